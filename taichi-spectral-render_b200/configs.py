"""Synthetic workloads in the ``create_scene()`` schema.

No public dataset is involved; every scene is generated from a seed:

  box_scene         closed 1 m box (12 triangles), 2,048-triangle UV sphere
                    (r = 0.25, GGX dielectric, alpha 0.1, Cauchy n), 0.2 m
                    ceiling light with a 5500 K blackbody shape, Oren-Nayar
                    walls (sigma 0.3) with logistic reflectance spectra;
                    25 bands 380-740 nm; 256^2, FOV 40 deg, depth 8, 64 spp
  terrain_scene     1024^2-vertex heightfield (2.09 M triangles, 6-octave value
                    noise) plus a 500k-triangle displaced sphere, GGX
                    conductors (alpha log-uniform in [0.02, 0.5], smooth n in
                    [0.2, 1.5], k in [2, 8]), 8 emissive quads; 1024^2, depth 12,
                    256 spp
  volume_scene      the box with the sphere replaced by a 20k-triangle closed
                    mesh holding a homogeneous Henyey-Greenstein medium (g 0.7,
                    sigma_s and sigma_a sums of two Gaussians) and one
                    fluorescent diffuse wall (Gaussian Stokes-shift EEM,
                    40 +- 15 nm, quantum yield 0.6); 512^2, depth 32, 512 spp

Material conventions follow the reference (main.py:90-175): roughness r gives
GGX alpha = r^2 in D (so r = sqrt(alpha)), Oren-Nayar sigma = r * pi / 2; a
diffuse reflectance rho is encoded as scattering 1 and k = lambda (1/rho - 1) /
(4 pi); an absorption coefficient sigma_a as k = sigma_a lambda / (4 pi).
Each generator returns (scene_dict, RenderConfig, extras) where extras holds
the EEM table, the CMF and the spp of the workload.
"""
import numpy as np

from . import spectral_data as sd
from .renderer import RenderConfig, fov_scale_for

BANDS = 25
LMIN, LMAX = 380.0, 740.0


def wavelengths(bands=BANDS, lmin=LMIN, lmax=LMAX):
    return np.linspace(lmin, lmax, bands)


def blocks_for(spp, bands=BANDS):
    """Passes needed for spp samples rounded up to whole spectral blocks."""
    return -(-int(spp) // bands) * bands


# --------------------------------------------------------------------------- geometry
def quad(p0, p1, p2, p3, material_id):
    """Two triangles (p0 p1 p2), (p0 p2 p3); the normal follows (p1 - p0) x (p2 - p0)."""
    return {"vertices": [list(p0), list(p1), list(p2), list(p3)], "faces": [[0, 1, 2], [0, 2, 3]],
            "material_id": material_id}


def box_walls(half, material_ids):
    """Six inward-facing walls of an axis-aligned cube [-half, half]^3, 2 triangles each.

    material_ids: 6 ids for floor, ceiling, back (-z), front (+z), left (-x), right (+x)."""
    h = half
    P = lambda x, y, z: (x * h, y * h, z * h)
    return [
        quad(P(-1, -1, -1), P(-1, -1, 1), P(1, -1, 1), P(1, -1, -1), material_ids[0]),  # floor, +y
        quad(P(-1, 1, -1), P(1, 1, -1), P(1, 1, 1), P(-1, 1, 1), material_ids[1]),      # ceiling, -y
        quad(P(-1, -1, -1), P(1, -1, -1), P(1, 1, -1), P(-1, 1, -1), material_ids[2]),  # back, +z
        quad(P(-1, -1, 1), P(-1, 1, 1), P(1, 1, 1), P(1, -1, 1), material_ids[3]),      # front, -z
        quad(P(-1, -1, -1), P(-1, 1, -1), P(-1, 1, 1), P(-1, -1, 1), material_ids[4]),  # left, +x
        quad(P(1, -1, -1), P(1, -1, 1), P(1, 1, 1), P(1, 1, -1), material_ids[5]),      # right, -x
    ]


def uv_sphere(center, radius, slices, stacks, material_id, displace=None, smooth=True):
    """UV sphere with pole fans: slices * (2 * stacks - 2) outward-facing triangles.

    displace(unit_dirs) -> relative radius offsets (optional)."""
    th = np.linspace(0.0, np.pi, stacks + 1)[1:-1]  # interior rings
    ph = np.linspace(0.0, 2 * np.pi, slices, endpoint=False)
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    ring = np.stack([st * np.cos(ph)[None, :], ct * np.ones_like(ph)[None, :], st * np.sin(ph)[None, :]], -1)
    dirs = np.concatenate([[[0.0, 1.0, 0.0]], ring.reshape(-1, 3), [[0.0, -1.0, 0.0]]], 0)
    r = np.full(dirs.shape[0], float(radius))
    if displace is not None:
        r = r * (1.0 + displace(dirs))
    verts = dirs * r[:, None] + np.asarray(center, np.float64)[None, :]
    R = stacks - 1
    idx = lambda i, j: 1 + i * slices + (j % slices)
    south = 1 + R * slices
    faces = []
    for j in range(slices):
        faces.append([0, idx(0, j + 1), idx(0, j)])
    for i in range(R - 1):
        for j in range(slices):
            a, b, c, d = idx(i, j), idx(i, j + 1), idx(i + 1, j + 1), idx(i + 1, j)
            faces.append([a, b, c])
            faces.append([a, c, d])
    for j in range(slices):
        faces.append([south, idx(R - 1, j), idx(R - 1, j + 1)])
    faces = np.asarray(faces, np.int64)
    mesh = {"vertices": verts.astype(np.float32), "faces": faces, "material_id": material_id}
    if smooth:
        if displace is None:
            mesh["vertex_normals"] = dirs.astype(np.float32)
        else:
            mesh["vertex_normals"] = vertex_normals(verts, faces).astype(np.float32)
    return mesh


def vertex_normals(verts, faces):
    v = np.asarray(verts, np.float64)
    f = np.asarray(faces, np.int64)
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    n = np.zeros_like(v)
    for k in range(3):
        np.add.at(n, f[:, k], fn)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-20)
    return n


def value_noise_2d(x, y, octaves, seed, base_freq=1.0, lacunarity=2.0, gain=0.5):
    """Fractal value noise: smoothstep-interpolated random lattice values, summed over octaves."""
    rng = np.random.default_rng(seed)
    out = np.zeros(np.broadcast(x, y).shape)
    amp, freq, norm = 1.0, base_freq, 0.0
    for _ in range(octaves):
        lattice = rng.uniform(-1.0, 1.0, size=(257, 257))
        fx, fy = x * freq, y * freq
        ix, iy = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64)
        tx, ty = fx - ix, fy - iy
        sx, sy = tx * tx * (3 - 2 * tx), ty * ty * (3 - 2 * ty)
        g = lambda a, b: lattice[a % 256, b % 256]
        top = g(ix, iy) * (1 - sx) + g(ix + 1, iy) * sx
        bot = g(ix, iy + 1) * (1 - sx) + g(ix + 1, iy + 1) * sx
        out += amp * (top * (1 - sy) + bot * sy)
        norm += amp
        amp *= gain
        freq *= lacunarity
    return out / norm


def heightfield(n, size, height, seed, material_id, octaves=6):
    """n x n vertex grid over [-size/2, size/2]^2 in x/z: 2 (n-1)^2 upward-facing triangles."""
    xs = np.linspace(-size / 2, size / 2, n)
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    Hh = height * value_noise_2d(X / size * 4.0 + 7.3, Z / size * 4.0 + 1.9, octaves, seed)
    verts = np.stack([X, Hh, Z], -1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="xy")
    a = (j * n + i).reshape(-1)
    b, c, d = a + 1, a + n + 1, a + n
    faces = np.empty((2 * a.shape[0], 3), np.int64)
    faces[0::2] = np.stack([a, c, b], -1)
    faces[1::2] = np.stack([a, d, c], -1)
    return {"vertices": verts.astype(np.float32), "faces": faces, "material_id": material_id,
            "vertex_normals": vertex_normals(verts, faces).astype(np.float32)}


# --------------------------------------------------------------------------- materials
def material(bands=BANDS, n=1.0, k=0.0, roughness=0.0, is_true_volume=0, scattering=0.0, emission=0.0,
             anisotropy=0.0, surface_emission=0, eem_id=0):
    vec = lambda v: np.broadcast_to(np.asarray(v, np.float64), (bands,)).tolist()
    ivec = lambda v: np.broadcast_to(np.asarray(v, np.int64), (bands,)).astype(int).tolist()
    return {"refractive_index": vec(n), "extinction_coefficient": vec(k), "roughness": vec(roughness),
            "is_true_volume": ivec(is_true_volume), "scattering_coefficient": vec(scattering),
            "anistropy_factor": vec(anisotropy), "surface_emission": ivec(surface_emission),
            "emission": vec(emission), "eem_id": int(eem_id)}


def air(bands=BANDS):
    return material(bands, n=1.0, k=0.0, roughness=0.0, is_true_volume=1)


def oren_nayar_wall(lam, rho, sigma=0.3, n=1.5, eem_id=0):
    return material(len(lam), n=n, k=sd.reflectance_to_k(rho, lam), roughness=sigma * 2.0 / np.pi,
                    scattering=1.0, is_true_volume=0, eem_id=eem_id)


def blackbody_light(lam, temperature=5500.0, peak=20.0):
    e = sd.planck(lam, temperature)
    return material(len(lam), n=1.0, emission=peak * e / e.max(), surface_emission=1)


def smooth_curve(rng, lam, lo, hi, terms=3):
    """A smooth random spectrum in [lo, hi] (a few low-frequency cosines)."""
    t = (lam - lam.min()) / max(lam.max() - lam.min(), 1e-9)
    v = np.zeros_like(t)
    for k in range(1, terms + 1):
        v += rng.uniform(-1, 1) / k * np.cos(np.pi * k * t + rng.uniform(0, 2 * np.pi))
    v = (v - v.min()) / max(v.max() - v.min(), 1e-9)
    return lo + (hi - lo) * v


# --------------------------------------------------------------------------- workloads
def box_scene(seed=0, sphere_slices=32, sphere_stacks=33, width=256, height=256, spp=64, depth=8):
    """Plain spectral render of a box and a dielectric sphere (2,062 triangles)."""
    rng = np.random.default_rng(seed)
    lam = wavelengths()
    mats = [air()]
    walls = []
    for _ in range(6):
        rho = sd.logistic(lam, rng.uniform(450, 650), rng.uniform(0.01, 0.05))
        walls.append(len(mats))
        mats.append(oren_nayar_wall(lam, rho))
    light_id = len(mats)
    mats.append(blackbody_light(lam))
    sphere_id = len(mats)
    mats.append(material(len(lam), n=sd.cauchy_n(lam), k=0.0, roughness=np.sqrt(0.1), is_true_volume=1))
    meshes = box_walls(0.5, walls)
    meshes.append(quad((-0.1, 0.499, -0.1), (0.1, 0.499, -0.1), (0.1, 0.499, 0.1), (-0.1, 0.499, 0.1), light_id))
    meshes.append(uv_sphere((0.0, -0.249, -0.05), 0.25, sphere_slices, sphere_stacks, sphere_id))
    camera = {"origin": [0.0, 0.0, 0.49], "lookat": [0.0, -0.05, -0.5], "up": [0.0, 1.0, 0.0]}
    cfg = RenderConfig(width=width, height=height, bands=BANDS, lambda_min=LMIN, lambda_max=LMAX,
                       max_path_length=depth, fov_scale=fov_scale_for(40.0), samples_per_pixel=blocks_for(spp),
                       image_width=width, image_height=height, seed=seed)
    extras = {"eems": None, "cmf": sd.cie1931_fit(lam), "spp": spp}
    return {"meshes": meshes, "materials": mats, "camera": camera}, cfg, extras


def terrain_scene(seed=1, grid=1024, sphere_slices=500, sphere_stacks=501, width=1024, height=1024, spp=256,
                  depth=12, size=24.0):
    """Large-mesh render: heightfield terrain plus a displaced sphere, GGX conductors."""
    rng = np.random.default_rng(seed)
    lam = wavelengths()
    mats = [air()]

    def conductor():
        alpha = float(np.exp(rng.uniform(np.log(0.02), np.log(0.5))))
        return material(len(lam), n=smooth_curve(rng, lam, 0.2, 1.5), k=smooth_curve(rng, lam, 2.0, 8.0),
                        roughness=np.sqrt(alpha), is_true_volume=0, scattering=0.0)

    terrain_id = len(mats)
    mats.append(conductor())
    sphere_id = len(mats)
    mats.append(conductor())
    light_ids = []
    for i in range(8):
        light_ids.append(len(mats))
        mats.append(blackbody_light(lam, temperature=float(rng.uniform(3500, 9000)), peak=float(rng.uniform(20, 60))))
    meshes = [heightfield(grid, size, 1.6, seed, terrain_id)]
    noise_seed = seed + 1000

    def bumps(d):
        return 0.04 * value_noise_2d(np.arctan2(d[:, 2], d[:, 0]) * 3.0 + 10.0, np.arccos(np.clip(d[:, 1], -1, 1)) * 3.0,
                                     4, noise_seed)

    meshes.append(uv_sphere((0.0, 3.0, 0.0), 2.2, sphere_slices, sphere_stacks, sphere_id, displace=bumps))
    for i, lid in enumerate(light_ids):
        ang = 2 * np.pi * i / len(light_ids)
        cx, cz, y, s = 7.0 * np.cos(ang), 7.0 * np.sin(ang), 9.0, 0.8
        meshes.append(quad((cx - s, y, cz - s), (cx + s, y, cz - s), (cx + s, y, cz + s), (cx - s, y, cz + s), lid))
    camera = {"origin": [0.0, 7.5, 13.0], "lookat": [0.0, 1.5, 0.0], "up": [0.0, 1.0, 0.0]}
    cfg = RenderConfig(width=width, height=height, bands=BANDS, lambda_min=LMIN, lambda_max=LMAX,
                       max_path_length=depth, fov_scale=fov_scale_for(45.0), samples_per_pixel=blocks_for(spp),
                       image_width=width, image_height=height, seed=seed)
    extras = {"eems": None, "cmf": sd.cie1931_fit(lam), "spp": spp}
    return {"meshes": meshes, "materials": mats, "camera": camera}, cfg, extras


def two_gaussians(rng, lam, amp=(0.5, 5.0), width=(20.0, 60.0)):
    v = np.zeros_like(lam)
    for _ in range(2):
        v += rng.uniform(*amp) * np.exp(-0.5 * ((lam - rng.uniform(lam.min(), lam.max())) / rng.uniform(*width)) ** 2)
    return v


def volume_scene(seed=2, medium_slices=100, medium_stacks=101, width=512, height=512, spp=512, depth=32,
                 fluorescent_medium=False, params=None):
    """Box with an HG medium in a closed mesh and one fluorescent diffuse wall.

    params (optional): overrides {"albedo_left", "albedo_right" (per band),
    "sigma_a" (per band), "g", "roughness" (3 values: medium boundary, left,
    right)} -- the parameters of the inverse-rendering workload."""
    rng = np.random.default_rng(seed)
    lam = wavelengths()
    mats = [air()]
    walls = []
    rhos = []
    for _ in range(6):
        rhos.append(sd.logistic(lam, rng.uniform(450, 650), rng.uniform(0.01, 0.05)))
    p = dict(params or {})
    rough = list(p.get("roughness", [0.001, 0.3 * 2 / np.pi, 0.3 * 2 / np.pi]))
    if "albedo_left" in p:
        rhos[4] = np.asarray(p["albedo_left"], np.float64)
    if "albedo_right" in p:
        rhos[5] = np.asarray(p["albedo_right"], np.float64)
    for w in range(6):
        walls.append(len(mats))
        eem_id = 1 if w == 2 else 0  # the back wall fluoresces
        r = rough[1] if w == 4 else (rough[2] if w == 5 else 0.3 * 2 / np.pi)
        m = oren_nayar_wall(lam, rhos[w], eem_id=eem_id)
        m["roughness"] = [float(r)] * len(lam)
        mats.append(m)
    light_id = len(mats)
    mats.append(blackbody_light(lam, peak=30.0))
    sigma_s = two_gaussians(rng, lam)
    sigma_a = np.asarray(p["sigma_a"], np.float64) if "sigma_a" in p else two_gaussians(rng, lam)
    g = float(p.get("g", 0.7))
    medium_id = len(mats)
    mats.append(material(len(lam), n=1.33, k=sd.absorption_to_k(sigma_a, lam), roughness=rough[0], is_true_volume=1,
                         scattering=sigma_s, anisotropy=g, eem_id=1 if fluorescent_medium else 0))
    meshes = box_walls(0.5, walls)
    meshes.append(quad((-0.1, 0.499, -0.1), (0.1, 0.499, -0.1), (0.1, 0.499, 0.1), (-0.1, 0.499, 0.1), light_id))
    meshes.append(uv_sphere((0.0, -0.24, -0.05), 0.25, medium_slices, medium_stacks, medium_id))
    camera = {"origin": [0.0, 0.0, 0.49], "lookat": [0.0, -0.05, -0.5], "up": [0.0, 1.0, 0.0]}
    eem = np.zeros((2, len(lam), len(lam)))
    eem[1] = sd.gaussian_stokes_eem(lam, 40.0, 15.0, 0.6)
    cfg = RenderConfig(width=width, height=height, bands=BANDS, lambda_min=LMIN, lambda_max=LMAX,
                       max_path_length=depth, fov_scale=fov_scale_for(40.0), samples_per_pixel=blocks_for(spp),
                       image_width=width, image_height=height, seed=seed)
    extras = {"eems": eem, "cmf": sd.cie1931_fit(lam), "spp": spp,
              "params": {"sigma_a": sigma_a, "sigma_s": sigma_s, "g": g, "roughness": rough,
                         "albedo_left": rhos[4], "albedo_right": rhos[5]}}
    return {"meshes": meshes, "materials": mats, "camera": camera}, cfg, extras


def batch_scene(seed):
    """One scene of the batched workload, drawn from the box / terrain / volume generators.

    Triangle count log-uniform in 1k-500k, resolution from {128^2, 256^2, 512^2},
    maximum depth uniform in 4..16; box and terrain scenes are surface-only,
    volume scenes carry the HG medium (half of them fluorescent)."""
    rng = np.random.default_rng(seed)
    tris = float(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
    res = int(rng.choice([128, 256, 512]))
    depth = int(rng.integers(4, 17))
    kind = str(rng.choice(["box", "terrain", "volume"]))
    if kind == "box":
        n = max(8, int(np.sqrt(tris / 2)))
        out = box_scene(seed=seed, sphere_slices=n, sphere_stacks=n + 1, width=res, height=res, depth=depth)
    elif kind == "volume":
        n = max(8, int(np.sqrt(tris / 2)))
        out = volume_scene(seed=seed, medium_slices=n, medium_stacks=n + 1, width=res, height=res, depth=depth,
                           fluorescent_medium=bool(rng.integers(2)))
    else:
        grid = max(8, int(np.sqrt(0.8 * tris / 2)))
        n = max(8, int(np.sqrt(0.2 * tris / 2)))
        out = terrain_scene(seed=seed, grid=grid, sphere_slices=n, sphere_stacks=n + 1, width=res, height=res,
                            depth=depth)
    out[2]["kind"] = kind
    return out


def batch_workload(first_seed=100, count=64):
    """The batched workload: scenes of seeds first_seed .. first_seed + count - 1."""
    return [batch_scene(s) for s in range(first_seed, first_seed + count)]
