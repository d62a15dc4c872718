"""The CUDA renderers against the reference's own estimator code.

``tests/golden/paths_ref.npz`` holds whole paths that the reference's
``cast_rays`` kernel (main.py:1502-1590), lifted unmodified from its source
and run with float32 arithmetic, computed for three scenes with the Philox
streams the library uses (``tests/golden/make_estimator_ref.py``).  Each scene
is uploaded exactly as the reference's ``setup_scene`` laid it out: triangles
in its BVH order, its node table adopted as the tree, its materials, EEMs and
camera.  The GPU renders the same passes and must agree per film cell (CUDA's
transcendental functions against NumPy's: 99.5 % of cells within 1e-3
relative, pass totals within 2e-3); where the reference's film cell is NaN
(the box's rough dielectric, after a path's throughput reached zero), the
GPU, which ends such paths, must be finite and equal to the sum of the
reference's finite deposits.
"""
import numpy as np
import pytest

from test_oracle_pinned import GOLD, reference_film

pytestmark = pytest.mark.gpu


def scene_from_fixture(P, name):
    """create_scene()-schema dictionary holding the fixture's triangles in its
    BVH order (unshared vertices, its per-vertex normals), its materials and
    camera, plus the node table as an adopted tree with identity permutation."""
    g = lambda k: P[f"{name}_{k}"]  # noqa: E731
    v0, v1, v2 = g("v0"), g("v1"), g("v2")
    mat = g("mat_id")
    meshes = []
    start = 0
    T = v0.shape[0]
    while start < T:
        end = start
        while end < T and mat[end] == mat[start]:
            end += 1
        k = end - start
        verts = np.stack([v0[start:end], v1[start:end], v2[start:end]], 1).reshape(-1, 3)
        norms = np.stack([g("n0")[start:end], g("n1")[start:end], g("n2")[start:end]], 1).reshape(-1, 3)
        meshes.append({"vertices": verts.tolist(), "faces": np.arange(3 * k).reshape(k, 3).tolist(),
                       "vertex_normals": norms.tolist(), "material_id": int(mat[start])})
        start = end
    mf, mi, me = g("mat_f32"), g("mat_i32"), g("mat_eem")
    keys = ("refractive_index", "extinction_coefficient", "roughness", "scattering_coefficient", "emission",
            "anistropy_factor")
    mats = []
    for m in range(mf.shape[0]):
        d = {k: mf[m, p].astype(np.float64).tolist() for p, k in enumerate(keys)}
        d["is_true_volume"] = mi[m, 0].tolist()
        d["surface_emission"] = mi[m, 1].tolist()
        d["eem_id"] = int(me[m])
        mats.append(d)
    cam = g("camera")
    scene = {"meshes": meshes, "materials": mats,
             "camera": {"origin": cam[0].tolist(), "lookat": cam[1].tolist(), "up": cam[2].tolist()}}
    bvh = {k: g(k) for k in ("node_min", "node_max", "node_left", "node_right", "node_num_tris", "node_tri_start")}
    bvh["tri_perm"] = np.arange(T, dtype=np.int32)
    return scene, bvh, g


@pytest.fixture(scope="module")
def paths():
    import os
    return dict(np.load(os.path.join(GOLD, "paths_ref.npz")))


@pytest.mark.parametrize("name", ["ref", "box", "volume"])
@pytest.mark.parametrize("kernel", ["mega", "wavefront"])
def test_gpu_paths_match_reference(name, kernel, paths):
    import spectral_b200 as sb
    scene, bvh, g = scene_from_fixture(paths, name)
    W, H, B, D, SB = (int(x) for x in g("config"))
    lmin, lmax, eps, esc, asp = (float(x) for x in g("lambda"))
    cfg = sb.RenderConfig(width=W, height=H, bands=B, lambda_min=lmin, lambda_max=lmax, max_path_length=D,
                          scatter_bounces=SB, epsilon=eps, escape=esc, aspect_ratio=asp, fov_scale=1.0,
                          seed=int(g("seed")), kernel=kernel, image_width=W, image_height=H)
    pix = g("pixels")
    with sb.Renderer(scene, cfg, eems=g("eem"), cmf=np.zeros((B, 3), np.float32), bvh=bvh) as r:
        assert np.array_equal(r.tri_perm(), bvh["tri_perm"])
        for p, b in zip(g("passes"), g("bands")):
            r.clear_pixel_space()
            r.cast_rays(int(b), pass_idx=int(p))
            film = r.block_film.cpu().numpy().reshape(B, -1).T[pix]
            assert r.check_device() == 0
            ref, nan = reference_film(g, int(p), B)
            assert np.isfinite(film).all()
            close = np.isclose(film, ref, rtol=1e-3, atol=1e-7)
            assert close.mean() >= 0.995, f"{name}/{kernel} pass {p}: {close.mean():.4f} of cells within 1e-3"
            assert abs(film.sum() - ref.sum()) <= 2e-3 * abs(ref.sum()) + 1e-9
            if name == "box":
                assert nan.sum() > 20  # the reference's NaN cells: finite here, equal to its finite deposits
                assert close[nan].mean() >= 0.99
