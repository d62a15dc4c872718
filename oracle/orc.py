"""ctypes binding of the CPU oracle (liborc.so) -- TEST INFRASTRUCTURE ONLY.

Used by tests/, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
bench.py as the checker.  The product path (the CUDA library) never imports
this module.  Parity status of the oracle: see oracle.h.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

F32P = ctypes.POINTER(ctypes.c_float)
I32P = ctypes.POINTER(ctypes.c_int32)


class OrcConfig(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("bands", ctypes.c_int32),
                ("lambda_min_nm", ctypes.c_float), ("lambda_step_nm", ctypes.c_float),
                ("epsilon", ctypes.c_float), ("escape", ctypes.c_float),
                ("max_path_length", ctypes.c_int32), ("scatter_bounces", ctypes.c_int32),
                ("aspect_ratio", ctypes.c_float), ("fov_scale", ctypes.c_float),
                ("seed", ctypes.c_uint32), ("scene_id", ctypes.c_uint32)]


class OrcScene(ctypes.Structure):
    _fields_ = [("num_tris", ctypes.c_int32),
                ("v0", F32P), ("v1", F32P), ("v2", F32P), ("n0", F32P), ("n1", F32P), ("n2", F32P),
                ("normal", F32P), ("area", F32P), ("mat_id", I32P),
                ("num_nodes", ctypes.c_int32), ("node_min", F32P), ("node_max", F32P),
                ("node_left", I32P), ("node_right", I32P), ("node_num_tris", I32P),
                ("node_tri_start", I32P),
                ("num_materials", ctypes.c_int32), ("mat_f32", F32P), ("mat_i32", I32P),
                ("mat_eem", I32P), ("num_eems", ctypes.c_int32), ("eem", F32P),
                ("max_lights", ctypes.c_int32), ("light_cdf", F32P), ("light_idx", I32P),
                ("num_lights", I32P), ("light_area", F32P),
                ("cam_origin", ctypes.c_float * 3), ("cam_u", ctypes.c_float * 3),
                ("cam_v", ctypes.c_float * 3), ("cam_w", ctypes.c_float * 3)]


class OrcStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_int64), ("vertices", ctypes.c_int64), ("traces", ctypes.c_int64),
                ("stack_overflow", ctypes.c_int64)]


def build():
    """Compile liborc.so in place (gcc, OpenMP, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_philox4x32_10.argtypes = [ctypes.POINTER(ctypes.c_uint32)] * 3
        L.orc_trace.argtypes = [ctypes.POINTER(OrcScene), ctypes.POINTER(OrcConfig), F32P, ctypes.c_int32,
                                I32P, F32P, F32P, F32P, ctypes.c_int32]
        L.orc_trace_brute.argtypes = [ctypes.POINTER(OrcScene), ctypes.POINTER(OrcConfig), F32P,
                                      ctypes.c_int32, I32P, F32P]
        L.orc_render_pass.argtypes = [ctypes.POINTER(OrcScene), ctypes.POINTER(OrcConfig), ctypes.c_uint32,
                                      ctypes.c_int32, I32P, ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
                                      ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(OrcStats)]
        L.orc_adjoint_pass.argtypes = [ctypes.POINTER(OrcScene), ctypes.POINTER(OrcConfig), ctypes.c_uint32,
                                       ctypes.c_int32, I32P, ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
                                       ctypes.c_int32, ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                       ctypes.c_int32, ctypes.c_int32]
        L.orc_build_bvh_sweep.argtypes = [ctypes.c_int32, F32P, F32P, F32P, ctypes.c_int32, F32P, F32P,
                                          I32P, I32P, I32P, I32P, I32P]
        L.orc_build_bvh_sweep.restype = ctypes.c_int32
        L.orc_eval.argtypes = [ctypes.POINTER(OrcScene), ctypes.POINTER(OrcConfig), ctypes.c_int32, ctypes.c_int32,
                               F32P, ctypes.c_int32, F32P, ctypes.c_int32, F32P, ctypes.c_int32, I32P]
        d = ctypes.c_double
        L.orc_fresnel.argtypes = [d, d, d, d, d, ctypes.c_int32]
        L.orc_fresnel.restype = d
        L.orc_ggx_d.argtypes = [d, d, ctypes.c_int32]
        L.orc_ggx_d.restype = d
        L.orc_hg_eval.argtypes = [d, d, ctypes.c_int32]
        L.orc_hg_eval.restype = d
        _LIB = L
    return _LIB


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _p(a, t):
    return a.ctypes.data_as(t)


def philox(ctr, key):
    c = (ctypes.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in ctr])
    k = (ctypes.c_uint32 * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    o = (ctypes.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return [o[i] for i in range(4)]


class Config:
    """Render constants of the reference (main.py:11-35) as runtime values."""

    def __init__(self, width=400, height=400, bands=25, lambda_min=10.0, lambda_max=1210.0, epsilon=1e-4,
                 escape=1e2, max_path_length=7, scatter_bounces=5, aspect_ratio=1.0, fov_scale=1.0, seed=0,
                 scene_id=0):
        self.c = OrcConfig(width, height, bands, lambda_min, (lambda_max - lambda_min) / (bands - 1), epsilon,
                           escape, max_path_length, scatter_bounces, aspect_ratio, fov_scale, seed, scene_id)


class Scene:
    """Scene in the reference layout: triangles in BVH order + reference BVH nodes.

    ``arrays`` keys: v0 v1 v2 n0 n1 n2 normal area mat_id (reordered order),
    node_min node_max node_left node_right node_num_tris node_tri_start,
    mat_f32 [M,6,B] mat_i32 [M,2,B] mat_eem [M], eem [E,B,B],
    light_cdf [B,L] light_idx [B,L] num_lights [B] light_area [B],
    cam_origin cam_u cam_v cam_w.
    """

    def __init__(self, arrays):
        a = {}
        for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area", "node_min", "node_max", "mat_f32", "eem",
                  "light_cdf", "light_area"):
            a[k] = _f32(arrays[k])
        for k in ("mat_id", "node_left", "node_right", "node_num_tris", "node_tri_start", "mat_i32", "mat_eem",
                  "light_idx", "num_lights"):
            a[k] = _i32(arrays[k])
        self._keep = a
        s = OrcScene()
        s.num_tris = a["area"].shape[0]
        for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area", "node_min", "node_max", "mat_f32", "eem",
                  "light_cdf", "light_area"):
            setattr(s, k, _p(a[k], F32P))
        for k in ("mat_id", "node_left", "node_right", "node_num_tris", "node_tri_start", "mat_i32", "mat_eem",
                  "light_idx", "num_lights"):
            setattr(s, k, _p(a[k], I32P))
        s.num_nodes = a["node_num_tris"].shape[0]
        s.num_materials = a["mat_f32"].shape[0]
        s.num_eems = a["eem"].shape[0]
        s.max_lights = a["light_cdf"].shape[1]
        for k in ("cam_origin", "cam_u", "cam_v", "cam_w"):
            v = np.asarray(arrays[k], dtype=np.float32)
            setattr(s, k, (ctypes.c_float * 3)(*v.tolist()))
        self.s = s


# function-level hooks of orc_eval: kind -> (id, output width)
EVAL_KINDS = {"triangle": (0, 3), "aabb": (1, 1), "trace": (2, 13), "complex": (3, 4), "fresnel": (4, 1),
              "ggx_d": (5, 1), "ggx_g": (6, 1), "ggx_sample": (7, 3), "hg": (8, 1), "hg_sample": (9, 3),
              "cos_hemisphere": (10, 3), "sphere": (11, 3), "bsdf": (12, 2), "shadow": (13, 1), "nee": (14, 3),
              "surface": (15, 7), "volume": (16, 17)}


def eval_fn(kind, cfg, inputs=None, draws=None, scene=None, n=None):
    """Run one restated reference function (FP32) on rows of inputs, each row
    with its own list of random draws.  Returns (outputs [n, w], draws used [n])."""
    k, width = EVAL_KINDS[kind]
    inp = None if inputs is None else _f32(inputs)
    if inp is not None and inp.ndim == 1:
        inp = inp[:, None]
    dr = None if draws is None else _f32(draws)
    n = n if n is not None else (inp.shape[0] if inp is not None else dr.shape[0])
    out = np.zeros((n, width), np.float32)
    used = np.zeros(n, np.int32)
    lib().orc_eval(ctypes.byref(scene.s) if scene is not None else None, ctypes.byref(cfg.c), k, n,
                   None if inp is None else _p(inp, F32P), 0 if inp is None else inp.shape[1],
                   None if dr is None else _p(dr, F32P), 0 if dr is None else dr.shape[1], _p(out, F32P), width,
                   _p(used, I32P))
    return out, used


def fresnel(cos_i, ni, ki, nt, kt, use_double=False):
    return lib().orc_fresnel(cos_i, ni, ki, nt, kt, int(use_double))


def ggx_d(ndh, rough, use_double=False):
    return lib().orc_ggx_d(ndh, rough, int(use_double))


def hg_eval(cos_t, g, use_double=False):
    return lib().orc_hg_eval(cos_t, g, int(use_double))


def trace(scene, cfg, rays, use_double=False):
    rays = _f32(rays).reshape(-1, 6)
    n = rays.shape[0]
    tri = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    u = np.empty(n, np.float32)
    v = np.empty(n, np.float32)
    lib().orc_trace(ctypes.byref(scene.s), ctypes.byref(cfg.c), _p(rays, F32P), n, _p(tri, I32P), _p(t, F32P),
                    _p(u, F32P), _p(v, F32P), int(use_double))
    return tri, t, u, v


def trace_brute(scene, cfg, rays):
    rays = _f32(rays).reshape(-1, 6)
    n = rays.shape[0]
    tri = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    lib().orc_trace_brute(ctypes.byref(scene.s), ctypes.byref(cfg.c), _p(rays, F32P), n, _p(tri, I32P),
                          _p(t, F32P))
    return tri, t


def render_pass(scene, cfg, pass_idx, band, pixel_ids, out=None, use_double=False, nthreads=0):
    """Add one cast_rays pass for ``pixel_ids`` into ``out`` [npix, B] (float64)."""
    pixel_ids = _i32(pixel_ids)
    npix = pixel_ids.shape[0]
    if out is None:
        out = np.zeros((npix, cfg.c.bands), np.float64)
    assert out.dtype == np.float64 and out.flags.c_contiguous and out.shape == (npix, cfg.c.bands)
    st = OrcStats()
    lib().orc_render_pass(ctypes.byref(scene.s), ctypes.byref(cfg.c), pass_idx, band, _p(pixel_ids, I32P), npix,
                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(use_double), nthreads,
                          ctypes.byref(st))
    return out, {"paths": st.paths, "vertices": st.vertices, "traces": st.traces,
                 "stack_overflow": st.stack_overflow}


def adjoint_pass(scene, cfg, pass_idx, band, pixel_ids, adj, param_ids, grad=None, out=None, use_double=True,
                 nthreads=0):
    """Forward-mode adjoint of one pass (FP64, or FP32 with use_double=False): ADDS d(sum adj * deposits)/d params into grad.

    adj: [npix, B] float64 deposit weights; param_ids: indices into the
    material table [M,6,B] followed by the EEM table [E,B,B].  out (optional,
    [npix, B] float64) receives the pass's FP64 film."""
    pixel_ids = _i32(pixel_ids)
    npix = pixel_ids.shape[0]
    adj = np.ascontiguousarray(adj, np.float64)
    assert adj.shape == (npix, cfg.c.bands)
    ids = np.ascontiguousarray(param_ids, np.int64)
    if grad is None:
        grad = np.zeros(ids.shape[0], np.float64)
    assert grad.dtype == np.float64 and grad.shape == ids.shape
    dp = ctypes.POINTER(ctypes.c_double)
    outp = None if out is None else out.ctypes.data_as(dp)
    if out is not None:
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.shape == (npix, cfg.c.bands)
    lib().orc_adjoint_pass(ctypes.byref(scene.s), ctypes.byref(cfg.c), pass_idx, band, _p(pixel_ids, I32P), npix,
                           adj.ctypes.data_as(dp), ids.shape[0], ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                           grad.ctypes.data_as(dp), outp, int(use_double), nthreads)
    return grad


def param_index(num_materials, bands, material, prop, band):
    """Index of material-table entry (material, prop, band) in the parameter vector."""
    return (material * 6 + prop) * bands + band


def eem_param_index(num_materials, bands, eem, row, col):
    return num_materials * 6 * bands + (eem * bands + row) * bands + col


def build_bvh_sweep(v0, v1, v2):
    """Reference SAH sweep builder (main.py:437-507) -> node table + permutation."""
    v0, v1, v2 = _f32(v0), _f32(v1), _f32(v2)
    T = v0.shape[0]
    M = max(2 * T - 1, 1)
    nmin = np.zeros((M, 3), np.float32)
    nmax = np.zeros((M, 3), np.float32)
    left = np.zeros(M, np.int32)
    right = np.zeros(M, np.int32)
    ntri = np.zeros(M, np.int32)
    tstart = np.zeros(M, np.int32)
    perm = np.zeros(T, np.int32)
    N = lib().orc_build_bvh_sweep(T, _p(v0, F32P), _p(v1, F32P), _p(v2, F32P), M, _p(nmin, F32P),
                                  _p(nmax, F32P), _p(left, I32P), _p(right, I32P), _p(ntri, I32P),
                                  _p(tstart, I32P), _p(perm, I32P))
    assert N >= 0
    return dict(node_min=nmin[:N], node_max=nmax[:N], node_left=left[:N], node_right=right[:N],
                node_num_tris=ntri[:N], node_tri_start=tstart[:N], perm=perm)


# ---------------------------------------------------------------- scene bridge
def camera_basis(origin, lookat, up):
    """update_camera (main.py:633-640) in float32."""
    f = np.float32
    o, l, u = (np.asarray(v, np.float32) for v in (origin, lookat, up))

    def nrm(a):
        return a / np.sqrt(f(a[0] * a[0]) + f(a[1] * a[1]) + f(a[2] * a[2]))

    def cr(a, b):
        return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], np.float32)

    w = nrm(o - l)
    uu = nrm(cr(u, w))
    v = cr(w, uu)
    return o, uu, v, w


def light_tables(mat_i32, slot_mat, slot_area, bands):
    """Per-band light CDF over triangle slots, float32 running sums (main.py:590-627)."""
    slot_area = np.asarray(slot_area, np.float32)
    lists = [np.nonzero(mat_i32[slot_mat, 1, b])[0] for b in range(bands)]
    L = max([1] + [len(x) for x in lists])
    cdf = np.zeros((bands, L), np.float32)
    idx = np.zeros((bands, L), np.int32)
    nl = np.zeros(bands, np.int32)
    area = np.zeros(bands, np.float32)
    for b, lst in enumerate(lists):
        nl[b] = len(lst)
        if not len(lst):
            continue
        a = slot_area[lst]
        tot = np.cumsum(a, dtype=np.float32)[-1]  # sequential float32 sum
        area[b] = tot
        cdf[b, :len(lst)] = np.cumsum((a / tot).astype(np.float32), dtype=np.float32)
        idx[b, :len(lst)] = lst
    return cdf, idx, nl, area


def oracle_scene(compiled, bvh, camera):
    """Oracle scene matching a GPU upload slot for slot.

    compiled: a CompiledScene of the package (original-order triangles and
    material tables); bvh: a tree in the reference layout with tri_perm (the
    same tree given to the GPU), so both sides see the same triangle slots and
    light CDF order."""
    perm = np.asarray(bvh["tri_perm"], np.int64)
    t = compiled.tris
    arrays = {k: t[k][perm] for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area", "mat_id")}
    for k in ("node_min", "node_max", "node_left", "node_right", "node_num_tris", "node_tri_start"):
        arrays[k] = bvh[k]
    B = compiled.mat_f32.shape[2]
    arrays["mat_f32"] = compiled.mat_f32
    arrays["mat_i32"] = compiled.mat_i32
    arrays["mat_eem"] = compiled.mat_eem
    arrays["eem"] = compiled.eem
    cdf, idx, nl, area = light_tables(compiled.mat_i32, arrays["mat_id"], arrays["area"], B)
    arrays.update(light_cdf=cdf, light_idx=idx, num_lights=nl, light_area=area)
    o, u, v, w = camera_basis(camera["origin"], camera["lookat"], camera["up"])
    arrays.update(cam_origin=o, cam_u=u, cam_v=v, cam_w=w)
    return Scene(arrays)


def oracle_config(cfg, scene_id=0):
    """Oracle config from a RenderConfig."""
    return Config(width=cfg.width, height=cfg.height, bands=cfg.bands, lambda_min=cfg.lambda_min,
                      lambda_max=cfg.lambda_max, epsilon=cfg.epsilon, escape=cfg.escape,
                      max_path_length=cfg.max_path_length, scatter_bounces=cfg.scatter_bounces,
                      aspect_ratio=cfg.aspect_ratio, fov_scale=cfg.fov_scale, seed=cfg.seed, scene_id=scene_id)
