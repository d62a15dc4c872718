"""ctypes binding of libspectral.so (include/spectral.h).

The library is the only compute path: if it is missing or no CUDA device is
present, the calls raise -- there is no CPU fallback.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libspectral.so")

TS_OK = 0
STATUS_NAMES = {0: "TS_OK", 1: "TS_ERR_INVALID_ARG", 2: "TS_ERR_CUDA", 3: "TS_ERR_OUT_OF_MEMORY",
                4: "TS_ERR_CAPACITY", 5: "TS_ERR_DEVICE_FAULT", 6: "TS_ERR_NO_SCENE"}
KERNEL_MEGA, KERNEL_WAVEFRONT = 0, 1
TRACE_FAST, TRACE_REFERENCE_ORDER = 0, 1
FILM_BLOCK, FILM_MEAN, FILM_M2 = 0, 1, 2

F32P = ctypes.POINTER(ctypes.c_float)
I32P = ctypes.POINTER(ctypes.c_int32)
F64P = ctypes.POINTER(ctypes.c_double)


class SpectralError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class TsConfig(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("bands", ctypes.c_int32),
                ("lambda_min_nm", ctypes.c_float), ("lambda_max_nm", ctypes.c_float),
                ("max_path_length", ctypes.c_int32), ("scatter_bounces", ctypes.c_int32),
                ("epsilon", ctypes.c_float), ("escape", ctypes.c_float), ("aspect_ratio", ctypes.c_float),
                ("fov_scale", ctypes.c_float), ("seed", ctypes.c_uint32), ("scene_id", ctypes.c_uint32),
                ("device", ctypes.c_int32), ("kernel", ctypes.c_int32), ("block_size", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("sort_keys", ctypes.c_int32), ("trace_budget", ctypes.c_int32),
                ("traversal", ctypes.c_int32), ("occupancy", ctypes.c_int32),
                ("queue_capacity", ctypes.c_int32), ("loop_host", ctypes.c_int32)]


class TsSceneDesc(ctypes.Structure):
    _fields_ = [("num_tris", ctypes.c_int32),
                ("v0", F32P), ("v1", F32P), ("v2", F32P), ("n0", F32P), ("n1", F32P), ("n2", F32P),
                ("normal", F32P), ("area", F32P), ("mat_id", I32P),
                ("num_materials", ctypes.c_int32), ("mat_f32", F32P), ("mat_i32", I32P), ("mat_eem", I32P),
                ("num_eems", ctypes.c_int32), ("eem", F32P), ("cmf", F32P),
                ("bvh_num_nodes", ctypes.c_int32), ("node_min", F32P), ("node_max", F32P),
                ("node_left", I32P), ("node_right", I32P), ("node_num_tris", I32P), ("node_tri_start", I32P),
                ("tri_perm", I32P),
                ("bvh_bins", ctypes.c_int32), ("bvh_leaf_max", ctypes.c_int32),
                ("bvh_cost_trav", ctypes.c_float), ("bvh_cost_tri", ctypes.c_float), ("bvh_width", ctypes.c_int32),
                ("bvh_quantized", ctypes.c_int32)]


class TsSceneInfo(ctypes.Structure):
    _fields_ = [("num_tris", ctypes.c_int32), ("num_nodes", ctypes.c_int32), ("num_ref_nodes", ctypes.c_int32),
                ("max_depth", ctypes.c_int32), ("leaves", ctypes.c_int32), ("sah_cost", ctypes.c_double),
                ("max_lights", ctypes.c_int32), ("device_bytes", ctypes.c_size_t), ("node_width", ctypes.c_int32),
                ("node_quantized", ctypes.c_int32)]


# (name, restype, argtypes) of every entry point declared in include/spectral.h
_VP = ctypes.c_void_p
SIGNATURES = [
    ("ts_create", ctypes.c_int, [ctypes.POINTER(TsConfig), ctypes.POINTER(_VP)]),
    ("ts_destroy", ctypes.c_int, [_VP]),
    ("ts_set_launch_config", ctypes.c_int, [_VP, ctypes.POINTER(TsConfig)]),
    ("ts_last_error", ctypes.c_char_p, [_VP]),
    ("ts_version", ctypes.c_char_p, []),
    ("ts_upload_scene", ctypes.c_int, [_VP, ctypes.POINTER(TsSceneDesc)]),
    ("ts_scene_info_get", ctypes.c_int, [_VP, ctypes.POINTER(TsSceneInfo)]),
    ("ts_get_tri_perm", ctypes.c_int, [_VP, I32P]),
    ("ts_build_bvh_host", ctypes.c_int, [ctypes.c_int32, F32P, F32P, F32P, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.c_float, ctypes.c_float, ctypes.c_int32, F32P, F32P, I32P, I32P,
                                         I32P, I32P, I32P, I32P]),
    ("ts_set_camera", ctypes.c_int, [_VP, F32P, F32P, F32P]),
    ("ts_render_pass", ctypes.c_int, [_VP, ctypes.c_uint32, ctypes.c_int32, _VP]),
    ("ts_render_passes", ctypes.c_int, [_VP, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, _VP]),
    ("ts_wave_loop_iterations", ctypes.c_int, [_VP, _VP, ctypes.POINTER(ctypes.c_int32)]),
    ("ts_set_loop_iteration_limit", ctypes.c_int, [_VP, ctypes.c_int32]),
    ("ts_create_view", ctypes.c_int, [_VP, ctypes.POINTER(TsConfig), ctypes.POINTER(_VP)]),
    ("ts_record_paths", ctypes.c_int, [_VP, ctypes.c_uint32, ctypes.c_int32]),
    ("ts_render_pass_counted", ctypes.c_int, [_VP, ctypes.c_uint32, ctypes.c_int32, _VP,
                                              ctypes.POINTER(ctypes.c_uint64)]),
    ("ts_render_tile_noalloc", ctypes.c_int, [_VP, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_int32, ctypes.c_int32, _VP, _VP]),
    ("ts_accumulate_block", ctypes.c_int, [_VP, ctypes.c_int32, _VP]),
    ("ts_reset", ctypes.c_int, [_VP, _VP]),
    ("ts_film_buffer", ctypes.c_int, [_VP, ctypes.c_int32, ctypes.POINTER(F64P), ctypes.POINTER(ctypes.c_size_t)]),
    ("ts_film_download", ctypes.c_int, [_VP, ctypes.c_int32, F64P, _VP]),
    ("ts_resolve_xyz", ctypes.c_int, [_VP, ctypes.c_double, _VP, _VP]),
    ("ts_resolve_xyz_host", ctypes.c_int, [_VP, ctypes.c_double, F32P, _VP]),
    ("ts_resolve_rgb", ctypes.c_int, [_VP, ctypes.c_double, F32P, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                      ctypes.c_int32, _VP, _VP]),
    ("ts_trace_batch", ctypes.c_int, [_VP, _VP, ctypes.c_int32, ctypes.c_int32, _VP, _VP, _VP, _VP, _VP]),
    ("ts_render_normals", ctypes.c_int, [_VP, _VP, _VP]),
    ("ts_param_count", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    ("ts_update_materials", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("ts_adjoint_pass", ctypes.c_int, [_VP, ctypes.c_uint32, ctypes.c_int32, _VP, _VP, _VP]),
    ("ts_adjoint_passes", ctypes.c_int, [_VP, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, _VP, _VP, _VP]),
    ("ts_check_device", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_uint32)]),
    ("ts_batch_create", ctypes.c_int, [_VP, ctypes.POINTER(_VP), ctypes.c_int32, ctypes.POINTER(_VP)]),
    ("ts_batch_destroy", ctypes.c_int, [_VP]),
    ("ts_batch_last_error", ctypes.c_char_p, [_VP]),
    ("ts_batch_reset", ctypes.c_int, [_VP, ctypes.c_uint32, _VP]),
    ("ts_batch_set_active", ctypes.c_int, [_VP, I32P, _VP]),
    ("ts_batch_step", ctypes.c_int, [_VP, _VP]),
    ("ts_batch_check", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_uint32)]),
]

_lib = None


def build(quiet=True):
    """Compile libspectral.so in place (nvcc, sm_100a)."""
    cmd = ["make", "-j8", "-C", _HERE]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)


def load():
    """Load libspectral.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libspectral.so not built at {LIB_PATH}; run __graft_entry__.build() or "
                          f"`make -C taichi-spectral-render_b200`")
    L = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def build_bvh_host(v0, v1, v2, bins=0, leaf_max=0, cost_trav=0.0, cost_tri=0.0):
    """The library's binned-SAH tree in the reference layout (host only, no GPU)."""
    import numpy as np
    v0, v1, v2 = (np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 3) for a in (v0, v1, v2))
    T = v0.shape[0]
    M = max(2 * T - 1, 1)
    nmin = np.zeros((M, 3), np.float32)
    nmax = np.zeros((M, 3), np.float32)
    left, right, ntri, tstart = (np.zeros(M, np.int32) for _ in range(4))
    perm = np.zeros(max(T, 1), np.int32)
    nn = ctypes.c_int32()
    f = lambda a: a.ctypes.data_as(F32P)
    i = lambda a: a.ctypes.data_as(I32P)
    check(load().ts_build_bvh_host(T, f(v0), f(v1), f(v2), bins, leaf_max, cost_trav, cost_tri, M, f(nmin), f(nmax),
                                   i(left), i(right), i(ntri), i(tstart), i(perm), ctypes.byref(nn)))
    N = nn.value
    return {"node_min": nmin[:N], "node_max": nmax[:N], "node_left": left[:N], "node_right": right[:N],
            "node_num_tris": ntri[:N], "node_tri_start": tstart[:N], "tri_perm": perm[:T]}


def check(status, ctx=None):
    if status != TS_OK:
        msg = load().ts_last_error(ctx)
        raise SpectralError(status, msg.decode() if msg else "")
