"""Shared helpers for the tests: oracle scenes that match a GPU upload slot for slot."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import orc  # noqa: E402
import spectral_b200 as sb  # noqa: E402
from spectral_b200 import _lib  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden_scene():
    return dict(np.load(os.path.join(GOLDEN, "scene_ref.npz")))


def golden_data():
    return dict(np.load(os.path.join(GOLDEN, "data_ref.npz")))


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
    """Per-band light CDF over triangle slots, float32 sums (main.py:590-627)."""
    T = slot_mat.shape[0]
    lists = [[s for s in range(T) if mat_i32[slot_mat[s], 1, b]] for b in range(bands)]
    L = max([1] + [len(x) for x in lists])
    cdf = np.zeros((bands, L), np.float32)
    idx = np.zeros((bands, L), np.int32)
    nl = np.zeros(bands, np.int32)
    area = np.zeros(bands, np.float32)
    for b, lst in enumerate(lists):
        nl[b] = len(lst)
        if not lst:
            continue
        tot = np.float32(0)
        for s in lst:
            tot = np.float32(tot + slot_area[s])
        area[b] = tot
        c = np.float32(0)
        for i, s in enumerate(lst):
            c = np.float32(c + np.float32(slot_area[s] / tot))
            cdf[b, i] = c
            idx[b, i] = s
    return cdf, idx, nl, area


def oracle_scene(compiled, bvh, camera):
    """Oracle scene with the triangles in the slot order of ``bvh`` (reference layout + tri_perm)."""
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
    return orc.Scene(arrays)


def oracle_config(cfg, scene_id=0):
    return orc.Config(width=cfg.width, height=cfg.height, bands=cfg.bands, lambda_min=cfg.lambda_min,
                      lambda_max=cfg.lambda_max, epsilon=cfg.epsilon, escape=cfg.escape,
                      max_path_length=cfg.max_path_length, scatter_bounces=cfg.scatter_bounces,
                      aspect_ratio=cfg.aspect_ratio, fov_scale=cfg.fov_scale, seed=cfg.seed, scene_id=scene_id)


def golden_compiled():
    """The reference's default scene as a CompiledScene + its own BVH (from the fixture)."""
    g = golden_scene()
    perm = g["bvh_perm"].astype(np.int64)
    inv = np.argsort(perm)
    tris = {k: np.ascontiguousarray(g[k][inv]) for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area",
                                                         "mat_id")}
    data = golden_data()
    B = 25
    eem = np.zeros((2, B, B), np.float32)
    eem[1] = data["ref_eem_uv_green"]
    cs = sb.scene.CompiledScene(tris=tris, mat_f32=g["mat_f32"], mat_i32=g["mat_i32"], mat_eem=g["mat_eem"],
                                eem=eem, cmf=np.ascontiguousarray(data["ref_cmf"], np.float32))
    bvh = {k: g[k] for k in ("node_min", "node_max", "node_left", "node_right", "node_num_tris", "node_tri_start")}
    bvh["tri_perm"] = g["bvh_perm"]
    cam = {"origin": g["camera"][0], "lookat": g["camera"][1], "up": g["camera"][2]}
    return cs, bvh, cam


def random_rays(n, seed, lo=-0.95, hi=0.95, origin_box=None):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3)) if origin_box is None else rng.uniform(origin_box[0], origin_box[1],
                                                                                 size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)


def camera_rays(cam, cfg_like_w, h, fov_scale=1.0, aspect=1.0, jitter_seed=None):
    o, u, v, w = camera_basis(cam["origin"], cam["lookat"], cam["up"])
    i, j = np.meshgrid(np.arange(cfg_like_w), np.arange(h), indexing="xy")
    off = 0.5 if jitter_seed is None else np.random.default_rng(jitter_seed).uniform(size=(2,) + i.shape)
    uu = (i + (off if np.isscalar(off) else off[0])) / cfg_like_w
    vv = (j + (off if np.isscalar(off) else off[1])) / h
    d = (u[None, None] * ((uu * 2 - 1) * aspect * fov_scale)[..., None] + v[None, None] * ((vv * 2 - 1) * fov_scale)[..., None]
         - w[None, None] * 2.0)
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    rays = np.concatenate([np.broadcast_to(o, d.shape), d], -1).reshape(-1, 6)
    return rays.astype(np.float32)
