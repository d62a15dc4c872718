"""Shared helpers for the tests: oracle scenes that match a GPU upload slot for slot."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import orc  # noqa: E402
from orc import camera_basis, light_tables, oracle_config, oracle_scene  # noqa: E402,F401
import spectral_b200 as sb  # noqa: E402
from spectral_b200 import _lib  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden_scene():
    return dict(np.load(os.path.join(GOLDEN, "scene_ref.npz")))


def golden_data():
    return dict(np.load(os.path.join(GOLDEN, "data_ref.npz")))


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
