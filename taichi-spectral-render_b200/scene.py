"""Scene compilation: ``create_scene()`` dictionaries -> flat arrays for the C ABI.

Mirrors the host half of the reference (main.py:398-631): the scene dictionary
schema (``meshes`` with ``vertices``/``faces``/``material_id``/optional
``vertex_normals``, ``materials`` with per-band property lists, ``camera``),
``get_scene_dimensions`` and the triangle flattening of ``setup_scene``.  The
BVH build, triangle reordering and light CDF construction happen inside the
library (``ts_upload_scene``).
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib

# material property indices, main.py:38-51
PROP_REFRACTIVE_INDEX = 0
PROP_EXTINCTION_COEFFICIENT = 1
PROP_ROUGHNESS = 2
PROP_SCATTERING_COEFFICIENT = 3
PROP_EMISSION = 4
PROP_ANISTROPY_FACTOR = 5
NUM_F32_PROPERTIES = 6
PROP_IS_TRUE_VOLUME = 0
PROP_SURFACE_EMISSION = 1
NUM_INT_PROPERTIES = 2

F32_KEYS = ("refractive_index", "extinction_coefficient", "roughness", "scattering_coefficient", "emission",
            "anistropy_factor")
I32_KEYS = ("is_true_volume", "surface_emission")


def get_scene_dimensions(scene_dict, spectral_bands=25):
    """Field sizes of a scene, as main.py:398-435 computes them (without printing)."""
    mats = scene_dict.get("materials", [])
    num_triangles = sum(len(m.get("faces", [])) for m in scene_dict.get("meshes", []))
    lights_per_band = [0] * spectral_bands
    for mesh in scene_dict.get("meshes", []):
        emis = mats[mesh["material_id"]].get("surface_emission", [False] * spectral_bands)
        if any(emis):
            n = len(mesh.get("faces", []))
            for i in range(spectral_bands):
                if emis[i]:
                    lights_per_band[i] += n
    return {"num_materials": len(mats), "num_triangles": num_triangles,
            "num_bvh_nodes": max(0, 2 * num_triangles - 1),
            "max_num_lights_per_band": max(lights_per_band) if lights_per_band else 0}


def flatten_triangles(scene_dict, exact=None):
    """Triangles in original order, flattened as setup_scene does (main.py:513-539).

    Geometric normal = cross(v1 - v0, v2 - v0) normalised when the area exceeds
    1e-6, area = |cross| / 2, vertex normals from ``vertex_normals`` or the
    geometric normal, all float32.  ``exact=True`` evaluates every
    triangle with the same numpy calls as the reference (bit-identical; slow for
    millions of triangles); ``exact=False`` vectorises (identical up to the
    rounding of the norm's summation).  Default: exact below 50k triangles.
    """
    meshes = scene_dict["meshes"]
    total = sum(len(m["faces"]) for m in meshes)
    if exact is None:
        exact = total < 50000
    out = {k: [] for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area", "mat_id")}
    for mesh in meshes:
        verts = np.asarray(mesh["vertices"], dtype=np.float32).reshape(-1, 3)
        faces = np.asarray(mesh["faces"], dtype=np.int64).reshape(-1, 3)
        if faces.size and (faces.min() < 0 or faces.max() >= verts.shape[0]):
            raise ValueError("mesh face index out of range")
        vn = None
        if "vertex_normals" in mesh:
            vn = np.asarray(mesh["vertex_normals"], dtype=np.float32).reshape(-1, 3)
        v0, v1, v2 = verts[faces[:, 0]], verts[faces[:, 1]], verts[faces[:, 2]]
        if exact:
            nrm = np.empty_like(v0)
            area = np.empty(v0.shape[0], np.float32)
            for t in range(v0.shape[0]):
                n = np.cross(v1[t] - v0[t], v2[t] - v0[t])
                a = np.linalg.norm(n) / 2.0
                if a > 1e-6:
                    n /= (a * 2.0)
                nrm[t] = n
                area[t] = a
        else:
            raw = np.cross(v1 - v0, v2 - v0).astype(np.float32)
            area = (np.sqrt(np.einsum("ij,ij->i", raw, raw)) / np.float32(2.0)).astype(np.float32)
            nrm = raw.copy()
            big = area > 1e-6
            nrm[big] /= (area[big] * np.float32(2.0))[:, None]
        if vn is not None:
            n0, n1, n2 = vn[faces[:, 0]], vn[faces[:, 1]], vn[faces[:, 2]]
        else:
            # the reference aliases n0/n1/n2 to the normal array that it then
            # normalises in place, so they end up as the unit normal
            n0 = n1 = n2 = nrm
        out["v0"].append(v0)
        out["v1"].append(v1)
        out["v2"].append(v2)
        out["n0"].append(n0)
        out["n1"].append(n1)
        out["n2"].append(n2)
        out["normal"].append(nrm)
        out["area"].append(area)
        out["mat_id"].append(np.full(v0.shape[0], int(mesh["material_id"]), np.int32))
    res = {}
    for k, v in out.items():
        if v:
            res[k] = np.ascontiguousarray(np.concatenate(v), dtype=np.int32 if k == "mat_id" else np.float32)
        else:
            res[k] = np.zeros((0,) if k in ("area", "mat_id") else (0, 3),
                              dtype=np.int32 if k == "mat_id" else np.float32)
    return res


def material_tables(materials, spectral_bands):
    """[M][6][B] f32, [M][2][B] i32 and [M] EEM ids with the defaults of main.py:545-561."""
    M, B = len(materials), spectral_bands
    mf = np.zeros((M, NUM_F32_PROPERTIES, B), np.float32)
    mi = np.zeros((M, NUM_INT_PROPERTIES, B), np.int32)
    me = np.zeros(M, np.int32)
    for i, m in enumerate(materials):
        for p, key in enumerate(F32_KEYS):
            v = np.asarray(m.get(key, [0.0] * B), dtype=np.float64).reshape(-1)
            if v.shape[0] != B:
                raise ValueError(f"material {i}: '{key}' has {v.shape[0]} bands, expected {B}")
            mf[i, p] = v
        for p, key in enumerate(I32_KEYS):
            v = np.asarray(m.get(key, [0] * B)).reshape(-1)
            if v.shape[0] != B:
                raise ValueError(f"material {i}: '{key}' has {v.shape[0]} bands, expected {B}")
            mi[i, p] = v.astype(np.int32)
        me[i] = int(m.get("eem_id", 0))
    return mf, mi, me


@dataclass
class CompiledScene:
    """Flat arrays for ``ts_upload_scene`` (kept alive while the descriptor is in use)."""
    tris: dict
    mat_f32: np.ndarray
    mat_i32: np.ndarray
    mat_eem: np.ndarray
    eem: np.ndarray
    cmf: np.ndarray
    bvh: dict = None
    bvh_params: dict = field(default_factory=dict)

    @property
    def num_tris(self):
        return int(self.tris["area"].shape[0])

    def desc(self):
        f = lambda a: a.ctypes.data_as(_lib.F32P)
        i = lambda a: a.ctypes.data_as(_lib.I32P)
        t = self.tris
        d = _lib.TsSceneDesc()
        d.num_tris = self.num_tris
        for k in ("v0", "v1", "v2", "n0", "n1", "n2", "normal", "area"):
            setattr(d, k, f(t[k]))
        d.mat_id = i(t["mat_id"])
        d.num_materials = self.mat_f32.shape[0]
        d.mat_f32, d.mat_i32, d.mat_eem = f(self.mat_f32), i(self.mat_i32), i(self.mat_eem)
        d.num_eems = self.eem.shape[0]
        d.eem = f(self.eem)
        d.cmf = f(self.cmf)
        if self.bvh is not None:
            b = self.bvh
            d.bvh_num_nodes = b["node_num_tris"].shape[0]
            d.node_min, d.node_max = f(b["node_min"]), f(b["node_max"])
            d.node_left, d.node_right = i(b["node_left"]), i(b["node_right"])
            d.node_num_tris, d.node_tri_start = i(b["node_num_tris"]), i(b["node_tri_start"])
            d.tri_perm = i(b["tri_perm"])
        p = self.bvh_params
        d.bvh_bins = int(p.get("bins", 0))
        d.bvh_leaf_max = int(p.get("leaf_max", 0))
        d.bvh_cost_trav = float(p.get("cost_trav", 0.0))
        d.bvh_cost_tri = float(p.get("cost_tri", 0.0))
        d.bvh_width = int(p.get("width", 0))
        d.bvh_quantized = 1 if p.get("quantize", False) else 0
        return d


def compile_scene(scene_dict, spectral_bands, eems=None, cmf=None, bvh=None, bvh_params=None, exact=None):
    """Flatten a ``create_scene()`` dictionary.

    eems: None, a [E][B][B] array indexed by EEM id (row 0 unused, as the
    reference's ``reemission_matrix`` field), or a dict {id: [B][B]}.
    cmf: [B][3] colour-matching functions (zeros if None).
    bvh: optional tree in the reference layout (keys node_min node_max
    node_left node_right node_num_tris node_tri_start tri_perm), e.g. the
    reference's own build_bvh output, adopted instead of building one.
    """
    B = spectral_bands
    tris = flatten_triangles(scene_dict, exact=exact)
    mf, mi, me = material_tables(scene_dict["materials"], B)
    if eems is None:
        E = int(me.max()) + 1 if me.size else 1
        eem = np.zeros((E, B, B), np.float32)
    elif isinstance(eems, dict):
        E = max(max(eems.keys()) + 1, int(me.max()) + 1)
        eem = np.zeros((E, B, B), np.float32)
        for k, v in eems.items():
            eem[k] = np.asarray(v, np.float32)
    else:
        eem = np.ascontiguousarray(eems, dtype=np.float32).reshape(-1, B, B)
    if cmf is None:
        cmf = np.zeros((B, 3), np.float32)
    cmf = np.ascontiguousarray(cmf, dtype=np.float32).reshape(B, 3)
    bv = None
    if bvh is not None:
        bv = {k: np.ascontiguousarray(bvh[k], dtype=np.float32 if k in ("node_min", "node_max") else np.int32)
              for k in ("node_min", "node_max", "node_left", "node_right", "node_num_tris", "node_tri_start",
                        "tri_perm")}
    return CompiledScene(tris=tris, mat_f32=mf, mat_i32=mi, mat_eem=me, eem=eem, cmf=cmf, bvh=bv,
                         bvh_params=dict(bvh_params or {}))
