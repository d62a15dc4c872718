"""The C-ABI library loads and exports every entry point include/spectral.h declares."""
import ctypes
import os
import re

import pytest

from helpers import ROOT, sb
from spectral_b200 import _lib


def declared_functions():
    src = open(os.path.join(ROOT, "include", "spectral.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ts_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_api():
    names = declared_functions()
    for must in ("ts_create", "ts_upload_scene", "ts_render_pass", "ts_accumulate_block", "ts_resolve_xyz",
                 "ts_reset", "ts_trace_batch", "ts_set_camera", "ts_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    bound = {n for n, _, _ in _lib.SIGNATURES}
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in bound, f"{name} has no ctypes signature"


def test_library_built_for_sm100a():
    assert os.path.exists(_lib.LIB_PATH)
    assert b"sm_100a" in _lib.load().ts_version()


def test_create_reports_missing_device_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = sb.RenderConfig(width=4, height=4).to_c()
    ctx = ctypes.c_void_p()
    st = _lib.load().ts_create(ctypes.byref(cfg), ctypes.byref(ctx))
    assert st == 2 and not ctx.value
    assert b"no CUDA device" in _lib.load().ts_last_error(None)


C_SIZES = {"int32_t": 4, "uint32_t": 4, "float": 4, "double": 8, "size_t": 8, "uint64_t": 8}


def header_struct(name):
    """(field name, byte size) of a typedef struct of include/spectral.h, in order."""
    src = open(os.path.join(ROOT, "include", "spectral.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    body = re.search(r"typedef struct\s*\{([^{}]*)\}\s*" + name + r"\s*;", src).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(?:const\s+)?([a-z0-9_]+)\s+(.*)", decl)
        base, rest = m.group(1), m.group(2)
        for item in rest.split(","):
            item = item.strip()
            arr = re.match(r"(\**)\s*([a-z0-9_]+)\s*(?:\[(\d+)\])?", item)
            size = 8 if arr.group(1) else C_SIZES[base]
            fields.append((arr.group(2), size * (int(arr.group(3)) if arr.group(3) else 1)))
    return fields


@pytest.mark.parametrize("cname,pytype", [("ts_config", "TsConfig"), ("ts_scene_desc", "TsSceneDesc"),
                                          ("ts_scene_info", "TsSceneInfo"), ("ts_batch_config", "TsBatchConfig")])
def test_ctypes_structs_match_the_header(cname, pytype):
    """Every field of the C structs, in order and size, has its ctypes twin."""
    from spectral_b200 import batch
    st = getattr(_lib, pytype, None) or getattr(batch, pytype)
    py = [(n, ctypes.sizeof(t)) for n, t in st._fields_]
    assert py == header_struct(cname)


def test_config_validation_on_host():
    lib = _lib.load()
    ctx = ctypes.c_void_p()
    for bad in (dict(width=0), dict(bands=0), dict(bands=65), dict(scatter_bounces=0), dict(max_path_length=-1),
                dict(lambda_min=800.0, lambda_max=400.0), dict(queue_capacity=-1), dict(queue_capacity=(1 << 25) + 1),
                dict(occupancy=3)):
        cfg = sb.RenderConfig(**{**dict(width=4, height=4), **bad}).to_c()
        assert lib.ts_create(ctypes.byref(cfg), ctypes.byref(ctx)) == 1, bad


def test_renderer_refuses_to_run_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from spectral_b200 import configs
    s, c, ex = configs.box_scene(width=8, height=8)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"])


def integration_python_blocks():
    """The ```python blocks of INTEGRATION.md."""
    src = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```python\n(.*?)```", src, flags=re.S)


def test_integration_doc_structs_match_the_header():
    """A host that copies INTEGRATION.md's ctypes binding gets structs of the
    header's layout: every documented Structure class is executed and compared
    field by field (name, size, offset) with include/spectral.h, and the
    documented positional constructor fills every field."""
    import ast
    found = 0
    for block in integration_python_blocks():
        tree = ast.parse(block)
        for node in tree.body:
            if not (isinstance(node, ast.ClassDef) and node.name.startswith("ts_")):
                continue
            ns = {"ctypes": ctypes}
            exec(compile(ast.Module(body=[node], type_ignores=[]), "INTEGRATION.md", "exec"), ns)
            st = ns[node.name]
            py = [(n, ctypes.sizeof(t)) for n, t in st._fields_]
            assert py == header_struct(node.name), node.name
            offs = [getattr(st, n).offset for n, _ in st._fields_]
            assert offs == [sum(sz for _, sz in py[:i]) for i in range(len(py))], node.name
            found += 1
            # positional constructions in the same block give a value for every field
            for call in ast.walk(tree):
                if isinstance(call, ast.Call) and isinstance(call.func, ast.Name) and call.func.id == node.name \
                        and call.args:
                    assert len(call.args) == len(st._fields_), (node.name, len(call.args))
    assert found >= 1


def test_new_entry_points_validate_arguments_without_a_gpu():
    """ts_create_view, ts_record_paths and ts_set_loop_iteration_limit reject
    null handles before touching a device."""
    lib = _lib.load()
    out = ctypes.c_void_p()
    cfg = sb.RenderConfig(width=4, height=4).to_c()
    assert lib.ts_create_view(None, ctypes.byref(cfg), ctypes.byref(out)) == 1 and not out.value
    assert b"null argument" in lib.ts_last_error(None)
    assert lib.ts_record_paths(None, 0, 4) == 1
    assert lib.ts_set_loop_iteration_limit(None, 3) == 1


def test_batch_config_carries_the_engine_fields():
    from spectral_b200 import batch
    names = [n for n, _ in batch.TsBatchConfig._fields_]
    assert names[-3:] == ["kernel", "queue_capacity", "trace_budget"]
    assert ctypes.sizeof(batch.TsBatchConfig) == 7 * 4
