"""Host logic of bench.py (no GPU): the workload description both arms print,
the second cameras of the batched workload, the committed traffic figures."""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_turned_camera_keeps_position_and_turns_the_view_about_up():
    cam = {"origin": [0.0, 0.0, 0.49], "lookat": [0.0, -0.05, -0.5], "up": [0.0, 1.0, 0.0]}
    t = bench.turned_camera(cam, 20.0)
    assert np.allclose(t["origin"], cam["origin"])
    assert np.allclose(t["up"], cam["up"])
    d0 = np.subtract(cam["lookat"], cam["origin"])
    d1 = np.subtract(t["lookat"], t["origin"])
    assert np.isclose(np.linalg.norm(d0), np.linalg.norm(d1))
    # the component along up is kept; the horizontal part turns by 20 degrees
    assert np.isclose(d0[1], d1[1])
    h0, h1 = d0[[0, 2]], d1[[0, 2]]
    cos = h0 @ h1 / (np.linalg.norm(h0) * np.linalg.norm(h1))
    assert np.isclose(np.degrees(np.arccos(cos)), 20.0)
    assert np.allclose(bench.turned_camera(cam, 0.0)["lookat"], cam["lookat"])


def test_step_config_is_the_same_dictionary_in_both_arms():
    from spectral_b200 import RenderConfig
    cfg = RenderConfig(width=64, height=32)
    ex = {"spp": 25}
    a = bench.step_config(cfg, ex, "desc", 1, 1000)
    b = bench.step_config(cfg, ex, "desc", 1, 1000)
    assert a == b
    assert a["paths_per_step"] == cfg.bands * 64 * 32 and a["passes_per_step"] == cfg.bands
    assert "fit in L2" in a["l2"]
    big = bench.step_config(RenderConfig(width=1024, height=1024), ex, "desc", 1, 2_590_000)
    assert "larger than L2" in big["l2"]


def test_committed_traffic_entries_are_per_pass_and_name_their_source():
    d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    for key, e in d.items():
        assert e["dram_bytes_per_launch"] > 0, key
        assert "ncu" in e["source"], key
    loop = d["terrain:wavefront:w4:bundle"]
    # 784 B per path x 1,048,576 paths per pass
    assert abs(loop["dram_bytes_per_launch"] - loop["bytes_per_path"] * 1048576) < 1e-3 * loop["dram_bytes_per_launch"]
    assert bench.profiled_traffic("wavefront", "terrain", 4, 0, True) == loop["dram_bytes_per_launch"]
