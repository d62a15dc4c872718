"""Host logic of the autotuner's candidate lists (no GPU)."""
from spectral_b200 import autotune


def test_bundle_wavefront_candidates_cover_capacities_up_to_the_bundle():
    c = autotune.bundle_wavefront_candidates(1024 * 1024, 25)
    caps = sorted({x.queue_capacity for x in c})
    assert caps == [2 << 20, 4 << 20, 8 << 20, 16 << 20, 25 << 20]
    # node layouts: two-child, 4-wide, and quantized 4- and 8-wide
    assert {(x.width, x.quantize) for x in c} == {(2, False), (4, False), (4, True), (8, True)}
    assert {x.trace_budget for x in c} == {8, 16} and len(c) == 4 * 5 * 2
    assert all(x.bvh_params() == {"width": x.width, "quantize": x.quantize} for x in c)
    assert all(x.kernel == "wavefront" and x.sort_keys == 0 for x in c)
    # small frames: capped by the whole bundle; huge frames: by the slot limit
    assert max(x.queue_capacity for x in autotune.bundle_wavefront_candidates(64 * 64, 25)) == 25 * 64 * 64
    assert max(x.queue_capacity for x in autotune.bundle_wavefront_candidates(4096 * 4096, 25)) == 1 << 25


def test_candidates_apply_the_queue_capacity():
    from spectral_b200 import RenderConfig
    cfg = autotune.Candidate(4, "default", "wavefront", 128, 0, 0, 16, queue_capacity=12345).apply(RenderConfig())
    assert cfg.kernel == "wavefront" and cfg.queue_capacity == 12345 and cfg.trace_budget == 16
