"""Host-side pieces of the batched ensemble (no GPU): the uneven mix and the
batch autotuner's cache key."""
import numpy as np

from licom4py_gpu_b200.ensemble import UV_PER_H, MemberSpec, uneven_mix


def test_uneven_mix_default_counts_and_ranges():
    specs = uneven_mix(seed=0)
    ns = [s.n for s in specs]
    assert ns.count(48) == 32 and ns.count(96) == 24 and ns.count(192) == 8
    assert all(200 <= s.nsub <= 2000 for s in specs)
    assert all(0.2 <= s.amplitude <= 2.0 for s in specs)
    assert len({s.seed for s in specs}) == len(specs)
    # deterministic per seed, different across seeds
    assert uneven_mix(seed=0) == specs
    assert uneven_mix(seed=1) != specs
    # the draws spread over their ranges (substeps uniform on 200..2000)
    steps = np.array([s.nsub for s in uneven_mix(counts={48: 4000}, seed=3)])
    assert abs(steps.mean() - 1100) < 30 and steps.min() < 260 and steps.max() > 1940


def test_mix_cells_and_uv_ratio():
    specs = uneven_mix(counts={12: 2, 24: 1}, nsub=(5, 5), amplitude=(1.0, 1.0), seed=7)
    assert [s.n for s in specs] == [12, 12, 24]
    assert sum(6 * s.n * s.n * s.nsub for s in specs) == 5 * 6 * (2 * 144 + 576)
    assert UV_PER_H == 0.3 and isinstance(specs[0], MemberSpec)


def test_batch_tune_key_depends_on_the_mix_only():
    import torch
    from licom4py_gpu_b200 import autotune
    orig = torch.cuda.get_device_name
    torch.cuda.get_device_name = lambda device=None: "B200"
    try:
        a = autotune._mix_key(uneven_mix(seed=0), torch.float32, 2, None)
        b = autotune._mix_key(uneven_mix(seed=5), torch.float32, 2, None)
        c = autotune._mix_key(uneven_mix(seed=0), torch.float64, 2, None)
    finally:
        torch.cuda.get_device_name = orig
    assert a == b and a != c and "C48x32" in a and "C192x8" in a
