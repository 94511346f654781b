"""Serving with continuous batching on the GPU.

Every request's result must be the same alone (one bt_round of all its
substeps, nothing else on the GPU) and in the mix (batched rounds shared with
whatever else is admitted, rounds of 8 substeps, admission limited by a
budget of three members): float32 within 1e-6 relative (max-norm over h0, ub,
vb), float64 within 1e-12.
"""
import numpy as np
import pytest
import torch

from helpers import rel_err
from licom4py_gpu_b200.batch import member_bytes
from licom4py_gpu_b200.ensemble import Geometry
from licom4py_gpu_b200.serving import BarotropicServer, Request, run_fifo

pytestmark = pytest.mark.gpu

TOL = {torch.float32: 1e-6, torch.float64: 1e-12}
MIX = [(12, 17), (24, 5), (16, 40), (12, 3), (24, 23), (16, 9), (12, 31), (24, 12)]


@pytest.fixture(scope="module")
def geo():
    g = Geometry(5000.0, device="cuda")
    yield g
    g.close()


@pytest.mark.parametrize("dtype,order", [(torch.float32, "fifo"), (torch.float64, "fifo"),
                                         (torch.float32, "shortest")])
def test_results_same_alone_and_in_the_mix(dtype, order, geo):
    reqs = [Request(rid=k, n=n, nsub=ns, seed=100 + 3 * k, arrival=0.0) for k, (n, ns) in enumerate(MIX)]
    budget = 3 * member_bytes(geo.plan(24, dtype), 2)
    srv = BarotropicServer(geo, dtype=dtype, round_substeps=8, hbm_budget=budget, max_members=8, order=order)
    stats = srv.run(reqs, realtime=False)
    srv.close()
    assert stats["requests"] == len(MIX) and stats["rejected"] == 0
    assert srv.sched.peak <= budget
    assert stats["rounds"] >= 40 // 8  # the longest request alone needs 5 rounds
    assert max(r.t_admit for r in reqs) > 0.0  # some requests waited for memory to free up
    alone = [Request(rid=r.rid, n=r.n, nsub=r.nsub, seed=r.seed) for r in reqs]
    run_fifo(geo, alone, dtype=dtype, realtime=False)
    for a, b in zip(reqs, alone):
        for k in ("h0", "ub", "vb"):
            err = rel_err(a.result[k], b.result[k])
            assert err <= TOL[dtype], f"request {a.rid} (C{a.n}, {a.nsub} substeps) {k}: {err:.2e}"
        assert np.isfinite(a.result["h0"]).all()


def test_requests_arriving_later_join_running_rounds(geo):
    """Real-time arrivals: a request arriving while others run is admitted at a
    round boundary and finishes before the long request that started first."""
    reqs = [Request(rid=0, n=24, nsub=2000, seed=1, arrival=0.0),
            Request(rid=1, n=12, nsub=8, seed=2, arrival=0.01)]
    srv = BarotropicServer(geo, dtype=torch.float32, round_substeps=4, max_members=4)
    stats = srv.run(reqs, realtime=True)
    srv.close()
    assert stats["requests"] == 2
    assert reqs[1].t_admit >= reqs[1].arrival and reqs[1].t_done < reqs[0].t_done
    assert stats["p99_s"] >= stats["p50_s"] > 0


@pytest.mark.parametrize("n,seed,amp", [(12, 5, 1.0), (24, 77, 0.37), (48, 1234, 1.9)])
def test_device_initial_state_equals_seeded_field_generator(n, seed, amp, geo):
    """The serving path's device-built initial state (HarmonicBasis) is the seeded
    harmonic field of fields.harmonic_state (h RMS = amplitude, u/v RMS = 0.3 x
    amplitude), up to float64 rounding of the reordered sums: 1e-12 relative."""
    from licom4py_gpu_b200.fields import harmonic_state
    from licom4py_gpu_b200.serving import HarmonicBasis
    basis = HarmonicBasis(geo, torch.device("cuda"))
    got = basis.state(Request(rid=0, n=n, nsub=1, seed=seed, amplitude=amp), torch.float64)
    want = harmonic_state(geo.grid(n), seed, amp, 0.3 * amp)
    for t, key in zip(got, ("h0", "ub", "vb")):
        err = rel_err(t.cpu().numpy(), want[key])
        assert err <= 1e-12, f"C{n} seed {seed} {key}: rel err {err:.2e}"
