"""Scheduler entry (Schedule.configure/run, schedule_core), on-device diagnostics and
conservation sums, and the W92 case-2 known-answer behaviour."""
import numpy as np
import pytest
import torch

from licom4py_gpu_b200 import schedule
from licom4py_gpu_b200.duogrid import Duogrid, make_consts
from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state, w92_case2_state
from licom4py_gpu_b200.momentum import Momentum, Namelist, conservation, interior_stats
from oracle import barotr_np as O

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def test_schedule_core_matches_oracle(grids):
    n = 12
    g = grids(n)
    consts = make_consts(g, 5000.0)
    st = harmonic_state(g, 21)
    m = n + 6
    state = [st["h0"], st["h0"], st["ub"], st["vb"], st["ub"], st["vb"]] + [np.zeros((6, m, m))] * 17
    extra = torch.ones(3, device="cuda")  # fields beyond the barotropic 23 pass through
    dtb = cfl_dtb(g, 5000.0)
    core = schedule._make_schedule_core(2)
    fn = schedule.make_plan_fn(core, tuple(dev(s) for s in state), consts)
    out = fn(tuple(dev(s) for s in state) + (extra,), consts, 3, 2, dtb)
    assert len(out) == 24 and out[23] is extra
    want = O.rk2_core(state, consts, 6, dtb)
    for k in range(16):
        np.testing.assert_array_equal(out[k].cpu().numpy(), want[k])


def test_interior_stats_and_conservation(grids):
    n = 24
    g = grids(n)
    st = harmonic_state(g, 3)
    h = dev(st["h0"])
    s = interior_stats(h).cpu().numpy()
    ih = st["h0"][:, 3:-3, 3:-3]
    assert s[0] == ih.max() and s[1] == ih.min()
    assert abs(s[2] - ih.mean()) <= 1e-15 * np.abs(ih).max()
    rda, c2l = dev(g["rda"]), dev(g["a_c2l"])
    mass, energy = conservation(h, dev(st["ub"]), dev(st["vb"]), rda, c2l, 5000.0).cpu().numpy()
    da = 1.0 / g["rda"][:, 3:-3, 3:-3]
    np.testing.assert_allclose(mass, (ih * da).sum(), rtol=1e-13)
    ul = g["a_c2l"][..., 0, 0] * st["ub"] + g["a_c2l"][..., 0, 1] * st["vb"]
    vl = g["a_c2l"][..., 1, 0] * st["ub"] + g["a_c2l"][..., 1, 1] * st["vb"]
    e = (0.5 * 9.8 * ih * ih + 0.5 * (5000.0 + ih) * (ul[:, 3:-3, 3:-3] ** 2 + vl[:, 3:-3, 3:-3] ** 2)) * da
    np.testing.assert_allclose(energy, e.sum(), rtol=1e-12)
    # float32 terms, compensated float64 sums: close to the float64 result
    m32, e32 = conservation(h.float(), dev(st["ub"]).float(), dev(st["vb"]).float(), rda.float(), c2l.float(),
                            5000.0).cpu().numpy()
    assert abs(m32 - mass) <= 1e-6 * (np.abs(ih) * da).sum()
    assert abs(e32 / energy - 1.0) < 1e-5


def test_schedule_run_w92_steady_state(capsys):
    """W92 case 2 is a steady geostrophic flow: after a model day the interior h changes little."""
    Duogrid.configure(24, depth=5600.0)
    nl = Namelist(barotropic_dt=600.0, baroclinic_dt=3600.0, integration_days=1.0, diag_freq=6.0,
                  async_threads=2, nx=24)
    mom = Momentum(nl, case="w92case2")
    h_init = mom.h0.clone()
    schedule.Schedule.configure(nl, mom)
    schedule.Schedule.run(mom)
    assert len(schedule.Schedule.reports) == 1 + 4  # initial + every 6 h of one day
    assert "Global h0:" in schedule.Schedule.reports[-1]
    dh = (mom.h0 - h_init)[:, 3:-3, 3:-3].abs().max().item()
    amp = h_init[:, 3:-3, 3:-3].abs().max().item()
    assert dh < 0.05 * amp, f"W92 drifted by {dh:.3f} m of {amp:.1f} m"
    # the same 24 substeps with the oracle
    g = Duogrid.grid_dict()
    consts = make_consts(g, 5600.0)
    s0 = w92_case2_state(g)
    m = 30
    state = [s0["h0"], s0["h0"], s0["ub"], s0["vb"], s0["ub"], s0["vb"]] + [np.zeros((6, m, m))] * 17
    want = O.rk2_core(state, consts, 24 * 6, 600.0)
    np.testing.assert_array_equal(mom.h0.cpu().numpy(), want[0])


def test_schedule_configure_with_reference_namelist():
    """Schedule.configure/run driven by an object shaped like the reference's Namelist
    (private _start_datetime / _total_baroclinic_steps only)."""
    from test_schedule_host import RefLikeNamelist
    Duogrid.configure(24, depth=5600.0)
    mom = Momentum(Namelist(barotropic_dt=600.0, baroclinic_dt=3600.0, integration_days=1.0, nx=24),
                   case="w92case2")
    mom.verbose = False
    ref_nl = RefLikeNamelist(baroclinic_dt=3600, diag_freq=12, async_threads=2, _total_baroclinic_steps=24)
    schedule.Schedule.configure(ref_nl, mom)
    assert schedule.Schedule.total_baroclinic_steps == 24
    schedule.Schedule.run(mom)
    reports = schedule.Schedule.reports
    assert len(reports) == 1 + 2  # initial + every 12 h of one day
    assert "2001-03-04-05" in reports[0] and "2001-03-05-05" in reports[-1]

