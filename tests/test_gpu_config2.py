"""Config 2 as stated: the plain drop-in at C96 over 1000 RK2 substeps, against the float64 oracle.

Workload: C96 (6 x 96 x 96 cells + 3-cell halos), seeded harmonic fields (seed 1,
h 1 m RMS, u/v 0.3 m/s RMS over H = 5000 m, the bench's inputs), dtb at CFL 0.5 of
sqrt(g H), 1000 midpoint-RK2 substeps (src/licom/momentum/barotr.py:41-61).

Tolerances:
  * float64 through ``_barotr_rk2_core`` and in resident mode: 1e-12 relative
    (max norm) on every state field, expected bit for bit;
  * float32 precision form: 1e-5 relative L2 on h after the 1000 substeps (the
    stated bound), u and v reported and held to the same bound.
The oracle run takes about 40 s on one host core; the fixture computes it once.
"""
import numpy as np
import pytest
import torch

from helpers import STATE_KEYS, rel_err
from licom4py_gpu_b200 import barotr
from licom4py_gpu_b200.duogrid import make_consts
from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state
from licom4py_gpu_b200.plan import BtPlan
from oracle import barotr_np as O

pytestmark = pytest.mark.gpu

N, NBB, SEED, DEPTH = 96, 1000, 1, 5000.0


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


@pytest.fixture(scope="module")
def case(grids):
    g = grids(N)
    consts = make_consts(g, DEPTH)
    st = harmonic_state(g, SEED)
    m = N + 6
    state = [st["h0"], st["h0"], st["ub"], st["vb"], st["ub"], st["vb"]] + [np.zeros((6, m, m))] * 17
    dtb = cfl_dtb(g, DEPTH)
    want = O.rk2_core(state, consts, NBB, dtb)
    return state, consts, dtb, want


def test_config2_float64_dropin_matches_oracle(case):
    state, consts, dtb, want = case
    got = barotr._barotr_rk2_core(tuple(dev(s) for s in state), consts, NBB, dtb, 1, 1)
    for k in range(16):
        err = rel_err(got[k].cpu().numpy(), want[k])
        assert err <= 1e-12, f"{STATE_KEYS[k]}: rel err {err:.3e}"
    for k in (0, 2, 3):
        np.testing.assert_array_equal(got[k].cpu().numpy(), want[k])


def test_config2_float64_resident_matches_oracle(case):
    state, consts, dtb, want = case
    p = BtPlan(consts, tile=(8, 16), mode="resident")
    out = p.round(*[dev(s) for s in state[:6]], nbb=NBB, dtb=dtb)
    p.check_device_error()
    for k, key in ((0, "h0"), (2, "ub"), (3, "vb")):
        np.testing.assert_array_equal(out[key].cpu().numpy(), want[k])
    p.close()


def test_config2_float32_within_1e5_of_oracle(case):
    state, consts, dtb, want = case
    p = BtPlan(consts, dtype=torch.float32, tile=(8, 16), mode="graph")
    out = p.round(*[dev(s, torch.float32) for s in state[:6]], nbb=NBB, dtb=dtb, diag=False)
    for k, key in ((0, "h0"), (2, "ub"), (3, "vb")):
        got = out[key].double().cpu().numpy()[:, 3:-3, 3:-3]
        ref = want[k][:, 3:-3, 3:-3]
        l2 = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert l2 <= 1e-5, f"{key}: relative L2 error {l2:.2e} after {NBB} substeps"
    p.close()
