"""bt_round_noalloc: the round for callers that cannot allocate device memory.

Such callers (a runtime's custom-call handler that is given only its operand
buffers, a model driver that reserves its GPU memory up front, a service whose
memory footprint is fixed) call bt_round_noalloc, which keeps its scratch in a
fixed array the library declares statically.  Its results must match the plan
based bt_round within the float64 tolerance of the other GPU tests (1e-12
relative; the same kernels run, so they are expected to be identical), on two
calls in a row (the second call finds the first call's contents in the shared
array).  This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from licom4py_gpu_b200 import _native as N
from licom4py_gpu_b200.duogrid import make_consts
from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state
from licom4py_gpu_b200.plan import DIAG_NAMES, BtPlan

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc_round(plan, ins, nbb, dtb, rk):
    c = plan.consts
    desc = N.GridDesc(plan.n, N.BT_F64 if plan.dtype == torch.float64 else N.BT_F32,
                      *[c[k].data_ptr() for k in ("dzph_x", "dzph_y", "rdx", "rdy", "a_f", "k2e_coef",
                                                  "loc_i_local", "loc_j_local", "a_c2l", "a_l2c", "inner",
                                                  "outer", "a_gct", "a_sina", "rda", "c_dy", "d_dx")])
    out = {k: plan.empty_field() for k in ("h0", "ub", "vb") + DIAG_NAMES}
    sin = N.StateIn(*[t.data_ptr() for t in ins])
    sout = N.StateOut(out["h0"].data_ptr(), out["ub"].data_ptr(), out["vb"].data_ptr(),
                      (ctypes.c_void_p * 10)(*[out[k].data_ptr() for k in DIAG_NAMES]))
    rc = N.lib().bt_round_noalloc(ctypes.byref(desc), ctypes.byref(sin), ctypes.byref(sout), nbb, float(dtb), rk,
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc)
    return out


def _rel(a, b):
    scale = b.abs().max().item()
    return (a - b).abs().max().item() / (scale if scale > 0 else 1.0)


@pytest.mark.parametrize("n,rk", [(24, 2), (48, 3)])
def test_noalloc_matches_round_on_two_calls(n, rk, grids):
    g = grids(n)
    consts = make_consts(g, 5000.0)
    dtb = cfl_dtb(g, 5000.0)
    plan = BtPlan(consts)
    for call, seed in enumerate((31, 32)):  # two calls in a row, different states
        st = harmonic_state(g, seed)
        ins = [torch.from_numpy(np.ascontiguousarray(st[k])).cuda() for k in ("h0", "h0", "ub", "vb", "ub", "vb")]
        want = plan.round(*ins, nbb=4, dtb=dtb, rk=rk)
        got = _noalloc_round(plan, ins, 4, dtb, rk)
        torch.cuda.synchronize()
        for k in want:
            assert _rel(got[k], want[k]) <= TOL, (call, k)
    plan.close()


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch(grids):
    g = grids(192)
    plan = BtPlan(make_consts(g, 5000.0))
    st = harmonic_state(g, 1)
    ins = [torch.from_numpy(np.ascontiguousarray(st[k])).cuda() for k in ("h0", "h0", "ub", "vb", "ub", "vb")]
    with pytest.raises(ValueError, match="scratch"):
        _noalloc_round(plan, ins, 1, 10.0, 2)
    plan.close()
