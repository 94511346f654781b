"""bt_round_noalloc: the round for callers that cannot allocate device memory.

Such callers (a runtime's custom-call handler that is given only its operand
buffers, a model driver that reserves its GPU memory up front, a service whose
memory footprint is fixed) call bt_round_noalloc, which keeps its scratch in a
fixed array the library declares statically.  Its results must match the plan
based bt_round within the float64 tolerance of the other GPU tests (1e-12
relative; the same kernels run, so they are expected to be identical), on two
calls in a row (the second call finds the first call's contents in the shared
array).  Float32 is held to 1e-6 relative.  The tests also check the
documented size limits, that the tables are checked as bt_plan_create checks
them, and that a call after a warm-up call leaves the device's free memory
unchanged.  This file is named to be collected last.
"""
import ctypes
import gc

import numpy as np
import pytest
import torch

from licom4py_gpu_b200 import _native as N
from licom4py_gpu_b200.duogrid import make_consts
from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state
from licom4py_gpu_b200.plan import DIAG_NAMES, BtPlan

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc_round(plan, ins, nbb, dtb, rk, out=None, consts=None):
    c = plan.consts if consts is None else consts
    desc = N.GridDesc(plan.n, N.BT_F64 if plan.dtype == torch.float64 else N.BT_F32,
                      *[c[k].data_ptr() for k in ("dzph_x", "dzph_y", "rdx", "rdy", "a_f", "k2e_coef",
                                                  "loc_i_local", "loc_j_local", "a_c2l", "a_l2c", "inner",
                                                  "outer", "a_gct", "a_sina", "rda", "c_dy", "d_dx")])
    if out is None:
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


def _inputs(g, seed, dtype=torch.float64):
    st = harmonic_state(g, seed)
    return [torch.from_numpy(np.ascontiguousarray(st[k])).to("cuda", dtype)
            for k in ("h0", "h0", "ub", "vb", "ub", "vb")]


# float64 at 1e-12; the float32 case at the float32 tolerance of the other GPU
# tests (1e-6 relative, max norm), against a float32 plan of the same tile shape
@pytest.mark.parametrize("n,rk,dtype", [(24, 2, torch.float64), (48, 3, torch.float64), (24, 2, torch.float32),
                                        (96, 3, torch.float64), (112, 2, torch.float64)])
def test_noalloc_matches_round_on_two_calls(n, rk, dtype, grids):
    g = grids(n)
    consts = make_consts(g, 5000.0)
    dtb = cfl_dtb(g, 5000.0)
    plan = BtPlan(consts, dtype=dtype, tile=(8, 16))
    tol = TOL if dtype == torch.float64 else 1e-6
    for call, seed in enumerate((31, 32)):  # two calls in a row, different states
        ins = _inputs(g, seed, dtype)
        want = plan.round(*ins, nbb=4, dtb=dtb, rk=rk)
        got = _noalloc_round(plan, ins, 4, dtb, rk)
        torch.cuda.synchronize()
        for k in want:
            assert _rel(got[k].double(), want[k].double()) <= tol, (call, k)
    plan.close()


def test_noalloc_allocates_no_device_memory(grids):
    """After a warm-up call, a second call changes neither torch's allocation
    count nor the device's free memory (cudaMemGetInfo)."""
    g = grids(48)
    plan = BtPlan(make_consts(g, 5000.0))
    ins = _inputs(g, 5)
    dtb = cfl_dtb(g, 5000.0)
    _noalloc_round(plan, ins, 2, dtb, 2)  # warm-up: set-up, table check, lazy kernel loading
    out = {k: plan.empty_field() for k in ("h0", "ub", "vb") + DIAG_NAMES}
    gc.collect()  # plans of earlier tests free their memory when collected, not during the call
    torch.cuda.synchronize()
    torch_before, free_before = torch.cuda.memory_allocated(), torch.cuda.mem_get_info()[0]
    _noalloc_round(plan, ins, 3, dtb, 2, out=out)
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated() == torch_before
    assert torch.cuda.mem_get_info()[0] >= free_before  # nothing was allocated on the device
    plan.close()


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch(grids):
    for n, rk in ((113, 2), (97, 3)):  # float64 limits: N <= 112 (rk 2), N <= 96 (rk 3)
        g = grids(n)
        plan = BtPlan(make_consts(g, 5000.0))
        with pytest.raises(ValueError, match="scratch"):
            _noalloc_round(plan, _inputs(g, 1), 1, 10.0, rk)
        plan.close()


def test_noalloc_checks_the_tables_like_plan_create(grids):
    """A k2e location outside the band (BT_EINVAL) and a mask that is not 0/1
    (BT_ENOTSUP) are refused, as bt_plan_create refuses them."""
    g = grids(24)
    consts = make_consts(g, 5000.0)
    plan = BtPlan(consts)
    ins = _inputs(g, 2)
    bad_loc = {k: v.clone() for k, v in plan.consts.items()}
    bad_loc["loc_i_local"][0, 10, 1] = 0  # W band cell of face 0
    with pytest.raises(ValueError, match="location"):
        _noalloc_round(plan, ins, 1, 10.0, 2, consts=bad_loc)
    bad_mask = {k: v.clone() for k, v in plan.consts.items()}
    bad_mask["inner"][2, 5, 5] = 0.5
    with pytest.raises(NotImplementedError, match="masks"):
        _noalloc_round(plan, ins, 1, 10.0, 2, consts=bad_mask)
    # the valid set still runs (and matches bt_round)
    want = plan.round(*ins, nbb=2, dtb=10.0)
    got = _noalloc_round(plan, ins, 2, 10.0, 2)
    torch.cuda.synchronize()
    assert _rel(got["h0"], want["h0"]) <= TOL
    plan.close()
