"""Drop-in barotropic RK cores: ``_barotr_rk2_core`` / ``_barotr_rk3_core``.

Same signature, argument meaning and state layout as the reference
(src/licom/momentum/barotr.py:41-87):

    state  -- the 23 STATE_KEYS arrays (src/licom/mymodule/schedule.py:62-92)
    consts -- the 17 CONST_SOURCES arrays (schedule.py:95-116)
    nbb    -- number of barotropic substeps (int)
    dtb    -- barotropic step (float)
    px, py -- per-tile mesh split; all six faces live on one GPU, so only
              px = py = 1 is valid (anything else raises ValueError)

Arrays are CUDA ``torch.Tensor`` (float64 for the drop-in, float32 for the
precision form); NumPy arrays are accepted and copied to the device once.
The return value is a new 23-tuple: h0 = h0p, ub = ubp, vb = vbp
(barotr.py:59), the ten diagnostics of the last stage, and the seven
coupling fields state[16:23] passed through as the very same objects.
"""

from __future__ import annotations

from typing import Dict, Sequence, Tuple

import numpy as np
import torch

from .plan import BtPlan, DIAG_NAMES, to_device

N_STATE = 23
N_CONSTS = 17

_PLANS: Dict[tuple, BtPlan] = {}
_PLAN_CACHE_MAX = 16


def _const_key(consts: Sequence, dtype, device) -> tuple:
    ids = []
    for c in consts[:N_CONSTS]:
        ids.append(("t", c.data_ptr(), tuple(c.shape), str(c.dtype)) if isinstance(c, torch.Tensor) else ("o", id(c)))
    return (str(dtype), str(device), tuple(ids))


def get_plan(consts: Sequence, dtype=torch.float64, device=None) -> BtPlan:
    """The cached plan for these constants (built on first use, like the JIT compile)."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    key = _const_key(consts, dtype, dev)
    plan = _PLANS.get(key)
    if plan is None:
        if len(_PLANS) >= _PLAN_CACHE_MAX:
            _PLANS.pop(next(iter(_PLANS))).close()
        plan = BtPlan(consts, dtype=dtype, device=dev)
        plan._const_refs = tuple(consts[:N_CONSTS])  # keep the key's objects alive
        _PLANS[key] = plan
    return plan


def clear_plans() -> None:
    while _PLANS:
        _PLANS.popitem()[1].close()


def _check_args(state, consts, nbb, px, py):
    if px != 1 or py != 1:
        raise ValueError(
            f"px = py = 1 is required: all six faces are held by one GPU (got px={px}, py={py})")
    if len(state) != N_STATE:
        raise ValueError(f"state must be the {N_STATE} STATE_KEYS arrays, got {len(state)}")
    if len(consts) < N_CONSTS:
        raise ValueError(f"consts must be the {N_CONSTS} CONST_SOURCES arrays, got {len(consts)}")
    if int(nbb) != nbb or nbb < 0:
        raise ValueError(f"nbb must be a non-negative integer, got {nbb}")


def _state_dtype(state) -> torch.dtype:
    h0 = state[0]
    if isinstance(h0, torch.Tensor):
        return h0.dtype
    return torch.float32 if np.asarray(h0).dtype == np.float32 else torch.float64


def _run_core(state, consts, nbb, dtb, px, py, rk: int):
    _check_args(state, consts, nbb, px, py)
    if nbb == 0:  # fori_loop(0, 0, ...) returns the state unchanged
        return tuple(state)
    dtype = _state_dtype(state)
    plan = get_plan(consts, dtype=dtype)
    ins = [to_device(s, dtype, plan.device) for s in state[:6]]
    out = plan.round(*ins, nbb=int(nbb), dtb=float(dtb), rk=rk, diag=True)
    h0, ub, vb = out["h0"], out["ub"], out["vb"]
    return (h0, h0, ub, vb, ub, vb) + tuple(out[k] for k in DIAG_NAMES) + tuple(state[16:23])


def _barotr_rk2_core(state, consts, nbb, dtb, px, py):
    """Midpoint RK2 over nbb substeps (src/licom/momentum/barotr.py:41-61)."""
    return _run_core(state, consts, nbb, dtb, px, py, rk=2)


def _barotr_rk3_core(state, consts, nbb, dtb, px, py):
    """Three-stage RK (dt/3, dt/2, dt; beta_d = 1) over nbb substeps (barotr.py:64-87)."""
    return _run_core(state, consts, nbb, dtb, px, py, rk=3)
