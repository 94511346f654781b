"""Drop-in single RK stage: ``_step_rk_logic`` (src/licom/momentum/barotr_pure.py:100-168).

Runs one stage on the GPU with the inputs' halo cells used as given and
returns the reference's 13 arrays: new_h0, new_ub, new_vb (halos filled by
ext_scalar / ext_vector) and celerity_x, celerity_y, ub_ct, vb_ct, ub_cx,
ub_cy, vb_cx, vb_cy, advx, advy of the stage.
"""

from __future__ import annotations

from .barotr import get_plan, _state_dtype
from .plan import DIAG_NAMES, to_device


def _step_rk_logic(h0, h0p, ub, vb, ubp, vbp, consts, dt, beta_d, is_laststep, px, py):
    if px != 1 or py != 1:
        raise ValueError(f"px = py = 1 is required (got px={px}, py={py})")
    dtype = _state_dtype((h0,))
    plan = get_plan(consts, dtype=dtype)
    ins = [to_device(a, dtype, plan.device) for a in (h0, h0p, ub, vb, ubp, vbp)]
    out = plan.stage(*ins, dt=float(dt), beta_d=float(beta_d), is_laststep=bool(is_laststep))
    return (out["h0"], out["ub"], out["vb"]) + tuple(out[k] for k in DIAG_NAMES)
