"""Shared helpers of the test suite (inputs rebuilt exactly as the golden script built them)."""
import hashlib

import numpy as np

STATE_KEYS = ("h0", "h0p", "ub", "vb", "ubp", "vbp", "celerity_x", "celerity_y", "ub_ct",
              "vb_ct", "ub_cx", "ub_cy", "vb_cx", "vb_cy", "advx", "advy",
              "pax", "pxb", "whx", "pay", "pyb", "why", "wgp")
STAGE_OUT = ("new_h0", "new_ub", "new_vb", "celerity_x", "celerity_y", "ub_ct", "vb_ct",
             "ub_cx", "ub_cy", "vb_cx", "vb_cy", "advx", "advy")


def sha(arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def golden_inputs(z, grid):
    """The 23-field input state and 17 consts a golden fixture was made from."""
    from licom4py_gpu_b200.duogrid import make_consts
    from licom4py_gpu_b200.fields import harmonic_state
    n = int(z["n"])
    consts = make_consts(grid, float(z["depth"]))
    m = n + 6
    if "in_h0" in z:
        six = [z["in_" + k] for k in STATE_KEYS[:6]]
    else:
        st = harmonic_state(grid, int(z["seed"]))
        base = st if int(z["base_seed"]) < 0 else harmonic_state(grid, int(z["base_seed"]), 0.5, 0.1)
        six = [st["h0"], base["h0"], st["ub"], st["vb"], base["ub"], base["vb"]]
    state = six + [np.zeros((6, m, m)) for _ in range(17)]
    return state, consts


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / (scale if scale > 0 else 1.0))
