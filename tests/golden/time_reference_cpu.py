"""Time the reference's own hot-path source against the float64 oracle port on the CPU.

The reference is Python (JAX); it cannot travel to the GPU machine, so the
timed CPU baseline there is the oracle port (oracle/barotr_np.py).  This script
shows what that stand-in is worth: on one host core it runs, on the same C{N}
inputs, (a) the reference's UNMODIFIED ``_barotr_rk2_core``
(src/licom/momentum/barotr.py:41-61, with barotr_pure.py, operators/*.py,
cube.py and communication.py) under the NumPy stand-in for ``jax`` that the
golden fixtures are made with, and (b) the oracle port, checks that both give
the same h/u/v bit for bit, and prints their cell-update rates as one JSON line.
JAX itself is not installed here, so ``jax.jit`` cannot be timed.

Usage:  python tests/golden/time_reference_cpu.py --ref PATH_TO_REFERENCE [--n 96] [--substeps 10]
        (or set LICOM_REFERENCE_ROOT)
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

for _var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ[_var] = "1"

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

import make_golden as G  # noqa: E402  (puts the jax stand-in and the repo on the path)
from oracle import barotr_np as O  # noqa: E402


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--ref", default=os.environ.get("LICOM_REFERENCE_ROOT"))
    p.add_argument("--n", type=int, default=96)
    p.add_argument("--substeps", type=int, default=10)
    p.add_argument("--seed", type=int, default=1)
    a = p.parse_args()
    if not a.ref:
        p.error("give --ref PATH_TO_REFERENCE or set LICOM_REFERENCE_ROOT")
    R = G.load_reference(a.ref, a.n)
    grid, consts, state, dtb = G.build_case(a.n, 5000.0, a.seed)
    cells = 6 * a.n * a.n
    st = tuple(G.A(s) for s in state)
    cs = tuple(G.A(c) for c in consts)
    R.barotr._barotr_rk2_core(st, cs, 1, dtb, 1, 1)  # warm-up
    t0 = time.perf_counter()
    ref = R.barotr._barotr_rk2_core(st, cs, a.substeps, dtb, 1, 1)
    t_ref = time.perf_counter() - t0
    O.rk2_core(state, consts, 1, dtb)
    t0 = time.perf_counter()
    port = O.rk2_core(state, consts, a.substeps, dtb)
    t_port = time.perf_counter() - t0
    same = all(np.array_equal(G.npy(ref[k]), port[k]) for k in (0, 2, 3))
    print(json.dumps({"n": a.n, "substeps": a.substeps, "cores": 1,
                      "reference_source_cell_updates_per_s": cells * a.substeps / t_ref,
                      "oracle_port_cell_updates_per_s": cells * a.substeps / t_port,
                      "port_over_reference": t_ref / t_port, "h_u_v_bitwise_equal": same}))


if __name__ == "__main__":
    main()
