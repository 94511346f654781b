"""Generate the golden fixtures of the barotropic path from the reference's own source.

Runs the UNMODIFIED reference hot-path modules

    src/licom/kernel/communication.py   (Topology, routing, update_domain, boundary_communication)
    src/licom/kernel/cube.py            (cube_rmp, ext_scalar, ext_vector)
    src/licom/operators/{poly,agrid,remap}.py
    src/licom/momentum/barotr_pure.py   (_step_rk_logic and its stage functions)
    src/licom/momentum/barotr.py        (_barotr_rk2_core, _barotr_rk3_core)

on the CPU in float64 under the NumPy stand-in for `jax` in ``_jaxshim/``
(single device: pdev = px = py = 1, so every all_gather is a reshape), on
geometry constants from this package's duogrid generator and seeded
spherical-harmonic initial states.  JAX itself is not installed in this
environment, so the stand-in is what executes the reference code.

The reference tree is only present in the development container, so the
outputs are committed as ``tests/golden/*.npz``; the tests never import the
reference.  Each fixture records the SHA-256 of the float64 constants it was
made with so the tests can check that the generator still reproduces them.

Usage:  python tests/golden/make_golden.py --ref PATH_TO_REFERENCE [--only NAME.npz ...]
        (or set LICOM_REFERENCE_ROOT to the reference checkout)
"""

from __future__ import annotations

import argparse
import hashlib
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(HERE, "_jaxshim"))
sys.path.insert(0, REPO)

import jax  # noqa: E402  (the stand-in)
import jax.numpy as jnp  # noqa: E402

from licom4py_gpu_b200 import duogrid_gen  # noqa: E402
from licom4py_gpu_b200.duogrid import make_consts  # noqa: E402
from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state  # noqa: E402

STATE_KEYS = ("h0", "h0p", "ub", "vb", "ubp", "vbp", "celerity_x", "celerity_y", "ub_ct",
              "vb_ct", "ub_cx", "ub_cy", "vb_cx", "vb_cy", "advx", "advy",
              "pax", "pxb", "whx", "pay", "pyb", "why", "wgp")
CONST_KEYS = ("dzph_x", "dzph_y", "rdx", "rdy", "a_f", "k2e_coef", "loc_i_local", "loc_j_local",
              "a_c2l", "a_l2c", "inner", "outer", "a_gct", "a_sina", "rda", "c_dy", "d_dx")
STAGE_OUT = ("new_h0", "new_ub", "new_vb", "celerity_x", "celerity_y", "ub_ct", "vb_ct",
             "ub_cx", "ub_cy", "vb_cx", "vb_cy", "advx", "advy")


def _pkg(name):
    m = types.ModuleType(name)
    m.__path__ = []
    sys.modules[name] = m
    return m


def _load(modname, path):
    spec = importlib.util.spec_from_file_location(modname, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[modname] = mod
    spec.loader.exec_module(mod)
    return mod


def load_reference(ref_root, n):
    """Import the reference hot-path modules under a minimal `licom` package."""
    src = os.path.join(ref_root, "src", "licom")
    _pkg("licom")
    kernel = _pkg("licom.kernel")
    ops = _pkg("licom.operators")
    mom = _pkg("licom.momentum")
    comm = _load("licom.kernel.communication", os.path.join(src, "kernel", "communication.py"))
    kernel.Communication = comm.Communication
    cube = _load("licom.kernel.cube", os.path.join(src, "kernel", "cube.py"))
    kernel.cube = cube
    poly = _load("licom.operators.poly", os.path.join(src, "operators", "poly.py"))
    agrid = _load("licom.operators.agrid", os.path.join(src, "operators", "agrid.py"))
    remap = _load("licom.operators.remap", os.path.join(src, "operators", "remap.py"))
    ops.Poly, ops.AGrid, ops.Remap = poly.Poly, agrid.AGrid, remap.Remap
    pure = _load("licom.momentum.barotr_pure", os.path.join(src, "momentum", "barotr_pure.py"))
    barotr = _load("licom.momentum.barotr", os.path.join(src, "momentum", "barotr.py"))
    mom.barotr_pure, mom.barotr = pure, barotr
    # Communication.configure(halo, nx_local, ny_local, mesh) (communication.py:269-291)
    comm.Communication.configure(3, n, n, jax.sharding.Mesh())
    return types.SimpleNamespace(comm=comm, cube=cube, pure=pure, barotr=barotr)


def A(x):
    return jnp.array(np.asarray(x))


def npy(x):
    return np.asarray(x).view(np.ndarray).copy()


def consts_sha(consts) -> str:
    h = hashlib.sha256()
    for c in consts:
        h.update(np.ascontiguousarray(c).tobytes())
    return h.hexdigest()


def build_case(n, depth, seed, base_seed=None):
    grid = duogrid_gen.generate(n)
    consts = make_consts(grid, depth)
    st = harmonic_state(grid, seed)
    if base_seed is None:
        base = st
    else:
        base = harmonic_state(grid, base_seed, h_rms=0.5, uv_rms=0.1)
    M = n + 6
    zeros = np.zeros((6, M, M))
    state = [st["h0"], base["h0"], st["ub"], st["vb"], base["ub"], base["vb"]] + \
        [zeros.copy() for _ in range(10)] + [zeros.copy() for _ in range(7)]
    dtb = cfl_dtb(grid, depth)
    return grid, consts, state, dtb


def save(path, **arrays):
    np.savez_compressed(path, **arrays)
    print(f"wrote {os.path.relpath(path, REPO)} ({os.path.getsize(path) / 1024:.0f} KiB)")


def gen_stage(ref_root, out):
    """One _step_rk_logic call (barotr_pure.py:100-168), mid and last stage, C8."""
    n, depth = 8, 5000.0
    R = load_reference(ref_root, n)
    grid, consts, state, dtb = build_case(n, depth, seed=11, base_seed=21)
    C = tuple(A(c) for c in consts) + tuple(A(np.zeros_like(consts[0])) for _ in range(7))
    arrays = {"n": n, "depth": depth, "dtb": dtb, "consts_sha": consts_sha(consts)}
    for k in range(6):
        arrays[f"in_{STATE_KEYS[k]}"] = state[k]
    for last in (False, True):
        res = R.pure._step_rk_logic(A(state[0]), A(state[1]), A(state[2]), A(state[3]),
                                    A(state[4]), A(state[5]), C, dtb / 2.0, 0.0, last, 1, 1)
        tag = "last" if last else "mid"
        for name, r in zip(STAGE_OUT, res):
            arrays[f"{tag}_{name}"] = npy(r)
    save(os.path.join(out, "stage_c8.npz"), **arrays)


def gen_halo(ref_root, out):
    """ext_scalar / ext_vector / boundary_communication on random fields, C8 and C12."""
    arrays = {}
    for n in (8, 12):
        R = load_reference(ref_root, n)
        grid = duogrid_gen.generate(n)
        consts = make_consts(grid, 5000.0)
        rng = np.random.default_rng(100 + n)
        M = n + 6
        s = rng.standard_normal((6, M, M))
        u = rng.standard_normal((6, M, M))
        v = rng.standard_normal((6, M, M))
        coef, li, lj, c2l, l2c, inner, outer = (A(consts[5]), A(consts[6]), A(consts[7]),
                                                A(consts[8]), A(consts[9]), A(consts[10]),
                                                A(consts[11]))
        es = R.cube.ext_scalar(A(s), coef, li, lj, 1, 1)
        eu, ev = R.cube.ext_vector(A(u), A(v), coef, li, lj, c2l, l2c, inner, outer, 1, 1)
        bu, bv = R.comm.Communication.boundary_communication(A(u), A(v))
        ud = R.comm.Communication.update_domain(A(s))
        arrays.update({f"c{n}_s": s, f"c{n}_u": u, f"c{n}_v": v,
                       f"c{n}_ext_scalar": npy(es), f"c{n}_ext_u": npy(eu), f"c{n}_ext_v": npy(ev),
                       f"c{n}_bc_u": npy(bu), f"c{n}_bc_v": npy(bv), f"c{n}_update_domain": npy(ud),
                       f"c{n}_routing": npy(R.comm.Communication._routing),
                       f"c{n}_consts_sha": consts_sha(consts)})
    save(os.path.join(out, "halo.npz"), **arrays)


def gen_core(ref_root, out, name, n, nbb, seed, rk=2, base_seed=None, keep_inputs=True,
             outputs=STATE_KEYS, depth=5000.0):
    R = load_reference(ref_root, n)
    grid, consts, state, dtb = build_case(n, depth, seed, base_seed)
    core = R.barotr._barotr_rk2_core if rk == 2 else R.barotr._barotr_rk3_core
    res = core(tuple(A(s) for s in state), tuple(A(c) for c in consts), nbb, dtb, 1, 1)
    arrays = {"n": n, "nbb": nbb, "dtb": dtb, "rk": rk, "seed": seed, "depth": depth,
              "base_seed": -1 if base_seed is None else base_seed,
              "consts_sha": consts_sha(consts), "inputs_sha": consts_sha(state)}
    if keep_inputs:
        for k in range(6):
            arrays[f"in_{STATE_KEYS[k]}"] = state[k]
    for k, key in enumerate(STATE_KEYS):
        if key in outputs:
            arrays[f"out_{key}"] = npy(res[k])
    save(os.path.join(out, name), **arrays)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--ref", default=os.environ.get("LICOM_REFERENCE_ROOT"),
                   help="root of the reference checkout (default: $LICOM_REFERENCE_ROOT)")
    p.add_argument("--out", default=HERE)
    p.add_argument("--only", nargs="*", default=None,
                   help="fixture file names to (re)generate; default: all of them")
    a = p.parse_args()
    if not a.ref:
        p.error("give --ref PATH_TO_REFERENCE or set LICOM_REFERENCE_ROOT")
    jobs = {
        "halo.npz": lambda: gen_halo(a.ref, a.out),
        "stage_c8.npz": lambda: gen_stage(a.ref, a.out),
        "rk2_c8.npz": lambda: gen_core(a.ref, a.out, "rk2_c8.npz", n=8, nbb=4, seed=1),
        "rk2_c12_base.npz": lambda: gen_core(a.ref, a.out, "rk2_c12_base.npz", n=12, nbb=3, seed=2, base_seed=3),
        "rk3_c8.npz": lambda: gen_core(a.ref, a.out, "rk3_c8.npz", n=8, nbb=3, seed=4, rk=3),
        "rk2_c8_nbb0.npz": lambda: gen_core(a.ref, a.out, "rk2_c8_nbb0.npz", n=8, nbb=0, seed=5),
        "rk2_c24.npz": lambda: gen_core(a.ref, a.out, "rk2_c24.npz", n=24, nbb=10, seed=6, keep_inputs=False,
                                        outputs=STATE_KEYS[:16]),
        "rk2_c48_100.npz": lambda: gen_core(a.ref, a.out, "rk2_c48_100.npz", n=48, nbb=100, seed=7,
                                            keep_inputs=False, outputs=("h0", "ub", "vb")),
        # the headline resolution (C96), RK2
        "rk2_c96_10.npz": lambda: gen_core(a.ref, a.out, "rk2_c96_10.npz", n=96, nbb=10, seed=9,
                                           keep_inputs=False, outputs=("h0", "ub", "vb")),
        # RK3 where tiles of the 8 x 16 and 16 x 16 shapes are full interior tiles
        "rk3_c48_30.npz": lambda: gen_core(a.ref, a.out, "rk3_c48_30.npz", n=48, nbb=30, seed=8, rk=3,
                                           keep_inputs=False, outputs=("h0", "ub", "vb")),
    }
    for name in (a.only if a.only else jobs):
        if name not in jobs:
            p.error(f"unknown fixture {name}; known: {', '.join(jobs)}")
        jobs[name]()


if __name__ == "__main__":
    main()
