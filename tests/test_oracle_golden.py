"""The float64 oracle against golden vectors produced by the reference's own source.

The fixtures in tests/golden were made by tests/golden/make_golden.py, which
runs the unmodified reference modules (barotr.py, barotr_pure.py, operators,
cube.py, communication.py) under a NumPy stand-in for jax.  The oracle must
reproduce them bit for bit.
"""
import numpy as np
import pytest

from conftest import load_golden
from helpers import STAGE_OUT, STATE_KEYS, golden_inputs, sha
from licom4py_gpu_b200.duogrid import make_consts
from oracle import barotr_np as O

CORE_FIXTURES = ["rk2_c8.npz", "rk2_c12_base.npz", "rk3_c8.npz", "rk2_c8_nbb0.npz", "rk2_c24.npz",
                 "rk2_c48_100.npz", "rk3_c48_30.npz", "rk2_c96_10.npz"]


@pytest.mark.parametrize("name", CORE_FIXTURES + ["stage_c8.npz"])
def test_generator_reproduces_fixture_consts(name, grids):
    z = load_golden(name)
    consts = make_consts(grids(int(z["n"])), float(z["depth"]))
    assert sha(consts) == str(z["consts_sha"])


@pytest.mark.parametrize("name", CORE_FIXTURES)
def test_core_bitexact(name, grids):
    z = load_golden(name)
    state, consts = golden_inputs(z, grids(int(z["n"])))
    assert sha(state) == str(z["inputs_sha"])
    core = O.rk2_core if int(z["rk"]) == 2 else O.rk3_core
    out = core(state, consts, int(z["nbb"]), float(z["dtb"]))
    checked = 0
    for k, key in enumerate(STATE_KEYS):
        if "out_" + key in z:
            np.testing.assert_array_equal(out[k], z["out_" + key], err_msg=key)
            checked += 1
    assert checked >= 3


@pytest.mark.parametrize("last", [False, True])
def test_stage_bitexact(last, grids):
    z = load_golden("stage_c8.npz")
    consts = make_consts(grids(8), float(z["depth"]))
    ins = [z["in_" + k] for k in STATE_KEYS[:6]]
    res = O.stage(*ins, consts, float(z["dtb"]) / 2.0, 0.0, last)
    tag = "last" if last else "mid"
    for name, a in zip(STAGE_OUT, res):
        np.testing.assert_array_equal(a, z[f"{tag}_{name}"], err_msg=name)


@pytest.mark.parametrize("n", [8, 12])
def test_halo_ops_bitexact(n, grids):
    z = load_golden("halo.npz")
    c = make_consts(grids(n), 5000.0)
    s, u, v = z[f"c{n}_s"], z[f"c{n}_u"], z[f"c{n}_v"]
    np.testing.assert_array_equal(O.copy_halo(s), z[f"c{n}_update_domain"])
    np.testing.assert_array_equal(O.fill_scalar(s, c[5], c[6], c[7]), z[f"c{n}_ext_scalar"])
    eu, ev = O.fill_vector(u, v, c[5], c[6], c[7], c[8], c[9], c[10], c[11])
    np.testing.assert_array_equal(eu, z[f"c{n}_ext_u"])
    np.testing.assert_array_equal(ev, z[f"c{n}_ext_v"])
    bu, bv = O.edge_average(u, v)
    np.testing.assert_array_equal(bu, z[f"c{n}_bc_u"])
    np.testing.assert_array_equal(bv, z[f"c{n}_bc_v"])


def test_routing_matches_reference():
    z = load_golden("halo.npz")
    routing = z["c8_routing"]  # Communication._routing[t, d] = (nb, dB, tid)
    for t in range(6):
        for d in range(4):
            nb, side, rev = O.face_neighbor(t, d)
            assert (nb, side, int(rev)) == tuple(int(x) for x in routing[t, d])


def test_oracle_detects_a_planted_mistake(grids):
    """The parity check has teeth: a perturbed viscosity constant changes the result."""
    z = load_golden("rk2_c8.npz")
    state, consts = golden_inputs(z, grids(8))
    orig = O.velocity_viscosity

    def bad(cx, cy, h, ucx, vcy):
        return orig(cx * 1.000001, cy, h, ucx, vcy)
    O.velocity_viscosity = bad
    try:
        out = O.rk2_core(state, consts, int(z["nbb"]), float(z["dtb"]))
    finally:
        O.velocity_viscosity = orig
    assert not np.array_equal(out[0], z["out_h0"])
