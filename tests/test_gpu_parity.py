"""GPU parity: the CUDA solver through the C-ABI against the golden vectors and the oracle.

Tolerances: the float64 path is compiled without FMA contraction and keeps the
reference's operand order, so it is expected to be bit-exact; the stated
bound, asserted here, is 1e-12 relative (max-norm) against the float64
oracle.  The float32 precision form is checked against float64 at 1e-5
relative h error after 100 substeps (C48).
"""
import numpy as np
import pytest
import torch

from conftest import load_golden
from helpers import STAGE_OUT, STATE_KEYS, golden_inputs, rel_err
from licom4py_gpu_b200 import barotr, barotr_pure
from licom4py_gpu_b200.duogrid import make_consts
from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state
from licom4py_gpu_b200 import _native as N
from licom4py_gpu_b200.plan import DIAG_NAMES, BtPlan
from oracle import barotr_np as O

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def host(t):
    return t.detach().cpu().numpy()


def assert_f64_close(got, want, what):
    got = host(got) if isinstance(got, torch.Tensor) else got
    err = rel_err(got, want)
    assert err <= F64_TOL, f"{what}: rel err {err:.3e} > {F64_TOL}"


@pytest.fixture(scope="module")
def plans(grids):
    cache = {}

    def get(n, depth=5000.0, dtype=torch.float64):
        key = (n, depth, dtype)
        if key not in cache:
            cache[key] = BtPlan(make_consts(grids(n), depth), dtype=dtype)
        return cache[key]
    yield get
    for p in cache.values():
        p.close()


@pytest.mark.parametrize("n", [8, 12])
def test_fill_halo_matches_reference(n, plans):
    z = load_golden("halo.npz")
    p = plans(n)
    s = dev(z[f"c{n}_s"])
    u, v = dev(z[f"c{n}_u"]), dev(z[f"c{n}_v"])
    p.fill_halo(h=s, u=u, v=v)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(s), z[f"c{n}_ext_scalar"])
    np.testing.assert_array_equal(host(u), z[f"c{n}_ext_u"])
    np.testing.assert_array_equal(host(v), z[f"c{n}_ext_v"])


@pytest.mark.parametrize("n", [8, 12])
def test_edge_average_matches_reference(n, plans):
    z = load_golden("halo.npz")
    p = plans(n)
    u, v = dev(z[f"c{n}_u"]), dev(z[f"c{n}_v"])
    p.edge_average(u, v)
    np.testing.assert_array_equal(host(u), z[f"c{n}_bc_u"])
    np.testing.assert_array_equal(host(v), z[f"c{n}_bc_v"])


@pytest.mark.parametrize("last", [False, True])
def test_stage_matches_reference(last, grids):
    z = load_golden("stage_c8.npz")
    consts = make_consts(grids(8), float(z["depth"]))
    ins = [dev(z["in_" + k]) for k in STATE_KEYS[:6]]
    res = barotr_pure._step_rk_logic(*ins, consts, float(z["dtb"]) / 2.0, 0.0, last, 1, 1)
    assert len(res) == 13
    tag = "last" if last else "mid"
    for name, a in zip(STAGE_OUT, res):
        assert_f64_close(a, z[f"{tag}_{name}"], f"{tag} {name}")


CORES = ["rk2_c8.npz", "rk2_c12_base.npz", "rk3_c8.npz", "rk2_c24.npz", "rk2_c48_100.npz", "rk3_c48_30.npz",
         "rk2_c96_10.npz"]


@pytest.mark.parametrize("name", CORES)
def test_core_matches_reference(name, grids):
    z = load_golden(name)
    state, consts = golden_inputs(z, grids(int(z["n"])))
    st = tuple(dev(s) for s in state)
    core = barotr._barotr_rk2_core if int(z["rk"]) == 2 else barotr._barotr_rk3_core
    out = core(st, consts, int(z["nbb"]), float(z["dtb"]), 1, 1)
    assert len(out) == 23
    checked = 0
    for k, key in enumerate(STATE_KEYS[:16]):
        if "out_" + key in z:
            assert_f64_close(out[k], z["out_" + key], f"{name}:{key}")
            checked += 1
    assert checked >= 3


def test_core_bitexact_against_oracle_c96(grids):
    g = grids(96)
    consts = make_consts(g, 5000.0)
    st = harmonic_state(g, 3)
    m = 102
    state = [st["h0"], st["h0"], st["ub"], st["vb"], st["ub"], st["vb"]] + [np.zeros((6, m, m))] * 17
    dtb = cfl_dtb(g, 5000.0)
    want = O.rk2_core(state, consts, 4, dtb)
    got = barotr._barotr_rk2_core(tuple(dev(s) for s in state), consts, 4, dtb, 1, 1)
    for k in range(16):
        assert_f64_close(got[k], want[k], STATE_KEYS[k])
    exact = sum(int(np.array_equal(host(got[k]), want[k])) for k in range(16))
    assert exact >= 3  # h0/ub/vb at least are expected to match bit for bit


def test_dropin_semantics(grids):
    z = load_golden("rk2_c8.npz")
    state, consts = golden_inputs(z, grids(8))
    st = tuple(dev(s) for s in state)
    out = barotr._barotr_rk2_core(st, consts, 2, float(z["dtb"]), 1, 1)
    assert out[0] is out[1] and out[2] is out[4] and out[3] is out[5]
    for k in range(16, 23):
        assert out[k] is st[k]  # coupling fields pass through as the same objects
    same = barotr._barotr_rk2_core(st, consts, 0, float(z["dtb"]), 1, 1)
    assert all(a is b for a, b in zip(same, st))
    with pytest.raises(ValueError):
        barotr._barotr_rk2_core(st, consts, 1, 1.0, 2, 1)
    with pytest.raises(ValueError):
        barotr._barotr_rk2_core(st[:20], consts, 1, 1.0, 1, 1)
    # inputs are not modified
    np.testing.assert_array_equal(host(st[0]), state[0])


def test_graph_mode_bitwise_equals_stream_mode(grids):
    g = grids(24)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 9)
    ins = [dev(s["h0"]), dev(s["h0"]), dev(s["ub"]), dev(s["vb"]), dev(s["ub"]), dev(s["vb"])]
    dtb = cfl_dtb(g, 5000.0)
    p = BtPlan(consts)
    a = p.round(*ins, nbb=5, dtb=dtb)
    p.set_mode("graph")
    b = p.round(*ins, nbb=5, dtb=dtb)
    c = p.round(*ins, nbb=5, dtb=dtb)  # replay of the cached graph
    torch.cuda.synchronize()
    for k in a:
        assert torch.equal(a[k], b[k]) and torch.equal(a[k], c[k]), k
    p.close()


@pytest.mark.parametrize("tile", [(7, 32), (8, 32), (15, 32), (16, 32), (8, 16), (16, 16)])
def test_tile_shapes_bitwise_identical(tile, grids):
    g = grids(48)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 4)
    ins = [dev(s["h0"]), dev(s["h0"]), dev(s["ub"]), dev(s["vb"]), dev(s["ub"]), dev(s["vb"])]
    dtb = cfl_dtb(g, 5000.0)
    ref = BtPlan(consts, tile=(8, 32)).round(*ins, nbb=3, dtb=dtb)
    got = BtPlan(consts, tile=tile).round(*ins, nbb=3, dtb=dtb)
    for k in ref:
        assert torch.equal(ref[k], got[k]), (tile, k)


@pytest.mark.parametrize("n,tile", [(10, (8, 32)), (17, (8, 16)), (18, (16, 16)), (34, (15, 32))])
def test_thin_last_tile_bitexact_against_oracle(n, tile, grids):
    """N with a last tile 1 or 2 cells thin: the previous tile's stencil region
    reaches the face halo without the tile touching that edge."""
    g = grids(n)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 31)
    m = n + 6
    state = [s["h0"], s["h0"], s["ub"], s["vb"], s["ub"], s["vb"]] + [np.zeros((6, m, m))] * 17
    dtb = cfl_dtb(g, 5000.0)
    want = O.rk2_core(state, consts, 3, dtb)
    p = BtPlan(consts, tile=tile)
    got = p.round(*[dev(x) for x in state[:6]], nbb=3, dtb=dtb)
    for k, name in ((0, "h0"), (2, "ub"), (3, "vb")):
        assert_f64_close(got[name], want[k], f"C{n} {tile} {name}")
    for k, name in enumerate(DIAG_NAMES):
        assert_f64_close(got[name], want[6 + k], f"C{n} {tile} {name}")
    p.close()


def test_float32_precision_form_c48(grids):
    """FP32 state/consts vs the float64 reference run (config-1 case, 100 substeps)."""
    z = load_golden("rk2_c48_100.npz")
    state, consts = golden_inputs(z, grids(48))
    st = tuple(dev(s, torch.float32) for s in state)
    out = barotr._barotr_rk2_core(st, tuple(np.asarray(c) for c in consts), 100, float(z["dtb"]), 1, 1)
    for k, key in ((0, "h0"), (2, "ub"), (3, "vb")):
        got = host(out[k]).astype(np.float64)[:, 3:-3, 3:-3]
        want = z["out_" + key][:, 3:-3, 3:-3]
        l2 = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert l2 <= 1e-5, f"{key}: relative L2 error {l2:.2e}"


def test_mass_conserved_c384(grids):
    """Size-independent property at full size: the averaged edge fluxes conserve sum(h * area)."""
    g = grids(384)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 8)
    da = torch.from_numpy(1.0 / g["rda"][:, 3:-3, 3:-3]).cuda()
    ins = [dev(s["h0"]), dev(s["h0"]), dev(s["ub"]), dev(s["vb"]), dev(s["ub"]), dev(s["vb"])]
    p = BtPlan(consts)
    out = p.round(*ins, nbb=20, dtb=cfl_dtb(g, 5000.0), diag=False)
    m0 = (ins[0][:, 3:-3, 3:-3] * da).sum().item()
    m1 = (out["h0"][:, 3:-3, 3:-3] * da).sum().item()
    scale = (ins[0][:, 3:-3, 3:-3].abs() * da).sum().item()
    assert abs(m1 - m0) <= 1e-12 * scale
    assert torch.isfinite(out["h0"]).all()
    p.close()


@pytest.mark.parametrize("rk", [2, 3])
def test_persistent_mode_bitwise_equals_stream_mode(rk, grids):
    g = grids(24)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 10)
    b = harmonic_state(g, 11, 0.5, 0.1)
    ins = [dev(s["h0"]), dev(b["h0"]), dev(s["ub"]), dev(s["vb"]), dev(b["ub"]), dev(b["vb"])]
    dtb = cfl_dtb(g, 5000.0)
    p = BtPlan(consts)
    a = p.round(*ins, nbb=6, dtb=dtb, rk=rk)
    p.set_mode("persistent")
    for ctas in (0, 7):  # occupancy-sized grid, and a small grid looping over many tiles
        p.set_max_ctas(ctas)
        c = p.round(*ins, nbb=6, dtb=dtb, rk=rk)
        p.check_device_error()
        assert p.last_grid >= 1
        for k in a:
            assert torch.equal(a[k], c[k]), (ctas, k)
    p.close()


def test_persistent_barrier_timeout_is_reported_and_recoverable(grids):
    """A grid-barrier wait given no polls gives up, flags the error and returns; no hang."""
    from licom4py_gpu_b200._native import BtError
    g = grids(24)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 12)
    ins = [dev(s["h0"]), dev(s["h0"]), dev(s["ub"]), dev(s["vb"]), dev(s["ub"]), dev(s["vb"])]
    dtb = cfl_dtb(g, 5000.0)
    p = BtPlan(consts, mode="persistent")
    p.set_max_ctas(16)
    p.set_spin_limit(-1)
    seen = False
    for _ in range(5):
        p.round(*ins, nbb=3, dtb=dtb)
        try:
            p.check_device_error()
        except BtError as e:
            assert "barrier" in str(e)
            seen = True
            break
    assert seen
    # the context stays usable: a normal round afterwards matches stream mode
    p.set_spin_limit(1 << 24)
    got = p.round(*ins, nbb=3, dtb=dtb)
    p.check_device_error()
    ref = BtPlan(consts).round(*ins, nbb=3, dtb=dtb)
    assert torch.equal(got["h0"], ref["h0"])
    p.close()


def test_misaligned_constant_views_give_the_same_round(grids):
    """Constant tensors that are views 8 bytes off a 16-byte boundary (the 2x2
    matrices are read with 16-byte loads) are copied aligned by the plan."""
    g = grids(24)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 5)
    ins = [dev(s["h0"]), dev(s["h0"]), dev(s["ub"]), dev(s["vb"]), dev(s["ub"]), dev(s["vb"])]
    dtb = cfl_dtb(g, 5000.0)
    ref_plan = BtPlan(consts)
    ref = ref_plan.round(*ins, nbb=3, dtb=dtb)
    shifted = []
    for c in consts:
        t = torch.from_numpy(np.ascontiguousarray(c)).cuda()
        buf = torch.empty(t.numel() + 1, dtype=t.dtype, device="cuda")
        view = buf[1:].view(t.shape)
        view.copy_(t)
        shifted.append(view)
    assert all(t.data_ptr() % 16 for t in shifted)
    p = BtPlan(shifted)
    assert all(t.data_ptr() % 16 == 0 for t in p.consts.values())
    got = p.round(*ins, nbb=3, dtb=dtb)
    torch.cuda.synchronize()
    for k in ref:
        assert torch.equal(ref[k], got[k]), k
    p.close()
    ref_plan.close()


# Tiles of 32 columns have full interior tiles (the whole stencil region inside
# the face, compiled without the edge logic) only from C96 on; these cases run
# every full-tile instantiation next to edge tiles.  A C96 launch is one wave,
# where the plan would pick the edge-path-only kernels, so the full-tile kernels
# are forced here and compared with the edge-path-only kernels of the 8 x 16 tile.
@pytest.mark.parametrize("tile", [(7, 32), (8, 32), (15, 32), (16, 32), (8, 16), (16, 16)])
def test_full_tile_shapes_bitwise_identical_c96(tile, grids):
    g = grids(96)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 12)
    ins = [dev(s["h0"]), dev(s["h0"]), dev(s["ub"]), dev(s["vb"]), dev(s["ub"]), dev(s["vb"])]
    dtb = cfl_dtb(g, 5000.0)
    ref_plan, plan = BtPlan(consts, tile=(8, 16)), BtPlan(consts, tile=tile)
    ref_plan.set_full_tiles(False)
    plan.set_full_tiles(True)
    for rk in (2, 3):
        ref = ref_plan.round(*ins, nbb=3, dtb=dtb, rk=rk)
        got = plan.round(*ins, nbb=3, dtb=dtb, rk=rk)
        for k in ref:
            assert torch.equal(ref[k], got[k]), (tile, rk, k)
    ref_plan.close()
    plan.close()


@pytest.mark.parametrize("tile", [(7, 32), (8, 32), (15, 32), (16, 32), (8, 16), (16, 16)])
def test_float32_full_tiles_c96(tile, grids):
    """Float32 rounds at C96 (full interior tiles of every shape) against the float64 path: 1e-5
    relative L2 on h, u, v after 100 substeps."""
    g = grids(96)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 13)
    dtb = cfl_dtb(g, 5000.0)
    keys = ("h0", "h0", "ub", "vb", "ub", "vb")
    p64 = BtPlan(consts, tile=(8, 16))
    want = p64.round(*[dev(s[k]) for k in keys], nbb=100, dtb=dtb, diag=False)
    p32 = BtPlan(consts, dtype=torch.float32, tile=tile)
    for full in (True, False):  # the full-tile kernels, then the edge-path-only kernels
        p32.set_full_tiles(full)
        got = p32.round(*[dev(s[k], torch.float32) for k in keys], nbb=100, dtb=dtb, diag=False)
        for key in ("h0", "ub", "vb"):
            a = got[key][:, 3:-3, 3:-3].double()
            b = want[key][:, 3:-3, 3:-3]
            l2 = ((a - b).norm() / b.norm()).item()
            assert l2 <= 1e-5, f"{tile} full={full} {key}: relative L2 error {l2:.2e}"
    p64.close()
    p32.close()


@pytest.mark.parametrize("full", [True, False])
@pytest.mark.parametrize("name,tile", [("rk3_c48_30.npz", (8, 16)), ("rk3_c48_30.npz", (16, 16)),
                                       ("rk2_c96_10.npz", (8, 16)), ("rk2_c96_10.npz", (16, 32))])
def test_both_kernel_builds_match_reference(name, tile, full, grids):
    """RK3 at C48 and RK2 at C96 (the headline resolution), both with full interior tiles at these
    shapes, against the reference's own runs, through the full-tile kernels and through the
    edge-path-only kernels."""
    z = load_golden(name)
    state, consts = golden_inputs(z, grids(int(z["n"])))
    plan = BtPlan(consts, tile=tile, mode="graph")
    plan.set_full_tiles(full)
    six = [dev(s) for s in state[:6]]
    out = plan.round(*six, nbb=int(z["nbb"]), dtb=float(z["dtb"]), rk=int(z["rk"]), diag=False)
    for key in ("h0", "ub", "vb"):
        assert_f64_close(out[key], z["out_" + key], f"{name} {tile} full={full}:{key}")
    plan.close()


@pytest.mark.parametrize("n,tile", [(48, (8, 16)), (96, (8, 16)), (192, (8, 32)), (384, (16, 32))])
def test_full_tile_choice_gives_the_same_round(n, tile, grids):
    """The kernel chosen by size, the full-tile kernels and the edge-path-only kernels give
    bit-identical float64 rounds (graph mode, RK2 and RK3)."""
    g = grids(n)
    consts = make_consts(g, 5000.0)
    s = harmonic_state(g, 21)
    ins = [dev(s["h0"]), dev(s["h0"]), dev(s["ub"]), dev(s["vb"]), dev(s["ub"]), dev(s["vb"])]
    dtb = cfl_dtb(g, 5000.0)
    plan = BtPlan(consts, tile=tile, mode="graph")
    plan.set_full_tiles(True)
    assert plan.full_tile_kernels == (True, True)
    plan.set_full_tiles(False)
    assert plan.full_tile_kernels == (False, False)
    for bad in (-2, 2):
        with pytest.raises(ValueError):
            plan.set_option(N.BT_OPT_FULL_TILES, bad)
    for rk in (2, 3):
        outs = []
        for full in (None, True, False):
            plan.set_full_tiles(full)
            outs.append(plan.round(*ins, nbb=2, dtb=dtb, rk=rk, diag=False))
        for got in outs[1:]:
            for k in outs[0]:
                assert torch.equal(outs[0][k], got[k]), (n, tile, rk, k)
    plan.close()
