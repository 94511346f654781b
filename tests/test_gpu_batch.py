"""Batched rounds (bt_batch_round) against single-member rounds (bt_round).

A member's result must not depend on the batch it runs in: the batched launch
runs the same tile code with the same tile shape, so the float64 results are
asserted bit-identical to bt_round (itself bit-exact against the oracle), and
float32 results within 1e-6 relative of the float32 bt_round.
"""
import numpy as np
import pytest
import torch

from helpers import rel_err
from licom4py_gpu_b200._native import BtError
from licom4py_gpu_b200.batch import BtBatch, MemberState, diag_buffers
from licom4py_gpu_b200.duogrid import make_consts
from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state
from licom4py_gpu_b200.plan import DIAG_NAMES, BtPlan

pytestmark = pytest.mark.gpu

F32_TOL = 1e-6


def dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


@pytest.fixture(scope="module")
def plans(grids):
    cache = {}

    def get(n, dtype=torch.float64):
        if (n, dtype) not in cache:
            cache[(n, dtype)] = BtPlan(make_consts(grids(n), 5000.0), dtype=dtype)
        return cache[(n, dtype)]
    yield get
    for p in cache.values():
        p.close()


# (resolution, seed, substeps): uneven sizes and counts, two members sharing a plan
MIX = [(12, 1, 5), (12, 2, 2), (16, 3, 7), (24, 4, 3), (8, 5, 1)]


def make_members(grids, plans, dtype, rk=2, mix=MIX):
    out = []
    for n, seed, nsub in mix:
        g = grids(n)
        s = harmonic_state(g, seed, h_rms=0.2 + 0.3 * seed, uv_rms=0.1 * seed)
        p = plans(n, dtype)
        out.append(MemberState(p, dev(s["h0"], dtype), dev(s["ub"], dtype), dev(s["vb"], dtype), nsub,
                               cfl_dtb(g, 5000.0), rk=rk, tag=(n, seed)))
    return out


def single(m: MemberState, init, rk=2, diag=False):
    h, u, v = init
    return m.plan.round(h, h, u, v, u, v, nbb=m.nsub, dtb=m.dtb, rk=rk, diag=diag)


@pytest.mark.parametrize("mode", ["persistent", "stream"])
@pytest.mark.parametrize("tile", [(8, 32), (16, 16)])
def test_batch_f64_identical_to_single_rounds(mode, tile, grids, plans):
    mem = make_members(grids, plans, torch.float64)
    init = [tuple(t.clone() for t in m.state) for m in mem]
    b = BtBatch(torch.float64, max_members=8, mode=mode, tile=tile)
    b.advance(mem)
    b.check_device_error()
    for m, x0 in zip(mem, init):
        m.plan.set_tile(*tile)
        want = single(m, x0)
        for k, name in enumerate(("h0", "ub", "vb")):
            assert torch.equal(m.state[k], want[name]), f"member {m.tag}: {name} differs from bt_round"
        assert m.remaining == 0
    b.close()


@pytest.mark.parametrize("mode", ["persistent", "stream"])
def test_batch_rk3_and_diagnostics(mode, grids, plans):
    mix = [(12, 7, 3), (16, 8, 2), (12, 9, 1)]
    mem = make_members(grids, plans, torch.float64, rk=3, mix=mix)
    init = [tuple(t.clone() for t in m.state) for m in mem]
    diag = [diag_buffers(m.plan) if k != 1 else None for k, m in enumerate(mem)]
    b = BtBatch(torch.float64, max_members=4, mode=mode)
    b.advance(mem, diag=diag)
    for k, (m, x0) in enumerate(zip(mem, init)):
        m.plan.set_tile(8, 32)
        want = single(m, x0, rk=3, diag=True)
        for q, name in enumerate(("h0", "ub", "vb")):
            assert torch.equal(m.state[q], want[name]), f"member {m.tag}: {name}"
        if diag[k] is not None:
            for q, name in enumerate(DIAG_NAMES):
                assert torch.equal(diag[k][q], want[name]), f"member {m.tag}: diagnostic {name}"
    b.close()


def test_batch_rounds_in_pieces_equal_one_round(grids, plans):
    """Members kept on the device across rounds of at most 2 substeps (each
    round re-fills the halos) end where one round of all substeps ends."""
    a = make_members(grids, plans, torch.float64)
    c = make_members(grids, plans, torch.float64)
    b = BtBatch(torch.float64, max_members=8)
    b.advance(a)
    rounds = 0
    while b.advance(c, max_substeps=2):
        rounds += 1
    assert rounds == 4  # the longest member has 7 substeps
    for x, y in zip(a, c):
        for k in range(3):
            assert rel_err(y.state[k].cpu().numpy(), x.state[k].cpu().numpy()) <= 1e-12
    b.close()


@pytest.mark.parametrize("mode", ["persistent", "stream"])
def test_batch_f32_matches_single_rounds(mode, grids, plans):
    mem = make_members(grids, plans, torch.float32)
    init = [tuple(t.clone() for t in m.state) for m in mem]
    b = BtBatch(torch.float32, max_members=8, mode=mode)
    b.advance(mem)
    for m, x0 in zip(mem, init):
        m.plan.set_tile(8, 32)
        want = single(m, x0)
        for k, name in enumerate(("h0", "ub", "vb")):
            err = rel_err(m.state[k].cpu().numpy(), want[name].cpu().numpy())
            assert err <= F32_TOL, f"member {m.tag}: {name} rel err {err:.2e}"
    b.close()


def test_batch_rejects_bad_members(grids, plans):
    mem = make_members(grids, plans, torch.float64, mix=[(12, 1, 2), (16, 2, 2)])
    b = BtBatch(torch.float64, max_members=1)
    with pytest.raises(ValueError, match="count"):
        b.advance(mem)
    b.close()
    b = BtBatch(torch.float32, max_members=4)
    with pytest.raises(ValueError, match="dtype"):
        b.advance(mem)
    b.close()
    b = BtBatch(torch.float64, max_members=4)
    rec = mem[0]._member(0)
    with pytest.raises(ValueError, match="nbb"):
        b.round_raw([rec])
    rec = mem[0]._member(1)
    rec.out.h0 = rec.inp.h0
    with pytest.raises(ValueError, match="alias"):
        b.round_raw([rec])
    rec = mem[0]._member(1)
    rec.scratch = rec.scratch + 8
    with pytest.raises(ValueError, match="aligned"):
        b.round_raw([rec])
    with pytest.raises(ValueError, match="tile"):
        b.set_tile(5, 7)
    b.close()


def test_batch_barrier_timeout_is_reported_and_recoverable(grids, plans):
    """A grid-barrier wait given no polls gives up, flags the error and returns; no hang."""
    b = BtBatch(torch.float64, max_members=8)
    b.set_max_ctas(16)
    b.set_spin_limit(-1)
    seen = False
    for _ in range(5):
        b.advance(make_members(grids, plans, torch.float64))
        try:
            b.check_device_error()
        except BtError as e:
            assert "barrier" in str(e)
            seen = True
            break
    assert seen
    b.set_spin_limit(1 << 24)
    mem = make_members(grids, plans, torch.float64)
    init = [tuple(t.clone() for t in m.state) for m in mem]
    b.advance(mem)
    b.check_device_error()
    m = mem[2]
    m.plan.set_tile(8, 32)
    assert torch.equal(m.state[0], single(m, init[2])["h0"])
    b.close()
