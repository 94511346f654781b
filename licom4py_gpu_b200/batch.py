"""Batched rounds: many independent barotropic integrations per launch.

The reference advances one state per ``rk_core`` call (src/licom/mymodule/
schedule.py:170, src/licom/momentum/barotr.py:41-87).  An ensemble of such
integrations, or the requests of a server, would call it once per member and
round; on a B200 each small member then leaves most SMs idle and pays its own
launch latency.  :class:`BtBatch` advances a list of members -- any mix of
resolutions (one :class:`~licom4py_gpu_b200.plan.BtPlan` each), time steps and
substep counts -- in one persistent launch per round (``bt_batch_round``).
Members with fewer substeps retire early inside the launch.

:class:`MemberState` keeps one integration device-resident between rounds:
two state buffers used in turn (input / output) and the stage scratch.
"""

from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import torch

from . import _native as N
from .plan import cuda_device, DIAG_NAMES, BtPlan

_MODES = {"persistent": N.BT_MODE_PERSISTENT, "stream": N.BT_MODE_STREAM}


def member_scratch_bytes(plan: BtPlan, rk: int = 2) -> int:
    """Device scratch bytes one member of ``plan``'s resolution needs."""
    out = ctypes.c_ulonglong()
    N.check(N.lib().bt_member_scratch_bytes(plan._h, int(rk), ctypes.byref(out)))
    return int(out.value)


def member_bytes(plan: BtPlan, rk: int = 2) -> int:
    """Device bytes of one :class:`MemberState`: two (h, u, v) states and the scratch."""
    esize = 8 if plan.dtype == torch.float64 else 4
    return 6 * 6 * plan.m * plan.m * esize + member_scratch_bytes(plan, rk) + 256


class MemberState:
    """One integration held on the device between rounds.

    ``state`` is the current (h0, ub, vb) with valid halos; the RK base of the
    next round is the state itself (h0p = h0, ..., barotr.py:59).  ``remaining``
    counts the substeps still to run.
    """

    def __init__(self, plan: BtPlan, h0: torch.Tensor, ub: torch.Tensor, vb: torch.Tensor, nsub: int,
                 dtb: float, rk: int = 2, tag=None):
        for name, t in (("h0", h0), ("ub", ub), ("vb", vb)):
            plan._check_field(name, t)
        self.plan = plan
        self.rk = int(rk)
        self.dtb = float(dtb)
        self.remaining = int(nsub)
        self.nsub = int(nsub)
        self.tag = tag
        self.bufs = [(h0, ub, vb), tuple(plan.empty_field() for _ in range(3))]
        self.cur = 0
        nbytes = member_scratch_bytes(plan, rk)
        self.scratch = torch.empty(nbytes + 256, dtype=torch.uint8, device=plan.device)
        off = (-self.scratch.data_ptr()) % 256
        self._scratch_ptr = self.scratch.data_ptr() + off

    @property
    def state(self) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        return self.bufs[self.cur]

    def _member(self, nbb: int, diag: Optional[Sequence[torch.Tensor]] = None) -> N.Member:
        src, dst = self.bufs[self.cur], self.bufs[1 - self.cur]
        sin = N.StateIn(src[0].data_ptr(), src[0].data_ptr(), src[1].data_ptr(), src[2].data_ptr(),
                        src[1].data_ptr(), src[2].data_ptr())
        dptrs = [t.data_ptr() for t in diag] if diag is not None else [0] * 10
        sout = N.StateOut(dst[0].data_ptr(), dst[1].data_ptr(), dst[2].data_ptr(), (ctypes.c_void_p * 10)(*dptrs))
        return N.Member(self.plan._h, sin, sout, self._scratch_ptr, int(nbb), self.dtb)


class BtBatch:
    """Batched-round executor for one dtype on one device."""

    def __init__(self, dtype: torch.dtype = torch.float32, max_members: int = 256, device=None,
                 mode: str = "persistent", tile: Tuple[int, int] = (8, 32)):
        if not torch.cuda.is_available():
            raise RuntimeError("licom4py_gpu_b200 needs a CUDA device (there is no CPU path)")
        if dtype not in (torch.float64, torch.float32):
            raise ValueError("dtype must be torch.float64 or torch.float32")
        self.device = cuda_device(device)
        self.dtype = dtype
        self.max_members = int(max_members)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            N.check(N.lib().bt_batch_create(N.BT_F64 if dtype == torch.float64 else N.BT_F32, self.max_members,
                                            ctypes.byref(h)))
        self._h = h
        self.set_mode(mode)
        self.set_tile(*tile)

    def set_mode(self, mode: str) -> None:
        if mode not in _MODES:
            raise ValueError(f"mode must be one of {sorted(_MODES)}")
        N.check(N.lib().bt_batch_set_mode(self._h, _MODES[mode]))
        self.mode = mode

    def set_tile(self, ti: int, tj: int) -> None:
        N.check(N.lib().bt_batch_set_tile(self._h, int(ti), int(tj)))
        self.tile = (int(ti), int(tj))

    def set_max_ctas(self, n: int) -> None:
        N.check(N.lib().bt_batch_set_option(self._h, N.BT_OPT_MAX_CTAS, int(n)))

    def set_spin_limit(self, polls: int) -> None:
        N.check(N.lib().bt_batch_set_option(self._h, N.BT_OPT_SPIN_LIMIT, int(polls)))

    @property
    def last_grid(self) -> int:
        return int(N.lib().bt_batch_get_info(self._h, N.BT_INFO_LAST_GRID))

    def round_raw(self, members: Sequence[N.Member], rk: int = 2, stream: Optional[torch.cuda.Stream] = None) -> None:
        """Advance prepared ``Member`` records (the C structures) by their nbb substeps."""
        if not members:
            return
        arr = (N.Member * len(members))(*members)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            N.check(N.lib().bt_batch_round(self._h, arr, len(members), int(rk), ctypes.c_void_p(s.cuda_stream)))

    def advance(self, states: Sequence[MemberState], max_substeps: Optional[int] = None,
                diag: Optional[Sequence[Optional[Sequence[torch.Tensor]]]] = None,
                stream: Optional[torch.cuda.Stream] = None) -> List[MemberState]:
        """One round over the states that still have substeps: each runs
        min(remaining, max_substeps) substeps (all remaining when None).
        Returns the states advanced in this round."""
        live = [m for m in states if m.remaining > 0]
        if not live:
            return []
        rks = {m.rk for m in live}
        if len(rks) != 1:
            raise ValueError("all members of one round must use the same RK order")
        recs = []
        for k, m in enumerate(live):
            nbb = m.remaining if max_substeps is None else min(m.remaining, int(max_substeps))
            d = None if diag is None else diag[states.index(m)]
            recs.append(m._member(nbb, d))
        self.round_raw(recs, rk=rks.pop(), stream=stream)
        for m, r in zip(live, recs):
            m.remaining -= r.nbb
            m.cur = 1 - m.cur
        return live

    def check_device_error(self) -> None:
        N.check(N.lib().bt_batch_check_device_error(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().bt_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def diag_buffers(plan: BtPlan) -> List[torch.Tensor]:
    """Ten fields for a member's STATE_KEYS[6:16] outputs."""
    return [plan.empty_field() for _ in DIAG_NAMES]
