"""Serving: a request loop over barotropic integrations with continuous batching.

A request is one integration the reference would run on its own
(``_barotr_rk2_core`` over ``nsub`` substeps from a seeded harmonic initial
state, src/licom/momentum/barotr.py:41-61), of any resolution.  The server
keeps every admitted request's state on the device and advances all of them
together, one batched launch (``bt_batch_round``) of up to ``round_substeps``
substeps per round.  Between rounds it

* retires the requests that finished (their result is copied to pinned host
  memory on a side stream; the request completes when that copy has landed),
* admits waiting requests in arrival order while the device-memory budget
  (``hbm_budget`` bytes of member state) and the member limit allow,

so requests that arrive while others are on the GPU join the next round and
their work overlaps on the device with the work already running.

:class:`Scheduler` is the host-side policy (no CUDA); :class:`BarotropicServer`
executes it on one GPU; :func:`run_fifo` is the one-request-at-a-time plain
path used for comparison.
"""

from __future__ import annotations

import heapq
import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Deque, Dict, List, Optional, Sequence, Tuple

import numpy as np

HALO = 3


@dataclass
class Request:
    rid: int
    n: int                  # cells per face edge
    nsub: int               # substeps
    seed: int               # harmonic initial state (h: seed, u/v: seed + 1, seed + 2)
    arrival: float = 0.0    # seconds after the start of the run
    amplitude: float = 1.0  # h RMS (m); u, v RMS = 0.3 * amplitude (m/s)
    t_admit: Optional[float] = None
    t_done: Optional[float] = None
    result: Optional[Dict[str, np.ndarray]] = None

    @property
    def latency(self) -> Optional[float]:
        return None if self.t_done is None else self.t_done - self.arrival

    @property
    def cell_updates(self) -> int:
        return 6 * self.n * self.n * self.nsub


def poisson_mix(count: int = 10_000, rate: float = 200.0, resolutions: Dict[int, float] = None,
                nsub: Tuple[int, int] = (100, 5000), seed: int = 0) -> List[Request]:
    """A Poisson arrival stream: exponential inter-arrival times of mean
    1 / rate, resolution drawn from ``resolutions`` {n: probability}
    (default C48 0.4, C96 0.35, C192 0.2, C384 0.05), substeps log-uniform in
    ``nsub`` (inclusive), a distinct harmonic seed per request."""
    res = resolutions if resolutions is not None else {48: 0.4, 96: 0.35, 192: 0.2, 384: 0.05}
    ns = np.array(sorted(res))
    p = np.array([res[n] for n in ns], dtype=np.float64)
    p = p / p.sum()
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    arrivals = np.cumsum(gaps) - gaps[0]
    which = rng.choice(len(ns), size=count, p=p)
    lo, hi = math.log(nsub[0]), math.log(nsub[1])
    steps = np.clip(np.rint(np.exp(rng.uniform(lo, hi, size=count))), nsub[0], nsub[1]).astype(int)
    return [Request(rid=k, n=int(ns[which[k]]), nsub=int(steps[k]), seed=1_000_003 * (seed + 1) + 7 * k,
                    arrival=float(arrivals[k])) for k in range(count)]


class Scheduler:
    """Admission and round planning, host only.

    ``member_bytes(n)`` gives the device bytes one request of resolution n
    holds while admitted.  Waiting requests are admitted while the budget and
    ``max_members`` allow, in the order ``order`` gives: "fifo" = arrival
    order with no overtaking (a large request is never starved), "shortest" =
    least work (cell-updates) first, arrival order among equals (lower median
    latency when the server is overloaded, at the cost of the largest
    requests).  A request larger than the whole budget is rejected.
    """

    def __init__(self, budget: int, member_bytes: Callable[[int], int], max_members: int = 1024,
                 round_substeps: int = 200, order: str = "fifo"):
        if order not in ("fifo", "shortest"):
            raise ValueError("order must be 'fifo' or 'shortest'")
        self.budget = int(budget)
        self.member_bytes = member_bytes
        self.max_members = int(max_members)
        self.round_substeps = int(round_substeps)
        self.order = order
        self.waiting: Deque[Request] = deque()
        self._heap: List[Tuple[int, float, int, Request]] = []
        self.active: Dict[int, Tuple[Request, int]] = {}  # rid -> (request, substeps left)
        self.used = 0
        self.peak = 0  # largest budget use seen
        self.rejected: List[Request] = []

    def arrive(self, req: Request) -> None:
        if self.member_bytes(req.n) > self.budget:
            self.rejected.append(req)
        elif self.order == "fifo":
            self.waiting.append(req)
        else:
            heapq.heappush(self._heap, (req.cell_updates, req.arrival, req.rid, req))

    def _next(self) -> Optional[Request]:
        if self.order == "fifo":
            return self.waiting[0] if self.waiting else None
        return self._heap[0][3] if self._heap else None

    def _pop(self) -> None:
        if self.order == "fifo":
            self.waiting.popleft()
        else:
            heapq.heappop(self._heap)

    @property
    def queued(self) -> int:
        return len(self.waiting) + len(self._heap)

    def admit(self) -> List[Request]:
        out = []
        while len(self.active) < self.max_members:
            req = self._next()
            if req is None:
                break
            need = self.member_bytes(req.n)
            if self.used + need > self.budget:
                break
            self._pop()
            self.used += need
            self.peak = max(self.peak, self.used)
            self.active[req.rid] = (req, req.nsub)
            out.append(req)
        return out

    def plan_round(self) -> Dict[int, int]:
        """Substeps each active request runs in the next round."""
        return {rid: min(left, self.round_substeps) for rid, (_, left) in self.active.items()}

    def finish_round(self, plan: Dict[int, int]) -> List[Request]:
        """Account a round; returns the requests it completed (their memory is released)."""
        done = []
        for rid, k in plan.items():
            req, left = self.active[rid]
            left -= k
            if left <= 0:
                del self.active[rid]
                self.used -= self.member_bytes(req.n)
                done.append(req)
            else:
                self.active[rid] = (req, left)
        return done

    @property
    def idle(self) -> bool:
        return self.queued == 0 and not self.active


def latency_stats(reqs: Sequence[Request]) -> Dict[str, float]:
    lat = np.array([r.latency for r in reqs if r.latency is not None], dtype=np.float64)
    if lat.size == 0:
        return {"p50_s": float("nan"), "p99_s": float("nan"), "mean_s": float("nan"), "max_s": float("nan")}
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
class HarmonicBasis:
    """Seeded harmonic initial states generated on the device.

    The 80 real spherical harmonics of degree 1..8 are evaluated once per
    resolution at every grid point (float64, on the device); a request's
    fields are then three matrix-vector products with its seeded N(0,1)
    coefficients, scaled to the target interior RMS and rotated to covariant
    components -- the construction of :func:`fields.harmonic_state`, with the
    sums taken in a different order (differences at float64 rounding level).
    """

    def __init__(self, geometry, device):
        import torch
        self.geo = geometry
        self.device = device
        self._basis: Dict[int, Tuple] = {}
        self.torch = torch

    def _get(self, n: int):
        torch = self.torch
        if n not in self._basis:
            from . import fields
            g = self.geo.grid(n)
            lon = g["a_pt"][..., 0]
            lat = g["a_pt"][..., 1]
            P = fields._legendre_all(8, np.sin(lat))
            rows = []
            for l in range(1, 9):
                for m in range(-l, l + 1):
                    am = abs(m)
                    if m == 0:
                        y = P[(l, 0)]
                    elif m > 0:
                        y = math.sqrt(2.0) * P[(l, am)] * np.cos(am * lon)
                    else:
                        y = math.sqrt(2.0) * P[(l, am)] * np.sin(am * lon)
                    rows.append(torch.from_numpy(np.ascontiguousarray(y).reshape(-1)).to(self.device))
            B = torch.stack(rows)  # (80, 6 M M)
            l2c = torch.from_numpy(np.ascontiguousarray(g["a_l2c"])).to(self.device)
            mask = torch.zeros((6, n + 6, n + 6), dtype=torch.bool, device=self.device)
            mask[:, HALO:-HALO, HALO:-HALO] = True
            self._basis[n] = (B, l2c, mask.reshape(-1))
        return self._basis[n]

    def state(self, req: Request, dtype):
        """(h0, ub, vb) device tensors of ``dtype`` for the request."""
        torch = self.torch
        B, l2c, mask = self._get(req.n)
        m = req.n + 6

        def series(seed):
            c = torch.from_numpy(np.random.default_rng(seed).standard_normal(B.shape[0])).to(self.device)
            return c @ B

        h = series(req.seed)
        h = h * (req.amplitude / torch.sqrt(torch.mean(h[mask] ** 2)))
        ul, vl = series(req.seed + 1), series(req.seed + 2)
        spd = torch.sqrt(torch.mean(ul[mask] ** 2 + vl[mask] ** 2) / 2.0)
        uv = 0.3 * req.amplitude
        ul, vl = (ul * (uv / spd)).reshape(6, m, m), (vl * (uv / spd)).reshape(6, m, m)
        ub = l2c[..., 0, 0] * ul + l2c[..., 0, 1] * vl
        vb = l2c[..., 1, 0] * ul + l2c[..., 1, 1] * vl
        return (h.reshape(6, m, m).to(dtype).contiguous(), ub.to(dtype).contiguous(), vb.to(dtype).contiguous())


class BarotropicServer:
    """Continuous-batching executor of :class:`Scheduler` on one GPU."""

    def __init__(self, geometry, dtype=None, rk: int = 2, round_substeps: int = 200,
                 hbm_budget: Optional[int] = None, max_members: int = 1024, mode: str = "stream",
                 tile: Tuple[int, int] = (16, 32), max_ctas: int = 0, keep_results: bool = True,
                 order: str = "fifo"):
        import torch
        from .batch import BtBatch, member_bytes
        self.torch = torch
        self.geo = geometry
        self.device = geometry.device
        self.dtype = dtype if dtype is not None else torch.float32
        self.rk = int(rk)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.5 * free)
        self._mbytes: Dict[int, int] = {}

        def mb(n: int) -> int:
            if n not in self._mbytes:
                self._mbytes[n] = member_bytes(self.geo.plan(n, self.dtype), self.rk)
            return self._mbytes[n]
        self.sched = Scheduler(hbm_budget, mb, max_members, round_substeps, order)
        self.batch = BtBatch(self.dtype, max_members=max_members, device=self.device, mode=mode, tile=tile)
        self.batch.set_max_ctas(max_ctas)
        self.basis = HarmonicBasis(geometry, self.device)
        self.keep_results = keep_results
        self.copy_stream = torch.cuda.Stream(self.device)
        self.states: Dict[int, object] = {}
        self.rounds = 0
        self.gpu_cell_updates = 0

    def _start(self, req: Request):
        from .batch import MemberState
        h, u, v = self.basis.state(req, self.dtype)
        st = MemberState(self.geo.plan(req.n, self.dtype), h, u, v, req.nsub, self.geo.dtb(req.n), rk=self.rk,
                         tag=req)
        self.states[req.rid] = st

    def run(self, requests: Sequence[Request], realtime: bool = True, clock=time.perf_counter) -> Dict[str, float]:
        """Serve ``requests`` (sorted by arrival).  With ``realtime`` a request
        becomes visible at its arrival time; otherwise all are visible at once.
        Returns throughput and latency figures."""
        torch = self.torch
        reqs = sorted(requests, key=lambda r: r.arrival)
        k = 0
        pending = []  # (request, member state, host tensors, event)
        t0 = clock()
        prev_round = None
        while k < len(reqs) or not self.sched.idle or pending:
            now = clock() - t0
            while k < len(reqs) and (not realtime or reqs[k].arrival <= now):
                self.sched.arrive(reqs[k])
                k += 1
            for req in self.sched.admit():
                req.t_admit = now
                self._start(req)
            plan = self.sched.plan_round()
            if plan:
                live = [self.states[rid] for rid in plan]
                self.batch.advance(live, max_substeps=self.sched.round_substeps)
                self.gpu_cell_updates += sum(6 * s.plan.n ** 2 * plan[s.tag.rid] for s in live)
                ev = torch.cuda.Event()
                ev.record()
                self.rounds += 1
                for req in self.sched.finish_round(plan):
                    st = self.states.pop(req.rid)
                    self.copy_stream.wait_event(ev)
                    with torch.cuda.stream(self.copy_stream):
                        host = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in st.state]
                        for hdst, src in zip(host, st.state):
                            hdst.copy_(src, non_blocking=True)
                        cev = torch.cuda.Event()
                        cev.record()
                    pending.append((req, st, host, cev))
                # keep the host at most one round ahead of the device
                if prev_round is not None:
                    prev_round.synchronize()
                prev_round = ev
            elif k < len(reqs) and realtime and not pending:
                time.sleep(max(0.0, min(reqs[k].arrival - (clock() - t0), 0.01)))
            still = []
            for item in pending:
                req, st, host, cev = item
                if cev.query():
                    req.t_done = clock() - t0
                    if self.keep_results:
                        req.result = {name: h.numpy() for name, h in zip(("h0", "ub", "vb"), host)}
                else:
                    still.append(item)
            pending = still
            if not plan and pending and (k >= len(reqs) or not realtime):
                pending[0][3].synchronize()
        wall = clock() - t0
        done = [r for r in reqs if r.t_done is not None]
        stats = latency_stats(done)
        work = sum(r.cell_updates for r in done)
        stats.update({"requests": len(done), "rejected": len(self.sched.rejected), "wall_s": wall,
                      "cell_updates": work, "cell_updates_per_s": work / wall if wall > 0 else float("nan"),
                      "rounds": self.rounds})
        return stats

    def close(self):
        self.batch.close()


def run_fifo(geometry, requests: Sequence[Request], dtype=None, configs: Optional[Dict[int, dict]] = None,
             realtime: bool = True, clock=time.perf_counter, keep_results: bool = True) -> Dict[str, float]:
    """The plain path: requests one at a time in arrival order, each a single
    ``bt_round`` of all its substeps on a plan of its resolution, the result
    copied back before the next starts.  ``configs[n]`` gives the plan's mode
    and tile (default stream mode, 8 x 32: every request has new buffers, so a
    captured graph would be captured again for each one)."""
    import torch
    from .duogrid import make_consts
    from .plan import BtPlan
    dtype = dtype if dtype is not None else torch.float32
    basis = HarmonicBasis(geometry, geometry.device)
    plans: Dict[int, BtPlan] = {}
    reqs = sorted(requests, key=lambda r: r.arrival)
    t0 = clock()
    for req in reqs:
        now = clock() - t0
        if realtime and req.arrival > now:
            time.sleep(req.arrival - now)
        if req.n not in plans:
            cfg = (configs or {}).get(req.n, {"mode": "stream", "tile": [8, 32]})
            plans[req.n] = BtPlan(make_consts(geometry.grid(req.n), geometry.depth), dtype=dtype,
                                  device=geometry.device, tile=tuple(cfg["tile"]), mode=cfg["mode"])
        p = plans[req.n]
        req.t_admit = clock() - t0
        h, u, v = basis.state(req, dtype)
        out = p.round(h, h, u, v, u, v, nbb=req.nsub, dtb=geometry.dtb(req.n), diag=False)
        res = {k: out[k].cpu().numpy() for k in ("h0", "ub", "vb")}
        req.t_done = clock() - t0
        if keep_results:
            req.result = res
    wall = clock() - t0
    for p in plans.values():
        p.close()
    stats = latency_stats(reqs)
    work = sum(r.cell_updates for r in reqs)
    stats.update({"requests": len(reqs), "wall_s": wall, "cell_updates": work,
                  "cell_updates_per_s": work / wall if wall > 0 else float("nan")})
    return stats
