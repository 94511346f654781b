"""Uneven ensembles: many independent barotropic integrations of mixed
resolution and length, advanced together by batched rounds.

An ensemble member is one integration the reference would run on its own
(``_barotr_rk2_core`` over ``nsub`` substeps, src/licom/momentum/barotr.py:41-61)
from a seeded harmonic initial state.  :func:`uneven_mix` draws the members of
a mix (resolution counts, perturbation amplitudes, substep counts);
:class:`Ensemble` holds their geometry (one plan per resolution), initial
states and time steps, and runs them either batched (all members in one
persistent launch per round, members retiring as their substeps run out) or
one integration at a time through the drop-in path, for comparison.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import duogrid_gen
from .batch import BtBatch, MemberState
from .duogrid import make_consts
from .fields import cfl_dtb, harmonic_state
from .plan import cuda_device, BtPlan

UV_PER_H = 0.3  # u, v RMS (m/s) per metre of h RMS: the 1 m / 0.3 m/s pairing of the seeded fields


@dataclass(frozen=True)
class MemberSpec:
    n: int            # cells per face edge
    seed: int         # harmonic field seed (h: seed, u/v: seed + 1, seed + 2)
    amplitude: float  # h perturbation RMS in metres; u, v RMS = UV_PER_H * amplitude
    nsub: int         # substeps of the integration


def uneven_mix(counts: Dict[int, int] = None, nsub: Tuple[int, int] = (200, 2000),
               amplitude: Tuple[float, float] = (0.2, 2.0), seed: int = 0) -> List[MemberSpec]:
    """Members of an uneven ensemble: ``counts[n]`` members at resolution n
    (default 32 x C48, 24 x C96, 8 x C192), each with its own seed, an h
    amplitude drawn U[amplitude] and a substep count drawn U{nsub} inclusive."""
    counts = counts if counts is not None else {48: 32, 96: 24, 192: 8}
    rng = np.random.default_rng(seed)
    out = []
    k = 0
    for n in sorted(counts):
        for _ in range(counts[n]):
            amp = float(rng.uniform(*amplitude))
            ns = int(rng.integers(nsub[0], nsub[1] + 1))
            out.append(MemberSpec(n=int(n), seed=10_000 * (seed + 1) + 3 * k, amplitude=amp, nsub=ns))
            k += 1
    return out


class Geometry:
    """Host geometry and device plans per (resolution, dtype), generated once."""

    def __init__(self, depth: float = 5000.0, device=None):
        self.depth = float(depth)
        self.device = cuda_device(device)
        self._grids: Dict[int, dict] = {}
        self._plans: Dict[Tuple[int, torch.dtype], BtPlan] = {}

    def grid(self, n: int) -> dict:
        if n not in self._grids:
            self._grids[n] = duogrid_gen.load_or_generate(n)[0]
        return self._grids[n]

    def plan(self, n: int, dtype: torch.dtype) -> BtPlan:
        key = (n, dtype)
        if key not in self._plans:
            self._plans[key] = BtPlan(make_consts(self.grid(n), self.depth), dtype=dtype, device=self.device)
        return self._plans[key]

    def dtb(self, n: int) -> float:
        return cfl_dtb(self.grid(n), self.depth)

    def initial_state(self, spec: MemberSpec) -> Dict[str, np.ndarray]:
        return harmonic_state(self.grid(spec.n), spec.seed, h_rms=spec.amplitude, uv_rms=UV_PER_H * spec.amplitude)

    def close(self) -> None:
        for p in self._plans.values():
            p.close()
        self._plans.clear()


class Ensemble:
    """The members of a mix, ready to run in one dtype."""

    def __init__(self, specs: Sequence[MemberSpec], dtype: torch.dtype = torch.float32, rk: int = 2,
                 geometry: Optional[Geometry] = None, depth: float = 5000.0, device=None):
        self.specs = list(specs)
        self.dtype = dtype
        self.rk = int(rk)
        self.geo = geometry if geometry is not None else Geometry(depth, device)
        self.device = self.geo.device
        self.init = []
        for s in self.specs:
            st = self.geo.initial_state(s)
            self.init.append(tuple(torch.from_numpy(st[k]).to(self.device, dtype) for k in ("h0", "ub", "vb")))

    def cell_updates(self) -> int:
        return sum(6 * s.n * s.n * s.nsub for s in self.specs)

    def members(self) -> List[MemberState]:
        """Fresh device states at the initial condition."""
        out = []
        for s, (h, u, v) in zip(self.specs, self.init):
            out.append(MemberState(self.geo.plan(s.n, self.dtype), h.clone(), u.clone(), v.clone(), s.nsub,
                                   self.geo.dtb(s.n), rk=self.rk, tag=s))
        return out

    def run_batched(self, batch: BtBatch, members: Optional[List[MemberState]] = None,
                    max_substeps: Optional[int] = None, stream=None) -> List[MemberState]:
        """All members to the end, batched; ``max_substeps`` caps a round
        (None: one round, one launch)."""
        mem = members if members is not None else self.members()
        while batch.advance(mem, max_substeps=max_substeps, stream=stream):
            pass
        return mem


class PlainRunner:
    """The one-integration-per-launch comparison: every member through the
    drop-in round (``bt_round``) with its own plan, in the single-member mode
    and tile shape the autotuner picked for its resolution."""

    def __init__(self, ens: Ensemble, configs: Dict[int, dict]):
        self.ens = ens
        self.plans = []
        self.bufs = []
        for s, x0 in zip(ens.specs, ens.init):
            cfg = configs[s.n]
            p = BtPlan(make_consts(ens.geo.grid(s.n), ens.geo.depth), dtype=ens.dtype, device=ens.device,
                       tile=tuple(cfg["tile"]), mode=cfg["mode"])
            self.plans.append(p)
            self.bufs.append({k: p.empty_field() for k in ("h0", "ub", "vb")})

    def run(self, stream=None) -> List[Dict[str, torch.Tensor]]:
        for s, p, x0, out in zip(self.ens.specs, self.plans, self.ens.init, self.bufs):
            h, u, v = x0
            p.round(h, h, u, v, u, v, nbb=s.nsub, dtb=self.ens.geo.dtb(s.n), rk=self.ens.rk, diag=False, out=out,
                    stream=stream)
        return self.bufs

    def close(self) -> None:
        for p in self.plans:
            p.close()
