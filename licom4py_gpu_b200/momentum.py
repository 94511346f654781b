"""Barotropic momentum state and its diagnostics.

``Momentum`` mirrors the part of the reference's ``Momentum``/``MomentumData``
(src/licom/momentum/momentum.py:26-43, src/licom/datatype/momentum_data.py:20-71)
that the barotropic path uses: the 23 STATE_KEYS fields as CUDA tensors,
``nbb = baroclinic_dt // barotropic_dt``, ``dtb`` and ``rk_barotr``, initial
fields from the W92 case-2 state or the seeded harmonic generator.

Diagnostics are computed on the device (``bt_interior_stats``), copied to
pinned host memory asynchronously, and formatted like
src/licom/mymodule/diag.py:45-75.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np
import torch

from . import _native as N
from .duogrid import Duogrid
from .fields import harmonic_state, w92_case2_state

STATE_KEYS = (
    "h0", "h0p", "ub", "vb", "ubp", "vbp",
    "celerity_x", "celerity_y", "ub_ct", "vb_ct", "ub_cx", "ub_cy", "vb_cx", "vb_cy",
    "advx", "advy",
    "pax", "pxb", "whx", "pay", "pyb", "why", "wgp",
)


@dataclass
class Namelist:
    """The namelist entries the barotropic path consumes (scripts/namelist; readnamelist/*)."""
    barotropic_dt: float = 30.0
    baroclinic_dt: float = 3600.0
    rk_barotr: int = 2
    case: str = "w92case2"
    nx: int = 96
    integration_days: float = 2.0
    diag_freq: Optional[float] = 24.0
    async_threads: int = 8
    start_year: int = 2000
    start_month: int = 1
    start_day: int = 1

    @property
    def total_baroclinic_steps(self) -> int:
        return int(round(self.integration_days * 86400.0 / self.baroclinic_dt))

    @property
    def start_datetime(self):
        import datetime
        return datetime.datetime(self.start_year, self.start_month, self.start_day)

    @classmethod
    def from_file(cls, path: str) -> "Namelist":
        """Read the INI namelist of the reference (scripts/namelist)."""
        import configparser
        cp = configparser.ConfigParser(inline_comment_prefixes=("#",))
        cp.read(path)
        nl = cls()
        r = cp["run_params"] if cp.has_section("run_params") else {}
        nl.barotropic_dt = float(r.get("barotropic_dt", nl.barotropic_dt))
        nl.baroclinic_dt = float(r.get("baroclinic_dt", nl.baroclinic_dt))
        nl.rk_barotr = int(r.get("rk_barotr", nl.rk_barotr))
        nl.case = r.get("case", nl.case)
        if cp.has_section("grid"):
            nl.nx = int(cp["grid"].get("nx", nl.nx))
        if cp.has_section("time_params"):
            t = cp["time_params"]
            nl.integration_days = float(t.get("integration_days", nl.integration_days))
            nl.start_year = int(t.get("start_year", nl.start_year))
            nl.start_month = int(t.get("start_month", nl.start_month))
            nl.start_day = int(t.get("start_day", nl.start_day))
        if cp.has_section("async_io"):
            a = cp["async_io"]
            nl.diag_freq = float(a.get("diag_freq", nl.diag_freq))
            nl.async_threads = int(a.get("async_threads", nl.async_threads))
        return nl


def interior_stats(field: torch.Tensor, out: Optional[torch.Tensor] = None,
                   stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """(max, min, mean) of the interior cells as a float64 device tensor of 3."""
    n = field.shape[-1] - 6
    if out is None:
        out = torch.empty(3, dtype=torch.float64, device=field.device)
    s = stream if stream is not None else torch.cuda.current_stream(field.device)
    dt = N.BT_F64 if field.dtype == torch.float64 else N.BT_F32
    N.check(N.lib().bt_interior_stats(n, dt, ctypes.c_void_p(field.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                      ctypes.c_void_p(s.cuda_stream)))
    return out


def conservation(h: torch.Tensor, u: torch.Tensor, v: torch.Tensor, rda: torch.Tensor, a_c2l: torch.Tensor,
                 depth: float, stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """(mass, energy) over the interior, compensated float64 sums of per-cell terms."""
    n = h.shape[-1] - 6
    out = torch.empty(2, dtype=torch.float64, device=h.device)
    s = stream if stream is not None else torch.cuda.current_stream(h.device)
    dt = N.BT_F64 if h.dtype == torch.float64 else N.BT_F32
    for t in (u, v, rda, a_c2l):
        if t.dtype != h.dtype or not t.is_contiguous():
            raise ValueError("conservation: all fields must be contiguous and share h's dtype")
    N.check(N.lib().bt_conservation(n, dt, *[ctypes.c_void_p(t.data_ptr()) for t in (h, u, v, rda, a_c2l)],
                                    float(depth), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s.cuda_stream)))
    return out


class Momentum:
    """Barotropic state container (the reference's Momentum, barotropic part)."""

    def __init__(self, namelist: Namelist, case: Optional[str] = None, seed: int = 1,
                 dtype: torch.dtype = torch.float64, device=None, verbose: bool = True):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.dtype = dtype
        self.verbose = verbose
        self.nbb = int(namelist.baroclinic_dt // namelist.barotropic_dt)  # momentum.py:37
        self.dtb = float(namelist.barotropic_dt)                           # momentum.py:39
        self.rk_barotr = int(namelist.rk_barotr)
        grid = Duogrid.grid_dict()
        case = case or namelist.case
        if case == "w92case2":
            st = w92_case2_state(grid)
        elif case == "harmonic":
            st = harmonic_state(grid, seed)
        else:
            raise ValueError(f"unknown initial case {case!r}")
        m = grid["rdx"].shape[-1]
        self.m = m
        to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device, dtype)  # noqa: E731
        self.h0, self.ub, self.vb = to(st["h0"]), to(st["ub"]), to(st["vb"])
        self.h0p, self.ubp, self.vbp = self.h0, self.ub, self.vb  # w92_field.py:93-96
        for k in STATE_KEYS[6:]:
            setattr(self, k, torch.zeros((6, m, m), dtype=dtype, device=self.device))
        self._stats_dev = torch.empty(9, dtype=torch.float64, device=self.device)

    def device_diag(self, state) -> Tuple[torch.Tensor, torch.cuda.Event]:
        """Interior max/min/mean of h0, ub, vb on the device, copied to pinned host memory."""
        stats = torch.empty(9, dtype=torch.float64, device=self.device)
        for k, idx in enumerate((0, 2, 3)):
            interior_stats(state[idx], out=stats[3 * k:3 * k + 3])
        host = torch.empty(9, dtype=torch.float64).pin_memory()
        host.copy_(stats, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        return host, ev

    @staticmethod
    def format_global_diag(time_str: str, stats) -> str:
        """The report of print_global_diag (src/licom/mymodule/diag.py:69-77)."""
        s = [float(x) for x in stats]
        out = [
            f"{time_str}",
            "                  max                  min                 mean",
            f"Global h0: {s[0]:20.16f}  {s[1]:20.16f}  {s[2]:20.16f}",
            f"Global ub: {s[3]:20.16f}  {s[4]:20.16f}  {s[5]:20.16f}",
            f"Global vb: {s[6]:20.16f}  {s[7]:20.16f}  {s[8]:20.16f}",
            "------------------------------------------------",
        ]
        return "\n".join(out)

    def print_global_diag(self, time_str: str) -> None:
        host, ev = self.device_diag(tuple(getattr(self, k) for k in STATE_KEYS))
        ev.synchronize()
        print(self.format_global_diag(time_str, host), flush=True)
