"""Solver plans: the compiled, device-resident form of one resolution's constants.

A :class:`BtPlan` is what ``make_spmd_jit`` + the closure-captured consts are
in the reference (src/licom/kernel/spmd.py:38-75,
md/SPMD_JIT_Architecture.md:66-77): built once from the 17 constants, it owns
the halo gather tables and the stage scratch, and advances states by rounds of
substeps through ``libbt.so``.  PyTorch only provides device memory and
streams here.
"""

from __future__ import annotations

import ctypes
from typing import Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _native as N

CONST_NAMES = ("dzph_x", "dzph_y", "rdx", "rdy", "a_f", "k2e_coef", "loc_i_local", "loc_j_local",
               "a_c2l", "a_l2c", "inner", "outer", "a_gct", "a_sina", "rda", "c_dy", "d_dx")
DIAG_NAMES = ("celerity_x", "celerity_y", "ub_ct", "vb_ct", "ub_cx", "ub_cy", "vb_cx", "vb_cy",
              "advx", "advy")
_INT_CONSTS = ("loc_i_local", "loc_j_local")

_MODES = {"stream": N.BT_MODE_STREAM, "graph": N.BT_MODE_GRAPH, "persistent": N.BT_MODE_PERSISTENT,
          "resident": N.BT_MODE_RESIDENT}


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream_handle(stream: Optional[torch.cuda.Stream]):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def cuda_device(device=None) -> torch.device:
    """``device`` as an indexed CUDA device (None / "cuda" -> the current device)."""
    d = torch.device(device) if device is not None else torch.device("cuda")
    if d.type != "cuda":
        raise ValueError(f"expected a CUDA device, got {d}")
    return d if d.index is not None else torch.device("cuda", torch.cuda.current_device())


def to_device(a, dtype: torch.dtype, device) -> torch.Tensor:
    """Contiguous CUDA tensor of ``dtype`` starting on a 16-byte boundary (the
    kernels read 2x2 matrices with 16-byte loads); numpy arrays and
    misaligned views are copied once."""
    if isinstance(a, np.ndarray):
        a = torch.from_numpy(np.ascontiguousarray(a))
    if not isinstance(a, torch.Tensor):
        raise TypeError(f"expected a torch.Tensor or numpy.ndarray, got {type(a).__name__}")
    t = a.to(device=device, dtype=dtype).contiguous()
    if t.data_ptr() % 16:
        t = t.clone()
    return t


class BtPlan:
    """Plan for one resolution N and one dtype (float64 drop-in or float32 precision form)."""

    def __init__(self, consts: Sequence, dtype: torch.dtype = torch.float64, device=None,
                 tile: Tuple[int, int] = (8, 32), mode: str = "stream"):
        if not torch.cuda.is_available():
            raise RuntimeError("licom4py_gpu_b200 needs a CUDA device (there is no CPU path)")
        if len(consts) < 17:
            raise ValueError(f"consts must hold the 17 CONST_SOURCES arrays, got {len(consts)}")
        if dtype not in (torch.float64, torch.float32):
            raise ValueError("dtype must be torch.float64 or torch.float32")
        self.device = cuda_device(device)
        self.dtype = dtype
        with torch.cuda.device(self.device):
            tens = []
            for name, c in zip(CONST_NAMES, consts[:17]):
                tens.append(to_device(c, torch.int32 if name in _INT_CONSTS else dtype, self.device))
        m = tens[2].shape[-1]
        for name, t in zip(CONST_NAMES, tens):
            if t.shape[:3] != (6, m, m):
                raise ValueError(f"const {name} has shape {tuple(t.shape)}, expected (6, {m}, {m}, ...)")
        self.n = m - 6
        self.m = m
        self.consts = dict(zip(CONST_NAMES, tens))
        desc = N.GridDesc(self.n, N.BT_F64 if dtype == torch.float64 else N.BT_F32,
                          *[t.data_ptr() for t in tens])
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            N.check(N.lib().bt_plan_create(ctypes.byref(desc), ctypes.byref(handle)))
        self._h = handle
        self.tile = tuple(tile)
        self.mode = mode
        self.set_tile(*tile)
        self.set_mode(mode)

    # -- configuration ---------------------------------------------------------
    def set_tile(self, ti: int, tj: int) -> None:
        N.check(N.lib().bt_plan_set_tile(self._h, int(ti), int(tj)))
        self.tile = (int(ti), int(tj))

    def set_mode(self, mode: str) -> None:
        if mode not in _MODES:
            raise ValueError(f"mode must be one of {sorted(_MODES)}")
        N.check(N.lib().bt_plan_set_mode(self._h, _MODES[mode]))
        self.mode = mode

    def set_option(self, key: int, value: int) -> None:
        N.check(N.lib().bt_plan_set_option(self._h, int(key), int(value)))

    def set_max_ctas(self, n: int) -> None:
        """Persistent mode: cap the cooperative grid (0 = as many as fit)."""
        self.set_option(N.BT_OPT_MAX_CTAS, n)

    def set_spin_limit(self, polls: int) -> None:
        """Persistent / resident mode: polls a grid-barrier or neighbour-tile wait may take
        before the round is abandoned."""
        self.set_option(N.BT_OPT_SPIN_LIMIT, polls)

    def enable_kernel_timing(self, on: bool = True) -> None:
        """Bracket the round kernel (persistent / resident mode) or each phase kernel
        (stream mode) with CUDA events on its stream; resets the record."""
        self.set_option(N.BT_OPT_KERNEL_TIMING, 1 if on else 0)

    def set_full_tiles(self, which) -> None:
        """Stream / graph mode phase kernels: None (default) by size -- the kernels with a
        path specialised for full interior tiles when a launch takes more than one wave of
        CTAs, the smaller edge-path-only kernels otherwise; True / False forces one of them.
        The results are the same."""
        self.set_option(N.BT_OPT_FULL_TILES, -1 if which is None else (1 if which else 0))

    KERNELS = {"round": N.BT_KERNEL_ROUND, "phase_h": N.BT_KERNEL_PHASE_H, "phase_uv": N.BT_KERNEL_PHASE_UV}

    def kernel_time(self, kind: str = "round") -> Tuple[float, int]:
        """(total ms, launches) of the timed kernels of ``kind`` since timing was enabled."""
        ms = ctypes.c_double()
        n = ctypes.c_int()
        N.check(N.lib().bt_plan_kernel_time(self._h, self.KERNELS[kind], ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    @property
    def last_grid(self) -> int:
        return int(N.lib().bt_plan_get_info(self._h, N.BT_INFO_LAST_GRID))

    @property
    def scratch_bytes(self) -> int:
        return int(N.lib().bt_plan_get_info(self._h, N.BT_INFO_SCRATCH_BYTES))

    @property
    def full_tile_kernels(self) -> Tuple[bool, bool]:
        """(phase H, phase UV): whether the stream / graph mode launches at this plan's tile and
        size run the kernels with the full-tile path (else the edge-path-only kernels)."""
        bits = int(N.lib().bt_plan_get_info(self._h, N.BT_INFO_FULL_TILES))
        return bool(bits & 1), bool(bits & 2)

    # -- validation --------------------------------------------------------------
    def _check_field(self, name: str, t: torch.Tensor) -> None:
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{name} must be a torch.Tensor")
        if t.shape != (6, self.m, self.m):
            raise ValueError(f"{name} has shape {tuple(t.shape)}, expected (6, {self.m}, {self.m})")
        if t.dtype != self.dtype:
            raise ValueError(f"{name} has dtype {t.dtype}, plan dtype is {self.dtype}")
        if t.device != self.device:
            raise ValueError(f"{name} is on {t.device}, plan is on {self.device}")
        if not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous")

    def empty_field(self) -> torch.Tensor:
        return torch.empty((6, self.m, self.m), dtype=self.dtype, device=self.device)

    # -- work ----------------------------------------------------------------
    def round(self, h0, h0p, ub, vb, ubp, vbp, nbb: int, dtb: float, rk: int = 2,
              diag: bool = True, out: Optional[Dict[str, torch.Tensor]] = None,
              stream: Optional[torch.cuda.Stream] = None) -> Dict[str, torch.Tensor]:
        """Advance ``nbb`` substeps; returns the new h0/ub/vb (+ the 10 diagnostics)."""
        ins = {"h0": h0, "h0p": h0p, "ub": ub, "vb": vb, "ubp": ubp, "vbp": vbp}
        for k, t in ins.items():
            self._check_field(k, t)
        if int(nbb) < 1:
            raise ValueError("nbb must be >= 1 (nbb = 0 is handled by the caller)")
        if out is None:
            out = {k: self.empty_field() for k in ("h0", "ub", "vb")}
            if diag:
                out.update({k: self.empty_field() for k in DIAG_NAMES})
        for k in ("h0", "ub", "vb") + (DIAG_NAMES if diag else ()):
            self._check_field("out." + k, out[k])
        sin = N.StateIn(*[t.data_ptr() for t in ins.values()])
        dptrs = [(out[k].data_ptr() if diag else 0) for k in DIAG_NAMES]
        sout = N.StateOut(out["h0"].data_ptr(), out["ub"].data_ptr(), out["vb"].data_ptr(),
                          (ctypes.c_void_p * 10)(*dptrs))
        with torch.cuda.device(self.device):
            N.check(N.lib().bt_round(self._h, ctypes.byref(sin), ctypes.byref(sout), int(nbb),
                                     float(dtb), int(rk), _stream_handle(stream)))
        return out

    def stage(self, h0, h0p, ub, vb, ubp, vbp, dt: float, beta_d: float, is_laststep: bool,
              diag: bool = True, stream: Optional[torch.cuda.Stream] = None) -> Dict[str, torch.Tensor]:
        """One RK stage on fields with valid halos (barotr_pure.py:100-168)."""
        ins = {"h0": h0, "h0p": h0p, "ub": ub, "vb": vb, "ubp": ubp, "vbp": vbp}
        for k, t in ins.items():
            self._check_field(k, t)
        out = {k: self.empty_field() for k in ("h0", "ub", "vb")}
        if diag:
            out.update({k: self.empty_field() for k in DIAG_NAMES})
        sin = N.StateIn(*[t.data_ptr() for t in ins.values()])
        dptrs = [(out[k].data_ptr() if diag else 0) for k in DIAG_NAMES]
        sout = N.StateOut(out["h0"].data_ptr(), out["ub"].data_ptr(), out["vb"].data_ptr(),
                          (ctypes.c_void_p * 10)(*dptrs))
        with torch.cuda.device(self.device):
            N.check(N.lib().bt_stage(self._h, ctypes.byref(sin), ctypes.byref(sout), float(dt),
                                     float(beta_d), 1 if is_laststep else 0, _stream_handle(stream)))
        return out

    def fill_halo(self, h=None, u=None, v=None, stream=None) -> None:
        """ext_scalar(h) / ext_vector(u, v) in place (src/licom/kernel/cube.py:130-153)."""
        for k, t in (("h", h), ("u", u), ("v", v)):
            if t is not None:
                self._check_field(k, t)
        with torch.cuda.device(self.device):
            N.check(N.lib().bt_fill_halo(self._h, _ptr(h), _ptr(u), _ptr(v), _stream_handle(stream)))

    def edge_average(self, u, v, stream=None) -> None:
        """boundary_communication(u, v) in place (src/licom/kernel/communication.py:504-570)."""
        self._check_field("u", u)
        self._check_field("v", v)
        with torch.cuda.device(self.device):
            N.check(N.lib().bt_edge_average(self._h, _ptr(u), _ptr(v), _stream_handle(stream)))

    def check_device_error(self) -> None:
        N.check(N.lib().bt_check_device_error(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().bt_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
