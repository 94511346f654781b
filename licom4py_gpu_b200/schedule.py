"""Scheduler entry of the barotropic path: field sets, schedule_core, Schedule.configure/run.

Same names, field order and call shapes as the reference's
src/licom/mymodule/schedule.py:

* ``STATE_KEYS`` (23 mutable fields) and ``CONST_SOURCES`` (17 read-only
  geometry fields, each ``(source, attribute)``), schedule.py:62-116;
* ``_make_schedule_core(rk_type)`` returns ``schedule_core(state, consts,
  chunk_size, nbb, dtb)`` running ``chunk_size`` baroclinic steps of ``nbb``
  barotropic substeps each (schedule.py:130-192);
* ``make_plan_fn(core_fn, state, consts)`` replaces ``make_spmd_jit``
  (src/licom/kernel/spmd.py:38-75): instead of tracing and compiling it builds
  the device plan of the constants once and returns ``fn(state, consts, n,
  nbb, dtb)``;
* ``Schedule.configure(namelist, momentum)`` / ``Schedule.run(momentum)``
  (schedule.py:209-313): chunked rounds with the diagnostics of each chunk
  computed on the device and reported from a host thread pool.

The state fields are CUDA tensors; there is no mesh: px = py = 1.
"""

from __future__ import annotations

import concurrent.futures
import datetime as _dt
from typing import Any, Callable, Optional, Sequence, Tuple

import torch

from .barotr import _barotr_rk2_core, _barotr_rk3_core, get_plan
from .duogrid import Duogrid as Dg

STATE_KEYS = (
    # --- Barotropic core state (0 ~ 15) ---
    "h0", "h0p", "ub", "vb", "ubp", "vbp",
    "celerity_x", "celerity_y", "ub_ct", "vb_ct", "ub_cx", "ub_cy", "vb_cx", "vb_cy",
    "advx", "advy",
    # --- Cross-module coupling fields (passed through by the barotropic core) ---
    "pax", "pxb", "whx", "pay", "pyb", "why", "wgp",
)

CONST_SOURCES = (
    (Dg, "dzph_x"), (Dg, "dzph_y"), (Dg, "rdx"), (Dg, "rdy"), (Dg, "a_f"),
    (Dg, "k2e_coef"), (Dg, "loc_i_local"), (Dg, "loc_j_local"), (Dg, "a_c2l"), (Dg, "a_l2c"),
    (Dg, "inner"), (Dg, "outer"),
    (Dg, "a_gct"), (Dg, "a_sina"), (Dg, "rda"), (Dg, "c_dy"), (Dg, "d_dx"),
)

N_BAROTR_STATE = 23
N_BAROTR_CONSTS = 17


def auto_pack(instance, state_keys, const_sources) -> Tuple[tuple, tuple]:
    """state and consts tuples from an instance and const sources (spmd.py:83-93)."""
    state = tuple(getattr(instance, k) for k in state_keys)
    consts = tuple(getattr(src, k) if src is not None else getattr(instance, k) for src, k in const_sources)
    return state, consts


def auto_unpack(instance, state_keys, state) -> None:
    """Write a state tuple back into the instance (spmd.py:96-102)."""
    for k, v in zip(state_keys, state):
        setattr(instance, k, v)


def _make_schedule_core(rk_type_barotr: int) -> Callable:
    """schedule_core(state, consts, chunk_size, nbb, dtb) for RK2 (rk = 2) or RK3."""
    rk_core = _barotr_rk2_core if rk_type_barotr == 2 else _barotr_rk3_core
    px = py = 1  # one GPU holds all six faces

    def schedule_core(state, consts, chunk_size, nbb, dtb):
        barotr_consts = tuple(consts[:N_BAROTR_CONSTS])
        s = tuple(state)
        for _ in range(int(chunk_size)):
            barotr_s = rk_core(s[:N_BAROTR_STATE], barotr_consts, nbb, dtb, px, py)
            s = tuple(barotr_s) + s[N_BAROTR_STATE:]
        return s

    return schedule_core


def make_plan_fn(core_fn: Callable, state: Sequence, consts: Sequence,
                 static_argnums=(2, 3, 4)) -> Callable:
    """Build the device plan of ``consts`` now and return ``fn(state, consts, *static)``.

    Stands in for make_spmd_jit: the plan (halo tables, scratch, kernel setup)
    is what a compile would produce; ``static_argnums`` is accepted for call
    compatibility.
    """
    dtype = state[0].dtype if isinstance(state[0], torch.Tensor) else torch.float64
    get_plan(consts, dtype=dtype)

    def fn(s, c, *static_args):
        return core_fn(s, c, *static_args)

    return fn


class Timer:
    """Model clock advanced by baroclinic steps (readnamelist/timemanager.py:16-73, subset)."""

    def __init__(self, start: _dt.datetime, step_seconds: float):
        self.current = start
        self.prev_dt = start
        self.step = _dt.timedelta(seconds=float(step_seconds))

    def advance(self, n: int) -> None:
        self.prev_dt = self.current
        self.current = self.current + n * self.step
        self.prev_dt = self.current


def _namelist_value(namelist, name: str):
    """A derived namelist value: the reference's private field ``_<name>`` if the
    object has it, else the public attribute ``name``; AttributeError if neither."""
    for attr in ("_" + name, name):
        if hasattr(namelist, attr):
            return getattr(namelist, attr)
    raise AttributeError(f"namelist has neither _{name} nor {name}")


class Schedule:
    """Global scheduler (schedule.py:200-313): configure once, then run in chunks."""

    @classmethod
    def configure(cls, namelist, momentum, routines: Optional[list] = None) -> None:
        """``namelist`` is the reference's ``Namelist`` (its derived values are the
        private ``_start_datetime`` / ``_total_baroclinic_steps`` fields,
        readnamelist/time_data.py:61, namelist_data.py:56, read as at
        schedule.py:216-218) or any object with the public names
        ``start_datetime`` / ``total_baroclinic_steps`` (this package's ``Namelist``)."""
        cls.current_time = Timer(_namelist_value(namelist, "start_datetime"), namelist.baroclinic_dt)
        cls.total_baroclinic_steps = int(_namelist_value(namelist, "total_baroclinic_steps"))
        cls.routines = ["barotropic", "baroclinic", "tracer"] if routines is None else routines
        diag_freq = getattr(namelist, "diag_freq", None)
        cls.diag_interval = (int(3600 / namelist.baroclinic_dt * diag_freq)
                             if diag_freq is not None and diag_freq > 0 else None)
        cls.async_threads = getattr(namelist, "async_threads", 8)
        cls._nbb = momentum.nbb
        cls._dtb = momentum.dtb
        cls._state, cls._consts = auto_pack(momentum, STATE_KEYS, CONST_SOURCES)
        core_fn = _make_schedule_core(momentum.rk_barotr)
        cls._jit_fn = make_plan_fn(core_fn, cls._state, cls._consts, static_argnums=(2, 3, 4))
        cls.reports = []

    @classmethod
    def _async_io_and_diag(cls, time_str: str, momentum, stats) -> None:
        """Background task: the device statistics of a chunk, already reduced, printed on the host."""
        text = momentum.format_global_diag(time_str, stats.cpu())
        cls.reports.append(text)
        if getattr(momentum, "verbose", True):
            print(text, flush=True)

    @classmethod
    def _dispatch_async_task(cls, executor, prefix: str, momentum) -> None:
        stats = momentum.device_diag(cls._state)  # on-device reduction, async copy to pinned host memory
        time_str = f"{prefix}: {cls.current_time.prev_dt.strftime('%Y-%m-%d-%H')}"
        executor.submit(cls._wait_and_report, time_str, momentum, stats)

    @classmethod
    def _wait_and_report(cls, time_str, momentum, stats) -> None:
        host, event = stats
        event.synchronize()
        cls._async_io_and_diag(time_str, momentum, host)

    @classmethod
    def run(cls, momentum) -> None:
        total = cls.total_baroclinic_steps
        chunk = cls.diag_interval if cls.diag_interval is not None else total
        with concurrent.futures.ThreadPoolExecutor(max_workers=cls.async_threads) as executor:
            cls._dispatch_async_task(executor, "Initial time", momentum)
            for start in range(0, total, chunk):
                n = min(chunk, total - start)
                cls._state = cls._jit_fn(cls._state, cls._consts, n, cls._nbb, cls._dtb)
                cls.current_time.advance(n)
                if cls.diag_interval is not None:
                    cls._dispatch_async_task(executor, "Time", momentum)
            if cls.diag_interval is None:
                cls._dispatch_async_task(executor, "Final time", momentum)
        auto_unpack(momentum, STATE_KEYS, cls._state)
