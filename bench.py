"""Benchmark of the barotropic RK2 path on the cubed-sphere duogrid (one JSON line).

Workload (one "step" = one call of the hot path): the plain drop-in
``_barotr_rk2_core`` round of ``--nbb`` substeps (default 1000) at C``--n``
(default C96: 6 x 96 x 96 cells + 3-cell halos) in float64, on seeded
synthetic fields: resting ocean of depth H = 5000 m, SSH perturbation = sum of
real spherical harmonics l = 1..8 scaled to 1 m RMS, lon/lat velocity the same
way at 0.3 m/s RMS, dtb at CFL 0.5 of sqrt(gH).

Metric: interior cell-updates per second (one cell advanced one substep of
two RK stages), whole job.  ``value`` is measured with inputs resident in HBM;
``e2e`` through the public call with host (pinned) buffers, host<->device
copies inside the timed region.  Between timed steps L2 is flushed by writing
a 512 MiB buffer (outside the per-step CUDA-event windows).

``--impl reference`` times the CPU implementation of the path instead (the
float64 oracle, which restates the reference's source bit for bit) on all
usable host cores (one single-threaded replica per core), on a bounded sample
of the same workload.

Multi-GPU (torchrun): replicas only, each rank integrates its own member; no
collective touches the data path.  Time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALG_WORDS = 41  # algorithmic words per cell-update over both RK stages (compulsory reads + writes of phase H and UV)
# Compulsory words per interior cell of each phase kernel, averaged over the two
# RK2 stages (stage 1 / stage 2): distinct field reads + writes of the kernel's work.
#   phase H : h, u, v, [h base], dzph_x, dzph_y, gct(4), sina, rda, c_dy, d_dx -> h     14 / 15
#   phase UV: u, v, h, new h, [u, v base], gct(4), sina, rda, rdx, rdy, a_f, c_dy,
#             d_dx, dzph_x, dzph_y -> u, v                                          18 / 20
KERNEL_WORDS = {"phase_h": 14.5, "phase_uv": 19.0}
KERNEL_NAMES = {"phase_h": "k_phase_h", "phase_uv": "k_phase_uv"}
METRIC = "barotropic cell-updates/s"
UNIT = "cell-updates/s"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=96)
    p.add_argument("--nbb", type=int, default=1000)
    p.add_argument("--depth", type=float, default=5000.0)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--mode", default="auto", choices=["auto", "resident", "persistent", "graph", "stream"])
    p.add_argument("--tile", default="auto")
    p.add_argument("--cpu-substeps", type=int, default=60,
                   help="substeps of the bounded CPU baseline sample")
    p.add_argument("--no-extras", action="store_true", help="skip the fp32 / mode comparison lines")
    p.add_argument("--case-only", action="store_true",
                   help="run one round of --nbb substeps (the profiling target) and exit, no timing")
    p.add_argument("--dtype", default="f64", choices=["f64", "f32"], help="dtype of --case-only")
    p.add_argument("--no-forms", action="store_true",
                   help="skip the layered forms (precision at C384, batched ensemble, serving)")
    p.add_argument("--serving-requests", type=int, default=100,
                   help="requests of the Poisson serving stream in the bounded serving sample")
    p.add_argument("--only-form", default=None, choices=["precision", "ensemble", "serving"],
                   help="run one layered form alone on one GPU and print its figures as one JSON line")
    p.add_argument("--no-oracle-check", action="store_true",
                   help="skip the float64 oracle run of the full timed round (error_vs_oracle)")
    return p.parse_args()


def run_case(args):
    """One round of the workload in the given mode/tile: the target of ncu captures."""
    import torch
    from licom4py_gpu_b200.plan import BtPlan
    _, consts, st, dtb = build_problem(args.n, args.depth, args.seed)
    dtype = torch.float64 if args.dtype == "f64" else torch.float32
    tile = (8, 16) if args.tile == "auto" else tuple(int(x) for x in args.tile.split("x"))
    mode = "stream" if args.mode == "auto" else args.mode
    p = BtPlan(consts, dtype=dtype, tile=tile, mode=mode)
    h = torch.from_numpy(st["h0"]).cuda().to(dtype)
    u = torch.from_numpy(st["ub"]).cuda().to(dtype)
    v = torch.from_numpy(st["vb"]).cuda().to(dtype)
    out = p.round(h, h, u, v, u, v, nbb=args.nbb, dtb=dtb)
    torch.cuda.synchronize()
    p.check_device_error()
    print(json.dumps({"case": f"C{args.n}", "dtype": args.dtype, "mode": mode, "tile": list(tile),
                      "nbb": args.nbb, "h_absmax": float(out["h0"].abs().max())}))


def dist_setup(args):
    from licom4py_gpu_b200 import replicas
    return replicas.setup("nccl")


def barrier(world):
    from licom4py_gpu_b200 import replicas
    replicas.barrier()


def max_over_ranks(x, world):
    from licom4py_gpu_b200 import replicas
    return replicas.max_over_ranks(x)


GEOMETRY_CACHE = {}  # resolution -> "hit" / "generated" (duogrid_C{N}.npz cache)


def build_problem(n, depth, seed):
    from licom4py_gpu_b200 import duogrid_gen
    from licom4py_gpu_b200.duogrid import make_consts
    from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state
    grid, hit = duogrid_gen.load_or_generate(n)
    GEOMETRY_CACHE[n] = "hit" if hit else "generated"
    consts = make_consts(grid, depth)
    st = harmonic_state(grid, seed)
    dtb = cfl_dtb(grid, depth)
    return grid, consts, st, dtb


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 7 and parts[0].isdigit():
                    rows.append(parts)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.remove(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [int(r[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][1]), "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU baseline (the float64 oracle, bit-exact to the reference's source)
# ---------------------------------------------------------------------------
def cpu_baseline(consts, st, dtb, n, substeps):
    from oracle import barotr_np as O
    m = n + 6
    state = [st["h0"], st["h0"], st["ub"], st["vb"], st["ub"], st["vb"]] + [np.zeros((6, m, m))] * 17
    t0 = time.perf_counter()
    O.rk2_core(state, consts, substeps, dtb)
    dt = time.perf_counter() - t0
    cells = 6 * n * n
    return {"value": cells * substeps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"C{n} float64, {substeps} RK2 substeps from the same initial state "
                      f"({dt:.1f} s, single-threaded NumPy oracle)"}


def l2_copy_gbs(dev, reps=100):
    """Device copy bandwidth of L2-resident buffers (48 MiB read + 48 MiB written per copy,
    96 MiB in all, under the 126 MB L2; large enough that the gaps between copies are
    small), bytes moved / time: the L2 figure the C48-C96 rounds are set against."""
    import torch
    src = torch.ones(12 << 20, dtype=torch.float32, device=dev)
    dst = torch.empty_like(src)
    for _ in range(5):
        dst.copy_(src)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        dst.copy_(src)
    b.record()
    torch.cuda.synchronize()
    return 2 * src.numel() * 4 * reps / (a.elapsed_time(b) * 1e-3) / 1e9


def _oracle_round(n, depth, seed, nbb):
    """The oracle's float64 h0, ub, vb after the full round of the timed workload."""
    from oracle import barotr_np as O
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    _, consts, st, dtb = build_problem(n, depth, seed)
    m = n + 6
    state = [st["h0"], st["h0"], st["ub"], st["vb"], st["ub"], st["vb"]] + [np.zeros((6, m, m))] * 17
    out = O.rk2_core(state, consts, nbb, dtb)
    return out[0], out[2], out[3]


class OracleCheck:
    """Part of the CPU-baseline leg: the float64 oracle runs the timed workload's
    full round (every substep, same inputs) in one spawned host process while the
    GPU legs run, and the GPU results of the timed runs are compared with it."""

    def __init__(self, n, depth, seed, nbb):
        import multiprocessing as mp
        self.nbb = nbb
        self.pool = mp.get_context("spawn").Pool(1)
        self.job = self.pool.apply_async(_oracle_round, (n, depth, seed, nbb))

    def compare(self, results, timeout_s=900.0):
        """results: {label: {"h0": t, "ub": t, "vb": t}} of device tensors; per label
        and field the relative L2 and max-norm error over the interior, and whether
        the field equals the oracle bit for bit."""
        try:
            want = self.job.get(timeout=timeout_s)
        except Exception as e:  # a report, not a failure of the bench
            return {"error": f"oracle run did not finish: {type(e).__name__}"}
        finally:
            self.pool.terminate()
        rep = {"substeps": self.nbb}
        for label, res in results.items():
            r = {}
            for key, ref in zip(("h0", "ub", "vb"), want):
                got = res[key].double().cpu().numpy()
                a, b = got[:, 3:-3, 3:-3], ref[:, 3:-3, 3:-3]
                r[key] = {"rel_l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                          "rel_linf": float(np.abs(a - b).max() / np.abs(b).max()),
                          "bitwise": bool(np.array_equal(got, ref))}
            rep[label] = r
        return rep


def _oracle_requests(depth, items):
    """The oracle's float64 h0 for each (n, substeps, seed, amplitude) request of the
    serving stream (initial state as fields.harmonic_state, dtb at CFL 0.5)."""
    from oracle import barotr_np as O
    from licom4py_gpu_b200 import duogrid_gen
    from licom4py_gpu_b200.duogrid import make_consts
    from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    res = []
    for n, nsub, seed, amp in items:
        grid = duogrid_gen.load_or_generate(n)[0]
        consts = make_consts(grid, depth)
        st = harmonic_state(grid, seed, amp, 0.3 * amp)
        m = n + 6
        state = [st["h0"], st["h0"], st["ub"], st["vb"], st["ub"], st["vb"]] + [np.zeros((6, m, m))] * 17
        res.append(O.rk2_core(state, consts, nsub, cfl_dtb(grid, depth))[0])
    return res


_REF_PROBLEM = None


def _ref_worker_init(n, depth, seed):
    """Pool initializer: each worker builds the problem once (single-threaded NumPy)."""
    global _REF_PROBLEM
    _, consts, st, dtb = build_problem(n, depth, seed)
    _REF_PROBLEM = (consts, st, dtb, n)


def _ref_worker_run(substeps):
    consts, st, dtb, n = _REF_PROBLEM
    return 6 * n * n * substeps / cpu_baseline(consts, st, dtb, n, substeps)["value"]


def ref_cores():
    """Host threads the reference arm uses: the usable cores, at most 64."""
    try:
        avail = len(os.sched_getaffinity(0))
    except AttributeError:
        avail = os.cpu_count() or 1
    return max(1, min(64, avail))


def cpu_baseline_all_cores(args):
    """The CPU-baseline leg of our own line: the same measurement as the reference arm (one
    single-threaded oracle replica of the workload per usable host core, spawned pool, a
    sample's time is the slowest replica's), on a bounded sample of the round."""
    import multiprocessing as mp
    cores = ref_cores()
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    sub = max(1, args.cpu_substeps // 10)
    cells = 6 * args.n * args.n
    with mp.get_context("spawn").Pool(cores, initializer=_ref_worker_init,
                                      initargs=(args.n, args.depth, args.seed)) as pool:
        pool.map(_ref_worker_run, [1] * cores)
        times = [max(pool.map(_ref_worker_run, [sub] * cores)) for _ in range(3)]
    t = statistics.median(times)
    return {"value": cores * cells * sub / t, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"C{args.n} float64, {cores} independent single-threaded replicas x {sub} RK2 substeps, "
                      f"3 samples (median; a sample's time is its slowest replica's), the oracle port"}


def run_reference(args, world, rank):
    """--impl reference: the CPU implementation of the path (the float64 oracle), rank 0 only, on
    every usable host core: one independent replica of the round per core in a process pool
    (started with spawn), each single-threaded; a step's time is the slowest replica's."""
    if rank != 0:
        return
    import multiprocessing as mp
    cores = ref_cores()
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"  # inherited by the workers: one thread each
    sub = max(1, args.cpu_substeps // max(1, args.steps))
    cells = 6 * args.n * args.n
    with mp.get_context("spawn").Pool(cores, initializer=_ref_worker_init,
                                      initargs=(args.n, args.depth, args.seed)) as pool:
        for _ in range(min(args.warmup, 1)):
            pool.map(_ref_worker_run, [1] * cores)
        vals, t_total = [], 0.0
        for _ in range(args.steps):
            times = pool.map(_ref_worker_run, [sub] * cores)
            t = max(times)
            vals.append(cores * cells * sub / t)
            t_total += t
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
            "data": "synthetic seeded spherical-harmonic fields",
            "config": {"workload": f"C{args.n} plain RK2, {sub} substeps per step (bounded sample of "
                                   f"the {args.nbb}-substep round), float64", "n": args.n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{cores} independent single-threaded replicas x {sub} substeps per step "
                                       f"x {args.steps} steps (time of the slowest replica)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Layered forms: precision at C384, batched uneven ensemble, serving
# ---------------------------------------------------------------------------
def _rel(a, b):
    """Relative L2 and max-norm error of a vs b over the interior cells (float64)."""
    a = a[:, 3:-3, 3:-3].double()
    b = b[:, 3:-3, 3:-3].double()
    return float((a - b).norm() / b.norm()), float((a - b).abs().max() / b.abs().max())


def form_precision(dev, depth, peak, seeds=8, nsub=2000):
    """Float32 precision form vs float64 at C384: 2000 substeps from 8 seeded
    states (h 1 m / u, v 0.3 m/s RMS); h/u/v errors, mass drift of both
    precisions from compensated float64 sums, throughput of both."""
    import torch
    from licom4py_gpu_b200 import duogrid_gen
    from licom4py_gpu_b200.autotune import choose_config
    from licom4py_gpu_b200.duogrid import make_consts
    from licom4py_gpu_b200.fields import cfl_dtb, harmonic_state
    from licom4py_gpu_b200.momentum import conservation
    from licom4py_gpu_b200.plan import BtPlan
    n = 384
    grid = duogrid_gen.load_or_generate(n)[0]
    consts = make_consts(grid, depth)
    dtb = cfl_dtb(grid, depth)
    rda = {}
    c2l = {}
    plans, times = {}, {torch.float64: 0.0, torch.float32: 0.0}
    for dt in (torch.float64, torch.float32):
        cfg = choose_config(n, dt, consts=consts, device=dev)
        plans[dt] = BtPlan(consts, dtype=dt, device=dev, tile=tuple(cfg["tile"]), mode=cfg["mode"])
        rda[dt] = torch.from_numpy(grid["rda"]).to(dev, dt)
        c2l[dt] = torch.from_numpy(np.ascontiguousarray(grid["a_c2l"])).to(dev, dt)
    err = {k: [0.0, 0.0] for k in ("h0", "ub", "vb")}
    drift = {"f64": [], "f32": []}
    da_abs = []
    for seed in range(1, seeds + 1):
        st = harmonic_state(grid, seed)
        outs = {}
        for dt in (torch.float64, torch.float32):
            h, u, v = (torch.from_numpy(st[k]).to(dev, dt) for k in ("h0", "ub", "vb"))
            p = plans[dt]
            p.round(h, h, u, v, u, v, nbb=2, dtb=dtb, diag=False)  # warm the graph path
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            o = p.round(h, h, u, v, u, v, nbb=nsub, dtb=dtb, diag=False)
            e1.record()
            torch.cuda.synchronize()
            times[dt] += e0.elapsed_time(e1)
            m0 = conservation(h, u, v, rda[dt], c2l[dt], depth).cpu().numpy()
            m1 = conservation(o["h0"], o["ub"], o["vb"], rda[dt], c2l[dt], depth).cpu().numpy()
            outs[dt] = (o, m0, m1)
        for k in err:
            l2, li = _rel(outs[torch.float32][0][k], outs[torch.float64][0][k])
            err[k][0] = max(err[k][0], l2)
            err[k][1] = max(err[k][1], li)
        hab = float((torch.from_numpy(np.abs(st["h0"][:, 3:-3, 3:-3]) / grid["rda"][:, 3:-3, 3:-3])).sum())
        da_abs.append(hab)
        for dt, tag in ((torch.float64, "f64"), (torch.float32, "f32")):
            _, m0, m1 = outs[dt]
            drift[tag].append((m1[0] - m0[0]) / hab)
    for p in plans.values():
        p.close()
    cu = 6 * n * n * nsub * seeds
    v64, v32 = cu / (times[torch.float64] * 1e-3), cu / (times[torch.float32] * 1e-3)
    return {"workload": f"C384, {nsub} RK2 substeps from {seeds} seeded states, float32 vs float64",
            "reference": "float64 path of this library, bit-identical to the float64 oracle of the reference source",
            "h_rel_l2": err["h0"][0], "h_rel_linf": err["h0"][1],
            "u_rel_l2": err["ub"][0], "u_rel_linf": err["ub"][1],
            "v_rel_l2": err["vb"][0], "v_rel_linf": err["vb"][1],
            "mass_drift_f64": float(max(abs(x) for x in drift["f64"])),
            "mass_drift_f32": float(max(abs(x) for x in drift["f32"])),
            "mass_drift_error": float(max(abs(a - b) for a, b in zip(drift["f32"], drift["f64"]))),
            "mass_drift_note": "mass sum(h da) change over the run / sum(|h0| da), compensated float64 sums",
            "f64": {"value": v64, "unit": UNIT, "round_frac_of_hbm": v64 * B_ALG_WORDS * 8 / 1e9 / peak},
            "f32": {"value": v32, "unit": UNIT, "round_frac_of_hbm": v32 * B_ALG_WORDS * 4 / 1e9 / peak}}


def form_ensemble(dev, depth):
    """Batched uneven ensemble (32 x C48, 24 x C96, 8 x C192; amplitudes
    U[0.2, 2] m, substeps U{200..2000}), float32, autotuned batch schedule:
    one persistent launch runs every member to its end.  Against the same
    members run one integration per launch through the drop-in path."""
    import torch
    from licom4py_gpu_b200 import autotune
    from licom4py_gpu_b200.batch import BtBatch
    from licom4py_gpu_b200.duogrid import make_consts
    from licom4py_gpu_b200.ensemble import Ensemble, Geometry, PlainRunner, uneven_mix
    import multiprocessing as mp
    specs = uneven_mix()
    # part of the CPU-baseline leg: the float64 oracle runs the 4 shortest C48 members (same seeded
    # initial states and CFL step) in a spawned host process while the GPU runs the ensemble
    pick = sorted(range(len(specs)), key=lambda k: (specs[k].n, specs[k].nsub))[:4]
    pool = mp.get_context("spawn").Pool(1)
    oracle_job = pool.apply_async(_oracle_requests, (depth, [(specs[k].n, specs[k].nsub, specs[k].seed,
                                                              specs[k].amplitude) for k in pick]))
    geo = Geometry(depth, device=dev)
    ens = Ensemble(specs, torch.float32, geometry=geo)
    cfg = autotune.choose_batch_config(ens)
    b = BtBatch(torch.float32, max_members=len(specs), device=dev, mode=cfg["mode"], tile=tuple(cfg["tile"]))
    b.set_max_ctas(cfg.get("max_ctas", 0))

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts), r

    work = ens.cell_updates()
    ens.run_batched(b)
    ms_b, mem32 = timed(lambda: ens.run_batched(b), 3)
    b.check_device_error()
    singles = {n: autotune.choose_config(n, torch.float32, consts=make_consts(geo.grid(n), depth), device=dev)
               for n in sorted({s.n for s in specs})}
    pr = PlainRunner(ens, singles)
    pr.run()
    ms_p, _ = timed(pr.run, 2)
    pr.close()
    # accuracy: every member against its float64 integration
    ens64 = Ensemble(specs, torch.float64, geometry=geo)
    b64 = BtBatch(torch.float64, max_members=len(specs), device=dev)
    mem64 = ens64.run_batched(b64)
    torch.cuda.synchronize()
    l2 = max(_rel(a.state[0], c.state[0])[0] for a, c in zip(mem32, mem64))
    li = max(_rel(a.state[0], c.state[0])[1] for a, c in zip(mem32, mem64))
    try:
        want = oracle_job.get(timeout=900)
        vs_oracle = max(_rel(mem32[k].state[0], torch.from_numpy(w).to(dev))[0] for k, w in zip(pick, want))
    except Exception as e:  # a report, not a failure of the bench
        vs_oracle = f"oracle run did not finish: {type(e).__name__}"
    finally:
        pool.terminate()
    b.close()
    b64.close()
    geo.close()
    vb, vp = work / (ms_b * 1e-3), work / (ms_p * 1e-3)
    return {"workload": "64 members (32 x C48, 24 x C96, 8 x C192), amplitude U[0.2, 2] m, substeps U{200..2000}, "
                        "RK2, float32; one persistent launch for the whole run, members retire early",
            "cell_updates": work, "batched": {"value": vb, "unit": UNIT, "ms": ms_b,
                                              "schedule": {k: cfg[k] for k in ("mode", "tile", "max_ctas", "source")
                                                           if k in cfg}},
            "plain_one_per_launch": {"value": vp, "unit": UNIT, "ms": ms_p,
                                     "configs": {str(k): [v["mode"], v["tile"]] for k, v in singles.items()}},
            "speedup": vb / vp, "h_rel_l2_max_vs_f64": l2, "h_rel_linf_max_vs_f64": li,
            "h_rel_l2_vs_oracle_shortest4_c48": vs_oracle}


def form_serving(dev, depth, count):
    """Serving sample: the first ``count`` requests of the Poisson stream
    (C48 0.4, C96 0.35, C192 0.2, C384 0.05; substeps log-uniform in
    [100, 5000]), float32, served in real time on one GPU with continuous
    batching (rounds of 200 substeps, admission by an HBM budget of half the
    free memory) and by the FIFO one-at-a-time plain path.  At the stream's
    200 requests/s the GPU is overloaded (the offered work exceeds its
    throughput several times), so the run is also repeated at 20 requests/s;
    at 200/s continuous batching is shown with arrival-order and with
    shortest-first admission."""
    import torch
    from licom4py_gpu_b200.ensemble import Geometry
    from licom4py_gpu_b200.serving import BarotropicServer, Request, poisson_mix, run_fifo
    import multiprocessing as mp
    geo = Geometry(depth, device=dev)
    for n in (48, 96, 192, 384):
        geo.plan(n, torch.float32)
        geo.dtb(n)
    keep = ("p50_s", "p99_s", "mean_s", "max_s", "requests", "wall_s", "cell_updates_per_s")
    # part of the CPU-baseline leg: the float64 oracle runs the 8 smallest requests of
    # the stream in a spawned host process while the GPU serves
    smallest = sorted(poisson_mix(count=count, rate=200.0, seed=0), key=lambda r: r.cell_updates)[:8]
    pool = mp.get_context("spawn").Pool(1)
    oracle_job = pool.apply_async(_oracle_requests, (depth, [(r.n, r.nsub, r.seed, r.amplitude)
                                                             for r in smallest]))
    out = {}
    first = None
    for rate, orders in ((200.0, ("fifo", "shortest")), (20.0, ("fifo",))):
        tag = f"rate_{int(rate)}"
        res = {"offered_cell_updates_per_s": None}
        for order in orders:
            reqs = poisson_mix(count=count, rate=rate, seed=0)
            srv = BarotropicServer(geo, dtype=torch.float32, round_substeps=200, order=order)
            for n in (48, 96, 192, 384):
                srv.basis._get(n)
            torch.cuda.synchronize()
            st = srv.run(reqs, realtime=True)
            srv.close()
            res[f"continuous_batching_{order}"] = {k: st[k] for k in keep + ("rounds",)}
            res["offered_cell_updates_per_s"] = sum(r.cell_updates for r in reqs) / max(reqs[-1].arrival, 1e-9)
            if first is None:
                first = reqs
        reqs_f = poisson_mix(count=count, rate=rate, seed=0)
        sf = run_fifo(geo, reqs_f, dtype=torch.float32, realtime=True)
        res["fifo_plain"] = {k: sf[k] for k in keep}
        res["throughput_ratio_fifo_order"] = (res["continuous_batching_fifo"]["cell_updates_per_s"] /
                                              sf["cell_updates_per_s"])
        if rate == 200.0:
            same = max(float(np.abs(a.result["h0"] - b.result["h0"]).max() / np.abs(b.result["h0"]).max())
                       for a, b in zip(first, reqs_f))
            res["same_result_alone_vs_mix_h_rel_max"] = same
        out[tag] = res
    # float64 check of the smallest requests (each alone, float64)
    small = sorted(first, key=lambda r: r.cell_updates)[:8]
    ref = [Request(rid=r.rid, n=r.n, nsub=r.nsub, seed=r.seed) for r in small]
    run_fifo(geo, ref, dtype=torch.float64, realtime=False)
    err64 = max(float(np.linalg.norm(a.result["h0"][:, 3:-3, 3:-3] - b.result["h0"][:, 3:-3, 3:-3]) /
                      np.linalg.norm(b.result["h0"][:, 3:-3, 3:-3])) for a, b in zip(small, ref))
    geo.close()
    out["workload"] = (f"first {count} requests of the 10k-request Poisson stream (seed 0), at 200 and at "
                       f"20 requests/s, float32, RK2")
    out["h_rel_l2_vs_f64_smallest8"] = err64
    try:
        want = oracle_job.get(timeout=900)
        served = {r.rid: r for r in first}
        out["h_rel_l2_vs_oracle_smallest8"] = max(
            float(np.linalg.norm(served[r.rid].result["h0"][:, 3:-3, 3:-3] - w[:, 3:-3, 3:-3]) /
                  np.linalg.norm(w[:, 3:-3, 3:-3])) for r, w in zip(smallest, want))
    except Exception as e:  # a report, not a failure of the bench
        out["h_rel_l2_vs_oracle_smallest8"] = f"oracle run did not finish: {type(e).__name__}"
    finally:
        pool.terminate()
    return out


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import torch
    from licom4py_gpu_b200 import barotr
    from licom4py_gpu_b200.plan import DIAG_NAMES, BtPlan
    from licom4py_gpu_b200.autotune import choose_config

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    grid, consts, st, dtb = build_problem(args.n, args.depth, args.seed + rank)
    # the oracle's run of the same full round, in a spawned host process meanwhile
    oracle = (OracleCheck(args.n, args.depth, args.seed, args.nbb)
              if rank == 0 and world == 1 and not args.no_oracle_check else None)
    checked = {}
    n, m, nbb = args.n, args.n + 6, args.nbb
    cells = 6 * n * n

    def dev_state(dtype):
        h = torch.from_numpy(st["h0"]).to(dev, dtype)
        u = torch.from_numpy(st["ub"]).to(dev, dtype)
        v = torch.from_numpy(st["vb"]).to(dev, dtype)
        return [h, h, u, v, u, v]

    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def timed_rounds(plan, ins, out, steps, warmup, kernel_timing=False, dtb_=None):
        dtb_ = dtb if dtb_ is None else dtb_  # the grid's own CFL step
        for _ in range(warmup):
            plan.round(*ins, nbb=nbb, dtb=dtb_, out=out)
        torch.cuda.synchronize()
        if kernel_timing:
            plan.enable_kernel_timing(True)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        barrier(world)
        torch.cuda.synchronize()
        for k in range(steps):
            flush.fill_(float(k))
            ev[k][0].record()
            plan.round(*ins, nbb=nbb, dtb=dtb_, out=out)
            ev[k][1].record()
        torch.cuda.synchronize()
        barrier(world)
        ms = sum(a.elapsed_time(b) for a, b in ev)
        kt = plan.kernel_time() if kernel_timing else (0.0, 0)
        if kernel_timing:
            plan.enable_kernel_timing(False)
        return ms, kt

    def make_plan(dtype, mode, tile):
        p = BtPlan(consts, dtype=dtype, device=dev, tile=tile, mode=mode)
        return p

    # configuration: autotuned (mode, tile) unless given
    cfg = choose_config(n, torch.float64, consts=consts, device=dev) if (args.mode == "auto" or args.tile == "auto") else None
    mode = cfg["mode"] if args.mode == "auto" else args.mode
    tile = tuple(cfg["tile"]) if args.tile == "auto" else tuple(int(x) for x in args.tile.split("x"))

    ins64 = dev_state(torch.float64)
    plan = make_plan(torch.float64, mode, tile)
    out = {k: plan.empty_field() for k in ("h0", "ub", "vb") + DIAG_NAMES}
    sampler = ClockSampler(local)
    with sampler:
        ms, (kms, klaunch) = timed_rounds(plan, ins64, out, args.steps, args.warmup,
                                          kernel_timing=(mode in ("persistent", "resident")))
    clocks = sampler.summary()
    ms = max_over_ranks(ms, world)
    ms_per_step = ms / args.steps
    value = world * cells * nbb * args.steps / (ms * 1e-3)
    launches_per_step = {"resident": 4, "persistent": 4, "graph": 4 * nbb + 3, "stream": 4 * nbb + 3}[mode]

    # roofline of the dominant kernel
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0

    def kernel_roofline(nn, dtype, tile_, nbb_, consts_, st_, dtb_):
        """Events around every phase kernel (stream mode, same stream) over one round."""
        p = BtPlan(consts_, dtype=dtype, device=dev, tile=tile_, mode="stream")
        h = torch.from_numpy(st_["h0"]).to(dev, dtype)
        u = torch.from_numpy(st_["ub"]).to(dev, dtype)
        v = torch.from_numpy(st_["vb"]).to(dev, dtype)
        o = {k: p.empty_field() for k in ("h0", "ub", "vb") + DIAG_NAMES}
        p.round(h, h, u, v, u, v, nbb=min(nbb_, 50), dtb=dtb_, out=o)
        p.enable_kernel_timing(True)
        flush.fill_(0.0)
        p.round(h, h, u, v, u, v, nbb=nbb_, dtb=dtb_, out=o)
        torch.cuda.synchronize()
        res = {k: p.kernel_time(k) for k in ("phase_h", "phase_uv")}
        fp = dict(zip(("phase_h", "phase_uv"), p.full_tile_kernels))  # which build of each kernel ran
        p.close()
        tot = sum(ms for ms, _ in res.values())
        dom = max(res, key=lambda k: res[k][0])
        ms, nl = res[dom]
        esz = 8 if dtype == torch.float64 else 4
        alg = KERNEL_WORDS[dom] * esz * 6 * nn * nn
        achieved = alg / (ms / nl * 1e-3) / 1e9
        traffic = None
        tfile = os.path.join(ROOT, "profiles", f"{KERNEL_NAMES[dom]}_c{nn}_{'f64' if esz == 8 else 'f32'}.json")
        if os.path.exists(tfile):
            try:
                traffic = json.load(open(tfile)).get("dram_bytes_per_launch")
            except (OSError, ValueError):
                traffic = None
        return {"bound": "hbm", "kernel": f"{KERNEL_NAMES[dom]}<{'double' if esz == 8 else 'float'},"
                                          f"{tile_[0]},{tile_[1]},{'true' if fp[dom] else 'false'}>",
                "achieved": achieved, "peak": peak, "peak_source": peak_src, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "launch_us": 1e3 * ms / nl,
                "alg_bytes_per_launch": alg, "launches_timed": nl,
                "share_of_phase_time": {k: res[k][0] / tot for k in res}}

    if mode in ("resident", "persistent") and klaunch > 0:
        # the round is one kernel: its event-timed launches in the headline run itself
        alg = B_ALG_WORDS * 8 * cells * nbb
        achieved = alg / (kms / klaunch * 1e-3) / 1e9
        l2 = l2_copy_gbs(dev)
        kname = "k_resident" if mode == "resident" else "k_round"
        traffic = None
        tfile = os.path.join(ROOT, "profiles", f"{kname}_c{n}_f64.json")
        if os.path.exists(tfile):
            try:
                traffic = json.load(open(tfile)).get("dram_bytes_per_launch")
            except (OSError, ValueError):
                traffic = None
        roofline = {"bound": "l2" if 41 * 8 * 6 * (n + 6) ** 2 < 64e6 else "hbm",
                    "kernel": f"{kname}<double,{tile[0]},{tile[1]}>", "achieved": achieved, "peak": peak,
                    "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                    "launch_us": 1e3 * kms / klaunch, "launches_timed": klaunch, "launches_per_step": 1,
                    "alg_bytes_per_launch": alg, "timed_in": "headline run (events around the round kernel)",
                    "l2_copy_gbs": l2, "frac_of_l2_copy": achieved / l2 if l2 else None}
    else:
        # graph / stream: the kernels' shares of phase time come from an event-timed stream-mode
        # pass (events around every launch remove the overlap of programmatic launch, so those
        # isolated launch times are upper bounds); the per-launch time of the headline run is the
        # dominant kernel's share of the headline step over its launches per step
        iso = kernel_roofline(n, torch.float64, tile, nbb, consts, st, dtb)
        dom = "phase_h" if iso["kernel"].startswith("k_phase_h") else "phase_uv"
        share = iso["share_of_phase_time"][dom]
        per_step = 2 * nbb  # launches of each phase kernel per RK2 round
        launch_us = 1e3 * ms_per_step * share / per_step
        achieved = iso["alg_bytes_per_launch"] / (launch_us * 1e-6) / 1e9
        l2 = l2_copy_gbs(dev)
        roofline = {"bound": "l2" if 41 * 8 * 6 * (n + 6) ** 2 < 64e6 else "hbm", "kernel": iso["kernel"],
                    "achieved": achieved, "peak": peak, "peak_source": peak_src, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": iso["traffic"], "launch_us": launch_us,
                    "launches_per_step": per_step, "alg_bytes_per_launch": iso["alg_bytes_per_launch"],
                    "timed_in": "headline run: share of phase time x ms_per_step / launches per step",
                    "share_of_phase_time": iso["share_of_phase_time"],
                    "isolated_launch_us": iso["launch_us"], "isolated_frac": iso["frac"],
                    "l2_copy_gbs": l2, "frac_of_l2_copy": achieved / l2 if l2 else None}
    round_roofline = {"achieved": B_ALG_WORDS * 8 * cells * nbb / (ms_per_step * 1e-3) / 1e9,
                      "peak": peak, "unit": "GB/s",
                      "frac": B_ALG_WORDS * 8 * cells * nbb / (ms_per_step * 1e-3) / 1e9 / peak,
                      "bytes_per_cell_update": B_ALG_WORDS * 8}

    # end to end through the public call, host (pinned) buffers
    pinned_in = [torch.from_numpy(a).pin_memory() for a in (st["h0"], st["h0"], st["ub"], st["vb"], st["ub"], st["vb"])]
    dev_in = [torch.empty((6, m, m), dtype=torch.float64, device=dev) for _ in range(6)]
    pinned_out = [torch.empty((6, m, m), dtype=torch.float64).pin_memory() for _ in range(13)]
    zeros = [torch.zeros((6, m, m), dtype=torch.float64, device=dev) for _ in range(17)]
    core_plan = barotr.get_plan(consts, dtype=torch.float64, device=dev)
    core_plan.set_mode(mode)
    core_plan.set_tile(*tile)

    def e2e_step():
        for d, h in zip(dev_in, pinned_in):
            d.copy_(h, non_blocking=True)
        state = tuple(dev_in) + tuple(zeros)
        res = barotr._barotr_rk2_core(state, consts, nbb, dtb, 1, 1)
        outs = [res[0], res[2], res[3]] + list(res[6:16])
        for h, d in zip(pinned_out, outs):
            h.copy_(d, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        e2e_step()
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    e2e = {"value": world * cells * nbb * args.steps / (e2e_ms * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": sum(t.numel() * t.element_size() for t in pinned_in),
           "d2h_bytes_per_step": sum(t.numel() * t.element_size() for t in pinned_out),
           "ms_per_step": e2e_ms / args.steps}

    extras = {}
    if not args.no_extras:
        # float32 precision form, same workload
        ins32 = dev_state(torch.float32)
        p32 = make_plan(torch.float32, mode, tile)
        out32 = {k: p32.empty_field() for k in ("h0", "ub", "vb") + DIAG_NAMES}
        ms32, _ = timed_rounds(p32, ins32, out32, args.steps, args.warmup)
        checked["f32"] = out32
        ms32 = max_over_ranks(ms32, world)
        h64 = out["h0"][:, 3:-3, 3:-3]
        h32 = out32["h0"][:, 3:-3, 3:-3].double()
        extras["fp32"] = {"value": world * cells * nbb * args.steps / (ms32 * 1e-3), "unit": UNIT,
                          "ms_per_step": ms32 / args.steps,
                          "h_rel_l2_vs_f64": float((h32 - h64).norm() / h64.norm())}
        p32.close()
        # round execution modes (CUDA graph vs persistent vs stream), float64
        modes = {}
        for md in ("resident", "persistent", "graph", "stream"):
            pm = make_plan(torch.float64, md, tile)
            steps = max(2, args.steps // 2)
            msm, _ = timed_rounds(pm, ins64, out, steps, 2)
            modes[md] = {"value": cells * nbb * steps / (msm * 1e-3), "ms_per_step": msm / steps}
            pm.close()
        extras["modes_f64"] = modes
        # the HBM-bound size: C384 rounds (float64 and float32), graph mode, tuned tile
        g384, c384, s384, d384 = build_problem(384, args.depth, args.seed)
        big = {}
        for dt_, tag in ((torch.float64, "f64"), (torch.float32, "f32")):
            cfg384 = choose_config(384, dt_, consts=c384, device=dev)
            t384 = tuple(cfg384["tile"])
            p = BtPlan(c384, dtype=dt_, device=dev, tile=t384, mode="graph")
            hh = torch.from_numpy(s384["h0"]).to(dev, dt_)
            uu = torch.from_numpy(s384["ub"]).to(dev, dt_)
            vv = torch.from_numpy(s384["vb"]).to(dev, dt_)
            ins384 = [hh, hh, uu, vv, uu, vv]
            o384 = {k: p.empty_field() for k in ("h0", "ub", "vb") + DIAG_NAMES}
            msb, _ = timed_rounds(p, ins384, o384, 3, 2, dtb_=d384)
            p.close()
            cu = 6 * 384 * 384 * nbb * 3 / (msb * 1e-3)
            esz = 8 if tag == "f64" else 4
            big[tag] = {"value": cu, "unit": UNIT, "ms_per_step": msb / 3, "tile": list(t384),
                        "round_frac_of_hbm": cu * B_ALG_WORDS * esz / 1e9 / peak,
                        "kernel": kernel_roofline(384, dt_, t384, 100, c384, s384, d384)}
        extras["c384"] = big

    if not args.no_forms and world == 1:
        extras["precision_c384"] = form_precision(dev, args.depth, peak)
        extras["ensemble"] = form_ensemble(dev, args.depth)
        extras["serving"] = form_serving(dev, args.depth, args.serving_requests)

    if oracle is not None:  # first, so that the oracle's process is done before the CPU timing
        checked["f64"] = out
        extras["error_vs_oracle"] = oracle.compare(checked)
    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_baseline_all_cores(args)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic: seeded spherical harmonics l=1..8 (h 1 m RMS, u/v 0.3 m/s RMS) over H=5000 m",
                "config": {"workload": f"C{n} plain drop-in RK2 round, {nbb} substeps per step, float64",
                           "n": n, "nbb": nbb, "rk": 2, "dtb_s": dtb, "mode": mode, "tile": list(tile),
                           "geometry": {f"C{k}": v for k, v in GEOMETRY_CACHE.items()},
                           "parallelism": f"replicas x{world}",
                           "l2": "flushed between steps (512 MiB write outside the timed windows); "
                                 "within a step the member's working set stays L2-resident"},
                "roofline": roofline, "round_roofline": round_roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches_per_step * args.steps, "clocks": clocks}
        line.update(extras)
        print(json.dumps(line), flush=True)
    plan.close()


def run_form(args):
    """One layered form alone (N = 1), e.g. the serving stream at its configured size."""
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs") or 6650.0
    if args.only_form == "precision":
        res = form_precision(dev, args.depth, peak)
    elif args.only_form == "ensemble":
        res = form_ensemble(dev, args.depth)
    else:
        res = form_serving(dev, args.depth, args.serving_requests)
    print(json.dumps({"form": args.only_form, "n_gpus": 1, **res}), flush=True)


def main():
    args = parse_args()
    if args.case_only:
        run_case(args)
        return
    if args.only_form:
        run_form(args)
        return
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        from licom4py_gpu_b200 import replicas
        replicas.teardown()


if __name__ == "__main__":
    main()
