"""Benchmark of the B200 dynamical core (one JSON line on rank 0).

A "step" is one pass of model_driver's time loop (driver_code.f90:304-676):
means + divergence, sources + Poisson rhs, the BiCGSTAB pressure solve, the
MPDATA advection of theta and the leap-frog momentum update, on seeded
synthetic fields of the 256 x 256 x 128 dry warm bubble (dx = dy = dz = 50 m,
dt = 1 s, kord = 3 monotone, ptol = 1e-10).  The timed steps are steps 1..K
of the run from the initial state (a warm-up run of W steps precedes them on
the same handle, then the initial state is uploaded again), so every arm
times the same time steps with the same solver iteration counts.

The headline `value` is the mixed-precision form (FP32 fields and BiCGSTAB
iterations, FP64 pressure, residual and dot products); the plain FP64 path
is timed on the same steps (`fp64`), and the per-field max / RMS errors of
the mixed form against the FP64 path after 1, 10 and --accuracy-steps steps
go in `accuracy_vs_fp64`.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
    python bench.py --run-case --case NAME --steps K [--precision 0|1] ...

The compact JSON line keeps the headline figures (mixed form, FP64 path,
speed-up, accuracy after --accuracy-steps, roofline, CPU baseline,
end-to-end); the long-form record (per-class kernel times, step models,
accuracy tables) goes to the file --details names (bench_details.json).
--run-case prints one line per step of a named case (profiling driver).

N > 1 (torchrun, one process per GPU): the single domain does not shard
(whole domain on one GPU), so each rank advances its own replica of the
workload ("replicas only"); value = all ranks' grid-point steps / max time.
--impl reference times the CPU restatement of the reference (oracle/, the
reference Fortran cannot be compiled here) on the host cores, rank 0 only.
"""
import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "dynamical-cloud-model_b200")
METRIC = "grid-pt-steps/s at 256x256x128: FP32+FP64-refine vs FP64 GPU at <=1e-6 rel err"


def metric_of(case):
    if case.name == "warm_bubble_256x256x128":
        return METRIC
    return "grid-pt-steps/s of %s (mixed precision, FP64 path beside it)" % case.name
PEAK_FALLBACK_GBS = 6650.0


def load_pkg():
    if "dcm_b200" in sys.modules:
        return sys.modules["dcm_b200"]
    spec = importlib.util.spec_from_file_location(
        "dcm_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dcm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return PEAK_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# algorithmic field passes per launch of each kernel class (reads + writes of
# an N-point field; stencil neighbours come from cache).  Jacobi sweeps:
# B1 3, B2 4, B3 5, C1 3, C2 4, C3 4 -> 23/6; matvecs: B4 (p, cr -> v1, vh) 4,
# C4 (cs, r, v1 -> t) 4; update (x p cs r v1 t cr -> x r rh) 10.  Other
# classes per launch at this configuration.
PASSES = {"jacobi": 23.0 / 6.0, "matvec": 4.0, "update": 10.0, "setup": 4.0,
          "means": 5.0, "sources": 7.0, "rhs": 4.0, "adv_ref": 3.0, "mp_shift": 1.0,
          "upwind": 5.0, "antidiff": 7.0, "beta": 7.0, "limit": 8.0, "momentum": 16.0}
# field passes of one BiCGSTAB iteration and of the rest of a step
ITER_PASSES = 41.0
STEP_PASSES = 60.0
# the reference's own algebra per iteration (dynamics.f90:391-423, every
# field pass the statements make, no stored quotients): the algorithmic
# model both forms' step_frac_algorithm count against
REF_ITER_PASSES = 39.0
# With the fused preconditioner (FP32) one "jacobi" launch applies all three
# sweeps of a phase: it reads r/a_p, v1/a_p (and old p) and writes p or cs,
# 4 passes in phase B and 3 in phase C; the iteration then moves 7 + 8 + 10 =
# 25 passes.  The three separate sweeps it replaces move 12 and 11.
FUSED_JACOBI_PASSES = 3.5
FUSED_REPLACED_PASSES = 11.5
FUSED_ITER_PASSES = 25.0
# With phase C's matvec as the fused kernel's fourth stage (launch shape
# fuse = 2) phase C's launch also reads r, v1 and writes t (6 passes moved;
# it replaces 11 + 4 = 15 algorithmic passes): per launch 5 moved and 13.5
# replaced on average, 24 passes per iteration.
FUSED_MV = {"jacobi": 5.0, "replaced": 13.5, "iter": 24.0}


def make_case(pkg, name):
    from dcm_b200 import cases
    if name == "warm_bubble":
        return cases.warm_bubble()
    if name == "kelvin_helmholtz":
        return cases.kelvin_helmholtz()
    if name.startswith("warm_bubble_"):
        ip, jp, kp = (int(x) for x in name.split("_")[-1].split("x"))
        return cases.warm_bubble(ip=ip, jp=jp, kp=kp)
    if name == "sheared_convection":
        return cases.sheared_convection()
    if name.startswith("sheared_convection_"):
        ip, jp, kp = (int(x) for x in name.split("_")[-1].split("x"))
        return cases.sheared_convection(ip=ip, jp=jp, kp=kp)
    raise SystemExit("unknown case " + name)


def pinned_like(a):
    """A pinned host copy of a Fortran-ordered field (page-locked through
    torch's caching host allocator), for the end-to-end copies."""
    import torch
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    v = t.numpy().reshape(a.shape[::-1]).transpose()
    v[...] = a
    return v, t


class Ranks:
    """The ranks of a torchrun launch (or one process): barrier and max / sum
    reductions of host scalars over the process group (NCCL on GPUs, gloo in
    the CPU tests)."""

    def __init__(self, dist=None):
        self.dist = dist
        self.rank = dist.get_rank() if dist is not None else 0
        self.world = dist.get_world_size() if dist is not None else 1

    def _device(self):
        return "cuda" if self.dist.get_backend() == "nccl" else "cpu"

    def barrier(self):
        if self.dist is not None:
            if self._device() == "cuda":
                import torch
                torch.cuda.synchronize()
            self.dist.barrier()

    def _reduce(self, x, op):
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, x):
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)


def partition(items, rank, world):
    """Ensemble members of one rank: every world-th member from `rank`
    (members are independent, so no data-path collective)."""
    return items[rank::world]


def live_mask_p(g):
    """Cells of p the reference computes and later reads (all but the halo
    rings of the top/bottom rows and the vertical halo edges)."""
    m = np.ones((g.kp + 2, g.jp + 2, g.ip + 2), dtype=bool, order="F")
    jh = np.zeros(g.jp + 2, dtype=bool)
    jh[[0, g.jp + 1]] = True
    ih = np.zeros(g.ip + 2, dtype=bool)
    ih[[0, g.ip + 1]] = True
    ring = jh[:, None] | ih[None, :]
    m[0][ring] = False
    m[g.kp + 1][ring] = False
    m[1:g.kp + 1][:, jh[:, None] & ih[None, :]] = False
    return m


def field_errors(g, ref, got):
    """Per-field max and RMS error of `got` relative to max|ref|.  p is
    compared on its live cells with each field's mean removed: the pressure
    equation is singular (Neumann / periodic), p is defined up to a constant
    and only its gradient enters the momentum update."""
    out = {}
    for n in ("u", "v", "w", "th", "p"):
        a, b = np.asarray(got[n]), np.asarray(ref[n])
        if n == "p":
            m = live_mask_p(g)
            a, b = a[m] - a[m].mean(), b[m] - b[m].mean()
        den = float(np.max(np.abs(b))) or 1.0
        d = a - b
        out[n] = {"max": float(np.max(np.abs(d)) / den),
                  "rms": float(np.sqrt(np.mean(d * d)) / den)}
    return out


def bench_config(case, args):
    """The workload of a bench line, the same dict in both arms (the GPU
    arm's mixed form and FP64 path and the reference arm's CPU restatement
    advance the same seeded case over the same time steps)."""
    g = case.grid
    mb = (g.ip + 2) * (g.jp + 2) * (g.kp + 2) * 8 / 1e6
    return {"workload": "%s: steps 1..%d from the seeded initial state" % (case.name, args.steps),
            "grid": "%dx%dx%d" % (g.ip, g.jp, g.kp), "dt": case.dt, "kord": case.kord,
            "monotone": bool(case.monotone), "ptol": case.ptol,
            "tracers": int(case.nq or 0),
            "l2": ("inputs larger than L2: one FP64 field is %.1f MB and a step streams "
                   "about 40 resident fields" % mb) if 40 * mb > 126 else
                  ("resident state (about 40 FP64 fields of %.2f MB) fits in the 126 MB "
                   "L2" % mb)}


def compact(obj, keep=("value", "ms_per_step")):
    """Floats to 4 significant digits (except the top-level `keep` keys), so
    that the JSON line stays short."""
    def r(o, top=False):
        if isinstance(o, dict):
            return {k: (v if top and k in keep else r(v)) for k, v in o.items()}
        if isinstance(o, list):
            return [r(v) for v in o]
        if isinstance(o, float):
            return float("%.4g" % o)
        return o
    return r(obj, True)


def write_details(d, name):
    """The long-form record (per-class kernel times, accuracy tables, step
    models, notes) beside the compact JSON line, at `name` (relative to the
    repository root); returns its path."""
    path = os.path.join(ROOT, name)
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(d, f, indent=1)
        return os.path.relpath(path, ROOT)
    except OSError:
        return None


def run_b200(args, rank, world, local_rank, dist):
    pkg = load_pkg()
    case = make_case(pkg, args.case)
    g = case.grid
    N = g.npoints
    core = pkg.DynamicalCore(g, device=local_rank)
    if args.host_loop:
        core.solver_graphs(False)
    kw = dict(ptol=case.ptol, kord=case.kord, monotone=case.monotone)
    if case.nq:
        kw.update(nq=case.nq, c_s=case.c_s, c_e=case.c_e)
    peak, peak_kind = peaks()

    # the mixed form's FP32 iterations use Chebyshev-weighted Jacobi sweeps
    # (same three sweeps, fewer iterations); FP64 keeps the reference's
    PRECOND = dict(precond=1, precond_lo=0.05)

    def fresh(prec, precond=None):
        pc = (PRECOND if prec == 1 else {}) if precond is None else precond
        core.upload_state(case.state, case.dt, precision=prec, **kw, **pc)
        core.driver_start()

    R = Ranks(dist)
    barrier, max_over_ranks = R.barrier, R.max

    def measure(prec, precond=None):
        """Steps 1..K of one precision: device time (CUDA events on the
        library stream, max over ranks), launches, clocks, then the same
        steps again with per-kernel-class events for the roofline.  The
        solver launch shape is the autotuner's for this grid (cached)."""
        shape = core.tune(precision=prec, use_cache=True)
        fresh(prec, precond)  # warm-up run (allocations, first launches)
        if args.warmup:
            core.step(args.warmup)
        fresh(prec, precond)
        core.profile(False)  # reset the launch counters, event timing off
        clocks = ClockSampler(local_rank)
        barrier()
        clocks.start()
        st = core.step(args.steps)
        clk = clocks.stop()
        barrier()
        ms = max_over_ranks(st.ms_total)
        launches = sum(c for _, c in core.profile_read().values())
        fresh(prec, precond)
        core.profile(True)
        core.step(args.steps)
        prof = core.profile_read()
        core.profile(False)
        classes = {k: v for k, v in prof.items() if v[1] > 0}
        return dict(ms=ms, iters=st.iters_total, launches=launches, clocks=clk,
                    classes=classes, value=world * N * args.steps / (ms / 1e3),
                    shape={"warps_per_sweep_block": shape[0], "tasks_per_warp": shape[1],
                           "march_depth": shape[2], "fused_preconditioner": shape[3],
                           "levels_per_lane": shape[4]})

    m32 = measure(1)
    m32ref = measure(1, precond={})  # mixed form with the reference's sweeps
    m64 = measure(0)

    # roofline of the dominant kernel class of the headline (mixed) form
    w32 = 4.0
    classes = m32["classes"]
    dom = max(classes, key=lambda k: classes[k][0])
    dom_ms, dom_n = classes[dom]
    fuse_level = int(m32["shape"]["fused_preconditioner"])
    fused = fuse_level > 0
    f_jac, f_rep, f_iter = ((FUSED_MV["jacobi"], FUSED_MV["replaced"], FUSED_MV["iter"])
                            if fuse_level == 2 else
                            (FUSED_JACOBI_PASSES, FUSED_REPLACED_PASSES, FUSED_ITER_PASSES))
    dom_passes = f_jac if (fused and dom == "jacobi") else PASSES.get(dom, 0.0)
    dom_bytes = dom_passes * N * w32
    dom_s = dom_ms / dom_n / 1e3 if dom_n else None
    # algorithmic bytes of one launch by the operator-fused model: a fused
    # preconditioner launch applies the three sweeps of a phase (11.5 passes
    # averaged over phases B and C)
    dom_bytes_alg = (f_rep * N * w32 if (fused and dom == "jacobi")
                     else dom_bytes)
    achieved_alg = dom_bytes_alg / dom_s / 1e9 if dom_n else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tr = json.load(f).get(case.name, {}).get("fp32", {})
        if not (dom == "jacobi" and fuse_level == 2):  # not captured for the fourth stage
            traffic = tr.get("jacobi_fused" if (fused and dom == "jacobi") else dom)

    def step_model(m, w, iter_passes):
        it = m["iters"] / args.steps
        b = (STEP_PASSES + iter_passes * it) * N * w
        gbs = b / (m["ms"] / args.steps / 1e3) / 1e9
        return {"bytes_per_step": b, "GBs": gbs, "frac": gbs / peak, "iters_per_step": it,
                "passes_per_iteration": iter_passes}

    # ---- accuracy: mixed against the FP64 path after the timed steps and
    #      after args.accuracy_steps
    acc = {}
    if args.accuracy_steps:
        # the FP64 run on a second handle, the mixed one on this handle, which
        # the end-to-end leg below uses next with the same layout
        cores = [pkg.DynamicalCore(g, device=local_rank), core]
        for prec, c in zip((0, 1), cores):
            c.upload_state(case.state, case.dt, precision=prec, **kw,
                           **(PRECOND if prec == 1 else {}))
            c.driver_start()
        done = 0
        for n in sorted({1, 10, args.accuracy_steps}):
            for c in cores:
                c.step(n - done)
            done = n
            acc[str(n)] = field_errors(g, cores[0].download_state(), cores[1].download_state())
        cores[0].close()

    # ---- end to end through the C-ABI with host buffers (pinned), mixed form
    host = {n: pinned_like(getattr(case.state, n)) for n in
            ("u", "v", "w", "zu", "zv", "zw", "tu", "tv", "tw", "th", "p")}
    st_host = case.state.copy()
    for n, (v, _) in host.items():
        setattr(st_host, n, v)
    # the result lands in pinned host buffers too (allocated before timing)
    zero = np.zeros(g.shape, order="F")
    dest = {n: pinned_like(zero) for n in ("u", "v", "w", "zu", "zv", "zw", "tu", "tv", "tw",
                                           "th", "p", "su", "sv", "sw", "psrc", "div", "sth")}
    outbufs = {n: v for n, (v, _) in dest.items()}
    barrier()
    t0 = time.perf_counter()
    core.upload_state(st_host, case.dt, precision=1, **kw, **PRECOND)
    core.driver_start()
    tu = time.perf_counter()
    core.step(args.steps)
    ts = time.perf_counter()
    out = core.download_state(out=outbufs)
    t1 = time.perf_counter()
    barrier()
    e2e_s = max_over_ranks(t1 - t0)
    field_bytes = g.shape[0] * g.shape[1] * g.shape[2] * 8
    h2d = 11 * field_bytes  # the 9 velocities, th and p (work fields start at zero)
    d2h = sum(a.nbytes for a in out.values() if isinstance(a, np.ndarray))
    e2e = {"value": world * N * args.steps / e2e_s, "unit": "grid-pt-steps/s",
           "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
           "host_ms": {"upload": (tu - t0) * 1e3, "steps": (ts - tu) * 1e3,
                       "download": (t1 - ts) * 1e3},
           "note": "mixed form: upload of the FP64 host state, K steps, download of the "
                   "state, per K-step call, on a handle whose device buffers an earlier "
                   "upload of the same layout allocated"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, case, min(args.cpu_steps, args.steps))
    core.close()
    if rank != 0:
        return None
    extra = other_configs(args, local_rank) if (world == 1 and not args.no_extra) else None
    sm32 = step_model(m32, w32, f_iter if fused else ITER_PASSES)
    sm64 = step_model(m64, 8.0, ITER_PASSES)
    acc_last = acc.get(str(args.accuracy_steps), {})
    details = {
        "fp64": {"tuned_launch_shape": m64["shape"], "gpu_launches": m64["launches"],
                 "clocks": m64["clocks"], "step_model": sm64,
                 "kernel_ms": {k: round(v[0], 3) for k, v in m64["classes"].items()}},
        "mixed": {"tuned_launch_shape": m32["shape"], "step_model": sm32,
                  "step_model_unfused_algorithm": step_model(m32, w32, ITER_PASSES),
                  "kernel_ms": {k: round(v[0], 3) for k, v in classes.items()},
                  "kernel_launches": {k: v[1] for k, v in classes.items()}},
        "mixed_reference_sweeps": {
            "value": m32ref["value"], "ms_per_step": m32ref["ms"] / args.steps,
            "bicgstab_iters_per_step": m32ref["iters"] / args.steps,
            "speedup_vs_fp64": m32ref["value"] / m64["value"],
            "note": "the mixed form with the reference's unweighted Jacobi sweeps: the part "
                    "of the speed-up that FP32 alone gives"},
        "accuracy_vs_fp64": acc,
        "roofline_note": "achieved = the algorithmic bytes of the three Jacobi sweeps one fused "
                         "launch applies (11.5 N-point FP32 passes, the operator-fused model) per "
                         "launch time; the fused kernel itself reads r/a_p, v1/a_p (and old p) "
                         "and writes p or cs, 3.5 passes, which min_bytes_frac counts",
        "e2e_host_ms": e2e.pop("host_ms"), "e2e_note": e2e.pop("note"),
        "preconditioner": "FP32 iterations: Chebyshev-weighted Jacobi sweeps (3 sweeps, "
                          "interval [0.05, 2]); FP64: the reference's 3 Jacobi sweeps",
    }
    min_bytes = f_jac * N * w32 if (fused and dom == "jacobi") else dom_bytes
    return {
        "metric": metric_of(case), "value": m32["value"], "unit": "grid-pt-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": m32["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded %s, numpy PCG64 seed %d)" % (case.name, case.seed),
        "fp64": {"value": m64["value"], "ms_per_step": m64["ms"] / args.steps,
                 "iters_per_step": m64["iters"] / args.steps, "step_frac": sm64["frac"],
                 "step_frac_algorithm": step_model(m64, 8.0, REF_ITER_PASSES)["frac"]},
        "speedup_vs_fp64": m32["value"] / m64["value"],
        "iters_per_step": m32["iters"] / args.steps, "step_frac": sm32["frac"],
        "step_frac_algorithm": step_model(m32, w32, REF_ITER_PASSES)["frac"],
        "accuracy_vs_fp64_steps": args.accuracy_steps,
        "accuracy_vs_fp64": {n: float("%.3g" % v["max"]) for n, v in acc_last.items()},
        "config": bench_config(case, args),
        "parallelism": "replicas" if world > 1 else "single GPU",
        "roofline": {"bound": "hbm", "kernel": dom + (" (fused preconditioner)" if fused else ""),
                     "achieved": achieved_alg, "peak": peak, "unit": "GB/s",
                     "frac": (achieved_alg / peak) if achieved_alg else None,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "bytes_per_launch": dom_bytes_alg, "launches": dom_n,
                     "avg_launch_us": dom_ms / dom_n * 1e3 if dom_n else None,
                     "min_bytes_frac": (min_bytes / dom_s / 1e9 / peak) if dom_n else None},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": m32["launches"],
        "clocks": {k: m32["clocks"].get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "other_configs": extra,
        "details": write_details(details, args.details),
    }


def other_configs(args, local_rank):
    """The benchmark's other configurations, one GPU, compactly: the
    128x1x64 shear layer (FP64, all 600 steps, beside the oracle on the host
    cores), the 512x512x256 sheared convection with 8 tracers (mixed form,
    steps 1..10), and the 64-member ensemble (steps 1..10, against the
    sequential per-member loop)."""
    pkg = load_pkg()
    from dcm_b200 import cases
    out = {}
    # config 1
    kh = cases.kelvin_helmholtz()
    core = pkg.DynamicalCore(kh.grid, device=local_rank)
    core.tune(precision=0, use_cache=True)
    kw = dict(ptol=kh.ptol, kord=kh.kord, monotone=kh.monotone)
    core.upload_state(kh.state, kh.dt, precision=0, **kw)
    core.driver_start()
    core.step(3)
    core.upload_state(kh.state, kh.dt, precision=0, **kw)
    core.driver_start()
    st = core.step(kh.nsteps)
    core.close()
    n1 = kh.grid.npoints
    c1 = {"workload": "%s FP64, steps 1..%d" % (kh.name, kh.nsteps),
          "value": n1 * kh.nsteps / (st.ms_total / 1e3), "ms_per_step": st.ms_total / kh.nsteps,
          "iters_per_step": st.iters_total / kh.nsteps}
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        oracle.set_threads(os.cpu_count() or 1, True)
        m = oracle.OracleModel(kh.grid, kh.state, kh.dt, **kw)
        m.driver_start()
        t0 = time.perf_counter()
        m.step(kh.nsteps)
        c1["oracle_value"] = n1 * kh.nsteps / (time.perf_counter() - t0)
        c1["oracle_cores"] = os.cpu_count() or 1
    out["1"] = c1
    # config 4
    sc = cases.sheared_convection()
    core = pkg.DynamicalCore(sc.grid, device=local_rank)
    core.tune(precision=1, use_cache=True)
    kw = dict(ptol=sc.ptol, kord=sc.kord, monotone=sc.monotone, nq=sc.nq, c_s=sc.c_s,
              c_e=sc.c_e, precision=1, precond=1, precond_lo=0.05)
    core.upload_state(sc.state, sc.dt, **kw)
    core.driver_start()
    core.step(2)
    core.upload_state(sc.state, sc.dt, **kw)
    core.driver_start()
    n4 = 10
    st = core.step(n4)
    core.close()
    out["4"] = {"workload": "%s mixed, 8 tracers, steps 1..%d" % (sc.name, n4),
                "value": sc.grid.npoints * n4 / (st.ms_total / 1e3),
                "ms_per_step": st.ms_total / n4, "iters_per_step": st.iters_total / n4}
    # config 5
    ea = argparse.Namespace(**vars(args))
    ea.steps, ea.warmup = 10, 3
    e = run_ensemble(ea, 0, 1, local_rank, None)
    out["5"] = {"workload": "%d-member ensemble mixed, steps 1..10" % args.members,
                "value": e["value"], "ms_per_step": e["ms_per_step"],
                "sequential_value": e["sequential"]["value"],
                "speedup_vs_sequential": e["speedup_vs_sequential"]}
    return out


def run_ensemble(args, rank, world, local_rank, dist):
    """Batched ensemble of seeded dry warm bubbles of uneven sizes (ip, jp
    from {64, 96, 128, 192}, kp from {48, 64, 96}, amplitude U(1, 3) K),
    mixed precision, solver launch shapes autotuned per grid shape.  Members
    are partitioned over ranks (no collective); each rank advances its
    members with one CUDA graph launch per step and, beside it, the same
    members one after another (sequential per-member loop)."""
    pkg = load_pkg()
    from dcm_b200 import cases
    spec = cases.ensemble_members(args.members)
    mine = partition(spec, rank, world)
    mcases = [cases.warm_bubble(ip=ip, jp=jp, kp=kp, amp=amp, seed=seed)
              for (ip, jp, kp, amp, seed) in mine]
    ens = pkg.Ensemble([c.grid for c in mcases], device=local_rank)
    shapes = {}
    for core, c in zip(ens.members, mcases):
        key = (c.grid.ip, c.grid.jp, c.grid.kp)
        shapes[key] = core.tune(precision=1, use_cache=True)
        if shapes[key] != core.tune(precision=1, use_cache=True):
            raise SystemExit("tuner cache is inconsistent")

    def fresh():
        for core, c in zip(ens.members, mcases):
            core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                              precision=1, precond=1, precond_lo=0.05)
            core.driver_start()

    R = Ranks(dist)
    barrier, max_over_ranks, sum_over_ranks = R.barrier, R.max, R.sum
    points = sum(c.grid.npoints for c in mcases)
    fresh()
    if args.warmup:
        ens.step(args.warmup)  # captures the three phase graphs
    fresh()
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    st = ens.step(args.steps)
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(st.ms_total)
    iters = st.iters_total
    # the same steps, one member after another
    fresh()
    for core in ens.members:
        if args.warmup:
            core.step(args.warmup)
    fresh()
    barrier()
    seq_ms = 0.0
    seq_iters = 0
    for core in ens.members:
        s2 = core.step(args.steps)
        seq_ms += s2.ms_total
        seq_iters += s2.iters_total
    barrier()
    seq_ms = max_over_ranks(seq_ms)
    total_points = sum_over_ranks(points)
    ens.close()
    if rank != 0:
        return None
    value = total_points * args.steps / (ms / 1e3)
    return {
        "metric": "aggregate grid-pt-steps/s of a %d-member warm-bubble ensemble" % args.members,
        "value": value, "unit": "grid-pt-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak" if world > 1 else "strong", "vs_baseline": None,
        "dtype": "f32+f64 (FP32 fields and BiCGSTAB, FP64 pressure, residual and dots)",
        "data": "synthetic (seeded warm bubbles, numpy PCG64 seeds 5000..5063)",
        "config": {"workload": "ensemble of %d dry warm bubbles, mixed precision" % args.members,
                   "members_per_rank": len(mine), "points_per_rank": points,
                   "grid_shapes": sorted(["%dx%dx%d" % k for k in shapes]),
                   "tuned_launch_shapes": {"%dx%dx%d" % k: list(v) for k, v in shapes.items()},
                   "timed_steps": "1..%d from the initial states" % args.steps,
                   "parallelism": "members partitioned over ranks" if world > 1 else
                   "single GPU"},
        "sequential": {"value": total_points * args.steps / (seq_ms / 1e3),
                       "ms_per_step": seq_ms / args.steps,
                       "note": "the same members, one dcm_step call after another"},
        "speedup_vs_sequential": seq_ms / ms,
        "bicgstab_iters": {"ensemble": iters, "sequential": seq_iters},
        "graph_launches": args.steps, "clocks": clk,
    }


def cpu_baseline(args, case, nsteps, budget=None, warmup=0):
    """The oracle (CPU restatement of the reference, not the reference
    binary: no Fortran compiler exists here) on all host cores, steps
    1..nsteps of the same case from its initial state, stopping early only
    past `budget` seconds.  warmup: untimed steps of the 128x1x64
    Kelvin-Helmholtz case first (thread pool and code paged in); the case's
    own arrays are first touched by the untimed set-up."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from dcm_b200 import cases
    cores = os.cpu_count() or 1
    oracle.set_threads(cores, True)
    if warmup:
        kh = cases.kelvin_helmholtz()
        w = oracle.OracleModel(kh.grid, kh.state, kh.dt, ptol=kh.ptol, kord=kh.kord,
                               monotone=kh.monotone)
        w.driver_start()
        w.step(warmup)
    m = oracle.OracleModel(case.grid, case.state, case.dt, ptol=case.ptol, kord=case.kord,
                           monotone=case.monotone)
    m.driver_start()
    budget = args.cpu_budget if budget is None else budget
    t0 = time.perf_counter()
    done = 0
    iters = 0
    while done < nsteps:
        it, _ = m.step(1)
        iters += it
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    return {"value": case.grid.npoints * done / dt, "unit": "grid-pt-steps/s", "cores": cores,
            "kind": "port", "steps_done": done, "ms_per_step": dt * 1e3 / done,
            "iters_per_step": iters / done,
            "sample": "%s steps 1..%d (%d BiCGSTAB iterations), FP64, %d OpenMP threads, "
                      "%.1f s" % (case.name, done, iters, cores, dt)}


def run_reference(args, rank, world):
    """The reference arm: the CPU restatement of the reference's FP64 time
    step (oracle/) on all host cores, timing steps 1..K of the GPU arm's
    workload from the same seeded initial state.  Rank 0 only."""
    if rank != 0:
        return None
    pkg = load_pkg()
    case = make_case(pkg, args.case)
    cpu = cpu_baseline(args, case, args.steps, budget=args.ref_budget, warmup=args.warmup)
    return {"impl": "reference", "metric": metric_of(case), "value": cpu["value"],
            "unit": "grid-pt-steps/s", "n_gpus": world, "steps": cpu["steps_done"],
            "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded %s, numpy PCG64 seed %d)" % (case.name, case.seed),
            "iters_per_step": cpu["iters_per_step"],
            "config": bench_config(case, args),
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "grid-pt-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_columns(args):
    """--columns N: the PAMM sedimentation transport (dcm_mpdata_vec_1d_device)
    on N seeded columns of 128 levels and two fields (fall speeds up to 8 m/s,
    dt 2 s, the microphysics' n_step per column), device-resident, timed with
    CUDA events over --steps calls after --warmup, L2 flushed before each;
    beside it the oracle on all host cores over the same columns, once.  One
    JSON line (kord 1, the sedimentation calls; kord 3 with the limiter)."""
    import ctypes as C

    import torch
    pkg = load_pkg()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.set_threads(os.cpu_count() or 1, False)
    lib = pkg.library()
    ncol, nq, kp = args.columns, 2, 128
    nw = kp + 2
    rng = np.random.default_rng(3)
    z = np.linspace(0.0, 1.0, nw)
    met = [np.ascontiguousarray(x) for x in (40.0 + 20.0 * z, 45.0 + 10.0 * z, 1.2 - 0.5 * z,
                                             1.2 - 0.5 * z)]
    w = -8.0 * rng.random((ncol, nw)) * rng.random((ncol, 1))
    psi = 1e-3 * rng.random((ncol, nq, kp + 2)) * (rng.random((ncol, nq, kp + 2)) > 0.3)
    dt = 2.0
    nsub = np.maximum(np.ceil(np.max(np.abs(w), axis=1) * dt / met[0].min() * 2.0),
                      1).astype(np.int32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to("cuda")  # noqa: E731
    d_dt, d_ns, d_w, d_psi0 = dev(np.full(ncol, dt)), dev(nsub), dev(w), dev(psi)
    d_met = [dev(a) for a in met]
    d_psi = d_psi0.clone()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    s = torch.cuda.current_stream()
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    out = {"metric": "columns/s of the sedimentation transport (mpdata_vec_1d)",
           "unit": "columns/s", "columns": ncol, "levels": kp, "fields": nq,
           "mean_passes": float(nsub.mean()), "steps": args.steps, "warmup": args.warmup}
    for kord, mono in ((1, 0), (3, 1)):
        def call():
            st = lib.dcm_mpdata_vec_1d_device(ncol, kp, nq, 1, 1, p(d_dt), p(d_ns),
                                              *[p(t) for t in d_met], 0, p(d_w), p(d_psi),
                                              kord, mono, 0, C.c_void_p(s.cuda_stream))
            if st:
                raise RuntimeError("dcm_mpdata_vec_1d_device: status %d" % st)
        for _ in range(args.warmup):
            d_psi.copy_(d_psi0)
            call()
        ms = []
        for _ in range(args.steps):
            d_psi.copy_(d_psi0)
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(s)
            call()
            e1.record(s)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        got = d_psi.cpu().numpy()
        ref = psi.copy()
        t0 = time.perf_counter()
        oracle.mpdata_vec_1d_columns(dt, nsub, *met, w, ref, kord=kord, monotone=mono)
        t_orc = time.perf_counter() - t0
        med = float(np.median(ms))
        out["kord%d" % kord] = {
            "monotone": bool(mono), "ms": med, "value": ncol / (med / 1e3),
            "gbs": (2 * psi.nbytes + w.nbytes) / (med / 1e3) / 1e9,
            "oracle_ms": t_orc * 1e3, "oracle_cores": os.cpu_count(),
            "max_rel_err_vs_oracle": float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))}
    print(json.dumps(compact(out)), flush=True)


def accuracy_vs_oracle(args):
    """--accuracy-vs-oracle N: the mixed form (as the benchmark runs it) and
    the FP64 path on the GPU, and the oracle's FP64 restatement of the
    reference on all host cores, each N steps from the same seeded state;
    per-field max and RMS errors (relative to max|oracle|; p on its live
    cells with the mean removed) after 1, 10 and N steps, one JSON line.
    The oracle's dot products are summed per thread (its fast mode), which
    moves its own result by the summation-order spread only."""
    pkg = load_pkg()
    case = make_case(pkg, args.case)
    g = case.grid
    n = args.accuracy_vs_oracle
    marks = sorted({1, 10, n})
    kw = dict(ptol=case.ptol, kord=case.kord, monotone=case.monotone)

    def keep(f):
        return {k: np.array(f[k], copy=True) for k in ("u", "v", "w", "th", "p")}

    snaps = {}
    for prec in (1, 0):
        core = pkg.DynamicalCore(g, device=args.device)
        core.upload_state(case.state, case.dt, precision=prec, **kw,
                          **(dict(precond=1, precond_lo=0.05) if prec else {}))
        core.driver_start()
        done = 0
        for mk in marks:
            core.step(mk - done)
            done = mk
            snaps[(prec, mk)] = keep(core.download_state())
        core.close()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.set_threads(os.cpu_count() or 1, True)
    m = oracle.OracleModel(g, case.state, case.dt, **kw)
    m.driver_start()
    t0 = time.perf_counter()
    done = 0
    out = {"case": case.name, "steps": n, "oracle_threads": os.cpu_count(), "errors": {}}
    for mk in marks:
        m.step(mk - done)
        done = mk
        ref = keep(m.fields())
        out["errors"][str(mk)] = {
            "mixed_vs_oracle": field_errors(g, ref, snaps[(1, mk)]),
            "fp64_vs_oracle": field_errors(g, ref, snaps[(0, mk)]),
            "mixed_vs_fp64": field_errors(g, snaps[(0, mk)], snaps[(1, mk)])}
    out["oracle_s"] = time.perf_counter() - t0
    print(json.dumps(out), flush=True)


def run_case(args):
    """--run-case: K time steps of a named case through the C-ABI, one line
    per step (solver iterations, FP64 updates and restarts of the mixed
    form, final residual, device time), for profiling single kernels
    (ncu -k ... over a few steps) and quick checks.  --host-loop drives the
    pressure solve from the host (the same kernels; a profiler then sees
    every launch); --graphs 2 keeps the graphs without programmatic
    dependent launch; --output FILE writes the reference's netCDF output
    before every --output-every steps; --profile prints the device time per
    kernel class over the steps after the first."""
    pkg = load_pkg()
    from dcm_b200 import cases
    c = make_case(pkg, args.case)
    core = pkg.DynamicalCore(c.grid, device=args.device)
    if args.host_loop or args.graphs != 1:
        core.solver_graphs(0 if args.host_loop else args.graphs)
    if args.fuse is not None:
        core.set_launch_shape(1, fuse=args.fuse)
    core.set_mpdata_shape(bool(args.mp_fuse), args.mp_rows)
    kw = dict(nq=c.nq, c_s=c.c_s, c_e=c.c_e) if c.nq else {}
    if args.viscous:
        kw["viscous"] = dict(lamsq=cases.mixing_length_sq(c.grid, 0.23, 0.1), z0=0.1, z0th=0.1)
    core.upload_state(c.state, c.dt, ptol=c.ptol, kord=c.kord, monotone=c.monotone,
                      precision=args.precision, precond=args.precond,
                      precond_lo=args.precond_lo, inner_tol=args.inner_tol, **kw)
    core.driver_start()
    out = pkg.Output(core, args.output) if args.output else None
    t_write = []
    for s in range(args.steps):
        if args.profile and s == min(1, args.steps - 1):
            core.profile(True)  # after the first step (module loading, first-call set-up)
        if out and s % args.output_every == 0:
            t0 = time.perf_counter()
            out.write(s * c.dt)
            t_write.append((time.perf_counter() - t0) * 1e3)
        st = core.step(1)
        print("%s precision %d step %d: %d iterations (%d updates, %d restarts), "
              "err %.3e, %.2f ms" % (c.name, args.precision, s + 1, st.iters_last,
                                     st.updates_last, st.restarts_last, st.err_last,
                                     st.ms_total), flush=True)
    if out:
        t0 = time.perf_counter()
        out.close()
        print("output: %d records, host ms per write call %s, close (drain) %.1f ms" % (
            len(t_write), " ".join("%.2f" % t for t in t_write),
            (time.perf_counter() - t0) * 1e3), flush=True)
    if args.profile:
        for name, (ms, n) in core.profile_read().items():
            if n:
                print("  %-9s %9.3f ms  %6d launches" % (name, ms, n))
    core.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--case", default="warm_bubble")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--cpu-budget", type=float, default=60.0,
                    help="seconds of the GPU arm's bounded cpu_baseline sample")
    ap.add_argument("--ref-budget", type=float, default=1800.0,
                    help="safety bound (s) of the reference arm, which times all K steps")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--details", default="bench_details.json",
                    help="file (relative to the repository root) for the long-form record")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other configurations (shear layer, sheared convection, "
                         "ensemble)")
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--host-loop", action="store_true",
                    help="host-polled solver loop instead of graph-driven solves (same "
                         "kernels; lets a profiler see every solver launch)")
    # --run-case: per-step lines of one case (profiling and quick checks)
    ap.add_argument("--run-case", action="store_true")
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1])
    ap.add_argument("--graphs", type=int, default=1, choices=[0, 1, 2],
                    help="solver loops: 1 graph-driven, 2 graph-driven without programmatic "
                         "dependent launch, 0 host-polled (as --host-loop)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--viscous", action="store_true",
                    help="Smagorinsky subgrid model on in sources (cvis 0.23, z0 = z0th = "
                         "0.1 m)")
    ap.add_argument("--precond", type=int, default=0, choices=[0, 1],
                    help="1: the mixed form's FP32 iterations use Chebyshev-weighted sweeps "
                         "on [--precond-lo, 2]")
    ap.add_argument("--precond-lo", type=float, default=0.05)
    ap.add_argument("--inner-tol", type=float, default=0.1,
                    help="mixed form: the reliable-update factor")
    ap.add_argument("--fuse", type=int, default=None, choices=[0, 1, 2],
                    help="FP32 preconditioner: separate sweeps (0), the fused kernel (1), or "
                         "the fused kernel with phase C's matvec as a fourth stage (2)")
    ap.add_argument("--mp-fuse", type=int, default=0, choices=[0, 1],
                    help="MPDATA: one fused kernel per antidiffusive iteration (1) or one "
                         "kernel per stage (0)")
    ap.add_argument("--mp-rows", type=int, default=32,
                    help="MPDATA: cap on the fused kernel's rows per block")
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--output", default=None,
                    help="netCDF file written before every --output-every steps")
    ap.add_argument("--output-every", type=int, default=1)
    ap.add_argument("--accuracy-vs-oracle", type=int, default=0,
                    help="N: errors of both forms against the oracle after 1, 10, N steps")
    ap.add_argument("--columns", type=int, default=0,
                    help="N: the PAMM sedimentation transport on N columns, timed, beside "
                         "the oracle")
    args = ap.parse_args()
    if args.run_case:
        run_case(args)
        return
    if args.accuracy_vs_oracle:
        accuracy_vs_oracle(args)
        return
    if args.columns:
        run_columns(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    else:
        if world > 1:
            import datetime

            import torch
            import torch.distributed as tdist
            torch.cuda.set_device(local_rank)
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
            dist = tdist
        if args.case == "ensemble":
            res = run_ensemble(args, rank, world, local_rank, dist)
        else:
            res = run_b200(args, rank, world, local_rank, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    if res is not None:
        print(json.dumps(compact(res)), flush=True)


if __name__ == "__main__":
    main()
