#!/usr/bin/env python
"""Benchmark of the Lippmann-Schwinger basic scheme on B200.

Workload (one GPU): 3D two-phase random spheres on a 128^3 grid (radius 8,
non-overlapping, volume fraction 0.3, seeded random sequential addition),
matrix mu=1 nu=0.3, spheres mu=100 nu=0.2, reference medium mu0=50.5
nu0=0.3, filtered Green operator, FP64, the 6 unit macroscopic load cases
iterated together.  One step = one basic-scheme iteration of all 6 load
cases (6 * 128^3 voxel-iterations); the metric is voxel-iterations/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (launched with torchrun): every rank solves its own replica (no
collective on the data path, weak scaling); the time is the max over ranks.
``--impl reference`` times the reference's own CPU path (its Cython modules
built in oracle/_ref, else the oracle's numpy restatement) on the same
workload, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "3D LS solve voxel-iter/s & time-to-1e-8 residual, mixed vs FP64; % HBM peak"
UNIT = "voxel-iter/s"
FALLBACK_HBM_GBS = 6650.0

MATRIX = (1.0, 0.3)
INCLUSION = (100.0, 0.2)
REF_MEDIUM = (50.5, 0.3)

# algorithmic bytes per voxel and load case of each pass (FP64, s = 6):
# r2c reads eps (48 B) + phase id (1 B) and writes the spectrum (48 B);
# column passes read and write the spectrum; c2r reads the spectrum and the
# old eps and writes the new eps.  Sum: 11*s*p + m = 529 B per voxel-iteration.
def pass_bytes(s, p, m=1):
    return {"rows_r2c_local": (2 * s * p + m), "cols_fwd_axis1": 2 * s * p,
            "cols_green_axis0": 2 * s * p, "cols_inv_axis1": 2 * s * p,
            "rows_c2r_update": 3 * s * p, "reduce_residual": 0}


def reduce_max(x, dist, device="cuda"):
    """Max of a per-rank float over all ranks (the job's time is its slowest
    rank); identity without a process group."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_step, steps, ms):
    """Units processed by all ranks per second: every rank runs its own
    replica of the workload (weak scaling), timed as the slowest rank."""
    return world * units_per_step * steps / (ms / 1e3)


def replica_seed(rank):
    """Seed of the microstructure rank `rank` solves (independent replicas)."""
    return 2024 + rank


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=5)
        return self.summarise(self.lines)

    @staticmethod
    def summarise(lines):
        """Median SM clock, the largest max clock and the throttle reasons seen
        active in nvidia-smi CSV lines of FIELDS (None without a sample)."""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def build_problem(n, seed, variant, dtype):
    import numpy as np

    import janus_b200.material.elastic.linear.isotropic as material
    from janus_b200 import microstructures as micro
    from janus_b200 import operators as ops
    from janus_b200.green import filtered, truncated

    phase, centres = micro.random_spheres(n, radius=8 * n / 128, volume_fraction=0.3,
                                          seed=seed)
    mat0 = material.create(*REF_MEDIUM, 3)
    tens = []
    for g, nu in (MATRIX, INCLUSION):
        m = material.create(g, nu, 3)
        tens.append(ops.isotropic_4(3 * (m.k - mat0.k), 2 * (m.g - mat0.g), 3))
    factory = filtered if variant == "filtered" else truncated
    green = factory(mat0.green_operator(), phase.shape, 1.0, dtype=dtype)
    return phase, tens, green, np.eye(6)


# ---------------------------------------------------------------------------
# CPU leg: the reference's serial path (or the oracle port) on one load case
# ---------------------------------------------------------------------------

def reference_available(fftw=None):
    from oracle import reference
    return reference.load(fftw=fftw)


# what the timed CPU baseline runs, by kind
CPU_LABELS = {
    "reference": "reference Cython + project FFT shim (not FFTW)",
    "reference+fftw": "reference Cython + FFTW",
    "port": "oracle numpy port of the reference (numpy.fft)",
}


def fftw_probe():
    """Path of a system libfftw3 (double precision), or None, and how it was
    looked for (ldconfig -p, then the usual library directories)."""
    found = None
    try:
        out = subprocess.run(["ldconfig", "-p"], capture_output=True, text=True,
                             timeout=10).stdout
        for line in out.splitlines():
            if "libfftw3.so.3" in line and "=>" in line:
                found = line.split("=>")[-1].strip()
                break
    except Exception:
        pass
    if found is None:
        for d in ("/usr/lib/x86_64-linux-gnu", "/usr/lib64", "/usr/lib", "/usr/local/lib"):
            cand = os.path.join(d, "libfftw3.so.3")
            if os.path.exists(cand):
                found = cand
                break
    info = {"ldconfig_libfftw3": found, "fftw3_h": os.path.exists("/usr/include/fftw3.h")}
    if found is None:
        info["fftw"] = "unavailable on this box"
    return found, info


def host_cpu():
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "logical_cores": os.cpu_count()}


def cpu_worker(n, seed, load, iters, variant, out_path, field_path=None, fftw=None):
    """Run `iters` basic-scheme iterations of one load case with the
    reference's own objects (the tutorial loop, square_basic.py:83-92);
    optionally save the last iterate (the parity leg's oracle field)."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    import numpy as np
    from janus_b200 import microstructures as micro
    phase, _ = micro.random_spheres(n, radius=8 * n / 128, volume_fraction=0.3, seed=seed)
    E = np.zeros(6)
    E[load] = 1.0
    ref = reference_available(fftw)
    times = []
    if ref is not None:
        kind = "reference+fftw" if fftw else "reference"
        import janus.fft.serial as rfft
        import janus.green as rgreen
        import janus.material.elastic.linear.isotropic as rmat
        import janus.operators as rops
        mat0 = rmat.create(*REF_MEDIUM, 3)
        tens = []
        for g, nu in (MATRIX, INCLUSION):
            m = rmat.create(g, nu, 3)
            tens.append(rops.isotropic_4(3 * (m.k - mat0.k), 2 * (m.g - mat0.g), 3))
        loc_arr = np.empty(phase.shape, dtype=object)
        loc_arr[phase == 0] = tens[0]
        loc_arr[phase == 1] = tens[1]
        loc = rops.block_diagonal_operator(loc_arr)
        fac = rgreen.filtered if variant == "filtered" else rgreen.truncated
        green = fac(mat0.green_operator(), phase.shape, 1.0, rfft.create_real(phase.shape))
        eps = np.empty(phase.shape + (6,))
        eps[...] = E
        new = np.empty_like(eps)
        norm = 1 / np.sqrt(eps[..., 0].size) / np.linalg.norm(E)
        for _ in range(iters):
            t0 = time.perf_counter()
            loc.apply(eps, new)
            green.apply(new, new)
            np.subtract(E, new, out=new)
            _ = norm * np.linalg.norm(new - eps)
            eps, new = new, eps
            times.append(time.perf_counter() - t0)
    else:
        kind = "port"
        from oracle import janus_oracle as O
        pars = [O.delta_c(*MATRIX, *REF_MEDIUM, 3), O.delta_c(*INCLUSION, *REF_MEDIUM, 3)]
        G = O.spectral_green_field(phase.shape, 1.0, *REF_MEDIUM, variant)
        eps = np.empty(phase.shape + (6,))
        eps[...] = E
        for _ in range(iters):
            t0 = time.perf_counter()
            tau = O.phase_apply(eps, phase, [p[0] for p in pars], [p[1] for p in pars], 3)
            y = O.green_apply(tau, *REF_MEDIUM, 1.0, variant, G=G)
            new = E - y
            _ = np.linalg.norm(new - eps)
            eps = new
            times.append(time.perf_counter() - t0)
    if field_path:
        np.save(field_path, eps)
    with open(out_path, "w") as f:
        json.dump({"kind": kind, "times": times}, f)


def run_cpu_workers(n, seed, loads, iters, variant, tag, save_field=False, fftw=None):
    import tempfile
    procs = []
    outs = []
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1",
               MKL_NUM_THREADS="1", CUDA_VISIBLE_DEVICES="")
    tmpdir = tempfile.mkdtemp(prefix="jb_cpu_")
    fields = []
    for load in loads:
        out = os.path.join(tmpdir, f"{tag}_{load}.json")
        outs.append(out)
        cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", "--n", str(n),
               "--seed", str(seed), "--load", str(load), "--iters", str(iters),
               "--variant", variant, "--out", out]
        if save_field:
            fields.append(os.path.join(tmpdir, f"{tag}_{load}_eps.npy"))
            cmd += ["--field", fields[-1]]
        if fftw:
            cmd += ["--fftw", fftw]
        procs.append(subprocess.Popen(cmd, env=env))
    for p in procs:
        p.wait()
    results = []
    for i, (p, out) in enumerate(zip(procs, outs)):
        if p.returncode != 0 or not os.path.exists(out):
            raise RuntimeError("CPU worker failed")
        with open(out) as f:
            results.append(json.load(f))
        if save_field:
            results[-1]["field"] = fields[i]
    return results


def cpu_baseline(n, seed, variant, budget_s=20.0, fftw=None):
    """1-core time of the reference's serial path on one load case:
    iterations until about `budget_s` of CPU work (at least 2).  The last
    iterate is kept (``field``, iteration count ``iterations``) for the
    parity leg."""
    probe = run_cpu_workers(n, seed, [5], 2, variant, "probe", fftw=fftw)[0]
    per_it = max(probe["times"][1], 1e-3)
    iters = max(2, min(20, int(budget_s / per_it)))
    res = run_cpu_workers(n, seed, [5], iters + 1, variant, "base", save_field=True,
                          fftw=fftw)[0]
    t = sum(res["times"][1:])
    vox = n ** 3
    return {"value": vox * iters / t, "unit": UNIT, "cores": 1,
            "kind": "reference" if res["kind"].startswith("reference") else "port",
            "label": CPU_LABELS[res["kind"]],
            "sample": f"{iters} basic-scheme iterations of one load case (E = xy) at {n}^3, "
                      "after 1 untimed iteration, single thread",
            "host_cpu": host_cpu(), "field": res["field"], "iterations": iters + 1}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def run_gpu(args, rank, world, dist):
    import numpy as np
    import torch

    from janus_b200 import operators as ops
    from janus_b200.solvers import BasicScheme

    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dtype = torch.float64 if args.dtype == "f64" else torch.float32
    n = args.n
    phase, tens, green, E = build_problem(n, replica_seed(rank), args.variant, dtype)
    loc = ops.BlockDiagonalOperator3D.from_phases(phase, tens, dtype=dtype)
    tuning = None
    if not args.no_tune:
        from janus_b200 import autotune
        tuning = autotune.tune(green, loc, nload=6, use_cache=False)
    solver = BasicScheme(green, loc, nload=6)
    solver.set_load(E)
    eps = solver.new_field()
    eps[...] = torch.from_numpy(E).to(dtype).cuda().view(6, 1, 1, 1, 6)
    res = torch.zeros(6, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        solver.step(eps, res)
    torch.cuda.synchronize()

    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    gpu_index = vis.split(",")[local] if vis else str(local)
    sampler = ClockSampler(gpu_index)
    sampler.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    solver.timing_begin(args.steps)
    start.record()
    for _ in range(args.steps):
        solver.step(eps, res)
    end.record()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = start.elapsed_time(end)
    passes, nrec = solver.timing_end()
    clocks = sampler.stop()
    ms = reduce_max(ms, dist)
    vox_step = 6 * n ** 3
    value = whole_job_rate(world, vox_step, args.steps, ms)

    # roofline of the dominant pass (algorithmic bytes / its mean duration)
    p = 8 if dtype == torch.float64 else 4
    pbytes = pass_bytes(6, p)
    dom = max(passes, key=lambda k: passes[k])
    dom_ms = passes[dom] / max(nrec, 1)
    peak, peak_kind = measured_peak()
    bytes_launch = pbytes[dom] * vox_step
    achieved = bytes_launch / (dom_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        key = f"{dom}@{n}^3x6/{args.variant}/{args.dtype}"
        if key in tj:
            traffic = tj[key]
    step_bytes = sum(pbytes.values()) * vox_step
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": bytes_launch,
                "step_achieved": round(step_bytes / (ms / args.steps / 1e3) / 1e9, 1),
                "step_frac": round(step_bytes / (ms / args.steps / 1e3) / 1e9 / peak, 4)}

    # end to end through the public API with host buffers: host phase map and
    # E in, strain field out (pinned), K iterations with the per-iteration
    # residual read back
    e2e = None
    if not args.no_e2e:
        out = torch.empty(solver.field_shape, dtype=dtype, pin_memory=True)
        # three repetitions, the median reported (each one complete: operators
        # built from the host phase map, K iterations, field copied out)
        reps = []
        for _ in range(3):
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()
            t0 = time.perf_counter()
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record()
            loc2 = ops.BlockDiagonalOperator3D.from_phases(phase, tens, dtype=dtype)
            sol2 = BasicScheme(green, loc2, nload=6)
            t1 = time.perf_counter()
            r = sol2.run(E, args.steps)
            t2 = time.perf_counter()
            out.copy_(r.eps, non_blocking=True)
            s1.record()
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            reps.append((max(s0.elapsed_time(s1), wall * 1e3),
                         {"setup_ms": round((t1 - t0) * 1e3, 2),
                          "solve_ms": round((t2 - t1) * 1e3, 2),
                          "copy_out_ms": round((time.perf_counter() - t2) * 1e3, 2)}))
            del r, sol2, loc2
        reps_sorted = sorted(reps, key=lambda x: x[0])
        e2e_ms, parts = reps_sorted[1]
        parts = dict(parts, repetitions_ms=[round(x[0], 2) for x in reps])
        e2e_ms = reduce_max(e2e_ms, dist)
        e2e = {"value": whole_job_rate(world, vox_step, args.steps, e2e_ms), "unit": UNIT,
               "h2d_bytes_per_step": int((phase.nbytes + E.nbytes) / args.steps),
               "d2h_bytes_per_step": int((out.numel() * out.element_size()) / args.steps
                                         + 6 * 8),
               "what": "operators from a host phase map, basic_scheme() for K iterations "
                       "(residuals read back every iteration), strain field copied to "
                       "pinned host memory; median of 3 repetitions", "parts": parts}

    solve = None
    if not args.no_solve and rank == 0 and world == 1 and args.dtype == "f64":
        import janus_b200.material.elastic.linear.isotropic as material
        solve = {"tol": args.tol, "workload": "the bench cell, 6 load cases"}
        solve.update(time_to_solution(
            green, loc, E, material.create(*REF_MEDIUM, 3), args.tol, args.inner,
            args.krylov_inner, args.solve_max_iter,
            legs=("fp64", "mixed", "mixed_bicgstab", "fp64_bicgstab", "gmres_fp64")))
        torch.cuda.empty_cache()

    target = None
    if not args.no_target and rank == 0 and world == 1 and args.dtype == "f64":
        target = target_leg(args, 2024)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(n, 2024, args.variant)
        except Exception as exc:  # pragma: no cover
            cpu = {"value": None, "unit": UNIT, "error": str(exc)}
        # the reference on real FFTW, where this machine has it
        fftw_path, fftw_info = fftw_probe()
        if fftw_path and os.path.isdir(os.path.join(ROOT, "oracle", "_ref_fftw", "janus")):
            try:
                cf = cpu_baseline(n, 2024, args.variant, fftw=fftw_path)
                os.remove(cf.pop("field"))
                cf.pop("iterations", None)
                fftw_info["reference_fftw"] = cf
            except Exception as exc:  # pragma: no cover
                fftw_info["reference_fftw"] = {"error": str(exc)}
        elif fftw_path:
            fftw_info["reference_fftw"] = "no FFTW build of the reference checker (oracle/_ref_fftw)"
        if cpu.get("value") is not None:
            cpu["fftw_probe"] = fftw_info
        # parity: the GPU FP64 iterate after the same iterations of the same
        # load case against the reference's own field
        field = cpu.pop("field", None)
        if field and args.dtype == "f64":
            import numpy as np
            ref_eps = np.load(field)
            os.remove(field)
            K = cpu.pop("iterations")
            E5 = np.zeros((1, 6))
            E5[0, 5] = 1.0
            r1 = BasicScheme(green, loc, nload=1).run(E5, K)
            got = r1.eps[0].cpu().numpy()
            err = float(np.abs(got - ref_eps).max() / np.abs(ref_eps).max())
            parity = {"max_rel_err": err, "bar": 1e-12, "ok": err <= 1e-12,
                      "what": f"GPU FP64 basic-scheme iterate after {K} iterations of load "
                              f"case E = xy at {n}^3 against the {cpu['label']} field of the "
                              "same iterations (the cpu_baseline run)"}
            del r1
        else:
            cpu.pop("iterations", None)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
            "config": {"workload": f"3D two-phase random spheres {n}^3 (radius {8 * n // 128}, "
                                   "vf 0.3, seeded RSA), mu 1/100, nu 0.3/0.2, mu0 50.5, "
                                   f"{args.variant} Green operator, 6 load cases, basic scheme",
                       "grid": [n, n, n], "load_cases": 6, "variant": args.variant,
                       "precision": args.dtype, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (strain fields "
                             f"{6 * n ** 3 * 6 * p / 1e6:.0f} MB per step)"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": nrec * len(passes),
            "passes_ms_per_step": {k: round(v / max(nrec, 1), 4) for k, v in passes.items()},
            "clocks": clocks, "solve": solve, "target": target, "parity": parity,
            "tuning": tuning,
        }
        print(json.dumps(line), flush=True)


def run_batch2d(args, rank, world):
    """Batched 2D workload: seeded two-phase ellipse cells of uneven sizes,
    3 load cases each, FP32 bulk + FP64 defect correction to a relative
    residual of args.batch_tol, all cells in one CUDA graph launch per outer
    step; the same cells solved one after another are timed beside it."""
    import numpy as np
    import torch

    import janus_b200.material.elastic.linear.isotropic as material
    from janus_b200 import microstructures as micro
    from janus_b200 import operators as ops
    from janus_b200.batch import BatchedMixedScheme
    from janus_b200.green import filtered, truncated
    from janus_b200.solvers import MixedScheme

    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    probs = micro.batch_2d_problems(args.batch_count, seed=2024 + rank)
    factory = filtered if args.variant == "filtered" else truncated
    built = []
    for p in probs:
        pars = [(2 * (material.create(g, nu, 2).k - material.create(p["mu0"], p["nu0"], 2).k),
                 2 * (g - p["mu0"])) for g, nu in zip(p["mu"], p["nu"])]
        tens = [ops.isotropic_4(a, b, 2) for a, b in pars]
        loc = ops.BlockDiagonalOperator2D.from_phases(p["phase"], tens)
        green = factory(material.create(p["mu0"], p["nu0"], 2).green_operator(),
                        p["phase"].shape, 1.0)
        built.append((green, loc, 3))
    E = [np.eye(3)] * len(probs)
    inner = args.krylov_inner if args.inner_method == "bicgstab" else args.inner
    batch = BatchedMixedScheme(built, inner=inner, branches=args.batch_branches,
                               method=args.inner_method)
    batch.run(E, tol=1e-2, max_outer=2)  # warm: tables, kernels, first capture
    torch.cuda.synchronize()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    sampler = ClockSampler(vis.split(",")[0] if vis else "0")
    sampler.start()
    time.sleep(0.3)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    res = batch.run(E, tol=args.batch_tol, max_outer=args.solve_max_iter)
    b.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    t_batch = a.elapsed_time(b) / 1e3
    nvox = [p["n"] ** 2 for p in probs]
    vi32 = sum(3 * v * r.fp32_iterations for v, r in zip(nvox, res))
    vi64 = sum(3 * v * r.outer_iterations for v, r in zip(nvox, res))
    # algorithmic bytes: 2D FP32 sweep 7*s*4 + 1, FP64 residual pass 7*s*8 + 1
    # (+ the FP32 residual written, 4*s) per voxel and load case
    traffic = vi32 * (7 * 3 * 4 + 1) + vi64 * (7 * 3 * 8 + 1 + 3 * 4)
    peak, peak_kind = measured_peak()
    seq = None
    if not args.no_sequential:
        # the batch runs every correction at the full sweep count, so the
        # one-by-one reference does too (the adaptive BiCGSTAB count of a lone
        # MixedScheme is a different schedule)
        seq_method = "bicgstab_fixed" if args.inner_method == "bicgstab" else args.inner_method
        schemes = [MixedScheme(g, l, 3, inner=inner, method=seq_method)
                   for g, l, _ in built]
        a.record()
        rs = [s.run(np.eye(3), tol=args.batch_tol, max_outer=args.solve_max_iter)
              for s in schemes]
        b.record()
        torch.cuda.synchronize()
        t_seq = a.elapsed_time(b) / 1e3
        same = all(torch.equal(x.eps, y.eps) for x, y in zip(res, rs))
        seq = {"method": seq_method, "seconds": round(t_seq, 4),
               "bitwise_equal_to_batch": bool(same),
               "outer_iterations_max": max(r.outer_iterations for r in rs),
               "batch_speedup": round(t_seq / t_batch, 3)}
    worst = max(float(r.residuals[-1].max()) for r in res)
    line = {
        "metric": "batched 2D LS solve voxel-iter/s (mixed FP32+FP64, one CUDA graph "
                  "launch per outer step)",
        "value": (vi32 + vi64) / t_batch, "unit": UNIT, "n_gpus": 1,
        "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"{len(probs)} two-phase 2D ellipse cells, n in "
                               f"{sorted(set(p['n'] for p in probs))}, 2-20 ellipses, "
                               "contrast log-U[10,1000], nu U[0.15,0.4], 3 load cases, "
                               f"{args.variant} Green operator, tol {args.batch_tol}",
                   "cells": len(probs), "voxels": int(sum(nvox)), "inner": inner,
                   "inner_method": args.inner_method,
                   "graph_branches": args.batch_branches},
        "time_to_solution_s": round(t_batch, 4),
        "graph_launches": batch.graph_launches,
        "outer_iterations_max": max(r.outer_iterations for r in res),
        "fp32_iterations_total": int(sum(r.fp32_iterations for r in res)),
        "final_residual_max": worst,
        "hbm": {"achieved": round(traffic / t_batch / 1e9, 1), "peak": peak, "unit": "GB/s",
                "frac": round(traffic / t_batch / 1e9 / peak, 4), "peak_source": peak_kind,
                "counts": "operator applications only (BiCGSTAB vector updates excluded)"
                if args.inner_method == "bicgstab" else "all passes"},
        "sequential": seq, "clocks": clocks,
        "per_cell": sorted([[p["n"], round(float(p["mu"][1]), 1), r.outer_iterations]
                            for p, r in zip(probs, res)], key=lambda v: -v[2])[:16],
    }
    print(json.dumps(line), flush=True)


def time_to_solution(green, loc, E, mat0, tol, inner, krylov_inner, max_outer,
                     legs=("fp64", "mixed", "mixed_bicgstab", "fp64_bicgstab")):
    """Solve (I + Gamma0 (C - C0)) eps = E to relative residual `tol` with the
    plain FP64 basic scheme and the defect-correction solvers, CUDA-event
    timed after a warm-up of each; C_eff of every leg against the FP64 basic
    scheme's.  Legs: fp64 (basic scheme), mixed (FP32 basic inner sweeps),
    mixed_bicgstab (FP32 BiCGSTAB inner), fp64_bicgstab (the same BiCGSTAB
    defect correction in FP64: the control separating the Krylov gain from
    the precision gain), gmres_fp64 (FP64 restarted GMRES)."""
    import numpy as np
    import torch

    from janus_b200.solvers import GMRES, BasicScheme, MixedScheme

    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    out = {}

    def timed(fn):
        torch.cuda.synchronize()
        a.record()
        r = fn()
        b.record()
        torch.cuda.synchronize()
        return r, a.elapsed_time(b) / 1e3

    fp64 = BasicScheme(green, loc, nload=len(E))
    fp64.run(E, 3)  # warm (tables, kernels)
    r64, t64 = timed(lambda: fp64.run(E, max_outer * inner, tol=tol))
    c64 = r64.mean_stress(mat0, E)
    del fp64
    out["fp64"] = {"iterations": r64.iterations, "seconds": round(t64, 4),
                   "final_residual_max": float(r64.residuals[-1].max()),
                   "status": r64.status_names}

    def rel(c):
        return float(np.abs(c - c64).max() / np.abs(c64).max())
    specs = {"mixed": dict(inner=inner, method="basic"),
             "mixed_bicgstab": dict(inner=krylov_inner, method="bicgstab"),
             "fp64_bicgstab": dict(inner=krylov_inner, method="bicgstab",
                                   inner_dtype=torch.float64)}
    for leg in legs:
        if leg in specs:
            sch = MixedScheme(green, loc, nload=len(E), **specs[leg])
            sch.run(E, tol=1e-30, max_outer=2)  # warm: kernels, work fields
            r, t = timed(lambda: sch.run(E, tol=tol, max_outer=max_outer))
            out[leg] = {"inner": specs[leg]["inner"], "outer_iterations": r.outer_iterations,
                        "inner_operator_applications": r.fp32_iterations,
                        "seconds": round(t, 4),
                        "final_residual_max": float(r.residuals[-1].max()),
                        "C_eff_max_rel_diff_vs_fp64": rel(r.mean_stress(mat0, E)),
                        "status": r.status_names}
            del sch
        elif leg == "gmres_fp64":
            gm = GMRES(green, loc, nload=len(E), restart=20)
            gm.run(E, tol=1e-30, max_iter=2)  # warm
            r, t = timed(lambda: gm.run(E, tol=tol, max_iter=max_outer * inner))
            out[leg] = {"restart": 20, "arnoldi_steps": r.iterations, "seconds": round(t, 4),
                        "final_residual_max": float(r.final_residuals.max()),
                        "C_eff_max_rel_diff_vs_fp64": rel(r.mean_stress(mat0, E)),
                        "status": r.status_names}
            del gm
        torch.cuda.empty_cache()
    for leg in list(out):
        if leg != "fp64":
            out[leg]["speedup_vs_fp64"] = round(t64 / out[leg]["seconds"], 3)
    if "fp64_bicgstab" in out and "mixed_bicgstab" in out:
        # precision alone: the same BiCGSTAB defect correction, FP64 vs FP32 inner
        out["precision_gain_bicgstab"] = round(
            out["fp64_bicgstab"]["seconds"] / out["mixed_bicgstab"]["seconds"], 3)
    if "mixed" in out:
        out["precision_gain_basic"] = out["mixed"]["speedup_vs_fp64"]
    out["C_eff_fp64"] = [[float(v) for v in row] for row in c64]
    return out


def target_leg(args, seed):
    """The time-to-solution target: a seeded 256^3 two-phase periodic
    Voronoi cell (512 cells, fair-coin phases), mu 1 / 100, nu 0.3,
    mu0 50.5, truncated Green operator, shear load case, to 1e-8."""
    import numpy as np
    import torch

    import janus_b200.material.elastic.linear.isotropic as material
    from janus_b200 import microstructures as micro
    from janus_b200 import operators as ops
    from janus_b200.green import truncated

    n, c, tol = args.target_n, 100.0, 1e-8
    t0 = time.perf_counter()
    phase = micro.voronoi(n, cells=512, seed=seed)
    gen_s = time.perf_counter() - t0
    mu0, nu0 = 0.5 * (1.0 + c), 0.3
    mat0 = material.create(mu0, nu0, 3)
    pars = [(3 * (material.create(g, 0.3, 3).k - mat0.k), 2 * (g - mu0)) for g in (1.0, c)]
    loc = ops.BlockDiagonalOperator3D.from_phases(phase, [ops.isotropic_4(a, b, 3)
                                                          for a, b in pars])
    green = truncated(mat0.green_operator(), (n, n, n), 1.0)
    E = np.eye(6)[-1:]
    res = time_to_solution(green, loc, E, mat0, tol, args.inner, args.krylov_inner,
                           args.solve_max_iter)
    del loc, green
    torch.cuda.empty_cache()
    return {"workload": f"3D two-phase Voronoi {n}^3, 512 cells (seed {seed}), mu 1/{c:g}, "
                        f"nu 0.3, mu0 {mu0:g}, truncated, E = xy shear, tol {tol:g}",
            "target": ">= 3x lower time-to-solution than the plain FP64 GPU solver, "
                      "C_eff within 1e-7 of FP64",
            "generation_s": round(gen_s, 1), "results": res}


def run_voronoi(args, rank):
    """Precision stress test: a 256^3 two-phase periodic Voronoi partition
    (512 seeded cells, fair-coin phases), phase A mu=1, phase B mu=contrast,
    nu=0.3, mu0 = (1 + contrast)/2, nu0 = 0.3; FP32 bulk + FP64 defect
    correction every `inner` iterations against the plain FP64 scheme, both
    to the same relative residual, for each Green variant."""
    import numpy as np
    import torch

    import janus_b200.material.elastic.linear.isotropic as material
    from janus_b200 import microstructures as micro
    from janus_b200 import operators as ops
    from janus_b200.green import filtered, truncated
    from janus_b200.solvers import GMRES, BasicScheme, MixedScheme

    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    n = args.voronoi_n
    t0 = time.perf_counter()
    phase = micro.voronoi(n, cells=512, seed=replica_seed(rank))
    gen_s = time.perf_counter() - t0
    c = args.contrast
    mu0, nu0 = 0.5 * (1.0 + c), 0.3
    mat0 = material.create(mu0, nu0, 3)
    pars = [(3 * (material.create(g, 0.3, 3).k - mat0.k), 2 * (g - mu0)) for g in (1.0, c)]
    tens = [ops.isotropic_4(a, b, 3) for a, b in pars]
    loc = ops.BlockDiagonalOperator3D.from_phases(phase, tens)
    E = np.eye(6)[-args.voronoi_loads:]
    out = {}
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    sampler = ClockSampler(vis.split(",")[0] if vis else "0")
    sampler.start()
    for name, factory in (("truncated", truncated), ("filtered", filtered)):
        if name not in args.voronoi_variants.split(","):
            continue
        green = factory(mat0.green_operator(), (n, n, n), 1.0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        fp64 = BasicScheme(green, loc, nload=len(E))
        fp64.run(E, 3)  # warm (tables, kernels)
        torch.cuda.synchronize()
        a.record()
        r64 = fp64.run(E, args.solve_max_iter * args.inner, tol=args.tol)
        b.record()
        torch.cuda.synchronize()
        t64 = a.elapsed_time(b) / 1e3
        c64 = r64.mean_stress(mat0, E)
        del fp64
        mixed = MixedScheme(green, loc, nload=len(E), inner=args.inner)
        mixed.run(E, tol=1e-2, max_outer=2)  # warm
        torch.cuda.synchronize()
        a.record()
        rm = mixed.run(E, tol=args.tol, max_outer=args.solve_max_iter)
        b.record()
        torch.cuda.synchronize()
        tm = a.elapsed_time(b) / 1e3
        cm = rm.mean_stress(mat0, E)
        out[name] = {
            "fp64": {"iterations": r64.iterations, "seconds": round(t64, 3),
                     "final_residual_max": float(r64.residuals[-1].max())},
            "mixed": {"outer_iterations": rm.outer_iterations,
                      "fp32_iterations": rm.fp32_iterations, "seconds": round(tm, 3),
                      "final_residual_max": float(rm.residuals[-1].max())},
            "speedup": round(t64 / tm, 3),
            "C_eff_rows": [[float(v) for v in row] for row in cm],
            "C_eff_max_rel_diff_vs_fp64": float(np.abs(cm - c64).max() / np.abs(c64).max()),
        }
        del mixed
        kry = MixedScheme(green, loc, nload=len(E), inner=args.krylov_inner, method="bicgstab")
        kry.run(E, tol=1e-30, max_outer=2)  # warm: one correction allocates the Krylov fields
        torch.cuda.synchronize()
        a.record()
        rk = kry.run(E, tol=args.tol, max_outer=args.solve_max_iter)
        b.record()
        torch.cuda.synchronize()
        tk = a.elapsed_time(b) / 1e3
        ck = rk.mean_stress(mat0, E)
        out[name]["mixed_bicgstab"] = {
            "inner": args.krylov_inner, "outer_iterations": rk.outer_iterations,
            "fp32_operator_applications": rk.fp32_iterations, "seconds": round(tk, 3),
            "final_residual_max": float(rk.residuals[-1].max()),
            "C_eff_max_rel_diff_vs_fp64": float(np.abs(ck - c64).max() / np.abs(c64).max())}
        out[name]["speedup_bicgstab"] = round(t64 / tk, 3)
        del kry
        gm = GMRES(green, loc, nload=len(E), restart=args.gmres_restart)
        gm.run(E, tol=1e-30, max_iter=2)  # warm
        torch.cuda.synchronize()
        a.record()
        rg = gm.run(E, tol=args.tol, max_iter=args.solve_max_iter * args.inner)
        b.record()
        torch.cuda.synchronize()
        tg = a.elapsed_time(b) / 1e3
        cg = rg.mean_stress(mat0, E)
        out[name]["gmres_fp64"] = {
            "restart": args.gmres_restart, "arnoldi_steps": rg.iterations,
            "seconds": round(tg, 3), "final_residual_max": float(rg.final_residuals.max()),
            "C_eff_max_rel_diff_vs_fp64": float(np.abs(cg - c64).max() / np.abs(c64).max())}
        out[name]["speedup_gmres_fp64"] = round(t64 / tg, 3)
        del gm, green
        torch.cuda.empty_cache()
    clocks = sampler.stop()
    line = {"metric": "time-to-solution, mixed (FP32 + FP64 defect correction) vs FP64",
            "unit": "s", "n_gpus": 1, "higher_is_better": False, "data": "synthetic",
            "config": {"workload": f"3D two-phase Voronoi {n}^3, 512 cells, mu 1/{c:g}, "
                                   f"nu 0.3, mu0 {mu0:g}, {len(E)} load case(s), "
                                   f"tol {args.tol:g}, inner {args.inner}",
                       "grid": [n, n, n], "contrast": c, "load_cases": len(E),
                       "generation_s": round(gen_s, 1)},
            "results": out, "clocks": clocks}
    print(json.dumps(line), flush=True)


def run_gradients(args, rank):
    """Differentiation workload: a batch of cells with a log-normal shear
    modulus mu(x) = exp(g(x)) (g a seeded Gaussian random field, squared-
    exponential correlation length 8 voxels, std 1.5, mean 0), nu = 0.3;
    forward FP32 + FP64 refinement to args.grad_tol, then the gradient of
    C_1212 with respect to mu(x) by the adjoint autograd.Function, checked
    against central differences (h = 1e-4 relative) of the same solver on
    seeded random directions and seeded voxels of the first cell."""
    import numpy as np
    import torch

    from janus_b200 import microstructures as micro
    from janus_b200.gradients import StiffnessFieldProblem, effective_shear_modulus

    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    n, B = args.grad_n, args.grad_batch
    mus = torch.stack([torch.from_numpy(np.exp(micro.gaussian_field(
        n, dim=3, corr_len=8.0, std=1.5, seed=replica_seed(rank) + b))) for b in range(B)])
    mus = mus.cuda()
    mu0 = [0.5 * float(m.min() + m.max()) for m in mus]
    prob = StiffnessFieldProblem(nu=0.3, tol=args.grad_tol, max_iter=400000, mixed=True,
                                 inner=args.krylov_inner, inner_method="bicgstab")
    # warm: kernels, tables
    effective_shear_modulus(mus[0, :16, :16, :16].contiguous(), StiffnessFieldProblem(
        nu=0.3, tol=1e-4))
    torch.cuda.synchronize()
    m = mus.clone().requires_grad_(True)
    a = torch.cuda.Event(enable_timing=True)
    b_ = torch.cuda.Event(enable_timing=True)
    c_ = torch.cuda.Event(enable_timing=True)
    a.record()
    c = effective_shear_modulus(m, prob, batched=True)
    b_.record()
    c.sum().backward()
    c_.record()
    torch.cuda.synchronize()
    t_fwd = a.elapsed_time(b_) / 1e3
    t_bwd = b_.elapsed_time(c_) / 1e3
    stats = list(prob.stats)
    nvox = n ** 3
    fwd_appl = sum(it for kind, it, _ in stats if kind == "forward")
    adj_appl = sum(it for kind, it, _ in stats if kind == "adjoint")
    grad = m.grad[0].detach()
    # central differences on cell 0 (mu0 held fixed, as in the gradient)
    p0 = StiffnessFieldProblem(nu=0.3, tol=args.fd_tol, max_iter=400000, mixed=True,
                               inner=args.krylov_inner, inner_method="bicgstab", mu0=mu0[0])
    rng = np.random.default_rng(7)

    def c1212(mu):
        with torch.no_grad():
            return float(effective_shear_modulus(mu, p0))

    dirs = []
    for _ in range(args.grad_dirs):
        d = torch.from_numpy(rng.standard_normal((n, n, n))).cuda()
        vals = [c1212(mus[0] * (1 + s * 1e-4 * d)) for s in (1.0, -1.0)]
        fd = (vals[0] - vals[1]) / 2e-4
        an = float((grad * mus[0] * d).sum())
        dirs.append({"fd": fd, "adjoint": an, "rel_err": abs(fd - an) / abs(an)})
    vox = []
    gmax = float(grad.abs().max())
    for v in rng.choice(nvox, args.grad_voxels, replace=False):
        idx = np.unravel_index(int(v), (n, n, n))
        h = 1e-4 * float(mus[0][idx])
        vals = []
        for s in (1.0, -1.0):
            mp = mus[0].clone()
            mp[idx] += s * h
            vals.append(c1212(mp))
        fd = (vals[0] - vals[1]) / (2 * h)
        an = float(grad[idx])
        vox.append({"voxel": [int(i) for i in idx], "fd": fd, "adjoint": an,
                    "err_rel_to_max": abs(fd - an) / gmax})
    line = {"metric": "gradient of C_1212 w.r.t. mu(x): forward + adjoint time",
            "unit": "s", "n_gpus": 1, "higher_is_better": False, "data": "synthetic",
            "config": {"workload": f"{B} cells {n}^3, mu = exp(g), g Gaussian (corr 8, std 1.5), "
                                   f"nu 0.3, mu0 mid-range, truncated, tol {args.grad_tol}, "
                                   f"mixed FP32 BiCGSTAB (inner {args.krylov_inner})",
                       "cells": B, "grid": [n, n, n]},
            "contrast_max": float(max(float(m_.max() / m_.min()) for m_ in mus)),
            "forward_s": round(t_fwd, 3), "backward_s": round(t_bwd, 3),
            "forward_voxel_iter_per_s": fwd_appl * nvox / t_fwd,
            "adjoint_voxel_iter_per_s": adj_appl * nvox / t_bwd,
            "operator_applications": {"forward": fwd_appl, "adjoint": adj_appl},
            "C_1212": [float(v) for v in c.detach().cpu()],
            "fd_tol": args.fd_tol,
            "final_residual_max": {k: max(r for kind, _, r in prob.stats + p0.stats if kind == k)
                                   for k in ("forward", "adjoint")},
            "fd_final_residual_max": max(r for _, _, r in p0.stats) if p0.stats else None,
            "fd_directions": dirs, "fd_voxels": vox}
    print(json.dumps(line), flush=True)


def run_kernels(args, rank):
    """Every product entry point once, 3D (128^3) and 2D (1024^2), FP64 and
    FP32, on fields larger than L2 where the call allows: the launch set an
    ncu pass reads for per-kernel DRAM traffic and duration.  Prints the list
    of calls made."""
    import numpy as np
    import torch

    import janus_b200.material.elastic.linear.isotropic as material
    from janus_b200 import _lib
    from janus_b200 import microstructures as micro
    from janus_b200 import operators as ops
    from janus_b200.fft.serial import create_real
    from janus_b200.gradients import _gradient
    from janus_b200.green import filtered, truncated, willot2015
    from janus_b200.solvers import GMRES, BasicScheme, MixedScheme

    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    calls = []
    rng = np.random.default_rng(0)
    for shape in ((128, 128, 128), (1024, 1024)):
        dim = len(shape)
        s = 3 if dim == 2 else 6
        phase = (rng.random(shape) < 0.3).astype(np.uint8)
        mat0 = material.create(50.5, 0.3, dim)
        pars = [(dim * (material.create(g, nu, dim).k - mat0.k), 2 * (g - 50.5))
                for g, nu in ((1.0, 0.3), (100.0, 0.2))]
        tens = [ops.isotropic_4(a, b, dim) for a, b in pars]
        for dt in (torch.float64, torch.float32):
            tag = "{}D/{}".format(dim, "f64" if dt == torch.float64 else "f32")
            # FFT objects: r2c / c2r of one scalar field
            fft = create_real(shape, dtype=dt)
            x = torch.from_numpy(rng.standard_normal(shape)).to("cuda", dt)
            c = fft.r2c(x)
            fft.c2r(c)
            calls.append(tag + " fft r2c/c2r")
            # Green operators on two fields (batch), every variant
            xf = torch.from_numpy(rng.standard_normal((2,) + shape + (s,))).to("cuda", dt)
            for f in (truncated, filtered, willot2015):
                g = f(mat0.green_operator(), shape, 1.0, dtype=dt)
                g.apply_batch(xf)
                calls.append(tag + " green apply " + f.__name__)
            g = filtered(mat0.green_operator(), shape, 1.0, dtype=dt)
            b = torch.from_numpy(rng.integers(0, shape[0], size=(1 << 20, dim)).astype(np.int32))
            tau = torch.from_numpy(rng.standard_normal((1 << 20, s, 2))).to("cuda", dt)
            g.apply_by_freq_device(b, tau)
            calls.append(tag + " green apply_by_freq_device")
            # local operators: phase map (isotropic, matrices), per-voxel blocks
            loc = (ops.BlockDiagonalOperator2D if dim == 2 else ops.BlockDiagonalOperator3D
                   ).from_phases(phase, tens, dtype=dt)
            y = torch.empty_like(xf)
            loc.local.apply_device(xf, y, batch=2)
            mats = np.stack([t.to_memoryview() for t in tens])
            locm = ops.LocalPhaseOperator(dim, shape, phase, None, None, dt, matrices=mats)
            locm.apply_device(xf, y, batch=2)
            a = torch.from_numpy(rng.standard_normal(shape + (s, s))).to("cuda", dt)
            lin = (ops.BlockDiagonalLinearOperator2D if dim == 2
                   else ops.BlockDiagonalLinearOperator3D)(a, dtype=dt)
            lin.apply(xf[0])
            lin.apply_transpose(xf[0])
            calls.append(tag + " local (phase, matrices), block linear (+transpose)")
            # solver steps (local + Green + update + residual), mean stress
            E = np.eye(s)[:2]
            sol = BasicScheme(g, loc, nload=2)
            r = sol.run(E, 2)
            calls.append(tag + " basic scheme (fill, passes, residual, mean)")
            if dt == torch.float64:
                for method in ("basic", "bicgstab"):
                    MixedScheme(g, loc, nload=2, inner=2, method=method).run(
                        E, tol=1e-30, max_outer=2)
                    calls.append(tag + " mixed scheme " + method)
                # two cycles of GMRES(3): Arnoldi steps, restart, update
                GMRES(g, loc, nload=2, restart=3).run(E, tol=1e-30, max_iter=5)
                calls.append(tag + " gmres")

                class _Cell:
                    pass
                cell = _Cell()
                cell.dim, cell.shape, cell.dsph_dmu = dim, shape, 1.0
                _gradient(cell, r.eps, r.eps.clone())
                calls.append(tag + " local gradient")
            torch.cuda.synchronize()
    # the 256-point tiles (rows, plain columns, in-place Green columns): one
    # truncated-operator basic-scheme iteration on one 256^3 field per precision
    shape = (256, 256, 256)
    phase = (rng.random(shape) < 0.3).astype(np.uint8)
    mat0 = material.create(50.5, 0.3, 3)
    pars = [(3 * (material.create(g, nu, 3).k - mat0.k), 2 * (g - 50.5))
            for g, nu in ((1.0, 0.3), (100.0, 0.2))]
    tens = [ops.isotropic_4(a, b, 3) for a, b in pars]
    for dt in (torch.float64, torch.float32):
        loc = ops.BlockDiagonalOperator3D.from_phases(phase, tens, dtype=dt)
        g = truncated(mat0.green_operator(), shape, 1.0, dtype=dt)
        BasicScheme(g, loc, nload=1).run(np.eye(6)[:1], 1)
        calls.append("3D 256^3/{} basic scheme (truncated)".format(
            "f64" if dt == torch.float64 else "f32"))
        del loc, g
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    print(json.dumps({"workload": "kernels", "calls": calls}), flush=True)


def run_passes2d(args, rank):
    """Per-pass device times of one basic-scheme step on n x n 2D grids
    (filtered, 3 load cases, 30% inclusions), n in --passes2d-n, FP64 and
    FP32: ms per pass (CUDA events around each pass, mean of --steps steps
    after --warmup) and the fraction of measured HBM bandwidth from the
    algorithmic bytes 2sp + 1 (r2c with the phase map), 2sp (Green pass), 3sp
    (c2r with the update) per voxel and load case."""
    import numpy as np
    import torch

    import janus_b200.material.elastic.linear.isotropic as material
    from janus_b200 import autotune
    from janus_b200 import operators as ops
    from janus_b200.green import filtered
    from janus_b200.solvers import BasicScheme

    peak, _ = measured_peak()
    for n in [int(v) for v in args.passes2d_n.split(",")]:
        for dt in (torch.float64, torch.float32):
            rng = np.random.default_rng(0)
            phase = (rng.random((n, n)) < 0.3).astype(np.uint8)
            mat0 = material.create(50.5, 0.3, 2)
            tens = [ops.isotropic_4(2 * (material.create(g, nu, 2).k - mat0.k), 2 * (g - 50.5), 2)
                    for g, nu in ((1.0, 0.3), (100.0, 0.2))]
            loc = ops.BlockDiagonalOperator2D.from_phases(phase, tens, dtype=dt)
            g = filtered(mat0.green_operator(), (n, n), 1.0, dtype=dt)
            sol = BasicScheme(g, loc, 3)
            sol.set_load(np.eye(3))
            eps = sol.new_field()
            res = torch.zeros(3, dtype=torch.float64, device=eps.device)
            t = autotune._time_passes(sol, eps, res, max(args.steps, 5), max(args.warmup, 3))
            p = 8 if dt == torch.float64 else 4
            vox = 3 * n * n
            alg = {"rows_r2c_local": (2 * 3 * p + 1) * vox, "cols_green_axis0": 2 * 3 * p * vox,
                   "rows_c2r_update": 3 * 3 * p * vox}
            out = {k: {"ms": round(v, 4),
                       "frac": round(alg[k] / (v * 1e-3) / 1e9 / peak, 3) if k in alg else None}
                   for k, v in t.items()}
            print(json.dumps({"workload": "passes2d", "n": n, "dtype": str(dt)[6:],
                              "passes": out}), flush=True)
            del sol, eps, g, loc
            torch.cuda.empty_cache()


def run_reference(args, rank):
    if rank != 0:
        return
    n = args.n
    results = run_cpu_workers(n, 2024, list(range(6)), args.warmup + args.steps, args.variant,
                              "ref")
    kind = results[0]["kind"]
    t = max(sum(r["times"][args.warmup:]) for r in results)
    value = 6 * n ** 3 * args.steps / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3D two-phase random spheres {n}^3 (radius {8 * n // 128}, "
                               "vf 0.3, seeded RSA), mu 1/100, nu 0.3/0.2, mu0 50.5, "
                               f"{args.variant} Green operator, 6 load cases, basic scheme",
                   "grid": [n, n, n], "load_cases": 6, "variant": args.variant,
                   "precision": "f64", "parallelism": "6 single-threaded processes"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 6,
                         "kind": "reference" if kind.startswith("reference") else "port",
                         "label": CPU_LABELS[kind],
                         "sample": f"{args.steps} timed iterations (after {args.warmup}) of "
                                   f"each of the 6 load cases at {n}^3, one process per load "
                                   "case (the reference's serial path is single-threaded)",
                         "host_cpu": host_cpu(), "fftw_probe": fftw_probe()[1]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="janus_b200", choices=["janus_b200", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--variant", default="filtered", choices=["filtered", "truncated"])
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--solve-max-iter", type=int, default=3000)
    ap.add_argument("--inner", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the column-schedule autotuner (built-in rules)")
    ap.add_argument("--workload", default="spheres3d",
                    choices=["spheres3d", "batch2d", "voronoi", "gradients", "kernels",
                             "passes2d"],
                    help="spheres3d: the headline step; batch2d: batched 2D cells; "
                         "voronoi: mixed vs FP64 time-to-solution on a 3D Voronoi cell")
    ap.add_argument("--passes2d-n", default="256,512,768,1024",
                    help="grid sizes of the passes2d workload")
    ap.add_argument("--voronoi-n", type=int, default=256)
    ap.add_argument("--grad-n", type=int, default=128)
    ap.add_argument("--grad-batch", type=int, default=8)
    ap.add_argument("--grad-tol", type=float, default=1e-8)
    ap.add_argument("--grad-dirs", type=int, default=4)
    ap.add_argument("--grad-voxels", type=int, default=32)
    ap.add_argument("--fd-tol", type=float, default=1e-13,
                    help="residual of the central-difference solves")
    ap.add_argument("--contrast", type=float, default=1000.0)
    ap.add_argument("--voronoi-loads", type=int, default=1)
    ap.add_argument("--voronoi-variants", default="truncated,filtered")
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--batch-tol", type=float, default=1e-8)
    ap.add_argument("--no-sequential", action="store_true")
    ap.add_argument("--batch-branches", type=int, default=8)
    ap.add_argument("--inner-method", default="basic", choices=["basic", "bicgstab"],
                    help="inner solver of the batched mixed scheme")
    ap.add_argument("--gmres-restart", type=int, default=20,
                    help="restart length of the FP64 GMRES time-to-solution leg")
    ap.add_argument("--krylov-inner", type=int, default=25,
                    help="BiCGSTAB iterations per defect-correction step")
    # internal: CPU worker process
    ap.add_argument("--cpu-worker", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--seed", type=int, default=2024, help=argparse.SUPPRESS)
    ap.add_argument("--load", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--iters", type=int, default=1, help=argparse.SUPPRESS)
    ap.add_argument("--out", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--field", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--fftw", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--no-target", action="store_true",
                    help="skip the time-to-solution target leg (256^3 Voronoi)")
    ap.add_argument("--target-n", type=int, default=256)
    args = ap.parse_args(argv)
    if args.warmup < 0 or args.steps < 1:
        ap.error("steps must be >= 1 and warmup >= 0")

    if args.cpu_worker:
        cpu_worker(args.n, args.seed, args.load, args.iters, args.variant, args.out,
                   args.field, args.fftw)
        return

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank)
        return

    if args.workload == "batch2d":
        if rank == 0:
            run_batch2d(args, rank, world)
        return
    if args.workload == "voronoi":
        if rank == 0:
            run_voronoi(args, rank)
        return
    if args.workload == "gradients":
        if rank == 0:
            run_gradients(args, rank)
        return
    if args.workload == "kernels":
        if rank == 0:
            run_kernels(args, rank)
        return
    if args.workload == "passes2d":
        if rank == 0:
            run_passes2d(args, rank)
        return

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(env_int("LOCAL_RANK", 0))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        run_gpu(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
