#!/usr/bin/env python
"""Benchmark: BEM solves/s of the per-frequency Nemoh solve on B200.

Workload (one "step"): the rectangular barge 100 x 20 m, draft 10 m, water
depth 50 m, y-symmetric half mesh of 2,400 panels, 40 frequencies
omega = 0.05..2.5 rad/s, 9 problems per frequency (headings 0/45/90 deg and
6 radiation DOFs). One solve = one (mesh, omega) system: assembly of D+/-,
S+/-, factorization of both symmetry classes, all 9 right-hand sides, the
boundary potential and the force integration. A step = the 40 solves.

Default (`--impl ours`): the mixed-precision path is the headline `value`
(solves/s with inputs resident on the GPU); the FP64 GPU path is timed beside
it (`fp64`) and the mixed result's error against it is reported per
coefficient family. `e2e` times the C-ABI call with host (pinned) buffers,
host<->device copies included. `--impl reference` times the reference's CPU
algorithm (the FP64 oracle restatement, faithful loop structure) on a bounded
sample per host core.

Multi-GPU: frequencies are independent, so each rank solves its own copy of
the 40-frequency workload (weak scaling, no data-path collective).
"""
import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_OMEGA = 40
NPROB = 9


def build_workload(n_omega=None):
    """The barge workload; n_omega < 40 keeps an evenly spaced subset (profiling)."""
    from nemoh_b200 import cases as C
    case = C.config_barge(n_omega=N_OMEGA)
    if n_omega and n_omega < N_OMEGA:
        case.omegas = case.omegas[np.linspace(0, N_OMEGA - 1, n_omega).round().astype(int)]
    nw = len(case.omegas)
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    nvel = np.asfortranarray(nv.reshape(nv.shape[0], nw, npb).transpose(0, 2, 1))
    nds = np.asfortranarray(C.generalised_normals(case))
    return case, nvel, nds


ASM_PROFILE = "profiles/assembly_counters_barge_4omega.md"


def assembly_counters():
    """Per-pair counts of the assembly passes from the committed ncu summary:
    the line `counters:` holds key=value pairs (FP64 FLOP executed per (I, J)
    pair by the Rankine pass of each depth regime, which runs once per call,
    and by the wave pass of each regime per frequency; DRAM bytes per pair of
    each). None when the summary is absent."""
    p = os.path.join(ROOT, ASM_PROFILE)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("counters:"):
            return {k: float(v) for k, v in (kv.split("=") for kv in line.split()[1:])}
    return None


def roofline_line(hbm_achieved, hbm_peak, hbm_src, traffic, alg_bytes, fp64):
    """The assembly passes' roofline: the binding roof is the FP64 pipe (their
    executed FP64 FLOP over the phase's time against the measured FMA peak);
    the HBM view beside it. Without the counters summary, the HBM view only."""
    kernel = ("rankine_cache_kernel (once per depth regime) + wave_sym_kernel (per frequency): "
              "influence-matrix assembly, FP64")
    hbm_view = {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_achieved / hbm_peak,
                "peak_source": hbm_src, "algorithmic_bytes_per_frequency": alg_bytes,
                "traffic": traffic, "traffic_unit": "DRAM bytes per frequency (ncu counts per pair, " + ASM_PROFILE + ")"}
    if fp64.get("achieved_tflops") and fp64.get("peak_tflops"):
        return {"bound": "fp64", "kernel": kernel, "achieved": fp64["achieved_tflops"], "peak": fp64["peak_tflops"],
                "unit": "TFLOP/s", "frac": fp64["frac"], "peak_source": fp64["peak_source"],
                "flop_source": fp64["flop_source"], "traffic": traffic,
                "traffic_unit": hbm_view["traffic_unit"], "hbm": hbm_view}
    out = dict(hbm_view, bound="hbm", kernel=kernel)
    out["fp64"] = fp64
    return out


def fp64_peak_tflops(device):
    import nemoh_b200 as nb
    L = nb.load_library()
    L.nemoh_b200_diag_fp64_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    v = ctypes.c_double()
    return v.value if L.nemoh_b200_diag_fp64_peak(int(device), ctypes.byref(v)) == 0 else None


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of one GPU during the timed
    region: read through NVML every 20 ms, or from `nvidia-smi -lms 200` where
    the NVML bindings are missing. Reads only; no GPU setting is changed."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event bits of hw_slowdown, hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    BITS = (0x8, 0x40, 0x20, 0x4)

    def __init__(self, index, period=0.02, nvml=None):
        self.index = index
        self.period = period
        self.rows = []
        self.proc = None
        self.nv = nvml
        self.stop = threading.Event()

    def __enter__(self):
        try:
            if self.nv is None:
                import pynvml
                self.nv = pynvml
            self.nv.nvmlInit()
            self.h = self.nv.nvmlDeviceGetHandleByIndex(self.index)
            self.mx = self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM)
            self.sample()   # one sample before the region starts, so a short region still has one
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def sample(self):
        """One NVML reading in the row layout of the nvidia-smi query."""
        nv = self.nv
        sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
        self.rows.append([str(self.index), str(sm), str(self.mx), "", ""] +
                         ["Active" if bits & b else "Not Active" for b in self.BITS])

    def _poll(self):
        while not self.stop.wait(self.period):
            try:
                self.sample()
            except Exception:
                return

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.nv is not None:
            self.stop.set()
            self.t.join(timeout=5)
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample(case, seconds):
    """The oracle (reference CPU algorithm, 1 core) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    L = O.lib()
    L.nemoh_oracle_sample_solve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                            ctypes.POINTER(ctypes.c_double)]
    L.nemoh_oracle_sample_solve.restype = ctypes.c_double
    m = case.mesh
    o = O.Oracle(m.nodes, m.panels, m.isym, case.rho, case.g, case.depth, cache_s=False)
    om = case.omegas
    kw = om * om / case.g
    fd = ~((case.depth == 0.0) | (kw * case.depth >= 20))
    picks = [(om[fd][len(om[fd]) // 2], int(fd.sum())), (om[~fd][len(om[~fd]) // 2], int((~fd).sum()))]
    total, detail = 0.0, []
    for w, count in picks:
        if count == 0:
            continue
        d = (ctypes.c_double * 8)()
        est = L.nemoh_oracle_sample_solve(o.h, float(w), NPROB, seconds / 2, d)
        if est < 0:
            raise RuntimeError("oracle sample failed")
        total += est * count
        detail.append({"omega": float(w), "solves": count, "s_per_solve": est, "s_per_pair": d[0],
                       "s_per_cmac": d[1]})
    return len(om) / total, detail


def max_over_ranks(ms, dist=None, device="cpu"):
    """The slowest rank's time: every rank times its own copy of the workload
    between barriers, and the job is done when the last rank is."""
    if dist is None:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, ms):
    """Units per second of the whole job: every rank processes its own units in
    `ms` (the max over ranks), so the job rate is world x units / time."""
    return world * units_per_rank / (ms / 1e3)


def single_gpu_extras(rank, world):
    """The CPU baseline sample and the single-GPU workloads beside the headline
    (output stages, batched bodies, serving streams) run once, on rank 0 of a
    one-GPU job: with more ranks they would only hold the other GPUs idle."""
    return rank == 0 and world == 1


def run_reference(args):
    """--impl reference: the reference CPU algorithm on all host threads.

    Default (a run of a few minutes): every step runs on every host thread
    the bounded per-core sample of `cpu_sample` (whole rows of Green
    evaluations and the first GAUSSZ elimination steps for one finite-depth and
    one deep-water frequency, timed, and extrapolated by operation counts to
    the 40-frequency workload); the step's rate is the sum over threads.

    --whole-solves: every timed step runs whole solves instead, one
    single-frequency case of the workload per host thread (the frequencies
    spread over the 40-frequency set, so the finite-depth / deep-water mix
    follows the workload's), each through the oracle executable in the
    reference's own loop structure (`faithful`), all threads at once; the
    step's rate is the sum over threads of 1 / (that thread's solve time).
    A whole solve takes minutes per thread, so this form is for a measurement
    run, not for the default."""
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from nemoh_b200 import cases as C
    case = C.config_barge(n_omega=N_OMEGA)
    cores = os.cpu_count() or 1
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            model = next((l.split(":", 1)[1].strip() for l in f if l.startswith("model name")), "")
    except OSError:
        pass
    per_step = float(os.environ.get("NEMOH_REF_SAMPLE_S", "8"))
    ctx = mp.get_context("spawn")
    times = []
    whole = None
    with ctx.Pool(cores) as pool:
        for step in range(args.warmup + (0 if args.whole_solves else args.steps)):
            t0 = time.time()
            res = pool.map(_ref_worker, [per_step] * cores)
            if step >= args.warmup:
                times.append((time.time() - t0, sum(r[0] for r in res)))
    if args.whole_solves:
        whole = whole_solves(case, cores, args.steps)
        times = [(max(d), sum(1.0 / t for t in d)) for d in whole["steps"]]
    value = float(np.mean([r for _, r in times]))
    if whole:
        sample = ("timed whole solves: per step one single-frequency case of the workload per host thread "
                  "(%d threads, %s), each the full faithful oracle solve at N=2400 with its 9 problems; "
                  "finite depth %.1f s and deep water %.1f s per solve (mean over threads)"
                  % (cores, model or "cpu", whole["t_fd"], whole["t_deep"]))
    else:
        sample = ("per thread per step (%d threads, %s): whole rows of Green evaluations and the first GAUSSZ "
                  "elimination steps at N=2400 for one finite-depth and one deep-water omega (%.0f s), timed and "
                  "extrapolated by operation counts to the 40-omega workload; --whole-solves times whole "
                  "solves instead" % (cores, model or "cpu", per_step))
    line = {
        "impl": "reference", "metric": "BEM solves/s (mixed vs FP64 GPU, rel err<=1e-6) at N=2400; serve p50/p99 ms",
        "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean([t for t, _ in times])) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "barge 100x20x10 m, depth 50 m, half mesh N=2400 (y-symmetric), 40 omega x 9 problems",
                   "n_panels": 2400, "omegas": N_OMEGA, "problems_per_omega": NPROB},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def whole_solves(case, threads, steps):
    """`steps` rounds of whole faithful oracle solves, one single-frequency
    case per host thread at once (frequency i * 40 / threads for thread i);
    returns each round's per-thread solve times and the mean finite-depth and
    deep-water times."""
    import tempfile
    import shutil
    from nemoh_b200 import cases as C
    exe = os.path.join(ROOT, "oracle", "_build", "nemoh_oracle")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    kw = case.omegas ** 2 / case.g
    fd = ~((case.depth == 0.0) | (kw * case.depth >= 20))
    pick = [i * N_OMEGA // threads for i in range(threads)] if threads < N_OMEGA else \
        [i % N_OMEGA for i in range(threads)]
    tmp = tempfile.mkdtemp(prefix="nemoh_ref_")
    rounds = []
    try:
        dirs = []
        for i, w in enumerate(pick):
            c = C.config_barge(n_omega=N_OMEGA)
            c.omegas = case.omegas[[w]]
            d = os.path.join(tmp, "t%03d" % i)
            C.write_case(c, d)
            dirs.append(d)
        for _ in range(steps):
            t0 = time.time()
            done = [None] * threads
            procs = [subprocess.Popen([exe, d, "faithful"], stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
                     for d in dirs]

            def wait(i):
                procs[i].wait()
                done[i] = time.time() - t0

            ths = [threading.Thread(target=wait, args=(i,)) for i in range(threads)]
            for t in ths:
                t.start()
            for t in ths:
                t.join()
            bad = [i for i, p in enumerate(procs) if p.returncode != 0]
            if bad:
                raise RuntimeError("oracle solve failed on thread %d: %s" % (bad[0], procs[bad[0]].stderr.read()))
            rounds.append(done)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    t_fd = [t for d in rounds for i, t in enumerate(d) if fd[pick[i]]]
    t_deep = [t for d in rounds for i, t in enumerate(d) if not fd[pick[i]]]
    return {"steps": rounds, "t_fd": float(np.mean(t_fd)) if t_fd else float("nan"),
            "t_deep": float(np.mean(t_deep)) if t_deep else float("nan")}


def _ref_worker(seconds):
    from nemoh_b200 import cases as C
    return cpu_sample(C.config_barge(n_omega=N_OMEGA), seconds)


def rel_err_families(F, F64, nbeta):
    """Per coefficient: |x - x64| / max(|x64|, 1e-6 * family max).

    A family is one force component and one problem over all frequencies
    (force(i, j) or excitation(i, beta) over omega). Families whose largest
    value is at most 1e-9 of the largest coefficient of the same kind
    (diffraction or radiation) vanish by the body's symmetry -- both paths
    hold round-off there, e.g. heave-surge coupling of a body symmetric in x
    and y -- and are measured against 1e-6 of that kind maximum instead.
    """
    a = np.abs(F64)
    fam = a.max(axis=2, keepdims=True)
    kind = np.empty_like(fam)
    kind[:, :nbeta] = a[:, :nbeta].max()
    kind[:, nbeta:] = a[:, nbeta:].max()
    floor = np.where(fam <= 1e-9 * kind, 1e-6 * kind, np.maximum(a, 1e-6 * fam))
    err = np.abs(F - F64) / floor
    return float(err.max()), float(np.median(err))


def _dof_name(d):
    axis = int(np.argmax(np.abs(np.asarray(d.direction, dtype=float))))
    return (("surge", "sway", "heave"), ("roll", "pitch", "yaw"))[d.icase - 1][axis] + (
        "" if d.body == 1 else "%d" % d.body)


def _part_err(x, x64):
    """|x - x64| / max(|x64|, 1e-6 * family max), families over the last axis,
    vanishing families (at most 1e-9 of the block's largest value) against
    1e-6 of the block maximum; the largest over the frequencies."""
    a = np.abs(x64)
    fam = a.max(axis=-1, keepdims=True)
    top = a.max()
    floor = np.where(fam <= 1e-9 * top, 1e-6 * top, np.maximum(a, 1e-6 * fam))
    return (np.abs(x - x64) / floor).max(axis=-1)


def coefficient_errors(F, F64, case):
    """Mixed against FP64 per coefficient: for every force component the
    largest relative error over the frequencies of the excitation force per
    heading, of the added mass (real part of the radiation force) and of the
    damping (imaginary part) per radiating degree of freedom. F[force,
    problem, omega], the diffraction problems first."""
    nb = len(case.betas_deg)
    forces = [_dof_name(d) for d in case.force]
    rad = [_dof_name(d) for d in case.rad]
    r2 = lambda v: float("%.2g" % v)
    exc = _part_err(F[:, :nb], F64[:, :nb])
    am = _part_err(F[:, nb:].real, F64[:, nb:].real)
    dmp = _part_err(F[:, nb:].imag, F64[:, nb:].imag)
    return {"forces": forces,
            "excitation": {"beta=%g" % b: [r2(exc[i, k]) for i in range(len(forces))]
                           for k, b in enumerate(case.betas_deg)},
            "added_mass": {r: [r2(am[i, k]) for i in range(len(forces))] for k, r in enumerate(rad)},
            "damping": {r: [r2(dmp[i, k]) for i in range(len(forces))] for k, r in enumerate(rad)}}


def _body_inputs(case):
    from nemoh_b200 import cases as C
    nw = len(case.omegas)
    nv = C.body_conditions(case)
    npb = len(case.betas_deg) + len(case.rad)
    nvel = np.asfortranarray(nv.reshape(nv.shape[0], nw, npb).transpose(0, 2, 1))
    return nvel, np.asfortranarray(C.generalised_normals(case))


def run_batched(local, n_bodies, n_omega=20, seed=4, steps=2):
    """Batched workload: n_bodies bodies from the seeded generator (cylinder, box
    or sphere, 200..3000 panels, infinite or 20..200 m depth), 20 frequencies
    0.1..2.5 rad/s, 6 DOF + heading 0 each. The bodies are resident on the
    device (nemoh_b200_add_body, not timed); one step is one
    nemoh_b200_solve_bodies call over all n_bodies x 20 (body, omega) items
    with host buffers (copies included): items of different bodies share
    ragged batches sized by free device memory. One untimed warm-up step, then
    `steps` timed steps (host wall clock)."""
    import nemoh_b200 as nb
    from nemoh_b200 import cases as C
    rng = np.random.default_rng(seed)
    omegas = np.linspace(0.1, 2.5, n_omega)
    cases, nvels = [], []
    for _ in range(n_bodies):
        mesh, depth = C.random_body(rng)
        case = C.Case(mesh, omegas, np.array([0.0]), C.six_dofs(), C.six_dofs(), depth=depth)
        nvel, _ = _body_inputs(case)
        cases.append(case)
        nvels.append(nvel)
    items_b = np.repeat(np.arange(n_bodies), n_omega)
    items_w = np.tile(omegas, n_bodies)
    items_v = [nvels[b][:, :, w] for b in range(n_bodies) for w in range(n_omega)]
    out, F = {}, {}
    for label, mode in (("fp64", nb.FP64), ("mixed", nb.MIXED)):
        with nb.Solver(local, mode) as s:
            for case in cases:
                s.add_body(case)
            res = s.solve_bodies(items_b, items_w, items_v)   # warm-up: workspace, kernel attributes
            t0 = time.perf_counter()
            for _ in range(steps):
                res = s.solve_bodies(items_b, items_w, items_v)
            dt = (time.perf_counter() - t0) / steps
            t = s.last_timings()
            # the same calls replayed as CUDA graphs: the first call in graph
            # mode runs directly, the second is captured, later ones replay
            s.set_graphs(True)
            for _ in range(2):
                s.solve_bodies(items_b, items_w, items_v)
            t0 = time.perf_counter()
            for _ in range(steps):
                rg = s.solve_bodies(items_b, items_w, items_v)
            dtg = (time.perf_counter() - t0) / steps
            cap, rep = s.graph_stats()
            fb = s.fallback_count()
        F[label] = [np.stack(res[b * n_omega:(b + 1) * n_omega], axis=2) for b in range(n_bodies)]
        out[label + "_solves_per_s"] = n_bodies * n_omega / dt
        out[label + "_s"] = dt
        out[label + "_phase_ms"] = {"assemble": t["assemble_ms"], "factor_solve": t["factor_ms"], "lu": t["lu_ms"],
                                    "solve": t["solve_ms"]}
        out[label + "_graph_solves_per_s"] = n_bodies * n_omega / dtg
        if mode == nb.MIXED:
            out["mixed_fp64_fallback"] = {"batches": fb[0], "systems": fb[1], "calls": 3 + steps * 2}
        out[label + "_graph"] = {"captured": cap, "replayed": rep,
                                 "max_diff_vs_direct": float(max(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
                                                                 for a, b in zip(rg, res)))}
    errs = [rel_err_families(a, b, 1)[0] for a, b in zip(F["mixed"], F["fp64"])]
    npan = [c.mesh.npanels for c in cases]
    out.update({"bodies": n_bodies, "omegas_per_body": n_omega, "solves": n_bodies * n_omega, "steps": steps,
                "panels_min": int(min(npan)), "panels_max": int(max(npan)), "panels_median": float(np.median(npan)),
                "finite_depth_bodies": int(sum(c.depth > 0 for c in cases)),
                "mixed_speedup": out["fp64_s"] / out["mixed_s"], "mixed_vs_fp64_max_rel_err": float(max(errs)),
                "path": "nemoh_b200_solve_bodies: all bodies and frequencies in one call, ragged batches",
                "timing": "host wall clock per call, host<->device copies included"})
    return out


def run_two_spheres(local, n_omega=30):
    """Precision workload: two floating spheres R=4 m, centres 20 m apart, deep
    water, 8,000 quad panels (quadrangulated icospheres, seed 3), 12 DOF + 2
    headings, 30 frequencies 0.2..3.0 rad/s: one step = the 30 solves through
    nemoh_b200_solve_frequencies_device (inputs resident on the device), FP64
    and mixed precision, CUDA events; the mixed result's error against FP64
    per coefficient."""
    import torch
    import nemoh_b200 as nb
    from nemoh_b200 import cases as C
    case = C.config_two_spheres(n_omega=n_omega)
    nvel_h, nds_h = _body_inputs(case)
    nc, nrhs, nw = nvel_h.shape
    nint = nds_h.shape[0]
    dev = torch.device("cuda", local)
    nvel_d = torch.from_numpy(np.ascontiguousarray(nvel_h.transpose(2, 1, 0)).view(np.float64)).to(dev)
    nds_d = torch.from_numpy(np.ascontiguousarray(nds_h.T)).to(dev)
    force_d = torch.zeros((nw, nrhs, nint, 2), dtype=torch.float64, device=dev)
    out, F = {"n_panels": case.mesh.npanels, "omegas": nw, "problems_per_omega": nrhs}, {}
    om = case.omegas.astype(np.float64)
    for label, mode in (("fp64", nb.FP64), ("mixed", nb.MIXED)):
        with nb.Solver(local, mode) as s:
            s.set_case(case)
            s.solve_frequencies_device(om, nvel_d.data_ptr(), nrhs, nint, nds_d.data_ptr(),
                                       force_d.data_ptr())   # warm-up: workspace, kernel attributes, tuning
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            s.solve_frequencies_device(om, nvel_d.data_ptr(), nrhs, nint, nds_d.data_ptr(), force_d.data_ptr())
            e1.record()
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1)
            t = s.last_timings()
            Fh = force_d.cpu().numpy()
            F[label] = (Fh[..., 0] + 1j * Fh[..., 1]).transpose(2, 1, 0)
            out[label] = {"solves_per_s": nw / (ms / 1e3), "ms_per_step": ms,
                          "phase_ms": {"assemble": t["assemble_ms"], "factor_solve": t["factor_ms"],
                                       "lu": t["lu_ms"], "solve": t["solve_ms"]}}
            if mode == nb.MIXED:
                out[label]["refinement"] = dict(zip(("iterations", "residual"), s.last_refinement()))
    N = case.mesh.npanels
    err_max, err_med = rel_err_families(F["mixed"], F["fp64"], len(case.betas_deg))
    lu_flop = 8.0 / 3.0 * N ** 3 * nw
    out.update({"mixed_speedup": out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"],
                "mixed_vs_fp64_max_rel_err": err_max, "mixed_vs_fp64_median_rel_err": err_med,
                "lu_effective_tflops": {k: lu_flop / (out[k]["phase_ms"]["lu"] / 1e3) / 1e12
                                        for k in ("fp64", "mixed") if out[k]["phase_ms"]["lu"] > 0},
                "mesh": "icosphere frequency 12 cut 0.055 R below the centre, 3 quads per triangle, 4,000 per "
                        "sphere, node jitter: areas within 10%, seed 3",
                "timing": "CUDA events around one 30-frequency call, inputs on the device"})
    return out


def _wall(fn, reps):
    fn()   # warm-up (workspace growth, first-touch)
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    return (time.perf_counter() - t0) / reps


def run_outputs(local, omega_index=10):
    """The solver's output stages beside the solve, on the barge at one
    finite-depth frequency and its 9 problems, each timed through the C-ABI
    with host buffers (copies included): Kochin function at 361 directions,
    free-surface elevation on the pre-processor's 101 x 101 grid over
    400 m x 400 m, the pre-processor's body conditions for the 40 x 9 problems,
    and the post-processor's impulse response functions (40 frequencies,
    6 x 6 coefficients, 1,000 time steps). Beside each, the CPU oracle (one
    core) on a bounded sample of the same work, scaled to the same unit."""
    import nemoh_b200 as nb
    from nemoh_b200 import cases as C
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    case = C.config_barge(n_omega=N_OMEGA)
    w = float(case.omegas[omega_index])
    T = 2 * np.pi / w
    nv = C.body_conditions(case)
    cols = range(omega_index * NPROB, (omega_index + 1) * NPROB)
    out = {"omega": w, "problems": NPROB, "n_panels": case.mesh.npanels,
           "timing": "host wall clock around the C-ABI call, host<->device copies included"}
    m = case.mesh
    with nb.Solver(local, nb.FP64) as s:
        s.set_case(case)
        res = [s.solve_potential(T, nv[:, j]) for j in cols]
        zigb = np.stack([r["zigb"] for r in res], axis=1)
        zigs = np.stack([r["zigs"] for r in res], axis=1)
        theta = np.linspace(0.0, 2 * np.pi, 361)
        t = _wall(lambda: s.kochin(T, theta, zigb, zigs), 5)
        out["kochin"] = {"directions": 361, "ms": t * 1e3, "unit": "directions x problems / s",
                         "value": 361 * NPROB / t}
        pts, _ = C.freesurface_grid(101, 101, 400.0, 400.0)
        t = _wall(lambda: s.free_surface(T, pts, zigb, zigs), 3)
        out["free_surface"] = {"points": len(pts), "ms": t * 1e3, "unit": "points x problems / s",
                               "value": len(pts) * NPROB / t,
                               "green_pairs_per_s": len(pts) * m.npanels / t}
        t = _wall(lambda: s.body_conditions(case), 5)
        out["body_conditions"] = {"problems": case.nproblems, "ms": t * 1e3, "unit": "problems / s",
                                  "value": case.nproblems / t}
        rng = np.random.default_rng(1)
        wv = np.linspace(0.05, 2.5, 40)
        Bc = rng.standard_normal((40, 6, 6)) * np.exp(-wv)[:, None, None]
        Ac = rng.standard_normal((40, 6, 6))
        t = _wall(lambda: s.irf(wv, Bc, Ac, 1000, 0.1), 5)
        out["irf"] = {"nw": 40, "pairs": 36, "ntime": 1000, "ms": t * 1e3}
    # CPU oracle on bounded samples (one core)
    o = O.Oracle(m.nodes, m.panels, m.isym, case.rho, case.g, case.depth)
    th8 = theta[:8]
    t = _wall(lambda: o.kochin(T, th8, zigb, zigs), 1)
    out["kochin"]["cpu_oracle_value"] = 8 * NPROB / t
    t = _wall(lambda: o.free_surface(T, pts[:64], zigb[:, :1], zigs[:, :1]), 1)
    out["free_surface"]["cpu_oracle_value"] = 64 / t
    t = _wall(lambda: (C.body_conditions(case), C.generalised_normals(case), C.froude_krylov(case)), 1)
    out["body_conditions"]["cpu_host_value"] = case.nproblems / t
    t = _wall(lambda: O.irf(wv, Bc, Ac, 1000, 0.1), 1)
    out["irf"]["cpu_oracle_ms"] = t * 1e3
    out["cpu"] = ("oracle (C++, 1 core) on 8 directions x 9 problems / 64 points x 1 problem, scaled; body conditions: "
                  "the numpy pre-processor restatement in nemoh_b200.cases")
    del o
    return out


def tc_split():
    """Operand split of the mixed LU's tensor-core updates (NEMOH_B200_TC_SPLIT)."""
    return "f16" if os.environ.get("NEMOH_B200_TC_SPLIT") == "f16" else "bf16"


def run_serving(local, n_bodies, n_req, rates=(0.25, 0.5, 0.75, 0.9, 1.0, 1.2), seed=5, n_check=64, workers=2):
    """Serving workload: Poisson request streams over the batched workload's
    bodies (one omega U(0.1, 2.5), heading U(0, 180) deg, 6 DOF per request)
    through the continuous-batching server (resident bodies, right-hand sides
    built on the device, cross-body batches). The saturation throughput is the
    median of the rates achieved on three streams offered well above capacity
    (one such stream's rate varies by tens of percent between runs with the
    batches the workers happen to take); streams at fractions of it then give
    the latency percentiles."""
    import nemoh_b200 as nb
    from nemoh_b200 import serving as S
    bodies = S.make_bodies(n_bodies, seed=4)
    srv = S.SolveServer(bodies, device=local, precision=nb.MIXED, workers=workers)
    try:
        srv.run(S.make_requests(min(256, n_req), 0, n_bodies, seed=seed + 100), realtime=False)   # warm-up
        sats = []
        for k in range(3):
            done, wall = srv.run(S.make_requests(min(n_req, 4000), 1e6, n_bodies, seed=seed + 1000 * k))
            sats.append(len(done) / wall)
        sat = float(np.median(sats))
        out = {"bodies": n_bodies, "requests_per_rate": n_req, "workers": workers, "precision": "mixed",
               "saturation_solves_per_s": sat, "saturation_streams_solves_per_s": sats, "rates": []}
        last = None
        for f in rates:
            done, wall = srv.run(S.make_requests(n_req, f * sat, n_bodies, seed=seed + int(100 * f)))
            st = S.latency_stats(done, wall, expected=n_req)
            st.update({"rate_frac": f, "offered_per_s": f * sat,
                       "mean_batch": float(np.mean([b[2] for b in srv.batches])),
                       "mean_bodies_per_batch": float(np.mean([b[1] for b in srv.batches]))})
            out["rates"].append(st)
            last = done
    finally:
        srv.close()
    # per-request error against the FP64 path on a sample of the last stream
    worst = 0.0
    check = sorted(last, key=lambda r: r.rid)[:n_check]
    with nb.Solver(local, nb.FP64) as s:
        for b in bodies:
            bid = s.add_body(b.case)
            s.set_body_dofs(bid, b.case.rad)
        f64s = s.solve_requests(np.array([r.body for r in check]), np.array([r.omega for r in check]),
                                np.radians([r.beta_deg for r in check]))
    for r, f64 in zip(check, f64s):
        a = np.abs(f64)
        # one frequency per request: each coefficient against itself, or
        # against 1e-6 of its kind's largest value where it vanishes by symmetry
        floor = np.empty_like(a)
        for cols in (slice(0, 1), slice(1, 7)):
            k = a[:, cols].max()
            floor[:, cols] = np.where(a[:, cols] <= 1e-9 * k, 1e-6 * k, a[:, cols])
        worst = max(worst, float((np.abs(r.force - f64) / floor).max()))
    out["mixed_vs_fp64_max_rel_err"] = worst
    out["checked_requests"] = len(check)
    out["latency"] = "host clock from arrival to result ready"
    return out


def run_ours(args):
    import torch
    import nemoh_b200 as nb
    from nemoh_b200 import build as B

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    B.build()
    case, nvel_h, nds_h = build_workload(args.omegas)
    nomega = len(case.omegas)
    dev = torch.device("cuda", local)
    omegas = case.omegas.astype(np.float64)
    nc, nrhs, nw = nvel_h.shape
    nint = nds_h.shape[0]
    # device-resident inputs (column-major layouts as the C-ABI expects)
    nvel_d = torch.from_numpy(np.ascontiguousarray(nvel_h.transpose(2, 1, 0)).view(np.float64)).to(dev)
    nds_d = torch.from_numpy(np.ascontiguousarray(nds_h.T)).to(dev)
    force_d = torch.zeros((nw, nrhs, nint, 2), dtype=torch.float64, device=dev)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    results = {}
    for label, mode in (("fp64", nb.FP64), ("mixed", nb.MIXED)):
        s = nb.Solver(local, mode)
        s.set_case(case)
        for _ in range(args.warmup):
            s.solve_frequencies_device(omegas, nvel_d.data_ptr(), nrhs, nint, nds_d.data_ptr(), force_d.data_ptr())
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        phase = np.zeros(4)
        l0 = s.launches
        with ClockSampler(local) as clk:
            barrier()
            ev0.record()
            for _ in range(args.steps):
                s.solve_frequencies_device(omegas, nvel_d.data_ptr(), nrhs, nint, nds_d.data_ptr(),
                                           force_d.data_ptr())
                t = s.last_timings()
                phase += [t["assemble_ms"], t["factor_ms"], t["solve_ms"], t["lu_ms"]]
            ev1.record()
            barrier()
        launches = s.launches - l0
        ms = max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
        F = force_d.cpu().numpy()
        F = (F[..., 0] + 1j * F[..., 1]).transpose(2, 1, 0)
        results[label] = dict(ms=ms / args.steps, phase=phase / args.steps, launches=launches, F=F,
                              clocks=clk.summary(), solver=s, refinement=s.last_refinement())
    # end-to-end through the C-ABI with pinned host buffers
    s = results["mixed"]["solver"]
    pin_nvel = torch.from_numpy(np.ascontiguousarray(nvel_h.transpose(2, 1, 0)).view(np.float64)).pin_memory()
    pin_nds = torch.from_numpy(np.ascontiguousarray(nds_h.T)).pin_memory()
    pin_force = torch.zeros((nw, nrhs, nint, 2), dtype=torch.float64).pin_memory()
    L = nb.load_library()
    dp = ctypes.POINTER(ctypes.c_double)
    om_arr = np.ascontiguousarray(omegas)

    def e2e_call():
        st = L.nemoh_b200_solve_frequencies(s._h, nw, om_arr.ctypes.data_as(dp), nrhs,
                                            ctypes.cast(pin_nvel.data_ptr(), dp), nint,
                                            ctypes.cast(pin_nds.data_ptr(), dp), ctypes.cast(pin_force.data_ptr(), dp))
        if st:
            raise RuntimeError("solve_frequencies failed: %d" % st)

    for _ in range(args.warmup):
        e2e_call()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        e2e_call()
    e1.record()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)

    mx, f64 = results["mixed"], results["fp64"]
    err_max, err_med = rel_err_families(mx["F"], f64["F"], len(case.betas_deg))
    value = whole_job_rate(world, nomega, mx["ms"])
    hbm, tc, src = peaks()
    # Dominant kernels of the mixed step: the two assembly passes (FP64 Green
    # functions). Algorithmic bytes = the influence matrices written, 4 x 16 N^2
    # per frequency, plus the FP32 copy of D+ and D- (2 x 8 N^2) that the wave
    # pass writes for the mixed LU, over the assembly phase's CUDA-event time.
    # The binding roof is the FP64 pipe: FP64 operations per pair as counted
    # by ncu on the current kernels (committed summary), over the same time,
    # against the FP64 FMA throughput measured here.
    N = case.mesh.npanels
    asm_ms = mx["phase"][0]
    asm_bytes = (4 * 16.0 + 2 * 8.0) * N * N * nomega
    achieved = asm_bytes / (asm_ms / 1e3) / 1e9
    kw = case.omegas ** 2 / case.g
    n_fd = int((~((case.depth == 0.0) | (kw * case.depth >= 20))).sum())
    cnt = assembly_counters()
    fp64_peak = fp64_peak_tflops(local)
    fp64 = {"peak_tflops": fp64_peak,
            "peak_source": "measured in this run (nemoh_b200_diag_fp64_peak: FMA chains on every SM)"}
    traffic = None
    keys = ("rankine_fd_flop", "rankine_deep_flop", "wave_fd_flop", "wave_deep_flop", "rankine_dram_bytes",
            "wave_fd_dram_bytes", "wave_deep_dram_bytes")
    if cnt and all(k in cnt for k in keys):
        # per step: the Rankine part once per depth regime met, the wave pass per frequency
        pairs, n_deep = N * N, nomega - n_fd
        flop = pairs * ((n_fd > 0) * cnt["rankine_fd_flop"] + (n_deep > 0) * cnt["rankine_deep_flop"] +
                        n_fd * cnt["wave_fd_flop"] + n_deep * cnt["wave_deep_flop"])
        traffic = pairs * (((n_fd > 0) + (n_deep > 0)) * cnt["rankine_dram_bytes"] + n_fd * cnt["wave_fd_dram_bytes"]
                           + n_deep * cnt["wave_deep_dram_bytes"]) / nomega
        ach = flop / (asm_ms / 1e3) / 1e12
        fp64.update({"achieved_tflops": ach, "frac": ach / fp64_peak if fp64_peak else None,
                     "flop_source": "FP64 instructions (DFMA x2, DADD, DMUL) per pair executed by the current "
                                    "kernels, ncu, " + ASM_PROFILE})
    line = {
        "metric": "BEM solves/s (mixed vs FP64 GPU, rel err<=1e-6) at N=2400; serve p50/p99 ms",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mx["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 assembly / f32 LU, tensor-core updates on split-%s operands / f64 refinement" % tc_split(),
        "data": "synthetic",
        "config": {"workload": "barge 100x20x10 m, depth 50 m, half mesh N=2400 (y-symmetric), 40 omega x 9 problems",
                   "n_panels": N, "omegas": nomega, "problems_per_omega": NPROB, "precision": "mixed",
                   "l2": "working set 15 GB of matrices per step, larger than L2 (no flush needed)"},
        "fp64": {"value": whole_job_rate(world, nomega, f64["ms"]), "unit": "solves/s", "ms_per_step": f64["ms"],
                 "phase_ms": {"assemble": f64["phase"][0], "factor_solve": f64["phase"][1], "lu": f64["phase"][3],
                              "solve": f64["phase"][2]}},
        "mixed_vs_fp64": {"max_rel_err": err_max, "median_rel_err": err_med, "speedup": f64["ms"] / mx["ms"],
                          "per_coefficient": coefficient_errors(mx["F"], f64["F"], case)},
        "phase_ms": {"assemble": mx["phase"][0], "factor_refine": mx["phase"][1], "lu": mx["phase"][3],
                     "solve": mx["phase"][2]},
        "refinement": dict(zip(("iterations", "residual"), mx["refinement"])),
        "sweep_choice": {"mixed": nb.sweep_choice(N, nomega * 2, NPROB, True)[0],
                         "fp64": nb.sweep_choice(N, nomega * 2, NPROB, False)[0],
                         "codes": "1-8: cluster sweep of that cluster size, 16: dataflow sweep"},
        "pipeline_pct": int(os.environ.get("NEMOH_B200_PIPELINE", "0")),
        "roofline": roofline_line(achieved, hbm, src, traffic, 80.0 * N * N, fp64),
        "e2e": {"value": whole_job_rate(world, nomega, e2e_ms), "unit": "solves/s",
                "h2d_bytes_per_step": int(pin_nvel.numel() * 8 + pin_nds.numel() * 8),
                "d2h_bytes_per_step": int(pin_force.numel() * 8)},
        "gpu_launches": int(mx["launches"]),
        "clocks": mx["clocks"],
    }
    if single_gpu_extras(rank, world) and not args.no_cpu:
        rate, detail = cpu_sample(case, args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": "solves/s", "cores": 1, "kind": "port",
                                "sample": "1 core: whole rows of Green evaluations and the first GAUSSZ elimination "
                                          "steps at N=2400 for one finite-depth and one deep-water omega "
                                          "(%.0f s total), extrapolated by operation counts to 40 omega; "
                                          "cross-checked against whole faithful solves timed on a B200 box's "
                                          "host core (finite depth 101.6 s, deep water 75.8 s per solve: "
                                          "0.0104 solves/s per core over the 40 omega)" % args.cpu_seconds}
    for r in results.values():
        r["solver"].close()
    results = {}
    if single_gpu_extras(rank, world) and not args.no_extras:
        for key, fn in (("outputs", lambda: run_outputs(local)),
                        ("two_spheres", lambda: run_two_spheres(local)),
                        ("batched", lambda: run_batched(local, args.bodies)),
                        ("serve", lambda: run_serving(local, args.bodies, args.requests))):
            if key not in args.extras.split(","):
                continue
            try:
                line[key] = fn()
            except Exception as e:   # reported in the line; the headline stands on its own
                line[key] = {"error": "%s: %s" % (type(e).__name__, e)}
    if rank == 0:
        print(json.dumps(line))
    for r in results.values():
        r["solver"].close()
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=16.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--omegas", type=int, default=N_OMEGA, help="frequency subset (profiling only)")
    ap.add_argument("--no-extras", action="store_true", help="skip the workloads beside the headline")
    ap.add_argument("--extras", default="outputs,two_spheres,batched,serve",
                    help="comma list of the workloads beside the headline to run")
    ap.add_argument("--bodies", type=int, default=256, help="bodies of the batched and serving workloads")
    ap.add_argument("--requests", type=int, default=10000, help="requests per serving rate")
    ap.add_argument("--whole-solves", action="store_true",
                    help="--impl reference: time whole faithful oracle solves (minutes per step)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
