#!/usr/bin/env python
"""UVLM time-step throughput on B200.

Workload (the configuration the headline metric is quoted on): free-wake UVLM, 16 x 128
bound panels (AIC 2048 x 2048), 200 wake rows (25 600 wake rings), linear twist and
NACA camber from a seeded RNG, cutoff kernel with core radius 1e-3 c, started from the
static solution.  A "step" is one UVLM time step (case_solve).

value   steps/s of the mixed-precision path (FP32 Biot-Savart, FP32 factors + FP64
        refinement), device-timed with CUDA events per step, L2 flushed between steps
        (a 256 MB write outside the timed events), max over ranks.
e2e     the same metric through the C ABI with host buffers: every step copies its node
        frames from pinned host memory, runs fj_solve_prescribed_dynamic, and reads the
        step's solution slot back to pinned host memory.
fp64_gpu  the plain FP64 path on the same steps, and the mixed path's CL/CD error
        against it.
autotune  the split counts of the step's three Biot-Savart sums, timed on the device before
        the timed regions (fj_autotune_vind) for both precisions, against the wave-filling
        rule the launches use untuned.
linear  the linearised UVLM at C1 size (8x32, W=64, frozen wake): assembly time of A, B, C,
        D on the device and a short march (--linear runs only this leg, with C1 prescribed
        and C3 as well, and a 1000-step march).
factorisation  the mixed solve's FP32 LU + FP32 inverse of this workload's AIC through the
        tensor-core path (tcgen05 TF32, three-pass split; the default) and through the FP32
        CUDA-core path, and the tensor-core GEMM alone at the LU's trailing-update shape
        (--factor runs only this leg).

--impl reference  times the FP64 oracle (the reference's arithmetic restated; the
        reference itself is JAX, which is not installed) with its pair sums in C++/OpenMP on
        every host thread, full time steps of the same workload, and prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "UVLM time-steps/s (free wake 16x128, W=200)"
UNIT = "steps/s"
FLOPS_PER_PAIR = 70.0  # Biot-Savart convention: FMA = 2, rsqrt/div = 1 per (target, filament)
VIND32_TRAFFIC_BYTES = 3.33e6  # DRAM bytes of one vind32 launch of this workload, from an ncu capture


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--small", action="store_true", help="a reduced workload (for quick checks)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only the autotuned, timed mixed steps, no other legs (for profiler runs)")
    ap.add_argument("--serving-cases", type=int, default=512, help="cases in the serving stream (0: skip)")
    ap.add_argument("--only-serving", action="store_true")
    ap.add_argument("--adjoint", action="store_true",
                    help="config 3: twist gradient of time-mean CL and CD by the hand-written adjoint")
    ap.add_argument("--adjoint-steps", type=int, default=1000)
    ap.add_argument("--residual", action="store_true",
                    help="only the time-step residual VJP (timestep_residual, config-3 wing) on the device")
    ap.add_argument("--linear", action="store_true",
                    help="only the linearised UVLM leg: A, B, C, D about the static solution (C1 and C3 wings, "
                         "frozen and prescribed wakes) and the linear system's time march")
    ap.add_argument("--factor", action="store_true",
                    help="only the factorisation leg (mixed solve's FP32 LU + inverse, tensor cores vs CUDA cores)")
    ap.add_argument("--configs", action="store_true",
                    help="the per-config table instead of the headline line: C1 heave 8x32/W64/50 steps, "
                         "C2 free wake 16x128/W200, C3 pitch 12x64/W100 primal")
    return ap.parse_args()


def workload(args, n_steps):
    from flapjax_b200 import cases

    if args.small:
        return cases.wing_free(m=8, n=32, m_star=40, n_steps=n_steps)
    return cases.wing_free(n_steps=n_steps)


# --------------------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0}
        loaded = [v for v in sm if v > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------------------
def make_case(case, precision, n_slots):
    import flapjax_b200 as fj

    kernel = fj.cutoff_kernel(case.r_cut) if case.kernel == "cutoff" else fj.biot_savart_epsilon
    uv = fj.UVLM([fj.GridDiscretisation(case.m, case.n, case.m_star)], np.arange(case.n + 1), kernel=kernel,
                 free_wake=case.free_wake, precision=precision)
    ff = fj.Constant(case.u_inf, case.rho, True)
    uv.set_design_variables(dt=case.dt, flowfield=ff, zeta_b0=case.zeta_b0, hg0=case.hg0)
    init = uv.solve_static()
    dc = uv.make_device_case(n_slots)
    uv.load_initial(dc, init)
    dc.set_hg(case.hg_t[:n_slots], case.hg_dot_t[:n_slots])
    return uv, dc


def coeffs(ft, case):
    a = np.deg2rad(case.alpha_deg)
    q = 0.5 * case.rho * case.u_mag**2 * case.s_ref
    return ft @ np.array((-np.sin(a), 0.0, np.cos(a))) / q, ft @ np.array((np.cos(a), 0.0, np.sin(a))) / q


def run_device_steps(dc, first, last, flush, torch, profile=False):
    """Steps first..last-1 one call each; returns per-step device ms (events) and the
    profile of the Biot-Savart kernels if requested."""
    from flapjax_b200 import _lib

    stream = torch.cuda.current_stream()
    times = []
    prof = _lib.FjProfile()
    if profile:
        _lib.call("fj_profile_begin")
    for i in range(first, last):
        if flush is not None:
            flush.fill_(i & 0xFF)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dc.solve_dynamic(i, i + 1, reuse_factors=i > 1)
        e1.record(stream)
        times.append((e0, e1))
    torch.cuda.synchronize()
    if profile:
        _lib.call("fj_profile_end", C_byref(prof))
    return [a.elapsed_time(b) for a, b in times], prof


def C_byref(x):
    import ctypes

    return ctypes.byref(x)


def e2e_run(uv, dc, case, first, last, torch, chunk=8):
    """Per step: H2D of the step's frames (pinned), the step through the C ABI, D2H of the
    step's solution slot (pinned).  The C ABI call advances `chunk` steps at a time (it
    synchronises once per call to report a zero pivot, a NaN or a failed refinement of
    any of its steps).  The copies run on a second stream: the next chunk's frames go up
    while a chunk computes, and its slots come back while the next chunk computes
    (results double-buffered in pinned memory).  The compute stream waits on the uploads
    before each call and on the last read-back before the closing event, so the one
    timed region (two events around the loop) holds every step's copies and compute.
    Returns ([ms of the loop], bytes in per step, bytes out per step)."""
    n_nodes = case.hg0.shape[0]
    hg = torch.from_numpy(np.ascontiguousarray(case.hg_t)).pin_memory()
    hgd = torch.from_numpy(np.ascontiguousarray(case.hg_dot_t)).pin_memory()
    fields = list(dc.arrays)
    outs = [{k: torch.empty(dc.arrays[k].shape[1], dtype=torch.float64).pin_memory() for k in fields}
            for _ in range(2 * chunk)]
    out_ft = [torch.empty(3, dtype=torch.float64).pin_memory() for _ in range(2 * chunk)]
    main = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    bytes_in = 2 * n_nodes * 16 * 8
    bytes_out = sum(v.numel() * 8 for v in outs[0].values()) + 3 * 8
    up = {i: torch.cuda.Event() for i in range(first, last)}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(main)
    copy.wait_event(e0)

    def upload(i0, i1):
        with torch.cuda.stream(copy):
            for i in range(i0, i1):
                dc.hg_t[i].copy_(hg[i], non_blocking=True)
                dc.hg_dot_t[i].copy_(hgd[i], non_blocking=True)
                up[i].record(copy)

    upload(first, min(first + chunk, last))
    for c0 in range(first, last, chunk):
        c1 = min(c0 + chunk, last)
        main.wait_event(up[c1 - 1])  # the copy stream uploads in order
        dc.solve_dynamic(c0, c1, reuse_factors=c0 > 1)
        done = torch.cuda.Event()
        done.record(main)
        upload(c1, min(c1 + chunk, last))
        with torch.cuda.stream(copy):
            copy.wait_event(done)
            for i in range(c0, c1):
                o = outs[(i - first) % (2 * chunk)]
                for k in fields:
                    o[k].copy_(dc.arrays[k][i], non_blocking=True)
                out_ft[(i - first) % (2 * chunk)].copy_(dc.force_total[i], non_blocking=True)
    main.wait_stream(copy)
    e1.record(main)
    torch.cuda.synchronize()
    return [e0.elapsed_time(e1)], bytes_in, bytes_out


def _cpu_uvlm(case):
    from oracle import uvlm_cpp as CP
    from oracle import uvlm_ref as R

    uv = CP.UVLMCpp([(case.m, case.n, case.m_star)], np.arange(case.n + 1), kernel=case.kernel, r_cut=case.r_cut,
                    free_wake=case.free_wake)
    uv.set_design_variables(case.dt, R.Constant(case.u_inf, case.rho, True), case.zeta_b0, case.hg0)
    return uv


def cpu_steps(case, threads, warmup, max_steps, budget_s):
    """Full UVLM time steps of the workload on the host: the FP64 oracle with its
    induced-velocity sums and AIC assembly in C++/OpenMP (``threads`` threads, SIMD over
    filaments) and the dense solve in LAPACK.  Static solve, ``warmup`` untimed steps,
    then up to ``max_steps`` timed steps while the budget lasts."""
    from oracle import uvlm_cpp as CP

    CP.set_threads(threads)
    uv = _cpu_uvlm(case)
    st = uv.solve_static()
    n_slots = min(case.hg_t.shape[0], 1 + warmup + max_steps)
    cs = uv._empty_case(n_slots)
    for key in ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
                "f_unsteady", "alpha"):
        for arr, val in zip(getattr(cs, key), getattr(st, key)):
            arr[0] = val[0]
    times = []
    for i in range(1, n_slots):
        t0 = time.perf_counter()
        uv.case_step(cs, i, case.hg_t[i], case.hg_t[i - 1], case.hg_dot_t[i])
        if i > warmup:
            times.append(time.perf_counter() - t0)
            if sum(times) >= budget_s:
                break
    return len(times) / sum(times), times


def cpu_single_thread(case, budget_s):
    """One-thread pair rate of the C++ oracle's induced-velocity sum (the free-wake
    convection targets against the bound and wake lattices), scaled to steps/s by the
    pairs of one step; the sums are > 99 % of a CPU step at this size."""
    from oracle import uvlm_cpp as CP

    CP.set_threads(1)
    zb = case.zeta_b0 + case.hg0[0, :3, 3]
    w = case.m_star
    zw = zb[-1][None] + np.arange(w + 1)[:, None, None] * (case.dt * case.u_inf)[None, None, :]
    rng = np.random.default_rng(0)
    gb = rng.normal(size=(case.m, case.n)) * 0.1
    gw = rng.normal(size=(w, case.n)) * 0.1
    targets = zw[:-1].reshape(-1, 3)
    filaments = sum(r * (c + 1) + (r + 1) * c for r, c in ((case.m, case.n), (w, case.n)))
    n_t, t0, chunk = 0, time.perf_counter(), 64
    while time.perf_counter() - t0 < budget_s and n_t < targets.shape[0]:
        CP.compute_v_ind(targets[n_t:n_t + chunk], [zb, zw], [gb, gw], case.kernel, None, case.r_cut)
        n_t += chunk
    el = time.perf_counter() - t0
    pairs = n_t * filaments
    return {"value": pairs / el / case.pairs_per_step(), "unit": UNIT, "cores": 1,
            "sample": f"induced velocity at {n_t} wake vertices from {filaments} filaments ({pairs:.3g} pairs in "
                      f"{el:.1f} s), scaled by {case.pairs_per_step():.4g} pairs per step",
            "pairs_per_s": pairs / el}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(case, budget_s):
    """cpu_baseline: full steps on all host threads plus the one-thread pair rate."""
    from flapjax_b200 import cases

    th = host_threads()
    cpu_case = cases.wing_free(m=case.m, n=case.n, m_star=case.m_star, n_steps=12, seed=case.seed)
    value, times = cpu_steps(cpu_case, th, 1, 10, budget_s)
    return {"value": value, "unit": UNIT, "cores": th, "kind": "port",
            "sample": f"C++/OpenMP FP64 oracle (uvlm_ref_cpu.cpp + LAPACK solve), static solve + 1 untimed step, "
                      f"then {len(times)} full time steps of the same workload on {th} threads "
                      f"({sum(times):.1f} s)",
            "step_s": times, "single_thread": cpu_single_thread(cpu_case, max(2.0, budget_s / 3))}


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import torch.distributed as dist

    from flapjax_b200 import _lib

    from flapjax_b200 import replicas

    rank, world, local = replicas.rank_env()
    torch.cuda.set_device(local)
    replicas.init("nccl")
    dev = torch.device("cuda", local)
    if args.configs:
        if rank == 0:
            print(json.dumps({"configs": config_table(args, torch)}))
        return 0
    if args.adjoint:
        if rank == 0:
            print(json.dumps({"adjoint": adjoint_bench(args, torch)}))
        return 0
    if args.residual:
        if rank == 0:
            print(json.dumps({"residual_vjp": residual_bench(torch)}))
        return 0
    if args.linear:
        if rank == 0:
            print(json.dumps({"linear": linear_bench(torch, small=args.small)}))
        return 0
    if args.factor:
        case = workload(args, 2)
        _, dcf = make_case(case, "mixed", 2)
        if rank == 0:
            print(json.dumps({"factorisation": factor_bench(dcf, case, torch)}))
        return 0
    if args.only_serving:
        serving = serving_bench(args, torch)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"serving": serving}))
        return 0
    assert args.warmup >= 3, "at least 3 warm-up steps"
    K, W = args.steps, args.warmup
    n_slots = 1 + W + K
    case = workload(args, n_slots - 1)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    # -- autotuning of the sum launches (outside every timed region) ----------------------
    from flapjax_b200 import tuning

    t_tune = time.perf_counter()
    kern = _lib.FJ_KERNEL_CUTOFF if case.kernel == "cutoff" else _lib.FJ_KERNEL_EPSILON
    shapes = tuning.step_shapes(case.m, case.n, case.m_star, case.free_wake)
    precs = ("mixed",) if args.kernels_only else ("mixed", "fp64")
    autotune = {p: tuning.autotune(shapes, p, kern, case.r_cut) for p in precs}
    autotune["seconds"] = time.perf_counter() - t_tune
    # -- mixed path: value ---------------------------------------------------------------
    uv, dc = make_case(case, "mixed", n_slots)
    run_device_steps(dc, 1, 1 + W, flush, torch)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.load().fj_launch_count()
    with ClockSampler(local) as clk:
        ms, prof = run_device_steps(dc, 1 + W, n_slots, flush, torch, profile=True)
    launches = _lib.load().fj_launch_count() - launches0
    torch.cuda.synchronize()
    t_ms = replicas.max_over_ranks(sum(ms), dev)
    if world > 1:
        dist.barrier()
    value = world * K / (t_ms * 1e-3)
    ft_mixed = dc.force_total[1 + W:n_slots].cpu().numpy()

    # -- roofline of the dominant kernel (Biot-Savart sums) -------------------------------
    peak = ctypes_peak(torch)
    # the FP32 sums only: the RHS's near-wake rows run in FP64 and are reported beside them
    v32_ms, v32_pairs = prof.vind_ms - prof.vind64_ms, prof.vind_pairs - prof.vind64_pairs
    achieved = v32_pairs * FLOPS_PER_PAIR / (v32_ms * 1e-3) / 1e12 if v32_ms > 0 else None
    roof = {"kernel": "vind32 (FP32 Biot-Savart sums)", "bound": "fp32", "achieved": achieved,
            "peak": peak, "unit": "TFLOP/s", "frac": (achieved / peak) if achieved and peak else None,
            "traffic": VIND32_TRAFFIC_BYTES,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the convection launch of this "
                              "workload (profiles/vind32_free_wake_16x128.md); the filament stream is the only "
                              "DRAM traffic, the rest stays in L2",
            "peak_source": "measured in-run (fj_peak_fp32: larger of scalar and packed FP32 FMA chains); "
                           "MEASURED_PEAKS.json has no FP32 CUDA-core figure",
            "pairs_per_launch": v32_pairs / max(prof.vind_launches - prof.vind64_launches, 1),
            "kernel_ms_per_step": v32_ms / K, "share_of_step": v32_ms / t_ms if t_ms else None,
            "pairs_per_s": v32_pairs / (v32_ms * 1e-3) if v32_ms > 0 else None,
            "fp64_near_wake_sums": {"ms_per_step": prof.vind64_ms / K, "pairs_per_step": prof.vind64_pairs / K,
                                    "share_of_step": prof.vind64_ms / t_ms if t_ms else None}}

    if args.kernels_only:
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_step": t_ms / K,
                              "steps": K, "warmup": W, "roofline": roof, "gpu_launches": int(launches),
                              "autotune": autotune, "note": "kernels only: no other legs"}))
        return 0

    # -- plain FP64 path and the mixed path's force-coefficient error -------------------
    # The free wake is chaotic: the FP64 path's own CL moves by many orders of magnitude
    # more than a 1e-13 input perturbation after a few dozen steps, so the trajectory error
    # is reported beside the one-step (local) error of the mixed step applied to FP64
    # states, and beside that FP64 self-sensitivity.
    fp64 = None
    if not args.no_fp64:
        _, d64 = make_case(case, "fp64", n_slots)
        run_device_steps(d64, 1, 1 + W, flush, torch)
        ms64, _ = run_device_steps(d64, 1 + W, n_slots, flush, torch)
        ft64 = d64.force_total[1 + W:n_slots].cpu().numpy()
        cl64, cd64 = coeffs(ft64, case)
        clm, cdm = coeffs(ft_mixed, case)
        # one-step error at sampled steps: mixed step from the FP64 state of slot i-1
        local, local_cd = [], []
        for i in np.linspace(1 + W, n_slots - 1, 5).astype(int):
            dc.copy_slot_from(d64, i - 1)
            dc.solve_dynamic(i, i + 1, reuse_factors=True)
            cl_i, cd_i = coeffs(dc.force_total[i].cpu().numpy()[None], case)
            cl_r, cd_r = coeffs(d64.force_total[i].cpu().numpy()[None], case)
            local.append(float(abs(cl_i[0] - cl_r[0]) / abs(cl_r[0])))
            local_cd.append(float(abs(cd_i[0] - cd_r[0]) / np.max(np.abs(cd64))))
        # FP64 self-sensitivity: the same run with zeta_b0 scaled by (1 + 1e-13)
        import copy as _copy

        cp = _copy.deepcopy(case)
        cp.zeta_b0 = case.zeta_b0 * (1.0 + 1e-13)
        _, dpp = make_case(cp, "fp64", n_slots)
        dpp.solve_dynamic(1, n_slots)
        clp, _ = coeffs(dpp.force_total[1 + W:n_slots].cpu().numpy(), case)
        fp64 = {"value": K / (sum(ms64) * 1e-3), "unit": UNIT, "ms_per_step": sum(ms64) / K,
                "speedup_mixed_over_fp64": (sum(ms64) / t_ms) if t_ms else None,
                "cl_rel_err_one_step_max": max(local),
                "cd_err_one_step_of_max_cd": max(local_cd),
                "cl_rel_err_traj_max": float(np.max(np.abs(clm - cl64) / np.abs(cl64))),
                "cd_rel_err_traj_max": float(np.max(np.abs(cdm - cd64)) / np.max(np.abs(cd64))),
                "fp64_cl_change_from_1e-13_input_perturbation": float(np.max(np.abs(clp - cl64) / np.abs(cl64)))}
        del d64, dpp
    factor = factor_bench(dc, case, torch) if not args.small else None
    del dc

    # -- e2e through the C ABI with host buffers -------------------------------------------
    e2e = None
    if not args.no_e2e:
        uv2, dce = make_case(case, "mixed", n_slots)
        e2e_run(uv2, dce, case, 1, 1 + W, torch)
        if world > 1:
            dist.barrier()
        ms_e, bi, bo = e2e_run(uv2, dce, case, 1 + W, n_slots, torch)
        te = replicas.max_over_ranks(sum(ms_e), dev)
        e2e = {"value": world * K / (te * 1e-3), "unit": UNIT, "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
               "copies": "each step's frames H2D and solution slot D2H (pinned) on a copy stream overlapping the "
                         "neighbouring chunk's compute; one event pair around the whole loop",
               "steps_per_call": 8}
        del dce

    torch.cuda.empty_cache()  # the serving budget is half of the free memory: return the cached blocks first
    serving = serving_bench(args, torch) if args.serving_cases > 0 else None
    # below capacity (about a sixth of what one GPU serves), so that latency is the step's
    # and not the queue's
    serving_low = serving_bench(args, torch, n=64, rate=10.0) if args.serving_cases > 0 else None
    linear = None
    if rank == 0 and not args.small:
        try:  # the linearised UVLM at C1 size (its own leg: --linear)
            linear = linear_bench(torch, small=True)
        except Exception as e:  # keep the headline line if this leg fails
            linear = {"error": f"{type(e).__name__}: {e}"}
    adjoint = None
    if rank == 0 and world == 1 and not args.small and args.adjoint_steps > 0:
        try:  # config 3's gradient on one GPU (its own leg: --adjoint)
            adjoint = adjoint_bench(args, torch)
        except Exception as e:  # keep the headline line if this leg fails
            adjoint = {"error": f"{type(e).__name__}: {e}"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    cpu = cpu_sample(case, args.cpu_seconds) if world == 1 else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32+fp64", "data": "synthetic (seeded wing geometry, no dataset)",
        "config": bench_config(case, args, world),
        "precision": "mixed (FP32 Biot-Savart with the first 4 wake rows of the RHS in FP64, FP32 factors + FP64 "
                     "refinement)",
        "e2e": e2e, "fp64_gpu": fp64, "roofline": roof, "cpu_baseline": cpu, "factorisation": factor,
        "gpu_launches": int(launches), "clocks": clk.summary(), "serving": serving,
        "serving_below_capacity": serving_low, "adjoint": adjoint, "autotune": autotune,
        "linear": linear,
    }
    print(json.dumps(line))
    return 0


def factor_bench(dc, case, torch):
    """The factorisation behind the mixed solve on this workload's own AIC (the bound
    lattice at slot 0, fj_aic_assemble): FP32 LU + FP32 inverse through each path
    (FJ_MIXED_FACTOR), device-timed per call with CUDA events, then the FP64-refined
    residual.  Beside it, the tensor-core GEMM alone at the LU's trailing-update shape
    (m = n = N - 128, k = 128, three passes) against the dense TF32 rate, taken as half the
    measured cuBLAS bf16 peak."""
    import ctypes as C

    from flapjax_b200 import _lib

    s = torch.cuda.current_stream().cuda_stream
    dev = torch.device("cuda", torch.cuda.current_device())
    m, n = case.m, case.n
    z = dc.arrays["zeta_b"][0].clone()
    nb = m * n
    zp = (C.c_void_p * 1)(z.data_ptr())
    mm, nn, ms = (C.c_int * 1)(m), (C.c_int * 1)(n), (C.c_int * 1)(0)
    nbytes = C.c_size_t()
    _lib.call("fj_aic_workspace_size", mm, nn, 1, C.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    a = torch.empty((nb, nb), dtype=torch.float64, device=dev)
    kern = _lib.FJ_KERNEL_CUTOFF if case.kernel == "cutoff" else _lib.FJ_KERNEL_EPSILON
    _lib.call("fj_aic_assemble", zp, mm, nn, 1, None, ms, None, None, kern, case.r_cut, a.data_ptr(), ws.data_ptr(),
              ws.numel(), s)
    b = torch.randn(nb, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))
    _lib.call("fj_solve_mixed_workspace_size", nb, C.byref(nbytes))
    wsm = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    x = torch.empty(nb, dtype=torch.float64, device=dev)
    res = torch.empty(1, dtype=torch.float64, device=dev)
    out = {"n": nb, "matrix": "AIC of the workload's bound lattice (slot 0)"}
    old = os.environ.get("FJ_MIXED_FACTOR")
    try:
        for mode in ("tf32x3", "tf32", "cuda"):
            os.environ["FJ_MIXED_FACTOR"] = mode
            times = []
            for it in range(6):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                _lib.call("fj_solve_mixed", a.data_ptr(), nb, b.data_ptr(), x.data_ptr(), 1, res.data_ptr(),
                          wsm.data_ptr(), wsm.numel(), s)
                e1.record()
                torch.cuda.synchronize()
                if it >= 2:
                    times.append(e0.elapsed_time(e1))
            out[mode] = {"factor_inverse_solve_ms": float(np.median(times)), "refined_rel_residual": float(res.item())}
    finally:
        if old is None:
            os.environ.pop("FJ_MIXED_FACTOR", None)
        else:
            os.environ["FJ_MIXED_FACTOR"] = old
    out["tensor_core_speedup_over_cuda_cores"] = (out["cuda"]["factor_inverse_solve_ms"] /
                                                   out["tf32x3"]["factor_inverse_solve_ms"])
    # the GEMM alone at the first trailing update's shape, through the factorisation's own
    # path (fj_gemm_tf32_tma: the hi/lo operand split, then the TMA-fed kernel; both inside
    # the events) and through the staged kernel (fj_gemm_tf32)
    g = max(nb - 128, 128)
    A = torch.randn((g, 128), dtype=torch.float32, device=dev)
    B = torch.randn((128, g), dtype=torch.float32, device=dev)
    Cm = torch.randn((g, g), dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    nf = C.c_size_t()
    _lib.call("fj_gemm_tf32_scratch_floats", g, g, 128, 3, C.byref(nf))
    scratch = torch.empty(nf.value, dtype=torch.float32, device=dev)
    peaks = measured_peaks()
    if "bf16_tflops" in peaks:
        tf32_peak = peaks["bf16_tflops"] / 2
        src = "half of measured MEASURED_PEAKS.json bf16_tflops (dense TF32 runs at half the bf16 rate)"
    else:
        tf32_peak = 1590.0 / 2
        src = "half of the fallback 1590 TFLOP/s bf16 (MEASURED_PEAKS.json absent; dense TF32 is half bf16)"

    def gemm_ms(path, calls):
        """Median over trials of the device time of `calls` back-to-back products, per call.
        With one call the host's work inside the call (tensor maps, launch set-up) shows
        as device idle time; with several, as in the factorisation, it overlaps the
        device's work."""
        times = []
        for it in range(8):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(calls):
                if path == "tma":
                    _lib.call("fj_gemm_tf32_tma", A.data_ptr(), 128, B.data_ptr(), g, Cm.data_ptr(), g, g, g, 128,
                              C.c_float(-1.0), C.c_float(1.0), 3, scratch.data_ptr(), scratch.numel(),
                              err.data_ptr(), s)
                else:
                    _lib.call("fj_gemm_tf32", A.data_ptr(), 128, B.data_ptr(), g, Cm.data_ptr(), g, g, g, 128,
                              C.c_float(-1.0), C.c_float(1.0), 3, err.data_ptr(), s)
            e1.record()
            torch.cuda.synchronize()
            if it >= 3:
                times.append(e0.elapsed_time(e1) / calls)
        return float(np.median(times))

    out["gemm"] = {"shape": [g, g, 128], "passes": 3, "tf32_peak_tflops": tf32_peak, "peak_source": src}
    for path in ("tma", "staged"):
        t1, t10 = gemm_ms(path, 1), gemm_ms(path, 10)
        achieved = 3 * 2.0 * g * g * 128 / (t10 * 1e-3) / 1e12
        out["gemm"][path] = {"ms": t10, "tflops_tf32_issued": achieved, "frac": achieved / tf32_peak,
                             "ms_single_call": t1, "timing": "10 calls back to back between events, per call"}
    out["gemm"]["tma"]["includes"] = "the operand split (one launch) and the TMA-fed product"
    return out


def residual_bench(torch):
    """Device time of one residual VJP (AeroResidual.vjp: the residual of the reference's
    timestep_residual and the cotangents of all its inputs) on the config-3 wing (12 x 64,
    W = 100, prescribed pitch) at slot 2, wall clock around the call (host algebra, transfers
    and device work), after one warm-up call."""
    import flapjax_b200 as fj
    from flapjax_b200 import cases
    from flapjax_b200.residual import AeroResidual

    c = cases.wing_pitch(m=12, n=64, m_star=100, n_steps=3)
    uv = fj.UVLM([fj.GridDiscretisation(c.m, c.n, c.m_star)], np.arange(c.n + 1), kernel=fj.biot_savart_epsilon,
                 precision="fp64")
    uv.set_design_variables(dt=c.dt, flowfield=fj.Constant(c.u_inf, c.rho, True), zeta_b0=c.zeta_b0, hg0=c.hg0)
    out = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    keys = ("gamma_b", "gamma_w", "gamma_b_dot", "zeta_w")
    q = lambda i: {k: [np.array(a[i]) for a in getattr(out, k)] for k in keys}
    ar = AeroResidual(uv)
    rng = np.random.default_rng(0)
    fb = rng.normal(size=(c.hg0.shape[0], 6))
    rbar = rng.normal(size=AeroResidual.ravel(q(2)).size + fb.size)
    args = (float(out.t[2]), c.hg_t[2], c.hg_dot_t[2], c.hg_t[1], q(2), q(1), fb, rbar)
    ar.vjp(*args)
    times = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r, _ = ar.vjp(*args)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    return {"workload": "config-3 wing 12x64, W=100, epsilon kernel, slot 2", "residual_size": int(r.size),
            "ms_per_vjp": 1e3 * float(np.median(times))}


def linear_bench(torch, small=False):
    """The linearised UVLM (aero/linear/linear_uvlm.py) about the static solution: wall time
    of the assembly of A, B, C, D on the device (the faster of two assemblies), the peak
    device memory, and the linear system's time march (x_n = A x_{n-1} + B u_n,
    y_n = C x_n + D u_n) over 1000 steps of seeded input perturbations, device-timed with
    CUDA events.  small: the C1 frozen-wake line only, with a 20-step march (the case the
    launch-list profile captures).  A line that runs out of device memory is recorded as
    such and the others still run."""
    out = []
    lines = (("C1 wing 8x32, W=64", (8, 32, 64), "frozen"), ("C1 wing 8x32, W=64", (8, 32, 64), "prescribed"),
             ("C3 wing 12x64, W=100", (12, 64, 100), "frozen"), ("C2 wing 16x128, W=200", (16, 128, 200), "frozen"))
    for label, (m, n, w), wt in lines[:1] if small else lines:
        torch.cuda.empty_cache()
        torch.cuda.reset_peak_memory_stats()
        try:
            out.append(_linear_line(torch, label, m, n, w, wt, 20 if small else 1000))
        except torch.cuda.OutOfMemoryError as e:
            out.append({"workload": f"{label}, {wt} wake", "error": f"OutOfMemoryError: {str(e)[:200]}"})
    torch.cuda.empty_cache()
    return out


def _linear_line(torch, label, m, n, w, wt, n_t):
    import flapjax_b200 as fj
    from flapjax_b200 import cases
    from flapjax_b200.linear import LinearUVLM

    c = cases.wing_heave(m=m, n=n, m_star=w, n_steps=1)
    uv = fj.UVLM([fj.GridDiscretisation(m, n, w)], np.arange(n + 1), kernel=fj.biot_savart_epsilon)
    uv.set_design_variables(dt=c.dt, flowfield=fj.Constant(c.u_inf, c.rho, True), zeta_b0=c.zeta_b0, hg0=c.hg0)
    lin = LinearUVLM(uv, uv.solve_static(), wt, skip_linearisation=True)
    times, sys_ = [], None
    for _ in range(2):
        sys_ = None  # one system alive at a time
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sys_ = lin.linearise()
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    peak = torch.cuda.max_memory_allocated() / 1e9
    rng = np.random.default_rng(0)
    u = torch.as_tensor(1e-4 * rng.normal(size=(n_t, lin.n_inputs))).cuda()
    sys_.run(u[:10])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sys_.run(u)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"workload": f"{label}, {wt} wake, epsilon kernel", "n_states": lin.n_states, "n_inputs": lin.n_inputs,
            "n_outputs": lin.n_outputs, "linearise_s": min(times),
            "matrix_bytes": 8 * (lin.n_states + lin.n_outputs) * (lin.n_states + lin.n_inputs),
            "peak_device_gb_assembly": peak, "run_steps_per_s": n_t / (ms * 1e-3),
            # the march reads A once per step (fj_lti_march); run() also does the B u, C x and D u
            # products, so this lower-bounds the march's own bandwidth
            "march_a_gbs": 8.0 * lin.n_states ** 2 * (n_t - 1) / (ms * 1e-3) / 1e9,
            "a_fits_l2": 8 * lin.n_states ** 2 < 126e6}


def measured_peaks():
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def config_table(args, torch):
    """Steps/s of the mixed and plain FP64 GPU paths and of the C++ FP64 oracle (1 thread
    and every host thread) on each single-case configuration, with the mixed path's CL/CD
    error against the FP64 path.  Prescribed wakes: the error over the whole run; the
    free wake (chaotic): the one-step error (FP64 state in, one mixed step)."""
    from flapjax_b200 import cases

    rows = {}
    specs = [("C1", cases.wing_heave(), 50), ("C2", cases.wing_free(n_steps=60), 60),
             ("C3", cases.wing_pitch(n_steps=200), 200)]
    for name, case, n_steps in specs:
        n_slots = n_steps + 1
        res = {"m": case.m, "n": case.n, "m_star": case.m_star, "steps": n_steps, "free_wake": case.free_wake,
               "pairs_per_step": case.pairs_per_step()}
        for prec in ("mixed", "fp64"):
            _, dc = make_case(case, prec, n_slots)
            run_device_steps(dc, 1, 4, None, torch)  # warm-up and the first (factorising) step
            # steps 4.. as one call (UVLM.solve_prescribed_dynamic): launched step by step,
            # then replayed from a captured step graph
            for graph in (False, True):
                st = torch.cuda.current_stream()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                dc.solve_dynamic(4, n_slots, reuse_factors=True, graph=graph)
                e1.record(st)
                e1.synchronize()
                ms = e0.elapsed_time(e1)
                key = prec if graph else f"{prec}_no_graph"
                res[f"{key}_steps_per_s"] = (n_slots - 4) / (ms * 1e-3)
                res[f"{key}_ms_per_step"] = ms / (n_slots - 4)
            res[f"_{prec}_dc"] = dc
        dm, d64 = res.pop("_mixed_dc"), res.pop("_fp64_dc")
        res["speedup_mixed_over_fp64"] = res["mixed_steps_per_s"] / res["fp64_steps_per_s"]
        cl64, cd64 = coeffs(d64.force_total[1:].cpu().numpy(), case)
        if case.free_wake:
            errs = []
            for i in np.linspace(2, n_slots - 1, 5).astype(int):
                dm.copy_slot_from(d64, i - 1)
                dm.solve_dynamic(i, i + 1, reuse_factors=True)
                cl_i, cd_i = coeffs(dm.force_total[i].cpu().numpy()[None], case)
                errs.append((abs(cl_i[0] - cl64[i - 1]) / abs(cl64[i - 1]),
                             abs(cd_i[0] - cd64[i - 1]) / np.max(np.abs(cd64))))
            res["cl_rel_err_one_step_max"] = max(e[0] for e in errs)
            res["cd_rel_err_one_step_max"] = max(e[1] for e in errs)
            res["cd_err_over_max_cl_one_step"] = res["cd_rel_err_one_step_max"] * float(
                np.max(np.abs(cd64)) / np.max(np.abs(cl64)))
        else:
            clm, cdm = coeffs(dm.force_total[1:].cpu().numpy(), case)
            res["cl_rel_err_max"] = float(np.max(np.abs(clm - cl64) / np.abs(cl64)))
            res["cd_rel_err_max_of_max"] = float(np.max(np.abs(cdm - cd64)) / np.max(np.abs(cd64)))
            # CD is a small projection of a force that is mostly lift: its error measured
            # against the lift scale shows the force accuracy itself
            res["cd_err_over_max_cl"] = float(np.max(np.abs(cdm - cd64)) / np.max(np.abs(cl64)))
            res["max_cd_over_max_cl"] = float(np.max(np.abs(cd64)) / np.max(np.abs(cl64)))
        if case.free_wake:
            # fluid-structure iterations: each step re-solved 3 times with new frames (a
            # structural iterate); iterations 2-3 reuse the convection velocities
            fsi = {}
            for prec in ("mixed", "fp64"):
                _, dc = make_case(case, prec, n_slots)
                run_device_steps(dc, 1, 4, None, torch)
                for reuse in (False, True):
                    st = torch.cuda.current_stream()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    n_it = 0
                    e0.record(st)
                    for i in range(4, min(n_slots, 14)):
                        for it in range(3):
                            dc.hg_t[i, :, 2, 3] += 1e-4  # the structure's new iterate
                            dc.solve_dynamic(i, i + 1, reuse_factors=True, reuse_convection=reuse and it > 0)
                            n_it += 1
                    e1.record(st)
                    e1.synchronize()
                    fsi[f"{prec}{'_reuse' if reuse else ''}_iterations_per_s"] = n_it / (e0.elapsed_time(e1) * 1e-3)
                del dc
            res["fsi_3_iterations_per_step"] = fsi
        del dm, d64
        th = host_threads()
        cpu_case = type(case)(**{**case.__dict__})
        v_all, t_all = cpu_steps(cpu_case, th, 1, min(10, n_steps - 1), 10.0)
        if case.free_wake:  # a free-wake step takes ~25 s on one core: sample its pair rate
            v_one, t_one = cpu_single_thread(cpu_case, 5.0)["value"], []
        else:
            v_one, t_one = cpu_steps(cpu_case, 1, 1, min(3, n_steps - 1), 10.0)
        res["cpu_all_threads_steps_per_s"] = v_all
        res["cpu_threads"] = th
        res["cpu_1_thread_steps_per_s"] = v_one
        res["cpu_sample_steps"] = [len(t_all), len(t_one)]
        rows[name] = res
    return rows


def adjoint_bench(args, torch):
    """Config 3: 12 x 64 wing, W = 100, 32 twist control angles ~ N(0, 1 deg), pitch 2 deg
    at k = 0.3, checkpoints every 10 steps.  Gradient of time-mean CL and CD with respect
    to the twist angles: FP64 forward, checkpointed recomputation, hand-written reverse
    sweep.  Two twist angles are also checked by central differences of the FP64 GPU
    forward (h = 1e-6; that forward's own roundoff limits such a difference to ~1e-4)."""
    import flapjax_b200 as fj
    from flapjax_b200 import cases
    from flapjax_b200.adjoint import PrescribedAdjoint, twist_jacobian

    c = cases.wing_pitch(n_steps=args.adjoint_steps)
    theta = c.extra["twist_ctrl_rad"]
    ctrl_y = np.linspace(0.0, c.span, len(theta))
    span_y = np.linspace(0.0, c.span, c.n + 1)
    jac = twist_jacobian(c.m, c.n, c.chord, 0.25, ctrl_y, span_y, np.interp(span_y, ctrl_y, theta))
    a = np.deg2rad(c.alpha_deg)
    q = 0.5 * c.rho * c.u_mag**2 * c.s_ref

    def weights(e):
        fw = np.zeros((c.n_tstep, 3))
        fw[1:] = np.asarray(e) / (q * c.n_steps)
        return fw

    def uvlm(zeta_b0):
        uv = fj.UVLM([fj.GridDiscretisation(c.m, c.n, c.m_star)], np.arange(c.n + 1), precision="fp64")
        uv.set_design_variables(dt=c.dt, flowfield=fj.Constant(c.u_inf, c.rho, True), zeta_b0=zeta_b0, hg0=c.hg0)
        return uv

    def mean_coeffs(zeta_b0):
        uv = uvlm(zeta_b0)
        out = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
        return [float(np.sum(weights(e)[1:] * out.force_total[1:])) for e in (e_l, e_d)]

    e_l, e_d = (-np.sin(a), 0.0, np.cos(a)), (np.cos(a), 0.0, np.sin(a))
    uv = uvlm(c.zeta_b0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    res = {"workload": "12x64 wing, W=100, 32 twist angles, pitch 2 deg at k=0.3, checkpoint 10",
           "steps": c.n_steps, "forward_s": t_fwd}
    # central differences of the FP64 GPU forward for two twist angles (both coefficients
    # from the same pair of runs)
    fd = {}
    for k in (3, 17):
        h = 1e-6
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        jp = mean_coeffs(cases.twisted_grid(c.m, c.n, c.chord, 0.25, np.interp(span_y, ctrl_y, tp)))
        jm = mean_coeffs(cases.twisted_grid(c.m, c.n, c.chord, 0.25, np.interp(span_y, ctrl_y, tm)))
        fd[k] = [(jp[i] - jm[i]) / (2 * h) for i in (0, 1)]
    for idx, (name, e) in enumerate((("CL", e_l), ("CD", e_d))):
        t0 = time.perf_counter()
        J, g = PrescribedAdjoint(uv).gradient(c.hg_t, c.hg_dot_t, weights(e), checkpoint=10)
        torch.cuda.synchronize()
        res[f"gradient_{name}_s"] = time.perf_counter() - t0
        grad = np.einsum("kmjd,mjd->k", jac, g)
        res[f"mean_{name}"] = J
        res[f"d{name}_dtwist"] = grad.tolist()
        res[f"fd_check_{name}"] = [{"param": k, "adjoint": float(grad[k]), "central_fd_fp64_gpu": fd[k][idx],
                                    "rel_diff": abs(fd[k][idx] - grad[k]) / max(abs(fd[k][idx]), 1e-30)}
                                   for k in (3, 17)]
    return res


def serving_bench(args, torch, n=None, rate=200.0):
    """Config 5: Poisson arrivals (200/s) of heaving wings with M ~ U{4..16},
    N ~ U{16..128}, W ~ U{20..200}, AoA ~ U[0, 8] deg, 100 steps each, mixed precision,
    continuously batched.  Reports whole-stream throughput and per-step latency, and the
    batched-step graph replays and captures.  With several ranks each serves every
    world-th arrival of the same stream (no collective on the data path); rank 0 merges
    the summaries."""
    import flapjax_b200 as fj
    from flapjax_b200 import cases, replicas
    from flapjax_b200.serving import Request, ServingLoop, graph_stats

    n = args.serving_cases if n is None else n
    stream, arrivals = cases.serving_stream(n_cases=n, rate=rate, n_steps=100, seed=0)

    def requests():
        out = []
        for k, (c, t) in enumerate(zip(stream, arrivals)):
            uv = fj.UVLM([fj.GridDiscretisation(c.m, c.n, c.m_star)], np.arange(c.n + 1), precision="mixed")
            uv.set_design_variables(dt=c.dt, flowfield=fj.Constant(c.u_inf, c.rho, True), zeta_b0=c.zeta_b0, hg0=c.hg0)
            out.append(Request(uv, c.hg_t, c.hg_dot_t, arrival=float(t), tag=k))
        return out

    rank, world, _ = replicas.rank_env()
    free = torch.cuda.mem_get_info()[0]
    loop = ServingLoop(memory_budget=int(0.5 * free), max_active=512, keep_results=False)
    loop.run(requests()[:8], realtime=False)  # warm-up (module load, allocator)
    torch.cuda.synchronize()
    g0 = graph_stats()
    res = loop.run(replicas.shard(requests(), rank, world), realtime=True)
    g1 = graph_stats()
    part = {"case_steps": res.case_steps, "wall_s": res.wall_s, "gpu_busy_s": res.gpu_busy_s,
            "step_latency_ms": res.step_latency_ms.tolist(), "admit_latency_s": res.admit_latency_s.tolist(),
            "max_active": res.max_active, "graph_replays": g1["replays"] - g0["replays"],
            "graph_captures": g1["captures"] - g0["captures"]}
    parts = replicas.gather_to_root(part)
    if parts is None:
        return None
    summ = replicas.merge_serving(parts)
    summ.update({"cases": n, "arrival_rate_per_s": rate, "steps_per_case": 100,
                 "graph_replays": sum(p["graph_replays"] for p in parts),
                 "graph_captures": sum(p["graph_captures"] for p in parts),
                 "workload": "heaving wings, M~U{4..16}, N~U{16..128}, W~U{20..200}, AoA~U[0,8] deg, mixed precision",
                 "pairs_total": float(sum(c.pairs_per_step() * c.n_steps for c in stream))})
    return summ


def bench_config(case, args, world):
    """The workload's description, the same on both arms."""
    return {"workload": "free-wake UVLM 16x128 bound, W=200 wake rows, cutoff kernel r=1e-3c, twist+camber seeded, "
                        "static-solve start" + (" [SMALL]" if args.small else ""),
            "m": case.m, "n": case.n, "m_star": case.m_star, "pairs_per_step": case.pairs_per_step(),
            "l2": "flushed between steps (256 MB write outside the timed events)",
            "parallelism": f"independent case replica per GPU x{world}", "seed": case.seed}


def ctypes_peak(torch):
    import ctypes

    from flapjax_b200 import _lib

    v = ctypes.c_double()
    _lib.call("fj_peak_fp32", ctypes.byref(v), torch.cuda.current_stream().cuda_stream)
    return v.value


def reference_arm(args):
    """The reference's arithmetic on the host CPU (the reference itself is JAX, absent on
    these machines): the C++/OpenMP FP64 oracle on every host thread, full time steps of
    the same workload.  Steps beyond what fits in about a minute are not run; the line
    reports how many were timed."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from flapjax_b200 import cases

    th = host_threads()
    n_max = max(1, min(args.steps, 50))
    case = cases.wing_free(n_steps=args.warmup + n_max) if not args.small else cases.wing_free(
        m=8, n=32, m_star=40, n_steps=args.warmup + n_max)
    value, times = cpu_steps(case, th, args.warmup, n_max, 60.0)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "dtype": "fp64", "data": "synthetic",
            "config": bench_config(case, args, int(os.environ.get("WORLD_SIZE", "1"))),
            "precision": "fp64",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": th, "kind": "port",
                             "sample": f"C++/OpenMP FP64 oracle, {args.warmup} untimed + {len(times)} timed full "
                                       f"time steps on {th} threads ({sum(times):.1f} s)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
