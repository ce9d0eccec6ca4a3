#!/usr/bin/env python
"""Benchmark of the explicit elastic FWI gradient evaluation on B200.

One step = one gradient evaluation of the plain inversion workload
(hirensi_b200.configs.inversion_config: 16x16x8 27-node hexahedra + 3-element
PML, 4 surface shots, 2000 RK4 steps): device assembly of C, K, G, M from the
current model, forward RK4 of all shots with the history kept in HBM, misfit,
adjoint RK4 with the zero-lag lambda/mu gradient fused in.  The metric is
fwd+adj GDOF-steps/s = DOF (regular-domain displacement DOF) x (forward +
adjoint steps) x shots / time.

    python bench.py [--gpus N --steps K --warmup W] [--impl native|reference]

Under torchrun each rank runs its own batch of shots (weak scaling) and the
gradients are summed over ranks with one NCCL all-reduce per step.
``--impl reference`` times the CPU restatement of the reference solver (the
reference itself needs Fortran + PETSc, which this image lacks) on the host
cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+adj GDOF-steps/s and FWI time-to-misfit, plain FP64 vs batched FP32+learned"
UNIT = "GDOF-steps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["native", "reference"], default="native")
    ap.add_argument("--nstep", type=int, default=2000, help="time steps per shot (2000 = the configuration)")
    ap.add_argument("--profile-case", action="store_true",
                    help="small run for profiler captures: 40 time steps, FP64 value leg only")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fwi", action="store_true", help="skip the FWI time-to-misfit leg")
    ap.add_argument("--fwi-iters", type=int, default=40,
                    help="iteration cap of each FWI time-to-misfit leg")
    ap.add_argument("--fwi-target", type=float, default=0.9,
                    help="FWI legs stop once the misfit has fallen by this fraction")
    ap.add_argument("--fwi-tv", action="store_true",
                    help="add the TV regularization to the gradient in the FWI legs (off: with it the plain "
                         "legs stall near a 6 %% reduction)")
    ap.add_argument("--fwi-fac", type=float, default=20.0,
                    help="Fac_Max_Update (largest model change per iteration) of the FWI legs")
    ap.add_argument("--profile-precision", choices=["fp64", "fp32"], default="fp64",
                    help="stepping precision of the --profile-case run")
    ap.add_argument("--variant", type=int, default=0,
                    help="stage-kernel variant for forward and adjoint (0 = chosen by timing on first use)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch every kernel directly instead of replaying the captured time loops")
    ap.add_argument("--workload", choices=["inversion", "uneven", "xl", "xl-fwi", "shot-scaling"], default="inversion",
                    help="inversion: the 16x16x8 plain inversion loop (default); uneven: batched uneven "
                         "shots on the 80x80x40 + PML 4 mesh, FP32 stepping, checkpointed adjoint; "
                         "xl: the same on the 160x160x80 + PML 6 mesh (86.6 M equations) with the "
                         "matrix-free operator; xl-fwi: inversion iterations on that mesh (8 shots in two "
                         "batches, records scaled by --length-scale); shot-scaling: stage-kernel time per shot "
                         "for 1, 2, 4 and 8 shots per pass over the 80x80x40 + PML 4 operator (FP32)")
    ap.add_argument("--max-batches", type=int, default=0, help="uneven / xl: time at most this many batches")
    ap.add_argument("--length-scale", type=float, default=0.03,
                    help="uneven workload: record lengths scaled by this factor (a bounded sample)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched FP32 leg (one full-length batch of 8 uneven shots on the "
                         "80x80x40 + PML 4 mesh) of the default run")
    ap.add_argument("--xl-error-steps", type=int, default=120,
                    help="xl workload: steps of the FP32-against-FP64 error check (2 shots); 0 skips it")
    ap.add_argument("--inflight", type=int, default=2,
                    help="uneven workload: batches in flight at once, each on its own context and stream")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# environment helpers

def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def stage_kernel_name(variant: int):
    """Kernel of a stage variant (FP64, 4 shots) and the committed ncu summary holding
    its DRAM traffic per launch."""
    if variant in (46, 86):
        return "rk4_stage_gt<double,4,runs>", "rk4_stage_gt46_fp64_inversion.md"
    if variant in (47, 87):
        return "rk4_stage_gtp<double,4>", "rk4_stage_gtp_fp64_inversion.md"
    if variant in (44, 45, 84, 85):
        return "rk4_stage_gt<double,4>", "rk4_stage_gt_fp64_inversion.md"
    if variant in (42, 43, 82, 83):
        return "rk4_stage_tile<double,4>", None
    if 90 <= variant <= 105:
        return "k_elem<double,4> + k_node<double,4>", None
    return "rk4_stage<double,4>", "rk4_stage_fp64_inversion.md"


def profile_traffic(name: str):
    """DRAM bytes per launch of a kernel from its committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"dram_bytes_per_launch\s*=\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic bytes of one fused stage launch (per-unit figure x units)

def stage_bytes(nnz_total: int, n: int, shots: int, bv: int) -> float:
    """Average algorithmic bytes of one RK4 stage launch: every stored entry once
    (value + 4-byte column), three row pointers, and per shot four stage vectors
    read/written per stage plus the x1..x3 update once per step
    (one quarter of the bytes of a whole RK4 step)."""
    matrix = nnz_total * (bv + 4) + (3 * 4 * (n + 1) if nnz_total else 0)
    vectors = shots * (4 * n * bv + 6 * n * bv / 4.0)
    return float(matrix + vectors)


# ---------------------------------------------------------------------------
# native arm

def run_native(args, rank, world, local_rank):
    import torch
    from hirensi_b200 import build
    from hirensi_b200.configs import RHO, inversion_config
    from hirensi_b200.solver import Solver

    build.build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nstep = 40 if args.profile_case else args.nstep
    prob = inversion_config(nstep=nstep)
    m = prob.mesh
    # one stream for the library and for torch (copies, the gradient all-reduce): the
    # library runs a null stream handle on a private non-blocking stream, which torch's
    # default stream would not be ordered with
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def make_solver(precision, variant=True):
        s = Solver(precision, device=local_rank)
        s.set_stream(stream.cuda_stream)
        s.set_mesh(m, RHO)
        s.assemble(prob.lam0, prob.mu0)
        s.set_history(m.store_eq)
        s.set_shots(prob.nstep, prob.dt, prob.src_eq, prob.src_b, prob.ftab)
        s.set_receivers(prob.eqdis, prob.eqdis_map)
        if variant and args.variant:
            s.set_variant(args.variant, args.variant)
        s.set_graphs(not args.no_graphs)
        return s

    # measured data: FP64 forward of the true model (set-up, untimed)
    fp32_profile = args.profile_case and args.profile_precision == "fp32"
    s64 = make_solver("fp64", variant=not fp32_profile)
    s64.assemble(prob.lam_true, prob.mu_true)
    s64.forward()
    dis = s64.traces()
    if fp32_profile:
        # profiler runs of the FP32 stepping: the value leg runs in FP32
        s64.close()
        s64 = make_solver("fp32")
    dis_dev = torch.from_numpy(dis).to(dev)
    lam_dev = torch.from_numpy(prob.lam0).to(dev)
    mu_dev = torch.from_numpy(prob.mu0).to(dev)
    g_dev = torch.zeros(2, m.nj, dtype=torch.float64, device=dev)
    s64.set_data(device_ptr=dis_dev.data_ptr())
    dis_pinned = torch.from_numpy(dis).pin_memory()
    lam_h, mu_h = prob.lam0.copy(), prob.mu0.copy()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def allreduce():
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(g_dev)

    def step_value(s):
        s.assemble_device(lam_dev.data_ptr(), mu_dev.data_ptr())
        s.forward()
        s.misfit(None)
        s.adjoint_gradient(None, to_host=False)
        s.gradient_device(g_dev[0].data_ptr(), g_dev[1].data_ptr())
        allreduce()

    def step_e2e(s):
        s.set_data(dis_pinned.numpy())
        s.assemble(lam_h, mu_h)
        s.forward()
        s.misfit(None)
        gl, gm = s.adjoint_gradient(None, to_host=True)
        if world > 1:
            g_dev[0].copy_(torch.from_numpy(gl))
            g_dev[1].copy_(torch.from_numpy(gm))
            allreduce()
        return gl

    def timed(fn, s, K, W, sample_clocks=False):
        for _ in range(W):
            fn(s)
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        clk = ClockSampler(local_rank) if sample_clocks else None
        if clk:
            clk.start()
        l0 = s.launch_count()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            fn(s)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        clocks = clk.stop() if clk else None
        launches = s.launch_count() - l0
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, launches, clocks

    K, W = args.steps, args.warmup
    units_per_step = prob.dof * ((prob.nstep + 1) + prob.nstep) * prob.nshot * world

    # value leg (inputs resident), FP64
    ms_val, launches, clocks = timed(step_value, s64, K, W, sample_clocks=True)
    # roofline: the stage kernel timed alone, 50 RK4 steps (200 launches) of the
    # tuned forward and adjoint variants back to back under one pair of CUDA events
    # on the library's stream (no per-launch events); the step's stage launches are
    # weighted by their count: 4 (nstep + 1) forward, 4 nstep adjoint
    n_fwd, n_adj = 4 * (prob.nstep + 1), 4 * prob.nstep
    st_fwd = s64.time_stage(adjoint=False, nsteps=50)
    st_adj = s64.time_stage(adjoint=True, nsteps=50)
    stage_avg_ms = (n_fwd * st_fwd + n_adj * st_adj) / (n_fwd + n_adj)
    stage_n = n_fwd + n_adj
    value = units_per_step * K / (ms_val * 1e-3)

    result = {"metric": METRIC, "value": value / 1e9, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
              "ms_per_step": ms_val / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
              "dtype": "f32" if (args.profile_case and args.profile_precision == "fp32") else "f64",
              "data": "synthetic (seeded layered model with a Gaussian anomaly; no dataset)"}
    nnz = [s64.operator_csr(w)[2].size for w in range(3)]
    result["config"] = {"workload": prob.name + f"_4shots_{prob.nstep}steps", "elements": m.nel, "nodes": m.nj,
                        "dof": prob.dof, "equations": m.neq, "nnz_CKG": nnz, "shots_per_gpu": prob.nshot,
                        "time_steps": prob.nstep, "dt": prob.dt,
                        "step": "assemble + forward (history in HBM) + misfit + adjoint with fused gradient",
                        "l2": "inputs larger than L2: FP64 operator 168 MB and 3.6 GB of histories per step"}
    result["gpu_launches"] = int(launches)
    result["config"]["stage_variant_fwd_adj"] = list(s64.variant())

    # roofline of the dominant kernel (fused RK4 stage, the variant the tuner chose)
    peak, peak_kind = measured_peaks()
    bytes_launch = stage_bytes(sum(nnz), m.neq, prob.nshot, 8)
    achieved = bytes_launch / (stage_avg_ms * 1e-3) / 1e9
    kname, kprofile = stage_kernel_name(s64.variant()[0])
    traffic = profile_traffic(kprofile) if kprofile else None
    result["roofline"] = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                          "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                          "bytes_per_launch": bytes_launch, "avg_launch_us": stage_avg_ms * 1e3,
                          "avg_launch_us_fwd_adj": [st_fwd * 1e3, st_adj * 1e3],
                          "timing": "200 back-to-back launches per direction under one event pair",
                          "stage_launches_per_step": int(stage_n),
                          "stage_share_of_step": stage_n * stage_avg_ms / (ms_val / K),
                          "traffic": traffic}
    result["clocks"] = clocks

    tuned = {"fp64": s64.variant()}   # the FWI legs reuse the variants tuned here
    if not args.profile_case:
        # e2e leg: host buffers through the C ABI, copies inside the timed region
        ms_e2e, _, _ = timed(step_e2e, s64, K, min(W, 1))
        h2d = dis.nbytes + lam_h.nbytes + mu_h.nbytes
        d2h = 2 * m.nj * 8 + 8
        result["e2e"] = {"value": units_per_step * K / (ms_e2e * 1e-3) / 1e9, "unit": UNIT,
                         "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e / K}
        # FP32 stepping with FP64 reductions, same workload
        if not args.no_fp32:
            g64 = g_dev.clone()
            tr64 = s64.traces()
            s32 = make_solver("fp32")
            s32.set_data(device_ptr=dis_dev.data_ptr())
            ms32, _, _ = timed(step_value, s32, K, W)
            tr32 = s32.traces()
            g32 = g_dev.clone()
            ms32e, _, _ = timed(step_e2e, s32, K, min(W, 1))
            tuned["fp32"] = s32.variant()

            def rel(a, b):
                return float(np.linalg.norm(a - b) / np.linalg.norm(b))

            result["fp32"] = {"value": units_per_step * K / (ms32 * 1e-3) / 1e9, "ms_per_step": ms32 / K,
                              "e2e": {"value": units_per_step * K / (ms32e * 1e-3) / 1e9, "unit": UNIT},
                              "seismogram_rel_l2_vs_fp64": rel(tr32, tr64),
                              "gradient_rel_l2_vs_fp64": rel(g32.cpu().numpy(), g64.cpu().numpy())}
            s32.close()
        if world == 1 and not args.no_cpu_baseline:      # the host-core baseline is a single-GPU figure
            cb = cpu_sample(prob, nsteps=200)
            cb.pop("seconds", None)
            result["cpu_baseline"] = cb
        if not args.no_fwi and world == 1:
            # time to a stated misfit reduction, each leg from the initial model
            result["fwi"] = {"target_reduction": args.fwi_target, "iteration_cap": args.fwi_iters,
                             "fac_max_update": args.fwi_fac, "regularization": "TV" if args.fwi_tv else None}
            legs = [("fp64", False)] if args.no_fp32 else [("fp64", False), ("fp32", False)]
            if not args.no_fp32 and os.path.exists(PRECOND_WEIGHTS):
                legs.append(("fp32", True))
            for prec, learned in legs:
                name = prec + ("_learned" if learned else "")
                result["fwi"][name] = fwi_leg(prec, prob, dis, local_rank, args.fwi_iters, learned=learned,
                                              target=args.fwi_target, variant=tuned.get(prec), fac=args.fwi_fac,
                                              tv=args.fwi_tv)
            f64, fl = result["fwi"]["fp64"], result["fwi"].get("fp32_learned")
            if fl and f64["reached_target"] and fl["reached_target"]:
                result["fwi"]["time_to_target_speedup_fp32_learned_vs_fp64"] = f64["time_to_target_s"] / fl["time_to_target_s"]
            f32 = result["fwi"].get("fp32")
            if f32 and f64["reached_target"] and f32["reached_target"]:
                result["fwi"]["time_to_target_speedup_fp32_vs_fp64"] = f64["time_to_target_s"] / f32["time_to_target_s"]
            if fl and f64["time_to_50pct_s"] and fl["time_to_50pct_s"]:
                result["fwi"]["time_to_50pct_speedup_fp32_learned_vs_fp64"] = f64["time_to_50pct_s"] / fl["time_to_50pct_s"]
    s64.close()
    if not args.profile_case and not args.no_batched and world == 1:
        result["batched_fp32"] = batched_leg(args, local_rank)
    return result


def batched_leg(args, local_rank):
    """One batch of the batched uneven-shot workload at full record length: 8 shots of
    the 64-shot plan on the 80x80x40 + PML 4 mesh (12.7 M equations), the batch with the
    shortest records (1500-2000 steps), FP32 stepping with FP64 reductions, forward with
    checkpoints every 100 steps, misfit, adjoint with recomputed segments and the fused
    gradient.  Warmed up on the same batch with its records scaled to 3 % (tuning,
    tables), then timed once with CUDA events.  Counts each shot's own steps."""
    import torch
    from hirensi_b200 import batching as B
    from hirensi_b200.configs import uneven_config
    from hirensi_b200.solver import Solver
    dev = torch.device("cuda", local_rank)
    t_setup = time.perf_counter()
    full = uneven_config(length_scale=1.0)
    short = uneven_config(length_scale=0.03)
    m = full.mesh
    lengths = [sh.nstep for sh in full.shots]
    ids = B.plan(lengths, 8)[-1]
    sv = Solver("fp32", device=local_rank)
    sv.set_graphs(False)   # launches are hidden behind millisecond stages; no capture in the timed batch
    sv.set_mesh(m, full.rho_el)
    sv.assemble(full.lam, full.mu)
    sv.set_history(m.store_eq)
    sv.set_checkpointing(100)

    def run(prob):
        b = B.pack(prob.shots, ids)
        B.configure(sv, b, prob.dt, m.store_position)
        sv.set_data(np.zeros((len(ids), len(b.eqdis), b.nstep + 1)))
        sv.forward()
        J = sv.misfit(None)
        sv.adjoint_gradient(None, to_host=False)
        return b, J

    run(short)
    b, _ = run(short)
    torch.cuda.synchronize(dev)
    setup_s = time.perf_counter() - t_setup
    # the full-length batch: its buffers (checkpoints, traces, source tables) are
    # allocated by the calls themselves, so the time is the device time the library
    # measures with CUDA events around each time loop (forward, adjoint), plus the misfit
    clk = ClockSampler(local_rank)
    clk.start()
    l0 = sv.launch_count()
    b = B.pack(full.shots, ids)
    B.configure(sv, b, full.dt, m.store_position)
    sv.set_data(np.zeros((len(ids), len(b.eqdis), b.nstep + 1)))
    sv.forward()
    t_fwd = sv.last_timing()[0]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sv.misfit(None)
    e1.record()
    torch.cuda.synchronize(dev)
    t_mis = e0.elapsed_time(e1)
    sv.adjoint_gradient(None, to_host=False)
    t_adj = sv.last_timing()[0]
    torch.cuda.synchronize(dev)
    ms = t_fwd + t_mis + t_adj
    clocks = clk.stop()
    launches = sv.launch_count() - l0
    units = sum(full.dof * (2 * lengths[i] + 1) for i in ids)
    st_f = sv.time_stage(adjoint=False, nsteps=20)
    st_a = sv.time_stage(adjoint=True, nsteps=20)
    nnz = [sv.operator_nnz(w) for w in range(3)]
    bytes_launch = stage_bytes(sum(nnz), m.neq, len(ids), 4)
    peak, peak_kind = measured_peaks()
    st = 0.5 * (st_f + st_a)
    out = {"value": units / (ms * 1e-3) / 1e9, "unit": UNIT, "ms": ms, "ms_forward_misfit_adjoint": [t_fwd, t_mis, t_adj],
           "dtype": "f32 stepping, f64 reductions",
           "workload": full.name, "shots_in_batch": len(ids), "record_lengths": [lengths[i] for i in ids],
           "receivers_per_shot": [len(full.shots[i].eqdis) // 3 for i in ids], "checkpoint_interval": 100,
           "equations": m.neq, "dof": full.dof, "nnz_CKG": nnz, "stage_variant_fwd_adj": list(sv.variant()),
           "gpu_launches": int(launches), "setup_s": setup_s, "clocks": clocks,
           "roofline": {"bound": "hbm", "achieved": bytes_launch / (st * 1e-3) / 1e9, "peak": peak,
                        "peak_kind": peak_kind, "unit": "GB/s", "frac": bytes_launch / (st * 1e-3) / 1e9 / peak,
                        "bytes_per_launch": bytes_launch, "avg_launch_us_fwd_adj": [st_f * 1e3, st_a * 1e3]},
           "step": "forward (checkpoints every 100 steps) + misfit + adjoint with recomputed segments and gradient"}
    sv.close()
    return out


PRECOND_WEIGHTS = os.path.join(ROOT, "hirensi_b200", "data", "precond_cnn6_16x16x8.npz")


# ---------------------------------------------------------------------------
# batched uneven shots on the large mesh

def run_uneven(args, rank, world, local_rank):
    """64 shots of uneven record length (1500-4000 steps scaled by --length-scale) and
    receiver count (100-900) on the 80x80x40 + PML 4 mesh (12.7 M equations), planned
    into batches of 8 by record length (hirensi_b200.batching); per batch: forward with
    the state checkpointed every 100 steps, misfit, adjoint with recomputed segments and
    the fused gradient, FP32 stepping with FP64 reductions.  Batches are sharded over
    ranks, and --inflight batches run at once on separate contexts (streams) of a GPU.
    The unit counts each shot's own steps: DOF x (2 nstep_s + 1) per shot.

    xl: 8 shots on the 160x160x80 + PML 6 mesh (86.6 M equations), four per batch,
    checkpoints every 50 steps, one context, matrix-free operator."""
    import torch
    from hirensi_b200 import batching as B
    from hirensi_b200 import build
    from hirensi_b200.configs import uneven_config
    from hirensi_b200.solver import Solver

    build.build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    t_setup = time.perf_counter()
    if args.workload == "xl":
        # The CSR of this mesh would exceed the 2^31 entry range: C, K, G are applied
        # element by element.  Four FP32 shots per batch hold about 40 GB of segment
        # history (50 steps) and 25 GB of checkpoints.
        prob = xl_problem(args.length_scale)
        per_batch, ckpt = 4, 50
    else:
        prob = uneven_config(length_scale=args.length_scale)
        per_batch, ckpt = 8, 100
    m = prob.mesh
    lengths = [sh.nstep for sh in prob.shots]
    plan = B.plan(lengths, per_batch)
    mine = plan[rank::world]
    if args.max_batches:
        mine = mine[:args.max_batches]
    import threading

    def make_solver():
        sv = Solver("fp32", device=local_rank)
        sv.set_graphs(not args.no_graphs)
        sv.set_mesh(m, prob.rho_el)
        if args.workload == "xl":
            sv.set_operator_mode(True)
        sv.assemble(prob.lam, prob.mu)
        sv.set_history(m.store_eq)
        sv.set_checkpointing(ckpt)
        return sv

    def run_batch(sv, ids):
        b = B.pack(prob.shots, ids)
        B.configure(sv, b, prob.dt, m.store_position)
        sv.set_data(np.zeros((len(ids), len(b.eqdis), b.nstep + 1)))
        sv.forward()
        sv.misfit(None)
        sv.adjoint_gradient(None, to_host=False)

    # warm-up: the first context tunes the stage variants on this operator; the others
    # take its choice; each builds its tables on one batch
    solvers = [make_solver() for _ in range(1 if args.workload == "xl" else max(1, args.inflight))]
    s = solvers[0]
    if args.variant:
        s.set_variant(args.variant, args.variant)
    run_batch(s, mine[0])
    for sv in solvers[1:]:
        sv.set_variant(*s.variant())
        run_batch(sv, mine[0])
    torch.cuda.synchronize(dev)
    setup_s = time.perf_counter() - t_setup
    clk = ClockSampler(local_rank)
    clk.start()
    l0 = sum(sv.launch_count() for sv in solvers)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # the batches in flight: each context (its own stream) takes the next batch in turn;
    # every library call blocks its host thread until its work is done
    queue = list(mine)
    lock = threading.Lock()
    errors = []

    def worker(sv):
        try:
            while True:
                with lock:
                    if not queue:
                        return
                    ids = queue.pop(0)
                run_batch(sv, ids)
        except Exception as exc:   # reported after the join
            errors.append(exc)

    e0.record()
    threads = [threading.Thread(target=worker, args=(sv,)) for sv in solvers]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    e1.record()
    torch.cuda.synchronize(dev)
    if errors:
        raise errors[0]
    ms = e0.elapsed_time(e1)
    clocks = clk.stop()
    launches = sum(sv.launch_count() for sv in solvers) - l0
    units = sum(prob.dof * (2 * lengths[i] + 1) for ids in mine for i in ids)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms, units], dtype=torch.float64, device=dev)
        dist.all_reduce(t[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        ms, units = float(t[0]), float(t[1])
    # roofline: per-launch stage times of one batch's forward
    b0 = B.pack(prob.shots, mine[0])
    B.configure(s, b0, prob.dt, m.store_position)
    s.set_timing(True)
    t0 = s.last_timing()
    s.forward()
    t1 = s.last_timing()
    s.set_timing(False)
    stage_us = (t1[1] - t0[1]) / max(t1[2] - t0[2], 1) * 1e3
    nnz = [s.operator_nnz(w) for w in range(3)]
    # matrix-free: no stored entries, so the vector part of the stage (the least any
    # stage moves) is the algorithmic figure
    bytes_launch = stage_bytes(sum(nnz), m.neq, len(mine[0]), 4)
    peak, peak_kind = measured_peaks()
    kname, _ = stage_kernel_name(s.variant()[0])
    achieved = bytes_launch / (stage_us * 1e-6) / 1e9
    result = {"metric": METRIC, "value": units / (ms * 1e-3) / 1e9, "unit": UNIT, "n_gpus": world,
              "steps": len(mine), "warmup": 1, "ms_per_step": ms / len(mine), "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "dtype": "f32",
              "data": "synthetic (seeded layered model with ellipsoidal inclusions; zero measured data)",
              "config": {"workload": prob.name, "equations": m.neq, "dof": prob.dof, "nnz_CKG": nnz,
                         "shots": len(prob.shots), "batches": len(plan), "batches_timed": len(mine),
                         "shots_per_batch": per_batch, "dt": prob.dt,
                         "record_lengths": [min(lengths), max(lengths)], "length_scale": args.length_scale,
                         "receivers_per_shot": [min(len(sh.eqdis) // 3 for sh in prob.shots),
                                                max(len(sh.eqdis) // 3 for sh in prob.shots)],
                         "checkpoint_interval": ckpt, "stage_variant_fwd_adj": list(s.variant()),
                         "batches_in_flight": len(solvers),
                         "setup_s": setup_s,
                         "operator": "matrix-free" if args.workload == "xl" else "csr",
                         "step": f"one batch of {per_batch} shots: forward + misfit + checkpointed adjoint with gradient",
                         "l2": "inputs larger than L2"},
              "gpu_launches": int(launches),
              "roofline": {"bound": "hbm", "kernel": kname.replace("double", "float").replace(",4>", f",{per_batch}>"),
                           "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                           "frac": achieved / peak, "bytes_per_launch": bytes_launch, "avg_launch_us": stage_us,
                           "traffic": None},
              "clocks": clocks}
    for sv in solvers:
        sv.close()
    if args.workload == "xl" and args.xl_error_steps > 0:
        result["fp32_error_vs_fp64"] = xl_error(prob, args.xl_error_steps, local_rank)
    return result


def xl_problem(length_scale):
    """The extra-large workload: 160x160x80 + PML 6, 8 shots of 6000-8000 steps scaled by
    length_scale, 2500 receivers, dt at 0.15 of the GLL-spacing CFL limit of the model
    distribution's fastest P wave (Vs 600 m/s, nu 0.40)."""
    from hirensi_b200.configs import uneven_config
    vp_max = 600.0 * np.sqrt(2.0 * (1.0 - 0.40) / (1.0 - 2.0 * 0.40))
    dt = 0.15 * (0.5 * 2.5) / vp_max
    return uneven_config(nx=160, ny=160, nz=80, npml=6, nshot=8, dt=dt, lengths=(6000, 8000),
                         receivers=(2500, 2500), length_scale=length_scale)


def run_xl_fwi(args, local_rank):
    """Inversion iterations on the extra-large mesh: the seeded model (layers + ellipsoidal
    inclusions) is the true model, its depth average (each level's mean lambda and mu) the
    initial one; 8 shots in two batches of four (hirensi_b200.inversion.BatchedBackend),
    FP32 stepping with FP64 reductions and L-BFGS, matrix-free operator, checkpointed
    adjoint; L-BFGS memory 5, the reference's step rules, Fac_Max_Update 20, no TV."""
    import torch
    from hirensi_b200 import batching as B
    from hirensi_b200 import build
    from hirensi_b200.configs import extend_into_pml
    from hirensi_b200.inversion import FWI, BatchedBackend, InversionConfig
    from hirensi_b200.solver import Solver
    build.build()
    torch.cuda.set_device(local_rank)
    t_setup = time.perf_counter()
    prob = xl_problem(args.length_scale)
    m = prob.mesh
    zlev = np.round(m.xyz[:, 2] / 1.25).astype(np.int64)
    _, inv = np.unique(zlev, return_inverse=True)
    cnt = np.bincount(inv)
    lam0 = extend_into_pml(m, (np.bincount(inv, prob.lam) / cnt)[inv])
    mu0 = extend_into_pml(m, (np.bincount(inv, prob.mu) / cnt)[inv])
    lengths = [sh.nstep for sh in prob.shots]
    plan = B.plan(lengths, 4)
    sv = Solver("fp32", device=local_rank)
    sv.set_mesh(m, prob.rho_el)
    sv.set_operator_mode(True)
    sv.assemble(prob.lam, prob.mu)
    sv.set_history(m.store_eq)
    sv.set_checkpointing(max(10, max(lengths) // 4))
    shots = list(prob.shots)
    for ids in plan:                        # measured data: the true model's traces
        b = B.pack(shots, ids)
        B.configure(sv, b, prob.dt, m.store_position)
        sv.forward()
        for k, tr in zip(ids, B.unpack_traces(b, sv.traces())):
            sh = shots[k]
            shots[k] = B.Shot(sh.src_eq, sh.src_b, sh.ftab, sh.eqdis, tr)
    batches = [B.pack(shots, ids) for ids in plan]
    cfg = InversionConfig(m_lbfgs=5, bounds_lambda=(1.0, 5000.0), bounds_mu=(1.0, 2000.0), regularization=None,
                          fac_max_update_lambda=20.0, fac_max_update_mu=20.0)
    backend = BatchedBackend(sv, m, batches, prob.dt, m.store_position)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    clk = ClockSampler(local_rank)
    clk.start()
    t0 = time.perf_counter()
    fwi = FWI(backend, cfg)
    failed = None
    try:
        hist = fwi.run(lam0, mu0, n_iter=args.fwi_iters)
    except RuntimeError as exc:     # ArmijoFailure: the reference would STOP here
        hist, failed = fwi.hist, str(exc)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = clk.stop()
    J0 = hist[0]["misfit"]
    rd = m.node_mat_id == 0
    err = {}
    if failed is None:
        mu_f = fwi.mu.cpu().numpy()
        err = {"mu_rel_l2_error": float(np.linalg.norm((mu_f - prob.mu)[rd]) / np.linalg.norm(prob.mu[rd])),
               "mu_rel_l2_error_initial": float(np.linalg.norm((mu0 - prob.mu)[rd]) / np.linalg.norm(prob.mu[rd]))}
    sv.close()
    out = {"metric": "FWI iterations on the extra-large mesh", "unit": "s", "value": wall, "higher_is_better": False,
           "n_gpus": 1, "dtype": "f32 stepping, f64 reductions and L-BFGS", "data": "synthetic (seeded true model)",
           "config": {"workload": prob.name.replace("_8shots", "") + "_fwi", "equations": m.neq, "dof": prob.dof,
                      "nodes": m.nj, "shots": len(shots), "batches": len(batches),
                      "record_lengths": [min(lengths), max(lengths)], "length_scale": args.length_scale,
                      "receivers_per_shot": 2500, "operator": "matrix-free",
                      "inversion": "L-BFGS memory 5, reference step rules, Fac_Max_Update 20, no TV; initial model = "
                                   "depth average of the true model"},
           "iterations": len(hist) - 1, "armijo_trials": [h["armijo"] for h in hist[1:]],
           "misfit_history": [h["misfit"] / J0 for h in hist], "misfit_reduction": 1.0 - hist[-1]["misfit"] / J0,
           "setup_s": setup_s, "clocks": clocks}
    if failed:
        out["armijo_failure"] = failed
    out.update(err)
    return out


def run_shot_scaling(args, local_rank):
    """How the cost of a stage grows with the shots that share one pass over the
    operator: on the 80x80x40 + PML 4 mesh (12.7 M equations, 312.6 M stored entries),
    FP32 stepping, for 1, 2, 4 and 8 shots the tuned stage variant is timed alone
    (hrn_time_stage, 50 RK4 steps per direction).  Per-shot time falling slowly with
    the shot count means the matrix stream is a small part of a stage, so batches
    larger than 8 would gain little."""
    import torch
    from hirensi_b200 import batching as B
    from hirensi_b200 import build
    from hirensi_b200.configs import uneven_config
    from hirensi_b200.solver import Solver
    build.build()
    torch.cuda.set_device(local_rank)
    prob = uneven_config(length_scale=0.01)
    m = prob.mesh
    rows = []
    for S in (1, 2, 4, 8):
        sv = Solver("fp32", device=local_rank)
        sv.set_mesh(m, prob.rho_el)
        sv.assemble(prob.lam, prob.mu)
        sv.set_history(m.store_eq)
        sv.set_checkpointing(10)
        b = B.pack(prob.shots, list(range(S)))
        B.configure(sv, b, prob.dt, m.store_position)
        sv.set_data(np.zeros((S, len(b.eqdis), b.nstep + 1)))
        sv.forward()
        sv.adjoint_gradient(None, to_host=False)
        f, a = sv.time_stage(False, 50), sv.time_stage(True, 50)
        rows.append({"shots": S, "variant_fwd_adj": list(sv.variant()), "stage_us_fwd_adj": [f * 1e3, a * 1e3],
                     "stage_us_per_shot": 0.5 * (f + a) * 1e3 / S})
        sv.close()
    base = rows[0]["stage_us_per_shot"]
    for r in rows:
        r["per_shot_vs_one_shot"] = r["stage_us_per_shot"] / base
    return {"metric": "stage-kernel time per shot against shots per pass", "unit": "us per shot-stage",
            "value": rows[-1]["stage_us_per_shot"], "higher_is_better": False, "n_gpus": 1, "dtype": "f32",
            "data": "synthetic", "config": {"workload": prob.name.replace("_64shots", ""), "equations": m.neq,
                                            "dof": prob.dof}, "rows": rows}


def xl_error(prob, nsteps, local_rank):
    """Seismogram and gradient error of FP32 stepping against FP64 stepping on the
    extra-large mesh (matrix-free operator): the first two shots of the workload, their
    records cut to `nsteps` steps, zero measured data (the residuals are the synthetics
    themselves), checkpoints every nsteps / 3 steps; relative L2 over all traces and
    over the whole gradient."""
    from hirensi_b200 import batching as B
    from hirensi_b200.solver import Solver
    m = prob.mesh
    shots = [B.Shot(sh.src_eq, sh.src_b, sh.ftab[: nsteps + 1], sh.eqdis) for sh in prob.shots[:2]]
    b = B.pack(shots, [0, 1])
    out = {}
    for prec in ("fp32", "fp64"):
        sv = Solver(prec, device=local_rank)
        sv.set_mesh(m, prob.rho_el)
        sv.set_operator_mode(True)
        sv.assemble(prob.lam, prob.mu)
        sv.set_history(m.store_eq)
        sv.set_checkpointing(max(1, nsteps // 3))
        B.configure(sv, b, prob.dt, m.store_position)
        sv.set_data(np.zeros((2, len(b.eqdis), b.nstep + 1)))
        sv.forward()
        tr = sv.traces()
        J = sv.misfit(None)
        gl, gm = sv.adjoint_gradient(None)
        out[prec] = (tr, J, gl, gm, list(sv.variant()))
        sv.close()

    def rel(a, b_):
        return float(np.linalg.norm(a - b_) / np.linalg.norm(b_))
    t32, J32, l32, m32, v32 = out["fp32"]
    t64, J64, l64, m64, v64 = out["fp64"]
    return {"shots": 2, "steps": nsteps, "receivers_per_shot": [len(sh.eqdis) // 3 for sh in shots],
            "seismogram_rel_l2": rel(t32, t64), "misfit_rel": abs(J32 - J64) / J64,
            "gradient_lambda_rel_l2": rel(l32, l64), "gradient_mu_rel_l2": rel(m32, m64),
            "variants_fp32_fp64": [v32, v64]}


def fwi_leg(precision, prob, dis, local_rank, iters, learned=False, target=None, variant=None, fac=5.0, tv=False):
    """Wall time of the inversion loop (L-BFGS memory 5, the reference's step rules, TV optional)
    from the initial model until the misfit has fallen by `target` or `iters` iterations
    have run, all vectors on the device; misfit reduction and model error reached.  With
    `learned`, each iteration first tries the trained CNN's scaled direction.  `variant` =
    the (forward, adjoint) stage variants tuned earlier on the same operator."""
    import torch
    from hirensi_b200.configs import RHO
    from hirensi_b200.inversion import FWI, DeviceBackend, InversionConfig
    from hirensi_b200.solver import Solver
    m = prob.mesh
    s = Solver(precision, device=local_rank)
    s.set_mesh(m, RHO)
    s.assemble(prob.lam0, prob.mu0)
    s.set_history(m.store_eq)
    s.set_shots(prob.nstep, prob.dt, prob.src_eq, prob.src_b, prob.ftab)
    s.set_receivers(prob.eqdis, prob.eqdis_map)
    s.set_data(dis)
    if variant:
        s.set_variant(*variant)
    cfg = InversionConfig(m_lbfgs=5, bounds_lambda=(10.0, 2000.0), bounds_mu=(10.0, 1000.0),
                          fac_max_update_lambda=fac, fac_max_update_mu=fac, regularization="TV" if tv else None)
    backend = DeviceBackend(s, m)
    pre = None
    if learned:
        from hirensi_b200.learned import DeviceNet, LearnedPreconditioner, Lattice, Net
        pre = LearnedPreconditioner(DeviceNet(Net.load(PRECOND_WEIGHTS), Lattice.of(m).shape), m, RHO)
    # warm-up outside the timed region, as a driver that keeps its solver between
    # inversions has it: one iteration builds the variant's tables, the inversion's
    # buffers and the captured time loops, and loads the network's kernels
    FWI(backend, cfg, preconditioner=pre).run(prob.lam0, prob.mu0, n_iter=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fwi = FWI(backend, cfg, preconditioner=pre)
    failed = None
    try:
        hist = fwi.run(prob.lam0, prob.mu0, n_iter=iters, target_reduction=target)
    except RuntimeError as exc:      # ArmijoFailure: the reference would STOP here
        hist, failed = fwi.hist, str(exc)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    J0, J = hist[0]["misfit"], hist[-1]["misfit"]
    rd = m.node_mat_id == 0
    err = {}
    if failed is None:
        mu_f = fwi.mu.cpu().numpy()
        vs = np.sqrt(np.maximum(mu_f, 0.0) / RHO)
        vs_t, vs_0 = np.sqrt(prob.mu_true / RHO), np.sqrt(prob.mu0 / RHO)
        err = {"vs_rel_l2_error": float(np.linalg.norm((vs - vs_t)[rd]) / np.linalg.norm(vs_t[rd])),
               "vs_rel_l2_error_initial": float(np.linalg.norm((vs_0 - vs_t)[rd]) / np.linalg.norm(vs_t[rd]))}
    t_target = next((h["wall_s"] for h in hist if target is not None and h["misfit"] <= (1.0 - target) * J0), None)
    t_half = next((h["wall_s"] for h in hist if h["misfit"] <= 0.5 * J0), None)
    it_half = next((h["iter"] for h in hist if h["misfit"] <= 0.5 * J0), None)
    s.close()
    out = {"iterations": len(hist) - 1, "wall_s": wall, "time_to_target_s": t_target,
           "time_to_50pct_s": t_half, "iterations_to_50pct": it_half,
           "misfit_initial": J0, "misfit_final": J, "misfit_reduction": 1.0 - J / J0,
           "misfit_history": [h["misfit"] for h in hist],
           "forward_solves": hist[-1]["forward_solves"], "adjoint_solves": hist[-1]["adjoint_solves"],
           "config": f"L-BFGS memory 5, {'TV regularization' if tv else 'no regularization'}, reference step "
                     f"rules (lambda bias on), Fac_Max_Update {fac}, bounds lambda [10,2000] mu [10,1000]",
           "warmup": "one inversion iteration (tables, buffers, captured time loops) before the timed inversion", **err}
    if failed:
        out["armijo_failure"] = failed
    if learned:
        out["learned_steps_accepted"] = int(sum(1 for h in hist[1:] if h.get("learned")))
        out["proposal_search"] = {"trials": [h["search"].get("trials", 0) for h in hist[1:]],
                                  "curvature_met": [h["search"].get("curvature") for h in hist[1:]],
                                  "rule": "weak Wolfe (Armijo c1 1e-4, curvature c2 0.9, up to two doublings)"}
        out["weights"] = os.path.relpath(PRECOND_WEIGHTS, ROOT)
    if target is not None:
        out["target_reduction"] = target
        out["reached_target"] = bool(failed is None and 1.0 - J / J0 >= target)
    return out


# ---------------------------------------------------------------------------
# CPU restatement of the reference (baseline leg and --impl reference)

_CPU_SYS = {}


def cpu_sample(prob, nsteps=100, shots=None):
    """Time the FP64 CPU restatement (OpenMP over all host cores: SpMV rows, vector
    updates and the gradient's element loop) on a bounded sample of the workload:
    every shot (or the first `shots`), `nsteps` forward + adjoint steps each with
    the gradient, one source per solve as the reference runs them."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from hirensi_b200.configs import RHO
    m = prob.mesh
    cores = os.cpu_count() or 1
    if "sys" not in _CPU_SYS:
        om = O.OracleMesh(m, RHO)
        _CPU_SYS["sys"] = (om, O.OracleSystem.assemble(om, prob.lam0, prob.mu0))
    om, S = _CPU_SYS["sys"]
    nshot = prob.nshot if shots is None else min(shots, prob.nshot)
    dis = np.zeros((prob.eqdis.size, nsteps + 1)) + 1e-12
    t0 = time.perf_counter()
    for k in range(nshot):
        b = np.zeros(m.neq)
        b[prob.src_eq[k]] = 1.0
        ftab = prob.ftab[k][: nsteps + 1]
        u = S.forward(b, ftab, nsteps, prob.dt, m.store_eq, nthreads=cores)
        p = S.adjoint(nsteps, prob.dt, m.store_eq, u, prob.eqdis, prob.eqdis_map, dis, nthreads=cores)
        O.control(om, nsteps, prob.dt, m.store_eq, u, p, nthreads=cores)
    dt = time.perf_counter() - t0
    units = prob.dof * ((nsteps + 1) + nsteps) * nshot
    return {"value": units / dt / 1e9, "unit": UNIT, "cores": cores, "kind": "port", "seconds": dt,
            "sample": f"{nshot} shots, {nsteps + 1} forward + {nsteps} adjoint RK4 steps each with the gradient, "
                      f"same mesh and model, {dt:.2f} s"}


def reference_config(prob):
    """The `config` of the native arm's line for this workload."""
    from hirensi_b200.configs import RHO
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    m = prob.mesh
    if "sys" not in _CPU_SYS:
        om = O.OracleMesh(m, RHO)
        _CPU_SYS["sys"] = (om, O.OracleSystem.assemble(om, prob.lam0, prob.mu0))
    S = _CPU_SYS["sys"][1]
    nnz = [int(S.csr(w)[2].size) for w in range(3)]
    return {"workload": prob.name + f"_4shots_{prob.nstep}steps", "elements": m.nel, "nodes": m.nj,
            "dof": prob.dof, "equations": m.neq, "nnz_CKG": nnz, "shots_per_gpu": prob.nshot,
            "time_steps": prob.nstep, "dt": prob.dt}


def run_reference(args, rank, world):
    """The CPU restatement on the host cores.  Each step is a bounded sample of the
    workload step: all 4 shots, each with the same number of forward and adjoint
    steps (200, fewer when --steps + --warmup would take more than about three
    minutes), timed whole; ms_per_step is the time of that sample."""
    if rank != 0:
        return None
    from hirensi_b200.configs import inversion_config
    prob = inversion_config(nstep=args.nstep)
    cfg = reference_config(prob)
    probe = cpu_sample(prob, nsteps=20)               # sizes the sample; untimed
    per_step = probe["seconds"] / 41.0                 # one forward or adjoint step of all shots
    budget = 180.0 / max(1, args.steps + args.warmup)
    nsteps = int(max(50, min(200, budget / (2.0 * per_step))))
    for _ in range(args.warmup):
        cpu_sample(prob, nsteps=nsteps)
    vals = [cpu_sample(prob, nsteps=nsteps) for _ in range(args.steps)]
    secs = [x["seconds"] for x in vals]
    units = prob.dof * ((nsteps + 1) + nsteps) * prob.nshot
    v = units * len(secs) / sum(secs) / 1e9
    cb = dict(vals[-1])
    cb["value"] = v
    cb.pop("seconds", None)
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference", "config": cfg,
            "sample": f"each step: all {prob.nshot} shots, {nsteps + 1} forward + {nsteps} adjoint steps with the "
                      f"gradient (the workload step has {prob.nstep + 1} + {prob.nstep}); CPU restatement of the "
                      "reference solver (Fortran + PETSc are not in the image)",
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "native":
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    elif args.workload in ("uneven", "xl"):
        res = run_uneven(args, rank, world, local_rank)
    elif args.workload == "xl-fwi":
        res = run_xl_fwi(args, local_rank) if rank == 0 else None
    elif args.workload == "shot-scaling":
        res = run_shot_scaling(args, local_rank) if rank == 0 else None
    else:
        res = run_native(args, rank, world, local_rank)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)
    if world > 1 and args.impl == "native":
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
