#!/usr/bin/env python
"""Benchmark of the MQCT hot paths on B200.

Headline (`value`): the state-to-state matrix build of the asymmetric top + atom
workload (A, B, C = 27.9, 14.5, 9.3 cm^-1, j <= 8 all tau and m: 969 states,
31 977 same-m pairs; 12-term site-site PES; angular grid 48 GL beta x 48 gamma x
48 alpha as written; 300 R points 3-25 bohr), in matrix elements (pairs x R
points) per second.  One step = one full build: rotor basis + PES tables +
contraction + units/cutoff/spline, inputs resident on the device.

Secondary (`expansion`): the PES-expansion build through its C ABI on the inputs of
two reference examples (with the reference's logged single-rank build times) and a
larger synthetic system.

Secondary (`propagation`): batched trajectory propagation on that matrix
(trajectories with b ~ U(0,15) bohr, E log-uniform 50-2000 cm^-1, RK4 dt=5 a.u.
until R > 25 bohr), trajectories per second, FP32 arithmetic, and the plain
FP64 GPU form of both paths for the speed-up.

`--impl reference` times the reference algorithm on the host cores instead: the
CPU restatement of INTEGRATOR_TEMP (wavefunctions re-evaluated at every grid
point for every element and R, as the reference does) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = json.load(open(os.path.join(ROOT, "BASELINE.json")))["metric"]
WORKLOAD = ("asym-top+atom matrix build: j<=8 (969 states, 31977 pairs), grid 48 GL beta x "
            "48 gamma x 48 alpha, 300 R 3-25 bohr")
L2_NOTE = "GPU arm: L2 flushed (256 MB write) between timed steps"


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="mqct", choices=["mqct", "reference"])
    p.add_argument("--precision", default="auto", choices=["auto", "f16x3", "bf16x3", "fp64"])
    p.add_argument("--c3-traj", type=int, default=4096,
                   help="trajectories of the propagation workload timed (4096 = full set)")
    p.add_argument("--no-propagation", action="store_true")
    p.add_argument("--no-fp64-form", action="store_true")
    p.add_argument("--no-expansion", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--only-projection", type=int, default=0, metavar="NR",
                   help="run the CALC_EXPANSION_TERMS block alone on NR R points and print "
                        "it (a small case for profiling)")
    return p.parse_args()


# ---------------------------------------------------------------- workload
def workload():
    import mqct_b200 as mq
    from mqct_b200 import synthetic as syn
    c2 = syn.config_c2(alpha_grid=True)
    s = mq.CollisionSystem(4, c2["channels"], A=c2["A"], B=c2["B"], C=c2["C"])
    R = mq.r_grid(c2["nR"], c2["rmin"], c2["rmax"])
    return c2, s, R


TC_PROFILE = os.path.join(ROOT, "profiles", "tc_contract_kernel_asymtop_j8_48x48x48_R300.md")
PROJ_PROFILE = os.path.join(ROOT, "profiles", "proj_kernels_nd3d2_calcexp_R32.md")


def _profiled_traffic(path, key="dram_bytes_per_launch"):
    """DRAM bytes per launch (or per unit) recorded by the committed ncu summary (None if
    absent)."""
    try:
        for ln in open(path):
            if ln.strip().startswith(key + ":"):
                return float(ln.split(":", 1)[1].strip().split()[0])
    except OSError:
        pass
    return None


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- GPU arm
def _matrix_bench(mq, s, R, c2, precision, steps, warmup, torch, flush):
    plan = mq.MatrixPlan(s, R, c2["grid"], c2["pes"], precision=precision)
    n = s.P * len(R)
    d_mat = torch.empty(n, dtype=torch.float64, device="cuda")
    d_y2 = torch.empty(n, dtype=torch.float64, device="cuda")
    d_sk = torch.empty(s.P, dtype=torch.int32, device="cuda")
    # epilogue layout of the tensor-core contraction: each timed (minimum of three executes), the faster kept
    plan.tune(d_mat.data_ptr(), d_y2.data_ptr(), d_sk.data_ptr())
    plan.sync()
    for _ in range(warmup):
        plan.execute(d_mat.data_ptr(), d_y2.data_ptr(), d_sk.data_ptr())
        plan.sync()
    seg = []
    for _ in range(steps):
        flush()
        torch.cuda.synchronize()
        plan.execute(d_mat.data_ptr(), d_y2.data_ptr(), d_sk.data_ptr())
        seg.append(plan.timing())
    plan.sync()  # raises if a device-side wait of the timed builds ran out of rounds
    torch.cuda.synchronize()
    return plan, d_mat, d_sk, np.array(seg)


def _layout(plan):
    q, ks, parts = plan.layout()
    warps, tune_ms = plan.epilogue()
    return {"alpha_points_per_fp64_drain": q, "grid_chunk_ranges": ks, "radial_column_parts": parts,
            "epilogue_warps": warps,
            "epilogue_tune_ms": {"8_warps": tune_ms[0], "16_warps": tune_ms[1]}}


def run_gpu(a):
    import torch
    import mqct_b200 as mq
    from mqct_b200 import replicas
    from mqct_b200 import synthetic as syn

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    c2, s, R = workload()
    peaks, peak_src = _peaks()
    prec = {"auto": mq.PREC_F16X3, "f16x3": mq.PREC_F16X3, "bf16x3": mq.PREC_BF16X3,
            "fp64": mq.PREC_FP64}[a.precision]
    if a.precision == "auto":
        try:
            mq.MatrixPlan(s, R[:4], (8, 8, 0, 0, 0, 0, 1), c2["pes"], precision=prec).close()
        except mq.MqctError:
            prec = mq.PREC_FP64
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def flush():  # write 256 MB (> 126 MB L2) between timed steps
        flush_buf.fill_(1.0)

    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0] or 0)
    barrier()
    with Clocks(gpu_index) as clk:
        t0 = time.perf_counter()
        plan, d_mat, d_sk, seg = _matrix_bench(mq, s, R, c2, prec, a.steps, a.warmup, torch, flush)
        barrier()
        wall = time.perf_counter() - t0
    step_ms = seg.sum(axis=1)
    ms = replicas.max_over_ranks(float(np.mean(step_ms)), dist, device="cuda")
    n_el = s.P * len(R)
    value = world * n_el / (ms / 1e3)
    flops = plan.flops
    layout = _layout(plan) if prec != mq.PREC_FP64 else None
    contract_ms = float(np.mean(seg[:, 1]))
    achieved_tf = flops / (contract_ms / 1e3) / 1e12
    out = {}

    # plain FP64 GPU form of the same build, and the accuracy of the split path
    fp64 = None
    acc = None
    mat64_host = None
    if not a.no_fp64_form and prec != mq.PREC_FP64:
        plan64, d_mat64, d_sk64, seg64 = _matrix_bench(mq, s, R, c2, mq.PREC_FP64, 1, 1, torch, flush)
        ms64 = float(seg64.sum(axis=1).mean())
        c64 = float(seg64[:, 1].mean())
        fp64 = {"ms_per_step": ms64, "speedup": ms64 / ms,
                "form": "FP64 tensor cores (mma.sync m8n8k4 f64), the same grid and alpha points",
                "contraction_ms": c64,
                "contraction_fp64_tflops": plan64.flops / (c64 / 1e3) / 1e12}
        m1 = d_mat.view(s.P, len(R)).double()
        m0 = d_mat64.view(s.P, len(R)).double()
        acc = matrix_accuracy(m1, m0, d_sk, d_sk64, torch)
        mat64_host = m0.cpu().numpy()
        plan64.close()
    plan.close()
    del d_mat

    # the reference's own 2-D form of the same build (alpha integrated analytically,
    # K = 48 x 48 = 2304): time and accuracy of the split path against its FP64 form
    ref_form = None
    if not a.no_fp64_form and prec != mq.PREC_FP64:
        c2d = dict(c2, grid=(48, 48, 0, 0, 0, 0, 1))
        p2, dm2, ds2, sg2 = _matrix_bench(mq, s, R, c2d, prec, max(1, a.steps), 1, torch, flush)
        p2b, dm2b, ds2b, sg2b = _matrix_bench(mq, s, R, c2d, mq.PREC_FP64, 1, 1, torch, flush)
        ms2, ms2b = float(sg2.sum(axis=1).mean()), float(sg2b.sum(axis=1).mean())
        ref_form = {"grid": "48 GL beta x 48 gamma, alpha analytic (K = 2304)",
                    "ms_per_step": ms2, "value": n_el / (ms2 / 1e3), "fp64_ms_per_step": ms2b,
                    "speedup_vs_fp64_form": ms2b / ms2,
                    "segments_ms": {"basis_pes": float(sg2[:, 0].mean()),
                                    "contraction": float(sg2[:, 1].mean()),
                                    "finalize": float(sg2[:, 2].mean())},
                    "layout": _layout(p2),
                    "accuracy": matrix_accuracy(dm2.view(s.P, len(R)).double(),
                                                dm2b.view(s.P, len(R)).double(), ds2, ds2b, torch)}
        p2.close()
        p2b.close()
        del dm2, dm2b

    # e2e through the C ABI with host buffers (H2D of the system, D2H of Mat_el, y2, flags),
    # the host output arrays in pinned memory, allocated once and reused from call to call
    # as a host loop keeps them; the first call (untimed) makes the plan that later calls on
    # the same inputs reuse
    pinned = (torch.empty((s.P, len(R)), dtype=torch.float64, pin_memory=True),
              torch.empty((s.P, len(R)), dtype=torch.float64, pin_memory=True),
              torch.empty(s.P, dtype=torch.int32, pin_memory=True))
    out = tuple(t.numpy() for t in pinned)
    e2e_ms = []
    for i in range(max(1, a.warmup)):
        mq.build_matrix(s, R, c2["grid"], c2["pes"], precision=prec, out=out)
    for i in range(max(3, min(a.steps, 5))):
        flush()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        mat, y2, sk = mq.build_matrix(s, R, c2["grid"], c2["pes"], precision=prec, out=out)
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    mat = mat.copy()
    mq.release_cached_build()
    h2d = (s.ind_mat.nbytes + R.nbytes + s.indx_chann.nbytes * 3 + s.vec1.nbytes +
           c2["pes"]["params"].nbytes + c2["pes"]["sites1"].nbytes)
    d2h = mat.nbytes + y2.nbytes + sk.nbytes

    # propagation (secondary)
    prop = None
    if not a.no_propagation:
        prop = run_propagation(mq, syn, s, R, mat, a, torch, world, dist, mat64=mat64_host)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    expansion = None if a.no_expansion else run_expansion(mq, syn)
    projection = None if a.no_expansion else run_projection(mq, peaks)
    cpu = cpu_baseline_matrix(oracle_c2_system(), a.cpu_seconds)
    tc = prec in (mq.PREC_BF16X3, mq.PREC_F16X3)
    tc_name = "F16x3" if prec == mq.PREC_F16X3 else "BF16x3"
    peak = peaks.get("bf16_tflops", 1590.0)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "matrix elements/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": (tc_name.lower() + "-fp32acc") if tc else "f64",
        "data": "synthetic (seeded site-site PES; no dataset)",
        "config": {"workload": WORKLOAD, "l2": L2_NOTE},
        "build": {"precision": (tc_name + " tcgen05") if tc else "FP64 tensor cores (mma.sync f64)",
                  "layout": layout,
                  "elements_per_step": n_el, "grid_points": 48 * 48 * 48,
                  "parallelism": f"replicas x{world}"},
        "segments_ms": {"basis_pes": float(seg[:, 0].mean()), "contraction": contract_ms,
                        "finalize": float(seg[:, 2].mean())},
        "roofline": {"bound": "tensor" if tc else "fp64", "achieved": achieved_tf,
                     "peak": peak if tc else None, "unit": "TFLOP/s",
                     "frac": achieved_tf / peak if tc else None,
                     "traffic": _profiled_traffic(TC_PROFILE) if tc else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                       "launch, " + os.path.relpath(TC_PROFILE, ROOT),
                     "peak_source": f"bf16_tflops ({peak_src}; dense FP16 and BF16 rates are equal)",
                     "flops_per_launch": flops, "kernel": "contraction"},
        "cpu_baseline": cpu,
        "e2e": {"value": n_el / (float(np.median(e2e_ms)) / 1e3), "unit": "matrix elements/s",
                "ms": float(np.median(e2e_ms)), "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h),
                "note": "mqct_build_matrix on host arrays: inputs copied up and Mat_el, y2, "
                        "flags copied down every call into pinned host arrays (allocated "
                        "once, reused); the plan of the first (untimed) call on the same "
                        "inputs is reused"},
        "clocks": clk.summary(),
        # per build: rotor tables, basis, PES weights, [W column scaling (F16x3)], W image,
        # basis image, contraction, finalize; the FP64 form: tables, basis, PES, contraction,
        # finalize
        "gpu_launches": int(a.steps * ((8 if prec == mq.PREC_F16X3 else 7) if tc else 5)),
        "fp64_form": fp64,
        "accuracy": acc,
        "reference_2d_form": ref_form,
        "propagation": prop,
        "expansion": expansion,
        "projection": projection,
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def matrix_accuracy(m1, m0, sk1, sk0, torch):
    """Error of the split-precision matrix against the FP64 form of the same build.
    Pairs whose FP64 radial function stays below 1e-9 of the largest element vanish by
    symmetry (rounding noise only) and are excluded; for the rest e_k = max_R |dM_k| /
    max_R |M_k| (relative max-norm error of the radial function) and, per entry above
    1e-3 of its row maximum, |dM| / |M|."""
    rowmax = m0.abs().amax(dim=1)
    gmax = rowmax.max()
    sig = rowmax >= 1e-9 * gmax
    d = (m1 - m0).abs()
    e_k = (d.amax(dim=1)[sig] / rowmax[sig])
    big = (m0.abs() >= 1e-3 * rowmax[:, None]) & sig[:, None]
    rel = (d[big] / m0.abs()[big])
    samp = rel[torch.randperm(rel.numel(), device=rel.device)[:4_000_000]] if rel.numel() > 4_000_000 else rel
    flag_diff = (sk1 != sk0)
    return {"pairs_compared": int(sig.sum()), "pairs_zero_by_symmetry": int((~sig).sum()),
            "pair_maxnorm_rel_err": {"median": float(e_k.median()),
                                     "p99": float(torch.quantile(e_k, 0.99)),
                                     "max": float(e_k.max())},
            "entry_rel_err_above_1e-3_rowmax": {"median": float(samp.median()),
                                                "p99": float(torch.quantile(samp, 0.99)),
                                                "max": float(rel.max())},
            "max_abs_err_hartree": float(d.max()),
            "cutoff_flags_differing": int(flag_diff.sum()),
            "max_fp64_element_of_differing_flags": float(rowmax[flag_diff].max()) if bool(flag_diff.any()) else 0.0}


def run_propagation(mq, syn, s, R, mat, a, torch, world, dist=None, mat64=None):
    from mqct_b200 import replicas
    c3 = syn.config_c3()
    tab = mq.PropagationTables.from_system(s, R, mat, syn.config_c2()["mass_amu"])
    n = min(a.c3_traj, c3["n_traj"])
    E = c3["E_cm"][:n] * syn.CM_TO_HARTREE
    k = np.sqrt(2 * tab.mass_au * E)
    b = c3["b"][:n]
    l = np.sqrt(np.maximum((b * k) ** 2 + 0.25, 0.0)) - 0.5   # b = sqrt(l(l+1))/k
    trajs = [mq.Trajectory(float(E[i]), float(l[i]), 1, c3["dt"], c3["r_fin"], c3["r_fin"],
                           max_steps=400000) for i in range(n)]
    res = {}
    # right-hand-side work of the lockstep engine: the four knot products per m-block,
    # 2 (re, im) x 2 flops per matrix entry, 4 right-hand sides per RK4 step
    _, blk = np.unique(tab.m12, return_counts=True)
    flops_per_step = 4.0 * 16.0 * float((blk.astype(np.float64) ** 2).sum())
    props = torch.cuda.get_device_properties(0)
    fp32_peak = props.multi_processor_count * 128 * 2 * _peaks()[0].get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    probs = {}
    # fp32: the plan's own choice (for 4 096 trajectories the lockstep engine with its last
    # trajectories handed to the resident engine); the engines alone beside it
    runs = (("fp32", mq.PROP_FP32, mq.ENGINE_AUTO),
            ("fp32_lockstep", mq.PROP_FP32, mq.ENGINE_LOCKSTEP),
            ("fp32_per_trajectory", mq.PROP_FP32, mq.ENGINE_PER_TRAJECTORY),
            ("fp64", mq.PROP_FP64, mq.ENGINE_PER_TRAJECTORY))
    names = {mq.ENGINE_LOCKSTEP: "lockstep", mq.ENGINE_PER_TRAJECTORY: "per-trajectory",
             mq.ENGINE_RESIDENT: "resident",
             mq.ENGINE_LOCKSTEP_TAIL: "lockstep, last trajectories on the resident engine"}
    for name, arith, engine in runs:
        nt = n
        plan = mq.PropagationPlan(tab, arith)
        plan.set_engine(engine)
        plan.run(trajs[:min(8, nt)])  # warm-up
        if engine == mq.ENGINE_PER_TRAJECTORY:
            plan.tune(trajs[:nt])     # launch shape for these tables (capped probe runs)
        t0 = time.perf_counter()
        amp, cls, diag = plan.run(trajs[:nt])
        wall = time.perf_counter() - t0
        ms = replicas.max_over_ranks(plan.timing(), dist, device="cuda")
        steps = float(diag[:, 1].sum())
        eng, rounds = plan.engine()
        r = {"n_traj": nt, "kernel_ms": ms, "wall_s": wall,
             "traj_per_s": world * nt / (ms / 1e3), "traj_steps": steps,
             "engine": names[eng],
             "max_status": float(diag[:, 4].max())}
        if eng == mq.ENGINE_LOCKSTEP_TAIL:
            r["handed_to_resident"] = plan.handed()
        if eng in (mq.ENGINE_LOCKSTEP, mq.ENGINE_LOCKSTEP_TAIL):
            r["rounds"] = rounds
            r["rhs_flops_per_step"] = flops_per_step
            r["achieved_tflops"] = steps * flops_per_step / (ms / 1e3) / 1e12
            if arith == mq.PROP_FP32:
                r["fp32_peak_tflops_nominal"] = fp32_peak
                r["frac_of_fp32_peak"] = r["achieved_tflops"] / fp32_peak
        else:
            r["table_bytes_per_step"] = plan.bytes_per_step
            r["achieved_table_GBs"] = steps * plan.bytes_per_step / (ms / 1e3) / 1e9
            r["frac_of_hbm_peak"] = r["achieved_table_GBs"] / _peaks()[0]["hbm_gbs"]
            r["launch_shape"] = dict(zip(("threads_per_cta", "ctas_per_sm", "probe_ms"), plan.shape()))
        res[name] = r
        probs[name] = mq.channel_probabilities(amp, s.indx_chann, s.n_channels)
        plan.close()
    p32, p64 = probs["fp32"], probs["fp64"]
    res["max_abs_prob_diff_fp32_vs_fp64"] = float(np.abs(p32 - p64).max())
    res["max_abs_prob_diff_engines_fp32"] = float(np.abs(p32 - probs["fp32_per_trajectory"]).max())
    res["max_abs_prob_diff_fp32_vs_fp32_lockstep"] = float(np.abs(p32 - probs["fp32_lockstep"]).max())
    # opacity-weighted sums sum_traj (2l+1) P_f (cross sections up to a common factor) of
    # the FP32 run (the plan's choice) and the FP64 form over the same trajectories
    w = 2 * l[:n] + 1
    s32, s64 = (w[:, None] * p32).sum(0), (w[:, None] * p64).sum(0)
    keep = s64 > 1e-4 * s64[1:].max()
    keep[0] = False  # elastic channel
    res["sigma_rel_diff_fp32_vs_fp64"] = {
        "channels": int(keep.sum()),
        "max": float(np.max(np.abs(s32[keep] - s64[keep]) / s64[keep]))}
    res["speedup_fp32_vs_fp32_per_trajectory"] = (res["fp32"]["traj_per_s"] /
                                                  res["fp32_per_trajectory"]["traj_per_s"])
    res["speedup_fp32_vs_fp32_lockstep"] = (res["fp32"]["traj_per_s"] /
                                            res["fp32_lockstep"]["traj_per_s"])
    res["speedup_fp32_vs_fp64_form"] = res["fp32"]["traj_per_s"] / res["fp64"]["traj_per_s"]
    # the coupled-states approximation (CS_APPROX) on the same trajectories: only the
    # m-block of the initial state is streamed and propagated
    plan = mq.PropagationPlan(tab, mq.PROP_FP32)
    plan.set_coupled_states(True)
    plan.run(trajs[:8])
    amp, cls, diag = plan.run(trajs)
    ms = replicas.max_over_ranks(plan.timing(), dist, device="cuda")
    res["fp32_cs"] = {"n_traj": n, "kernel_ms": ms, "traj_per_s": world * n / (ms / 1e3),
                      "traj_steps": float(diag[:, 1].sum()),
                      "max_status": float(diag[:, 4].max())}
    plan.close()
    # a batch that cannot fill the GPU (132 trajectories, every 31st of the set): the
    # cluster-resident engine (the plan's choice for FP32 batches up to 1024) against the
    # per-trajectory kernel in FP32 and in FP64 (the FP64 form)
    small = trajs[::31][:132]
    sb = {"n_traj": len(small)}
    sp = {}
    for name, arith, engine in (("fp32_resident", mq.PROP_FP32, mq.ENGINE_RESIDENT),
                                ("fp32_per_trajectory", mq.PROP_FP32, mq.ENGINE_PER_TRAJECTORY),
                                ("fp64", mq.PROP_FP64, mq.ENGINE_PER_TRAJECTORY)):
        plan = mq.PropagationPlan(tab, arith)
        plan.set_engine(engine)
        plan.run(small[:8])
        amp, cls, diag = plan.run(small)
        ms = replicas.max_over_ranks(plan.timing(), dist, device="cuda")
        sb[name] = {"kernel_ms": ms, "traj_per_s": world * len(small) / (ms / 1e3),
                    "max_status": float(diag[:, 4].max())}
        if engine == mq.ENGINE_RESIDENT:
            sb[name]["cluster_ctas"], sb[name]["clusters"] = plan.cluster()
        sp[name] = mq.channel_probabilities(amp, s.indx_chann, s.n_channels)
        plan.close()
    sb["speedup_resident_vs_fp32_per_trajectory"] = (sb["fp32_per_trajectory"]["kernel_ms"] /
                                                     sb["fp32_resident"]["kernel_ms"])
    sb["speedup_resident_vs_fp64_form"] = sb["fp64"]["kernel_ms"] / sb["fp32_resident"]["kernel_ms"]
    sb["max_abs_prob_diff_resident_vs_fp64"] = float(np.abs(sp["fp32_resident"] - sp["fp64"]).max())
    res["small_batch"] = sb
    # cross sections from the split-precision matrix against those from the FP64 form's
    # matrix: the same 256 trajectories propagated in FP64 on each
    if mat64 is not None:
        tab64 = mq.PropagationTables.from_system(s, R, mat64, syn.config_c2()["mass_amu"])
        ns_ = min(256, n)
        sig = []
        for tb in (tab, tab64):
            pl = mq.PropagationPlan(tb, mq.PROP_FP64)
            amp_, _, _ = pl.run(trajs[:ns_])
            pl.close()
            p_ = mq.channel_probabilities(amp_, s.indx_chann, s.n_channels)
            sig.append(((2 * l[:ns_] + 1)[:, None] * p_).sum(0))
        keep = sig[1] > 1e-4 * sig[1][1:].max()
        keep[0] = False
        res["sigma_rel_diff_matrix_split_vs_fp64"] = {
            "trajectories": ns_, "channels": int(keep.sum()),
            "max": float(np.max(np.abs(sig[0][keep] - sig[1][keep]) / sig[1][keep]))}
    res["workload"] = (f"{n} of the 4096 trajectories (b~U(0,15), E log-uniform 50-2000 cm^-1, "
                       "dt=5 a.u., R>25 stop), c2 matrix, retained pairs "
                       f"{tab.P} of {s.P}")
    return res


# ---------------------------------------------------------------- CPU / reference arm
def _synthetic():
    """mqct_b200/synthetic.py loaded on its own (numpy only): the seeded inputs of the
    workloads, without importing the CUDA library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "mqct_synthetic_inputs", os.path.join(ROOT, "mqct_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def oracle_c2_system():
    """The c2 build's inputs from the oracle alone: levels and eigenvectors
    (orc_asym_top), states, pairs (orc_ind_mat), R grid (orc_rgrid) and the seeded PES;
    nothing of the CUDA library is loaded."""
    from oracle import pyoracle as po
    po.build()
    syn = _synthetic()
    c2 = syn.config_c2(alpha_grid=True)
    ch = np.asarray(c2["channels"], np.int32)
    ldv = 2 * int(ch[:, 0].max()) + 1
    e_ch = np.zeros(len(ch))
    vec = np.zeros((len(ch), ldv))
    for i, (j, ka, kc) in enumerate(ch):
        e, v = po.asym_top(c2["A"], c2["B"], c2["C"], int(j), int(ka), int(kc))
        e_ch[i] = e
        vec[i, :len(v)] = v
    osys = po.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=e_ch, vec1=vec.reshape(-1),
                           ldv=ldv)
    states = osys.states()
    ind = po.ind_mat(states[2])
    R = po.rgrid(c2["nR"], c2["rmin"], c2["rmax"])
    pd = c2["pes"]
    pes = po.OraclePes(pd["kind"], pd["n_terms"], pd["params"], sites1=pd["sites1"])
    return dict(c2=c2, osys=osys, states=states, ind=ind, R=R, pes=pes)


def cpu_baseline_matrix(sysd, seconds, n_threads=0, seed=0):
    """The reference algorithm (INTEGRATOR_TEMP restated, wavefunctions re-evaluated
    at every grid point for every element and R, as the reference does) on a bounded
    sample of the build: seeded elements spread over the whole pair list (every
    m-block and j), each at three R points spread over the grid (small, middle and
    large R).  A short probe sizes the sample to about `seconds` of work."""
    from oracle import pyoracle as po
    ind, R = sysd["ind"], sysd["R"]
    P = len(ind)
    cores = n_threads or os.cpu_count()
    r_sel = np.array([R[len(R) // 10], R[len(R) // 2], R[(9 * len(R)) // 10]])
    rng = np.random.default_rng(seed)

    def run(n_el):
        sel = np.sort(rng.choice(P, n_el, replace=False))
        sub = np.ascontiguousarray(ind[sel])
        t0 = time.perf_counter()
        po.integrate_elements(sysd["osys"], sysd["states"], sub, r_sel, sysd["c2"]["grid"],
                              sysd["pes"], literal=True, n_threads=n_threads)
        return time.perf_counter() - t0

    t1 = run(cores)
    n2 = int(max(cores, min(P, cores * max(1.0, seconds / max(t1, 1e-3)))))
    n2 = max(cores, (n2 // cores) * cores)
    t2 = run(n2)
    n_work = n2 * len(r_sel)
    return {"value": n_work / t2, "unit": "matrix elements/s", "cores": cores, "kind": "port",
            "sample": f"{n2} seeded elements spread over the {P} pairs x 3 R points "
                      f"({', '.join(f'{r:.2f}' for r in r_sel)} bohr) of the same build "
                      f"(literal INTEGRATOR_TEMP restatement of the oracle, {cores} OpenMP "
                      f"threads), {t2:.1f} s"}


GOLDEN = os.path.join(ROOT, "tests", "golden")


def run_expansion(mq, syn):
    """The PES-expansion build (EXPANSION_MATRIX_ELEMENT, MIJ_CUTOFF, spline) end to end
    through mqct_build_matrix_expansion (host arrays in, Mat_el and y2 out; transfers and
    set-up inside the time), on the inputs of two reference examples whose logs give the
    reference's single-rank build time, and on a larger asymmetric top + diatom system
    (j1 <= 6 all levels, j2 = 0, 2) with the same 83 terms.  The oracle's restatement of
    the same formulas (OpenMP, all host threads) is timed beside it."""
    from oracle import pyoracle as po
    po.build()
    g3 = np.load(os.path.join(GOLDEN, "g3_h2o_h2_type8.npz"))
    g5 = np.load(os.path.join(GOLDEN, "g5_h2o_h2_expansion_terms.npz"))
    g1 = np.load(os.path.join(GOLDEN, "g1_h2o_h2o_at.npz"))
    s8 = mq.CollisionSystem(8, g3["channels"], A=float(g3["A"]), B=float(g3["B"]),
                            C=float(g3["C"]), BE=float(g3["BE"]))
    s0 = mq.CollisionSystem(0, g1["channels"], A=float(g1["A"]), B=float(g1["B"]),
                            C=float(g1["C"]))
    big = [c + (j2,) for j2 in (0, 2) for c in syn.asym_channels(6)]
    sb = mq.CollisionSystem(8, big, A=float(g3["A"]), B=float(g3["B"]), C=float(g3["C"]),
                            BE=float(g3["BE"]))
    cases = [
        ("h2o_h2_type8", "H2O+H2 example (EXAMPLES_IO/SYS_TYPE_8/H2O_H2_MTRXCalculation): "
         "104 states, 891 pairs, 101 R, 83 terms", s8, g5, "CM-1", 127.174),
        ("h2o_h2o_type0", "H2O+H2O AT example, 2nd run (EXAMPLES_IO/SYS_TYPE_0/"
         "H2O_H2O_AT_Approximation): 81 states, 594 pairs, 171 R, 28 terms", s0, g1, "KCAL",
         283.947),
        ("asymtop_j6_diatom_j02", f"asym top j1<=6 + diatom j2=0,2: {sb.n_states} states, "
         f"{sb.P} pairs, 101 R, the 83 terms of the H2O+H2 example", sb, g5, "CM-1", None),
    ]
    import torch
    out = {}
    for key, desc, s, g, unit, ref_s in cases:
        R, lab, T = g["R"], g["labels"], g["terms"]
        times = []
        for i in range(12):
            t0 = time.perf_counter()
            mq.build_matrix_expansion(s, R, lab, T, e_unit=unit)
            times.append(time.perf_counter() - t0)
        ms = float(np.median(times[2:])) * 1e3
        ms_min = float(np.min(times[2:])) * 1e3
        n_el = s.P * len(R)
        # device times of the plan: the angular set-up, and one execute (contraction,
        # cut-off, spline) from terms resident on the device
        plan = mq.ExpansionPlan(s, R, lab)
        dT = torch.from_numpy(np.ascontiguousarray(T.T)).cuda()
        dm = torch.empty((s.P, len(R)), dtype=torch.float64, device="cuda")
        dy = torch.empty_like(dm)
        dk = torch.empty(s.P, dtype=torch.int32, device="cuda")
        ex = []
        for i in range(5):
            plan.execute(dT, dm, dy, dk, e_unit=unit)
            plan.sync()
            ex.append(plan.timing()[1])
        ang_ms = plan.timing()[0]
        ex_ms = float(np.median(ex[2:]))
        plan.close()
        del dT, dm, dy, dk
        # the oracle on a bounded sample of pairs (all of them for the small examples)
        ch = s.channels
        kp = min(s.P, 4000)
        ind = np.ascontiguousarray(s.ind_mat[:kp])
        t0 = time.perf_counter()
        if s.sys_type == 0:
            osys = po.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                                   e_ch=s.e_ch, vec1=s.vec1.reshape(-1),
                                   vec2=s.vec2.reshape(-1), ldv=s.ldv)
            po.expansion_matrix_type0(osys, osys.states(), ind, lab, T, mq.E_UNIT[unit])
        else:
            osys = po.OracleSystem(8, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], e_ch=s.e_ch,
                                   vec1=s.vec1.reshape(-1), ldv=s.ldv)
            po.expansion_matrix_type8(osys, osys.states(), ind, lab, T)
        tc = time.perf_counter() - t0
        out[key] = {"workload": desc, "elements": n_el, "ms_per_build_e2e": ms,
                    "ms_per_build_e2e_min": ms_min,
                    "elements_per_s_e2e": n_el / (ms / 1e3),
                    "device_ms_angular_setup": ang_ms, "device_ms_execute": ex_ms,
                    "elements_per_s_device": n_el / ((ang_ms + ex_ms) / 1e3),
                    "cpu_port_elements_per_s": kp * len(R) / tc,
                    "cpu_port_sample": f"{kp} pairs x {len(R)} R, {os.cpu_count()} OpenMP threads, "
                                       f"{tc:.2f} s",
                    "reference_log_single_rank_s": ref_s,
                    "speedup_vs_reference_log": (ref_s / (ms / 1e3)) if ref_s else None}
    return out


def run_projection(mq, peaks, nR=86):
    """CALC_EXPANSION_TERMS at the size of the reference's CALC_EXPANSION example for
    ND3+D2 (EXAMPLES_IO/SYS_TYPE_7/NH3_H2_CalcExpansion: 377 terms, GRD_R = 86,
    GRD_ANG1 = 40,40 (alpha2 40), GRD_ANG2 = 20,20 (beta1, beta2 20), GRD_ANG3 = 40,40
    (gamma1 40)), on a seeded PES table of that shape (the example's PES is a user
    Fortran routine).  Device times of the three contractions with V resident (V larger
    than L2, so every execute reads it from HBM), the end-to-end one-shot call on host
    buffers (V up, terms and terms_im down), and the oracle restatement on a bounded
    sample of (term, R) pairs, scaled to the full workload."""
    import torch

    from oracle import pyoracle as po
    labels = np.load(os.path.join(GOLDEN, "g5b_nd3_d2_type7.npz"))["labels"]
    shape = (40, 20, 20, 40)
    rng = np.random.default_rng(7)
    V = (rng.standard_normal((nR,) + shape) * 500.0).astype(np.float64)
    G = int(np.prod(shape))
    nt = len(labels)
    pp = mq.ProjectionPlan(7, labels, shape)
    dV = torch.from_numpy(V).cuda()
    dT = torch.empty((nt, nR), dtype=torch.float64, device="cuda")
    dI = torch.empty_like(dT)
    torch.cuda.synchronize()
    seg = []
    for i in range(8):
        pp.execute(dV, nR, dT, dI)
        pp.sync()
        seg.append(pp.timing())
    seg = np.array(seg[3:])
    ga, al, te = (float(np.median(seg[:, k])) for k in range(3))
    pp.close()
    del dV, dT, dI
    n_out = nt * nR
    # end to end: host V (pinned) in, both term arrays out; plan set-up inside the time
    Vp = torch.from_numpy(V).pin_memory()
    Vh = Vp.numpy()
    e2e = []
    for i in range(6):
        t0 = time.perf_counter()
        mq.project_terms(7, labels, Vh)
        e2e.append(time.perf_counter() - t0)
    e2e_ms = float(np.median(e2e[2:])) * 1e3
    # the oracle on a sample: 4 terms (one per nju1 and the largest l) at 2 R points
    pick = [0, int(np.argmax(labels[:, 1] == 3)), int(np.argmax(labels[:, 1] == 6)),
            int(np.argmax(labels[:, 0] + labels[:, 2]))]
    t0 = time.perf_counter()
    po.project_terms(7, labels[pick], V[:2])
    tc = time.perf_counter() - t0
    per_pair_s = tc / (len(pick) * 2)
    # algorithmic HBM bytes of the gamma contraction: V read once, F written once
    n_pairs = len(set(int(x) for x in labels[:, 1]))
    f_bytes = nR * shape[0] * shape[1] * shape[2] * n_pairs * 16
    alg = V.nbytes + f_bytes
    hbm = peaks.get("hbm_gbs", 6650.0)
    return {"workload": "ND3+D2 CALC_EXPANSION size (SYS_TYPE 7): 377 terms, 86 R, grid "
                        "alpha2 40 x beta1 20 x beta2 20 x gamma1 40 (640000 points), "
                        "seeded PES table",
            "V_bytes": int(V.nbytes), "terms_per_call": n_out,
            "device_ms": {"gamma": ga, "alpha2": al, "beta_terms": te, "total": ga + al + te},
            "terms_per_s_device": n_out / ((ga + al + te) / 1e3),
            "e2e": {"ms": e2e_ms, "terms_per_s": n_out / (e2e_ms / 1e3),
                    "h2d_bytes": int(V.nbytes), "d2h_bytes": int(2 * n_out * 8)},
            "roofline_gamma": {"bound": "hbm", "algorithmic_bytes": int(alg),
                               "traffic": (None if _profiled_traffic(PROJ_PROFILE,
                                                                     "dram_bytes_per_R_point")
                                           is None else
                                           _profiled_traffic(PROJ_PROFILE,
                                                             "dram_bytes_per_R_point") * nR),
                               "traffic_source": "ncu DRAM bytes of the gamma kernel at 32 R "
                                                 "points, scaled by R points, "
                                                 + os.path.relpath(PROJ_PROFILE, ROOT),
                               "achieved_gbs": alg / (ga / 1e3) / 1e9, "peak_gbs": hbm,
                               "frac": alg / (ga / 1e3) / 1e9 / hbm},
            "cpu_port": {"terms_per_s": 1.0 / per_pair_s,
                         "sample": f"{len(pick)} terms x 2 R (each a sum over the 640000 grid "
                                   f"points), {os.cpu_count()} OpenMP threads, {tc:.2f} s",
                         "full_workload_s_estimate": per_pair_s * n_out}}


def run_reference(a):
    """--impl reference: the oracle's restatement of the reference's INTEGRATOR_TEMP on
    the host cores, inputs built by the oracle alone (the CUDA library is not loaded);
    every step a bounded sample of the c2 build, the line's value the median over the
    timed steps."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sysd = oracle_c2_system()
    for i in range(a.warmup):
        cpu_baseline_matrix(sysd, 0.5, seed=1000 + i)
    t0 = time.perf_counter()
    vals, last = [], None
    for i in range(a.steps):
        last = cpu_baseline_matrix(sysd, a.cpu_seconds / 3, seed=i)
        vals.append(last["value"])
    v = float(np.median(vals))
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "matrix elements/s",
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": (time.perf_counter() - t0) / a.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded site-site PES; no dataset)",
            "config": {"workload": WORKLOAD, "l2": L2_NOTE},
            "cpu_baseline": dict(last, value=v,
                                 sample=f"median of {a.steps} steps, each: " + last["sample"]),
            "e2e": {"value": v, "unit": "matrix elements/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    a = _args()
    if a.only_projection:
        import mqct_b200 as mq
        print(json.dumps(run_projection(mq, _peaks()[0], nR=a.only_projection)), flush=True)
        return
    if a.impl == "reference":
        run_reference(a)
    else:
        run_gpu(a)


if __name__ == "__main__":
    main()
