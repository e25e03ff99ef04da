#!/usr/bin/env python
"""Benchmark: N=5 10-eigenpair shift-and-invert Lanczos solve on one B200
(mixed precision form vs plain FP64), one JSON line on stdout.

A step is one complete solve of the 10 smallest eigenpairs of the
null-space-free reduced Maxwell operator at N=5 (NF = 10^6 modes,
2*NF = 2e6 complex unknowns; golden-ratio cut matrix, eps = 1 + 12 prod
(1+cos x_d)/2, q = (0.05,0.04,0.03); Krylov block 40, outer tol 1e-8, inner
Mhat PCG tol 1e-10), followed by a Rayleigh-Ritz step with the exact K_r on the
10 Ritz vectors.  Setup (mass/basis/operator handles) is outside the timed region,
as in the reference's timing.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fame|reference]

Multi-GPU runs are replicas (independent solves, one per rank, no data-path
collective); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "null--space-free-6d-projection-method_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "N=5 10-eigenpair solve s & Yee pts/s, mixed vs FP64 on 1 B200 at 1e-8 resid"
N_BENCH = 5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["fame", "reference"], default="fame")
    ap.add_argument("--N", type=int, default=N_BENCH)
    ap.add_argument("--case", choices=["chain", "pcg", "solve", "yee", "recon", "grad", "osi", "rank1", "peaks"],
                    default=None,
                    help="run one piece of the step alone (for profiling), print its device time")
    ap.add_argument("--precision", choices=["fp32", "fp64", "mixed"], default="mixed")
    ap.add_argument("--reps", type=int, default=3)
    return ap.parse_args()


def workload_config(N):
    return {
        "workload": "N=%d null-space-free Maxwell, NF=%d, 2NF=%d complex unknowns, 10 smallest "
                    "eigenpairs, shift 0, Krylov block 40, outer tol 1e-8, inner Mhat PCG tol 1e-10"
                    % (N, (2 * N) ** 6, 2 * (2 * N) ** 6),
        "material": "eps = 1 + 12*prod_d (1+cos x_d)/2",
        "cut_matrix": "[I3; diag(phi, 1/phi, phi^2)]",
        "q": [0.05, 0.04, 0.03],
        "form": "mixed: complex64 mass + FP32 PCG inside FP64 refinement; FP64 Lanczos",
        "l2": "Krylov basis (1.28 GB) larger than L2, plus a 256 MB L2 flush between steps",
        "setup": "excluded (mass/basis/operator handles built before timing)",
    }


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.strip().split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if "Active" in v and "Not" not in v:
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


TAYLOR_TC_FORM = ("moments as split-FP32 (3xTF32) tcgen05 MMAs, operands generated in shared memory, FP32 TMEM "
                  "accumulation over 512-mode slices, FP64 slice sum and evaluation")


def ncu_traffic(kind):
    """Per-launch DRAM bytes of the dominant chain from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "mhat_chain_traffic.json")) as f:
            return json.load(f).get(kind)
    except Exception:
        return None


# ----------------------------------------------------------------- fame arm
def reduce_max_over_ranks(x, world, device):
    """The largest value of x over the ranks of the process group (every rank calls it
    at the same point); the job's time is the slowest replica's."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_line(world, rank, seconds_per_step, steps, device):
    """Whole-job figures of independent replicas (one solve per rank and step): the
    step time is the maximum over ranks and the throughput counts every rank's solves."""
    t = reduce_max_over_ranks(seconds_per_step, world, device)
    return {"seconds_per_step": t, "ms_per_step": round(t * 1e3, 3), "solves_per_s_all_gpus": round(world / t, 4),
            "n_gpus": world, "steps": steps}


def run_fame(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import fame_b200 as F

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", torch.cuda.current_device())
    N = args.N
    NF = (2 * N) ** 6
    cfg = F.configs
    S = cfg.SOLVE

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max_over_ranks(x, world, dev)

    # ---- setup (untimed)
    E = cfg.material_separable_cos(N, 12.0, device=dev)
    mass = F.MassBackend(E, N)
    sysq = F.build_q_system(mass, cfg.P_GOLDEN, cfg.Q_PHYS)
    v0 = F.start_vector(cfg.SEED, sysq.nr)
    ops = {}
    ops["mixed"] = F.make_explicit_krinv_compact(sysq, S["tolCG"], S["maxitCG"], precision="mixed",
                                                 **cfg.MIXED_OPTS)[0]
    ops["fp64"] = F.make_explicit_krinv_compact(sysq, S["tolCG"], S["maxitCG"], precision="fp64")[0]
    # the reference algorithm's inner solve (plain Mhat CG, exp1/make_explicit_krinv_compact.m:43) in FP64
    ops["fp64_plain"] = F.make_explicit_krinv_compact(sysq, S["tolCG"], S["maxitCG"], precision="fp64",
                                                      mhatPreconditioner=0)[0]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def solve(prec):
        """One step: the 10-eigenpair Lanczos solve, then Rayleigh-Ritz with the exact K_r."""
        Y, theta, steps, info = F.Lanczos(ops[prec], None, None, sysq.nr, S["nev"], S["tol"], S["maxRestart"],
                                          S["p"], v0)
        lam, relres = F.rayleigh_ritz(sysq, Y)
        return dict(Y=Y, theta=theta, info=info, lam=lam, relres=relres, lam_raw=np.sort(1.0 / theta))

    def timed_steps(prec, steps):
        times, launches = [], 0
        res = None
        for _ in range(steps):
            # the previous step's eigenvectors go back to the allocator first, so that every
            # step reuses one cached output block instead of one step mapping a second one
            res = None
            flush.zero_()
            barrier()
            l0 = F.kernel_launches()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            res = solve(prec)
            e1.record()
            barrier()
            launches += F.kernel_launches() - l0
            times.append(e0.elapsed_time(e1) / 1e3)
        return times, launches, res

    for _ in range(max(args.warmup, 0)):
        solve("mixed")
    solve("fp64")
    solve("fp64_plain")
    barrier()

    sampler = ClockSampler(dev.index)
    sampler.start()
    time.sleep(1.0)  # let the sampler's NVML start-up finish before the timed region
    for prec in ops:
        ops[prec].reset_stats()
    t_mixed, launches, res_mixed = timed_steps("mixed", args.steps)
    st_mixed = ops["mixed"].stats()
    clocks = sampler.stop()
    job = replica_line(world, rank, sum(t_mixed) / len(t_mixed), args.steps, dev)
    step_s = job["seconds_per_step"]
    # the comparison forms: median of three solves each (one solve alone is exposed to the
    # occasional slow step)
    t_fp64, _, res_fp64 = timed_steps("fp64", 3)
    fp64_s = max_over_ranks(sorted(t_fp64)[1])
    st_fp64 = ops["fp64"].stats()
    t_plain, _, res_plain = timed_steps("fp64_plain", 3)
    plain_s = max_over_ranks(sorted(t_plain)[1])
    st_plain = ops["fp64_plain"].stats()

    def rel_max(a, b):
        return float(np.max(np.abs(np.asarray(a) - np.asarray(b)) / np.abs(np.asarray(b))))

    lam_err = rel_max(res_mixed["lam"], res_fp64["lam"])
    lam_err_raw = rel_max(res_mixed["lam_raw"], res_fp64["lam_raw"])

    # ---- dominant kernel chain: Mhat (3 fields through passes A/B/C)
    def chain_time(dtype, reps=40):
        x = torch.randn(NF, dtype=dtype, device=dev)
        for _ in range(5):
            F.apply_Mhat_C_scalar_compact(x, sysq)
        torch.cuda.synchronize()
        s = torch.cuda.current_stream()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            F.apply_Mhat_C_scalar_compact(x, sysq)
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    peak, peak_kind = measured_peaks()
    bytes32 = 156.0 * NF  # algorithmic bytes per FP32 Mhat chain (3 passes, 3 fields)
    bytes64 = 312.0 * NF
    t32 = chain_time(torch.complex64)
    t64 = chain_time(torch.complex128)
    ach32 = bytes32 / t32 / 1e9
    ach64 = bytes64 / t64 / 1e9

    # ---- Yee-field reconstruction of eigenmode 10 (h = 0.0125, n = 40; 3 components)
    yee = None
    try:
        y10 = res_fp64["Y"][:, 9].contiguous()  # refined vectors are in ascending lambda order
        X, MX, _ = F.recover_original_eigenvectors(y10.reshape(-1, 1), sysq, 1e-12, 3000)
        x10 = X[:, 0].contiguous()
        n_yee, h_yee = 40, 0.0125
        pts, axes, sz = F.build_yee_points(n_yee, h_yee)
        M = pts[0].shape[0]
        Qm = F.build_projected_q_modes(sysq)
        blocks = F.build_yee_block_partition(sz, 4)

        def recon(method):
            if method.startswith("direct"):  # the three components in one call (GEMMs batched over them)
                return F.reconstruct_fields_direct_grid(x10, sysq, axes, tensor_cores=(method == "direct_tc"))
            return [F.taylor_on_blocks(x10[c * NF:(c + 1) * NF], Qm, pts[c], 10, blocks,
                                       tensor_cores=(method == "taylor_tc")) for c in range(3)]

        times = {}
        fields = {}
        for method in ("direct", "direct_tc", "taylor", "taylor_tc"):
            recon(method)
            samples = []
            for _ in range(5):  # median of 5 (three components each)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                fields[method] = recon(method)
                torch.cuda.synchronize()
                samples.append(time.perf_counter() - t0)
            times[method] = sorted(samples)[len(samples) // 2]

        def field_err(x, y):
            return float(sum(torch.linalg.norm(a - b) ** 2 for a, b in zip(x, y)) ** 0.5 /
                         sum(torch.linalg.norm(b) ** 2 for b in y) ** 0.5)
        err = field_err(fields["taylor"], fields["direct"])
        yee = {"points_per_component": M, "n": n_yee, "h": h_yee, "mode": 10,
               "direct_pts_per_s": round(3 * M / times["direct"], 1),
               "taylor_p10_64c_pts_per_s": round(3 * M / times["taylor"], 1),
               "taylor_rel_err_vs_direct": err, "timing": "median of 5 repetitions, 3 components each",
               "direct_3xtf32_pts_per_s": round(3 * M / times["direct_tc"], 1),
               "direct_3xtf32_rel_err_vs_fp64": field_err(fields["direct_tc"], fields["direct"]),
               "taylor_3xtf32_pts_per_s": round(3 * M / times["taylor_tc"], 1),
               "taylor_3xtf32_rel_err_vs_fp64_taylor": field_err(fields["taylor_tc"], fields["taylor"]),
               "taylor_3xtf32_rel_err_vs_direct": field_err(fields["taylor_tc"], fields["direct"]),
               "taylor_3xtf32_form": TAYLOR_TC_FORM,
               "direct_form": "factorised tensor-grid sum (axis-block cut matrix), three components per GEMM launch, FP64",
               "taylor_form": "multi-center Taylor p=10, 4^3 centers, FP64"}
        # LWRQ validation of the reconstructed field (material sampled on the Yee edges)
        lam10 = float(res_fp64["lam"][9])
        F.compute_yee_lwrq_metrics(fields["direct"], lam10, cfg.P_GOLDEN, n_yee, h_yee, ("cos", 12.0))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lw, _ = F.compute_yee_lwrq_metrics(fields["direct"], lam10, cfg.P_GOLDEN, n_yee, h_yee, ("cos", 12.0))
        t_lw = time.perf_counter() - t0
        yee["lwrq"] = {k: lw[k] for k in ("lambda3D", "eta3D", "deltaLambda", "nuLWRQ", "deltaPart")}
        yee["lwrq"]["seconds"] = round(t_lw, 5)
    except Exception as exc:  # reported, not hidden
        yee = {"error": repr(exc)}

    # ---- batched Bloch path: 12 q-points, N = 3,4,5 round-robin, mixed precision
    bloch = None
    try:
        qs, Ns = cfg.bloch_path(4)
        qs = [np.array(qv) for qv in qs]
        qs[0] = qs[0] + cfg.GAMMA_SHIFT  # the reduction is singular at Gamma
        mats = [cfg.material_separable_cos(Nq, 12.0, device=dev) for Nq in Ns]
        F.solve_batch(Ns, mats, qs, cfg.P_GOLDEN, nev=S["nev"], tol=S["tol"], p=S["p"], tolCG=S["tolCG"], **cfg.MIXED_OPTS)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lam_b, infos_b = F.solve_batch(Ns, mats, qs, cfg.P_GOLDEN, nev=S["nev"], tol=S["tol"], p=S["p"],
                                       tolCG=S["tolCG"], **cfg.MIXED_OPTS)
        torch.cuda.synchronize()
        t_batch = time.perf_counter() - t0

        def sequential(prec):
            t0 = time.perf_counter()
            for i in range(len(Ns)):
                F.solve_batch([Ns[i]], [mats[i]], [qs[i]], cfg.P_GOLDEN, nev=S["nev"], tol=S["tol"], p=S["p"],
                              tolCG=S["tolCG"], precision=prec, **(cfg.MIXED_OPTS if prec == "mixed" else {}))
            torch.cuda.synchronize()
            return time.perf_counter() - t0
        t_seq = sequential("mixed")
        t_seq64 = sequential("fp64")
        # the autotuner's schedule and pass tile shape per N (tuning untimed, like the handles)
        t0 = time.perf_counter()
        tuned = F.tune_batch(Ns, mats, qs, cfg.P_GOLDEN, tolCG=S["tolCG"], **cfg.MIXED_OPTS)
        t_tune = time.perf_counter() - t0
        F.solve_batch(Ns, mats, qs, cfg.P_GOLDEN, nev=S["nev"], tol=S["tol"], p=S["p"], tolCG=S["tolCG"], tuned=tuned,
                      **cfg.MIXED_OPTS)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lam_t, _ = F.solve_batch(Ns, mats, qs, cfg.P_GOLDEN, nev=S["nev"], tol=S["tol"], p=S["p"], tolCG=S["tolCG"],
                                 tuned=tuned, **cfg.MIXED_OPTS)
        torch.cuda.synchronize()
        t_tuned = time.perf_counter() - t0
        bloch = {"points": len(Ns), "N": Ns, "batched_s": round(t_batch, 4), "sequential_s": round(t_seq, 4),
                 "batch_speedup": round(t_seq / t_batch, 3),
                 "batched_tuned_s": round(t_tuned, 4), "tuned": {str(k): v for k, v in tuned.items()},
                 "tuning_s": round(t_tune, 2),
                 "tuned_lambda_max_rel_diff": float(np.max(np.abs(lam_t - lam_b) / np.abs(lam_b))),
                 "fp64_sequential_s": round(t_seq64, 4),
                 "mixed_batched_vs_fp64_sequential": round(t_seq64 / t_batch, 3),
                 "converged": all(i["converged"] for i in infos_b),
                 "gamma": "q = Gamma + %s (the null-space-free reduction is singular at Gamma)"
                          % [float(v) for v in cfg.GAMMA_SHIFT],
                 "lambda_1": [float(v) for v in lam_b[:, 0]]}
    except Exception as exc:
        bloch = {"error": repr(exc)}

    # ---- end to end through the public API from host buffers
    e2e = None
    if rank == 0 or world > 1:
        E_h = E.cpu().pin_memory()
        v0_h = v0.cpu().pin_memory()
        torch.cuda.synchronize()

        def e2e_once():
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            Ed = E_h.to(dev, non_blocking=True)
            vd = v0_h.to(dev, non_blocking=True)
            m2 = F.MassBackend(Ed, N)
            s2 = F.build_q_system(m2, cfg.P_GOLDEN, cfg.Q_PHYS)
            op2, _ = F.make_explicit_krinv_compact(s2, S["tolCG"], S["maxitCG"], precision="mixed",
                                                   **cfg.MIXED_OPTS)
            Y, theta, _, _ = F.Lanczos(op2, None, None, s2.nr, S["nev"], S["tol"], S["maxRestart"], S["p"], vd)
            lam, _ = F.rayleigh_ritz(s2, Y)  # the eigenvalues arrive on the host with the call
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            del op2, s2, m2, Y
            return dt, lam

        # cold: the device memory pool returned to the driver first, so every handle maps fresh memory
        torch.cuda.empty_cache()
        F._lib.lib.fame_device_trim_memory(dev.index)
        cold, lam = e2e_once()
        reps = max(1, min(args.steps, 2))
        tot = 0.0
        for _ in range(reps):
            dt, lam = e2e_once()
            tot += dt
        h2d = E_h.numel() * 8 + v0_h.numel() * 16
        d2h = 8 * len(lam)
        e2e = {"value": max_over_ranks(tot / reps), "unit": "s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "cold_first_call_s": max_over_ranks(cold),
               "includes": "H2D of eps and v0 from pinned memory, handle setup (mass, basis, K_r^{-1}), solve, "
                           "Rayleigh-Ritz, D2H of the 10 eigenvalues; the eigenvectors stay in device memory, as "
                           "the reference's gpuArray results do; value: warm (pool blocks cached by the previous "
                           "call), cold_first_call_s: first call after the pool was returned to the driver"}

    # ---- CPU baseline and parity against the oracle (rank 0, N=1 only)
    cpu = None
    parity = None
    if rank == 0 and world == 1:
        legs = cpu_oracle_legs(N, n3_solve=True, tight=True)
        cpu = cpu_line(legs, steps_in_solve=res_mixed["info"]["steps"])
        parity = gpu_parity(F, legs, ops, sysq, S, dev)

    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(step_s, 6), "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_s * 1e3, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64/f32 mass+PCG, f64 refinement+Lanczos+Rayleigh-Ritz", "data": "synthetic",
            "config": workload_config(N),
            "fp64_solve_s": round(fp64_s, 6), "mixed_speedup_vs_fp64": round(fp64_s / step_s, 3),
            "fp64_plain_solve_s": round(plain_s, 6), "mixed_speedup_vs_fp64_plain": round(plain_s / step_s, 3),
            "forms": {"mixed": "FP32 preconditioned Mhat PCG inside FP64 refinement",
                      "fp64": "FP64 Mhat PCG preconditioned by the inverse-material operator",
                      "fp64_plain": "FP64 plain Mhat CG, the reference's pcg(Mhat, ...)"},
            "eig_rel_err_mixed_vs_fp64": lam_err, "eig_rel_err_mixed_vs_fp64_raw": lam_err_raw,
            "rayleigh_ritz_relres_max": float(np.max(res_mixed["relres"])),
            "lanczos_steps": res_mixed["info"]["steps"], "converged": res_mixed["info"]["converged"],
            "step_s": [round(t, 6) for t in t_mixed],
            "inner": {"mixed": {"krinv_calls": st_mixed.inverseCalls,
                                "fp32_pcg_iters_per_call": round(st_mixed.fp32Iterations / max(1, st_mixed.inverseCalls), 2),
                                "fp64_refinements_per_call": round(st_mixed.refineSteps / max(1, st_mixed.inverseCalls), 2)},
                      "fp64": {"krinv_calls": st_fp64.inverseCalls,
                               "pcg_iters_per_call": round(st_fp64.totalIterations / max(1, st_fp64.inverseCalls), 2)},
                      "fp64_plain": {"krinv_calls": st_plain.inverseCalls,
                                     "pcg_iters_per_call": round(st_plain.totalIterations / max(1, st_plain.inverseCalls), 2)}},
            "solves_per_s_all_gpus": job["solves_per_s_all_gpus"],
            "parity": parity,
            "yee_pts_per_s": (yee or {}).get("direct_pts_per_s"),
            "yee": yee,
            "bloch_path": bloch,
            "roofline": {"bound": "hbm", "achieved": round(ach32, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(ach32 / peak, 4), "traffic": ncu_traffic("fp32"),
                         "kernel": "Mhat chain FP32 (passes A/B/C, 3 fields), %.1f us/launch" % (t32 * 1e6),
                         "algorithmic_bytes": bytes32, "peak_source": peak_kind,
                         "fp64_chain": {"achieved": round(ach64, 1), "frac": round(ach64 / peak, 4),
                                        "us": round(t64 * 1e6, 2), "algorithmic_bytes": bytes64,
                                        "traffic": ncu_traffic("fp64")}},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    del ops
    if world > 1:
        dist.destroy_process_group()


# ------------------------------------------------------------ CPU reference
def cpu_oracle_legs(N, n3_solve=True, tight=False):
    """CPU legs on the host cores, through the oracle only (this function loads no CUDA
    library): (i) one explicit K_r^{-1} action at N on the normalised start vector, with
    the reference algorithm (plain Mhat PCG, tolCG 1e-10: exp1/make_explicit_krinv_compact.m);
    (ii) optionally the full N=3 10-eigenpair solve at the benchmark settings
    (exp2/Lanczos.m + the explicit K_r^{-1}), followed by the oracle's Rayleigh-Ritz."""
    import numpy as np
    import oracle as O
    from oracle import workloads as W
    cores = os.cpu_count() or 1
    O.set_fft_workers(cores)
    SV = W.SOLVE
    out = {"cores": cores}
    E = O.material_separable_cos(N, 12.0)
    S = O.build_q_system(N, W.P_GOLDEN, W.Q_PHYS, E)
    op, stats = O.make_explicit_krinv_compact(S, SV["tolCG"], SV["maxitCG"])
    v0 = O.start_vector(W.SEED, S.nr)
    v0 = v0 / np.linalg.norm(v0)
    t0 = time.perf_counter()
    y = op(v0)
    out["action"] = {"N": N, "seconds": time.perf_counter() - t0, "iters": stats()["totalMhatIterations"],
                     "y": y, "v0": v0}
    if tight:  # the same action at tolCG 1e-13 (untimed): the common exact reference for parity
        out["action"]["y_tight"] = O.make_explicit_krinv_compact(S, 1e-13, SV["maxitCG"])[0](v0)
    if n3_solve:
        S3 = O.build_q_system(3, W.P_GOLDEN, W.Q_PHYS, O.material_separable_cos(3, 12.0))
        t0 = time.perf_counter()
        sol = O.solve_modes(S3, nev=SV["nev"], p=SV["p"], tol=SV["tol"], maxRestart=SV["maxRestart"],
                            tolCG=SV["tolCG"], seed=W.SEED, maxitCG=SV["maxitCG"])
        dt = time.perf_counter() - t0
        out["n3"] = {"seconds": dt, "steps": int(sol["steps"]), "lam": sol["lam"],
                     "lam_rr": O.rayleigh_ritz_Kr(sol["Y"], S3)[0]}
    return out


def cpu_line(legs, steps_in_solve, kind="port"):
    """The cpu_baseline object: the N=5 solve extrapolated from the measured K_r^{-1}
    action (labelled), and the measured full N=3 solve."""
    a = legs["action"]
    d = {"value": round(a["seconds"] * steps_in_solve, 6), "unit": "s", "cores": legs["cores"], "kind": kind,
         "extrapolated": True, "action_seconds": round(a["seconds"], 6), "lanczos_steps": steps_in_solve,
         "sample": "one explicit K_r^{-1} action at N=%d (FP64 NumPy/pocketfft oracle of the reference algorithm, "
                   "%d threads, %d plain Mhat PCG iterations, %.2f s) x %d Lanczos steps of the solve"
                   % (a["N"], legs["cores"], a["iters"], a["seconds"], steps_in_solve)}
    if "n3" in legs:
        d["n3_full_solve_s"] = round(legs["n3"]["seconds"], 3)
        d["n3_lanczos_steps"] = legs["n3"]["steps"]
    return d


def gpu_parity(F, legs, ops, sysq, S, dev):
    """Parity of the benchmarked GPU paths against the oracle on the same inputs: the N=5
    K_r^{-1} action on the normalised start vector (both precision forms, and a tight FP64
    action as the common exact reference; at tolCG 1e-10 the oracle's own action is ~3e-9
    from the exact one, so the GPU and the oracle are also compared with both at tolCG
    1e-13), and the N=3 eigenvalues at the benchmark settings
    (raw 1/theta and after Rayleigh-Ritz, against the oracle's raw and refined values)."""
    import numpy as np
    import torch
    out = {"settings": "tol %g, tolCG %g, p %d, nev %d" % (S["tol"], S["tolCG"], S["p"], S["nev"])}
    a = legs["action"]
    y_o = a["y"]
    vd = torch.as_tensor(a["v0"], device=dev)

    def rel(x, y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    tight = F.make_explicit_krinv_compact(sysq, 1e-13, 3000, precision="fp64")[0]
    y_t = tight(vd).cpu().numpy()
    out["krinv_n%d_oracle_rel_vs_tight" % a["N"]] = rel(y_o, y_t)
    if "y_tight" in a:  # both sides at tolCG 1e-13: GPU FP64 vs the oracle
        out["krinv_n%d_tight_rel_vs_oracle_tight" % a["N"]] = rel(y_t, a["y_tight"])
    for prec in ("fp64", "mixed"):
        y = ops[prec](vd).cpu().numpy()
        out["krinv_n%d_%s_rel_vs_oracle" % (a["N"], prec)] = rel(y, y_o)
        out["krinv_n%d_%s_rel_vs_tight" % (a["N"], prec)] = rel(y, y_t)
    del tight
    if "n3" in legs:
        E3 = F.configs.material_separable_cos(3, 12.0, device=dev)
        m3 = F.MassBackend(E3, 3)
        s3 = F.build_q_system(m3, F.configs.P_GOLDEN, F.configs.Q_PHYS)
        op3 = F.make_explicit_krinv_compact(s3, S["tolCG"], S["maxitCG"], precision="mixed",
                                            **F.configs.MIXED_OPTS)[0]
        Y, theta, _, info = F.Lanczos(op3, None, None, s3.nr, S["nev"], S["tol"], S["maxRestart"], S["p"],
                                      F.start_vector(F.configs.SEED, s3.nr))
        lam_raw = np.sort(1.0 / theta)
        lam_rr, _ = F.rayleigh_ritz(s3, Y)
        o = legs["n3"]
        out["eig_n3_mixed_raw_rel_vs_oracle_raw"] = float(np.max(np.abs(lam_raw - o["lam"]) / o["lam"]))
        out["eig_n3_mixed_rr_rel_vs_oracle_rr"] = float(np.max(np.abs(lam_rr - o["lam_rr"]) / o["lam_rr"]))
        out["eig_n3_oracle_raw_rel_vs_oracle_rr"] = float(np.max(np.abs(o["lam"] - o["lam_rr"]) / o["lam_rr"]))
    return out


def run_case(args):
    """One piece of the benchmark step, repeated ``--reps`` times on cuda:0:

    * ``chain``: the Mhat action (passes A/B/C over 3 fields), FP32 (``--precision
      fp32``/``mixed``) or FP64 — the kernel chain the roofline line reports;
    * ``pcg``: one explicit K_r^{-1} action (``--precision mixed|fp64``);
    * ``solve``: one full 10-eigenpair Lanczos solve (the timed step).
    """
    import torch
    import fame_b200 as F
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if args.case == "grad":
        return grad_case(F, args)
    if args.case == "osi":
        return osi_case(F, args)
    if args.case == "rank1":
        return rank1_case(F, args)
    if args.case == "peaks":
        return peaks_case(args)
    N = args.N
    NF = (2 * N) ** 6
    cfg = F.configs
    S = cfg.SOLVE
    E = cfg.material_separable_cos(N, 12.0, device=dev)
    mass = F.MassBackend(E, N)
    sysq = F.build_q_system(mass, cfg.P_GOLDEN, cfg.Q_PHYS)
    v0 = F.start_vector(cfg.SEED, sysq.nr)
    prec = "fp64" if args.precision == "fp64" else "mixed"
    if args.case == "yee":
        return yee_sweep(F, cfg, sysq, v0, args)
    if args.case == "recon":
        return recon_case(F, cfg, sysq, v0, args)
    if args.case == "chain":
        x = torch.randn(NF, dtype=torch.complex128 if prec == "fp64" else torch.complex64, device=dev)
        body = lambda: F.apply_Mhat_C_scalar_compact(x, sysq)  # noqa: E731
    else:
        op = F.make_explicit_krinv_compact(sysq, S["tolCG"], S["maxitCG"], precision=prec,
                                           **(cfg.MIXED_OPTS if prec == "mixed" else {}))[0]
        if args.case == "pcg":
            q = (v0 / torch.linalg.norm(v0)).reshape(-1, 1)
            body = lambda: op(q)  # noqa: E731
        else:
            body = lambda: F.Lanczos(op, None, None, sysq.nr, S["nev"], S["tol"],  # noqa: E731
                                     S["maxRestart"], S["p"], v0)
    body()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = F.kernel_launches()
    e0.record()
    for _ in range(args.reps):
        body()
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"case": args.case, "N": N, "precision": prec, "reps": args.reps,
                      "s_per_rep": e0.elapsed_time(e1) / 1e3 / args.reps,
                      "launches_per_rep": (F.kernel_launches() - l0) / args.reps}), flush=True)


def grad_case(F, args):
    """Hellmann-Feynman gradients of the 10 smallest eigenvalues with respect to the 7
    material parameters theta = (delta = 12, a_1..a_6 ~ U[0.5, 1], seeded) at N = 6 (NF =
    2,985,984): time of solve + eigenvector recovery + mass adjoint, and a central finite
    difference (step 1e-6) of d lambda / d delta as the check."""
    import numpy as np
    import torch
    N = 6 if args.N == N_BENCH else args.N
    prec = "fp64" if args.precision == "fp64" else "mixed"
    kw = dict(nev=10, tolCG=1e-12, tol=1e-10, precision=prec)
    theta = np.concatenate([[12.0], F.configs.gradient_amplitudes()])
    F.grad.eigenvalue_gradients(2, theta, **kw)  # warm-up (kernels, workspaces)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lam, dlam = F.grad.eigenvalue_gradients(N, theta, **kw)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    h = 1e-6
    tp, tm = theta.copy(), theta.copy()
    tp[0] += h
    tm[0] -= h
    fd = (F.grad.eigenpairs(N, tp, **kw)[0] - F.grad.eigenpairs(N, tm, **kw)[0]) / (2 * h)
    print(json.dumps({"case": "grad", "N": N, "NF": (2 * N) ** 6, "precision": prec, "modes": 10, "params": 7,
                      "seconds_solve_recover_adjoint": t, "lambda": lam.tolist(),
                      "dlambda_ddelta": dlam[:, 0].tolist(),
                      "fd_rel_err_ddelta": float(np.max(np.abs(dlam[:, 0] - fd) / np.abs(fd)))}), flush=True)


def peaks_case(args):
    """Roofline denominators for the tensor-core and FP64 kernels, measured on this GPU with
    the vendor library (cuBLAS through torch.matmul; used as the yardstick only, never on the
    solver path): dense TF32 GEMM and FP64 GEMM throughput, 8192^3, after warm-up, median of
    ``--reps`` bursts of 10 products timed with CUDA events."""
    import torch
    dev = torch.device("cuda", 0)
    out = {"case": "peaks"}
    prev = torch.backends.cuda.matmul.allow_tf32
    try:
        for name, dt, tf32 in (("tf32_tflops", torch.float32, True), ("fp64_tflops", torch.float64, False),
                               ("fp32_simt_tflops", torch.float32, False)):
            torch.backends.cuda.matmul.allow_tf32 = tf32
            n = 8192
            a = torch.randn(n, n, dtype=dt, device=dev)
            b = torch.randn(n, n, dtype=dt, device=dev)
            c = torch.empty(n, n, dtype=dt, device=dev)
            for _ in range(3):
                torch.matmul(a, b, out=c)
            torch.cuda.synchronize()
            rates = []
            for _ in range(max(3, args.reps)):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(10):
                    torch.matmul(a, b, out=c)
                e1.record()
                torch.cuda.synchronize()
                rates.append(10 * 2 * n ** 3 / (e0.elapsed_time(e1) / 1e3) / 1e12)
            out[name] = sorted(rates)[len(rates) // 2]
            del a, b, c
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    print(json.dumps(out), flush=True)


def rank1_case(F, args):
    """The rank-1 lattice transforms of the radix plan at N (exp1/rank1_exact_fft_scatter.m,
    exp1/rank1_exact_ifft_gather.m; M = 2N (4N-1)^5): device time of one scatter (embed +
    length-M FFT) and one gather (length-M inverse FFT + gather), median of ``--reps``, and the
    HBM rate of their Stockham passes (each pass reads and writes M complex128)."""
    import numpy as np
    import torch
    N = args.N
    n = 2 * N
    B = 2 * n - 1
    NF, M = n ** 6, n * B ** 5
    codes = np.zeros(NF, dtype=np.int64)
    tmp = np.arange(NF, dtype=np.int64)
    for j in range(6):  # exp1/build_radix_exact_rank1_plan_scalar.m:33-41
        codes += (tmp % n) * B ** j
        tmp //= n
    target = (codes + (n - 1) * sum(B ** j for j in range(6))) % M
    plan = dict(NF=NF, M=M, inputIdx=(codes + 1).astype(np.uint32), targetIdx=(target + 1).astype(np.uint32))
    x = F.start_vector(7, NF)
    ts = {"scatter": [], "gather": []}
    for _ in range(max(1, args.reps) + 1):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        X = F.rank1_exact_fft_scatter(x, plan)
        e[1].record()
        F.rank1_exact_ifft_gather(X, plan)
        e[2].record()
        torch.cuda.synchronize()
        ts["scatter"].append(e[0].elapsed_time(e[1]) / 1e3)
        ts["gather"].append(e[1].elapsed_time(e[2]) / 1e3)
    med = {k: sorted(v[1:])[len(v[1:]) // 2] for k, v in ts.items()}
    passes, m = 0, M
    for r in (27, 23, 19, 16, 15, 14, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2):
        while m % r == 0:
            m //= r
            passes += 1
    print(json.dumps({"case": "rank1", "N": N, "M": M, "NF": NF, "passes": passes,
                      "scatter_s": med["scatter"], "gather_s": med["gather"],
                      "stockham_gbs_gather": passes * 2 * M * 16 / med["gather"] / 1e9}), flush=True)


def osi_case(F, args):
    """Method A (the original shift-invert, exp1/run_method_A_fig1a.m) against method C on
    the same Bloch point: reference material (epsC = 4, alpha = 1.2), P = [I; diag(sqrt 2,
    sqrt 3, sqrt 5)], q = (0.13, 0.21, 0.17), 10 eigenvalues to 1e-10, sigma = 1e-4,
    MINRES and CG tolerance 1e-10; N = 3 and 5 (or --N)."""
    import numpy as np
    import torch
    cfg = F.configs
    dev = torch.device("cuda", 0)
    for N in ([3, 5] if args.N == N_BENCH else [args.N]):
        E = cfg.material_smooth_exp(N, 4.0, 1.2, device=dev)
        eMean, eMax = float(E.mean()), float(E.max())
        m = F.MassBackend(E, N)
        s = F.build_q_system(m, cfg.P_REFERENCE, cfg.Q_TRACKING)
        F.eigs_method_A(s, nev=10, sigma=1e-4, epsMean=eMean, epsMax=eMax, tol=1e-10, p=40)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lamA, _, infoA, stA = F.eigs_method_A(s, nev=10, sigma=1e-4, epsMean=eMean, epsMax=eMax, tol=1e-10, p=40)
        torch.cuda.synchronize()
        tA = time.perf_counter() - t0
        out = {}
        for prec in ("fp64", "mixed"):
            op = F.make_explicit_krinv_compact(s, 1e-10, 3000, precision=prec)[0]
            v0 = F.start_vector(cfg.SEED, s.nr)
            F.Lanczos(op, None, None, s.nr, 10, 1e-10, 30, 40, v0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, th, _, infoC = F.Lanczos(op, None, None, s.nr, 10, 1e-10, 30, 40, v0)
            torch.cuda.synchronize()
            out[prec] = (time.perf_counter() - t0, np.sort(1.0 / th), infoC)
        lamC = out["fp64"][1]
        print(json.dumps({"case": "osi", "N": N, "NF": (2 * N) ** 6, "method_A_s": round(tA, 4),
                          "method_A_lanczos_steps": infoA["steps"], "method_A_converged": infoA["converged"],
                          "method_A_minres_iterations": stA["totalMINRESIterations"],
                          "method_A_shifted_solves": stA["topVectorApplications"],
                          "method_A_plateau_accepts": stA["totalPlateauAccepts"],
                          "method_A_max_true_relres": stA["maxTrueRelres"],
                          "method_C_fp64_s": round(out["fp64"][0], 4), "method_C_mixed_s": round(out["mixed"][0], 4),
                          "method_C_lanczos_steps": out["fp64"][2]["steps"],
                          "speedup_C_mixed_over_A": round(tA / out["mixed"][0], 2),
                          "lambda_rel_diff_A_vs_C": float(np.max(np.abs(lamA - lamC) / lamC)),
                          "lambda": lamC.tolist()}), flush=True)


def recon_case(F, cfg, sysq, v0, args):
    """Eigenmode 10 at N=5 on the n = 40 window (h = 0.0125): ``--reps`` times the three
    components by the batched direct grid (FP64 and 3xTF32) and by 3xTF32 Taylor (p = 10,
    4^3 centers), timed per repetition (for profiling the reconstruction kernels)."""
    import numpy as np
    import torch
    S = cfg.SOLVE
    op = F.make_explicit_krinv_compact(sysq, S["tolCG"], S["maxitCG"], precision="fp64")[0]
    Y, theta = F.Lanczos(op, None, None, sysq.nr, S["nev"], S["tol"], S["maxRestart"], S["p"], v0)[:2]
    F.rayleigh_ritz(sysq, Y)
    X, _, _ = F.recover_original_eigenvectors(Y[:, 9].reshape(-1, 1).contiguous(), sysq, 1e-12, 3000)
    x3 = X[:, 0].contiguous()
    NF = sysq.NF
    pts, axes, sz = F.build_yee_points(40, 0.0125)
    Qm = F.build_projected_q_modes(sysq)
    blocks = F.build_yee_block_partition(sz, 4)
    out = {}
    for name, fn in (("direct_fp64", lambda: F.reconstruct_fields_direct_grid(x3, sysq, axes, tensor_cores=False)),
                     ("direct_3xtf32", lambda: F.reconstruct_fields_direct_grid(x3, sysq, axes, tensor_cores=True)),
                     ("taylor_3xtf32", lambda: [F.taylor_on_blocks(x3[c * NF:(c + 1) * NF], Qm, pts[c], 10, blocks,
                                                                   tensor_cores=True) for c in range(3)])):
        ts = []
        for _ in range(max(1, args.reps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        out[name] = sorted(ts)[len(ts) // 2]
    M3 = sum(int(p.shape[0]) for p in pts)
    print(json.dumps({"case": "recon", "n": 40, "points": M3,
                      **{k + "_pts_per_s": M3 / v for k, v in out.items()}}), flush=True)


def yee_sweep(F, cfg, sysq, v0, args):
    """Yee-field reconstruction of eigenmode 10 over the window sizes n = 40..200 (h =
    0.0125), Taylor orders p = 6, 8, 10 and m^3 centers, m = 1..6: points/s (median of
    ``--reps``, three components) and the field error against the FP64 direct sum."""
    import numpy as np
    import torch
    S = cfg.SOLVE
    op = F.make_explicit_krinv_compact(sysq, S["tolCG"], S["maxitCG"], precision="fp64")[0]
    Y, theta = F.Lanczos(op, None, None, sysq.nr, S["nev"], S["tol"], S["maxRestart"], S["p"], v0)[:2]
    th = theta.cpu().numpy() if torch.is_tensor(theta) else np.asarray(theta)
    i10 = int(np.argsort(1.0 / th)[9])
    X, _, _ = F.recover_original_eigenvectors(Y[:, i10].reshape(-1, 1).contiguous(), sysq, 1e-12, 3000)
    NF = sysq.NF
    xc = [X[c * NF:(c + 1) * NF, 0].contiguous() for c in range(3)]
    Qm = F.build_projected_q_modes(sysq)

    def timed(fn):
        fn()
        ts = []
        for _ in range(max(1, args.reps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return sorted(ts)[len(ts) // 2], out

    def err(a, b):
        return float(sum(torch.linalg.norm(x - y) ** 2 for x, y in zip(a, b)) ** 0.5 /
                     sum(torch.linalg.norm(y) ** 2 for y in b) ** 0.5)

    for n in (40, 80, 120, 160, 200):
        pts, axes, sz = F.build_yee_points(n, 0.0125)
        M3 = sum(int(p.shape[0]) for p in pts)
        x3 = X[:, 0].contiguous()
        t64, ref = timed(lambda: F.reconstruct_fields_direct_grid(x3, sysq, axes))
        ttc, dtc = timed(lambda: F.reconstruct_fields_direct_grid(x3, sysq, axes, tensor_cores=True))
        print(json.dumps({"case": "yee", "n": n, "method": "direct", "pts_per_s_fp64": M3 / t64,
                          "pts_per_s_3xtf32": M3 / ttc, "rel_err_3xtf32": err(dtc, ref)}), flush=True)
        for p in (6, 8, 10):
            for m in range(1, 7):
                blocks = F.build_yee_block_partition(sz, m)
                row = {"case": "yee", "n": n, "method": "taylor", "p": p, "m": m}
                for tc in (False, True):
                    t, u = timed(lambda: [F.taylor_on_blocks(xc[c], Qm, pts[c], p, blocks, tensor_cores=tc)
                                          for c in range(3)])
                    key = "3xtf32" if tc else "fp64"
                    row["pts_per_s_" + key] = M3 / t
                    row["rel_err_" + key] = err(u, ref)
                print(json.dumps(row), flush=True)
                del u
        del pts, ref, dtc
        torch.cuda.empty_cache()


def run_reference(args):
    """The reference arm: the reference's algorithm on the host cores through the FP64
    oracle (MATLAB/Octave are not installed here; nothing of the CUDA library is loaded).
    A timed step is one explicit K_r^{-1} action at N=5 (the unit of the solve: the
    solve is 40 of them); the line's value is the N=5 solve time extrapolated from the
    mean step (labelled), and one full N=3 solve is timed beside it.  Under torchrun
    only rank 0 runs; the other ranks exit without work."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    N = args.N
    steps_in_solve = 40  # Lanczos steps of the N=5 solve: p = 40, converged in the first cycle
    secs = []
    legs = None
    for i in range(args.warmup + args.steps):
        legs = cpu_oracle_legs(N, n3_solve=False)
        if i >= args.warmup:
            secs.append(legs["action"]["seconds"])
    per_action = sum(secs) / len(secs)
    legs["action"]["seconds"] = per_action
    legs["n3"] = cpu_oracle_legs(3, n3_solve=True)["n3"]
    cb = cpu_line(legs, steps_in_solve, kind="port")
    v = cb["value"]
    line = {
        "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(per_action * 1e3, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(N), "impl": "reference", "cpu_baseline": cb, "extrapolated": True,
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "MATLAB/Octave are not installed; the reference path is the NumPy FP64 restatement of the reference "
                "algorithm (oracle), timed on the host cores.  Each timed step is one explicit K_r^{-1} action at "
                "N=%d (ms_per_step); value = the mean step x %d Lanczos steps (extrapolated N=%d solve); "
                "cpu_baseline.n3_full_solve_s is a measured full N=3 solve." % (N, steps_in_solve, N),
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.case:
        run_case(args)
    else:
        run_fame(args)


if __name__ == "__main__":
    main()
