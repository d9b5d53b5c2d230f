"""LGF-FMM Poisson benchmark (one JSON line on rank 0).

A step is one PoissonSolver::apply_lgf on the AMR workload (8^3 base blocks of
16^3 cells, 3 mesh levels, seeded sum-of-Gaussians source): every FMM sweep of
every level, the level transfers and the correction, as the reference's
"Rate" (tests/poisson/vortexrings.hpp:292-298) times it. `value` is cells per
second with the source already in HBM (device-timed, CUDA events on the
library's stream, max over ranks); `e2e` adds the pinned host->device copy of
the source and the device->host copy of the solution through the C ABI, both as
the leaf blocks' interiors (iblgf_field_upload_leaves /
download_leaves_async: a step's solution copy overlaps the next step's upload
and solve; every copy completes inside the timed region).

--gpus N runs N independent replicas (one process per GPU); the solve has no
data-path collective.
--impl reference times the CPU restatement of the reference algorithm (oracle)
on the host cores for the same workload and metric.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "iblgf-amr_b200"))

import iblgf_setups as S  # noqa: E402

METRIC = "LGF-FMM cells/s, NS step ms: FP32-batched vs FP64 plain, 1 B200, rel err\u22641e-5"
# DRAM bytes (read + written) of the spectral MAC per solve, from one ncu capture of the five
# MAC launches of an amr_3level solve on the FP32 path (dram__bytes_read.sum +
# dram__bytes_write.sum, profiles/group_mac_dram_amr_3level.md); per solve like `achieved`
MAC_DRAM_BYTES = {("amr_3level", "fp32", 0): 4232.1e6}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            # the timed region starts once sampling has started
            self.first = self.proc.stdout.readline()
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in [self.first] + out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def build_case(name):
    return S.GaussianPoisson(name)


def cpu_reference(case, steps, warmup, sample_levels=None):
    """Time the oracle (CPU restatement, all host threads) on the workload."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    d = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    src = case.fields(d)
    cells = case.n_cells(d)
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        d.apply_lgf(src)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    return cells, times, os.cpu_count()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="amr_3level")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="with --gpus N > 1: one octree sharded over the ranks (the reference server's partition, "
                         "an NCCL all-reduce of each sweep's level targets) instead of N independent replicas")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 plain comparison run")
    ap.add_argument("--no-ns", action="store_true", help="skip the IF-HERK step measurement")
    ap.add_argument("--no-adapt", action="store_true", help="skip the adaptive IF-HERK march measurement")
    ap.add_argument("--ns-only", action="store_true", help="only the IF-HERK step measurement (profiling)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-problems measurement")
    ap.add_argument("--batch-only", action="store_true", help="only the batched-problems measurement (profiling)")
    ap.add_argument("--no-ib", action="store_true", help="skip the immersed-boundary NS step measurement")
    ap.add_argument("--mac-variant", type=int, default=-1, choices=[-1, 0, 1, 2, 3],
                    help="pin the sibling-group MAC variant (-1: autotune per plan)")
    ap.add_argument("--ib-only", action="store_true", help="only the immersed-boundary NS step measurement")
    ap.add_argument("--helm-only", action="store_true",
                    help="only the Fourier-in-z 2-D block operators (bandwidth of each)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    case = build_case(args.workload)
    wl = ("%s: %d^3 base blocks of %d^3 cells, %d refinement levels, sum-of-Gaussians source (seeded)"
          % (case.name, case.blocks[0][1][0] // case.block_extent, case.block_extent, case.n_levels))

    if args.impl == "reference":
        if rank != 0:
            return
        # warm spectrum cache, as the metric defines cells/s: one untimed solve
        steps = max(1, min(args.steps, 2))
        warm = 1
        cells, times, cores = cpu_reference(case, steps, warm)
        v = cells / float(np.mean(times))
        line = {"metric": METRIC, "value": v, "unit": "cells/s", "n_gpus": args.gpus, "steps": steps,
                "warmup": warm, "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "impl": "reference",
                "config": {"workload": wl, "cells_per_step": cells},
                "cpu_baseline": {"value": v, "unit": "cells/s", "cores": cores, "kind": "port",
                                 "sample": "full apply_lgf per step (steps capped at 2) after one untimed "
                                           "solve that fills the LGF spectrum cache"},
                "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch

    import iblgf_b200 as B
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    if args.ns_only:
        if rank == 0:
            out = {"ns_step": ns_bench(B, stream, local, args.steps, args.warmup)}
            if not args.no_adapt:
                out["ns_step_adaptive"] = ns_adapt_bench(B, stream, local, args.steps, args.warmup)
            print(json.dumps(out), flush=True)
        return
    if args.ib_only:
        if rank == 0:
            print(json.dumps({"ns_step_ib": ib_bench(B, stream, local, args.steps, args.warmup)}), flush=True)
        return
    if args.helm_only:
        if rank == 0:
            print(json.dumps({"helm_ops": helm_bench(B, stream, local, args.steps, args.warmup)}), flush=True)
        return
    if args.batch_only:
        if rank == 0:
            print(json.dumps({"batch": batch_bench(B, stream, local, args.steps, args.warmup)}), flush=True)
        return
    prec = B.FP32 if args.precision == "fp32" else B.FP64
    g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate, precision=prec, device=local,
                 stream=stream.cuda_stream)
    g.mac_variant(args.mac_variant)
    src_host = case.fields(g)
    cells = case.n_cells(g)
    sharded = args.shard and world > 1
    if sharded:
        import sharding
        g.set_owner(g.partition(world), rank, sharding.torch_allreduce_exchange())
    fs, ft = g.field(src_host), g.field()
    for _ in range(args.warmup):
        g.apply_lgf(fs, ft)
    g.synchronize()
    # the group-MAC autotuner's measurements (first warm-up solve, per plan)
    tuning = g.mac_tuning()

    # ---- device-timed region: inputs resident in HBM (> L2: fields and spectra)
    g.profile(True)
    l0 = g.launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as ck:
        ev0.record(stream)
        for _ in range(args.steps):
            g.apply_lgf(fs, ft)
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = g.launches() - l0
    ms = ev0.elapsed_time(ev1)
    phases = g.profile_read()
    stats = g.stats()
    g.profile(False)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    # replicas: every rank solves the whole problem; sharded: one problem
    value = (1 if sharded else world) * cells / (ms_step * 1e-3)

    # ---- end to end through the C ABI with pinned host buffers: the leaf
    # interiors (the cells the metric counts) in, the solution on them out
    leaf = (g.flags & 1) != 0
    hsrc = torch.from_numpy(np.ascontiguousarray(src_host[leaf][:, 1:-1, 1:-1, 1:-1])).pin_memory()
    hout = torch.empty(hsrc.shape, dtype=torch.float64).pin_memory()
    nbytes = hsrc.numel() * 8
    L = B.lib()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # untimed: the first asynchronous copies create the copy stream and the
    # device staging buffers
    g._check(L.iblgf_field_upload_leaves_async(g.h, fs, hsrc.data_ptr(), hsrc.numel()))
    g.apply_lgf(fs, ft)
    g._check(L.iblgf_field_download_leaves_async(g.h, ft, hout.data_ptr(), hout.numel()))
    g.synchronize()
    e0.record(stream)
    # every step copies its input in and its solution out through the C ABI;
    # both copies run on the library's copy stream: the next step's input is
    # issued right after this step's solve and copies under it, the solution
    # copies under the next solve; all copies end before e1
    g._check(L.iblgf_field_upload_leaves_async(g.h, fs, hsrc.data_ptr(), hsrc.numel()))
    for k in range(args.steps):
        g.apply_lgf(fs, ft)
        if k + 1 < args.steps:
            g._check(L.iblgf_field_upload_leaves_async(g.h, fs, hsrc.data_ptr(), hsrc.numel()))
        g._check(L.iblgf_field_download_leaves_async(g.h, ft, hout.data_ptr(), hout.numel()))
    g.synchronize()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    # ---- launch overhead: the same solve replayed from a CUDA graph (every
    # launch of one apply_lgf recorded once); equal times mean the step is not
    # launch-bound, the premise a persistent work-queue sweep would need
    graph_rec = None
    if rank == 0 and not sharded:
        try:
            g.synchronize()
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg, stream=stream, capture_error_mode="relaxed"):
                g.apply_lgf(fs, ft)
            for _ in range(2):
                cg.replay()
            torch.cuda.synchronize()
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream)
            with torch.cuda.stream(stream):
                for _ in range(args.steps):
                    cg.replay()
            q1.record(stream)
            torch.cuda.synchronize()
            graph_rec = {"ms_per_step_graph_replay": q0.elapsed_time(q1) / args.steps,
                         "ms_per_step_direct_launches": ms_step, "launches_per_step": launches / args.steps}
            del cg
        except Exception as ex:  # a capture the runtime refuses is reported, not fatal
            graph_rec = {"unavailable": str(ex)[:200]}

    # ---- FP64 plain path on the same input, and accuracy of this run against it
    extra = {}
    out64 = None
    if rank == 0 and prec == B.FP32 and not args.no_fp64:
        g64 = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                       n_levels=case.n_levels, predicate=case.predicate, precision=B.FP64, device=local,
                       stream=stream.cuda_stream)
        f64s, f64t = g64.field(src_host), g64.field()
        for _ in range(2):
            g64.apply_lgf(f64s, f64t)
        g64.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(max(2, args.steps // 2)):
            g64.apply_lgf(f64s, f64t)
        a1.record(stream)
        torch.cuda.synchronize()
        ms64 = a0.elapsed_time(a1) / max(2, args.steps // 2)
        out32 = g.download(ft)
        out64 = g64.download(f64t)
        rel = float(np.abs(out32 - out64).max() / np.abs(out64).max())
        extra = {"fp64_plain": {"value": cells / (ms64 * 1e-3), "ms_per_step": ms64},
                 "speedup_vs_fp64_plain": ms64 / ms_step, "rel_linf_vs_fp64": rel}
        g64.close()

    # ---- roofline of the dominant phase (phase times from CUDA events on the stream)
    hbm, peak_kind = peaks()
    fma = g.fma_peak(prec)
    # the tensor cores' issue rate at the MAC's product shape and at full width
    tc_rate = {str(n): g.tc_mma_rate(n) for n in (16, 64, 256)} if rank == 0 else None
    names = ["forward transforms", "spectral MAC", "inverse transforms+interp+add", "zero/copy/anterp"]
    k = int(np.argmax(phases))
    per_step = phases / args.steps
    nc = g.Nb * (2 * g.Nb - 1) ** 2
    cb = 8 if prec == B.FP32 else 16
    sweeps, nsrc, ntgt, npairs, nuniq = [int(x) / args.steps for x in stats[:5]]
    if k == 1:
        flops = 8.0 * nc * npairs
        bytes_alg = (nuniq + nsrc + ntgt) * nc * cb
    elif k == 0:
        P = 2 * g.Nb - 1
        flops = nsrc * 8.0 * (g.Nb ** 3 * g.Nb / 2 + P * g.Nb ** 3 + P * P * g.Nb * g.Nb)
        bytes_alg = nsrc * (g.Nb ** 3 * 8 + nc * cb)
    else:
        P = 2 * g.Nb - 1
        flops = ntgt * 8.0 * (P * P * g.Nb * g.Nb + P * g.Nb ** 3 + g.Nb ** 4 / 2)
        bytes_alg = ntgt * (nc * cb + g.Nb ** 3 * 16)
    t_k = per_step[k] * 1e-3
    # the CUDA-core roofline is taken on the floating-point work the kernels
    # execute; for the MAC that is less than the pair list's 8 Nc flops per
    # pair (block-Toeplitz products), which is reported beside it
    exec_flops = float(stats[9]) / args.steps * nc if k == 1 else flops
    ai = flops / max(bytes_alg, 1)
    if ai > fma * 1e12 / (hbm * 1e9):
        roof = {"bound": "fp-cuda-core", "achieved": exec_flops / t_k / 1e12, "peak": fma, "unit": "TFLOP/s",
                "frac": exec_flops / t_k / 1e12 / fma,
                "peak_source": "measured FMA-chain kernel (iblgf_fma_peak)"}
    else:
        roof = {"bound": "hbm", "achieved": bytes_alg / t_k / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": bytes_alg / t_k / 1e9 / hbm, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"}
    chosen = {r["choice"] for r in tuning} if args.mac_variant < 0 else {args.mac_variant}
    traffic = MAC_DRAM_BYTES.get((args.workload, args.precision, min(chosen) if len(chosen) == 1 else -1)) \
        if k == 1 else None
    roof.update({"kernel": names[k], "traffic": traffic,
                 "traffic_source": "ncu capture of the MAC launches of one solve (profiles/group_mac_dram_amr_3level.md)"
                 if traffic else None,
                 "phase_ms_per_step": dict(zip(names, per_step.tolist())),
                 "algorithmic_flops": flops, "algorithmic_bytes": bytes_alg})
    if k == 1:
        # the pair list's work (8 Nc flops per (target, source) pair) per
        # second, and the products the sibling groups cover
        nexec = int(stats[8]) / args.steps
        roof.update({"executed_flops": exec_flops, "pair_list_equivalent_tflops": flops / t_k / 1e12,
                     "covered_products_per_step": nexec, "pair_share_of_covered": npairs / max(nexec, 1)})

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        # the oracle's solution of the same source: parity of the timed
        # configuration (relative L-inf over every node of every block)
        cpu, ref = cpu_baseline(case, src_host)
        scale = max(float(np.abs(ref).max()), 1e-300)
        extra["rel_linf_vs_oracle"] = float(np.abs(g.download(ft) - ref).max() / scale)
        if out64 is not None:
            extra["fp64_plain"]["rel_linf_vs_oracle"] = float(np.abs(out64 - ref).max() / scale)
    if rank == 0 and not args.no_cpu_baseline:
        extra["reference_gpu"] = reference_gpu_baseline(g.Nb, ntgt, npairs, cells, extra.get("fp64_plain"))
    if rank == 0 and not args.no_ns:
        extra["ns_step"] = ns_bench(B, stream, local, args.steps, args.warmup)
        if not args.no_adapt:
            extra["ns_step_adaptive"] = ns_adapt_bench(B, stream, local, args.steps, args.warmup)
    if rank == 0 and not args.no_ib:
        extra["ns_step_ib"] = ib_bench(B, stream, local, args.steps, args.warmup)
    if rank == 0 and not args.no_batch:
        extra["batch"] = batch_bench(B, stream, local, args.steps, args.warmup)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "strong" if sharded else "weak",
                "vs_baseline": None, "dtype": "f32" if prec == B.FP32 else "f64", "data": "synthetic",
                "config": {"workload": wl, "cells_per_step": cells, "octants": g.n,
                           "precision": args.precision + " FFT/MAC, f64 fields and LGF table",
                           "l2": "inputs larger than L2 (fields %.0f MB, spectra cache > 126 MB)" % (g.n * g.Nb ** 3 * 8 / 1e6),
                           "parallelism": ("sharded octree (NCCL all-reduce per sweep)" if sharded else "replicas")
                           if world > 1 else "single GPU",
                           "sweeps_per_step": sweeps, "pairs_per_step": npairs,
                           "targets_per_step": ntgt, "group_mac_targets_per_step": int(stats[7]) / args.steps},
                "e2e": {"value": (1 if sharded else world) * cells / (e2e_ms * 1e-3), "unit": "cells/s",
                        "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
                "gpu_launches": int(launches),
                "mac_autotune": {"variants": "0, 1: direct sibling-group kernel (64 x 768, 32 x 512 FP32); "
                                             "2: block-Toeplitz kernel (TMA-staged coefficients); "
                                             "3: tensor-core kernel (tcgen05 TF32, 3-product split, "
                                             "M = 128 groups, N = 16, K = 8 per MMA)",
                                 "pinned": args.mac_variant,
                                 "plans": tuning},
                "launch_overhead": graph_rec,
                "roofline": roof,
                "tensor_core_mma_clocks": {"per_instruction_by_N": tc_rate,
                                           "shape": "tcgen05.mma kind::tf32, M = 128, K = 8, one issuing "
                                                    "thread per SM"},
                "clocks": ck.summary(),
                "cpu_baseline": cpu}
        line.update(extra)
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.destroy_process_group()


def ns_bench(B, stream, device, steps, warmup):
    """IF-HERK time step (NS step ms) on the vortex-ring configuration: FP32
    FFT/MAC path and FP64 plain path from the same initial velocity, each
    timed with CUDA events over `steps` steps after `warmup` steps, and the
    FP32 velocity's relative L-inf deviation from FP64 after the same steps."""
    import torch
    case = S.VortexRingNS("c4")
    dt = case.dt()
    out = {}
    res = {}
    for name, prec in (("fp32", B.FP32), ("fp64", B.FP64)):
        g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                     n_levels=case.n_levels, predicate=case.predicate, precision=prec, device=device,
                     stream=stream.cuda_stream)
        u0 = case.initial_velocity(g)
        uf = [g.field(u0[k]) for k in range(3)]
        pf = g.field()
        T = g.ns_step(uf, pf, dt, case.Re, 0.0, warmup)
        g.synchronize()
        l0 = g.launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        T = g.ns_step(uf, pf, dt, case.Re, T, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        out["ms_per_step_" + name] = e0.elapsed_time(e1) / steps
        out["launches_per_step"] = (g.launches() - l0) / steps
        res[name] = np.stack([g.download(uf[k]) for k in range(3)])
        out["octants"], out["leaves"] = int(g.n), int(np.count_nonzero(g.leaf))
        g.close()
    out.update({"workload": "vortex ring R=1, sigma=0.2R, Re=1000, dx_finest=R/32, 16^3 blocks, 3 mesh levels",
                "dt": dt, "Re": case.Re, "steps": steps, "warmup": warmup,
                "speedup_fp32_vs_fp64": out["ms_per_step_fp64"] / out["ms_per_step_fp32"],
                "rel_linf_u_fp32_vs_fp64": float(np.abs(res["fp32"] - res["fp64"]).max() / np.abs(res["fp64"]).max())})
    return out


def helm_bench(B, stream, device, steps, warmup):
    """The Fourier-in-z family of block operators on 2-D blocks, each timed
    with CUDA events over `steps` launches after `warmup`, on fields larger
    than L2 (2048 blocks of 18^2 nodes; 16 z modes, i.e. 32 real components
    per scalar field, or 48 z planes). Achieved bandwidth counts every input
    component read once and every output component written once per launch
    (the one-cell neighbours come from cache)."""
    import torch
    g = B.Solver((-32, -32, -32), (64, 64, 64), 16, 1.0, [((-16, -16, -16), (32, 32, 32))], device=device,
                 stream=stream.cuda_stream)
    hbm, kind = peaks()
    nblk, nb, nm, npl = 2048, 18, 16, 48
    sep, per = 2 * nm, nblk * nb * nb * 8
    gen = torch.Generator(device="cuda").manual_seed(7)

    def rnd(c):
        return torch.randn((nblk, c, nb, nb), dtype=torch.float64, device="cuda", generator=gen)

    cases = []
    for op, cin, cout in (("laplace", sep, sep), ("gradient", sep, 3 * sep), ("divergence", 3 * sep, sep),
                          ("curl", 3 * sep, 3 * sep), ("curl_transpose", 3 * sep, 3 * sep)):
        src, dst = rnd(cin), rnd(cout)
        cases.append((op + "_helmholtz_complex", (cin + cout) * per,
                      lambda op=op, src=src, dst=dst: g.helm2d_op(op, src, dst, nm, 0.1, 2.0, 1.0)))
    face, edge, dnl = rnd(3 * npl), rnd(3 * npl), rnd(3 * npl)
    cases.append(("nonlinear_helmholtz", 9 * npl * per, lambda: g.helm2d_nonlinear(face, edge, dnl, npl)))
    cases.append(("curl_helmholtz_planes", 6 * npl * per,
                  lambda: g.helm2d_real_op("curl_planes", face, dnl, n_planes=npl, dx_level=0.1, dx_fine=0.05)))
    torch.cuda.synchronize()
    out = {}
    for name, nbytes, fn in cases:
        for _ in range(warmup):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / steps * 1e-3
        out[name] = {"ms": t * 1e3, "bytes": nbytes, "GB/s": nbytes / t / 1e9, "frac_of_hbm": nbytes / t / 1e9 / hbm}
    out.update({"workload": "2048 blocks of 18^2 nodes, 16 z modes (complex operators) or 48 z planes",
                "hbm_gbs": hbm, "hbm_peak": kind, "steps": steps, "warmup": warmup})
    g.close()
    return out


def ns_adapt_bench(B, stream, device, steps, warmup, adapt_freq=5):
    """IF-HERK time loop with adaptation on the vortex-ring configuration
    (FP32): Solver.ns_march with the NS setup's adapt condition every
    adapt_freq iterations against the same number of plain steps; wall time
    per iteration (host tree update, field remap and plan rebuild included)."""
    import time
    case = S.VortexRingNS("c4")
    dt = case.dt()
    out = {"workload": "vortex ring (as ns_step), adapt condition of the NS setup (refinement_factor 1/8, "
                       "base_level_threshold 1e-4), adapt_frequency %d" % adapt_freq}

    def cond(sv, mc, mk, me, sm):
        return S.adapt_level_change(sv.keys, sv.levels, sv.flags, sv.base_level, mc, mk, me, sm,
                                    n_level_refinement=case.n_levels)

    for name, freq in (("plain", 0), ("adaptive", adapt_freq)):
        g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                     n_levels=case.n_levels, predicate=case.predicate, precision=B.FP32, device=device,
                     stream=stream.cuda_stream)
        u0 = case.initial_velocity(g)
        uf = [g.field(u0[k]) for k in range(3)]
        pf = g.field()
        T = g.ns_step(uf, pf, dt, case.Re, 0.0, warmup)
        g.synchronize()
        n0 = g.n
        t0 = time.perf_counter()
        T, sm, hist = g.ns_march(uf, pf, dt, case.Re, T, steps, adapt_freq=freq, adapt_condition=cond)
        g.synchronize()
        out["ms_per_iteration_" + name] = (time.perf_counter() - t0) * 1e3 / steps
        if freq:
            out["adaptations"] = len(hist)
            out["attempts"] = [int(len(h[0])) for h in hist]
            out["octants_before_after"] = [int(n0), int(g.n)]
        g.close()
    out["adapt_overhead_ms_per_adaptation"] = (
        (out["ms_per_iteration_adaptive"] - out["ms_per_iteration_plain"]) * steps / max(out.get("adaptations", 0), 1))
    return out


def ib_bench(B, stream, device, steps, warmup):
    """IF-HERK step with the immersed boundary, flow past a sphere (D = 1,
    Re = 300, uniform stream via frame velocity, dx_finest = D/40, 2009 IB
    points, wake refinement): step time (CUDA events) and IB CG iterations per
    step, FP32 and FP64, warm start = previous step's force per stage."""
    import torch
    case = S.SphereIB("c5")
    out = {"workload": "sphere D=1, Re=300, uniform stream, dx_finest=D/40, 16^3 blocks, 3 mesh levels, "
                       "2009 IB points, CG threshold 1e-3, max 40; warm start: previous force per stage "
                       "(reference), its linear extrapolation (fp32_extrapolated) and the learned 1-D conv net "
                       "correcting the previous force (fp32_learned, trained on 8 steps x 3 stages)"}
    dt = 0.35 * case.dx_base / 4 / 1.0
    res = {}
    train_steps = 8
    for name, prec, mode in (("fp32", B.FP32, 0), ("fp64", B.FP64, 0), ("fp32_extrapolated", B.FP32, 2),
                             ("fp32_learned", B.FP32, 1)):
        learned = mode == 1
        g = B.Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                     n_levels=case.n_levels, predicate=case.predicate, precision=prec, device=device,
                     stream=stream.cuda_stream)
        X = sphere_points(case.dx_base, g.depth - 1 - g.base_level, case.ibph)
        g.ib_set_points(X, case.Re)
        g.ns_options((-1.0, 0.0, 0.0))
        if mode == 1:
            # steps 2 .. train_steps + 1 record samples; the network is
            # trained before the timed steps
            g.ib_warmstart(1, train_steps=train_steps, epochs=1000, lr=2e-3, seed=7)
        elif mode == 2:
            g.ib_warmstart(2)
        u0 = case.velocity(g, U=(0.0, 0.0, 0.0))
        uf = [g.field(u0[k]) for k in range(3)]
        pf = g.field()
        T = 0.0
        # the learned leg trains at the end of its warm-up; one more untimed
        # step runs the first prediction, which pays a one-time set-up cost
        for _ in range(max(warmup, train_steps + 2) + 1 if learned else warmup):
            T = g.ns_step(uf, pf, dt, case.Re, T, 1)
        torch.cuda.synchronize()
        its = []
        ms = 0.0
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            T = g.ns_step(uf, pf, dt, case.Re, T, 1)
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            its.append(sum(g.ib_iterations()))
        out["ms_per_step_" + name] = ms / steps
        out["cg_iterations_per_step_" + name] = float(np.mean(its))
        if mode:
            if learned:
                out["warm_start_training"] = g.ib_warmstart_info()
            g.close()
            continue
        out["octants"], out["leaves"], out["ib_points"] = int(g.n), int(np.count_nonzero(g.leaf)), len(X)
        res[name] = np.stack([g.download(uf[k]) for k in range(3)])
        g.close()
    out.update({"dt": dt, "steps": steps, "warmup": warmup,
                "speedup_fp32_vs_fp64": out["ms_per_step_fp64"] / out["ms_per_step_fp32"],
                "rel_linf_u_fp32_vs_fp64": float(np.abs(res["fp32"] - res["fp64"]).max() / np.abs(res["fp64"]).max())})
    return out


def sphere_points(dx_base, ib_level, ibph):
    """IB points on the sphere R = 0.5 (ib.hpp:179-210), Fibonacci order."""
    dx = dx_base / 2 ** ib_level * ibph
    n = int(np.floor(np.pi / (dx * dx * 0.86602540378))) + 1
    lam = (1.0 + np.sqrt(5.0)) / 2.0
    x = np.arange(n) + 0.5
    phi = np.arccos(1.0 - 2 * x / n)
    theta = 2 * np.pi * x / lam
    return np.stack([0.5 * np.cos(theta) * np.sin(phi), 0.5 * np.sin(theta) * np.sin(phi), 0.5 * np.cos(phi)], 1)


def batch_bench(B, stream, device, steps, warmup):
    """Batch of 256 independent Poisson problems of 1..64 blocks of 16^3
    cells: one batched apply_lgf (every sweep stage one launch for all
    problems) in FP32, timed with CUDA events over `steps` solves after
    `warmup`, against the same problems solved one after another through
    single-problem contexts on the same stream, and against the FP64 batch."""
    import torch
    case = S.BatchPoisson("c3")
    out = {"workload": "256 unbounded Poisson problems, 1..64 blocks of 16^3 cells (log-uniform, seeded), dx = 1",
           "problems": len(case.problems), "blocks": int(sum(p["n_blocks"] for p in case.problems))}

    def timed(run):
        for _ in range(warmup):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            run()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    res = {}
    for name, prec in (("fp32", B.FP32), ("fp64", B.FP64)):
        g = B.BatchSolver(case.block_extent, case.dx_base, case.problems, precision=prec, device=device,
                          stream=stream.cuda_stream)
        src = g.zeros()
        for i in range(len(case.problems)):
            v = g.problem(i)
            src[v.offset:v.offset + v.n] = case.fields(v, i)
        fs, ft = g.field(src), g.field()
        l0 = g.launches()
        g.apply_lgf(fs, ft)
        g.synchronize()
        out["launches_per_solve"] = g.launches() - l0
        ms = timed(lambda: g.apply_lgf(fs, ft))
        cells = int(np.count_nonzero(g.leaf)) * case.block_extent ** 3
        out["cells_per_solve"] = cells
        out["ms_per_solve_" + name] = ms
        out["cells_per_s_" + name] = cells / (ms * 1e-3)
        res[name] = g.download(ft)
        g.close()
    out["rel_linf_fp32_vs_fp64"] = float(np.abs(res["fp32"] - res["fp64"]).max() / np.abs(res["fp64"]).max())
    # the same problems one context each, solved one after another (FP32)
    solvers = []
    for i, p in enumerate(case.problems):
        s = B.Solver(p["bd_base"], p["bd_extent"], case.block_extent, case.dx_base, p["blocks"], precision=B.FP32,
                     device=device, stream=stream.cuda_stream)
        solvers.append((s, s.field(case.fields(s, i)), s.field()))
    ms_seq = timed(lambda: [s.apply_lgf(a, b) for s, a, b in solvers])
    out["ms_per_solve_sequential_fp32"] = ms_seq
    out["speedup_batched_vs_sequential"] = ms_seq / out["ms_per_solve_fp32"]
    for s, _, _ in solvers:
        s.close()
    return out


def reference_gpu_baseline(Nb, targets, pairs, cells, fp64_ours):
    """The reference's own GPU path for the block convolutions (its cuFFT
    Convolution_GPU, FP64, built from the reference tree into
    oracle/_ref/ref_conv_gpu) driven through its stock per-pair calls on
    synthetic pairs: wall time per target for 64 and 160 pairs per target
    (100 targets, after one pass that caches the LGF spectra) fitted as
    a + b pairs, then evaluated for the workload's targets and pairs per
    solve. Only the convolutions: the reference's anterpolation,
    interpolation and bookkeeping would add to it, so the result is an upper
    bound of the reference's cells/s."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_conv_gpu")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_conv_gpu not built (needs the reference tree at build time)"}
    pts = []
    for q in (64, 160):
        r = subprocess.run([exe, "time", str(Nb), "100", str(q), "2"], capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            return {"unavailable": "ref_conv_gpu exited %d" % r.returncode}
        pts.append((q, json.loads(r.stdout.strip().splitlines()[-1])["ms_per_target"]))
    (q0, t0), (q1, t1) = pts
    b = (t1 - t0) / (q1 - q0)
    a = t0 - b * q0
    ms = targets * a + pairs * b
    out = {"kind": "reference fft::Convolution_GPU<3> (cuFFT D2Z/Z2D FP64, batches of 10), stock "
                   "apply_forward_add / apply_backward per pair / target, synthetic pairs",
           "ms_per_target_measured": {str(q): t for q, t in pts},
           "ms_per_target_fit": {"per_target": a, "per_pair": b},
           "ms_per_solve_convolutions_only": ms, "cells_per_s_upper_bound": cells / (ms * 1e-3)}
    if fp64_ours:
        out["fp64_ours_speedup"] = ms / fp64_ours["ms_per_step"]
    return out


def cpu_baseline(case, src=None):
    """Oracle (CPU restatement, OpenMP over targets, all host threads): one
    full apply_lgf of the workload timed after one untimed solve that fills
    the LGF spectrum cache (cells/s is defined on a warm cache). Returns the
    baseline record and the oracle's solution (for the parity check)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    d = O.Domain(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                 n_levels=case.n_levels, predicate=case.predicate)
    if src is None:
        src = case.fields(d)
    cells = case.n_cells(d)
    t0 = time.perf_counter()
    d.apply_lgf(src)
    t1 = time.perf_counter()
    out = d.apply_lgf(src)
    t2 = time.perf_counter()
    return ({"value": cells / (t2 - t1), "unit": "cells/s", "cores": os.cpu_count(), "kind": "port",
             "sample": "one full apply_lgf of the same workload (%.1f s) after one untimed solve "
                       "(%.1f s, fills the spectrum cache)" % (t2 - t1, t1 - t0)}, out)


if __name__ == "__main__":
    main()
