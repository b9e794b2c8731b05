#!/usr/bin/env python
"""Benchmark of LAMB's sector multiply C = A.B on B200.

Workload (default): 6144 waters (18,432 atoms, O block 13 / H block 5,
matrix dimension 141,312) in a 56.8 A periodic box, cutoff 8 A, A and B from
seeds 1 and 2, eps 1e-10, synthetic (seeded generator, include/lamb_gen.h).
One step = one full multiply (symbolic phase + numeric phase + result filter)
on inputs resident in HBM.  The inputs (1.9 GB each) exceed the 126 MB L2, so
no flush is needed between steps.

Printed JSON line (rank 0): metric GFLOP/s (FP64-equivalent flops counted
from the block pattern: sum of 2*b_i*b_k*b_j over executed products), the
dominant kernel's roofline against the FP64 tensor-pipe peak measured live on
the same GPU, the whole multiply's fraction of the measured HBM copy
bandwidth, the end-to-end number through the C ABI with host buffers, and the
CPU baseline (the oracle restatement on a bounded row sample).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun) every rank runs an independent replica (nothing in the
multiply shards at one rank); value is the sum over ranks of flops divided by
the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "block-SpGEMM GFLOP/s (FP64-equivalent), LAMB sector multiply"
# Every CPU timing (the cpu_baseline leg and the reference arm) runs the
# oracle on every CPU_ROW_STRIDE-th C block row of the same workload.
CPU_ROW_STRIDE = 6


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="water6144_cut8",
                   choices=["water6144_cut8", "water1536_cut7", "water768_cut7", "water192_cut6", "batch64", "mcweeny384",
                            "adjoint96"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--no-positions", action="store_true", help="order work from the block pattern only")
    p.add_argument("--mixed-steps", type=int, default=3, help="timed steps of the int8-slice path (0 skips it)")
    p.add_argument("--no-full-check", action="store_true", help="skip the whole-product check against the oracle")
    p.add_argument("--batch-steps", type=int, default=3, help="timed full runs of the 64-box batch (0 skips it)")
    return p.parse_args()


def workload(name):
    from lamb_b200 import gen
    return {"water6144_cut8": gen.WATER_6144, "water1536_cut7": gen.WATER_1536, "water768_cut7": gen.WATER_768,
            "water192_cut6": gen.WATER_192}[name]


def workload_config(wl, g) -> dict:
    """The workload (identical in both arms)."""
    return {"workload": wl.name, "n_mol": wl.n_mol, "n_atoms": int(g.n_atoms), "box": wl.box, "cutoff": wl.cutoff,
            "eps": wl.eps, "seeds": {"geometry": wl.geom_seed, "A": wl.seed_a, "B": wl.seed_b},
            "blocks": {"O": wl.blk_o, "H": wl.blk_h}}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def algorithmic_bytes(a, b, c) -> int:
    """Compulsory bytes of one multiply: FP64 elements of A, B, C plus the
    index (row_p 8 B per row, col_i 2 B and extents 16 B per block)."""
    tot = 0
    for m in (a, b, c):
        for s in m.sectors:
            used = int((s.extents[:, 1] - s.extents[:, 0] + 1).sum()) if s.n_blks else 0
            tot += 8 * used + 8 * (s.n_rows + 1) + 18 * s.n_blks
    return tot


class Clocks:
    """SM clock and throttle-reason sampler (NVML, in-process thread, 200 ms).

    Started before the warm-up so that NVML is initialised before the timed
    region; mark() / stop() bracket the timed region and only samples taken
    inside it are reported."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, device):
        import threading
        self.rows, self.t0, self.t1 = [], None, None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self._nv, self._h = pynvml, h
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self._nv = None
            return
        self._th = threading.Thread(target=self._run, daemon=True)
        self._th.start()

    def _run(self):
        nv, h = self._nv, self._h
        while not self._stop.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.rows.append((time.perf_counter(), mhz, rs))
            except Exception:
                pass
            self._stop.wait(0.2)

    def mark(self):
        self.t0 = time.perf_counter()

    def stop(self):
        self.t1 = time.perf_counter()
        if self._nv is None:
            return None
        self._stop.set()
        self._th.join(timeout=2)
        rows = [r for r in self.rows if self.t0 is not None and self.t0 <= r[0] <= self.t1]
        if not rows:  # timed region shorter than one period: nearest sample after it
            rows = [r for r in self.rows if r[0] >= (self.t0 or 0)][:1]
        if not rows:
            return None
        reasons = sorted({k for _, _, rs in rows for k, bit in self.REASONS.items() if rs & bit})
        return {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(rows), "source": "NVML"}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def committed_traffic(kernel, wl):
    """DRAM bytes per multiply of `kernel` at workload `wl`, from the
    committed summary profiles/<kernel>_traffic.json (a small-case ncu capture
    and its scaling to each workload); None when absent."""
    path = os.path.join(REPO, "profiles", f"{kernel}_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)["per_multiply_bytes"].get(wl)
    except Exception:
        return None


def cpu_sample(a, b, eps, threads, reps=1):
    """Times the oracle on every CPU_ROW_STRIDE-th C row (`reps` runs)."""
    import oracle
    fl, dt, c = 0.0, 0.0, None
    for _ in range(reps):
        t = time.perf_counter()
        c, st = oracle.multiply(a, b, eps, threads=threads, row_stride=CPU_ROW_STRIDE)
        dt += time.perf_counter() - t
        fl += st["flops"]
    return c, fl, dt


def rows_of(m, stride):
    out = {}
    for s in m.sectors:
        rows = s.block_rows()
        for bi in range(s.n_blks):
            r = int(rows[bi])
            if r % stride == 0:
                f, l = int(s.extents[bi, 0]), int(s.extents[bi, 1])
                out[(s.subset_row, s.subset_col, r, int(s.col_i[bi]))] = s.data[f - 1:l]
    return out


def sampled_error(c_gpu, c_ref, stride):
    import numpy as np
    g, r = rows_of(c_gpu, stride), rows_of(c_ref, stride)
    if set(g) != set(r):
        return float("inf")
    num = sum(float(np.sum((g[k] - r[k]) ** 2)) for k in r)
    den = sum(float(np.sum(r[k] ** 2)) for k in r)
    return float(np.sqrt(num / den)) if den > 0 else 0.0


def pin_matrix(m):
    """Copies a host matrix into page-locked buffers (the e2e inputs)."""
    import numpy as np
    import torch
    from lamb_b200.matrix import LambMatrix, Sector
    keep = []

    def pin(x):
        t = torch.empty(x.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(x.dtype).reshape(x.shape)
        v[...] = x
        keep.append(t)
        return v
    secs = [Sector(s.subset_row, s.subset_col, pin(s.row_blk_sizes), pin(s.col_blk_sizes), pin(s.row_p),
                   pin(s.col_i), pin(s.extents), pin(s.data)) for s in m.sectors]
    out = LambMatrix(secs, m.name)
    out._keep = keep
    return out


def matrix_bytes(m):
    return sum(x.nbytes for s in m.sectors for x in (s.row_blk_sizes, s.col_blk_sizes, s.row_p, s.col_i,
                                                      s.extents, s.data))


def run_reference(args):
    """CPU arm: the oracle (the reference's multiply is a stub and its Fortran
    does not build here), all host threads, every CPU_ROW_STRIDE-th C block
    row of the same workload per step.  Inputs come from the same generator
    (liblamb_gen.so) outside the timed region."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = workload(args.workload)
    g, a, b = wl.build()
    threads = os.cpu_count() or 1
    import oracle
    for _ in range(args.warmup):
        oracle.multiply(a, b, wl.eps, threads=threads, row_stride=CPU_ROW_STRIDE)
    fl, tt = 0.0, 0.0
    for _ in range(args.steps):
        _, f, dt = cpu_sample(a, b, wl.eps, threads)
        tt += dt
        fl += f
    v = fl / tt / 1e9
    sample = f"every {CPU_ROW_STRIDE}th C block row of {wl.name} per step ({fl / args.steps / 1e9:.1f} GFLOP)"
    cpu = {"value": v, "unit": "GFLOP/s", "cores": threads, "kind": "port", "sample": sample, "cpu": cpu_model()}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(wl, g),
            "cpu_baseline": cpu,
            "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "oracle restatement in C + OpenMP (the reference's sector_multiply is a stub and needs "
                    "gfortran+MPI); inputs from liblamb_gen.so, built outside the timed region"}
    print(json.dumps(line), flush=True)


def run_mixed_leg(ctx, lib, local, da, db, dc, wl, args, flops, ms_fp64):
    """The mixed multiply (int8 digit products on the tensor cores, FP64
    recombination) on the FP64 leg's inputs: time per phase, error against
    the FP64 result, and the tensor-core roofline of the tile kernel."""
    import ctypes
    from lamb_b200 import gpu
    dcm = ctx.create_like(da)
    ctx.multiply(da, db, dcm, wl.eps, gpu.MIXED)  # warm-up: pool growth
    mst = [ctx.multiply(da, db, dcm, wl.eps, gpu.MIXED) for _ in range(args.mixed_steps)]
    rel = ctx.diff_frobenius(dcm, dc) / ctx.frobenius(dc)
    dcm.destroy()
    mean = lambda k: statistics.mean(x[k] for x in mst)
    ms_m, ms_num = mean("ms_total"), mean("ms_numeric")
    s_m = int(mst[-1]["mixed_slices"])
    out = {"value": flops / (ms_m * 1e-3) / 1e9, "unit": "GFLOP/s", "ms_per_step": ms_m, "steps": args.mixed_steps,
           "phases_ms": {"exponents_and_pattern": mean("ms_symbolic") - mean("ms_prepare"),
                         "panels_tiles_inner_lists": mean("ms_prepare"), "numeric": ms_num,
                         "result_filter": mean("ms_filter")},
           "ms_symbolic": mean("ms_symbolic"), "ms_numeric": ms_num, "slices": s_m,
           "rel_frobenius_err_vs_fp64": rel, "ms_ratio_vs_fp64": ms_m / ms_fp64}
    t_ops = mst[-1]["tensor_ops"]
    if t_ops > 0:
        f = lib.lamb_probe_int8_tcgen05_tops
        f.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
        peak = ctypes.c_double()
        ctx.check(f(local, 0, 5, ctypes.byref(peak)))
        achieved = t_ops / (ms_num * 1e-3) / 1e12
        out["path"] = ("tcgen05.mma kind::i8 (M=128, K=32, N=64..256: one MMA per A digit plane and run of up to "
                       "four B digit planes, nine per 32-row stage) on 128x64 spatial cluster tiles, six base-254 "
                       "digits per operand, 21 digit-pair products into six int32 TMEM level accumulators, exact "
                       "int64 level recombination, FP64 scaling")
        out["roofline"] = {"bound": "tensor", "kernel": "k_tc_tiles", "achieved": achieved, "peak": peak.value,
                           "unit": "TOP/s (int8)", "frac": achieved / peak.value,
                           "peak_source": "tcgen05 kind::i8 probe issuing the tile kernel's own nine-MMA stage "
                                          "(lamb_probe_int8_tcgen05_tops n=0) on this GPU in this run",
                           "tensor_ops_per_multiply": t_ops,
                           "traffic": committed_traffic("k_tc_tiles", wl.name),
                           "traffic_scope": "DRAM bytes of the multiply's tile-kernel launch, scaled by tensor ops "
                                            "from the committed small-case capture; null when none",
                           "useful_fraction": flops * s_m * (s_m + 1) / 2 / t_ops,
                           "note": "executed ops include the zero padding of the cluster tiles; useful_fraction = "
                                   "FP64-equivalent flops x 21 digit pairs / executed ops"}
    else:
        out["path"] = "int8 digit slices through mma.m16n8k32.s8 (the tile limits of the tensor-core kernel were exceeded)"
    return out


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from lamb_b200 import build, gpu
    build.build_all()
    from lamb_b200.gpu import Context
    import ctypes
    wl = workload(args.workload)
    g, a, b = wl.build()
    ctx = Context(local)
    lib = gpu.lib()
    lib.lamb_probe_fp64_tflops.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
    peak = ctypes.c_double()
    ctx.check(lib.lamb_probe_fp64_tflops(local, 5, ctypes.byref(peak)))
    fp64_peak = peak.value
    da, db = ctx.upload(a), ctx.upload(b)
    if not args.no_positions:
        da.set_positions(g.sector_positions(), g.box)
    dc = ctx.create_like(da)
    ext = torch.cuda.ExternalStream(ctx.stream_ptr(), device=torch.device("cuda", local))
    clk = Clocks(local)
    for _ in range(args.warmup):
        st = ctx.multiply(da, db, dc, wl.eps)

    def barrier():
        if world > 1:
            dist.barrier()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk.mark()
    with torch.cuda.stream(ext):
        e0.record()
    stats = []
    for _ in range(args.steps):
        stats.append(ctx.multiply(da, db, dc, wl.eps))
    with torch.cuda.stream(ext):
        e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier()
    ms = e0.elapsed_time(e1)
    ms_t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    flops = stats[-1]["flops"]
    value = flops * args.steps * world / (ms_max * 1e-3) / 1e9
    ms_num = statistics.mean(s["ms_numeric"] for s in stats)
    ms_kern = statistics.mean(s["ms_kernel"] for s in stats)  # the k_stacked launches alone
    ms_tot = statistics.mean(s["ms_total"] for s in stats)
    c_host = dc.download()
    alg_bytes = algorithmic_bytes(a, b, c_host)
    peaks, peak_kind = measured_peaks()
    achieved_tf = flops / (ms_kern * 1e-3) / 1e12
    # the mixed path on the same inputs, its error taken against the FP64 result
    mixed = None
    if args.mixed_steps > 0:
        mixed = run_mixed_leg(ctx, lib, local, da, db, dc, wl, args, flops, ms_tot)
    # cfg2: the 64-box batch, full multiply per step (rank 0 of a single-GPU run)
    batch = None
    if world == 1 and args.batch_steps > 0:
        batch = batch_leg(ctx, args, args.batch_steps, 2)
    # e2e through the C ABI with page-locked host buffers
    pa, pb = pin_matrix(a), pin_matrix(b)
    c_out = dc.download(pinned=True)
    pos = g.sector_positions()
    h2d = matrix_bytes(pa) + matrix_bytes(pb)
    d2h = matrix_bytes(c_out)
    barrier()
    t_e2e = []
    # one untimed pass first: the device memory pool grows to the working set
    for it in range(1 + max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        xa, xb = ctx.upload(pa), ctx.upload(pb)
        if not args.no_positions:
            xa.set_positions(pos, g.box)
        xc = ctx.create_like(xa)
        # async: the download below copies C row chunk by row chunk as the numeric phase completes them
        st_e = ctx.multiply(xa, xb, xc, wl.eps, gpu.ASYNC)
        c_out = xc.download(out=c_out)
        xc.destroy(); xb.destroy(); xa.destroy()
        if it > 0:
            t_e2e.append(time.perf_counter() - t)
    e2e_t = torch.tensor([statistics.mean(t_e2e)], device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = flops * world / float(e2e_t.item()) / 1e9
    cpu = None
    err = None
    full = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        c_ref, fl_ref, dt = cpu_sample(a, b, wl.eps, threads, reps=2)
        cpu = {"value": fl_ref / dt / 1e9, "unit": "GFLOP/s", "cores": threads, "kind": "port",
               "sample": f"every {CPU_ROW_STRIDE}th C block row of {wl.name}, twice ({fl_ref / 1e9:.1f} GFLOP, "
                         f"{dt:.1f} s)", "cpu": cpu_model()}
        err = sampled_error(c_host, c_ref, CPU_ROW_STRIDE)
        del c_ref
    if rank == 0 and world == 1 and not args.no_full_check:
        # every row of the FP64 result against the oracle (pattern under the
        # filter rule, relative Frobenius error), outside the timed regions
        import oracle
        t = time.perf_counter()
        full = oracle.check_product(a, b, wl.eps, c_host)
        full["seconds"] = time.perf_counter() - t
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded water boxes)",
            "config": workload_config(wl, g),
            "setup": {"path": "plain FP64 (DMMA)",
                      "row_order": "pattern (Cuthill-McKee)" if args.no_positions else "Morton (atom coordinates)",
                      "l2": "inputs 2x1.9 GB exceed L2; no flush", "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "tensor", "kernel": "k_stacked", "achieved": achieved_tf,
                         "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved_tf / fp64_peak,
                         "peak_source": "FP64 DMMA probe measured on this GPU in this run",
                         "traffic": committed_traffic("k_stacked", wl.name),
                         "traffic_scope": "DRAM bytes of one multiply's k_stacked launches (all row chunks), "
                                          "scaled from the committed small-case capture; null when none",
                         "flops_per_multiply": flops, "ms_per_multiply": ms_kern,
                         "timing": "CUDA events around each row chunk's k_stacked launch, summed per multiply "
                                   "(the chunks' stack fills excluded); numeric phase with fills: "
                                   f"{ms_num:.2f} ms"},
            "roofline_hbm": {"bound": "hbm", "achieved": alg_bytes / (ms_tot * 1e-3) / 1e9,
                             "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                             "frac": alg_bytes / (ms_tot * 1e-3) / 1e9 / peaks.get("hbm_gbs"),
                             "note": f"algorithmic bytes of the whole multiply over its device time; {peak_kind}",
                             "bytes": alg_bytes},
            "e2e": {"value": e2e_value, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": statistics.mean(t_e2e) * 1e3},
            "cpu_baseline": cpu,
            "max_rel_err_vs_oracle": err,
            "full_check_vs_oracle": full,
            "mixed": mixed,
            "batch": batch,
            "stats": {k: stats[-1][k] for k in ("n_products", "n_c_blocks", "ms_symbolic", "ms_numeric", "ms_total")},
            # timed region per step minus the multiply's own device time: host-side
            # stalls between and inside the multiplies (the GPU idles meanwhile)
            "host_gap_ms_per_step": ms_max / args.steps - ms_tot,
            "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    for m in (dc, db, da):
        m.destroy()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def batch_leg(ctx, args, steps, warmup):
    """cfg2: 64 uneven independent water boxes.  Every timed step is a full
    run of the batch: symbolic phase of every instance, one graph-replayed
    persistent numeric launch over the global queue, result filter of every
    instance (lamb_gpu_batch_run with LAMB_GPU_BATCH_FULL)."""
    import torch
    from lamb_b200.gen import batch_instances
    wls = batch_instances()
    devs = []
    t0 = time.perf_counter()
    for wl in wls:
        g, a, b = wl.build()
        da, db = ctx.upload(a), ctx.upload(b)
        if not args.no_positions:
            da.set_positions(g.sector_positions(), g.box)
        devs.append((da, db, ctx.create_like(da)))
        del a, b
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    batch = ctx.batch([d[0] for d in devs], [d[1] for d in devs], [d[2] for d in devs], eps=1e-10)
    t_create = time.perf_counter() - t0
    for _ in range(warmup):
        batch.run_full()
    torch.cuda.synchronize()
    clk = Clocks(ctx.device)
    clk.mark()
    sts = [batch.run_full() for _ in range(steps)]
    clocks = clk.stop()
    mean = lambda k: statistics.mean(x[k] for x in sts)
    st = sts[-1]
    out = {"metric": METRIC + " (batched, full multiply per step)", "value": st["flops"] / (mean("ms_total") * 1e-3) / 1e9,
           "unit": "GFLOP/s", "steps": steps, "warmup": warmup, "ms_per_step": mean("ms_total"),
           "phases_ms": {"symbolic": mean("ms_symbolic"), "numeric_graph_replay": mean("ms_numeric"),
                         "result_filter": mean("ms_filter")},
           "numeric_only_gflops": st["flops"] / (mean("ms_numeric") * 1e-3) / 1e9,
           "config": {"workload": "batch64: 64 boxes of 96-1536 waters (log-uniform, seed 3), cutoffs U[5,9] A, "
                                  "O 23 / H 5 in half, O 13 / H 5 in the rest", "eps": 1e-10,
                      "graph": "numeric launch captured once, replayed per step", "tuned": batch.config()},
           "stats": {"flops": st["flops"], "n_products": st["n_products"], "n_c_blocks": st["n_c_blocks"],
                     "n_c_blocks_dropped": st["n_c_blocks_dropped"], "build_s": t_build, "create_s": t_create},
           "gpu_launches_per_step": int(st["kernel_launches"]), "clocks": clocks}
    batch.destroy()
    for m in devs:
        for x in m:
            x.destroy()
    return out


def run_batch(args):
    """64 uneven independent water boxes, the standalone line."""
    from lamb_b200 import build
    build.build_all()
    from lamb_b200.gpu import Context
    ctx = Context(0)
    out = batch_leg(ctx, args, args.steps, args.warmup)
    line = {"metric": out.pop("metric"), "value": out.pop("value"), "unit": "GFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": out.pop("ms_per_step"),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded water boxes)", "config": out.pop("config"),
            "gpu_launches": out["gpu_launches_per_step"] * args.steps, **out}
    print(json.dumps(line), flush=True)
    ctx.close()


def run_mcweeny(args):
    """McWeeny purification of a gapped water Hamiltonian: 30 steps of
    P <- 3P^2 - 2P^3, the first 25 with int8-slice products and the last 5 in
    FP64, against the same 30 steps all in FP64.  384 waters (1,152 atoms),
    cutoff 6 A, eps 1e-10: P fills in to a dense block matrix after the
    first steps, which bounds the system size on one GPU."""
    import torch
    from lamb_b200 import build
    build.build_all()
    from lamb_b200.gen import WaterGeometry, gapped_hamiltonian
    from lamb_b200.gpu import Context
    g = WaterGeometry(384, None, 6.0, seed=1)
    h = gapped_hamiltonian(g, 1)
    ctx = Context(0)
    dh = ctx.upload(h)
    dh.set_positions(g.sector_positions(), g.box)
    p64, pmx = ctx.create_like(dh), ctx.create_like(dh)
    clk = Clocks(0)
    ctx.purify(dh, p64, mu=0.0, steps=3, fp64_tail=3, eps=1e-10)  # warm-up: pool growth, row order
    torch.cuda.synchronize()
    clk.mark()
    r64 = ctx.purify(dh, p64, mu=0.0, steps=30, fp64_tail=30, eps=1e-10)
    rmx = ctx.purify(dh, pmx, mu=0.0, steps=30, fp64_tail=5, eps=1e-10)
    clocks = clk.stop()
    rel = ctx.diff_frobenius(pmx, p64) / ctx.frobenius(p64)
    e64, emx = ctx.trace_product(p64, dh), ctx.trace_product(pmx, dh)
    line = {"metric": "McWeeny purification time, 30 steps (2 multiplies each)", "value": rmx["ms_total"],
            "unit": "ms", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": rmx["ms_total"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "int8 slices + f64",
            "data": "synthetic (seeded gapped water Hamiltonian)",
            "config": {"workload": "mcweeny384: 384 waters (1,152 atoms), cutoff 6 A, gap 0.2 at mu = 0, "
                                   "eps 1e-10, 25 int8-slice steps + 5 FP64 steps"},
            "fp64_ms": r64["ms_total"], "mixed_over_fp64_time": rmx["ms_total"] / r64["ms_total"],
            "rel_frobenius_err_P_vs_fp64": rel, "band_energy": emx, "band_energy_fp64": e64,
            "band_energy_rel_err": abs(emx - e64) / abs(e64), "trace": rmx["trace"], "trace_fp64": r64["trace"],
            "idempotency": rmx["idempotency"], "idempotency_fp64": r64["idempotency"],
            "steps_mixed": rmx["steps_mixed"], "clocks": clocks}
    print(json.dumps(line), flush=True)
    for m in (pmx, p64, dh):
        m.destroy()
    ctx.close()


def run_adjoint(args):
    """dL/dH of L = Tr(P_K H) after K = 20 McWeeny steps in FP64, from the
    masked-adjoint kernels with a checkpoint every 4th P_k (recomputation in
    between), against the dense FP64 torch gradient and central differences
    (step 1e-6) on 200 random entries of H.  96 waters (288 atoms), O 13 /
    H 5, cutoff 7 A, seed 4: with no filter P_K is dense, which bounds the
    size the recomputation can hold and the 400 finite-difference solves."""
    import numpy as np
    import torch
    from lamb_b200 import build
    build.build_all()
    from lamb_b200 import autograd as AG
    from lamb_b200.gen import WaterGeometry, gapped_hamiltonian
    from lamb_b200.gpu import Context
    g = WaterGeometry(96, None, 7.0, seed=4)
    h = gapped_hamiltonian(g, 4, coupling=0.05)
    ctx = Context(0)
    K, cp = 20, 4
    lam = AG.gershgorin_lambda(h)
    eng = AG.PurifyEngine(ctx, K, lam, checkpoint=cp)
    flat = lambda: torch.from_numpy(np.concatenate([s.data for s in h.sectors]))
    hv = flat().requires_grad_(True)
    AG.PurifyTrace.apply(flat().requires_grad_(True), h, eng).backward()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = AG.PurifyTrace.apply(hv, h, eng)
    loss.backward()
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    grad = hv.grad.numpy()
    # dense FP64 reference on the GPU (cuBLAS)
    ri, ci = AG.dense_index(h)
    n = int(h.to_dense().shape[0])
    hv2 = flat().cuda().requires_grad_(True)
    t0 = time.perf_counter()
    ref = AG.dense_purify_loss(hv2, ri, ci, n, lam, K)
    ref.backward()
    torch.cuda.synchronize()
    t_dense = time.perf_counter() - t0
    gref = hv2.grad.cpu().numpy()
    grad_err = float(np.linalg.norm(grad - gref) / np.linalg.norm(gref))
    # central differences on 200 random entries; the FD error floor is about
    # eps_mach |L| / step, so entries whose derivative is far above it are
    # held to 1e-6 relative and the rest to the floor
    step = 1e-6
    roundoff = np.finfo(np.float64).eps * abs(loss.item()) / step   # FD error floor from rounding L
    floor = 8 * roundoff
    rng = np.random.default_rng(4)
    picks = rng.choice(hv.shape[0], 200, replace=False)
    # 100 more among the largest derivatives, where a relative check means most
    big_pool = np.argsort(-np.abs(grad))[:2000]
    picks = np.concatenate([picks, rng.choice(big_pool, 100, replace=False)])
    worst_rel, n_rel, n_ok, worst_abs = 0.0, 0, 0, 0.0
    t0 = time.perf_counter()
    for i in picks:
        e = torch.zeros_like(hv)
        e[i] = step
        with torch.no_grad():
            lp = AG.PurifyTrace.apply(flat() + e, h, eng).item()
            lm = AG.PurifyTrace.apply(flat() - e, h, eng).item()
        fd = (lp - lm) / (2 * step)
        worst_abs = max(worst_abs, abs(fd - grad[i]))
        if abs(grad[i]) >= 1e6 * roundoff:  # relative 1e-6 is resolvable
            n_rel += 1
            r = abs(fd - grad[i]) / abs(grad[i])
            worst_rel = max(worst_rel, r)
            n_ok += r <= 1e-6
        else:
            n_ok += abs(fd - grad[i]) <= floor + 1e-6 * abs(grad[i])
    t_fd = time.perf_counter() - t0
    line = {"metric": "gradient of Tr(P_K H) through K=20 McWeeny steps (masked adjoint, checkpoint every 4th)",
            "value": t_grad * 1e3, "unit": "ms (forward + backward)", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": t_grad * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded gapped water Hamiltonian, coupling 0.05)",
            "config": {"workload": "adjoint96: 96 waters (288 atoms, dim 2,208), O 13 / H 5, cutoff 7 A, seed 4",
                       "K": K, "checkpoint_every": cp},
            "loss": loss.item(), "loss_dense": ref.item(),
            "grad_rel_err_vs_dense_fp64": grad_err, "dense_torch_ms": t_dense * 1e3,
            "fd": {"entries": int(len(picks)), "random": 200, "largest": 100, "step": step, "passed": int(n_ok),
                   "relative_checked": int(n_rel), "worst_rel_err": worst_rel, "worst_abs_err": worst_abs,
                   "roundoff_floor": roundoff, "seconds": t_fd,
                   "criterion": "|fd-g| <= 1e-6 |g| where |g| >= 1e6 * eps |L| / step, else <= 8 eps |L| / step + 1e-6 |g|"}}
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    args = parse()
    if args.workload == "adjoint96":
        run_adjoint(args)
    elif args.workload == "mcweeny384":
        run_mcweeny(args)
    elif args.workload == "batch64":
        run_batch(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
