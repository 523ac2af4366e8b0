"""Benchmark of the block-sparse contraction path (btod_contract2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ltg|reference]
                    [--workload ladder-large|ladder-split|ladder-small|ring] [--mode plain|...]

One step = one btod_contract2::perform over the whole synthetic workload.
value   = algorithmic FP64 flops / device time, inputs resident in HBM
          (effective FP64 TFLOP/s; flops = sum over non-zero C blocks and
          coalesced pairs of 2*|C block|*K, the reference's get_cost x 2000);
e2e     = same flops / time of the C-ABI call sequence with host buffers:
          H2D of both operand arenas, the contraction, D2H of the result.
N > 1 runs independent replicas (the path does not shard); value sums ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "ladder-large": "LADDER_LARGE",
    "ladder-split": "LADDER_SPLIT",
    "ladder-small": "LADDER_SMALL",
    "ladder-ccd": "LADDER_CCD",
    "ladder-prof": "LADDER_PROF",
    "ring": "RING_D2H",
    "ring-small": "RING_D2H_SMALL",
    "dense": "DENSE_6144",
}
# HBM-bound operations (btod_copy / btod_add / btod_dotprod) on the CCD
# iteration's tensors, o=30 v=300 (blocks 15 / 50,50,50 per spin).
TRANSFER_WORKLOADS = ("copy-vvvv", "add-x4", "dot-vvvv")
# One CCD amplitude iteration (copy, ladder, ring, antisymmetrising add,
# denominator, energy) replayed as one CUDA graph, o=30 v=300.
GRAPH_WORKLOADS = ("ccd-iter",)
MODES = {"plain": 0, "ozaki-bf16": 1, "ozaki-fp8": 2, "ozaki-int8": 3, "ozaki-crt": 4}
FP64_NOMINAL = 40.0


def max_over_ranks(values, device, world):
    """Per-rank times -> their maximum over all ranks (every rank gets it).
    Replicas run independently; the job's time is that of the slowest rank."""
    if world <= 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def replica_rate(work_per_rank, ms, world):
    """Whole-job rate of `world` replicas that each did `work_per_rank` in at
    most `ms` milliseconds (units of work per second)."""
    return world * work_per_rank / (ms * 1e-3)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ltg", choices=["ltg", "reference"])
    # Headline: the split-precision ladder o=40 v=240 (blocks 64/56 per spin)
    # at <= 1e-12 (modular INT8 mode, 13 moduli), with the plain FP64 DMMA path
    # timed on the same workload.
    p.add_argument("--workload", default="ladder-split",
                   choices=sorted(WORKLOADS) + list(TRANSFER_WORKLOADS) + list(GRAPH_WORKLOADS))
    p.add_argument("--mode", default="ozaki-crt", choices=sorted(MODES))
    p.add_argument("--nslices", type=int, default=None,
                   help="slices (moduli for ozaki-crt); default 7, 8 for FP8, 13 for the modular mode")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--no-plain", action="store_true", help="skip the plain-DMMA companion timing")
    p.add_argument("--no-slices", action="store_true",
                   help="skip the companion timing of the BF16 x7 and FP8 x8 slice modes")
    p.add_argument("--fused-split", type=int, default=0, choices=[0, 1, 2],
                   help="modular mode: one-read split of row families in kernel shape 1 or 2 (0: exponent and "
                        "residue passes)")
    p.add_argument("--symmetrize", default="", choices=["", "asymm01", "asymm-p0123"],
                   help="also time the result antisymmetrized over indexes (0,1) or the pair exchange "
                        "(0 1)(2 3), fused into the contraction's kernels against the contraction followed by "
                        "the symmetrizer pass (slice modes at their default slice counts)")
    p.add_argument("--crt-stage", type=int, default=0, choices=[0, 2, 3, 4, 6],
                   help="modular mode: k blocks per products pipeline stage (0: default)")
    p.add_argument("--tile", type=int, default=-1, help="force one tile shape (debug)")
    p.add_argument("--split-k", type=int, default=0, choices=[0, 1, 2, 3, 4],
                   help="plain mode: k chunks per tile (0 automatic, 1 never)")
    p.add_argument("--crt-rows", type=int, default=0, choices=[0, 128, 256],
                   help="modular mode: rows of the products kernel's work items (0: default, 256)")
    a = p.parse_args()
    if a.mode == "plain":
        a.nslices = 0
    elif a.nslices is None:
        a.nslices = {"ozaki-fp8": 8, "ozaki-crt": 13}.get(a.mode, 7)
    return a


def workload(name):
    from libtensor_b200 import spec as S
    cfg = getattr(S, WORKLOADS[name])
    a = cfg.t_spec()
    b = cfg.v_spec() if hasattr(cfg, "v_spec") else cfg.w_spec()
    return cfg, a, b


def contraction_of(cfg):
    from libtensor_b200.core import contraction2
    c = cfg.contraction
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    return contr


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- reference

def build_reference(a_spec, b_spec, cfg):
    """The workload on the reference compiled from its sources: operands
    filled with the seeded inputs inside the reference library (the same bits
    the product generates on the device), the contraction and its result
    tensor.  Nothing of the product library is loaded."""
    from oracle import refapi as R
    ra, rb = R.RefBT(a_spec), R.RefBT(b_spec)
    ra.fill_seeded(11, cfg.t_scale)
    rb.fill_seeded(23, cfg.v_scale)
    c = cfg.contraction
    op = R.RefContract2(c["n"], c["m"], c["k"], c["permc"], c["pairs"], ra, rb, 1.0, 1.0, cfg.kc)
    rc = op.make_result()
    return ra, rb, op, rc


def time_reference(op, rc, steps, warmup, budget_s=30.0):
    """Times the reference's perform() (wall clock); returns (seconds/step, runs)."""
    from oracle import refapi as R
    R.set_threads(os.cpu_count() or 1)
    for _ in range(warmup):
        op.perform(rc)
    ts = []
    t_start = time.perf_counter()
    for _ in range(steps):
        t0 = time.perf_counter()
        op.perform(rc)
        ts.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    return float(np.median(ts)), len(ts)


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import refapi as R
    cfg, a_spec, b_spec = workload(args.workload)
    metric, unit = metric_name(), "TFLOP/s"
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libltref.so was not built"}))
        return
    R.set_threads(os.cpu_count() or 1)
    ra, rb, op, rc = build_reference(a_spec, b_spec, cfg)
    flops = 2.0 * op.cost()[0]       # the reference's task cost of the schedule, before its /1000
    sec, runs = time_reference(op, rc, args.steps, min(args.warmup, 1), budget_s=120.0)
    v = flops / sec / 1e12
    out = {"metric": metric, "value": v, "unit": unit, "impl": "reference", "n_gpus": args.gpus,
           "steps": runs, "warmup": min(args.warmup, 1), "ms_per_step": sec * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, symmetrised)",
           "config": config_of(args, cfg, flops),
           "cpu_baseline": {"value": v, "unit": unit, "cores": os.cpu_count(), "kind": "reference",
                            "sample": f"full workload, {runs} perform() calls, median"},
           "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def metric_name():
    return "btod_contract2 eff. FP64 TFLOP/s: split-prec vs plain DMMA @ rel err<=1e-12"


def config_of(args, cfg, flops):
    return {"workload": f"{cfg.name} ({args.workload})", "mode": args.mode, "nslices": args.nslices,
            "o": cfg.o, "v": cfg.v, "algorithmic_flops": flops,
            "l2": "inputs larger than L2 (no flush)" if args.workload in ("ladder-large", "ladder-split", "ring", "ladder-ccd", "dense") else "small inputs, L2-resident"}


# ---------------------------------------------------------------- ltg arm

def measure_fp64_peak(torch, dev):
    """cuBLAS DGEMM 8192^3 (best of 3): the FP64 denominator of the roofline."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def ltg_arm(args):
    import torch
    import torch.distributed as dist
    from libtensor_b200.core import Context, block_tensor, btod_contract2

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)

    cfg, a_spec, b_spec = workload(args.workload)
    mode = MODES[args.mode]
    ctx = Context(local)
    A, B = block_tensor(ctx, a_spec), block_tensor(ctx, b_spec)
    A.fill_seeded(11, cfg.t_scale)
    B.fill_seeded(23, cfg.v_scale)
    op = btod_contract2(contraction_of(cfg), A, B, kc=cfg.kc)
    C = op.make_result()
    flops = op.flops()
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ctx.synchronize()

    tiles = None
    if args.crt_rows:
        op.set_crt_rows(args.crt_rows)
    if args.split_k:
        op.set_split_k(args.split_k)
    if args.fused_split:
        op.set_fused_split(args.fused_split)
    if args.crt_stage:
        op.set_crt_stage(args.crt_stage)
    if args.tile >= 0:
        op.set_tile(args.tile)
    elif not args.no_autotune:
        # tile shapes of the plain FP64 kernel (also the companion timing below)
        tiles = op.autotune(C, mode=0, nslices=0, reps=1)
    clocks = ClockSampler(local)
    clocks.start()            # nvidia-smi needs a moment to start: begin before the warm-up
    for _ in range(max(3, args.warmup)):
        op.perform(C, mode=mode, nslices=args.nslices)
    barrier()

    # ---- device-resident timing
    n0 = ctx.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ctx.set_timing(True)          # event pair around every kernel launch of the library
    e0.record(stream)
    for _ in range(args.steps):
        op.perform(C, mode=mode, nslices=args.nslices)
    e1.record(stream)
    barrier()
    ktimes = ctx.kernel_times()
    ctx.set_timing(False)
    launches = ctx.launch_count() - n0
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()

    # results kept for the accuracy check against the reference (below)
    results = {}
    if rank == 0:
        results[args.mode] = C.download()
        if mode != 0:
            Cp = op.make_result()
            op.perform(Cp, mode=0)
            results["plain"] = Cp.download()
            Cp.close()

    # plain FP64 DMMA companion on the same workload (the metric's denominator)
    plain = None
    if mode != 0 and not args.no_plain:
        for _ in range(3):
            op.perform(C, mode=0)
        barrier()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(args.steps):
            op.perform(C, mode=0)
        p1.record(stream)
        barrier()
        pms = max_over_ranks([p0.elapsed_time(p1) / args.steps], dev, world)[0]
        plain = {"value": replica_rate(flops, pms, world) / 1e12, "unit": "TFLOP/s", "ms_per_step": pms}
    # slice split-precision companions (Ozaki BF16 / FP8 slices, FP32
    # accumulation) on the same workload: throughput, and their results for
    # the accuracy check against the reference -- the counts that reach the
    # metric's bound (BF16 x7) or near it (FP8 x8), and 3 and 4 slices
    slices = None
    if args.mode == "ozaki-crt" and not args.no_slices:
        slices = {}
        for key, sname, S in (("ozaki-bf16", "ozaki-bf16", 7), ("ozaki-fp8", "ozaki-fp8", 8),
                              ("ozaki-bf16x3", "ozaki-bf16", 3), ("ozaki-bf16x4", "ozaki-bf16", 4),
                              ("ozaki-fp8x3", "ozaki-fp8", 3), ("ozaki-fp8x4", "ozaki-fp8", 4)):
            sm = MODES[sname]
            for _ in range(3):
                op.perform(C, mode=sm, nslices=S)
            barrier()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            for _ in range(args.steps):
                op.perform(C, mode=sm, nslices=S)
            s1.record(stream)
            barrier()
            sms = max_over_ranks([s0.elapsed_time(s1) / args.steps], dev, world)[0]
            slices[key] = {"value": replica_rate(flops, sms, world) / 1e12, "unit": "TFLOP/s", "slices": S,
                           "ms_per_step": sms}
            if rank == 0:
                results[key] = C.download()
    # symmetrizer companion (plain mode): fused into the contraction epilogue
    # against the contraction into a temporary followed by the symmetrizer
    symm = None
    if args.symmetrize:
        from libtensor_b200.core import btod_symmetrize
        kw = dict(symm=False, idx=(0, 1)) if args.symmetrize == "asymm01" else dict(symm=False, perm=(1, 0, 3, 2))
        Rf = op.make_symmetrized(**kw)
        G = op.make_result()
        sy = btod_symmetrize(G, **kw)
        Ru = sy.make_result()

        def timed(fn):
            for _ in range(3):
                fn()
            barrier()
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream)
            for _ in range(args.steps):
                fn()
            q1.record(stream)
            barrier()
            return max_over_ranks([q0.elapsed_time(q1) / args.steps], dev, world)[0]

        def unfused():
            op.perform(G, mode=mode, nslices=args.nslices)
            sy.perform(Ru)
        fms = timed(lambda: op.perform_symmetrized(Rf, mode=mode, nslices=args.nslices, **kw))
        ums = timed(unfused)
        diff = None
        if rank == 0:
            # relative to the contraction's largest element (a symmetrizer
            # whose terms cancel leaves a result of rounding size)
            a, b = Rf.download(), Ru.download()
            diff = float(np.max(np.abs(a - b))) / max(1e-300, float(np.max(np.abs(G.download()))))
        symm = {"terms": args.symmetrize, "fused_ms": fms, "unfused_ms": ums,
                "fused_vs_unfused": ums / fms, "max_diff_rel_to_contraction": diff,
                "temporary_bytes_saved": 8 * G.nelems}
        for t in (Rf, Ru, G):
            t.close()
    ms = max_over_ranks([ms], dev, world)[0]
    value = replica_rate(flops, ms, world) / 1e12

    # ---- end-to-end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        ha = torch.empty(max(1, A.nelems), dtype=torch.float64, pin_memory=True)
        hb = torch.empty(max(1, B.nelems), dtype=torch.float64, pin_memory=True)
        hc = torch.empty(max(1, C.nelems), dtype=torch.float64, pin_memory=True)
        A.download_async(ha.data_ptr()); B.download_async(hb.data_ptr())
        ctx.synchronize()
        for _ in range(2):
            A.upload_async(ha.data_ptr()); B.upload_async(hb.data_ptr())
            op.perform(C, mode=mode, nslices=args.nslices)
            C.download_async(hc.data_ptr())
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            A.upload_async(ha.data_ptr()); B.upload_async(hb.data_ptr())
            op.perform(C, mode=mode, nslices=args.nslices)
            C.download_async(hc.data_ptr())
        f1.record(stream)
        barrier()
        ems = max_over_ranks([f0.elapsed_time(f1) / args.steps], dev, world)[0]
        e2e = {"value": replica_rate(flops, ems, world) / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": 8 * (A.nelems + B.nelems), "d2h_bytes_per_step": 8 * C.nelems,
               "ms_per_step": ems}
        del ha, hb, hc

    # ---- roofline of the dominant kernel, timed by events inside the timed region
    roofline = None
    if rank == 0:
        split = op.split_bytes(C, mode, args.nslices) if mode != 0 else None
        roofline = contraction_roofline(torch, dev, args, flops, ktimes, split)

    cpu, accuracy = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, accuracy = cpu_baseline(cfg, a_spec, b_spec, C, results, flops, op.get_schedule())

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    out = {"metric": metric_name(), "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
           "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, symmetrised; no public dataset)",
           "config": config_of(args, cfg, flops), "roofline": roofline,
           "kernels": {k: {"launches": n, "ms_total": v, "share": v / sum(x for x, _ in ktimes.values())}
                       for k, (v, n) in ktimes.items()},
           "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk}
    if tiles:
        out["config"]["autotuned_tiles"] = {f"{m}x{n}": t for (m, n), t in tiles.items()}
    if plain:
        out["plain_fp64_dmma"] = plain
        out["split_vs_plain"] = value / plain["value"]
    if slices:
        out["slice_modes"] = slices
    if symm:
        out["symmetrizer"] = symm
    if accuracy:
        out["accuracy"] = accuracy
    print(json.dumps(out))


def measure_int8_peak(torch, dev):
    """cuBLASLt INT8 GEMM 8192^3 (torch._int_mm, best of 3), TOP/s."""
    n = 8192
    a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device=dev)
    b = torch.randint(-64, 64, (n, n), dtype=torch.int8, device=dev)
    torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def contraction_roofline(torch, dev, args, flops, ktimes, split=None):
    """Roofline of the kernel with the largest device time in the timed region.

    Plain mode: the DMMA contraction against the live cuBLAS DGEMM rate.
    Split modes: the slice-product kernel; its algorithmic work is the
    S(S+1)/2 slice products per FP64 multiply-add of the schedule
    (2*|C|*K each), against the live dense rate of the slice type."""
    if not ktimes:
        return None
    kname = max(ktimes, key=lambda k: ktimes[k][0])
    kms, kn = ktimes[kname]
    sec = kms * 1e-3 / max(1, kn)                       # average launch
    per_launch = flops * args.steps / max(1, kn)        # algorithmic FP64 flops per launch
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        t = json.load(open(tpath)).get(f"{kname}:{args.workload}:{args.mode}")
        traffic = t.get("bytes_per_launch") if isinstance(t, dict) else t
    if kname == "contract_fp64":
        peak = measure_fp64_peak(torch, dev)
        ach = per_launch / sec / 1e12
        return {"bound": "tensor", "kernel": kname, "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                "frac": ach / peak, "traffic": traffic, "avg_launch_ms": sec * 1e3,
                "peak_source": "measured live: cuBLAS DGEMM 8192^3 (FP64 tensor path), "
                               f"nominal {FP64_NOMINAL} TFLOP/s"}
    if kname == "oz_gemm":
        S = args.nslices if args.nslices > 0 else (8 if args.mode == "ozaki-fp8" else (13 if args.mode == "ozaki-crt" else 7))
        # slice products per FP64 multiply-add: S(S+1)/2 for the slice modes,
        # one per modulus for the modular mode
        prods = S if args.mode == "ozaki-crt" else S * (S + 1) // 2
        ach = prods * per_launch / sec / 1e12
        if args.mode in ("ozaki-int8", "ozaki-crt"):
            try:
                peak, src = measure_int8_peak(torch, dev), "measured live: cuBLASLt INT8 GEMM 8192^3 (torch._int_mm)"
            except Exception as e:     # no INT8 GEMM in this torch build
                peak, src = None, f"INT8 GEMM unavailable: {e}"
            unit = "TFLOP/s"       # INT8 multiply-adds counted as 2 operations, like flops
        else:
            mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
                os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"bf16_tflops": 1590.0}
            bf = float(mp["bf16_tflops"])
            peak = bf if args.mode == "ozaki-bf16" else 2 * bf
            src = ("measured bf16 dense (MEASURED_PEAKS.json bf16_tflops)" if args.mode == "ozaki-bf16" else
                   "2 x measured bf16 dense (FP8 E4M3 is twice the bf16 rate on this part)")
            unit = "TFLOP/s"
        return {"bound": "tensor", "kernel": kname, "achieved": ach, "peak": peak, "unit": unit,
                "frac": ach / peak if peak else None, "traffic": traffic, "avg_launch_ms": sec * 1e3,
                "slice_products": prods, "effective_fp64_tflops": per_launch / sec / 1e12,
                "peak_source": src}
    if kname == "oz_split" and split is not None:
        rb, wb = split
        peak, src = hbm_peak()
        ach = (rb + wb) / sec / 1e9
        return {"bound": "hbm", "kernel": kname, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "traffic": traffic, "avg_launch_ms": sec * 1e3,
                "algorithmic_bytes": {"read": rb, "write": wb,
                                      "note": "FP64 operands read by the exponent and residue passes, "
                                              "residue (or slice) images written"},
                "peak_source": src}
    return {"bound": "hbm", "kernel": kname, "achieved": None, "peak": None, "unit": "GB/s",
            "frac": None, "traffic": traffic, "avg_launch_ms": sec * 1e3}


def block_accuracy(C, arena, rc):
    """Block max-norm relative error (worst block) and RMS relative error of a
    product result against the reference's result tensor."""
    worst, num, den = 0.0, 0.0, 0.0
    for bidx, g in C.blocks(arena):
        r = rc.get_block(bidx, g.shape)
        m = float(np.max(np.abs(r))) if r.size else 0.0
        if m > 0:
            worst = max(worst, float(np.max(np.abs(g - r))) / m)
        num += float(np.sum((g - r) ** 2))
        den += float(np.sum(r ** 2))
    return {"max_block_rel_err": worst, "rms_rel_err": (num / den) ** 0.5 if den > 0 else 0.0}


def cpu_baseline(cfg, a_spec, b_spec, C, results, flops, sched):
    """The reference's perform() on the same seeded inputs, timed on the host
    cores, and the product's results (this mode and the plain path) compared
    block by block with the reference's result."""
    try:
        from oracle import refapi as R
        if not R.available():
            return None, None
        R.set_threads(os.cpu_count() or 1)
        ra, rb, op, rc = build_reference(a_spec, b_spec, cfg)
        sec, runs = time_reference(op, rc, 2, 0, budget_s=30.0)
        cpu = {"value": flops / sec / 1e12, "unit": "TFLOP/s", "cores": os.cpu_count(), "kind": "reference",
               "sample": f"full workload, {runs} perform() call(s) of the reference built from its sources "
                         f"(OpenBLAS, 1 BLAS thread x {os.cpu_count()} libutil threads, one batch per operand)",
               "ms_per_step": sec * 1e3}
        acc = {k: block_accuracy(C, v, rc) for k, v in results.items()}
        acc["against"] = ("the reference CPU btod_contract2 (built from its sources) on the same seeded "
                          "inputs, per canonical C block")
        acc["nonzero_blocks_identical"] = op.schedule() == list(sched)
        for x in (rc, ra, rb):
            x.close()
        op.close()
        return cpu, acc
    except Exception as e:   # the baseline is reported, never required
        return ({"value": None, "unit": "TFLOP/s", "cores": os.cpu_count(), "kind": "reference",
                 "sample": f"failed: {e}"}, None)


# ---------------------------------------------------------------- HBM-bound operations

def hbm_peak():
    """Measured copy bandwidth of this GPU model (GB/s) and where it came from."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, torch copy)"
    return 6650.0, "fallback 6.65 TB/s"


def transfer_setup(name, ctx):
    """Operands, the operation and its algorithmic bytes per call."""
    from libtensor_b200 import spec as S
    from libtensor_b200.core import block_tensor, btod_add, btod_copy, btod_dotprod
    cfg = S.LADDER_CCD
    if name == "copy-vvvv":
        a = block_tensor(ctx, cfg.v_spec())
        a.fill_seeded(31, 1.0)
        b = a.permuted((0, 2, 1, 3))
        op = btod_copy(a, (0, 2, 1, 3), 1.0)
        run = lambda: op.perform(b)                       # noqa: E731
        return dict(srcs=[a], dst=b, run=run, bytes=16 * b.nelems, terms=1,
                    desc="B = P(0,2,1,3) V, V(a,b,c,d) v=300 antisym ab, cd + spin")
    if name == "add-x4":
        x = block_tensor(ctx, cfg.x_spec())
        x.fill_seeded(32, 1.0)
        r = block_tensor(ctx, cfg.x_spec())
        op = btod_add(x, None, 1.0)
        op.add_op(x, (1, 0, 2, 3), -1.0)
        op.add_op(x, (0, 1, 3, 2), -0.5)
        op.add_op(x, (1, 0, 3, 2), 0.5)
        run = lambda: op.perform(r)                       # noqa: E731
        return dict(srcs=[x], dst=r, run=run, bytes=(8 * 4 + 8) * r.nelems, terms=4,
                    desc="r = X - P(ij)X - 0.5 P(ab)X + 0.5 P(ij)P(ab)X, X(i,j,a,b) o=30 v=300 spin blocks")
    if name == "dot-vvvv":
        a = block_tensor(ctx, cfg.v_spec())
        b = block_tensor(ctx, cfg.v_spec())
        a.fill_seeded(33, 1.0)
        b.fill_seeded(34, 1.0)
        op = btod_dotprod(a, None, b, (1, 0, 3, 2))
        out = {}
        run = lambda: out.__setitem__("v", op.calculate())   # noqa: E731
        return dict(srcs=[a, b], dst=None, run=run, bytes=16 * a.nelems, terms=2, out=out, op=op,
                    desc="<V, P(1,0,3,2) V'>, V v=300 antisym ab, cd + spin")
    raise ValueError(name)


def transfer_arm(args):
    import torch
    from libtensor_b200.core import Context
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    ctx = Context(local)
    w = transfer_setup(args.workload, ctx)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(max(3, args.warmup)):
        w["run"]()
    ctx.synchronize()
    torch.cuda.synchronize()
    n0 = ctx.launch_count()
    ctx.set_timing(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        w["run"]()
    e1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    launches = ctx.launch_count() - n0
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    ms = max_over_ranks([ms], dev, world)[0]
    gbs = replica_rate(w["bytes"], ms, world) / 1e9
    kname = "dot" if args.workload.startswith("dot") else "transfer"
    kms, kn = kt.get(kname, (0.0, 0))
    peak, peak_src = hbm_peak()
    achieved = w["bytes"] * args.steps / (kms * 1e-3) / 1e9 if kms > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(f"{kname}:{args.workload}")

    e2e = None
    if not args.no_e2e:
        hs = [torch.empty(max(1, t.nelems), dtype=torch.float64, pin_memory=True) for t in w["srcs"]]
        hd = torch.empty(max(1, w["dst"].nelems), dtype=torch.float64, pin_memory=True) if w["dst"] else None
        for t, h in zip(w["srcs"], hs):
            t.download_async(h.data_ptr())
        ctx.synchronize()

        def e2e_step():
            for t, h in zip(w["srcs"], hs):
                t.upload_async(h.data_ptr())
            w["run"]()
            if hd is not None:
                w["dst"].download_async(hd.data_ptr())
        for _ in range(2):
            e2e_step()
        ctx.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        f1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        ems = max_over_ranks([f0.elapsed_time(f1) / args.steps], dev, world)[0]
        h2d = sum(8 * t.nelems for t in w["srcs"])
        d2h = 8 * w["dst"].nelems if w["dst"] else 8
        e2e = {"value": replica_rate(w["bytes"], ems, world) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    out = {"metric": f"{args.workload}: algorithmic GB/s", "value": gbs, "unit": "GB/s", "n_gpus": world,
           "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, symmetrised)",
           "config": {"workload": f"{args.workload}: {w['desc']}", "algorithmic_bytes": w["bytes"],
                      "l2": "operands larger than L2 (no flush)"},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak if achieved else None, "traffic": traffic,
                        "peak_source": peak_src, "kernel": kname},
           "kernels": {k: {"launches": n, "ms_total": v} for k, (v, n) in kt.items()},
           "e2e": e2e, "gpu_launches": launches, "clocks": clk, "cpu_baseline": None}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = transfer_cpu_baseline(args.workload, w)
    print(json.dumps(out))


def transfer_elems(name):
    """Elements of the result (copy, add) or of each operand (dot): the
    canonical allowed blocks of the tensor, counted on the description, each
    block rounded up to 4 elements as the product's arenas store them."""
    from oracle import restate as X
    spec = transfer_inputs(name)[0][0]
    if name == "copy-vvvv":
        from libtensor_b200.spec import permuted_spec
        spec = permuted_spec(spec, (0, 2, 1, 3))
    bid = spec.bidims()
    n = 0
    for a in X.canonical_blocks(spec):
        bidx = X._unabs(a, bid)
        m = 1
        for d, b in enumerate(bidx):
            m *= spec.block_extent(d, b)
        n += (m + 3) // 4 * 4
    return n


def transfer_inputs(name):
    """(spec, seed) of each operand of a transfer workload (scale 1.0), as
    transfer_setup fills them."""
    from libtensor_b200 import spec as S
    cfg = S.LADDER_CCD
    return {"copy-vvvv": [(cfg.v_spec(), 31)], "add-x4": [(cfg.x_spec(), 32)],
            "dot-vvvv": [(cfg.v_spec(), 33), (cfg.v_spec(), 34)]}[name]


def transfer_reference(name):
    """The reference's own btod_copy / btod_add / btod_dotprod on the same
    seeded inputs (generated inside the reference library); returns
    (callable, tensors to close)."""
    from oracle import refapi as R
    refs = []
    for spec, seed in transfer_inputs(name):
        r = R.RefBT(spec)
        r.fill_seeded(seed, 1.0)
        refs.append(r)
    if name == "copy-vvvv":
        from libtensor_b200.spec import permuted_spec
        rb = R.RefBT(permuted_spec(refs[0].spec, (0, 2, 1, 3)))
        return (lambda: R.ref_copy(refs[0], (0, 2, 1, 3), 1.0, rb)), refs + [rb]
    if name == "add-x4":
        rr = R.RefBT(refs[0].spec)
        x = refs[0]
        ops = [(x, None, 1.0), (x, (1, 0, 2, 3), -1.0), (x, (0, 1, 3, 2), -0.5), (x, (1, 0, 3, 2), 0.5)]
        return (lambda: R.ref_add(ops, rr)), refs + [rr]
    return (lambda: R.ref_dotprod(refs[0], None, refs[1], (1, 0, 3, 2))), refs


def transfer_cpu_baseline(name, w, steps=2, budget_s=30.0):
    try:
        from oracle import refapi as R
        if not R.available():
            return None
        R.set_threads(os.cpu_count() or 1)
        fn, refs = transfer_reference(name)
        ts = []
        t_start = time.perf_counter()
        for _ in range(steps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
            if time.perf_counter() - t_start > budget_s:
                break
        for r in refs:
            r.close()
        sec = float(np.median(ts))
        return {"value": w["bytes"] / sec / 1e9, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"full workload, {len(ts)} call(s) of the reference built from its sources",
                "ms_per_step": sec * 1e3}
    except Exception as e:
        return {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"failed: {e}"}


def ccd_arm(args):
    """CCD iteration graph: value = contraction flops (ladder + ring) per second."""
    import torch
    from libtensor_b200.ccd import CCDIteration
    from libtensor_b200.core import Context
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    ctx = Context(local)
    mode = MODES[args.mode]
    it = CCDIteration(ctx, [15], [50, 50, 50], mode, args.nslices)
    # per-operation device times of one eager iteration (the first
    # iteration's energy is compared with the reference's first iteration)
    it.step()
    ctx.synchronize()
    energy0 = it.energy()
    ctx.set_timing(True)
    n0 = ctx.launch_count()
    it.step()
    per_iter = ctx.launch_count() - n0          # kernels in one iteration (and in the graph)
    kt = ctx.kernel_times()
    ctx.set_timing(False)
    it.capture()
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(max(3, args.warmup)):
        it.launch()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        it.launch()
    e1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    energy = it.energy()
    # end to end: amplitudes uploaded from pinned host memory, the graph, the
    # energy read back, every step
    nt = it.t.nelems
    ht = torch.empty(max(1, nt), dtype=torch.float64, pin_memory=True)
    he = torch.empty(1, dtype=torch.float64, pin_memory=True)
    it.t.download_async(ht.data_ptr())
    ctx.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        it.t.upload_async(ht.data_ptr())
        it.launch()
        with torch.cuda.stream(stream):
            he.copy_(it.energy_dev, non_blocking=True)
    f1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ems = f0.elapsed_time(f1) / args.steps
    ms, ems = max_over_ranks([ms, ems], dev, world)
    flops = it.flops
    it.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import refapi as R
            if R.available():
                sec, runs, rflops, e_ref = ccd_reference(1, 60.0)
                cpu = {"value": rflops / sec / 1e12, "unit": "TFLOP/s", "cores": os.cpu_count(),
                       "kind": "reference", "ms_per_step": sec * 1e3,
                       "sample": f"full workload, {runs} iteration(s) of the reference's operations in sequence",
                       "energy": e_ref, "energy_rel_diff": abs(energy0 - e_ref) / abs(e_ref) if e_ref else None}
        except Exception as e:   # the baseline is reported, never required
            cpu = {"value": None, "unit": "TFLOP/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    tot = sum(v for v, _ in kt.values())
    out = {"metric": "CCD iteration (CUDA graph): contraction TFLOP/s eff. FP64",
           "value": replica_rate(flops, ms, world) / 1e12, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
           "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, symmetrised)",
           "config": {"workload": "ccd-iter: o=30 (15 per spin) v=300 (50,50,50 per spin); copy P(0,2,1,3), "
                                  "ladder, ring, 5-term add, denominator, energy, t <- R; one graph launch per step",
                      "mode": args.mode, "nslices": args.nslices, "algorithmic_flops": flops,
                      "l2": "operands larger than L2 (no flush)"},
           "kernels_eager_iteration": {k: {"launches": n, "ms_total": v, "share": v / tot} for k, (v, n) in kt.items()},
           "energy": energy,
           "e2e": {"value": replica_rate(flops, ems, world) / 1e12, "unit": "TFLOP/s",
                   "h2d_bytes_per_step": 8 * nt, "d2h_bytes_per_step": 8, "ms_per_step": ems},
           "gpu_launches": per_iter * args.steps, "clocks": clk, "cpu_baseline": cpu, "roofline": None,
           "first_iteration_energy": energy0}
    print(json.dumps(out))


def ccd_reference(steps, budget_s):
    """The CCD iteration on the reference built from its sources, one
    operation after the other (oracle/ref_ccd.py), on the host cores: each
    timed step is the first iteration of freshly built tensors (the
    reference's assigning add stores R with the add's own, spin-only,
    symmetry, so later iterations would run on a less symmetric t).
    Returns (seconds per step, steps run, flops, energy)."""
    from oracle import refapi as R
    from oracle.ref_ccd import RefCCDIteration
    R.set_threads(os.cpu_count() or 1)
    ts, flops, energy = [], None, None
    t_start = time.perf_counter()
    for _ in range(max(1, steps)):
        it = RefCCDIteration([15], [50, 50, 50])
        t0 = time.perf_counter()
        it.step()
        ts.append(time.perf_counter() - t0)
        flops, energy = it.flops, it.energy
        it.close()
        if time.perf_counter() - t_start > budget_s:
            break
    return float(np.median(ts)), len(ts), flops, energy


def ccd_reference_arm(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from oracle import refapi as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libltref.so was not built"}))
        return
    sec, runs, flops, energy = ccd_reference(args.steps, 120.0)
    v = flops / sec / 1e12
    print(json.dumps({
        "metric": "CCD iteration (CUDA graph): contraction TFLOP/s eff. FP64", "value": v, "unit": "TFLOP/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": runs, "warmup": 0, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, symmetrised)",
        "config": {"workload": "ccd-iter: o=30 (15 per spin) v=300 (50,50,50 per spin); the reference's "
                               "btod_copy, btod_contract2 (ladder, ring), btod_add, denominator, btod_dotprod, "
                               "btod_copy in sequence", "algorithmic_flops": flops},
        "energy": energy,
        "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": os.cpu_count(), "kind": "reference",
                         "sample": f"full workload, {runs} iteration(s), median"},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def main():
    args = parse()
    if args.workload in GRAPH_WORKLOADS:
        if args.impl == "reference":
            ccd_reference_arm(args)
        else:
            ccd_arm(args)
        return
    if args.workload in TRANSFER_WORKLOADS:
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) != 0:
                return
            nbytes = {"copy-vvvv": 16, "add-x4": 40, "dot-vvvv": 16}[args.workload]
            from oracle import refapi as R
            if not R.available():
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libltref.so was not built"}))
                return
            w = {"bytes": nbytes * transfer_elems(args.workload)}
            b = transfer_cpu_baseline(args.workload, w, steps=args.steps, budget_s=120.0)
            print(json.dumps({"metric": f"{args.workload}: algorithmic GB/s", "value": b["value"], "unit": "GB/s",
                              "impl": "reference", "n_gpus": args.gpus, "higher_is_better": True,
                              "cpu_baseline": b, "e2e": {"value": b["value"], "unit": "GB/s",
                                                         "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        else:
            transfer_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        ltg_arm(args)


if __name__ == "__main__":
    main()
