#!/usr/bin/env python
"""Benchmark: SP2 density-matrix purification on the ELLPACK N=64000 lattice
Hamiltonian (40^3 sites, neighbours within radius 3, threshold 1e-5,
occupation N/2), FP64, through libbml_b200's C ABI.

One step = one SP2 run from H: Gershgorin bounds, X0 = (emax I - H)/(emax -
emin), then SP2_ITERS iterations of X^2 (thresholded, traces) and the branch
update X <- X^2 or X <- 2X - X^2.  The full solve of this Hamiltonian fills in
to a dense 64000^2 matrix (the system is metallic at half filling: its density
matrix decays too slowly for the threshold to keep rows sparse), so the timed
solve is the first SP2_ITERS iterations, in which rows grow from 123 to ~1500
entries; the stop rule |tr X - tr X^2| < 1e-8 is not reached within them.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) one solve is split over the ranks (bml_b200/sharded.py):
each rank forms its block of rows of X^2, the partial traces are summed, and
the new iterate's rows are all-gathered over NCCL after every iteration;
rank 0 prints one JSON line with the slowest rank's time (strong scaling).
`value` is seconds per SP2 solve.  `e2e` is the same metric through the C ABI
with host buffers: H uploaded from host arrays and the density matrix
downloaded every step.  --impl reference runs the reference
bml CPU library (built from its sources into oracle/_ref) on the host cores
with the same inputs and loop.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L, RADIUS, SEED = 40, 3, 0
N = L ** 3
M_H = 256          # stored width of H (interior rows hold 123)
M_X = 2048         # stored width of the iterates (iteration 5 needs 1792)
THRESHOLD = 1e-5
OCC = N / 2.0
SP2_ITERS = 4
# B200 FP64 (vector and tensor) nominal rate, HGX figure per GPU; no measured
# FP64 peak is available, so fractions against it are "of nominal"
FP64_NOMINAL_TFLOPS = 37.0
METRIC = "s per SP2 solve & X² HBM GB/s, ELLPACK N=64K: FP64 vs mixed at ≤1e-6 err"
WORKLOAD = ("SP2 on the 40^3 lattice Hamiltonian (N=64000, radius 3, M=%d, thr 1e-5, occ N/2, FP64), "
            "first %d iterations from X0 (the full solve fills in to dense)" % (M_X, SP2_ITERS))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-tc", action="store_true",
                    help="run the small tensor-core ELLBLOCK case for an ncu capture (10^3 block lattice)")
    ap.add_argument("--profile-tc-wide", action="store_true",
                    help="the same for the SP2 iterate after one iteration (the second iteration's product)")
    ap.add_argument("--tc-split", type=int, default=0, choices=[0, 1],
                    help="split of the tensor-core X^2 in the profile cases: 0 FP16 hi/lo, 1 8-bit slices")
    ap.add_argument("--profile-eb-sp2", action="store_true",
                    help="one mixed ELLBLOCK SP2 run (16^3, 5 iterations, 8-bit split, 1 closing FP64 iteration) "
                         "inside the NVTX range sp2, for an ncu launch list")
    ap.add_argument("--profile-eb-ops", action="store_true",
                    help="the one-pass ELLBLOCK operations, once each, for an ncu capture (7^3 block lattice)")
    ap.add_argument("--eb-ops-L", type=int, default=7, help="block lattice side for --profile-eb-ops")
    ap.add_argument("--profile-eb", action="store_true",
                    help="run the small exact ELLBLOCK case for an ncu capture (10^3 block lattice)")
    ap.add_argument("--no-ellblock", action="store_true", help="skip the ELLBLOCK tensor-core leg")
    ap.add_argument("--exchange", default="gather", choices=["gather", "halo"],
                    help="with --gpus > 1: all-gather the iterate after each update, or send each rank only "
                         "the rows its next X^2 reads")
    ap.add_argument("--step-only", action="store_true",
                    help="time the SP2 steps only (no e2e, roofline, mixed, chain, ELLBLOCK or CPU legs), for a "
                         "launch-list capture; the timed steps run inside an NVTX range \"step\"")
    ap.add_argument("--profile", action="store_true",
                    help="small case for ncu: 30^3 lattice, 3 SP2 iterations then one X^2")
    ap.add_argument("--profile-ops", action="store_true",
                    help="case for ncu of the one-pass ELLPACK operations (add, threshold, copy, scale, "
                         "trace, Gershgorin, transpose) on the 30^3 lattice's SP2 iterate X and X^2")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
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
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def inputs():
    import bml_b200 as B
    return B.gen_lattice(L, RADIUS, N, M_H, SEED)


def bench_config(world, exchange="gather"):
    """The `config` object of the JSON line, the same in both arms."""
    how = {"gather": "NCCL all-gather of the iterate",
           "halo": "NCCL point-to-point rows within each rank's column range"}[exchange]
    return {"workload": WORKLOAD, "N": N, "M": M_X, "threshold": THRESHOLD,
            "sp2_iterations": SP2_ITERS,
            "parallelism": ("rows sharded over %d GPUs (%s)" % (world, how)) if world > 1 else "1 GPU",
            "l2": "inputs larger than L2 (iterates ~0.8-1.3 GB)"}


# ---------------------------------------------------------------------------
# libbml_b200 arm
# ---------------------------------------------------------------------------
def run_b200(args, rank, world, local):
    import numpy as np
    import bml_b200 as B
    B.check(B.lib.bml_b200_set_device(local))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        pg = dist
    v, ix, nz = inputs()
    H = B.Ellpack.from_arrays(v, ix, nz, N, M_H)
    D = B.Ellpack(N, M_X)
    info = (C.c_double * 6)()
    dv = np.zeros(N * M_X)
    dix = np.zeros(N * M_X, np.int32)
    dnz = np.zeros(N, np.int32)
    # pinned host buffers for the end-to-end leg
    import torch
    h_v = torch.from_numpy(v).pin_memory().numpy()
    h_ix = torch.from_numpy(ix).pin_memory().numpy()
    h_nz = torch.from_numpy(nz).pin_memory().numpy()
    o_v = torch.empty(N * M_X, dtype=torch.float64).pin_memory().numpy()
    o_ix = torch.empty(N * M_X, dtype=torch.int32).pin_memory().numpy()
    o_nz = torch.empty(N, dtype=torch.int32).pin_memory().numpy()

    sharded = None
    if world > 1:
        # One solve split over the ranks: each forms its rows of X^2, the
        # traces are summed and the new iterate's rows all-gathered (NCCL).
        from bml_b200.sharded import GpuOps, ShardedSP2
        ops = GpuOps(B.lib, H.h, M_X, THRESHOLD, pg, torch)
        sharded = ShardedSP2(ops, pg, rank, world, args.exchange)

    def step():
        if sharded is not None:
            t0 = time.perf_counter()
            res = sharded.run(OCC, SP2_ITERS, 1e-8, 0)
            info[0], info[1], info[2], info[3] = res["iterations"], res["rule"], res["trace"], res["idempotency"]
            info[5] = time.perf_counter() - t0
            return
        st = B.lib.bml_b200_sp2(H.h, D.h, THRESHOLD, OCC, SP2_ITERS, 1e-8, 0, info)
        B.check(st)

    def barrier():
        if pg:
            pg.barrier()

    def max_over_ranks(x):
        if not pg:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    # The clock sampler starts before the last warm-up step, so that its own
    # start-up (nvidia-smi and NVML) falls outside the timed region.
    clocks = ClockSampler(local)
    for k in range(args.warmup):
        if k == args.warmup - 1:
            clocks.start()
        step()
    if args.warmup == 0:
        clocks.start()
    B.check(B.lib.bml_b200_synchronize())
    # X^2 roofline inputs from the last warm-up run
    x2_seconds_per_run = info[5]
    widths = info[4]
    barrier()
    launches0 = B.lib.bml_b200_launch_count()
    B.check(B.lib.bml_b200_event_record(0))
    step_ev = []
    nvtx = _nvtx()
    for k in range(args.steps):
        nvtx.range_push("step")
        step()
        nvtx.range_pop()
        if k < 32:
            slot = 16 + k
            B.check(B.lib.bml_b200_event_record(slot))
            step_ev.append(slot)
    B.check(B.lib.bml_b200_event_record(1))
    ms = B.event_ms(0, 1)
    step_ms = [B.event_ms(a, b) for a, b in zip([0] + step_ev[:-1], step_ev)]
    launches = B.lib.bml_b200_launch_count() - launches0
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(ms)
    sec_per_step = ms / 1e3 / args.steps
    value = sec_per_step  # one solve, split over the ranks when world > 1
    if args.step_only:
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return {"metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "step_ms": step_ms,
                "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "config": bench_config(world, args.exchange), "gpu_launches": int(B.lib.bml_b200_launch_count() - launches0),
                "note": "--step-only: the SP2 steps alone"} if rank == 0 else None

    # end-to-end through the C ABI with host buffers
    barrier()
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 3))):
        B.check(B.lib.bml_b200_ellpack_upload(H.h, h_v.ctypes.data_as(C.c_void_p),
                                             h_ix.ctypes.data_as(C.POINTER(C.c_int)),
                                             h_nz.ctypes.data_as(C.POINTER(C.c_int))))
        step()
        B.check(B.lib.bml_b200_ellpack_download(ops.X if sharded is not None else D.h,
                                               o_v.ctypes.data_as(C.c_void_p),
                                               o_ix.ctypes.data_as(C.POINTER(C.c_int)),
                                               o_nz.ctypes.data_as(C.POINTER(C.c_int))))
    e2e_steps = max(1, min(args.steps, 3))
    e2e = (time.perf_counter() - t0) / e2e_steps
    e2e = max_over_ranks(e2e)

    # per-X^2 roofline: one X^2 on the iterate of iteration SP2_ITERS-1
    rl = x2_roofline(B, H, info)
    # the single-GPU legs (mixed precision, ELLBLOCK tensor cores) run only
    # without the sharded solve
    mixed = mixed_leg(B, v, ix, nz, max(3, min(args.steps, 5))) if world == 1 else None
    chain = chain_solve_leg(B) if world == 1 else None
    ellb = None if (args.no_ellblock or world > 1) else ellblock_leg()
    ellb_sp2 = None if (args.no_ellblock or world > 1) else ellblock_sp2_leg()
    res = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "step_ms": step_ms, "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded splitmix64 lattice Hamiltonian, generated on the host)",
        "config": bench_config(world, args.exchange),
        # the transfers move each row's columns up to the widest row
        "e2e": {"value": e2e, "unit": "s",
                "h2d_bytes_per_step": int(N * int(nz.max()) * (v.itemsize + ix.itemsize) + nz.nbytes),
                "d2h_bytes_per_step": int(N * int(o_nz.max()) * (o_v.itemsize + o_ix.itemsize) + o_nz.nbytes)},
        "gpu_launches": int(launches),
        "roofline": rl,
        "clocks": clk,
        "sp2": {"iterations": info[0], "trace": info[2], "idempotency": info[3], "max_row_width": widths,
                "x2_seconds_per_run": x2_seconds_per_run},
        "mixed": mixed,
        "chain_solve": chain,
        "ellblock_tc": ellb,
        "ellblock_sp2": ellb_sp2,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res["cpu_baseline"] = cpu_baseline()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return res if rank == 0 else None


def mixed_leg(B, v, ix, nz, reps):
    """The mixed-precision form on the same workload: the first SP2_ITERS-2
    iterations in FP32 (FP64 traces, branch and stop tests), the last two in
    FP64.  Timed like the main leg (CUDA events on the library stream around
    `reps` runs), then compared with the FP64 solve: relative errors of tr D
    and of the band energy tr(DH), ||D_mixed - D_fp64||_F / ||D_fp64||_F, and
    the idempotency ||X^2 - X||_F of both results (X^2 thresholded at 1e-5)."""
    import numpy as np
    pad = lambda a: np.pad(a.reshape(N, M_H), ((0, 0), (0, M_X - M_H))).reshape(-1)
    Hp = B.Ellpack.from_arrays(pad(v), pad(ix), nz, N, M_X)
    nclose = 2

    def timed(fn, reps):
        fn()
        B.check(B.lib.bml_b200_synchronize())
        B.check(B.lib.bml_b200_event_record(4))
        for _ in range(reps):
            fn()
        B.check(B.lib.bml_b200_event_record(5))
        return B.event_ms(4, 5) / 1e3 / reps

    D64, Dm = B.Ellpack(N, M_X), B.Ellpack(N, M_X)
    i64, im = (C.c_double * 6)(), (C.c_double * 8)()
    t64 = timed(lambda: B.check(B.lib.bml_b200_sp2(Hp.h, D64.h, THRESHOLD, OCC, SP2_ITERS, 1e-8, 0, i64)), reps)
    tm = timed(lambda: B.check(B.lib.bml_b200_sp2_mixed(Hp.h, Dm.h, THRESHOLD, OCC, SP2_ITERS, 1e-8, 0,
                                                        nclose, im)), reps)
    e64 = B.lib.bml_trace_mult(D64.h, Hp.h)
    em = B.lib.bml_trace_mult(Dm.h, Hp.h)
    n64 = B.lib.bml_fnorm(D64.h)
    dist = B.lib.bml_fnorm2(Dm.h, D64.h)
    T = B.Ellpack(N, 2 * M_X)

    def idem(D):
        st, _ = B.multiply_x2(D, T, THRESHOLD)
        B.check(st)
        return B.lib.bml_fnorm2(T.h, D.h)

    res = {"value": tm, "unit": "s", "fp64_value": t64, "speedup_vs_fp64": t64 / tm,
           "fp32_iterations": int(im[6]), "fp64_closing_iterations": nclose,
           "trace_rel_err": abs(im[2] - i64[2]) / abs(i64[2]),
           "energy_trDH_rel_err": abs(em - e64) / abs(e64),
           "density_rel_fro_err": dist / n64,
           "idempotency_fro": {"fp64": idem(D64), "mixed": idem(Dm)},
           "target": "mixed >= 2x faster than FP64 at <= 1e-6 relative trace/energy error"}
    # the same with one FP32 iteration and the rest in FP64
    D1, i1 = B.Ellpack(N, M_X), (C.c_double * 8)()
    t1 = timed(lambda: B.check(B.lib.bml_b200_sp2_mixed(Hp.h, D1.h, THRESHOLD, OCC, SP2_ITERS, 1e-8, 0,
                                                        SP2_ITERS - 1, i1)), reps)
    e1 = B.lib.bml_trace_mult(D1.h, Hp.h)
    res["one_fp32_iteration"] = {"value": t1, "speedup_vs_fp64": t64 / t1, "fp32_iterations": int(i1[6]),
                                 "trace_rel_err": abs(i1[2] - i64[2]) / abs(i64[2]),
                                 "energy_trDH_rel_err": abs(e1 - e64) / abs(e64),
                                 "density_rel_fro_err": B.lib.bml_fnorm2(D1.h, D64.h) / n64}
    for m in (Hp, D64, Dm, D1, T):
        m.free()
    return res


def chain_solve_leg(B, reps=3, nclose=2):
    """Config 1 timed as a full SP2 solve: the 1-D chain Hamiltonian (N=4096,
    H_ij = u exp(-|i-j|/4) for |i-j| <= 16, seed 0), threshold 1e-5,
    occupation N/2, M = 512 (the iterates' widths reach ~390; the stated
    M = 128 overflows, as it does on the reference), run until
    |tr X - tr X^2| < 1e-8, until that error has not improved for 10
    iterations, or for 100 iterations.  FP64 against the mixed form (FP32
    bulk on the unordered kernel, FP64 traces/branch/stop tests, `nclose`
    closing FP64 iterations).  Device time by CUDA events on the library
    stream, `reps` solves each; errors of the mixed result against the FP64
    one: tr D, band energy tr(DH), ||D_mixed - D||_F / ||D||_F, and the
    idempotency ||D^2 - D||_F of both."""
    import numpy as np
    Nc, MHc, Mc = 4096, 128, 512
    v, ix, nz = B.gen_chain(Nc, MHc, 0)
    pad = lambda a: np.pad(a.reshape(Nc, MHc), ((0, 0), (0, Mc - MHc))).reshape(-1)
    H = B.Ellpack.from_arrays(pad(v), pad(ix), nz, Nc, Mc)
    thr, occ, maxit, tol, stall = 1e-5, Nc / 2.0, 100, 1e-8, 10

    def timed(fn):
        fn()
        B.check(B.lib.bml_b200_synchronize())
        B.check(B.lib.bml_b200_event_record(4))
        for _ in range(reps):
            fn()
        B.check(B.lib.bml_b200_event_record(5))
        return B.event_ms(4, 5) / 1e3 / reps

    D64, Dm = B.Ellpack(Nc, Mc), B.Ellpack(Nc, Mc)
    i64, im = (C.c_double * 6)(), (C.c_double * 8)()
    t64 = timed(lambda: B.check(B.lib.bml_b200_sp2(H.h, D64.h, thr, occ, maxit, tol, stall, i64)))
    tm = timed(lambda: B.check(B.lib.bml_b200_sp2_mixed(H.h, Dm.h, thr, occ, maxit, tol, stall, nclose, im)))
    e64, em = B.lib.bml_trace_mult(D64.h, H.h), B.lib.bml_trace_mult(Dm.h, H.h)
    T = B.Ellpack(Nc, 2 * Mc)

    def idem(D):
        st, _ = B.multiply_x2(D, T, thr)
        B.check(st)
        return B.lib.bml_fnorm2(T.h, D.h)

    rules = {1: "tol", 2: "stall", 3: "maxiter", 4: "error"}
    res = {"workload": "SP2 solve on the 1-D chain Hamiltonian (N=4096, M=512, thr 1e-5, occ N/2) to the stop "
                       "rule (|trX - trX^2| < 1e-8, no improvement in 10 iterations, or 100 iterations)",
           "fp64": {"s": t64, "iterations": int(i64[0]), "rule": rules.get(int(i64[1])), "trace": i64[2],
                    "trace_err_t_minus_t2": i64[3], "energy_trDH": e64, "idempotency_fro": idem(D64)},
           "mixed": {"s": tm, "iterations": int(im[0]), "fp32_iterations": int(im[6]),
                     "fp64_closing_iterations": nclose, "rule": rules.get(int(im[1])), "trace": im[2],
                     "energy_trDH": em, "idempotency_fro": idem(Dm)},
           "speedup": t64 / tm,
           "trace_rel_err": abs(im[2] - i64[2]) / abs(i64[2]),
           "energy_trDH_rel_err": abs(em - e64) / abs(e64),
           "density_rel_fro_err": B.lib.bml_fnorm2(Dm.h, D64.h) / B.lib.bml_fnorm(D64.h),
           "target": "mixed >= 2x faster than FP64 at <= 1e-6 relative trace/energy error"}
    for m in (H, D64, Dm, T):
        m.free()
    return res


def products(X, n):
    """Product terms of X^2: P = sum_i sum_{j in row i} nnz_j."""
    import numpy as np
    xv, xix, xnz = X.download()
    rows = xix.reshape(n, -1)
    width = rows.shape[1]
    P = 0
    for i in range(0, n, 4096):
        blk = rows[i:i + 4096]
        mask = np.arange(width)[None, :] < xnz[i:i + 4096, None]
        P += int(xnz[blk[mask]].astype(np.int64).sum())
    return P


def formed_fraction(X, n, sample=400, seed=0):
    """Share of X^2's product terms that the symmetric form computes (those
    with k >= i), from a sample of rows."""
    import numpy as np
    xv, xix, xnz = X.download()
    rows = xix.reshape(n, -1)
    width = rows.shape[1]
    rng = np.random.default_rng(seed)
    tot = part = 0
    for i in rng.choice(n, size=min(sample, n), replace=False):
        js = rows[i, :xnz[i]]
        sub = rows[js]                                   # the rows j of row i
        valid = np.arange(width)[None, :] < xnz[js][:, None]
        tot += int(valid.sum())
        part += int((valid & (sub >= i)).sum())
    return part / max(tot, 1)


# ncu capture of one X^2 call on the 30^3 lattice's SP2 iterate (bench.py
# --profile, 18.57 G reference product terms; profiles/x2_symmetric_lattice30.md):
# the product kernel's dram__bytes_read.sum + dram__bytes_write.sum
NCU_X2_PRODUCTS = 18570945128
NCU_X2_KERNEL_DRAM = 1111612672 + 169511936


def x2_roofline(B, H, info):
    """One X^2 on the SP2 iterate entering iteration SP2_ITERS-1: the
    compulsory HBM bytes of the call over the product kernel's device time
    (CUDA events on the library stream around that kernel, averaged over the
    calls), and the same figures for the whole call."""
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs")
    src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    X = B.Ellpack(N, M_X)
    info2 = (C.c_double * 6)()
    B.check(B.lib.bml_b200_sp2(H.h, X.h, THRESHOLD, OCC, SP2_ITERS - 1, 1e-8, 0, info2))
    X2 = B.Ellpack(N, M_X)
    tr = (C.c_double * 2)()
    old_timing = B.lib.bml_b200_set_kernel_timing(1)
    B.check(B.lib.bml_b200_multiply_x2(X.h, X2.h, THRESHOLD, tr))  # warm
    reps = 3
    kms = []
    B.check(B.lib.bml_b200_event_record(2))
    for _ in range(reps):
        B.check(B.lib.bml_b200_multiply_x2(X.h, X2.h, THRESHOLD, tr))
        kms.append(B.lib.bml_b200_last_x2_kernel_ms())
    B.check(B.lib.bml_b200_event_record(3))
    B.lib.bml_b200_set_kernel_timing(old_timing)
    t_call = B.event_ms(2, 3) / 1e3 / reps
    t_k = sum(kms) / len(kms) / 1e3
    symmetric = B.lib.bml_b200_last_x2_symmetric()
    nnz_x = B.lib.bml_b200_nnz(X.h)
    nnz_x2 = B.lib.bml_b200_nnz(X2.h)
    P = products(X, N)
    frac_formed = formed_fraction(X, N) if symmetric else 1.0
    formed = P * frac_formed
    bytes_alg = 12 * nnz_x + 12 * nnz_x2 + 8 * N
    achieved = bytes_alg / t_k / 1e9
    X.free()
    X2.free()
    return {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_source": src,
            "traffic": NCU_X2_KERNEL_DRAM / NCU_X2_PRODUCTS * P,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the product kernel "
                              "(fast_x2_kernel, symmetric form) on the 30^3 case (bench.py --profile: 1.28 GB for "
                              "18.57 G reference product terms), scaled by this call's product terms",
            "kernel": "fast_x2_kernel (symmetric form: columns k >= i), one ELLPACK X^2 on the SP2 iterate of "
                      "iteration %d; kernel_seconds by CUDA events around it on the library stream" % (SP2_ITERS - 1),
            "kernel_seconds": t_k, "x2_call_seconds": t_call, "symmetric_form": bool(symmetric),
            "nnz_x": int(nnz_x), "nnz_x2": int(nnz_x2), "products_reference": P,
            "products_formed": int(formed), "products_formed_share": frac_formed,
            "reference_products_per_s": P / t_call,
            "fp64_gflops_formed": 2.0 * formed / t_k / 1e9,
            "compute_frac": 2.0 * formed / t_k / 1e12 / (FP64_NOMINAL_TFLOPS / 2),
            "compute_frac_of": "nominal FP64 %.0f TFLOP/s halved (each product is a multiply and a separate "
                               "atomic add)" % FP64_NOMINAL_TFLOPS,
            "busiest_unit": {"unit": "L1/shared-memory pipe (l1tex__throughput)", "busy_pct": 92.6,
                             "shared_atomic_wavefronts_share": 0.59, "l2_pct": 23.5, "dram_pct_of_elapsed": None,
                             "source": "ncu --set full of fast_x2_kernel on the 30^3 case (bench.py --profile): the "
                                       "kernel is bound by its shared-memory atomic adds (59% of the shared "
                                       "wavefronts), neither by HBM bytes nor by FP64 flops"},
            "gathered_gbs": 12.0 * formed / t_k / 1e9}


# ---------------------------------------------------------------------------
# reference (CPU) arm and the CPU baseline
# ---------------------------------------------------------------------------
def _omp_env():
    ncpu = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncpu))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    os.environ.setdefault("OMP_STACKSIZE", "64M")
    return int(os.environ["OMP_NUM_THREADS"])


def ref_sp2(O, H, D, X2, iters):
    """The SP2 loop of bml_b200_sp2, on the reference library."""
    lib = O.ref()
    lib.bml_copy(H, D)
    b = lib.bml_gershgorin(H)
    bb = (C.c_double * 2).from_address(b)
    emin, emax = bb[0], bb[1]
    lib.bml_free_memory(b)
    lib.bml_normalize(D, emin, emax)
    for _ in range(iters):
        tr = O.ref_x2(D, X2, THRESHOLD)
        if abs(tr[1] - OCC) <= abs(2 * tr[0] - tr[1] - OCC):
            lib.bml_copy(X2, D)
        else:
            lib.bml_add(D, X2, 2.0, -1.0, THRESHOLD)
    return tr


def _ref_setup():
    threads = _omp_env()
    from oracle import oracle as O
    if not O.available():
        raise RuntimeError("oracle/_ref is not built")
    import numpy as np
    # the oracle's own copy of the seeded generator: this process never loads
    # the library under test
    v, ix, nz = O.gen_lattice(L, RADIUS, N, M_H, SEED)
    # the reference copies whole padded rows: H and the iterates share M
    pad = lambda a: np.pad(a.reshape(N, M_H), ((0, 0), (0, M_X - M_H))).reshape(-1)
    H = O.ref_ellpack(pad(v), pad(ix), nz, N, M_X)
    D = O.ref().bml_zero_matrix(2, 2, N, M_X, 0)
    X2 = O.ref().bml_zero_matrix(2, 2, N, M_X, 0)
    return O, H, D, X2, threads


def cpu_baseline():
    O, H, D, X2, threads = _ref_setup()
    t0 = time.perf_counter()
    ref_sp2(O, H, D, X2, SP2_ITERS)
    dt = time.perf_counter() - t0
    return {"value": dt, "unit": "s", "cores": threads, "kind": "reference",
            "sample": "one full step (SP2 from H, %d iterations) on the reference bml ELLPACK "
                      "OpenMP CPU path, built -O3 -std=c99 -fopenmp from its sources" % SP2_ITERS}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    O, H, D, X2, threads = _ref_setup()
    warm, steps = args.warmup, args.steps
    for _ in range(warm):
        ref_sp2(O, H, D, X2, SP2_ITERS)
    t0 = time.perf_counter()
    for _ in range(steps):
        ref_sp2(O, H, D, X2, SP2_ITERS)
    dt = (time.perf_counter() - t0) / steps
    sample = ("%d timed step(s) after %d warm-up, each a full SP2 run from H (%d iterations), reference "
              "bml ELLPACK OpenMP CPU path on %d threads" % (steps, warm, SP2_ITERS, threads))
    return {"impl": "reference", "metric": METRIC, "value": dt, "unit": "s", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": dt * 1e3, "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded splitmix64 lattice Hamiltonian)",
            "config": bench_config(world, args.exchange),
            "cpu_baseline": {"value": dt, "unit": "s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": dt, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_profile_case():
    """A case small enough for an ncu capture (about 3 GB on the device):
    the 30^3 lattice (N=27000), three SP2 iterations, then one more X^2 whose
    kernels are the ones to capture (skip the launches of the first three)."""
    import bml_b200 as B
    Lp = 30
    Np = Lp ** 3
    v, ix, nz = B.gen_lattice(Lp, RADIUS, Np, M_H, SEED)
    H = B.Ellpack.from_arrays(v, ix, nz, Np, M_H)
    D = B.Ellpack(Np, M_X)
    info = (C.c_double * 6)()
    B.check(B.lib.bml_b200_sp2(H.h, D.h, THRESHOLD, Np / 2.0, 3, 1e-8, 0, info))
    X2 = B.Ellpack(Np, M_X)
    tr = (C.c_double * 2)()
    B.check(B.lib.bml_b200_multiply_x2(D.h, X2.h, THRESHOLD, tr))
    print(json.dumps({"profile_case": "30^3 lattice, X^2 after 3 SP2 iterations", "trace": list(tr),
                      "tiers": B.last_tier_counts(), "width": B.lib.bml_b200_last_required_M(),
                      "products": products(D, Np), "nnz_x": B.lib.bml_b200_nnz(D.h),
                      "nnz_x2": B.lib.bml_b200_nnz(X2.h)}))


def run_profile_ops():
    """The one-pass ELLPACK operations, each launched once, on matrices larger
    than L2: X = the SP2 iterate after 3 iterations on the 30^3 lattice
    (N = 27000, threshold 1e-5, as in --profile) and X2 = X^2.  The SP2 start
    and iterations launch gershgorin, scale, copy (3), add (1) and diag (1)
    kernels first; the operations below follow, in the order written.
    Prints the entry counts from which each operation's compulsory bytes
    follow."""
    import bml_b200 as B
    Lp, Mp = 30, M_X
    Np = Lp ** 3
    v, ix, nz = B.gen_lattice(Lp, RADIUS, Np, M_H, SEED)
    H = B.Ellpack.from_arrays(v, ix, nz, Np, M_H)
    X = B.Ellpack(Np, Mp)
    info = (C.c_double * 6)()
    B.check(B.lib.bml_b200_sp2(H.h, X.h, THRESHOLD, Np / 2.0, 3, 1e-8, 0, info))
    X2 = B.Ellpack(Np, Mp)
    tr = (C.c_double * 2)()
    B.check(B.lib.bml_b200_multiply_x2(X.h, X2.h, THRESHOLD, tr))
    nnz = lambda m: int(B.lib.bml_b200_nnz(m.h))
    n_x, n_x2 = nnz(X), nnz(X2)
    # the operations, in launch order, inside an NVTX range "ops" (ncu
    # --nvtx --nvtx-include "ops/" captures only these)
    nvtx = _nvtx()
    nvtx.range_push("ops")
    S = B.Ellpack(Np, Mp)
    B.lib.bml_copy(X.h, S.h)                       # copy_kernel: X -> S
    B.lib.bml_add(S.h, X2.h, 2.0, -1.0, THRESHOLD)  # add_kernel: S = 2 S - X2
    n_add = nnz(S)
    T = B.Ellpack(Np, Mp)
    B.lib.bml_copy(X2.h, T.h)                      # copy_kernel: X2 -> T
    B.lib.bml_threshold(T.h, 1e-4)                 # threshold_kernel, in place
    n_thr = nnz(T)
    alpha = C.c_double(0.5)
    B.lib.bml_scale_inplace(C.byref(alpha), X2.h)  # scale_kernel on X2
    trace = B.lib.bml_trace(X2.h)                  # diag_kernel
    eb = B.lib.bml_gershgorin(X2.h)                # gershgorin_kernel
    B.lib.bml_free_memory(eb)
    Xt = B.lib.bml_transpose_new(X2.h)             # transpose_scatter_kernel + row_sort_kernel
    B.check()
    nvtx.range_pop()
    hh = C.c_void_p(Xt)
    B.lib.bml_deallocate(C.byref(hh))
    print(json.dumps({"profile_case": "one-pass ELLPACK operations on the 30^3 lattice's SP2 iterate X and X^2",
                      "N": Np, "M": Mp, "nnz_x": n_x, "nnz_x2": n_x2, "nnz_add": n_add, "nnz_threshold": n_thr,
                      "trace": trace}))


def _nvtx():
    """NVTX range markers (torch's bindings), for the ncu captures of the
    profile cases; no-ops where torch has none."""
    try:
        import torch
        return torch.cuda.nvtx
    except (ImportError, AttributeError):
        class _Nop:
            def range_push(self, _):
                pass

            def range_pop(self):
                pass
        return _Nop()


class _StdoutToStderr:
    """Route the process's stdout (fd 1) to stderr while the library prints
    its partition messages (bml_set_block_sizes prints, as the reference
    does), so that stdout keeps exactly one JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        C.CDLL(None).fflush(None)
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        C.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def ellblock_case(L):
    """H on the L^3 block lattice of 32x32 blocks (radius 2, N(0,1) exp(-d)
    entries, seed 0) with MB = 257 (room for X^2's radius-4 block rows)."""
    import bml_b200 as B
    nb = L ** 3
    arr = (C.c_int * nb)(*([32] * nb))
    with _StdoutToStderr():
        B.lib.bml_b200_reset_block_sizes()
        B.lib.bml_set_block_sizes(arr, nb, 257)
        H = B.lib.bml_b200_gen_block_lattice(L, 2.0, 32, SEED, 2)
    B.check()
    return H, nb * 32


def run_profile_tc(wide=False, split=0):
    """Three tensor-core X^2 calls on the 10^3 block lattice (N = 32000): of
    H, or (wide) of X1, the iterate after one exact SP2 iteration from H
    (the product of the second SP2 iteration); the three calls run inside the
    NVTX range "tc"."""
    import bml_b200 as B
    B.lib.bml_b200_set_tc_split(split)
    H, n = ellblock_case(10)
    X = H
    if wide:
        X = B.lib.bml_zero_matrix(3, 2, n, n, 0)
        info = (C.c_double * 8)()
        B.check()
        B.check(B.lib.bml_b200_ellblock_sp2_mixed(H, X, 1e-6, n / 2.0, 1, -1.0, 0, 1, info))
    X2 = B.lib.bml_zero_matrix(3, 2, n, n, 0)
    tr = (C.c_double * 2)()
    B.check(B.lib.bml_b200_synchronize())
    nvtx = _nvtx()
    nvtx.range_push("tc")
    for _ in range(3):
        B.check(B.lib.bml_b200_ellblock_multiply_x2_tc(X, X2, 1e-6, tr))
    B.check(B.lib.bml_b200_synchronize())
    nvtx.range_pop()
    print(json.dumps({"profile_case": "10^3 block lattice, tensor-core X^2 of %s" % ("the SP2 iterate X1" if wide else "H"),
                      "trace": list(tr), "blocks_x": int(B.lib.bml_b200_nnz(X)) // 1024,
                      "blocks_x2": int(B.lib.bml_b200_nnz(X2)) // 1024}))


def run_profile_eb_sp2(iters=5, nclose=1):
    """The mixed ELLBLOCK SP2 of the ellblock_sp2 leg's mixed_8bit_close1
    entry (16^3 block lattice, the 8-bit split for the bulk iterations, one
    closing FP64 iteration), once to size the device memory, then once
    inside the NVTX range "sp2"; prints its device time, the trace and the
    number of tensor-core iterations."""
    import bml_b200 as B
    H, n = ellblock_case(16)
    old = B.lib.bml_b200_set_tc_split(1)
    nvtx = _nvtx()
    for timed in (False, True):
        D = B.lib.bml_zero_matrix(3, 2, n, n, 0)
        B.check()
        info = (C.c_double * 8)()
        B.check(B.lib.bml_b200_synchronize())
        if timed:
            nvtx.range_push("sp2")
        B.check(B.lib.bml_b200_event_record(6))
        B.check(B.lib.bml_b200_ellblock_sp2_mixed(H, D, 1e-6, n / 2.0, iters, -1.0, 0, nclose, info))
        B.check(B.lib.bml_b200_event_record(7))
        B.check(B.lib.bml_b200_synchronize())
        if timed:
            nvtx.range_pop()
            print(json.dumps({"profile_case": "mixed ELLBLOCK SP2, 16^3 block lattice, %d iterations, 8-bit split, "
                                              "%d closing FP64" % (iters, nclose),
                              "s": B.event_ms(6, 7) / 1e3, "trace": B.lib.bml_trace(D),
                              "tc_iterations": int(info[6])}))
        hh = C.c_void_p(D)
        B.lib.bml_deallocate(C.byref(hh))
    B.lib.bml_b200_set_tc_split(old)


def block_lattice_products(L, radius):
    """Block products of X^2 on the L^3 block lattice: the (ib, jb, kb)
    triples, sum over ib and its neighbours jb of jb's neighbour count."""
    import itertools
    import numpy as np
    r = int(radius)
    offs = [o for o in itertools.product(range(-r, r + 1), repeat=3) if sum(x * x for x in o) <= radius ** 2 + 1e-9]
    pos = np.array([(x, y, z) for z in range(L) for y in range(L) for x in range(L)])
    deg = np.zeros(L ** 3, np.int64)
    for o in offs:
        deg += np.all((pos + o >= 0) & (pos + o < L), axis=1)
    total = 0
    for o in offs:
        q = pos + o
        ok = np.all((q >= 0) & (q < L), axis=1)
        q = q[ok]
        total += int(deg[q[:, 0] + L * q[:, 1] + L * L * q[:, 2]].sum())
    return total


def run_profile_eb():
    """Three exact FP64 X^2 calls on the 10^3 block lattice (N = 32000)."""
    import bml_b200 as B
    H, n = ellblock_case(10)
    X2 = B.lib.bml_zero_matrix(3, 2, n, n, 0)
    B.check()
    for _ in range(3):
        B.lib.bml_free_memory(C.c_void_p(B.lib.bml_multiply_x2(H, X2, C.c_double(1e-6))))
        B.check()
    print(json.dumps({"profile_case": "10^3 block lattice, exact FP64 X^2", "trace": B.lib.bml_trace(X2)}))


def run_profile_eb_ops(L=7):
    """The one-pass ELLBLOCK operations, each launched once, on the L^3 block
    lattice (radius 2, MB = 257; L = 7: 343 block rows of 32x32, N = 10976):
    H, and X2 = H^2 (exact, threshold 1e-6), at L = 7 about 280 MB of blocks,
    larger than L2.  Prints the block counts from which each operation's
    compulsory bytes follow."""
    import bml_b200 as B
    H, n = ellblock_case(L)
    X2 = B.lib.bml_zero_matrix(3, 2, n, n, 0)
    S = B.lib.bml_zero_matrix(3, 2, n, n, 0)
    T = B.lib.bml_zero_matrix(3, 2, n, n, 0)
    B.check()
    B.lib.bml_free_memory(C.c_void_p(B.lib.bml_multiply_x2(H, X2, C.c_double(1e-6))))
    B.check()
    blocks = lambda h: int(B.lib.bml_b200_nnz(h)) // 1024
    n_h, n_x2 = blocks(H), blocks(X2)
    # the operations, in launch order, inside an NVTX range "ops"
    nvtx = _nvtx()
    nvtx.range_push("ops")
    B.lib.bml_copy(X2, S)                                   # eb_copy_kernel: X2 -> S
    B.lib.bml_add(S, H, C.c_double(2.0), C.c_double(-1.0), C.c_double(1e-6))  # eb_add_kernel: S = 2 S - H
    n_add = blocks(S)
    B.lib.bml_copy(X2, T)                                   # eb_copy_kernel: X2 -> T
    B.lib.bml_threshold(T, C.c_double(1e-1))                # eb_threshold_kernel, in place
    n_thr = blocks(T)
    alpha = C.c_double(0.5)
    B.lib.bml_scale_inplace(C.byref(alpha), X2)             # eb_scale_kernel on X2
    trace = B.lib.bml_trace(X2)                             # eb_diag_kernel
    eb = B.lib.bml_gershgorin(X2)                           # eb_gersh_kernel
    B.lib.bml_free_memory(eb)
    Xt = B.lib.bml_transpose_new(X2)                        # eb_transpose_kernel
    tm = B.lib.bml_trace_mult(X2, H)                        # eb_trace_mult_kernel
    B.check()
    nvtx.range_pop()
    for h in (X2, S, T, Xt, H):
        hh = C.c_void_p(h)
        B.lib.bml_deallocate(C.byref(hh))
    B.lib.bml_b200_reset_block_sizes()
    print(json.dumps({"profile_case": "one-pass ELLBLOCK operations on the %d^3 block lattice's H and H^2" % L,
                      "N": n, "blocks_h": n_h, "blocks_x2": n_x2, "blocks_add": n_add, "blocks_threshold": n_thr,
                      "trace": trace, "trace_mult": tm}))


def ellblock_sp2_leg(iters=5, nclose=2):
    """The mixed ELLBLOCK SP2 configuration on the 16^3 block lattice (4096
    block rows of 32, N = 131072, threshold 1e-6, occupation N/2): the first
    `iters` iterations from X0, every X^2 in FP64 against bulk X^2 on the
    tensor cores and the last `nclose` in FP64, with their errors, for both
    splits of the tensor-core X^2 (FP16 hi/lo with FP32 accumulation, and
    8-bit slices with exact INT32 accumulation); the 8-bit split also with a
    single closing FP64 iteration, which its exact accumulation allows at
    the same error target.  Device time by CUDA events on the library
    stream."""
    import bml_b200 as B
    H, n = ellblock_case(16)
    # warm-up: the exact and tensor-core X^2 size their device scratch once
    W = B.lib.bml_zero_matrix(3, 2, n, n, 0)
    B.check()
    B.lib.bml_free_memory(C.c_void_p(B.lib.bml_multiply_x2(H, W, C.c_double(1e-6))))
    B.check(B.lib.bml_b200_ellblock_multiply_x2_tc(H, W, 1e-6, None))
    hh = C.c_void_p(W)
    B.lib.bml_deallocate(C.byref(hh))
    out = {}
    old_split = B.lib.bml_b200_set_tc_split(0)
    for name, nc, split in (("fp64", iters, 0), ("mixed", nclose, 0), ("mixed_8bit", nclose, 1),
                            ("mixed_8bit_close1", 1, 1)):
        D = B.lib.bml_zero_matrix(3, 2, n, n, 0)
        B.check()
        info = (C.c_double * 8)()
        B.lib.bml_b200_set_tc_split(split)
        if split:  # size the 8-bit split's scratch outside the timed call
            Wm = B.lib.bml_zero_matrix(3, 2, n, n, 0)
            B.check(B.lib.bml_b200_ellblock_multiply_x2_tc(H, Wm, 1e-6, None))
            hh = C.c_void_p(Wm)
            B.lib.bml_deallocate(C.byref(hh))
        with _StdoutToStderr():
            B.check(B.lib.bml_b200_synchronize())
            B.check(B.lib.bml_b200_event_record(6))
            B.check(B.lib.bml_b200_ellblock_sp2_mixed(H, D, 1e-6, n / 2.0, iters, -1.0, 0, nc, info))
            B.check(B.lib.bml_b200_event_record(7))
        t = B.event_ms(6, 7) / 1e3
        out[name] = {"s": t, "trace": B.lib.bml_trace(D), "energy_trDH": B.lib.bml_trace_mult(D, H),
                     "idempotency_t_minus_t2": info[3], "tc_iterations": int(info[6]), "nnz": int(B.lib.bml_b200_nnz(D))}
        hh = C.c_void_p(D)
        B.lib.bml_deallocate(C.byref(hh))
    B.lib.bml_b200_set_tc_split(old_split)
    hh = C.c_void_p(H)
    B.lib.bml_deallocate(C.byref(hh))
    B.lib.bml_b200_reset_block_sizes()
    e, m, m8, m81 = out["fp64"], out["mixed"], out["mixed_8bit"], out["mixed_8bit_close1"]
    rel = lambda a, b: abs(a - b) / abs(b)
    for x, nc in ((m8, nclose), (m81, 1)):
        x.update({"speedup": e["s"] / x["s"], "trace_rel_err": rel(x["trace"], e["trace"]),
                  "energy_rel_err": rel(x["energy_trDH"], e["energy_trDH"]), "closing_fp64": nc,
                  "split": "8-bit slices (5 per entry), exact INT32 accumulation, FP64 recombination"})
    return {"workload": "SP2 on the 16^3 block lattice Hamiltonian (4096 block rows of 32x32, N=131072, radius 2, "
                        "thr 1e-6, occ N/2), first %d iterations from X0" % iters,
            "iterations": iters, "closing_fp64": nclose, "fp64": e, "mixed": m, "speedup": e["s"] / m["s"],
            "trace_rel_err": rel(m["trace"], e["trace"]),
            "energy_rel_err": rel(m["energy_trDH"], e["energy_trDH"]),
            "mixed_8bit": m8, "mixed_8bit_close1": m81,
            "note": "bulk X^2 on the tensor cores (mixed: FP16 hi/lo split, FP32 accumulation; mixed_8bit: "
                    "8-bit slices, exact INT32 accumulation), the closing iterations on the FP64 block product"}


def ellblock_leg(reps=3):
    """The mixed ELLBLOCK configuration's product: X^2 of H on the 16^3 block
    lattice (4096 block rows of 32, N = 131072, threshold 1e-6), on the
    tensor cores (scaled FP16 hi/lo split) against the FP64 block product, device
    times by CUDA events and the tensor-core result's trace error."""
    import bml_b200 as B
    H, n = ellblock_case(16)
    Xe = B.lib.bml_zero_matrix(3, 2, n, n, 0)
    Xt = B.lib.bml_zero_matrix(3, 2, n, n, 0)
    B.check()
    tr = (C.c_double * 2)()

    def timed(fn):
        fn()
        B.check(B.lib.bml_b200_synchronize())
        B.check(B.lib.bml_b200_event_record(6))
        for _ in range(reps):
            fn()
        B.check(B.lib.bml_b200_event_record(7))
        return B.event_ms(6, 7) / 1e3 / reps

    def exact():
        p = B.lib.bml_multiply_x2(H, Xe, C.c_double(1e-6))
        B.lib.bml_free_memory(C.c_void_p(p))
        B.check()

    te = timed(exact)
    old_split = B.lib.bml_b200_set_tc_split(1)
    t8 = timed(lambda: B.check(B.lib.bml_b200_ellblock_multiply_x2_tc(H, Xt, 1e-6, tr)))
    tr8 = B.lib.bml_trace(Xt)
    B.lib.bml_b200_set_tc_split(0)
    tt = timed(lambda: B.check(B.lib.bml_b200_ellblock_multiply_x2_tc(H, Xt, 1e-6, tr)))
    B.lib.bml_b200_set_tc_split(old_split)
    tre, trt = B.lib.bml_trace(Xe), B.lib.bml_trace(Xt)
    nnz_h = B.lib.bml_b200_nnz(H)
    P = block_lattice_products(16, 2.0)
    flops = 2.0 * 32 ** 3 * P
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    tc_peak = peaks.get("bf16_tflops") or 1590.0
    res = {"workload": "X^2 of H, 16^3 block lattice, 4096 block rows of 32x32 (N=131072), radius 2, thr 1e-6",
           "tc_s": tt, "fp64_s": te, "speedup": te / tt, "trace_rel_err": abs(trt - tre) / abs(tre),
           "tc_8bit_s": t8, "tc_8bit_trace_rel_err": abs(tr8 - tre) / abs(tre),
           "nnz_h": int(nnz_h), "nnz_x2": int(B.lib.bml_b200_nnz(Xt)), "block_products": P,
           "fp64_tflops": flops / te / 1e12,
           "fp64_ceiling_tflops": FP64_NOMINAL_TFLOPS,
           "fp64_ceiling": "nominal B200 FP64 %.0f TFLOP/s: the library's default (unordered) form sums each "
                           "block product by fused multiply-adds; the ordered form (bml_b200_set_x2_exact(1)) "
                           "rounds every multiply and add separately, as the reference, at half that "
                           "ceiling" % FP64_NOMINAL_TFLOPS,
           "tc_tflops": 3 * flops / tt / 1e12, "tc_peak_tflops": tc_peak,
           "tc_tflops_note": "three block products (hi*hi, hi*lo, lo*hi) per block pair over the measured "
                             "dense bf16 peak (f16 runs at the same rate)",
           "method": "tcgen05 kind::f16, FP16 hi*hi + hi*lo + lo*hi of X scaled by 2^s, FP32 accumulation in TMEM"}
    for h in (H, Xe, Xt):
        hh = C.c_void_p(h)
        B.lib.bml_deallocate(C.byref(hh))
    B.lib.bml_b200_reset_block_sizes()
    return res


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.profile:
        run_profile_case()
        return
    if args.profile_eb_sp2:
        run_profile_eb_sp2()
        return
    if args.profile_tc or args.profile_tc_wide:
        run_profile_tc(wide=args.profile_tc_wide, split=args.tc_split)
        return
    if args.profile_ops:
        run_profile_ops()
        return
    if args.profile_eb:
        run_profile_eb()
        return
    if args.profile_eb_ops:
        run_profile_eb_ops(args.eb_ops_L)
        return
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    else:
        res = run_b200(args, rank, world, local)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
