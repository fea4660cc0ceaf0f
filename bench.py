#!/usr/bin/env python
"""Benchmark: factor + batched solve of the 1024^2 2D Helmholtz HPS problem on B200, mixed precision
against FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision mixed|fp64]
    python bench.py --serve [--requests R]
    python bench.py --forest | --three-d
    python bench.py --gemm fp64|tf32x3|int8 [--gemm-shape m,n,k,count]   (one GEMM engine alone)

One step = the reference's hot path on one batch: robin_tree%factor of the 1024^2, L=12 tree
(16x16 leaves, kb=200, seeded 100-bump potential with 0.002i*kb damping) followed by one batched
solve of its 32 seeded plane-wave right-hand sides and get_solution.  ``value`` is right-hand
sides per second with the factorization inside every step, so it moves with both factor time
and solve throughput.  Three arms run on the same inputs in the same run: the plain FP64 path
(the headline arm, ``value``, the reference's precision), the mixed-precision path (``mixed``:
RB_PREC_MIXED, the B1, Y1, Y2 and parent-map GEMMs of merge levels 2-4 on the tcgen05 tensor
cores in int8 digit slices with exact integer accumulation, FP64 elsewhere including the top two
levels, every solve refined to 1e-10 against the FP64 residual), and ``mixed_int8_top``, the
same with the top two levels' GEMMs on the int8 engine too (RB_FLAG_MIXED_INT8_TOP; their
inversions stay FP64), each with its factor, solve and step ratios against FP64
(``mixed_vs_fp64``, ``mixed_int8_top_vs_fp64``).  ``--precision mixed`` makes the mixed arm the
headline.

* value:  device-resident inputs (rb_tree_factor_device / rb_tree_solve_device /
          rb_get_solution_device), CUDA events on the library's stream, max over ranks.
* e2e:    the same steps through the host C-ABI calls a user makes (rb_tree_factor,
          rb_tree_solve, rb_get_solution_async per RHS, rb_tree_sync after the last step) from
          pinned host buffers: H2D of the potential and right-hand sides and D2H of every
          solution inside the timed region, each step's read-back beside the next step's factor.
          The plane waves' interior sources are zero and go in as f_centres = NULL (the library
          zeroes its source array on the device; the kernels are the same).
* accuracy: mixed against FP64 GPU on every right-hand side; both against an FP64 CPU solve of
          the same global FD system (SuperLU, run in a spawned process beside the GPU work) for
          the first and last right-hand side; the normwise backward error of the e2e solutions.
* roofline: per-launch CUDA events over a second pass of the same steps give the dominant
          kernel family's algorithmic flops / time, against the peak of the pipe it runs on: the
          complex128 cuBLAS GEMM measured in this run (FP64 kernels; MEASURED_PEAKS.json has no
          FP64 entry) or, for the tcgen05 kernel, MEASURED_PEAKS.json's bf16 rate x 2 (int8) / 15
          (int8 operations per algorithmic flop of the digit-slice product; split TF32: / 2 / 3).
* cpu_baseline / --impl reference: the reference's LAPACK/BLAS call sequence (oracle port, scipy
          OpenBLAS, all host threads) MEASURED on the whole workload: the full factor (every leaf
          and merge) and a few single-RHS solves (the reference solves one right-hand side per
          call); RHS/s = nrhs / (factor + nrhs x mean solve).  The reference arm cuts that one
          pass into K consecutive measured steps.
* --serve: the serving loop (rb_server_*): 8 resident trees (grids 256^2..1024^2, kb 50..200), a
          Poisson stream of device-sampled point-source / plane-wave solve requests (1-64 RHS)
          with 20 refactors, at 0.5x and 0.9x of the measured saturated rate; p50/p99 latency
          from arrival to solution in host memory, mixed and FP64 servers.
Multi-GPU: replicas only (every rank factors and solves its own copy of the problem); the only
collective is the max-reduction of the timings.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Factor time + solves/s on 1024² 2D Helmholtz, mixed vs FP64 GPU @1e-10; p99 ms"

# DRAM bytes (read + write) per algorithmic flop of the contiguous-k FP64 tensor-core GEMM
# ("zgemm_tc"), from an ncu capture of dram__bytes_read.sum + dram__bytes_write.sum over two full
# factors of the 512^2, L=10 workload (--config 2 --single-arm): 0.76 GB for 71.2 GFLOP.  ncu cannot
# run inside this script, and a capture of that kind on the 1024^2 workload would be too large, so
# the ratio is carried here and scaled to the timed launches by their flops.  The tile reads each
# operand panel once per output tile, so its traffic grows with the flops at a fixed tile shape.
DRAM_BYTES_PER_FLOP = {"zgemm_tc": 0.0107}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nrhs", type=int, default=None, help="right-hand sides per step (default: the config's)")
    ap.add_argument("--config", type=int, default=4, choices=[1, 2, 4],
                    help="workload: 4 = 1024^2 L=12 (the headline), 2 = 512^2 L=10, 1 = 64^2 L=4 (profiling/tests)")
    ap.add_argument("--precision", default="fp64", choices=["mixed", "fp64"],
                    help="the headline arm (value, e2e, roofline); the other precision is timed beside it")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forward-error", action="store_true")
    ap.add_argument("--single-arm", action="store_true",
                    help="time the headline precision only (no second arm, no mixed-vs-FP64 block): "
                         "a launch list of the headline step alone")
    ap.add_argument("--serve", action="store_true",
                    help="serving bench: 8 resident trees, Poisson solve stream at 0.5x and 0.9x of saturation")
    ap.add_argument("--requests", type=int, default=4000, help="solve requests per offered load (--serve)")
    ap.add_argument("--forest", action="store_true",
                    help="batching bench: 64 trees of uneven sizes factored as one forest vs one at a time")
    ap.add_argument("--gemm", default=None, choices=["fp64", "tf32x3", "int8"],
                    help="one batched complex GEMM on one engine (the FP64 tiles, or the tcgen05 kernel in split "
                         "TF32 or int8 digit slices): device time per launch and algorithmic TFLOP/s; "
                         "--gemm-shape m,n,k,count")
    ap.add_argument("--gemm-shape", default="2048,2048,512,4")
    ap.add_argument("--three-d", action="store_true",
                    help="3D bench: factor and 8-RHS solve of the unit cube at 16^3 (L=6) and 32^3 (L=9), "
                         "4^3 leaves, with the manufactured solution's error")
    return ap.parse_args()


WORKLOAD_TEXT = {
    4: "2D Helmholtz 1024^2, L=12 (4096 leaves of 16x16), kb=200, 100-bump potential, 0.002i*kb damping",
    2: "2D Helmholtz 512^2, L=10 (1024 leaves of 16x16), kb=100, 40-bump potential, 0.005i*kb damping",
    1: "2D Helmholtz 64^2, L=4 (16 leaves of 16x16), kb=20, 5-bump potential, 0.01i*kb damping",
}


def config_dict(cfg, nrhs, precision):
    from robinsolver_b200 import workloads as W
    c = W.CONFIGS[cfg]
    solve = "RHS batched solve" if precision == "fp64" else \
        "RHS batched solve refined to 1e-10 against the FP64 residual"
    return {
        "workload": f"{WORKLOAD_TEXT[cfg]}, impedance boundary; per step: factor ({precision}) + {nrhs} "
                    f"{'plane-wave' if cfg == 4 else 'point-source/plane-wave'} {solve} + get_solution",
        "grid": c["N"], "L": c["L"], "leaf": "16x16", "nrhs": nrhs, "precision": precision,
        "l2": "no flush: per-step working set and inputs larger than L2 (126 MB)" if cfg != 1
              else "small case: fits in L2",
    }


# ------------------------------------------------------------------------------------------------
# CPU baseline: the reference's LAPACK/BLAS call sequence, run on the whole workload
# ------------------------------------------------------------------------------------------------

def _oracle_tree(wl):
    from oracle import hps_ref as H
    T = H.RobinTree()
    T.bndry_params = wl.bndry_params
    T.nlvls = wl.L
    T.ell_op = H.EllipticOperator(2, wl.domain, wl.potential)
    T.opts = H.SolveOpts(h_tgt=wl.h_tgt, kb=wl.opts_kb)
    T.root, T.levels = H.build_tree(wl.L, np.asarray(wl.domain, dtype=np.float64), 2)
    T.keep_leaf = True
    return T


def reference_items(wl, nsolves):
    """The reference's call sequence on the whole workload as a list of work items: every leaf
    and merge of robin_tree%factor in compute_RTR's post order, then nsolves robin_tree%solve
    calls of one right-hand side each (the reference solves one per call).  Returns the oracle
    tree and the items; run_item executes one."""
    T = _oracle_tree(wl)
    order = []

    def post(n):
        if n.isleaf:
            order.append(("leaf", n))
        else:
            post(n.child1)
            post(n.child2)
            order.append(("merge", n))
    post(T.root)
    order += [("solve", r) for r in range(nsolves)]
    return T, order


def run_item(T, wl, item):
    from oracle import hps_ref as H
    kind, x = item
    if kind == "leaf":
        T._leaf(x)
    elif kind == "merge":
        T._merge(x)
        if x is T.root:
            T.factored = True
    else:
        r = wl.rhs[x % len(wl.rhs)]
        T.solve([H.EllipticRHS(2, r.f, r.g)])


def timed_items(T, wl, items):
    """(LAPACK/BLAS seconds, wall seconds) of a run of items.  The Python index loops of the
    restatement are compiled loops in the reference, so the LAPACK/BLAS time is its CPU cost."""
    from oracle import hps_ref as H
    prof = [0.0, 0]
    H.PROFILE = prof
    t0 = time.perf_counter()
    try:
        for it in items:
            run_item(T, wl, it)
    finally:
        H.PROFILE = None
    return prof[0], time.perf_counter() - t0


def cpu_full_pass(wl, nrhs, nsolves, chunks=1, on_chunk=None):
    """The full factor plus nsolves single-RHS solves, measured (not extrapolated), in `chunks`
    consecutive slices of the item list.  Returns per-chunk (lapack_s, wall_s) and the factor and
    mean solve times."""
    T, items = reference_items(wl, nsolves)
    nf = len(items) - nsolves
    per = [(0.0, 0.0)] * chunks
    fac = sol = 0.0
    walls = 0.0
    bounds = np.linspace(0, len(items), chunks + 1).astype(int)
    for c in range(chunks):
        lo, hi = bounds[c], bounds[c + 1]
        lap_f = lap_s = 0.0
        wall = 0.0
        # split the chunk at the factor/solve boundary to attribute the time
        for a, b in ((lo, min(hi, nf)), (max(lo, nf), hi)):
            if b > a:
                lp, wl_s = timed_items(T, wl, items[a:b])
                wall += wl_s
                if a < nf:
                    lap_f += lp
                else:
                    lap_s += lp
        fac += lap_f
        sol += lap_s
        walls += wall
        per[c] = (lap_f + lap_s, wall)
        if on_chunk:
            on_chunk(c)
    return per, fac, sol / max(nsolves, 1), walls


def cpu_sample_threads(wl, threads):
    """LAPACK/BLAS seconds of a fixed sample (16 leaves, the deepest merge whose interface has
    256 points with children given random maps of the true sizes, one leaf solve) at a given
    thread count: the CPU's own thread scaling on this workload's kernels."""
    from threadpoolctl import threadpool_limits
    from oracle import hps_ref as H
    with threadpool_limits(limits=threads):
        T = _oracle_tree(wl)
        leaves = T.levels[-1][:16]
        lap, _ = timed_items(T, wl, [("leaf", n) for n in leaves])
        rng = np.random.default_rng(7)
        for l in range(wl.L - 1, -1, -1):
            node = T.levels[l][0]
            kids = (node.child1, node.child2)
            grids = [tuple(int(round(w * wl.N)) for w in (c.box[1] - c.box[0])[:2]) for c in kids]
            cut = int(np.argmax(np.abs((node.box[1] - node.box[0]) - (kids[0].box[1] - kids[0].box[0]))[:2]))
            if grids[0][1 - cut] >= 256:
                break
        for c, (ga, gb) in zip(kids, grids):
            c.ptbox = [ga, gb, -1]
            nbc = 2 * (ga + gb)
            c.rtr = np.asfortranarray((rng.standard_normal((nbc, nbc)) + 1j * rng.standard_normal((nbc, nbc)))
                                      / np.sqrt(2.0 * nbc))
        prof = [0.0, 0]
        H.PROFILE = prof
        try:
            T._merge(node)
            lf = leaves[0]
            b = np.zeros((lf.lu.shape[0], 1), dtype=np.complex128, order="F")
            H._getrs((lf.lu, lf.piv), b)
        finally:
            H.PROFILE = None
    return lap + prof[0]


def cpu_model():
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def cpu_baseline_block(wl, nrhs, nsolves=2):
    threads = os.cpu_count() or 1
    per, fac, sol, wall = cpu_full_pass(wl, nrhs, nsolves)
    step = fac + nrhs * sol
    t1 = cpu_sample_threads(wl, 1)
    tn = cpu_sample_threads(wl, threads)
    return {
        "value": nrhs / step, "unit": "RHS/s", "cores": threads, "kind": "port",
        "cpu": cpu_model(), "factor_s": fac, "solve_s_per_rhs": sol, "wall_s": wall,
        "thread_scaling": {"sample_s_1_thread": t1, f"sample_s_{threads}_threads": tn, "speedup": t1 / tn},
        "sample": f"measured on the whole workload: the full factor (every leaf and merge of the reference's "
                  f"call sequence) and {nsolves} single-RHS solves, LAPACK/BLAS time (scipy OpenBLAS, {threads} "
                  f"threads; the restatement's Python loops are compiled in the reference and not counted, "
                  f"{wall:.0f} s wall); RHS/s = {nrhs} / (factor + {nrhs} x mean solve)",
    }


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from robinsolver_b200 import workloads as W
    nrhs = args.nrhs or W.CONFIGS[args.config]["nrhs"]
    wl = W.make_workload(args.config, nrhs=nrhs)
    threads = os.cpu_count() or 1
    # warm-up: the factor of config 1's small tree, W times
    small = W.make_workload(1)
    for _ in range(args.warmup):
        T, items = reference_items(small, 1)
        timed_items(T, small, items)
    # timed: ONE pass over the whole workload -- full factor + 4 single-RHS solves -- cut into
    # `steps` consecutive slices; every slice is measured
    nsolves = 4
    per, fac, sol, wall = cpu_full_pass(wl, nrhs, nsolves, chunks=args.steps)
    tot = sum(p[0] for p in per)
    value = nrhs / (fac + nrhs * sol)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "RHS/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic (seeded)",
        "config": config_dict(args.config, nrhs, "fp64"),
        "factor_ms": 1e3 * fac, "solve_ms_per_rhs": 1e3 * sol, "wall_s": wall,
        "cpu_baseline": {"value": value, "unit": "RHS/s", "cores": threads, "kind": "port", "cpu": cpu_model(),
                         "sample": f"one pass over the whole workload (full factor: every leaf and merge; then "
                                   f"{nsolves} single-RHS solves), cut into {args.steps} consecutive measured "
                                   f"steps; LAPACK/BLAS time of the reference's call sequence (scipy OpenBLAS, "
                                   f"{threads} threads); RHS/s = {nrhs} / (factor + {nrhs} x mean solve)"},
        "e2e": {"value": value, "unit": "RHS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def zgemm_peak_tflops(torch, dev):
    """complex128 cuBLAS GEMM rate (8 n^3 flops), the FP64 denominator of the roofline."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device=dev)
    b = torch.randn(n, n, dtype=torch.complex128, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 8.0 * n ** 3 / (best * 1e-3) / 1e12


def _superlu_reference(wl, kv, F, G, rows):
    """FP64 CPU solutions of the global FD system (SuperLU) for the listed right-hand sides; runs
    in a spawned process beside the GPU measurement (one host core)."""
    from oracle import fd_global as FG
    S = FG.SparseFD(wl.L, wl.domain, wl.h_tgt, wl.opts_kb, wl.bndry_params, kv)
    return [S.solve(F[r], G[r]) for r in rows]


def _start_superlu(wl_args, kv, F, G, rows):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    pool = ctx.Pool(1)
    return pool, pool.apply_async(_superlu_from_args, (wl_args, kv, F[rows], G[rows]))


def _superlu_from_args(wl_args, kv, F, G):
    sys.path.insert(0, str(ROOT))
    from robinsolver_b200 import workloads as W
    wl = W.make_workload(*wl_args[0], **wl_args[1])
    return _superlu_reference(wl, kv, F, G, range(F.shape[0]))


class Arm:
    """One tree of the bench workload at one precision, driven through the C-ABI."""

    def __init__(self, rb, _lib, wl, precision, kv, d_k, d_f, d_g, nrhs):
        self.lib = _lib.lib
        self._lib = _lib
        # "mixed_int8_top": the mixed factor with its top two levels' GEMMs on the int8 engine too
        self.precision = "mixed" if precision.startswith("mixed") else "fp64"
        self.prec = _lib.RB_PREC_MIXED if self.precision == "mixed" else _lib.RB_PREC_FP64
        # RB_FLAG_ASYNC_FACTOR: the host factor call returns once enqueued, so that the e2e step's
        # right-hand-side upload overlaps the factor (the device-path calls are asynchronous anyway)
        self.T = rb.robin_tree(async_factor=True, mixed_int8_top=(precision == "mixed_int8_top"))
        self.T.bndry_params = wl.bndry_params
        op = rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential)
        opts = rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb)
        self.inf = self.T.plan(wl.L, op, opts)
        self.h = self.T.handle
        self.kv, self.d_k, self.d_f, self.d_g, self.nrhs = kv, d_k, d_f, d_g, nrhs
        import torch
        self.d_u = torch.empty((nrhs, self.inf.nleaves, self.inf.leaf_n), dtype=torch.complex128, device=d_k.device)

    def ck(self, code):
        if code != 0:
            raise RuntimeError(self._lib.last_error(self.h))

    def step(self):
        lib = self.lib
        self.ck(lib.rb_tree_factor_device(self.h, self.d_k.data_ptr(), self.prec, 0))
        self.ck(lib.rb_tree_solve_device(self.h, self.nrhs, self.d_f.data_ptr(), self.d_g.data_ptr(), 0))
        self.ck(lib.rb_get_solution_device(self.h, self.d_u.data_ptr(), 0))

    def stream(self, torch, dev):
        return torch.cuda.ExternalStream(self.lib.rb_tree_stream(self.h), device=dev)

    def timed(self, torch, dev, steps, warmup):
        """Per-step ms and total ms of `steps` steps after `warmup`, CUDA events on the library's
        stream."""
        self.T.factor_samples(self.kv, self.precision)   # first calls allocate and build descriptors
        F = self.d_f.cpu().numpy()
        G = self.d_g.cpu().numpy()
        self.T.solve_samples(F, G)
        for _ in range(warmup):
            self.step()
        torch.cuda.synchronize()
        st = self.stream(torch, dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        with torch.cuda.stream(st):
            ev[0].record(st)
            for i in range(steps):
                self.step()
                ev[i + 1].record(st)
        torch.cuda.synchronize()
        return [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)], ev[0].elapsed_time(ev[-1])

    def split(self, torch, dev):
        """(factor ms, solve ms) of one step: the factor's own device time and the solve alone."""
        self.T.factor_samples(self.kv, self.precision)
        self.T._update_times()
        factor_ms = self.T.f_time * 1e3
        st = self.stream(torch, dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(st):
            e0.record(st)
            self.ck(self.lib.rb_tree_solve_device(self.h, self.nrhs, self.d_f.data_ptr(), self.d_g.data_ptr(), 0))
            e1.record(st)
        torch.cuda.synchronize()
        return factor_ms, e0.elapsed_time(e1)


def roofline_block(arm, torch, dev, steps, zpeak, bf16_peak):
    """Per-launch events over `steps` more steps: the dominant kernel family, its algorithmic
    rate and its fraction of the peak of the pipe it runs on."""
    arm.T.set_timing(2)
    arm.T.clear_stage_times()
    for _ in range(steps):
        arm.step()
    torch.cuda.synchronize()
    entries = arm.T.stage_times(with_flops=True)
    arm.T.set_timing(0)
    per = {}
    for name, ms, flops in entries:
        d = per.setdefault(name, [0, 0.0, 0.0])
        d[0] += 1
        d[1] += ms
        d[2] += flops
    tot = sum(v[1] for v in per.values())
    shares = {k: round(v[1] / tot, 4) for k, v in per.items()}
    dname, (dcnt, dms, dflops) = max(per.items(), key=lambda kv_: kv_[1][1])
    achieved = dflops / (dms * 1e-3) / 1e12 if dflops > 0 else None
    # the tcgen05 kernel's ceiling in algorithmic flops.  int8 digit slices (the default engine):
    # the dense int8 rate is twice the measured bf16 rate, and a 128 x 48 complex tile takes 30
    # int8 MMAs of 128 x 96 x 32 per 32-deep k-block, 23.6 M int8 operations for 1.57 M algorithmic
    # flops (15 per flop).  Split TF32: the TF32 rate is half the bf16 rate, and every complex
    # multiply-add is 4 real ones x 3 split products (3 per flop).
    int8 = os.environ.get("RB_MIXED_ENGINE", "int8") != "tf32x3"
    tc5_peak = (bf16_peak * 2.0 / 15.0 if int8 else bf16_peak / 2.0 / 3.0) if bf16_peak else None
    fams = {}
    for k, v in per.items():
        if v[2] > 0:
            pk = tc5_peak if k == "zgemm_tc5" else zpeak
            fams[k] = {"launches": v[0], "ms": round(v[1], 3), "tflops": round(v[2] / (v[1] * 1e-3) / 1e12, 2),
                       "frac": round(v[2] / (v[1] * 1e-3) / 1e12 / pk, 3) if pk else None}
    if dname == "zgemm_tc5":
        peak, pipe, src = (tc5_peak, "int8 (tcgen05, 5 digit slices)",
                           "MEASURED_PEAKS.json bf16_tflops x 2 (dense int8) / 15 (int8 operations per algorithmic "
                           "flop)") if int8 else \
            (tc5_peak, "tf32 (tcgen05, split x3)",
             "MEASURED_PEAKS.json bf16_tflops / 2 (dense TF32) / 3 (split products per complex term)")
    else:
        peak, pipe, src = zpeak, "fp64", "complex128 cuBLAS GEMM 4096^3 measured in this run (no FP64 entry in " \
                                         "MEASURED_PEAKS.json)"
    return {
        "bound": "tensor", "pipe": pipe, "kernel": dname, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
        "frac": (achieved / peak) if (achieved and peak) else None,
        "traffic": (DRAM_BYTES_PER_FLOP[dname] * dflops / dcnt) if (dname in DRAM_BYTES_PER_FLOP and dcnt) else None,
        "traffic_note": "bytes per launch: a measured bytes-per-flop ratio of this kernel (512^2 capture) times this "
                        "run's flops per launch" if dname in DRAM_BYTES_PER_FLOP else None,
        "launches": dcnt, "ms_total": dms,
        "share_of_step": shares.get(dname), "peak_source": src,
        "flop_count": "algorithmic 8mnk per complex GEMM, 8m^3 per Gauss-Jordan inverse",
        "families": fams, "shares": shares,
    }


def our_arm(args):
    import torch

    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib
    from robinsolver_b200 import workloads as W
    from robinsolver_b200.replicas import Replicas

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # replicas only: each rank runs the whole workload on its GPU; no data-path collective
    rep = Replicas("nccl", device=dev, timeout_s=300)
    world, rank = rep.world, rep.rank

    nrhs = args.nrhs or W.CONFIGS[args.config]["nrhs"]
    wl = W.make_workload(args.config, nrhs=nrhs)
    Tp = rb.robin_tree()
    Tp.bndry_params = wl.bndry_params
    inf = Tp.plan(wl.L, rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential),
                  rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb))
    kv = np.ascontiguousarray(wl.potential(Tp.sample_points(_lib.RB_POINTS_POTENTIAL)))
    F, G = Tp.sample_rhs([rb.elliptic_rhs(d=2, f=r.f, g=[rb.bndry_rhs(g) for g in r.g]) for r in wl.rhs])
    Tp.close()
    nleaf, nper = inf.nleaves, inf.leaf_n

    # the FP64 CPU solve of the same FD system for the forward errors, beside the GPU work
    check_rows = [0, nrhs - 1] if nrhs > 1 else [0]
    superlu = None
    if rank == 0 and not args.no_forward_error:
        superlu = _start_superlu(((args.config,), {"nrhs": nrhs}), kv.reshape(nleaf, -1), F, G, check_rows)

    d_k = torch.from_numpy(kv).to(dev)
    d_f = torch.from_numpy(F).to(dev)
    d_g = torch.from_numpy(G).to(dev)
    main = args.precision
    other = "fp64" if main == "mixed" else "mixed"
    # the third arm: the mixed factor with the top two levels' GEMMs on the int8 engine as well
    # (RB_FLAG_MIXED_INT8_TOP), beyond the configuration's FP64 top levels
    order = (main,) if args.single_arm else (main, other, "mixed_int8_top")
    arms = {p: Arm(rb, _lib, wl, p, kv, d_k, d_f, d_g, nrhs) for p in order}

    # ---- timed regions: the headline precision, then the other one --------------------------------
    res = {}
    clocks = ClockSampler(local)
    for p in order:
        rep.barrier()
        torch.cuda.synchronize()
        if p == main:
            clocks.start()
        step_ms, tot_ms = arms[p].timed(torch, dev, args.steps, args.warmup)
        rep.barrier()
        if p == main:
            clk = clocks.stop()
        value, total_ms = rep.rate(nrhs * args.steps, tot_ms)
        fl, sl = arms[p].T.launch_counts()
        fms, sms = arms[p].split(torch, dev)
        res[p] = {"value": value, "total_ms": total_ms, "step_ms": step_ms, "launches": (fl + sl) * args.steps,
                  "factor_ms": fms, "solve_ms": sms}

    # ---- accuracy: mixed vs FP64 GPU on every right-hand side, both vs the FP64 CPU solve ------------
    U = {p: arms[p].d_u.cpu().numpy() for p in arms}
    both = len(arms) >= 2

    def vs_fp64(p):
        errs = [float(np.abs(U[p][r] - U["fp64"][r]).max() / np.abs(U["fp64"][r]).max()) for r in range(nrhs)]
        it, rho, est, resid = arms[p].T.refine_info()
        return {"step_speedup": res["fp64"]["total_ms"] / res[p]["total_ms"],
                "factor_speedup": res["fp64"]["factor_ms"] / res[p]["factor_ms"],
                "solve_speedup": res["fp64"]["solve_ms"] / res[p]["solve_ms"],
                "max_rel_err_all_rhs": max(errs), "refine_corrections": it, "contraction": rho,
                "estimated_error": est, "residual": resid}

    # ---- roofline of the headline precision ---------------------------------------------------------
    zpeak = zgemm_peak_tflops(torch, dev)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    roof = roofline_block(arms[main], torch, dev, args.steps, zpeak, peaks.get("bf16_tflops"))

    # ---- forward errors against the FP64 CPU solve: joined here, so that the SuperLU process (all host
    # cores, ~10 GB of host memory traffic) is done before the host-copy-bound e2e leg is timed ----------
    from oracle import fd_global as FG
    fwd = None
    if superlu is not None:
        pool, job = superlu
        ref = job.get(timeout=1800)
        pool.close()
        pool.join()
        fwd = {p: max(FG.forward_error(U[p][r], ref[i]) for i, r in enumerate(check_rows)) for p in U}
        fwd["rhs_checked"] = check_rows
        fwd["reference"] = "SuperLU solve of the assembled global FD system (oracle/fd_global.SparseFD), FP64, CPU"

    # ---- e2e through the host C-ABI ---------------------------------------------------------------------
    e2e = None
    if not args.no_e2e:
        arm = arms[main]
        lib, h = arm.lib, arm.h
        pk = torch.from_numpy(kv).pin_memory()
        pf = torch.from_numpy(F).pin_memory()
        pg = torch.from_numpy(G).pin_memory()
        pu = torch.empty((nrhs, nleaf, nper), dtype=torch.complex128).pin_memory()
        pk_p, pf_p, pg_p = (_lib.C.cast(t.data_ptr(), _lib.C.POINTER(_lib.C.c_double)) for t in (pk, pf, pg))
        u_ptrs = [_lib.C.cast(pu[r].data_ptr(), _lib.C.POINTER(_lib.C.c_double)) for r in range(nrhs)]

        # the solutions come back with rb_get_solution_async: each step's read-back (671 MB at the
        # PCIe rate) runs beside the next step's factor, and rb_tree_sync ends the timed region
        # plane waves have no interior source (f = 0): with f_centres = NULL the library zeroes its
        # source array on the device and solves as for uploaded zeros
        zero_f = args.config == 4 and not np.any(F)
        f_arg = None if zero_f else pf_p

        def host_step():
            arm.ck(lib.rb_tree_factor(h, pk_p, arm.prec))
            arm.ck(lib.rb_tree_solve(h, nrhs, f_arg, pg_p))
            for r in range(nrhs):
                arm.ck(lib.rb_get_solution_async(h, r, u_ptrs[r], None))

        for _ in range(max(1, args.warmup)):
            host_step()
        arm.ck(lib.rb_tree_sync(h))
        rep.barrier()
        torch.cuda.synchronize()
        st = arm.stream(torch, dev)
        t0 = time.perf_counter()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(st)
        for _ in range(args.steps):
            host_step()
        arm.ck(lib.rb_tree_sync(h))
        a1.record(st)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        e2e_ms = rep.max(max(a0.elapsed_time(a1), wall * 1e3))
        e2e = {"value": world * nrhs * args.steps / (e2e_ms * 1e-3), "unit": "RHS/s",
               "calls": "rb_tree_factor (RB_FLAG_ASYNC_FACTOR), rb_tree_solve, rb_get_solution_async per RHS "
                        "(each step's read-back beside the next step's factor), rb_tree_sync at the end; pinned "
                        "host buffers", "precision": main,
               "h2d_bytes_per_step": int(kv.nbytes + (0 if zero_f else F.nbytes) + G.nbytes),
               "zero_sources": "f_centres = NULL (plane waves: f = 0; zeroed on the device, same kernels)"
               if zero_f else None,
               "d2h_bytes_per_step": int(pu.numel() * 16)}
        U_e2e = pu.numpy().copy()
    else:
        U_e2e = U[main]

    # backward error of the solutions the user read back
    bw = max(FG.backward_error(wl.L, wl.domain, wl.h_tgt, wl.opts_kb, wl.bndry_params, kv.reshape(nleaf, -1),
                               U_e2e[r], F[r].reshape(nleaf, -1), G[r]) for r in check_rows)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_block(wl, nrhs)

    if rank == 0:
        r0, r1, r2 = res[main], res.get(other), res.get("mixed_int8_top")
        out = {
            "metric": METRIC, "value": r0["value"], "unit": "RHS/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r0["total_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex128" if main == "fp64" else
            "complex128 storage; int8 digit-slice tensor-core GEMMs on levels 2-4, fp64 elsewhere",
            "data": "synthetic (seeded potential and plane waves, no dataset)",
            "config": config_dict(args.config, nrhs, main),
            "factor_ms": r0["factor_ms"], "solve_ms": r0["solve_ms"],
            "solves_per_s_resident": nrhs / (r0["solve_ms"] * 1e-3),
            "p50_ms": float(np.percentile(r0["step_ms"], 50)), "p99_ms": float(np.percentile(r0["step_ms"], 99)),
            other: None if r1 is None else {
                "value": r1["value"], "ms_per_step": r1["total_ms"] / args.steps, "factor_ms": r1["factor_ms"],
                "solve_ms": r1["solve_ms"], "solves_per_s_resident": nrhs / (r1["solve_ms"] * 1e-3)},
            "mixed_int8_top": None if not both else {
                "value": r2["value"], "ms_per_step": r2["total_ms"] / args.steps, "factor_ms": r2["factor_ms"],
                "solve_ms": r2["solve_ms"], "solves_per_s_resident": nrhs / (r2["solve_ms"] * 1e-3),
                "what": "RB_FLAG_MIXED_INT8_TOP: the mixed factor with the top two merge levels' GEMMs on the "
                        "int8 engine as well (their inversions FP64)"},
            "mixed_vs_fp64": None if not both else vs_fp64("mixed"),
            "mixed_int8_top_vs_fp64": None if not both else vs_fp64("mixed_int8_top"),
            "backward_error": bw, "forward_error": fwd,
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(r0["launches"]), "clocks": clk,
        }
        print(json.dumps(out), flush=True)
    for a in arms.values():
        a.T.close()
    rep.close()
    return 0


# ------------------------------------------------------------------------------------------------
# Serving: resident trees, a Poisson stream of solve requests and refactors (rb_server_*)
# ------------------------------------------------------------------------------------------------

SERVE_GRIDS = [(256, 6), (384, 8), (512, 8), (768, 10), (1024, 12)]
SERVE_BUFFERS = 8


def serve_trees(seed=5000, ntrees=8):
    """8 trees with grids drawn from {256^2 (L6), 384^2 (L8), 512^2 (L8), 768^2 (L10), 1024^2 (L12)},
    kb ~ U(50, 200) and seeded 40-bump potentials with 0.005i kb damping."""
    from robinsolver_b200 import workloads as W
    rng = np.random.default_rng(seed)
    out = []
    for i in range(ntrees):
        N, L = SERVE_GRIDS[int(rng.integers(len(SERVE_GRIDS)))]
        kb = float(rng.uniform(50.0, 200.0))
        out.append(W.make_workload(2, instance=100 + i, N=N, L=L, kb=kb, nbumps=40, delta=0.005, nrhs=0))
    return out


def _bump_params(wl, rng=None):
    pot = wl.potential
    if rng is None:
        cs, amps = pot.centres, pot.amps
    else:
        cs = rng.uniform(0.2, 0.8, size=pot.centres.shape)
        amps = rng.uniform(-1.0, 1.0, size=pot.amps.shape)
    return (pot.kb, pot.delta, pot.width, [(c[0], c[1], a) for c, a in zip(cs, amps)])


def serve_stream(srv, trees, tids, requests, rate_rhs, rng, nfactor, bufs, collect, max_rhs=64):
    """Submits `requests` solve requests (1..max_rhs RHS, point sources or plane waves sampled on
    the device) at Poisson arrivals of rate_rhs right-hand sides per second, with nfactor refactors
    (new seeded potentials) spread through the stream; returns once every request completed.
    Each tree has a few pinned output buffers: a request waits for a free one (its latency still
    counts from its scheduled arrival)."""
    import queue
    from robinsolver_b200 import _lib
    sizes = rng.integers(1, max_rhs + 1, size=requests)
    mean_rhs = float(sizes.mean())
    gaps = rng.exponential(mean_rhs / rate_rhs, size=requests)
    which = rng.integers(len(trees), size=requests)
    kinds = rng.integers(2, size=requests)
    fac_at = set(np.linspace(0, requests - 1, nfactor + 2).astype(int)[1:-1].tolist()) if nfactor else set()
    pending = [[] for _ in trees]          # per tree, in submission order: (request, buffer)

    def release(i, block):
        while pending[i]:
            rr, b = pending[i][0]
            if not srv.wait(rr, -1.0 if block else 0.0):
                return
            pending[i].pop(0)
            if b is not None:
                bufs[i].put(b)
            if block:
                return

    t0 = srv.now()
    arrival = t0
    for q in range(requests):
        arrival += gaps[q]
        while srv.now() < arrival:
            dt = arrival - srv.now()
            if dt > 2e-4:
                time.sleep(dt - 1e-4)
        ti = int(which[q])
        wl = trees[ti]
        if q in fac_at:
            pending[ti].append((srv.submit_factor(tids[ti], bumps=_bump_params(wl, rng), arrival=arrival), None))
        nr = int(sizes[q])
        if kinds[q] == 0:
            par = np.stack([rng.uniform(0.1, 0.9, nr), rng.uniform(0.1, 0.9, nr), np.full(nr, 0.05)], axis=1)
            field = _lib.RB_FIELD_POINT_SOURCE
        else:
            th = rng.uniform(0.0, 2 * np.pi, nr)
            par = np.stack([np.full(nr, wl.kb), np.cos(th), np.sin(th)], axis=1)
            field = _lib.RB_FIELD_PLANE_WAVE
        while True:
            try:
                buf = bufs[ti].get_nowait()
                break
            except queue.Empty:
                release(ti, True)
        pending[ti].append((srv.submit_solve(tids[ti], nr, field=field, params=par, u=buf[:nr * collect[ti]],
                                             arrival=arrival), buf))
        for i in range(len(trees)):
            release(i, False)
    for i in range(len(trees)):
        while pending[i]:
            release(i, True)
    return srv.now() - t0


def serve_arm(args):
    import queue

    import torch

    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib

    torch.cuda.set_device(0)
    trees = serve_trees()
    out = {"metric": "serving: solve latency p50/p99 (arrival -> solution in host memory) and RHS/s, "
                     "8 resident trees, Poisson stream", "unit": "ms", "requests": args.requests}
    for prec in ("mixed", "fp64"):
        srv = rb.robin_server(max_batch_rhs=64, precision=prec, tol=1e-10)
        tids = []
        for wl in trees:
            tids.append(srv.add_tree(wl.L, rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential),
                                     rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb), wl.bndry_params))
        per = []
        for t in tids:
            inf = srv.tree_info(t)
            per.append(inf.nleaves * inf.leaf_n)
        reqs = [srv.submit_factor(t, bumps=_bump_params(wl)) for t, wl in zip(tids, trees)]
        for r in reqs:
            srv.wait(r)
        # pinned output buffers: NBUF per tree of 64 right-hand sides (a request waits for a free one
        # of its tree; too few make the single submitter a head-of-line block for every tree)
        bufs = []
        for p in per:
            qq = queue.Queue()
            for _ in range(SERVE_BUFFERS):
                qq.put(torch.empty(64 * p, dtype=torch.complex128).pin_memory().numpy())
            bufs.append(qq)
        srv.stats(reset=True)
        rng = np.random.default_rng(777)
        # saturation: a closed burst of requests submitted at once
        dur = serve_stream(srv, trees, tids, max(50, args.requests // 10), 1e9, rng, 0, bufs, per)
        st = srv.stats(reset=True)
        sat = st["rhs"] / dur
        res = {"saturated_rhs_per_s": sat, "saturation_burst": {k: st[k] for k in ("solves", "rhs", "batches")}}
        for load in (0.5, 0.9):
            rng = np.random.default_rng(int(load * 1000))
            dur = serve_stream(srv, trees, tids, args.requests, load * sat, rng, 20, bufs, per)
            st = srv.stats(reset=True)
            res[f"load_{load}"] = {"offered_rhs_per_s": load * sat, "rhs_per_s": st["rhs"] / dur,
                                   "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                                   "max_ms": st["max_ms"], "solves": st["solves"], "batches": st["batches"],
                                   "factors": st["factors"], "factor_p50_ms": st["factor_p50_ms"],
                                   "failed": st["failed"], "duration_s": dur}
        res["reserved_gb"] = st["reserved_bytes"] / 1e9
        out[prec] = res
        srv.close()
    out["trees"] = [f"{wl.N}^2 L={wl.L} kb={wl.kb:.1f}" for wl in trees]
    out["output_buffers_per_tree"] = SERVE_BUFFERS
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------
# Forest: 64 trees of uneven sizes factored in one schedule (rb_forest_*)
# ------------------------------------------------------------------------------------------------

FOREST_GRIDS = [(128, 4), (192, 6), (256, 6), (384, 8), (512, 8)]


def forest_workloads(ntrees=64, seed=3000):
    """64 trees, grids drawn from {128^2, 192^2, 256^2, 384^2, 512^2} with L giving 24^2 to 32^2
    leaves, kb ~ U(20, 120), 20-60 bumps, 8 point-source right-hand sides each."""
    from robinsolver_b200 import workloads as W
    rng = np.random.default_rng(seed)
    out = []
    for i in range(ntrees):
        N, L = FOREST_GRIDS[int(rng.integers(len(FOREST_GRIDS)))]
        out.append(W.make_workload(2, instance=200 + i, N=N, L=L, kb=float(rng.uniform(20.0, 120.0)),
                                   nbumps=int(rng.integers(20, 61)), delta=0.005, nrhs=8, kinds="point"))
    return out


def forest_arm(args):
    import torch

    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    wls = forest_workloads()
    trees, d_k, FG = [], [], []
    for wl in wls:
        T = rb.robin_tree()
        T.bndry_params = wl.bndry_params
        T.plan(wl.L, rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential),
               rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb))
        kv = np.ascontiguousarray(wl.potential(T.sample_points(_lib.RB_POINTS_POTENTIAL)))
        F, G = T.sample_rhs([rb.elliptic_rhs(d=2, f=r.f, g=[rb.bndry_rhs(g) for g in r.g]) for r in wl.rhs])
        trees.append(T)
        d_k.append(torch.from_numpy(kv).to(dev))
        FG.append((torch.from_numpy(F).to(dev), torch.from_numpy(G).to(dev)))
    lib = _lib.lib

    # (a) every tree factored on its own, as graphs (second call on), one after the other
    for T, k in zip(trees, d_k):
        for _ in range(2):
            assert lib.rb_tree_factor_device(T.handle, k.data_ptr(), _lib.RB_PREC_FP64, 1) == 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    reps = max(1, args.steps)
    for _ in range(reps):
        for T, k in zip(trees, d_k):
            assert lib.rb_tree_factor_device(T.handle, k.data_ptr(), _lib.RB_PREC_FP64, 0) == 0
    torch.cuda.synchronize()
    single_s = (time.perf_counter() - t0) / reps
    # (b) the forest: autotune once, capture, replay
    Fo = rb.robin_forest(trees)
    ptrs = [k.data_ptr() for k in d_k]
    ta = time.perf_counter()
    Fo.factor(ptrs, autotune=True)
    tune_s = time.perf_counter() - ta
    for _ in range(max(1, args.warmup)):
        Fo.factor(ptrs, autotune=True)
    ft = []
    for _ in range(reps):
        Fo.factor(ptrs, autotune=True)
        ft.append(Fo.info()["f_time"])
    forest_s = float(np.median(ft))
    info = Fo.info()
    # the forest's factors solve: 8 point sources per tree
    t1 = time.perf_counter()
    for T, (F, G) in zip(trees, FG):
        assert lib.rb_tree_solve_device(T.handle, 8, F.data_ptr(), G.data_ptr(), 0) == 0
    torch.cuda.synchronize()
    solve_s = time.perf_counter() - t1
    picks = {}
    for h, st, eng, ms in Fo.tuning():
        if ms >= 0:                      # -1: the shape could not launch on that stage
            picks.setdefault((h, st), []).append((ms, eng))
    chosen = {f"h{h}s{st}": min(v)[1] for (h, st), v in sorted(picks.items())}
    out = {"metric": "64-tree batched factor: trees/s, forest vs one tree at a time (FP64, CUDA graphs)",
           "value": len(trees) / forest_s, "unit": "trees/s", "forest_factor_ms": forest_s * 1e3,
           "single_trees_factor_ms": single_s * 1e3, "speedup": single_s / forest_s,
           "forest_launches": info["launches"], "tuned_stages": info["tuned_stages"], "autotune_s": tune_s,
           "solve_8rhs_all_trees_ms": solve_s * 1e3, "engines": chosen,
           "trees": {f"{N}^2 L={L}": sum(1 for w in wls if w.N == N) for N, L in FOREST_GRIDS}}
    print(json.dumps(out), flush=True)
    Fo.close()
    for T in trees:
        T.close()
    return 0


def three_d_arm(args):
    """The 3D path (d = 3): the unit cube, 4^3-cell leaves, k = 1, kb = 1, bndry_params of the
    reference's example, boundary data of the exact solution cos(x/sqrt3) cos(y/sqrt3) cos(z/sqrt3)
    (Laplace u + u = 0).  Per grid: factor time (library device events, graph replay), solve time for
    8 right-hand sides, the factor's stage shares (timing mode 1), and the max-norm error against the
    exact solution (O(h^2) discretisation error, not a parity figure: parity is in the tests)."""
    import torch

    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib

    torch.cuda.set_device(0)
    s3 = 1.0 / np.sqrt(3.0)
    dom = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]])

    def exact(X):
        return np.cos(s3 * X[:, 0]) * np.cos(s3 * X[:, 1]) * np.cos(s3 * X[:, 2])

    def face(f):
        ax, side = f // 2, f % 2
        tang = [t for t in range(3) if t != ax]

        def g(P):
            X = np.zeros((P.shape[0], 3))
            X[:, ax] = dom[side, ax]
            X[:, tang[0]], X[:, tang[1]] = P[:, 0], P[:, 1]
            d = -s3 * np.sin(s3 * X[:, ax])
            for j in tang:
                d = d * np.cos(s3 * X[:, j])
            return (1.0 if side else -1.0) * d + 1j * exact(X)
        return g

    out = {"metric": "3D factor ms and 8-RHS solve ms (FP64, unit cube, 4^3 leaves)", "grids": {}}
    for N, L in ((16, 6), (32, 9)):
        T = rb.robin_tree()
        T.bndry_params = np.array([[1j, 1.0], [-1j, 1.0]])
        op = rb.elliptic_operator(d=3, domain=dom, k=lambda X: np.ones(X.shape[0], dtype=complex))
        opts = rb.solve_opts(h_tgt=1.0 / N, kb=1.0)
        T.factor(L, op, opts)
        rhs = [rb.elliptic_rhs(d=3, f=lambda X: np.zeros(X.shape[0]), g=[face(f) for f in range(6)])] * 8
        F, G = T.sample_rhs(rhs)
        kv = np.ones(T.info().n_interior, dtype=np.complex128)
        fts, sts = [], []
        for it in range(max(3, args.warmup) + max(3, args.steps)):
            T.factor_samples(kv)
            T.solve_samples(F, G)
            if it >= max(3, args.warmup):
                fts.append(T.f_time)
                sts.append(T.s_time)
        X = T.sample_points(_lib.RB_POINTS_SOLUTION)
        err = float(np.max(np.abs(T.solution_array(0).ravel() - exact(X))))
        T.set_timing(1)
        T.clear_stage_times()
        T.factor_samples(kv)
        st = T.stage_times(with_flops=True)
        T.set_timing(0)
        tot = sum(ms for _, ms, _ in st) or 1.0
        fam = {}
        for name, ms, fl in st:
            a = fam.setdefault(name, [0.0, 0.0])
            a[0] += ms
            a[1] += fl
        inf = T.info()
        out["grids"][f"{N}^3 L={L}"] = {
            "leaves": inf.nleaves, "leaf_unknowns": inf.leaf_n, "root_boundary": inf.root_nb,
            "factor_ms": float(np.median(fts)) * 1e3, "solve_8rhs_ms": float(np.median(sts)) * 1e3,
            "max_err_vs_exact": err,
            "factor_stages": {k: {"ms": round(v[0], 3), "share": round(v[0] / tot, 3),
                                  "tflops": round(v[1] / v[0] / 1e9, 2) if v[0] > 0 and v[1] > 0 else None}
                              for k, v in sorted(fam.items(), key=lambda kv: -kv[1][0])},
        }
        T.close()
    print(json.dumps(out), flush=True)
    return 0


def gemm_arm(args):
    """One batched complex GEMM D_i = A_i B_i (column-major, random normal entries) on one engine,
    timed with CUDA events over --steps launches after --warmup (rb_test_zgemm_timed, operand
    split passes included), and its error against torch's complex128 product relative to
    max|A| max|B| k."""
    import ctypes

    import torch

    from robinsolver_b200 import _lib
    m, n, k, cnt = (int(x) for x in args.gemm_shape.split(","))
    engine = {"fp64": 0, "tf32x3": 1, "int8": 2}[args.gemm]
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(7)
    A = torch.randn(cnt, k, m, dtype=torch.complex128, device=dev, generator=g)
    B = torch.randn(cnt, n, k, dtype=torch.complex128, device=dev, generator=g)
    C = torch.zeros(cnt, n, m, dtype=torch.complex128, device=dev)
    ms = ctypes.c_double()
    for reps in (max(args.warmup, 1), args.steps):
        rc = _lib.lib.rb_test_zgemm_timed(engine, m, n, k, A.data_ptr(), m, m * k, B.data_ptr(), k, k * n,
                                          C.data_ptr(), m, m * n, 1.0, 0.0, 0.0, 0.0, cnt, reps, ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"rb_test_zgemm_timed: {rc} {_lib.last_error(None)}")
    ref = torch.matmul(A.transpose(1, 2), B.transpose(1, 2))
    err = float((C.transpose(1, 2) - ref).abs().max() / (A.abs().max() * B.abs().max() * k))
    flops = 8.0 * m * n * k * cnt
    print(json.dumps({"gemm": args.gemm, "shape": {"m": m, "n": n, "k": k, "count": cnt}, "ms_per_launch": ms.value,
                      "tflops_algorithmic": flops / (ms.value * 1e-3) / 1e12, "err_rel_scale": err,
                      "launches_timed": args.steps}), flush=True)
    return 0


def main():
    args = parse()
    if args.three_d:
        return three_d_arm(args)
    if args.gemm:
        return gemm_arm(args)
    if args.serve:
        return serve_arm(args)
    if args.forest:
        return forest_arm(args)
    if args.impl == "reference":
        return reference_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
