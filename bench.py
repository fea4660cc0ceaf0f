#!/usr/bin/env python
"""Benchmark: factor + batched solve of the 1024^2 2D Helmholtz HPS problem on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the reference's hot path on one batch: robin_tree%factor of the 1024^2, L=12 tree
(16x16 leaves, kb=200, seeded 100-bump potential with 0.002i*kb damping) followed by one batched
solve of its 32 seeded plane-wave right-hand sides and get_solution.  ``value`` is right-hand
sides per second with the factorization inside every step, so it moves with both factor time
and solve throughput; factor_ms, solve_ms and per-step p50/p99 are reported beside it.

* value:  device-resident inputs (rb_tree_factor_device / rb_tree_solve_device /
          rb_get_solution_device), CUDA events on the library's stream, max over ranks.
* e2e:    the same steps through the host C-ABI calls a user makes (rb_tree_factor,
          rb_tree_solve, rb_get_solution per RHS) from pinned host buffers: H2D of the
          potential and right-hand sides and D2H of every solution inside the timed region.
* roofline: per-launch CUDA events over a second pass of the same steps give the dominant
          kernel's algorithmic flops / time; the denominator is the complex128 cuBLAS GEMM
          rate measured in this run (MEASURED_PEAKS.json has no FP64 entry).
* cpu_baseline / --impl reference: the reference's LAPACK/BLAS call sequence (oracle port,
          scipy OpenBLAS, all host threads) timed on a sample of the same workload -- 16 leaves,
          one node per merge level (children with random Robin-to-Robin maps of the true sizes),
          leaf and node solves of one right-hand side -- and scaled by the node counts to the full
          step (the reference solves one right-hand side per call).
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

# DRAM bytes (read + write) per launch of a stage's kernel in one step of the 1024^2 / L=12
# workload, from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, one pass):
# profiles/zgemm_dmma_kc_1024sq_L12_fp64.md.  ncu cannot run inside this script, so the figure
# is carried here and reported for the bench's own workload only.
DRAM_BYTES_PER_LAUNCH = {4: {"zgemm_tc": 1.912e8}}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nrhs", type=int, default=None, help="right-hand sides per step (default: the config's)")
    ap.add_argument("--config", type=int, default=4, choices=[1, 2, 4],
                    help="workload: 4 = 1024^2 L=12 (the headline), 2 = 512^2 L=10, 1 = 64^2 L=4 (profiling/tests)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


WORKLOAD_TEXT = {
    4: "2D Helmholtz 1024^2, L=12 (4096 leaves of 16x16), kb=200, 100-bump potential, 0.002i*kb damping",
    2: "2D Helmholtz 512^2, L=10 (1024 leaves of 16x16), kb=100, 40-bump potential, 0.005i*kb damping",
    1: "2D Helmholtz 64^2, L=4 (16 leaves of 16x16), kb=20, 5-bump potential, 0.01i*kb damping",
}


def config_dict(cfg, nrhs):
    from robinsolver_b200 import workloads as W
    c = W.CONFIGS[cfg]
    return {
        "workload": f"{WORKLOAD_TEXT[cfg]}, impedance boundary; per step: factor + {nrhs} "
                    f"{'plane-wave' if cfg == 4 else 'point-source/plane-wave'} RHS batched solve + get_solution",
        "grid": c["N"], "L": c["L"], "leaf": "16x16", "nrhs": nrhs, "precision": "fp64",
        "l2": "no flush: per-step working set and inputs larger than L2 (126 MB)" if cfg != 1
              else "small case: fits in L2",
    }


# ------------------------------------------------------------------------------------------------
# CPU baseline: the reference's LAPACK/BLAS call sequence on a sample of the workload
# ------------------------------------------------------------------------------------------------

def cpu_reference_step_seconds(wl, nrhs, threads):
    """Seconds the reference's LAPACK/BLAS calls would take for one full step (factor + nrhs
    single-RHS solves), from timed samples scaled by node counts."""
    from threadpoolctl import threadpool_limits

    from oracle import hps_ref as H

    rng = np.random.default_rng(4242)
    with threadpool_limits(limits=threads):
        root, levels = H.build_tree(wl.L, wl.domain, 2)
        T = H.RobinTree()
        T.bndry_params = wl.bndry_params
        T.opts = H.SolveOpts(h_tgt=wl.h_tgt, kb=wl.opts_kb)
        T.ell_op = H.EllipticOperator(2, wl.domain, wl.potential)
        T.levels = levels
        T.keep_leaf = True
        prof = [0.0, 0]
        H.PROFILE = prof
        try:
            # leaves: FD_solve's zgetrf + zgetrs(64 RHS) on real leaves
            nsamp = 16
            idx = rng.choice(len(levels[-1]), nsamp, replace=False)
            for i in idx:
                T._leaf(levels[-1][i])
            leaf_factor = prof[0] / nsamp
            # leaf solves: fd_leaf_solve + fd_leaf_update = two zgetrs with one RHS
            prof[0] = 0.0
            for i in idx:
                lf = levels[-1][i]
                b = np.zeros((lf.lu.shape[0], 1), dtype=np.complex128, order="F")
                H._getrs((lf.lu, lf.piv), b)
                H._getrs((lf.lu, lf.piv), b)
            leaf_solve = prof[0] / nsamp
            a, bb = levels[-1][idx[0]].ptbox[:2]
            total_factor = len(levels[-1]) * leaf_factor
            total_solve = len(levels[-1]) * leaf_solve
            # one node per merge level, children with random RtR maps of the true sizes
            child_grid = (a, bb)
            grids = {wl.L: child_grid}
            for l in range(wl.L - 1, -1, -1):
                node = levels[l][0]
                c1, c2 = node.child1, node.child2
                for c in (c1, c2):
                    c.ptbox = [grids[l + 1][0], grids[l + 1][1], -1]
                    nbc = 2 * (c.ptbox[0] + c.ptbox[1])
                    c.rtr = np.asfortranarray((rng.standard_normal((nbc, nbc)) + 1j * rng.standard_normal((nbc, nbc)))
                                              / np.sqrt(2.0 * nbc))
                prof[0] = 0.0
                T._merge(node)
                total_factor += len(levels[l]) * prof[0]
                grids[l] = tuple(node.ptbox[:2])
                # node solve work of one RHS: apply_invm in both sweeps + the T_ji g_i / T_in g_n products
                m = H.get_pt_face(c1.ptbox)[c1.iface - 1]
                x = rng.standard_normal((m, 1)) + 0j
                prof[0] = 0.0
                H.apply_invm(None, None, x, x, 0.0, node.D, node.S, node.nu)
                H.apply_invm(x, x, x, x, 1.0, node.D, node.S, node.nu)
                for c in (c1, c2):
                    nbc = c.rtr.shape[0]
                    H._gemm(1.0, np.asfortranarray(c.rtr[:, :m]), x)
                    H._gemm(1.0, np.asfortranarray(c.rtr[:m, :]), rng.standard_normal((nbc, 1)) + 0j)
                total_solve += len(levels[l]) * prof[0]
                c1.rtr = c2.rtr = None
                node.rtr = None
        finally:
            H.PROFILE = None
    return total_factor + nrhs * total_solve, total_factor, total_solve


def cpu_baseline_block(wl, nrhs, reps):
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(reps):
        t0 = time.perf_counter()
        step, fac, sol = cpu_reference_step_seconds(wl, nrhs, threads)
        vals.append((step, fac, sol, time.perf_counter() - t0))
    step, fac, sol, wall = sorted(vals)[len(vals) // 2]
    return {
        "value": nrhs / step, "unit": "RHS/s", "cores": threads, "kind": "port",
        "factor_s": fac, "solve_s_per_rhs": sol,
        "sample": f"LAPACK/BLAS time of the reference's call sequence (scipy OpenBLAS, {threads} threads) on "
                  f"16 leaves, one node per merge level (random child RtR maps of the true sizes) and one-RHS "
                  f"leaf/node solves, scaled by node counts to a full factor + {nrhs} single-RHS solves; "
                  f"median of {reps} samples of ~{wall:.1f} s wall each",
    }


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from robinsolver_b200 import workloads as W
    nrhs = args.nrhs or W.CONFIGS[args.config]["nrhs"]
    wl = W.make_workload(args.config, nrhs=nrhs)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_reference_step_seconds(wl, nrhs, threads)
    steps = []
    t_wall = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step, fac, sol = cpu_reference_step_seconds(wl, nrhs, threads)
        t_wall += time.perf_counter() - t0
        steps.append((step, fac, sol))
    tot = sum(s[0] for s in steps)
    value = nrhs * len(steps) / tot
    ms = 1e3 * tot / len(steps)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "RHS/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic (seeded)",
        "config": config_dict(args.config, nrhs),
        "factor_ms": 1e3 * np.mean([s[1] for s in steps]),
        "solve_ms_per_rhs": 1e3 * np.mean([s[2] for s in steps]),
        "cpu_baseline": {"value": value, "unit": "RHS/s", "cores": threads, "kind": "port",
                         "sample": "each step: LAPACK/BLAS time of the reference's call sequence on 16 leaves, one "
                                   "node per merge level and one-RHS solves, scaled by node counts to the full "
                                   f"step ({t_wall / max(len(steps), 1):.1f} s wall per step)"},
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
    barrier = rep.barrier
    max_over_ranks = rep.max

    nrhs = args.nrhs or W.CONFIGS[args.config]["nrhs"]
    wl = W.make_workload(args.config, nrhs=nrhs)
    # RB_FLAG_ASYNC_FACTOR: the host factor call returns once enqueued, so that the e2e step's
    # right-hand-side upload overlaps the factor (the device-path calls are asynchronous anyway)
    T = rb.robin_tree(async_factor=True)
    T.bndry_params = wl.bndry_params
    op = rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential)
    opts = rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb)
    inf = T.plan(wl.L, op, opts)
    kv = np.ascontiguousarray(wl.potential(T.sample_points(_lib.RB_POINTS_POTENTIAL)))
    rhs = [rb.elliptic_rhs(d=2, f=r.f, g=[rb.bndry_rhs(g) for g in r.g]) for r in wl.rhs]
    F, G = T.sample_rhs(rhs)
    nleaf, nper = inf.nleaves, inf.leaf_n
    # device-resident inputs/outputs for `value`
    d_k = torch.from_numpy(kv).to(dev)
    d_f = torch.from_numpy(F).to(dev)
    d_g = torch.from_numpy(G).to(dev)
    d_u = torch.empty((nrhs, nleaf, nper), dtype=torch.complex128, device=dev)
    lib = _lib.lib
    h = T.handle

    def ck(code):
        if code != 0:
            raise RuntimeError(_lib.last_error(h))

    def device_step():
        ck(lib.rb_tree_factor_device(h, d_k.data_ptr(), _lib.RB_PREC_FP64, 0))
        ck(lib.rb_tree_solve_device(h, nrhs, d_f.data_ptr(), d_g.data_ptr(), 0))
        ck(lib.rb_get_solution_device(h, d_u.data_ptr(), 0))

    # first call allocates and builds the launch descriptors
    T.factor_samples(kv)
    T.solve_samples(F, G)
    stream = torch.cuda.ExternalStream(lib.rb_tree_stream(h), device=dev)
    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize()

    # ---- timed region: value -----------------------------------------------------------------
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    fl0 = sl0 = 0
    launches = 0
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for i in range(args.steps):
            device_step()
            ev[i + 1].record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    fl, sl = T.launch_counts()
    launches = (fl + sl) * args.steps
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    value, total_ms = rep.rate(nrhs * args.steps, ev[0].elapsed_time(ev[-1]))

    # factor / solve split from the library's own events on the last step
    T.factor_samples(kv)
    T._update_times()                # waits for the (asynchronous) factor and takes its time
    factor_ms = T.f_time * 1e3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        ck(lib.rb_tree_solve_device(h, nrhs, d_f.data_ptr(), d_g.data_ptr(), 0))
        e1.record(stream)
    torch.cuda.synchronize()
    solve_ms = e0.elapsed_time(e1)

    # ---- roofline: per-launch events over the same steps ----------------------------------------
    T.set_timing(2)
    T.clear_stage_times()
    for _ in range(args.steps):
        device_step()
    torch.cuda.synchronize()
    entries = T.stage_times(with_flops=True)
    T.set_timing(0)
    per = {}
    for name, ms, flops in entries:
        d = per.setdefault(name, [0, 0.0, 0.0])
        d[0] += 1
        d[1] += ms
        d[2] += flops
    dom = max(per.items(), key=lambda kv_: kv_[1][1])
    peak = zgemm_peak_tflops(torch, dev)
    dname, (dcnt, dms, dflops) = dom
    achieved = dflops / (dms * 1e-3) / 1e12 if dflops > 0 else None
    shares = {k: round(v[1] / sum(x[1] for x in per.values()), 4) for k, v in per.items()}

    # ---- e2e through the host C-ABI ---------------------------------------------------------------
    e2e = None
    if not args.no_e2e:
        pk = torch.from_numpy(kv).pin_memory()
        pf = torch.from_numpy(F).pin_memory()
        pg = torch.from_numpy(G).pin_memory()
        pu = torch.empty((nrhs, nleaf, nper), dtype=torch.complex128).pin_memory()
        pk_p, pf_p, pg_p = (_lib.C.cast(t.data_ptr(), _lib.C.POINTER(_lib.C.c_double)) for t in (pk, pf, pg))
        u_ptrs = [_lib.C.cast(pu[r].data_ptr(), _lib.C.POINTER(_lib.C.c_double)) for r in range(nrhs)]

        def host_step():
            ck(lib.rb_tree_factor(h, pk_p, _lib.RB_PREC_FP64))
            ck(lib.rb_tree_solve(h, nrhs, pf_p, pg_p))
            for r in range(nrhs):
                ck(lib.rb_get_solution(h, r, u_ptrs[r], None))

        for _ in range(max(1, args.warmup)):
            host_step()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.steps):
            host_step()
        a1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        e2e_ms = max_over_ranks(max(a0.elapsed_time(a1), wall * 1e3))
        e2e = {"value": world * nrhs * args.steps / (e2e_ms * 1e-3), "unit": "RHS/s",
               "calls": "rb_tree_factor (RB_FLAG_ASYNC_FACTOR), rb_tree_solve, rb_get_solution per RHS; "
                        "pinned host buffers",
               "h2d_bytes_per_step": int(kv.nbytes + F.nbytes + G.nbytes),
               "d2h_bytes_per_step": int(pu.numel() * 16)}
        # the solution the user read back: backward error of two right-hand sides
        from oracle import fd_global as FG
        bw = max(FG.backward_error(wl.L, wl.domain, wl.h_tgt, wl.opts_kb, wl.bndry_params, kv.reshape(nleaf, -1),
                                   pu[r].numpy(), F[r].reshape(nleaf, -1), G[r]) for r in (0, nrhs - 1))
    else:
        bw = None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_block(wl, nrhs, reps=3)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "RHS/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
            "data": "synthetic (seeded potential and plane waves, no dataset)",
            "config": config_dict(args.config, nrhs),
            "factor_ms": factor_ms, "solve_ms": solve_ms,
            "solves_per_s_resident": nrhs / (solve_ms * 1e-3),
            "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
            "backward_error": bw,
            "roofline": {
                "bound": "tensor", "pipe": "fp64", "kernel": dname, "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None,
                "traffic": DRAM_BYTES_PER_LAUNCH.get(args.config, {}).get(dname),
                "launches": dcnt, "ms_total": dms, "share_of_step": shares.get(dname),
                "flop_count": "algorithmic 8mnk per complex GEMM (the tensor-core kernel issues three real "
                              "MMAs per complex product, so achieved can exceed a four-product peak)",
                # the MMA pipe's own work is 6mnk of the 8mnk counted: its busy fraction
                "executed_frac": (0.75 * achieved / peak) if achieved else None,
                "peak_source": "complex128 cuBLAS GEMM 4096^3 measured in this run (no FP64 entry in "
                               "MEASURED_PEAKS.json)",
                "shares": shares,
            },
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(out), flush=True)
    T.close()
    rep.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
