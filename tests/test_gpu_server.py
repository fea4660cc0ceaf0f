"""The serving loop (rb_server_*): resident trees of different sizes, continuously batched solve
requests, refactors ordered with their tree's solves (run on a GPU).

Each served result must equal the same right-hand sides solved alone on a separate handle of
the same tree: bit for bit for FP64 trees (the solve's GEMMs sum in an order that does not depend
on the batch), within the 1e-10 refinement tolerance for a mixed-precision tree.
"""
import numpy as np
import pytest

import robinsolver_b200 as rb
from robinsolver_b200 import _lib
from robinsolver_b200 import workloads as W
from helpers import gpu_rhs, gpu_tree, rel_err

pytestmark = pytest.mark.gpu

# (config, N, L): 16x16 leaves at 64^2/L4 and 128^2/L6, 24x24 leaves at 96^2/L4
TREES = [(1, 64, 4), (2, 128, 6), (1, 96, 4)]


def _alone(wl, F, G, precision="fp64"):
    """F, G for a list of right-hand sides solved on a fresh handle in one call."""
    T, op, opts = gpu_tree(wl)
    T.factor(wl.L, op, opts, precision=precision)
    T.solve_samples(F, G)
    U = np.stack([T.solution_array(r) for r in range(F.shape[0])])
    T.close()
    return U


def _setup(srv, precision="fp64"):
    trees = []
    for i, (cfg, N, L) in enumerate(TREES):
        wl = W.make_workload(cfg, instance=10 + i, N=N, L=L, nrhs=8, kinds="alternate")
        T, op, opts = gpu_tree(wl)
        T.plan(wl.L, op, opts)
        kv = np.ascontiguousarray(wl.potential(T.sample_points(_lib.RB_POINTS_POTENTIAL)))
        F, G = T.sample_rhs(gpu_rhs(wl.rhs))
        inf = T.info()
        T.close()
        tid = srv.add_tree(wl.L, op, opts, wl.bndry_params)
        trees.append(dict(wl=wl, tid=tid, k=kv, F=F, G=G, per=inf.nleaves * inf.leaf_n, inf=inf))
    return trees


def test_served_results_equal_alone_fp64():
    srv = rb.robin_server(max_batch_rhs=16)
    trees = _setup(srv)
    reqs = [srv.submit_factor(t["tid"], k=t["k"]) for t in trees]
    rng = np.random.default_rng(3)
    jobs = []
    # submit everything at once: each tree's queue is batched while earlier batches run
    for n in range(30):
        t = trees[rng.integers(len(trees))]
        nr = int(rng.integers(1, 5))
        idx = rng.choice(8, nr, replace=False)
        F = np.ascontiguousarray(t["F"][idx])
        G = np.ascontiguousarray(t["G"][idx])
        u = np.zeros(nr * t["per"], dtype=np.complex128)
        jobs.append((t, idx, u, srv.submit_solve(t["tid"], nr, f=F, g=G, u=u)))
    for r in reqs:
        assert srv.wait(r)
    for _, _, _, r in jobs:
        assert srv.wait(r)
    st = srv.stats()
    assert st["solves"] == 30 and st["failed"] == 0
    assert st["batches"] < 30            # requests were merged
    assert st["p99_ms"] >= st["p50_ms"] > 0.0
    ref = {id(t): _alone(t["wl"], t["F"], t["G"]) for t in trees}
    for t, idx, u, _ in jobs:
        U = u.reshape(len(idx), t["inf"].nleaves, t["inf"].leaf_n)
        for j, q in enumerate(idx):
            assert np.array_equal(U[j], ref[id(t)][q])
    srv.close()


def test_refactor_is_ordered_with_solves_and_fields():
    """Solves before a refactor use the old potential, solves after it the new one; device-side
    fields (point sources, plane waves) give what host samples of the same fields give."""
    srv = rb.robin_server(max_batch_rhs=8)
    trees = _setup(srv)
    t = trees[1]
    wl = t["wl"]
    wl_new = W.make_workload(2, instance=99, N=wl.N, L=wl.L, nrhs=2, kinds="alternate")
    T, op, opts = gpu_tree(wl_new)
    T.plan(wl_new.L, op, opts)
    k_new = np.ascontiguousarray(wl_new.potential(T.sample_points(_lib.RB_POINTS_POTENTIAL)))
    T.close()
    per = t["per"]
    r0 = srv.submit_factor(t["tid"], k=t["k"])
    u_old = np.zeros(per, dtype=np.complex128)
    s_old = srv.submit_solve(t["tid"], 1, f=np.ascontiguousarray(t["F"][:1]), g=np.ascontiguousarray(t["G"][:1]), u=u_old)
    r1 = srv.submit_factor(t["tid"], k=k_new)
    u_new = np.zeros(per, dtype=np.complex128)
    s_new = srv.submit_solve(t["tid"], 1, f=np.ascontiguousarray(t["F"][:1]), g=np.ascontiguousarray(t["G"][:1]), u=u_new)
    # device-sampled fields: one point source (x0, y0, w) and one plane wave (kb, dx, dy)
    ps = wl.rhs[0].f
    pw = wl.rhs[1].g[0]
    u_f = np.zeros(2 * per, dtype=np.complex128)
    s_f = srv.submit_solve(t["tid"], 1, field=_lib.RB_FIELD_POINT_SOURCE, params=[ps.x0[0], ps.x0[1], ps.width],
                           u=u_f[:per])
    s_g = srv.submit_solve(t["tid"], 1, field=_lib.RB_FIELD_PLANE_WAVE, params=[pw.kb, pw.d[0], pw.d[1]],
                           u=u_f[per:])
    for r in (r0, s_old, r1, s_new, s_f, s_g):
        assert srv.wait(r)
    old = _alone(wl, t["F"][:1], t["G"][:1])[0]
    new = _alone(wl_new, t["F"][:1], t["G"][:1])[0]
    assert np.array_equal(u_old.reshape(old.shape), old)
    assert np.array_equal(u_new.reshape(new.shape), new)
    both = _alone(wl_new, t["F"][:2], t["G"][:2])
    assert rel_err(u_f[:per].reshape(old.shape), both[0]) < 1e-12
    assert rel_err(u_f[per:].reshape(old.shape), both[1]) < 1e-12
    srv.close()


def test_admission_refuses_a_tree_beyond_the_budget():
    srv = rb.robin_server(device_budget=64 << 20, max_batch_rhs=4)
    wl = W.make_workload(2, N=512, L=10, nrhs=1)
    T, op, opts = gpu_tree(wl)
    tid = srv.add_tree(wl.L, op, opts, wl.bndry_params)
    r = srv.submit_factor(tid, bumps=(100.0, 0.005, 0.08, [(0.5, 0.5, 0.3)]))
    with pytest.raises(rb.RobinSolverError) as e:
        srv.wait(r)
    assert e.value.code == _lib.RB_ERR_OUT_OF_MEMORY
    srv.close()


def test_mixed_server_within_tolerance():
    """A mixed-precision server (256^2/L=6: one tensor-core level) against FP64 solves alone."""
    srv = rb.robin_server(max_batch_rhs=8, precision="mixed", tol=1e-10)
    wl = W.make_workload(2, instance=5, N=256, L=6, nrhs=6, kinds="alternate")
    T, op, opts = gpu_tree(wl)
    T.plan(wl.L, op, opts)
    kv = np.ascontiguousarray(wl.potential(T.sample_points(_lib.RB_POINTS_POTENTIAL)))
    F, G = T.sample_rhs(gpu_rhs(wl.rhs))
    inf = T.info()
    T.close()
    tid = srv.add_tree(wl.L, op, opts, wl.bndry_params)
    per = inf.nleaves * inf.leaf_n
    reqs = [srv.submit_factor(tid, k=kv)]
    outs = []
    for q in range(6):
        u = np.zeros(per, dtype=np.complex128)
        outs.append(u)
        reqs.append(srv.submit_solve(tid, 1, f=np.ascontiguousarray(F[q:q + 1]), g=np.ascontiguousarray(G[q:q + 1]), u=u))
    for r in reqs:
        assert srv.wait(r)
    ref = _alone(wl, F, G)
    for q in range(6):
        assert rel_err(outs[q].reshape(ref[q].shape), ref[q]) < 1e-10
    srv.close()
