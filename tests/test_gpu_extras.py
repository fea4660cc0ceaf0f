"""Device-side sampling, check_solution and save/load of a factorized tree (beyond the
reference's factor/solve: the steps on either side of the path and persistence)."""
import numpy as np
import pytest

from robinsolver_b200 import workloads as W
from helpers import gpu_rhs, gpu_tree

pytestmark = pytest.mark.gpu


def _tree(wl, **kw):
    T, op, opts = gpu_tree(wl, **kw)
    T.plan(wl.L, op, opts)
    return T, op, opts


def test_device_sampling_matches_the_host_definitions():
    import torch
    from robinsolver_b200 import _lib
    wl = W.make_workload(2, N=128, L=6, nrhs=4)          # point, plane, point, plane
    T, _, _ = _tree(wl)
    inf = T.info()
    # potential
    pot = wl.potential
    par = np.concatenate([[pot.kb, pot.delta, pot.width],
                          np.column_stack([pot.centres, pot.amps]).ravel()])
    dk = torch.empty(inf.n_interior, dtype=torch.complex128, device="cuda")
    T.sample_device(_lib.RB_FIELD_BUMP_POTENTIAL, len(pot.amps), par, dk.data_ptr())
    kh = pot(T.sample_points(_lib.RB_POINTS_POTENTIAL))
    assert np.max(np.abs(dk.cpu().numpy() - kh)) <= 1e-14 * np.max(np.abs(kh))
    # point sources (f) and plane waves (g)
    pts = [r for r in wl.rhs if r.kind == "point"]
    pws = [r for r in wl.rhs if r.kind == "plane"]
    df = torch.empty((len(pts), inf.n_interior), dtype=torch.complex128, device="cuda")
    dg = torch.empty((len(pws), inf.root_nb), dtype=torch.complex128, device="cuda")
    T.sample_device(_lib.RB_FIELD_POINT_SOURCE, len(pts), [[r.f.x0[0], r.f.x0[1], r.f.width] for r in pts],
                    df.data_ptr(), 0)
    T.sample_device(_lib.RB_FIELD_PLANE_WAVE, len(pws), [[r.g[0].kb, r.g[0].d[0], r.g[0].d[1]] for r in pws],
                    0, dg.data_ptr())
    F, G = T.sample_rhs(gpu_rhs(pts + pws))
    assert np.max(np.abs(df.cpu().numpy() - F[:len(pts)])) <= 1e-14
    gh = G[len(pts):]
    assert np.max(np.abs(dg.cpu().numpy() - gh)) <= 1e-13 * np.max(np.abs(gh))
    T.close()


@pytest.mark.parametrize("norm, rel", [("1", False), ("2", False), ("M", False), ("M", True)])
def test_check_solution_matches_a_host_computation(norm, rel):
    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib
    wl = W.make_workload(2, N=128, L=6, nrhs=2)
    T, op, opts = gpu_tree(wl)
    T.factor(wl.L, op, opts)
    T.solve(gpu_rhs(wl.rhs))
    # a smooth stand-in for an exact solution, vectorised over points
    true_sol = lambda X: np.exp(1j * 3.0 * X[:, 0]) * (1.0 + X[:, 1]) + 0.5
    err = rb.check_solution(T, true_sol, irhs=1, norm=norm, rel=rel)
    U = T.solution_array(1)
    ue = true_sol(T.sample_points(_lib.RB_POINTS_SOLUTION)).reshape(U.shape)
    d = np.abs((U - ue) / ue) if rel else np.abs(U - ue)
    ref = {"1": d.sum(axis=1), "2": np.sqrt((d * d).sum(axis=1))}.get(norm, d.max(axis=1))
    assert np.allclose(err, ref, rtol=1e-12, atol=0.0)
    T.close()


def test_save_and_load_give_the_same_solver(tmp_path):
    import robinsolver_b200 as rb
    wl = W.make_workload(2, N=128, L=6, nrhs=3)
    T, op, opts = gpu_tree(wl)
    T.factor(wl.L, op, opts)
    path = tmp_path / "tree.rbt"
    T.save(path)
    Tl = rb.robin_tree.load(path)
    rhs = gpu_rhs(wl.rhs)
    T.solve(rhs)
    F, G = T.sample_rhs(rhs)
    Tl.solve_samples(F, G)
    for r in range(len(rhs)):
        assert np.array_equal(T.solution_array(r), Tl.solution_array(r))
    assert np.array_equal(T.get_rtr(1, 0), Tl.get_rtr(1, 0))
    T.close()
    Tl.close()


def test_async_readback_equals_sync_and_orders_with_the_next_solve():
    """rb_get_solution_async + rb_tree_sync give the same bytes as rb_get_solution, and a solve
    issued right after the asynchronous read-back (other right-hand sides) does not overwrite the
    solution before the copy has landed."""
    import ctypes

    import torch

    from robinsolver_b200 import _lib
    wl = W.make_workload(2, N=256, L=6, nrhs=4)
    T, op, opts = gpu_tree(wl)
    T.factor(wl.L, op, opts)
    rhs = gpu_rhs(wl.rhs)
    T.solve(rhs)
    ref = [T.solution_array(r) for r in range(4)]
    inf = T.info()
    bufs = [torch.zeros((inf.nleaves, inf.leaf_n), dtype=torch.complex128).pin_memory() for _ in range(4)]
    ptr = [ctypes.cast(b.data_ptr(), ctypes.POINTER(ctypes.c_double)) for b in bufs]
    lib = _lib.lib
    for r in range(4):
        assert lib.rb_get_solution_async(T.handle, r, ptr[r], None) == 0, _lib.last_error(T.handle)
    T.solve(rhs[::-1])              # writes the solution buffer: must wait for the copies above
    assert lib.rb_tree_sync(T.handle) == 0
    for r in range(4):
        assert np.array_equal(bufs[r].numpy(), ref[r]), r
    # and the new solve is the reversed set
    assert np.array_equal(T.solution_array(0), ref[3])
    T.close()


def test_null_sources_solve_as_zeros():
    """rb_tree_solve with f_centres = NULL (every interior source zero) gives the bytes of a solve
    with an uploaded array of zeros, FP64 and mixed precision."""
    wl = W.make_workload(2, N=256, L=6, nrhs=3)
    for prec in ("fp64", "mixed"):
        T, op, opts = gpu_tree(wl)
        T.factor(wl.L, op, opts, precision=prec)
        F, G = T.sample_rhs(gpu_rhs(wl.rhs))
        T.solve_samples(np.zeros_like(F), G)
        ref = [T.solution_array(r) for r in range(3)]
        T.solve_samples(None, G)
        for r in range(3):
            assert np.array_equal(T.solution_array(r), ref[r]), (prec, r)
        T.close()


def test_changing_rhs_counts_reuse_cached_solve_plans():
    """Solves whose RHS counts change from call to call (a serving loop's batches) switch between
    cached launch plans and graphs: every solution equals the first solve of that count, bit for
    bit, across switches, and more counts than the cache holds still solve correctly."""
    wl = W.make_workload(2, N=256, L=6, nrhs=12)
    T, op, opts = gpu_tree(wl)
    T.factor(wl.L, op, opts)
    rhs = gpu_rhs(wl.rhs)
    first = {}
    for c in [3, 5, 3, 7, 5, 3, 7, 7, 1, 2, 4, 6, 8, 9, 10, 11, 12, 3, 5]:
        T.solve(rhs[:c])
        U = [T.solution_array(r) for r in range(c)]
        if c not in first:
            first[c] = U
        for r in range(c):
            assert np.array_equal(U[r], first[c][r]), (c, r)
    # batches are independent of their size: the first RHS agrees across counts
    for c in first:
        assert np.array_equal(first[c][0], first[1][0]), c
    T.close()
