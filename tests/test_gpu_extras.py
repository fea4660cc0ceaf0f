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
