"""CPU tests of the oracle (oracle/hps_ref.py, oracle/fd_global.py) and the workload generator."""
import numpy as np
import pytest

from oracle import fd_global as G
from oracle import hps_ref as H
from robinsolver_b200 import workloads as W
from helpers import oracle_run, rel_err

S2 = np.sqrt(2.0)


def _manufactured(N, L):
    """example.f90's 2D known-answer problem: u = cos(x/sqrt2) cos(y/sqrt2), Laplace(u) + u = 0,
    kb = 1, faces x1/y1 get zero2D and x2/y2 get one2D (example.f90:37-41, 136-186)."""
    T = H.RobinTree()
    T.bndry_params = np.array([[1j, 1.0], [-1j, 1.0]])
    T.factor(L, H.EllipticOperator(2, np.array([[0, 0, 0], [1, 1, 1.0]]), lambda X: np.ones(len(X)) + 0j),
             H.SolveOpts(h_tgt=1.0 / N, kb=1.0))
    zero2d = lambda X: 1j * np.cos(X[:, 0] / S2)
    one2d = lambda X: 1j * np.cos(1 / S2) * np.cos(X[:, 0] / S2) - 1 / S2 * np.sin(1 / S2) * np.cos(X[:, 0] / S2)
    T.solve([H.EllipticRHS(2, lambda X: np.zeros(len(X)) + 0j, [zero2d, one2d, zero2d, one2d])])
    err = 0.0
    for (box, u), lf in zip(T.get_solution(), T.leaves()):
        a, b = lf.ptbox[:2]
        P = H.leaf_all_points(a, b, lf.h, box)
        err = max(err, np.max(np.abs(u[:, 0] - np.cos(P[:, 0] / S2) * np.cos(P[:, 1] / S2))))
    return err


def test_manufactured_solution_second_order():
    e16, e32, e64 = _manufactured(16, 2), _manufactured(32, 2), _manufactured(64, 4)
    assert e64 < 3e-6
    assert 3.3 < e16 / e32 < 4.7 and 3.3 < e32 / e64 < 4.7


def test_oracle_matches_global_sparse_solve():
    wl = W.make_workload(1)
    T, U = oracle_run(wl)
    g = G.GlobalFD(wl.L, wl.domain, wl.h_tgt, wl.opts_kb, wl.bndry_params, wl.potential)
    ug = g.solve(wl.rhs[0].f, wl.rhs[0].g)
    assert rel_err(U[0], ug) < 1e-11


def test_oracle_backward_error_is_tiny(golden1):
    wl = W.make_workload(1)
    T, U = oracle_run(wl)
    k = golden1["k"].reshape(16, -1)
    e = G.backward_error(wl.L, wl.domain, wl.h_tgt, wl.opts_kb, wl.bndry_params, k, U[0],
                         golden1["F"][0].reshape(16, -1), golden1["G"][0])
    assert e < 1e-14
    e2 = G.backward_error(wl.L, wl.domain, wl.h_tgt, wl.opts_kb, wl.bndry_params, k, U[0] * (1 + 1e-9),
                          golden1["F"][0].reshape(16, -1), golden1["G"][0])
    assert e2 > 100 * e


def test_oracle_reproduces_golden(golden1):
    wl = W.make_workload(1)
    wl2 = W.make_workload(1, instance=1, kinds="plane")
    T, U = oracle_run(wl, wl.rhs + wl2.rhs)
    assert rel_err(U, golden1["U"]) < 1e-13
    assert rel_err(T.leaves()[0].rtr, golden1["rtr_leaf0"]) < 1e-13
    assert rel_err(T.levels[3][0].rtr, golden1["rtr_l3n0"]) < 1e-13


def test_leaf_matrix_structure():
    """Boundary rows of the leaf FD matrix couple only to themselves and two inward points,
    so A_bb is diagonal (the fact the B200 leaf condensation relies on)."""
    h = np.array([1 / 64, 1 / 64, 0.0])
    A = H.fd_matrix(16, 16, h, np.full(256, 20.0 + 0.2j), -20.0)
    nb = 64
    assert np.count_nonzero(A[:nb, :nb] - np.diag(np.diag(A[:nb, :nb]))) == 0
    assert np.all(np.count_nonzero(A[:nb], axis=1) == 3)
    assert np.all(np.count_nonzero(A[nb:], axis=1) <= 5)


def test_workload_is_seeded():
    a, b = W.make_workload(2), W.make_workload(2)
    assert np.array_equal(a.potential.centres, b.potential.centres)
    assert [r.kind for r in a.rhs] == ["point", "plane"] * 8
    X = np.random.default_rng(0).uniform(size=(7, 3))
    assert np.array_equal(a.rhs[1].g[2](X), b.rhs[1].g[2](X))
