"""Mixed precision (RB_PREC_MIXED): split-TF32 tcgen05 GEMMs on the factor's merge levels l >= 2
whose interface has at least 128 points, FP64 elsewhere, and solves that apply that factor (with
FP64 GEMMs) refined against the FP64 residual of the global FD system (run on a GPU).

Bars: every refined solution within 1e-10 relative (max norm) of the FP64 GPU solution of the
same problem, as BASELINE's precision configuration asks; the merged maps of a tensor-core level
within 1e-5 of the FP64 ones (the split keeps ~22 bits) but not equal to them (the tensor-core
path did run); the refinement contracts by at least 1e-3 per correction.
"""
import numpy as np
import pytest

from robinsolver_b200 import workloads as W
from helpers import gpu_rhs, gpu_tree, rel_err

pytestmark = pytest.mark.gpu


def _pair(wl, **kw):
    Tf, op, opts = gpu_tree(wl, **kw)
    Tf.factor(wl.L, op, opts)
    Tm, op2, opts2 = gpu_tree(wl, **kw)
    Tm.factor(wl.L, op2, opts2, precision="mixed")
    return Tf, Tm


def _solve(T, rhs, tol=None):
    T.solve(gpu_rhs(rhs), tol=tol)
    return np.stack([T.solution_array(r) for r in range(len(rhs))])


@pytest.mark.parametrize("N,L", [(256, 6), (512, 10)])
def test_mixed_refined_solution_matches_fp64(N, L):
    """256^2/L=6 (32x32 leaves; levels 1-2 have 128-point interfaces, level 2 runs on tcgen05)
    and config 2's 512^2/L=10 (levels 2-4 on tcgen05), point sources and plane waves."""
    wl = W.make_workload(2, N=N, L=L, nrhs=6)
    Tf, Tm = _pair(wl)
    Uf = _solve(Tf, wl.rhs)
    Um = _solve(Tm, wl.rhs)
    for r in range(len(wl.rhs)):
        assert rel_err(Um[r], Uf[r]) < 1e-10, (r, rel_err(Um[r], Uf[r]))
    it, rho, est, res = Tm.refine_info()
    assert 1 <= it <= 4, (it, rho, est)
    assert rho < 1e-3, rho
    assert est < 1e-11
    # a tensor-core level's merged map: close to FP64, but computed differently
    d = rel_err(Tm.get_rtr(2, 0), Tf.get_rtr(2, 0))
    assert 1e-13 < d < 1e-5, d
    Tf.close()
    Tm.close()


def test_mixed_tolerance_and_repeat_solves():
    """A looser tolerance takes no more corrections; repeated solves on one factor agree."""
    wl = W.make_workload(2, N=256, L=6, nrhs=3)
    Tf, Tm = _pair(wl)
    Uf = _solve(Tf, wl.rhs)
    U1 = _solve(Tm, wl.rhs, tol=1e-10)
    it1 = Tm.refine_info()[0]
    U2 = _solve(Tm, wl.rhs, tol=1e-6)
    it2 = Tm.refine_info()[0]
    assert it2 <= it1
    for r in range(3):
        assert rel_err(U2[r], Uf[r]) < 1e-6
    U3 = _solve(Tm, wl.rhs, tol=1e-10)
    assert np.array_equal(U1, U3)
    Tf.close()
    Tm.close()


def test_mixed_small_tree():
    """A tree without 128-point interfaces below level 1 (64^2, L=4): every merge is FP64, so the
    refined solve recovers the FP64 solution at once."""
    wl = W.make_workload(1)
    Tf, Tm = _pair(wl)
    Uf = _solve(Tf, wl.rhs)
    Um = _solve(Tm, wl.rhs)
    assert rel_err(Um[0], Uf[0]) < 1e-10
    Tf.close()
    Tm.close()


@pytest.mark.slow
def test_mixed_full_size_matches_fp64():
    """1024^2, L=12, kb=200 (the headline configuration), 4 plane waves: refined to 1e-10 against
    the FP64 GPU solve."""
    wl = W.make_workload(4, nrhs=4)
    Tf, Tm = _pair(wl)
    Uf = _solve(Tf, wl.rhs)
    Um = _solve(Tm, wl.rhs)
    for r in range(len(wl.rhs)):
        assert rel_err(Um[r], Uf[r]) < 1e-10, (r, rel_err(Um[r], Uf[r]))
    Tf.close()
    Tm.close()
