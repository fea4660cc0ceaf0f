"""Mixed precision (RB_PREC_MIXED): the factor's merge levels l >= 2 with interfaces of at least 256
points run their B1, Y1, Y2 and parent-map GEMMs on the tcgen05 tensor cores in int8 digit
slices with exact integer accumulation (the default engine), FP64 elsewhere; solves apply that
factor with FP64 GEMMs and are refined against the FP64 residual of the global FD system (run on a
GPU).

Bars: every refined solution within 1e-10 relative (max norm) of the FP64 GPU solution of the
same problem (the mixed-precision configuration's bar); the merged maps of a tensor-core level
within 1e-8 of the FP64 ones (the digit slices keep ~35 bits) but not equal to them (the
tensor-core path did run); the refinement contracts by at least 1e-5 per correction.
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


@pytest.mark.parametrize("N,L,tc_level", [(256, 6, None), (512, 10, 2)])
def test_mixed_refined_solution_matches_fp64(N, L, tc_level):
    """256^2/L=6 (32x32 leaves; no interface below level 1 reaches 256 points: every merge FP64)
    and config 2's 512^2/L=10 (level 2, 256-point interfaces, on the tensor cores), point sources
    and plane waves."""
    wl = W.make_workload(2, N=N, L=L, nrhs=6)
    Tf, Tm = _pair(wl)
    Uf = _solve(Tf, wl.rhs)
    Um = _solve(Tm, wl.rhs)
    for r in range(len(wl.rhs)):
        assert rel_err(Um[r], Uf[r]) < 1e-10, (r, rel_err(Um[r], Uf[r]))
    it, rho, est, res = Tm.refine_info()
    assert 1 <= it <= 2, (it, rho, est)
    assert rho < 1e-5, rho
    assert est < 1e-11
    if tc_level is not None:
        # a tensor-core level's merged map: close to FP64, but computed differently
        d = rel_err(Tm.get_rtr(tc_level, 0), Tf.get_rtr(tc_level, 0))
        assert 1e-15 < d < 1e-8, d
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
    """A tree without 256-point interfaces below level 1 (64^2, L=4): every merge is FP64, so the
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


def test_mixed_int8_top_levels():
    """RB_FLAG_MIXED_INT8_TOP (512^2/L=10): the top two levels' GEMMs on the int8 engine as well
    (their 512- and 256-point interfaces' inversions stay FP64); refined within 1e-10 of FP64 with
    one correction, and the root level's map differs from the FP64 one within the engine's bar."""
    wl = W.make_workload(2, N=512, L=10, nrhs=4)
    Tf, op, opts = gpu_tree(wl)
    Tf.factor(wl.L, op, opts)
    Tm, op2, opts2 = gpu_tree(wl, mixed_int8_top=True)
    Tm.factor(wl.L, op2, opts2, precision="mixed")
    Uf = _solve(Tf, wl.rhs)
    Um = _solve(Tm, wl.rhs)
    for r in range(len(wl.rhs)):
        assert rel_err(Um[r], Uf[r]) < 1e-10, (r, rel_err(Um[r], Uf[r]))
    it, rho, est, res = Tm.refine_info()
    assert it == 1 and rho < 1e-5, (it, rho)
    for lvl in (1, 2):
        d = rel_err(Tm.get_rtr(lvl, 0), Tf.get_rtr(lvl, 0))
        assert 1e-15 < d < 1e-8, (lvl, d)
    Tf.close()
    Tm.close()
