"""Forests (rb_forest_*): trees of uneven sizes factored together in one level-synchronous
schedule with autotuned GEMM tile shapes (run on a GPU).

Every tree of the forest must solve like the same tree factored alone (1e-12 relative: the tile
shapes the autotuner picks differ from the one-tree rule only in FP64 rounding) and, for the
config-1 tree, like the oracle (1e-11).
"""
import numpy as np
import pytest

import robinsolver_b200 as rb
from robinsolver_b200 import _lib
from robinsolver_b200 import workloads as W
from helpers import gpu_rhs, gpu_tree, oracle_run, rel_err

pytestmark = pytest.mark.gpu

# (config, N, L): leaves 16^2, 24^2, 16^2, 32^2, 24^2 -> uneven interface lengths per height
SHAPES = [(1, 64, 4), (1, 96, 4), (2, 128, 6), (2, 128, 4), (2, 192, 6)]


def _trees(instance0=0):
    out = []
    for i, (cfg, N, L) in enumerate(SHAPES):
        wl = W.make_workload(cfg, instance=instance0 + i, N=N, L=L, nrhs=2, kinds="alternate")
        T, op, opts = gpu_tree(wl)
        T.plan(wl.L, op, opts)
        kv = np.ascontiguousarray(wl.potential(T.sample_points(_lib.RB_POINTS_POTENTIAL)))
        out.append((wl, T, kv))
    return out


def _solve(T, wl):
    T.solve(gpu_rhs(wl.rhs))
    return np.stack([T.solution_array(r) for r in range(len(wl.rhs))])


def _alone(wl):
    T, op, opts = gpu_tree(wl)
    T.factor(wl.L, op, opts)
    U = _solve(T, wl)
    T.close()
    return U


@pytest.mark.parametrize("autotune", [True, False])
def test_forest_factor_matches_single_trees(autotune):
    import torch
    dev = torch.device("cuda", 0)
    trees = _trees()
    d_k = [torch.from_numpy(kv).to(dev) for _, _, kv in trees]
    F = rb.robin_forest([T for _, T, _ in trees])
    F.factor([t.data_ptr() for t in d_k], autotune=autotune)
    info = F.info()
    assert info["f_time"] > 0 and info["launches"] > 0
    if autotune:
        assert info["tuned_stages"] > 0 and len(F.tuning()) > 0
    for wl, T, _ in trees:
        U = _solve(T, wl)
        Ua = _alone(wl)
        for r in range(len(wl.rhs)):
            assert rel_err(U[r], Ua[r]) < 1e-12, (wl.N, wl.L, r)
    # the oracle on the config-1 tree
    wl, T, _ = trees[0]
    _, Uo = oracle_run(wl)
    assert rel_err(_solve(T, wl)[0], Uo[0]) < 1e-11
    # refactor through the captured graph with other potentials
    trees2 = _trees(instance0=50)
    for (wl2, T2, kv2), d in zip(trees2, d_k):
        d.copy_(torch.from_numpy(kv2))
        T2.close()
    F.factor([t.data_ptr() for t in d_k], autotune=autotune)
    F.factor([t.data_ptr() for t in d_k], autotune=autotune)
    for (wl, T, _), (wl2, _, _) in zip(trees, trees2):
        U = _solve(T, wl2)
        Ua = _alone(wl2)
        assert rel_err(U[0], Ua[0]) < 1e-12
    F.close()
    for _, T, _ in trees:
        T.close()
