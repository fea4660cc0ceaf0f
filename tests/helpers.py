"""Shared test helpers: run the oracle and the B200 path on the same seeded workload."""
import numpy as np

from oracle import hps_ref as H
from robinsolver_b200 import workloads as W


def oracle_run(wl, rhs=None):
    """Oracle factor + solve; returns (tree, U) with U = (nrhs, nleaves, n)."""
    rhs = wl.rhs if rhs is None else rhs
    T = H.RobinTree()
    T.bndry_params = wl.bndry_params
    T.factor(wl.L, H.EllipticOperator(2, wl.domain, wl.potential), H.SolveOpts(h_tgt=wl.h_tgt, kb=wl.opts_kb))
    T.solve([H.EllipticRHS(2, r.f, r.g) for r in rhs])
    sol = T.get_solution()
    U = np.stack([np.stack([u[:, r] for _, u in sol]) for r in range(len(rhs))])
    return T, U


def gpu_tree(wl, **kw):
    import robinsolver_b200 as rb
    T = rb.robin_tree(**kw)
    T.bndry_params = wl.bndry_params
    op = rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential)
    opts = rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb)
    return T, op, opts


def gpu_rhs(rhs_list):
    import robinsolver_b200 as rb
    return [rb.elliptic_rhs(d=2, f=r.f, g=[rb.bndry_rhs(g_face=gf) for gf in r.g] + [rb.bndry_rhs()] * 2)
            for r in rhs_list]


def rel_err(u, ref):
    """max |u - ref| / max |ref| over all leaves (normwise, per right-hand side)."""
    u = np.asarray(u)
    ref = np.asarray(ref)
    return float(np.max(np.abs(u - ref)) / np.max(np.abs(ref)))
