"""Writes the golden fixtures under tests/golden/ from the CPU oracle (oracle/hps_ref.py).

    python tests/golden/make_golden.py

config1.npz -- the 64^2, L=4 plain-method case (kb=20, 5 bumps, 0.01i*kb damping, one Gaussian
point source, g=0), seed 1000, plus a second right-hand side (a plane wave, seed 1001) so that
boundary data is exercised:
    k, F, G        potential / source / boundary samples in the C-ABI layouts
    U              get_solution of every right-hand side, (nrhs, nleaves, n)
    rtr_leaf0      leaf 0's Robin-to-Robin matrix (64 x 64)
    rtr_l3n0       node 0 of level 3 (96 x 96)
The reference itself cannot run here (no Fortran compiler), so these pin the restatement
against future changes; they are not outputs of the reference.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import hps_ref as H  # noqa: E402
from robinsolver_b200 import workloads as W  # noqa: E402


def samples(T, wl_rhs):
    leaves = T.leaves()
    a, b = leaves[0].ptbox[:2]
    F = np.stack([np.concatenate([r.f(H.interior_points(a, b, T.opts.h, lf.box)) for lf in leaves])
                  for r in wl_rhs])
    G = []
    for r in wl_rhs:
        g = []
        for f in range(1, 5):
            for lf in leaves:
                if lf.isbndry[f - 1]:
                    g.append(r.g[f - 1](H.face_points(a, b, T.opts.h, lf.box, f)))
        G.append(np.concatenate(g))
    return F, np.stack(G)


def main():
    wl = W.make_workload(1)
    wl2 = W.make_workload(1, instance=1, kinds="plane")
    rhs = wl.rhs + wl2.rhs
    T = H.RobinTree()
    T.bndry_params = wl.bndry_params
    T.factor(wl.L, H.EllipticOperator(2, wl.domain, wl.potential), H.SolveOpts(h_tgt=wl.h_tgt, kb=wl.opts_kb))
    T.solve([H.EllipticRHS(2, r.f, r.g) for r in rhs])
    leaves = T.leaves()
    a, b = leaves[0].ptbox[:2]
    k = np.concatenate([wl.potential(H.interior_points(a, b, lf.h, lf.box)) for lf in leaves])
    F, G = samples(T, rhs)
    sol = T.get_solution()
    U = np.stack([np.stack([u[:, r] for _, u in sol]) for r in range(len(rhs))])
    np.savez_compressed(Path(__file__).with_name("config1.npz"), k=k, F=F, G=G, U=U,
                        rtr_leaf0=leaves[0].rtr, rtr_l3n0=T.levels[3][0].rtr,
                        bndry_params=wl.bndry_params, opts_kb=wl.opts_kb, h_tgt=wl.h_tgt, L=wl.L)
    print("wrote config1.npz", U.shape)


if __name__ == "__main__":
    main()
