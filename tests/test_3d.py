"""3D (d = 3) path: the oracle's restatement against an independently assembled global system and
the manufactured solution (CPU), the library's 3D plan against the oracle's tree (CPU), and the
CUDA factor/solve against the oracle (GPU)."""
import numpy as np
import pytest

from oracle import hps_ref as H
from oracle import hps_ref3d as H3

# bndry_params of example.f90 (nu = -1, zeta = 0: the transmission conditions of continuous u and
# du/dn), and a general pair for the algebra (nu, zeta both complex and nonzero)
BP = np.array([[1j, 1.0], [-1j, 1.0]], dtype=np.complex128)
BP_GEN = np.array([[1.0 + 0.5j, 1.0], [-1.0j, 0.7]], dtype=np.complex128)
S3 = 1.0 / np.sqrt(3.0)


def exact(X):
    """cos(x/sqrt3) cos(y/sqrt3) cos(z/sqrt3): Laplace u + u = 0 (example.f90:188-196 in form)."""
    return np.cos(S3 * X[:, 0]) * np.cos(S3 * X[:, 1]) * np.cos(S3 * X[:, 2])


def exact_dn(X, axis, sign):
    """Outward normal derivative on a face of normal `axis` and direction `sign`."""
    c = [np.cos(S3 * X[:, j]) for j in range(3)]
    d = -S3 * np.sin(S3 * X[:, axis])
    prod = d
    for j in range(3):
        if j != axis:
            prod = prod * c[j]
    return sign * prod


def robin_faces(domain, kb):
    """g on the six faces for the exact solution: du/dn + i kb u at face-local coordinates."""
    lo, hi = domain[0], domain[1]
    faces = []
    for f in range(6):
        ax, side = f // 2, f % 2
        tang = [t for t in range(3) if t != ax]

        def g(P, ax=ax, side=side, tang=tang):
            X = np.zeros((P.shape[0], 3))
            X[:, ax] = hi[ax] if side else lo[ax]
            X[:, tang[0]] = P[:, 0]
            X[:, tang[1]] = P[:, 1]
            return exact_dn(X, ax, 1.0 if side else -1.0) + 1j * kb * exact(X)
        faces.append(g)
    return faces


def bump_potential(X):
    """A smooth, complex, non-constant potential: 1 + 0.3 exp(-|x - c|^2 / 0.05) + 0.01i."""
    r2 = ((X - np.array([0.4, 0.55, 0.45])) ** 2).sum(axis=1)
    return 1.0 + 0.3 * np.exp(-r2 / 0.05) + 0.01j


def source(X):
    return np.sin(3.0 * X[:, 0]) * np.cos(2.0 * X[:, 1]) + 0.5j * X[:, 2]


def plane_faces():
    """Arbitrary smooth boundary data on the six faces (face-local coordinates)."""
    return [lambda P, f=f: np.cos(1.5 * P[:, 0] + 0.7 * f) + 1j * np.sin(2.0 * P[:, 1] - 0.3 * f) for f in range(6)]


def oracle_tree(L, N, kfun, kb=1.0, domain=None, bp=BP):
    domain = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]) if domain is None else domain
    O = H3.RobinTree3D()
    O.bndry_params = bp
    O.factor(L, H.EllipticOperator(3, domain, kfun), H.SolveOpts(h_tgt=1.0 / N, kb=kb))
    return O


# ---- oracle (CPU) ------------------------------------------------------------------------------

@pytest.mark.parametrize("bp", [BP, BP_GEN])
def test_oracle3d_matches_global_system(bp):
    L, N, kb = 3, 8, 1.0
    dom = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]])
    O = oracle_tree(L, N, bump_potential, kb, dom, bp)
    gf = plane_faces()
    O.solve([H.EllipticRHS(3, source, gf)])
    tree = np.stack([u[:, 0] for _, u in O.get_solution()])
    glob = H3.global_solve(L, dom, 1.0 / N, kb, bp, bump_potential, source, gf)
    assert np.max(np.abs(tree - glob)) / np.max(np.abs(glob)) < 1e-11


def test_oracle3d_manufactured_solution_converges():
    errs = []
    for N, L in ((8, 3), (16, 6)):
        dom = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]])
        O = oracle_tree(L, N, lambda X: np.ones(X.shape[0], dtype=complex), 1.0, dom)
        O.solve([H.EllipticRHS(3, lambda X: np.zeros(X.shape[0]), robin_faces(dom, 1.0))])
        e = 0.0
        for box, u in O.get_solution():
            idx = O.index(O.levels[-1][0].ptbox)
            X = H3.leaf_all_points(idx, O.opts.h, box)
            e = max(e, np.max(np.abs(u[:, 0] - exact(X))))
        errs.append(e)
    assert errs[1] < errs[0] / 3.0, errs          # O(h^2)
    assert errs[1] < 2e-3, errs


# ---- plan (CPU) ----------------------------------------------------------------------------------

def _planned3d(L, N, kfun=bump_potential, kb=1.0):
    import robinsolver_b200 as rb
    T = rb.robin_tree()
    T.bndry_params = BP
    T.plan(L, rb.elliptic_operator(d=3, domain=np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]), k=kfun),
           rb.solve_opts(h_tgt=1.0 / N, kb=kb))
    return T


@pytest.mark.parametrize("L,N", [(3, 8), (4, 16), (6, 16)])
def test_plan3d_matches_oracle(L, N):
    from robinsolver_b200 import _lib
    T = _planned3d(L, N)
    inf = T.info()
    O = oracle_tree(L, N, bump_potential)
    leaves = O.levels[-1]
    a, b, c = leaves[0].ptbox
    idx = O.index(leaves[0].ptbox)
    assert (inf.d, inf.nleaves, inf.leaf_a, inf.leaf_b, inf.leaf_c) == (3, len(leaves), a, b, c)
    assert (inf.leaf_nb, inf.leaf_n) == (idx.nb, idx.n)
    assert inf.n_interior == len(leaves) * a * b * c
    for l in range(L + 1):
        assert T._level_grid(l) == tuple(O.levels[l][0].ptbox[:3])
    hl = O.opts.h
    pot = np.concatenate([H3.interior_points(idx, lf.h, lf.box) for lf in leaves])
    src = np.concatenate([H3.interior_points(idx, hl, lf.box) for lf in leaves])
    bnd = np.concatenate([H3.face_points(idx, hl, lf.box, f) for f in range(1, 7) for lf in leaves
                          if lf.isbndry[f - 1]])
    sol = np.concatenate([H3.leaf_all_points(idx, hl, lf.box) for lf in leaves])
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_POTENTIAL), pot)
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_SOURCE), src)
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_BOUNDARY)[:, :2], bnd[:, :2])
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_SOLUTION), sol)
    assert inf.root_nb == bnd.shape[0]
    T.close()


def test_plan3d_refusals():
    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib
    T = rb.robin_tree()
    T.bndry_params = BP
    op = rb.elliptic_operator(d=3, domain=np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]), k=bump_potential)
    # 64^3 in 4^3 leaves: the root interface holds 4096 points
    with pytest.raises(rb.RobinSolverError) as ei:
        T.plan(12, op, rb.solve_opts(h_tgt=1.0 / 64, kb=1.0))
    assert ei.value.code == _lib.RB_ERR_UNSUPPORTED and "1024" in str(ei.value)
    # one 12^3 leaf: 864 + 1728 unknowns
    with pytest.raises(rb.RobinSolverError) as ei:
        T.plan(1, op, rb.solve_opts(h_tgt=1.0 / 24, kb=1.0))
    assert ei.value.code == _lib.RB_ERR_UNSUPPORTED


# ---- CUDA path against the oracle (GPU) ------------------------------------------------------------

def _gpu_tree(L, N, kfun, kb=1.0, bp=BP):
    import robinsolver_b200 as rb
    T = rb.robin_tree()
    T.bndry_params = bp
    T.factor(L, rb.elliptic_operator(d=3, domain=np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]), k=kfun),
             rb.solve_opts(h_tgt=1.0 / N, kb=kb))
    return T


def rel_err(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("L,N,bp", [(3, 8, BP), (6, 16, BP), (5, 16, BP_GEN)])
def test_gpu3d_factor_and_solve_match_oracle(L, N, bp):
    import robinsolver_b200 as rb
    T = _gpu_tree(L, N, bump_potential, bp=bp)
    O = oracle_tree(L, N, bump_potential, bp=bp)
    for l in range(1, L + 1):
        for i in (0, len(O.levels[l]) - 1):
            assert rel_err(T.get_rtr(l, i), O.levels[l][i].rtr) < 1e-11, (l, i)
    gf = plane_faces()
    rhs = [rb.elliptic_rhs(d=3, f=source, g=gf),
           rb.elliptic_rhs(d=3, f=lambda X: np.zeros(X.shape[0]), g=plane_faces()[::-1])]
    T.solve(rhs)
    O.solve([H.EllipticRHS(3, r.f, r.g) for r in rhs])
    ref = [np.stack([u[:, j] for _, u in O.get_solution()]) for j in range(2)]
    for j in range(2):
        assert rel_err(T.solution_array(j), ref[j]) < 1e-11, j
    T.close()


@pytest.mark.gpu
def test_gpu3d_manufactured_solution():
    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib
    N, L = 32, 9
    dom = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]])
    T = _gpu_tree(L, N, lambda X: np.ones(X.shape[0], dtype=complex))
    T.solve(rb.elliptic_rhs(d=3, f=lambda X: np.zeros(X.shape[0]), g=robin_faces(dom, 1.0)))
    X = T.sample_points(_lib.RB_POINTS_SOLUTION)
    u = T.solution_array(0).ravel()
    err = np.max(np.abs(u - exact(X)))
    assert err < 5e-4, err
    T.close()


@pytest.mark.gpu
def test_gpu3d_refuses_mixed_precision():
    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib
    with pytest.raises(rb.RobinSolverError) as ei:
        T = rb.robin_tree()
        T.bndry_params = BP
        T.factor(3, rb.elliptic_operator(d=3, domain=np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]),
                                         k=bump_potential), rb.solve_opts(h_tgt=1.0 / 8, kb=1.0), precision="mixed")
    assert ei.value.code == _lib.RB_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_gpu3d_reference_merge_form_matches_oracle():
    """The reference's interface solve (inv(D), inv(S), RB_FLAG_MERGE_DS) in 3D: maps and a solve
    within 1e-11 of the oracle at 16^3, L=5."""
    import robinsolver_b200 as rb
    L, N = 5, 16
    T = rb.robin_tree(merge_ds=True)
    T.bndry_params = BP_GEN
    T.factor(L, rb.elliptic_operator(d=3, domain=np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]]), k=bump_potential),
             rb.solve_opts(h_tgt=1.0 / N, kb=1.0))
    O = oracle_tree(L, N, bump_potential, bp=BP_GEN)
    for l in (1, 3, L):
        assert rel_err(T.get_rtr(l, 0), O.levels[l][0].rtr) < 1e-11, l
    T.solve(rb.elliptic_rhs(d=3, f=source, g=plane_faces()))
    O.solve([H.EllipticRHS(3, source, plane_faces())])
    ref = np.stack([u[:, 0] for _, u in O.get_solution()])
    assert rel_err(T.solution_array(0), ref) < 1e-11
    T.close()


@pytest.mark.gpu
def test_gpu3d_save_load_solves_identically(tmp_path):
    import robinsolver_b200 as rb
    T = _gpu_tree(4, 16, bump_potential)
    rhs = rb.elliptic_rhs(d=3, f=source, g=plane_faces())
    T.solve(rhs)
    U = T.solution_array(0)
    T.save(str(tmp_path / "tree3d.bin"))
    T2 = rb.robin_tree.load(str(tmp_path / "tree3d.bin"))
    F, G = T.sample_rhs([rhs])
    T2.solve_samples(F, G)
    assert np.array_equal(T2.solution_array(0), U)
    T.close()
    T2.close()


@pytest.mark.gpu
def test_gpu3d_refuses_2d_only_features():
    """Forests and device-side sampling are 2D only: RB_ERR_UNSUPPORTED, no device fault."""
    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib
    T = _planned3d(3, 8)
    with pytest.raises(rb.RobinSolverError) as ei:
        rb.robin_forest([T])
    assert ei.value.code == _lib.RB_ERR_UNSUPPORTED
    T.close()
    T = _gpu_tree(3, 8, bump_potential)
    with pytest.raises(rb.RobinSolverError) as ei:
        T.sample_device(_lib.RB_FIELD_PLANE_WAVE, 1, [[1.0, 1.0, 0.0]])
    assert ei.value.code == _lib.RB_ERR_UNSUPPORTED
    T.close()
