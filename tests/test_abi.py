"""CPU tests of the C-ABI library: it loads, exports what include/robin_b200.h declares, and its
host-side plan (tree geometry, sample points, validation) matches the oracle.  No device calls."""
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import hps_ref as H
from robinsolver_b200 import workloads as W

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    from robinsolver_b200 import _lib
    hdr = (ROOT / "include" / "robin_b200.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|double|void\*|const char\*)\s+(rb_\w+)\s*\(", hdr, re.M))
    assert declared == set(_lib.EXPORTS)
    for name in declared:
        assert hasattr(_lib.lib, name), name


def _planned(wl):
    import robinsolver_b200 as rb
    T = rb.robin_tree()
    T.bndry_params = wl.bndry_params
    T.plan(wl.L, rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential),
           rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb))
    return T


@pytest.mark.parametrize("cfg,leaves,n,root_nb", [(1, 16, 320, 256), (2, 1024, 320, 2048), (4, 4096, 320, 4096)])
def test_plan_sizes(cfg, leaves, n, root_nb):
    T = _planned(W.make_workload(cfg))
    inf = T.info()
    assert (inf.nleaves, inf.leaf_n, inf.root_nb, inf.leaf_a, inf.leaf_b) == (leaves, n, root_nb, 16, 16)
    assert inf.device_bytes == 0 and inf.factored == 0
    T.close()


@pytest.mark.parametrize("cfg,kw", [(1, {}), (2, dict(N=128, L=6)), (1, dict(N=48, L=3))])
def test_sample_points_match_oracle(cfg, kw):
    from robinsolver_b200 import _lib
    wl = W.make_workload(cfg, **kw)
    T = _planned(wl)
    root, levels = H.build_tree(wl.L, wl.domain, 2)
    leaves = levels[-1]
    grids = [H.get_h(wl.h_tgt, lf.box, 2) for lf in leaves]
    hl, gl = grids[-1]
    a, b = gl[0], gl[1]
    pot = np.concatenate([H.interior_points(g[0], g[1], h, lf.box) for (h, g), lf in zip(grids, leaves)])
    src = np.concatenate([H.interior_points(a, b, hl, lf.box) for lf in leaves])
    bnd = np.concatenate([H.face_points(a, b, hl, lf.box, f) for f in range(1, 5) for lf in leaves if lf.isbndry[f - 1]])
    sol = np.concatenate([H.leaf_all_points(a, b, hl, lf.box) for lf in leaves])
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_POTENTIAL), pot)
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_SOURCE), src)
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_BOUNDARY), bnd)
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_SOLUTION), sol)
    for l in range(wl.L + 1):
        assert T._level_grid(l)[:2] == tuple(levels[l][0].ptbox[:2]) if levels[l][0].ptbox else True
    T.close()


def test_level_grids_match_oracle_ptbox():
    wl = W.make_workload(1)
    T = _planned(wl)
    O = H.RobinTree()
    O.bndry_params = wl.bndry_params
    O.factor(wl.L, H.EllipticOperator(2, wl.domain, wl.potential), H.SolveOpts(h_tgt=wl.h_tgt, kb=wl.opts_kb))
    for l in range(wl.L + 1):
        assert T._level_grid(l) == (*O.levels[l][0].ptbox[:2], 1)
    T.close()


def _expect(code, fn):
    import robinsolver_b200 as rb
    with pytest.raises(rb.RobinSolverError) as ei:
        fn()
    assert ei.value.code == code
    return str(ei.value)


def test_validation_errors_match_reference_messages():
    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib
    wl = W.make_workload(1)
    op = rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential)
    opts = rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb)
    T = rb.robin_tree()
    T.bndry_params = np.array([[1.0, 2.0], [0.5, 1.0]], dtype=complex)        # det = 0
    msg = _expect(_lib.RB_ERR_BNDRY_PARAMS, lambda: T.plan(4, op, opts))
    assert "nearly singular" in msg
    T.bndry_params = wl.bndry_params
    bad = rb.elliptic_operator(d=2, domain=np.array([[0, 0, 0], [-1, 1, 1.0]]), k=wl.potential)
    assert "Invalid operator domain" in _expect(_lib.RB_ERR_DOMAIN, lambda: T.plan(4, bad, opts))
    assert "Dimension" in _expect(_lib.RB_ERR_DOMAIN, lambda: T.plan(4, rb.elliptic_operator(d=4), opts))
    _expect(_lib.RB_ERR_INVALID, lambda: T.plan(4, op, rb.solve_opts(h_tgt=wl.h_tgt, kb=1.0, ordering=2)))
    T.plan(4, op, opts)
    assert "factored first" in _expect(_lib.RB_ERR_NOT_FACTORED, lambda: T.solve(rb.elliptic_rhs()))
    T.close()


def test_device_budget_refusal_happens_before_any_device_call():
    import robinsolver_b200 as rb
    from robinsolver_b200 import _lib
    wl = W.make_workload(4)
    T = rb.robin_tree(device_budget=1 << 30)
    T.bndry_params = wl.bndry_params
    msg = _expect(_lib.RB_ERR_OUT_OF_MEMORY,
                  lambda: T.plan(wl.L, rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential),
                                 rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb)))
    assert "budget" in msg


@pytest.mark.parametrize("h_tgt,uniform", [(0.0123, True), (0.02, False)])
def test_non_dyadic_domain_plans_like_the_oracle(h_tgt, uniform):
    """On [0.1,0.7]x[-0.3,0.5] with h_tgt = 0.02 the rounded leaf widths give leaf grids of 15 and
    16 points (the oracle's get_h agrees); the reference would stop with "Interface sizes of node
    children do not match", this build refuses at plan time.  h_tgt = 0.0123 is uniform."""
    from robinsolver_b200 import _lib
    import robinsolver_b200 as rb
    dom = np.array([[0.1, -0.3, 0.0], [0.7, 0.5, 1.0]])
    root, levels = H.build_tree(3, dom, 2)
    leaves = levels[-1]
    grids = [H.get_h(h_tgt, lf.box, 2) for lf in leaves]
    assert (len(set(tuple(g[:2]) for _, g in grids)) == 1) == uniform
    T = rb.robin_tree()
    T.bndry_params = W.make_workload(1).bndry_params
    op = rb.elliptic_operator(d=2, domain=dom, k=None)
    opts = rb.solve_opts(h_tgt=h_tgt, kb=-5.0)
    if not uniform:
        assert "Interface sizes" in _expect(_lib.RB_ERR_GEOMETRY, lambda: T.plan(3, op, opts))
        return
    T.plan(3, op, opts)
    pot = np.concatenate([H.interior_points(g[0], g[1], h, lf.box) for (h, g), lf in zip(grids, leaves)])
    assert np.array_equal(T.sample_points(_lib.RB_POINTS_POTENTIAL), pot)
    T.close()


def test_load_refuses_missing_and_foreign_files(tmp_path):
    import ctypes
    from robinsolver_b200 import _lib
    h = ctypes.c_void_p()
    assert _lib.lib.rb_tree_load(str(tmp_path / "none.rbt").encode(), ctypes.byref(h)) == _lib.RB_ERR_INVALID
    assert "cannot open" in _lib.last_error(None)
    bad = tmp_path / "bad.rbt"
    bad.write_bytes(b"not a tree" * 20)
    assert _lib.lib.rb_tree_load(str(bad).encode(), ctypes.byref(h)) == _lib.RB_ERR_INVALID
    assert "not a factorized tree" in _lib.last_error(None)


def test_load_refuses_another_file_version(tmp_path):
    """A file of this library's magic but another format version (version 1 lacked the levels'
    [Y1; Y2]) is refused from its header, before any device work."""
    import ctypes
    import struct
    from robinsolver_b200 import _lib
    old = tmp_path / "v1.rbt"
    old.write_bytes(b"RBTREEF1" + struct.pack("<II", 1, ctypes.sizeof(_lib.rb_geom)) + bytes(1024))
    h = ctypes.c_void_p()
    assert _lib.lib.rb_tree_load(str(old).encode(), ctypes.byref(h)) == _lib.RB_ERR_INVALID
    assert "not a factorized tree" in _lib.last_error(None)
    assert not h.value


def test_save_needs_a_factorization(tmp_path):
    import robinsolver_b200 as rb
    from robinsolver_b200 import workloads as W
    wl = W.make_workload(1)
    T = rb.robin_tree()
    T.bndry_params = wl.bndry_params
    T.plan(wl.L, rb.elliptic_operator(d=2, domain=wl.domain, k=wl.potential), rb.solve_opts(h_tgt=wl.h_tgt, kb=wl.opts_kb))
    with pytest.raises(rb.RobinSolverError):
        T.save(tmp_path / "t.rbt")
    T.close()
