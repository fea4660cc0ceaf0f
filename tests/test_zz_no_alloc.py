"""GPU test of rb_leaf_rtr_noalloc, the entry point for callers that cannot allocate device memory:
a framework that owns the device's memory through its own pool and forbids allocations by
libraries, or a latency-critical loop that cannot afford cudaMalloc's implicit synchronisation.
Its leaf Robin-to-Robin maps, computed in a static device scratch array, must match the ones the
allocating path produces (rb_tree_factor, read back with rb_tree_get_rtr) within the 1e-11 parity
tolerance of the GPU tests, on two calls in a row that share that array.  This file is collected
last so that a run stopping at the first failure has already run every other test."""
import numpy as np
import pytest

from helpers import gpu_tree, rel_err

pytestmark = pytest.mark.gpu


# (grid N, leaf engine): 16x16 leaves on the tensor-core warp kernel (the default) and on the DFMA
# warp kernel (RB_LEAF_ENGINE=dfma), and 12x12 leaves on the one-CTA-per-leaf kernel
CASES = [(64, None), (64, "dfma"), (48, None)]


@pytest.mark.parametrize("N,engine", CASES, ids=["16x16-tc", "16x16-dfma", "12x12-block"])
def test_noalloc_leaf_rtr_matches_allocating_factor(N, engine, monkeypatch):
    import torch

    from robinsolver_b200 import _lib
    from robinsolver_b200 import workloads as W

    if engine:
        monkeypatch.setenv("RB_LEAF_ENGINE", engine)     # read at every leaf launch
    else:
        monkeypatch.delenv("RB_LEAF_ENGINE", raising=False)
    wl = W.make_workload(1, N=N)                 # L=4: 16 leaves of (N/4)^2
    T, op, opts = gpu_tree(wl)
    T.factor(wl.L, op, opts)
    inf = T.info()
    nl, a, b = inf.nleaves, inf.leaf_a, inf.leaf_b
    assert a == N // 4 and b == N // 4
    nb = 2 * (a + b)
    ref = [T.get_rtr(wl.L, i) for i in range(nl)]
    kv = np.ascontiguousarray(wl.potential(T.sample_points(_lib.RB_POINTS_POTENTIAL)))
    T.close()

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    # dyadic domain: every leaf has the spacing the tree reports for its last leaf
    d_h = torch.tensor(np.tile(np.array(inf.h_last[:2]), nl), dtype=torch.float64, device=dev)
    d_k = torch.from_numpy(kv).to(dev)
    out = torch.empty((nl, nb, nb), dtype=torch.complex128, device=dev)
    torch.cuda.synchronize()
    for call in range(2):
        out.fill_(complex(float("nan"), float("nan")))
        torch.cuda.synchronize()
        rc = _lib.lib.rb_leaf_rtr_noalloc(a, b, opts.kb, d_h.data_ptr(), d_k.data_ptr(), nl, out.data_ptr(), None)
        assert rc == _lib.RB_OK, _lib.last_error(None)
        got = out.cpu().numpy()
        for i in range(nl):
            # each leaf's block is nb x nb column-major: row-major view transposed
            assert rel_err(got[i].T, ref[i]) < 1e-11, (call, i)

    # a batch one leaf beyond the scratch array is refused before any device work, and the
    # largest one that fits is accepted
    per_leaf = (b * a * a + nb * (nb + a * b)) * 16
    limit = (32 * 2 ** 20 - 256) // per_leaf
    rc = _lib.lib.rb_leaf_rtr_noalloc(a, b, opts.kb, d_h.data_ptr(), d_k.data_ptr(), limit + 1, out.data_ptr(), None)
    assert rc == _lib.RB_ERR_INVALID
    assert "limit" in _lib.last_error(None)
    big = limit
    d_hb = torch.tensor(np.tile(np.array(inf.h_last[:2]), big), dtype=torch.float64, device=dev)
    d_kb = d_k.reshape(nl, -1).repeat((big + nl - 1) // nl, 1)[:big].contiguous()
    outb = torch.empty((big, nb, nb), dtype=torch.complex128, device=dev)
    rc = _lib.lib.rb_leaf_rtr_noalloc(a, b, opts.kb, d_hb.data_ptr(), d_kb.data_ptr(), big, outb.data_ptr(), None)
    assert rc == _lib.RB_OK, _lib.last_error(None)
    got = outb.cpu().numpy()
    for i in (0, nl - 1, big - 1):
        assert rel_err(got[i].T, ref[i % nl]) < 1e-11, i
