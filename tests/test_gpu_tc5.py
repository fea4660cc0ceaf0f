"""The tcgen05 split-TF32 complex GEMM of the mixed-precision levels, held directly against a
host FP64 product (run on a GPU).

Tolerance: the split keeps ~22 significant bits of every operand and accumulates in FP32, so
the max-norm error relative to max|A| max|B| k is bounded near 1e-6; the bar is 2e-6 of that
scale.  The FP64 engine on the same problems is held to 1e-13.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(engine, A, B, C0, alpha, beta):
    import torch

    from robinsolver_b200 import _lib
    cnt, m, k = A.shape
    n = B.shape[2]
    dev = torch.device("cuda", 0)
    # column-major per problem: torch row-major (cnt, cols, rows)
    dA = torch.from_numpy(np.ascontiguousarray(A.transpose(0, 2, 1))).to(dev)
    dB = torch.from_numpy(np.ascontiguousarray(B.transpose(0, 2, 1))).to(dev)
    dC = torch.from_numpy(np.ascontiguousarray(C0.transpose(0, 2, 1))).to(dev)
    rc = _lib.lib.rb_test_zgemm(engine, m, n, k, dA.data_ptr(), m, m * k, dB.data_ptr(), k, k * n,
                                dC.data_ptr(), m, m * n, alpha.real, alpha.imag, beta.real, beta.imag, cnt)
    assert rc == 0, (rc, _lib.last_error(None))
    return dC.cpu().numpy().transpose(0, 2, 1)


SHAPES = [(128, 64, 16, 1), (128, 64, 256, 3), (300, 70, 123, 2), (512, 512, 512, 2), (96, 200, 40, 5),
          (1024, 32, 1024, 1), (257, 31, 33, 4)]


@pytest.mark.parametrize("m,n,k,cnt", SHAPES)
def test_tc5_gemm_matches_host_product(m, n, k, cnt):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = rng.standard_normal((cnt, m, k)) + 1j * rng.standard_normal((cnt, m, k))
    B = rng.standard_normal((cnt, k, n)) + 1j * rng.standard_normal((cnt, k, n))
    C0 = rng.standard_normal((cnt, m, n)) + 1j * rng.standard_normal((cnt, m, n))
    alpha, beta = 0.7 - 0.2j, -0.5 + 0.25j
    ref = alpha * (A @ B) + beta * C0
    scale = np.abs(A).max() * np.abs(B).max() * k
    got = _run(1, A, B, C0, alpha, beta)
    err = np.abs(got - ref).max() / scale
    assert err < 2e-6, err
    # and not merely FP32-accurate by accident of cancellation: the plain TF32 bound is ~5e-4
    f64 = _run(0, A, B, C0, alpha, beta)
    assert np.abs(f64 - ref).max() / scale < 1e-13


def test_tc5_gemm_beta_zero_overwrites():
    """beta = 0 overwrites D without reading it (NaN in D stays out of the result)."""
    rng = np.random.default_rng(5)
    m, n, k = 200, 64, 48
    A = rng.standard_normal((1, m, k)) + 1j * rng.standard_normal((1, m, k))
    B = rng.standard_normal((1, k, n)) + 1j * rng.standard_normal((1, k, n))
    C0 = np.full((1, m, n), np.nan + 1j * np.nan)
    got = _run(1, A, B, C0, 1.0 + 0j, 0j)
    ref = A @ B
    assert np.isfinite(got).all()
    assert np.abs(got - ref).max() / (np.abs(A).max() * np.abs(B).max() * k) < 2e-6
