"""The tcgen05 complex GEMM of the mixed-precision levels, in both of its arithmetics, held directly
against a host FP64 product (run on a GPU).

Tolerances, as max-norm error relative to max|A| max|B| k:
- split TF32 (engine 1) keeps ~22 significant bits of every operand and accumulates in FP32:
  bounded near 1e-6, bar 2e-6;
- int8 digit slices (engine 2, the default) keep 35 bits of every row-scaled (A) or column-scaled
  (B) operand and accumulate exactly in int32: the error is about 2^-35 of
  max|A_i.| max|B_.j| k per element; bar 1e-10 of that row/column scale.
The FP64 engine on the same problems is held to 1e-13.
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
    got8 = _run(2, A, B, C0, alpha, beta)
    assert np.abs(got8 - ref).max() / scale < 1e-10


def _rowcol_scale(A, B):
    """max|A_i.| max|B_.j| k per output element, (cnt, m, n)."""
    ra = np.abs(A).max(axis=2)
    cb = np.abs(B).max(axis=1)
    return ra[:, :, None] * cb[:, None, :] * A.shape[2]


@pytest.mark.parametrize("m,n,k,cnt", [(256, 100, 96, 3), (130, 49, 700, 2), (64, 300, 33, 1)])
def test_int8_engine_scales_rows_and_columns(m, n, k, cnt):
    """Rows of A and columns of B spanning 2^-40 .. 2^40 in magnitude (and an all-zero row): each
    output element keeps its own row/column-relative accuracy, which a single global scale would
    lose."""
    rng = np.random.default_rng(k)
    A = (rng.standard_normal((cnt, m, k)) + 1j * rng.standard_normal((cnt, m, k))) * \
        np.exp2(rng.uniform(-40, 40, (cnt, m, 1)))
    B = (rng.standard_normal((cnt, k, n)) + 1j * rng.standard_normal((cnt, k, n))) * \
        np.exp2(rng.uniform(-40, 40, (cnt, 1, n)))
    A[:, 3, :] = 0.0
    C0 = np.zeros((cnt, m, n), dtype=np.complex128)
    ref = A @ B
    got = _run(2, A, B, C0, 1.0 + 0j, 0j)
    err = (np.abs(got - ref) / np.maximum(_rowcol_scale(A, B), 1e-300)).max()
    assert err < 1e-10, err
    assert (got[:, 3, :] == 0).all()


def test_tc5_gemm_beta_zero_overwrites():
    """beta = 0 overwrites D without reading it (NaN in D stays out of the result)."""
    rng = np.random.default_rng(5)
    m, n, k = 200, 64, 48
    A = rng.standard_normal((1, m, k)) + 1j * rng.standard_normal((1, m, k))
    B = rng.standard_normal((1, k, n)) + 1j * rng.standard_normal((1, k, n))
    C0 = np.full((1, m, n), np.nan + 1j * np.nan)
    ref = A @ B
    for engine, bar in ((1, 2e-6), (2, 1e-10)):
        got = _run(engine, A, B, C0.copy(), 1.0 + 0j, 0j)
        assert np.isfinite(got).all()
        assert np.abs(got - ref).max() / (np.abs(A).max() * np.abs(B).max() * k) < bar
