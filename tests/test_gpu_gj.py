"""The batched Gauss-Jordan inversion of the interface systems, held directly against a host
inverse (run on a GPU): every size path (whole-matrix m <= 32, resident panels above), batches,
a leading dimension above m, and matrices that need row exchanges on every panel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _invert(A, ld=None, reps=1):
    import torch

    from robinsolver_b200 import _lib
    cnt, m, _ = A.shape
    ld = ld or m
    buf = np.zeros((cnt, m, ld), dtype=np.complex128)        # per matrix: m columns of ld rows
    buf[:, :, :m] = A.transpose(0, 2, 1)
    d = torch.from_numpy(buf).to(torch.device("cuda", 0))
    ms = _lib.C.c_double()
    rc = _lib.lib.rb_test_zinvert(m, cnt, d.data_ptr(), ld, m * ld, reps, _lib.C.byref(ms))
    assert rc == 0, (rc, _lib.last_error(None))
    out = d.cpu().numpy()[:, :, :m].transpose(0, 2, 1)
    return out, ms.value


def _matrices(m, cnt, seed, permute):
    rng = np.random.default_rng(seed)
    A = (rng.standard_normal((cnt, m, m)) + 1j * rng.standard_normal((cnt, m, m))) / np.sqrt(m)
    A += (2.0 + 1.0j) * np.eye(m)
    if permute:
        # a row permutation moves the dominant entries off the diagonal: every pivot is an exchange
        for i in range(cnt):
            A[i] = A[i][rng.permutation(m)]
    return A


@pytest.mark.parametrize("m,cnt", [(16, 7), (32, 3), (40, 5), (64, 4), (100, 3), (128, 6), (200, 2), (256, 8),
                                   (300, 2), (512, 4), (700, 1), (1024, 1), (1024, 2)])
@pytest.mark.parametrize("permute", [False, True])
def test_gj_inverse_matches_host(m, cnt, permute):
    A = _matrices(m, cnt, 11 * m + cnt, permute)
    X, _ = _invert(A)
    ref = np.linalg.inv(A)
    for i in range(cnt):
        err = np.abs(X[i] - ref[i]).max() / np.abs(ref[i]).max()
        assert err < 1e-12, (i, err)


def test_gj_leading_dimension_and_repeat():
    A = _matrices(300, 3, 5, True)
    X, ms = _invert(A, ld=320, reps=2)       # inverting twice returns the input
    assert ms > 0.0
    assert np.abs(X - A).max() / np.abs(A).max() < 1e-12
