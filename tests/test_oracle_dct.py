"""The DCT-step oracle (pfo_dct_q): FFTW's unnormalized REDFT10 (type 2) and
REDFT01 (type 3) definitions, summed directly in __float128.

Checked here on the CPU against the same definitions written with numpy in
double (the closed-form cosine sums), against Makhoul's FFT-based evaluation
(numpy.fft) that the GPU kernel follows, and by the round trip
type 3 of type 2 = 2N x.  There is no reference output to pin it on: the
transform belongs to the VkFFT that PfSolve grew out of, whose generators are
not part of the reference, so these definitions are the contract.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _dct2_direct(x):
    N = x.shape[-1]
    n = np.arange(N)
    C = np.cos(np.pi * np.outer(n, 2 * n + 1) / (2 * N))
    return 2.0 * x @ C.T


def _dct3_direct(X):
    N = X.shape[-1]
    n = np.arange(N)
    C = np.cos(np.pi * np.outer(2 * n + 1, n) / (2 * N))  # [k, j] -> cos(pi j (2k+1) / 2N)
    return X[..., :1] + 2.0 * X[..., 1:] @ C[:, 1:].T


def _dct2_makhoul(x):
    N = x.shape[-1]
    v = np.empty_like(x)
    v[..., : N // 2] = x[..., 0::2]
    v[..., N // 2:] = x[..., 1::2][..., ::-1]
    k = np.arange(N)
    return 2.0 * np.real(np.exp(-1j * np.pi * k / (2 * N)) * np.fft.fft(v, axis=-1))


@pytest.mark.parametrize("N", [2, 8, 16, 64, 128, 500, 1024])
def test_dct_oracle_definitions(N):
    rng = np.random.default_rng(N)
    nsys = 5
    x = rng.standard_normal((nsys, N))
    X = O.dct(2, x.ravel(), N, nsys).reshape(nsys, N)
    ref2 = _dct2_direct(x)
    assert np.abs(X - ref2).max() <= 1e-12 * np.abs(ref2).max()
    if N % 2 == 0:
        mk = _dct2_makhoul(x)
        assert np.abs(X - mk).max() <= 1e-12 * np.abs(mk).max()
    Y = O.dct(3, X.ravel(), N, nsys).reshape(nsys, N)
    ref3 = _dct3_direct(X)
    assert np.abs(Y - ref3).max() <= 1e-12 * np.abs(ref3).max()
    # the round trip in __float128 is exact to the rounding of X and Y
    assert np.abs(Y - 2 * N * x).max() <= 1e-14 * 2 * N * np.abs(x).max()


def test_dct_oracle_strides_and_types():
    rng = np.random.default_rng(3)
    N, nsys, si, so = 16, 4, 21, 19
    x = rng.standard_normal(si * nsys)
    X = O.dct(2, x, N, nsys, in_stride=si, out_stride=so)
    for y in range(nsys):
        assert np.allclose(X[y * so:y * so + N], _dct2_direct(x[y * si:y * si + N]), rtol=0, atol=1e-12)
    with pytest.raises(ValueError):
        O.dct(4, x, N, nsys)
