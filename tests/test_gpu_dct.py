"""GPU parity of the DCT step (performDCT 2 / 3: the radial DCT that feeds the
JW chain) against the __float128 oracle (pfo_dct_q), through the C ABI.

Tolerance: <= 1e-13 relative L2 per row (an FP64 FFT of up to 4096 points;
observed ~1e-15).  Rows of 8 .. 4096 points, batches that leave partial CTA
rounds, in place and out of place, padded strides, launch-time buffers and
strides; the round trip type 3 of type 2 = 2N x at a larger batch; and the
plan's rejections (lengths that are not powers of two, precisions other than
FP64, types other than 2 and 3)."""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _app(N, nsys, dct_type, buf, out=None, **kw):
    from pfsolve_b200.api import App
    return App(buffer=buf, outputBuffer=out, FFTdim=1, size=(N, nsys), performDCT=dct_type, doublePrecision=1, **kw)


def _rows_err(got, ref, N, nsys, so):
    worst = 0.0
    for y in range(nsys):
        g, r = got[y * so:y * so + N], ref[y * so:y * so + N]
        worst = max(worst, float(np.linalg.norm(g - r) / np.linalg.norm(r)))
    return worst


@pytest.mark.parametrize("dct_type", [2, 3])
@pytest.mark.parametrize("N", [8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
def test_dct_against_oracle(N, dct_type):
    import torch

    from pfsolve_b200.api import last_launch, launch_count
    rng = np.random.default_rng(10 * N + dct_type)
    nsys = 37
    x = rng.standard_normal(N * nsys)
    tx = torch.from_numpy(x.copy()).cuda()
    to = torch.zeros_like(tx)
    app = _app(N, nsys, dct_type, tx, to)
    n0 = launch_count()
    app.append()
    torch.cuda.synchronize()
    assert launch_count() == n0 + 1
    assert last_launch()["kernel"] == capi.PFSOLVE_KERNEL_DCT
    got = to.cpu().numpy()
    app.close()
    ref = O.dct(dct_type, x, N, nsys)
    assert _rows_err(got, ref, N, nsys, N) <= TOL
    np.testing.assert_array_equal(tx.cpu().numpy(), x)  # out of place: input untouched


@pytest.mark.parametrize("dct_type", [2, 3])
@pytest.mark.parametrize("N", [8, 64, 512, 4096])
def test_dct_in_place_and_strides(N, dct_type):
    import torch
    rng = np.random.default_rng(N + dct_type)
    nsys, si = 21, N + 6
    x = rng.standard_normal(si * nsys)
    # in place on `buffer` (no outputBuffer), padded stride: the padding stays
    tx = torch.from_numpy(x.copy()).cuda()
    app = _app(N, nsys, dct_type, tx, None, inputBufferStride=si, outputBufferStride=si)
    app.append()
    torch.cuda.synchronize()
    got = tx.cpu().numpy()
    app.close()
    ref = O.dct(dct_type, x, N, nsys, in_stride=si, out_stride=si)
    assert _rows_err(got, ref, N, nsys, si) <= TOL
    for y in range(nsys):
        np.testing.assert_array_equal(got[y * si + N:(y + 1) * si], x[y * si + N:(y + 1) * si])
    # out of place with a different output stride, buffers and strides given at launch
    so = N + 2
    tx = torch.from_numpy(x.copy()).cuda()
    to = torch.zeros(so * nsys, dtype=torch.float64, device="cuda")
    app = _app(N, nsys, dct_type, None, None,
               jw_control_bitmask=capi.RUNTIME_INPUTBUFFERSTRIDE | capi.RUNTIME_OUTPUTBUFFERSTRIDE)
    app.append(buffer=tx, outputBuffer=to, inputBufferStride=si, outputBufferStride=so)
    torch.cuda.synchronize()
    got = to.cpu().numpy()
    app.close()
    ref = O.dct(dct_type, x, N, nsys, in_stride=si, out_stride=so)
    assert _rows_err(got, ref, N, nsys, so) <= TOL


@pytest.mark.parametrize("N", [256, 1024])
def test_dct_round_trip_many_rows(N):
    """Type 3 of type 2 is 2N times the identity, on 20 000 rows (many rows per
    CTA, every round of the persistent grid)."""
    import torch
    rng = np.random.default_rng(N)
    nsys = 20000
    x = torch.from_numpy(rng.standard_normal(N * nsys)).cuda()
    X = torch.empty_like(x)
    y = torch.empty_like(x)
    a2 = _app(N, nsys, 2, x, X)
    a3 = _app(N, nsys, 3, X, y)
    a2.append()
    a3.append()
    torch.cuda.synchronize()
    err = ((y / (2 * N) - x).view(nsys, N).norm(dim=1) / x.view(nsys, N).norm(dim=1)).max().item()
    assert err <= 1e-14, err
    a2.close()
    a3.close()


def test_dct_plan_rejections():
    import torch
    t = torch.zeros(4096, dtype=torch.float64, device="cuda")
    for N, kw, code in [(100, {}, capi.PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_DCT),
                        (8192, {}, capi.PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_DCT),
                        (4, {}, capi.PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_DCT),
                        (64, dict(performDCT=4), capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION),
                        (64, dict(doublePrecision=0), capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION)]:
        args = dict(FFTdim=1, size=(N, 1), performDCT=2, doublePrecision=1)
        args.update(kw)
        from pfsolve_b200.api import App
        with pytest.raises(capi.PfSolveError) as ei:
            App(buffer=t, **args)
        assert ei.value.code == code, (N, kw)
