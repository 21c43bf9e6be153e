"""GPU parity of ALT stride-2 mode (jw_type / 100 % 10 == 1) through the C
ABI: the streaming kernel (FP64, whole row sets staged by TMA, both parities
solved together) and the group kernel with one parity per group, against the
oracle's ALT restatement (pinned on the reference's ALT outputs,
tests/test_golden_alt.py).
FP64 to 1e-13 relative L2 per system; mixed precision to 1e-12 after two
refinement sweeps."""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

import jwcases as J

pytestmark = pytest.mark.gpu


def _errs(x, ref, case):
    S, off, M = case.out_stride, case.offset_solution, case.M
    return max(np.linalg.norm(x[off + y * S: off + y * S + M] - ref[off + y * S: off + y * S + M]) /
               max(np.linalg.norm(ref[off + y * S: off + y * S + M]), 1e-300) for y in range(case.batch))


KINDS = [(2, 113), (1, 110), (1, 111), (1, 112), (1, 113), (0, 110), (0, 111), (0, 112), (0, 113)]


@pytest.mark.parametrize("ub,jwt", KINDS)
@pytest.mark.parametrize("M", [2, 3, 64, 255, 512, 1001, 4096, 8192])
def test_alt_modes_sizes(ub, jwt, M):
    rng = np.random.default_rng(30000 + 10 * ub + jwt + M)
    bands = WL.alt_bands(rng, M, ub)
    case = O.Case(M=M, batch=37, upperBanded=ub, jw_type=jwt)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    x = J.run_app(case, bands, rhs)
    assert _errs(x, O.jw_step_alt(case, bands, rhs), case) <= 1e-13


@pytest.mark.parametrize("ub,jwt", KINDS)
@pytest.mark.parametrize("M", [64, 512, 1000, 2048, 4096])
def test_alt_streaming_kernel(ub, jwt, M):
    """FP64 ALT on the streaming kernel (a row set staged by TMA, its even and
    odd systems solved together): one streaming launch, against the oracle
    and against the group kernel (kernelPath 1)."""
    from pfsolve_b200.api import streaming_launch_count
    rng = np.random.default_rng(36000 + 10 * ub + jwt + M)
    bands = WL.alt_bands(rng, M, ub)
    case = O.Case(M=M, batch=301, upperBanded=ub, jw_type=jwt)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    n0 = streaming_launch_count()
    x = J.run_app(case, bands, rhs)
    assert streaming_launch_count() == n0 + 1
    assert _errs(x, O.jw_step_alt(case, bands, rhs, nthreads=8), case) <= 1e-13
    xg = J.run_app(case, bands, rhs, kernelPath=1)
    assert streaming_launch_count() == n0 + 1
    assert np.abs(x - xg).max() <= 1e-13 * np.abs(xg).max()


@pytest.mark.parametrize("off", [3, 4])
def test_alt_streaming_input_window_scaleC(off):
    """Launch-time input window, scaleC and solution offset on the streaming
    ALT kernel (offset 4: 16-byte-aligned row sets, streamed; offset 3: the
    group kernel takes the launch)."""
    from pfsolve_b200.api import streaming_launch_count
    rng = np.random.default_rng(37000 + off)
    M = 320
    bm = capi.RUNTIME_OFFSETSOLUTION | capi.RUNTIME_INPUTZEROPAD | capi.RUNTIME_SCALEC
    for ub, jwt in [(2, 113), (1, 110), (0, 110), (1, 111), (0, 112)]:
        case = O.Case(M=M, batch=9, upperBanded=ub, jw_type=jwt, bitmask=bm, run_offsetSolution=off,
                      run_inputZeropad=(3, 290), run_scaleC=0.5)
        bands = WL.alt_bands(rng, M, ub)
        rhs = rng.uniform(-1, 1, case.rhs_len() + 8)
        n0 = streaming_launch_count()
        x = J.run_app(case, bands, rhs)
        assert streaming_launch_count() == n0 + (1 if off == 4 else 0)
        ref = O.jw_step_alt(case, bands, rhs)
        assert np.abs(x - ref).max() <= 1e-13 * np.abs(ref).max(), (ub, jwt)


def test_alt_windows_offsets_scaleC():
    rng = np.random.default_rng(31000)
    M = 300
    bm = (capi.RUNTIME_OFFSETSOLUTION | capi.RUNTIME_INPUTZEROPAD | capi.RUNTIME_OUTPUTZEROPAD |
          capi.RUNTIME_SCALEC | capi.RUNTIME_OUTPUTBUFFERSTRIDE)
    for ub, jwt in [(2, 113), (1, 110), (0, 110)]:
        for off in (3, 4):
            case = O.Case(M=M, batch=5, upperBanded=ub, jw_type=jwt, bitmask=bm, run_offsetSolution=off,
                          run_inputZeropad=(3, 290), run_outputZeropad=(1, 297), run_scaleC=0.5,
                          run_outputBufferStride=M + 5)
            bands = WL.alt_bands(rng, M, ub)
            rhs = rng.uniform(-1, 1, case.rhs_len() + 8)
            x = J.run_app(case, bands, rhs)
            ref = O.jw_step_alt(case, bands, rhs)
            assert np.abs(x - ref).max() <= 1e-13 * np.abs(ref).max(), (ub, off)


def test_alt_many_systems():
    """Batches of 1, 2, odd and large sizes: every group keeps one parity."""
    rng = np.random.default_rng(32000)
    M = 1000
    bands = WL.alt_bands(rng, M, 2)
    for B in (1, 2, 3, 999, 40000):
        case = O.Case(M=M, batch=B, upperBanded=2, jw_type=113)
        rhs = rng.uniform(-1, 1, case.rhs_len())
        x = J.run_app(case, bands, rhs)
        assert _errs(x, O.jw_step_alt(case, bands, rhs, nthreads=8), case) <= 1e-13, B


@pytest.mark.parametrize("ub,jwt", [(2, 113), (1, 110), (0, 110)])
def test_alt_mixed_precision(ub, jwt):
    rng = np.random.default_rng(33000 + ub)
    M = 512
    bands = WL.alt_bands(rng, M, ub)
    case = O.Case(M=M, batch=65, upperBanded=ub, jw_type=jwt)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    x = J.run_app(case, bands, rhs, mixedPrecisionRefinement=2)
    assert _errs(x, O.jw_step_alt(case, bands, rhs), case) <= 1e-12


def test_alt_rejected():
    import torch

    from pfsolve_b200.api import App
    rng = np.random.default_rng(34000)
    M = 64
    bands = torch.from_numpy(WL.alt_bands(rng, M, 1)).cuda()
    x = torch.zeros(M * 2, dtype=torch.float64, device="cuda")
    for extra in (dict(numConsecutiveJWIterations=2), dict(jw_control_bitmask=capi.RUNTIME_OFFSETM),
                  dict(quadDoubleDoublePrecisionDoubleMemory=1), dict(M_size=8194, size=(8194, 2))):
        kw = dict(M_size=M, size=(M, 2), upperBanded=1, jw_type=110, doublePrecision=1)
        kw.update(extra)
        with pytest.raises(capi.PfSolveError):
            App(buffer=bands, outputBuffer=x, **kw)


@pytest.mark.parametrize("KL,KU", [(0, 2), (0, 1), (2, 0), (1, 0), (3, 0), (2, 2), (1, 1), (0, 6), (5, 0)])
@pytest.mark.parametrize("M", [33, 256, 1000])
def test_alt_dgbmv(KL, KU, M):
    """ALT_dgbmv: alternate bands of the general band matrix dropped, on the
    fused-weight group/streaming kernels (KL, KU <= 2) and the generic one."""
    rng = np.random.default_rng(35000 + 100 * KL + 10 * KU + M)
    A = WL.band_major(rng, M, KL, KU)
    case = O.Case(M=M, batch=11, LDA=KL + KU + 1, KU=KU, KL=KL, jw_type=0, ALT_dgbmv=1)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    ref = O.dgbmv(case, A, rhs)
    x = J.run_app(case, A, rhs)
    assert np.abs(x - ref).max() <= 1e-13 * max(np.abs(ref).max(), 1e-300)


def test_alt_device_status_clean():
    from pfsolve_b200.api import device_status
    assert device_status() == 0
