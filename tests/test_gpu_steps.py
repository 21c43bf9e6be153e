"""GPU parity of the K-step JW kernel (numConsecutiveJWIterations = K > 1)
through the C ABI, against the oracle's K-step restatement (itself pinned on
the reference's own K-step outputs, tests/test_golden_steps.py).  Tolerance:
relative L2 <= 1e-13 per system, as for the single-step kernels."""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

import jwcases as J

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _errs(x, ref, case, Mrows):
    S, off = case.out_stride, case.offset_solution
    e = 0.0
    for y in range(case.batch):
        a = x[off + y * S: off + y * S + Mrows]
        b = ref[off + y * S: off + y * S + Mrows]
        e = max(e, np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    return e


def _case(rng, M, B, ub, jwt, K, **kw):
    bands = WL.steps_bands(rng, M, ub, K)
    kw.setdefault("cfg_outputBufferStride", (M + K + 2) // 2 * 2)  # even: 16-byte-aligned rows
    case = O.Case(M=M, batch=B, upperBanded=ub, jw_type=jwt, **kw)
    rhs = rng.uniform(-1, 1, case.rhs_len() + K + 2)
    return case, bands, rhs


KINDS = [(1, 10), (1, 11), (1, 12), (0, 10), (0, 11), (0, 12)]


@pytest.mark.parametrize("ub,jwt", KINDS)
@pytest.mark.parametrize("K", [2, 4, 8])
@pytest.mark.parametrize("M", [17, 128, 512, 1000, 2048])
def test_steps_modes_sizes(ub, jwt, K, M):
    rng = np.random.default_rng(20000 + 100 * ub + jwt + 7 * K + M)
    case, bands, rhs = _case(rng, M, 37, ub, jwt, K)
    ref = O.jw_steps(case, K, bands, rhs)
    for path in (0, 1):  # one system per lane (TMA sweep) / the K-step kernel
        try:
            x, shape = J.run_steps(case, K, bands, rhs, kernelPath=path)
        except capi.PfSolveError as e:
            # the step tables of long systems may not fit shared memory
            assert e.code == capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION and M * K > 8000, (M, K, path)
            continue
        if path == 0 and shape["streaming"] == 4:
            assert shape["tma_launches"] == 1
        else:
            assert shape["streaming"] == 3 and shape["tma_launches"] == 0
        assert _errs(x, ref, case, M + K) <= TOL, path
        # rows beyond the system slots are untouched
        assert np.array_equal(x[case.rhs_len() + K:], rhs[case.rhs_len() + K:])


@pytest.mark.parametrize("M", [100, 1024, 2047])
def test_steps_tridiagonal_two_steps(M):
    rng = np.random.default_rng(21000 + M)
    case, bands, rhs = _case(rng, M, 65, 2, 13, 2)
    x, shape = J.run_steps(case, 2, bands, rhs)
    assert shape["streaming"] == 3
    assert _errs(x, O.jw_steps(case, 2, bands, rhs), case, M) <= TOL


def test_steps_long_system_two_steps():
    rng = np.random.default_rng(21500)
    for ub, jwt in [(1, 10), (0, 10), (2, 13)]:
        M = 4096 if ub else 4095
        case, bands, rhs = _case(rng, M, 9, ub, jwt, 2)
        x, shape = J.run_steps(case, 2, bands, rhs, kernelPath=1)
        assert shape["streaming"] == 3 and shape["rowsPerThread"] == 16
        assert _errs(x, O.jw_steps(case, 2, bands, rhs), case, M + 1) <= TOL


def test_steps_one_buffer_and_windows_and_offsets():
    rng = np.random.default_rng(22000)
    M, K = 300, 3  # odd offsets: the K-step kernel; even ones: the sweep kernel
    bm = (capi.RUNTIME_OFFSETSOLUTION | capi.RUNTIME_INPUTZEROPAD | capi.RUNTIME_OUTPUTZEROPAD |
          capi.RUNTIME_SCALEC | capi.RUNTIME_OUTPUTBUFFERSTRIDE)
    for ub in (0, 1):
        buf = WL.steps_bands(rng, M, ub, K, per_step=False)
        # odd solution offset: rows are not 16-byte aligned (scalar accesses)
        for off in (3, 4):
            case = O.Case(M=M, batch=5, upperBanded=ub, jw_type=10, bitmask=bm, run_offsetSolution=off,
                          run_inputZeropad=(2, 290), run_outputZeropad=(1, 295), run_scaleC=0.5,
                          run_outputBufferStride=M + K + 5)
            rhs = rng.uniform(-1, 1, case.rhs_len() + K + 8)
            x, _ = J.run_steps(case, K, buf, rhs)
            ref = O.jw_steps(case, K, buf, rhs)
            assert np.abs(x - ref).max() <= 1e-13 * np.abs(ref).max()


def test_steps_many_systems():
    rng = np.random.default_rng(23000)
    for ub in (0, 1):
        for B in (1, 2, 33, 1001, 20000):
            case, bands, rhs = _case(rng, 512, B, ub, 10, 4)
            x, shape = J.run_steps(case, 4, bands, rhs)
            assert shape["tma_launches"] == 1
            assert _errs(x, O.jw_steps(case, 4, bands, rhs, nthreads=8), case, 512 + 3) <= TOL


def test_steps_sweep_sizes_and_ks():
    """Every K up to 8 and sizes around the boxes (16 rows up to K = 4, 8
    above), both sweep directions."""
    rng = np.random.default_rng(23500)
    for ub in (0, 1):
        for K in range(2, 9):
            for M in (9, 15, 16, 17, 31, 32, 33, 63, 257):
                if M - K + 1 < 1:
                    continue
                case, bands, rhs = _case(rng, M, 70, ub, 10, K)
                x, shape = J.run_steps(case, K, bands, rhs)
                assert shape["tma_launches"] == 1, (ub, K, M)
                assert _errs(x, O.jw_steps(case, K, bands, rhs), case, M + K) <= TOL, (ub, K, M)


def test_steps_rejected_combinations():
    rng = np.random.default_rng(24000)
    # launch-time band offsets with K > 1 crash the reference's plan creation
    cases = [((2, 13, 3), {}), ((1, 13, 2), {}), ((1, 10, 9), {}), ((1, 10, 2), dict(mixedPrecisionRefinement=2)),
             ((0, 10, 3), dict(useMultipleInputBuffers_override=2)),
             ((1, 10, 2), dict(jw_control_bitmask=capi.RUNTIME_OFFSETM)),
             ((0, 10, 2), dict(jw_control_bitmask=capi.RUNTIME_OFFSETV))]
    for (ub, jwt, K), extra in cases:
        case, bands, rhs = _case(rng, 64, 2, ub, jwt, min(K, 8))
        import torch

        from pfsolve_b200.api import App
        tbs = [torch.from_numpy(b).cuda() for b in bands]
        to = torch.from_numpy(rhs).cuda()
        nbuf = extra.pop("useMultipleInputBuffers_override", len(tbs))
        with pytest.raises(capi.PfSolveError) as ei:
            App(buffer=tbs, outputBuffer=to, numConsecutiveJWIterations=K, useMultipleInputBuffers=nbuf,
                **J.case_fields(case, **extra))
        assert ei.value.code == capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION, (ub, jwt, K)


def test_steps_device_status_clean():
    from pfsolve_b200.api import device_status
    assert device_status() == 0
