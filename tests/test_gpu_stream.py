"""GPU parity of the streaming (TMA-staged) JW kernel, through the C ABI.

Every case checks three things: the plan chose the streaming kernel and the
launch ran on it (PfSolveStreamingLaunchCount), the result matches the
__float128 oracle within the FP64 tolerance of the group kernel's tests
(relative L2 <= 1e-13 per system), and it agrees with the group kernel
(kernelPath = 1) on the same inputs.  Launches whose buffers do not allow the
streaming layout (odd row offsets, partial output windows, accumulation) must
fall back to the group kernel and stay correct.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

import jwcases as J

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _run(case, bands, rhs, **extra):
    from pfsolve_b200.api import streaming_launch_count
    n0 = streaming_launch_count()
    x = J.run_app(case, bands, rhs, **extra)
    return x, streaming_launch_count() - n0


def _case(rng, M, B, ub, jwt, **kw):
    nat = J.random_bands(rng, M, ub)
    bands = WL.permute_bands(nat, M)
    case = O.Case(M=M, batch=B, upperBanded=ub, jw_type=jwt, **kw)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    return case, bands, rhs


@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (1, 11), (1, 12), (1, 13),
                                    (0, 10), (0, 11), (0, 12), (0, 13)])
@pytest.mark.parametrize("M", [256, 512, 1000, 1024, 2048, 4096])
def test_streaming_modes_and_sizes(ub, jwt, M):
    rng = np.random.default_rng(7000 + 100 * ub + jwt + M)
    case, bands, rhs = _case(rng, M, 301, ub, jwt)
    x, n = _run(case, bands, rhs)
    assert n == 1, "the launch did not run on the streaming kernel"
    ref = O.jw_step(case, bands, rhs, "q")
    e, emax = J.rel_err(x, ref, case)
    assert e <= TOL, (e, emax)
    xg, ng = _run(case, bands, rhs, kernelPath=1)
    assert ng == 0
    eg, _ = J.rel_err(x, xg, case)
    assert eg <= TOL


@pytest.mark.parametrize("R", [8, 16, 32])
@pytest.mark.parametrize("M", [256, 1024, 4096])
def test_streaming_rows_per_thread(R, M):
    W = -(-M // (32 * R))
    if W not in (1, 2, 4):
        pytest.skip("no streaming variant with that many warps per system")
    rng = np.random.default_rng(R + M)
    case, bands, rhs = _case(rng, M, 77, 2, 13)
    x, n = _run(case, bands, rhs, rowsPerThread=R)
    assert n == 1
    e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= TOL


def test_plan_shape_reports_streaming():
    import torch

    from pfsolve_b200.api import App
    M, B = 1024, 8
    tb = torch.zeros(3 * M, dtype=torch.float64, device="cuda")
    tr = torch.zeros(M * B, dtype=torch.float64, device="cuda")
    app = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=1)
    sh = app.shape()
    assert sh["streaming"] == 1 and sh["rowsPerThread"] * sh["warpsPerSystem"] * 32 >= M and sh["groupsPerCTA"] >= 1
    app.close()
    app = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=1,
              kernelPath=1)
    assert app.shape()["streaming"] == 0
    app.close()


def test_batch_not_multiple_of_groups_and_single_system():
    rng = np.random.default_rng(5)
    for B in (1, 2, 1001, 4097):
        case, bands, rhs = _case(rng, 512, B, 2, 13)
        x, n = _run(case, bands, rhs)
        assert n == 1
        e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
        assert e <= TOL


def test_input_window_partial_stays_streaming():
    rng = np.random.default_rng(6)
    M = 1024
    for ub, jwt in [(2, 13), (1, 10), (0, 11)]:
        case, bands, rhs = _case(rng, M, 65, ub, jwt, bitmask=capi.RUNTIME_INPUTZEROPAD, run_inputZeropad=(3, 1000))
        x, n = _run(case, bands, rhs)
        assert n == 1
        e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
        assert e <= TOL


def test_fallbacks_to_group_kernel():
    """Odd row offset (rows not 16-byte aligned), odd stride, partial output
    window: the group kernel runs, results stay exact."""
    rng = np.random.default_rng(8)
    M, B = 512, 33
    cases = [
        dict(bitmask=capi.RUNTIME_OFFSETSOLUTION, run_offsetSolution=3),
        dict(bitmask=capi.RUNTIME_OUTPUTBUFFERSTRIDE, run_outputBufferStride=M + 1),
        dict(bitmask=capi.RUNTIME_OUTPUTZEROPAD, run_outputZeropad=(5, 400)),
    ]
    for kw in cases:
        case, bands, rhs = _case(rng, M, B, 2, 13, **kw)
        x, n = _run(case, bands, rhs)
        assert n == 0, kw
        e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
        assert e <= TOL, kw


def test_even_offset_and_stride_stay_streaming():
    rng = np.random.default_rng(9)
    M, B = 512, 40
    case, bands, rhs = _case(rng, M, B, 2, 13,
                             bitmask=capi.RUNTIME_OFFSETSOLUTION | capi.RUNTIME_OUTPUTBUFFERSTRIDE,
                             run_offsetSolution=6, run_outputBufferStride=M + 10)
    x, n = _run(case, bands, rhs)
    assert n == 1
    e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= TOL


def _chain(wl, Y, block, lshift, **extra):
    import torch

    from pfsolve_b200.api import App, append_chain, streaming_launch_count
    M = wl.M
    tA = torch.from_numpy(wl.dgbmv).cuda()
    tb = torch.from_numpy(wl.jw_bands).cuda()
    rhs = wl.rhs[:2 * M * Y].copy()
    tr = torch.from_numpy(rhs).cuda()
    tout = torch.zeros(2 * M * Y, dtype=torch.float64, device="cuda")
    dg = App(buffer=tA, outputBuffer=tr, M_size=M, size=(M, 2 * Y), LDA=5, KU=2, KL=2, doublePrecision=1, scaleC=1.0)
    jw = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, 2 * Y), upperBanded=2, jw_type=13, doublePrecision=1,
             scaleC=1.0, **extra)
    bl = App(buffer=tr, outputBuffer=tout, M_size=M, size=(M, Y), block=block, lshift=lshift,
             jw_control_bitmask=capi.RUNTIME_SCALEC, doublePrecision=1)
    n0 = streaming_launch_count()
    append_chain([dg, jw, bl], [dg.launch_params(), jw.launch_params(), bl.launch_params(scaleC=0.5)])
    torch.cuda.synchronize()
    n = streaming_launch_count() - n0
    return rhs, tout.cpu().numpy(), n


@pytest.mark.parametrize("R", [0, 16, 32])
@pytest.mark.parametrize("block,lshift", [(7, 0), (307, 3)])
def test_streaming_chain_config2_form(R, block, lshift):
    wl = WL.config2(B=130)
    M, Y = wl.M, 130
    rhs, got, n = _chain(wl, Y, block, lshift, rowsPerThread=R)
    assert n == 1
    c1 = O.Case(M=M, batch=2 * Y, LDA=5, KU=2, KL=2, jw_type=0)
    y = O.dgbmv(c1, wl.dgbmv, rhs)
    c2 = O.Case(M=M, batch=2 * Y, upperBanded=2, jw_type=13)
    x = O.jw_step(c2, wl.jw_bands, y, "q")
    cb = O.Case(M=M, batch=Y, block=block, lshift=lshift, jw_type=0, bitmask=O.RUNTIME_SCALEC, run_scaleC=0.5)
    ref = O.block(cb, x, np.zeros(2 * M * Y)).reshape(Y, M, 2)
    got = got.reshape(Y, M, 2)
    e = max(np.linalg.norm(got[k] - ref[k]) / np.linalg.norm(ref[k]) for k in range(Y))
    assert e <= TOL
    _, got_g, ng = _chain(wl, Y, block, lshift, kernelPath=1)
    assert ng == 0
    eg = max(np.linalg.norm(got[k] - got_g.reshape(Y, M, 2)[k]) / np.linalg.norm(ref[k]) for k in range(Y))
    assert eg <= TOL


def test_device_status_clean():
    from pfsolve_b200.api import device_status
    assert device_status() == 0


# Mixed precision on the streaming kernel: FP32 solves with FP64 residual
# refinement; <= 1e-12 relative L2 after two refinement sweeps (1e-10 after
# one) against the __float128 oracle, as for the group kernel.
@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (1, 12), (1, 13), (0, 10), (0, 12), (0, 13)])
@pytest.mark.parametrize("M", [256, 512, 1024, 4096])
def test_streaming_mixed_precision(ub, jwt, M):
    rng = np.random.default_rng(8100 + 10 * ub + jwt + M)
    case, bands, rhs = _case(rng, M, 129, ub, jwt)
    ref = O.jw_step(case, bands, rhs, "q")
    for refine, tol in ((1, 1e-10), (2, 1e-12)):
        x, n = _run(case, bands, rhs, mixedPrecisionRefinement=refine)
        assert n == 1, "the mixed launch did not run on the streaming kernel"
        e, _ = J.rel_err(x, ref, case)
        assert e <= tol, (refine, e)


def test_streaming_mixed_config3_weakly_dominant():
    wl = WL.config3(B=256)
    case = O.Case(M=wl.M, batch=wl.nrhs, upperBanded=2, jw_type=13)
    ref = O.jw_step(case, wl.jw_bands, wl.rhs, "q")
    x, n = _run(case, wl.jw_bands, wl.rhs, mixedPrecisionRefinement=2)
    assert n == 1
    e, _ = J.rel_err(x, ref, case)
    assert e <= 1e-12, e
    xg, ng = _run(case, wl.jw_bands, wl.rhs, mixedPrecisionRefinement=2, kernelPath=1)
    assert ng == 0
    assert J.rel_err(xg, ref, case)[0] <= 1e-12


def test_streaming_mixed_chain_config2_form():
    wl = WL.config2(B=64)
    M, Y = wl.M, 64
    rhs, got, n = _chain(wl, Y, 7, 0, mixedPrecisionRefinement=2)
    assert n == 1
    c1 = O.Case(M=M, batch=2 * Y, LDA=5, KU=2, KL=2, jw_type=0)
    y = O.dgbmv(c1, wl.dgbmv, rhs)
    c2 = O.Case(M=M, batch=2 * Y, upperBanded=2, jw_type=13)
    x = O.jw_step(c2, wl.jw_bands, y, "q")
    cb = O.Case(M=M, batch=Y, block=7, jw_type=0, bitmask=O.RUNTIME_SCALEC, run_scaleC=0.5)
    ref = O.block(cb, x, np.zeros(2 * M * Y)).reshape(Y, M, 2)
    got = got.reshape(Y, M, 2)
    e = max(np.linalg.norm(got[k] - ref[k]) / np.linalg.norm(ref[k]) for k in range(Y))
    assert e <= 1e-12, e


@pytest.mark.parametrize("nb", [0, 2, 3, 4])
@pytest.mark.parametrize("refine", [0, 2])
@pytest.mark.parametrize("M,B,ub,jwt", [(512, 4097, 2, 13), (1024, 3001, 1, 10), (256, 6000, 0, 13)])
def test_staging_buffers(nb, refine, M, B, ub, jwt):
    """stagingBuffers (TMA staging buffers per group, 2-4; 0: the default):
    enough systems that every group cycles through its buffers many times,
    FP64 and the mixed mode (2 refinement sweeps), against the __float128
    oracle (1e-13; mixed: 1e-12)."""
    rng = np.random.default_rng(M + B + nb + refine)
    case, bands, rhs = _case(rng, M, B, ub, jwt)
    x, n = _run(case, bands, rhs, stagingBuffers=nb, mixedPrecisionRefinement=refine)
    assert n == 1, "the launch did not run on the streaming kernel"
    e, emax = J.rel_err(x, O.jw_step(case, bands, rhs, "q", nthreads=8), case)
    assert e <= (1e-12 if refine else TOL), (e, emax)
