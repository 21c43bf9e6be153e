"""FP32-storage precisions on the GPU, through the C ABI: the reference's
default precision (FP32 storage and arithmetic, doublePrecision = 0) and
doublePrecisionFloatMemory (FP64 arithmetic on FP32 storage)
(PfSolve/pfSolve_PlanManagement/pfSolve_API_handles/pfSolve_InitAPIParameters.h:148-245,
pfSolve_Plans/pfSolve_Plan_JonesWorland.h:244-264).

Oracle: the same FP32 inputs through the __float128 restatement, rounded to
FP32 at the end.  Tolerances (relative L2 per system):
  * FP64 arithmetic on FP32 storage: 3e-7 -- the result is the FP64 step
    rounded once to FP32, so it differs from the rounded oracle by at most
    about an FP32 unit in the last place (2^-23 = 1.2e-7) per value;
  * FP32 arithmetic: 2e-5 on the diagonally dominant systems used here (the
    reference's own FP32 kernel is within 2e-6 of the oracle on its golden
    vector; this build's FP32 solve orders its operations differently).
"""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

import jwcases as J

pytestmark = pytest.mark.gpu
F32, F32MEM = "f32", "f32mem"
TOL = {F32: 2e-5, F32MEM: 3e-7}


def prec_fields(prec):
    return dict(doublePrecision=0, doublePrecisionFloatMemory=1 if prec == F32MEM else 0)


def run_f32(case, buffer, out, prec, **extra):
    """One app on FP32 buffers; returns (output buffer, launch info)."""
    import torch

    from pfsolve_b200.api import App, last_launch
    tb = torch.from_numpy(np.ascontiguousarray(buffer, dtype=np.float32)).cuda()
    to = torch.from_numpy(np.array(out, dtype=np.float32, copy=True)).cuda()
    fields = J.case_fields(case, **extra)
    fields.update(prec_fields(prec))
    app = App(buffer=tb, outputBuffer=to, **fields)
    app.append(**J.launch_fields(case))
    torch.cuda.synchronize()
    info = last_launch()
    res = to.cpu().numpy()
    app.close()
    return res, info


def rel(x, ref, case):
    return O.rel_errors(np.asarray(x, np.float64), np.asarray(ref, np.float64), case.M, case.batch, case.out_stride,
                        case.offset_solution)[0]


def jw_case32(rng, M, B, ub, jwt, **kw):
    bands = WL.permute_bands(J.random_bands(rng, M, ub), M).astype(np.float32)
    case = O.Case(M=M, batch=B, upperBanded=ub, jw_type=jwt, **kw)
    rhs = rng.uniform(-1, 1, case.rhs_len()).astype(np.float32)
    return case, bands, rhs


@pytest.mark.parametrize("prec", [F32, F32MEM])
@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (1, 11), (1, 12), (1, 13), (0, 10), (0, 11), (0, 12), (0, 13)])
@pytest.mark.parametrize("M", [7, 64, 256, 1000, 1024])
def test_jw_modes(prec, ub, jwt, M):
    rng = np.random.default_rng(7000 + 100 * ub + jwt + M)
    case, bands, rhs = jw_case32(rng, M, 41, ub, jwt)
    x, info = run_f32(case, bands, rhs, prec)
    assert info["precision"] == (4 if prec == F32 else 5)
    ref = O.jw_step(case, bands, rhs, "f32")
    e = rel(x, ref, case)
    assert e <= TOL[prec], (e, info)


@pytest.mark.parametrize("prec", [F32, F32MEM])
@pytest.mark.parametrize("nb", [0, 2, 3, 4])
def test_staging_buffers(prec, nb):
    """stagingBuffers 2-4 (0: the default, three for FP32 storage and
    arithmetic where they fit beside as many groups as two) on the streaming
    kernel's steady state."""
    rng = np.random.default_rng(610 + nb)
    case, bands, rhs = jw_case32(rng, 512, 8193, 2, 13)
    x, info = run_f32(case, bands, rhs, prec, stagingBuffers=nb)
    assert info["kernel"] == capi.PFSOLVE_KERNEL_STREAMING, info
    ref = O.jw_step(case, bands, rhs, "f32", nthreads=8)
    assert rel(x, ref, case) <= TOL[prec]


@pytest.mark.parametrize("prec", [F32, F32MEM])
@pytest.mark.parametrize("M,B", [(512, 4097), (2048, 300), (4096, 150)])
@pytest.mark.parametrize("path", [0, 1])
def test_streaming_and_group_kernels(prec, M, B, path):
    """Many systems per group (the streaming kernel's steady state), and the
    group kernel (kernelPath 1) on the same inputs."""
    rng = np.random.default_rng(M + B + path)
    case, bands, rhs = jw_case32(rng, M, B, 2, 13)
    x, info = run_f32(case, bands, rhs, prec, kernelPath=path)
    want = capi.PFSOLVE_KERNEL_GROUP if path == 1 else capi.PFSOLVE_KERNEL_STREAMING
    assert info["kernel"] == want, info
    ref = O.jw_step(case, bands, rhs, "f32", nthreads=8)
    assert rel(x, ref, case) <= TOL[prec]


@pytest.mark.parametrize("prec", [F32, F32MEM])
def test_runtime_offsets_strides_zeropad_scaleC(prec):
    """Odd runtime offsets and strides (not 16-byte aligned in FP32: the group
    kernel), keep-windows and scaleC."""
    rng = np.random.default_rng(31)
    M, B = 300, 9
    bm = (capi.RUNTIME_OFFSETSOLUTION | capi.RUNTIME_INPUTZEROPAD | capi.RUNTIME_OUTPUTZEROPAD |
          capi.RUNTIME_SCALEC | capi.RUNTIME_OUTPUTBUFFERSTRIDE)
    for ub, jwt in [(1, 10), (0, 13), (2, 13)]:
        case, bands, _ = jw_case32(rng, M, B, ub, jwt, bitmask=bm, run_offsetSolution=17,
                                   run_inputZeropad=(3, 280), run_outputZeropad=(10, 250), run_scaleC=0.75,
                                   run_outputBufferStride=M + 129)
        rhs = rng.uniform(-1, 1, case.rhs_len() + 64).astype(np.float32)
        x, info = run_f32(case, bands, rhs, prec)
        assert info["kernel"] == capi.PFSOLVE_KERNEL_GROUP
        ref = O.jw_step(case, bands, rhs, "f32")
        assert rel(x, ref, case) <= TOL[prec], (ub, jwt)
        np.testing.assert_array_equal(x[:17], rhs[:17])


@pytest.mark.parametrize("prec", [F32, F32MEM])
@pytest.mark.parametrize("KL,KU", [(1, 1), (2, 2), (0, 1), (3, 3)])
def test_dgbmv(prec, KL, KU):
    """dgbmv on FP32 storage against the oracle's FP64-storage dgbmv of the
    same (FP32-representable) values, rounded to FP32."""
    rng = np.random.default_rng(KL * 10 + KU)
    M, B = 257, 13
    A = WL.band_major(rng, M, KL, KU).astype(np.float32)
    case = O.Case(M=M, batch=B, LDA=KL + KU + 1, KU=KU, KL=KL, jw_type=0)
    rhs = rng.uniform(-1, 1, case.rhs_len()).astype(np.float32)
    y, info = run_f32(case, A, rhs, prec)
    ref = O.dgbmv(case, A.astype(np.float64), rhs.astype(np.float64)).astype(np.float32)
    assert rel(y, ref, case) <= (TOL[prec] if prec == F32 else 3e-7), info


@pytest.mark.parametrize("prec", [F32, F32MEM])
@pytest.mark.parametrize("block", [1, 2, 4, 7, 21, 27, 101, 301, 401])
def test_block(prec, block):
    rng = np.random.default_rng(block)
    N, Y = 130, 7
    bt = block % 10
    cin, cout = bt in (2, 3, 4), bt in (5, 6, 7)
    iS, oS = N + 3, N + 5
    n_in = (2 if (cin or bt == 7) else 1) * (Y * iS + 8)
    n_out = (2 if (cout or bt == 4) else 1) * (Y * oS + 8)
    inp = rng.standard_normal(n_in).astype(np.float32)
    out0 = rng.standard_normal(n_out).astype(np.float32)
    case = O.Case(M=N, batch=Y, block=block, lshift=2, jw_type=0, cfg_inputBufferStride=iS, cfg_outputBufferStride=oS,
                  bitmask=capi.RUNTIME_SCALEC | capi.RUNTIME_INPUTZEROPAD, run_scaleC=0.5, run_inputZeropad=(2, 120))
    got, info = run_f32(case, inp, out0, prec)
    assert info["kernel"] == capi.PFSOLVE_KERNEL_BLOCK
    ref = O.block(case, inp.astype(np.float64), out0.astype(np.float64)).astype(np.float32)
    # FP64 products rounded once to FP32: one unit in the last place at most
    np.testing.assert_allclose(got, ref, rtol=2.5e-7, atol=1e-30)


@pytest.mark.parametrize("prec", [F32, F32MEM])
def test_chain_config2_form(prec):
    """dgbmv(5) -> tridiagonal JW -> block 7 (XXII -> packed) fused on FP32
    storage, on the streaming kernel."""
    import torch

    from pfsolve_b200.api import App, append_chain, last_launch
    wl = WL.config2(B=300)
    M, Y = wl.M, 300
    A32, b32 = wl.dgbmv.astype(np.float32), wl.jw_bands.astype(np.float32)
    rhs = wl.rhs[:2 * M * Y].astype(np.float32)
    tA, tb = torch.from_numpy(A32).cuda(), torch.from_numpy(b32).cuda()
    tr = torch.from_numpy(rhs.copy()).cuda()
    tout = torch.zeros(2 * M * Y, dtype=torch.float32, device="cuda")
    pf = prec_fields(prec)
    dg = App(buffer=tA, outputBuffer=tr, M_size=M, size=(M, 2 * Y), LDA=5, KU=2, KL=2, **pf)
    jw = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, 2 * Y), upperBanded=2, jw_type=13, scaleC=1.0, **pf)
    bl = App(buffer=tr, outputBuffer=tout, M_size=M, size=(M, Y), block=7, **pf)
    append_chain([dg, jw, bl], [dg.launch_params(), jw.launch_params(), bl.launch_params()])
    torch.cuda.synchronize()
    info = last_launch()
    assert (info["kernel"], info["layoutIn"], info["layoutOut"]) == (capi.PFSOLVE_KERNEL_STREAMING, 1, 2), info
    got = tout.cpu().numpy().reshape(Y, M * 2).astype(np.float64)
    y = O.dgbmv(O.Case(M=M, batch=2 * Y, LDA=5, KU=2, KL=2, jw_type=0), A32.astype(np.float64),
                rhs.astype(np.float64))
    x = O.jw_step(O.Case(M=M, batch=2 * Y, upperBanded=2, jw_type=13), b32.astype(np.float64), y, "q", nthreads=8)
    ref = O.block(O.Case(M=M, batch=Y, block=7, jw_type=0), x, np.zeros(2 * M * Y)).reshape(Y, -1)
    e = (np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)).max()
    # FP64 arithmetic: only the storage roundings (inputs exact, output once); FP32: its arithmetic too
    assert e <= (2e-5 if prec == F32 else 3e-7), e


def test_precision_precedence_and_rejections():
    """doublePrecision wins over doublePrecisionFloatMemory (FP64 storage), as
    in the reference; the FP32-storage precisions reject the modes they do
    not cover (mixed refinement, K > 1, ALT, long systems)."""
    import torch

    from pfsolve_b200.api import App
    b = torch.zeros(3 * 64, dtype=torch.float64, device="cuda")
    r = torch.zeros(64, dtype=torch.float64, device="cuda")
    app = App(buffer=b, outputBuffer=r, M_size=64, size=(64, 1), upperBanded=2, jw_type=13, doublePrecision=1,
              doublePrecisionFloatMemory=1, scaleC=1.0)
    app.append()
    torch.cuda.synchronize()
    from pfsolve_b200.api import last_launch
    assert last_launch()["precision"] == 0
    app.close()
    for fields in (dict(mixedPrecisionRefinement=2), dict(numConsecutiveJWIterations=2, upperBanded=1, jw_type=10),
                   dict(jw_type=113), dict(M_size=8192, size=(8192, 1))):
        f = dict(M_size=64, size=(64, 1), upperBanded=2, jw_type=13, doublePrecision=0)
        f.update(fields)
        with pytest.raises(capi.PfSolveError) as ei:
            App(buffer=b, outputBuffer=r, **f)
        assert ei.value.code in (capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION, capi.PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH)
