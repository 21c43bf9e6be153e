"""GPU parity of the sm_100a kernels against the oracle, through the C ABI.

Tolerance (FP64 storage and arithmetic): the relative L2 error of every
system against the __float128 oracle is at most 1e-13 for the diagonally
dominant systems used here (the reference's own FP64 PCR reaches 1e-15..8e-15
absolute on such systems); at least one system must be checked.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

import jwcases as J

pytestmark = pytest.mark.gpu
TOL = 1e-13


def jw_case(rng, M, B, ub, jwt, **kw):
    nat = J.random_bands(rng, M, ub)
    bands = WL.permute_bands(nat, M)
    case = O.Case(M=M, batch=B, upperBanded=ub, jw_type=jwt, **kw)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    return case, bands, rhs


@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (1, 11), (1, 12), (1, 13),
                                    (0, 10), (0, 11), (0, 12), (0, 13)])
@pytest.mark.parametrize("M", [1, 7, 32, 33, 100, 256, 257, 512, 1000, 1024])
def test_jw_modes_and_sizes(ub, jwt, M):
    rng = np.random.default_rng(1000 * ub + 10 * jwt + M)
    B = 37
    case, bands, rhs = jw_case(rng, M, B, ub, jwt)
    x = J.run_app(case, bands, rhs)
    ref = O.jw_step(case, bands, rhs, "q")
    e, emax = J.rel_err(x, ref, case)
    assert e <= TOL, (e, emax)


@pytest.mark.parametrize("R", [2, 4, 8, 16])
@pytest.mark.parametrize("M", [64, 300, 1024, 2048, 4096])
def test_rows_per_thread_choices(R, M):
    if -(-M // (32 * R)) > 8 and R < 16:
        pytest.skip("more than 8 warps per system; the plan raises R")
    rng = np.random.default_rng(R * 7 + M)
    case, bands, rhs = jw_case(rng, M, 19, 2, 13)
    x = J.run_app(case, bands, rhs, rowsPerThread=R)
    e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= TOL


def test_runtime_offsets_strides_zeropad_scaleC():
    rng = np.random.default_rng(11)
    M, B = 300, 9
    bm = (capi.RUNTIME_OFFSETM | capi.RUNTIME_OFFSETV | capi.RUNTIME_OFFSETSOLUTION | capi.RUNTIME_INPUTZEROPAD |
          capi.RUNTIME_OUTPUTZEROPAD | capi.RUNTIME_SCALEC | capi.RUNTIME_OUTPUTBUFFERSTRIDE)
    for ub, jwt in [(1, 10), (0, 10), (1, 13), (0, 13), (2, 13)]:
        nat = J.random_bands(rng, M, ub)
        perm = WL.permute_bands(nat, M)  # md = perm[:M], mo = perm[M:2M], solve band = perm[2M:]
        # bands placed at runtime offsets: offsetM region holds the two matvec bands, offsetV the solve band
        big = np.full(8 * M, np.nan)
        oM, oV = 2 * M + 5, 6 * M + 3
        if ub == 2:
            big[:3 * M] = perm
        else:
            md, mo, sv = perm[:M], perm[M:2 * M], perm[2 * M:]
            if jwt % 10 == 3:  # the solve reuses the band loaded beside md
                if ub == 1:
                    big[oM:oM + M] = md
                    big[oM + M:oM + 2 * M] = sv
                else:
                    big[oM + M:oM + 2 * M] = md
                    big[oM:oM + M] = sv
            else:
                if ub == 1:
                    big[oM + M:oM + 2 * M] = md
                    big[oM:oM + M] = mo
                else:
                    big[oM:oM + M] = md
                    big[oM + M:oM + 2 * M] = mo
                big[oV:oV + M] = sv
        big = np.nan_to_num(big, nan=1e300)  # any stray read would blow the error up
        case = O.Case(M=M, batch=B, upperBanded=ub, jw_type=jwt, bitmask=bm, run_offsetM=oM, run_offsetV=oV,
                      run_offsetSolution=17, run_inputZeropad=(3, 280), run_outputZeropad=(10, 250),
                      run_scaleC=0.75, run_outputBufferStride=M + 128)
        rhs = rng.uniform(-1, 1, case.rhs_len() + 64)
        x = J.run_app(case, big, rhs)
        ref = O.jw_step(case, big, rhs, "q")
        e, _ = J.rel_err(x, ref, case)
        assert e <= TOL, (ub, jwt, e)
        # rows outside the output window keep their input values
        np.testing.assert_array_equal(x[:17], rhs[:17])


def test_plan_time_values():
    rng = np.random.default_rng(12)
    M, B = 200, 5
    case, bands, rhs = jw_case(rng, M, B, 2, 13, cfg_offsetSolution=8, cfg_outputBufferStride=M + 16,
                               cfg_inputZeropad=(4, 0), cfg_outputZeropad=(0, 150), cfg_scaleC=2.0)
    x = J.run_app(case, bands, rhs)
    e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= TOL


def test_empty_windows_and_batch():
    rng = np.random.default_rng(13)
    M = 64
    case, bands, rhs = jw_case(rng, M, 4, 2, 13, bitmask=capi.RUNTIME_OUTPUTZEROPAD, run_outputZeropad=(5, 5))
    x = J.run_app(case, bands, rhs)
    np.testing.assert_array_equal(x, rhs)  # nothing written


def test_unsupported_combinations_return_codes():
    import torch

    from pfsolve_b200.api import App
    b = torch.zeros(3 * 64, dtype=torch.float64, device="cuda")
    r = torch.zeros(64, dtype=torch.float64, device="cuda")
    for fields, code in [(dict(upperBanded=2, jw_type=10), capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION),
                         (dict(upperBanded=2, jw_type=12), capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION),
                         # K > 2 tridiagonal steps: the reference never reloads the middle steps' diagonal
                         (dict(upperBanded=2, jw_type=13, numConsecutiveJWIterations=3),
                          capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION),
                         # ALT mode with launch-time band offsets
                         (dict(upperBanded=2, jw_type=113, jw_control_bitmask=capi.RUNTIME_OFFSETM),
                          capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION)]:
        with pytest.raises(capi.PfSolveError) as ei:
            App(buffer=b, outputBuffer=r, M_size=64, size=(64, 1), doublePrecision=1, **fields)
        assert ei.value.code == code
    # longer than 64 slices of 1024 rows, in either long-system form
    for M, path in ((65544, 0), (65544, 3)):
        with pytest.raises(capi.PfSolveError) as ei:
            App(buffer=b, outputBuffer=r, M_size=M, size=(M, 1), doublePrecision=1, upperBanded=2, jw_type=13,
                kernelPath=path)
        assert ei.value.code == capi.PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH


@pytest.mark.parametrize("KL,KU", [(1, 1), (2, 2), (0, 1), (2, 1), (3, 3), (0, 6)])
@pytest.mark.parametrize("M", [33, 256, 1000])
def test_dgbmv_app(KL, KU, M):
    rng = np.random.default_rng(KL * 100 + KU * 10 + M)
    B = 11
    A = WL.band_major(rng, M, KL, KU)
    case = O.Case(M=M, batch=B, LDA=KL + KU + 1, KU=KU, KL=KL, jw_type=0)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    y = J.run_app(case, A, rhs)
    ref = O.dgbmv(case, A, rhs)
    e, _ = J.rel_err(y, ref, case)
    assert e <= 1e-14


@pytest.mark.parametrize("block", [1, 2, 3, 4, 5, 6, 7, 21, 27, 101, 201, 301, 401, 307, 325])
def test_block_app(block):
    rng = np.random.default_rng(block)
    N, Y = 130, 7
    bt = block % 10
    cin = bt in (2, 3, 4)
    cout = bt in (5, 6, 7)
    iS, oS = N + 3, N + 5
    n_in = (2 if (cin or bt == 7) else 1) * (Y * iS + 8)
    n_out = (2 if (cout or bt == 4) else 1) * (Y * oS + 8)
    inp = rng.standard_normal(n_in)
    out0 = rng.standard_normal(n_out)
    case = O.Case(M=N, batch=Y, block=block, lshift=2, jw_type=0, cfg_inputBufferStride=iS, cfg_outputBufferStride=oS,
                  bitmask=capi.RUNTIME_SCALEC | capi.RUNTIME_INPUTZEROPAD, run_scaleC=0.5,
                  run_inputZeropad=(2, 120))
    got = J.run_app(case, inp, out0)
    ref = O.block(case, inp, out0)
    np.testing.assert_allclose(got, ref, rtol=1e-14, atol=1e-300)


def test_chain_dgbmv_jw_config1_form():
    """config 1 at full size: 3-band V then upper-bidiagonal M, fused."""
    import torch

    from pfsolve_b200.api import App, append_chain
    wl = WL.config1()
    M, B = wl.M, wl.nrhs
    tA = torch.from_numpy(wl.dgbmv).cuda()
    tb = torch.from_numpy(wl.jw_bands).cuda()
    tr = torch.from_numpy(wl.rhs.copy()).cuda()
    dg = App(buffer=tA, outputBuffer=tr, M_size=M, size=(M, B), LDA=3, KU=1, KL=1, doublePrecision=1, scaleC=1.0)
    jw = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, B), upperBanded=0, jw_type=13, doublePrecision=1, scaleC=1.0)
    append_chain([dg, jw], [dg.launch_params(), jw.launch_params()])
    torch.cuda.synchronize()
    x = tr.cpu().numpy()
    c1 = O.Case(M=M, batch=B, LDA=3, KU=1, KL=1, jw_type=0)
    y = O.dgbmv(c1, wl.dgbmv, wl.rhs)
    c2 = O.Case(M=M, batch=B, upperBanded=0, jw_type=13)
    ref = O.jw_step(c2, wl.jw_bands, y, "q")
    e, _ = O.rel_errors(x, ref, M, B, M)
    assert e <= TOL
    # unfused chain gives the same answer within rounding
    tr2 = torch.from_numpy(wl.rhs.copy()).cuda()
    dg2 = App(buffer=tA, outputBuffer=tr2, M_size=M, size=(M, B), LDA=3, KU=1, KL=1, doublePrecision=1, scaleC=1.0)
    jw2 = App(buffer=tb, outputBuffer=tr2, M_size=M, size=(M, B), upperBanded=0, jw_type=13, doublePrecision=1, scaleC=1.0)
    dg2.append()
    jw2.append()
    torch.cuda.synchronize()
    e2, _ = O.rel_errors(tr2.cpu().numpy(), ref, M, B, M)
    assert e2 <= TOL


def _config2_chain(wl, ncplx, scale_block=7, lshift=0):
    import torch

    from pfsolve_b200.api import App, append_chain
    M = wl.M
    tA = torch.from_numpy(wl.dgbmv).cuda()
    tb = torch.from_numpy(wl.jw_bands).cuda()
    rhs = wl.rhs[:2 * M * ncplx].copy()
    tr = torch.from_numpy(rhs).cuda()
    tout = torch.zeros(2 * M * ncplx, dtype=torch.float64, device="cuda")
    dg = App(buffer=tA, outputBuffer=tr, M_size=M, size=(M, 2 * ncplx), LDA=5, KU=2, KL=2, doublePrecision=1, scaleC=1.0)
    jw = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, 2 * ncplx), upperBanded=2, jw_type=13, doublePrecision=1, scaleC=1.0)
    bl = App(buffer=tr, outputBuffer=tout, M_size=M, size=(M, ncplx), block=scale_block, lshift=lshift,
             jw_control_bitmask=capi.RUNTIME_SCALEC, doublePrecision=1)
    append_chain([dg, jw, bl], [dg.launch_params(), jw.launch_params(), bl.launch_params(scaleC=0.5)])
    torch.cuda.synchronize()
    return rhs, tout.cpu().numpy()


@pytest.mark.parametrize("block,lshift", [(7, 0), (307, 3)])
def test_chain_config2_form(block, lshift):
    wl = WL.config2(B=64)
    M, Y = wl.M, 64
    rhs, got = _config2_chain(wl, Y, block, lshift)
    c1 = O.Case(M=M, batch=2 * Y, LDA=5, KU=2, KL=2, jw_type=0)
    y = O.dgbmv(c1, wl.dgbmv, rhs)
    c2 = O.Case(M=M, batch=2 * Y, upperBanded=2, jw_type=13)
    x = O.jw_step(c2, wl.jw_bands, y, "q")
    cb = O.Case(M=M, batch=Y, block=block, lshift=lshift, jw_type=0, bitmask=O.RUNTIME_SCALEC, run_scaleC=0.5)
    ref = O.block(cb, x, np.zeros(2 * M * Y))
    got_c = got.reshape(Y, M, 2)
    ref_c = ref.reshape(Y, M, 2)
    for y_ in range(Y):
        num = np.linalg.norm(got_c[y_] - ref_c[y_])
        den = np.linalg.norm(ref_c[y_])
        assert num / den <= TOL


def test_config3_full_size_sampled():
    """config 3 at full size (N=512, 131072 RHS): every system solved on the
    GPU; a seeded sample of 96 systems checked against the __float128 oracle,
    and the whole batch checked by linearity (solve(b) for b = e_k sums)."""
    import torch

    from pfsolve_b200.api import App
    wl = WL.config3()
    M, B = wl.M, wl.nrhs
    tb = torch.from_numpy(wl.jw_bands).cuda()
    tr = torch.from_numpy(wl.rhs).cuda()
    app = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=1, scaleC=1.0)
    app.append()
    torch.cuda.synchronize()
    x = tr.view(B, M)
    pick = np.random.default_rng(99).choice(B, 96, replace=False)
    sub_rhs = wl.rhs.reshape(B, M)[pick].ravel()
    case = O.Case(M=M, batch=96, upperBanded=2, jw_type=13)
    ref = O.jw_step(case, wl.jw_bands, sub_rhs, "q")
    e, _ = O.rel_errors(x[torch.from_numpy(pick).cuda()].cpu().numpy().ravel(), ref, M, 96, M)
    assert e <= TOL
    # size-independent property: A x = b for every system (residual in the
    # normalised form md*b - (x + ld x_{i-1} + ud x_{i+1}), FP64 on the GPU)
    nat = torch.zeros(3 * M, dtype=torch.float64, device="cuda")
    perm = torch.from_numpy(WL.reference_band_order(M)).cuda()
    for k in range(3):
        nat[k * M:(k + 1) * M] = tb[k * M + perm]
    ld, md, ud = nat[:M], nat[M:2 * M], nat[2 * M:]
    b = torch.from_numpy(wl.rhs).cuda().view(B, M)
    r = md * b - x
    r[:, 1:] -= ld[1:] * x[:, :-1]
    r[:, :-1] -= ud[:-1] * x[:, 1:]
    rel = (r.norm(dim=1) / (md * b).norm(dim=1)).max().item()
    assert rel <= 1e-13


# ---------------------------------------------------------------------------
# Mixed precision: FP32 factor-solve + FP64 residual refinement (FP64 storage).
# Bound: 1e-12 relative L2 against the __float128 oracle after 2 refinement
# sweeps on the weakly dominant config-3 system (the accuracy the mixed mode
# is meant to reach); one sweep is allowed 1e-10.

@pytest.mark.parametrize("refine,tol", [(1, 1e-10), (2, 1e-12), (3, 1e-12)])
def test_mixed_precision_config3(refine, tol):
    import torch

    from pfsolve_b200.api import App
    wl = WL.config3(B=512)
    M, B = wl.M, wl.nrhs
    tb = torch.from_numpy(wl.jw_bands).cuda()
    tr = torch.from_numpy(wl.rhs.copy()).cuda()
    app = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=1,
              scaleC=1.0, mixedPrecisionRefinement=refine)
    app.append()
    torch.cuda.synchronize()
    case = O.Case(M=M, batch=B, upperBanded=2, jw_type=13)
    ref = O.jw_step(case, wl.jw_bands, wl.rhs, "q")
    e, _ = O.rel_errors(tr.cpu().numpy(), ref, M, B, M)
    assert e <= tol, e


@pytest.mark.parametrize("ub,jwt", [(1, 10), (0, 10), (1, 12), (0, 12), (1, 13), (0, 13)])
@pytest.mark.parametrize("M", [100, 300, 1000])
def test_mixed_precision_bidiagonal(ub, jwt, M):
    rng = np.random.default_rng(500 + 10 * ub + jwt + M)
    case, bands, rhs = jw_case(rng, M, 23, ub, jwt)
    x = J.run_app(case, bands, rhs, mixedPrecisionRefinement=2)
    e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= 1e-12, e


def test_mixed_precision_chain_config1_form():
    import torch

    from pfsolve_b200.api import App, append_chain
    wl = WL.config1(B=128)
    M, B = wl.M, wl.nrhs
    tA = torch.from_numpy(wl.dgbmv).cuda()
    tb = torch.from_numpy(wl.jw_bands).cuda()
    tr = torch.from_numpy(wl.rhs.copy()).cuda()
    dg = App(buffer=tA, outputBuffer=tr, M_size=M, size=(M, B), LDA=3, KU=1, KL=1, doublePrecision=1)
    jw = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, B), upperBanded=0, jw_type=13, doublePrecision=1,
             scaleC=1.0, mixedPrecisionRefinement=2)
    append_chain([dg, jw], [dg.launch_params(), jw.launch_params()])
    torch.cuda.synchronize()
    y = O.dgbmv(O.Case(M=M, batch=B, LDA=3, KU=1, KL=1, jw_type=0), wl.dgbmv, wl.rhs)
    ref = O.jw_step(O.Case(M=M, batch=B, upperBanded=0, jw_type=13), wl.jw_bands, y, "q")
    e, _ = O.rel_errors(tr.cpu().numpy(), ref, M, B, M)
    assert e <= 1e-12, e
