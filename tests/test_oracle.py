"""The oracle checked against independent dense linear algebra and against the
reference's own band layout (CPU only)."""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import workloads as WL


@pytest.mark.parametrize("M", [1, 2, 7, 31, 32, 33, 100, 255, 256, 257, 511, 512, 513, 1000, 1024, 2048, 4352,
                               4353, 4360, 5000, 6144, 8192, 12000, 16383, 16384])
def test_band_order_matches_reference_formula(M):
    perm_c = O.permutation(M)
    perm_py = WL.reference_band_order(M)
    assert sorted(perm_c.tolist()) == list(range(M))
    np.testing.assert_array_equal(perm_c, perm_py)


def test_band_order_register_major_small():
    # M=100 -> 32 lanes, r = 4 rows per lane, 25 lanes active: row t*4+j at j*25+t
    perm = O.permutation(100)
    for t in range(25):
        for j in range(4):
            assert perm[4 * t + j] == j * 25 + t


def _dense(a, d, c):
    M = d.shape[0]
    return np.diag(d) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)


@pytest.mark.parametrize("M", [1, 2, 5, 64, 100, 300])
def test_tridiagonal_matches_dense(M):
    rng = np.random.default_rng(M)
    a, d, c = WL.tridiagonal(rng, M)
    B = 3
    bands = WL.permute_bands(WL.tri_bands(a, d, c), M)
    rhs = rng.uniform(-1, 1, M * B)
    case = O.Case(M=M, batch=B, upperBanded=2, jw_type=13)
    x = O.jw_step(case, bands, rhs, "q")
    ref = np.linalg.solve(_dense(a, d, c), rhs.reshape(B, M).T).T.ravel()
    assert np.abs(x - ref).max() < 1e-12


def _jw_dense(ub, jwt, md, mo, sl, su, M):
    """Dense operator of one JW step in natural order."""
    V = np.eye(M)
    if jwt % 10 != 2:
        if jwt % 10 == 3:
            V = np.diag(md)
        elif ub == 1:
            V = np.diag(md) + np.diag(mo[:-1], 1)
        else:
            V = np.diag(md) + np.diag(mo[1:], -1)
    S = np.eye(M)
    if jwt % 10 != 1:
        if ub == 1:
            S = np.eye(M) + np.diag(sl[1:], -1)
        elif ub == 0:
            S = np.eye(M) + np.diag(su[:-1], 1)
        else:
            S = np.eye(M) + np.diag(sl[1:], -1) + np.diag(su[:-1], 1)
    return np.linalg.solve(S, V)


@pytest.mark.parametrize("ub", [0, 1])
@pytest.mark.parametrize("jwt", [10, 11, 12, 13])
@pytest.mark.parametrize("M", [40, 257])
def test_bidiagonal_modes_match_dense(ub, jwt, M):
    rng = np.random.default_rng(ub * 100 + jwt + M)
    # every band may act as a solve band in some mode: |entries| < 1/2 keeps the
    # unit-diagonal recurrences stable
    nat = rng.uniform(-.5, .5, 3 * M)
    bands = WL.permute_bands(nat, M)
    B = 2
    rhs = rng.uniform(-1, 1, M * B)
    case = O.Case(M=M, batch=B, upperBanded=ub, jw_type=jwt, cfg_scaleC=1.0)
    x = O.jw_step(case, bands, rhs, "q")
    mv, sv, md, mo, sl, su = O.jw_operator(case, bands)
    T = _jw_dense(ub, jwt, md, mo, sl, su, M)
    ref = (T @ rhs.reshape(B, M).T).T.ravel()
    assert np.abs(x - ref).max() < 1e-11


def test_operator_offsets_follow_code_not_readme():
    # upperBanded=1, jw_type=10: V = md at [0,M) + ud at [M,2M); M solve uses ld at [2M,3M)
    M = 64
    nat = np.concatenate([np.full(M, 2.0), np.full(M, 3.0), np.full(M, 5.0)])
    bands = WL.permute_bands(nat, M)
    mv, sv, md, mo, sl, su = O.jw_operator(O.Case(M=M, batch=1, upperBanded=1, jw_type=10), bands)
    assert (mv, sv) == (O.MV_UPPER, O.SV_LOWER)
    assert md[0] == 2.0 and mo[0] == 3.0 and sl[0] == 5.0
    # runtime offsetM swaps the matvec bands: ud at offsetM, md at offsetM+M
    case = O.Case(M=M, batch=1, upperBanded=1, jw_type=10, bitmask=O.RUNTIME_OFFSETM | O.RUNTIME_OFFSETV,
                  run_offsetM=0, run_offsetV=2 * M)
    mv, sv, md, mo, sl, su = O.jw_operator(case, bands)
    assert md[0] == 3.0 and mo[0] == 2.0 and sl[0] == 5.0
    # jw_type%10 == 3 with upperBanded=1 takes md from [M,2M) (flipped
    # orientation) and solves with the band at [0,M) loaded beside it
    mv, sv, md, mo, sl, su = O.jw_operator(O.Case(M=M, batch=1, upperBanded=1, jw_type=13), bands)
    assert (mv, sv) == (O.MV_DIAG, O.SV_LOWER) and md[0] == 3.0 and sl[0] == 2.0
    mv, sv, md, mo, sl, su = O.jw_operator(O.Case(M=M, batch=1, upperBanded=0, jw_type=13), bands)
    assert (mv, sv) == (O.MV_DIAG, O.SV_UPPER) and md[0] == 2.0 and su[0] == 3.0


@pytest.mark.parametrize("jwt", [10, 11, 12])
def test_undefined_combination_rejected(jwt):
    M = 16
    with pytest.raises(ValueError):
        O.jw_step(O.Case(M=M, batch=1, upperBanded=2, jw_type=jwt), np.ones(3 * M), np.ones(M))


def test_zeropad_keep_windows_and_scaleC():
    M = 50
    rng = np.random.default_rng(5)
    a, d, c = WL.tridiagonal(rng, M)
    bands = WL.permute_bands(WL.tri_bands(a, d, c), M)
    rhs = rng.uniform(-1, 1, M)
    # runtime windows: read [5, 40), write [10, 30), scaleC on row 0 only
    case = O.Case(M=M, batch=1, bitmask=O.RUNTIME_INPUTZEROPAD | O.RUNTIME_OUTPUTZEROPAD | O.RUNTIME_SCALEC,
                  run_inputZeropad=(5, 40), run_outputZeropad=(0, 30), run_scaleC=3.0)
    x = O.jw_step(case, bands, rhs, "q")
    b = rhs.copy()
    b[:5] = 0
    b[40:] = 0
    ref = np.linalg.solve(_dense(a, d, c), b)
    ref[0] *= 3.0
    np.testing.assert_allclose(x[:30], ref[:30], atol=1e-13)
    np.testing.assert_array_equal(x[30:], rhs[30:])  # not written
    # plan-time windows: 0 means unbounded
    case = O.Case(M=M, batch=1, cfg_inputZeropad=(0, 20))
    x = O.jw_step(case, bands, rhs, "q")
    b = rhs.copy()
    b[20:] = 0
    np.testing.assert_allclose(x, np.linalg.solve(_dense(a, d, c), b), atol=1e-13)


@pytest.mark.parametrize("KL,KU", [(1, 1), (2, 2), (0, 3), (3, 0)])
def test_dgbmv_matches_dense(KL, KU):
    M, B = 37, 3
    rng = np.random.default_rng(KL * 10 + KU)
    A = WL.band_major(rng, M, KL, KU)
    x = rng.uniform(-1, 1, M * B)
    case = O.Case(M=M, batch=B, LDA=KL + KU + 1, KU=KU, KL=KL)
    y = O.dgbmv(case, A, x)
    D = np.zeros((M, M))
    for r in range(M):
        for j in range(KL + KU + 1):
            cc = r + KU - j
            if 0 <= cc < M:
                D[r, cc] = A[j * M + cc]
    ref = (D @ x.reshape(B, M).T).T.ravel()
    assert np.abs(y - ref).max() < 1e-13


def test_block_layouts():
    N, Y = 6, 3
    rng = np.random.default_rng(9)
    cplx = rng.standard_normal((Y, N)) + 1j * rng.standard_normal((Y, N))
    packed = np.stack([cplx.real, cplx.imag], -1).ravel()
    xxii = np.concatenate([np.concatenate([cplx[y].real, cplx[y].imag]) for y in range(Y)])
    # 4: packed -> XXII
    out = O.block(O.Case(M=N, batch=Y, block=4), packed, np.zeros(2 * N * Y))
    np.testing.assert_array_equal(out, xxii)
    # 7: XXII -> packed
    out = O.block(O.Case(M=N, batch=Y, block=7), xxii, np.zeros(2 * N * Y))
    np.testing.assert_array_equal(out, packed)
    # 2 / 3: Re / Im
    out = O.block(O.Case(M=N, batch=Y, block=2), packed, np.zeros(N * Y))
    np.testing.assert_array_equal(out, cplx.real.ravel())
    out = O.block(O.Case(M=N, batch=Y, block=3), packed, np.zeros(N * Y))
    np.testing.assert_array_equal(out, cplx.imag.ravel())
    # 1 + accumulate + ScaleC (runtime)
    r = rng.standard_normal(N * Y)
    o0 = rng.standard_normal(N * Y)
    out = O.block(O.Case(M=N, batch=Y, block=121, bitmask=O.RUNTIME_SCALEC, run_scaleC=2.5), r, o0)
    np.testing.assert_allclose(out, o0 + 2.5 * r, rtol=1e-15)


def test_scale_factors_closed_form():
    L, s = 3, 0.5
    for x in range(5):
        X = float(x)
        assert O.scale_factor(2, x, L, s) == pytest.approx(2 * (X + L + 1) * np.sqrt((X + 1) / (X + s + L + 1.5)))
        assert O.scale_factor(3, x, L, s) == pytest.approx(
            4 * (X + L + 2) * (X + L + 3) * np.sqrt((X + 1) * (X + 2) / ((X + s + L + 2.5) * (X + s + L + 3.5))))
        assert O.scale_factor(4, x, L, s) == pytest.approx((4 * L + 6) * (X + L + 1) * np.sqrt((X + 1) / (X + s + L + 1.5)))


def test_double_path_close_to_quad():
    wl = WL.config3(M=512, B=8)
    case = O.Case(M=wl.M, batch=wl.nrhs, upperBanded=2, jw_type=13)
    xq = O.jw_step(case, wl.jw_bands, wl.rhs, "q")
    xd = O.jw_step(case, wl.jw_bands, wl.rhs, "d")
    e, _ = O.rel_errors(xd, xq, wl.M, wl.nrhs, wl.M)
    assert e < 1e-13


def test_dd_storage_round_trip():
    M, B = 64, 2
    rng = np.random.default_rng(3)
    a, d, c = WL.tridiagonal(rng, M)
    bands = WL.permute_bands(WL.tri_bands(a, d, c), M)
    rhs = rng.uniform(-1, 1, M * B)
    bdd = np.stack([bands, np.zeros_like(bands)], -1).ravel()
    rdd = np.stack([rhs, np.zeros_like(rhs)], -1).ravel()
    case = O.Case(M=M, batch=B, upperBanded=2, jw_type=13)
    xdd = O.jw_step(case, bdd, rdd, "dd").reshape(-1, 2)
    xq = O.jw_step(case, bands, rhs, "q")
    np.testing.assert_allclose(xdd[:, 0], xq, rtol=1e-15)
    assert np.all(np.abs(xdd[:, 1]) <= np.abs(xdd[:, 0]) * 2.0 ** -52 + 1e-300)
