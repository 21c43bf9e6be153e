"""Seeded synthetic inputs with the shapes and distributions of the JW-step
workloads this library is measured on, plus the reference's band layout.

Band layout: PfSolve's JW kernel reads band arrays in a register-major order
(reorder_i0, PfSolve/pfSolve_PlanManagement/pfSolve_Plans/pfSolve_Plan_JonesWorland.h:66-142):
row ``t*r + j`` of a band is stored at ``S_j + t`` where ``r = ceil(M/T)``
rows per lane (``T`` = 32 lanes below 512 rows, else ``64*ceil(M/1024)``) and
``S_j`` counts the rows held by registers ``0..j-1``.  Callers of the
reference pre-permute bands this way (sample_0_benchmark_VkFFT_single.cpp:306-310);
this library reads the same layout so the buffers are interchangeable.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def reference_band_order(M: int) -> np.ndarray:
    """perm[i] = storage position of logical row i in the reference's band
    order (reorder_i0, CUDA backend): register-major over the whole system up
    to 4352 rows; beyond, register-major within each piece of 256 rows (the
    partial last piece with its own counts)."""
    piece = 256 if M > 4352 else 0
    size1 = piece if piece else M
    warp = 64 * ((size1 + 1023) // 1024)
    if size1 < 512:
        warp = 32
    warp = max(warp, 32)
    if warp % 32:
        warp = 32 * ((warp + 31) // 32)
    r = max(1, (size1 + warp - 1) // warp)
    i = np.arange(M, dtype=np.int64)
    if piece:
        base = (i // piece) * piece
        li = i - base
        size0 = np.where(base + piece > M, M % piece, piece)
    else:
        base = np.zeros_like(i)
        li = i
        size0 = np.full_like(i, M)
    t, j = li // r, li % r
    m = size0 % r
    ceil_n, floor_n = (size0 + r - 1) // r, size0 // r
    return base + t + np.where(j < m, j * ceil_n, m * ceil_n + (j - m) * floor_n)


def permute_bands(natural: np.ndarray, M: int) -> np.ndarray:
    """Natural-order bands (band k occupies [k*M, (k+1)*M)) -> reference layout."""
    natural = np.asarray(natural)
    out = np.empty_like(natural)
    perm = reference_band_order(M)
    for k in range(natural.shape[0] // M):
        out[k * M + perm] = natural[k * M:(k + 1) * M]
    return out


def steps_registers(M: int, upperBanded: int, K: int) -> int:
    """Rows per lane of the reference's band order for a K-step application:
    computed from M + K - 1 rows when the steps grow the system (upperBanded 0),
    else from M (pfSolve_Plan_JonesWorland.h:276-283, 342-346)."""
    tm = M if upperBanded else M + K - 1
    warp = 64 * ((tm + 1023) // 1024)
    if tm < 512:
        warp = 32
    warp = max(warp, 32)
    if warp % 32:
        warp = 32 * ((warp + 31) // 32)
    return max(1, (tm + warp - 1) // warp)


def step_rows(M: int, upperBanded: int, s: int) -> int:
    """Rows of step s: M - s (upperBanded 1, 2) or M + s (upperBanded 0)."""
    return M - s if upperBanded else M + s


def steps_band_order(Ms: int, r: int) -> np.ndarray:
    """perm[i] for Ms rows with r rows per lane (one piece, Ms <= 4352)."""
    i = np.arange(Ms, dtype=np.int64)
    t, j = i // r, i % r
    m, ce, fl = Ms % r, -(-Ms // r), Ms // r
    return t + np.where(j < m, j * ce, m * ce + (j - m) * fl)


def steps_bands(rng, M: int, upperBanded: int, K: int, per_step: bool = True):
    """Band buffers of a K-step application, three bands of Ms rows each per
    step, stored in the step's band order.  upperBanded 2: normalised
    tridiagonal (ld | md | ud).  upperBanded 0/1: three bands in U(-1/2, 1/2)
    (every section is read as some band by one of the jw_types).  Row 0 of
    every band is zero; the last row's entry of the third band stays random
    (it couples to the row that leaves or enters the system) unless the step
    fills the reference's registers exactly.  per_step False: one buffer of
    3 * max(Ms) values read by every step at its own offsets.  Tridiagonal
    bands need per_step."""
    r = steps_registers(M, upperBanded, K)
    Mmax = max(step_rows(M, upperBanded, s) for s in range(K))
    tm = M if upperBanded else M + K - 1
    lanes = 32 if tm < 512 else 64 * ((tm + 1023) // 1024)
    capacity = r * lanes  # rows held in the reference's registers

    def one(Ms):
        if upperBanded == 2:
            a, d, c = tridiagonal(rng, Ms)
            c[-1] = rng.uniform(-0.25, 0.25)
            nat = tri_bands(a, d, c)
        else:
            nat = rng.uniform(-0.5, 0.5, 3 * Ms)
            nat[0] = nat[Ms] = nat[2 * Ms] = 0.0
        if Ms == capacity:  # no row below the last: its upper coupling is unused
            nat[Ms - 1] = nat[2 * Ms - 1] = nat[3 * Ms - 1] = 0.0
        out = np.empty_like(nat)
        perm = steps_band_order(Ms, r)
        for k in range(3):
            out[k * Ms + perm] = nat[k * Ms:(k + 1) * Ms]
        return out

    if per_step:
        return [one(step_rows(M, upperBanded, s)) for s in range(K)]
    buf = rng.uniform(-0.5, 0.5, 3 * Mmax)
    for s_ in range(K):  # row 0 of every band any step reads
        Ms = step_rows(M, upperBanded, s_)
        buf[[0, Ms, 2 * Ms]] = 0.0
    return buf


def alt_positions(M: int) -> np.ndarray:
    """pos[r] = storage position of row r in the ALT (stride-2) band layout:
    T lanes and R = ceil(M / T) rows per lane as for any JW plan; lane t < T/2
    holds the even rows 2 (t R + i), lane t >= T/2 the odd rows
    2 ((t - T/2) R + i) + 1, and the entry of register i of lane t sits at
    i T + t (pfSolve_TridiagonalSolve.h:1319-1330, pfSolve_ReadWrite.h:1705-1711)."""
    warp = 64 * ((M + 1023) // 1024)
    if M < 512:
        warp = 32
    warp = max(warp, 32)
    if warp % 32:
        warp = 32 * ((warp + 31) // 32)
    R = (M + warp - 1) // warp
    r = np.arange(M, dtype=np.int64)
    h, e = r & 1, r >> 1
    t = h * (warp // 2) + e // R
    return (e % R) * warp + t


def alt_band_span(M: int) -> int:
    """Entries between consecutive ALT bands (R T, the lanes' register capacity)."""
    warp = 64 * ((M + 1023) // 1024)
    if M < 512:
        warp = 32
    warp = max(warp, 32)
    return ((M + warp - 1) // warp) * warp


def alt_bands(rng, M: int, upperBanded: int) -> np.ndarray:
    """Three ALT-layout bands of R T entries each.  Natural rows: upperBanded 2
    a normalised tridiagonal per parity (ld | md | ud, couplings r -+ 2);
    otherwise U(-1/2, 1/2).  Couplings that leave a parity's rows (lower bands
    at rows 0, 1; upper bands at the last two rows) and the padding are zero."""
    span = alt_band_span(M)
    pos = alt_positions(M)
    lower = np.arange(M) < 2
    upper = np.arange(M) >= M - 2
    if upperBanded == 2:
        a = rng.uniform(-1, 1, M)
        c = rng.uniform(-1, 1, M)
        a[lower] = 0.0
        c[upper] = 0.0
        d = np.abs(a) + np.abs(c) + rng.uniform(1, 2, M)
        nat = [a / d, 1.0 / d, c / d]
    else:
        nat = [rng.uniform(-0.5, 0.5, M) for _ in range(3)]
        for k in range(3):  # each band is a lower or an upper coupling in some jw_type
            nat[k][lower | upper] = 0.0
    out = np.zeros(3 * span)
    for k in range(3):
        out[k * span + pos] = nat[k]
    return out


def tridiagonal(rng, M, dominance=None):
    """(a, d, c): a_0 = c_{M-1} = 0.  d = |a|+|c|+U(1,2), or dominance*(|a|+|c|)."""
    a = rng.uniform(-1.0, 1.0, M)
    c = rng.uniform(-1.0, 1.0, M)
    a[0] = 0.0
    c[-1] = 0.0
    if dominance is None:
        d = np.abs(a) + np.abs(c) + rng.uniform(1.0, 2.0, M)
    else:
        d = dominance * (np.abs(a) + np.abs(c))
        d[d == 0] = 1.0
    return a, d, c


def tri_bands(a, d, c):
    """JW tridiagonal bands in natural order: ld = a/d at [0,M), md = 1/d at
    [M,2M), ud = c/d at [2M,3M) (host normalisation of sample_0...cpp:306-310)."""
    return np.concatenate([a / d, 1.0 / d, c / d])


def upper_bidiag_bands(d, s):
    """Bands of an upperBanded=0, jw_type%10=3 step solving (diag d, super s):
    md = 1/d at [0,M) and ud = s/d at [M,2M) -- with jw_type%10 == 3 the
    reference's solve reuses the band loaded next to md (pfSolve_JonesWorland.h:
    133-206, 337-344); [2M,3M) is unused."""
    M = d.shape[0]
    s = s.copy()
    s[-1] = 0.0
    return np.concatenate([1.0 / d, s / d, np.zeros(M)])


def band_major(rng, M, KL, KU, low=-1.0, high=1.0):
    """dgbmv band-major storage A[j*M + c] (j = 0..KL+KU), U(low, high)."""
    return rng.uniform(low, high, (KL + KU + 1) * M)


@dataclass
class Workload:
    name: str
    M: int
    nrhs: int          # right-hand sides (complex ones count once)
    complex: bool
    jw_bands: np.ndarray   # reference layout
    dgbmv: np.ndarray | None
    rhs: np.ndarray        # real rows (XXII for complex)
    desc: dict


def config1(seed=0, M=256, B=512) -> Workload:
    """Plain FP64 JW step, test-1 form: 3-band V then upper-bidiagonal M
    (diag ~U(1,2), super ~U(-0.5,0.5)), B real RHS ~U(-1,1), stride M."""
    rng = np.random.default_rng(seed)
    d = rng.uniform(1.0, 2.0, M)
    s = rng.uniform(-0.5, 0.5, M)
    A = band_major(rng, M, 1, 1)
    rhs = rng.uniform(-1.0, 1.0, M * B)
    return Workload("config1", M, B, False, permute_bands(upper_bidiag_bands(d, s), M), A, rhs,
                    dict(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1))


def config2(seed=1, M=1024, B=65536) -> Workload:
    """Batched FP64 tridiagonal solve fused with a 5-band matvec: N=1024, B
    complex RHS ~N(0,1) in XXII layout, written packed.  a,c ~U(-1,1),
    d = |a|+|c|+U(1,2); band matrix ~U(-1,1)."""
    rng = np.random.default_rng(seed)
    a, d, c = tridiagonal(rng, M)
    A = band_major(rng, M, 2, 2)
    rhs = rng.standard_normal(2 * M * B)
    return Workload("config2", M, B, True, permute_bands(tri_bands(a, d, c), M), A, rhs,
                    dict(upperBanded=2, jw_type=13, LDA=5, KU=2, KL=2, block=7))


def config3(seed=2, M=512, B=131072) -> Workload:
    """Weakly dominant tridiagonal (d = 1.05(|a|+|c|)), B real RHS ~U(-1,1)."""
    rng = np.random.default_rng(seed)
    a, d, c = tridiagonal(rng, M, dominance=1.05)
    rhs = rng.uniform(-1.0, 1.0, M * B)
    return Workload("config3", M, B, False, permute_bands(tri_bands(a, d, c), M), None, rhs,
                    dict(upperBanded=2, jw_type=13))


def config4_sizes(lmax=511, Nmax=512):
    ls = np.arange(lmax + 1)
    return ls, Nmax - ls // 2, 2 * ls + 1


@dataclass
class UnevenStep:
    """One spectral timestep: harmonic degrees l = 0..lmax, N_l rows and
    2l+1 complex RHS per degree; coefficients as config 1 per degree."""
    ls: np.ndarray
    Ns: np.ndarray
    nsys: np.ndarray
    jw_bands: list      # per degree, reference layout
    dgbmv: list         # per degree, band-major (3 bands)
    rhs_offsets: np.ndarray  # per degree, element offset of its XXII block in `rhs`
    rhs: np.ndarray     # all degrees' XXII right-hand sides, concatenated
    scale_s: float


def config4(seed=3, lmax=511, Nmax=512, scale_s=-0.5, rhs=True) -> UnevenStep:
    """Uneven batch of one timestep: N_l = Nmax - floor(l/2), 2l+1 complex RHS
    ~N(0,1) per degree (XXII), V 3-band ~U(-1,1) and upper-bidiagonal M
    (diag ~U(1,2), super ~U(-0.5,0.5)) per degree; SphLaplA with lshift = l."""
    rng = np.random.default_rng(seed)
    ls, Ns, nsys = config4_sizes(lmax, Nmax)
    jw, dg, offs = [], [], []
    off = 0
    for l, N, ns in zip(ls, Ns, nsys):
        d = rng.uniform(1.0, 2.0, N)
        s = rng.uniform(-0.5, 0.5, N)
        jw.append(permute_bands(upper_bidiag_bands(d, s), N))
        dg.append(band_major(rng, N, 1, 1))
        offs.append(off)
        off += 2 * N * ns
    data = rng.standard_normal(off) if rhs else np.zeros(0)
    return UnevenStep(ls, Ns, nsys, jw, dg, np.array(offs, dtype=np.int64), data, scale_s)


def serve_operator_bands(rng, M):
    """Test-0 form operator (upperBanded 2, jw_type 13: diagonal scale then unit
    tridiagonal solve) with config-1 coefficient distributions: d ~ U(1,2),
    a, c ~ U(-0.5, 0.5), a_0 = c_{M-1} = 0; normalised md = 1/d, ld = a/d,
    ud = c/d and stored in the reference's band order."""
    d = rng.uniform(1.0, 2.0, M)
    a = rng.uniform(-0.5, 0.5, M)
    c = rng.uniform(-0.5, 0.5, M)
    a[0] = 0.0
    c[-1] = 0.0
    return permute_bands(np.concatenate([a / d, 1.0 / d, c / d]), M)


@dataclass
class ServeRequestSpec:
    M: int
    nrhs: int
    precision: int  # 1 mixed, 2 double-double storage


def config5_requests(n, seed=4, n_min=32, n_max=1024, r_min=1, r_max=4096, dd_fraction=0.2):
    """Request mix of the serving loop: N log-uniform in [n_min, n_max], RHS
    count log-uniform in [r_min, r_max], 80 % mixed precision, 20 %
    double-double."""
    rng = np.random.default_rng(seed)
    Ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max + 1), n)).astype(np.int64).clip(n_min, n_max)
    Rs = np.exp(rng.uniform(np.log(r_min), np.log(r_max + 1), n)).astype(np.int64).clip(r_min, r_max)
    dd = rng.uniform(0, 1, n) < dd_fraction
    return [ServeRequestSpec(int(N), int(R), 2 if d else 1) for N, R, d in zip(Ns, Rs, dd)]


def poisson_arrivals(n, rate, seed=4):
    """Arrival times (s) of n requests of a Poisson process of the given rate."""
    rng = np.random.default_rng(seed + 1)
    return np.cumsum(rng.exponential(1.0 / rate, n))
