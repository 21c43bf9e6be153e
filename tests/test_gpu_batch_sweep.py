"""The uneven batch's sweep kernel (one complex system per lane, each
system's rows in sequence) through the C ABI: every bidiagonal operator kind
it takes, ragged sizes and system counts, odd strides and 8-byte-aligned rows,
against the __float128 oracle chain per entry (dgbmv -> JW step -> block), and
against the group kernel on a spectral timestep.

Tolerance: relative L2 error <= 1e-13 per complex system, as for the group
kernel; rows past M in the output strides stay untouched.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import workloads as WL

pytestmark = pytest.mark.gpu
TOL = 1e-13
SENTINEL = 7.0

# (upperBanded, jw_type, LDA, KU, block): the fused V*A stays within rows
# i-1..i+1 and the solve is bidiagonal (descending, ascending) or absent
MODES = {
    "ub0_j13_dg3_sphlapla": (0, 13, 3, 1, 307),
    "ub1_j13_dg3_scalec": (1, 13, 3, 1, 107),
    "ub1_j10_dg2_sphlapl": (1, 10, 2, 0, 207),
    "ub0_j11_dg2_nosolve": (0, 11, 2, 1, 7),
    "ub1_j12_plain": (1, 12, 0, 0, 407),
    "ub0_j10_plain": (0, 10, 0, 0, 307),
}
SIZES = [(1, 3), (2, 1), (7, 33), (8, 32), (9, 31), (31, 2), (33, 64), (64, 5), (255, 40), (257, 1),
         (1000, 7), (4096, 3)]


def make_entries(rng, LDA, KU, sizes, istr_pad=0, ostr_pad=0):
    ents = []
    for k, (M, ns) in enumerate(sizes):
        nat = rng.uniform(-0.5, 0.5, 3 * M)
        dg = WL.band_major(rng, M, LDA - 1 - KU, KU) if LDA else None
        ents.append(dict(M=M, ns=ns, bands=WL.permute_bands(nat, M), dg=dg, rhs=rng.standard_normal(2 * M * ns),
                         lshift=k % 7, scaleS=-0.55 + 0.1 * k, scaleC=1.0 + 0.25 * (k % 3), istr=M + istr_pad,
                         ostr=M + ostr_pad))
    return ents


def oracle_entry(e, ub, jwt, LDA, KU, block):
    M, ns = e["M"], e["ns"]
    y = e["rhs"]
    if LDA:
        y = O.dgbmv(O.Case(M=M, batch=2 * ns, LDA=LDA, KU=KU, KL=LDA - 1 - KU, jw_type=0), e["dg"], y)
    x = O.jw_step(O.Case(M=M, batch=2 * ns, upperBanded=ub, jw_type=jwt, cfg_scaleC=e["scaleC"]), e["bands"], y,
                  "q")
    cb = O.Case(M=M, batch=ns, block=block, lshift=e["lshift"], jw_type=0, bitmask=O.RUNTIME_SCALEC,
                run_scaleC=e["scaleS"])
    return O.block(cb, x, np.zeros(2 * M * ns)).reshape(ns, 2 * M)


def run_batch(ents, mode, in_shift=0, in_place=False, **shape):
    """Entries back to back in one input and one output buffer (the input's
    row padding NaN, the output's SENTINEL); returns each entry's output rows
    (ns x 2*ostr) and the plan's shape."""
    import torch

    from pfsolve_b200.api import Batch
    ub, jwt, LDA, KU, block = mode
    n_in = sum(2 * e["ns"] * e["istr"] for e in ents) + in_shift
    hin = np.full(n_in, np.nan)
    offs_in, offs_out = [], []
    o_in, o_out = in_shift, 0
    for e in ents:
        M, ns, s = e["M"], e["ns"], e["istr"]
        hin[o_in:o_in + 2 * ns * s].reshape(2 * ns, s)[:, :M] = e["rhs"].reshape(2 * ns, M)
        offs_in.append(o_in)
        offs_out.append(o_out)
        o_in += 2 * ns * s
        o_out += 2 * ns * e["ostr"]
    inp = torch.from_numpy(hin).cuda()
    out = inp if in_place else torch.full((o_out,), SENTINEL, dtype=torch.float64, device="cuda")
    if in_place:
        offs_out = offs_in
    keep, entries = [], []
    for e, oi, oo in zip(ents, offs_in, offs_out):
        tb = torch.from_numpy(e["bands"]).cuda()
        ta = torch.from_numpy(e["dg"]).cuda() if e["dg"] is not None else None
        keep += [tb, ta]
        entries.append(dict(M=e["M"], nsys=e["ns"], bands=tb, dgbmvBands=ta, input=inp.data_ptr() + 8 * oi,
                            output=out.data_ptr() + 8 * oo, inputStride=e["istr"], outputStride=e["ostr"],
                            lshift=e["lshift"], scaleS=e["scaleS"], scaleC=e["scaleC"]))
    b = Batch(entries, upperBanded=ub, jw_type=jwt, LDA=LDA, KU=KU, KL=max(0, LDA - 1 - KU), block=block, **shape)
    b.append()
    torch.cuda.synchronize()
    got_shape = b.shape()
    b.close()
    hout = out.cpu().numpy()
    return [hout[oo:oo + 2 * e["ns"] * e["ostr"]].reshape(e["ns"], 2 * e["ostr"]) for e, oo in zip(ents, offs_out)], \
        got_shape


def check(ents, outs, mode, untouched=True):
    for k, (e, g) in enumerate(zip(ents, outs)):
        M = e["M"]
        ref = oracle_entry(e, *mode)
        rel = np.linalg.norm(g[:, :2 * M] - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert rel.max() <= TOL, (k, M, e["ns"], rel.max())
        if untouched:
            assert np.all(g[:, 2 * M:] == SENTINEL), (k, M)


@pytest.mark.parametrize("rows", [0, 8, 16])
@pytest.mark.parametrize("name", list(MODES))
def test_sweep_matches_oracle(name, rows):
    """Chunks of 8 and 16 rows (0: the plan's default)."""
    mode = MODES[name]
    rng = np.random.default_rng(11)
    ents = make_entries(rng, mode[2], mode[3], SIZES)
    outs, shape = run_batch(ents, mode, sweepRows=rows)
    assert shape["rowsPerThread"] == 0 and shape["systemsPerItem"] == 32, shape
    assert shape["sweepRows"] == (rows or 16), shape
    check(ents, outs, mode)


@pytest.mark.parametrize("rows", [8, 16])
@pytest.mark.parametrize("istr_pad,ostr_pad,in_shift", [(1, 3, 0), (2, 1, 1), (0, 0, 1), (3, 2, 1), (4, 0, 0)])
def test_sweep_strides_and_alignment(istr_pad, ostr_pad, in_shift, rows):
    """Odd input strides take the shifted imaginary box, an input 8 bytes off
    a 16-byte boundary the 8-byte copies; padded strides leave the padding
    out of the results and untouched in the output."""
    for name in ("ub0_j13_dg3_sphlapla", "ub1_j10_dg2_sphlapl"):
        mode = MODES[name]
        rng = np.random.default_rng(12 + istr_pad)
        ents = make_entries(rng, mode[2], mode[3], SIZES[:10], istr_pad, ostr_pad)
        outs, shape = run_batch(ents, mode, in_shift=in_shift, sweepRows=rows)
        assert shape["rowsPerThread"] == 0, shape
        check(ents, outs, mode)


def test_sweep_equals_group_kernel_on_a_timestep():
    import torch

    from pfsolve_b200.api import Batch
    step = WL.config4(lmax=63, Nmax=200, seed=9)
    res = []
    for shape in (dict(), dict(rowsPerThread=8)):
        inp = torch.from_numpy(step.rhs).cuda()
        out = torch.zeros_like(inp)
        keep, entries = [], []
        for k, (l, N, ns) in enumerate(zip(step.ls, step.Ns, step.nsys)):
            tb = torch.from_numpy(step.jw_bands[k]).cuda()
            ta = torch.from_numpy(step.dgbmv[k]).cuda()
            keep += [tb, ta]
            off = 8 * int(step.rhs_offsets[k])
            entries.append(dict(M=int(N), nsys=int(ns), bands=tb, dgbmvBands=ta, input=inp.data_ptr() + off,
                                output=out.data_ptr() + off, inputStride=int(N), outputStride=int(N), lshift=int(l),
                                scaleS=step.scale_s, scaleC=1.0))
        b = Batch(entries, upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307, **shape)
        b.append()
        torch.cuda.synchronize()
        assert (b.shape()["rowsPerThread"] == 0) == (not shape)
        b.close()
        res.append(out.cpu().numpy())
    for k in range(len(step.ls)):
        N, ns, off = int(step.Ns[k]), int(step.nsys[k]), int(step.rhs_offsets[k])
        a = res[0][off:off + 2 * N * ns].reshape(ns, 2 * N)
        g = res[1][off:off + 2 * N * ns].reshape(ns, 2 * N)
        assert (np.linalg.norm(a - g, axis=1) / np.linalg.norm(g, axis=1)).max() <= TOL, k


def test_in_place_batch_takes_the_group_kernel():
    """XXII -> packed in place: the sweep would overwrite rows it has not yet
    read, so the plan keeps the group kernel (a system at a time)."""
    mode = MODES["ub0_j13_dg3_sphlapla"]
    rng = np.random.default_rng(13)
    ents = make_entries(rng, mode[2], mode[3], [(64, 40), (200, 33), (511, 5)])
    outs, shape = run_batch(ents, mode, in_place=True)
    assert shape["rowsPerThread"] != 0, shape
    check(ents, outs, mode, untouched=False)


def test_sweep_rejects_wide_operators_and_keeps_the_group_kernel():
    """V*A reaching rows i-2 / i+2 (a 3-band dgbmv on a bidiagonal matvec) is
    not the sweep kernel's: the config-4 shape with rowsPerThread 0 still runs
    the group kernel where one is compiled, else the plan reports the
    combination as unsupported."""
    import ctypes

    from pfsolve_b200 import capi
    lib = capi.load()
    e = (capi.PfSolveBatchEntry * 1)()
    e[0].M, e[0].nsys = 64, 0
    e[0].bands = e[0].dgbmvBands = e[0].input = e[0].output = 16
    e[0].inputStride = e[0].outputStride = 64
    h = ctypes.c_void_p()
    for rows in (0, 8):
        d = capi.PfSolveBatchDesc(upperBanded=0, jw_type=10, LDA=3, KU=1, KL=1, block=307, sweepRows=rows)
        assert lib.PfSolveBatchCreate(ctypes.byref(h), 0, ctypes.byref(d), e, 1) == \
            capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION
    # the group kernel's operator with sweepRows asks for what the batch cannot do
    d = capi.PfSolveBatchDesc(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=301, sweepRows=16)
    assert lib.PfSolveBatchCreate(ctypes.byref(h), 0, ctypes.byref(d), e, 1) == \
        capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION
