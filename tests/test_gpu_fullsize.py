"""The benchmarked kernel instances, checked at the sizes they are benchmarked at.

Config 2 (N = 1024, 65 536 complex systems, 5-band dgbmv -> tridiagonal JW
step -> XXII-to-packed block, one fused launch) and config 3 in mixed
precision (N = 512, 131 072 real systems, FP32 solve + 2 FP64 refinement
sweeps), through the C ABI:

  * the launch ran on the streaming kernel instance the benchmark times
    (PfSolveGetLastLaunch);
  * a sample of at least 512 systems, spread over the whole batch and holding
    systems that their group solves first, second and last (the steady-state
    path: next system's TMA load in flight, buffer swap, mbarrier phase flip),
    against the __float128 oracle: relative L2 per system <= 1e-13 (FP64) and
    <= 1e-12 (mixed);
  * every system by its residual, computed in FP64 on the GPU from the
    natural-order bands: ||md*(A b) - (x + ld x_{i-1} + ud x_{i+1})|| /
    ||md*(A b)|| <= 1e-13 (FP64), <= 1e-12 (mixed).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def spread_sample(nsys, ngroups, seed, each=160):
    """Systems solved first, second and last by their group, plus others, as
    the persistent kernels hand them out (group y mod ngroups takes system y
    at its (y div ngroups)-th turn)."""
    rng = np.random.default_rng(seed)
    g1 = min(ngroups, nsys)
    first = rng.choice(g1, min(each, g1), replace=False)
    parts = [first]
    if nsys > ngroups:
        g2 = min(ngroups, nsys - ngroups)
        parts.append(ngroups + rng.choice(g2, min(each, g2), replace=False))
    g = rng.choice(g1, min(each, g1), replace=False)
    parts.append(g + ngroups * ((nsys - 1 - g) // ngroups))
    parts.append(rng.choice(nsys, min(each, nsys), replace=False))
    return np.unique(np.concatenate(parts))


def natural_bands(tb, M):
    """(ld, md, ud) in row order from the reference-layout band buffer."""
    import torch
    perm = torch.from_numpy(WL.reference_band_order(M)).to(tb.device)
    return tuple(tb[k * M + perm] for k in range(3))


def band_matvec(A, b, KL, KU):
    """y = A b for a band-major matrix (A[j*M + c] multiplies b_c in row
    c + j - KU), rows of b being systems."""
    M = b.shape[1]
    y = b.new_zeros(b.shape)
    for j in range(KL + KU + 1):
        k = KU - j  # row r reads column r + k
        lo, hi = max(0, -k), min(M, M - k)
        y[:, lo:hi] += A[j * M + lo + k:j * M + hi + k] * b[:, lo + k:hi + k]
    return y


def tri_residual(ld, md, ud, g, x):
    """Per-system ||md*g - (x + ld x_{i-1} + ud x_{i+1})|| and ||md*g||."""
    t = md * g
    r = t - x
    r[:, 1:] -= ld[1:] * x[:, :-1]
    r[:, :-1] -= ud[:-1] * x[:, 1:]
    return r.norm(dim=1), t.norm(dim=1)


def test_config2_chain_full_size():
    import torch

    from pfsolve_b200.api import App, append_chain, last_launch, streaming_launch_count
    wl = WL.config2()
    M, B = wl.M, wl.nrhs
    assert (M, B) == (1024, 65536)
    tA = torch.from_numpy(wl.dgbmv).cuda()
    tb = torch.from_numpy(wl.jw_bands).cuda()
    rhs = torch.from_numpy(wl.rhs).cuda()
    out = torch.zeros(2 * M * B, dtype=torch.float64, device="cuda")
    dg = App(buffer=tA, outputBuffer=rhs, M_size=M, size=(M, 2 * B), LDA=5, KU=2, KL=2, doublePrecision=1)
    jw = App(buffer=tb, outputBuffer=rhs, M_size=M, size=(M, 2 * B), upperBanded=2, jw_type=13, doublePrecision=1,
             scaleC=1.0)
    bl = App(buffer=rhs, outputBuffer=out, M_size=M, size=(M, B), block=7, doublePrecision=1)
    n0 = streaming_launch_count()
    append_chain([dg, jw, bl], [dg.launch_params(), jw.launch_params(), bl.launch_params()])
    torch.cuda.synchronize()
    info = last_launch()
    assert streaming_launch_count() == n0 + 1
    # StCfg<16, 2, 2, 2, SV_TRI, LAY_XXII, LAY_PACKED, no Scale, FP64>: the benchmarked instance
    assert (info["kernel"], info["rowsPerThread"], info["warpsPerSystem"]) == (capi.PFSOLVE_KERNEL_STREAMING, 16, 2)
    assert (info["bandsBelow"], info["bandsAbove"], info["solve"]) == (2, 2, 3)
    assert (info["layoutIn"], info["layoutOut"], info["scale"], info["precision"]) == (1, 2, 0, 0)
    ngroups = info["gridCTAs"] * info["groupsPerCTA"]
    assert B > 2 * ngroups, "every group solves several systems"
    ys = spread_sample(B, ngroups, seed=21)
    assert len(ys) >= 512
    # oracle: the same chain in __float128 on the sampled systems
    sub = wl.rhs.reshape(B, 2, M)[ys].ravel()
    n = len(ys)
    th = os.cpu_count() or 1
    y = O.dgbmv(O.Case(M=M, batch=2 * n, LDA=5, KU=2, KL=2, jw_type=0), wl.dgbmv, sub, nthreads=th)
    x = O.jw_step(O.Case(M=M, batch=2 * n, upperBanded=2, jw_type=13), wl.jw_bands, y, "q", nthreads=th)
    ref = O.block(O.Case(M=M, batch=n, block=7, jw_type=0), x, np.zeros(2 * M * n)).reshape(n, M, 2)
    got = out.view(B, M, 2)[torch.from_numpy(ys).cuda()].cpu().numpy()
    rel = np.linalg.norm((got - ref).reshape(n, -1), axis=1) / np.linalg.norm(ref.reshape(n, -1), axis=1)
    assert rel.max() <= 1e-13, (rel.max(), ys[rel.argmax()])
    # every system: the residual of the chain, in chunks of systems
    ld, md, ud = natural_bands(tb, M)
    b3 = rhs.view(B, 2, M)
    x3 = out.view(B, M, 2)
    worst = 0.0
    for y0 in range(0, B, 8192):
        y1 = min(B, y0 + 8192)
        for part in range(2):
            g = band_matvec(tA, b3[y0:y1, part], 2, 2)
            num, den = tri_residual(ld, md, ud, g, x3[y0:y1, :, part].contiguous())
            worst = max(worst, (num / den).max().item())
    assert worst <= 1e-13, worst


@pytest.mark.parametrize("refine,tol", [(2, 1e-12)])
def test_config3_mixed_full_size(refine, tol):
    import torch

    from pfsolve_b200.api import App, last_launch
    wl = WL.config3()
    M, B = wl.M, wl.nrhs
    assert (M, B) == (512, 131072)
    tb = torch.from_numpy(wl.jw_bands).cuda()
    x = torch.from_numpy(wl.rhs.copy()).cuda()
    app = App(buffer=tb, outputBuffer=x, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=1,
              scaleC=1.0, mixedPrecisionRefinement=refine)
    app.append()
    torch.cuda.synchronize()
    info = last_launch()
    assert (info["kernel"], info["precision"], info["solve"]) == (capi.PFSOLVE_KERNEL_STREAMING, 1, 3)
    ngroups = info["gridCTAs"] * info["groupsPerCTA"]
    assert B > 2 * ngroups
    ys = spread_sample(B, ngroups, seed=22)
    assert len(ys) >= 512
    n = len(ys)
    sub = wl.rhs.reshape(B, M)[ys].ravel()
    ref = O.jw_step(O.Case(M=M, batch=n, upperBanded=2, jw_type=13), wl.jw_bands, sub, "q",
                    nthreads=os.cpu_count() or 1).reshape(n, M)
    got = x.view(B, M)[torch.from_numpy(ys).cuda()].cpu().numpy()
    rel = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert rel.max() <= tol, (rel.max(), ys[rel.argmax()])
    ld, md, ud = natural_bands(tb, M)
    b = torch.from_numpy(wl.rhs).cuda().view(B, M)
    num, den = tri_residual(ld, md, ud, b, x.view(B, M))
    assert (num / den).max().item() <= tol
    app.close()
