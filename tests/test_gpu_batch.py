"""Uneven batches (one spectral timestep, harmonic degrees of different sizes)
in one persistent launch, through the C ABI.

Tolerance: relative L2 error <= 1e-13 per complex system against the
__float128 oracle chain (dgbmv -> JW step -> block 307).
"""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import workloads as WL

pytestmark = pytest.mark.gpu
TOL = 1e-13


def build(step, desc_extra=None):
    import torch

    from pfsolve_b200.api import Batch
    dev = torch.device("cuda")
    inp = torch.from_numpy(step.rhs).to(dev)
    out = torch.zeros_like(inp)
    keep = []
    entries = []
    for k, (l, N, ns) in enumerate(zip(step.ls, step.Ns, step.nsys)):
        tb = torch.from_numpy(step.jw_bands[k]).to(dev)
        ta = torch.from_numpy(step.dgbmv[k]).to(dev)
        keep += [tb, ta]
        off = int(step.rhs_offsets[k])
        entries.append(dict(M=int(N), nsys=int(ns), bands=tb, dgbmvBands=ta,
                            input=inp.data_ptr() + 8 * off, output=out.data_ptr() + 8 * off,
                            inputStride=int(N), outputStride=int(N), lshift=int(l), scaleS=step.scale_s,
                            scaleC=1.0))
    desc = dict(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307)
    desc.update(desc_extra or {})
    b = Batch(entries, **desc)
    return b, inp, out, keep


def oracle_degree(step, k):
    l, N, ns = int(step.ls[k]), int(step.Ns[k]), int(step.nsys[k])
    off = int(step.rhs_offsets[k])
    rhs = step.rhs[off:off + 2 * N * ns]
    y = O.dgbmv(O.Case(M=N, batch=2 * ns, LDA=3, KU=1, KL=1, jw_type=0), step.dgbmv[k], rhs)
    x = O.jw_step(O.Case(M=N, batch=2 * ns, upperBanded=0, jw_type=13), step.jw_bands[k], y, "q")
    cb = O.Case(M=N, batch=ns, block=307, lshift=l, jw_type=0, bitmask=O.RUNTIME_SCALEC, run_scaleC=step.scale_s)
    return O.block(cb, x, np.zeros(2 * N * ns))


def check(step, got):
    for k in range(len(step.ls)):
        N, ns = int(step.Ns[k]), int(step.nsys[k])
        off = int(step.rhs_offsets[k])
        ref = oracle_degree(step, k).reshape(ns, 2 * N)
        g = got[off:off + 2 * N * ns].reshape(ns, 2 * N)
        rel = np.linalg.norm(g - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert rel.max() <= TOL, (k, rel.max())


def test_uneven_step_matches_oracle():
    import torch
    step = WL.config4(lmax=47, Nmax=160)
    b, inp, out, keep = build(step)
    b.append()
    torch.cuda.synchronize()
    check(step, out.cpu().numpy())
    b.close()


def test_graph_capture_replays_identically():
    import torch
    step = WL.config4(lmax=31, Nmax=128, seed=5)
    b, inp, out, keep = build(step)
    s = torch.cuda.Stream()
    b.capture(s)
    b.append(s)
    s.synchronize()
    first = out.cpu().numpy()
    out.zero_()
    b.append(s)
    b.append(s)
    s.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), first)
    check(step, first)
    b.close()


def test_autotune_keeps_results():
    import torch
    step = WL.config4(lmax=31, Nmax=256, seed=6)
    b, inp, out, keep = build(step)
    b.autotune(iterations=2)
    shape = b.shape()
    assert shape["rowsPerThread"] in (0, 2, 4, 8, 16) and shape["tunedMs"] > 0
    out.zero_()
    b.append()
    torch.cuda.synchronize()
    check(step, out.cpu().numpy())
    b.close()


def test_each_degree_alone_equals_in_the_mix():
    import torch
    step = WL.config4(lmax=23, Nmax=96, seed=7)
    b, inp, out, keep = build(step, dict(rowsPerThread=4))
    b.append()
    torch.cuda.synchronize()
    mixed = out.cpu().numpy()
    for k in (0, 7, 23):
        sub = WL.UnevenStep(step.ls[k:k + 1], step.Ns[k:k + 1], step.nsys[k:k + 1], step.jw_bands[k:k + 1],
                            step.dgbmv[k:k + 1], np.array([0]),
                            step.rhs[int(step.rhs_offsets[k]):int(step.rhs_offsets[k]) + 2 * int(step.Ns[k]) *
                                     int(step.nsys[k])].copy(), step.scale_s)
        b1, i1, o1, k1 = build(sub, dict(rowsPerThread=4))
        b1.append()
        torch.cuda.synchronize()
        off = int(step.rhs_offsets[k])
        n = 2 * int(step.Ns[k]) * int(step.nsys[k])
        np.testing.assert_array_equal(o1.cpu().numpy(), mixed[off:off + n])
        b1.close()
    b.close()


def test_full_timestep_sampled():
    """The full timestep (l = 0..511, 262144 complex systems) in one launch;
    every degree's first and last systems checked against the oracle."""
    import torch
    step = WL.config4()
    b, inp, out, keep = build(step)
    b.append()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for k in (0, 1, 100, 255, 400, 511):
        N, ns = int(step.Ns[k]), int(step.nsys[k])
        off = int(step.rhs_offsets[k])
        ref = oracle_degree(step, k).reshape(ns, 2 * N)
        g = got[off:off + 2 * N * ns].reshape(ns, 2 * N)
        rel = np.linalg.norm(g - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert rel.max() <= TOL, (k, rel.max())
    b.close()
