"""PfSolveBatchAppendNoAlloc (the uneven batch staged in the library's fixed
device array, allocating nothing) against PfSolveBatchCreate +
PfSolveBatchAppend on the same descriptor, through the C ABI.

Both run the same kernel with the same rows per thread and systems per item,
so every system agrees to 1e-13 relative L2 (observed: identical); checked on
two calls in a row.  A sample of degrees is also checked against the
__float128 oracle chain (dgbmv -> JW step -> block 307) at 1e-13, so that the
two paths cannot agree on a wrong answer.  After a warm-up call, further calls
leave the device's free memory unchanged, launch exactly one kernel each and
leave the caller's current device as it was.  Capacity errors need no device
work."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _oracle_degree(step, k):
    """The degree-k systems of an uneven step by the __float128 oracle chain."""
    l, N, ns = int(step.ls[k]), int(step.Ns[k]), int(step.nsys[k])
    off = int(step.rhs_offsets[k])
    rhs = step.rhs[off:off + 2 * N * ns]
    y = O.dgbmv(O.Case(M=N, batch=2 * ns, LDA=3, KU=1, KL=1, jw_type=0), step.dgbmv[k], rhs)
    x = O.jw_step(O.Case(M=N, batch=2 * ns, upperBanded=0, jw_type=13), step.jw_bands[k], y, "q")
    cb = O.Case(M=N, batch=ns, block=307, lshift=l, jw_type=0, bitmask=O.RUNTIME_SCALEC, run_scaleC=step.scale_s)
    return O.block(cb, x, np.zeros(2 * N * ns))


def _entry_array(entries):
    arr = (capi.PfSolveBatchEntry * max(1, len(entries)))()
    for i, e in enumerate(entries):
        a = arr[i]
        a.M, a.nsys = int(e["M"]), int(e["nsys"])
        a.bands, a.dgbmvBands = e["bands"], e["dgbmvBands"]
        a.input, a.output = e["input"], e["output"]
        a.inputStride, a.outputStride = int(e["M"]), int(e["M"])
        a.lshift, a.scaleS, a.scaleC = int(e["lshift"]), float(e["scaleS"]), 1.0
    return arr


def test_noalloc_matches_batch_append_twice():
    import torch

    from pfsolve_b200.api import Batch
    lib = capi.load()
    step = WL.config4(lmax=95)
    inp = torch.from_numpy(step.rhs).cuda()
    out_ref = torch.zeros_like(inp)
    out = torch.zeros_like(inp)
    keep, ents_ref, ents = [], [], []
    for k, (l, N, ns) in enumerate(zip(step.ls, step.Ns, step.nsys)):
        tj = torch.from_numpy(step.jw_bands[k]).cuda()
        ta = torch.from_numpy(step.dgbmv[k]).cuda()
        keep += [tj, ta]
        off = 8 * int(step.rhs_offsets[k])
        common = dict(M=int(N), nsys=int(ns), bands=tj.data_ptr(), dgbmvBands=ta.data_ptr(), lshift=int(l),
                      scaleS=step.scale_s)
        ents_ref.append(dict(common, input=inp.data_ptr() + off, output=out_ref.data_ptr() + off,
                             inputStride=int(N), outputStride=int(N)))
        ents.append(dict(common, input=inp.data_ptr() + off, output=out.data_ptr() + off))
    shape = dict(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307, rowsPerThread=8, systemsPerItem=32)
    b = Batch(ents_ref, **shape)
    b.append()
    torch.cuda.synchronize()
    ref = out_ref.cpu().numpy()
    b.close()
    desc = capi.PfSolveBatchDesc(**shape)
    arr = _entry_array(ents)
    # the oracle on a sample of degrees (first, middle, last) of the reference path
    for k in (0, len(step.ls) // 2, len(step.ls) - 1):
        N, ns = int(step.Ns[k]), int(step.nsys[k])
        off = int(step.rhs_offsets[k])
        o = _oracle_degree(step, k).reshape(ns, 2 * N)
        r = ref[off:off + 2 * N * ns].reshape(ns, 2 * N)
        assert (np.linalg.norm(r - o, axis=1) / np.linalg.norm(o, axis=1)).max() <= TOL, k
    for call in range(2):
        out.zero_()
        torch.cuda.synchronize()
        rc = lib.PfSolveBatchAppendNoAlloc(0, ctypes.byref(desc), arr, len(ents), None)
        assert rc == capi.PFSOLVE_SUCCESS, rc
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        worst = 0.0
        for k, (N, ns) in enumerate(zip(step.Ns, step.nsys)):
            off = int(step.rhs_offsets[k])
            g = got[off:off + 2 * N * ns].reshape(ns, 2 * N)
            r = ref[off:off + 2 * N * ns].reshape(ns, 2 * N)
            worst = max(worst, float((np.linalg.norm(g - r, axis=1) / np.linalg.norm(r, axis=1)).max()))
        assert worst <= TOL, (call, worst)


def test_noalloc_allocates_nothing_and_keeps_the_device():
    """After a warm-up call (which loads the kernel and looks up the array's
    address), calls change neither the device's free memory nor the caller's
    current device, and each launches exactly one kernel."""
    import torch

    lib = capi.load()
    step = WL.config4(lmax=31, Nmax=128, seed=9)
    inp = torch.from_numpy(step.rhs).cuda()
    out = torch.zeros_like(inp)
    keep, ents = [], []
    for k, (l, N, ns) in enumerate(zip(step.ls, step.Ns, step.nsys)):
        tj = torch.from_numpy(step.jw_bands[k]).cuda()
        ta = torch.from_numpy(step.dgbmv[k]).cuda()
        keep += [tj, ta]
        off = 8 * int(step.rhs_offsets[k])
        ents.append(dict(M=int(N), nsys=int(ns), bands=tj.data_ptr(), dgbmvBands=ta.data_ptr(), lshift=int(l),
                         scaleS=step.scale_s, input=inp.data_ptr() + off, output=out.data_ptr() + off))
    desc = capi.PfSolveBatchDesc(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307)
    arr = _entry_array(ents)
    assert lib.PfSolveBatchAppendNoAlloc(0, ctypes.byref(desc), arr, len(ents), None) == capi.PFSOLVE_SUCCESS
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    dev0 = torch.cuda.current_device()
    for _ in range(5):
        n0 = lib.PfSolveLaunchCount()
        assert lib.PfSolveBatchAppendNoAlloc(0, ctypes.byref(desc), arr, len(ents), None) == capi.PFSOLVE_SUCCESS
        assert lib.PfSolveLaunchCount() == n0 + 1
        assert torch.cuda.current_device() == dev0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    # the result of the last call against the oracle on one degree
    k = len(step.ls) - 1
    N, ns = int(step.Ns[k]), int(step.nsys[k])
    off = int(step.rhs_offsets[k])
    o = _oracle_degree(step, k).reshape(ns, 2 * N)
    g = out.cpu().numpy()[off:off + 2 * N * ns].reshape(ns, 2 * N)
    assert (np.linalg.norm(g - o, axis=1) / np.linalg.norm(o, axis=1)).max() <= TOL


def test_noalloc_capacity_and_argument_errors():
    lib = capi.load()
    desc = capi.PfSolveBatchDesc(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307)
    n = capi.PFSOLVE_NOALLOC_MAX_ENTRIES + 1
    arr = (capi.PfSolveBatchEntry * n)()
    for a in arr:
        a.M, a.nsys, a.bands, a.dgbmvBands, a.input, a.output = 64, 1, 8, 8, 8, 8
    assert lib.PfSolveBatchAppendNoAlloc(0, ctypes.byref(desc), arr, n, None) == capi.PFSOLVE_ERROR_CAPACITY
    # too many work items: one system per item
    big = (capi.PfSolveBatchEntry * 1)()
    big[0].M, big[0].nsys, big[0].bands, big[0].dgbmvBands, big[0].input, big[0].output = \
        64, capi.PFSOLVE_NOALLOC_MAX_ITEMS + 1, 8, 8, 8, 8
    d1 = capi.PfSolveBatchDesc(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307, systemsPerItem=1)
    assert lib.PfSolveBatchAppendNoAlloc(0, ctypes.byref(d1), big, 1, None) == capi.PFSOLVE_ERROR_CAPACITY
    assert lib.PfSolveBatchAppendNoAlloc(0, None, big, 1, None) == capi.PFSOLVE_ERROR_INVALID_ARGUMENT


def test_noalloc_refused_under_stream_capture():
    """The descriptors are copied from host arrays that the next call
    rewrites, so a call on a stream under capture must enqueue nothing and
    return PFSOLVE_ERROR_INVALID_ARGUMENT; the same call outside the capture
    still runs."""
    import torch

    lib = capi.load()
    step = WL.config4(lmax=15, Nmax=64, seed=11)
    inp = torch.from_numpy(step.rhs).cuda()
    out = torch.zeros_like(inp)
    keep, ents = [], []
    for k, (l, N, ns) in enumerate(zip(step.ls, step.Ns, step.nsys)):
        tj = torch.from_numpy(step.jw_bands[k]).cuda()
        ta = torch.from_numpy(step.dgbmv[k]).cuda()
        keep += [tj, ta]
        off = 8 * int(step.rhs_offsets[k])
        ents.append(dict(M=int(N), nsys=int(ns), bands=tj.data_ptr(), dgbmvBands=ta.data_ptr(), lshift=int(l),
                         scaleS=step.scale_s, input=inp.data_ptr() + off, output=out.data_ptr() + off))
    desc = capi.PfSolveBatchDesc(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307)
    arr = _entry_array(ents)
    s = torch.cuda.Stream()
    # set-up (the array's address) outside any capture
    assert lib.PfSolveBatchAppendNoAlloc(0, ctypes.byref(desc), arr, len(ents),
                                         ctypes.c_void_p(s.cuda_stream)) == capi.PFSOLVE_SUCCESS
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    marker = torch.zeros(1, device="cuda")
    n0 = lib.PfSolveLaunchCount()
    with torch.cuda.graph(g, stream=s):
        marker.add_(1.0)
        rc = lib.PfSolveBatchAppendNoAlloc(0, ctypes.byref(desc), arr, len(ents), ctypes.c_void_p(s.cuda_stream))
    assert rc == capi.PFSOLVE_ERROR_INVALID_ARGUMENT, rc
    assert lib.PfSolveLaunchCount() == n0
    del g
    out.zero_()
    torch.cuda.synchronize()
    assert lib.PfSolveBatchAppendNoAlloc(0, ctypes.byref(desc), arr, len(ents),
                                         ctypes.c_void_p(s.cuda_stream)) == capi.PFSOLVE_SUCCESS
    s.synchronize()
    k = len(step.ls) - 1
    N, ns = int(step.Ns[k]), int(step.nsys[k])
    off = int(step.rhs_offsets[k])
    o = _oracle_degree(step, k).reshape(ns, 2 * N)
    got = out.cpu().numpy()[off:off + 2 * N * ns].reshape(ns, 2 * N)
    assert (np.linalg.norm(got - o, axis=1) / np.linalg.norm(o, axis=1)).max() <= TOL
