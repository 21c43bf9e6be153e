"""GPU parity of the long-system JW kernels, through the C ABI.

Systems of 4 096 < N <= 65 536 rows run over slices of 1 024 rows
(PfSolveGetShape streaming = 5): by default in two passes with no waits
between CTAs at any N (launches whose rows no tensor map can describe fall
back to the single pass, one cooperative launch whose CTAs wait (bounded)
for the other slices of each system); kernelPath 3 asks for two passes
only, kernelPath 4 for the single pass only.  With
kernelPath 2, systems of up to 16 384 rows run on one thread-block cluster of
3, 4, 6 or 8 CTAs per system (streaming = 2).  Every case checks that the
plan chose the kernel asked for, that the launch ran on it, and that every
system matches the __float128 oracle to 1e-13 relative L2 (the FP64
tolerance of the other kernels).  The app works in place, so the halo rows
of neighbouring slices are exercised."""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

import jwcases as J

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _case(rng, M, B, ub, jwt, **kw):
    nat = J.random_bands(rng, M, ub)
    bands = WL.permute_bands(nat, M)
    case = O.Case(M=M, batch=B, upperBanded=ub, jw_type=jwt, **kw)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    return case, bands, rhs


def _run(case, bands, rhs, **extra):
    import torch

    from pfsolve_b200.api import App, streaming_launch_count
    tb = torch.from_numpy(np.ascontiguousarray(bands)).cuda()
    to = torch.from_numpy(np.array(rhs, copy=True)).cuda()
    app = App(buffer=tb, outputBuffer=to, **J.case_fields(case, **extra))
    shape = app.shape()
    n0 = streaming_launch_count()
    app.append(**J.launch_fields(case))
    torch.cuda.synchronize()
    n = streaming_launch_count() - n0
    x = to.cpu().numpy()
    app.close()
    return x, shape, n


PATHS = {0: 5, 3: 5, 4: 5, 2: 2}  # kernelPath -> PfSolveGetShape streaming


@pytest.mark.parametrize("path", list(PATHS))
@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (1, 11), (1, 12), (0, 10), (0, 11), (0, 13)])
@pytest.mark.parametrize("M", [4104, 4360, 5000, 6000, 6144, 8192, 12000, 16384, 20000, 40000, 65536])
def test_long_modes_and_sizes(ub, jwt, M, path):
    if path == 2 and M > 16384:
        pytest.skip("the cluster kernel holds one system on 8 CTAs of 2048 rows at most")
    rng = np.random.default_rng(9000 + 10 * ub + jwt + M)
    case, bands, rhs = _case(rng, M, 7, ub, jwt)
    x, shape, n = _run(case, bands, rhs, kernelPath=path)
    assert shape["streaming"] == PATHS[path] and n == 1, shape
    ref = O.jw_step(case, bands, rhs, "q")
    e, emax = J.rel_err(x, ref, case)
    assert e <= TOL, (e, emax)


@pytest.mark.parametrize("path", list(PATHS))
def test_long_many_systems_and_windows(path):
    rng = np.random.default_rng(77)
    for M, B, kw in [(8192, 301, {}), (8192, 65, dict(bitmask=capi.RUNTIME_INPUTZEROPAD, run_inputZeropad=(5, 8000))),
                     (8192, 2000, {}),
                     (8192, 40, dict(bitmask=capi.RUNTIME_INPUTZEROPAD, run_inputZeropad=(1030, 3100))),
                     (65536, 150, {})]:
        if path == 2 and M > 16384:
            continue
        case, bands, rhs = _case(rng, M, B, 2, 13, **kw)
        x, shape, n = _run(case, bands, rhs, kernelPath=path)
        assert n == 1
        e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
        assert e <= TOL


@pytest.mark.parametrize("path", [3, 2])
def test_long_rejects_buffers_it_cannot_take(path):
    """The two-pass form asked for alone (kernelPath 3) and the cluster form
    have no fallback for rows a TMA tensor map cannot describe: a misaligned
    launch returns UNSUPPORTED_COMBINATION instead of running."""
    rng = np.random.default_rng(3)
    case, bands, rhs = _case(rng, 6144, 3, 2, 13, bitmask=capi.RUNTIME_OFFSETSOLUTION, run_offsetSolution=1)
    with pytest.raises(capi.PfSolveError) as ei:
        _run(case, bands, rhs, kernelPath=path)
    assert ei.value.code == capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION


@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (0, 13), (1, 11)])
@pytest.mark.parametrize("M,kw", [(6144, dict(bitmask=capi.RUNTIME_OFFSETSOLUTION, run_offsetSolution=1)),
                                  (5000, dict(cfg_outputBufferStride=5003)),
                                  (9001, dict(bitmask=capi.RUNTIME_INPUTZEROPAD | capi.RUNTIME_OFFSETSOLUTION,
                                              run_inputZeropad=(7, 8990), run_offsetSolution=3))])
def test_single_pass_unaligned_rows(ub, jwt, M, kw):
    """Rows that are not 16-byte aligned (odd offsets and strides): the single
    pass moves them with plain loads and stores and still matches the oracle;
    rows outside the systems keep their values."""
    rng = np.random.default_rng(M + ub + jwt)
    case, bands, rhs = _case(rng, M, 21, ub, jwt, **kw)
    x, shape, n = _run(case, bands, rhs)
    assert shape["streaming"] == 5 and n == 1
    e, emax = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= TOL, (e, emax)
    off = case.offset_solution
    np.testing.assert_array_equal(x[:off], rhs[:off])


@pytest.mark.parametrize("M", [4097, 5001, 12345, 30001])
@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (0, 13)])
def test_single_pass_any_length(M, ub, jwt):
    """Odd lengths at the packed stride M: rows no tensor map can describe,
    so the default plan's launch falls back to the single pass, which moves
    every row with plain loads and stores."""
    rng = np.random.default_rng(M + 10 * ub + jwt)
    case, bands, rhs = _case(rng, M, 37, ub, jwt)
    x, shape, n = _run(case, bands, rhs)
    assert shape["streaming"] == 5 and n == 1, shape
    e, emax = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= TOL, (e, emax)


@pytest.mark.parametrize("path", [0, 3, 4])
@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (0, 13), (1, 11)])
@pytest.mark.parametrize("M", [4104, 4097, 5001, 12345, 30001])
def test_two_passes_any_length(M, ub, jwt, path):
    """Lengths that are not a multiple of the 16 rows per thread, with even
    strides (rows 16-byte aligned): two passes (pivot products for a
    tridiagonal solve, tables, pass 1, carries unless there is no solve,
    pass 2; kernelPath 0 and 3) or the single pass (tables and one
    cooperative launch; kernelPath 4), the last partial chunk moved by its
    thread with plain loads and stores; in place, against the oracle, with
    the rows between the systems left as they were."""
    import torch

    from pfsolve_b200.api import App, launch_count
    rng = np.random.default_rng(M + 7 * ub + jwt)
    stride = M + (M & 1) + 2
    case, bands, rhs = _case(rng, M, 37, ub, jwt, cfg_outputBufferStride=stride)
    tb = torch.from_numpy(np.ascontiguousarray(bands)).cuda()
    x = torch.from_numpy(np.array(rhs, copy=True)).cuda()
    app = App(buffer=tb, outputBuffer=x, **J.case_fields(case, kernelPath=path))
    n0 = launch_count()
    app.append(**J.launch_fields(case))
    torch.cuda.synchronize()
    solve = not (ub == 1 and jwt == 11)
    assert launch_count() - n0 == (1 if ub == 2 else 0) + (2 if path == 4 else (4 if solve else 3))
    got = x.cpu().numpy()
    app.close()
    e, emax = J.rel_err(got, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= TOL, (e, emax)
    gaps = np.concatenate([got[y * stride + M:(y + 1) * stride] for y in range(37)])
    ref_gaps = np.concatenate([rhs[y * stride + M:(y + 1) * stride] for y in range(37)])
    np.testing.assert_array_equal(gaps, ref_gaps)


@pytest.mark.parametrize("M,path,launches", [(16384, 0, 5), (16384, 4, 3), (12345, 0, 3)])
def test_long_default_forms_and_repeats(M, path, launches):
    """The default plan runs two passes (pivot products, tables, pass 1,
    carries, pass 2: five launches for a tridiagonal solve), and the single
    pass (tables and one cooperative launch: three) for launches whose rows
    no tensor map can describe (M = 12 345 at a stride of M); kernelPath 4
    asks for the single pass.
    Repeated launches of one plan (new flag epochs each time) give the same
    result."""
    import torch

    from pfsolve_b200.api import App, last_launch, launch_count
    rng = np.random.default_rng(5)
    B = 600
    case, bands, rhs = _case(rng, M, B, 2, 13)
    tb = torch.from_numpy(bands).cuda()
    base = torch.from_numpy(rhs).cuda()
    x = base.clone()
    app = App(buffer=tb, outputBuffer=x, **J.case_fields(case, kernelPath=path))
    n0 = launch_count()
    app.append()
    torch.cuda.synchronize()
    assert launch_count() - n0 == launches
    assert last_launch()["kernel"] == capi.PFSOLVE_KERNEL_LONG
    first = x.cpu().numpy()
    for _ in range(3):
        x.copy_(base)
        app.append()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(x.cpu().numpy(), first)
    e, _ = J.rel_err(first, O.jw_step(case, bands, rhs, "q"), case)
    assert e <= TOL
    app.close()


def test_cluster_device_status_clean():
    from pfsolve_b200.api import device_status
    assert device_status() == 0
