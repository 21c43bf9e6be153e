"""GPU parity of the long-system JW kernels, through the C ABI.

Systems of 4 096 < N <= 16 384 rows run on the two-pass kernel (slices, no
waits between CTAs; the default, PfSolveGetShape streaming = 5) or, with
kernelPath 2, on one thread-block cluster of 3, 4, 6 or 8 CTAs per system
(streaming = 2).  Every case checks that the plan chose the kernel asked for,
that the launch ran on it, and that every system matches the __float128
oracle to 1e-13 relative L2 (the FP64 tolerance of the other kernels).  The
app works in place, so the two-pass kernel's halo records are exercised."""
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


PATHS = {0: 5, 2: 2}  # kernelPath -> PfSolveGetShape streaming


@pytest.mark.parametrize("path", list(PATHS))
@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (1, 11), (1, 12), (0, 10), (0, 11), (0, 13)])
@pytest.mark.parametrize("M", [4104, 4360, 5000, 6000, 6144, 8192, 12000, 16384])
def test_long_modes_and_sizes(ub, jwt, M, path):
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
    M = 8192
    for B, kw in [(301, {}), (65, dict(bitmask=capi.RUNTIME_INPUTZEROPAD, run_inputZeropad=(5, 8000))),
                  (2000, {}), (40, dict(bitmask=capi.RUNTIME_INPUTZEROPAD, run_inputZeropad=(1030, 3100)))]:
        case, bands, rhs = _case(rng, M, B, 2, 13, **kw)
        x, shape, n = _run(case, bands, rhs, kernelPath=path)
        assert n == 1
        e, _ = J.rel_err(x, O.jw_step(case, bands, rhs, "q"), case)
        assert e <= TOL


@pytest.mark.parametrize("path", list(PATHS))
def test_long_rejects_buffers_it_cannot_take(path):
    """No group-kernel fallback exists beyond 4096 rows: a misaligned launch
    returns UNSUPPORTED_COMBINATION instead of running."""
    rng = np.random.default_rng(3)
    case, bands, rhs = _case(rng, 6144, 3, 2, 13, bitmask=capi.RUNTIME_OFFSETSOLUTION, run_offsetSolution=1)
    with pytest.raises(capi.PfSolveError) as ei:
        _run(case, bands, rhs, kernelPath=path)
    assert ei.value.code == capi.PFSOLVE_ERROR_UNSUPPORTED_COMBINATION


def test_cluster_device_status_clean():
    from pfsolve_b200.api import device_status
    assert device_status() == 0
