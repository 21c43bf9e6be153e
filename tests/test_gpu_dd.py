"""Double-double (quad emulation) JW steps on the GPU against the __float128
oracle, through the C ABI.

Tolerances: double-double storage <= 1e-27 relative L2 per system (the
format carries ~106 significand bits; the oracle 113); double-double
arithmetic on FP64 storage: the result is the correctly rounded FP64 of a
quad-accurate solve, <= 2e-16 relative L2.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import workloads as WL

import jwcases as J

pytestmark = pytest.mark.gpu


def run_dd(case, bands, rhs, **extra):
    return J.run_app(case, bands, rhs, doublePrecision=0, quadDoubleDoublePrecision=1, **extra)


@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (0, 10), (1, 11), (0, 11), (1, 12), (0, 12), (1, 13), (0, 13)])
@pytest.mark.parametrize("M", [33, 256, 513, 1024])
def test_dd_storage_modes(ub, jwt, M):
    rng = np.random.default_rng(900 + 10 * ub + jwt + M)
    bands = WL.permute_bands(J.random_bands(rng, M, ub), M)
    case = O.Case(M=M, batch=9, upperBanded=ub, jw_type=jwt)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    # give the inputs genuine low parts so the double-double path is exercised
    bdd = O.to_dd(bands)
    bdd[1::2] = bands * rng.uniform(-1, 1, bands.shape) * 2.0 ** -60
    rdd = O.to_dd(rhs)
    rdd[1::2] = rhs * rng.uniform(-1, 1, rhs.shape) * 2.0 ** -60
    got = J.run_app(case, bdd, rdd, doublePrecision=0, quadDoubleDoublePrecision=1)
    ref = O.jw_step(case, bdd, rdd, "dd")
    e, _ = O.rel_errors_dd(got, ref, case.M, case.batch, case.out_stride, case.offset_solution)
    assert e <= 1e-27, e


def test_dd_double_memory_config3():
    wl = WL.config3(B=128)
    case = O.Case(M=wl.M, batch=wl.nrhs, upperBanded=2, jw_type=13)
    got = J.run_app(case, wl.jw_bands, wl.rhs, doublePrecision=0, quadDoubleDoublePrecisionDoubleMemory=1)
    ref = O.jw_step(case, wl.jw_bands, wl.rhs, "q")
    e, _ = O.rel_errors(got, ref, case.M, case.batch, case.M)
    assert e <= 2e-16, e


@pytest.mark.parametrize("rows", [0, 4, 8, 16])
@pytest.mark.parametrize("ub,jwt", [(2, 13), (1, 10), (0, 13), (1, 11)])
@pytest.mark.parametrize("M", [200, 512, 1000])
def test_dd_table_and_register_forms(ub, jwt, M, rows):
    """Both forms of the double-double kernel on many systems per group (so
    every group swaps its staging buffers several times): the table form
    (coefficients, chunk products and scan multipliers built once per CTA in
    shared memory; the default, 16 rows per thread for systems of up to 512
    rows, else 8) and the register form (rowsPerThread 4), against the
    __float128 oracle at 1e-27 relative L2 per system."""
    from pfsolve_b200.api import App
    import torch
    rng = np.random.default_rng(4000 + 10 * ub + jwt + M + rows)
    bands = WL.permute_bands(J.random_bands(rng, M, ub), M)
    case = O.Case(M=M, batch=700, upperBanded=ub, jw_type=jwt)
    rhs = rng.uniform(-1, 1, case.rhs_len())
    bdd = O.to_dd(bands)
    bdd[1::2] = bands * rng.uniform(-1, 1, bands.shape) * 2.0 ** -60
    rdd = O.to_dd(rhs)
    rdd[1::2] = rhs * rng.uniform(-1, 1, rhs.shape) * 2.0 ** -60
    tb = torch.from_numpy(bdd).cuda()
    to = torch.from_numpy(rdd.copy()).cuda()
    app = App(buffer=tb, outputBuffer=to,
              **J.case_fields(case, doublePrecision=0, quadDoubleDoublePrecision=1, rowsPerThread=rows))
    want = rows if rows else (16 if M <= 512 else 8)
    assert app.shape()["rowsPerThread"] == want, app.shape()
    app.append(**J.launch_fields(case))
    torch.cuda.synchronize()
    got = to.cpu().numpy()
    app.close()
    ref = O.jw_step(case, bdd, rdd, "dd")
    e, _ = O.rel_errors_dd(got, ref, case.M, case.batch, case.out_stride, case.offset_solution)
    assert e <= 1e-27, e
