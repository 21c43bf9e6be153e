"""Double-double JW steps: golden vectors from the reference's own
double-double app (quadDoubleDoublePrecision = 1, {hi, lo} storage with
non-zero lo parts; tests/golden/make_golden.py --only dd).

The reference generates these kernels only for the bidiagonal kinds at
M <= 32 with one step (its sequential-Thomas generation,
pfSolve_Plan_JonesWorland.h:306); for every other case its double-double code
generation stops with SIGSEGV inside initializePfSolve (a double-double
constant moved into a register with its {hi, lo} parts unset,
pfSolve_ReadWrite.h:1567-1682, pfSolve_TridiagonalSolve.h:1048), so no larger
fixture exists.  Larger sizes and the tridiagonal kind are checked against the
__float128 oracle in test_gpu_dd.py.

CPU: the oracle reproduces the reference's double-double outputs to <= 1e-30
relative (seen: 1.2e-32; the {hi, lo} format carries ~106 bits).
GPU: the double-double kernel reproduces them through the C ABI to <= 1e-27
relative L2 per system, the tolerance its oracle tests use.
"""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "dd", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FILES]


def load(path):
    z = np.load(path, allow_pickle=False)
    p = json.loads(str(z["params"]))
    for k in ("cfg_inputZeropad", "cfg_outputZeropad", "run_inputZeropad", "run_outputZeropad"):
        p[k] = tuple(p[k])
    assert str(z["precision"]) == "dd"
    return O.Case(**p), z["buffer"], z["rhs"], z["ref_out"]


def dd_value_error(a, b):
    """max |a - b| / max |b| over {hi, lo} pairs, formed as (hi_a - hi_b) + (lo_a - lo_b)."""
    d = (a[0::2] - b[0::2]) + (a[1::2] - b[1::2])
    return np.abs(d).max() / np.abs(b[0::2]).max()


def test_fixture_set_is_present():
    assert len(FILES) >= 3
    assert {"dd_ub1_t10_M16", "dd_ub1_t10_M32", "dd_ub0_t13_M32"} <= set(IDS)


@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_fixture_inputs_carry_low_parts(path):
    case, buf, rhs, ref = load(path)
    assert np.count_nonzero(buf[1::2]) > 0 and np.count_nonzero(rhs[1::2]) > 0
    # the reference's outputs are genuine double-double values, not FP64
    assert np.count_nonzero(ref[1::2]) > ref.size // 4


@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_oracle_against_reference(path):
    case, buf, rhs, ref = load(path)
    got = O.jw_step(case, buf, rhs, "dd")
    assert dd_value_error(got, ref) <= 1e-30


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_kernel_against_reference(path):
    import jwcases as J
    case, buf, rhs, ref = load(path)
    got = J.run_app(case, buf, rhs, doublePrecision=0, quadDoubleDoublePrecision=1)
    e, _ = O.rel_errors_dd(got, ref, case.M, case.batch, case.out_stride, case.offset_solution)
    assert e <= 1e-27, e
    assert dd_value_error(got, ref) <= 1e-27
