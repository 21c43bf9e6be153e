"""Golden vectors of K consecutive JW steps (numConsecutiveJWIterations = K),
produced by the reference's own GPU kernel (oracle/ref_harness.cpp driving the
unmodified PfSolve library; tests/golden/make_golden.py --only steps).

CPU: the oracle's K-step restatement reproduces every fixture (pins it).
GPU: the sm_100a K-step kernel reproduces every fixture through the C ABI.
Tolerance: max |x - ref| / max |ref| <= 2e-15 (oracle, __float128 rounded to
FP64) and <= 2e-13 (FP64 kernels), as for the single-step fixtures.
"""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "steps", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FILES]


def load(path):
    z = np.load(path, allow_pickle=False)
    p = json.loads(str(z["params"]))
    for k in ("cfg_inputZeropad", "cfg_outputZeropad", "run_inputZeropad", "run_outputZeropad"):
        p[k] = tuple(p[k])
    n = int(z["nbuf"])
    bufs = [z[f"buffer_{k}"] for k in range(n)]
    return O.Case(**p), int(z["K"]), bufs, z["rhs"], z["ref_out"]


def test_fixture_set_is_present():
    names = set(IDS)
    assert len(FILES) >= 30
    for ub in (0, 1, 2):
        assert any(n.startswith(f"steps_ub{ub}") for n in names)
    assert any(n.startswith("steps_onebuf") for n in names)


@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_oracle_matches_reference(path):
    case, K, bufs, rhs, ref = load(path)
    got = O.jw_steps(case, K, bufs if len(bufs) > 1 else bufs[0], rhs)
    assert np.abs(got - ref).max() <= 2e-15 * np.abs(ref).max()


def test_rows_beyond_last_step_untouched():
    """A shrinking run writes M - K + 1 rows: the rows that left the system
    keep their input values (the reference writes only the final M_size)."""
    path = [f for f in FILES if "steps_ub1_t10_K5_M250" in f][0]
    case, K, bufs, rhs, ref = load(path)
    M, S = case.M, case.out_stride
    for y in range(case.batch):
        tail = slice(y * S + M - K + 1, y * S + M)
        assert np.array_equal(ref[tail], rhs[tail])


def test_undefined_step_combinations_rejected():
    rng = np.random.default_rng(0)
    from pfsolve_b200 import workloads as WL
    for ub, jwt, K in [(2, 13, 3), (1, 13, 2), (0, 13, 2)]:
        case = O.Case(M=64, batch=1, upperBanded=ub, jw_type=jwt)
        with pytest.raises(ValueError):
            O.jw_steps(case, K, WL.steps_bands(rng, 64, ub, K), np.zeros(64 + K))


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_kernel_matches_reference(path):
    import jwcases as J
    case, K, bufs, rhs, ref = load(path)
    for path in (0, 1):  # sweep kernel where the buffers allow it; the K-step kernel
        got, shape = J.run_steps(case, K, bufs if len(bufs) > 1 else bufs[0], rhs, kernelPath=path)
        assert shape["streaming"] == (4 if path == 0 and case.upperBanded != 2 else 3), shape
        assert np.abs(got - ref).max() <= 2e-13 * np.abs(ref).max(), path
