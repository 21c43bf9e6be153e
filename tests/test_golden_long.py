"""Long systems (N > 4352): golden vectors from the reference's own GPU path,
which splits such a system over several kernel launches with reduced systems
in its temporary buffer (multi-upload, pfSolve_InitializeApp.h:1540-1583;
tests/golden/make_golden.py --only long).

CPU: the oracle reproduces the tridiagonal fixtures (N = 4352 .. 16384) and the
single-launch bidiagonal one at N = 4352 (pins it); the reference's bidiagonal
multi-upload outputs are recorded as a defect (below).
GPU: the long-system kernels (the default plan: two passes, the single pass
for rows no tensor map can describe; two passes alone, kernelPath 3; the
single pass alone, kernelPath 4; the cluster kernel, kernelPath 2, up to
16 384 rows)
reproduce the fixtures through the C ABI, and match the oracle where the
reference's output is defective.
Tolerances as for the single-step fixtures: 2e-15 (oracle), 2e-13 (kernels
against the reference), 1e-13 (kernels against the oracle).
"""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "long", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FILES]

# The reference's reduced-system kernels (pfSolve_TridiagonalSolve.h:1795-1856,
# pfSolve_ReadWrite.h:2014-2198) carry the three bands of a tridiagonal
# solve; for the bidiagonal kinds (upperBanded 0/1) split over several
# launches its output is not the step: NaN everywhere (upperBanded 0,
# jw_type 13) or values up to 1e209 (upperBanded 1, jw_type 10).  The same
# kind at N = 4352, in one launch, matches the oracle.
LONG_REFERENCE_DEFECTS = {"long_ub1_t10_M4360", "long_ub0_t13_M4400"}


def load(path):
    z = np.load(path, allow_pickle=False)
    p = json.loads(str(z["params"]))
    for k in ("cfg_inputZeropad", "cfg_outputZeropad", "run_inputZeropad", "run_outputZeropad"):
        p[k] = tuple(p[k])
    return O.Case(**p), z["buffer"], z["rhs"], z["ref_out"]


def test_fixture_set_is_present():
    assert len(FILES) >= 8
    assert any(n.startswith("long_ub2") and n.endswith("M16384") for n in IDS)
    assert LONG_REFERENCE_DEFECTS <= set(IDS)


@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_oracle_against_reference(path):
    case, buf, rhs, ref = load(path)
    got = O.jw_step(case, buf, rhs, "q")
    name = os.path.basename(path)[:-4]
    if name in LONG_REFERENCE_DEFECTS:
        bad = ~np.isfinite(ref) | (np.abs(ref - got) > 0.5 * np.abs(got).max())
        assert bad.mean() > 0.05, "the reference's bidiagonal multi-upload output is expected to be wrong"
    else:
        assert np.abs(got - ref).max() <= 2e-15 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("kernel_path", [0, 3, 4, 2], ids=["default", "two_pass", "single_pass", "cluster"])
@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_kernel_against_reference(path, kernel_path):
    import jwcases as J
    case, buf, rhs, ref = load(path)
    if kernel_path == 2 and (case.M > 16384 or case.M % 8):
        pytest.skip("the cluster kernel holds one system of at most 8 x 2048 rows, a multiple of 8")
    if kernel_path == 3 and case.M % 2:
        pytest.skip("odd M at the packed stride: rows no tensor map can describe, which two passes alone refuse")
    name = os.path.basename(path)[:-4]
    got = J.run_app(case, buf, rhs, kernelPath=kernel_path)
    if name in LONG_REFERENCE_DEFECTS:
        ref, tol = O.jw_step(case, buf, rhs, "q"), 1e-13
    else:
        tol = 2e-13
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
