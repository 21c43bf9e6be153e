"""Golden vectors of the FP32-storage precisions, produced by the reference's
own GPU kernels (tests/golden/make_golden.py --only f32, into
tests/golden/f32/): its default precision ("f32": FP32 storage and
arithmetic) and doublePrecisionFloatMemory ("f32mem": FP64 arithmetic on FP32
storage), for every JW mode, launch-time values, dgbmv and block layouts.

Tolerances, as max |x - ref| / max |ref|:
  * oracle vs reference: 2.5e-7 for f32mem (both round an exact-to-FP64
    result to FP32 once: one FP32 unit in the last place, 2^-23), 5e-6 for f32
    (the reference's FP32 rounding);
  * kernels vs reference: 2.5e-7 for f32mem, 2e-5 for f32 (two FP32 solves
    that order their operations differently).
"""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

import jwcases as J

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "f32", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FILES]


def load(path):
    z = np.load(path, allow_pickle=False)
    p = json.loads(str(z["params"]))
    for k in ("cfg_inputZeropad", "cfg_outputZeropad", "run_inputZeropad", "run_outputZeropad"):
        p[k] = tuple(p[k])
    return O.Case(**p), str(z["precision"]), z["buffer"], z["rhs"], z["ref_out"]


def oracle_out(case, buf, rhs):
    """The oracle on the FP32 inputs, rounded to FP32."""
    if case.block:
        return O.block(case, buf.astype(np.float64), rhs.astype(np.float64)).astype(np.float32)
    if case.LDA:
        return O.dgbmv(case, buf.astype(np.float64), rhs.astype(np.float64)).astype(np.float32)
    return O.jw_step(case, buf, rhs, "f32")


def test_fixture_set_is_present():
    names = set(IDS)
    assert len(FILES) >= 40, "FP32 fixtures missing: run make_golden.py --only f32 on a GPU"
    for prec in ("f32", "f32mem"):
        assert any(n.startswith(prec + "_jw_ub2") for n in names)
        assert any(n.startswith(prec + "_jw_ub0") for n in names)
        assert any(n.startswith(prec + "_jw_ub1") for n in names)
        assert any(n.startswith(prec + "_dgbmv") for n in names)
        assert any(n.startswith(prec + "_block") for n in names)


@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_oracle_matches_reference(path):
    case, prec, buf, rhs, ref = load(path)
    assert buf.dtype == np.float32 and rhs.dtype == np.float32 and ref.dtype == np.float32
    got = oracle_out(case, buf, rhs).astype(np.float64)
    ref = ref.astype(np.float64)
    tol = 2.5e-7 if prec == "f32mem" else 5e-6
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_kernels_match_reference(path):
    case, prec, buf, rhs, ref = load(path)
    got = J.run_app_prec(case, buf, rhs, prec).astype(np.float64)
    ref = ref.astype(np.float64)
    tol = 2.5e-7 if prec == "f32mem" else 2e-5
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
