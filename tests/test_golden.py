"""Golden vectors produced by the reference's own GPU kernels (the unmodified
PfSolve library driven by oracle/ref_harness.cpp; generated by
tests/golden/make_golden.py).

CPU: the oracle reproduces every fixture -- this pins the oracle.
GPU: the sm_100a kernels reproduce every fixture through the C ABI.
Tolerance: max |x - ref| / max |ref| <= 2e-15 for FP64 oracle vs reference
(the two differ only by the reference's FP64 rounding), <= 2e-13 for the FP64
kernels, <= 2e-6 for FP32 storage.
"""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

import jwcases as J

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load(path):
    z = np.load(path, allow_pickle=False)
    p = json.loads(str(z["params"]))
    for k in ("cfg_inputZeropad", "cfg_outputZeropad", "run_inputZeropad", "run_outputZeropad"):
        p[k] = tuple(p[k])
    return O.Case(**p), str(z["precision"]), z["buffer"], z["rhs"], z["ref_out"]


def oracle_out(case, prec, buf, rhs):
    if case.block:
        return O.block(case, buf, rhs)
    if case.LDA:
        return O.dgbmv(case, buf, rhs)
    return O.jw_step(case, buf, rhs, {"f32": "f32", "dd": "dd"}.get(prec, "q"))


def test_fixture_set_is_present():
    names = {os.path.basename(f) for f in FILES}
    assert len(FILES) >= 40
    assert any(n.startswith("jw_ub2") for n in names)
    assert any(n.startswith("dgbmv") for n in names)
    assert any(n.startswith("block") for n in names)


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_oracle_matches_reference(path):
    case, prec, buf, rhs, ref = load(path)
    got = oracle_out(case, prec, buf, rhs).astype(np.float64)
    ref = ref.astype(np.float64)
    tol = 2e-6 if prec == "f32" else 2e-15
    assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("path", [f for f in FILES if "_f32_" not in f and "_dd_" not in f],
                         ids=[os.path.basename(f)[:-4] for f in FILES if "_f32_" not in f and "_dd_" not in f])
def test_kernels_match_reference(path):
    case, prec, buf, rhs, ref = load(path)
    got = J.run_app(case, buf, rhs)
    assert np.abs(got - ref).max() <= 2e-13 * np.abs(ref).max()
