"""Python access to the test oracle (TEST INFRASTRUCTURE ONLY).

Wraps ``oracle/libjw_oracle.so`` -- the CPU restatement of PfSolve's
Jones-Worland step, dgbmv and block kernels in ``__float128`` and ``double``
(see ``jw_oracle.h`` for the reference citations) -- and drives the reference's
own library through ``oracle/_ref/pfsolve_ref`` to produce golden vectors.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.  The product (``pfsolve_b200``) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field, fields

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjw_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "pfsolve_ref")

RUNTIME_MSIZE = 1
RUNTIME_OFFSETM = 2
RUNTIME_OFFSETV = 4
RUNTIME_OFFSETSOLUTION = 8
RUNTIME_INPUTZEROPAD = 16
RUNTIME_OUTPUTZEROPAD = 32
RUNTIME_SCALEC = 64
RUNTIME_INPUTBUFFERSTRIDE = 128
RUNTIME_OUTPUTBUFFERSTRIDE = 256

MV_NONE, MV_DIAG, MV_UPPER, MV_LOWER = 0, 1, 2, 3
SV_NONE, SV_LOWER, SV_UPPER, SV_TRI = 0, 1, 2, 3


class _Params(ctypes.Structure):
    _fields_ = [
        ("M", ctypes.c_int64), ("batch", ctypes.c_int64),
        ("upperBanded", ctypes.c_int32), ("jw_type", ctypes.c_int32),
        ("bitmask", ctypes.c_int64),
        ("cfg_offsetM", ctypes.c_int64), ("cfg_offsetV", ctypes.c_int64),
        ("cfg_offsetSolution", ctypes.c_int64),
        ("cfg_inputZeropad", ctypes.c_int64 * 2), ("cfg_outputZeropad", ctypes.c_int64 * 2),
        ("cfg_inputBufferStride", ctypes.c_int64), ("cfg_outputBufferStride", ctypes.c_int64),
        ("cfg_scaleC", ctypes.c_double),
        ("run_offsetM", ctypes.c_int64), ("run_offsetV", ctypes.c_int64),
        ("run_offsetSolution", ctypes.c_int64),
        ("run_inputZeropad", ctypes.c_int64 * 2), ("run_outputZeropad", ctypes.c_int64 * 2),
        ("run_inputBufferStride", ctypes.c_int64), ("run_outputBufferStride", ctypes.c_int64),
        ("run_scaleC", ctypes.c_double),
        ("bandsPermuted", ctypes.c_int32),
        ("LDA", ctypes.c_int32), ("KU", ctypes.c_int32), ("KL", ctypes.c_int32),
        ("block", ctypes.c_int32), ("lshift", ctypes.c_int32),
        ("size0", ctypes.c_int64), ("size1", ctypes.c_int64),
        ("ALT_dgbmv", ctypes.c_int32),
    ]


class _Step(ctypes.Structure):
    _fields_ = [("M", ctypes.c_int64), ("r", ctypes.c_int64),
                ("mv", ctypes.c_int32), ("sv", ctypes.c_int32), ("diag", ctypes.c_int32),
                ("off_md", ctypes.c_int64), ("off_mo", ctypes.c_int64),
                ("off_sl", ctypes.c_int64), ("off_su", ctypes.c_int64)]


@dataclass
class Case:
    """Plan-time and launch-time values of one PfSolve application.

    Field names follow ``PfSolveConfiguration`` (``cfg_*``) and
    ``PfSolveLaunchParams`` (``run_*``) of the reference
    (PfSolve/pfSolve_Structs/pfSolve_Structs.h:119-449).
    """
    M: int
    batch: int
    upperBanded: int = 2
    jw_type: int = 13
    bitmask: int = 0
    cfg_offsetM: int = 0
    cfg_offsetV: int = 0
    cfg_offsetSolution: int = 0
    cfg_inputZeropad: tuple = (0, 0)
    cfg_outputZeropad: tuple = (0, 0)
    cfg_inputBufferStride: int = 0
    cfg_outputBufferStride: int = 0
    cfg_scaleC: float = 1.0
    run_offsetM: int = 0
    run_offsetV: int = 0
    run_offsetSolution: int = 0
    run_inputZeropad: tuple = (0, 0)
    run_outputZeropad: tuple = (0, 0)
    run_inputBufferStride: int = 0
    run_outputBufferStride: int = 0
    run_scaleC: float = 1.0
    bandsPermuted: int = 1
    LDA: int = 0
    KU: int = 0
    KL: int = 0
    block: int = 0
    lshift: int = 0
    size0: int = 0
    size1: int = 0
    ALT_dgbmv: int = 0

    def __post_init__(self):
        if self.cfg_inputBufferStride == 0:
            self.cfg_inputBufferStride = self.M
        if self.cfg_outputBufferStride == 0:
            self.cfg_outputBufferStride = self.M
        if self.run_inputBufferStride == 0:
            self.run_inputBufferStride = self.cfg_inputBufferStride
        if self.run_outputBufferStride == 0:
            self.run_outputBufferStride = self.cfg_outputBufferStride
        if self.size0 == 0:
            self.size0 = self.M
        if self.size1 == 0:
            self.size1 = self.batch

    def resolved(self, bit, name):
        return getattr(self, "run_" + name) if (self.bitmask & bit) else getattr(self, "cfg_" + name)

    @property
    def out_stride(self):
        return self.resolved(RUNTIME_OUTPUTBUFFERSTRIDE, "outputBufferStride")

    @property
    def in_stride(self):
        return self.resolved(RUNTIME_INPUTBUFFERSTRIDE, "inputBufferStride")

    @property
    def offset_solution(self):
        return self.resolved(RUNTIME_OFFSETSOLUTION, "offsetSolution")

    def rhs_len(self):
        """Elements the RHS buffer must hold for this case."""
        return self.offset_solution + (self.batch - 1) * self.out_stride + self.M

    def to_c(self) -> _Params:
        p = _Params()
        for f in fields(self):
            v = getattr(self, f.name)
            if isinstance(v, tuple):
                arr = getattr(p, f.name)
                arr[0], arr[1] = int(v[0]), int(v[1])
            else:
                setattr(p, f.name, v)
        return p


_lib = None


def lib():
    """Load (building on first use when the C compiler is present) the oracle library."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER(_Params)
    dp = ctypes.POINTER(ctypes.c_double)
    fp = ctypes.POINTER(ctypes.c_float)
    L.pfo_reorder_i0.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]
    L.pfo_reorder_i0.restype = ctypes.c_int64
    for name, bt in (("pfo_jw_step_q", dp), ("pfo_jw_step_d", dp), ("pfo_jw_step_q_dd", dp),
                     ("pfo_dgbmv_q", dp), ("pfo_dgbmv_d", dp)):
        fn = getattr(L, name)
        fn.argtypes = [P, bt, bt, ctypes.c_int]
        fn.restype = ctypes.c_int
    L.pfo_jw_step_q_f32.argtypes = [P, fp, fp, ctypes.c_int]
    L.pfo_jw_step_q_f32.restype = ctypes.c_int
    L.pfo_block_q.argtypes = [P, dp, dp]
    L.pfo_block_q.restype = ctypes.c_int
    L.pfo_jw_operator.argtypes = [P, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  dp, dp, dp, dp]
    L.pfo_jw_operator.restype = ctypes.c_int
    L.pfo_scale_factor.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_double]
    L.pfo_scale_factor.restype = ctypes.c_double
    L.pfo_rel_errors.argtypes = [dp, dp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                 dp, dp]
    L.pfo_rel_errors.restype = None
    L.pfo_rel_errors_dd.argtypes = L.pfo_rel_errors.argtypes
    L.pfo_rel_errors_dd.restype = None
    for name in ("pfo_jw_steps_q", "pfo_jw_steps_d"):
        fn = getattr(L, name)
        fn.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(dp), dp, ctypes.c_int]
        fn.restype = ctypes.c_int
    L.pfo_alt_position.argtypes = [ctypes.c_int64, ctypes.c_int64]
    L.pfo_alt_position.restype = ctypes.c_int64
    L.pfo_jw_step_alt_q.argtypes = [P, dp, dp, ctypes.c_int]
    L.pfo_jw_step_alt_q.restype = ctypes.c_int
    L.pfo_steps_registers.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int]
    L.pfo_steps_registers.restype = ctypes.c_int64
    L.pfo_jw_steps_layout.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Step)]
    L.pfo_jw_steps_layout.restype = ctypes.c_int
    L.pfo_dct_q.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, dp, ctypes.c_int64, dp, ctypes.c_int64,
                            ctypes.c_int]
    L.pfo_dct_q.restype = ctypes.c_int
    _lib = L
    return L


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def reorder_i0(i, M, Msplit0=0):
    return lib().pfo_reorder_i0(int(i), int(M), int(Msplit0))


def permutation(M):
    """perm[i] = storage position of logical row i in the reference's band layout."""
    L = lib()
    return np.array([L.pfo_reorder_i0(i, M, 0) for i in range(M)], dtype=np.int64)


def permute_bands(natural, M):
    """Natural-order bands (k*M + i) -> reference register-major storage."""
    natural = np.asarray(natural)
    nb = natural.shape[0] // M
    out = np.empty_like(natural)
    perm = permutation(M)
    for k in range(nb):
        out[k * M + perm] = natural[k * M:(k + 1) * M]
    return out


def jw_operator(case: Case, bands: np.ndarray):
    """(mv_kind, sv_kind, md, mo, sl, su) in natural row order."""
    M = case.M
    arrs = [np.zeros(M) for _ in range(4)]
    mv = ctypes.c_int()
    sv = ctypes.c_int()
    b = np.ascontiguousarray(bands, dtype=np.float64)
    rc = lib().pfo_jw_operator(ctypes.byref(case.to_c()), _dptr(b), ctypes.byref(mv), ctypes.byref(sv),
                               *[_dptr(a) for a in arrs])
    if rc:
        raise ValueError("combination not defined by the reference")
    return mv.value, sv.value, *arrs


def jw_step(case: Case, bands: np.ndarray, rhs: np.ndarray, mode: str = "q", nthreads: int = 1) -> np.ndarray:
    """One JW step on a copy of ``rhs``.  mode: 'q' (__float128), 'd' (double),
    'f32' (float storage), 'dd' (double-double storage: arrays of {hi, lo} pairs)."""
    p = case.to_c()
    L = lib()
    if mode == "f32":
        b = np.ascontiguousarray(bands, dtype=np.float32)
        out = np.array(rhs, dtype=np.float32, copy=True)
        rc = L.pfo_jw_step_q_f32(ctypes.byref(p), b.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), nthreads)
    else:
        b = np.ascontiguousarray(bands, dtype=np.float64)
        out = np.array(rhs, dtype=np.float64, copy=True)
        fn = {"q": L.pfo_jw_step_q, "d": L.pfo_jw_step_d, "dd": L.pfo_jw_step_q_dd}[mode]
        rc = fn(ctypes.byref(p), _dptr(b), _dptr(out), nthreads)
    if rc:
        raise ValueError("combination not defined by the reference")
    return out


def alt_positions(M):
    """Storage position of row r in the ALT band layout (stride-2 mode)."""
    L = lib()
    return np.array([L.pfo_alt_position(r, M) for r in range(M)], dtype=np.int64)


def jw_step_alt(case: Case, bands: np.ndarray, rhs: np.ndarray, nthreads: int = 1) -> np.ndarray:
    """One ALT-mode JW step (jw_type / 100 % 10 == 1) on a copy of ``rhs``."""
    b = np.ascontiguousarray(bands, dtype=np.float64)
    out = np.array(rhs, dtype=np.float64, copy=True)
    if lib().pfo_jw_step_alt_q(ctypes.byref(case.to_c()), _dptr(b), _dptr(out), nthreads):
        raise ValueError("combination not defined by the reference")
    return out


def steps_layout(case: Case, K: int, s: int) -> dict:
    """Rows, band-order register count, operator kinds and band offsets of step
    ``s`` of a K-step application (raises for undefined combinations)."""
    st = _Step()
    if lib().pfo_jw_steps_layout(ctypes.byref(case.to_c()), int(K), int(s), ctypes.byref(st)):
        raise ValueError("combination not defined by the reference")
    return {f: getattr(st, f) for f, _ in _Step._fields_}


def steps_permutation(M, r):
    """Register-major band order of M rows with r registers per lane."""
    i = np.arange(M, dtype=np.int64)
    t, j = i // r, i % r
    m, ce, fl = M % r, -(-M // r), M // r
    return t + np.where(j < m, j * ce, m * ce + (j - m) * fl)


def jw_steps(case: Case, K: int, bands, rhs: np.ndarray, mode: str = "q", nthreads: int = 1) -> np.ndarray:
    """K consecutive JW steps on a copy of ``rhs``; ``bands`` is one buffer read
    by every step or a list of K per-step buffers."""
    bufs = [np.ascontiguousarray(b, dtype=np.float64) for b in (bands if isinstance(bands, (list, tuple)) else [bands])]
    arr = (ctypes.POINTER(ctypes.c_double) * len(bufs))(*[_dptr(b) for b in bufs])
    out = np.array(rhs, dtype=np.float64, copy=True)
    fn = lib().pfo_jw_steps_q if mode == "q" else lib().pfo_jw_steps_d
    if fn(ctypes.byref(case.to_c()), int(K), len(bufs), arr, _dptr(out), nthreads):
        raise ValueError("combination not defined by the reference")
    return out


def dgbmv(case: Case, A: np.ndarray, rhs: np.ndarray, mode: str = "q", nthreads: int = 1) -> np.ndarray:
    out = np.array(rhs, dtype=np.float64, copy=True)
    a = np.ascontiguousarray(A, dtype=np.float64)
    fn = lib().pfo_dgbmv_q if mode == "q" else lib().pfo_dgbmv_d
    if fn(ctypes.byref(case.to_c()), _dptr(a), _dptr(out), nthreads):
        raise ValueError("invalid dgbmv parameters")
    return out


def block(case: Case, inp: np.ndarray, out: np.ndarray) -> np.ndarray:
    o = np.array(out, dtype=np.float64, copy=True)
    i = np.ascontiguousarray(inp, dtype=np.float64)
    if lib().pfo_block_q(ctypes.byref(case.to_c()), _dptr(i), _dptr(o)):
        raise ValueError("block combination not defined by the reference")
    return o


def scale_factor(kind, x, lshift, s):
    return lib().pfo_scale_factor(int(kind), int(x), int(lshift), float(s))


def rel_errors(a, ref, M, batch, stride, offset=0):
    """(max over systems of relative L2 error, max-abs error / max-abs value)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    r = np.ascontiguousarray(ref, dtype=np.float64)
    e1 = ctypes.c_double()
    e2 = ctypes.c_double()
    lib().pfo_rel_errors(_dptr(a), _dptr(r), M, batch, stride, offset, ctypes.byref(e1), ctypes.byref(e2))
    return e1.value, e2.value


def rel_errors_dd(a, ref, M, batch, stride, offset=0):
    """rel_errors for double-double arrays ({hi, lo} pairs), evaluated in __float128."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    r = np.ascontiguousarray(ref, dtype=np.float64)
    e1 = ctypes.c_double()
    e2 = ctypes.c_double()
    lib().pfo_rel_errors_dd(_dptr(a), _dptr(r), M, batch, stride, offset, ctypes.byref(e1), ctypes.byref(e2))
    return e1.value, e2.value


def to_dd(x):
    """FP64 array -> double-double pairs {x, 0}."""
    x = np.asarray(x, dtype=np.float64)
    return np.stack([x, np.zeros_like(x)], -1).ravel()


# --------------------------------------------------------------------------
# The reference itself (oracle/_ref/pfsolve_ref, built from the reference's
# sources by `make -C oracle ref`; runs only where a GPU is present).

def reference_available() -> bool:
    return os.path.exists(REF_BIN)


def write_reference_case(case_dir: str, case: Case, bands, rhs: np.ndarray, *,
                         precision: str = "f64", inp: np.ndarray | None = None, iters: int = 0, K: int = 1):
    """Write the files ``pfsolve_ref`` reads for one case.  ``bands`` may be a
    list of per-step buffers (K consecutive steps with one input buffer each)."""
    os.makedirs(case_dir, exist_ok=True)
    kv = {
        "M": case.M, "size0": case.size0, "size1": case.size1 if (case.block) else case.batch,
        "jw_type": case.jw_type, "upperBanded": case.upperBanded, "bitmask": case.bitmask,
        "cfg_offsetM": case.cfg_offsetM, "cfg_offsetV": case.cfg_offsetV,
        "cfg_offsetSolution": case.cfg_offsetSolution,
        "cfg_iz0": case.cfg_inputZeropad[0], "cfg_iz1": case.cfg_inputZeropad[1],
        "cfg_oz0": case.cfg_outputZeropad[0], "cfg_oz1": case.cfg_outputZeropad[1],
        "cfg_scaleC": repr(float(case.cfg_scaleC)),
        "cfg_inputBufferStride": case.cfg_inputBufferStride,
        "cfg_outputBufferStride": case.cfg_outputBufferStride,
        "run_offsetM": case.run_offsetM, "run_offsetV": case.run_offsetV,
        "run_offsetSolution": case.run_offsetSolution,
        "run_iz0": case.run_inputZeropad[0], "run_iz1": case.run_inputZeropad[1],
        "run_oz0": case.run_outputZeropad[0], "run_oz1": case.run_outputZeropad[1],
        "run_scaleC": repr(float(case.run_scaleC)),
        "run_inputBufferStride": case.run_inputBufferStride,
        "run_outputBufferStride": case.run_outputBufferStride,
        "LDA": case.LDA, "KU": case.KU, "KL": case.KL, "block": case.block, "lshift": case.lshift,
        "ALT_dgbmv": case.ALT_dgbmv,
        "doublePrecision": 1 if precision in ("f64",) else 0,
        "doublePrecisionFloatMemory": 1 if precision == "f32mem" else 0,
        "quadDoubleDoublePrecision": 1 if precision == "dd" else 0,
        "iters": iters,
        "K": K,
        # K > 1 on one buffer: no multiple-buffer binding (inputs<k> would not exist)
        "useMultipleInputBuffers": len(bands) if isinstance(bands, (list, tuple)) else (1 if K == 1 else 0),
    }
    with open(os.path.join(case_dir, "params.txt"), "w") as f:
        for k, v in kv.items():
            f.write(f"{k}={v}\n")
    dt = np.float32 if precision in ("f32", "f32mem") else np.float64
    if isinstance(bands, (list, tuple)):
        for k, b in enumerate(bands):
            np.ascontiguousarray(b, dtype=dt).tofile(os.path.join(case_dir, f"bands_{k}.bin"))
    elif bands is not None:
        np.ascontiguousarray(bands, dtype=dt).tofile(os.path.join(case_dir, "bands.bin"))
    np.ascontiguousarray(rhs, dtype=dt).tofile(os.path.join(case_dir, "rhs.bin"))
    if inp is not None:
        np.ascontiguousarray(inp, dtype=dt).tofile(os.path.join(case_dir, "in.bin"))


def run_reference(case_dir: str, timeout: float = 120.0):
    """Run the reference on one case directory; returns (output array bytes path, ms or None)."""
    r = subprocess.run([REF_BIN, case_dir], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"pfsolve_ref failed ({r.returncode}): {r.stderr.strip()}")
    t = None
    tp = os.path.join(case_dir, "time.txt")
    if os.path.exists(tp):
        t = float(open(tp).read().strip())
    return os.path.join(case_dir, "out.bin"), t


def dct(dct_type: int, x: np.ndarray, N: int, nsys: int, in_stride: int = 0, out_stride: int = 0,
        nthreads: int = 4) -> np.ndarray:
    """The DCT step (type 2 or 3, FFTW's unnormalized REDFT10 / REDFT01) of
    nsys rows of N points, in __float128 (pfo_dct_q); rows at in_stride
    (default N), results packed at out_stride (default N)."""
    in_stride = in_stride or N
    out_stride = out_stride or N
    xi = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(max(1, (nsys - 1) * out_stride + N))
    if lib().pfo_dct_q(int(dct_type), N, nsys, _dptr(xi), in_stride, _dptr(out), out_stride, nthreads) != 0:
        raise ValueError("DCT type must be 2 or 3")
    return out
