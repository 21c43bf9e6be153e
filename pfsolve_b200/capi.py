"""ctypes binding of the C ABI in ``include/pfsolve_b200.h``.

The structures mirror the header field for field; ``tests/test_abi.py`` checks
their sizes against the compiled library's own view.  The library is the
in-tree ``pfsolve_b200/libpfsolve_b200.so``; importing this module never falls
back to anything else -- a missing library raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfsolve_b200.so")

RUNTIME_MSIZE = 1
RUNTIME_OFFSETM = 2
RUNTIME_OFFSETV = 4
RUNTIME_OFFSETSOLUTION = 8
RUNTIME_INPUTZEROPAD = 16
RUNTIME_OUTPUTZEROPAD = 32
RUNTIME_SCALEC = 64
RUNTIME_INPUTBUFFERSTRIDE = 128
RUNTIME_OUTPUTBUFFERSTRIDE = 256

BLOCK_READ_REAL_WRITE_REAL = 1
BLOCK_READ_COMPLEX_R_WRITE_REAL = 2
BLOCK_READ_COMPLEX_I_WRITE_REAL = 3
BLOCK_READ_COMPLEX_STRIDED_WRITE_COMPLEX_PACKED = 4
BLOCK_READ_REAL_WRITE_COMPLEX_R = 5
BLOCK_READ_REAL_WRITE_COMPLEX_I = 6
BLOCK_READ_COMPLEX_PACKED_WRITE_COMPLEX_STRIDED = 7
BLOCK_ADD_OUTPUTBUFFER_VALUES = 20
BLOCK_SCALEC = 100
BLOCK_SCALED = 200
BLOCK_SCALESPHLAPLA = 300
BLOCK_SCALESPHLAPLB = 400

PFSOLVE_SUCCESS = 0
PFSOLVE_ERROR_INVALID_DEVICE = 1002
PFSOLVE_ERROR_EMPTY_FFTdim = 2001
PFSOLVE_ERROR_EMPTY_size = 2002
PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH = 3002
PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_DCT = 3004
PFSOLVE_ERROR_UNSUPPORTED_COMBINATION = 5001
PFSOLVE_ERROR_INVALID_ARGUMENT = 5002
PFSOLVE_ERROR_CAPACITY = 5003

u64 = ctypes.c_uint64
i64 = ctypes.c_int64
c_int = ctypes.c_int
vpp = ctypes.POINTER(ctypes.c_void_p)


class PfSolveConfiguration(ctypes.Structure):
    _fields_ = [
        ("FFTdim", u64), ("size", u64 * 3),
        ("device", ctypes.POINTER(c_int)), ("stream", ctypes.POINTER(ctypes.c_void_p)), ("num_streams", u64),
        ("bufferSize", ctypes.POINTER(u64)), ("outputBufferSize", ctypes.POINTER(u64)),
        ("kernelSize", ctypes.POINTER(u64)),
        ("buffer", vpp), ("outputBuffer", vpp), ("kernel", vpp),
        ("upperBanded", c_int), ("jw_type", c_int), ("block", c_int), ("lshift", c_int),
        ("LDA", c_int), ("KU", c_int), ("KL", c_int), ("ALT_dgbmv", c_int),
        ("Msplit", u64 * 3), ("performDCT", u64),
        ("jw_control_bitmask", i64), ("M_size", i64), ("offsetM", i64), ("offsetV", i64),
        ("offsetSolution", i64), ("inputZeropad", i64 * 2), ("outputZeropad", i64 * 2),
        ("scaleC", ctypes.c_double),
        ("doublePrecision", u64), ("quadDoubleDoublePrecision", u64),
        ("quadDoubleDoublePrecisionDoubleMemory", u64), ("halfPrecision", u64),
        ("doublePrecisionFloatMemory", u64),
        ("inputBufferStride", u64 * 3), ("outputBufferStride", u64 * 3),
        ("isInputFormatted", u64), ("isOutputFormatted", u64),
        ("keepShaderCode", u64), ("printMemoryLayout", u64), ("disableCaching", c_int),
        ("disableSetLocale", u64), ("useUint64", u64),
        ("numConsecutiveJWIterations", c_int), ("useMultipleInputBuffers", c_int),
        ("mixedPrecisionRefinement", c_int), ("rowsPerThread", c_int), ("kernelPath", c_int),
        ("stagingBuffers", c_int),
    ]


class PfSolveLaunchParams(ctypes.Structure):
    _fields_ = [
        ("buffer", vpp), ("outputBuffer", vpp), ("kernel", vpp),
        ("M_size", u64), ("offsetM", u64), ("offsetV", u64), ("offsetSolution", u64),
        ("inputZeropad", u64 * 2), ("outputZeropad", u64 * 2),
        ("scaleC", ctypes.c_longdouble),
        ("inputBufferStride", u64), ("outputBufferStride", u64), ("batchSize", u64),
    ]


class PfSolveApplication(ctypes.Structure):
    _fields_ = [("configuration", PfSolveConfiguration), ("internal", ctypes.c_void_p)]


class MapKeyJW(ctypes.Structure):
    _fields_ = [("size", i64 * 2), ("upperBanded", i64), ("outputBufferStride", i64), ("type", i64)]


class MapKeyDgbmv(ctypes.Structure):
    _fields_ = [("size", i64 * 2), ("outputBufferStride", i64), ("LDA", i64), ("KU", i64), ("KL", i64)]


class MapKeyBlock(ctypes.Structure):
    _fields_ = [("size", i64 * 2), ("inputBufferStride", i64), ("outputBufferStride", i64), ("type", i64),
                ("lshift", i64)]


class PfSolveBatchEntry(ctypes.Structure):
    _fields_ = [("M", i64), ("nsys", i64), ("bands", ctypes.c_void_p), ("dgbmvBands", ctypes.c_void_p),
                ("input", ctypes.c_void_p), ("output", ctypes.c_void_p), ("inputStride", i64),
                ("outputStride", i64), ("lshift", c_int), ("scaleS", ctypes.c_double), ("scaleC", ctypes.c_double)]


class PfSolveBatchDesc(ctypes.Structure):
    _fields_ = [("upperBanded", c_int), ("jw_type", c_int), ("LDA", c_int), ("KU", c_int), ("KL", c_int),
                ("block", c_int), ("mixedPrecisionRefinement", c_int), ("rowsPerThread", c_int),
                ("systemsPerItem", c_int), ("sweepRows", c_int)]


class PfSolveServerDesc(ctypes.Structure):
    _fields_ = [("device", c_int), ("hbmBudgetBytes", u64), ("streams", c_int), ("maxBatchRequests", c_int),
                ("refineSweeps", c_int)]


class PfSolveRequest(ctypes.Structure):
    _fields_ = [("op", c_int), ("precision", c_int), ("nrhs", i64), ("input", ctypes.c_void_p),
                ("output", ctypes.c_void_p), ("stride", i64), ("scaleC", ctypes.c_double),
                ("stream", ctypes.c_void_p), ("inputReady", c_int)]


class PfSolveLaunchInfo(ctypes.Structure):
    _fields_ = [("kernel", c_int), ("rowsPerThread", c_int), ("warpsPerSystem", c_int), ("groupsPerCTA", c_int),
                ("bandsBelow", c_int), ("bandsAbove", c_int), ("solve", c_int), ("layoutIn", c_int),
                ("layoutOut", c_int), ("scale", c_int), ("precision", c_int), ("alt", c_int), ("gridCTAs", i64)]


PFSOLVE_KERNEL_NONE, PFSOLVE_KERNEL_GROUP, PFSOLVE_KERNEL_STREAMING, PFSOLVE_KERNEL_LONG = 0, 1, 2, 3
PFSOLVE_KERNEL_CLUSTER, PFSOLVE_KERNEL_STEPS, PFSOLVE_KERNEL_STEPS_SWEEP = 4, 5, 6
PFSOLVE_KERNEL_DGBMV, PFSOLVE_KERNEL_BLOCK, PFSOLVE_KERNEL_DCT = 7, 8, 9


class PfSolveServerStats(ctypes.Structure):
    _fields_ = [("submitted", u64), ("completed", u64), ("batches", u64), ("rhs", u64),
                ("peakInflightBytes", u64), ("p50Ms", ctypes.c_double), ("p99Ms", ctypes.c_double),
                ("maxMs", ctypes.c_double), ("p99QueueMs", ctypes.c_double), ("p99DeviceMs", ctypes.c_double)]


PFSOLVE_SERVE_MIXED, PFSOLVE_SERVE_DD, PFSOLVE_SERVE_DD_FP64MEM = 1, 2, 3
PFSOLVE_NOALLOC_MAX_ENTRIES, PFSOLVE_NOALLOC_MAX_ITEMS = 1024, 16384

# Every function the header declares, with its ctypes signature.
_APP_P = ctypes.POINTER(PfSolveApplication)
_LP_P = ctypes.POINTER(PfSolveLaunchParams)
SIGNATURES = {
    "initializePfSolve": (c_int, [_APP_P, PfSolveConfiguration]),
    "PfSolveAppend": (c_int, [_APP_P, c_int, _LP_P]),
    "PfSolveSync": (c_int, [_APP_P]),
    "deletePfSolve": (None, [_APP_P]),
    "getPfSolveErrorString": (ctypes.c_char_p, [c_int]),
    "PfSolveGetVersion": (c_int, []),
    "PfSolveAppLibraryCreate": (ctypes.c_void_p, []),
    "PfSolveAppLibraryDestroy": (None, [ctypes.c_void_p]),
    "checkLibrary_JonesWorland": (c_int, [ctypes.c_void_p, MapKeyJW, ctypes.POINTER(_APP_P)]),
    "addToLibrary_JonesWorland": (c_int, [ctypes.c_void_p, MapKeyJW, _APP_P]),
    "checkLibrary_dgbmv": (c_int, [ctypes.c_void_p, MapKeyDgbmv, ctypes.POINTER(_APP_P)]),
    "addToLibrary_dgbmv": (c_int, [ctypes.c_void_p, MapKeyDgbmv, _APP_P]),
    "checkLibrary_block": (c_int, [ctypes.c_void_p, MapKeyBlock, ctypes.POINTER(_APP_P)]),
    "addToLibrary_block": (c_int, [ctypes.c_void_p, MapKeyBlock, _APP_P]),
    "PfSolveAppendChain": (c_int, [ctypes.POINTER(_APP_P), ctypes.POINTER(_LP_P), c_int, c_int]),
    "PfSolveLaunchCount": (u64, []),
    "PfSolveGetDeviceStatus": (c_int, []),
    "PfSolveGetShape": (c_int, [_APP_P] + [ctypes.POINTER(c_int)] * 4),
    "PfSolveStreamingLaunchCount": (u64, []),
    "PfSolveGetLastLaunch": (c_int, [ctypes.POINTER(PfSolveLaunchInfo)]),
    "PfSolveServerCreate": (c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(PfSolveServerDesc)]),
    "PfSolveServerAddOperator": (c_int, [ctypes.c_void_p, i64, ctypes.c_void_p, c_int, c_int,
                                         ctypes.POINTER(c_int)]),
    "PfSolveServerSubmit": (c_int, [ctypes.c_void_p, ctypes.POINTER(PfSolveRequest), ctypes.POINTER(u64)]),
    "PfSolveServerWait": (c_int, [ctypes.c_void_p, u64, ctypes.POINTER(ctypes.c_double)]),
    "PfSolveServerGetStats": (c_int, [ctypes.c_void_p, ctypes.POINTER(PfSolveServerStats)]),
    "PfSolveServerDestroy": (None, [ctypes.c_void_p]),
    "PfSolveBatchCreate": (c_int, [ctypes.POINTER(ctypes.c_void_p), c_int, ctypes.POINTER(PfSolveBatchDesc),
                                   ctypes.POINTER(PfSolveBatchEntry), c_int]),
    "PfSolveBatchAppend": (c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "PfSolveBatchCaptureGraph": (c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "PfSolveBatchAutotune": (c_int, [ctypes.c_void_p, ctypes.c_void_p, c_int]),
    "PfSolveBatchGetShape": (c_int, [ctypes.c_void_p] + [ctypes.POINTER(c_int)] * 4 + [ctypes.POINTER(ctypes.c_double)]),
    "PfSolveBatchGetSweepShape": (c_int, [ctypes.c_void_p] + [ctypes.POINTER(c_int)] * 3),
    "PfSolveBatchDestroy": (None, [ctypes.c_void_p]),
    "PfSolveBatchAppendNoAlloc": (c_int, [c_int, ctypes.POINTER(PfSolveBatchDesc), ctypes.POINTER(PfSolveBatchEntry),
                                          c_int, ctypes.c_void_p]),
}

_lib = None


def load():
    """Load the in-tree library; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C pfsolve_b200` "
                           "(or __graft_entry__.build()); there is no fallback implementation")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class PfSolveError(RuntimeError):
    def __init__(self, code, what=""):
        s = load().getPfSolveErrorString(code).decode()
        super().__init__(f"{what}: {s} ({code})")
        self.code = code


def check(code, what=""):
    if code != PFSOLVE_SUCCESS:
        raise PfSolveError(code, what)
