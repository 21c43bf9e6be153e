"""Host-side mirror of PfSolve's plan/application interface for the JW path.

``App`` wraps one ``PfSolveApplication`` created through the C ABI
(``initializePfSolve`` -> ``PfSolveAppend`` -> ``deletePfSolve``), with field
names taken verbatim from ``PfSolveConfiguration`` / ``PfSolveLaunchParams``
(PfSolve/pfSolve_Structs/pfSolve_Structs.h:119-449).  Device buffers are torch
CUDA tensors (plumbing only: every kernel launch goes through the library).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

from . import capi
from .capi import check


def _ptr(t) -> int:
    if t is None:
        return 0
    if isinstance(t, int):
        return t
    return int(t.data_ptr())


class App:
    """One initialised PfSolve application (JW, dgbmv or block).

    Construct with the configuration fields as keyword arguments, e.g.
    ``App(M_size=256, size=(256, 512), jw_type=13, upperBanded=2,
    doublePrecision=1, buffer=bands, outputBuffer=rhs)``.
    """

    def __init__(self, *, device: int = 0, stream=None, buffer=None, outputBuffer=None, **fields):
        self._lib = capi.load()
        self._keep = []
        cfg = capi.PfSolveConfiguration()
        cfg.FFTdim = 1
        self._dev = ctypes.c_int(device)
        cfg.device = ctypes.pointer(self._dev)
        if stream is not None:
            self._stream = (ctypes.c_void_p * 1)(int(stream))
            cfg.stream = ctypes.cast(self._stream, ctypes.POINTER(ctypes.c_void_p))
            cfg.num_streams = 1
        size = fields.pop("size", None)
        if size is not None:
            for k, v in enumerate(size):
                cfg.size[k] = int(v)
        for key in ("inputBufferStride", "outputBufferStride", "inputZeropad", "outputZeropad", "Msplit"):
            if key in fields:
                v = fields.pop(key)
                arr = getattr(cfg, key)
                if isinstance(v, (list, tuple)):
                    for k, x in enumerate(v):
                        arr[k] = int(x)
                else:
                    arr[0] = int(v)
        for k, v in fields.items():
            if not hasattr(cfg, k):
                raise AttributeError(f"PfSolveConfiguration has no field {k!r}")
            setattr(cfg, k, v)
        if buffer is not None:
            cfg.buffer = self._vpp(buffer)
        if outputBuffer is not None:
            cfg.outputBuffer = self._vpp(outputBuffer)
        self.app = capi.PfSolveApplication()
        check(self._lib.initializePfSolve(ctypes.byref(self.app), cfg), "initializePfSolve")
        self.alive = True

    def _vpp(self, t):
        """void** for one buffer, or for a list of buffers (one per step of a
        K-step application with useMultipleInputBuffers)."""
        ts = list(t) if isinstance(t, (list, tuple)) else [t]
        arr = (ctypes.c_void_p * len(ts))(*[_ptr(x) for x in ts])
        self._keep.append(arr)
        return ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p))

    def launch_params(self, *, buffer=None, outputBuffer=None, scaleC=None, inputZeropad=None,
                      outputZeropad=None, **vals) -> capi.PfSolveLaunchParams:
        lp = capi.PfSolveLaunchParams()
        if buffer is not None:
            lp.buffer = self._vpp(buffer)
        if outputBuffer is not None:
            lp.outputBuffer = self._vpp(outputBuffer)
        if scaleC is not None:
            lp.scaleC = float(scaleC)
        if inputZeropad is not None:
            lp.inputZeropad[0], lp.inputZeropad[1] = int(inputZeropad[0]), int(inputZeropad[1])
        if outputZeropad is not None:
            lp.outputZeropad[0], lp.outputZeropad[1] = int(outputZeropad[0]), int(outputZeropad[1])
        for k, v in vals.items():
            setattr(lp, k, int(v))
        return lp

    def append(self, lp: Optional[capi.PfSolveLaunchParams] = None, **kw):
        if lp is None:
            lp = self.launch_params(**kw)
        check(self._lib.PfSolveAppend(ctypes.byref(self.app), 0, ctypes.byref(lp)), "PfSolveAppend")
        return lp

    def sync(self):
        check(self._lib.PfSolveSync(ctypes.byref(self.app)), "PfSolveSync")

    def shape(self) -> dict:
        """Kernel shape of this plan (``PfSolveGetShape``)."""
        v = [ctypes.c_int() for _ in range(4)]
        check(self._lib.PfSolveGetShape(ctypes.byref(self.app), *[ctypes.byref(x) for x in v]), "PfSolveGetShape")
        return dict(streaming=v[0].value, rowsPerThread=v[1].value, warpsPerSystem=v[2].value,
                    groupsPerCTA=v[3].value)

    def close(self):
        if getattr(self, "alive", False):
            self._lib.deletePfSolve(ctypes.byref(self.app))
            self.alive = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def streaming_launch_count() -> int:
    """Launches that ran on the streaming kernel (``PfSolveStreamingLaunchCount``)."""
    return int(capi.load().PfSolveStreamingLaunchCount())


def last_launch() -> dict:
    """The kernel instance of this thread's most recent launch (``PfSolveGetLastLaunch``)."""
    info = capi.PfSolveLaunchInfo()
    check(capi.load().PfSolveGetLastLaunch(ctypes.byref(info)), "PfSolveGetLastLaunch")
    return {k: getattr(info, k) for k, _ in info._fields_}


def device_status() -> int:
    """``PfSolveGetDeviceStatus``: 0, or PFSOLVE_ERROR_DEVICE_FAULT after a bounded wait ran out."""
    return int(capi.load().PfSolveGetDeviceStatus())


def append_chain(apps: Sequence[App], lps: Sequence[capi.PfSolveLaunchParams], allow_unfused: bool = False):
    """Run apps as one fused kernel (``PfSolveAppendChain``)."""
    lib = capi.load()
    n = len(apps)
    app_ptrs = (ctypes.POINTER(capi.PfSolveApplication) * n)(*[ctypes.pointer(a.app) for a in apps])
    lp_ptrs = (ctypes.POINTER(capi.PfSolveLaunchParams) * n)(*[ctypes.pointer(l) for l in lps])
    check(lib.PfSolveAppendChain(app_ptrs, lp_ptrs, n, 1 if allow_unfused else 0), "PfSolveAppendChain")


def launch_count() -> int:
    return int(capi.load().PfSolveLaunchCount())


class Batch:
    """One uneven batch plan (``PfSolveBatchCreate``): a JW step over many
    groups of systems of different sizes in one persistent launch.

    ``entries`` is a list of dicts with the ``PfSolveBatchEntry`` fields; device
    buffers may be torch tensors or raw pointers.
    """

    def __init__(self, entries, *, device: int = 0, **desc_fields):
        self._lib = capi.load()
        self._keep = entries
        d = capi.PfSolveBatchDesc()
        for k, v in desc_fields.items():
            setattr(d, k, int(v))
        arr = (capi.PfSolveBatchEntry * max(1, len(entries)))()
        for i, e in enumerate(entries):
            a = arr[i]
            a.M, a.nsys = int(e["M"]), int(e["nsys"])
            a.bands = _ptr(e["bands"])
            a.dgbmvBands = _ptr(e.get("dgbmvBands"))
            a.input = _ptr(e["input"])
            a.output = _ptr(e["output"])
            a.inputStride = int(e["inputStride"])
            a.outputStride = int(e["outputStride"])
            a.lshift = int(e.get("lshift", 0))
            a.scaleS = float(e.get("scaleS", 0.0))
            a.scaleC = float(e.get("scaleC", 1.0))
        self.handle = ctypes.c_void_p()
        check(self._lib.PfSolveBatchCreate(ctypes.byref(self.handle), int(device), ctypes.byref(d), arr,
                                           len(entries)), "PfSolveBatchCreate")

    def append(self, stream=None):
        check(self._lib.PfSolveBatchAppend(self.handle, _stream(stream)), "PfSolveBatchAppend")

    def capture(self, stream):
        check(self._lib.PfSolveBatchCaptureGraph(self.handle, _stream(stream)), "PfSolveBatchCaptureGraph")

    def autotune(self, stream=None, iterations=3):
        check(self._lib.PfSolveBatchAutotune(self.handle, _stream(stream), int(iterations)), "PfSolveBatchAutotune")

    def shape(self):
        r, w, spi, items = (ctypes.c_int() for _ in range(4))
        ms = ctypes.c_double()
        check(self._lib.PfSolveBatchGetShape(self.handle, ctypes.byref(r), ctypes.byref(w), ctypes.byref(spi),
                                             ctypes.byref(items), ctypes.byref(ms)), "PfSolveBatchGetShape")
        ch, nb, nw = (ctypes.c_int() for _ in range(3))
        check(self._lib.PfSolveBatchGetSweepShape(self.handle, ctypes.byref(ch), ctypes.byref(nb), ctypes.byref(nw)),
              "PfSolveBatchGetSweepShape")
        return dict(rowsPerThread=r.value, warpsPerSystem=w.value, systemsPerItem=spi.value, items=items.value,
                    tunedMs=ms.value, sweepRows=ch.value, sweepBuffers=nb.value, sweepWarps=nw.value)

    def close(self):
        if getattr(self, "handle", None):
            self._lib.PfSolveBatchDestroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stream(s):
    if s is None:
        return None
    if isinstance(s, int):
        return s
    return int(s.cuda_stream)
