"""Serving engine client: ``Server`` wraps the C ABI's PfSolveServer*
functions (request queue, HBM-footprint admission, continuous batching on
several streams; see include/pfsolve_b200.h), and ``run_load`` drives it with
timed arrivals.  Device buffers are torch CUDA tensors (plumbing only: every
kernel launch goes through the library)."""
from __future__ import annotations

import ctypes
import time

from . import capi
from .capi import check


class Server:
    def __init__(self, device=0, hbm_budget_bytes=8 << 30, streams=4, max_batch_requests=32, refine_sweeps=2):
        self._lib = capi.load()
        d = capi.PfSolveServerDesc(device=device, hbmBudgetBytes=int(hbm_budget_bytes), streams=streams,
                                   maxBatchRequests=max_batch_requests, refineSweeps=refine_sweeps)
        self.h = ctypes.c_void_p()
        check(self._lib.PfSolveServerCreate(ctypes.byref(self.h), ctypes.byref(d)), "PfSolveServerCreate")
        self._keep = []

    def add_operator(self, M, bands, upperBanded=2, jw_type=13) -> int:
        """Register device bands (a CUDA tensor of 3*M doubles, reference layout)."""
        op = ctypes.c_int()
        self._keep.append(bands)
        check(self._lib.PfSolveServerAddOperator(self.h, int(M), ctypes.c_void_p(bands.data_ptr()), upperBanded,
                                                 jw_type, ctypes.byref(op)), "PfSolveServerAddOperator")
        return op.value

    def submit(self, op, precision, nrhs, inp, out, stride=0, scaleC=1.0, stream=None, input_ready=False) -> int:
        """Queue one request.  Unless ``input_ready``, the request's kernel
        waits for the work enqueued so far on ``stream`` (a torch stream or a
        raw handle; None: the legacy default stream, torch's default)."""
        sh = None if stream is None else (stream if isinstance(stream, int) else int(stream.cuda_stream))
        r = capi.PfSolveRequest(op=op, precision=precision, nrhs=int(nrhs), input=inp.data_ptr(),
                                output=out.data_ptr(), stride=int(stride), scaleC=float(scaleC), stream=sh,
                                inputReady=1 if input_ready else 0)
        t = ctypes.c_uint64()
        check(self._lib.PfSolveServerSubmit(self.h, ctypes.byref(r), ctypes.byref(t)), "PfSolveServerSubmit")
        return t.value

    def wait(self, ticket) -> float:
        ms = ctypes.c_double()
        check(self._lib.PfSolveServerWait(self.h, ctypes.c_uint64(ticket), ctypes.byref(ms)), "PfSolveServerWait")
        return ms.value

    def stats(self) -> dict:
        s = capi.PfSolveServerStats()
        check(self._lib.PfSolveServerGetStats(self.h, ctypes.byref(s)), "PfSolveServerGetStats")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if self.h:
            self._lib.PfSolveServerDestroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_load(server, requests, arrivals, input_ready=True):
    """Submit ``requests`` (tuples (op, precision, nrhs, input, output)) at the
    given arrival times (seconds from start, busy-waited), then wait for all.
    The inputs are device-resident and complete before the load starts
    (``input_ready``: no ordering event per request).
    Returns (latencies in ms per request, wall seconds, seconds the submitter
    ran behind the schedule at most)."""
    tickets = []
    lag = 0.0
    t0 = time.perf_counter()
    for (op, prec, nrhs, inp, out), ta in zip(requests, arrivals):
        while True:
            now = time.perf_counter() - t0
            if now >= ta:
                break
        lag = max(lag, now - ta)
        tickets.append(server.submit(op, prec, nrhs, inp, out, input_ready=input_ready))
    lat = [server.wait(t) for t in tickets]
    wall = time.perf_counter() - t0
    return lat, wall, lag
