"""The C-ABI library loads, exports every entry point its header declares, and
the ctypes mirror has the C layout (CPU only; no kernel runs)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

from pfsolve_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        for m in re.finditer(r"PFSOLVE_API\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.append(m.group(1))
    return names


def test_library_builds_and_loads():
    assert os.path.exists(capi.LIB_PATH), "run make -C pfsolve_b200"
    lib = capi.load()
    # the reference returns the literal 00102 (pfSolve.h:101-103): octal, value 66
    assert lib.PfSolveGetVersion() == 0o102 == 66


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 16
    lib = ctypes.CDLL(capi.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
    assert set(names) == set(capi.SIGNATURES), "capi.SIGNATURES must cover exactly the header's functions"


PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "pfsolve_b200.h"
#define F(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  printf("cfg %zu\nlp %zu\napp %zu\nkjw %zu\nkdg %zu\nkbl %zu\nbent %zu\nbdesc %zu\n",
         sizeof(PfSolveConfiguration), sizeof(PfSolveLaunchParams), sizeof(PfSolveApplication),
         sizeof(PfSolve_MapKey_JonesWorland), sizeof(PfSolve_MapKey_dgbmv), sizeof(PfSolve_MapKey_block),
         sizeof(PfSolveBatchEntry), sizeof(PfSolveBatchDesc));
  printf("sdesc %zu\nsreq %zu\nsstat %zu\nlinfo %zu\n", sizeof(PfSolveServerDesc), sizeof(PfSolveRequest),
         sizeof(PfSolveServerStats), sizeof(PfSolveLaunchInfo));
  F(PfSolveRequest, nrhs) F(PfSolveRequest, scaleC) F(PfSolveRequest, stream) F(PfSolveRequest, inputReady)
  F(PfSolveLaunchInfo, precision) F(PfSolveLaunchInfo, gridCTAs) F(PfSolveServerDesc, hbmBudgetBytes)
  F(PfSolveServerStats, p50Ms) F(PfSolveServerStats, p99DeviceMs) F(PfSolveConfiguration, kernelPath)
  F(PfSolveConfiguration, jw_type) F(PfSolveConfiguration, jw_control_bitmask)
  F(PfSolveConfiguration, scaleC) F(PfSolveConfiguration, doublePrecision)
  F(PfSolveConfiguration, outputBufferStride) F(PfSolveConfiguration, numConsecutiveJWIterations)
  F(PfSolveConfiguration, rowsPerThread)
  F(PfSolveLaunchParams, scaleC) F(PfSolveLaunchParams, batchSize)
  return 0;
}
"""


def test_ctypes_layout_matches_c(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.strip().splitlines())
    assert int(out["cfg"]) == ctypes.sizeof(capi.PfSolveConfiguration)
    assert int(out["lp"]) == ctypes.sizeof(capi.PfSolveLaunchParams)
    assert int(out["app"]) == ctypes.sizeof(capi.PfSolveApplication)
    assert int(out["kjw"]) == ctypes.sizeof(capi.MapKeyJW)
    assert int(out["kdg"]) == ctypes.sizeof(capi.MapKeyDgbmv)
    assert int(out["kbl"]) == ctypes.sizeof(capi.MapKeyBlock)
    assert int(out["bent"]) == ctypes.sizeof(capi.PfSolveBatchEntry)
    assert int(out["bdesc"]) == ctypes.sizeof(capi.PfSolveBatchDesc)
    assert int(out["sdesc"]) == ctypes.sizeof(capi.PfSolveServerDesc)
    assert int(out["sreq"]) == ctypes.sizeof(capi.PfSolveRequest)
    assert int(out["sstat"]) == ctypes.sizeof(capi.PfSolveServerStats)
    assert int(out["linfo"]) == ctypes.sizeof(capi.PfSolveLaunchInfo)
    for key, val in out.items():
        if "." in key:
            T, f = key.split(".")
            cls = getattr(capi, T)
            assert getattr(cls, f).offset == int(val), key


def _init(**fields):
    lib = capi.load()
    cfg = capi.PfSolveConfiguration()
    dev = ctypes.c_int(0)
    cfg.device = ctypes.pointer(dev)
    cfg.FFTdim = 1
    for k, v in fields.items():
        if k == "size":
            for i, x in enumerate(v):
                cfg.size[i] = x
        else:
            setattr(cfg, k, v)
    app = capi.PfSolveApplication()
    return lib.initializePfSolve(ctypes.byref(app), cfg), app


def test_validation_errors_before_device_use():
    assert _init(FFTdim=0, size=(8, 1), jw_type=13)[0] == capi.PFSOLVE_ERROR_EMPTY_FFTdim
    assert _init(size=(0, 1), jw_type=13)[0] == capi.PFSOLVE_ERROR_EMPTY_size
    lib = capi.load()
    cfg = capi.PfSolveConfiguration()
    cfg.FFTdim = 1
    cfg.size[0] = 8
    app = capi.PfSolveApplication()
    assert lib.initializePfSolve(ctypes.byref(app), cfg) == capi.PFSOLVE_ERROR_INVALID_DEVICE
    assert lib.initializePfSolve(None, cfg) == capi.PFSOLVE_ERROR_INVALID_ARGUMENT
    # an uninitialised app is rejected, not dereferenced
    assert lib.PfSolveAppend(ctypes.byref(capi.PfSolveApplication()), 0, None) == 4


def header_result_codes():
    """(name, value) of every PfSolveResult code the header declares."""
    text = open(os.path.join(ROOT, "include", "pfsolve_b200.h")).read()
    body = text[text.index("typedef enum PfSolveResult {"):text.index("} PfSolveResult;")]
    return [(m.group(1), int(m.group(2))) for m in re.finditer(r"(PFSOLVE_\w+)\s*=\s*(\d+)", body)]


def test_error_strings():
    """Every declared code has its own name (as the reference's
    getPfSolveErrorString, pfSolve_Structs.h:545 onward); the 92 reference
    codes keep their numbers."""
    lib = capi.load()
    codes = header_result_codes()
    assert len(codes) == 96 and len({v for _, v in codes}) == 96
    for name, value in codes:
        assert lib.getPfSolveErrorString(value) == name.encode(), (name, value)
    assert lib.getPfSolveErrorString(0) == b"PFSOLVE_SUCCESS"
    assert lib.getPfSolveErrorString(4029) == b"PFSOLVE_ERROR_FAILED_TO_COPY"
    assert lib.getPfSolveErrorString(4055) == b"PFSOLVE_ERROR_FAILED_TO_SUBMIT_BARRIER"
    assert lib.getPfSolveErrorString(5001) == b"PFSOLVE_ERROR_UNSUPPORTED_COMBINATION"
    assert lib.getPfSolveErrorString(12345) == b"PFSOLVE_ERROR_UNKNOWN"


def test_app_library_keys_order_and_lookup():
    lib = capi.load()
    L = lib.PfSolveAppLibraryCreate()
    try:
        k = capi.MapKeyJW()
        k.size[0], k.size[1], k.upperBanded, k.outputBufferStride, k.type = 256, 512, 2, 256, 13
        out = ctypes.POINTER(capi.PfSolveApplication)()
        assert lib.checkLibrary_JonesWorland(L, k, ctypes.byref(out)) == 0
        assert not out  # miss
        app = capi.PfSolveApplication()
        app.configuration.M_size = 256
        assert lib.addToLibrary_JonesWorland(L, k, ctypes.byref(app)) == 0
        assert lib.checkLibrary_JonesWorland(L, k, ctypes.byref(out)) == 0
        assert out and out.contents.configuration.M_size == 256
        k2 = capi.MapKeyJW()
        k2.size[0], k2.size[1], k2.upperBanded, k2.outputBufferStride, k2.type = 256, 512, 2, 256, 12
        assert lib.checkLibrary_JonesWorland(L, k2, ctypes.byref(out)) == 0
        assert not out
    finally:
        lib.PfSolveAppLibraryDestroy(L)


def test_server_argument_checks_before_device_use():
    lib = capi.load()
    h = ctypes.c_void_p()
    assert lib.PfSolveServerCreate(ctypes.byref(h), None) == capi.PFSOLVE_ERROR_INVALID_ARGUMENT
    for bad in (dict(streams=0), dict(streams=17), dict(maxBatchRequests=0), dict(refineSweeps=4),
                dict(hbmBudgetBytes=0)):
        kw = dict(device=0, hbmBudgetBytes=1 << 20, streams=2, maxBatchRequests=4, refineSweeps=2)
        kw.update(bad)
        d = capi.PfSolveServerDesc(**kw)
        assert lib.PfSolveServerCreate(ctypes.byref(h), ctypes.byref(d)) == capi.PFSOLVE_ERROR_INVALID_ARGUMENT, bad
    r = capi.PfSolveRequest()
    t = ctypes.c_uint64()
    assert lib.PfSolveServerSubmit(None, ctypes.byref(r), ctypes.byref(t)) == capi.PFSOLVE_ERROR_INVALID_ARGUMENT
    lib.PfSolveServerDestroy(None)


def test_integration_example_compiles_and_links(tmp_path):
    """The C caller quoted in the integration guide (tests/abi_example.c)
    builds against the header and links the library."""
    code = open(os.path.join(ROOT, "tests", "abi_example.c")).read()
    src = tmp_path / "jw_step.c"
    src.write_text(code + "\nint main(void) { return 0; }\n")
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    libdir = os.path.dirname(capi.LIB_PATH)
    subprocess.run([cc, "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-L", libdir, "-lpfsolve_b200", "-Wl,-rpath," + libdir, "-o", str(tmp_path / "jw_step")],
                   check=True)
