"""Generate golden vectors from the reference's own GPU kernels.

Runs ``oracle/_ref/pfsolve_ref`` (the unmodified PfSolve library, compiled from
its sources by ``make -C oracle ref``) on seeded inputs and stores inputs plus
the reference's outputs as ``<out>/<case>.npz``.  Needs a CUDA GPU; run it as
``python tests/golden/make_golden.py --out <dir>`` and copy the fixtures into
``tests/golden/``.  ``--time`` also times the reference's JW
kernel on the full-size configurations and writes ``ref_timing.json``.
Subsets (``--only``): K-step fixtures, ALT mode, long systems (into
``<out>/long/``), double-double (into ``<out>/dd/``, copied to
``tests/golden/dd/``), ``dd-crash``, which re-runs the double-double cases
the reference's code generation crashes on and stores no fixtures, and
``f32``: the FP32-storage precisions (into ``<out>/f32/``, copied to
``tests/golden/f32/``).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import traceback
from dataclasses import asdict

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from pfsolve_b200 import workloads as WL  # noqa: E402

RT = O


def jw_bands(rng, M, ub):
    """Natural-order bands; out-of-range couplings zero (reference convention)."""
    if ub == 2:
        return WL.tri_bands(*WL.tridiagonal(rng, M))
    # each band is the solve band in some jw_type: |entries| < 1/2 keeps the
    # unit-diagonal recurrences stable
    bands = [rng.uniform(-.5, .5, M) for _ in range(3)]
    for k in range(3):
        bands[k][0] = 0.0
        bands[k][-1] = 0.0
    return np.concatenate(bands)


def jw_cases():
    """(name, Case, bands, rhs, precision) for the JW application."""
    out = []
    for ub, jwt in [(2, 13), (1, 10), (1, 11), (1, 12), (1, 13), (0, 10), (0, 11), (0, 12), (0, 13)]:
        for M in ([7, 33, 100, 256, 513, 1024] if (ub, jwt) in [(2, 13), (1, 10), (0, 10)] else [33, 300]):
            rng = np.random.default_rng(7000 + 100 * ub + jwt + M)
            bands = WL.permute_bands(jw_bands(rng, M, ub), M)
            case = O.Case(M=M, batch=3, upperBanded=ub, jw_type=jwt)
            rhs = rng.uniform(-1, 1, case.rhs_len())
            out.append((f"jw_ub{ub}_t{jwt}_M{M}", case, bands, rhs, "f64"))
    # runtime values: offsets, strides, zeropads, scaleC (sample_0 form: stride N+128)
    M = 200
    bm = (RT.RUNTIME_OFFSETSOLUTION | RT.RUNTIME_INPUTZEROPAD | RT.RUNTIME_OUTPUTZEROPAD | RT.RUNTIME_SCALEC |
          RT.RUNTIME_OUTPUTBUFFERSTRIDE)
    for ub, jwt in [(2, 13), (1, 10), (0, 13)]:
        rng = np.random.default_rng(8000 + ub)
        nat = jw_bands(rng, M, ub)
        case = O.Case(M=M, batch=4, upperBanded=ub, jw_type=jwt, bitmask=bm, run_offsetSolution=6,
                      run_inputZeropad=(3, 190), run_outputZeropad=(5, 180), run_scaleC=0.625,
                      run_outputBufferStride=M + 128)
        rhs = rng.uniform(-1, 1, case.rhs_len() + 8)
        out.append((f"jw_runtime_ub{ub}_t{jwt}", case, WL.permute_bands(nat, M), rhs, "f64"))
    # runtime offsetM / offsetV (band order swap)
    for ub in (0, 1):
        rng = np.random.default_rng(8100 + ub)
        md, mo, sv = rng.uniform(-.5, .5, M), rng.uniform(-.5, .5, M), rng.uniform(-.5, .5, M)
        mo[0] = mo[-1] = sv[0] = sv[-1] = 0.0
        perm = WL.reference_band_order(M)
        big = np.zeros(5 * M)
        oM, oV = M + 3, 4 * M - 7
        first, second = (mo, md) if ub == 1 else (md, mo)
        big[oM + perm] = first
        big[oM + M + perm] = second
        big[oV + perm] = sv
        case = O.Case(M=M, batch=3, upperBanded=ub, jw_type=10, bitmask=RT.RUNTIME_OFFSETM | RT.RUNTIME_OFFSETV,
                      run_offsetM=oM, run_offsetV=oV)
        rhs = rng.uniform(-1, 1, case.rhs_len())
        out.append((f"jw_offsetMV_ub{ub}", case, big, rhs, "f64"))
    # plan-time values (compile-time windows, scaleC, offsetSolution)
    rng = np.random.default_rng(8200)
    case = O.Case(M=M, batch=3, upperBanded=2, jw_type=13, cfg_offsetSolution=4, cfg_outputBufferStride=M + 16,
                  cfg_inputZeropad=(4, 0), cfg_outputZeropad=(0, 150), cfg_scaleC=2.0)
    out.append(("jw_plantime", case, WL.permute_bands(WL.tri_bands(*WL.tridiagonal(rng, M)), M),
                rng.uniform(-1, 1, case.rhs_len()), "f64"))
    # double-double storage (test-0 form, quad emulation)
    for M in (64, 256):
        rng = np.random.default_rng(8300 + M)
        bands = WL.permute_bands(WL.tri_bands(*WL.tridiagonal(rng, M)), M)
        case = O.Case(M=M, batch=2, upperBanded=2, jw_type=13)
        rhs = rng.uniform(-1, 1, case.rhs_len())
        bdd = np.stack([bands, np.zeros_like(bands)], -1).ravel()
        rdd = np.stack([rhs, np.zeros_like(rhs)], -1).ravel()
        out.append((f"jw_dd_M{M}", case, bdd, rdd, "dd"))
    # FP32 (the reference's default precision)
    rng = np.random.default_rng(8400)
    M = 256
    case = O.Case(M=M, batch=3, upperBanded=2, jw_type=13)
    out.append(("jw_f32_M256", case, WL.permute_bands(WL.tri_bands(*WL.tridiagonal(rng, M)), M),
                rng.uniform(-1, 1, case.rhs_len()), "f32"))
    return out


def f32_cases():
    """(name, Case, buffer, rhs, precision) on FP32 storage: the reference's
    default precision ("f32": FP32 arithmetic) and doublePrecisionFloatMemory
    ("f32mem": FP64 arithmetic), for every JW mode, launch-time values, the
    dgbmv application and the block layouts.  Inputs are FP32 values."""
    out = []
    f = np.float32
    for prec in ("f32", "f32mem"):
        for ub, jwt in [(2, 13), (1, 10), (1, 11), (1, 12), (1, 13), (0, 10), (0, 11), (0, 12), (0, 13)]:
            for M in ([33, 256, 1000] if (ub, jwt) in [(2, 13), (1, 10), (0, 10)] else [100]):
                rng = np.random.default_rng(15000 + 100 * ub + jwt + M)
                bands = WL.permute_bands(jw_bands(rng, M, ub), M).astype(f)
                case = O.Case(M=M, batch=3, upperBanded=ub, jw_type=jwt)
                out.append((f"{prec}_jw_ub{ub}_t{jwt}_M{M}", case, bands,
                            rng.uniform(-1, 1, case.rhs_len()).astype(f), prec))
        M = 200
        bm = (RT.RUNTIME_OFFSETSOLUTION | RT.RUNTIME_INPUTZEROPAD | RT.RUNTIME_OUTPUTZEROPAD | RT.RUNTIME_SCALEC |
              RT.RUNTIME_OUTPUTBUFFERSTRIDE)
        for ub, jwt in [(2, 13), (1, 10), (0, 13)]:
            rng = np.random.default_rng(15500 + ub)
            case = O.Case(M=M, batch=4, upperBanded=ub, jw_type=jwt, bitmask=bm, run_offsetSolution=5,
                          run_inputZeropad=(3, 190), run_outputZeropad=(5, 180), run_scaleC=0.625,
                          run_outputBufferStride=M + 131)
            out.append((f"{prec}_jw_runtime_ub{ub}_t{jwt}", case, WL.permute_bands(jw_bands(rng, M, ub), M).astype(f),
                        rng.uniform(-1, 1, case.rhs_len() + 8).astype(f), prec))
        for M, KL, KU in [(128, 2, 2), (64, 3, 1)]:
            rng = np.random.default_rng(15700 + M + KL)
            case = O.Case(M=M, batch=2, LDA=KL + KU + 1, KU=KU, KL=KL, jw_type=0)
            out.append((f"{prec}_dgbmv_M{M}_kl{KL}_ku{KU}", case, WL.band_major(rng, M, KL, KU).astype(f),
                        rng.uniform(-1, 1, case.rhs_len()).astype(f), prec))
        N, Y = 40, 3
        for block in (1, 4, 7, 27, 301):
            rng = np.random.default_rng(15900 + block)
            bt = block % 10
            nin = (2 if bt in (2, 3, 4, 7) else 1) * N * Y
            nout = (2 if bt in (4, 5, 6, 7) else 1) * N * Y
            case = O.Case(M=N, batch=Y, block=block, lshift=2, jw_type=0, bitmask=RT.RUNTIME_SCALEC, run_scaleC=0.5)
            out.append((f"{prec}_block_{block}", case, rng.standard_normal(nin).astype(f),
                        rng.standard_normal(nout).astype(f), prec))
    return out


def dgbmv_cases():
    out = []
    for M, KL, KU in [(33, 1, 1), (128, 2, 2), (100, 0, 2), (64, 3, 1)]:
        rng = np.random.default_rng(9000 + M + KL)
        A = WL.band_major(rng, M, KL, KU)
        case = O.Case(M=M, batch=2, LDA=KL + KU + 1, KU=KU, KL=KL, jw_type=0)
        out.append((f"dgbmv_M{M}_kl{KL}_ku{KU}", case, A, rng.uniform(-1, 1, case.rhs_len()), "f64"))
    return out


def alt_dgbmv_cases():
    """dgbmv with ALT_dgbmv: alternate bands dropped (stored with the dgbmv
    fixtures; the rule is restated literally, including its one-sided forms)."""
    out = []
    for M, KL, KU in [(64, 0, 2), (100, 0, 4), (64, 2, 0), (65, 3, 0), (80, 2, 2), (50, 1, 3)]:
        rng = np.random.default_rng(9200 + M + 10 * KL + KU)
        A = WL.band_major(rng, M, KL, KU)
        case = O.Case(M=M, batch=2, LDA=KL + KU + 1, KU=KU, KL=KL, jw_type=0, ALT_dgbmv=1)
        out.append((f"dgbmv_alt_M{M}_kl{KL}_ku{KU}", case, A, rng.uniform(-1, 1, case.rhs_len()), "f64"))
    return out


def block_cases():
    out = []
    N, Y = 40, 3
    for block in (1, 2, 3, 4, 5, 6, 7, 21, 27, 101, 201, 301, 401):
        rng = np.random.default_rng(9500 + block)
        bt = block % 10
        nin = (2 if bt in (2, 3, 4, 7) else 1) * N * Y
        nout = (2 if bt in (4, 5, 6, 7) else 1) * N * Y
        case = O.Case(M=N, batch=Y, block=block, lshift=2, jw_type=0, bitmask=RT.RUNTIME_SCALEC, run_scaleC=0.5)
        out.append((f"block_{block}", case, rng.standard_normal(nin), rng.standard_normal(nout), "f64"))
    return out


def steps_cases():
    """(name, Case, K, band buffers, rhs) for K consecutive steps
    (numConsecutiveJWIterations), stored under tests/golden/steps/."""
    out = []
    combos = [(1, 10, (2, 3, 5)), (0, 10, (2, 3, 5)), (1, 11, (3,)), (0, 11, (3,)), (1, 12, (3,)), (0, 12, (3,)),
              (2, 13, (2,))]
    for ub, jwt, Ks in combos:
        for K in Ks:
            for M in (33, 250, 1000):
                rng = np.random.default_rng(12000 + 1000 * ub + 10 * jwt + K + M)
                bands = WL.steps_bands(rng, M, ub, K)
                case = O.Case(M=M, batch=3, upperBanded=ub, jw_type=jwt, cfg_outputBufferStride=M + K + 3)
                rhs = rng.uniform(-1, 1, case.rhs_len() + K)
                out.append((f"steps_ub{ub}_t{jwt}_K{K}_M{M}", case, K, bands, rhs))
    # one buffer read by every step at its own offsets
    for ub in (0, 1):
        M, K = 120, 3
        rng = np.random.default_rng(12500 + ub)
        buf = WL.steps_bands(rng, M, ub, K, per_step=False)
        case = O.Case(M=M, batch=2, upperBanded=ub, jw_type=10, cfg_outputBufferStride=M + 8)
        out.append((f"steps_onebuf_ub{ub}", case, K, [buf], rng.uniform(-1, 1, case.rhs_len() + K)))
    # launch-time windows, scaleC, stride and solution offset
    bm = (RT.RUNTIME_OFFSETSOLUTION | RT.RUNTIME_INPUTZEROPAD | RT.RUNTIME_OUTPUTZEROPAD | RT.RUNTIME_SCALEC |
          RT.RUNTIME_OUTPUTBUFFERSTRIDE)
    for ub in (0, 1, 2):
        M, K = 200, (2 if ub == 2 else 4)
        rng = np.random.default_rng(12600 + ub)
        case = O.Case(M=M, batch=3, upperBanded=ub, jw_type=13 if ub == 2 else 10, bitmask=bm,
                      run_offsetSolution=4, run_inputZeropad=(2, 190), run_outputZeropad=(3, 199),
                      run_scaleC=0.75, run_outputBufferStride=M + K + 9)
        out.append((f"steps_runtime_ub{ub}", case, K, WL.steps_bands(rng, M, ub, K),
                    rng.uniform(-1, 1, case.rhs_len() + K + 8)))
    return out


def steps_offset_cases():
    """Launch-time offsetM / offsetV with K > 1 (the reference's generator
    was seen to fail on the host for these; kept apart so the others run)."""
    out = []
    for ub in (0, 1):
        M, K = 200, 3
        rng = np.random.default_rng(12700 + ub)
        oM, oV = 5, 3 * (M + K) + 2
        bufs = []
        for s_ in range(K):
            Ms = WL.step_rows(M, ub, s_)
            b = rng.uniform(-0.5, 0.5, oV + M + K + 4)
            b[oV] = 0.0
            b[oM + Ms] = b[oM] = 0.0
            bufs.append(b)
        case = O.Case(M=M, batch=3, upperBanded=ub, jw_type=10, bitmask=RT.RUNTIME_OFFSETM | RT.RUNTIME_OFFSETV,
                      run_offsetM=oM, run_offsetV=oV, cfg_outputBufferStride=M + K + 3)
        out.append((f"steps_offsetMV_ub{ub}", case, K, bufs, rng.uniform(-1, 1, case.rhs_len() + K)))
    return out


def alt_cases():
    """(name, Case, bands, rhs, precision) for the ALT stride-2 mode
    (jw_type / 100 % 10 == 1), stored under tests/golden/alt/."""
    out = []
    for ub, jwt in [(2, 113), (1, 110), (1, 111), (1, 112), (1, 113), (0, 110), (0, 111), (0, 112), (0, 113)]:
        for M in ([20, 33, 100, 256, 511, 512, 1000, 2048] if jwt == 113 or jwt == 110 else [33, 300]):
            rng = np.random.default_rng(13000 + 1000 * ub + jwt + M)
            bands = WL.alt_bands(rng, M, ub)
            case = O.Case(M=M, batch=3, upperBanded=ub, jw_type=jwt)
            rhs = rng.uniform(-1, 1, case.rhs_len())
            out.append((f"alt_ub{ub}_t{jwt}_M{M}", case, bands, rhs, "f64"))
    # launch-time windows, scaleC, stride and solution offset
    M = 200
    bm = (RT.RUNTIME_OFFSETSOLUTION | RT.RUNTIME_INPUTZEROPAD | RT.RUNTIME_OUTPUTZEROPAD | RT.RUNTIME_SCALEC |
          RT.RUNTIME_OUTPUTBUFFERSTRIDE)
    for ub, jwt in [(2, 113), (1, 110), (0, 110)]:
        rng = np.random.default_rng(13500 + ub)
        case = O.Case(M=M, batch=4, upperBanded=ub, jw_type=jwt, bitmask=bm, run_offsetSolution=6,
                      run_inputZeropad=(3, 190), run_outputZeropad=(5, 180), run_scaleC=0.625,
                      run_outputBufferStride=M + 16)
        out.append((f"alt_runtime_ub{ub}_t{jwt}", case, WL.alt_bands(rng, M, ub),
                    rng.uniform(-1, 1, case.rhs_len() + 8), "f64"))
    return out


def long_cases():
    """(name, Case, bands, rhs, precision) for long systems, N > 4352: the
    reference splits them over several kernel launches (multi-upload,
    pfSolve_InitializeApp.h:1540-1583, reduced systems in its temporary buffer);
    stored under tests/golden/long/."""
    out = []
    for ub, jwt in [(2, 13), (1, 10), (0, 10), (1, 12), (0, 13)]:
        for M in ([4352, 4360, 5000, 8192, 16384] if (ub, jwt) in [(2, 13), (1, 10)] else [4400, 8192]):
            rng = np.random.default_rng(17000 + 100 * ub + jwt + M)
            bands = WL.permute_bands(jw_bands(rng, M, ub), M)
            case = O.Case(M=M, batch=2, upperBanded=ub, jw_type=jwt)
            rhs = rng.uniform(-1, 1, case.rhs_len())
            out.append((f"long_ub{ub}_t{jwt}_M{M}", case, bands, rhs, "f64"))
    # beyond one cluster of 8 x 2048 rows: up to 64 slices of 1024 rows; and
    # lengths that are not a multiple of 16 rows (an even one, whose rows are
    # 16-byte aligned at the packed stride, and an odd one)
    for M in (20000, 32768, 65536, 20002, 12345):
        rng = np.random.default_rng(17500 + M)
        bands = WL.permute_bands(jw_bands(rng, M, 2), M)
        case = O.Case(M=M, batch=2, upperBanded=2, jw_type=13)
        out.append((f"long_ub2_t13_M{M}", case, bands, rng.uniform(-1, 1, case.rhs_len()), "f64"))
    return out


REF_BIN_FP128 = os.path.join(ROOT, "oracle", "_ref", "pfsolve_ref_fp128")


# The reference's double-double code generation stops with SIGSEGV inside
# initializePfSolve whenever it moves a double-double constant into a
# register: the constant is declared with the double-double type but only its
# plain value is set (pfSolve_ReadWrite.h:1567-1568, moved at :1682 and
# :1692; the same in pfSolve_TridiagonalSolve.h, e.g. :1048), so
# PfCopyContainer (pfSolve_MathUtils.h:51-55) follows its unallocated
# {hi, lo} parts.  The sequential-Thomas generation, taken only for M <= 32
# with one step (pfSolve_Plan_JonesWorland.h:306), avoids those moves for the
# bidiagonal kinds; those cases are the fixtures.  DD_CRASHING lists the
# kinds and sizes seen to crash, kept to re-run the evidence (--only dd-crash).
DD_PINNED = [(1, 10, 16), (1, 10, 32), (0, 13, 32)]
DD_CRASHING = [(2, 13, 16), (2, 13, 32), (2, 13, 64), (2, 13, 256), (2, 13, 1000), (1, 10, 100), (1, 10, 512),
               (0, 10, 32), (0, 10, 100), (0, 10, 512), (0, 13, 300)]


def dd_cases(which=DD_PINNED):
    """(name, Case, bands, rhs, precision) in double-double storage ({hi, lo}
    pairs, non-zero lo parts), stored under tests/golden/dd/."""
    out = []
    for ub, jwt, M in which:
        rng = np.random.default_rng(18000 + 100 * ub + jwt + M)
        bands = WL.permute_bands(jw_bands(rng, M, ub), M)
        case = O.Case(M=M, batch=2, upperBanded=ub, jw_type=jwt)
        rhs = rng.uniform(-1, 1, case.rhs_len())
        bdd = O.to_dd(bands)
        bdd[1::2] = bands * rng.uniform(-1, 1, bands.shape) * 2.0 ** -60
        rdd = O.to_dd(rhs)
        rdd[1::2] = rhs * rng.uniform(-1, 1, rhs.shape) * 2.0 ** -60
        out.append((f"dd_ub{ub}_t{jwt}_M{M}", case, bdd, rdd, "dd"))
    return out


def run_dd_case(tmp, name, case, buf, rhs):
    """The reference's double-double JW app (default build first, then the
    PfSolve_use_FP128 build).  Its code-generation buffers are raised above
    the defaults (maxTempLength, maxCodeLength); that does not change the
    crash described above.  A crash report carries the harness phase and the
    return addresses, for addr2line on the same binary."""
    import subprocess
    d = os.path.join(tmp, name)
    O.write_reference_case(d, case, buf, rhs, precision="dd")
    with open(os.path.join(d, "params.txt"), "a") as f:
        f.write(f"maxTempLength={1 << 20}\nmaxCodeLength={1 << 27}\n")
    errs = []
    for binary in (O.REF_BIN, REF_BIN_FP128):
        if not os.path.exists(binary):
            continue
        r = subprocess.run([binary, d], capture_output=True, text=True, timeout=300)
        if r.returncode == 0:
            return np.fromfile(os.path.join(d, "out.bin"), dtype=np.float64), os.path.basename(binary)
        errs.append(f"{os.path.basename(binary)} rc={r.returncode}: {r.stderr.strip()[-4000:]}")
    raise RuntimeError("; ".join(errs))


def run_case(tmp, name, case, buf, rhs, prec):
    d = os.path.join(tmp, name)
    if prec == "dd" and os.path.exists(REF_BIN_FP128):
        O.write_reference_case(d, case, buf, rhs, precision=prec)
        import subprocess
        r = subprocess.run([REF_BIN_FP128, d], capture_output=True, text=True, timeout=120)
        if r.returncode != 0:
            raise RuntimeError(f"pfsolve_ref_fp128 failed ({r.returncode}): {r.stderr.strip()}")
        return np.fromfile(os.path.join(d, "out.bin"), dtype=np.float64)
    if case.block:
        O.write_reference_case(d, case, None, rhs, precision=prec, inp=buf)
    else:
        O.write_reference_case(d, case, buf, rhs, precision=prec)
    path, _ = O.run_reference(d)
    dt = np.float32 if prec in ("f32", "f32mem") else np.float64
    return np.fromfile(path, dtype=dt)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "golden_out"))
    ap.add_argument("--time", action="store_true")
    ap.add_argument("--only", default="all", choices=["all", "steps", "alt", "long", "dd", "dd-crash", "f32"],
                    help="steps: only the K-step fixtures (and K-step timing with --time); alt: only ALT mode; "
                         "long: only long systems (N > 4352, and their timing with --time); dd: only the double-double "
                         "fixtures; dd-crash: the double-double cases the reference crashes on (no fixtures); "
                         "f32: the FP32-storage precisions")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    tmp = os.path.join(args.out, "_cases")
    summary = {}
    single = (jw_cases() + dgbmv_cases() + alt_dgbmv_cases() + block_cases() if args.only == "all" else
              alt_dgbmv_cases() if args.only == "alt" else [])
    for name, case, buf, rhs, prec in single:
        try:
            ref = run_case(tmp, name, case, buf, rhs, prec)
            np.savez_compressed(os.path.join(args.out, name + ".npz"), params=json.dumps(asdict(case)),
                                precision=prec, buffer=buf, rhs=rhs, ref_out=ref)
            summary[name] = "ok"
        except Exception as e:  # record and continue: one failing case must not hide the others
            summary[name] = f"error: {e}"
            traceback.print_exc()
    if args.time and args.only == "all":
        timing = {}
        for label, M, B in [("config3_jw_t13_N512_B131072", 512, 131072),
                            ("config2_jw_t13_N1024_B131072real", 1024, 131072),
                            ("config1_jw_ub0_t13_N256_B512", 256, 512)]:
            rng = np.random.default_rng(1)
            ub = 0 if "ub0" in label else 2
            nat = (WL.tri_bands(*WL.tridiagonal(rng, M)) if ub == 2 else
                   WL.upper_bidiag_bands(rng.uniform(1, 2, M), rng.uniform(-.5, .5, M)))
            case = O.Case(M=M, batch=B, upperBanded=ub, jw_type=13)
            d = os.path.join(tmp, label)
            os.makedirs(d, exist_ok=True)
            O.write_reference_case(d, case, WL.permute_bands(nat, M), np.zeros(1), precision="f64", iters=20)
            os.remove(os.path.join(d, "rhs.bin"))
            with open(os.path.join(d, "params.txt"), "a") as f:
                f.write(f"rhs_bytes={8 * M * B}\n")
            try:
                _, ms = O.run_reference(d, timeout=300)
                bytes_alg = 2 * 8 * M * B
                timing[label] = dict(ms=ms, rhs_per_s=B / (ms * 1e-3), gbs=bytes_alg / (ms * 1e-3) / 1e9)
            except Exception as e:
                timing[label] = dict(error=str(e))
        with open(os.path.join(args.out, "ref_timing.json"), "w") as f:
            json.dump(timing, f, indent=1)
        print(json.dumps(timing, indent=1))
    adir = os.path.join(args.out, "alt")
    os.makedirs(adir, exist_ok=True)
    for name, case, buf, rhs, prec in (alt_cases() if args.only in ("all", "alt") else []):
        try:
            ref = run_case(tmp, name, case, buf, rhs, prec)
            np.savez_compressed(os.path.join(adir, name + ".npz"), params=json.dumps(asdict(case)),
                                precision=prec, buffer=buf, rhs=rhs, ref_out=ref)
            summary[name] = "ok"
        except Exception as e:
            summary[name] = f"error: {e}"
            traceback.print_exc()
    sdir = os.path.join(args.out, "steps")
    os.makedirs(sdir, exist_ok=True)
    for name, case, K, bufs, rhs in (steps_cases() + steps_offset_cases() if args.only in ("all", "steps") else []):
        try:
            d = os.path.join(tmp, name)
            O.write_reference_case(d, case, list(bufs) if len(bufs) > 1 else bufs[0], rhs, K=K)
            path, _ = O.run_reference(d)
            ref = np.fromfile(path, dtype=np.float64)
            np.savez_compressed(os.path.join(sdir, name + ".npz"), params=json.dumps(asdict(case)), K=K,
                                nbuf=len(bufs), rhs=rhs, ref_out=ref,
                                **{f"buffer_{k}": b for k, b in enumerate(bufs)})
            summary[name] = "ok"
        except Exception as e:
            summary[name] = f"error: {e}"
            traceback.print_exc()
    if args.time and args.only in ("all", "steps"):
        # K consecutive steps in one reference kernel (upperBanded 1, jw_type 10)
        timing = {}
        for K in (1, 2, 4):
            M, B = 512, 131072
            rng = np.random.default_rng(5)
            label = f"steps_ub1_t10_N512_K{K}_B131072"
            case = O.Case(M=M, batch=B, upperBanded=1, jw_type=10)
            d = os.path.join(tmp, label)
            os.makedirs(d, exist_ok=True)
            bufs = WL.steps_bands(rng, M, 1, K) if K > 1 else [WL.steps_bands(rng, M, 1, 2)[0]]
            O.write_reference_case(d, case, bufs if K > 1 else bufs[0], np.zeros(1), precision="f64",
                                   iters=20, K=K)
            os.remove(os.path.join(d, "rhs.bin"))
            with open(os.path.join(d, "params.txt"), "a") as f:
                f.write(f"rhs_bytes={8 * M * B}\n")
            try:
                _, ms = O.run_reference(d, timeout=300)
                timing[label] = dict(ms=ms, rhs_per_s=B / (ms * 1e-3), gbs=2 * 8 * M * B / (ms * 1e-3) / 1e9)
            except Exception as e:
                timing[label] = dict(error=str(e))
        with open(os.path.join(args.out, "ref_timing_steps.json"), "w") as f:
            json.dump(timing, f, indent=1)
        print(json.dumps(timing, indent=1))
    ldir = os.path.join(args.out, "long")
    os.makedirs(ldir, exist_ok=True)
    for name, case, buf, rhs, prec in (long_cases() if args.only in ("all", "long") else []):
        try:
            ref = run_case(tmp, name, case, buf, rhs, prec)
            np.savez_compressed(os.path.join(ldir, name + ".npz"), params=json.dumps(asdict(case)),
                                precision=prec, buffer=buf, rhs=rhs, ref_out=ref)
            summary[name] = "ok"
        except Exception as e:
            summary[name] = f"error: {e}"
            traceback.print_exc()
    if args.time and args.only in ("all", "long"):
        # long tridiagonal systems, 1 GiB of right-hand sides (jw_type 13)
        timing = {}
        for M, B in ((8192, 16384), (16384, 8192)):
            rng = np.random.default_rng(6)
            label = f"long_jw_t13_N{M}_B{B}"
            case = O.Case(M=M, batch=B, upperBanded=2, jw_type=13)
            d = os.path.join(tmp, label)
            os.makedirs(d, exist_ok=True)
            O.write_reference_case(d, case, WL.permute_bands(WL.tri_bands(*WL.tridiagonal(rng, M)), M), np.zeros(1),
                                   precision="f64", iters=20)
            os.remove(os.path.join(d, "rhs.bin"))
            with open(os.path.join(d, "params.txt"), "a") as f:
                f.write(f"rhs_bytes={8 * M * B}\n")
            try:
                _, ms = O.run_reference(d, timeout=300)
                timing[label] = dict(ms=ms, rhs_per_s=B / (ms * 1e-3), gbs=2 * 8 * M * B / (ms * 1e-3) / 1e9)
            except Exception as e:
                timing[label] = dict(error=str(e))
        with open(os.path.join(args.out, "ref_timing_long.json"), "w") as f:
            json.dump(timing, f, indent=1)
        print(json.dumps(timing, indent=1))
    fdir = os.path.join(args.out, "f32")
    os.makedirs(fdir, exist_ok=True)
    for name, case, buf, rhs, prec in (f32_cases() if args.only in ("all", "f32") else []):
        try:
            ref = run_case(tmp, name, case, buf, rhs, prec)
            np.savez_compressed(os.path.join(fdir, name + ".npz"), params=json.dumps(asdict(case)),
                                precision=prec, buffer=buf, rhs=rhs, ref_out=ref)
            summary[name] = "ok"
        except Exception as e:
            summary[name] = f"error: {e}"
            traceback.print_exc()
    ddir = os.path.join(args.out, "dd")
    os.makedirs(ddir, exist_ok=True)
    dd_set = {"all": DD_PINNED, "dd": DD_PINNED, "dd-crash": DD_CRASHING}.get(args.only, [])
    for name, case, buf, rhs, prec in dd_cases(dd_set):
        try:
            ref, binary = run_dd_case(tmp, name, case, buf, rhs)
            np.savez_compressed(os.path.join(ddir, name + ".npz"), params=json.dumps(asdict(case)),
                                precision=prec, buffer=buf, rhs=rhs, ref_out=ref, binary=binary)
            summary[name] = "ok"
        except Exception as e:
            summary[name] = f"error: {e}"
            traceback.print_exc()
    with open(os.path.join(args.out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)
    bad = [k for k, v in summary.items() if v != "ok"]
    print(f"{len(summary) - len(bad)} ok, {len(bad)} failed: {bad}")


if __name__ == "__main__":
    main()
