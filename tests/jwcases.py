"""Shared helpers: run one PfSolve application through the C ABI on the GPU and
compare with the oracle."""
import numpy as np

from oracle import oracle as O


def case_fields(case: O.Case, **extra):
    """PfSolveConfiguration fields of an oracle Case."""
    f = dict(M_size=case.M, size=(case.size0, case.size1 if case.block else case.batch),
             upperBanded=case.upperBanded, jw_type=case.jw_type, jw_control_bitmask=case.bitmask,
             offsetM=case.cfg_offsetM, offsetV=case.cfg_offsetV, offsetSolution=case.cfg_offsetSolution,
             inputZeropad=case.cfg_inputZeropad, outputZeropad=case.cfg_outputZeropad,
             scaleC=case.cfg_scaleC, inputBufferStride=case.cfg_inputBufferStride,
             outputBufferStride=case.cfg_outputBufferStride, LDA=case.LDA, KU=case.KU, KL=case.KL,
             block=case.block, lshift=case.lshift, doublePrecision=1, ALT_dgbmv=case.ALT_dgbmv)
    f.update(extra)
    return f


def launch_fields(case: O.Case):
    return dict(offsetM=case.run_offsetM, offsetV=case.run_offsetV, offsetSolution=case.run_offsetSolution,
                inputZeropad=case.run_inputZeropad, outputZeropad=case.run_outputZeropad,
                scaleC=case.run_scaleC, inputBufferStride=case.run_inputBufferStride,
                outputBufferStride=case.run_outputBufferStride)


def run_app(case: O.Case, buffer: np.ndarray, out: np.ndarray, **extra):
    """Initialise + append one app; returns the output buffer after the launch."""
    import torch

    from pfsolve_b200.api import App
    tb = torch.from_numpy(np.ascontiguousarray(buffer, dtype=np.float64)).cuda()
    to = torch.from_numpy(np.array(out, dtype=np.float64, copy=True)).cuda()
    app = App(buffer=tb, outputBuffer=to, **case_fields(case, **extra))
    app.append(**launch_fields(case))
    torch.cuda.synchronize()
    res = to.cpu().numpy()
    app.close()
    return res


def precision_fields(prec: str) -> dict:
    """PfSolveConfiguration precision fields: "f64", "f32" (FP32 storage and
    arithmetic, the reference's default) or "f32mem" (FP64 arithmetic on FP32
    storage, doublePrecisionFloatMemory)."""
    if prec == "f64":
        return dict(doublePrecision=1)
    return dict(doublePrecision=0, doublePrecisionFloatMemory=1 if prec == "f32mem" else 0)


def run_app_prec(case: O.Case, buffer: np.ndarray, out: np.ndarray, prec: str, **extra):
    """run_app in a given precision; FP32-storage precisions take and return
    float32 buffers."""
    import torch

    from pfsolve_b200.api import App
    dt = np.float64 if prec == "f64" else np.float32
    tb = torch.from_numpy(np.ascontiguousarray(buffer, dtype=dt)).cuda()
    to = torch.from_numpy(np.array(out, dtype=dt, copy=True)).cuda()
    fields = case_fields(case, **extra)
    fields.update(precision_fields(prec))
    app = App(buffer=tb, outputBuffer=to, **fields)
    app.append(**launch_fields(case))
    torch.cuda.synchronize()
    res = to.cpu().numpy()
    app.close()
    return res


def run_steps(case: O.Case, K: int, bufs, out: np.ndarray, **extra):
    """K consecutive steps in one app: ``bufs`` is one band buffer read by every
    step or a list of K per-step buffers (useMultipleInputBuffers = K).
    Returns (output buffer after the launch, the plan's shape with the number
    of TMA-staged launches it made under "tma_launches")."""
    import torch

    from pfsolve_b200.api import App, streaming_launch_count
    bl = bufs if isinstance(bufs, (list, tuple)) else [bufs]
    tbs = [torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).cuda() for b in bl]
    to = torch.from_numpy(np.array(out, dtype=np.float64, copy=True)).cuda()
    app = App(buffer=tbs, outputBuffer=to, numConsecutiveJWIterations=K,
              useMultipleInputBuffers=len(tbs) if len(tbs) > 1 else 0, **case_fields(case, **extra))
    shape = app.shape()
    n0 = streaming_launch_count()
    app.append(**launch_fields(case))
    torch.cuda.synchronize()
    shape["tma_launches"] = streaming_launch_count() - n0
    res = to.cpu().numpy()
    app.close()
    return res, shape


def rel_err(x, ref, case: O.Case):
    return O.rel_errors(x, ref, case.M, case.batch, case.out_stride, case.offset_solution)


def random_bands(rng, M, ub):
    """Natural-order JW bands for the given orientation.  Off-diagonal entries
    that couple to rows outside the system (row 0 of a lower band, row M-1 of
    an upper band) are zero, as in the reference's own inputs
    (sample_0_benchmark_VkFFT_single.cpp:191-192): the reference reads an
    unrelated register value for such a neighbour."""
    if ub == 2:
        a = rng.uniform(-1, 1, M)
        c = rng.uniform(-1, 1, M)
        a[0] = 0
        c[-1] = 0
        d = np.abs(a) + np.abs(c) + rng.uniform(1, 2, M)
        return np.concatenate([a / d, 1 / d, c / d])
    # Any of the three bands is the solve band in some jw_type: |entries| < 1/2
    # keeps every unit-diagonal recurrence stable.
    bands = [rng.uniform(-0.5, 0.5, M) for _ in range(3)]
    for k in range(3):
        bands[k][0] = 0.0
        bands[k][-1] = 0.0
    return np.concatenate(bands)
