"""Serving engine on the GPU, through the C ABI (PfSolveServer*).

Checks and tolerances (relative L2 per system):
  * every request against the __float128 oracle: mixed precision (FP32 solve,
    two FP64 refinement sweeps) <= 1e-12; double-double storage <= 1e-27;
  * each result is the same alone and in a concurrent mix: mixed <= 1e-13,
    double-double <= 1e-28 between the two runs;
  * admission by HBM footprint: the peak of admitted in-flight bytes stays
    within the budget and every request completes;
  * a Poisson run at the serving workload's arrival rate completes every
    request and reports p50/p99 latency.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pfsolve_b200 import capi
from pfsolve_b200 import workloads as WL

pytestmark = pytest.mark.gpu
MIXED, DD = capi.PFSOLVE_SERVE_MIXED, capi.PFSOLVE_SERVE_DD


def _prepare(server, specs, seed):
    import torch
    rng = np.random.default_rng(seed)
    ops, reqs = {}, []
    for sp in specs:
        if sp.M not in ops:
            bands = WL.serve_operator_bands(np.random.default_rng(sp.M), sp.M)
            tb = torch.from_numpy(bands).cuda()
            ops[sp.M] = (server.add_operator(sp.M, tb), bands, tb)
        rhs = rng.uniform(-1, 1, sp.M * sp.nrhs)
        if sp.precision == DD:
            rhs = O.to_dd(rhs)
            rhs[1::2] = rhs[0::2] * rng.uniform(-1, 1, sp.M * sp.nrhs) * 2.0 ** -60
        inp = torch.from_numpy(rhs).cuda()
        out = torch.zeros_like(inp)
        reqs.append(dict(spec=sp, op=ops[sp.M][0], bands=ops[sp.M][1], rhs=rhs, inp=inp, out=out))
    return ops, reqs


def _oracle_err(r, got):
    sp = r["spec"]
    case = O.Case(M=sp.M, batch=sp.nrhs, upperBanded=2, jw_type=13)
    if sp.precision == DD:
        ref = O.jw_step(case, O.to_dd(r["bands"]), r["rhs"], "dd")
        return O.rel_errors_dd(got, ref, sp.M, sp.nrhs, sp.M)[0]
    ref = O.jw_step(case, r["bands"], r["rhs"], "q")
    return O.rel_errors(got, ref, sp.M, sp.nrhs, sp.M)[0]


def _specs(n, seed, r_max=512):
    return WL.config5_requests(n, seed=seed, r_max=r_max)


def test_each_request_matches_oracle_alone_and_in_mix():
    import torch

    from pfsolve_b200.serving import Server
    specs = _specs(40, seed=4)
    assert any(s.precision == DD for s in specs) and any(s.precision == MIXED for s in specs)
    srv = Server(streams=4, max_batch_requests=16)
    _, reqs = _prepare(srv, specs, seed=5)
    # alone: one request at a time
    alone = []
    for r in reqs:
        t = srv.submit(r["op"], r["spec"].precision, r["spec"].nrhs, r["inp"], r["out"])
        srv.wait(t)
        alone.append(r["out"].cpu().numpy().copy())
        r["out"].zero_()
    # the clears are done before the mix starts (each request also waits for
    # the default stream's work queued before its submit)
    torch.cuda.synchronize()
    # in the mix: all submitted back to back, batched and overlapped
    tickets = [srv.submit(r["op"], r["spec"].precision, r["spec"].nrhs, r["inp"], r["out"]) for r in reqs]
    for t in tickets:
        srv.wait(t)
    torch.cuda.synchronize()
    st = srv.stats()
    assert st["completed"] == 2 * len(reqs)
    assert st["batches"] < 2 * len(reqs), "the mix was not batched"
    bad = []
    for i, (r, a) in enumerate(zip(reqs, alone)):
        sp = r["spec"]
        mixed = r["out"].cpu().numpy()
        e_alone = _oracle_err(r, a)
        e_mix = _oracle_err(r, mixed)
        tol = 1e-27 if sp.precision == DD else 1e-12
        if sp.precision == DD:
            d = O.rel_errors_dd(mixed, a, sp.M, sp.nrhs, sp.M)[0]
            dtol = 1e-28
        else:
            d = O.rel_errors(mixed, a, sp.M, sp.nrhs, sp.M)[0]
            dtol = 1e-13
        if not (e_alone <= tol and e_mix <= tol and d <= dtol):
            bad.append((i, sp, e_alone, e_mix, d))
    srv.close()
    assert not bad, bad


@pytest.mark.parametrize("precision", [MIXED, DD])
def test_submit_waits_for_pending_default_stream_write(precision):
    """A request submitted while the caller's default-stream write of its input
    (and clear of its output) is still queued behind a long kernel reads the
    written input: the request's kernel waits for the event Submit records on
    the caller's stream.  Checked against the __float128 oracle."""
    import torch

    from pfsolve_b200.serving import Server
    M, nrhs = 256, 64
    srv = Server(streams=2, max_batch_requests=4)
    bands = WL.serve_operator_bands(np.random.default_rng(M), M)
    tb = torch.from_numpy(bands).cuda()
    op = srv.add_operator(M, tb)
    rng = np.random.default_rng(17)
    rhs = rng.uniform(-1, 1, M * nrhs)
    if precision == DD:
        rhs = O.to_dd(rhs)
    src = torch.from_numpy(rhs).cuda()
    inp = torch.full_like(src, 1e30)   # a stale input the request must not see
    out = torch.full_like(src, 7.0)
    torch.cuda.synchronize()
    torch.cuda._sleep(200_000_000)     # ~0.1 s of GPU spinning on the default stream (bounded by its cycle count)
    inp.copy_(src)                     # queued behind it
    out.zero_()
    t = srv.submit(op, precision, nrhs, inp, out)   # stream None: the legacy default stream
    srv.wait(t)
    got = out.cpu().numpy()
    srv.close()
    r = dict(spec=WL.ServeRequestSpec(M, nrhs, precision), bands=bands, rhs=rhs)
    e = _oracle_err(r, got)
    assert e <= (1e-27 if precision == DD else 1e-12), e


def test_admission_by_hbm_budget():
    from pfsolve_b200.serving import Server
    specs = _specs(60, seed=6, r_max=2048)
    budget = 24 << 20
    srv = Server(hbm_budget_bytes=budget, streams=8, max_batch_requests=8)
    _, reqs = _prepare(srv, specs, seed=7)
    tickets = []
    for r in reqs:
        sp = r["spec"]
        nbytes = sp.M * sp.nrhs * (16 if sp.precision == DD else 8) * 2
        if nbytes > budget:
            with pytest.raises(capi.PfSolveError):
                srv.submit(r["op"], sp.precision, sp.nrhs, r["inp"], r["out"])
            continue
        tickets.append(srv.submit(r["op"], sp.precision, sp.nrhs, r["inp"], r["out"]))
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    assert st["completed"] == len(tickets) > 0
    assert 0 < st["peakInflightBytes"] <= budget
    srv.close()


def test_poisson_load_short():
    from pfsolve_b200.serving import Server, run_load
    specs = _specs(400, seed=8)
    srv = Server(streams=8, max_batch_requests=32)
    _, reqs = _prepare(srv, specs, seed=9)
    arrivals = WL.poisson_arrivals(len(reqs), 20000.0, seed=8)
    lat, wall, lag = run_load(srv, [(r["op"], r["spec"].precision, r["spec"].nrhs, r["inp"], r["out"]) for r in reqs],
                              arrivals)
    st = srv.stats()
    assert st["completed"] == len(reqs)
    assert all(x > 0 for x in lat)
    assert st["p50Ms"] <= st["p99Ms"] <= st["maxMs"]
    srv.close()


def test_invalid_requests_rejected():
    import torch

    from pfsolve_b200.serving import Server
    srv = Server(hbm_budget_bytes=1 << 20)
    tb = torch.from_numpy(WL.serve_operator_bands(np.random.default_rng(0), 64)).cuda()
    op = srv.add_operator(64, tb)
    x = torch.zeros(64 * 4096, dtype=torch.float64, device="cuda")
    with pytest.raises(capi.PfSolveError):
        srv.submit(op + 1, MIXED, 1, x, x)
    with pytest.raises(capi.PfSolveError):
        srv.submit(op, 7, 1, x, x)
    with pytest.raises(capi.PfSolveError):  # 64 * 4096 * 8 B in place = 2 MiB > 1 MiB budget
        srv.submit(op, MIXED, 4096, x, x)
    t = srv.submit(op, MIXED, 16, x, x)
    srv.wait(t)
    srv.close()
