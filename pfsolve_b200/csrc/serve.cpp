// serve.cpp -- the serving engine: JW-step requests of mixed size and
// precision, admitted by HBM footprint and batched continuously.
//
// One worker thread owns dispatch.  A request joins the queue on submit; the
// worker takes the queue head's precision class, gathers the queued requests
// of that class that fit the HBM budget (bytes of every admitted, unfinished
// request) up to maxBatchRequests, and launches them on a free stream:
//   * mixed precision (FP32 solve + FP64 refinement): one persistent
//     uneven-batch launch over all requests of the batch (jw_batch_kernel),
//     descriptors copied from pinned staging on the same stream;
//   * double-double: one JW-step launch per request (jw_dd_kernel).
// Ordering with the caller: the server's streams are non-blocking, so they do
// not follow the caller's (legacy default or other) stream.  Submit records an
// event on the request's `stream` (unless the caller marks the input ready)
// and the flight waits for it before the request's kernel: whatever the
// caller enqueued before Submit (writing the input, clearing the output)
// happens first.
// An event is recorded behind every batch; the worker polls the events of
// the batches in flight (at least every 20 us while any is), stamps the
// requests' completion time, releases their bytes and wakes the waiters.
// With `streams` batches in flight, requests that arrive while others run are
// admitted as soon as a stream and bytes free up, and their kernels overlap on
// the device.  Mixed-precision batches prefer high-priority streams;
// double-double requests run one per flight (one launch each) on the
// low-priority ones.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/pfsolve_b200.h"
#include "plan.h"

using namespace pfb;

namespace {

using Clock = std::chrono::steady_clock;

struct ServeOp {
    int64_t M;
    const double* bands;
    double* bands_dd;  // {hi, lo} copy (lo = 0), owned
    JwLayout L;
    int KL, KU;
};

struct Req {
    uint64_t id;
    PfSolveRequest r;
    int64_t M;
    uint64_t bytes;
    int cls;  // batch class: precision class and operator kind (one kernel per batch)
    PfSolveResult status = PFSOLVE_SUCCESS;
    cudaEvent_t ready = nullptr;  // recorded on the caller's stream at submit (nullptr: input ready)
    Clock::time_point t_submit, t_dispatch, t_done;
    bool done = false;
};

struct Shape {
    int G = 0, max_blocks = 0;
    size_t smem = 0;
};

struct Flight {
    PfSolveServer* srv = nullptr;
    cudaStream_t stream = nullptr;
    BatchEntryDev* h_entries = nullptr;  // pinned staging
    WorkItem* h_items = nullptr;
    BatchEntryDev* d_entries = nullptr;
    WorkItem* d_items = nullptr;
    unsigned int* d_counter = nullptr;
    int items_cap = 0;
    cudaEvent_t done = nullptr;  // recorded behind the batch; the worker polls it
    std::vector<Req*> reqs;
    bool busy = false;
    bool launched = false;  // the batch (and its event) has been enqueued
    bool high = false;      // high-priority stream: mixed-precision batches only
    int cls = 0;        // batch class of the requests in flight
};


}  // namespace

struct PfSolveServer {
    PfSolveServerDesc desc;
    int num_sms = 0;
    std::deque<ServeOp> ops;  // references stay valid while operators are added
    std::map<std::pair<const void*, int>, Shape> shapes;  // (kernel, W) -> groups, blocks
    std::mutex shape_mu;                                   // guards `shapes`
    std::mutex mu;
    std::condition_variable cv;       // worker
    std::condition_variable done_cv;  // waiters
    std::deque<Req*> pending;
    std::unordered_map<uint64_t, Req*> reqs;
    std::vector<Flight> flights;
    std::vector<cudaEvent_t> ready_pool;  // ordering events not in use (guarded by mu)
    uint64_t next_id = 1;
    uint64_t inflight_bytes = 0, peak_inflight = 0;
    uint64_t submitted = 0, completed = 0, batches = 0, rhs = 0;
    std::vector<double> lat_ms, queue_ms, device_ms;
    bool stop = false;
    std::thread worker;
};

namespace {

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Rows per thread and warps per system for systems of up to Mmax rows.
void serve_rows(int64_t Mmax, int& R, int& W)
{
    R = (Mmax <= 128) ? 4 : 8;
    W = (int)((Mmax + 32 * R - 1) / (32 * R));
    int p = 1;
    while (p < W) p <<= 1;
    W = p;
}

// Double-double kernel for systems of M rows: the register form at 4 rows
// per thread up to 128 rows, else the table form (coefficients built once per
// CTA in shared memory), 16 rows per thread up to 512 rows (one warp), else 8.
const JwVariant* serve_dd_variant(int64_t M, int KL, int KU, int sv, int prec, int& W)
{
    int R = 4, tbl = 0;
    if (M > 128) {
        R = (M <= 512) ? 16 : 8;
        tbl = 1;
    }
    W = (int)((M + 32 * R - 1) / (32 * R));
    int p = 1;
    while (p < W) p <<= 1;
    W = p;
    return find_jw_variant(R, KL, KU, sv, LAY_REAL, LAY_REAL, 0, prec, tbl);
}

bool batch_shape(PfSolveServer* s, const BatchVariant* v, int W, Shape& out)
{
    std::lock_guard<std::mutex> lk(s->shape_mu);
    auto key = std::make_pair(v->func, W);
    auto it = s->shapes.find(key);
    if (it != s->shapes.end()) { out = it->second; return true; }
    for (int G = std::max(1, 8 / W); G >= 1; --G) {
        const size_t smem = v->smem_bytes(W, G);
        if (smem > 227 * 1024) continue;
        if (!allow_max_smem(v->func)) continue;
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, v->func, 32 * W * G, smem) != cudaSuccess ||
            blocks < 1)
            continue;
        out.G = G;
        out.max_blocks = blocks * s->num_sms;
        out.smem = smem;
        s->shapes[key] = out;
        return true;
    }
    cudaGetLastError();
    return false;
}

bool jw_shape(PfSolveServer* s, const JwVariant* v, int W, Shape& out)
{
    std::lock_guard<std::mutex> lk(s->shape_mu);
    auto key = std::make_pair(v->func, W);
    auto it = s->shapes.find(key);
    if (it != s->shapes.end()) { out = it->second; return true; }
    int G = 0, maxb = 0;
    if (!choose_groups(v, W, s->num_sms, G, maxb)) { cudaGetLastError(); return false; }
    out.G = G;
    out.max_blocks = maxb;
    out.smem = v->smem_bytes(W, G);
    s->shapes[key] = out;
    return true;
}

JwOperator make_operator(const PfSolveServer* s, const ServeOp& o, const PfSolveRequest& r)
{
    JwOperator op;
    memset(&op, 0, sizeof(op));
    op.bands = (r.precision == PFSOLVE_SERVE_DD) ? o.bands_dd : o.bands;
    op.off_md = o.L.off_md;
    op.off_mo = o.L.off_mo;
    op.off_sl = o.L.off_sl;
    op.off_su = o.L.off_su;
    op.mvj = o.L.mvj;
    op.scaleC = r.scaleC;
    op.M = o.M;
    set_band_order(o.M, op);
    op.refine_sweeps = 1 + s->desc.refineSweeps;
    return op;
}

JwIO make_io(const ServeOp& o, const PfSolveRequest& r)
{
    JwIO io;
    memset(&io, 0, sizeof(io));
    io.in = static_cast<const double*>(r.input);
    io.out = static_cast<double*>(r.output);
    io.in_stride = io.out_stride = r.stride ? r.stride : o.M;
    io.iz0 = io.oz0 = 0;
    io.iz1 = io.oz1 = INT64_MAX / 4;
    io.nsys = r.nrhs;
    io.M = o.M;
    return io;
}

// Complete the requests of flight `fl` (its event has fired).  Called by the
// worker with the server lock held.
void complete_flight(PfSolveServer* s, Flight& fl, Clock::time_point now)
{
    for (Req* r : fl.reqs) {
        r->t_done = now;
        r->done = true;
        s->inflight_bytes -= r->bytes;
        s->completed++;
        s->rhs += (uint64_t)r->r.nrhs;
        s->lat_ms.push_back(ms_between(r->t_submit, now));
        s->queue_ms.push_back(ms_between(r->t_submit, r->t_dispatch));
        s->device_ms.push_back(ms_between(r->t_dispatch, now));
    }
    fl.reqs.clear();
    fl.busy = false;
    s->batches++;
}

// Complete every flight whose work has finished; true when any did.
bool reap_flights(PfSolveServer* s)
{
    bool any = false;
    const Clock::time_point now = Clock::now();
    for (Flight& fl : s->flights) {
        if (!fl.busy || !fl.launched) continue;
        const cudaError_t e = cudaEventQuery(fl.done);
        if (e == cudaErrorNotReady) continue;
        if (e != cudaSuccess) {
            cudaGetLastError();
            for (Req* r : fl.reqs) r->status = PFSOLVE_ERROR_FAILED_TO_SYNCHRONIZE;
        }
        complete_flight(s, fl, now);
        any = true;
    }
    return any;
}

// Enqueue the batch of flight `fl` (mixed: one uneven-batch launch; dd: one
// launch per request), then its completion event.  First the flight's
// stream waits for each request's ordering event; a wait captures the
// event's state when it is enqueued, so the events go back to the pool
// right after.
void launch_flight(PfSolveServer* s, Flight& fl, int cls)
{
    for (Req* r : fl.reqs) {
        if (!r->ready) continue;
        if (cudaStreamWaitEvent(fl.stream, r->ready, 0) != cudaSuccess) {
            cudaGetLastError();
            r->status = PFSOLVE_ERROR_FAILED_TO_SYNCHRONIZE;
        }
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Req* r : fl.reqs)
            if (r->ready) {
                s->ready_pool.push_back(r->ready);
                r->ready = nullptr;
            }
    }
    if (cls == 0) {
        int64_t Mmax = 0, S = 0;
        for (Req* r : fl.reqs) {
            Mmax = std::max(Mmax, r->M);
            S += r->r.nrhs;
        }
        int R, W;
        serve_rows(Mmax, R, W);
        const ServeOp& o0 = s->ops[fl.reqs[0]->r.op];
        const BatchVariant* v = find_batch_variant(R, o0.KL, o0.KU, o0.L.sv, LAY_REAL, LAY_REAL, 0, PREC_MIXED);
        Shape sh;
        if (!v || !batch_shape(s, v, W, sh)) {
            for (Req* r : fl.reqs) r->status = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        } else {
            // items: enough per group for balance, within the staging capacity
            const int64_t groups = (int64_t)sh.max_blocks * sh.G;
            int64_t spi = std::max<int64_t>(1, std::min<int64_t>(64, (S + 2 * groups - 1) / (2 * groups)));
            int64_t nitems = 0;
            for (;;) {
                nitems = 0;
                for (Req* r : fl.reqs) nitems += (r->r.nrhs + spi - 1) / spi;
                if (nitems <= fl.items_cap) break;
                spi *= 2;
            }
            int k = 0, e = 0;
            for (Req* r : fl.reqs) {
                const ServeOp& o = s->ops[r->r.op];
                fl.h_entries[e].op = make_operator(s, o, r->r);
                fl.h_entries[e].io = make_io(o, r->r);
                for (int64_t y0 = 0; y0 < r->r.nrhs; y0 += spi) {
                    fl.h_items[k].entry = e;
                    fl.h_items[k].pad = 0;
                    fl.h_items[k].y0 = y0;
                    fl.h_items[k].y1 = std::min<int64_t>(r->r.nrhs, y0 + spi);
                    ++k;
                }
                ++e;
            }
            cudaMemcpyAsync(fl.d_entries, fl.h_entries, e * sizeof(BatchEntryDev), cudaMemcpyHostToDevice, fl.stream);
            cudaMemcpyAsync(fl.d_items, fl.h_items, k * sizeof(WorkItem), cudaMemcpyHostToDevice, fl.stream);
            cudaMemsetAsync(fl.d_counter, 0, sizeof(unsigned int), fl.stream);
            const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((k + sh.G - 1) / sh.G, sh.max_blocks));
            v->launch(dim3((unsigned)grid), dim3(32 * W * sh.G), sh.smem, fl.stream, fl.d_entries, fl.d_items, k,
                      fl.d_counter, W);
            note_launch(false);
            if (cudaGetLastError() != cudaSuccess)
                for (Req* r : fl.reqs) r->status = PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
        }
    } else {
        for (Req* r : fl.reqs) {
            const ServeOp& o = s->ops[r->r.op];
            int W;
            const int prec = (r->r.precision == PFSOLVE_SERVE_DD) ? 2 : 3;
            const JwVariant* v = serve_dd_variant(o.M, o.KL, o.KU, o.L.sv, prec, W);
            Shape sh;
            if (!v || !jw_shape(s, v, W, sh)) {
                r->status = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
                continue;
            }
            const JwOperator op = make_operator(s, o, r->r);
            const JwIO io = make_io(o, r->r);
            // one system per group (no persistent CTAs): short CTAs let the
            // high-priority streams' blocks in between
            const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((io.nsys + sh.G - 1) / sh.G, INT32_MAX));
            v->launch(dim3((unsigned)grid), dim3(32 * W * sh.G), sh.smem, fl.stream, op, io, W);
            note_launch(false);
            if (cudaGetLastError() != cudaSuccess) r->status = PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
        }
    }
    cudaEventRecord(fl.done, fl.stream);
}

// A free stream for a batch of class `cls`: mixed precision prefers the
// high-priority streams, double-double only uses the low-priority ones.
int free_flight(PfSolveServer* s, int cls)
{
    const bool dd = cls >= 1000;
    for (int pass = 0; pass < 2; ++pass)
        for (size_t i = 0; i < s->flights.size(); ++i) {
            const Flight& fl = s->flights[i];
            if (fl.busy) continue;
            if (dd && fl.high) continue;
            if (!dd && pass == 0 && !fl.high) continue;
            return (int)i;
        }
    return -1;
}

// Double-double requests run one launch each, one request per flight and
// only on the low-priority streams: short mixed-precision batches are never
// queued behind them, and a short double-double request never waits for a
// long one batched with it (a flight completes as a whole).
constexpr int kDdBatch = 1;

// The request that opens the next batch: the first queued request whose class
// has a free stream; nullptr when none has (or its bytes do not fit yet:
// admission is first come, first served).
Req* next_head(PfSolveServer* s, int& flight)
{
    for (Req* r : s->pending) {
        const int f = free_flight(s, r->cls);
        if (f < 0) continue;
        if (s->inflight_bytes + r->bytes > s->desc.hbmBudgetBytes) return nullptr;
        flight = f;
        return r;
    }
    return nullptr;
}

void worker_loop(PfSolveServer* s)
{
    cudaSetDevice(s->desc.device);
    std::unique_lock<std::mutex> lk(s->mu);
    const uint64_t budget = s->desc.hbmBudgetBytes;
    for (;;) {
        if (reap_flights(s)) s->done_cv.notify_all();
        Req* head = nullptr;
        int f = -1;
        if (!s->pending.empty()) head = next_head(s, f);
        if (!head) {
            bool busy = false;
            for (const Flight& fl : s->flights) busy = busy || fl.busy;
            if (s->stop && s->pending.empty() && !busy) break;  // drained
            // sleep until a submission, or poll the flights in flight again shortly
            if (busy) s->cv.wait_for(lk, std::chrono::microseconds(20));
            else s->cv.wait(lk);
            continue;
        }
        Flight& fl = s->flights[f];
        const int cls = head->cls;
        const int cap = (cls >= 1000) ? std::min(kDdBatch, s->desc.maxBatchRequests) : s->desc.maxBatchRequests;
        uint64_t add = 0;
        for (auto it = s->pending.begin(); it != s->pending.end() && (int)fl.reqs.size() < cap;) {
            Req* r = *it;
            if (r->cls != cls) {
                ++it;
                continue;
            }
            if (s->inflight_bytes + add + r->bytes > budget) break;
            fl.reqs.push_back(r);
            add += r->bytes;
            it = s->pending.erase(it);
        }
        s->inflight_bytes += add;
        s->peak_inflight = std::max(s->peak_inflight, s->inflight_bytes);
        fl.busy = true;
        fl.launched = false;
        fl.cls = cls;
        const Clock::time_point now = Clock::now();
        for (Req* r : fl.reqs) r->t_dispatch = now;
        lk.unlock();
        launch_flight(s, fl, cls / 1000);
        lk.lock();
        fl.launched = true;
    }
}

void free_flight_resources(Flight& fl)
{
    if (fl.stream) cudaStreamDestroy(fl.stream);
    if (fl.done) cudaEventDestroy(fl.done);
    if (fl.h_entries) cudaFreeHost(fl.h_entries);
    if (fl.h_items) cudaFreeHost(fl.h_items);
    if (fl.d_entries) cudaFree(fl.d_entries);
    if (fl.d_items) cudaFree(fl.d_items);
    if (fl.d_counter) cudaFree(fl.d_counter);
}

}  // namespace

extern "C" {

PfSolveResult PfSolveServerCreate(PfSolveServer** server, const PfSolveServerDesc* desc)
{
    if (!server || !desc) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    *server = nullptr;
    if (desc->hbmBudgetBytes == 0 || desc->streams < 1 || desc->streams > 16 || desc->maxBatchRequests < 1 ||
        desc->maxBatchRequests > 256 || desc->refineSweeps < 1 || desc->refineSweeps > 3)
        return PFSOLVE_ERROR_INVALID_ARGUMENT;
    if (cudaSetDevice(desc->device) != cudaSuccess) return PFSOLVE_ERROR_INVALID_DEVICE;
    PfSolveServer* s = new (std::nothrow) PfSolveServer();
    if (!s) return PFSOLVE_ERROR_MALLOC_FAILED;
    s->desc = *desc;
    if (cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, desc->device) != cudaSuccess) {
        delete s;
        return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;
    }
    s->flights.resize(desc->streams);
    const int cap = desc->maxBatchRequests * 64;
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    bool ok = true;
    for (size_t i = 0; i < s->flights.size(); ++i) {
        Flight& fl = s->flights[i];
        fl.srv = s;
        fl.items_cap = cap;
        // one stream: shared by both classes; otherwise half high priority
        fl.high = desc->streams > 1 && (int)i < desc->streams / 2;
        ok = ok && cudaStreamCreateWithPriority(&fl.stream, cudaStreamNonBlocking, fl.high ? prio_high : prio_low) ==
                       cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&fl.done, cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaMallocHost(&fl.h_entries, desc->maxBatchRequests * sizeof(BatchEntryDev)) == cudaSuccess;
        ok = ok && cudaMallocHost(&fl.h_items, cap * sizeof(WorkItem)) == cudaSuccess;
        ok = ok && cudaMalloc(&fl.d_entries, desc->maxBatchRequests * sizeof(BatchEntryDev)) == cudaSuccess;
        ok = ok && cudaMalloc(&fl.d_items, cap * sizeof(WorkItem)) == cudaSuccess;
        ok = ok && cudaMalloc(&fl.d_counter, sizeof(unsigned int)) == cudaSuccess;
    }
    if (!ok) {
        for (Flight& fl : s->flights) free_flight_resources(fl);
        delete s;
        return PFSOLVE_ERROR_FAILED_TO_ALLOCATE;
    }
    s->worker = std::thread(worker_loop, s);
    *server = s;
    return PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveServerAddOperator(PfSolveServer* s, int64_t M, const double* bands, int upperBanded, int jw_type,
                                       int* opId)
{
    if (!s || !bands || !opId || M < 1 || M > 1024) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    PfSolveConfiguration c;
    memset(&c, 0, sizeof(c));
    c.M_size = M;
    c.upperBanded = upperBanded;
    c.jw_type = jw_type;
    ServeOp o;
    memset(&o, 0, sizeof(o));
    o.M = M;
    o.bands = bands;
    if (upperBanded < 0 || upperBanded > 2 || jw_type < 10 || !jw_layout(c, false, false, 0, 0, o.L) ||
        o.L.sv == SV_NONE)
        return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    o.KL = (o.L.mvj == MVJ_LOWER) ? 1 : 0;
    o.KU = (o.L.mvj == MVJ_UPPER) ? 1 : 0;
    for (int R : {4, 8}) {
        if (!find_batch_variant(R, o.KL, o.KU, o.L.sv, LAY_REAL, LAY_REAL, 0, PREC_MIXED))
            return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    }
    for (int prec : {PREC_DD, PREC_DD_F64MEM}) {
        int W;
        if (!serve_dd_variant(M, o.KL, o.KU, o.L.sv, prec, W)) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    }
    cudaSetDevice(s->desc.device);
    if (cudaMalloc(&o.bands_dd, 3 * M * 2 * sizeof(double)) != cudaSuccess) return PFSOLVE_ERROR_FAILED_TO_ALLOCATE;
    if (cudaMemset(o.bands_dd, 0, 3 * M * 2 * sizeof(double)) != cudaSuccess ||
        cudaMemcpy2D(o.bands_dd, 2 * sizeof(double), bands, sizeof(double), sizeof(double), 3 * M,
                     cudaMemcpyDeviceToDevice) != cudaSuccess) {
        cudaFree(o.bands_dd);
        return PFSOLVE_ERROR_FAILED_TO_COPY;
    }
    // Resolve every launch shape this operator can need now, so that the
    // worker never queries (and first loads) a kernel while serving.
    for (int R : {4, 8}) {
        for (int W = 1; W <= (R == 4 ? 1 : 4); W *= 2) {  // the shapes serve_rows picks for M <= 1024
            Shape sh;
            batch_shape(s, find_batch_variant(R, o.KL, o.KU, o.L.sv, LAY_REAL, LAY_REAL, 0, PREC_MIXED), W, sh);
        }
    }
    for (int64_t Mr : {(int64_t)64, (int64_t)256, (int64_t)768, (int64_t)1024})  // every dd variant and W
        for (int prec : {PREC_DD, PREC_DD_F64MEM}) {
            int W;
            Shape sh;
            const JwVariant* v = serve_dd_variant(Mr, o.KL, o.KU, o.L.sv, prec, W);
            if (v) jw_shape(s, v, W, sh);
        }
    std::lock_guard<std::mutex> lk(s->mu);
    s->ops.push_back(o);
    *opId = (int)s->ops.size() - 1;
    return PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveServerSubmit(PfSolveServer* s, const PfSolveRequest* r, uint64_t* ticket)
{
    if (!s || !r || !ticket || !r->input || !r->output || r->nrhs < 1 || r->stride < 0) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    if (r->precision < PFSOLVE_SERVE_MIXED || r->precision > PFSOLVE_SERVE_DD_FP64MEM) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    Req* q = new (std::nothrow) Req();
    if (!q) return PFSOLVE_ERROR_MALLOC_FAILED;
    if (!r->inputReady) {
        // the ordering event, recorded on the caller's stream on the server's
        // device (the caller's current device is restored)
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (!s->ready_pool.empty()) {
                q->ready = s->ready_pool.back();
                s->ready_pool.pop_back();
            }
        }
        int saved = -1;
        if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
        bool ok = cudaSetDevice(s->desc.device) == cudaSuccess;
        if (ok && !q->ready) ok = cudaEventCreateWithFlags(&q->ready, cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaEventRecord(q->ready, r->stream) == cudaSuccess;
        if (saved >= 0 && saved != s->desc.device) cudaSetDevice(saved);
        if (!ok) {
            cudaGetLastError();
            if (q->ready) {
                std::lock_guard<std::mutex> lk(s->mu);
                s->ready_pool.push_back(q->ready);
            }
            delete q;
            return PFSOLVE_ERROR_FAILED_TO_EVENT_RECORD;
        }
    }
    // a rejected request returns its ordering event to the pool
    auto reject = [&](Req* q_) {
        if (q_->ready) s->ready_pool.push_back(q_->ready);
        delete q_;
    };
    std::unique_lock<std::mutex> lk(s->mu);
    if (r->op < 0 || r->op >= (int)s->ops.size()) {
        reject(q);
        return PFSOLVE_ERROR_INVALID_ARGUMENT;
    }
    q->r = *r;
    const ServeOp& o = s->ops[r->op];
    q->M = o.M;
    q->cls = (r->precision == PFSOLVE_SERVE_MIXED ? 0 : 1000) + 100 * o.KL + 10 * o.KU + o.L.sv;
    if (r->stride && r->stride < q->M) {
        reject(q);
        return PFSOLVE_ERROR_INVALID_ARGUMENT;
    }
    const uint64_t elem = (r->precision == PFSOLVE_SERVE_DD) ? 16 : 8;
    q->bytes = (uint64_t)r->nrhs * (uint64_t)q->M * elem * (r->input == r->output ? 1 : 2);
    if (q->bytes > s->desc.hbmBudgetBytes) {
        reject(q);
        return PFSOLVE_ERROR_CAPACITY;
    }
    q->id = s->next_id++;
    q->t_submit = Clock::now();
    s->reqs[q->id] = q;
    s->pending.push_back(q);
    s->submitted++;
    *ticket = q->id;
    lk.unlock();
    s->cv.notify_all();
    return PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveServerWait(PfSolveServer* s, uint64_t ticket, double* latencyMs)
{
    if (!s) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    Req* q = it->second;
    s->done_cv.wait(lk, [&] { return q->done; });
    if (latencyMs) *latencyMs = ms_between(q->t_submit, q->t_done);
    const PfSolveResult status = q->status;
    s->reqs.erase(it);
    delete q;
    return status;
}

PfSolveResult PfSolveServerGetStats(PfSolveServer* s, PfSolveServerStats* out)
{
    if (!s || !out) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    std::vector<double> lat, qm, dm;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        out->submitted = s->submitted;
        out->completed = s->completed;
        out->batches = s->batches;
        out->rhs = s->rhs;
        out->peakInflightBytes = s->peak_inflight;
        lat = s->lat_ms;
        qm = s->queue_ms;
        dm = s->device_ms;
    }
    auto quantile = [](std::vector<double>& v, double f) {
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        return v[std::min(v.size() - 1, (size_t)(f * (v.size() - 1) + 0.5))];
    };
    out->p50Ms = quantile(lat, 0.50);
    out->p99Ms = quantile(lat, 0.99);
    out->maxMs = lat.empty() ? 0.0 : lat.back();
    out->p99QueueMs = quantile(qm, 0.99);
    out->p99DeviceMs = quantile(dm, 0.99);
    return PFSOLVE_SUCCESS;
}

void PfSolveServerDestroy(PfSolveServer* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->desc.device);
    for (Flight& fl : s->flights)
        if (fl.stream) cudaStreamSynchronize(fl.stream);
    for (Flight& fl : s->flights) free_flight_resources(fl);
    for (ServeOp& o : s->ops)
        if (o.bands_dd) cudaFree(o.bands_dd);
    for (auto& kv : s->reqs) {
        if (kv.second->ready) cudaEventDestroy(kv.second->ready);
        delete kv.second;
    }
    for (cudaEvent_t e : s->ready_pool) cudaEventDestroy(e);
    delete s;
}

}  // extern "C"
