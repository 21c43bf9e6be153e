// noalloc.cu -- PfSolveBatchAppendNoAlloc: an uneven batch (the persistent
// jw_batch_kernel) run without allocating anything.
//
// PfSolveBatchCreate keeps its work list, entry descriptors and work counter
// in cudaMalloc'd buffers.  This entry point stages them instead in a fixed
// file-scope device array (g_noalloc_scratch) and in fixed host arrays, so a
// call never reaches the device allocator.  Limits: kMaxEntries entries and
// kMaxItems work items per call.  The work counter must start at zero: every
// call clears it with cudaMemsetAsync on its stream before the launch.  All
// calls share the one scratch array, so calls whose work overlaps in time
// (other streams, other host threads) race on it.  The host staging arrays
// are pageable: cudaMemcpyAsync stages them before it returns, so the next
// call may rewrite them at once.  Because the next call rewrites them, a call
// on a stream that is being captured is refused (PFSOLVE_ERROR_INVALID_ARGUMENT)
// before it enqueues anything.  The caller's current device is restored on
// every return.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/pfsolve_b200.h"
#include "plan.h"

using namespace pfb;

namespace {

constexpr int kMaxEntries = PFSOLVE_NOALLOC_MAX_ENTRIES;
constexpr int kMaxItems = PFSOLVE_NOALLOC_MAX_ITEMS;
constexpr size_t kCounterBytes = 256;
constexpr size_t kEntryBytes = (size_t)kMaxEntries * sizeof(BatchEntryDev);
constexpr size_t kItemBytes = (size_t)kMaxItems * sizeof(WorkItem);
constexpr size_t kScratchBytes = kCounterBytes + kEntryBytes + kItemBytes;

// [work counter | entry descriptors | work items]
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// host staging of one call (fixed, not allocated)
BatchEntryDev g_entries[kMaxEntries];
WorkItem g_items[kMaxItems];

constexpr int kMaxDevices = 64;
unsigned char* g_scratch_ptr[kMaxDevices];
std::mutex g_setup_mu;

// Device address of the scratch array on the current device, looked up once
// per device.
PfSolveResult scratch_address(int device, unsigned char** out)
{
    if (device < 0 || device >= kMaxDevices) return PFSOLVE_ERROR_INVALID_DEVICE;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;
        }
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[device];
    return PFSOLVE_SUCCESS;
}

// Restores the calling thread's current device when the call returns.
struct DeviceGuard {
    int saved = -1;
    DeviceGuard()
    {
        if (cudaGetDevice(&saved) != cudaSuccess) {
            cudaGetLastError();
            saved = -1;
        }
    }
    ~DeviceGuard()
    {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

// Work items largest first; ties by (entry, first system), so the order is
// the same on every call.  std::sort sorts in place: no temporary buffer.
bool item_before(const WorkItem& x, const WorkItem& y)
{
    const int64_t a = g_entries[x.entry].op.M * (x.y1 - x.y0), b = g_entries[y.entry].op.M * (y.y1 - y.y0);
    if (a != b) return a > b;
    if (x.entry != y.entry) return x.entry < y.entry;
    return x.y0 < y.y0;
}

}  // namespace

extern "C" PfSolveResult PfSolveBatchAppendNoAlloc(CUdevice device, const PfSolveBatchDesc* desc,
                                                   const PfSolveBatchEntry* entries, int nentries,
                                                   cudaStream_t stream)
{
    if (!desc || nentries < 0 || (nentries > 0 && !entries)) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    if (nentries > kMaxEntries) return PFSOLVE_ERROR_CAPACITY;
    if (desc->sweepRows) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;  // the group kernel only
    if (desc->mixedPrecisionRefinement < 0 || desc->mixedPrecisionRefinement > 3) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    const int bt = desc->block % 10, sk = desc->block / 100;
    if (!(bt == 0 || bt == 1 || bt == 7) || ((desc->block / 10) % 10 != 0 && (desc->block / 10) % 10 != 2) || sk > 4 ||
        (bt == 0 && desc->block != 0))
        return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    PfSolveConfiguration c;
    memset(&c, 0, sizeof(c));
    c.upperBanded = desc->upperBanded;
    c.jw_type = desc->jw_type;
    c.M_size = 16;
    JwLayout L0;
    if (desc->jw_type < 10 || !jw_layout(c, false, false, 0, 0, L0)) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    int KL = (L0.mvj == MVJ_LOWER) ? 1 : 0, KU = (L0.mvj == MVJ_UPPER) ? 1 : 0;
    if (desc->LDA > 0) {
        if (desc->KU < 0 || desc->KU >= desc->LDA) return PFSOLVE_ERROR_INVALID_ARGUMENT;
        KL += desc->LDA - 1 - desc->KU;
        KU += desc->KU;
    }
    const int LIN = (bt == 7) ? LAY_XXII : LAY_REAL, LOUT = (bt == 7) ? LAY_PACKED : LAY_REAL;
    const int PREC = (desc->mixedPrecisionRefinement > 0 && L0.sv != SV_NONE) ? PREC_MIXED : PREC_F64;

    // entry descriptors (same operator and data description as PfSolveBatchCreate)
    int64_t Mmax = 0;
    for (int e = 0; e < nentries; ++e) {
        const PfSolveBatchEntry& en = entries[e];
        if (en.M < 1 || en.M > 4096 || en.nsys < 0 || !en.bands || !en.input || !en.output)
            return PFSOLVE_ERROR_INVALID_ARGUMENT;
        if (desc->LDA > 0 && !en.dgbmvBands) return PFSOLVE_ERROR_INVALID_ARGUMENT;
        c.M_size = en.M;
        JwLayout L;
        jw_layout(c, false, false, 0, 0, L);
        BatchEntryDev& d = g_entries[e];
        memset(&d, 0, sizeof(d));
        d.op.M = en.M;
        set_band_order(en.M, d.op);
        d.op.refine_sweeps = 1 + desc->mixedPrecisionRefinement;
        d.op.bands = static_cast<const double*>(en.bands);
        d.op.off_md = L.off_md;
        d.op.off_mo = L.off_mo;
        d.op.off_sl = L.off_sl;
        d.op.off_su = L.off_su;
        d.op.mvj = L.mvj;
        d.op.scaleC = en.scaleC;
        if (desc->LDA > 0) {
            d.op.dgbmv = static_cast<const double*>(en.dgbmvBands);
            d.op.dg_lda = desc->LDA;
            d.op.dg_ku = desc->KU;
        }
        d.op.scale_kind = sk;
        d.op.lshift = en.lshift;
        d.op.scale_s = en.scaleS;
        d.io.in = static_cast<const double*>(en.input);
        d.io.out = static_cast<double*>(en.output);
        d.io.in_stride = en.inputStride;
        d.io.out_stride = en.outputStride;
        d.io.iz1 = INT64_MAX / 4;
        d.io.oz1 = INT64_MAX / 4;
        d.io.nsys = en.nsys;
        d.io.M = en.M;
        d.io.accumulate = ((desc->block / 10) % 10) == 2;
        Mmax = std::max<int64_t>(Mmax, en.M);
    }

    // work items: systemsPerItem systems each, largest first
    const int64_t spi = desc->systemsPerItem > 0 ? desc->systemsPerItem : 64;
    int nitems = 0;
    for (int e = 0; e < nentries; ++e)
        for (int64_t y0 = 0; y0 < entries[e].nsys; y0 += spi) {
            if (nitems >= kMaxItems) return PFSOLVE_ERROR_CAPACITY;
            WorkItem& w = g_items[nitems++];
            w.entry = e;
            w.pad = 0;
            w.y0 = y0;
            w.y1 = std::min<int64_t>(entries[e].nsys, y0 + spi);
        }
    std::sort(g_items, g_items + nitems, item_before);
    if (nitems == 0) return PFSOLVE_SUCCESS;

    DeviceGuard keep_device;
    if (cudaSetDevice(device) != cudaSuccess) return PFSOLVE_ERROR_INVALID_DEVICE;
    // The descriptors are copied from g_entries / g_items, which the next call
    // rewrites: a captured copy would replay whatever the latest call left
    // there.  A stream under capture (or one whose capture state cannot be
    // read, e.g. the legacy stream while another stream captures globally)
    // is refused before anything is enqueued.
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
            cudaGetLastError();
            return PFSOLVE_ERROR_INVALID_ARGUMENT;
        }
        if (cs != cudaStreamCaptureStatusNone) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    }
    int num_sms = 0;
    if (cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;
    unsigned char* scratch = nullptr;
    PfSolveResult res = scratch_address(device, &scratch);
    if (res != PFSOLVE_SUCCESS) return res;

    int maxopt = 0;
    if (cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess)
        return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;

    // launch shape: as PfSolveBatchCreate (rows per thread 8, else 4)
    const BatchVariant* v = nullptr;
    int W = 1, G = 1, blocks = 0;
    const int Rs[2] = {desc->rowsPerThread ? desc->rowsPerThread : 8, 4};
    for (int k = 0; k < (desc->rowsPerThread ? 1 : 2) && !v; ++k) {
        const int R = Rs[k];
        const int64_t w = (Mmax + 32 * (int64_t)R - 1) / (32 * (int64_t)R);
        if (w < 1 || w > 8) continue;
        const BatchVariant* cand = find_batch_variant(R, KL, KU, L0.sv, LIN, LOUT, sk ? 1 : 0, PREC);
        if (!cand) continue;
        const int g = std::max(1, 8 / (int)w);
        const size_t smem = cand->smem_bytes((int)w, g);
        // the shared-memory opt-in, set directly to the device's maximum as
        // the plan path sets it (idempotent; the plan path's cache of
        // opted-in kernels is a std::set, which would allocate)
        if (smem > 48 * 1024 &&
            (smem > (size_t)maxopt ||
             cudaFuncSetAttribute(cand->func, cudaFuncAttributeMaxDynamicSharedMemorySize, maxopt) != cudaSuccess)) {
            cudaGetLastError();
            continue;
        }
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, cand->func, 32 * (int)w * g, smem) != cudaSuccess || b < 1)
            continue;
        v = cand;
        W = (int)w;
        G = g;
        blocks = b;
    }
    if (!v) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;

    unsigned int* d_counter = reinterpret_cast<unsigned int*>(scratch);
    BatchEntryDev* d_entries = reinterpret_cast<BatchEntryDev*>(scratch + kCounterBytes);
    WorkItem* d_items = reinterpret_cast<WorkItem*>(scratch + kCounterBytes + kEntryBytes);
    if (cudaMemcpyAsync(d_entries, g_entries, nentries * sizeof(BatchEntryDev), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(d_items, g_items, nitems * sizeof(WorkItem), cudaMemcpyHostToDevice, stream) != cudaSuccess ||
        cudaMemsetAsync(d_counter, 0, sizeof(unsigned int), stream) != cudaSuccess)
        return PFSOLVE_ERROR_FAILED_TO_COPY;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((nitems + G - 1) / G, (int64_t)blocks * num_sms));
    v->launch(dim3((unsigned)grid), dim3(32 * W * G), v->smem_bytes(W, G), stream, d_entries, d_items, nitems,
              d_counter, W);
    note_launch(false);
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    return PFSOLVE_SUCCESS;
}
