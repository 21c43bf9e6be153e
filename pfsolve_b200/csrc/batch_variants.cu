// batch_variants.cu -- instantiations of the persistent uneven-batch kernel.
#include "jw_batch_seq.cuh"
#include "jw_kernel.cuh"
#include "jw_variants.h"
#include "stream_variant_defs.h"

namespace pfb {

template <class C>
static size_t batch_smem_fn(int W, int G)
{
    return jw_batch_smem_bytes<C>(W, G);
}

template <class C>
static void batch_launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const BatchEntryDev* entries,
                            const WorkItem* items, int nitems, unsigned int* counter, int W)
{
    jw_batch_kernel<C><<<grid, block, smem, st>>>(entries, items, nitems, counter, W);
}

#define PFB_BV(R, KL, KU, SV, LIN, LOUT, SC, P)                                                   \
    BatchVariant{R, KL, KU, SV, LIN, LOUT, SC, P,                                                 \
                 (const void*)&jw_batch_kernel<JwCfg<R, KL, KU, SV, LIN, LOUT, SC, P>>,           \
                 &batch_smem_fn<JwCfg<R, KL, KU, SV, LIN, LOUT, SC, P>>,                          \
                 &batch_launch_fn<JwCfg<R, KL, KU, SV, LIN, LOUT, SC, P>>}
#define PFB_BV2(KL, KU, SV, LIN, LOUT, SC, P) PFB_BV(4, KL, KU, SV, LIN, LOUT, SC, P), PFB_BV(8, KL, KU, SV, LIN, LOUT, SC, P)

static const BatchVariant kBatchVariants[] = {
    // one spectral timestep: 3-band V + upper-bidiagonal M, SphLaplA, XXII -> packed
    PFB_BV2(1, 1, SV_UPPER, LAY_XXII, LAY_PACKED, true, PREC_F64),
    PFB_BV2(1, 1, SV_UPPER, LAY_XXII, LAY_PACKED, false, PREC_F64),
    // request batches of the serving loop (real systems, in place)
    PFB_BV2(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, false, PREC_F64),
    PFB_BV2(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, false, PREC_MIXED),
    PFB_BV2(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false, PREC_F64),
    PFB_BV2(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false, PREC_MIXED),
    PFB_BV2(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false, PREC_F64),
    PFB_BV2(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false, PREC_MIXED),
    PFB_BV2(0, 0, SV_LOWER, LAY_REAL, LAY_REAL, false, PREC_MIXED),
    PFB_BV2(0, 1, SV_LOWER, LAY_REAL, LAY_REAL, false, PREC_MIXED),
    PFB_BV2(1, 0, SV_UPPER, LAY_REAL, LAY_REAL, false, PREC_MIXED),
};

const BatchVariant* find_batch_variant(int R, int KL, int KU, int SV, int LIN, int LOUT, int SCALE, int PREC)
{
    for (const BatchVariant& v : kBatchVariants)
        if (v.R == R && v.KL == KL && v.KU == KU && v.SV == SV && v.LIN == LIN && v.LOUT == LOUT &&
            v.SCALE == (SCALE ? 1 : 0) && v.PREC == PREC)
            return &v;
    return nullptr;
}

template <int SVK, int CH, int NBUF, int NW>
static void batch_seq_launch_fn(dim3 grid, size_t smem, cudaStream_t st, const BatchEntryDev* entries,
                                const BatchSeqEntry* seq, const double* coefs, const WorkItem* items, int nitems,
                                unsigned int* counter)
{
    jw_batch_seq_kernel<SVK, CH, NBUF, NW><<<grid, 32 * NW, smem, st>>>(entries, seq, coefs, items, nitems, counter);
}
template <int SVK>
static void batch_seq_coef_fn(int nentries, cudaStream_t st, const BatchEntryDev* entries, const BatchSeqEntry* seq,
                              double* coefs)
{
    jw_batch_seq_coef_kernel<SVK><<<nentries, 128, 0, st>>>(entries, seq, coefs);
}

// warps per CTA: as many as the shared memory of one SM holds
#define PFB_BSV(SVK, CH, NBUF, NW)                                                                  \
    BatchSeqVariant{SVK, CH, NBUF, NW, (const void*)&jw_batch_seq_kernel<SVK, CH, NBUF, NW>,       \
                    &batch_seq_launch_fn<SVK, CH, NBUF, NW>, &batch_seq_coef_fn<SVK>}
// shapes in order of preference: 16-row chunks first (128-byte rows per system
// and part: fewer, longer DRAM bursts than 8-row chunks)
#define PFB_BSV_SHAPES(SVK) PFB_BSV(SVK, 16, 4, 5), PFB_BSV(SVK, 16, 3, 6), PFB_BSV(SVK, 8, 4, 10)

static const BatchSeqVariant kBatchSeqVariants[] = {
    PFB_BSV_SHAPES(SV_UPPER),
    PFB_BSV_SHAPES(SV_LOWER),
    PFB_BSV_SHAPES(SV_NONE),
};

const BatchSeqVariant* find_batch_seq_variant(int SV, int shape)
{
    int n = 0;
    for (const BatchSeqVariant& v : kBatchSeqVariants)
        if (v.SV == SV && n++ == shape) return &v;
    return nullptr;
}

size_t batch_seq_smem(const BatchSeqVariant* v) { return batch_seq_smem_bytes(v->CH, v->NBUF, v->NW); }
int64_t batch_seq_rows(int64_t M) { return batch_seq_coef_rows(M); }

PFB_STREAM_STATUS_ACCESSOR(batch_status_fetch_clear)

}  // namespace pfb
