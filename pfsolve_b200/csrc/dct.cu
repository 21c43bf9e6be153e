// dct.cu -- instantiations and launch of the DCT-step kernel (dct.cuh), and
// its twiddle tables.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <new>

#include "dct.cuh"
#include "jw_variants.h"

namespace pfb {

namespace {

template <int LOGN, int TYPE>
cudaError_t dct_launch_t(const DctIO& io, const double2* tw, const double2* pt, int num_sms, cudaStream_t st)
{
    using S = DctShape<LOGN>;
    const void* f = (const void*)&dct_kernel<LOGN, TYPE>;
    // per device on first use: the shared-memory opt-in and the resident CTAs
    static std::mutex mu;
    static int blocks_of[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    int blocks;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!blocks_of[dev]) {
            if (S::SMEM > 48 * 1024 &&
                cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM) != cudaSuccess)
                return cudaGetLastError();
            int b = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, S::NT, S::SMEM) != cudaSuccess || b < 1)
                return cudaErrorInvalidConfiguration;
            blocks_of[dev] = b;
        }
        blocks = blocks_of[dev];
    }
    const int64_t want = ((io.nsys + 1) / 2 + S::SPC - 1) / S::SPC;  // row pairs per CTA round: SPC
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)blocks * num_sms));
    dct_kernel<LOGN, TYPE><<<(unsigned)grid, S::NT, S::SMEM, st>>>(io, tw, pt);
    return cudaPeekAtLastError();
}

template <int TYPE>
cudaError_t dct_launch_type(int logn, const DctIO& io, const double2* tw, const double2* pt, int num_sms,
                            cudaStream_t st)
{
    switch (logn) {
    case 3: return dct_launch_t<3, TYPE>(io, tw, pt, num_sms, st);
    case 4: return dct_launch_t<4, TYPE>(io, tw, pt, num_sms, st);
    case 5: return dct_launch_t<5, TYPE>(io, tw, pt, num_sms, st);
    case 6: return dct_launch_t<6, TYPE>(io, tw, pt, num_sms, st);
    case 7: return dct_launch_t<7, TYPE>(io, tw, pt, num_sms, st);
    case 8: return dct_launch_t<8, TYPE>(io, tw, pt, num_sms, st);
    case 9: return dct_launch_t<9, TYPE>(io, tw, pt, num_sms, st);
    case 10: return dct_launch_t<10, TYPE>(io, tw, pt, num_sms, st);
    case 11: return dct_launch_t<11, TYPE>(io, tw, pt, num_sms, st);
    case 12: return dct_launch_t<12, TYPE>(io, tw, pt, num_sms, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t dct_launch(int logn, int type, const DctIO& io, const double2* tw, const double2* pt, int num_sms,
                       cudaStream_t st)
{
    if (type == 2) return dct_launch_type<2>(logn, io, tw, pt, num_sms, st);
    if (type == 3) return dct_launch_type<3>(logn, io, tw, pt, num_sms, st);
    return cudaErrorInvalidValue;
}

// tw[j] = e^{-2 pi i j/N}, pt[k] = (cos, sin)(pi k/(2N)), from long double
// values rounded once; both in one allocation (tw first).
cudaError_t dct_tables(int64_t N, double2** tables)
{
    const size_t n = (size_t)2 * N;
    double2* h = new (std::nothrow) double2[n];
    if (!h) return cudaErrorMemoryAllocation;
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int64_t j = 0; j < N; ++j) {
        const long double a = -2.0L * pi * (long double)j / (long double)N;
        h[j] = make_double2((double)cosl(a), (double)sinl(a));
        const long double t = pi * (long double)j / (long double)(2 * N);
        h[N + j] = make_double2((double)cosl(t), (double)sinl(t));
    }
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(tables), n * sizeof(double2));
    if (e == cudaSuccess) e = cudaMemcpy(*tables, h, n * sizeof(double2), cudaMemcpyHostToDevice);
    delete[] h;
    return e;
}

}  // namespace pfb
