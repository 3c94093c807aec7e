// range_compress.cu -- range compression kernels.
//
// The reference forms range profiles with a batched in-place cuFFT inverse
// transform of the raw phase history (no zero pad, no window), then two more
// kernels: cufftNormalize_1DBatch_kernel (x /= N) and cufftShift_1DBatch_kernel
// (swap halves) (src/gpuBackProjection/cuda_sar_focusing/cuda_sar_focusing.hpp:
// 616-620, cuda_BackProjectionKernels.cuh:95-135).  Here:
//  1. rc_prep_kernel writes the FFT input in one pass: sample k < K becomes
//     ph[k] * fac[k] with fac[k] = w_k / Nfft * exp(+j 2 pi ((k s) mod Nfft) / Nfft),
//     s = (Nfft+1)/2, and k >= K is the zero pad (matlab/bpBasic.m:82).
//     The twiddle is the fftshift (cshift by s, cpuBackProjection_fft.hpp:81-84)
//     moved to the input side: ifft(x .* e^{j 2 pi k s/N})[n] = ifft(x)[n + s].
//     The 1/Nfft scale and the taper ride along, so no normalise or shift pass.
//  2. cuFFT batched C2C (Z2Z for FP64) inverse, in place.
//  3. rc_pairs_kernel stores pair entries {rc[b], rc[b+1] - rc[b]} in rows of
//     `row_stride` entries with `guard` zero entries on each side, the layout
//     the backprojection kernels stage into shared memory.
#include "sarbp_internal.h"

namespace sarbp {
namespace {

template <typename C>
__global__ void rc_prep_kernel(const float2 *__restrict__ ph, const C *__restrict__ fac, C *__restrict__ out, int K,
                               int nfft, long long total) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long p = i / nfft;
        const int k = static_cast<int>(i - p * nfft);
        C v;
        v.x = 0;
        v.y = 0;
        if (k < K) {
            const float2 x = ph[p * K + k];
            const C f = fac[k];
            v.x = x.x * f.x - x.y * f.y;
            v.y = x.x * f.y + x.y * f.x;
        }
        out[i] = v;
    }
}

struct __align__(16) PairD {
    double vr, vi, dr, di;
};

__device__ __forceinline__ void make_pair(const float2 &v, const float2 &vn, float4 *dst) {
    *dst = make_float4(v.x, v.y, vn.x - v.x, vn.y - v.y);
}
__device__ __forceinline__ void make_pair(const double2 &v, const double2 &vn, PairD *dst) {
    PairD e;
    e.vr = v.x;
    e.vi = v.y;
    e.dr = vn.x - v.x;
    e.di = vn.y - v.y;
    *dst = e;
}

template <typename C, typename E>
__global__ void rc_pairs_kernel(const C *__restrict__ X, E *__restrict__ pairs, int nfft, long long total,
                                long long row_stride, int guard) {
    const int per = nfft + 1;  // entries b = -1 .. nfft-1 of each row
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long p = i / per;
        const int b = static_cast<int>(i - p * per) - 1;
        C v, vn;
        v.x = 0;
        v.y = 0;
        vn.x = 0;
        vn.y = 0;
        if (b >= 0) v = X[p * nfft + b];
        if (b + 1 < nfft) vn = X[p * nfft + b + 1];
        make_pair(v, vn, pairs + p * row_stride + guard + b);
    }
}

// Batch forms: scene blockIdx.y of the table, grid-stride over its elements.
__global__ void rc_prep_batch_kernel(const BatchScene *__restrict__ scenes) {
    const BatchScene &S = scenes[blockIdx.y];
    const float2 *__restrict__ ph = static_cast<const float2 *>(S.ph);
    const float2 *__restrict__ fac = static_cast<const float2 *>(S.fac);
    float2 *__restrict__ out = static_cast<float2 *>(S.fft);
    const int K = S.K, nfft = S.L.nfft;
    const long long total = static_cast<long long>(S.L.np) * nfft;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long p = i / nfft;
        const int k = static_cast<int>(i - p * nfft);
        float2 v = make_float2(0.0f, 0.0f);
        if (k < K) {
            const float2 x = ph[p * K + k];
            const float2 f = fac[k];
            v.x = x.x * f.x - x.y * f.y;
            v.y = x.x * f.y + x.y * f.x;
        }
        out[i] = v;
    }
}

__global__ void rc_pairs_batch_kernel(const BatchScene *__restrict__ scenes) {
    const BatchScene &S = scenes[blockIdx.y];
    const float2 *__restrict__ X = static_cast<const float2 *>(S.fft);
    float4 *__restrict__ pairs = static_cast<float4 *>(const_cast<void *>(S.L.pairs));
    const int nfft = S.L.nfft, guard = S.L.guard;
    const int per = nfft + 1;
    const long long total = static_cast<long long>(S.L.np) * per;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long p = i / per;
        const int b = static_cast<int>(i - p * per) - 1;
        float2 v = make_float2(0.0f, 0.0f), vn = make_float2(0.0f, 0.0f);
        if (b >= 0) v = X[p * nfft + b];
        if (b + 1 < nfft) vn = X[p * nfft + b + 1];
        make_pair(v, vn, pairs + p * S.row_stride + guard + b);
    }
}

int grid_for(long long total) {
    long long blocks = (total + 255) / 256;
    const long long cap = 148LL * 16;
    return static_cast<int>(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

}  // namespace

cudaError_t launch_rc_prep(int precision, const void *ph, const void *fac, void *fft_buf, int K, int nfft, int np,
                           cudaStream_t s) {
    const long long total = static_cast<long long>(np) * nfft;
    if (precision == SARBP_PRECISION_FP64)
        rc_prep_kernel<double2><<<grid_for(total), 256, 0, s>>>(static_cast<const float2 *>(ph),
                                                                 static_cast<const double2 *>(fac),
                                                                 static_cast<double2 *>(fft_buf), K, nfft, total);
    else
        rc_prep_kernel<float2><<<grid_for(total), 256, 0, s>>>(static_cast<const float2 *>(ph),
                                                               static_cast<const float2 *>(fac),
                                                               static_cast<float2 *>(fft_buf), K, nfft, total);
    return cudaGetLastError();
}

cudaError_t launch_rc_pairs(int precision, const void *fft_buf, void *pairs, int nfft, int np, long long row_stride,
                            int guard, cudaStream_t s) {
    const long long total = static_cast<long long>(np) * (nfft + 1);
    if (precision == SARBP_PRECISION_FP64)
        rc_pairs_kernel<double2, PairD><<<grid_for(total), 256, 0, s>>>(
            static_cast<const double2 *>(fft_buf), static_cast<PairD *>(pairs), nfft, total, row_stride, guard);
    else
        rc_pairs_kernel<float2, float4><<<grid_for(total), 256, 0, s>>>(
            static_cast<const float2 *>(fft_buf), static_cast<float4 *>(pairs), nfft, total, row_stride, guard);
    return cudaGetLastError();
}

cudaError_t launch_rc_prep_batch(const BatchScene *scenes, int nscenes, cudaStream_t s) {
    if (nscenes < 1 || nscenes > 65535) return cudaErrorInvalidValue;
    rc_prep_batch_kernel<<<dim3(128, nscenes), 256, 0, s>>>(scenes);
    return cudaGetLastError();
}

cudaError_t launch_rc_pairs_batch(const BatchScene *scenes, int nscenes, cudaStream_t s) {
    if (nscenes < 1 || nscenes > 65535) return cudaErrorInvalidValue;
    rc_pairs_batch_kernel<<<dim3(128, nscenes), 256, 0, s>>>(scenes);
    return cudaGetLastError();
}

}  // namespace sarbp
