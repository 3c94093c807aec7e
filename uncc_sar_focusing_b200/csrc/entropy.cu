// entropy.cu -- the autofocus loss on the device (sarbp_image_entropy,
// sarbp_image_entropy_grad).
//
// Shannon entropy of an image's normalised intensity,
//     E = -sum_j p_j log p_j,  p_j = w_j / S,  w_j = |I_j|^2,  S = sum_j w_j,
// the loss the gradient autofocus descends (the reference's grid search
// scores images by a 2-D DFT cost instead; its Shannon form is the usual
// entropy autofocus objective).  With T = sum_j w_j log w_j,
//     E = log S - T / S,
// so one pass accumulates S and T together; and
//     dE/dw_j = -(log p_j + E) / S,
// so the gradient with respect to the image (for a real loss of a complex
// input: dL/dRe + j dL/dIm) is  g * 2 I_j * dE/dw_j,  one elementwise pass.
// Intensities are formed in FP32 as the image is stored; S and T are summed
// in FP64 in a fixed order (per-thread, warp, block, then the blocks in
// index order), so results repeat bit for bit.  log p is taken at no less
// than 1e-30, as the torch formula's clamp does.
//
// Three launches per forward-and-backward instead of the dozen elementwise
// and reduction kernels of the same formula written with torch operations.
#include <cstdint>

#include "host_common.h"
#include "sarbp_internal.h"

namespace sarbp {
namespace {

constexpr int kEntThreads = 256;
constexpr int kEntMaxBlocks = 296;
constexpr float kMinP = 1e-30f;

// Workspace: [kEntMaxBlocks][2] block sums (S, T), then S, T, E.
constexpr size_t kEntWorkDoubles = 2 * kEntMaxBlocks + 4;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sums of (S, T), fixed order: each block's threads in a grid-stride
// pattern, then the warps in order.
__device__ __forceinline__ void block_sum2(double &s, double &t) {
    __shared__ double ws[kEntThreads / 32][2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    s = warp_sum(s);
    t = warp_sum(t);
    if (lane == 0) {
        ws[warp][0] = s;
        ws[warp][1] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s = 0.0;
        t = 0.0;
        for (int w = 0; w < kEntThreads / 32; ++w) {
            s += ws[w][0];
            t += ws[w][1];
        }
    }
}

__global__ void __launch_bounds__(kEntThreads) entropy_partial_kernel(const float2 *__restrict__ img, long long n,
                                                                     double *__restrict__ work) {
    double s = 0.0, t = 0.0;
    for (long long j = blockIdx.x * static_cast<long long>(kEntThreads) + threadIdx.x; j < n;
         j += static_cast<long long>(gridDim.x) * kEntThreads) {
        const float2 v = img[j];
        const float w = fmaf(v.x, v.x, v.y * v.y);
        s += static_cast<double>(w);
        if (w > 0.0f) t += static_cast<double>(w) * static_cast<double>(logf(w));
    }
    block_sum2(s, t);
    if (threadIdx.x == 0) {
        work[2 * blockIdx.x] = s;
        work[2 * blockIdx.x + 1] = t;
    }
}

// One block: the block sums in index order, then E = log S - T / S.  The
// torch formula's clamp of p at 1e-30 changes E only for pixels whose
// p log p is below 1e-28; they are left out of T as zero intensities are.
__global__ void __launch_bounds__(kEntThreads) entropy_finish_kernel(int nblocks, double *__restrict__ work,
                                                                    float *__restrict__ out) {
    double s = 0.0, t = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += kEntThreads) {
        s += work[2 * b];
        t += work[2 * b + 1];
    }
    block_sum2(s, t);
    if (threadIdx.x == 0) {
        const double e = s > 0.0 ? log(s) - t / s : 0.0;
        double *r = work + 2 * kEntMaxBlocks;
        r[0] = s;
        r[1] = t;
        r[2] = e;
        if (out) *out = static_cast<float>(e);
    }
}

// grad[j] = g * 2 I_j * dE/dw_j, dE/dw_j = -(log max(p_j, 1e-30) + E) / S.
__global__ void __launch_bounds__(kEntThreads) entropy_grad_kernel(const float2 *__restrict__ img, long long n,
                                                                  const double *__restrict__ work,
                                                                  const float *__restrict__ grad_e,
                                                                  float2 *__restrict__ grad) {
    const double *r = work + 2 * kEntMaxBlocks;
    const double s = r[0];
    const float inv_s = s > 0.0 ? static_cast<float>(1.0 / s) : 0.0f;
    const float e = static_cast<float>(r[2]);
    const float g2 = 2.0f * (grad_e ? *grad_e : 1.0f);
    for (long long j = blockIdx.x * static_cast<long long>(kEntThreads) + threadIdx.x; j < n;
         j += static_cast<long long>(gridDim.x) * kEntThreads) {
        const float2 v = img[j];
        const float p = fmaf(v.x, v.x, v.y * v.y) * inv_s;
        const float d = -(logf(fmaxf(p, kMinP)) + e) * inv_s * g2;
        grad[j] = make_float2(d * v.x, d * v.y);
    }
}

int entropy_blocks(long long n) {
    const long long b = (n + 8LL * kEntThreads - 1) / (8LL * kEntThreads);
    return static_cast<int>(b < 1 ? 1 : (b > kEntMaxBlocks ? kEntMaxBlocks : b));
}

}  // namespace
}  // namespace sarbp

using namespace sarbp;

extern "C" {

size_t sarbp_image_entropy_work_bytes(void) { return kEntWorkDoubles * sizeof(double); }

int sarbp_image_entropy(const void *image, long long n, void *work, float *entropy, void *stream) {
    host::NvtxRange range("sarbp_image_entropy");
    if (!image || !work) return SARBP_ERR_NULL_POINTER;
    if (n < 1) return SARBP_ERR_INVALID_ARGUMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nb = entropy_blocks(n);
    double *w = static_cast<double *>(work);
    entropy_partial_kernel<<<nb, kEntThreads, 0, s>>>(static_cast<const float2 *>(image), n, w);
    SARBP_TRY_CUDA(cudaGetLastError());
    entropy_finish_kernel<<<1, kEntThreads, 0, s>>>(nb, w, entropy);
    SARBP_TRY_CUDA(cudaGetLastError());
    return SARBP_OK;
}

int sarbp_image_entropy_grad(const void *image, long long n, const void *work, const float *grad_entropy,
                             void *grad_image, void *stream) {
    host::NvtxRange range("sarbp_image_entropy_grad");
    if (!image || !work || !grad_image) return SARBP_ERR_NULL_POINTER;
    if (n < 1) return SARBP_ERR_INVALID_ARGUMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long b = (n + kEntThreads - 1) / kEntThreads;
    const int nb = static_cast<int>(b > 148LL * 16 ? 148LL * 16 : b);
    entropy_grad_kernel<<<nb, kEntThreads, 0, s>>>(static_cast<const float2 *>(image), n,
                                                   static_cast<const double *>(work), grad_entropy,
                                                   static_cast<float2 *>(grad_image));
    SARBP_TRY_CUDA(cudaGetLastError());
    return SARBP_OK;
}

}  // extern "C"
