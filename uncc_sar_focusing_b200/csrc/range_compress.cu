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
#include <cmath>
#include <vector>

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
    if (S.fused) return;  // range-compressed by its own fused launch
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
    if (S.fused) return;
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

// ---- fused range compression: nfft = R K, K = 32 K2 ------------------------
//
// With y[k] = fac[k] ph[k] (taper x 1/N x shift twiddle) and N = R K the
// zero-padded inverse DFT splits into R inverse DFTs of length K:
//     rc[R m + r] = sum_k (y[k] W_N^{k r}) W_K^{k m},   W_L = exp(+j 2 pi / L).
// One CTA per pulse (grid-stride), one warp per sub-transform r.  Each
// length-K transform is done in four steps with K = 32 K2, k = k1 + 32 k2,
// m = m2 + K2 m1:  lane k1 transforms its K2 samples in registers (over k2),
// multiplies by W_K^{k1 m2}, the warp transposes through shared memory, and
// lane m2 transforms the 32 values over k1 in registers.  The R results are
// read back interleaved to write the pair entries {rc[b], rc[b+1] - rc[b]},
// b = -1 .. N-1, straight to HBM: 8 bytes read per input sample, 16 bytes
// written per pair entry, no FFT buffer.  Twiddles come from one table built
// in double on the host and staged into shared memory.
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

template <int L>
__host__ __device__ constexpr int log2_of() {
    int n = 0;
    for (int v = L; v > 1; v >>= 1) ++n;
    return n;
}

template <int L>
__device__ __forceinline__ constexpr int bit_reverse(int x) {
    int r = 0;
    for (int b = 1; b < L; b <<= 1) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

// exp(+j 2 pi e / 32) for e in [0, 16) as FP32 constants (correctly rounded);
// after unrolling every e is a compile-time constant
__device__ __forceinline__ float2 w32(int e) {
    constexpr float c1 = 0.980785251f, s1 = 0.195090324f, c2 = 0.923879504f, s2 = 0.382683426f;
    constexpr float c3 = 0.831469595f, s3 = 0.555570245f, h = 0.707106769f;
    switch (e) {
        case 1: return make_float2(c1, s1);
        case 2: return make_float2(c2, s2);
        case 3: return make_float2(c3, s3);
        case 4: return make_float2(h, h);
        case 5: return make_float2(s3, c3);
        case 6: return make_float2(s2, c2);
        case 7: return make_float2(s1, c1);
        case 9: return make_float2(-s1, c1);
        case 10: return make_float2(-s2, c2);
        case 11: return make_float2(-s3, c3);
        case 12: return make_float2(-h, h);
        case 13: return make_float2(-c3, s3);
        case 14: return make_float2(-c2, s2);
        case 15: return make_float2(-c1, s1);
        default: return make_float2(1.0f, 0.0f);
    }
}

// In-register inverse DFT of L points (L divides 32): radix-2 decimation in
// frequency, natural-order input, bit-reversed output.  The twiddles W_L^e =
// W_32^(e 32 / L) are constants, 1 and +j without a multiply (68.5 vs 72.2 us
// with the twiddles loaded from a shared-memory table; same results).
template <int L>
__device__ __forceinline__ void ifft_dif(float2 (&v)[L]) {
    constexpr int LOG = log2_of<L>();
#pragma unroll
    for (int st = 0; st < LOG; ++st) {
        const int half = (L >> 1) >> st;
#pragma unroll
        for (int i = 0; i < L; i += 2 * half) {
#pragma unroll
            for (int j = 0; j < half; ++j) {
                const float2 a = v[i + j], b = v[i + j + half];
                v[i + j] = make_float2(a.x + b.x, a.y + b.y);
                const float2 d = make_float2(a.x - b.x, a.y - b.y);
                const int e = j * (L / (2 * half));
                constexpr int kScale = 32 / L;
                const int e32 = e * kScale;
                v[i + j + half] = e32 == 0 ? d : (e32 == 8 ? make_float2(-d.y, d.x) : cmulf(d, w32(e32)));
            }
        }
    }
}

// Layout of the twiddle table (complex64 entries) for K = 32 K2, N = R K.
template <int K2, int R>
struct RcTable {
    static constexpr int K = 32 * K2, N = K * R, NW = N / 32;
    static constexpr int kTwk = 0;                 // W_K^{k1 m2} at m2 * 32 + k1
    static constexpr int kWn = kTwk + K;           // W_N^i, i < 32 R
    static constexpr int kWnr = kWn + 32 * R;      // W_{N/32}^i, i < N / 32
    static constexpr int kSize = kWnr + NW;
    // shared row of one sub-transform.  The pair-row writes read element
    // (r, m) = (b mod R, b / R) for consecutive b: 16 lanes (one 128-byte
    // wavefront of 8-byte reads) cover R values of r and 16/R of m, first
    // bank 2 (r kReg + m) mod 32; kReg = 16/R mod 16 makes these 16
    // distinct even banks for every R (K + 36, right for R = 4, put r and
    // r + 4 on the same banks for R = 8)
    static constexpr int kReg = K + 32 + 16 / R;
    static constexpr size_t kSmem = (static_cast<size_t>(K) + kSize + static_cast<size_t>(R) * kReg) * 8;
};

template <int K2, int R>
__device__ __forceinline__ void rc_fused_body(const float2 *__restrict__ ph, const float2 *__restrict__ fac,
                                              const float2 *__restrict__ tab, float4 *__restrict__ pairs, int np,
                                              long long row_stride, int guard) {
    using T = RcTable<K2, R>;
    constexpr int K = T::K, N = T::N, REG = T::kReg, LOGR = log2_of<R>();
    extern __shared__ __align__(16) float2 rc_sm[];
    float2 *y = rc_sm, *tb = y + K, *regions = tb + T::kSize;
    const int tid = threadIdx.x, r = tid >> 5, lane = tid & 31;
    for (int i = tid; i < T::kSize; i += 32 * R) tb[i] = tab[i];
    float2 *reg = regions + r * REG;
    // a pulse's input samples, loaded one pulse ahead: issued before the
    // current pulse's row writes (the long phase), consumed after the barrier
    constexpr int KPT = (K + 32 * R - 1) / (32 * R);
    float2 pre[KPT];
    auto prefetch = [&](int q) {
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const int k = tid + j * 32 * R;
            pre[j] = (q < np && k < K) ? ph[static_cast<long long>(q) * K + k] : make_float2(0.0f, 0.0f);
        }
    };
    prefetch(blockIdx.x);
    for (int p = blockIdx.x; p < np; p += gridDim.x) {
        __syncthreads();  // the previous pulse's reads of the regions are done; the table is staged
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
            const int k = tid + j * 32 * R;
            if (k < K) y[k] = cmulf(pre[j], fac[k]);
        }
        __syncthreads();
        // z[k1 + 32 k2] = y[.] W_N^{k1 r} W_{N/32}^{k2 r}, transformed over k2
        const float2 a = tb[T::kWn + lane * r];
        float2 v[K2];
#pragma unroll
        for (int k2 = 0; k2 < K2; ++k2)
            v[k2] = cmulf(y[lane + 32 * k2], cmulf(a, tb[T::kWnr + ((k2 * r) & (T::NW - 1))]));
        ifft_dif<K2>(v);
        // times W_K^{k1 m2}, transposed: element (k1, m2) at m2 * 33 + k1
#pragma unroll
        for (int m2 = 0; m2 < K2; ++m2) reg[m2 * 33 + lane] = cmulf(v[bit_reverse<K2>(m2)], tb[T::kTwk + m2 * 32 + lane]);
        __syncwarp();
        float2 w[32];
        if (lane < K2) {
#pragma unroll
            for (int k1 = 0; k1 < 32; ++k1) w[k1] = reg[lane * 33 + k1];
        }
        __syncwarp();
        if (lane < K2) {
            ifft_dif<32>(w);
#pragma unroll
            for (int m1 = 0; m1 < 32; ++m1) reg[lane + K2 * m1] = w[bit_reverse<32>(m1)];
        }
        __syncthreads();
        prefetch(p + gridDim.x);
        // rc[R m + r] = regions[r][m]
        float4 *row = pairs + static_cast<long long>(p) * row_stride + guard;
        for (int b = tid - 1; b < N; b += 32 * R) {
            float2 u = make_float2(0.0f, 0.0f), un = make_float2(0.0f, 0.0f);
            if (b >= 0) u = regions[(b & (R - 1)) * REG + (b >> LOGR)];
            if (b + 1 < N) un = regions[((b + 1) & (R - 1)) * REG + ((b + 1) >> LOGR)];
            row[b] = make_float4(u.x, u.y, un.x - u.x, un.y - u.y);
        }
    }
}

template <int K2, int R>
__global__ void __launch_bounds__(32 * R) rc_fused_kernel(const float2 *__restrict__ ph,
                                                         const float2 *__restrict__ fac,
                                                         const float2 *__restrict__ tab, float4 *__restrict__ pairs,
                                                         int np, long long row_stride, int guard) {
    rc_fused_body<K2, R>(ph, fac, tab, pairs, np, row_stride, guard);
}

// The same for one scene of a batch: every pointer and size from the scene's
// slot of the device table, so a captured graph replays with new buffers.
template <int K2, int R>
__global__ void __launch_bounds__(32 * R) rc_fused_scene_kernel(const BatchScene *__restrict__ scene,
                                                               const float2 *__restrict__ tab) {
    const BatchScene &S = *scene;
    rc_fused_body<K2, R>(static_cast<const float2 *>(S.ph), static_cast<const float2 *>(S.fac), tab,
                         static_cast<float4 *>(const_cast<void *>(S.L.pairs)), S.L.np, S.row_stride, S.L.guard);
}

template <int K2, int R>
void fill_rc_table(std::vector<float> &t) {
    using T = RcTable<K2, R>;
    t.assign(2 * static_cast<size_t>(T::kSize), 0.0f);
    auto put = [&](int at, double num, double den) {
        const double a = 2.0 * M_PI * num / den;
        t[2 * static_cast<size_t>(at)] = static_cast<float>(std::cos(a));
        t[2 * static_cast<size_t>(at) + 1] = static_cast<float>(std::sin(a));
    };
    for (int m2 = 0; m2 < K2; ++m2)
        for (int k1 = 0; k1 < 32; ++k1) put(T::kTwk + m2 * 32 + k1, static_cast<double>(k1) * m2, T::K);
    for (int i = 0; i < 32 * R; ++i) put(T::kWn + i, i, T::N);
    for (int i = 0; i < T::NW; ++i) put(T::kWnr + i, i, T::NW);
}

template <int K2, int R>
cudaError_t launch_fused(const float2 *ph, const float2 *fac, const float2 *tab, float4 *pairs, int np,
                         long long row_stride, int guard, int grid, cudaStream_t s) {
    using T = RcTable<K2, R>;
    auto kern = rc_fused_kernel<K2, R>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(T::kSmem));
    if (e != cudaSuccess) return e;
    const int g = np < grid ? np : grid;
    kern<<<g > 0 ? g : 1, 32 * R, T::kSmem, s>>>(ph, fac, tab, pairs, np, row_stride, guard);
    return cudaGetLastError();
}

// Range profiles rc[b] back out of the pair rows (sarbp_get_range_profiles
// after fused range compression).
__global__ void pairs_to_rc_kernel(const float4 *__restrict__ pairs, float2 *__restrict__ rc, int nfft,
                                   long long total, long long row_stride, int guard) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long p = i / nfft;
        const int b = static_cast<int>(i - p * nfft);
        const float4 e = pairs[p * row_stride + guard + b];
        rc[i] = make_float2(e.x, e.y);
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

#define SARBP_RC_SHAPES(X) \
    X(8, 1) X(8, 2) X(8, 4) X(8, 8) X(8, 16) X(16, 1) X(16, 2) X(16, 4) X(16, 8) X(16, 16) X(32, 1) X(32, 2) \
        X(32, 4) X(32, 8) X(32, 16)

bool rc_fused_shape(int K, int R, size_t *smem, std::vector<float> *table) {
#define SARBP_RC_CASE(K2_, R_)                                        \
    if (K == 32 * K2_ && R == R_) {                                   \
        if (smem) *smem = RcTable<K2_, R_>::kSmem;                    \
        if (table) fill_rc_table<K2_, R_>(*table);                    \
        return true;                                                  \
    }
    SARBP_RC_SHAPES(SARBP_RC_CASE)
#undef SARBP_RC_CASE
    return false;
}

cudaError_t launch_rc_fused(const void *ph, const void *fac, const void *table, void *pairs, int K, int R, int np,
                            long long row_stride, int guard, int grid, cudaStream_t s) {
#define SARBP_RC_CASE(K2_, R_)                                                                                   \
    if (K == 32 * K2_ && R == R_)                                                                                 \
        return launch_fused<K2_, R_>(static_cast<const float2 *>(ph), static_cast<const float2 *>(fac),          \
                                     static_cast<const float2 *>(table), static_cast<float4 *>(pairs), np,        \
                                     row_stride, guard, grid, s);
    SARBP_RC_SHAPES(SARBP_RC_CASE)
#undef SARBP_RC_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_rc_fused_scene(const BatchScene *scene, const void *table, int K, int R, int grid,
                                  cudaStream_t s) {
#define SARBP_RC_CASE(K2_, R_)                                                                                   \
    if (K == 32 * K2_ && R == R_) {                                                                               \
        auto kern = rc_fused_scene_kernel<K2_, R_>;                                                               \
        const size_t smem = RcTable<K2_, R_>::kSmem;                                                              \
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                             static_cast<int>(smem));                                             \
        if (e != cudaSuccess) return e;                                                                           \
        kern<<<grid > 0 ? grid : 1, 32 * R_, smem, s>>>(scene, static_cast<const float2 *>(table));               \
        return cudaGetLastError();                                                                                \
    }
    SARBP_RC_SHAPES(SARBP_RC_CASE)
#undef SARBP_RC_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_pairs_to_rc(const void *pairs, void *rc, int nfft, int np, long long row_stride, int guard,
                               cudaStream_t s) {
    const long long total = static_cast<long long>(np) * nfft;
    pairs_to_rc_kernel<<<grid_for(total), 256, 0, s>>>(static_cast<const float4 *>(pairs), static_cast<float2 *>(rc),
                                                      nfft, total, row_stride, guard);
    return cudaGetLastError();
}

}  // namespace sarbp
