// probes.cu -- pipe-throughput probes for the backprojection roofline.
//
// The backprojection is bounded by the FP32, FP64, MUFU (sin/cos) and
// shared-memory pipes, not by HBM or tensor cores.  Each probe kernel issues
// a known number of one operation from 148 x 8 CTAs of 256 threads with eight
// independent chains per thread; sarbp_probe times it with CUDA events and
// returns the operation rate, so the bench divides by peaks measured on the
// same GPU in the same run.  Built into libsarbp_probes.so, used by bench.py.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;

__global__ void probe_ffma(float *out, int iters) {
    float a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) a[j] = threadIdx.x * 1e-3f + j;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int j = 0; j < kChains; ++j) a[j] = fmaf(a[j], 0.9999999f, 1e-7f);
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += a[j];
    if (s == 123.456f) out[0] = s;  // keeps the chains alive
}

__global__ void probe_dfma(double *out, int iters) {
    double a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) a[j] = threadIdx.x * 1e-3 + j;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int j = 0; j < kChains; ++j) a[j] = fma(a[j], 0.9999999999, 1e-12);
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += a[j];
    if (s == 123.456) out[0] = s;
}

// one __sincosf = MUFU.SIN + MUFU.COS (+ the range scaling multiply)
__global__ void probe_sincos(float *out, int iters) {
    float x[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) x[j] = threadIdx.x * 1e-4f + 0.1f * j;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int j = 0; j < kChains; ++j) {
            float s, c;
            __sincosf(x[j], &s, &c);
            x[j] = s + c;
        }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += x[j];
    if (s == 123.456f) out[0] = s;
}

// conflict-free 16-byte shared-memory loads
__global__ void probe_lds128(float *out, int iters) {
    __shared__ float4 buf[2048];
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) buf[i] = make_float4(i, i + 1, i + 2, i + 3);
    __syncthreads();
    float4 acc[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) acc[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned idx = threadIdx.x;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < kChains; ++j) {
            const float4 v = buf[(idx + 256u * j) & 2047u];
            acc[j].x += v.x;
            acc[j].y += v.y;
            acc[j].z += v.z;
            acc[j].w += v.w;
        }
        idx += 32u;
    }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += acc[j].x + acc[j].y + acc[j].z + acc[j].w;
    if (s == 123.456f) out[0] = s;
}

}  // namespace

extern "C" {

// which: 0 FP32 FMA, 1 FP64 FMA, 2 __sincosf, 3 LDS.128.
// Returns 0 and *ops_per_s (FMA, sincos or 16-byte loads per second) and
// *ms, or a CUDA error code.
__attribute__((visibility("default"))) int sarbp_probe(int which, int iters, double *ops_per_s, float *ms) {
    if (!ops_per_s || !ms || iters <= 0 || which < 0 || which > 3) return -1;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256;
    void *scratch = nullptr;
    cudaError_t e = cudaMalloc(&scratch, 64);
    if (e != cudaSuccess) return static_cast<int>(e);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int rep = 0; rep < 2; ++rep) {  // first launch warms up
        cudaEventRecord(a);
        switch (which) {
            case 0: probe_ffma<<<blocks, threads>>>(static_cast<float *>(scratch), iters); break;
            case 1: probe_dfma<<<blocks, threads>>>(static_cast<double *>(scratch), iters); break;
            case 2: probe_sincos<<<blocks, threads>>>(static_cast<float *>(scratch), iters); break;
            default: probe_lds128<<<blocks, threads>>>(static_cast<float *>(scratch), iters); break;
        }
        cudaEventRecord(b);
    }
    e = cudaEventSynchronize(b);
    float t = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(scratch);
    if (e != cudaSuccess) return static_cast<int>(e);
    *ms = t;
    *ops_per_s = static_cast<double>(blocks) * threads * kChains * static_cast<double>(iters) / (t * 1e-3);
    return 0;
}

}  // extern "C"
