// oracle/ref_gpu_harness.cu -- BENCH / TEST INFRASTRUCTURE (the reference's
// own GPU kernels as a timed baseline), not product code.
//
// Compiles the reference's GPU kernels from
// src/gpuBackProjection/cuda_sar_focusing/cuda_BackProjectionKernels.cuh where
// it lies (oracle/Makefile, output in oracle/_ref/) and launches them as
// cuda_focus_SAR_image does (cuda_sar_focusing.hpp:612-667):
//   cuifft              in-place batched C2C inverse over N_fft x Np
//                       (cuda_sar_focusing.hpp:372-399)
//   cufftNormalize_1DBatch, cufftShift_1DBatch   (cuda_BackProjectionKernels.cuh:106-135)
//   backprojection_loop<float> on 16 x 16 blocks (cuda_sar_focusing.hpp:627-667)
// with range_vec, minRange and maxRange built as cuda_sar_focusing.hpp:570-590
// builds them (float).  Left out, because they are not the kernels: the
// per-call device allocation and copies, cufftPlan1d per call and the
// cudaDeviceReset of the reference's host function.  The reference FFTs
// N_fft samples per pulse in place, so the caller passes the phase history
// already tapered and zero-padded to N_fft per pulse (the reference C++ has
// neither a window nor a pad).
//
// Guard: backprojection_loop brackets a sample with roundf(dR_idx) - 1 and
// roundf(dR_idx); for dR_idx < 0.5 (a pixel within half a bin of the swath's
// lower edge) that reads index -1.  ref_gpu_focus computes, in double, every
// pulse's smallest range to the image rectangle and refuses (status -2) any
// scene in which some pixel-pulse comes within 2 bins of that edge, before it
// touches the GPU, so every read the kernel makes stays inside its buffers.
#define CUDAFUNCTION __host__ __device__

#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "cuda_BackProjectionKernels.cuh"

namespace {

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    template <typename T>
    T *as() const {
        return static_cast<T *>(p);
    }
};

// smallest distance from antenna (x, y, z) to the image rectangle at z = 0,
// the kernel's pixel model (cuda_BackProjectionKernels.cuh:55-63)
double min_range(double x, double y, double z, double left, double right, double bottom, double top) {
    const double cx = std::min(std::max(x, left), right);
    const double cy = std::min(std::max(y, bottom), top);
    return std::sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy) + z * z);
}

}  // namespace

extern "C" {

// ph: complex64 [np][nfft] (re, im), host, tapered and zero-padded.
// ax..f0: float [np], host.  img: complex64 [nx][ny] (x-major), host.
// Returns 0, -1 (CUDA / cuFFT error), -2 (guard: scene reaches the swath's
// lower edge), -3 (bad argument).  fft_ms / bp_ms: mean per repetition
// (CUDA events on the legacy stream, after one untimed repetition).
int ref_gpu_focus(const float *ph, int nfft, int np, const float *ax, const float *ay, const float *az,
                  const float *r0, const float *f0, double max_wy, int nx, int ny, double x0, double y0, double wx,
                  double wy, int reps, float *img, double *fft_ms, double *bp_ms) {
    if (!ph || !ax || !ay || !az || !r0 || !f0 || !img || nfft < 2 || np < 1 || nx < 2 || ny < 2 || reps < 1 ||
        !(max_wy > 0.0))
        return -3;
    using T = float;
    SAR_ImageFormationParameters<T> params;
    params.N_fft = nfft;
    params.N_x_pix = nx;
    params.N_y_pix = ny;
    params.x0_m = static_cast<T>(x0);
    params.y0_m = static_cast<T>(y0);
    params.Wx_m = static_cast<T>(wx);
    params.Wy_m = static_cast<T>(wy);
    params.max_Wy_m = static_cast<T>(max_wy);

    // range bins and window limits, as the reference host code builds them
    std::vector<T> range_vec(nfft);
    T minRange = INFINITY, maxRange = -INFINITY;
    for (int i = 0; i < nfft; ++i) {
        const T r = ((float)i / nfft - 0.5f) * params.max_Wy_m;
        range_vec[i] = r;
        minRange = std::min(minRange, r);
        maxRange = std::max(maxRange, r);
    }
    const T dx = params.Wx_m / (params.N_x_pix - 1);
    const T dy = params.Wy_m / (params.N_y_pix - 1);
    const T left = params.x0_m - params.Wx_m / 2;
    const T bottom = params.y0_m - params.Wy_m / 2;

    // guard (see the header): no pixel-pulse within 2 bins of the lower edge
    const double right = left + static_cast<double>(dx) * (nx - 1), top = bottom + static_cast<double>(dy) * (ny - 1);
    for (int p = 0; p < np; ++p) {
        const double dr = min_range(ax[p], ay[p], az[p], left, right, bottom, top) - r0[p];
        const double idx = (dr / params.max_Wy_m + 0.5) * nfft;
        if (!(idx >= 2.0)) return -2;
    }

    const size_t n_ph = static_cast<size_t>(nfft) * np, n_img = static_cast<size_t>(nx) * ny;
    DevBuf d_pristine, d_sample, d_ax, d_ay, d_az, d_r0, d_f0, d_params, d_rv, d_img;
    if (cudaMalloc(&d_pristine.p, n_ph * sizeof(cufftComplex)) != cudaSuccess ||
        cudaMalloc(&d_sample.p, n_ph * sizeof(cufftComplex)) != cudaSuccess ||
        cudaMalloc(&d_ax.p, np * sizeof(T)) != cudaSuccess || cudaMalloc(&d_ay.p, np * sizeof(T)) != cudaSuccess ||
        cudaMalloc(&d_az.p, np * sizeof(T)) != cudaSuccess || cudaMalloc(&d_r0.p, np * sizeof(T)) != cudaSuccess ||
        cudaMalloc(&d_f0.p, np * sizeof(T)) != cudaSuccess ||
        cudaMalloc(&d_params.p, sizeof(params)) != cudaSuccess ||
        cudaMalloc(&d_rv.p, nfft * sizeof(T)) != cudaSuccess ||
        cudaMalloc(&d_img.p, n_img * sizeof(cufftComplex)) != cudaSuccess)
        return -1;
    if (cudaMemcpy(d_pristine.p, ph, n_ph * sizeof(cufftComplex), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_ax.p, ax, np * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_ay.p, ay, np * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_az.p, az, np * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_r0.p, r0, np * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_f0.p, f0, np * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_params.p, &params, sizeof(params), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_rv.p, range_vec.data(), nfft * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        return -1;
    cufftHandle plan;
    if (cufftPlan1d(&plan, nfft, CUFFT_C2C, np) != CUFFT_SUCCESS) return -1;
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    const dim3 block(16, 16, 1);
    const dim3 grid(static_cast<unsigned>(std::ceil(static_cast<float>(nx) / 16)),
                    static_cast<unsigned>(std::ceil(static_cast<float>(ny) / 16)));
    int status = 0;
    double fsum = 0.0, bsum = 0.0;
    for (int r = 0; r <= reps && status == 0; ++r) {
        // fresh input for the in-place transform (untimed)
        if (cudaMemcpy(d_sample.p, d_pristine.p, n_ph * sizeof(cufftComplex), cudaMemcpyDeviceToDevice) !=
            cudaSuccess) {
            status = -1;
            break;
        }
        cudaEventRecord(e0);
        if (cufftExecC2C(plan, d_sample.as<cufftComplex>(), d_sample.as<cufftComplex>(), CUFFT_INVERSE) !=
            CUFFT_SUCCESS) {
            status = -1;
            break;
        }
        cufftNormalize_1DBatch(d_sample.as<cufftComplex>(), nfft, np);
        cufftShift_1DBatch<cufftComplex>(d_sample.as<cufftComplex>(), nfft, np);
        cudaEventRecord(e1);
        backprojection_loop<T><<<grid, block>>>(d_sample.as<cufftComplex>(), nfft, np, dx, dy, left, bottom,
                                                 minRange, maxRange, d_ax.as<T>(), d_ay.as<T>(), d_az.as<T>(),
                                                 d_r0.as<T>(), d_f0.as<T>(),
                                                 d_params.as<SAR_ImageFormationParameters<T>>(), d_rv.as<T>(),
                                                 d_img.as<cufftComplex>());
        cudaEventRecord(e2);
        if (cudaEventSynchronize(e2) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            status = -1;
            break;
        }
        float a = 0.0f, b = 0.0f;
        cudaEventElapsedTime(&a, e0, e1);
        cudaEventElapsedTime(&b, e1, e2);
        if (r > 0) {
            fsum += a;
            bsum += b;
        }
    }
    if (status == 0 &&
        cudaMemcpy(img, d_img.p, n_img * sizeof(cufftComplex), cudaMemcpyDeviceToHost) != cudaSuccess)
        status = -1;
    cufftDestroy(plan);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    if (status == 0) {
        if (fft_ms) *fft_ms = fsum / reps;
        if (bp_ms) *bp_ms = bsum / reps;
    }
    return status;
}

}  // extern "C"
