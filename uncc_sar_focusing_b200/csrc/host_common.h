// host_common.h -- host-side helpers shared by the plan (api.cu) and batch
// (batch.cu) entry points: status mapping, device guard, descriptor checks,
// grid axes, window geometry and the range-compression factors.
#pragma once

#include <atomic>
#include <cmath>
#include <cuda_runtime.h>
#include <cufft.h>
#include <nvtx3/nvToolsExt.h>
#include <vector>

#include "bp_common.cuh"
#include "sarbp_internal.h"

namespace sarbp {
namespace host {

inline int from_cuda(cudaError_t e) {
    if (e == cudaSuccess) return SARBP_OK;
    if (e == cudaErrorMemoryAllocation) return SARBP_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SARBP_ERR_NO_DEVICE;
    return SARBP_ERR_CUDA;
}

// Failure injection for device allocations (sarbp_test_fail_device_alloc):
// the number of allocations to let through before one fails, -1: off.
inline std::atomic<long long> g_alloc_countdown{-1};

// cudaMalloc, or cudaErrorMemoryAllocation (nothing allocated) when the
// injection countdown reaches this allocation.
inline cudaError_t device_malloc(void **p, size_t bytes) {
    long long c = g_alloc_countdown.load();
    while (c >= 0) {
        if (g_alloc_countdown.compare_exchange_weak(c, c - 1)) {
            if (c == 0) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
            break;
        }
    }
    return cudaMalloc(p, bytes);
}

// NVTX range over an entry point's host work (enqueueing, copies, waits), so
// that Nsight Systems timelines and ncu's --nvtx filters can name the calls;
// without a tool attached a push/pop costs a few nanoseconds.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

inline int from_cufft(cufftResult r) {
    if (r == CUFFT_SUCCESS) return SARBP_OK;
    if (r == CUFFT_ALLOC_FAILED) return SARBP_ERR_OUT_OF_MEMORY;
    return SARBP_ERR_CUFFT;
}

#define SARBP_TRY(call)                  \
    do {                                 \
        const int st_ = (call);          \
        if (st_ != SARBP_OK) return st_; \
    } while (0)

#define SARBP_TRY_CUDA(call)                         \
    do {                                             \
        const cudaError_t e_ = (call);               \
        if (e_ != cudaSuccess) {                     \
            cudaGetLastError();                      \
            return ::sarbp::host::from_cuda(e_);     \
        }                                            \
    } while (0)

// Makes a device current for the duration of a call and restores the
// caller's device afterwards.
struct DeviceGuard {
    int prev = -1;
    bool changed = false;
    cudaError_t status = cudaSuccess;
    explicit DeviceGuard(int dev) {
        status = cudaGetDevice(&prev);
        if (status == cudaSuccess && prev != dev) {
            status = cudaSetDevice(dev);
            changed = status == cudaSuccess;
        }
    }
    ~DeviceGuard() {
        if (changed) cudaSetDevice(prev);
    }
};

inline bool finite_nonneg(double v) { return std::isfinite(v) && v >= 0.0; }

inline int validate_desc(const sarbp_plan_desc *d) {
    if (!d) return SARBP_ERR_NULL_POINTER;
    const sarbp_grid &g = d->grid;
    if (d->num_range_samples < 1 || d->num_pulses < 1 || d->nfft < 2 || d->nfft < d->num_range_samples ||
        d->nfft > (1 << 24))
        return SARBP_ERR_INVALID_ARGUMENT;
    if (!(std::isfinite(d->max_wr) && d->max_wr > 0.0)) return SARBP_ERR_INVALID_ARGUMENT;
    if (g.nx < 1 || g.ny < 1 || g.nz < 1 || g.nx > (1 << 20) || g.ny > (1 << 20) || g.nz > 65535)
        return SARBP_ERR_INVALID_ARGUMENT;
    if (!(std::isfinite(g.x0) && std::isfinite(g.y0) && std::isfinite(g.z0) && finite_nonneg(g.wx) &&
          finite_nonneg(g.wy) && finite_nonneg(g.wz)))
        return SARBP_ERR_INVALID_ARGUMENT;
    if (d->precision != SARBP_PRECISION_MIXED && d->precision != SARBP_PRECISION_FP64)
        return SARBP_ERR_INVALID_ARGUMENT;
    if (d->window != SARBP_WINDOW_NONE && d->window != SARBP_WINDOW_HAMMING && d->window != SARBP_WINDOW_TAYLOR)
        return SARBP_ERR_INVALID_ARGUMENT;
    const double samples = static_cast<double>(d->num_pulses) * static_cast<double>(d->nfft);
    if (samples > 4.0e9) return SARBP_ERR_UNSUPPORTED;
    return SARBP_OK;
}

// First coordinate and step of a linspace axis of n points of width w
// centred on c (cpuBackProjection.hpp:55-62).
inline void axis(int n, double c, double w, double *lo, double *step) {
    if (n > 1) {
        *step = w / static_cast<double>(n - 1);
        *lo = c - 0.5 * w;
    } else {
        *step = 0.0;
        *lo = c;
    }
}

// Range-bin window of a tile of (8 mx) x 64 pixels with steps dx, dy at
// lambda bins per metre: W = ceil(lambda * half-diagonal) + 3 bins each side,
// wsize = 2W + 2 pair entries; hd the half-diagonal in metres.
inline void tile_window(double lambda, double dx, double dy, int mx, int *W, int *wsize, double *hd) {
    const double hx = 0.5 * 8.0 * mx * dx, hy = 0.5 * 64.0 * dy;
    *hd = std::sqrt(hx * hx + hy * hy);
    *W = static_cast<int>(std::ceil(lambda * *hd)) + 3;
    *wsize = 2 * (*W) + 2;
}

// Far-field test constants of the mixed kernel for a tile half-diagonal hd:
// the remainder after the e (h + t hr) expansion is <= 0.625 hd^4 / Rc^3
// metres; a pulse whose k times that exceeds 1e-7 revolutions takes the
// exact path.
inline void near_field_consts(double hd, double *near_hd16, double *near_coef) {
    *near_hd16 = 16.0 * hd;
    *near_coef = 0.625 * hd * hd * hd * hd / 1.0e-7;
}

// fac[k] = w_k / nfft * exp(+j 2 pi ((k s) mod nfft) / nfft), s = (nfft+1)/2,
// interleaved re, im: taper (Hamming or none), the 1/nfft of the inverse FFT
// and the fftshift as an input twiddle.
// Taylor window of n samples with nbar nearly constant sidelobes at sll dB
// (sll < 0), not normalised: w_k = 1 + 2 sum_{m=1}^{nbar-1} F_m cos(2 pi m x_k),
// x_k = (k - n/2 + 1/2) / n, with the coefficients of Carrara, Goodman and
// Majewski, "Spotlight Synthetic Aperture Radar" (1995), sec. on Taylor
// weighting: A = acosh(10^(-sll/20)) / pi, sigma^2 = nbar^2 / (A^2 + (nbar -
// 1/2)^2), F_m = (-1)^(m+1) prod_i (1 - m^2 / (sigma^2 (A^2 + (i - 1/2)^2)))
// / (2 prod_{i != m} (1 - m^2 / i^2)), i = 1 .. nbar-1.  This is the taper
// matlab/rangeCompress.m:11 applies as taylorwin(K, 5, -35).
inline std::vector<double> taylor_window(int n, int nbar, double sll) {
    std::vector<double> w(static_cast<size_t>(n > 0 ? n : 0), 1.0);
    if (n <= 1) return w;  // a single sample keeps unit weight
    const double A = std::acosh(std::pow(10.0, -sll / 20.0)) / M_PI;
    const double sig2 = nbar * nbar / (A * A + (nbar - 0.5) * (nbar - 0.5));
    for (int m = 1; m < nbar; ++m) {
        double num = 1.0, den = 1.0;
        for (int i = 1; i < nbar; ++i) {
            num *= 1.0 - (static_cast<double>(m) * m / sig2) / (A * A + (i - 0.5) * (i - 0.5));
            if (i != m) den *= 1.0 - static_cast<double>(m) * m / (static_cast<double>(i) * i);
        }
        const double Fm = ((m % 2) ? 1.0 : -1.0) * num / (2.0 * den);
        for (int k = 0; k < n; ++k) {
            const double x = (k - 0.5 * n + 0.5) / n;
            w[k] += 2.0 * Fm * std::cos(2.0 * M_PI * m * x);
        }
    }
    return w;
}

// Real taper w_k of a plan's window (all ones for SARBP_WINDOW_NONE).
inline std::vector<double> taper(int K, int window) {
    if (window == SARBP_WINDOW_TAYLOR) return taylor_window(K, 5, -35.0);
    std::vector<double> w(static_cast<size_t>(K), 1.0);
    if (window == SARBP_WINDOW_HAMMING && K > 1)
        for (int k = 0; k < K; ++k)
            w[k] = 0.54 - 0.46 * std::cos(2.0 * M_PI * static_cast<double>(k) / static_cast<double>(K - 1));
    return w;
}

// Per-sample complex weights c_k (interleaved): the caller's, else the taper.
inline std::vector<double> range_weights(const sarbp_plan_desc &d, const double *user) {
    const int K = d.num_range_samples;
    std::vector<double> c(2 * static_cast<size_t>(K), 0.0);
    if (user) {
        c.assign(user, user + 2 * static_cast<size_t>(K));
        return c;
    }
    const std::vector<double> w = taper(K, d.window);
    for (int k = 0; k < K; ++k) c[2 * k] = w[k];
    return c;
}

// fac[k] = c_k / nfft * exp(+j 2 pi ((k s) mod nfft) / nfft), s = (nfft+1)/2:
// weight, 1/nfft scale and the fftshift moved to the input side as a twiddle.
inline std::vector<double> range_factors(const sarbp_plan_desc &d, const double *user = nullptr) {
    const int K = d.num_range_samples, N = d.nfft;
    const long long s = (N + 1) / 2;
    const std::vector<double> c = range_weights(d, user);
    std::vector<double> fac(2 * static_cast<size_t>(K));
    for (int k = 0; k < K; ++k) {
        const long long m = (static_cast<long long>(k) * s) % N;
        const double ang = 2.0 * M_PI * static_cast<double>(m) / static_cast<double>(N);
        const double tr = std::cos(ang) / N, ti = std::sin(ang) / N;
        fac[2 * k] = c[2 * k] * tr - c[2 * k + 1] * ti;
        fac[2 * k + 1] = c[2 * k] * ti + c[2 * k + 1] * tr;
    }
    return fac;
}

inline int status_from_bits(unsigned bits) {
    if (bits & ERRBIT_TIMEOUT) return SARBP_ERR_KERNEL_TIMEOUT;
    if (bits & ERRBIT_NOT_FINITE) return SARBP_ERR_NOT_FINITE;
    if (bits & ERRBIT_BOUNDS) return SARBP_ERR_KERNEL_BOUNDS;
    return SARBP_OK;
}

}  // namespace host
}  // namespace sarbp
