// mf.cu -- matched-filter focusing (sarbp_matched_filter).
//
// The reference's second focusing algorithm: computeDifferentialRangeAndPhase
// CorrectionsMF / run_mf (src/cpuBackProjection/cpuBackProjection.hpp:165-228)
// and matlab/mfBasic.m:73-89:
//     img[q] = sum_p sum_k w_k ph_p[k] exp(+j 4 pi (f0_p + k dF) dR_pq / c).
// With a_p = exp(+j 4 pi f0_p dR / c) and z_p = exp(+j 4 pi dF dR / c) the
// inner sum is a_p * P_p(z_p), P_p the polynomial with coefficients w_k ph_p[k],
// evaluated by Horner's rule: K complex multiply-adds per pixel-pulse instead
// of K complex exponentials.  Both phases are reduced modulo one revolution
// in FP64 before sincospi; Horner and accumulation run in FP32 (MIXED) or
// FP64.  One thread per pixel; each pulse's tapered samples are staged in
// shared memory by the CTA in chunks and read as broadcasts.  K times the work
// of backprojection: a reference for it on small images and the reference's
// own alternative, not a fast path.
#include <cstdint>

#include "bp_common.cuh"
#include "sarbp_internal.h"

namespace sarbp {
namespace {

constexpr int kMfThreads = 256;
constexpr int kMfChunk = 2048;  // samples staged per pass

template <typename R>
struct C2 {
    R x, y;
};

template <typename R>
__global__ void __launch_bounds__(kMfThreads) mf_kernel(const float2 *__restrict__ ph, const double *__restrict__ win,
                                                       MfLaunch M) {
    __shared__ C2<R> s[kMfChunk];
    const long long npix = static_cast<long long>(M.nx) * M.ny * M.nz;
    const long long q = blockIdx.x * static_cast<long long>(kMfThreads) + threadIdx.x;
    const bool live = q < npix;
    const int iy = static_cast<int>(q % M.ny);
    const long long r = q / M.ny;
    const int ix = static_cast<int>(r % M.nx);
    const int iz = static_cast<int>(r / M.nx);
    const double x = M.left + ix * M.dx, y = M.bottom + iy * M.dy, z = M.zlow + iz * M.dz;
    R acc_re = 0, acc_im = 0;
    for (int p = 0; p < M.np; ++p) {
        const double ex = M.ax[p] - x, ey = M.ay[p] - y, ez = M.az[p] - z;
        const double dR = sqrt(ex * ex + ey * ey + ez * ez) - M.r0[p];
        // revolutions: 2 f0 dR / c and 2 dF dR / c, reduced mod 1
        double a0 = 2.0 * M.f0[p] * dR / kClight, th = 2.0 * M.df * dR / kClight;
        a0 -= rint(a0);
        th -= rint(th);
        double sa, ca, sz, cz;
        sincospi(2.0 * a0, &sa, &ca);
        sincospi(2.0 * th, &sz, &cz);
        const R zr = static_cast<R>(cz), zi = static_cast<R>(sz);
        // P(z) = sum_k c_k z^k by Horner from the highest power, in chunks
        R hr = 0, hi = 0;
        for (int c1 = M.K; c1 > 0; c1 -= kMfChunk) {
            const int c0 = c1 > kMfChunk ? c1 - kMfChunk : 0;
            __syncthreads();
            for (int k = c0 + threadIdx.x; k < c1; k += kMfThreads) {
                const float2 v = ph[static_cast<long long>(p) * M.K + k];
                const double wr = win ? win[2 * k] : 1.0, wi = win ? win[2 * k + 1] : 0.0;
                s[k - c0].x = static_cast<R>(wr * v.x - wi * v.y);
                s[k - c0].y = static_cast<R>(wr * v.y + wi * v.x);
            }
            __syncthreads();
            for (int k = c1 - 1; k >= c0; --k) {
                const C2<R> v = s[k - c0];
                const R nr = hr * zr - hi * zi + v.x;
                const R ni = hr * zi + hi * zr + v.y;
                hr = nr;
                hi = ni;
            }
        }
        const R ar = static_cast<R>(ca), ai = static_cast<R>(sa);
        acc_re += hr * ar - hi * ai;
        acc_im += hr * ai + hi * ar;
    }
    if (!live) return;
    if (sizeof(R) == 8) {
        double2 *img = static_cast<double2 *>(M.img);
        img[q] = make_double2(static_cast<double>(acc_re), static_cast<double>(acc_im));
    } else {
        float2 *img = static_cast<float2 *>(M.img);
        img[q] = make_float2(static_cast<float>(acc_re), static_cast<float>(acc_im));
    }
}

}  // namespace

cudaError_t launch_mf(const void *ph, const double *win, const MfLaunch &M, bool fp64, cudaStream_t s) {
    const long long npix = static_cast<long long>(M.nx) * M.ny * M.nz;
    const long long blocks = (npix + kMfThreads - 1) / kMfThreads;
    if (blocks < 1 || blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    if (fp64)
        mf_kernel<double><<<static_cast<unsigned>(blocks), kMfThreads, 0, s>>>(static_cast<const float2 *>(ph), win, M);
    else
        mf_kernel<float><<<static_cast<unsigned>(blocks), kMfThreads, 0, s>>>(static_cast<const float2 *>(ph), win, M);
    return cudaGetLastError();
}

}  // namespace sarbp
