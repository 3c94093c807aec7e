// bp_mixed.cu -- mixed-precision forward backprojection for sm_100a.
//
// Replaces the reference kernel backprojection_loop
// (src/gpuBackProjection/cuda_sar_focusing/cuda_BackProjectionKernels.cuh:33-93)
// and its CPU twin computeDifferentialRangeAndPhaseCorrections
// (src/cpuBackProjection/cpuBackProjection.hpp:49-93):
//     img[q] += lerp(rc_p, bin(dR)) * exp(+j 4 pi f0_p dR / c),
//     dR = |a_p - x_q| - R0_p,  gate rmin < dR < rmax,
//     bracket [floor(bin), floor(bin)+1]  (CPU/MATLAB semantics, not the
//     GPU kernel's roundf bracket, cuda_BackProjectionKernels.cuh:68-74).
//
// Design (one CTA = one pixel tile of (8*MX) x 64 pixels of one z-slice,
// 256 threads, each thread MX rows x 2 adjacent columns):
//  * per (tile, pulse), warp 0 computes the geometry record in FP64 (tile
//    centre range, unit vector, phase and bin offsets reduced mod 1) and
//    issues one cp.async.bulk copy of the pulse's range-bin window (the bins
//    any pixel of the tile can touch, a conservative +-|tile half-diagonal|)
//    into shared memory; two stages, PB pulses per stage, one mbarrier each;
//  * range profiles live in HBM as pair entries {rc[b], rc[b+1]-rc[b]}
//    (float4) so each pixel-pulse needs one 16-byte shared-memory load and
//    two FMAs for the linear interpolation;
//  * per pixel-pulse all arithmetic is FP32: the differential range is
//    (Rc - R0) - u.d + g with the FP64 per-tile part carried as revolution
//    and bin offsets, g = e (h + t hr) the far-field remainder (exact
//    sqrt form for near-field pulses), phase reduced mod 1 before
//    __sincosf, floor/fraction of the bin by a round-down add;
//  * complex64 results leave as float4 stores of two adjacent pixels.
#include <cstdint>

#include "bp_common.cuh"
#include "sarbp_internal.h"

namespace sarbp {
namespace {

constexpr int kThreads = 256;
constexpr int kTY = 64;
constexpr float kRoundMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kRoundMagicBits = 0x4B400000;

__device__ __forceinline__ PulseGeo make_geo(const BpLaunch &L, int p, double cx, double cy, double cz) {
    PulseGeo g;
    g.flags = 0;
    const double ax = L.ax[p], ay = L.ay[p], az = L.az[p], r0 = L.r0[p], f0 = L.f0[p];
    const double vx = ax - cx, vy = ay - cy, vz = az - cz;
    const double rc = sqrt(vx * vx + vy * vy + vz * vz);
    const double inv = 1.0 / rc;
    const double ux = vx * inv, uy = vy * inv;
    const double D = rc - r0;
    const double k = 2.0 * f0 / kClight;
    const double bc = D * L.lambda + L.half_nfft;
    const double kd = k * D;
    if (!(isfinite(bc) && isfinite(kd) && isfinite(ux) && isfinite(uy) && rc > 0.0 && fabs(bc) < 1.0e9 &&
          fabs(kd) < 1.0e12)) {
        atomicOr(L.err, ERRBIT_NOT_FINITE);
        return g;
    }
    const int ws = static_cast<int>(floor(bc)) - L.W;
    g.ws = ws;
    g.B0 = bc - static_cast<double>(ws);
    g.A = frac_rev(kd);
    const double al = frac_rev(-k * ux * L.dx);
    const double be = frac_rev(-k * uy * L.dy);
    g.alpha = al;
    g.beta = be;
    g.gam = -L.lambda * ux * L.dx;
    g.eta = -L.lambda * uy * L.dy;
    g.a8 = static_cast<float>(frac_rev(8.0 * al));
    g.b1 = static_cast<float>(be);
    g.g8 = static_cast<float>(8.0 * g.gam);
    g.e1 = static_cast<float>(g.eta);
    g.tx = static_cast<float>(ux * L.dx);
    g.ty = static_cast<float>(uy * L.dy);
    g.h = static_cast<float>(0.5 * inv);
    g.hr = static_cast<float>(0.5 * inv * inv);
    g.kappa = static_cast<float>(k);
    g.rc = static_cast<float>(rc);
    g.lo = static_cast<float>(-ws);
    g.hi = static_cast<float>(L.nfft - 1 - ws);
    int flags = 0;
    if (!(ws + L.wsize - 2 <= 0 || ws + 1 >= L.nfft - 1)) flags |= PG_ACTIVE;
    if (!(ws >= 0 && ws + L.wsize <= L.nfft)) flags |= PG_GATE;
    if (rc < L.near_hd16 || rc * rc * rc < k * L.near_coef) flags |= PG_NEAR;
    g.flags = flags;
    return g;
}

// Warp 0: geometry of block b's pulses into geo_s, then one bulk copy per
// active pulse of its window into win_s, all completing on `bar`.
template <int PB>
__device__ __forceinline__ void produce_block(const BpLaunch &L, int b, PulseGeo *geo_s, float4 *win_s,
                                              uint32_t bar, int lane, double cx, double cy, double cz) {
    const int p = b * PB + lane;
    uint32_t bytes = 0;
    const float4 *src = nullptr;
    if (lane < PB) {
        PulseGeo g;
        g.flags = 0;
        if (p < L.np) g = make_geo(L, p, cx, cy, cz);
        if (g.flags & PG_ACTIVE) {
            bytes = static_cast<uint32_t>(L.wsize) * 16u;
            src = static_cast<const float4 *>(L.pairs) + static_cast<long long>(p) * L.row_stride + L.guard + g.ws;
        }
        geo_s[lane] = g;
    }
    const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
    if (lane == 0) mbar_arrive_expect_tx(bar, total);
    __syncwarp();
    if (bytes) bulk_copy_g2s(smem_addr(win_s + lane * L.wsize), src, bytes, bar);
}

template <int MX, bool GATE, bool NEAR, bool CHECKED>
__device__ __forceinline__ void accumulate_pulse(const PulseGeo &g, const float4 *__restrict__ w,
                                                 const float4 *zero, int i0, int j0, float lam,
                                                 const float (&d2)[MX][2], float (&acc_re)[MX][2],
                                                 float (&acc_im)[MX][2], int wsize, unsigned *err) {
    const double pd = fma(static_cast<double>(i0), g.alpha, fma(static_cast<double>(j0), g.beta, g.A));
    const float P00 = static_cast<float>(pd - rint(pd));
    const float B00 = static_cast<float>(fma(static_cast<double>(i0), g.gam, fma(static_cast<double>(j0), g.eta, g.B0)));
    const float t00 = fmaf(static_cast<float>(i0), g.tx, static_cast<float>(j0) * g.ty);
    const float tx8 = 8.0f * g.tx;
#pragma unroll
    for (int k = 0; k < MX; ++k) {
        const float Pk = fmaf(static_cast<float>(k), g.a8, P00);
        const float Bk = fmaf(static_cast<float>(k), g.g8, B00);
        const float tk = fmaf(static_cast<float>(k), tx8, t00);
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const float t = l ? tk + g.ty : tk;
            const float Pb = l ? Pk + g.b1 : Pk;
            const float Bb = l ? Bk + g.e1 : Bk;
            const float e = fmaf(-t, t, d2[k][l]);
            float gg;
            if (NEAR) {
                const float sv = g.rc - t;
                gg = e / (sv + sqrtf(fmaf(sv, sv, e)));
            } else {
                gg = e * fmaf(t, g.hr, g.h);
            }
            const float P = fmaf(g.kappa, gg, Pb);
            const float B = fmaf(lam, gg, Bb);
            const float f = P - rintf(P);
            float sn, cs;
            __sincosf(6.28318530717958647692f * f, &sn, &cs);
            const float y = __fadd_rd(B, kRoundMagic);
            const float a = B - (y - kRoundMagic);
            const int idx = __float_as_int(y) - kRoundMagicBits;
            const float4 *src = w + idx;
            if (GATE) {
                const bool valid = (B > g.lo) && (B < g.hi);
                src = valid ? src : zero;
            }
            if (CHECKED) {
                if (static_cast<unsigned>(idx) > static_cast<unsigned>(wsize - 2)) {
                    atomicOr(err, ERRBIT_BOUNDS);
                    src = zero;
                }
            }
            const float4 v = *src;
            const float re = fmaf(a, v.z, v.x);
            const float im = fmaf(a, v.w, v.y);
            acc_re[k][l] = fmaf(re, cs, fmaf(-im, sn, acc_re[k][l]));
            acc_im[k][l] = fmaf(re, sn, fmaf(im, cs, acc_im[k][l]));
        }
    }
}

template <int MX, int PB, bool CHECKED>
__global__ void __launch_bounds__(kThreads, 2) bp_mixed_kernel(const BpLaunch L) {
    constexpr int TX = 8 * MX;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    float4 *zero = reinterpret_cast<float4 *>(smem + 16);
    PulseGeo *geo = reinterpret_cast<PulseGeo *>(smem + 32);
    float4 *win = reinterpret_cast<float4 *>(smem + 32 + 2 * PB * sizeof(PulseGeo));
    const int wsize = L.wsize;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ty0 = blockIdx.x * kTY, tx0 = blockIdx.y * TX, iz = blockIdx.z;
    const double cx = L.left + static_cast<double>(tx0 + TX / 2) * L.dx;
    const double cy = L.bottom + static_cast<double>(ty0 + kTY / 2) * L.dy;
    const double cz = L.zlow + static_cast<double>(iz) * L.dz;
    const int i0 = warp - TX / 2;
    const int j0 = 2 * lane - kTY / 2;
    const float lam = static_cast<float>(L.lambda);

    float d2[MX][2], acc_re[MX][2], acc_im[MX][2];
    {
        const float dxf = static_cast<float>(L.dx), dyf = static_cast<float>(L.dy);
#pragma unroll
        for (int k = 0; k < MX; ++k)
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                const float di = static_cast<float>(i0 + 8 * k) * dxf;
                const float dj = static_cast<float>(j0 + l) * dyf;
                d2[k][l] = fmaf(di, di, dj * dj);
                acc_re[k][l] = 0.0f;
                acc_im[k][l] = 0.0f;
            }
    }

    const uint32_t bar_base = smem_addr(&bars[0]);  // stage s barrier at bar_base + 8*s
    if (threadIdx.x == 0) {
        mbar_init(bar_base, 1);
        mbar_init(bar_base + 8, 1);
        *zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        fence_mbar_init();
    }
    __syncthreads();

    const int nblocks = (L.np + PB - 1) / PB;
    if (warp == 0 && nblocks > 0) produce_block<PB>(L, 0, geo, win, bar_base, lane, cx, cy, cz);
    __syncthreads();

    int last_issued = 0;
    bool timed_out = false;
    for (int b = 0; b < nblocks; ++b) {
        const int s = b & 1;
        if (warp == 0 && b + 1 < nblocks) {
            produce_block<PB>(L, b + 1, geo + (s ^ 1) * PB, win + (s ^ 1) * PB * wsize, bar_base + 8 * (s ^ 1), lane, cx,
                              cy, cz);
            last_issued = b + 1;
        }
        const bool ok = mbar_wait_bounded(bar_base + 8 * s, (b >> 1) & 1, L.err);
        if (ok) {
            const int nq = min(PB, L.np - b * PB);
            for (int q = 0; q < nq; ++q) {
                const PulseGeo &g = geo[s * PB + q];
                const int flags = g.flags;
                if (!(flags & PG_ACTIVE)) continue;
                const float4 *w = win + (s * PB + q) * wsize;
                if (flags & PG_NEAR)
                    accumulate_pulse<MX, true, true, CHECKED>(g, w, zero, i0, j0, lam, d2, acc_re, acc_im, wsize,
                                                              L.err);
                else if (flags & PG_GATE)
                    accumulate_pulse<MX, true, false, CHECKED>(g, w, zero, i0, j0, lam, d2, acc_re, acc_im,
                                                               wsize, L.err);
                else
                    accumulate_pulse<MX, false, false, CHECKED>(g, w, zero, i0, j0, lam, d2, acc_re, acc_im,
                                                                wsize, L.err);
            }
        }
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
    }
    if (timed_out) {
        // let the copies already issued for the other stage land before the
        // CTA's shared memory goes away (again bounded)
        if (threadIdx.x == 0 && last_issued > 0) mbar_wait_bounded(bar_base + 8 * (last_issued & 1), (last_issued >> 1) & 1, L.err);
        return;
    }

    float2 *img = static_cast<float2 *>(L.img);
#pragma unroll
    for (int k = 0; k < MX; ++k) {
        const int row = tx0 + warp + 8 * k;
        const int col = ty0 + 2 * lane;
        if (row >= L.nx || col >= L.ny) continue;
        const long long o = (static_cast<long long>(iz) * L.nx + row) * L.ny + col;
        if (L.vec_store && col + 1 < L.ny) {
            float4 v = make_float4(acc_re[k][0], acc_im[k][0], acc_re[k][1], acc_im[k][1]);
            float4 *dst = reinterpret_cast<float4 *>(img + o);
            if (L.accumulate) {
                const float4 old = *dst;
                v.x += old.x;
                v.y += old.y;
                v.z += old.z;
                v.w += old.w;
            }
            *dst = v;
        } else {
            float2 v0 = make_float2(acc_re[k][0], acc_im[k][0]);
            if (L.accumulate) {
                const float2 old = img[o];
                v0.x += old.x;
                v0.y += old.y;
            }
            img[o] = v0;
            if (col + 1 < L.ny) {
                float2 v1 = make_float2(acc_re[k][1], acc_im[k][1]);
                if (L.accumulate) {
                    const float2 old = img[o + 1];
                    v1.x += old.x;
                    v1.y += old.y;
                }
                img[o + 1] = v1;
            }
        }
    }
}

template <int MX, int PB>
cudaError_t launch_mx_pb(const BpLaunch &L, bool checked, size_t smem, cudaStream_t s) {
    constexpr int TX = 8 * MX;
    const dim3 grid((L.ny + kTY - 1) / kTY, (L.nx + TX - 1) / TX, L.nz);
    auto kern = checked ? bp_mixed_kernel<MX, PB, true> : bp_mixed_kernel<MX, PB, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    kern<<<grid, kThreads, smem, s>>>(L);
    return cudaGetLastError();
}

}  // namespace

size_t bp_mixed_smem_bytes(const TileConfig &tc, int wsize) {
    return 32 + 2 * static_cast<size_t>(tc.pb) * sizeof(PulseGeo) +
           2 * static_cast<size_t>(tc.pb) * static_cast<size_t>(wsize) * 16;
}

cudaError_t launch_bp_mixed(const BpLaunch &L, const TileConfig &tc, bool checked, size_t smem, cudaStream_t s) {
#define SARBP_MIXED_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_) return launch_mx_pb<MX_, PB_>(L, checked, smem, s);
    SARBP_MIXED_CASE(4, 4)
    SARBP_MIXED_CASE(4, 8)
    SARBP_MIXED_CASE(4, 16)
    SARBP_MIXED_CASE(2, 4)
    SARBP_MIXED_CASE(2, 8)
    SARBP_MIXED_CASE(2, 16)
    SARBP_MIXED_CASE(1, 8)
    SARBP_MIXED_CASE(1, 16)
#undef SARBP_MIXED_CASE
    return cudaErrorInvalidValue;
}

}  // namespace sarbp
