// bp_tile.cuh -- the (tile, pulse) machinery shared by the mixed-precision
// forward and adjoint backprojection kernels: tile constants, the FP64
// geometry record of one pulse relative to one pixel tile, the per-warp
// producer that writes records and issues the window bulk copies, and the
// shared-memory load of one pair entry.  See bp_mixed.cu for the design.
#pragma once

#include <cstdint>

#include "bp_common.cuh"
#include "sarbp_internal.h"

namespace sarbp {
namespace tile {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTY = 64;
constexpr float kRoundMagic = 12582912.0f;  // 1.5 * 2^23: adding it rounds to an integer
constexpr uint32_t kRoundMagicBits = 0x4B400000u;
constexpr double kTwoPi = 6.283185307179586476925286766559;

__device__ __forceinline__ PulseGeo make_geo(const BpLaunch &L, int p, long long goff, double cx, double cy,
                                             double cz) {
    PulseGeo g;
    g.flags = 0;
    const long long gi = goff + p;  // geometry of hypothesis goff / np
    const double ax = L.ax[gi], ay = L.ay[gi], az = L.az[gi], r0 = L.r0[gi], f0 = L.f0[gi];
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
    const double al = frac_rev(-k * ux * L.dx);
    const double be = frac_rev(-k * uy * L.dy);
    g.A = frac_rev(kd);
    g.alpha = al;
    g.beta = be;
    g.B0 = bc - static_cast<double>(ws);
    g.gam = -L.lambda * ux * L.dx;
    g.eta = -L.lambda * uy * L.dy;
    g.a8r = static_cast<float>(kTwoPi * frac_rev(8.0 * al));
    g.b1r = static_cast<float>(kTwoPi * be);
    g.g8 = static_cast<float>(8.0 * g.gam);
    g.e1 = static_cast<float>(g.eta);
    g.tx = static_cast<float>(ux * L.dx);
    g.ty = static_cast<float>(uy * L.dy);
    g.h = static_cast<float>(0.5 * inv);
    g.hr = static_cast<float>(0.5 * inv * inv);
    g.kr = static_cast<float>(kTwoPi * k);
    g.rc = static_cast<float>(rc);
    g.lo = static_cast<float>(-ws);
    g.hi = static_cast<float>(L.nfft - 1 - ws);
    g.ws = ws;
    g.ux = static_cast<float>(ux);
    g.uy = static_cast<float>(uy);
    g.uz = static_cast<float>(vz * inv);
    g.rinv = static_cast<float>(inv);
    int flags = 0;
    if (!(ws + L.wsize - 2 <= 0 || ws + 1 >= L.nfft - 1)) flags |= PG_ACTIVE;
    if (!(ws >= 0 && ws + L.wsize <= L.nfft)) flags |= PG_GATE;
    if (rc < L.near_hd16 || rc * rc * rc < k * L.near_coef) flags |= PG_NEAR;
    g.flags = flags;
    return g;
}

// Pulse slots of block b handled by this warp (slot q = warp, warp + 8, ...):
// lane 0 writes the geometry record and either arrives with the window's byte
// count and issues its bulk copy, or just arrives (inactive / past the end).
template <int PB>
__device__ __forceinline__ void produce_slots(const BpLaunch &L, int b, PulseGeo *geo_s, uint32_t win_s,
                                              uint32_t bar, int warp, int lane, double cx, double cy, double cz,
                                              long long goff = 0) {
    if (lane != 0) return;
    for (int q = warp; q < PB; q += kWarps) {
        const int p = b * PB + q;
        PulseGeo g;
        g.flags = 0;
        if (p < L.np) g = make_geo(L, p, goff, cx, cy, cz);
        geo_s[q] = g;
        if (g.flags & PG_ACTIVE) {
            const uint32_t bytes = static_cast<uint32_t>(L.wsize) * 16u;
            const float4 *src =
                static_cast<const float4 *>(L.pairs) + static_cast<long long>(p) * L.row_stride + L.guard + g.ws;
            mbar_arrive_expect_tx(bar, bytes);
            bulk_copy_g2s(win_s + static_cast<uint32_t>(q) * bytes, src, bytes, bar);
        } else {
            mbar_arrive(bar);
        }
    }
}

__device__ __forceinline__ float4 lds128(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(addr));
    return v;
}

__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }

}  // namespace tile
}  // namespace sarbp
