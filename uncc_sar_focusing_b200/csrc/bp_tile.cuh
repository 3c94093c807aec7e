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

// ---- work split over (tile, pulse-stage) units ---------------------------
//
// Tiles are numbered t = (zz * tiles_x + tx) * tiles_y + ty (zz = hypothesis
// * nz + z-slice) and unit u = t * stages + stage.  CTA c of G takes units
// [lo(c), lo(c+1)), lo(c) = floor(c U / G): with G = tiles every CTA gets
// exactly one tile; with G = the resident CTA count every SM gets the same
// number of pulse stages, whatever the tile count (no partial last wave).
struct TileGrid {
    int tiles_y, tiles_x;
    long long tiles;
    int stages;
    long long units;
};

__host__ __device__ __forceinline__ TileGrid tile_grid(const BpLaunch &L, int TX, int PB) {
    TileGrid g;
    g.tiles_y = (L.ny + kTY - 1) / kTY;
    g.tiles_x = (L.nx + TX - 1) / TX;
    g.tiles = static_cast<long long>(g.tiles_y) * g.tiles_x * L.nz * L.nhyp;
    g.stages = (L.np + PB - 1) / PB;
    g.units = g.tiles * g.stages;
    return g;
}

__host__ __device__ __forceinline__ long long sk_lo(long long c, long long units, long long G) {
    return c * units / G;
}

// The CTA whose range holds unit u: the largest c with lo(c) <= u.
__device__ __forceinline__ long long sk_owner(long long u, long long units, long long G) {
    long long c = u * G / units;
    while (c + 1 < G && sk_lo(c + 1, units, G) <= u) ++c;
    while (c > 0 && sk_lo(c, units, G) > u) --c;
    return c;
}

// Partial-sum slot of CTA c's segment of the tile whose first unit is
// `first`: its first segment (the one holding unit lo(c)) uses slot 2c, a
// later one slot 2c + 1.
__device__ __forceinline__ long long sk_slot(long long c, long long first, long long units, long long G) {
    return sk_lo(c, units, G) >= first ? 2 * c : 2 * c + 1;
}

// Pixel origin (row tx0, column ty0) and hypothesis-major slice zz of tile t.
__device__ __forceinline__ void tile_origin(const TileGrid &g, long long t, int TX, int &tx0, int &ty0, int &zz) {
    const long long r = t / g.tiles_y;
    ty0 = static_cast<int>(t - r * g.tiles_y) * kTY;
    const long long q = r / g.tiles_x;
    tx0 = static_cast<int>(r - q * g.tiles_x) * TX;
    zz = static_cast<int>(q);
}

// Position of a unit, advanced one unit at a time without divisions: stage
// b of the tile at tile column ty, tile row tx, z-slice iz of hypothesis hyp.
struct UnitCursor {
    int b, ty, tx, iz, hyp;

    __device__ __forceinline__ void init(const TileGrid &g, const BpLaunch &L, long long u) {
        const long long t = u / g.stages;
        b = static_cast<int>(u - t * g.stages);
        const long long r = t / g.tiles_y;
        ty = static_cast<int>(t - r * g.tiles_y);
        const long long q = r / g.tiles_x;
        tx = static_cast<int>(r - q * g.tiles_x);
        hyp = static_cast<int>(q / L.nz);
        iz = static_cast<int>(q - static_cast<long long>(hyp) * L.nz);
    }
    __device__ __forceinline__ void advance(const TileGrid &g, const BpLaunch &L) {
        if (++b < g.stages) return;
        b = 0;
        if (++ty < g.tiles_y) return;
        ty = 0;
        if (++tx < g.tiles_x) return;
        tx = 0;
        if (++iz < L.nz) return;
        iz = 0;
        ++hyp;
    }
};

#ifndef SARBP_GEO_RSQ
#define SARBP_GEO_RSQ 1
#endif

// 1/sqrt(s) in double by Newton-Raphson for the reciprocal square root,
// y <- y (3 - s y^2) / 2, from the single-precision hardware estimate (about
// 2^-22 relative): each step squares the relative error, two reach double
// precision.  In place of a double sqrt and a double division on the
// producing lane, whose instruction sequences are several times longer.
__device__ __forceinline__ double rsqrt_newton(double s) {
    double y = static_cast<double>(rsqrtf(static_cast<float>(s)));
    const double hs = 0.5 * s;
    y = y * fma(-hs * y, y, 1.5);
    y = y * fma(-hs * y, y, 1.5);
    return y;
}

// tx_half: half the tile's rows (its columns are 64: 32 each side)
__device__ __forceinline__ PulseGeo make_geo(const BpLaunch &L, int p, long long goff, double cx, double cy,
                                             double cz, int tx_half) {
    PulseGeo g;
    g.flags = 0;
    const long long gi = goff + p;  // geometry of hypothesis goff / np
    const double ax = L.ax[gi], ay = L.ay[gi], az = L.az[gi], r0 = L.r0[gi], f0 = L.f0[gi];
    const double vx = ax - cx, vy = ay - cy, vz = az - cz;
#if SARBP_GEO_RSQ
    const double s2 = vx * vx + vy * vy + vz * vz;
    const double inv = rsqrt_newton(s2);
    const double rc = s2 * inv;
    constexpr double kTwoOverC = 2.0 / kClight;
    const double k = f0 * kTwoOverC;
#else
    const double rc = sqrt(vx * vx + vy * vy + vz * vz);
    const double inv = 1.0 / rc;
    const double k = 2.0 * f0 / kClight;
#endif
    const double ux = vx * inv, uy = vy * inv;
    const double D = rc - r0;
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
    g.b32r = static_cast<float>(kTwoPi * frac_rev(32.0 * be));
    g.g8 = static_cast<float>(8.0 * g.gam);
    g.e32 = static_cast<float>(32.0 * g.eta);
    g.tx = static_cast<float>(ux * L.dx);
    g.ty = static_cast<float>(uy * L.dy);
    g.h = static_cast<float>(0.5 * inv);
    g.hr = static_cast<float>(0.5 * inv * inv);
    g.kr = static_cast<float>(kTwoPi * k);
    g.rc = static_cast<float>(rc);
    // validity bounds of the window-centred bin (bin - ws - W)
    g.lo = static_cast<float>(-ws - L.W);
    g.hi = static_cast<float>(L.nfft - 1 - ws - L.W);
    g.ws = ws;
    g.ux = static_cast<float>(ux);
    g.uy = static_cast<float>(uy);
    g.uz = static_cast<float>(vz * inv);
    g.rinv = static_cast<float>(inv);

    int flags = 0;
    if (rc < L.near_hd16 || rc * rc * rc < k * L.near_coef) flags |= PG_NEAR;
    // Tight window: a pixel (i, j) of the tile has bin - bc = i gam + j eta +
    // lambda g with 0 <= g <= hd^2 / (2 (Rc - hd)) (hd the tile
    // half-diagonal), |i| <= tx_half, |j| <= 32, so its floor(bin) and
    // floor(bin) + 1 lie within floor(bc) -/+ (ceil(span) + 1): wp =
    // ceil(span) + 3, at most W (the triangle-inequality bound |bin - bc| <=
    // lambda hd the full window is sized for).  Near-field pulses keep W.
    int wp = L.W;
    if (!(flags & PG_NEAR)) {
        const double hd = L.near_hd16 * (1.0 / 16.0);
        const double span = fabs(g.gam) * tx_half + fabs(g.eta) * 32.0 + L.lambda * hd * hd / (2.0 * (rc - hd));
        if (span < L.W) {
            const int w = static_cast<int>(ceil(span)) + 3;
            wp = w < L.W ? w : L.W;
        }
    }
    g.wp = wp;
    // the part of the window this pulse copies: bins [wsp, wsp + 2 wp + 2)
    const int wsp = ws + (L.W - wp), wsz = 2 * wp + 2;
    if (!(wsp + wsz - 2 <= 0 || wsp + 1 >= L.nfft - 1)) flags |= PG_ACTIVE;
    if (!(wsp >= 0 && wsp + wsz <= L.nfft)) flags |= PG_GATE;
    g.flags = flags;
    return g;
}

// Pulse slots of block b handled by this warp (slot q = warp, warp + 8, ...):
// lane 0 writes the geometry record and either arrives with the window's byte
// count and issues its bulk copy, or just arrives (inactive / past the end).
// Per-(tile, pulse) base tables of the mixed kernels (forward and adjoint),
// kBaseEntries float4 words: row entries 0..7, one per warp, for
// i0 = warp - TX/2: (2 pi frac(A + i0 alpha), B0 + i0 gam, i0 tx, -kr), then
// 32 floats, one per lane, for j0 = lane - 32 (a lane's pixels are columns
// lane and lane + 32 of the tile): the column phase 2 pi frac(j0 beta).  The
// phase parts are reduced modulo one revolution in FP64; a thread's phase
// base is row + column, its bin and projection bases row + j0 eta and
// row + j0 ty, formed in FP32 from the record (eta = e32 / 32 exactly).
constexpr int kBaseEntries = kWarps + 32 / 4;

// Records (and base tables when base_s != nullptr) and window copies of
// stage b into one buffer.  Warp w produces slots w, w + 8, ...: lane 0
// computes the FP64 record (or lanes 0..7 move the prefetched pre-pass
// record into place), the warp's lanes fill the base tables from it, then
// lane 0 issues the window's bulk copy (or a plain arrival), whose release
// on the stage's mbarrier also publishes the record and the tables
// (__syncwarp orders the other lanes' stores before it).
// Pre-pass records (BpLaunch::geo_tab) of pulse stage b of the tile whose
// record row is `rec` into a staging slot of shared memory, asynchronously
// (cp.async, 16 bytes by each of lanes 0..7 of warp q for slot q): issued a
// stage ahead of produce_slots, which waits for them.
template <int PB>
__device__ __forceinline__ void prefetch_records(const BpLaunch &L, const PulseGeo *rec, int b, PulseGeo *stg,
                                                 int warp, int lane) {
    for (int q = warp; q < PB; q += kWarps) {
        const int p = b * PB + q;
        if (p < L.np && lane < 8) {
            const uint32_t dst = smem_addr(reinterpret_cast<const float4 *>(stg + q) + lane);
            const float4 *src = reinterpret_cast<const float4 *>(rec + p) + lane;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Base tables of one (tile, pulse) from its record's FP64 steps (every lane
// of the warp writes its column entry, lanes 0..7 the row entries; the row
// entries carry -kr in their fourth word, so the forward kernel's
// consumers read it with the row part).
__device__ __forceinline__ void write_base_table(float4 *tab, int lane, int tx_half, int W, double A, double alpha,
                                                 double beta, double B0, double gam, float tx, float kr) {
    const int j0 = lane - kTY / 2;
    const double pc = static_cast<double>(j0) * beta;
    reinterpret_cast<float *>(tab + kWarps)[lane] = static_cast<float>(kTwoPi * (pc - rint(pc)));
    if (lane < kWarps) {
        const int i0 = lane - tx_half;
        const double pr = fma(static_cast<double>(i0), alpha, A);
        tab[lane] = make_float4(static_cast<float>(kTwoPi * (pr - rint(pr))),
                                static_cast<float>(fma(static_cast<double>(i0), gam, B0 - W)),
                                static_cast<float>(i0) * tx, -kr);
    }
}

// Lane 0: the window copy of pulse p (slot q) into the stage buffer, or a
// plain arrival when the tile's window misses the pulse's range bins.  The
// test hook L.drop_pulse expects that pulse's bytes without copying them.
__device__ __forceinline__ void issue_window(const BpLaunch &L, int p, int q, int flags, int wp, int ws,
                                             uint32_t win_s, uint32_t bar) {
    if (flags & PG_ACTIVE) {
        // the pulse's tight window, at its place inside the slot's full one
        const int off = L.W - wp;
        const uint32_t bytes = static_cast<uint32_t>(2 * wp + 2) * 16u;
        if (p == L.drop_pulse) {
            mbar_arrive_expect_tx(bar, bytes);
            return;
        }
        const float4 *src =
            static_cast<const float4 *>(L.pairs) + static_cast<long long>(p) * L.row_stride + L.guard + ws + off;
        mbar_arrive_expect_tx(bar, bytes);
        bulk_copy_g2s(win_s + (static_cast<uint32_t>(q) * static_cast<uint32_t>(L.wsize) + static_cast<uint32_t>(off)) *
                                  16u,
                      src, bytes, bar);
    } else {
        mbar_arrive(bar);
    }
}

// Records, base tables and window copies of stage b (see below).  stg: the
// stage's prefetched records (prefetch_records), or nullptr: lane 0 computes
// them (make_geo).
template <int PB>
__device__ __forceinline__ void produce_slots(const BpLaunch &L, int b, PulseGeo *geo_s, float4 *base_s,
                                              uint32_t win_s, uint32_t bar, int warp, int lane, int tx_half,
                                              double cx, double cy, double cz, long long goff = 0,
                                              const PulseGeo *stg = nullptr) {
    if (stg) {
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
        for (int q = warp; q < PB; q += kWarps) {
            const int p = b * PB + q;
            const bool valid = p < L.np;
            // lanes 0..7 move the record's 16-byte words into the stage's
            // record slot (zeros past the last pulse: flags 0); every lane
            // reads the steps of the tables itself (broadcast loads)
            const float4 *rec = reinterpret_cast<const float4 *>(stg + q);
            if (lane < 8)
                reinterpret_cast<float4 *>(geo_s + q)[lane] = valid ? rec[lane] : make_float4(0.f, 0.f, 0.f, 0.f);
            if (base_s) {
                double2 d0 = make_double2(0.0, 0.0), d1 = d0;
                double gam = 0.0;
                float tx = 0.0f, kr = 0.0f;
                if (valid) {
                    const double2 *rd = reinterpret_cast<const double2 *>(stg + q);
                    d0 = rd[0];  // A, alpha
                    d1 = rd[1];  // beta, B0
                    gam = stg[q].gam;
                    tx = stg[q].tx;
                    kr = stg[q].kr;
                }
                write_base_table(base_s + q * kBaseEntries, lane, tx_half, L.W, d0.x, d0.y, d1.x, d1.y, gam, tx, kr);
            }
            __syncwarp();
            if (lane == 0 && valid) {
                const int4 f = *reinterpret_cast<const int4 *>(&stg[q].ws);  // ws, flags, wp, pad
                issue_window(L, p, q, f.y, f.z, f.x, win_s, bar);
            } else if (lane == 0) {
                mbar_arrive(bar);
            }
        }
        return;
    }
    for (int q = warp; q < PB; q += kWarps) {
        const int p = b * PB + q;
        PulseGeo g = {};
        if (lane == 0 && p < L.np) g = make_geo(L, p, goff, cx, cy, cz, tx_half);
        if (base_s) {
            const unsigned full = 0xffffffffu;
            const double A = __shfl_sync(full, g.A, 0), alpha = __shfl_sync(full, g.alpha, 0);
            const double beta = __shfl_sync(full, g.beta, 0), B0 = __shfl_sync(full, g.B0, 0);
            const double gam = __shfl_sync(full, g.gam, 0);
            const float tx = __shfl_sync(full, g.tx, 0), kr = __shfl_sync(full, g.kr, 0);
            write_base_table(base_s + q * kBaseEntries, lane, tx_half, L.W, A, alpha, beta, B0, gam, tx, kr);
            __syncwarp();
        }
        if (lane != 0) continue;
        geo_s[q] = g;
        issue_window(L, p, q, g.flags, g.wp, g.ws, win_s, bar);
    }
}

__device__ __forceinline__ float4 lds128(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(addr));
    return v;
}

__device__ __forceinline__ void sts64(uint32_t addr, float x, float y) {
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(x), "f"(y) : "memory");
}

__device__ __forceinline__ void sts128(uint32_t addr, float x, float y, float z, float w) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(x), "f"(y), "f"(z), "f"(w) : "memory");
}

__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }

// Intercept form of the windows: entry n of a pulse's window holds
// {v_n, v'_n} (v'_n = v_(n+1) - v_n); rewritten in place to
// {v_n - (n - W) v'_n, v'_n}, a pixel whose window-centred bin is
// B = bin - ws - W (floor(B) + W = n) interpolates
//     v(B) = v_n + (B + W - n) v'_n = c_n + B v'_n
// with one fused multiply-add and no fraction.  Warp `warp` rewrites the
// slots it produced (q = warp, warp + 8, ...) of one stage buffer once their
// copies have landed (bounded wait on the buffer's mbarrier; a timeout sets
// the error bit and leaves the windows as they are).  The barrier that
// follows publishes them.
// ZFORM (the adjoint, which needs only Z(B) = v'(B) + j nu v(B), nu = kr /
// lambda radians per bin): the entry becomes {Zc, Zv} with Zc = v'_n + j nu
// c_n and Zv = j nu v'_n, so that Z(B) = Zc + B Zv is again one fused
// multiply-add per component and the pixel loop neither interpolates v nor
// forms Z.
template <int PB, bool ZFORM = false>
__device__ __forceinline__ bool intercept_slots(const PulseGeo *geo_s, uint32_t win_s, uint32_t bar, uint32_t parity,
                                                int wsize, int W, int warp, int lane, unsigned *err,
                                                float inv_lam = 0.0f) {
    if (warp >= PB) return true;
    if (!mbar_wait_bounded(bar, parity, err)) return false;
    for (int q = warp; q < PB; q += kWarps) {
        if (!(geo_s[q].flags & PG_ACTIVE)) continue;
        const uint32_t w = win_s + static_cast<uint32_t>(q) * static_cast<uint32_t>(wsize) * 16u;
        // the entries the pulse's tight window copied
        const int wp = geo_s[q].wp;
        const float nu = ZFORM ? geo_s[q].kr * inv_lam : 0.0f;
        for (int n = W - wp + lane; n < W + wp + 2; n += 32) {
            const uint32_t a = w + static_cast<uint32_t>(n) * 16u;
            const float4 e = lds128(a);
            const float m = static_cast<float>(n - W);
            const float cr = fmaf(-m, e.z, e.x), ci = fmaf(-m, e.w, e.y);
            if (ZFORM)
                sts128(a, fmaf(-nu, ci, e.z), fmaf(nu, cr, e.w), -nu * e.w, nu * e.z);
            else
                sts64(a, cr, ci);
        }
    }
    // these generic-proxy stores precede the next bulk copy (async proxy) into
    // the same buffer, issued after the CTA barrier
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    return true;
}

}  // namespace tile
}  // namespace sarbp
