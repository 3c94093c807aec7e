// bp_adjoint.cu -- gradient of an image loss with respect to the per-pulse
// geometry (antenna position and slant range), for sm_100a.
//
// The forward operator is img_q = sum_p v_p(b_pq) exp(j phi_pq) with
// b = lambda dR + nfft/2, phi = kr dR (kr = 2 pi 2 f0 / c) and
// dR = |a_p - x_q| - R0_p (bp_mixed.cu).  For a real loss with upstream
// gradient G_q = dL/dRe(img_q) + j dL/dIm(img_q):
//     dL/d(dR_pq) = s_pq = Re(conj(G_q) (lambda v'_p(b) + j kr v_p(b)) exp(j phi))
//     dL/da_p = sum_q s_pq u_pq (u_pq the unit vector pixel -> antenna),
//     dL/dR0_p = -sum_q s_pq.
// v'_p(b) is the slope of the linear interpolation, rc[b+1] - rc[b], which the
// pair entries already hold.  Nothing per pixel-pulse is stored: the kernel
// recomputes the geometry of every (tile, pulse) exactly as the forward kernel
// does (same records, base tables, shared-memory windows and FP32 per-pixel
// arithmetic).
//
// Per pixel the kernel holds G_q as |G_q| exp(j psi_q), so that with
// nu = kr / lambda and Z = v' + j nu v
//     s_pq = lambda |G_q| Re(Z exp(j (phi - psi_q))):
// the conjugate product with G becomes a phase offset folded into the sine /
// cosine argument, and lambda leaves the pixel loop.  The producing warps
// rewrite each window entry to {v' + j nu c, j nu v'} (the intercept form's
// c = v_n - (n - W) v'_n), so Z at a pixel's window-centred bin B is one
// fused multiply-add per component, Z = Zc + B Zv.  Writing d = (i dx, j dy, 0)
// for a pixel's offset from the tile centre (i, j its row and column offsets)
// and Rc/R_q = 1 + t_eff/Rc, d/R_q = d_eff/Rc (far field: t_eff = u.d =
// i ux dx + j uy dy, d_eff = d; near field: the exact ratios),
//     sum_q s u_q = u (E0 + Et/Rc) - (dx Ei, dy Ej, 0)/Rc
// with E0 = sum s, Ei = sum s i (Rc/R), Ej = sum s j (Rc/R) and Et = sum s t_eff.
// In the far field t_eff is linear in (i, j), so a thread accumulates only
// sum |G| Re(..) per column and sum row * |G| Re(..) over its pixels (two
// paired FP32 accumulators) and Et follows from Ei and Ej.
//
// Work split: the (tile, pulse-stage) units are divided over the resident
// CTAs in contiguous ranges (bp_tile.cuh); every unit writes the per-tile
// partial gradients of its own pulses, so no fix-up pass is needed.  Stages
// are up to 8 pulses deep (record production and the stage barrier are paid
// per stage); the warp reduces the 4 sums of each group of up to 4 pulses with
// one transposed butterfly (each step halves the values a lane holds), the
// CTA adds its 8 warps, and
// adjoint_reduce_kernel sums the tiles per pulse in double, in a fixed order.
#include <algorithm>
#include <cstdint>

#include "bp_common.cuh"
#include "bp_tile.cuh"
#include "sarbp_internal.h"

namespace sarbp {
namespace {

using namespace tile;

// Far field: T += |G| s~ per column (x: l = 0, y: l = 1; s~ = Re(Z exp(j
// theta))) and, after each of the thread's rows k = 0..MX-2, V += T, so that
// sum_k k |G| s~ = (MX - 1) T - V without per-row weights.
// Near field: E += (s^, s^ r i, s^ r j, s^ Rc (r - 1)), s^ = |G| s~, r = Rc/R.
template <int MX, bool GATE, bool NEAR>
__device__ __forceinline__ void adjoint_pulse(const PulseGeo &g, const float4 *base, uint32_t w_addr,
                                              uint32_t zero_addr, int warp, int lane, float lam,
                                              const float2 (&nd2)[MX], const float2 (&npsi)[MX],
                                              const float2 (&gm)[MX], float i0f, float j0f, int W,
                                              float2 &T, float2 &V, float4 &E) {
    const float4 c0 = *reinterpret_cast<const float4 *>(&g.a8r);  // a8r, b32r, g8, e32
    const float4 c1 = *reinterpret_cast<const float4 *>(&g.tx);   // tx, ty, h, hr
    const float4 c2 = *reinterpret_cast<const float4 *>(&g.kr);   // kr, rc, lo, hi
    const float4 rowv = base[warp];
    const float P00 = rowv.x + reinterpret_cast<const float *>(base + kWarps)[lane];
    const float B00 = fmaf(j0f, c0.w * (1.0f / 32.0f), rowv.y);
    const float t00 = fmaf(j0f, c1.y, rowv.z);
    float2 t2 = make_float2(t00, fmaf(32.0f, c1.y, t00));  // second pixel: 32 columns on
    float2 Pb = make_float2(P00, P00 + c0.y);
    float2 Bb = make_float2(B00, B00 + c0.w);
    const float2 TX8 = splat(8.0f * c1.x), A8 = splat(c0.x), G8 = splat(c0.z);
    const float2 HR = splat(c1.w), H = splat(c1.z), NKR = splat(-c2.x), NLAM = splat(-lam);
    const float2 MAGIC = splat(kRoundMagic);
    // B is the window-centred bin (entry floor(B) + W, intercept form)
    const uint32_t w_adj = w_addr + (static_cast<uint32_t>(W) - kRoundMagicBits) * 16u;
#pragma unroll
    for (int k = 0; k < MX; ++k) {
        if (k > 0) {
            t2 = __fadd2_rn(t2, TX8);
            Pb = __fadd2_rn(Pb, A8);
            Bb = __fadd2_rn(Bb, G8);
        }
        float2 ng;
        float2 rr = make_float2(1.0f, 1.0f);  // Rc / R_q (near field only)
        if (NEAR) {
            const float e0 = -fmaf(t2.x, t2.x, nd2[k].x), e1 = -fmaf(t2.y, t2.y, nd2[k].y);
            const float s0 = c2.y - t2.x, s1 = c2.y - t2.y;
            const float g0 = e0 / (s0 + sqrtf(fmaf(s0, s0, e0))), g1 = e1 / (s1 + sqrtf(fmaf(s1, s1, e1)));
            ng = make_float2(-g0, -g1);
            rr = make_float2(c2.y / (s0 + g0), c2.y / (s1 + g1));
        } else {
            const float2 ne = __ffma2_rn(t2, t2, nd2[k]);
            ng = __fmul2_rn(ne, __ffma2_rn(t2, HR, H));
        }
        // theta = phi - psi, bin B and its floor split as in the forward kernel
        const float2 TH = __ffma2_rn(NKR, ng, __fadd2_rn(Pb, npsi[k]));
        const float2 B = __ffma2_rn(NLAM, ng, Bb);
        const float2 y = __fadd2_rd(B, MAGIC);
        float2 ZR, NZI, CS, SN;  // the pair's Re Z, -Im Z and rotations
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const float Tl = l ? TH.y : TH.x;
            const float yl = l ? y.y : y.x;
            const float Bl = l ? B.y : B.x;
            float sn, cs;
            __sincosf(Tl, &sn, &cs);
            uint32_t addr = __float_as_uint(yl) * 16u + w_adj;
            if (GATE) {
                const bool valid = (Bl > c2.z) && (Bl < c2.w);
                addr = valid ? addr : zero_addr;
            }
            // Z-form entry {Zc, Zv}: Z(B) = v' + j nu v(B) = Zc + B Zv
            const float4 v = lds128(addr);
            const float zr = fmaf(Bl, v.z, v.x);
            const float nzi = fmaf(-Bl, v.w, -v.y);
            if (l) {
                ZR.y = zr;
                NZI.y = nzi;
                CS.y = cs;
                SN.y = sn;
            } else {
                ZR.x = zr;
                NZI.x = nzi;
                CS.x = cs;
                SN.x = sn;
            }
        }
        // s~ = Re(Z exp(j theta)) of the pair as paired FP32
        const float2 st = __ffma2_rn(ZR, CS, __fmul2_rn(NZI, SN));
        if (NEAR) {
            const float2 sh = __fmul2_rn(gm[k], st);
            const float ik = i0f + static_cast<float>(8 * k);
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                const float s = l ? sh.y : sh.x;
                const float r = l ? rr.y : rr.x;
                const float sr = s * r;
                E.x += s;
                E.y = fmaf(sr, ik, E.y);
                E.z = fmaf(sr, j0f + static_cast<float>((kTY / 2) * l), E.z);
                E.w = fmaf(s, c2.y * (r - 1.0f), E.w);
            }
        } else {
            T = __ffma2_rn(gm[k], st, T);
            if (k < MX - 1) V = __fadd2_rn(V, T);
        }
    }
}

// The warp sums of N values (N = 4, 8, 16 or 32) at once: each step swaps
// half of a lane's values with the partner lane and adds, so N - 1 + 5 -
// log2(N) shuffles give lane L the sum of value (L >> (5 - log2 N)).
template <int N>
__device__ __forceinline__ float warp_reduce_scatter(float (&v)[N], int lane) {
    static_assert(N == 4 || N == 8 || N == 16 || N == 32, "value count");
    int o = 16;
#pragma unroll
    for (int h = N / 2; h >= 1; h >>= 1, o >>= 1) {
        const bool upper = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const float send = upper ? v[i] : v[i + h];
            const float keep = upper ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    float r = v[0];
#pragma unroll
    for (; o >= 1; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    return r;
}

template <int N>
struct Log2 {
    static constexpr int value = N <= 1 ? 0 : 1 + Log2<N / 2>::value;
};
template <>
struct Log2<1> {
    static constexpr int value = 0;
};

template <int MX, int PB>
__global__ void __launch_bounds__(kThreads, 2)
    bp_adjoint_kernel(const __grid_constant__ BpLaunch L, const float2 *__restrict__ grad,
                      float4 *__restrict__ partials) {
    constexpr int TX = 8 * MX;
    constexpr int RG = PB < 4 ? PB : 4;  // pulses per warp reduction
    constexpr int NV = 4 * RG;           // its sums: (E0, Ei, Ej, Et) per pulse
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    float4 *zero = reinterpret_cast<float4 *>(smem + 16);
    PulseGeo *geo = reinterpret_cast<PulseGeo *>(smem + 32);
    float4 *bases = reinterpret_cast<float4 *>(smem + 32 + 2 * PB * sizeof(PulseGeo));
    float *red = reinterpret_cast<float *>(smem + 32 + 2 * PB * (sizeof(PulseGeo) + kBaseEntries * sizeof(float4)));
    unsigned char *win_ptr = smem + 32 + 2 * PB * (sizeof(PulseGeo) + kBaseEntries * sizeof(float4)) +
                             2 * kWarps * 4 * PB * sizeof(float);
    const uint32_t win_addr = smem_addr(win_ptr);
    const uint32_t zero_addr = smem_addr(zero);
    const int wsize = L.wsize;
    const uint32_t pulse_bytes = static_cast<uint32_t>(wsize) * 16u;
    const uint32_t buf_bytes = static_cast<uint32_t>(PB) * pulse_bytes;

    const TileGrid tg = tile_grid(L, TX, PB);
    const long long G = gridDim.x;
    const long long lo = sk_lo(blockIdx.x, tg.units, G);
    const int n = static_cast<int>(sk_lo(blockIdx.x + 1, tg.units, G) - lo);
    if (n <= 0) return;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = warp - TX / 2;
    const int j0 = lane - kTY / 2;  // columns lane and lane + 32 of the tile
    const float i0f = static_cast<float>(i0), j0f = static_cast<float>(j0);
    const float lam = static_cast<float>(L.lambda), inv_lam = static_cast<float>(1.0 / L.lambda);
    const float dxf = static_cast<float>(L.dx), dyf = static_cast<float>(L.dy);

    float2 nd2[MX];  // -|d|^2 of the thread's pixel pairs
#pragma unroll
    for (int k = 0; k < MX; ++k) {
        const float di = static_cast<float>(i0 + 8 * k) * dxf;
        const float dj0 = j0f * dyf, dj1 = static_cast<float>(j0 + kTY / 2) * dyf;
        nd2[k] = make_float2(-fmaf(di, di, dj0 * dj0), -fmaf(di, di, dj1 * dj1));
    }

    UnitCursor cc, pc;  // consumer at unit i, producer at unit i + 1
    cc.init(tg, L, lo);
    pc = cc;

    // the consumer tile's upstream gradient as -psi and |G| per pixel pair
    float2 npsi[MX], gm[MX];
    auto load_tile = [&]() {
        const int tx0 = cc.tx * TX, ty0 = cc.ty * kTY;
#pragma unroll
        for (int k = 0; k < MX; ++k) {
            const int row = tx0 + warp + 8 * k;
            float ps[2], mg[2];
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                const int col = ty0 + lane + (kTY / 2) * l;
                const float2 q = (row < L.nx && col < L.ny)
                                     ? grad[(static_cast<long long>(cc.iz) * L.nx + row) * L.ny + col]
                                     : make_float2(0.0f, 0.0f);
                ps[l] = -atan2f(q.y, q.x);
                mg[l] = sqrtf(fmaf(q.x, q.x, q.y * q.y));
            }
            npsi[k] = make_float2(ps[0], ps[1]);
            gm[k] = make_float2(mg[0], mg[1]);
        }
    };
    load_tile();

    const uint32_t bar_base = smem_addr(&bars[0]);  // buffer s barrier at bar_base + 8*s
    if (threadIdx.x == 0) {
        mbar_init(bar_base, PB);
        mbar_init(bar_base + 8, PB);
        *zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        fence_mbar_init();
    }
    __syncthreads();

    // Pre-pass records (BpLaunch::geo_tab, [tile][pulse]): the producing
    // warps copy them from a staging ring filled a stage ahead, after the
    // two stage buffers' windows.
    const bool pregeo = L.geo_tab != nullptr;
    PulseGeo *stg = reinterpret_cast<PulseGeo *>(win_ptr + 2 * buf_bytes);
    auto prefetch = [&](const UnitCursor &u, int slot) {
        const long long t = ((static_cast<long long>(u.hyp) * L.nz + u.iz) * tg.tiles_x + u.tx) * tg.tiles_y + u.ty;
        prefetch_records<PB>(L, static_cast<const PulseGeo *>(L.geo_tab) + t * L.np, u.b, stg + slot * PB, warp,
                             lane);
    };
    // records, base tables and windows of the producer cursor's unit into
    // buffer s (every lane of the warp enters produce_slots)
    auto produce = [&](int s) {
        const double cx = L.left + static_cast<double>(pc.tx * TX + TX / 2) * L.dx;
        const double cy = L.bottom + static_cast<double>(pc.ty * kTY + kTY / 2) * L.dy;
        const double cz = L.zlow + static_cast<double>(pc.iz) * L.dz;
        produce_slots<PB>(L, pc.b, geo + s * PB, bases + s * PB * kBaseEntries, win_addr + s * buf_bytes,
                          bar_base + 8 * s, warp, lane, TX / 2, cx, cy, cz, 0, pregeo ? stg + s * PB : nullptr);
    };
    if (pregeo) {
        prefetch(pc, 0);
        if (n > 1) {
            UnitCursor nx = pc;
            nx.advance(tg, L);
            prefetch(nx, 1);
        }
    }
    produce(0);
    intercept_slots<PB, true>(geo, win_addr, bar_base, 0, L.wsize, L.W, warp, lane, L.err, inv_lam);
    __syncthreads();

    int last_issued = 0;
    for (int i = 0; i < n; ++i) {
        const int s = i & 1;
        if (i + 1 < n) {
            pc.advance(tg, L);
            produce(s ^ 1);
            last_issued = i + 1;
            // stage i + 2's records into the staging slot stage i's producer
            // read before the last barrier
            if (pregeo && i + 2 < n) {
                UnitCursor nx = pc;
                nx.advance(tg, L);
                prefetch(nx, s);
            }
        }
        const int b = cc.b;
        const bool ok = mbar_wait_bounded(bar_base + 8 * s, (i >> 1) & 1, L.err);
        const int nq = min(PB, L.np - b * PB);
        // the record fields the final sum of pulse q = threadIdx.x needs
        int rflags = 0;
        float rtx = 0.0f, rty = 0.0f, rux = 0.0f, ruy = 0.0f, ruz = 0.0f, rinv = 0.0f;
        bool fast = false;
        if (ok) {
            const int my_flags = lane < nq ? geo[s * PB + lane].flags : 0;
            const int any_f = __reduce_or_sync(0xffffffffu, my_flags);
            const int all_f = __reduce_and_sync(0xffffffffu, lane < nq ? my_flags : PG_ACTIVE);
            fast = nq == PB && (all_f & PG_ACTIVE) && !(any_f & (PG_GATE | PG_NEAR));
            if (threadIdx.x < nq) {
                const PulseGeo &g = geo[s * PB + threadIdx.x];
                rflags = g.flags;
                rtx = g.tx;
                rty = g.ty;
                rux = g.ux;
                ruy = g.uy;
                ruz = g.uz;
                rinv = g.rinv;
            }
        }
        // pulses in groups of RG: the group's 4 RG sums, then their warp sums
        // (lane L holds value L >> shift) into this stage's half of red; after
        // the stage barrier thread q adds the 8 warps for pulse q (the next
        // stage writes the other half, so one barrier per stage)
        constexpr int shift = 5 - Log2<NV>::value;
        float *red_s = red + s * (kWarps * 4 * PB);
        const uint32_t w0 = win_addr + s * buf_bytes;
#pragma unroll
        for (int gi = 0; gi < PB / RG; ++gi) {
            float v[NV];
#pragma unroll
            for (int c = 0; c < NV; ++c) v[c] = 0.0f;
            // far field: E0, Ei = i0 E0 + 8 sum k s^, Ej = j0 E0 + 32 sum_(l=1) s^, Et later
            auto far_sums = [&](int r, float2 T, float2 V) {
                const float S = T.x + T.y;
                const float Sk = fmaf(static_cast<float>(MX - 1), S, -(V.x + V.y));
                v[4 * r + 0] = S;
                v[4 * r + 1] = fmaf(i0f, S, 8.0f * Sk);
                v[4 * r + 2] = fmaf(j0f, S, static_cast<float>(kTY / 2) * T.y);
            };
            if (fast) {
#pragma unroll
                for (int r = 0; r < RG; ++r) {
                    const int q = gi * RG + r;
                    float2 T = make_float2(0.0f, 0.0f), V = make_float2(0.0f, 0.0f);
                    float4 E;
                    adjoint_pulse<MX, false, false>(geo[s * PB + q], bases + (s * PB + q) * kBaseEntries,
                                                    w0 + q * pulse_bytes, zero_addr, warp, lane, lam, nd2, npsi, gm,
                                                    i0f, j0f, L.W, T, V, E);
                    far_sums(r, T, V);
                }
            } else if (ok) {
#pragma unroll
                for (int r = 0; r < RG; ++r) {
                    const int q = gi * RG + r;
                    const PulseGeo &g = geo[s * PB + q];
                    if (q >= nq || !(g.flags & PG_ACTIVE)) continue;
                    const float4 *bq = bases + (s * PB + q) * kBaseEntries;
                    const uint32_t w = w0 + q * pulse_bytes;
                    float2 T = make_float2(0.0f, 0.0f), V = make_float2(0.0f, 0.0f);
                    float4 E = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    if (g.flags & PG_NEAR) {
                        adjoint_pulse<MX, true, true>(g, bq, w, zero_addr, warp, lane, lam, nd2, npsi, gm, i0f, j0f,
                                                      L.W, T, V, E);
                        v[4 * r + 0] = E.x;
                        v[4 * r + 1] = E.y;
                        v[4 * r + 2] = E.z;
                        v[4 * r + 3] = E.w;
                    } else {
                        adjoint_pulse<MX, true, false>(g, bq, w, zero_addr, warp, lane, lam, nd2, npsi, gm, i0f,
                                                       j0f, L.W, T, V, E);
                        far_sums(r, T, V);
                    }
                }
            }
            const float rs = warp_reduce_scatter<NV>(v, lane);
            if ((lane & ((1 << shift) - 1)) == 0) red_s[warp * 4 * PB + gi * NV + (lane >> shift)] = rs;
        }
        // the next stage's windows into intercept form, published by the barrier
        if (i + 1 < n)
            intercept_slots<PB, true>(geo + (s ^ 1) * PB, win_addr + (s ^ 1) * buf_bytes, bar_base + 8 * (s ^ 1),
                                      ((i + 1) >> 1) & 1, wsize, L.W, warp, lane, L.err, inv_lam);
        if (__syncthreads_or(!ok)) {
            // let the copies already issued for the other buffer (and the
            // record prefetches) land before the CTA's shared memory goes
            // away (again bounded)
            asm volatile("cp.async.wait_all;" ::: "memory");
            if (threadIdx.x == 0 && last_issued > i)
                mbar_wait_bounded(bar_base + 8 * (last_issued & 1), (last_issued >> 1) & 1, L.err);
            return;
        }
        if (threadIdx.x < nq) {
            const int q = threadIdx.x;
            float4 t = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                const float4 x = *reinterpret_cast<const float4 *>(red_s + w * 4 * PB + 4 * q);
                t.x += x.x;
                t.y += x.y;
                t.z += x.z;
                t.w += x.w;
            }
            float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (rflags & PG_ACTIVE) {
                // sum s u_q = u (E0 + Et/Rc) - (dx Ei, dy Ej, 0)/Rc, times lambda;
                // dL/dR0 = -lambda E0
                const float Et = (rflags & PG_NEAR) ? t.w : fmaf(rtx, t.y, rty * t.z);
                const float c = fmaf(Et, rinv, t.x);
                out.x = lam * fmaf(rux, c, -dxf * t.y * rinv);
                out.y = lam * fmaf(ruy, c, -dyf * t.z * rinv);
                out.z = lam * ruz * c;
                out.w = -lam * t.x;
            }
            const long long tile =
                ((static_cast<long long>(cc.hyp) * L.nz + cc.iz) * tg.tiles_x + cc.tx) * tg.tiles_y + cc.ty;
            partials[tile * L.np + b * PB + q] = out;
        }
        if (i + 1 < n) {
            cc.advance(tg, L);
            if (cc.b == 0) load_tile();
        }
    }
}

// out[p] = sum over tiles of partials[t][p], in double.  Block: 32 pulses
// (the lanes) x kRedWarps warps; warp w sums tiles w, w + kRedWarps, ...,
// then warp 0 adds the warps in order (a fixed order: the result does not
// depend on scheduling).  Outputs: grad_ant [3][np] (x, y, z) and
// grad_r0 [np] (may be null).
constexpr int kRedWarps = 16;

__global__ void __launch_bounds__(32 * kRedWarps)
    adjoint_reduce_kernel(const float4 *__restrict__ partials, long long ntiles, int np, double *__restrict__ grad_ant,
                          double *__restrict__ grad_r0, int accumulate) {
    __shared__ double sums[kRedWarps][4][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int p = blockIdx.x * 32 + lane;
    double gx = 0.0, gy = 0.0, gz = 0.0, gr = 0.0;
    if (p < np) {
        for (long long t = w; t < ntiles; t += kRedWarps) {
            const float4 v = partials[t * np + p];
            gx += v.x;
            gy += v.y;
            gz += v.z;
            gr += v.w;
        }
    }
    sums[w][0][lane] = gx;
    sums[w][1][lane] = gy;
    sums[w][2][lane] = gz;
    sums[w][3][lane] = gr;
    __syncthreads();
    if (w != 0 || p >= np) return;
    for (int u = 1; u < kRedWarps; ++u) {
        gx += sums[u][0][lane];
        gy += sums[u][1][lane];
        gz += sums[u][2][lane];
        gr += sums[u][3][lane];
    }
    if (accumulate) {
        grad_ant[p] += gx;
        grad_ant[np + p] += gy;
        grad_ant[2 * np + p] += gz;
        if (grad_r0) grad_r0[p] += gr;
    } else {
        grad_ant[p] = gx;
        grad_ant[np + p] = gy;
        grad_ant[2 * np + p] = gz;
        if (grad_r0) grad_r0[p] = gr;
    }
}

template <int MX, int PB>
cudaError_t launch_adj(const BpLaunch &L, const void *grad, void *partials, size_t smem, cudaStream_t s) {
    constexpr int TX = 8 * MX;
    auto kern = bp_adjoint_kernel<MX, PB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    // one CTA per resident slot, each taking a contiguous range of units
    int dev = 0, sms = 0, occ = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    const long long units = tile_grid(L, TX, PB).units;
    const long long ctas = std::min<long long>(units, static_cast<long long>(sms) * occ);
    if (ctas < 1 || ctas > 0x7fffffffLL) return cudaErrorInvalidValue;
    // the (tile, pulse) records from the pre-pass when the plan holds room
    // for them, else computed by the producing lanes
    BpLaunch La = L;
    bool pregeo = false;
    e = launch_geo_records(La, MX, &pregeo, s);
    if (e != cudaSuccess) return e;
    if (!pregeo) La.geo_tab = nullptr;
    kern<<<static_cast<unsigned>(ctas), kThreads, smem, s>>>(La, static_cast<const float2 *>(grad),
                                                              static_cast<float4 *>(partials));
    return cudaGetLastError();
}

}  // namespace

long long bp_tile_count(const BpLaunch &L, const TileConfig &tc) {
    const long long TX = 8 * tc.mx;
    return ((L.ny + 63) / 64) * ((L.nx + TX - 1) / TX) * static_cast<long long>(L.nz);
}

size_t bp_adjoint_smem_bytes(const TileConfig &tc, int wsize) {
    const size_t pb = static_cast<size_t>(tc.pb);
    return 32 + 2 * pb * (sizeof(PulseGeo) + kBaseEntries * sizeof(float4)) + 2 * kWarps * 4 * pb * sizeof(float) +
           2 * pb * static_cast<size_t>(wsize) * 16 + 2 * pb * sizeof(PulseGeo);
}

cudaError_t launch_bp_adjoint(const BpLaunch &L, const void *grad, void *partials, const TileConfig &tc, size_t smem,
                              cudaStream_t s) {
#define SARBP_ADJ_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_) return launch_adj<MX_, PB_>(L, grad, partials, smem, s);
    SARBP_ADJ_CASE(8, 8)
    SARBP_ADJ_CASE(8, 4)
    SARBP_ADJ_CASE(8, 2)  // wide windows: the stage depth halves below 4 at 64-row tiles too
    SARBP_ADJ_CASE(8, 1)
    SARBP_ADJ_CASE(4, 8)
    SARBP_ADJ_CASE(2, 8)
    SARBP_ADJ_CASE(1, 8)
    SARBP_ADJ_CASE(4, 4)
    SARBP_ADJ_CASE(4, 2)
    SARBP_ADJ_CASE(4, 1)
    SARBP_ADJ_CASE(2, 4)
    SARBP_ADJ_CASE(2, 2)
    SARBP_ADJ_CASE(2, 1)
    SARBP_ADJ_CASE(1, 4)
    SARBP_ADJ_CASE(1, 2)
    SARBP_ADJ_CASE(1, 1)
#undef SARBP_ADJ_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_adjoint_reduce(const void *partials, long long ntiles, int np, double *grad_ant, double *grad_r0,
                                  int accumulate, cudaStream_t s) {
    const int blocks = (np + 31) / 32;
    adjoint_reduce_kernel<<<blocks > 0 ? blocks : 1, 32 * kRedWarps, 0, s>>>(
        static_cast<const float4 *>(partials), ntiles, np, grad_ant, grad_r0, accumulate);
    return cudaGetLastError();
}

}  // namespace sarbp
