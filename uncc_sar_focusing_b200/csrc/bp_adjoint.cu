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
// does (same records, same shared-memory windows, same FP32 per-pixel
// arithmetic).  Per tile and pulse each thread accumulates
//     E0 = sum s,  Et = sum s t_eff,  Ex = sum s dx_eff,  Ey = sum s dy_eff
// over its pixels, where Rc/R_q = 1 + t_eff/Rc and d/R_q = d_eff/Rc (far field:
// t_eff = u.d, d_eff = d; near field: the exact ratios), so that
//     sum_q s u_q = u (E0 + Et/Rc) - (Ex, Ey, 0)/Rc.
// The CTA reduces the four sums per pulse and writes the tile's gradient;
// adjoint_reduce_kernel sums the tiles in double.
#include <cstdint>

#include "bp_common.cuh"
#include "bp_tile.cuh"
#include "sarbp_internal.h"

namespace sarbp {
namespace {

using namespace tile;

template <int MX, bool NEAR>
__device__ __forceinline__ void adjoint_pulse(const PulseGeo &g, uint32_t w_addr, uint32_t zero_addr, int i0, int j0,
                                              float lam, const float2 (&nd2)[MX], const float2 (&G)[MX][2],
                                              const float (&dxk)[MX], const float (&dyl)[2], float4 &E) {
    const double2 A_al = *reinterpret_cast<const double2 *>(&g.A);
    const double2 be_B0 = *reinterpret_cast<const double2 *>(&g.beta);
    const double2 ga_et = *reinterpret_cast<const double2 *>(&g.gam);
    const float4 c0 = *reinterpret_cast<const float4 *>(&g.a8r);  // a8r, b1r, g8, e1
    const float4 c1 = *reinterpret_cast<const float4 *>(&g.tx);   // tx, ty, h, hr
    const float4 c2 = *reinterpret_cast<const float4 *>(&g.kr);   // kr, rc, lo, hi
    const double pd = fma(static_cast<double>(i0), A_al.y, fma(static_cast<double>(j0), be_B0.x, A_al.x));
    const float P00 = static_cast<float>(kTwoPi * (pd - rint(pd)));
    const float B00 =
        static_cast<float>(fma(static_cast<double>(i0), ga_et.x, fma(static_cast<double>(j0), ga_et.y, be_B0.y)));
    const float t00 = fmaf(static_cast<float>(i0), c1.x, static_cast<float>(j0) * c1.y);
    float2 t2 = make_float2(t00, t00 + c1.y);
    float2 Pb = make_float2(P00, P00 + c0.y);
    float2 Bb = make_float2(B00, B00 + c0.w);
    const float2 TX8 = splat(8.0f * c1.x), A8 = splat(c0.x), G8 = splat(c0.z);
    const float2 HR = splat(c1.w), H = splat(c1.z), NKR = splat(-c2.x), NLAM = splat(-lam);
    const float2 MAGIC = splat(kRoundMagic), NMAGIC = splat(-kRoundMagic), NEG1 = splat(-1.0f);
    const uint32_t w_adj = w_addr - kRoundMagicBits * 16u;
    const float kr = c2.x;
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
        const float2 P = __ffma2_rn(NKR, ng, Pb);
        const float2 B = __ffma2_rn(NLAM, ng, Bb);
        const float2 y = __fadd2_rd(B, MAGIC);
        const float2 a = __ffma2_rn(__fadd2_rn(y, NMAGIC), NEG1, B);
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const float Pl = l ? P.y : P.x;
            const float Bl = l ? B.y : B.x;
            const float yl = l ? y.y : y.x;
            const float al = l ? a.y : a.x;
            float sn, cs;
            __sincosf(Pl, &sn, &cs);
            uint32_t addr = __float_as_uint(yl) * 16u + w_adj;
            const bool valid = (Bl > c2.z) && (Bl < c2.w);
            addr = valid ? addr : zero_addr;
            const float4 v = lds128(addr);
            const float vr = fmaf(al, v.z, v.x);
            const float vi = fmaf(al, v.w, v.y);
            const float2 Gq = G[k][l];
            // W = conj(G) exp(j phi)
            const float Wre = fmaf(Gq.x, cs, Gq.y * sn);
            const float Wim = fmaf(Gq.x, sn, -Gq.y * cs);
            // s = lambda Re(W v') - kr Im(W v)
            const float X = fmaf(Wre, v.z, -Wim * v.w);
            const float Y = fmaf(Wre, vi, Wim * vr);
            const float s = fmaf(lam, X, -kr * Y);
            const float tl = l ? t2.y : t2.x;
            if (NEAR) {
                const float rl = l ? rr.y : rr.x;
                // t_eff = Rc (Rc/R - 1), d_eff = d Rc/R
                E.x += s;
                E.y = fmaf(s, c2.y * (rl - 1.0f), E.y);
                E.z = fmaf(s * rl, dxk[k], E.z);
                E.w = fmaf(s * rl, dyl[l], E.w);
            } else {
                E.x += s;
                E.y = fmaf(s, tl, E.y);
                E.z = fmaf(s, dxk[k], E.z);
                E.w = fmaf(s, dyl[l], E.w);
            }
        }
    }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int MX, int PB>
__global__ void __launch_bounds__(kThreads, 2)
    bp_adjoint_kernel(const BpLaunch L, const float2 *__restrict__ grad, float4 *__restrict__ partials) {
    constexpr int TX = 8 * MX;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    float4 *zero = reinterpret_cast<float4 *>(smem + 16);
    PulseGeo *geo = reinterpret_cast<PulseGeo *>(smem + 32);
    float4 *red = reinterpret_cast<float4 *>(smem + 32 + 2 * PB * sizeof(PulseGeo));  // [kWarps][PB]
    const uint32_t win_addr = smem_addr(smem + 32 + 2 * PB * sizeof(PulseGeo) + kWarps * PB * sizeof(float4));
    const uint32_t zero_addr = smem_addr(zero);
    const int wsize = L.wsize;
    const uint32_t pulse_bytes = static_cast<uint32_t>(wsize) * 16u;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ty0 = blockIdx.x * kTY, tx0 = blockIdx.y * TX, iz = blockIdx.z;
    const long long tile = (static_cast<long long>(blockIdx.z) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    const double cx = L.left + static_cast<double>(tx0 + TX / 2) * L.dx;
    const double cy = L.bottom + static_cast<double>(ty0 + kTY / 2) * L.dy;
    const double cz = L.zlow + static_cast<double>(iz) * L.dz;
    const int i0 = warp - TX / 2;
    const int j0 = 2 * lane - kTY / 2;
    const float lam = static_cast<float>(L.lambda);

    float2 nd2[MX], G[MX][2];
    float dxk[MX], dyl[2];
    {
        const float dxf = static_cast<float>(L.dx), dyf = static_cast<float>(L.dy);
#pragma unroll
        for (int l = 0; l < 2; ++l) dyl[l] = static_cast<float>(j0 + l) * dyf;
#pragma unroll
        for (int k = 0; k < MX; ++k) {
            dxk[k] = static_cast<float>(i0 + 8 * k) * dxf;
            nd2[k] = make_float2(-fmaf(dxk[k], dxk[k], dyl[0] * dyl[0]), -fmaf(dxk[k], dxk[k], dyl[1] * dyl[1]));
            const int row = tx0 + warp + 8 * k;
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                const int col = ty0 + 2 * lane + l;
                G[k][l] = (row < L.nx && col < L.ny)
                              ? grad[(static_cast<long long>(iz) * L.nx + row) * L.ny + col]
                              : make_float2(0.0f, 0.0f);
            }
        }
    }

    const uint32_t bar_base = smem_addr(&bars[0]);
    if (threadIdx.x == 0) {
        mbar_init(bar_base, PB);
        mbar_init(bar_base + 8, PB);
        *zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        fence_mbar_init();
    }
    __syncthreads();

    const int nblocks = (L.np + PB - 1) / PB;
    if (nblocks > 0) produce_slots<PB>(L, 0, geo, nullptr, win_addr, bar_base, warp, lane, 0, cx, cy, cz);
    __syncthreads();

    int last_issued = 0;
    bool timed_out = false;
    for (int b = 0; b < nblocks; ++b) {
        const int s = b & 1;
        if (b + 1 < nblocks) {
            produce_slots<PB>(L, b + 1, geo + (s ^ 1) * PB, nullptr, win_addr + (s ^ 1) * PB * pulse_bytes,
                              bar_base + 8 * (s ^ 1), warp, lane, 0, cx, cy, cz);
            last_issued = b + 1;
        }
        const bool ok = mbar_wait_bounded(bar_base + 8 * s, (b >> 1) & 1, L.err);
        const int nq = min(PB, L.np - b * PB);
        float4 E[PB];
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            E[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (!ok || q >= nq) continue;
            const PulseGeo &g = geo[s * PB + q];
            const int flags = g.flags;
            if (!(flags & PG_ACTIVE)) continue;
            const uint32_t w = win_addr + (s * PB + q) * pulse_bytes;
            if (flags & PG_NEAR)
                adjoint_pulse<MX, true>(g, w, zero_addr, i0, j0, lam, nd2, G, dxk, dyl, E[q]);
            else
                adjoint_pulse<MX, false>(g, w, zero_addr, i0, j0, lam, nd2, G, dxk, dyl, E[q]);
        }
        // CTA sums per pulse: warp butterflies, then across the 8 warps
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            const float4 r = make_float4(warp_sum(E[q].x), warp_sum(E[q].y), warp_sum(E[q].z), warp_sum(E[q].w));
            if (lane == 0) red[warp * PB + q] = r;
        }
        __syncthreads();
        if (ok && threadIdx.x < nq) {
            const int q = threadIdx.x;
            const int p = b * PB + q;
            float4 t = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                const float4 r = red[w * PB + q];
                t.x += r.x;
                t.y += r.y;
                t.z += r.z;
                t.w += r.w;
            }
            const PulseGeo &g = geo[s * PB + q];
            float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (g.flags & PG_ACTIVE) {
                // sum s u_q = u (E0 + Et/Rc) - (Ex, Ey, 0)/Rc; dL/dR0 = -E0
                const float c = fmaf(t.y, g.rinv, t.x);
                out.x = fmaf(g.ux, c, -t.z * g.rinv);
                out.y = fmaf(g.uy, c, -t.w * g.rinv);
                out.z = g.uz * c;
                out.w = -t.x;
            }
            partials[tile * L.np + p] = out;
        }
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
    }
    if (timed_out && threadIdx.x == 0 && last_issued > 0)
        mbar_wait_bounded(bar_base + 8 * (last_issued & 1), (last_issued >> 1) & 1, L.err);
}

// out[p] = sum over tiles of partials[t][p], in double; layout of the
// outputs: grad_ant [3][np] (x, y, z) and grad_r0 [np] (may be null).
__global__ void adjoint_reduce_kernel(const float4 *__restrict__ partials, long long ntiles, int np,
                                      double *__restrict__ grad_ant, double *__restrict__ grad_r0, int accumulate) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x) {
        double gx = 0.0, gy = 0.0, gz = 0.0, gr = 0.0;
        for (long long t = 0; t < ntiles; ++t) {
            const float4 v = partials[t * np + p];
            gx += v.x;
            gy += v.y;
            gz += v.z;
            gr += v.w;
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
}

template <int MX, int PB>
cudaError_t launch_adj(const BpLaunch &L, const void *grad, void *partials, size_t smem, cudaStream_t s) {
    constexpr int TX = 8 * MX;
    const dim3 grid((L.ny + kTY - 1) / kTY, (L.nx + TX - 1) / TX, L.nz);
    auto kern = bp_adjoint_kernel<MX, PB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    kern<<<grid, kThreads, smem, s>>>(L, static_cast<const float2 *>(grad), static_cast<float4 *>(partials));
    return cudaGetLastError();
}

}  // namespace

long long bp_tile_count(const BpLaunch &L, const TileConfig &tc) {
    const long long TX = 8 * tc.mx;
    return ((L.ny + 63) / 64) * ((L.nx + TX - 1) / TX) * static_cast<long long>(L.nz);
}

size_t bp_adjoint_smem_bytes(const TileConfig &tc, int wsize) {
    return 32 + 2 * static_cast<size_t>(tc.pb) * sizeof(PulseGeo) + kWarps * static_cast<size_t>(tc.pb) * 16 +
           2 * static_cast<size_t>(tc.pb) * static_cast<size_t>(wsize) * 16;
}

cudaError_t launch_bp_adjoint(const BpLaunch &L, const void *grad, void *partials, const TileConfig &tc, size_t smem,
                              cudaStream_t s) {
#define SARBP_ADJ_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_) return launch_adj<MX_, PB_>(L, grad, partials, smem, s);
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
    const int blocks = (np + 255) / 256;
    adjoint_reduce_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(static_cast<const float4 *>(partials), ntiles, np,
                                                                  grad_ant, grad_r0, accumulate);
    return cudaGetLastError();
}

}  // namespace sarbp
