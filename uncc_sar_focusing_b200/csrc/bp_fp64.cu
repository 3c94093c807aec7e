// bp_fp64.cu -- all-FP64 forward backprojection for sm_100a.
//
// Same tiling, shared-memory window staging (cp.async.bulk + mbarrier) and
// output layout as the mixed kernel in bp_mixed.cu, but every pixel-pulse is
// computed directly in double: |a_p - x_q| with a double sqrt, the bin
// index, the linear interpolation of FP64 range profiles and the rotation
// exp(+j 2 pi k dR) (k = 2 f0 / c, reduced mod one revolution, sincospi),
// accumulated in double.  It is the accuracy path and the FP64 baseline the
// mixed kernel is measured against; semantics as bp_mixed.cu.
#include <cstdint>

#include "bp_common.cuh"
#include "bp_tile.cuh"
#include "sarbp_internal.h"

namespace sarbp {
namespace {

constexpr int kThreads = 256;
constexpr int kTY = 64;

struct __align__(16) PairD {
    double vr, vi, dr, di;  // rc[b] and rc[b+1] - rc[b]
};

__device__ __forceinline__ PulseGeo64 make_geo64(const BpLaunch &L, int p, double cx, double cy, double cz) {
    PulseGeo64 g;
    g.flags = 0;
    g.ax = L.ax[p];
    g.ay = L.ay[p];
    g.az = L.az[p];
    g.r0 = L.r0[p];
    g.k = 2.0 * L.f0[p] / kClight;
    const double vx = g.ax - cx, vy = g.ay - cy, vz = g.az - cz;
    const double D = sqrt(vx * vx + vy * vy + vz * vz) - g.r0;
    const double bc = D * L.lambda + L.half_nfft;
    if (!(isfinite(bc) && isfinite(g.k) && fabs(bc) < 1.0e9)) {
        atomicOr(L.err, ERRBIT_NOT_FINITE);
        return g;
    }
    g.ws = static_cast<int>(floor(bc)) - L.W;
    if (!(g.ws + L.wsize - 2 <= 0 || g.ws + 1 >= L.nfft - 1)) g.flags = PG_ACTIVE;
    return g;
}

// As produce_slots in bp_mixed.cu: warp w handles pulse slots w, w + 8, ...
template <int PB>
__device__ __forceinline__ void produce_slots64(const BpLaunch &L, int b, PulseGeo64 *geo_s, uint32_t win_s,
                                                uint32_t bar, int warp, int lane, double cx, double cy, double cz) {
    if (lane != 0) return;
    for (int q = warp; q < PB; q += kThreads / 32) {
        const int p = b * PB + q;
        PulseGeo64 g;
        g.flags = 0;
        if (p < L.np) g = make_geo64(L, p, cx, cy, cz);
        geo_s[q] = g;
        if (g.flags & PG_ACTIVE) {
            const uint32_t bytes = static_cast<uint32_t>(L.wsize) * 32u;
            const PairD *src =
                static_cast<const PairD *>(L.pairs) + static_cast<long long>(p) * L.row_stride + L.guard + g.ws;
            mbar_arrive_expect_tx(bar, bytes);
            bulk_copy_g2s(win_s + static_cast<uint32_t>(q) * bytes, src, bytes, bar);
        } else {
            mbar_arrive(bar);
        }
    }
}

// Store (or add) a thread's MX x 2 pixels of the tile at (tx0, ty0, z-slice iz).
template <int MX>
__device__ __forceinline__ void store_pixels64(const BpLaunch &L, int tx0, int ty0, int iz, int warp, int lane,
                                               const double (&re)[MX][2], const double (&im)[MX][2]) {
    double2 *img = static_cast<double2 *>(L.img);
#pragma unroll
    for (int k = 0; k < MX; ++k) {
        const int row = tx0 + warp + 8 * k;
        if (row >= L.nx) continue;
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const int col = ty0 + 2 * lane + l;
            if (col >= L.ny) continue;
            const long long o = (static_cast<long long>(iz) * L.nx + row) * L.ny + col;
            double2 v = make_double2(re[k][l], im[k][l]);
            if (L.accumulate) {
                const double2 old = img[o];
                v.x += old.x;
                v.y += old.y;
            }
            img[o] = v;
        }
    }
}

// Tile-local index of pixel (row warp + 8k, column 2 lane + l) in a
// partial-sum slot of TX x 64 complex128 values.
__device__ __forceinline__ int slot_pixel(int warp, int lane, int k, int l) { return (warp + 8 * k) * kTY + 2 * lane + l; }

// Units of (tile, stage) split over the CTAs as in bp_mixed.cu (tile::sk_lo).
template <int MX, int PB>
__global__ void __launch_bounds__(kThreads, 1) bp_fp64_kernel(const BpLaunch L) {
    constexpr int TX = 8 * MX;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    PulseGeo64 *geo = reinterpret_cast<PulseGeo64 *>(smem + 32);
    PairD *win = reinterpret_cast<PairD *>(smem + 32 + 2 * PB * sizeof(PulseGeo64));
    const int wsize = L.wsize;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const tile::TileGrid tg = tile::tile_grid(L, TX, PB);
    const long long G = gridDim.x;
    const long long lo = tile::sk_lo(blockIdx.x, tg.units, G);
    const int n = static_cast<int>(tile::sk_lo(blockIdx.x + 1, tg.units, G) - lo);
    if (n <= 0) return;
    const int S = tg.stages;

    double xs[MX], ys[2], z = 0.0, acc_re[MX][2], acc_im[MX][2];
#pragma unroll
    for (int k = 0; k < MX; ++k)
#pragma unroll
        for (int l = 0; l < 2; ++l) acc_re[k][l] = acc_im[k][l] = 0.0;
    const double top = static_cast<double>(L.nfft - 1);

    const uint32_t bar_base = smem_addr(&bars[0]);  // buffer s barrier at bar_base + 8*s
    if (threadIdx.x == 0) {
        mbar_init(bar_base, PB);
        mbar_init(bar_base + 8, PB);
        fence_mbar_init();
    }
    __syncthreads();

    auto produce = [&](const tile::UnitCursor &pc, int s) {
        if (lane != 0) return;
        const double cx = L.left + static_cast<double>(pc.tx * TX + TX / 2) * L.dx;
        const double cy = L.bottom + static_cast<double>(pc.ty * kTY + kTY / 2) * L.dy;
        const double cz = L.zlow + static_cast<double>(pc.iz) * L.dz;
        produce_slots64<PB>(L, pc.b, geo + s * PB, smem_addr(win + s * PB * wsize), bar_base + 8 * s, warp, lane, cx,
                            cy, cz);
    };

    tile::UnitCursor cc, pc;  // consumer at unit i, producer at unit i + 1
    cc.init(tg, L, lo);
    pc = cc;
    produce(pc, 0);
    __syncthreads();

    int last_issued = 0;
    int seg = 0;
    int seg_first = cc.b;
    bool new_tile = true;
    for (int i = 0; i < n; ++i) {
        const int s = i & 1;
        if (i + 1 < n) {
            pc.advance(tg, L);
            produce(pc, s ^ 1);
            last_issued = i + 1;
        }
        const int b = cc.b;
        if (new_tile) {
            const int tx0 = cc.tx * TX, ty0 = cc.ty * kTY;
#pragma unroll
            for (int k = 0; k < MX; ++k) xs[k] = L.left + static_cast<double>(tx0 + warp + 8 * k) * L.dx;
#pragma unroll
            for (int l = 0; l < 2; ++l) ys[l] = L.bottom + static_cast<double>(ty0 + 2 * lane + l) * L.dy;
            z = L.zlow + static_cast<double>(cc.iz) * L.dz;
            new_tile = false;
        }
        const bool ok = mbar_wait_bounded(bar_base + 8 * s, (i >> 1) & 1, L.err);
        if (ok) {
            const int nq = min(PB, L.np - b * PB);
            for (int q = 0; q < nq; ++q) {
                const PulseGeo64 &g = geo[s * PB + q];
                if (!(g.flags & PG_ACTIVE)) continue;
                const PairD *w = win + (s * PB + q) * wsize;
                const double gax = g.ax, gay = g.ay, gaz = g.az, gr0 = g.r0, gk = g.k;
                const int gws = g.ws;
                const double ez = gaz - z;
#pragma unroll
                for (int k = 0; k < MX; ++k) {
                    const double ex = gax - xs[k];
#pragma unroll
                    for (int l = 0; l < 2; ++l) {
                        const double ey = gay - ys[l];
                        const double dR = sqrt(ex * ex + ey * ey + ez * ez) - gr0;
                        const double B = dR * L.lambda + L.half_nfft;
                        if (!(B > 0.0 && B < top)) continue;  // rmin < dR < rmax
                        const double fl = floor(B);
                        const int idx = static_cast<int>(fl) - gws;
                        if (static_cast<unsigned>(idx) > static_cast<unsigned>(wsize - 2)) {
                            atomicOr(L.err, ERRBIT_BOUNDS);
                            continue;
                        }
                        const double a = B - fl;
                        const PairD v = w[idx];
                        const double re = fma(a, v.dr, v.vr);
                        const double im = fma(a, v.di, v.vi);
                        const double ph = gk * dR;
                        double sn, cs;
                        sincospi(2.0 * (ph - rint(ph)), &sn, &cs);
                        acc_re[k][l] = fma(re, cs, fma(-im, sn, acc_re[k][l]));
                        acc_im[k][l] = fma(re, sn, fma(im, cs, acc_im[k][l]));
                    }
                }
            }
        }
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0 && last_issued > i)
                mbar_wait_bounded(bar_base + 8 * (last_issued & 1), (last_issued >> 1) & 1, L.err);
            return;
        }
        if (i + 1 == n || b == S - 1) {
            if (seg_first == 0 && b == S - 1) {
                store_pixels64<MX>(L, cc.tx * TX, cc.ty * kTY, cc.iz, warp, lane, acc_re, acc_im);
            } else {
                double2 *slot = static_cast<double2 *>(L.sk_partial) +
                                (2 * static_cast<long long>(blockIdx.x) + (seg > 0 ? 1 : 0)) * (TX * kTY);
#pragma unroll
                for (int k = 0; k < MX; ++k)
#pragma unroll
                    for (int l = 0; l < 2; ++l)
                        slot[slot_pixel(warp, lane, k, l)] = make_double2(acc_re[k][l], acc_im[k][l]);
            }
#pragma unroll
            for (int k = 0; k < MX; ++k)
#pragma unroll
                for (int l = 0; l < 2; ++l) acc_re[k][l] = acc_im[k][l] = 0.0;
            ++seg;
            seg_first = 0;
            new_tile = true;
        }
        cc.advance(tg, L);
    }
}

template <int MX>
__global__ void __launch_bounds__(kThreads) bp_sk_fixup64_kernel(const BpLaunch L, long long G, int PB) {
    constexpr int TX = 8 * MX;
    const tile::TileGrid tg = tile::tile_grid(L, TX, PB);
    const long long t = blockIdx.x;
    const long long c0 = tile::sk_owner(t * tg.stages, tg.units, G);
    const long long c1 = tile::sk_owner(t * tg.stages + tg.stages - 1, tg.units, G);
    if (c0 == c1) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double re[MX][2], im[MX][2];
#pragma unroll
    for (int k = 0; k < MX; ++k)
#pragma unroll
        for (int l = 0; l < 2; ++l) re[k][l] = im[k][l] = 0.0;
    const double2 *part = static_cast<const double2 *>(L.sk_partial);
    for (long long c = c0; c <= c1; ++c) {
        const double2 *slot = part + tile::sk_slot(c, t * tg.stages, tg.units, G) * (TX * kTY);
#pragma unroll
        for (int k = 0; k < MX; ++k)
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                const double2 v = slot[slot_pixel(warp, lane, k, l)];
                re[k][l] += v.x;
                im[k][l] += v.y;
            }
    }
    int tx0, ty0, iz;
    tile::tile_origin(tg, t, TX, tx0, ty0, iz);
    store_pixels64<MX>(L, tx0, ty0, iz, warp, lane, re, im);
}

template <int MX, int PB>
cudaError_t launch64(const BpLaunch &L, size_t smem, cudaStream_t s) {
    constexpr int TX = 8 * MX;
    auto kern = bp_fp64_kernel<MX, PB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const tile::TileGrid tg = tile::tile_grid(L, TX, PB);
    if (tg.units < 1) return cudaSuccess;
    long long G = tg.tiles;
    if (L.sk_partial && L.sk_resident > 0 && tg.tiles % L.sk_resident != 0) {
        const long long g = L.sk_resident < tg.units ? L.sk_resident : tg.units;
        if (2 * g * TX * kTY * static_cast<long long>(sizeof(double2)) <= L.sk_slot_bytes) G = g;
    }
    if (G > 0x7fffffffLL) return cudaErrorInvalidValue;
    kern<<<static_cast<unsigned>(G), kThreads, smem, s>>>(L);
    e = cudaGetLastError();
    if (e != cudaSuccess || G == tg.tiles) return e;
    bp_sk_fixup64_kernel<MX><<<static_cast<unsigned>(tg.tiles), kThreads, 0, s>>>(L, G, PB);
    return cudaGetLastError();
}

template <int MX, int PB>
int resident64(size_t smem) {
    auto kern = bp_fp64_kernel<MX, PB>;
    int dev = 0, sms = 0, occ = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return occ * sms;
}

}  // namespace

size_t bp_fp64_smem_bytes(const TileConfig &tc, int wsize) {
    return 32 + 2 * static_cast<size_t>(tc.pb) * sizeof(PulseGeo64) +
           2 * static_cast<size_t>(tc.pb) * static_cast<size_t>(wsize) * 32;
}

int bp_fp64_resident(const TileConfig &tc, size_t smem) {
#define SARBP_FP64_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_) return resident64<MX_, PB_>(smem);
    SARBP_FP64_CASE(4, 16)
    SARBP_FP64_CASE(4, 8)
    SARBP_FP64_CASE(4, 4)
    SARBP_FP64_CASE(4, 2)
    SARBP_FP64_CASE(4, 1)
    SARBP_FP64_CASE(2, 16)
    SARBP_FP64_CASE(2, 8)
    SARBP_FP64_CASE(2, 4)
    SARBP_FP64_CASE(2, 2)
    SARBP_FP64_CASE(2, 1)
    SARBP_FP64_CASE(1, 16)
    SARBP_FP64_CASE(1, 8)
    SARBP_FP64_CASE(1, 4)
    SARBP_FP64_CASE(1, 2)
    SARBP_FP64_CASE(1, 1)
#undef SARBP_FP64_CASE
    return 0;
}

cudaError_t launch_bp_fp64(const BpLaunch &L, const TileConfig &tc, size_t smem, cudaStream_t s) {
#define SARBP_FP64_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_) return launch64<MX_, PB_>(L, smem, s);
    SARBP_FP64_CASE(4, 16)
    SARBP_FP64_CASE(4, 8)
    SARBP_FP64_CASE(4, 4)
    SARBP_FP64_CASE(4, 2)
    SARBP_FP64_CASE(4, 1)
    SARBP_FP64_CASE(2, 16)
    SARBP_FP64_CASE(2, 8)
    SARBP_FP64_CASE(2, 4)
    SARBP_FP64_CASE(2, 2)
    SARBP_FP64_CASE(2, 1)
    SARBP_FP64_CASE(1, 16)
    SARBP_FP64_CASE(1, 8)
    SARBP_FP64_CASE(1, 4)
    SARBP_FP64_CASE(1, 2)
    SARBP_FP64_CASE(1, 1)
#undef SARBP_FP64_CASE
    return cudaErrorInvalidValue;
}

}  // namespace sarbp
