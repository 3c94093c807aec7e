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

template <int MX, int PB>
__global__ void __launch_bounds__(kThreads, 1) bp_fp64_kernel(const BpLaunch L) {
    constexpr int TX = 8 * MX;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    PulseGeo64 *geo = reinterpret_cast<PulseGeo64 *>(smem + 32);
    PairD *win = reinterpret_cast<PairD *>(smem + 32 + 2 * PB * sizeof(PulseGeo64));
    const int wsize = L.wsize;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ty0 = blockIdx.x * kTY, tx0 = blockIdx.y * TX, iz = blockIdx.z;
    const double cx = L.left + static_cast<double>(tx0 + TX / 2) * L.dx;
    const double cy = L.bottom + static_cast<double>(ty0 + kTY / 2) * L.dy;
    const double z = L.zlow + static_cast<double>(iz) * L.dz;
    const double cz = z;

    double xs[MX], ys[2], acc_re[MX][2], acc_im[MX][2];
#pragma unroll
    for (int k = 0; k < MX; ++k) {
        xs[k] = L.left + static_cast<double>(tx0 + warp + 8 * k) * L.dx;
#pragma unroll
        for (int l = 0; l < 2; ++l) acc_re[k][l] = acc_im[k][l] = 0.0;
    }
#pragma unroll
    for (int l = 0; l < 2; ++l) ys[l] = L.bottom + static_cast<double>(ty0 + 2 * lane + l) * L.dy;
    const double top = static_cast<double>(L.nfft - 1);

    const uint32_t bar_base = smem_addr(&bars[0]);  // stage s barrier at bar_base + 8*s
    if (threadIdx.x == 0) {
        mbar_init(bar_base, PB);
        mbar_init(bar_base + 8, PB);
        fence_mbar_init();
    }
    __syncthreads();

    const int nblocks = (L.np + PB - 1) / PB;
    if (nblocks > 0) produce_slots64<PB>(L, 0, geo, smem_addr(win), bar_base, warp, lane, cx, cy, cz);
    __syncthreads();

    int last_issued = 0;
    bool timed_out = false;
    for (int b = 0; b < nblocks; ++b) {
        const int s = b & 1;
        if (b + 1 < nblocks) {
            produce_slots64<PB>(L, b + 1, geo + (s ^ 1) * PB, smem_addr(win + (s ^ 1) * PB * wsize),
                                bar_base + 8 * (s ^ 1), warp, lane, cx, cy, cz);
            last_issued = b + 1;
        }
        const bool ok = mbar_wait_bounded(bar_base + 8 * s, (b >> 1) & 1, L.err);
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
            timed_out = true;
            break;
        }
    }
    if (timed_out) {
        if (threadIdx.x == 0 && last_issued > 0) mbar_wait_bounded(bar_base + 8 * (last_issued & 1), (last_issued >> 1) & 1, L.err);
        return;
    }

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
            double2 v = make_double2(acc_re[k][l], acc_im[k][l]);
            if (L.accumulate) {
                const double2 old = img[o];
                v.x += old.x;
                v.y += old.y;
            }
            img[o] = v;
        }
    }
}

template <int MX, int PB>
cudaError_t launch64(const BpLaunch &L, size_t smem, cudaStream_t s) {
    constexpr int TX = 8 * MX;
    const dim3 grid((L.ny + kTY - 1) / kTY, (L.nx + TX - 1) / TX, L.nz);
    auto kern = bp_fp64_kernel<MX, PB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    kern<<<grid, kThreads, smem, s>>>(L);
    return cudaGetLastError();
}

}  // namespace

size_t bp_fp64_smem_bytes(const TileConfig &tc, int wsize) {
    return 32 + 2 * static_cast<size_t>(tc.pb) * sizeof(PulseGeo64) +
           2 * static_cast<size_t>(tc.pb) * static_cast<size_t>(wsize) * 32;
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
