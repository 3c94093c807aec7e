// bp_common.cuh -- shared device helpers of the sm_100a backprojection kernels.
//
// * mbarrier + cp.async.bulk (the non-tensor TMA copy, no multicast) used to
//   stage each pulse's range-bin window of a pixel tile into shared memory;
// * bounded waits: every wait gives up after a fixed wall time, sets an error
//   bit and lets the kernel return instead of hanging;
// * the per-(tile, pulse) geometry record computed in FP64 once per tile and
//   pulse and read by every thread of the tile.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sarbp {

// Device error bits (plan->d_err)
enum : unsigned {
    ERRBIT_NOT_FINITE = 1u,
    ERRBIT_TIMEOUT = 2u,
    ERRBIT_BOUNDS = 4u,
};

// speed of light, include/uncc_sar_focusing.hpp:34
constexpr double kClight = 299792458.0;

// Wall-clock limit of a bounded wait (ns).
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of the barrier; false (and an error bit) after the
// wall-clock limit.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, unsigned *err) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_timer_ns();
    for (unsigned it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0u && global_timer_ns() - t0 > kWaitLimitNs) {
            atomicOr(err, ERRBIT_TIMEOUT);
            return false;
        }
    }
}

// Plain (non-multicast) bulk copy global -> this CTA's shared memory,
// completing transaction bytes on `bar`.  dst, src and bytes are multiples
// of 16 (the callers copy whole 16- or 32-byte entries from 256-byte aligned
// allocations).
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

__device__ __forceinline__ double frac_rev(double x) { return x - rint(x); }

// Flags of a PulseGeo record
enum : int {
    PG_ACTIVE = 1,  // the tile's window meets the valid range bins
    PG_GATE = 2,    // some pixels may fall outside (0, nfft-1): test each
    PG_NEAR = 4,    // tile too large for the far-field expansion: exact path
};

// Geometry of one pulse relative to one pixel tile (mixed-precision kernel).
//
// With the tile centre c on the pixel grid, pixel offset d = (i*dx, j*dy, 0)
// (integers i, j), u = (a - c)/|a - c|, Rc = |a - c|, t = u.d and
// e = |d|^2 - t^2, the differential range is exactly
//     dR = (Rc - R0) - t + g,   g = e / ((Rc - t) + sqrt((Rc - t)^2 + e))
// and g = e (h + t hr) (1 + O((|d|/Rc)^2)) with h = 1/(2Rc), hr = 1/(2Rc^2).
// Phase 2 pi k dR (k = 2 f0 / c), range bin lambda dR + nfft/2
// (lambda = nfft / max_wr).  The per-tile and per-step phase terms are
// reduced modulo one revolution in FP64, so what is left for FP32 is small.
// Field groups are 16-byte aligned so a thread reads them with vector loads.
struct __align__(16) PulseGeo {
    double A, alpha;   // frac(k (Rc - R0)); frac(-k ux dx): revolutions per x step
    double beta, B0;   // frac(-k uy dy); tile-centre bin relative to the window start
    double gam, eta;   // -lambda ux dx, -lambda uy dy: bins per x / y step
    float a8r, b32r, g8, e32;  // 2 pi frac(8 alpha), 2 pi frac(32 beta) (rad); 8 gam, 32 eta (bins)
    float tx, ty, h, hr;     // ux dx, uy dy (m); 1/(2 Rc), 1/(2 Rc^2)
    float kr, rc, lo, hi;    // 2 pi k (rad/m); Rc; valid iff lo < B_rel < hi
    int ws;                  // start bin of the tile's full window (W bins each side; may be negative)
    int flags;               // PG_*
    int wp;                  // this pulse's half-width (<= W): the bins it can reach from the tile
    int pad1;
    float ux, uy, uz, rinv;  // unit vector tile centre -> antenna, 1/Rc (adjoint kernel)
};
static_assert(sizeof(PulseGeo) == 128, "PulseGeo layout");

// Geometry of one pulse for the FP64 kernel (per-pixel exact computation).
struct __align__(16) PulseGeo64 {
    double ax, ay, az;  // antenna position
    double r0;          // slant range to scene centre
    double k;           // 2 f0 / c
    int ws;             // window start bin
    int flags;          // PG_ACTIVE
};
static_assert(sizeof(PulseGeo64) % 16 == 0, "PulseGeo64 must keep 16-byte alignment");

}  // namespace sarbp
