// noalloc.cu -- backprojection that allocates nothing.
//
// sarbp_backproject normally reads range profiles from a plan whose device
// buffers sarbp_plan_create allocated.  Some callers cannot allocate device
// memory when they need an image: a data-collection loop that hands pulses to
// a callback as they arrive (the way the reference's charlotte_sar_api.hpp
// callbacks are meant to be driven) cannot afford the device-wide
// synchronisation and unbounded latency of cudaMalloc/cudaFree, and a host
// application that owns the GPU's memory through its own pool or a fixed
// budget does not allow a library to take more behind its back.  For them,
// sarbp_backproject_noalloc takes range profiles, geometry and the image in
// memory the caller already owns, and keeps the only scratch it needs -- the
// pair-entry rows the kernel stages from, plus one error word -- in the
// file-scope array below.
//
// The array is a fixed 32 MiB per GPU that loads this library, held until the
// process exits.  Every call shares it and leaves its contents behind, so each
// call rewrites whole rows (guard bands included) and zeroes the error word
// before its kernels run; two calls that overlap on the GPU (different
// streams, or different host threads on one device) race on it.  The first
// call on a device looks up the array's device address with
// cudaGetSymbolAddress (once per device, that device current) and caches it;
// make that first call before any stream capture.  The call is synchronous:
// it waits for its stream and reports kernel-side errors as a status.
#include <cmath>
#include <cstdint>
#include <mutex>

#include "bp_common.cuh"
#include "host_common.h"
#include "sarbp_internal.h"

namespace {

using namespace sarbp;

// 2^21 16-byte entries = 32 MiB.  Entry 0 holds the error word; pair rows
// start at entry 1 (16-byte aligned, as the bulk copies need).
constexpr size_t kScratchEntries = size_t(1) << 21;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float4 g_noalloc_scratch[kScratchEntries];

std::mutex g_scratch_mutex;
float4 *g_scratch_addr[kMaxDevices] = {};

int scratch_for(int dev, float4 **out) {
    if (dev < 0 || dev >= kMaxDevices) return SARBP_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return SARBP_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<float4 *>(p);
    }
    *out = g_scratch_addr[dev];
    return SARBP_OK;
}

// Whole pair rows {rc[b], rc[b+1] - rc[b]}, zero outside 0 <= b < nfft
// (including the guard bands, which a previous call may have filled).
__global__ void noalloc_pair_rows(const float2 *__restrict__ rc, float4 *__restrict__ rows, int nfft, int guard,
                                  long long row_stride, long long total) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long p = i / row_stride;
        const int b = static_cast<int>(i - p * row_stride) - guard;
        float2 v = make_float2(0.0f, 0.0f), vn = make_float2(0.0f, 0.0f);
        if (b >= 0 && b < nfft) v = rc[p * nfft + b];
        if (b + 1 >= 0 && b + 1 < nfft) vn = rc[p * nfft + b + 1];
        rows[i] = make_float4(v.x, v.y, vn.x - v.x, vn.y - v.y);
    }
}

bool finite_nonneg(double v) { return std::isfinite(v) && v >= 0.0; }

void axis(int n, double c, double w, double *lo, double *step) {
    if (n > 1) {
        *step = w / static_cast<double>(n - 1);
        *lo = c - 0.5 * w;
    } else {
        *step = 0.0;
        *lo = c;
    }
}

}  // namespace

extern "C" SARBP_API int sarbp_backproject_noalloc(const sarbp_plan_desc *desc, const void *range_profiles,
                                                   const sarbp_geometry *geo, void *image, int flags,
                                                   void *stream) {
    host::NvtxRange range("sarbp_backproject_noalloc");
    if (!desc || !range_profiles || !geo || !image || !geo->ant_x || !geo->ant_y || !geo->ant_z ||
        !geo->slant_range || !geo->start_freq)
        return SARBP_ERR_NULL_POINTER;
    const sarbp_grid &g = desc->grid;
    if (geo->memory != SARBP_MEMORY_DEVICE || geo->num_pulses < 1 || desc->nfft < 2 || desc->nfft > (1 << 24) ||
        !(std::isfinite(desc->max_wr) && desc->max_wr > 0.0) || g.nx < 1 || g.ny < 1 || g.nz < 1 ||
        g.nx > (1 << 20) || g.ny > (1 << 20) || g.nz > 65535 || !std::isfinite(g.x0) || !std::isfinite(g.y0) ||
        !std::isfinite(g.z0) || !finite_nonneg(g.wx) || !finite_nonneg(g.wy) || !finite_nonneg(g.wz) ||
        (flags & ~SARBP_ACCUMULATE))
        return SARBP_ERR_INVALID_ARGUMENT;
    if (desc->precision != SARBP_PRECISION_MIXED) return SARBP_ERR_UNSUPPORTED;

    BpLaunch L{};
    double left, bottom, zlow, dx, dy, dz;
    axis(g.nx, g.x0, g.wx, &left, &dx);
    axis(g.ny, g.y0, g.wy, &bottom, &dy);
    axis(g.nz, g.z0, g.wz, &zlow, &dz);
    const double lambda = static_cast<double>(desc->nfft) / desc->max_wr;

    // tile: 32 x 64 pixels when the windows allow two CTAs per SM, else the
    // deepest stage of smaller tiles that fits one CTA per SM
    static const int cand[][2] = {{4, 8}, {4, 4}, {2, 8}, {2, 4}, {1, 8}, {1, 4}, {2, 2}, {1, 2}, {1, 1}};
    TileConfig tc{0, 0};
    int W = 0, wsize = 0;
    size_t smem = 0;
    for (int pass = 0; pass < 2 && !tc.mx; ++pass) {
        const size_t limit = pass == 0 ? 110u * 1024u : 227u * 1024u;
        for (const auto &c : cand) {
            const double hx = 0.5 * 8.0 * c[0] * dx, hy = 0.5 * 64.0 * dy;
            const int w = static_cast<int>(std::ceil(lambda * std::sqrt(hx * hx + hy * hy))) + 3;
            const TileConfig t{c[0], c[1]};
            const size_t sm = bp_mixed_smem_bytes(t, 2 * w + 2);
            if (2 * w + 2 > (1 << 16) || sm > limit) continue;
            tc = t;
            W = w;
            wsize = 2 * w + 2;
            smem = sm;
            break;
        }
    }
    if (!tc.mx) return SARBP_ERR_UNSUPPORTED;
    const int guard = wsize + 2;
    const long long row_stride = static_cast<long long>(desc->nfft) + 2LL * guard;
    const long long total = row_stride * geo->num_pulses;
    if (total > static_cast<long long>(kScratchEntries) - 1) return SARBP_ERR_UNSUPPORTED;  // beyond 32 MiB

    // desc->device >= 0: run on that device (as sarbp_plan_create does), the
    // caller's current device restored on return; -1: the current device
    if (desc->device < -1) return SARBP_ERR_INVALID_ARGUMENT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return SARBP_ERR_NO_DEVICE;
    }
    if (desc->device >= 0) {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess) {
            cudaGetLastError();
            return SARBP_ERR_NO_DEVICE;
        }
        if (desc->device >= count) return SARBP_ERR_INVALID_ARGUMENT;
        dev = desc->device;
    }
    host::DeviceGuard on_device(dev);
    if (on_device.status != cudaSuccess) {
        cudaGetLastError();
        return SARBP_ERR_CUDA;
    }
    float4 *scratch = nullptr;
    int st = scratch_for(dev, &scratch);
    if (st != SARBP_OK) return st;
    unsigned *err = reinterpret_cast<unsigned *>(scratch);
    float4 *rows = scratch + 1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) {
        const long long blocks = (total + 255) / 256;
        noalloc_pair_rows<<<static_cast<int>(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, s>>>(
            static_cast<const float2 *>(range_profiles), rows, desc->nfft, guard, row_stride, total);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        L.pairs = rows;
        L.row_stride = row_stride;
        L.guard = guard;
        L.ax = geo->ant_x;
        L.ay = geo->ant_y;
        L.az = geo->ant_z;
        L.r0 = geo->slant_range;
        L.f0 = geo->start_freq;
        L.np = geo->num_pulses;
        L.nfft = desc->nfft;
        L.lambda = lambda;
        L.half_nfft = 0.5 * desc->nfft;
        L.nx = g.nx;
        L.ny = g.ny;
        L.nz = g.nz;
        L.left = left;
        L.bottom = bottom;
        L.zlow = zlow;
        L.dx = dx;
        L.dy = dy;
        L.dz = dz;
        L.W = W;
        L.wsize = wsize;
        const double hx = 0.5 * 8.0 * tc.mx * dx, hy = 0.5 * 64.0 * dy;
        const double hd = std::sqrt(hx * hx + hy * hy);
        L.near_hd16 = 16.0 * hd;
        L.near_coef = 0.625 * hd * hd * hd * hd / 1.0e-7;
        L.img = image;
        L.accumulate = (flags & SARBP_ACCUMULATE) ? 1 : 0;
        L.err = err;
        L.nhyp = 1;
        e = launch_bp_mixed(L, tc, false, smem, s);
    }
    // the error word comes back on the call's own stream, behind its kernels:
    // one stream synchronisation, nothing ordered against other streams
    unsigned bits = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, err, sizeof(bits), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return SARBP_ERR_CUDA;
    }
    if (bits & ERRBIT_TIMEOUT) return SARBP_ERR_KERNEL_TIMEOUT;
    if (bits & ERRBIT_NOT_FINITE) return SARBP_ERR_NOT_FINITE;
    if (bits & ERRBIT_BOUNDS) return SARBP_ERR_KERNEL_BOUNDS;
    return SARBP_OK;
}
