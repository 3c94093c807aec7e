// api.cu -- the C ABI of include/sarbp.h.
//
// Host-side driver in place of the reference's cuda_focus_SAR_image
// (src/gpuBackProjection/cuda_sar_focusing/cuda_sar_focusing.hpp:526-723):
// plan creation holds what the reference re-creates on every call
// (GPUMemoryManager allocations :93-348, the cuFFT plan :372-399, the range
// bin vector :574-598), every call is stream-ordered, errors come back as
// status codes, and nothing resets the device.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "bp_common.cuh"
#include "host_common.h"
#include "sarbp_internal.h"

using namespace sarbp;
using namespace sarbp::host;

namespace {

// Window geometry for a tile of (8*mx) x 64 pixels centred on an integer pixel.
void window_for(const sarbp_plan *p, int mx, int *W, int *wsize) {
    double hd;
    tile_window(p->lambda, p->dx, p->dy, mx, W, wsize, &hd);
}

// Largest stage depth whose shared memory fits 2 CTAs per SM (mixed) or one
// (FP64); environment SARBP_TILE="mx,pb" overrides (tuning runs).
int choose_tile(sarbp_plan *p) {
    // (mx, pb) candidates, best first; the first pass keeps two CTAs per SM
    // for the mixed kernel, the second accepts one CTA per SM (coarse grids
    // whose range-bin windows are wide).  64-row tiles (mx = 8, mixed only)
    // halve the per-pulse record, base-table and setup work per pixel: on
    // 1024 x 2048 x 1024^2 a pixel-pulse costs ~1.87 (mx 8) against ~2.25
    // (mx 4) time units, so they are taken unless padding the rows to 64
    // instead of 32 adds more than 15% pixels.
    static const int cand[][2] = {{8, 8}, {8, 4}, {4, 8}, {4, 4}, {2, 8}, {2, 4}, {1, 8}, {1, 4}, {2, 2}, {1, 2}, {1, 1}};
    const int ncand = static_cast<int>(sizeof(cand) / sizeof(cand[0]));
    const bool fp64 = p->precision == SARBP_PRECISION_FP64;
    const long long nx = p->desc.grid.nx;
    const bool tall_tiles = !fp64 && (nx + 63) / 64 * 64 * 100 <= (nx + 31) / 32 * 32 * 115;
    int forced_mx = 0, forced_pb = 0;
    if (const char *env = std::getenv("SARBP_TILE")) {
        if (std::sscanf(env, "%d,%d", &forced_mx, &forced_pb) != 2) forced_mx = forced_pb = 0;
    }
    const size_t limits[2] = {fp64 ? 220u * 1024u : 110u * 1024u, 227u * 1024u};
    for (int pass = -1; pass < 2; ++pass) {
        for (int i = 0; i < ncand; ++i) {
            int mx = cand[i][0], pb = cand[i][1];
            if (pass < 0) {
                if (!forced_mx || i > 0) break;
                mx = forced_mx;
                pb = forced_pb;
            }
            if (pass >= 0 && mx == 8 && !tall_tiles) continue;
            int W, wsize;
            window_for(p, mx, &W, &wsize);
            if (wsize > (1 << 16)) continue;
            TileConfig tc{mx, pb};
            const size_t smem = fp64 ? bp_fp64_smem_bytes(tc, wsize) : bp_mixed_smem_bytes(tc, wsize);
            if (smem > limits[pass < 0 ? 1 : pass]) continue;
            p->tile = tc;
            p->W = W;
            p->wsize = wsize;
            p->smem = smem;
            return SARBP_OK;
        }
    }
    return SARBP_ERR_UNSUPPORTED;
}

}  // namespace

// Pipelined host-buffer focusing: three streams (uploads, kernels, downloads)
// and kDepth staging slots.  Submission t uses slot t % kDepth; its upload is
// enqueued only after submission t - kDepth has been collected on the host,
// which also orders the slot's reuse.  Per-slot error words travel back with
// the image into page-locked host memory.
struct sarbp_pipe {
    static constexpr int kDepth = 2;
    cudaStream_t in = nullptr, work = nullptr, out = nullptr;
    cudaEvent_t in_ready[kDepth] = {}, work_done[kDepth] = {}, out_done[kDepth] = {};
    void *d_ph[kDepth] = {};
    double *d_geo[kDepth] = {};
    void *d_img[kDepth] = {};
    unsigned *d_err = nullptr;  // [kDepth]
    unsigned *h_err = nullptr;  // [kDepth], page-locked
    unsigned long long submitted = 0, collected = 0;
    int pending = SARBP_OK;  // first error of a collected submission, not yet reported
};

namespace {

void destroy_pipe(sarbp_pipe *q) {
    if (!q) return;
    for (cudaStream_t s : {q->in, q->work, q->out})
        if (s) cudaStreamSynchronize(s);
    for (int i = 0; i < sarbp_pipe::kDepth; ++i) {
        for (cudaEvent_t e : {q->in_ready[i], q->work_done[i], q->out_done[i]})
            if (e) cudaEventDestroy(e);
        cudaFree(q->d_ph[i]);
        cudaFree(q->d_geo[i]);
        cudaFree(q->d_img[i]);
    }
    cudaFree(q->d_err);
    if (q->h_err) cudaFreeHost(q->h_err);
    for (cudaStream_t s : {q->in, q->work, q->out})
        if (s) cudaStreamDestroy(s);
    cudaGetLastError();
    delete q;
}

void release(sarbp_plan *p) {
    if (!p) return;
    destroy_pipe(p->pipe);
    if (p->fft_ok) cufftDestroy(p->fft);
    cudaFree(p->d_ph);
    cudaFree(p->d_geo);
    cudaFree(p->d_fft);
    cudaFree(p->d_pairs);
    cudaFree(p->d_fac);
    cudaFree(p->d_img);
    cudaFree(p->d_err);
    cudaFree(p->d_partials);
    cudaFree(p->d_gout);
    cudaFree(p->d_hyp);
    cudaFree(p->d_sk);
    cudaFree(p->d_geotab);
    cudaFree(p->d_hyprec);
    cudaFree(p->d_rctab);
    cudaFree(p->d_win);
    delete p;
}

int alloc(sarbp_plan *p, void **ptr, size_t bytes) {
    const cudaError_t e = host::device_malloc(ptr, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return from_cuda(e);
    }
    p->bytes += bytes;
    return SARBP_OK;
}

size_t cplx_bytes(const sarbp_plan *p) { return p->precision == SARBP_PRECISION_FP64 ? 16 : 8; }

// The per-sample factor table of the range-compression kernels from the
// plan's weights (the caller's, else the desc's taper).
int upload_range_factors(sarbp_plan *p) {
    const std::vector<double> fac = range_factors(p->desc, p->range_w.empty() ? nullptr : p->range_w.data());
    if (p->precision == SARBP_PRECISION_FP64) {
        SARBP_TRY_CUDA(cudaMemcpy(p->d_fac, fac.data(), fac.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f32(fac.begin(), fac.end());
        SARBP_TRY_CUDA(cudaMemcpy(p->d_fac, f32.data(), f32.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    return SARBP_OK;
}

int check_geometry_host(const sarbp_geometry *g) {
    const double *arrs[5] = {g->ant_x, g->ant_y, g->ant_z, g->slant_range, g->start_freq};
    for (const double *a : arrs)
        for (int i = 0; i < g->num_pulses; ++i)
            if (!std::isfinite(a[i])) return SARBP_ERR_NOT_FINITE;
    return SARBP_OK;
}

int read_errors(sarbp_plan *p, cudaStream_t s) {
    SARBP_TRY_CUDA(cudaStreamSynchronize(s));
    unsigned bits = 0;
    SARBP_TRY_CUDA(cudaMemcpy(&bits, p->d_err, sizeof(bits), cudaMemcpyDeviceToHost));
    if (bits) SARBP_TRY_CUDA(cudaMemset(p->d_err, 0, sizeof(unsigned)));
    return status_from_bits(bits);
}

int range_compress_impl(sarbp_plan *p, const void *ph, int np, int memory, cudaStream_t s) {
    if (!ph) return SARBP_ERR_NULL_POINTER;
    if (np < 1 || np > p->np_cap) return SARBP_ERR_INVALID_ARGUMENT;
    if (memory != SARBP_MEMORY_HOST && memory != SARBP_MEMORY_DEVICE) return SARBP_ERR_INVALID_ARGUMENT;
    const void *src = ph;
    if (memory == SARBP_MEMORY_HOST) {
        SARBP_TRY_CUDA(cudaMemcpyAsync(p->d_ph, ph, static_cast<size_t>(np) * p->K * 8, cudaMemcpyHostToDevice, s));
        src = p->d_ph;
    }
    if (p->d_rctab) {
        SARBP_TRY_CUDA(launch_rc_fused(src, p->d_fac, p->d_rctab, p->d_pairs, p->K, p->rc_R, np, p->row_stride,
                                       p->guard, p->rc_grid, s));
        p->np_ready = np;
        if (memory == SARBP_MEMORY_HOST) SARBP_TRY_CUDA(cudaStreamSynchronize(s));
        return SARBP_OK;
    }
    SARBP_TRY_CUDA(launch_rc_prep(p->precision, src, p->d_fac, p->d_fft, p->K, p->nfft, np, s));
    const cufftResult r0 = cufftSetStream(p->fft, s);
    if (r0 != CUFFT_SUCCESS) return from_cufft(r0);
    const cufftResult r1 =
        p->precision == SARBP_PRECISION_FP64
            ? cufftExecZ2Z(p->fft, static_cast<cufftDoubleComplex *>(p->d_fft),
                           static_cast<cufftDoubleComplex *>(p->d_fft), CUFFT_INVERSE)
            : cufftExecC2C(p->fft, static_cast<cufftComplex *>(p->d_fft), static_cast<cufftComplex *>(p->d_fft),
                           CUFFT_INVERSE);
    if (r1 != CUFFT_SUCCESS) return from_cufft(r1);
    SARBP_TRY_CUDA(launch_rc_pairs(p->precision, p->d_fft, p->d_pairs, p->nfft, np, p->row_stride, p->guard, s));
    p->np_ready = np;
    if (memory == SARBP_MEMORY_HOST) SARBP_TRY_CUDA(cudaStreamSynchronize(s));
    return SARBP_OK;
}

BpLaunch launch_params(const sarbp_plan *p, const double *ax, const double *ay, const double *az, const double *r0,
                       const double *f0, int np, void *img, int flags) {
    const sarbp_grid &g = p->desc.grid;
    BpLaunch L{};
    L.pairs = p->d_pairs;
    L.row_stride = p->row_stride;
    L.guard = p->guard;
    L.ax = ax;
    L.ay = ay;
    L.az = az;
    L.r0 = r0;
    L.f0 = f0;
    L.np = np;
    L.nfft = p->nfft;
    L.lambda = p->lambda;
    L.half_nfft = 0.5 * p->nfft;
    L.nx = g.nx;
    L.ny = g.ny;
    L.nz = g.nz;
    L.left = p->left;
    L.bottom = p->bottom;
    L.zlow = p->zlow;
    L.dx = p->dx;
    L.dy = p->dy;
    L.dz = p->dz;
    L.W = p->W;
    L.wsize = p->wsize;
    L.near_hd16 = p->near_hd16;
    L.near_coef = p->near_coef;
    L.img = img;
    L.accumulate = (flags & SARBP_ACCUMULATE) ? 1 : 0;
    L.err = p->d_err;
    L.nhyp = 1;
    L.sk_partial = p->d_sk;
    L.sk_slot_bytes = static_cast<long long>(p->sk_bytes);
    L.sk_resident = p->sk_resident;
    L.geo_tab = p->d_geotab;
    L.geo_tab_records = p->geotab_records;
    L.drop_pulse = p->drop_pulse;
    return L;
}

// Geometry arrays on the device: the caller's, or the plan's staging copy.
int device_geometry(sarbp_plan *p, const sarbp_geometry *geo, cudaStream_t s, const double **out) {
    const int np = geo->num_pulses;
    const double *src[5] = {geo->ant_x, geo->ant_y, geo->ant_z, geo->slant_range, geo->start_freq};
    if (geo->memory == SARBP_MEMORY_HOST) {
        const int st = check_geometry_host(geo);
        if (st != SARBP_OK) return st;
        for (int i = 0; i < 5; ++i) {
            SARBP_TRY_CUDA(cudaMemcpyAsync(p->d_geo + static_cast<size_t>(i) * p->np_cap, src[i],
                                           sizeof(double) * np, cudaMemcpyHostToDevice, s));
            out[i] = p->d_geo + static_cast<size_t>(i) * p->np_cap;
        }
    } else {
        for (int i = 0; i < 5; ++i) out[i] = src[i];
    }
    return SARBP_OK;
}

int backproject_impl(sarbp_plan *p, const sarbp_geometry *geo, void *image, int image_memory, int flags,
                     cudaStream_t s) {
    if (!geo || !image || !geo->ant_x || !geo->ant_y || !geo->ant_z || !geo->slant_range || !geo->start_freq)
        return SARBP_ERR_NULL_POINTER;
    if (geo->num_pulses < 1 || geo->num_pulses > p->np_ready) return SARBP_ERR_INVALID_ARGUMENT;
    if ((geo->memory != SARBP_MEMORY_HOST && geo->memory != SARBP_MEMORY_DEVICE) ||
        (image_memory != SARBP_MEMORY_HOST && image_memory != SARBP_MEMORY_DEVICE) ||
        (flags & ~(SARBP_ACCUMULATE | SARBP_CHECKED)))
        return SARBP_ERR_INVALID_ARGUMENT;
    const int np = geo->num_pulses;
    const double *gp[5];
    const int gst = device_geometry(p, geo, s, gp);
    if (gst != SARBP_OK) return gst;
    const double *ax = gp[0], *ay = gp[1], *az = gp[2], *r0 = gp[3], *f0 = gp[4];
    const sarbp_grid &g = p->desc.grid;
    const size_t img_bytes = static_cast<size_t>(g.nx) * g.ny * g.nz * cplx_bytes(p);
    void *dimg = image;
    if (image_memory == SARBP_MEMORY_HOST) {
        dimg = p->d_img;
        if (flags & SARBP_ACCUMULATE)
            SARBP_TRY_CUDA(cudaMemcpyAsync(dimg, image, img_bytes, cudaMemcpyHostToDevice, s));
    }

    BpLaunch L = launch_params(p, ax, ay, az, r0, f0, np, dimg, flags);
    cudaError_t e;
    if (p->precision == SARBP_PRECISION_FP64)
        e = launch_bp_fp64(L, p->tile, p->smem, s);
    else
        e = launch_bp_mixed(L, p->tile, (flags & SARBP_CHECKED) != 0, p->smem, s);
    SARBP_TRY_CUDA(e);
    if (image_memory == SARBP_MEMORY_HOST) {
        SARBP_TRY_CUDA(cudaMemcpyAsync(image, dimg, img_bytes, cudaMemcpyDeviceToHost, s));
        return read_errors(p, s);
    }
    if (geo->memory == SARBP_MEMORY_HOST) SARBP_TRY_CUDA(cudaStreamSynchronize(s));
    return SARBP_OK;
}

int hypotheses_impl(sarbp_plan *p, const sarbp_geometry *geo, int nhyp, void *images, int image_memory, int flags,
                    cudaStream_t s) {
    if (!geo || !images || !geo->ant_x || !geo->ant_y || !geo->ant_z || !geo->slant_range || !geo->start_freq)
        return SARBP_ERR_NULL_POINTER;
    if (p->precision != SARBP_PRECISION_MIXED) return SARBP_ERR_UNSUPPORTED;
    const sarbp_grid &g = p->desc.grid;
    if (nhyp < 1 || static_cast<long long>(nhyp) * g.nz > 65535 || geo->num_pulses < 1 ||
        geo->num_pulses > p->np_ready || (geo->memory != SARBP_MEMORY_HOST && geo->memory != SARBP_MEMORY_DEVICE) ||
        (image_memory != SARBP_MEMORY_HOST && image_memory != SARBP_MEMORY_DEVICE) || (flags & ~SARBP_ACCUMULATE))
        return SARBP_ERR_INVALID_ARGUMENT;
    const int np = geo->num_pulses;
    const size_t ngeo = static_cast<size_t>(nhyp) * np;
    const size_t img_bytes = static_cast<size_t>(nhyp) * g.nx * g.ny * g.nz * 8;
    const double *src[5] = {geo->ant_x, geo->ant_y, geo->ant_z, geo->slant_range, geo->start_freq};
    const double *dg[5];
    const size_t need = (geo->memory == SARBP_MEMORY_HOST ? 5 * ngeo * sizeof(double) : 0) +
                        (image_memory == SARBP_MEMORY_HOST ? img_bytes : 0);
    if (need > p->hyp_bytes) {
        p->bytes -= p->hyp_bytes;
        cudaFree(p->d_hyp);
        p->d_hyp = nullptr;
        p->hyp_bytes = 0;
        const int st = alloc(p, &p->d_hyp, need);
        if (st != SARBP_OK) return st;
        p->hyp_bytes = need;
    }
    unsigned char *stage = static_cast<unsigned char *>(p->d_hyp);
    if (geo->memory == SARBP_MEMORY_HOST) {
        for (int i = 0; i < 5; ++i) {
            for (size_t j = 0; j < ngeo; ++j)
                if (!std::isfinite(src[i][j])) return SARBP_ERR_NOT_FINITE;
            double *d = reinterpret_cast<double *>(stage) + i * ngeo;
            SARBP_TRY_CUDA(cudaMemcpyAsync(d, src[i], ngeo * sizeof(double), cudaMemcpyHostToDevice, s));
            dg[i] = d;
        }
        stage += 5 * ngeo * sizeof(double);
    } else {
        for (int i = 0; i < 5; ++i) dg[i] = src[i];
    }
    void *dimg = images;
    if (image_memory == SARBP_MEMORY_HOST) {
        dimg = stage;
        if (flags & SARBP_ACCUMULATE) SARBP_TRY_CUDA(cudaMemcpyAsync(dimg, images, img_bytes, cudaMemcpyHostToDevice, s));
    }
    BpLaunch L = launch_params(p, dg[0], dg[1], dg[2], dg[3], dg[4], np, dimg, flags);
    L.nhyp = nhyp;
    // geometry records of every (hypothesis, tile, pulse) from the pre-pass
    // in the plan's hypothesis records buffer, grown on demand (not while the
    // stream is being captured; a failed allocation leaves the producers
    // computing the records); plans without records (SARBP_PREGEO=0) skip it
    L.geo_tab = nullptr;
    L.geo_tab_records = 0;
    if (p->d_geotab) {
        const long long recs = static_cast<long long>(nhyp) * ((g.ny + 63) / 64) *
                               ((g.nx + 8 * p->tile.mx - 1) / (8 * p->tile.mx)) * g.nz * np;
        const size_t bytes = static_cast<size_t>(recs) * sizeof(PulseGeo);
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
            cudaGetLastError();
            cap = cudaStreamCaptureStatusActive;
        }
        if (bytes > p->hyprec_bytes && cap == cudaStreamCaptureStatusNone) {
            p->bytes -= p->hyprec_bytes;
            cudaFree(p->d_hyprec);
            p->d_hyprec = nullptr;
            p->hyprec_bytes = 0;
            if (alloc(p, &p->d_hyprec, bytes) == SARBP_OK) p->hyprec_bytes = bytes;
        }
        if (bytes <= p->hyprec_bytes) {
            L.geo_tab = p->d_hyprec;
            L.geo_tab_records = recs;
        }
    }
    SARBP_TRY_CUDA(launch_bp_mixed(L, p->tile, false, p->smem, s));
    if (image_memory == SARBP_MEMORY_HOST) {
        SARBP_TRY_CUDA(cudaMemcpyAsync(images, dimg, img_bytes, cudaMemcpyDeviceToHost, s));
        return read_errors(p, s);
    }
    if (geo->memory == SARBP_MEMORY_HOST) SARBP_TRY_CUDA(cudaStreamSynchronize(s));
    return SARBP_OK;
}

int adjoint_impl(sarbp_plan *p, const sarbp_geometry *geo, const void *grad, int grad_memory, double *grad_ant,
                 double *grad_r0, int out_memory, int flags, cudaStream_t s) {
    if (!geo || !grad || !grad_ant || !geo->ant_x || !geo->ant_y || !geo->ant_z || !geo->slant_range ||
        !geo->start_freq)
        return SARBP_ERR_NULL_POINTER;
    if (p->precision != SARBP_PRECISION_MIXED) return SARBP_ERR_UNSUPPORTED;
    if (geo->num_pulses < 1 || geo->num_pulses > p->np_ready) return SARBP_ERR_INVALID_ARGUMENT;
    if ((geo->memory != SARBP_MEMORY_HOST && geo->memory != SARBP_MEMORY_DEVICE) ||
        (grad_memory != SARBP_MEMORY_HOST && grad_memory != SARBP_MEMORY_DEVICE) ||
        (out_memory != SARBP_MEMORY_HOST && out_memory != SARBP_MEMORY_DEVICE) || (flags & ~SARBP_ACCUMULATE))
        return SARBP_ERR_INVALID_ARGUMENT;
    const int np = geo->num_pulses;
    const double *gp[5];
    const int gst = device_geometry(p, geo, s, gp);
    if (gst != SARBP_OK) return gst;
    const sarbp_grid &g = p->desc.grid;
    const size_t npix = static_cast<size_t>(g.nx) * g.ny * g.nz;
    const void *dgrad = grad;
    if (grad_memory == SARBP_MEMORY_HOST) {
        SARBP_TRY_CUDA(cudaMemcpyAsync(p->d_img, grad, npix * 8, cudaMemcpyHostToDevice, s));
        dgrad = p->d_img;
    }
    // stage depth: the deepest of 8, 4, 2, 1 pulses whose shared memory fits
    // two CTAs per SM
    TileConfig tc{p->tile.mx, 8};
    size_t smem = bp_adjoint_smem_bytes(tc, p->wsize);
    while (tc.pb > 1 && smem > 110u * 1024u) {
        tc.pb /= 2;
        smem = bp_adjoint_smem_bytes(tc, p->wsize);
    }
    if (smem > 227u * 1024u) return SARBP_ERR_UNSUPPORTED;
    BpLaunch L = launch_params(p, gp[0], gp[1], gp[2], gp[3], gp[4], np, nullptr, 0);
    const long long ntiles = bp_tile_count(L, tc);
    const size_t need = static_cast<size_t>(ntiles) * p->np_cap * 16;
    if (p->partials_bytes < need) {
        p->bytes -= p->partials_bytes;
        cudaFree(p->d_partials);
        p->d_partials = nullptr;
        p->partials_bytes = 0;
        const int st = alloc(p, &p->d_partials, need);
        if (st != SARBP_OK) return st;
        p->partials_bytes = need;
    }
    double *gant = grad_ant, *gr0 = grad_r0;
    if (out_memory == SARBP_MEMORY_HOST) {
        if (!p->d_gout) {
            const int st = alloc(p, reinterpret_cast<void **>(&p->d_gout), 4 * sizeof(double) * p->np_cap);
            if (st != SARBP_OK) return st;
        }
        gant = p->d_gout;
        gr0 = grad_r0 ? p->d_gout + 3 * np : nullptr;
        if (flags & SARBP_ACCUMULATE) {
            SARBP_TRY_CUDA(cudaMemcpyAsync(gant, grad_ant, 3 * sizeof(double) * np, cudaMemcpyHostToDevice, s));
            if (gr0) SARBP_TRY_CUDA(cudaMemcpyAsync(gr0, grad_r0, sizeof(double) * np, cudaMemcpyHostToDevice, s));
        }
    }
    SARBP_TRY_CUDA(launch_bp_adjoint(L, dgrad, p->d_partials, tc, smem, s));
    SARBP_TRY_CUDA(launch_adjoint_reduce(p->d_partials, ntiles, np, gant, gr0, (flags & SARBP_ACCUMULATE) ? 1 : 0, s));
    if (out_memory == SARBP_MEMORY_HOST) {
        SARBP_TRY_CUDA(cudaMemcpyAsync(grad_ant, gant, 3 * sizeof(double) * np, cudaMemcpyDeviceToHost, s));
        if (grad_r0) SARBP_TRY_CUDA(cudaMemcpyAsync(grad_r0, gr0, sizeof(double) * np, cudaMemcpyDeviceToHost, s));
        return read_errors(p, s);
    }
    if (geo->memory == SARBP_MEMORY_HOST || grad_memory == SARBP_MEMORY_HOST)
        SARBP_TRY_CUDA(cudaStreamSynchronize(s));
    return SARBP_OK;
}

int create_pipe(sarbp_plan *p) {
    sarbp_pipe *q = new (std::nothrow) sarbp_pipe();
    if (!q) return SARBP_ERR_OUT_OF_MEMORY;
    p->pipe = q;  // release() tears down whatever was created if a step fails
    for (cudaStream_t *s : {&q->in, &q->work, &q->out})
        SARBP_TRY_CUDA(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
    const sarbp_grid &g = p->desc.grid;
    const size_t npix = static_cast<size_t>(g.nx) * g.ny * g.nz;
    const size_t np = static_cast<size_t>(p->np_cap);
    for (int i = 0; i < sarbp_pipe::kDepth; ++i) {
        for (cudaEvent_t *e : {&q->in_ready[i], &q->work_done[i], &q->out_done[i]})
            SARBP_TRY_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        int st;
        if ((st = alloc(p, &q->d_ph[i], np * p->K * 8)) ||
            (st = alloc(p, reinterpret_cast<void **>(&q->d_geo[i]), 5 * np * sizeof(double))) ||
            (st = alloc(p, &q->d_img[i], npix * cplx_bytes(p))))
            return st;
    }
    const int st = alloc(p, reinterpret_cast<void **>(&q->d_err), sarbp_pipe::kDepth * sizeof(unsigned));
    if (st != SARBP_OK) return st;
    SARBP_TRY_CUDA(cudaMemset(q->d_err, 0, sarbp_pipe::kDepth * sizeof(unsigned)));
    SARBP_TRY_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&q->h_err), sarbp_pipe::kDepth * sizeof(unsigned),
                                 cudaHostAllocDefault));
    return SARBP_OK;
}

// Wait on the host for submission t (the oldest not yet collected) and keep
// the first error it recorded.
int collect_one(sarbp_pipe *q) {
    const unsigned long long t = q->collected + 1;
    const int slot = static_cast<int>(t % sarbp_pipe::kDepth);
    SARBP_TRY_CUDA(cudaEventSynchronize(q->out_done[slot]));
    const int st = status_from_bits(q->h_err[slot]);
    if (q->pending == SARBP_OK) q->pending = st;
    q->collected = t;
    return SARBP_OK;
}

int drain_pipe(sarbp_plan *p) {
    sarbp_pipe *q = p->pipe;
    if (!q) return SARBP_OK;
    while (q->collected < q->submitted) {
        const int st = collect_one(q);
        if (st != SARBP_OK) return st;
    }
    return SARBP_OK;
}

int focus_submit_impl(sarbp_plan *p, const sarbp_aperture *ap, void *image, unsigned long long *ticket) {
    if (!ap || !image || !ticket) return SARBP_ERR_NULL_POINTER;
    const sarbp_geometry *geo = &ap->geometry;
    if (!ap->phase_history || !geo->ant_x || !geo->ant_y || !geo->ant_z || !geo->slant_range || !geo->start_freq)
        return SARBP_ERR_NULL_POINTER;
    const int np = geo->num_pulses;
    if (np < 1 || np > p->np_cap || ap->phase_history_memory != SARBP_MEMORY_HOST ||
        geo->memory != SARBP_MEMORY_HOST)
        return SARBP_ERR_INVALID_ARGUMENT;
    int st = check_geometry_host(geo);
    if (st != SARBP_OK) return st;
    if (!p->pipe && (st = create_pipe(p)) != SARBP_OK) {
        destroy_pipe(p->pipe);
        p->pipe = nullptr;
        return st;
    }
    sarbp_pipe *q = p->pipe;
    const unsigned long long t = q->submitted + 1;
    const int slot = static_cast<int>(t % sarbp_pipe::kDepth);
    // the slot's previous user (t - kDepth) must have left the device: after
    // this, its upload, kernels and download have all completed
    while (q->collected + sarbp_pipe::kDepth < t)
        if ((st = collect_one(q)) != SARBP_OK) return st;

    // uploads
    SARBP_TRY_CUDA(cudaMemcpyAsync(q->d_ph[slot], ap->phase_history, static_cast<size_t>(np) * p->K * 8,
                                   cudaMemcpyHostToDevice, q->in));
    const double *src[5] = {geo->ant_x, geo->ant_y, geo->ant_z, geo->slant_range, geo->start_freq};
    const double *dg[5];
    for (int i = 0; i < 5; ++i) {
        double *d = q->d_geo[slot] + static_cast<size_t>(i) * p->np_cap;
        SARBP_TRY_CUDA(cudaMemcpyAsync(d, src[i], sizeof(double) * np, cudaMemcpyHostToDevice, q->in));
        dg[i] = d;
    }
    SARBP_TRY_CUDA(cudaEventRecord(q->in_ready[slot], q->in));

    // kernels: range compression into the plan's rows, then backprojection
    SARBP_TRY_CUDA(cudaStreamWaitEvent(q->work, q->in_ready[slot], 0));
    st = range_compress_impl(p, q->d_ph[slot], np, SARBP_MEMORY_DEVICE, q->work);
    if (st != SARBP_OK) return st;
    BpLaunch L = launch_params(p, dg[0], dg[1], dg[2], dg[3], dg[4], np, q->d_img[slot], 0);
    L.err = q->d_err + slot;
    SARBP_TRY_CUDA(p->precision == SARBP_PRECISION_FP64 ? launch_bp_fp64(L, p->tile, p->smem, q->work)
                                                         : launch_bp_mixed(L, p->tile, false, p->smem, q->work));
    SARBP_TRY_CUDA(cudaEventRecord(q->work_done[slot], q->work));

    // downloads: the image, then the slot's error word (cleared for reuse)
    const sarbp_grid &g = p->desc.grid;
    const size_t img_bytes = static_cast<size_t>(g.nx) * g.ny * g.nz * cplx_bytes(p);
    SARBP_TRY_CUDA(cudaStreamWaitEvent(q->out, q->work_done[slot], 0));
    SARBP_TRY_CUDA(cudaMemcpyAsync(image, q->d_img[slot], img_bytes, cudaMemcpyDeviceToHost, q->out));
    SARBP_TRY_CUDA(cudaMemcpyAsync(q->h_err + slot, q->d_err + slot, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                   q->out));
    SARBP_TRY_CUDA(cudaMemsetAsync(q->d_err + slot, 0, sizeof(unsigned), q->out));
    SARBP_TRY_CUDA(cudaEventRecord(q->out_done[slot], q->out));
    q->submitted = t;
    *ticket = t;
    return SARBP_OK;
}

int focus_wait_impl(sarbp_plan *p, unsigned long long ticket) {
    sarbp_pipe *q = p->pipe;
    const unsigned long long last = q ? q->submitted : 0;
    if (ticket == 0) ticket = last;
    if (ticket > last) return SARBP_ERR_INVALID_ARGUMENT;
    while (q && q->collected < ticket) {
        const int st = collect_one(q);
        if (st != SARBP_OK) return st;
    }
    if (!q) return SARBP_OK;
    const int st = q->pending;
    q->pending = SARBP_OK;
    return st;
}

int matched_filter_impl(sarbp_plan *p, const sarbp_aperture *ap, void *image, int image_memory, cudaStream_t s) {
    if (!ap || !image || !ap->phase_history) return SARBP_ERR_NULL_POINTER;
    const sarbp_geometry *geo = &ap->geometry;
    if (!geo->ant_x || !geo->ant_y || !geo->ant_z || !geo->slant_range || !geo->start_freq)
        return SARBP_ERR_NULL_POINTER;
    const int np = geo->num_pulses;
    if (np < 1 || np > p->np_cap ||
        (ap->phase_history_memory != SARBP_MEMORY_HOST && ap->phase_history_memory != SARBP_MEMORY_DEVICE) ||
        (geo->memory != SARBP_MEMORY_HOST && geo->memory != SARBP_MEMORY_DEVICE) ||
        (image_memory != SARBP_MEMORY_HOST && image_memory != SARBP_MEMORY_DEVICE))
        return SARBP_ERR_INVALID_ARGUMENT;
    const bool weighted = p->desc.window != SARBP_WINDOW_NONE || !p->range_w.empty();
    if (weighted && (!p->d_win || p->win_stale)) {
        const std::vector<double> w = range_weights(p->desc, p->range_w.empty() ? nullptr : p->range_w.data());
        if (!p->d_win) SARBP_TRY(alloc(p, reinterpret_cast<void **>(&p->d_win), w.size() * sizeof(double)));
        SARBP_TRY_CUDA(cudaMemcpy(p->d_win, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice));
        p->win_stale = false;
    }
    const void *ph = ap->phase_history;
    if (ap->phase_history_memory == SARBP_MEMORY_HOST) {
        SARBP_TRY_CUDA(cudaMemcpyAsync(p->d_ph, ph, static_cast<size_t>(np) * p->K * 8, cudaMemcpyHostToDevice, s));
        ph = p->d_ph;
    }
    const double *gp[5];
    SARBP_TRY(device_geometry(p, geo, s, gp));
    const sarbp_grid &g = p->desc.grid;
    const size_t img_bytes = static_cast<size_t>(g.nx) * g.ny * g.nz * cplx_bytes(p);
    void *dimg = image_memory == SARBP_MEMORY_HOST ? p->d_img : image;
    MfLaunch M{};
    M.ax = gp[0];
    M.ay = gp[1];
    M.az = gp[2];
    M.r0 = gp[3];
    M.f0 = gp[4];
    M.np = np;
    M.K = p->K;
    M.df = kClight / (2.0 * p->desc.max_wr);
    M.nx = g.nx;
    M.ny = g.ny;
    M.nz = g.nz;
    M.left = p->left;
    M.bottom = p->bottom;
    M.zlow = p->zlow;
    M.dx = p->dx;
    M.dy = p->dy;
    M.dz = p->dz;
    M.img = dimg;
    SARBP_TRY_CUDA(launch_mf(ph, weighted ? p->d_win : nullptr, M, p->precision == SARBP_PRECISION_FP64, s));
    if (image_memory == SARBP_MEMORY_HOST) {
        SARBP_TRY_CUDA(cudaMemcpyAsync(image, dimg, img_bytes, cudaMemcpyDeviceToHost, s));
        return read_errors(p, s);
    }
    if (geo->memory == SARBP_MEMORY_HOST || ap->phase_history_memory == SARBP_MEMORY_HOST)
        SARBP_TRY_CUDA(cudaStreamSynchronize(s));
    return SARBP_OK;
}

}  // namespace

extern "C" {

int sarbp_abi_version(void) { return SARBP_ABI_VERSION; }

const char *sarbp_status_string(int status) {
    switch (status) {
        case SARBP_OK: return "ok";
        case SARBP_ERR_INVALID_ARGUMENT: return "invalid argument";
        case SARBP_ERR_NULL_POINTER: return "null pointer";
        case SARBP_ERR_UNSUPPORTED: return "unsupported configuration";
        case SARBP_ERR_OUT_OF_MEMORY: return "out of memory";
        case SARBP_ERR_CUDA: return "CUDA runtime error";
        case SARBP_ERR_CUFFT: return "cuFFT error";
        case SARBP_ERR_NOT_FINITE: return "non-finite geometry";
        case SARBP_ERR_KERNEL_TIMEOUT: return "device wait timed out";
        case SARBP_ERR_KERNEL_BOUNDS: return "kernel index out of range (clamped)";
        case SARBP_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

int sarbp_plan_create(const sarbp_plan_desc *desc, sarbp_plan **out) {
    NvtxRange range("sarbp_plan_create");
    if (!out) return SARBP_ERR_NULL_POINTER;
    *out = nullptr;
    int st = validate_desc(desc);
    if (st != SARBP_OK) return st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SARBP_ERR_NO_DEVICE;
    }
    int dev = desc->device;
    if (dev < 0) SARBP_TRY_CUDA(cudaGetDevice(&dev));
    if (dev >= ndev) return SARBP_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(dev);
    SARBP_TRY_CUDA(guard.status);

    sarbp_plan *p = new (std::nothrow) sarbp_plan();
    if (!p) return SARBP_ERR_OUT_OF_MEMORY;
    p->desc = *desc;
    p->device = dev;
    p->K = desc->num_range_samples;
    p->np_cap = desc->num_pulses;
    p->nfft = desc->nfft;
    p->precision = desc->precision;
    p->lambda = static_cast<double>(desc->nfft) / desc->max_wr;
    const sarbp_grid &g = desc->grid;
    axis(g.nx, g.x0, g.wx, &p->left, &p->dx);
    axis(g.ny, g.y0, g.wy, &p->bottom, &p->dy);
    axis(g.nz, g.z0, g.wz, &p->zlow, &p->dz);
    st = choose_tile(p);
    if (st != SARBP_OK) {
        delete p;
        return st;
    }
    {
        int W, wsize;
        double hd;
        tile_window(p->lambda, p->dx, p->dy, p->tile.mx, &W, &wsize, &hd);
        near_field_consts(hd, &p->near_hd16, &p->near_coef);
    }
    p->guard = p->wsize + 2;
    p->row_stride = static_cast<long long>(p->nfft) + 2LL * p->guard;
    const size_t cb = cplx_bytes(p);
    const size_t entry = p->precision == SARBP_PRECISION_FP64 ? 32 : 16;
    const size_t npix = static_cast<size_t>(g.nx) * g.ny * g.nz;
    const size_t np = static_cast<size_t>(p->np_cap);
    if ((st = alloc(p, &p->d_ph, np * p->K * 8)) ||
        (st = alloc(p, reinterpret_cast<void **>(&p->d_geo), 5 * np * sizeof(double))) ||
        (st = alloc(p, &p->d_fft, np * p->nfft * cb)) ||
        (st = alloc(p, &p->d_pairs, np * static_cast<size_t>(p->row_stride) * entry)) ||
        (st = alloc(p, &p->d_fac, static_cast<size_t>(p->K) * cb)) || (st = alloc(p, &p->d_img, npix * cb)) ||
        (st = alloc(p, reinterpret_cast<void **>(&p->d_err), sizeof(unsigned)))) {
        release(p);
        return st;
    }
    // partial-sum slots for launches split over the resident CTAs (two tiles
    // per CTA); without them every launch runs one CTA per tile
    p->sk_resident = p->precision == SARBP_PRECISION_FP64 ? bp_fp64_resident(p->tile, p->smem)
                                                          : bp_mixed_resident(p->tile, p->smem);
    if (p->sk_resident > 0) {
        const size_t sk = 2 * static_cast<size_t>(p->sk_resident) * (8 * p->tile.mx) * 64 * cb;
        if (alloc(p, &p->d_sk, sk) == SARBP_OK) {
            p->sk_bytes = sk;
        } else {
            p->sk_resident = 0;
        }
    }
    // geometry records of a single-image launch from a pre-pass kernel
    // (environment SARBP_PREGEO=0: computed by the producing lanes instead)
    if (p->precision == SARBP_PRECISION_MIXED) {
        const char *env = std::getenv("SARBP_PREGEO");
        if (!(env && std::strcmp(env, "0") == 0)) {
            const long long recs = static_cast<long long>((g.ny + 63) / 64) *
                                   ((g.nx + 8 * p->tile.mx - 1) / (8 * p->tile.mx)) * g.nz * p->np_cap;
            if (alloc(p, &p->d_geotab, static_cast<size_t>(recs) * sizeof(PulseGeo)) == SARBP_OK)
                p->geotab_records = recs;
        }
    }
    if (cudaMemset(p->d_pairs, 0, np * static_cast<size_t>(p->row_stride) * entry) != cudaSuccess ||
        cudaMemset(p->d_fft, 0, np * p->nfft * cb) != cudaSuccess ||
        cudaMemset(p->d_err, 0, sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        release(p);
        return SARBP_ERR_CUDA;
    }
    // fac[k] = w_k / nfft * exp(+j 2 pi ((k s) mod nfft) / nfft), s = (nfft+1)/2
    st = upload_range_factors(p);
    if (st != SARBP_OK) {
        release(p);
        return st;
    }
    // fused range compression when the shape has a kernel (environment
    // SARBP_RC=cufft keeps the taper / cuFFT / pair-row path)
    {
        const int K = p->K, N = p->nfft;
        const int R = (N % K == 0) ? N / K : 0;
        const char *env = std::getenv("SARBP_RC");
        const bool want = !(env && std::strcmp(env, "cufft") == 0);
        size_t rc_smem = 0;
        std::vector<float> tab;
        int dev_smem = 0, sms = 0;
        cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaGetLastError();
        if (want && p->precision == SARBP_PRECISION_MIXED && R >= 1 && rc_fused_shape(K, R, &rc_smem, &tab) &&
            rc_smem <= static_cast<size_t>(dev_smem)) {
            if (alloc(p, &p->d_rctab, tab.size() * sizeof(float)) == SARBP_OK &&
                cudaMemcpy(p->d_rctab, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess) {
                p->rc_R = R;
                // CTAs resident at once: the kernel loops over pulses
                const int per_sm = rc_smem > 0 ? static_cast<int>((228u * 1024u) / (rc_smem + 1024u)) : 1;
                p->rc_grid = (sms > 0 ? sms : 148) * (per_sm > 0 ? (per_sm < 4 ? per_sm : 4) : 1);
            } else {
                cudaGetLastError();
                cudaFree(p->d_rctab);
                p->d_rctab = nullptr;
            }
        }
    }
    const cufftResult r = cufftPlan1d(&p->fft, p->nfft, p->precision == SARBP_PRECISION_FP64 ? CUFFT_Z2Z : CUFFT_C2C,
                                      p->np_cap);
    if (r != CUFFT_SUCCESS) {
        release(p);
        return from_cufft(r);
    }
    p->fft_ok = true;
    size_t ws = 0;
    if (cufftGetSize(p->fft, &ws) == CUFFT_SUCCESS) p->bytes += ws;
    *out = p;
    return SARBP_OK;
}

int sarbp_plan_destroy(sarbp_plan *plan) {
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    release(plan);
    return SARBP_OK;
}

int sarbp_plan_workspace_bytes(const sarbp_plan *plan, size_t *bytes) {
    if (!plan || !bytes) return SARBP_ERR_NULL_POINTER;
    *bytes = plan->bytes;
    return SARBP_OK;
}

int sarbp_plan_get_info(const sarbp_plan *plan, sarbp_plan_info *info) {
    if (!plan || !info) return SARBP_ERR_NULL_POINTER;
    std::memset(info, 0, sizeof(*info));
    const sarbp_grid &g = plan->desc.grid;
    info->tile_mx = plan->tile.mx;
    info->stage_pulses = plan->tile.pb;
    info->window_bins = plan->wsize;
    info->resident_ctas = plan->sk_resident;
    info->tiles = static_cast<long long>((g.ny + 63) / 64) * ((g.nx + 8 * plan->tile.mx - 1) / (8 * plan->tile.mx)) *
                  g.nz;
    info->smem_bytes = static_cast<long long>(plan->smem);
    info->kernels_per_backproject = (plan->d_sk && plan->sk_resident > 0 && info->tiles % plan->sk_resident != 0) ? 2 : 1;
    info->fused_range_compression = plan->d_rctab ? 1 : 0;
    return SARBP_OK;
}

int sarbp_test_fail_device_alloc(int after) {
    host::g_alloc_countdown.store(after < 0 ? -1 : after);
    return SARBP_OK;
}

int sarbp_test_drop_window_copy(sarbp_plan *plan, int pulse) {
    if (!plan) return SARBP_ERR_NULL_POINTER;
    if (plan->precision != SARBP_PRECISION_MIXED) return SARBP_ERR_UNSUPPORTED;
    SARBP_TRY(drain_pipe(plan));
    plan->drop_pulse = pulse < 0 ? -1 : pulse;
    return SARBP_OK;
}

int sarbp_plan_set_range_weights(sarbp_plan *plan, const double *weights) {
    NvtxRange range("sarbp_plan_set_range_weights");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    if (weights)
        for (int k = 0; k < 2 * plan->K; ++k)
            if (!std::isfinite(weights[k])) return SARBP_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    SARBP_TRY(drain_pipe(plan));
    // the kernels of earlier calls on any stream may still read the table
    SARBP_TRY_CUDA(cudaDeviceSynchronize());
    if (weights)
        plan->range_w.assign(weights, weights + 2 * static_cast<size_t>(plan->K));
    else
        plan->range_w.clear();
    plan->win_stale = true;
    return upload_range_factors(plan);
}

int sarbp_range_compress(sarbp_plan *plan, const void *phase_history, int num_pulses, int memory, void *stream) {
    NvtxRange range("sarbp_range_compress");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    SARBP_TRY(drain_pipe(plan));
    return range_compress_impl(plan, phase_history, num_pulses, memory, static_cast<cudaStream_t>(stream));
}

int sarbp_get_range_profiles(sarbp_plan *plan, void *out, int memory, void *stream) {
    NvtxRange range("sarbp_get_range_profiles");
    if (!plan || !out) return SARBP_ERR_NULL_POINTER;
    if (memory != SARBP_MEMORY_HOST && memory != SARBP_MEMORY_DEVICE) return SARBP_ERR_INVALID_ARGUMENT;
    if (plan->np_ready < 1) return SARBP_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    SARBP_TRY(drain_pipe(plan));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t bytes = static_cast<size_t>(plan->np_ready) * plan->nfft * cplx_bytes(plan);
    if (plan->d_rctab)  // fused range compression keeps the profiles only in the pair rows
        SARBP_TRY_CUDA(launch_pairs_to_rc(plan->d_pairs, plan->d_fft, plan->nfft, plan->np_ready, plan->row_stride,
                                          plan->guard, s));
    SARBP_TRY_CUDA(cudaMemcpyAsync(out, plan->d_fft, bytes,
                                   memory == SARBP_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                   s));
    if (memory == SARBP_MEMORY_HOST) SARBP_TRY_CUDA(cudaStreamSynchronize(s));
    return SARBP_OK;
}

int sarbp_backproject(sarbp_plan *plan, const sarbp_geometry *geometry, void *image, int image_memory, int flags,
                      void *stream) {
    NvtxRange range("sarbp_backproject");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    SARBP_TRY(drain_pipe(plan));
    return backproject_impl(plan, geometry, image, image_memory, flags, static_cast<cudaStream_t>(stream));
}

int sarbp_focus(sarbp_plan *plan, const sarbp_aperture *ap, void *image, int image_memory, void *stream) {
    NvtxRange range("sarbp_focus");
    if (!plan || !ap) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    SARBP_TRY(drain_pipe(plan));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    {
        NvtxRange rc("range compression");
        const int st = range_compress_impl(plan, ap->phase_history, ap->geometry.num_pulses,
                                           ap->phase_history_memory, s);
        if (st != SARBP_OK) return st;
    }
    NvtxRange bp("backprojection");
    return backproject_impl(plan, &ap->geometry, image, image_memory, 0, s);
}

int sarbp_focus_image(const sarbp_plan_desc *desc, const sarbp_aperture *ap, void *image, int image_memory) {
    if (!desc || !ap) return SARBP_ERR_NULL_POINTER;
    sarbp_plan *plan = nullptr;
    int st = sarbp_plan_create(desc, &plan);
    if (st != SARBP_OK) return st;
    st = sarbp_focus(plan, ap, image, image_memory, nullptr);
    if (st == SARBP_OK) st = sarbp_plan_check(plan, nullptr);
    sarbp_plan_destroy(plan);
    return st;
}

int sarbp_backproject_hypotheses(sarbp_plan *plan, const sarbp_geometry *geometry, int num_hypotheses, void *images,
                                 int image_memory, int flags, void *stream) {
    NvtxRange range("sarbp_backproject_hypotheses");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    SARBP_TRY(drain_pipe(plan));
    return hypotheses_impl(plan, geometry, num_hypotheses, images, image_memory, flags,
                           static_cast<cudaStream_t>(stream));
}

int sarbp_backproject_adjoint(sarbp_plan *plan, const sarbp_geometry *geometry, const void *grad_image,
                              int grad_memory, double *grad_ant, double *grad_r0, int out_memory, int flags,
                              void *stream) {
    NvtxRange range("sarbp_backproject_adjoint");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    SARBP_TRY(drain_pipe(plan));
    return adjoint_impl(plan, geometry, grad_image, grad_memory, grad_ant, grad_r0, out_memory, flags,
                        static_cast<cudaStream_t>(stream));
}

int sarbp_focus_submit(sarbp_plan *plan, const sarbp_aperture *aperture, void *image, unsigned long long *ticket) {
    NvtxRange range("sarbp_focus_submit");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    return focus_submit_impl(plan, aperture, image, ticket);
}

int sarbp_focus_wait(sarbp_plan *plan, unsigned long long ticket) {
    NvtxRange range("sarbp_focus_wait");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    return focus_wait_impl(plan, ticket);
}

int sarbp_matched_filter(sarbp_plan *plan, const sarbp_aperture *aperture, void *image, int image_memory,
                         void *stream) {
    NvtxRange range("sarbp_matched_filter");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    SARBP_TRY(drain_pipe(plan));
    return matched_filter_impl(plan, aperture, image, image_memory, static_cast<cudaStream_t>(stream));
}

int sarbp_plan_check(sarbp_plan *plan, void *stream) {
    NvtxRange range("sarbp_plan_check");
    if (!plan) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(plan->device);
    SARBP_TRY_CUDA(guard.status);
    return read_errors(plan, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
