// batch.cu -- batches of independent scenes of uneven sizes (sarbp_batch_*).
//
// Each scene keeps its own range-compression buffers and cuFFT plan; a
// device-resident scene table (BatchScene) holds every per-call pointer, so
// the work of one call -- table upload, batched taper/twiddle/zero-pad, one
// FFT per scene, batched pair rows, ONE backprojection launch over the
// (tile, pulse-stage) units of all scenes split evenly over the resident
// CTAs, the fix-up of split tiles, and the read-back of per-image completion
// times -- is captured once as a CUDA graph and replayed on later calls with
// only the table contents changed.  Changing a scene's pulse count changes
// the unit count and re-captures.  The reference has no batch mode: its
// cuda_focus_SAR_image focuses one aperture per call, allocating and freeing
// everything each time (cuda_sar_focusing.hpp:526-723).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "bp_common.cuh"
#include "bp_tile.cuh"
#include "host_common.h"
#include "sarbp_internal.h"

using namespace sarbp;
using namespace sarbp::host;

struct sarbp_batch {
    int device = 0;
    int n = 0;
    std::vector<sarbp_plan_desc> desc;
    std::vector<void *> d_pairs, d_fft, d_fac;
    std::vector<cufftHandle> fft;
    std::vector<char> fft_ok;
    std::vector<int> guard;
    std::vector<long long> row_stride;
    std::vector<double> lambda, dx, dy, dz, left, bottom, zlow;
    void *fft_work = nullptr;
    std::vector<void *> rctab;     // per scene: fused range-compression table (null: cuFFT path)
    std::vector<int> rc_R;         // per scene: nfft / K of the fused path
    std::vector<void *> rc_tables; // the distinct tables (one per (K, R))
    int rc_grid = 0;
    // tile shape and the per-scene windows it implies
    TileConfig tile{0, 0};
    size_t smem = 0;
    int resident = 0, max_wsize = 0;
    int per_tile = -1;  // -1: choose per call (split below four waves of tiles)
    std::vector<int> W, wsize;
    std::vector<double> near_hd16, near_coef;
    // per call
    BatchScene *h_table = nullptr, *d_table = nullptr;  // h_table page-locked
    void *d_partial = nullptr;
    size_t partial_bytes = 0;
    // pre-pass geometry records of every scene, [scene][tile][pulse] at the
    // current tile shape (null: the producers compute them)
    void *d_geotab = nullptr;
    size_t geotab_bytes = 0;
    bool records_now = false;    // this call's table slots carry record rows
    long long max_records = 0;   // the largest scene's tiles x pulses in this call
    unsigned long long *d_times = nullptr, *h_times = nullptr;  // [n] completion, [n] start; h page-locked
    unsigned *d_err = nullptr, *h_err = nullptr;
    long long units = 0, tiles = 0;
    std::vector<int> np_now;
    // graph
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<int> graph_np;
    bool graph_valid = false, use_graph = true;
    cudaEvent_t done_ev = nullptr;
    bool launched = false;
    size_t bytes = 0;
};

namespace {

__global__ void stamp_kernel(unsigned long long *t) { *t = global_timer_ns(); }

int balloc(sarbp_batch *b, void **p, size_t bytes) {
    const cudaError_t e = host::device_malloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return from_cuda(e);
    }
    b->bytes += bytes;
    return SARBP_OK;
}

void drop_graph(sarbp_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_valid = false;
}

void release(sarbp_batch *b) {
    if (!b) return;
    if (b->launched && b->done_ev) cudaEventSynchronize(b->done_ev);
    drop_graph(b);
    for (int i = 0; i < b->n; ++i) {
        if (i < static_cast<int>(b->fft_ok.size()) && b->fft_ok[i]) cufftDestroy(b->fft[i]);
        if (i < static_cast<int>(b->d_pairs.size())) cudaFree(b->d_pairs[i]);
        if (i < static_cast<int>(b->d_fft.size())) cudaFree(b->d_fft[i]);
        if (i < static_cast<int>(b->d_fac.size())) cudaFree(b->d_fac[i]);
    }
    cudaFree(b->fft_work);
    for (void *t : b->rc_tables) cudaFree(t);
    cudaFree(b->d_table);
    cudaFree(b->d_partial);
    cudaFree(b->d_geotab);
    cudaFree(b->d_times);
    cudaFree(b->d_err);
    if (b->h_table) cudaFreeHost(b->h_table);
    if (b->h_times) cudaFreeHost(b->h_times);
    if (b->h_err) cudaFreeHost(b->h_err);
    if (b->done_ev) cudaEventDestroy(b->done_ev);
    if (b->cap) cudaStreamDestroy(b->cap);
    cudaGetLastError();
    delete b;
}

// Windows, shared memory and resident CTAs for tile shape tc; false if the
// stage does not fit one CTA's shared memory.
bool configure(sarbp_batch *b, const TileConfig &tc) {
    std::vector<int> W(b->n), ws(b->n);
    std::vector<double> h16(b->n), hc(b->n);
    int wmax = 0;
    for (int i = 0; i < b->n; ++i) {
        double hd;
        tile_window(b->lambda[i], b->dx[i], b->dy[i], tc.mx, &W[i], &ws[i], &hd);
        near_field_consts(hd, &h16[i], &hc[i]);
        if (ws[i] + 2 > b->guard[i] || ws[i] > (1 << 16)) return false;
        wmax = ws[i] > wmax ? ws[i] : wmax;
    }
    const size_t smem = bp_mixed_smem_bytes(tc, wmax);
    if (smem > 227u * 1024u) return false;
    const int res = bp_mixed_batch_resident(tc, smem);
    if (res < 1) return false;
    const size_t need = 2 * static_cast<size_t>(res) * (8 * tc.mx) * 64 * sizeof(float2);
    if (need > b->partial_bytes) {
        cudaFree(b->d_partial);
        b->d_partial = nullptr;
        b->partial_bytes = 0;
        if (balloc(b, &b->d_partial, need) != SARBP_OK) return false;
        b->partial_bytes = need;
    }
    // room for every scene's records at this tile shape (environment
    // SARBP_PREGEO=0, or no room: the producers compute the records)
    const char *pregeo_env = std::getenv("SARBP_PREGEO");
    if (!(pregeo_env && std::strcmp(pregeo_env, "0") == 0)) {
        size_t recs = 0;
        for (int i = 0; i < b->n; ++i) {
            const sarbp_grid &g = b->desc[i].grid;
            recs += static_cast<size_t>((g.ny + 63) / 64) * ((g.nx + 8 * tc.mx - 1) / (8 * tc.mx)) * g.nz *
                    static_cast<size_t>(b->desc[i].num_pulses);
        }
        const size_t need = recs * sizeof(PulseGeo);
        if (need > b->geotab_bytes) {
            cudaFree(b->d_geotab);
            b->d_geotab = nullptr;
            b->geotab_bytes = 0;
            if (balloc(b, &b->d_geotab, need) == SARBP_OK) b->geotab_bytes = need;
        }
    }
    b->tile = tc;
    b->smem = smem;
    b->resident = res;
    b->max_wsize = wmax;
    b->W = W;
    b->wsize = ws;
    b->near_hd16 = h16;
    b->near_coef = hc;
    drop_graph(b);
    return true;
}

int choose_default_tile(sarbp_batch *b) {
    // 64-row tiles unless padding every scene's rows to 64 instead of 32 adds
    // more than 15% pixel-pulses over the batch (the plan's rule, api.cu)
    double pad64 = 0.0, pad32 = 0.0;
    for (int s = 0; s < b->n; ++s) {
        const sarbp_grid &g = b->desc[s].grid;
        const double w = static_cast<double>(g.ny) * g.nz * b->desc[s].num_pulses;
        pad64 += w * ((g.nx + 63) / 64 * 64);
        pad32 += w * ((g.nx + 31) / 32 * 32);
    }
    const bool tall_tiles = pad64 <= 1.15 * pad32;
    for (const size_t limit : {110u * 1024u, 227u * 1024u})
        for (int i = 0; i < bp_batch_tile_count; ++i) {
            const TileConfig tc = bp_batch_tiles[i];
            if (tc.mx == 8 && !tall_tiles) continue;
            // quick shared-memory check before configure allocates anything
            int wmax = 0;
            for (int s = 0; s < b->n; ++s) {
                int W, ws;
                double hd;
                tile_window(b->lambda[s], b->dx[s], b->dy[s], tc.mx, &W, &ws, &hd);
                wmax = ws > wmax ? ws : wmax;
            }
            if (bp_mixed_smem_bytes(tc, wmax) > limit) continue;
            if (configure(b, tc)) return SARBP_OK;
        }
    return SARBP_ERR_UNSUPPORTED;
}

// Scene table of one call into the page-locked host copy.
int fill_table(sarbp_batch *b, const sarbp_aperture *aps, void *const *images) {
    long long units = 0, tiles = 0;
    for (int i = 0; i < b->n; ++i) {
        const sarbp_aperture &a = aps[i];
        const sarbp_geometry &g = a.geometry;
        if (!a.phase_history || !g.ant_x || !g.ant_y || !g.ant_z || !g.slant_range || !g.start_freq || !images[i])
            return SARBP_ERR_NULL_POINTER;
        if (a.phase_history_memory != SARBP_MEMORY_DEVICE || g.memory != SARBP_MEMORY_DEVICE || g.num_pulses < 1 ||
            g.num_pulses > b->desc[i].num_pulses)
            return SARBP_ERR_INVALID_ARGUMENT;
        const sarbp_plan_desc &d = b->desc[i];
        BatchScene &T = b->h_table[i];
        std::memset(&T, 0, sizeof(T));
        BpLaunch &L = T.L;
        L.drop_pulse = -1;
        L.pairs = b->d_pairs[i];
        L.row_stride = b->row_stride[i];
        L.guard = b->guard[i];
        L.ax = g.ant_x;
        L.ay = g.ant_y;
        L.az = g.ant_z;
        L.r0 = g.slant_range;
        L.f0 = g.start_freq;
        L.np = g.num_pulses;
        L.nfft = d.nfft;
        L.lambda = b->lambda[i];
        L.half_nfft = 0.5 * d.nfft;
        L.nx = d.grid.nx;
        L.ny = d.grid.ny;
        L.nz = d.grid.nz;
        L.left = b->left[i];
        L.bottom = b->bottom[i];
        L.zlow = b->zlow[i];
        L.dx = b->dx[i];
        L.dy = b->dy[i];
        L.dz = b->dz[i];
        L.W = b->W[i];
        L.wsize = b->wsize[i];
        L.near_hd16 = b->near_hd16[i];
        L.near_coef = b->near_coef[i];
        L.img = images[i];
        L.accumulate = 0;
        L.err = b->d_err;
        L.nhyp = 1;
        T.fused = b->rctab[i] ? 1 : 0;
        T.ph = a.phase_history;
        T.fac = b->d_fac[i];
        T.fft = b->d_fft[i];
        T.K = d.num_range_samples;
        T.row_stride = b->row_stride[i];
        const tile::TileGrid tg = tile::tile_grid(L, 8 * b->tile.mx, b->tile.pb);
        T.unit_begin = units;
        T.tile_begin = tiles;
        units += tg.units;
        tiles += tg.tiles;
        b->np_now[i] = g.num_pulses;
    }
    b->units = units;
    b->tiles = tiles;
    // record rows of every scene at this call's pulse counts, [tile][pulse]
    // per scene, back to back; all scenes or none
    long long off = 0, biggest = 0;
    for (int i = 0; i < b->n; ++i) {
        const BpLaunch &L = b->h_table[i].L;
        const long long r = tile::tile_grid(L, 8 * b->tile.mx, 1).tiles * L.np;
        off += r;
        biggest = r > biggest ? r : biggest;
    }
    b->records_now = b->d_geotab && static_cast<size_t>(off) * sizeof(PulseGeo) <= b->geotab_bytes &&
                     biggest < 0x7fffffffLL;
    b->max_records = biggest;
    off = 0;
    for (int i = 0; i < b->n; ++i) {
        BpLaunch &L = b->h_table[i].L;
        const long long r = tile::tile_grid(L, 8 * b->tile.mx, 1).tiles * L.np;
        L.geo_tab = b->records_now ? static_cast<void *>(static_cast<PulseGeo *>(b->d_geotab) + off) : nullptr;
        L.geo_tab_records = b->records_now ? r : 0;
        off += r;
    }
    return SARBP_OK;
}

bool per_tile_now(const sarbp_batch *b) {
    return b->per_tile >= 0 ? b->per_tile != 0 : b->tiles >= 4LL * b->resident;
}

// The work of one call on stream s (captured into the graph, or run eagerly).
int enqueue(sarbp_batch *b, cudaStream_t s) {
    const int n = b->n;
    SARBP_TRY_CUDA(cudaMemcpyAsync(b->d_table, b->h_table, n * sizeof(BatchScene), cudaMemcpyHostToDevice, s));
    SARBP_TRY_CUDA(cudaMemsetAsync(b->d_times, 0, (n + 1) * sizeof(unsigned long long), s));
    stamp_kernel<<<1, 1, 0, s>>>(b->d_times + n);
    SARBP_TRY_CUDA(cudaGetLastError());
    if (b->records_now)
        SARBP_TRY_CUDA(launch_geo_records_batch(b->d_table, n, b->tile.mx, b->max_records, s));
    SARBP_TRY_CUDA(launch_rc_prep_batch(b->d_table, n, s));
    for (int i = 0; i < n; ++i) {
        if (b->rctab[i]) {
            SARBP_TRY_CUDA(launch_rc_fused_scene(b->d_table + i, b->rctab[i], b->desc[i].num_range_samples,
                                                 b->rc_R[i], b->rc_grid, s));
            continue;
        }
        const cufftResult r0 = cufftSetStream(b->fft[i], s);
        if (r0 != CUFFT_SUCCESS) return from_cufft(r0);
        const cufftResult r1 = cufftExecC2C(b->fft[i], static_cast<cufftComplex *>(b->d_fft[i]),
                                            static_cast<cufftComplex *>(b->d_fft[i]), CUFFT_INVERSE);
        if (r1 != CUFFT_SUCCESS) return from_cufft(r1);
    }
    SARBP_TRY_CUDA(launch_rc_pairs_batch(b->d_table, n, s));
    SARBP_TRY_CUDA(launch_bp_mixed_batch(b->d_table, n, b->units, b->tiles, b->tile, b->smem, b->resident,
                                         b->d_partial, b->d_times, s, b->max_wsize, per_tile_now(b),
                                         b->records_now ? b->d_geotab : nullptr));
    SARBP_TRY_CUDA(cudaMemcpyAsync(b->h_times, b->d_times, (n + 1) * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, s));
    SARBP_TRY_CUDA(cudaMemcpyAsync(b->h_err, b->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    SARBP_TRY_CUDA(cudaMemsetAsync(b->d_err, 0, sizeof(unsigned), s));
    return SARBP_OK;
}

int capture(sarbp_batch *b) {
    drop_graph(b);
    SARBP_TRY_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const int st = enqueue(b, b->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &g);
    if (st != SARBP_OK || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return st != SARBP_OK ? st : SARBP_ERR_CUDA;
    }
    b->graph = g;
    const cudaError_t ei = cudaGraphInstantiate(&b->exec, g, 0);
    if (ei != cudaSuccess) {
        cudaGetLastError();
        drop_graph(b);
        return SARBP_ERR_CUDA;
    }
    b->graph_valid = true;
    b->graph_np = b->np_now;
    return SARBP_OK;
}

int focus_impl(sarbp_batch *b, const sarbp_aperture *aps, void *const *images, cudaStream_t s) {
    if (!aps || !images) return SARBP_ERR_NULL_POINTER;
    // the previous call must have read the table before it is rewritten
    if (b->launched) SARBP_TRY_CUDA(cudaEventSynchronize(b->done_ev));
    SARBP_TRY(fill_table(b, aps, images));
    if (b->use_graph && (!b->graph_valid || b->graph_np != b->np_now)) {
        if (capture(b) != SARBP_OK) b->use_graph = false;  // run the same work eagerly from now on
    }
    if (b->use_graph) {
        SARBP_TRY_CUDA(cudaGraphLaunch(b->exec, s));
    } else {
        SARBP_TRY(enqueue(b, s));
    }
    SARBP_TRY_CUDA(cudaEventRecord(b->done_ev, s));
    b->launched = true;
    return SARBP_OK;
}

int wait_impl(sarbp_batch *b, double *image_ms) {
    if (!b->launched) return SARBP_OK;
    SARBP_TRY_CUDA(cudaEventSynchronize(b->done_ev));
    if (image_ms)
        for (int i = 0; i < b->n; ++i) {
            const unsigned long long t0 = b->h_times[b->n], t = b->h_times[i];
            image_ms[i] = t >= t0 ? static_cast<double>(t - t0) * 1.0e-6 : 0.0;
        }
    return status_from_bits(*b->h_err);
}

}  // namespace

extern "C" {

int sarbp_batch_create(const sarbp_plan_desc *descs, int num_scenes, sarbp_batch **out) {
    NvtxRange range("sarbp_batch_create");
    if (!out || !descs) return SARBP_ERR_NULL_POINTER;
    *out = nullptr;
    if (num_scenes < 1 || num_scenes > 65535) return SARBP_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < num_scenes; ++i) {
        SARBP_TRY(validate_desc(&descs[i]));
        if (descs[i].precision != SARBP_PRECISION_MIXED) return SARBP_ERR_UNSUPPORTED;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SARBP_ERR_NO_DEVICE;
    }
    int dev = descs[0].device;
    if (dev < 0) SARBP_TRY_CUDA(cudaGetDevice(&dev));
    if (dev >= ndev) return SARBP_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(dev);
    SARBP_TRY_CUDA(guard.status);

    sarbp_batch *b = new (std::nothrow) sarbp_batch();
    if (!b) return SARBP_ERR_OUT_OF_MEMORY;
    b->device = dev;
    b->n = num_scenes;
    b->desc.assign(descs, descs + num_scenes);
    const int n = num_scenes;
    b->d_pairs.assign(n, nullptr);
    b->d_fft.assign(n, nullptr);
    b->d_fac.assign(n, nullptr);
    b->fft.assign(n, 0);
    b->fft_ok.assign(n, 0);
    b->guard.assign(n, 0);
    b->row_stride.assign(n, 0);
    b->np_now.assign(n, 0);
    for (auto *v : {&b->lambda, &b->dx, &b->dy, &b->dz, &b->left, &b->bottom, &b->zlow}) v->assign(n, 0.0);
    b->rctab.assign(n, nullptr);
    b->rc_R.assign(n, 0);
    int st = SARBP_OK;
    size_t work = 0;
    // fused range compression where the shape has a kernel (environment
    // SARBP_RC=cufft keeps the cuFFT path); one table per distinct (K, R)
    const char *rc_env = std::getenv("SARBP_RC");
    const bool want_fused = !(rc_env && std::strcmp(rc_env, "cufft") == 0);
    int dev_smem = 0, sms = 0;
    cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    b->rc_grid = 2 * (sms > 0 ? sms : 148);
    std::vector<std::pair<long long, void *>> tab_of;  // key K * 64 + R
    for (int i = 0; i < n && st == SARBP_OK; ++i) {
        const sarbp_plan_desc &d = descs[i];
        b->lambda[i] = static_cast<double>(d.nfft) / d.max_wr;
        axis(d.grid.nx, d.grid.x0, d.grid.wx, &b->left[i], &b->dx[i]);
        axis(d.grid.ny, d.grid.y0, d.grid.wy, &b->bottom[i], &b->dy[i]);
        axis(d.grid.nz, d.grid.z0, d.grid.wz, &b->zlow[i], &b->dz[i]);
        // rows guarded for the largest tile shape any autotuning may pick
        int mx_max = 1;
        for (int t = 0; t < bp_batch_tile_count; ++t) mx_max = bp_batch_tiles[t].mx > mx_max ? bp_batch_tiles[t].mx : mx_max;
        int W, ws;
        double hd;
        tile_window(b->lambda[i], b->dx[i], b->dy[i], mx_max, &W, &ws, &hd);
        b->guard[i] = ws + 2;
        b->row_stride[i] = static_cast<long long>(d.nfft) + 2LL * b->guard[i];
        const size_t np = static_cast<size_t>(d.num_pulses);
        const size_t pair_bytes = np * static_cast<size_t>(b->row_stride[i]) * 16;
        const size_t fft_bytes = np * d.nfft * sizeof(float2);
        const int R = d.nfft % d.num_range_samples == 0 ? d.nfft / d.num_range_samples : 0;
        size_t rc_smem = 0;
        std::vector<float> tab;
        const bool fused = want_fused && R >= 1 && rc_fused_shape(d.num_range_samples, R, &rc_smem, &tab) &&
                           rc_smem <= static_cast<size_t>(dev_smem);
        if (fused) {
            const long long key = static_cast<long long>(d.num_range_samples) * 64 + R;
            void *t = nullptr;
            for (const auto &kv : tab_of)
                if (kv.first == key) t = kv.second;
            if (!t) {
                if ((st = balloc(b, &t, tab.size() * sizeof(float)))) break;
                b->rc_tables.push_back(t);
                tab_of.emplace_back(key, t);
                if (cudaMemcpy(t, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
                    cudaGetLastError();
                    st = SARBP_ERR_CUDA;
                    break;
                }
            }
            b->rctab[i] = t;
            b->rc_R[i] = R;
        }
        if ((st = balloc(b, &b->d_pairs[i], pair_bytes)) || (!fused && (st = balloc(b, &b->d_fft[i], fft_bytes))) ||
            (st = balloc(b, &b->d_fac[i], static_cast<size_t>(d.num_range_samples) * sizeof(float2))))
            break;
        if (cudaMemset(b->d_pairs[i], 0, pair_bytes) != cudaSuccess ||
            (!fused && cudaMemset(b->d_fft[i], 0, fft_bytes) != cudaSuccess)) {
            cudaGetLastError();
            st = SARBP_ERR_CUDA;
            break;
        }
        const std::vector<double> fac = range_factors(d);
        const std::vector<float> f32(fac.begin(), fac.end());
        if (cudaMemcpy(b->d_fac[i], f32.data(), f32.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            st = SARBP_ERR_CUDA;
            break;
        }
        if (fused) continue;
        // FFT plans share one work area (their executions are serialised)
        cufftResult r = cufftCreate(&b->fft[i]);
        if (r == CUFFT_SUCCESS) {
            b->fft_ok[i] = 1;
            r = cufftSetAutoAllocation(b->fft[i], 0);
        }
        size_t ws_bytes = 0;
        if (r == CUFFT_SUCCESS) r = cufftMakePlan1d(b->fft[i], d.nfft, CUFFT_C2C, d.num_pulses, &ws_bytes);
        if (r != CUFFT_SUCCESS) {
            st = from_cufft(r);
            break;
        }
        work = ws_bytes > work ? ws_bytes : work;
    }
    if (st == SARBP_OK && work > 0) st = balloc(b, &b->fft_work, work);
    for (int i = 0; i < n && st == SARBP_OK; ++i) {
        if (!b->fft_ok[i]) continue;
        const cufftResult r = cufftSetWorkArea(b->fft[i], b->fft_work);
        if (r != CUFFT_SUCCESS) st = from_cufft(r);
    }
    if (st == SARBP_OK) st = balloc(b, reinterpret_cast<void **>(&b->d_table), n * sizeof(BatchScene));
    if (st == SARBP_OK) st = balloc(b, reinterpret_cast<void **>(&b->d_times), (n + 1) * sizeof(unsigned long long));
    if (st == SARBP_OK) st = balloc(b, reinterpret_cast<void **>(&b->d_err), sizeof(unsigned));
    if (st == SARBP_OK) {
        if (cudaHostAlloc(reinterpret_cast<void **>(&b->h_table), n * sizeof(BatchScene), cudaHostAllocDefault) !=
                cudaSuccess ||
            cudaHostAlloc(reinterpret_cast<void **>(&b->h_times), (n + 1) * sizeof(unsigned long long),
                          cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc(reinterpret_cast<void **>(&b->h_err), sizeof(unsigned), cudaHostAllocDefault) !=
                cudaSuccess ||
            cudaMemset(b->d_err, 0, sizeof(unsigned)) != cudaSuccess ||
            cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->done_ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            st = SARBP_ERR_CUDA;
        } else {
            *b->h_err = 0;
        }
    }
    if (st == SARBP_OK) st = choose_default_tile(b);
    if (st != SARBP_OK) {
        release(b);
        return st;
    }
    *out = b;
    return SARBP_OK;
}

int sarbp_batch_destroy(sarbp_batch *b) {
    if (!b) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(b->device);
    release(b);
    return SARBP_OK;
}

int sarbp_batch_focus(sarbp_batch *b, const sarbp_aperture *aps, void *const *images, void *stream) {
    NvtxRange range("sarbp_batch_focus");
    if (!b) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(b->device);
    SARBP_TRY_CUDA(guard.status);
    return focus_impl(b, aps, images, static_cast<cudaStream_t>(stream));
}

int sarbp_batch_wait(sarbp_batch *b, double *image_ms) {
    NvtxRange range("sarbp_batch_wait");
    if (!b) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(b->device);
    SARBP_TRY_CUDA(guard.status);
    return wait_impl(b, image_ms);
}

int sarbp_batch_autotune(sarbp_batch *b, const sarbp_aperture *aps, void *const *images, void *stream,
                         double *best_ms) {
    NvtxRange range("sarbp_batch_autotune");
    if (!b) return SARBP_ERR_NULL_POINTER;
    if (!aps || !images) return SARBP_ERR_NULL_POINTER;
    DeviceGuard guard(b->device);
    SARBP_TRY_CUDA(guard.status);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const TileConfig start = b->tile;
    const int start_sched = b->per_tile;
    TileConfig best{0, 0};
    int best_sched = 0;
    double best_t = 0.0;
    cudaEvent_t e0, e1;
    SARBP_TRY_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaGetLastError();
        return SARBP_ERR_CUDA;
    }
    int st = SARBP_OK;
    for (int c = 0; c < 2 * bp_batch_tile_count && st == SARBP_OK; ++c) {
        if (b->launched && cudaEventSynchronize(b->done_ev) != cudaSuccess) {
            st = SARBP_ERR_CUDA;
            break;
        }
        if (!configure(b, bp_batch_tiles[c / 2])) continue;
        b->per_tile = c & 1;
        // two warm-up calls (the first captures the graph), then three timed
        for (int w = 0; w < 2 && st == SARBP_OK; ++w) st = focus_impl(b, aps, images, s);
        if (st == SARBP_OK) st = wait_impl(b, nullptr);
        if (st != SARBP_OK) break;
        float ms = 0.0f;
        if (cudaEventRecord(e0, s) != cudaSuccess) st = SARBP_ERR_CUDA;
        for (int r = 0; r < 3 && st == SARBP_OK; ++r) st = focus_impl(b, aps, images, s);
        if (st == SARBP_OK && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                               cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
            st = SARBP_ERR_CUDA;
        if (st == SARBP_OK) st = wait_impl(b, nullptr);
        if (st == SARBP_OK && (!best.mx || ms / 3.0 < best_t)) {
            best = bp_batch_tiles[c / 2];
            best_sched = c & 1;
            best_t = ms / 3.0;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGetLastError();
    if (b->launched) cudaEventSynchronize(b->done_ev);
    if (st == SARBP_OK && !best.mx) st = SARBP_ERR_UNSUPPORTED;
    if (!configure(b, st == SARBP_OK ? best : start) && st == SARBP_OK) st = SARBP_ERR_CUDA;
    b->per_tile = st == SARBP_OK ? best_sched : start_sched;
    if (st == SARBP_OK && best_ms) *best_ms = best_t;
    return st;
}

int sarbp_batch_set_schedule(sarbp_batch *b, int per_tile) {
    if (!b) return SARBP_ERR_NULL_POINTER;
    if (per_tile < -1 || per_tile > 1) return SARBP_ERR_INVALID_ARGUMENT;
    DeviceGuard guard(b->device);
    SARBP_TRY_CUDA(guard.status);
    if (b->launched) SARBP_TRY_CUDA(cudaEventSynchronize(b->done_ev));
    b->per_tile = per_tile;
    drop_graph(b);
    return SARBP_OK;
}

int sarbp_batch_get_info(const sarbp_batch *b, sarbp_batch_info *info) {
    if (!b || !info) return SARBP_ERR_NULL_POINTER;
    std::memset(info, 0, sizeof(*info));
    info->num_scenes = b->n;
    info->tile_mx = b->tile.mx;
    info->stage_pulses = b->tile.pb;
    info->max_window_bins = b->max_wsize;
    info->resident_ctas = b->resident;
    info->graph = b->use_graph && b->graph_valid ? 1 : 0;
    info->tiles = b->tiles;
    info->units = b->units;
    info->smem_bytes = static_cast<long long>(b->smem);
    info->workspace_bytes = static_cast<long long>(b->bytes);
    info->per_tile = per_tile_now(b) ? 1 : 0;
    return SARBP_OK;
}

}  // extern "C"
