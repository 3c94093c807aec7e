// sarbp_internal.h -- plan state and kernel launchers behind include/sarbp.h.
#pragma once

#include <cstddef>
#include <vector>
#include <cuda_runtime.h>
#include <cufft.h>

#include "../../include/sarbp.h"

namespace sarbp {

// Launch parameters of the forward backprojection kernels.
struct BpLaunch {
    const void *pairs;      // float4 (MIXED) / double4 (FP64) pair entries
    long long row_stride;   // entries per pulse row
    int guard;              // zero entries before bin 0 of each row
    const double *ax, *ay, *az, *r0, *f0;
    int np, nfft;
    double lambda;          // nfft / max_wr (bins per metre)
    double half_nfft;       // nfft / 2
    int nx, ny, nz;
    double left, bottom, zlow;  // coordinates of pixel (0, 0, 0)
    double dx, dy, dz;
    int W, wsize;           // window half-width and size (entries)
    double near_hd16;       // 16 * tile half-diagonal (m)
    double near_coef;       // 0.625 * hd^4 / tolerance (revolutions)
    void *img;              // complex64 / complex128 [nz][nx][ny]
    int accumulate;
    unsigned *err;
    int nhyp;               // geometry hypotheses (mixed forward kernel): arrays [nhyp][np], images [nhyp][nz][nx][ny]
    // Work split of the forward kernels.  The (tile, pulse-stage) units of a
    // launch, tile-major, are divided evenly over the launch's CTAs; a tile
    // whose stages end up on several CTAs leaves per-CTA partial sums in
    // sk_partial (two slots of one tile each per CTA) that bp_sk_fixup adds
    // in CTA order.  sk_partial == nullptr: one CTA per tile, no partials.
    void *sk_partial;
    long long sk_slot_bytes;  // bytes reserved for sk_partial (launch checks the need)
    int sk_resident;          // CTAs of the kernel resident at once on the device (0: do not split)
    // Geometry records of every (tile, pulse) of the launch written by a
    // pre-pass kernel ([tile][pulse], one PulseGeo each; the mixed forward kernel's
    // producing lanes then load them instead of computing them), and the
    // records the buffer holds; nullptr: computed in the kernel.
    void *geo_tab;
    long long geo_tab_records;
    // test hook (sarbp_test_drop_window_copy): the pulse whose window copy the
    // producers leave out while still expecting its bytes; -1: none
    int drop_pulse = -1;
};

// One scene of a batch (sarbp_batch_focus), in device memory.  The forward
// kernel walks the units of all scenes, scene-major: scene s owns units
// [unit_begin, unit_begin + its tiles x stages) and tiles
// [tile_begin, tile_begin + its tiles) of the launch.
struct BatchScene {
    BpLaunch L;                 // the scene's backprojection (pairs, geometry, grid, image, window)
    const void *ph;             // complex64 [np][K] phase history (device)
    const void *fac;            // per-sample taper x scale x shift twiddle [K]
    void *fft;                  // complex64 [np][nfft] FFT buffer
    int K;
    int fused;                  // 1: range-compressed by its own fused launch (batched taper/pair kernels skip it)
    long long row_stride;       // pair entries per pulse row
    long long unit_begin, tile_begin;
};

// Matched-filter launch (mf.cu): geometry on the device, pixel grid, image
// complex64 (MIXED) or complex128 (FP64) [nz][nx][ny].
struct MfLaunch {
    const double *ax, *ay, *az, *r0, *f0;
    int np, K;
    double df;  // frequency step (Hz)
    int nx, ny, nz;
    double left, bottom, zlow, dx, dy, dz;
    void *img;
};
// win: complex range weights (interleaved double re, im) [K], or null (all ones)
cudaError_t launch_mf(const void *ph, const double *win, const MfLaunch &M, bool fp64, cudaStream_t s);

// Tile shape of the forward kernels (see bp_mixed.cu).
struct TileConfig {
    int mx;   // rows per thread; tile = (8*mx) x 64 pixels, 256 threads
    int pb;   // pulses per pipeline stage
};

cudaError_t launch_bp_mixed(const BpLaunch &L, const TileConfig &tc, bool checked, size_t smem,
                            cudaStream_t s);
// Geometry records of every (tile, pulse) of L into L.geo_tab for tiles of
// (8 mx) x 64 pixels (bp_mixed.cu).  *ran is false (nothing launched) when
// L.geo_tab is null or holds fewer records than the launch has; the kernels
// then compute the records themselves.
cudaError_t launch_geo_records(const BpLaunch &L, int mx, bool *ran, cudaStream_t s);
// The same for every scene of a batch whose table slot has record rows
// (L.geo_tab non-null), tiles of (8 mx) x 64 pixels; max_records: the
// largest scene's tiles x pulses.
cudaError_t launch_geo_records_batch(const BatchScene *scenes, int nscenes, int mx, long long max_records,
                                     cudaStream_t s);
cudaError_t launch_bp_fp64(const BpLaunch &L, const TileConfig &tc, size_t smem, cudaStream_t s);
size_t bp_mixed_smem_bytes(const TileConfig &tc, int wsize);
// Adjoint (bp_adjoint.cu): per-(tile, pulse) gradient partials, then a sum
// over tiles into grad_ant [3][np] and grad_r0 [np].
cudaError_t launch_bp_adjoint(const BpLaunch &L, const void *grad, void *partials, const TileConfig &tc, size_t smem,
                              cudaStream_t s);
cudaError_t launch_adjoint_reduce(const void *partials, long long ntiles, int np, double *grad_ant, double *grad_r0,
                                  int accumulate, cudaStream_t s);
size_t bp_adjoint_smem_bytes(const TileConfig &tc, int wsize);
long long bp_tile_count(const BpLaunch &L, const TileConfig &tc);
size_t bp_fp64_smem_bytes(const TileConfig &tc, int wsize);
// CTAs of the forward kernel for this tile and shared-memory size that are
// resident at once on the current device (0 if the query fails).  A split
// launch with that many CTAs needs 2 * resident * (8 mx * 64) complex values
// of sk_partial.
int bp_mixed_resident(const TileConfig &tc, size_t smem);
// Batch forward launch over `nscenes` scenes (table in device memory,
// `units` = their total units, `tiles` = their total tiles): the split kernel
// and, when tiles are split, the fix-up.  Completion time of each scene's
// image (%globaltimer ns) goes to done[scene] (atomic max) when done != null.
// max_wsize: the largest scene window (entries), the stage buffers' stride.
// per_tile: one CTA per tile in scene order instead of the even split (no
// partial sums; scenes complete one after another).  records: non-null when
// every scene's slot carries pre-pass record rows (launch_geo_records_batch
// filled them), else the producers compute the records.
// Instantiated for the tile shapes in bp_batch_tiles.
cudaError_t launch_bp_mixed_batch(const BatchScene *scenes, int nscenes, long long units, long long tiles,
                                  const TileConfig &tc, size_t smem, int resident, void *partial,
                                  unsigned long long *done, cudaStream_t s, int max_wsize, bool per_tile,
                                  void *records);
int bp_mixed_batch_resident(const TileConfig &tc, size_t smem);
extern const TileConfig bp_batch_tiles[];
extern const int bp_batch_tile_count;
int bp_fp64_resident(const TileConfig &tc, size_t smem);

// Range compression kernels (range_compress.cu)
cudaError_t launch_rc_prep(int precision, const void *ph, const void *fac, void *fft_buf, int K, int nfft, int np,
                           cudaStream_t s);
cudaError_t launch_rc_pairs(int precision, const void *fft_buf, void *pairs, int nfft, int np, long long row_stride,
                            int guard, cudaStream_t s);
// Range compression steps 1 and 3 for every scene of a batch in one launch
// each (blockIdx.y = scene); the FFT in between runs per scene.
cudaError_t launch_rc_prep_batch(const BatchScene *scenes, int nscenes, cudaStream_t s);
// Fused range compression (mixed precision): taper, zero pad, inverse FFT and
// pair rows in one kernel for nfft = R K with K = 32 K2, K2 in {8, 16, 32},
// R in {1, 2, 4, 8, 16}.  rc_fused_shape says whether (K, R) is one of those
// and fills the twiddle table (interleaved float re, im) and the kernel's
// shared-memory bytes; grid: CTAs (each loops over pulses).
bool rc_fused_shape(int K, int R, size_t *smem, std::vector<float> *table);
cudaError_t launch_rc_fused(const void *ph, const void *fac, const void *table, void *pairs, int K, int R, int np,
                            long long row_stride, int guard, int grid, cudaStream_t s);
cudaError_t launch_pairs_to_rc(const void *pairs, void *rc, int nfft, int np, long long row_stride, int guard,
                               cudaStream_t s);
// Fused range compression of one batch scene, parameters read from its table
// slot (grid CTAs loop over the scene's pulses).
cudaError_t launch_rc_fused_scene(const BatchScene *scene, const void *table, int K, int R, int grid,
                                  cudaStream_t s);
cudaError_t launch_rc_pairs_batch(const BatchScene *scenes, int nscenes, cudaStream_t s);

}  // namespace sarbp

struct sarbp_plan {
    sarbp_plan_desc desc;
    int device;
    int K, np_cap, nfft, precision;
    double lambda;
    int W, wsize, guard;
    long long row_stride;
    sarbp::TileConfig tile;
    size_t smem;
    double near_hd16, near_coef;
    double dx, dy, dz, left, bottom, zlow;

    void *d_ph;       // complex64 [np][K] staging for host phase histories
    double *d_geo;    // 5 x np staging for host geometry
    void *d_fft;      // complex64/128 [np][nfft]
    void *d_pairs;    // pair entries [np][row_stride]
    void *d_fac;      // per-sample window * scale * shift twiddle [K]
    void *d_img;      // image staging for host outputs
    unsigned *d_err;  // device error bits
    void *d_partials; // adjoint per-(tile, pulse) partial gradients (allocated on first use)
    size_t partials_bytes;
    double *d_gout;   // adjoint output staging for host outputs [4][np] (allocated on first use)
    void *d_hyp;      // host-memory staging for hypothesis batches (allocated on first use)
    size_t hyp_bytes;
    double *d_win;    // complex range weights c_k for the matched filter (allocated on first use)
    bool win_stale;   // d_win no longer holds the current weights
    std::vector<double> range_w;  // caller's complex range weights [2 K] (empty: desc.window)
    void *d_rctab;    // twiddle table of the fused range compression (null: cuFFT path)
    int rc_R;         // nfft / K of the fused range compression
    int rc_grid;      // its CTAs
    void *d_geotab;   // pre-pass geometry records (BpLaunch::geo_tab), tiles x np_cap PulseGeo
    long long geotab_records;
    void *d_hyprec;   // pre-pass records of hypothesis launches (grown on first use)
    size_t hyprec_bytes;
    void *d_sk;       // partial sums of tiles split over CTAs (BpLaunch::sk_partial)
    size_t sk_bytes;
    int sk_resident;  // resident CTAs of the plan's forward kernel
    int drop_pulse = -1;  // test hook: BpLaunch::drop_pulse of the plan's launches
    size_t bytes;     // device bytes held
    cufftHandle fft;
    bool fft_ok;
    int np_ready;     // pulses in the current range profiles
    struct sarbp_pipe *pipe;  // pipelined host-buffer focusing (created on first submit)
};
