// bp_mixed.cu -- mixed-precision forward backprojection for sm_100a.
//
// Replaces the reference kernel backprojection_loop
// (src/gpuBackProjection/cuda_sar_focusing/cuda_BackProjectionKernels.cuh:33-93)
// and its CPU twin computeDifferentialRangeAndPhaseCorrections
// (src/cpuBackProjection/cpuBackProjection.hpp:49-93):
//     img[q] += lerp(rc_p, bin(dR)) * exp(+j 4 pi f0_p dR / c),
//     dR = |a_p - x_q| - R0_p,  gate rmin < dR < rmax,
//     bracket [floor(bin), floor(bin)+1]  (CPU/MATLAB semantics, not the
//     GPU kernel's roundf bracket, cuda_BackProjectionKernels.cuh:68-74).
//
// Design (one CTA = one pixel tile of (8*MX) x 64 pixels of one z-slice,
// 256 threads = 8 warps, each thread MX rows (8 apart) x 2 columns (lane and
// lane + 32, so the lanes of one gather are one column apart):
//  * pulses go through shared memory in stages of PB pulses, two stage
//    buffers, each with three mbarriers: "full" (PB arrivals and the window
//    bytes), "ready" (all 8 warps have put their windows into intercept
//    form) and "empty" (all 8 warps have consumed the stage).  A warp waits
//    only for the buffer it touches next, so the warps of a CTA drift up to
//    a stage apart instead of meeting at a CTA barrier every stage (1.72 vs
//    1.76 ms on the large workload, same image).  For each pulse slot of the next
//    stage one warp (slot mod 8) computes the (tile, pulse) geometry record in
//    FP64 (tile-centre range, unit vector, phase and bin steps reduced mod 1)
//    and issues one cp.async.bulk copy of the pulse's range-bin window (the
//    bins any pixel of the tile can touch: +-|tile half-diagonal|), so the
//    FP64 work and the copy issue are spread evenly over the warps;
//  * range profiles live in HBM as pair entries {rc[b], rc[b+1]-rc[b]}
//    (float4); once a window lands its producing warp rewrites it in
//    shared memory to intercept form {rc[b] - (n - W) slope, slope}, so one
//    16-byte load and two FMAs on the window-centred bin interpolate;
//  * per pixel-pulse all arithmetic is FP32: dR = (Rc - R0) - u.d + g with
//    the FP64 per-tile part carried as a per-thread phase and bin base,
//    g = e (h + t hr) the far-field remainder (exact sqrt form for near-field
//    pulses); the phase stays in radians within a few multiples of pi of
//    zero and goes straight to __sincosf; the floor of the bin comes from one
//    round-down add whose result bits also form the shared-memory address;
//  * MX = 8 (64 x 64-pixel tiles) by default: the per-(tile, pulse) and
//    per-(thread, pulse) work is spread over 16 pixels per thread;
//  * complex64 results leave as float2 stores, 32 consecutive pixels per warp.
#include <cstdint>

#include "bp_common.cuh"
#include "bp_tile.cuh"
#include "sarbp_internal.h"

namespace sarbp {
namespace {

using namespace tile;

// pulses of a common-path stage unrolled together (0: the default per tile shape)
#ifndef SARBP_FAST_UNROLL
#define SARBP_FAST_UNROLL 0
#endif
constexpr int kFastUnroll = SARBP_FAST_UNROLL;

// CTAs per SM the register budget is sized for when shared memory allows
// more than one (launch bounds of the default instantiation)
#ifndef SARBP_CTAS_PER_SM
#define SARBP_CTAS_PER_SM 2
#endif
constexpr int kCtasPerSm = SARBP_CTAS_PER_SM;

constexpr int kTabEntries = kBaseEntries;

// Header of the shared memory: six mbarriers (full, ready and empty, two
// buffers each) and the zero entry.
constexpr int kHdr = 64;

// Dynamic shared memory of the forward kernel: the header, two stage
// buffers of PB records, base tables and windows, and two staging slots of
// PB pre-pass records.
__host__ __device__ constexpr size_t smem_bytes_of(int pb, int wsize) {
    return kHdr + 2 * static_cast<size_t>(pb) * (sizeof(PulseGeo) + kTabEntries * sizeof(float4)) +
           2 * static_cast<size_t>(pb) * static_cast<size_t>(wsize) * 16 +
           2 * static_cast<size_t>(pb) * sizeof(PulseGeo);
}

// pulse stages of split tiles walked in step across the resident CTAs
#ifndef SARBP_STAGE_ROTATION
#define SARBP_STAGE_ROTATION 1
#endif
constexpr bool kRotate = SARBP_STAGE_ROTATION != 0;


// One pulse into the thread's MX x 2 pixels.  The two columns l = 0, 1 (32 apart) of a
// row form a pair and their geometry arithmetic and complex
// multiply-accumulate run as paired FP32 instructions (__ffma2_rn and
// friends); the sine/cosine, the shared-memory gather and the interpolation
// are per pixel.
// Sign conventions avoid negations: nd2 = -|d|^2, so ne = t^2 - |d|^2 = -e,
// ng = ne (h + t hr) = -g, and the phase / bin add -kr * ng, -lam * ng.
template <int MX, bool GATE, bool NEAR, bool CHECKED>
__device__ __forceinline__ void accumulate_pulse(const PulseGeo &g, const float4 *base, uint32_t w_addr,
                                                 uint32_t zero_addr, int warp, int lane, float lam, float j0f,
                                                 const float2 (&nd2)[MX], float (&acc_re)[MX][2],
                                                 float (&acc_im)[MX][2], int wsize, int W, unsigned *err) {
    const float4 c0 = *reinterpret_cast<const float4 *>(&g.a8r);  // a8r, b32r, g8, e32
    const float4 c1 = *reinterpret_cast<const float4 *>(&g.tx);   // tx, ty, h, hr
    const float4 c2 = *reinterpret_cast<const float4 *>(&g.kr);   // kr, rc, lo, hi
    // per-thread phase, bin and projection bases: row part + column part,
    // each reduced in FP64 by the producer (|phase| <= 2 pi); the pair's
    // second pixel is 32 columns on
    const float4 rowv = base[warp];
    const float P00 = rowv.x + reinterpret_cast<const float *>(base + kWarps)[lane];
    const float B00 = fmaf(j0f, c0.w * (1.0f / 32.0f), rowv.y);
    const float t00 = fmaf(j0f, c1.y, rowv.z);
    float2 t2 = make_float2(t00, fmaf(32.0f, c1.y, t00));
    float2 Pb = make_float2(P00, P00 + c0.y);
    float2 Bb = make_float2(B00, B00 + c0.w);
    const float2 TX8 = splat(8.0f * c1.x), A8 = splat(c0.x), G8 = splat(c0.z);
    const float2 HR = splat(c1.w), H = splat(c1.z), NKR = splat(rowv.w), NLAM = splat(-lam);
    const float2 MAGIC = splat(kRoundMagic);
    // B is the window-centred bin; shared address of pair entry floor(B) + W:
    // bits(B + 1.5*2^23, rounded down) * 16 + w_adj (mod 2^32)
    const uint32_t w_adj = w_addr + (static_cast<uint32_t>(W) - kRoundMagicBits) * 16u;
#pragma unroll
    for (int k = 0; k < MX; ++k) {
        if (k > 0) {
            t2 = __fadd2_rn(t2, TX8);
            Pb = __fadd2_rn(Pb, A8);
            Bb = __fadd2_rn(Bb, G8);
        }
        float2 ng;
        if (NEAR) {
            const float e0 = -fmaf(t2.x, t2.x, nd2[k].x), e1 = -fmaf(t2.y, t2.y, nd2[k].y);
            const float s0 = c2.y - t2.x, s1 = c2.y - t2.y;
            ng = make_float2(-e0 / (s0 + sqrtf(fmaf(s0, s0, e0))), -e1 / (s1 + sqrtf(fmaf(s1, s1, e1))));
        } else {
            const float2 ne = __ffma2_rn(t2, t2, nd2[k]);
            ng = __fmul2_rn(ne, __ffma2_rn(t2, HR, H));
        }
        const float2 P = __ffma2_rn(NKR, ng, Pb);
        const float2 B = __ffma2_rn(NLAM, ng, Bb);
        const float2 y = __fadd2_rd(B, MAGIC);
        float2 RE, IM, CS, SN;  // the pair's interpolated samples and rotations
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const float Pl = l ? P.y : P.x;
            const float Bl = l ? B.y : B.x;
            const float yl = l ? y.y : y.x;
            float sn, cs;
            __sincosf(Pl, &sn, &cs);
            uint32_t addr = __float_as_uint(yl) * 16u + w_adj;
            if (GATE) {
                const bool valid = (Bl > c2.z) && (Bl < c2.w);
                addr = valid ? addr : zero_addr;
            }
            if (CHECKED) {
                // entry floor(B) + W must lie in the pulse's tight window
                // [W - wp, W + wp] (its next entry too)
                const uint32_t idx = __float_as_uint(yl) - kRoundMagicBits + static_cast<uint32_t>(g.wp);
                if (idx > static_cast<uint32_t>(2 * g.wp)) {
                    atomicOr(err, ERRBIT_BOUNDS);
                    addr = zero_addr;
                }
            }
            // intercept-form entry {c, v'}: v(B) = c + B v'
            const float4 v = lds128(addr);
            const float re = fmaf(Bl, v.z, v.x);
            const float im = fmaf(Bl, v.w, v.y);
            if (l) {
                RE.y = re;
                IM.y = im;
                CS.y = cs;
                SN.y = sn;
            } else {
                RE.x = re;
                IM.x = im;
                CS.x = cs;
                SN.x = sn;
            }
        }
        // complex multiply-accumulate of the pair as paired FP32 (same fused
        // operations as per pixel, half the instructions)
        float2 ar = make_float2(acc_re[k][0], acc_re[k][1]), ai = make_float2(acc_im[k][0], acc_im[k][1]);
        ar = __ffma2_rn(RE, CS, __ffma2_rn(make_float2(-IM.x, -IM.y), SN, ar));
        ai = __ffma2_rn(RE, SN, __ffma2_rn(IM, CS, ai));
        acc_re[k][0] = ar.x;
        acc_re[k][1] = ar.y;
        acc_im[k][0] = ai.x;
        acc_im[k][1] = ai.y;
    }
}

// Store (or add, L.accumulate) a thread's MX x 2 pixels of the tile at
// (tx0, ty0, slice zz) into the complex64 image: columns lane and lane + 32,
// so every store of a warp is 32 consecutive pixels.
template <int MX>
__device__ __forceinline__ void store_pixels(const BpLaunch &L, int tx0, int ty0, int zz, int warp, int lane,
                                             const float (&re)[MX][2], const float (&im)[MX][2]) {
    float2 *img = static_cast<float2 *>(L.img);
#pragma unroll
    for (int k = 0; k < MX; ++k) {
        const int row = tx0 + warp + 8 * k;
        if (row >= L.nx) continue;
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const int col = ty0 + lane + (kTY / 2) * l;
            if (col >= L.ny) continue;
            const long long o = (static_cast<long long>(zz) * L.nx + row) * L.ny + col;
            float2 v = make_float2(re[k][l], im[k][l]);
            if (L.accumulate) {
                const float2 old = img[o];
                v.x += old.x;
                v.y += old.y;
            }
            img[o] = v;
        }
    }
}

// Index of thread (warp, lane)'s pixel pair of row group k in a partial-sum
// slot of TX x 64 complex64 values (written and read by the same mapping).
__device__ __forceinline__ int slot_pair(int warp, int lane, int k) { return (warp + 8 * k) * kTY + 2 * lane; }

// Unit cursor over one launch (BATCH = false: the kernel parameter's scene)
// or over the scenes of a batch table, scene-major.
//
// Pulse-stage order within a tile (single-scene launches split over the
// resident CTAs): unit t S + b of tile t processes stage (b + rot_t) mod S
// with rot_t = t S - lo(owner of unit t S) mod S, the local step at which
// that CTA reaches the tile.  A CTA's k-th unit then works on stage k mod S,
// except on its first, partial tile, so the CTAs resident together walk the
// pulses in step and share the range profiles they stage through L2.  For
// the tiles a CTA reaches at their first stage rot_t = -lo(c) mod S, one
// value per CTA (rot_later); only the first tile has its own.  Every stage
// of a tile is still processed exactly once; only the order of the per-tile
// sums changes.
template <int TX, int PB, bool BATCH>
struct SceneCursor {
    const BpLaunch *L;
    TileGrid g;
    UnitCursor u;
    int scene;
    int rot;  // stage rotation of the current tile

    // pulse stage of the current unit
    __device__ __forceinline__ int stage() const {
        const int e = u.b + rot;
        return e >= g.stages ? e - g.stages : e;
    }

    // cursor at `unit` of U units split over the launch's G = gridDim.x CTAs
    __device__ __forceinline__ void init(const BpLaunch *L0, const BatchScene *scenes, int nscenes, long long unit,
                                         long long U) {
        scene = 0;
        L = L0;
        if constexpr (BATCH) {
            int a = 0, z = nscenes - 1;  // last scene with unit_begin <= unit
            while (a < z) {
                const int m = (a + z + 1) >> 1;
                if (scenes[m].unit_begin <= unit) a = m;
                else z = m - 1;
            }
            scene = a;
            L = &scenes[a].L;
            unit -= scenes[a].unit_begin;
        }
        g = tile_grid(*L, TX, PB);
        u.init(g, *L, unit);
        rot = 0;
        if constexpr (!BATCH && kRotate) {
            const long long G = gridDim.x;
            const long long first = unit - u.b;  // the tile's first unit
            rot = static_cast<int>((first - sk_lo(sk_owner(first, U, G), U, G)) % g.stages);
        }
    }
    // true when the cursor moved on to the next scene; rot_later: the stage
    // rotation of tiles entered at their first stage
    __device__ __forceinline__ bool advance(const BatchScene *scenes, int nscenes, int rot_later) {
        u.advance(g, *L);
        if (u.b == 0) rot = rot_later;
        if constexpr (BATCH) {
            if (u.hyp >= L->nhyp && scene + 1 < nscenes) {
                ++scene;
                L = &scenes[scene].L;
                g = tile_grid(*L, TX, PB);
                u.b = u.ty = u.tx = u.iz = u.hyp = 0;
                return true;
            }
        }
        return false;
    }
};

// BATCH = false: one scene, L0.  BATCH = true: the scenes of the table; L0
// carries only the batch-wide window size (the largest scene window: the
// stage buffers' stride) and sk_partial; each scene's image completion time
// goes to done[scene].
template <int MX, int PB, bool CHECKED, int MINB, bool BATCH>
__global__ void __launch_bounds__(kThreads, MINB)
    bp_mixed_kernel(const __grid_constant__ BpLaunch L0, const BatchScene *__restrict__ scenes, int nscenes,
                    long long batch_units, unsigned long long *__restrict__ done, int tile_mode) {
    constexpr int TX = 8 * MX;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    float4 *zero = reinterpret_cast<float4 *>(smem + kHdr - 16);
    PulseGeo *geo = reinterpret_cast<PulseGeo *>(smem + kHdr);
    float4 *bases = reinterpret_cast<float4 *>(smem + kHdr + 2 * PB * sizeof(PulseGeo));
    const uint32_t win_addr = smem_addr(smem + kHdr + 2 * PB * (sizeof(PulseGeo) + kTabEntries * sizeof(float4)));
    const uint32_t zero_addr = smem_addr(zero);
    const uint32_t buf_bytes = static_cast<uint32_t>(PB) * static_cast<uint32_t>(L0.wsize) * 16u;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this CTA's units [lo, lo + n) of the launch's (tile, stage) units
    const long long U = BATCH ? batch_units : tile_grid(L0, TX, PB).units;
    const long long G = gridDim.x;
    long long lo = sk_lo(blockIdx.x, U, G);
    int n = static_cast<int>(sk_lo(blockIdx.x + 1, U, G) - lo);
    if (BATCH && tile_mode) {
        // one CTA per tile of the batch, in scene order: CTA t takes tile t's stages
        int a = 0, z = nscenes - 1;  // last scene with tile_begin <= t
        while (a < z) {
            const int m = (a + z + 1) >> 1;
            if (scenes[m].tile_begin <= static_cast<long long>(blockIdx.x)) a = m;
            else z = m - 1;
        }
        const int S = tile_grid(scenes[a].L, TX, PB).stages;
        lo = scenes[a].unit_begin + (static_cast<long long>(blockIdx.x) - scenes[a].tile_begin) * S;
        n = S;
    }
    if (n <= 0) return;
    const int i0 = warp - TX / 2;
    const int j0 = lane - kTY / 2;  // column offset of the first pixel (the second is 32 on)
    const float j0f = static_cast<float>(j0);

    SceneCursor<TX, PB, BATCH> cc, pc;  // consumer at unit i, producer at unit i + 1
    cc.init(&L0, scenes, nscenes, lo, U);
    // stage rotation of the tiles this CTA enters at their first stage
    const int rot_later =
        (!BATCH && kRotate) ? static_cast<int>((cc.g.stages - lo % cc.g.stages) % cc.g.stages) : 0;
    pc = cc;

    // per-scene constants of the consumer
    float2 nd2[MX];  // -|d|^2 of the thread's pixel pairs
    float lam;
    int wsize;
    uint32_t pulse_bytes;
    auto scene_consts = [&]() {
        const BpLaunch &L = *cc.L;
        lam = static_cast<float>(L.lambda);
        wsize = L.wsize;
        pulse_bytes = static_cast<uint32_t>(wsize) * 16u;
        const float dxf = static_cast<float>(L.dx), dyf = static_cast<float>(L.dy);
#pragma unroll
        for (int k = 0; k < MX; ++k) {
            const float di = static_cast<float>(i0 + 8 * k) * dxf;
            const float dj0 = static_cast<float>(j0) * dyf, dj1 = static_cast<float>(j0 + kTY / 2) * dyf;
            nd2[k] = make_float2(-fmaf(di, di, dj0 * dj0), -fmaf(di, di, dj1 * dj1));
        }
    };
    scene_consts();
    float acc_re[MX][2], acc_im[MX][2];
#pragma unroll
    for (int k = 0; k < MX; ++k)
#pragma unroll
        for (int l = 0; l < 2; ++l) acc_re[k][l] = acc_im[k][l] = 0.0f;

    // buffer s: full (windows landed) at bar_base + 8 s, ready at
    // bar_base + 16 + 8 s, empty at bar_base + 32 + 8 s
    const uint32_t bar_base = smem_addr(&bars[0]);
    auto ready_bar = [&](int b) { return bar_base + 16u + 8u * b; };
    auto empty_bar = [&](int b) { return bar_base + 32u + 8u * b; };
    if (threadIdx.x == 0) {
        mbar_init(bar_base, PB);
        mbar_init(bar_base + 8, PB);
        for (int b = 0; b < 2; ++b) {
            mbar_init(ready_bar(b), kWarps);
            mbar_init(empty_bar(b), kWarps);
        }
        *zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        fence_mbar_init();
    }
    __syncthreads();

    // records, base tables and windows of the producer cursor's unit into
    // buffer s
    // Pre-pass records (single-scene launches: L0.geo_tab; batches: each
    // scene's L.geo_tab, L0.geo_tab non-null when every scene has them): the
    // records of the stage after the producer's are copied asynchronously
    // into the staging ring (two stages of PB records after the stage
    // buffers' windows) while the current stage accumulates, so their
    // global-memory latency does not stall the producing warps.
    const bool pregeo = L0.geo_tab != nullptr;
    PulseGeo *stg = reinterpret_cast<PulseGeo *>(smem + smem_bytes_of(PB, L0.wsize) - 2 * PB * sizeof(PulseGeo));
    // stage after the producer cursor's unit (last: the CTA has no more)
    auto prefetch_next = [&](int slot, bool last) {
        if (last) return;
        if constexpr (BATCH) {
            // the next unit may be the next scene's
            SceneCursor<TX, PB, BATCH> nx = pc;
            nx.advance(scenes, nscenes, rot_later);
            const BpLaunch &L = *nx.L;
            const long long t =
                ((static_cast<long long>(nx.u.hyp) * L.nz + nx.u.iz) * nx.g.tiles_x + nx.u.tx) * nx.g.tiles_y +
                nx.u.ty;
            prefetch_records<PB>(L, static_cast<const PulseGeo *>(L.geo_tab) + t * L.np, nx.stage(),
                                 stg + slot * PB, warp, lane);
            return;
        }
        const BpLaunch &L = *pc.L;
        long long t =
            ((static_cast<long long>(pc.u.hyp) * L.nz + pc.u.iz) * pc.g.tiles_x + pc.u.tx) * pc.g.tiles_y + pc.u.ty;
        int st;
        if (pc.u.b + 1 < pc.g.stages) {
            st = pc.stage() + 1;
            if (st == pc.g.stages) st = 0;
        } else {
            ++t;  // the next tile, entered at its first stage
            st = rot_later;
        }
        prefetch_records<PB>(L, static_cast<const PulseGeo *>(L.geo_tab) + t * L.np, st, stg + slot * PB, warp, lane);
    };
    auto produce = [&](int s, const PulseGeo *staged) {
        // every lane of the warp enters: the base tables take the whole warp
        // (the records come from the staging slot, or lane 0 computes them
        // and shuffles their steps to the warp), lane 0 issues the copy
        const BpLaunch &L = *pc.L;
        const double cx = L.left + static_cast<double>(pc.u.tx * TX + TX / 2) * L.dx;
        const double cy = L.bottom + static_cast<double>(pc.u.ty * kTY + kTY / 2) * L.dy;
        const double cz = L.zlow + static_cast<double>(pc.u.iz) * L.dz;
        produce_slots<PB>(L, pc.stage(), geo + s * PB, bases + s * PB * kTabEntries, win_addr + s * buf_bytes,
                          bar_base + 8 * s, warp, lane, TX / 2, cx, cy, cz,
                          static_cast<long long>(pc.u.hyp) * L.np, staged);
    };

    if (pregeo) {
        // stage 0's records now, stage 1's ahead
        const BpLaunch &L = *pc.L;
        const long long t =
            ((static_cast<long long>(pc.u.hyp) * L.nz + pc.u.iz) * pc.g.tiles_x + pc.u.tx) * pc.g.tiles_y + pc.u.ty;
        prefetch_records<PB>(L, static_cast<const PulseGeo *>(L.geo_tab) + t * L.np, pc.stage(), stg, warp, lane);
        produce(0, stg);
        prefetch_next(1, n < 2);
    } else {
        produce(0, nullptr);
    }
    const bool ok0 = intercept_slots<PB>(geo, win_addr, bar_base, 0, pc.L->wsize, pc.L->W, warp, lane, pc.L->err);
    __syncwarp();
    if (lane == 0) mbar_arrive(ready_bar(0));
    if (__any_sync(0xffffffffu, !ok0)) {
        // stage 0's copies never completed (error bit set): leave once the
        // record prefetches have landed; the other warps leave at their next
        // wait (every arrival on the incomplete barrier's phase is made)
        asm volatile("cp.async.wait_all;" ::: "memory");
        return;
    }

    int last_issued = 0;
    int seg = 0;                 // segments flushed so far
    int seg_first = cc.u.b;      // first stage of the open segment
    for (int i = 0; i < n; ++i) {
        const int s = i & 1;
        bool ok = true;
        if (i + 1 < n) {
            pc.advance(scenes, nscenes, rot_later);
            // buffer s ^ 1 last held stage i - 1: every warp has consumed it
            if (i >= 1) ok = mbar_wait_bounded(empty_bar(s ^ 1), ((i - 1) >> 1) & 1, pc.L->err);
        }
        if (i + 1 < n && ok) {
            if (pregeo) {
                // stage i + 1's records were prefetched into staging slot
                // (i + 1) & 1; stage i + 2's go to the other one, whose
                // records this warp read when it produced stage i (a warp
                // fills and reads only its own pulse slots of the ring)
                produce(s ^ 1, stg + (s ^ 1) * PB);
                prefetch_next(s, i + 2 >= n);
            } else {
                produce(s ^ 1, nullptr);
            }
            last_issued = i + 1;
        }
        const BpLaunch &L = *cc.L;
        const int S = cc.g.stages;
        const int b = cc.u.b;  // position in the tile's stage order
        if (ok) ok = mbar_wait_bounded(ready_bar(s), (i >> 1) & 1, L.err);
        if (ok) {
            const int nq = min(PB, L.np - cc.stage() * PB);
            // stage summary: all PB pulses active, none gated or near-field
            const int my_flags = lane < nq ? geo[s * PB + lane].flags : 0;
            const int any_f = __reduce_or_sync(0xffffffffu, my_flags);
            const int all_f = __reduce_and_sync(0xffffffffu, lane < nq ? my_flags : PG_ACTIVE);
            const uint32_t w0 = win_addr + s * buf_bytes;
            if (nq == PB && (all_f & PG_ACTIVE) && !(any_f & (PG_GATE | PG_NEAR))) {
                // the whole stage unrolled (64-row tiles: 1.762 vs 1.771 ms for a
                // half-stage unroll, no spill either way; 32 rows: 2.250 vs 2.283 ms)
                constexpr int kUnroll = kFastUnroll > 0 ? kFastUnroll : PB;
#pragma unroll kUnroll
                for (int q = 0; q < PB; ++q)
                    accumulate_pulse<MX, false, false, CHECKED>(geo[s * PB + q], bases + (s * PB + q) * kTabEntries,
                                                                w0 + q * pulse_bytes, zero_addr, warp, lane, lam, j0f,
                                                                nd2, acc_re, acc_im, wsize, L.W, L.err);
            } else {
                for (int q = 0; q < nq; ++q) {
                    const PulseGeo &g = geo[s * PB + q];
                    const float4 *bq = bases + (s * PB + q) * kTabEntries;
                    const int flags = g.flags;
                    if (!(flags & PG_ACTIVE)) continue;
                    const uint32_t w = w0 + q * pulse_bytes;
                    if (flags & PG_NEAR)
                        accumulate_pulse<MX, true, true, CHECKED>(g, bq, w, zero_addr, warp, lane, lam, j0f, nd2,
                                                                  acc_re, acc_im, wsize, L.W, L.err);
                    else if (flags & PG_GATE)
                        accumulate_pulse<MX, true, false, CHECKED>(g, bq, w, zero_addr, warp, lane, lam, j0f, nd2,
                                                                   acc_re, acc_im, wsize, L.W, L.err);
                    else
                        accumulate_pulse<MX, false, false, CHECKED>(g, bq, w, zero_addr, warp, lane, lam, j0f, nd2,
                                                                    acc_re, acc_im, wsize, L.W, L.err);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty_bar(s));
        // the next stage's windows into intercept form, published by the
        // ready mbarrier
        if (i + 1 < n && ok) {
            ok = intercept_slots<PB>(geo + (s ^ 1) * PB, win_addr + (s ^ 1) * buf_bytes, bar_base + 8 * (s ^ 1),
                                     ((i + 1) >> 1) & 1, pc.L->wsize, pc.L->W, warp, lane, L.err);
            __syncwarp();
            if (lane == 0) mbar_arrive(ready_bar(s ^ 1));
        }
        // a wait ran out (error bit set): this warp stops, the others at
        // their next wait for it; its own copies and record prefetches land
        // before the CTA's shared memory goes away (again bounded)
        if (__any_sync(0xffffffffu, !ok)) {
            asm volatile("cp.async.wait_all;" ::: "memory");
            if (lane == 0 && last_issued > i)
                mbar_wait_bounded(bar_base + 8 * (last_issued & 1), (last_issued >> 1) & 1, L.err);
            return;
        }
        if (i + 1 == n || b == S - 1) {
            // the segment of this tile ends: whole tile -> image, else -> partial slot
            if (seg_first == 0 && b == S - 1) {
                store_pixels<MX>(L, cc.u.tx * TX, cc.u.ty * kTY, cc.u.hyp * L.nz + cc.u.iz, warp, lane, acc_re,
                                 acc_im);
                // completion time: the latest of the warps' stores
                if (BATCH && done) {
                    __syncwarp();
                    if (lane == 0) atomicMax(done + cc.scene, global_timer_ns());
                }
            } else {
                float4 *slot = static_cast<float4 *>(L0.sk_partial) +
                               (2 * static_cast<long long>(blockIdx.x) + (seg > 0 ? 1 : 0)) * (TX * kTY / 2);
#pragma unroll
                for (int k = 0; k < MX; ++k)
                    slot[slot_pair(warp, lane, k) / 2] =
                        make_float4(acc_re[k][0], acc_im[k][0], acc_re[k][1], acc_im[k][1]);
            }
#pragma unroll
            for (int k = 0; k < MX; ++k)
#pragma unroll
                for (int l = 0; l < 2; ++l) acc_re[k][l] = acc_im[k][l] = 0.0f;
            ++seg;
            seg_first = 0;
        }
        if (cc.advance(scenes, nscenes, rot_later)) scene_consts();
    }
}

// Tiles whose stages were split over several CTAs: add the CTAs' partial
// sums in CTA order (a fixed order, so results repeat bit for bit) and store
// the tile.  One CTA per tile of the launch; tiles held whole by one CTA
// return at once.
template <int MX, int PB, bool BATCH>
__global__ void __launch_bounds__(kThreads)
    bp_sk_fixup_kernel(const __grid_constant__ BpLaunch L0, const BatchScene *__restrict__ scenes, int nscenes,
                       long long units, long long G, unsigned long long *__restrict__ done) {
    constexpr int TX = 8 * MX;
    long long t = blockIdx.x, unit0 = 0;
    const BpLaunch *Lp = &L0;
    int scene = 0;
    if constexpr (BATCH) {
        int a = 0, z = nscenes - 1;  // last scene with tile_begin <= t
        while (a < z) {
            const int m = (a + z + 1) >> 1;
            if (scenes[m].tile_begin <= t) a = m;
            else z = m - 1;
        }
        scene = a;
        Lp = &scenes[a].L;
        t -= scenes[a].tile_begin;
        unit0 = scenes[a].unit_begin;
    }
    const BpLaunch &L = *Lp;
    const TileGrid tg = tile_grid(L, TX, PB);
    const long long first = unit0 + t * tg.stages;
    const long long c0 = sk_owner(first, units, G);
    const long long c1 = sk_owner(first + tg.stages - 1, units, G);
    if (c0 == c1) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float re[MX][2], im[MX][2];
#pragma unroll
    for (int k = 0; k < MX; ++k)
#pragma unroll
        for (int l = 0; l < 2; ++l) re[k][l] = im[k][l] = 0.0f;
    const float4 *part = static_cast<const float4 *>(L0.sk_partial);
    for (long long c = c0; c <= c1; ++c) {
        const float4 *slot = part + sk_slot(c, first, units, G) * (TX * kTY / 2);
#pragma unroll
        for (int k = 0; k < MX; ++k) {
            const float4 v = slot[slot_pair(warp, lane, k) / 2];
            re[k][0] += v.x;
            im[k][0] += v.y;
            re[k][1] += v.z;
            im[k][1] += v.w;
        }
    }
    int tx0, ty0, zz;
    tile_origin(tg, t, TX, tx0, ty0, zz);
    store_pixels<MX>(L, tx0, ty0, zz, warp, lane, re, im);
    if (BATCH && done) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(done + scene, global_timer_ns());
    }
}

// Geometry records of every (tile, pulse) of a launch, [tile][pulse], one
// thread each (make_geo, full warps), for the forward kernel's producers to
// load.  Each CTA computes 256 records into shared memory, then writes them
// out as consecutive 16-byte words (a warp stores 512 contiguous bytes).  In
// shared memory word k of record r sits at [k][r] with a row stride of 257
// words, so both the record-per-thread stores and the word-per-thread reads
// hit 8 distinct bank groups per quarter warp (a [r][k] layout put all 32
// lanes of each 16-byte store on the same four banks).  Indexes are 32-bit:
// the launch checks n < 2^31.
template <int MX>
__device__ __forceinline__ void geo_records_chunk(const BpLaunch &L, unsigned n, unsigned i0, float4 *words) {
    constexpr int TX = 8 * MX;
    constexpr int kWords = sizeof(PulseGeo) / sizeof(float4);
    constexpr int kStride = 257;
    const TileGrid tg = tile_grid(L, TX, 1);
    const unsigned np = static_cast<unsigned>(L.np), ty_n = static_cast<unsigned>(tg.tiles_y),
                   tx_n = static_cast<unsigned>(tg.tiles_x), nz = static_cast<unsigned>(L.nz);
    const unsigned i = i0 + threadIdx.x;
    if (i < n) {
        const unsigned t = i / np, p = i - t * np;
        const unsigned r = t / ty_n, ty = t - r * ty_n;
        const unsigned zz = r / tx_n, tx = r - zz * tx_n;
        const unsigned hyp = zz / nz, iz = zz - hyp * nz;
        const double cx = L.left + static_cast<double>(static_cast<int>(tx) * TX + TX / 2) * L.dx;
        const double cy = L.bottom + static_cast<double>(static_cast<int>(ty) * kTY + kTY / 2) * L.dy;
        const double cz = L.zlow + static_cast<double>(iz) * L.dz;
        const PulseGeo g = make_geo(L, static_cast<int>(p), static_cast<long long>(hyp) * L.np, cx, cy, cz, TX / 2);
        const float4 *gw = reinterpret_cast<const float4 *>(&g);
#pragma unroll
        for (int k = 0; k < kWords; ++k) words[k * kStride + threadIdx.x] = gw[k];
    }
    __syncthreads();
    float4 *out = static_cast<float4 *>(L.geo_tab);
    const unsigned left = n - i0;
    const int nw = static_cast<int>((left < 256u ? left : 256u) * kWords);
    for (int w = threadIdx.x; w < nw; w += 256)
        out[static_cast<long long>(i0) * kWords + w] = words[(w % kWords) * kStride + w / kWords];
    __syncthreads();
}

template <int MX>
__global__ void __launch_bounds__(256) bp_geo_records_kernel(const __grid_constant__ BpLaunch L, int n) {
    __shared__ float4 words[(sizeof(PulseGeo) / sizeof(float4)) * 257];
    for (unsigned i0 = blockIdx.x * 256u; i0 < static_cast<unsigned>(n); i0 += gridDim.x * 256u)
        geo_records_chunk<MX>(L, static_cast<unsigned>(n), i0, words);
}

// The same for every scene of a batch (blockIdx.y = scene), into each
// scene's record rows (BatchScene::L.geo_tab).
template <int MX>
__global__ void __launch_bounds__(256) bp_geo_records_batch_kernel(const BatchScene *__restrict__ scenes) {
    __shared__ float4 words[(sizeof(PulseGeo) / sizeof(float4)) * 257];
    const BpLaunch &L = scenes[blockIdx.y].L;
    if (!L.geo_tab) return;
    const unsigned n = static_cast<unsigned>(tile_grid(L, 8 * MX, 1).tiles) * static_cast<unsigned>(L.np);
    for (unsigned i0 = blockIdx.x * 256u; i0 < n; i0 += gridDim.x * 256u) geo_records_chunk<MX>(L, n, i0, words);
}

template <int MX>
cudaError_t launch_records_mx(const BpLaunch &L, bool *ran, cudaStream_t s) {
    *ran = false;
    const long long nrec = tile_grid(L, 8 * MX, 1).tiles * L.np;
    if (!L.geo_tab || nrec < 1 || nrec > L.geo_tab_records || nrec >= 0x7fffffffLL) return cudaSuccess;
    const long long blocks = (nrec + 255) / 256;
    bp_geo_records_kernel<MX><<<static_cast<unsigned>(blocks < 148 * 64 ? blocks : 148 * 64), 256, 0, s>>>(
        L, static_cast<int>(nrec));
    const cudaError_t e = cudaGetLastError();
    *ran = e == cudaSuccess;
    return e;
}

}  // namespace

cudaError_t launch_geo_records(const BpLaunch &L, int mx, bool *ran, cudaStream_t s) {
    switch (mx) {
        case 8: return launch_records_mx<8>(L, ran, s);
        case 4: return launch_records_mx<4>(L, ran, s);
        case 2: return launch_records_mx<2>(L, ran, s);
        case 1: return launch_records_mx<1>(L, ran, s);
        default: *ran = false; return cudaSuccess;
    }
}

cudaError_t launch_geo_records_batch(const BatchScene *scenes, int nscenes, int mx, long long max_records,
                                     cudaStream_t s) {
    if (nscenes < 1 || nscenes > 65535 || max_records < 1 || max_records >= 0x7fffffffLL)
        return cudaErrorInvalidValue;
    const long long bx = (max_records + 255) / 256;
    const dim3 grid(static_cast<unsigned>(bx < 1024 ? bx : 1024), static_cast<unsigned>(nscenes));
    switch (mx) {
        case 8: bp_geo_records_batch_kernel<8><<<grid, 256, 0, s>>>(scenes); break;
        case 4: bp_geo_records_batch_kernel<4><<<grid, 256, 0, s>>>(scenes); break;
        case 2: bp_geo_records_batch_kernel<2><<<grid, 256, 0, s>>>(scenes); break;
        case 1: bp_geo_records_batch_kernel<1><<<grid, 256, 0, s>>>(scenes); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

namespace {

template <int MX, int PB, bool CHECKED, int MINB>
cudaError_t launch_kernels(const BpLaunch &L0, size_t smem, cudaStream_t s) {
    constexpr int TX = 8 * MX;
    auto kern = bp_mixed_kernel<MX, PB, CHECKED, MINB, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const TileGrid tg = tile_grid(L0, TX, PB);
    if (tg.units < 1) return cudaSuccess;
    BpLaunch L = L0;
    bool pregeo = false;
    e = launch_geo_records(L, MX, &pregeo, s);
    if (e != cudaSuccess) return e;
    if (!pregeo) L.geo_tab = nullptr;
    // split the units over the resident CTAs unless the tiles fill whole waves
    long long G = tg.tiles;
    if (L.sk_partial && L.sk_resident > 0 && tg.tiles % L.sk_resident != 0) {
        const long long g = L.sk_resident < tg.units ? L.sk_resident : tg.units;
        if (2 * g * TX * kTY * static_cast<long long>(sizeof(float2)) <= L.sk_slot_bytes) G = g;
    }
    if (G > 0x7fffffffLL) return cudaErrorInvalidValue;
    kern<<<static_cast<unsigned>(G), kThreads, smem, s>>>(L, nullptr, 0, 0, nullptr, 0);
    e = cudaGetLastError();
    if (e != cudaSuccess || G == tg.tiles) return e;
    bp_sk_fixup_kernel<MX, PB, false>
        <<<static_cast<unsigned>(tg.tiles), kThreads, 0, s>>>(L, nullptr, 0, tg.units, G, nullptr);
    return cudaGetLastError();
}

template <int MX, int PB>
cudaError_t launch_mx_pb(const BpLaunch &L, bool checked, size_t smem, cudaStream_t s) {
    // two CTAs per SM (128 registers) by default; one CTA per SM (up to 255
    // registers) when the stage needs more shared memory than two CTAs get
    const bool one_cta = smem > 113u * 1024u;
    if (checked)
        return one_cta ? launch_kernels<MX, PB, true, 1>(L, smem, s) : launch_kernels<MX, PB, true, kCtasPerSm>(L, smem, s);
    return one_cta ? launch_kernels<MX, PB, false, 1>(L, smem, s) : launch_kernels<MX, PB, false, kCtasPerSm>(L, smem, s);
}

template <typename K>
int resident_of(K kern, size_t smem) {
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

template <int MX, int PB>
int resident_mx_pb(size_t smem) {
    const bool one_cta = smem > 113u * 1024u;
    return one_cta ? resident_of(bp_mixed_kernel<MX, PB, false, 1, false>, smem)
                   : resident_of(bp_mixed_kernel<MX, PB, false, kCtasPerSm, false>, smem);
}

template <int MX, int PB, int MINB>
cudaError_t launch_batch_kernels(const BatchScene *scenes, int nscenes, long long units, long long tiles,
                                 size_t smem, int resident, const BpLaunch &L0, unsigned long long *done,
                                 bool per_tile, cudaStream_t s) {
    auto kern = bp_mixed_kernel<MX, PB, false, MINB, true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    if (tiles < 1 || tiles > 0x7fffffffLL) return cudaErrorInvalidValue;
    if (per_tile) {
        // one CTA per tile: no partial sums, scenes finish in order
        kern<<<static_cast<unsigned>(tiles), kThreads, smem, s>>>(L0, scenes, nscenes, units, done, 1);
        return cudaGetLastError();
    }
    const long long G = resident < units ? resident : units;
    if (G < 1 || G > 0x7fffffffLL) return cudaErrorInvalidValue;
    kern<<<static_cast<unsigned>(G), kThreads, smem, s>>>(L0, scenes, nscenes, units, done, 0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    bp_sk_fixup_kernel<MX, PB, true>
        <<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(L0, scenes, nscenes, units, G, done);
    return cudaGetLastError();
}

template <int MX, int PB>
cudaError_t launch_batch_mx_pb(const BatchScene *scenes, int nscenes, long long units, long long tiles, size_t smem,
                               int resident, const BpLaunch &L0, unsigned long long *done, bool per_tile,
                               cudaStream_t s) {
    return smem > 113u * 1024u
               ? launch_batch_kernels<MX, PB, 1>(scenes, nscenes, units, tiles, smem, resident, L0, done, per_tile, s)
               : launch_batch_kernels<MX, PB, 2>(scenes, nscenes, units, tiles, smem, resident, L0, done, per_tile,
                                                 s);
}

template <int MX, int PB>
int batch_resident_mx_pb(size_t smem) {
    return smem > 113u * 1024u ? resident_of(bp_mixed_kernel<MX, PB, false, 1, true>, smem)
                               : resident_of(bp_mixed_kernel<MX, PB, false, 2, true>, smem);
}

}  // namespace

size_t bp_mixed_smem_bytes(const TileConfig &tc, int wsize) { return smem_bytes_of(tc.pb, wsize); }

int bp_mixed_resident(const TileConfig &tc, size_t smem) {
#define SARBP_MIXED_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_) return resident_mx_pb<MX_, PB_>(smem);
    SARBP_MIXED_CASE(8, 8)
    SARBP_MIXED_CASE(8, 4)
    SARBP_MIXED_CASE(4, 16)
    SARBP_MIXED_CASE(4, 8)
    SARBP_MIXED_CASE(4, 4)
    SARBP_MIXED_CASE(4, 2)
    SARBP_MIXED_CASE(4, 1)
    SARBP_MIXED_CASE(2, 16)
    SARBP_MIXED_CASE(2, 8)
    SARBP_MIXED_CASE(2, 4)
    SARBP_MIXED_CASE(2, 2)
    SARBP_MIXED_CASE(2, 1)
    SARBP_MIXED_CASE(1, 16)
    SARBP_MIXED_CASE(1, 8)
    SARBP_MIXED_CASE(1, 4)
    SARBP_MIXED_CASE(1, 2)
    SARBP_MIXED_CASE(1, 1)
#undef SARBP_MIXED_CASE
    return 0;
}

// Tile shapes instantiated for batches; the batch autotuner times these.
const TileConfig bp_batch_tiles[] = {{8, 8}, {8, 4}, {4, 8}, {4, 4}, {2, 8}, {2, 4}, {1, 8}, {1, 4}};
const int bp_batch_tile_count = static_cast<int>(sizeof(bp_batch_tiles) / sizeof(bp_batch_tiles[0]));

cudaError_t launch_bp_mixed_batch(const BatchScene *scenes, int nscenes, long long units, long long tiles,
                                  const TileConfig &tc, size_t smem, int resident, void *partial,
                                  unsigned long long *done, cudaStream_t s, int max_wsize, bool per_tile,
                                  void *records) {
    BpLaunch L0{};
    L0.wsize = max_wsize;
    L0.sk_partial = partial;
    L0.geo_tab = records;  // non-null: every scene's table slot has its record rows
#define SARBP_BATCH_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_)  \
        return launch_batch_mx_pb<MX_, PB_>(scenes, nscenes, units, tiles, smem, resident, L0, done, per_tile, s);
    SARBP_BATCH_CASE(8, 8)
    SARBP_BATCH_CASE(8, 4)
    SARBP_BATCH_CASE(4, 8)
    SARBP_BATCH_CASE(4, 4)
    SARBP_BATCH_CASE(2, 8)
    SARBP_BATCH_CASE(2, 4)
    SARBP_BATCH_CASE(1, 8)
    SARBP_BATCH_CASE(1, 4)
#undef SARBP_BATCH_CASE
    return cudaErrorInvalidValue;
}

int bp_mixed_batch_resident(const TileConfig &tc, size_t smem) {
#define SARBP_BATCH_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_) return batch_resident_mx_pb<MX_, PB_>(smem);
    SARBP_BATCH_CASE(8, 8)
    SARBP_BATCH_CASE(8, 4)
    SARBP_BATCH_CASE(4, 8)
    SARBP_BATCH_CASE(4, 4)
    SARBP_BATCH_CASE(2, 8)
    SARBP_BATCH_CASE(2, 4)
    SARBP_BATCH_CASE(1, 8)
    SARBP_BATCH_CASE(1, 4)
#undef SARBP_BATCH_CASE
    return 0;
}

cudaError_t launch_bp_mixed(const BpLaunch &L, const TileConfig &tc, bool checked, size_t smem, cudaStream_t s) {
#define SARBP_MIXED_CASE(MX_, PB_) \
    if (tc.mx == MX_ && tc.pb == PB_) return launch_mx_pb<MX_, PB_>(L, checked, smem, s);
    SARBP_MIXED_CASE(8, 8)
    SARBP_MIXED_CASE(8, 4)
    SARBP_MIXED_CASE(4, 16)
    SARBP_MIXED_CASE(4, 8)
    SARBP_MIXED_CASE(4, 4)
    SARBP_MIXED_CASE(4, 2)
    SARBP_MIXED_CASE(4, 1)
    SARBP_MIXED_CASE(2, 16)
    SARBP_MIXED_CASE(2, 8)
    SARBP_MIXED_CASE(2, 4)
    SARBP_MIXED_CASE(2, 2)
    SARBP_MIXED_CASE(2, 1)
    SARBP_MIXED_CASE(1, 16)
    SARBP_MIXED_CASE(1, 8)
    SARBP_MIXED_CASE(1, 4)
    SARBP_MIXED_CASE(1, 2)
    SARBP_MIXED_CASE(1, 1)
#undef SARBP_MIXED_CASE
    return cudaErrorInvalidValue;
}

}  // namespace sarbp
