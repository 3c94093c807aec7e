// cuda_focus_sar_image.cpp -- the reference's C++ focusing symbols on top of
// the C ABI of include/sarbp.h.
//
// Exports exactly the two instantiations the reference's
// libuncc_sar_focusing_gpu.so exports
// (src/gpuBackProjection/cuda_sar_focusing/libcuda_sar_focusing.cu:26-32):
//
//   void cuda_focus_SAR_image<float, float>(SAR_Aperture<float> const&,
//            SAR_ImageFormationParameters<float> const&, std::valarray<unccComplex<float>>&);
//   void cuda_focus_SAR_image<double, double>(...)
//
// so callers such as sph_sar_data_callback_gpu (include/charlotte_sar_api.hpp:
// 261-316) and the MATLAB MEX front-end (cuda_sar_focusing_mex.cuh:27-65) link
// against libsarbp_compat.so instead and run unchanged.  It is compiled
// against the caller's own headers (include/uncc_sar_focusing.hpp), which
// define the argument types.
//
// Semantics: the grid, N_fft and max_Wy_m come from the image parameters, the
// phase history / antenna positions / slant range / start frequency from the
// aperture (uncc_sar_focusing.hpp:63-174), output x-major N_x_pix * N_y_pix.
// N_fft >= numRangeSamples zero-pads each pulse (the reference leaves this as
// a TODO, cpuBackProjection.hpp:107-110); no taper is applied, as in the
// reference.  <float,float> runs the mixed-precision engine, <double,double>
// the FP64 engine.  Like the reference the call is synchronous and void;
// unlike it, it never calls cudaDeviceReset() and reports failures on stderr
// with the engine's status string.  The plan (device buffers and FFT plan) of
// the last shape is kept for the next call with the same shape.
#include <cstdio>
#include <mutex>
#include <vector>

#include <uncc_sar_focusing.hpp>

#include "sarbp.h"

namespace {

struct CachedPlan {
    sarbp_plan_desc desc{};
    sarbp_plan *plan = nullptr;
};

std::mutex g_mutex;
CachedPlan g_cache[2];  // [precision]

bool same_desc(const sarbp_plan_desc &a, const sarbp_plan_desc &b) {
    return a.num_range_samples == b.num_range_samples && a.num_pulses == b.num_pulses && a.nfft == b.nfft &&
           a.max_wr == b.max_wr && a.grid.nx == b.grid.nx && a.grid.ny == b.grid.ny && a.grid.nz == b.grid.nz &&
           a.grid.x0 == b.grid.x0 && a.grid.y0 == b.grid.y0 && a.grid.z0 == b.grid.z0 && a.grid.wx == b.grid.wx &&
           a.grid.wy == b.grid.wy && a.grid.wz == b.grid.wz && a.precision == b.precision &&
           a.window == b.window && a.device == b.device;
}

template <typename T>
std::vector<double> to_double(const SimpleMatrix<T> &m, size_t n) {
    std::vector<double> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = static_cast<double>(m.data[i]);
    return v;
}

template <typename T, typename P>
void focus(const SAR_Aperture<T> &ap, const SAR_ImageFormationParameters<P> &ip, CArray<T> &out) {
    if (ip.algorithm != SAR_ImageFormationParameters<P>::ALGORITHM::BACKPROJECTION) {
        std::fprintf(stderr, "cuda_focus_SAR_image: only the backprojection algorithm is available\n");
        return;
    }
    const int K = ap.numRangeSamples, Np = ap.numAzimuthSamples;
    const size_t npix = static_cast<size_t>(ip.N_x_pix) * static_cast<size_t>(ip.N_y_pix);
    if (K < 1 || Np < 1 || ap.sampleData.data.size() < static_cast<size_t>(K) * Np ||
        ap.Ant_x.data.size() < static_cast<size_t>(Np) || ap.Ant_y.data.size() < static_cast<size_t>(Np) ||
        ap.Ant_z.data.size() < static_cast<size_t>(Np) || ap.slant_range.data.size() < static_cast<size_t>(Np) ||
        ap.startF.data.size() < static_cast<size_t>(Np) || out.size() < npix) {
        std::fprintf(stderr, "cuda_focus_SAR_image: aperture or output sizes are inconsistent\n");
        return;
    }
    sarbp_plan_desc d{};
    d.num_range_samples = K;
    d.num_pulses = Np;
    d.nfft = ip.N_fft;
    d.max_wr = static_cast<double>(ip.max_Wy_m);
    d.grid.nx = ip.N_x_pix;
    d.grid.ny = ip.N_y_pix;
    d.grid.nz = 1;
    d.grid.x0 = static_cast<double>(ip.x0_m);
    d.grid.y0 = static_cast<double>(ip.y0_m);
    d.grid.z0 = 0.0;  // the reference images the plane z = 0 (cpuBackProjection.hpp:57)
    d.grid.wx = static_cast<double>(ip.Wx_m);
    d.grid.wy = static_cast<double>(ip.Wy_m);
    d.grid.wz = 0.0;
    const bool fp64 = sizeof(T) == sizeof(double);
    d.precision = fp64 ? SARBP_PRECISION_FP64 : SARBP_PRECISION_MIXED;
    d.window = SARBP_WINDOW_NONE;
    d.device = -1;

    std::vector<float> ph(2 * static_cast<size_t>(K) * Np);
    for (size_t i = 0; i < static_cast<size_t>(K) * Np; ++i) {
        ph[2 * i] = static_cast<float>(ap.sampleData.data[i].real());
        ph[2 * i + 1] = static_cast<float>(ap.sampleData.data[i].imag());
    }
    const std::vector<double> ax = to_double(ap.Ant_x, Np), ay = to_double(ap.Ant_y, Np),
                              az = to_double(ap.Ant_z, Np), r0 = to_double(ap.slant_range, Np),
                              f0 = to_double(ap.startF, Np);
    sarbp_aperture a{};
    a.phase_history = ph.data();
    a.phase_history_memory = SARBP_MEMORY_HOST;
    a.geometry = {ax.data(), ay.data(), az.data(), r0.data(), f0.data(), Np, SARBP_MEMORY_HOST};

    std::lock_guard<std::mutex> lock(g_mutex);
    CachedPlan &c = g_cache[fp64 ? 1 : 0];
    if (!c.plan || !same_desc(c.desc, d)) {
        if (c.plan) sarbp_plan_destroy(c.plan);
        c.plan = nullptr;
        const int st = sarbp_plan_create(&d, &c.plan);
        if (st != SARBP_OK) {
            std::fprintf(stderr, "cuda_focus_SAR_image: %s\n", sarbp_status_string(st));
            c.plan = nullptr;
            return;
        }
        c.desc = d;
    }
    std::vector<double> img(2 * npix);
    std::vector<float> img32;
    void *dst = img.data();
    if (!fp64) {
        img32.resize(2 * npix);
        dst = img32.data();
    }
    int st = sarbp_focus(c.plan, &a, dst, SARBP_MEMORY_HOST, nullptr);
    if (st == SARBP_OK) st = sarbp_plan_check(c.plan, nullptr);
    if (st != SARBP_OK) {
        std::fprintf(stderr, "cuda_focus_SAR_image: %s\n", sarbp_status_string(st));
        return;
    }
    for (size_t i = 0; i < npix; ++i) {
        const double re = fp64 ? img[2 * i] : img32[2 * i];
        const double im = fp64 ? img[2 * i + 1] : img32[2 * i + 1];
        out[i]._M_real = static_cast<T>(re);
        out[i]._M_imag = static_cast<T>(im);
    }
}

}  // namespace

template <typename __nTp, typename __nTpParams>
void cuda_focus_SAR_image(const SAR_Aperture<__nTp> &sar_data,
                          const SAR_ImageFormationParameters<__nTpParams> &sar_image_params,
                          CArray<__nTp> &output_image) {
    focus(sar_data, sar_image_params, output_image);
}

template __attribute__((visibility("default"))) void cuda_focus_SAR_image<float, float>(
    SAR_Aperture<float> const &, SAR_ImageFormationParameters<float> const &, std::valarray<unccComplex<float>> &);
template __attribute__((visibility("default"))) void cuda_focus_SAR_image<double, double>(
    SAR_Aperture<double> const &, SAR_ImageFormationParameters<double> const &,
    std::valarray<unccComplex<double>> &);
