/*
 * oracle/ref_harness.cpp -- TEST INFRASTRUCTURE (the oracle), not product code.
 *
 * Thin extern "C" entry into the reference CPU backprojection, compiled by
 * oracle/Makefile directly against the reference's own headers where they
 * lie (include/, src/cpuBackProjection/; nothing is copied into this repo).
 * Output goes to oracle/_ref/ only.
 *
 * It drives the reference exactly as its MATLAB front-end does
 * (src/cpuBackProjection/cpuBackProjection_mex.hpp:100-163,
 * cpu_SARFocusingAlgorithm): import phase history, freq, antenna positions and
 * slant range into a SAR_Aperture, initialize_SAR_Aperture_Data(), set the
 * image grid, SAR_ImageFormationParameters::update(), focus_SAR_image().
 * The reference does no zero padding or windowing (cpuBackProjection.hpp:
 * 107-110), so callers pass a phase history that is already windowed and
 * zero-padded to N_fft samples per pulse, with freq extended at the same step.
 */
#define CUDAFUNCTION

#include <cstring>
#include <iostream>
#include <mutex>

#include <cpuBackProjection.hpp>

namespace {

// The reference prints progress to std::cout and its FILE logger on every
// call.  Both are switched off once per process (never toggled back, so calls
// from several threads at once do not race on the stream state).
struct QuietReference {
    QuietReference() {
        static std::once_flag once;
        std::call_once(once, [] {
            std::cout.rdbuf(nullptr);
            Output2FILE::Stream() = nullptr;
        });
    }
};

template <typename T>
int focus_with_reference(int nfft, int Np, const T *ph, const T *freq, const T *ax, const T *ay, const T *az,
                         const T *r0, int nx, int ny, T x0, T y0, T wx, T wy, T *img, T *max_wy_out,
                         T *start_f_out, bool matched_filter = false) {
    QuietReference quiet;
    SAR_Aperture<T> ap;
    SAR_ImageFormationParameters<T> params;

    int ph_dims[2] = {nfft, Np};
    int freq_dims[2] = {nfft, 1};
    int pulse_dims[2] = {1, Np};
    ap.numAzimuthSamples = Np;
    ap.numRangeSamples = nfft;
    import_MatrixComplex<const T, Complex<T>>(ph, ph_dims, 2, ap.sampleData);
    import_MatrixReal<const T, T>(freq, freq_dims, 2, ap.freq);
    import_MatrixReal<const T, T>(ax, pulse_dims, 2, ap.Ant_x);
    import_MatrixReal<const T, T>(ay, pulse_dims, 2, ap.Ant_y);
    import_MatrixReal<const T, T>(az, pulse_dims, 2, ap.Ant_z);
    import_MatrixReal<const T, T>(r0, pulse_dims, 2, ap.slant_range);

    params.N_x_pix = nx;
    params.N_y_pix = ny;
    params.N_fft = nfft;
    params.x0_m = x0;
    params.y0_m = y0;
    params.Wx_m = wx;
    params.Wy_m = wy;

    ap.polarity_channel = 0;
    if (initialize_SAR_Aperture_Data(ap) != EXIT_SUCCESS) return -1;
    params.update(ap);
    if (matched_filter) params.algorithm = SAR_ImageFormationParameters<T>::ALGORITHM::MATCHED_FILTER;

    CArray<T> out(params.N_y_pix * params.N_x_pix);
    focus_SAR_image(ap, params, out);
    for (size_t i = 0; i < out.size(); i++) {
        img[2 * i] = out[i].real();
        img[2 * i + 1] = out[i].imag();
    }
    if (max_wy_out) *max_wy_out = params.max_Wy_m;
    if (start_f_out)
        for (int p = 0; p < Np; p++) start_f_out[p] = ap.startF.data[p];
    return 0;
}

}  // namespace

extern "C" {

/* run_bp<float> via focus_SAR_image<float,float>; arrays interleaved re,im. */
int ref_focus_bp_f32(int nfft, int Np, const float *ph, const float *freq, const float *ax, const float *ay,
                     const float *az, const float *r0, int nx, int ny, float x0, float y0, float wx, float wy,
                     float *img, float *max_wy_out, float *start_f_out) {
    return focus_with_reference<float>(nfft, Np, ph, freq, ax, ay, az, r0, nx, ny, x0, y0, wx, wy, img,
                                       max_wy_out, start_f_out);
}

/* run_mf<double> via focus_SAR_image<double,double> with the MATCHED_FILTER
 * algorithm (cpuBackProjection.hpp:165-228); K = nfft samples per pulse, no
 * zero pad needed. */
int ref_focus_mf_f64(int K, int Np, const double *ph, const double *freq, const double *ax, const double *ay,
                     const double *az, const double *r0, int nx, int ny, double x0, double y0, double wx,
                     double wy, double *img) {
    return focus_with_reference<double>(K, Np, ph, freq, ax, ay, az, r0, nx, ny, x0, y0, wx, wy, img, nullptr,
                                        nullptr, true);
}

/* run_bp<double> via focus_SAR_image<double,double>. */
int ref_focus_bp_f64(int nfft, int Np, const double *ph, const double *freq, const double *ax, const double *ay,
                     const double *az, const double *r0, int nx, int ny, double x0, double y0, double wx,
                     double wy, double *img, double *max_wy_out, double *start_f_out) {
    return focus_with_reference<double>(nfft, Np, ph, freq, ax, ay, az, r0, nx, ny, x0, y0, wx, wy, img,
                                        max_wy_out, start_f_out);
}

}
