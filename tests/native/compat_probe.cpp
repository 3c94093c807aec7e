// compat_probe.cpp -- test helper: drives cuda_focus_SAR_image<T,T> exactly as
// the reference's MATLAB front-end does (cuda_sar_focusing_mex.cuh:27-65 with
// import_MATLABMexArguments, cpuBackProjection_mex.hpp:100-123):
// aperture from raw arrays, initialize_SAR_Aperture_Data, grid,
// SAR_ImageFormationParameters::update, then the focusing call, which the
// dynamic linker resolves to libsarbp_compat.so.  Compiled against the
// reference's own headers by tests/native/Makefile.
#define CUDAFUNCTION

#include <uncc_sar_focusing.hpp>

template <typename __nTp, typename __nTpParams>
void cuda_focus_SAR_image(const SAR_Aperture<__nTp> &, const SAR_ImageFormationParameters<__nTpParams> &,
                          CArray<__nTp> &);

namespace {
template <typename T>
int run(int K, int Np, const T *ph, const T *freq, const T *ax, const T *ay, const T *az, const T *r0, int nfft,
        int nx, int ny, T x0, T y0, T wx, T wy, T *img, T *max_wy) {
    SAR_Aperture<T> ap;
    SAR_ImageFormationParameters<T> params;
    int ph_dims[2] = {K, Np}, freq_dims[2] = {K, 1}, pulse_dims[2] = {1, Np};
    ap.numAzimuthSamples = Np;
    ap.numRangeSamples = K;
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
    CArray<T> out(params.N_y_pix * params.N_x_pix);
    cuda_focus_SAR_image(ap, params, out);
    for (size_t i = 0; i < out.size(); i++) {
        img[2 * i] = out[i].real();
        img[2 * i + 1] = out[i].imag();
    }
    *max_wy = params.max_Wy_m;
    return 0;
}
}  // namespace

extern "C" {
int compat_focus_f32(int K, int Np, const float *ph, const float *freq, const float *ax, const float *ay,
                     const float *az, const float *r0, int nfft, int nx, int ny, float x0, float y0, float wx,
                     float wy, float *img, float *max_wy) {
    return run<float>(K, Np, ph, freq, ax, ay, az, r0, nfft, nx, ny, x0, y0, wx, wy, img, max_wy);
}
int compat_focus_f64(int K, int Np, const double *ph, const double *freq, const double *ax, const double *ay,
                     const double *az, const double *r0, int nfft, int nx, int ny, double x0, double y0, double wx,
                     double wy, double *img, double *max_wy) {
    return run<double>(K, Np, ph, freq, ax, ay, az, r0, nfft, nx, ny, x0, y0, wx, wy, img, max_wy);
}
}
