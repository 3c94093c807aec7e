// callback_probe.cpp -- test helper: drives the reference's raw-array callback
// API exactly as an external data source would (include/charlotte_sar_api.hpp:
// sph_sar_data_callback_gpu<float>, :261-316): Sandia-style arrays (samples
// interleaved re, im, K per pulse; per-pulse start frequency and chirp rate;
// antenna x, y, z; the A/D rate), from which the header's own code builds the
// aperture (create_SARAperture, :130-166, the derived-frequency path of
// initialize_SAR_Aperture_Data), picks the full-scene grid
// (create_SARImageFormationParams, :168-197), calls cuda_focus_SAR_image --
// resolved by the dynamic linker to libsarbp_compat.so -- and writes the 8-bit
// BMP (writeBMPFile, uncc_sar_globals.hpp:66-117).  Compiled against the
// reference's headers by tests/native/Makefile.
#define CUDAFUNCTION
#define LOADBMP_IMPLEMENTATION

#include <numeric>

#include <uncc_sar_focusing.hpp>
#include <uncc_sar_globals.hpp>
#include <charlotte_sar_api.hpp>

extern "C" {

// The grid the callback will use for these arrays: nx, ny, nfft and
// x0, y0, wx, wy, max_wy (metres).
int probe_callback_grid(float adf, float *samples, int K, float *start_f, float *chirp, float *x, float *y,
                        float *z, int np, int *dims, double *geom) {
    SAR_Aperture<float> ap;
    create_SARAperture<float>(adf, samples, K, start_f, chirp, x, y, z, np, ap);
    SAR_ImageFormationParameters<float> params;
    create_SARImageFormationParams(ap, params);
    dims[0] = params.N_x_pix;
    dims[1] = params.N_y_pix;
    dims[2] = params.N_fft;
    geom[0] = params.x0_m;
    geom[1] = params.y0_m;
    geom[2] = params.Wx_m;
    geom[3] = params.Wy_m;
    geom[4] = params.max_Wy_m;
    return 0;
}

// The callback itself; the BMP goes to bmp_path.
int probe_callback_gpu(const char *bmp_path, float adf, float *samples, int K, float *start_f, float *chirp,
                       float *x, float *y, float *z, int np) {
    outputfile = bmp_path;
    return sph_sar_data_callback_gpu<float>(0, adf, samples, K, start_f, chirp, x, y, z, np);
}

}  // extern "C"
