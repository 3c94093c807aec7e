/*
 * oracle/bp_oracle.c -- TEST INFRASTRUCTURE (the oracle), not product code.
 *
 * CPU restatement of the reference's backprojection (BP) hot path, used only
 * by tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg as the
 * checker.  Two instantiations of the same algorithm:
 *
 *   *_fp64  -- the accuracy oracle.  All arithmetic in double: geometry,
 *              differential range, phase, interpolation and accumulation.
 *              Follows matlab/bpBasic.m:61-97 and
 *              src/cpuBackProjection/cpuBackProjection.hpp:24-163 step for step
 *              (range-bin vector, strict swath gate, interp1 bracket search,
 *              phase exp(+j*4*pi*f0*dR/c), x-major accumulation).
 *
 *   *_ref32 -- the reference's own float semantics, operation for operation,
 *              so that it can be pinned against run_bp<float> compiled from
 *              the reference sources (oracle/ref_harness.cpp).  Float pixel
 *              accumulation (cpuBackProjection.hpp:55-62,89-91), float
 *              differential range (:65-70), phase argument formed in double
 *              and cast to float (:75-76), cosf/sinf through polar()
 *              (include/uncc_complex.hpp:81-84), index map
 *              RANGE_VALUE_TO_RANGE_INDEX (:47), interp1 (:24-42), the
 *              valarray "x /= x.size()" of ifftw that divides by a complex N
 *              (src/cpuBackProjection/cpuBackProjection_fft.hpp:44-46 with
 *              uncc_complex.hpp:193-200) and fftshift = cshift((N+1)/2)
 *              (cpuBackProjection_fft.hpp:81-84).
 *
 * Both build with -ffp-contract=off so every float operation rounds once,
 * as in the reference build; see oracle/Makefile.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

#define ORACLE_CLIGHT 299792458.0         /* include/uncc_sar_focusing.hpp:34 */
#define ORACLE_PI 3.141592653589793       /* include/uncc_sar_focusing.hpp:36 */

/* ------------------------------------------------------------------------- */
/* range compression                                                          */
/* ------------------------------------------------------------------------- */

/*
 * rc[p][i] = fftshift(ifft(w .* ph[p], nfft))[i] in double (matlab/bpBasic.m:82,
 * matlab/formImage3DSAR.m:115-116 for the taper).  ph is complex64 [Np][K]
 * (frequency fastest, as SAR_Aperture::sampleData, uncc_sar_focusing.hpp:68),
 * window is K doubles or NULL, rc is complex128 [Np][nfft].
 * ifft includes the 1/nfft scale; fftshift moves element (i + (nfft+1)/2) % nfft
 * to position i.
 */
static int range_compress_fp64_impl(int K, int Np, int nfft, const float *ph, const double *window,
                                    const double *cweights, double *rc);

int oracle_range_compress_fp64(int K, int Np, int nfft, const float *ph, const double *window, double *rc) {
    return range_compress_fp64_impl(K, Np, nfft, ph, window, NULL, rc);
}

/*
 * The same with complex per-sample weights c_k (interleaved doubles [K]) in
 * place of the real taper: rc_p = fftshift(ifft(c .* ph_p, nfft)), the
 * caller-supplied range weights of sarbp_plan_set_range_weights (a taper, a
 * range reference function, or both; matlab/rangeCompress.m:6-7).
 */
int oracle_range_compress_fp64_cw(int K, int Np, int nfft, const float *ph, const double *cweights, double *rc) {
    return range_compress_fp64_impl(K, Np, nfft, ph, NULL, cweights, rc);
}

static int range_compress_fp64_impl(int K, int Np, int nfft, const float *ph, const double *window,
                                    const double *cweights, double *rc) {
    if (K <= 0 || Np <= 0 || nfft < K || !ph || !rc) return -1;
    const int shift = (nfft + 1) / 2;
    int err = 0;
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)nfft);
        if (!buf) err = -2;
#pragma omp for schedule(static)
        for (int p = 0; p < Np; p++) {
            if (!buf) continue;
            for (int k = 0; k < nfft; k++) {
                double re = 0.0, im = 0.0;
                if (k < K) {
                    const double vr = (double)ph[2 * ((size_t)p * K + k)];
                    const double vi = (double)ph[2 * ((size_t)p * K + k) + 1];
                    if (cweights) {
                        re = cweights[2 * k] * vr - cweights[2 * k + 1] * vi;
                        im = cweights[2 * k] * vi + cweights[2 * k + 1] * vr;
                    } else {
                        const double w = window ? window[k] : 1.0;
                        re = w * vr;
                        im = w * vi;
                    }
                }
                buf[2 * k] = re;
                buf[2 * k + 1] = im;
            }
            oracle_dft_c128(nfft, buf, buf, FFTW_BACKWARD);
            double *out = rc + 2 * (size_t)p * nfft;
            for (int i = 0; i < nfft; i++) {
                const int src = (i + shift) % nfft;
                out[2 * i] = buf[2 * src] / (double)nfft;
                out[2 * i + 1] = buf[2 * src + 1] / (double)nfft;
            }
        }
        free(buf);
    }
    return err;
}

/*
 * The reference's float range compression of one pulse, run_bp<float>
 * (cpuBackProjection.hpp:151-158): ifftw on an N-sample slice, then the
 * valarray division by a Complex<float>(N, 0), then cshift((N+1)/2).
 * ph is complex64 [Np][nfft] (already zero-padded by the caller, since the
 * reference slices the phase history with stride N_fft), rc complex64 [Np][nfft].
 */
int oracle_range_compress_ref32(int nfft, int Np, const float *ph, float *rc) {
    if (nfft <= 0 || Np <= 0 || !ph || !rc) return -1;
    const int shift = (nfft + 1) / 2;
#pragma omp parallel
    {
        float *buf = (float *)malloc(sizeof(float) * 2 * (size_t)nfft);
#pragma omp for schedule(static)
        for (int p = 0; p < Np; p++) {
            if (!buf) continue;
            memcpy(buf, ph + 2 * (size_t)p * nfft, sizeof(float) * 2 * (size_t)nfft);
            fftwf_plan plan = fftwf_plan_dft_1d(nfft, (fftwf_complex *)buf, (fftwf_complex *)buf, FFTW_BACKWARD,
                                                FFTW_ESTIMATE);
            fftwf_execute(plan);
            fftwf_destroy_plan(plan);
            /* x /= Complex<float>(N, 0): complex division, uncc_complex.hpp:193-200 */
            const float nr = (float)nfft, ni = 0.0f;
            for (int i = 0; i < nfft; i++) {
                const float re = buf[2 * i], im = buf[2 * i + 1];
                const float r = re * nr + im * ni;
                const float n2 = nr * nr + ni * ni;
                const float imq = (im * nr - re * ni) / n2;
                buf[2 * i] = r / n2;
                buf[2 * i + 1] = imq;
            }
            float *out = rc + 2 * (size_t)p * nfft;
            for (int i = 0; i < nfft; i++) {
                const int src = (i + shift) % nfft;
                out[2 * i] = buf[2 * src];
                out[2 * i + 1] = buf[2 * src + 1];
            }
        }
        free(buf);
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* backprojection, FP64                                                       */
/* ------------------------------------------------------------------------- */

static inline double grid_coord(int i, int n, double c, double w) {
    /* linspace(c - w/2, c + w/2, n) (cpuBackProjection.hpp:55-62, bpBasic.m x_vec) */
    return (n > 1) ? (c - 0.5 * w) + (double)i * (w / (double)(n - 1)) : c;
}

/*
 * Contribution of every pulse to the pixel at (x, y, z); FP64.
 * rc: complex128 [Np][nfft] range profiles (fftshifted), r_vec the range-bin
 * vector r[i] = (i/nfft - 0.5) * max_wr (cpuBackProjection.hpp:114-135).
 */
static void bp_pixel_fp64(int Np, int nfft, const double *rc, const double *r_vec, const double *ax,
                          const double *ay, const double *az, const double *r0, const double *f0, double max_wr,
                          double x, double y, double z, double *out_re, double *out_im) {
    const double rmin = r_vec[0], rmax = r_vec[nfft - 1];
    double acc_re = 0.0, acc_im = 0.0;
    for (int p = 0; p < Np; p++) {
        const double dx = ax[p] - x, dy = ay[p] - y, dz = az[p] - z;
        const double dR = sqrt(dx * dx + dy * dy + dz * dz) - r0[p];
        if (!(dR > rmin && dR < rmax)) continue; /* strict swath gate, :71 */
        /* interp1 bracket search (:24-42) starting from floor(index) - 1 */
        const double idx = (dR / max_wr + 0.5) * (double)nfft;
        int right = (int)floor(idx) - 1;
        if (right < -1) right = -1;
        while (++right < nfft && r_vec[right] <= dR) {
        }
        if (right == nfft || right == 0) continue;
        const double alpha = (dR - r_vec[right - 1]) / (r_vec[right] - r_vec[right - 1]);
        const double *lo = rc + 2 * ((size_t)p * nfft + right - 1);
        const double *hi = rc + 2 * ((size_t)p * nfft + right);
        const double v_re = alpha * hi[0] + (1.0 - alpha) * lo[0];
        const double v_im = alpha * hi[1] + (1.0 - alpha) * lo[1];
        const double phi = 4.0 * ORACLE_PI * f0[p] * dR / ORACLE_CLIGHT;
        const double c = cos(phi), s = sin(phi);
        acc_re += v_re * c - v_im * s;
        acc_im += v_re * s + v_im * c;
    }
    *out_re = acc_re;
    *out_im = acc_im;
}

static double *make_rvec_fp64(int nfft, double max_wr) {
    double *r = (double *)malloc(sizeof(double) * (size_t)nfft);
    if (!r) return NULL;
    for (int i = 0; i < nfft; i++) r[i] = ((double)i / (double)nfft - 0.5) * max_wr;
    return r;
}

/*
 * Full image, FP64.  img is complex128 laid out [nz][nx][ny] (x-major within a
 * z-slice, img[x*Ny + y] as cpuBackProjection.hpp:87); z = z0 when nz == 1.
 */
int oracle_bp_fp64(int Np, int nfft, const double *rc, const double *ax, const double *ay, const double *az,
                   const double *r0, const double *f0, double max_wr, int nx, int ny, int nz, double x0,
                   double y0, double z0, double wx, double wy, double wz, double *img) {
    if (Np <= 0 || nfft < 2 || nx <= 0 || ny <= 0 || nz <= 0 || !rc || !img) return -1;
    double *r_vec = make_rvec_fp64(nfft, max_wr);
    if (!r_vec) return -2;
    const long long nxy = (long long)nx * ny;
#pragma omp parallel for schedule(dynamic, 16)
    for (long long row = 0; row < (long long)nz * nx; row++) {
        const int iz = (int)(row / nx), ix = (int)(row % nx);
        const double x = grid_coord(ix, nx, x0, wx);
        const double z = grid_coord(iz, nz, z0, wz);
        for (int iy = 0; iy < ny; iy++) {
            const double y = grid_coord(iy, ny, y0, wy);
            double re, im;
            bp_pixel_fp64(Np, nfft, rc, r_vec, ax, ay, az, r0, f0, max_wr, x, y, z, &re, &im);
            const long long o = (long long)iz * nxy + (long long)ix * ny + iy;
            img[2 * o] = re;
            img[2 * o + 1] = im;
        }
    }
    free(r_vec);
    return 0;
}

/*
 * Selected pixels only (flat indices into the [nz][nx][ny] image), FP64.
 * Used to check full-size images on a sample of pixels in seconds.
 */
int oracle_bp_fp64_pixels(int Np, int nfft, const double *rc, const double *ax, const double *ay,
                          const double *az, const double *r0, const double *f0, double max_wr, int nx, int ny,
                          int nz, double x0, double y0, double z0, double wx, double wy, double wz, long long npix,
                          const long long *pix, double *out) {
    if (Np <= 0 || nfft < 2 || nx <= 0 || ny <= 0 || nz <= 0 || !rc || !pix || !out) return -1;
    double *r_vec = make_rvec_fp64(nfft, max_wr);
    if (!r_vec) return -2;
    const long long nxy = (long long)nx * ny;
#pragma omp parallel for schedule(dynamic, 64)
    for (long long q = 0; q < npix; q++) {
        const long long o = pix[q];
        const int iz = (int)(o / nxy);
        const long long rem = o % nxy;
        const int ix = (int)(rem / ny), iy = (int)(rem % ny);
        double re, im;
        bp_pixel_fp64(Np, nfft, rc, r_vec, ax, ay, az, r0, f0, max_wr, grid_coord(ix, nx, x0, wx),
                      grid_coord(iy, ny, y0, wy), grid_coord(iz, nz, z0, wz), &re, &im);
        out[2 * q] = re;
        out[2 * q + 1] = im;
    }
    free(r_vec);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* backprojection, reference double semantics                                 */
/* ------------------------------------------------------------------------- */

/*
 * The reference's double path, run_bp<double,double> (cpuBackProjection.hpp:
 * 49-163 instantiated with double), restated with the float roundings it
 * contains switched on and nothing else changed from bp_pixel_fp64 above:
 *   - pixel coordinates are float and accumulate (:55-62,89-91);
 *   - dR is computed in double and stored to a float (:65-70);
 *   - interp1's xInterpLocation parameter is float (:25);
 *   - the range-bin vector is ((float)i/N - 0.5f) * maxWr in double (:45);
 *   - Complex<double>::operator*= keeps the real part in a float temporary
 *     (include/uncc_complex.hpp:186-191).
 * Pinning this against the compiled reference pins bp_pixel_fp64, which is
 * the same sequence of operations without those roundings.
 */
int oracle_range_compress_ref64(int nfft, int Np, const double *ph, double *rc) {
    if (nfft <= 0 || Np <= 0 || !ph || !rc) return -1;
    const int shift = (nfft + 1) / 2;
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)nfft);
#pragma omp for schedule(static)
        for (int p = 0; p < Np; p++) {
            if (!buf) continue;
            memcpy(buf, ph + 2 * (size_t)p * nfft, sizeof(double) * 2 * (size_t)nfft);
            oracle_dft_c128(nfft, buf, buf, FFTW_BACKWARD);
            const double nr = (double)nfft, ni = 0.0;
            for (int i = 0; i < nfft; i++) {
                const double re = buf[2 * i], im = buf[2 * i + 1];
                const double r = re * nr + im * ni;
                const double n2 = nr * nr + ni * ni;
                const double imq = (im * nr - re * ni) / n2;
                buf[2 * i] = r / n2;
                buf[2 * i + 1] = imq;
            }
            double *out = rc + 2 * (size_t)p * nfft;
            for (int i = 0; i < nfft; i++) {
                const int src = (i + shift) % nfft;
                out[2 * i] = buf[2 * src];
                out[2 * i + 1] = buf[2 * src + 1];
            }
        }
        free(buf);
    }
    return 0;
}

int oracle_bp_ref64(int Np, int nfft, const double *rc, const double *ax, const double *ay, const double *az,
                    const double *r0, const double *f0, double max_wr, int nx, int ny, double x0, double y0,
                    double wx, double wy, double *img) {
    if (Np <= 0 || nfft < 2 || nx <= 1 || ny <= 1 || !rc || !img) return -1;
    double *r_vec = (double *)malloc(sizeof(double) * (size_t)nfft);
    float *tx = (float *)malloc(sizeof(float) * (size_t)nx);
    float *ty = (float *)malloc(sizeof(float) * (size_t)ny);
    if (!r_vec || !tx || !ty) {
        free(r_vec); free(tx); free(ty);
        return -2;
    }
    double rmin = INFINITY, rmax = -INFINITY;
    for (int i = 0; i < nfft; i++) {
        r_vec[i] = (double)((float)i / (float)nfft - 0.5f) * max_wr;
        if (rmin > r_vec[i]) rmin = r_vec[i];
        if (rmax < r_vec[i]) rmax = r_vec[i];
    }
    const float delta_x = (float)(wx / (double)(nx - 1));
    const float delta_y = (float)(wy / (double)(ny - 1));
    float t = (float)(x0 - (wx / 2.0));
    for (int i = 0; i < nx; i++) { tx[i] = t; t += delta_x; }
    t = (float)(y0 - (wy / 2.0));
    for (int i = 0; i < ny; i++) { ty[i] = t; t += delta_y; }
    const float target_z = 0.0f;

#pragma omp parallel for schedule(dynamic, 4)
    for (int ix = 0; ix < nx; ix++) {
        for (int iy = 0; iy < ny; iy++) {
            double acc_re = 0.0, acc_im = 0.0;
            const double x = (double)tx[ix], y = (double)ty[iy], z = (double)target_z;
            for (int p = 0; p < Np; p++) {
                const double ex = ax[p] - x, ey = ay[p] - y, ez = az[p] - z;
                const float dR = (float)(sqrt(ex * ex + ey * ey + ez * ez) - r0[p]);
                if (!((double)dR > rmin && (double)dR < rmax)) continue;
                const double phi = (4.0 * ORACLE_PI * f0[p] * (double)dR) / ORACLE_CLIGHT;
                const double c = (double)1.0f * cos(phi), s = (double)1.0f * sin(phi);
                const double dR_idx = ((double)dR / max_wr + 0.5f) * (double)nfft;
                int right = (int)(floor(dR_idx) - 1);
                while (++right < nfft && r_vec[right] <= (double)dR) {
                }
                if (right == nfft || right == 0) continue;
                const double alpha = ((double)dR - r_vec[right - 1]) / (r_vec[right] - r_vec[right - 1]);
                const double *lo = rc + 2 * ((size_t)p * nfft + right - 1);
                const double *hi = rc + 2 * ((size_t)p * nfft + right);
                const double v_re = alpha * hi[0] + (1.0 - alpha) * lo[0];
                const double v_im = alpha * hi[1] + (1.0 - alpha) * lo[1];
                const float m_re = (float)(v_re * c - v_im * s);
                const double m_im = v_re * s + v_im * c;
                acc_re += (double)m_re;
                acc_im += m_im;
            }
            img[2 * ((size_t)ix * ny + iy)] = acc_re;
            img[2 * ((size_t)ix * ny + iy) + 1] = acc_im;
        }
    }
    free(r_vec);
    free(tx);
    free(ty);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* backprojection, reference float semantics                                  */
/* ------------------------------------------------------------------------- */

/*
 * run_bp<float> / computeDifferentialRangeAndPhaseCorrections<float,float>
 * (cpuBackProjection.hpp:49-93,95-163) restated operation for operation.
 * rc: complex64 [Np][nfft] range profiles produced by oracle_range_compress_ref32.
 * Pixel coordinates accumulate in float along x and y (:55-62,89-91); the
 * scene plane is z = 0 (:57).  img: complex64 [nx][ny].
 */
int oracle_bp_ref32(int Np, int nfft, const float *rc, const float *ax, const float *ay, const float *az,
                    const float *r0, const float *f0, float max_wr, int nx, int ny, float x0, float y0, float wx,
                    float wy, float *img) {
    if (Np <= 0 || nfft < 2 || nx <= 1 || ny <= 1 || !rc || !img) return -1;
    float *r_vec = (float *)malloc(sizeof(float) * (size_t)nfft);
    float *tx = (float *)malloc(sizeof(float) * (size_t)nx);
    float *ty = (float *)malloc(sizeof(float) * (size_t)ny);
    if (!r_vec || !tx || !ty) {
        free(r_vec); free(tx); free(ty);
        return -2;
    }
    /* RANGE_INDEX_TO_RANGE_VALUE: ((float) idx / N - 0.5f) * maxWr (:45) */
    float rmin = INFINITY, rmax = -INFINITY;
    for (int i = 0; i < nfft; i++) {
        r_vec[i] = ((float)i / (float)nfft - 0.5f) * max_wr;
        if (rmin > r_vec[i]) rmin = r_vec[i];
        if (rmax < r_vec[i]) rmax = r_vec[i];
    }
    const float delta_x = wx / (float)(nx - 1);
    const float delta_y = wy / (float)(ny - 1);
    float t = x0 - (wx / 2.0f);
    for (int i = 0; i < nx; i++) { tx[i] = t; t += delta_x; }
    t = y0 - (wy / 2.0f);
    for (int i = 0; i < ny; i++) { ty[i] = t; t += delta_y; }
    const float target_z = 0.0f;

#pragma omp parallel for schedule(dynamic, 4)
    for (int ix = 0; ix < nx; ix++) {
        for (int iy = 0; iy < ny; iy++) {
            float acc_re = 0.0f, acc_im = 0.0f;
            const float x = tx[ix], y = ty[iy];
            for (int p = 0; p < Np; p++) {
                const float ex = ax[p] - x, ey = ay[p] - y, ez = az[p] - target_z;
                const float dR = sqrtf(ex * ex + ey * ey + ez * ez) - r0[p];
                if (!(dR > rmin && dR < rmax)) continue;
                const float phi = (float)((4.0 * ORACLE_PI * (double)f0[p] * (double)dR) / ORACLE_CLIGHT);
                const float c = 1.0f * cosf(phi), s = 1.0f * sinf(phi);
                const float dR_idx = (dR / max_wr + 0.5f) * (float)nfft;
                int right = (int)(floorf(dR_idx) - 1);
                while (++right < nfft && r_vec[right] <= dR) {
                }
                if (right == nfft || right == 0) continue;
                const float alpha = (dR - r_vec[right - 1]) / (r_vec[right] - r_vec[right - 1]);
                const float *lo = rc + 2 * ((size_t)p * nfft + right - 1);
                const float *hi = rc + 2 * ((size_t)p * nfft + right);
                const float one_m = 1.0f - alpha;
                const float v_re = alpha * hi[0] + one_m * lo[0];
                const float v_im = alpha * hi[1] + one_m * lo[1];
                const float m_re = v_re * c - v_im * s;
                const float m_im = v_re * s + v_im * c;
                acc_re += m_re;
                acc_im += m_im;
            }
            img[2 * ((size_t)ix * ny + iy)] = acc_re;
            img[2 * ((size_t)ix * ny + iy) + 1] = acc_im;
        }
    }
    free(r_vec);
    free(tx);
    free(ty);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* gradient of a real image loss with respect to the pulse geometry, FP64     */
/* ------------------------------------------------------------------------- */

/*
 * For img_q = sum_p v_p(b_pq) exp(j phi_pq) (bp_pixel_fp64 above) and the
 * upstream gradient G_q = dL/dRe(img_q) + j dL/dIm(img_q):
 *   s_pq = Re(conj(G_q) (lambda v'_p(b) + j 2 pi k_p v_p(b)) exp(j phi_pq)),
 *   dL/da_p = sum_q s_pq (a_p - x_q)/|a_p - x_q|,   dL/dR0_p = -sum_q s_pq,
 * with lambda = nfft / max_wr, k_p = 2 f0_p / c and v'_p the slope of the
 * linear interpolation on the bracket interp1 selects.  G and the image are
 * [nz][nx][ny]; outputs are double [Np].  There is no reference counterpart
 * (the reference's autofocus is a grid search); this is the exact derivative
 * of the FP64 forward restatement, used to check the GPU adjoint.
 */
int oracle_bp_grad_fp64(int Np, int nfft, const double *rc, const double *ax, const double *ay, const double *az,
                        const double *r0, const double *f0, double max_wr, int nx, int ny, int nz, double x0,
                        double y0, double z0, double wx, double wy, double wz, const double *G, double *gax,
                        double *gay, double *gaz, double *gr0) {
    if (Np <= 0 || nfft < 2 || nx <= 0 || ny <= 0 || nz <= 0 || !rc || !G || !gax || !gay || !gaz) return -1;
    double *r_vec = make_rvec_fp64(nfft, max_wr);
    if (!r_vec) return -2;
    const double rmin = r_vec[0], rmax = r_vec[nfft - 1];
    const double lam = (double)nfft / max_wr;
    const long long nxy = (long long)nx * ny;
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < Np; p++) {
        const double k = 2.0 * f0[p] / ORACLE_CLIGHT;
        double sx = 0.0, sy = 0.0, sz = 0.0, s0 = 0.0;
        for (int iz = 0; iz < nz; iz++) {
            const double z = grid_coord(iz, nz, z0, wz);
            for (int ix = 0; ix < nx; ix++) {
                const double x = grid_coord(ix, nx, x0, wx);
                for (int iy = 0; iy < ny; iy++) {
                    const double y = grid_coord(iy, ny, y0, wy);
                    const double dx = ax[p] - x, dy = ay[p] - y, dz = az[p] - z;
                    const double R = sqrt(dx * dx + dy * dy + dz * dz);
                    const double dR = R - r0[p];
                    if (!(dR > rmin && dR < rmax)) continue;
                    const double idx = (dR / max_wr + 0.5) * (double)nfft;
                    int right = (int)floor(idx) - 1;
                    if (right < -1) right = -1;
                    while (++right < nfft && r_vec[right] <= dR) {
                    }
                    if (right == nfft || right == 0) continue;
                    const double alpha = (dR - r_vec[right - 1]) / (r_vec[right] - r_vec[right - 1]);
                    const double *lo = rc + 2 * ((size_t)p * nfft + right - 1);
                    const double *hi = rc + 2 * ((size_t)p * nfft + right);
                    const double vr = alpha * hi[0] + (1.0 - alpha) * lo[0];
                    const double vi = alpha * hi[1] + (1.0 - alpha) * lo[1];
                    const double dr = hi[0] - lo[0], di = hi[1] - lo[1];
                    const double phi = 4.0 * ORACLE_PI * f0[p] * dR / ORACLE_CLIGHT;
                    const double c = cos(phi), s = sin(phi);
                    /* D = (lambda v' + j 2 pi k v) exp(j phi) */
                    const double pr = lam * dr - 2.0 * ORACLE_PI * k * vi;
                    const double pi_ = lam * di + 2.0 * ORACLE_PI * k * vr;
                    const double Dr = pr * c - pi_ * s, Di = pr * s + pi_ * c;
                    const long long o = (long long)iz * nxy + (long long)ix * ny + iy;
                    const double sv = G[2 * o] * Dr + G[2 * o + 1] * Di; /* Re(conj(G) D) */
                    sx += sv * dx / R;
                    sy += sv * dy / R;
                    sz += sv * dz / R;
                    s0 += sv;
                }
            }
        }
        gax[p] = sx;
        gay[p] = sy;
        gaz[p] = sz;
        if (gr0) gr0[p] = -s0;
    }
    free(r_vec);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* matched filter, FP64                                                       */
/* ------------------------------------------------------------------------- */

/*
 * Matched-filter image (matlab/mfBasic.m:73-89; cpuBackProjection.hpp:165-228):
 *     img[q] += ph_p[k] * exp(+j 4 pi (f0_p + k dF) dR_pq / c)
 * for pulses p >= first_pulse and samples k < K, dR = |a_p - x_q| - R0_p,
 * every term in double with cos / sin of the full phase.  ph: complex128
 * [Np][K] (any taper already applied).  first_pulse = 0 is MATLAB's loop;
 * the reference C++ loop starts at pulse 2 (cpuBackProjection.hpp:216-218).
 * img: complex128 [nz][nx][ny].
 */
int oracle_mf_fp64(int Np, int K, const double *ph, const double *ax, const double *ay, const double *az,
                   const double *r0, const double *f0, double df, int nx, int ny, int nz, double x0, double y0,
                   double z0, double wx, double wy, double wz, int first_pulse, double *img) {
    if (Np <= 0 || K <= 0 || nx <= 0 || ny <= 0 || nz <= 0 || !ph || !img) return -1;
    const long long nxy = (long long)nx * ny;
#pragma omp parallel for schedule(dynamic, 16)
    for (long long row = 0; row < (long long)nz * nx; row++) {
        const int iz = (int)(row / nx), ix = (int)(row % nx);
        const double x = grid_coord(ix, nx, x0, wx);
        const double z = grid_coord(iz, nz, z0, wz);
        for (int iy = 0; iy < ny; iy++) {
            const double y = grid_coord(iy, ny, y0, wy);
            double acc_re = 0.0, acc_im = 0.0;
            for (int p = first_pulse; p < Np; p++) {
                const double dx = ax[p] - x, dy = ay[p] - y, dz = az[p] - z;
                const double dR = sqrt(dx * dx + dy * dy + dz * dz) - r0[p];
                const double *s = ph + 2 * (size_t)p * K;
                for (int k = 0; k < K; k++) {
                    const double phi = 4.0 * ORACLE_PI * (f0[p] + (double)k * df) * dR / ORACLE_CLIGHT;
                    const double c = cos(phi), sn = sin(phi);
                    acc_re += s[2 * k] * c - s[2 * k + 1] * sn;
                    acc_im += s[2 * k] * sn + s[2 * k + 1] * c;
                }
            }
            const long long o = (long long)iz * nxy + (long long)ix * ny + iy;
            img[2 * o] = acc_re;
            img[2 * o + 1] = acc_im;
        }
    }
    return 0;
}
