/*
 * oracle/fftw3.h -- TEST INFRASTRUCTURE (the oracle), not product code.
 *
 * The subset of the FFTW3 C API that the reference CPU backprojection uses
 * (src/cpuBackProjection/cpuBackProjection_fft.hpp:31-69: fftw{f}_plan_dft_1d,
 * fftw{f}_execute, fftw{f}_destroy_plan, FFTW_FORWARD/BACKWARD, FFTW_ESTIMATE).
 * FFTW itself is not installed in this image, so the reference header is
 * compiled against this declaration and the project FFT in oracle/fft.c,
 * which computes the same unnormalised DFT
 *     out[n] = sum_k in[k] * exp(sign * 2*pi*i * k*n / N),  sign = -1 / +1
 * for FFTW_FORWARD / FFTW_BACKWARD, exactly as FFTW documents it.
 * Only the oracle (oracle/Makefile) includes this file.
 */
#ifndef SARBP_ORACLE_FFTW3_H
#define SARBP_ORACLE_FFTW3_H

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef double fftw_complex[2];
typedef float fftwf_complex[2];

typedef struct oracle_fft_plan_s *fftw_plan;
typedef struct oracle_fft_plan_s *fftwf_plan;

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);

/* Project-level entry used by the oracle's own restatement (same transform,
 * double precision, out-of-place allowed, in == out allowed). */
int oracle_dft_c128(int n, const double *in, double *out, int sign);

#ifdef __cplusplus
}
#endif

#endif /* SARBP_ORACLE_FFTW3_H */
