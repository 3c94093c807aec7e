/*
 * oracle/fft.c -- TEST INFRASTRUCTURE (the oracle), not product code.
 *
 * A double-precision FFT behind the FFTW3 API subset declared in
 * oracle/fftw3.h.  It exists because FFTW is not installed here and the
 * reference CPU backprojection (src/cpuBackProjection/cpuBackProjection_fft.hpp:
 * 31-79, fftw_engine/ifftw) needs it; the project's own oracle
 * (oracle/bp_oracle.c) uses the same transform for its range compression.
 *
 * Method (textbook, no library code):
 *   - recursive decimation-in-time Cooley-Tukey over the prime factorisation
 *     of N (radix 4 and 2 butterflies written out, any other radix p <= 64 by
 *     a direct p-point DFT of the twiddled inputs);
 *   - Bluestein's chirp-z algorithm (Bluestein 1970; Rabiner, Schafer & Rader
 *     1969) when N has a prime factor > 64: the DFT becomes a circular
 *     convolution of length M = 2^ceil(log2(2N-1)) done with the radix-2 path.
 * All arithmetic is in double; twiddles come from cos/sin of 2*pi*t/N with t
 * reduced modulo N first, so the float API is accurate to float rounding.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double re, im;
} cplx;

typedef struct fft_core {
    int n;
    int sign;
    int nfac;
    int fac[64];
    cplx *tw; /* tw[t] = exp(sign * 2*pi*i * t / n), t < n */
    /* Bluestein state (used when blu_m > 0) */
    int blu_m;
    cplx *blu_chirp; /* b[t] = exp(sign * pi*i * t^2 / n), t < n */
    cplx *blu_hf;    /* forward FFT (length m) of the conjugate chirp, pre-scaled by 1/m */
    struct fft_core *blu_fwd, *blu_inv;
    cplx *blu_buf;
} fft_core;

struct oracle_fft_plan_s {
    fft_core *core;
    int is_float;
    void *in, *out;
    cplx *work_in, *work_out;
};

static const double TWO_PI = 6.283185307179586476925286766559;

static int factorize(int n, int *fac, int *nfac) {
    int k = 0;
    while (n % 4 == 0) { fac[k++] = 4; n /= 4; }
    while (n % 2 == 0) { fac[k++] = 2; n /= 2; }
    for (int p = 3; p <= 64 && n > 1; p += 2) {
        while (n % p == 0) { fac[k++] = p; n /= p; }
    }
    *nfac = k;
    return n; /* remaining factor (> 1 means a prime > 64 is left) */
}

static void core_free(fft_core *c);
void oracle_fft_core_exec(const fft_core *c, const cplx *in, cplx *out);

static fft_core *core_new(int n, int sign) {
    fft_core *c = (fft_core *)calloc(1, sizeof(fft_core));
    if (!c) return NULL;
    c->n = n;
    c->sign = sign;
    c->tw = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    if (!c->tw) { free(c); return NULL; }
    for (int t = 0; t < n; t++) {
        double a = TWO_PI * (double)t / (double)n;
        c->tw[t].re = cos(a);
        c->tw[t].im = (double)sign * sin(a);
    }
    int rest = factorize(n, c->fac, &c->nfac);
    if (rest > 1) {
        /* Bluestein: X_k = b_k * sum_j (x_j b_j) conj(b_{k-j}), b_t = exp(sign*pi*i*t^2/n) */
        int m = 1;
        while (m < 2 * n - 1) m <<= 1;
        c->nfac = 0;
        c->blu_m = m;
        c->blu_chirp = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        c->blu_hf = (cplx *)calloc((size_t)m, sizeof(cplx));
        c->blu_buf = (cplx *)malloc(sizeof(cplx) * (size_t)m);
        c->blu_fwd = core_new(m, -1);
        c->blu_inv = core_new(m, +1);
        if (!c->blu_chirp || !c->blu_hf || !c->blu_buf || !c->blu_fwd || !c->blu_inv) {
            core_free(c);
            return NULL;
        }
        for (int t = 0; t < n; t++) {
            long long t2 = ((long long)t * (long long)t) % (2LL * n);
            double a = M_PI * (double)t2 / (double)n;
            c->blu_chirp[t].re = cos(a);
            c->blu_chirp[t].im = (double)sign * sin(a);
        }
        /* h_t = conj(b_|t|) laid out circularly for t in (-n, n) */
        cplx *h = (cplx *)calloc((size_t)m, sizeof(cplx));
        if (!h) { core_free(c); return NULL; }
        for (int t = 0; t < n; t++) {
            cplx v = {c->blu_chirp[t].re, -c->blu_chirp[t].im};
            h[t] = v;
            if (t > 0) h[m - t] = v;
        }
        oracle_fft_core_exec(c->blu_fwd, h, c->blu_hf);
        for (int t = 0; t < m; t++) {
            c->blu_hf[t].re /= (double)m;
            c->blu_hf[t].im /= (double)m;
        }
        free(h);
    }
    return c;
}

static void core_free(fft_core *c) {
    if (!c) return;
    free(c->tw);
    free(c->blu_chirp);
    free(c->blu_hf);
    free(c->blu_buf);
    core_free(c->blu_fwd);
    core_free(c->blu_inv);
    free(c);
}

/* out[0..n) = DFT of in[0], in[stride], ..., using factors fac[fi..] */
static void rec(const fft_core *c, const cplx *in, int stride, cplx *out, int n, int fi) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int p = c->fac[fi];
    const int m = n / p;
    for (int j = 0; j < p; j++) rec(c, in + (size_t)j * stride, stride * p, out + (size_t)j * m, m, fi + 1);
    const int N = c->n;
    const int tstep = N / n; /* w_n^x = tw[x * tstep] */
    cplx y[64];
    for (int k = 0; k < m; k++) {
        for (int j = 0; j < p; j++) {
            cplx a = out[(size_t)j * m + k];
            if (j == 0 || k == 0) {
                y[j] = a;
            } else {
                cplx w = c->tw[(int)(((long long)j * k * tstep) % N)];
                y[j].re = a.re * w.re - a.im * w.im;
                y[j].im = a.re * w.im + a.im * w.re;
            }
        }
        if (p == 2) {
            out[k].re = y[0].re + y[1].re;
            out[k].im = y[0].im + y[1].im;
            out[k + m].re = y[0].re - y[1].re;
            out[k + m].im = y[0].im - y[1].im;
        } else if (p == 4) {
            /* w_4 = exp(sign*i*pi/2) = sign*i */
            const double s = (double)c->sign;
            cplx a0 = {y[0].re + y[2].re, y[0].im + y[2].im};
            cplx a1 = {y[0].re - y[2].re, y[0].im - y[2].im};
            cplx b0 = {y[1].re + y[3].re, y[1].im + y[3].im};
            cplx b1 = {y[1].re - y[3].re, y[1].im - y[3].im};
            /* (sign*i) * b1 */
            cplx rb1 = {-s * b1.im, s * b1.re};
            out[k].re = a0.re + b0.re;
            out[k].im = a0.im + b0.im;
            out[k + m].re = a1.re + rb1.re;
            out[k + m].im = a1.im + rb1.im;
            out[k + 2 * m].re = a0.re - b0.re;
            out[k + 2 * m].im = a0.im - b0.im;
            out[k + 3 * m].re = a1.re - rb1.re;
            out[k + 3 * m].im = a1.im - rb1.im;
        } else {
            const int pstep = N / p; /* w_p^x = tw[x * pstep] */
            for (int q = 0; q < p; q++) {
                double sr = 0.0, si = 0.0;
                for (int j = 0; j < p; j++) {
                    cplx w = c->tw[((j * q) % p) * pstep];
                    sr += y[j].re * w.re - y[j].im * w.im;
                    si += y[j].re * w.im + y[j].im * w.re;
                }
                out[k + (size_t)q * m].re = sr;
                out[k + (size_t)q * m].im = si;
            }
        }
    }
}

void oracle_fft_core_exec(const fft_core *c, const cplx *in, cplx *out) {
    const int n = c->n;
    if (c->blu_m == 0) {
        if (in == out) {
            cplx *tmp = (cplx *)malloc(sizeof(cplx) * (size_t)n);
            memcpy(tmp, in, sizeof(cplx) * (size_t)n);
            rec(c, tmp, 1, out, n, 0);
            free(tmp);
        } else {
            rec(c, in, 1, out, n, 0);
        }
        return;
    }
    const int m = c->blu_m;
    cplx *a = (cplx *)calloc((size_t)m, sizeof(cplx));
    cplx *af = c->blu_buf;
    for (int t = 0; t < n; t++) {
        cplx b = c->blu_chirp[t];
        a[t].re = in[t].re * b.re - in[t].im * b.im;
        a[t].im = in[t].re * b.im + in[t].im * b.re;
    }
    rec(c->blu_fwd, a, 1, af, m, 0);
    for (int t = 0; t < m; t++) {
        cplx h = c->blu_hf[t];
        double r = af[t].re * h.re - af[t].im * h.im;
        double i = af[t].re * h.im + af[t].im * h.re;
        af[t].re = r;
        af[t].im = i;
    }
    rec(c->blu_inv, af, 1, a, m, 0);
    for (int t = 0; t < n; t++) {
        cplx b = c->blu_chirp[t];
        out[t].re = a[t].re * b.re - a[t].im * b.im;
        out[t].im = a[t].re * b.im + a[t].im * b.re;
    }
    free(a);
}

int oracle_dft_c128(int n, const double *in, double *out, int sign) {
    if (n <= 0) return -1;
    fft_core *c = core_new(n, sign < 0 ? -1 : +1);
    if (!c) return -2;
    oracle_fft_core_exec(c, (const cplx *)in, (cplx *)out);
    core_free(c);
    return 0;
}

static struct oracle_fft_plan_s *plan_new(int n, void *in, void *out, int sign, int is_float) {
    if (n <= 0) return NULL;
    struct oracle_fft_plan_s *p = (struct oracle_fft_plan_s *)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->core = core_new(n, sign < 0 ? -1 : +1);
    p->work_in = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    p->work_out = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    if (!p->core || !p->work_in || !p->work_out) {
        core_free(p->core);
        free(p->work_in);
        free(p->work_out);
        free(p);
        return NULL;
    }
    p->is_float = is_float;
    p->in = in;
    p->out = out;
    return p;
}

static void plan_exec(struct oracle_fft_plan_s *p) {
    const int n = p->core->n;
    if (p->is_float) {
        const float *fi = (const float *)p->in;
        for (int t = 0; t < n; t++) {
            p->work_in[t].re = fi[2 * t];
            p->work_in[t].im = fi[2 * t + 1];
        }
    } else {
        memcpy(p->work_in, p->in, sizeof(cplx) * (size_t)n);
    }
    oracle_fft_core_exec(p->core, p->work_in, p->work_out);
    if (p->is_float) {
        float *fo = (float *)p->out;
        for (int t = 0; t < n; t++) {
            fo[2 * t] = (float)p->work_out[t].re;
            fo[2 * t + 1] = (float)p->work_out[t].im;
        }
    } else {
        memcpy(p->out, p->work_out, sizeof(cplx) * (size_t)n);
    }
}

static void plan_free(struct oracle_fft_plan_s *p) {
    if (!p) return;
    core_free(p->core);
    free(p->work_in);
    free(p->work_out);
    free(p);
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags;
    return plan_new(n, in, out, sign, 0);
}
void fftw_execute(const fftw_plan p) { plan_exec(p); }
void fftw_destroy_plan(fftw_plan p) { plan_free(p); }

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags) {
    (void)flags;
    return plan_new(n, in, out, sign, 1);
}
void fftwf_execute(const fftwf_plan p) { plan_exec(p); }
void fftwf_destroy_plan(fftwf_plan p) { plan_free(p); }
