/*
 * TEST INFRASTRUCTURE -- not part of the shipped library.
 *
 * The six FFTW 3 single-precision entry points that the reference's
 * frequency-domain datuming tool calls (src/kirchdat2d_frequency_cs.cpp:1335-1339,
 * :309, :479, :1406-1407 and its fftwf_malloc/fftwf_free buffers), restated from
 * the published definition of the real discrete Fourier transform so that the
 * UNMODIFIED tool can be compiled from its own sources and linked here.  The
 * vendored FFTW (3.3.x, under fftw/ of the reference) needs its own configure or
 * cmake build and generated codelets, so it is not built.
 *
 * Conventions (FFTW 3 manual, "What FFTW Really Computes"):
 *   r2c, n real -> n/2+1 complex:   Y[k] = sum_j x[j] exp(-2 pi i j k / n)
 *   c2r, n/2+1 complex -> n real:   y[j] = sum_{k=0}^{n-1} X[k] exp(+2 pi i j k / n),
 *       with X[n-k] = conj(X[k]) (Hermitian extension; the imaginary parts of
 *       X[0] and, for even n, X[n/2] do not contribute); both unnormalised.
 * Computed in double (iterative radix-2 Cooley-Tukey for powers of two, the
 * direct O(n^2) sum otherwise) and rounded to float once, so the results differ
 * from an FFTW build by FFTW's own float rounding only.
 */
#include <fftw3.h>

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

struct fftwf_plan_s {
    int n, kind; /* kind 0: r2c, 1: c2r */
    float *rbuf;
    fftwf_complex *cbuf;
    double *wr, *wi; /* cos and sin of 2 pi k / n, k < n/2 */
    double *xr, *xi; /* work vectors, n each */
};

void *fftwf_malloc(size_t n)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1)) return NULL;
    return p;
}

void fftwf_free(void *p) { free(p); }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static fftwf_plan make_plan(int n, int kind, float *r, fftwf_complex *c)
{
    if (n <= 0) return NULL;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->n = n;
    p->kind = kind;
    p->rbuf = r;
    p->cbuf = c;
    p->xr = (double *)malloc(sizeof(double) * (size_t)n);
    p->xi = (double *)malloc(sizeof(double) * (size_t)n);
    const int nt = n > 1 ? n / 2 : 1;
    p->wr = (double *)malloc(sizeof(double) * (size_t)nt);
    p->wi = (double *)malloc(sizeof(double) * (size_t)nt);
    for (int k = 0; k < nt; k++) {
        const double a = 2.0 * M_PI * (double)k / (double)n;
        p->wr[k] = cos(a);
        p->wi[k] = sin(a);
    }
    return p;
}

fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags)
{
    (void)flags;
    return make_plan(n, 0, in, out);
}

fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags)
{
    (void)flags;
    return make_plan(n, 1, out, in);
}

void fftwf_destroy_plan(fftwf_plan p)
{
    if (!p) return;
    free(p->xr);
    free(p->xi);
    free(p->wr);
    free(p->wi);
    free(p);
}

/* in-place complex DFT of (xr, xi): X[k] = sum_j x[j] exp(sign 2 pi i j k / n),
   sign -1 (forward) or +1 (backward) */
static void dft(const struct fftwf_plan_s *p, int sign)
{
    const int n = p->n;
    double *xr = p->xr, *xi = p->xi;
    if (is_pow2(n)) {
        for (int i = 1, j = 0; i < n; i++) { /* bit reversal */
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double t = xr[i]; xr[i] = xr[j]; xr[j] = t;
                t = xi[i]; xi[i] = xi[j]; xi[j] = t;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1, stride = n / len;
            for (int s = 0; s < n; s += len) {
                for (int k = 0; k < half; k++) {
                    const double wr = p->wr[k * stride], wi = sign * p->wi[k * stride];
                    const int a = s + k, b = a + half;
                    const double tr = xr[b] * wr - xi[b] * wi, ti = xr[b] * wi + xi[b] * wr;
                    xr[b] = xr[a] - tr;
                    xi[b] = xi[a] - ti;
                    xr[a] += tr;
                    xi[a] += ti;
                }
            }
        }
        return;
    }
    double *yr = (double *)malloc(sizeof(double) * (size_t)n), *yi = (double *)malloc(sizeof(double) * (size_t)n);
    for (int k = 0; k < n; k++) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; j++) {
            const double a = sign * 2.0 * M_PI * (double)(((long long)j * k) % n) / (double)n;
            const double c = cos(a), s = sin(a);
            sr += xr[j] * c - xi[j] * s;
            si += xr[j] * s + xi[j] * c;
        }
        yr[k] = sr;
        yi[k] = si;
    }
    memcpy(xr, yr, sizeof(double) * (size_t)n);
    memcpy(xi, yi, sizeof(double) * (size_t)n);
    free(yr);
    free(yi);
}

void fftwf_execute(const fftwf_plan p)
{
    if (!p) return;
    const int n = p->n, nh = n / 2 + 1;
    if (p->kind == 0) {
        for (int j = 0; j < n; j++) {
            p->xr[j] = p->rbuf[j];
            p->xi[j] = 0.0;
        }
        dft(p, -1);
        for (int k = 0; k < nh; k++) {
            p->cbuf[k][0] = (float)p->xr[k];
            p->cbuf[k][1] = (float)p->xi[k];
        }
    } else {
        for (int k = 0; k < n; k++) {
            if (k < nh) {
                p->xr[k] = p->cbuf[k][0];
                p->xi[k] = p->cbuf[k][1];
            } else {
                p->xr[k] = p->cbuf[n - k][0];
                p->xi[k] = -p->cbuf[n - k][1];
            }
        }
        p->xi[0] = 0.0;
        if (n % 2 == 0) p->xi[n / 2] = 0.0;
        dft(p, +1);
        for (int j = 0; j < n; j++) p->rbuf[j] = (float)p->xr[j];
    }
}
