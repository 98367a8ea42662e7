/*
 * FFTW-API shim — TEST INFRASTRUCTURE ONLY (oracle).  Not part of the product.
 *
 * FFTW 3.3.3 (the dependency named in Readme.md:24, not vendored in the
 * reference and not installed here) is replaced by this file when the
 * reference solvers are compiled as the CPU oracle.  It implements the six
 * entry points the reference calls (see fftw3.h for the call sites) from the
 * transform definitions FFTW publishes (FFTW 3.3 manual, section 4.8):
 *
 *   complex DFT  : Y[k] = sum_j X[j] w^(jk),  w = exp(sign 2 pi i / n), unnormalised
 *   r2c          : the forward DFT of real data, outputs k = 0..n/2 of the last axis
 *   c2r          : the backward DFT of Hermitian data (imaginary parts of the
 *                  k=0 and k=n/2 entries of the last axis are ignored)
 *   REDFT10      : Y[k] = 2 sum_j X[j] cos(pi (j + 1/2) k / n)
 *   REDFT01      : Y[k] = X[0] + 2 sum_{j>=1} X[j] cos(pi j (k + 1/2) / n)
 *
 * Algorithms (own code): a batched mixed-radix Stockham FFT (radix 4, 2, 3, 5,
 * generic odd factors) whose inner loop runs over a batch of L lines laid out
 * [n][L]; r2c/c2r of even length by the half-length complex transform;
 * DCT-II / DCT-III of even length by Makhoul's reordering (IEEE TASSP 28(1),
 * 1980).  Twiddles are evaluated in long double and rounded once.
 * Multi-dimensional transforms apply the 1-D transforms axis by axis.
 * Lines are processed in parallel with OpenMP.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SHIM_BATCH 16
static const long double SHIM_PI = 3.141592653589793238462643383279502884L;

/* ------------------------------------------------------------------------- */
/* 1-D complex FFT plans (cached per length)                                  */
/* ------------------------------------------------------------------------- */
typedef struct cplan {
    int n;
    int nfac;
    int fac[32];
    double* wre; /* exp(-2 pi i k / n), k < n */
    double* wim;
    struct cplan* next;
} cplan;

static cplan* g_cplans = NULL;

static cplan* cplan_get(int n) {
    cplan* p;
    for (p = __atomic_load_n(&g_cplans, __ATOMIC_ACQUIRE); p; p = p->next)
        if (p->n == n) return p;
#ifdef _OPENMP
#pragma omp critical(crysscft_shim_plan)
#endif
    {
        for (p = g_cplans; p; p = p->next)
            if (p->n == n) break;
        if (!p) {
            p = (cplan*)calloc(1, sizeof(cplan));
            p->n = n;
            int m = n;
            while (m % 4 == 0) { p->fac[p->nfac++] = 4; m /= 4; }
            while (m % 2 == 0) { p->fac[p->nfac++] = 2; m /= 2; }
            while (m % 3 == 0) { p->fac[p->nfac++] = 3; m /= 3; }
            while (m % 5 == 0) { p->fac[p->nfac++] = 5; m /= 5; }
            for (int f = 7; m > 1; f += 2)
                while (m % f == 0) { p->fac[p->nfac++] = f; m /= f; }
            p->wre = (double*)malloc(sizeof(double) * (size_t)n);
            p->wim = (double*)malloc(sizeof(double) * (size_t)n);
            for (int k = 0; k < n; ++k) {
                long double a = -2.0L * SHIM_PI * (long double)k / (long double)n;
                p->wre[k] = (double)cosl(a);
                p->wim[k] = (double)sinl(a);
            }
            p->next = g_cplans;
            __atomic_store_n(&g_cplans, p, __ATOMIC_RELEASE);
        }
    }
    return p;
}

/*
 * Batched Stockham autosort FFT.  Data: xr/xi[j*L + l], j < n, l < L.
 * sign = -1 forward, +1 backward.  yr/yi are scratch of the same size.
 * The result is written back to xr/xi.
 */
static void cfft_batch(const cplan* P, double* xr, double* xi, double* yr, double* yi,
                       int L, int sign) {
    const int n = P->n;
    if (n == 1) return;
    int len = n, s = 1;
    double *ar = xr, *ai = xi, *br = yr, *bi = yi;
    for (int f = 0; f < P->nfac; ++f) {
        const int r = P->fac[f];
        const int m = len / r;
        const int tws = n / len; /* W_len^e = W_n^(e*tws) */
        const size_t blk = (size_t)s * (size_t)L;
        for (int p = 0; p < m; ++p) {
            if (r == 2) {
                const int e = (p * tws) % n;
                const double wr = P->wre[e], wi = sign < 0 ? P->wim[e] : -P->wim[e];
                const double* a0r = ar + (size_t)(p) * blk;
                const double* a0i = ai + (size_t)(p) * blk;
                const double* a1r = ar + (size_t)(p + m) * blk;
                const double* a1i = ai + (size_t)(p + m) * blk;
                double* b0r = br + (size_t)(2 * p) * blk;
                double* b0i = bi + (size_t)(2 * p) * blk;
                double* b1r = br + (size_t)(2 * p + 1) * blk;
                double* b1i = bi + (size_t)(2 * p + 1) * blk;
                for (size_t t = 0; t < blk; ++t) {
                    double ur = a0r[t], ui = a0i[t], vr = a1r[t], vi = a1i[t];
                    b0r[t] = ur + vr;
                    b0i[t] = ui + vi;
                    double dr = ur - vr, di = ui - vi;
                    b1r[t] = dr * wr - di * wi;
                    b1i[t] = dr * wi + di * wr;
                }
            } else if (r == 4) {
                double w1r, w1i, w2r, w2i, w3r, w3i;
                {
                    int e1 = (p * tws) % n, e2 = (2 * p * tws) % n, e3 = (3 * p * tws) % n;
                    double sg = sign < 0 ? 1.0 : -1.0;
                    w1r = P->wre[e1]; w1i = sg * P->wim[e1];
                    w2r = P->wre[e2]; w2i = sg * P->wim[e2];
                    w3r = P->wre[e3]; w3i = sg * P->wim[e3];
                }
                const double* a0r = ar + (size_t)(p) * blk;
                const double* a0i = ai + (size_t)(p) * blk;
                const double* a1r = ar + (size_t)(p + m) * blk;
                const double* a1i = ai + (size_t)(p + m) * blk;
                const double* a2r = ar + (size_t)(p + 2 * m) * blk;
                const double* a2i = ai + (size_t)(p + 2 * m) * blk;
                const double* a3r = ar + (size_t)(p + 3 * m) * blk;
                const double* a3i = ai + (size_t)(p + 3 * m) * blk;
                double* b0r = br + (size_t)(4 * p) * blk;
                double* b0i = bi + (size_t)(4 * p) * blk;
                double* b1r = br + (size_t)(4 * p + 1) * blk;
                double* b1i = bi + (size_t)(4 * p + 1) * blk;
                double* b2r = br + (size_t)(4 * p + 2) * blk;
                double* b2i = bi + (size_t)(4 * p + 2) * blk;
                double* b3r = br + (size_t)(4 * p + 3) * blk;
                double* b3i = bi + (size_t)(4 * p + 3) * blk;
                /* DFT_4 with w4 = exp(sign i pi/2): multiplying by w4 is (x,y)->(-sign*y, sign*x) */
                const double sg = (double)sign;
                for (size_t t = 0; t < blk; ++t) {
                    double x0r = a0r[t], x0i = a0i[t], x1r = a1r[t], x1i = a1i[t];
                    double x2r = a2r[t], x2i = a2i[t], x3r = a3r[t], x3i = a3i[t];
                    double s02r = x0r + x2r, s02i = x0i + x2i;
                    double d02r = x0r - x2r, d02i = x0i - x2i;
                    double s13r = x1r + x3r, s13i = x1i + x3i;
                    double d13r = x1r - x3r, d13i = x1i - x3i;
                    /* j*d13 where j = exp(sign i pi/2) */
                    double jd13r = -sg * d13i, jd13i = sg * d13r;
                    double c0r = s02r + s13r, c0i = s02i + s13i;
                    double c1r = d02r + jd13r, c1i = d02i + jd13i;
                    double c2r = s02r - s13r, c2i = s02i - s13i;
                    double c3r = d02r - jd13r, c3i = d02i - jd13i;
                    b0r[t] = c0r;
                    b0i[t] = c0i;
                    b1r[t] = c1r * w1r - c1i * w1i;
                    b1i[t] = c1r * w1i + c1i * w1r;
                    b2r[t] = c2r * w2r - c2i * w2i;
                    b2i[t] = c2r * w2i + c2i * w2r;
                    b3r[t] = c3r * w3r - c3i * w3i;
                    b3i[t] = c3r * w3i + c3i * w3r;
                }
            } else {
                /* generic radix r: b_k = (sum_j a_j W_r^(jk)) * W_len^(pk) */
                const int wr_step = n / r; /* W_r^q = W_n^(q * n / r) */
                const double sg = sign < 0 ? 1.0 : -1.0;
                for (int k = 0; k < r; ++k) {
                    const int et = (p * k * tws) % n;
                    const double twr = P->wre[et], twi = sg * P->wim[et];
                    double* bkr = br + (size_t)(r * p + k) * blk;
                    double* bki = bi + (size_t)(r * p + k) * blk;
                    for (size_t t = 0; t < blk; ++t) { bkr[t] = 0.0; bki[t] = 0.0; }
                    for (int j = 0; j < r; ++j) {
                        const int e = (int)(((long long)j * k * wr_step) % n);
                        const double cr = P->wre[e], ci = sg * P->wim[e];
                        const double* ajr = ar + (size_t)(p + j * m) * blk;
                        const double* aji = ai + (size_t)(p + j * m) * blk;
                        for (size_t t = 0; t < blk; ++t) {
                            bkr[t] += ajr[t] * cr - aji[t] * ci;
                            bki[t] += ajr[t] * ci + aji[t] * cr;
                        }
                    }
                    for (size_t t = 0; t < blk; ++t) {
                        double ur = bkr[t], ui = bki[t];
                        bkr[t] = ur * twr - ui * twi;
                        bki[t] = ur * twi + ui * twr;
                    }
                }
            }
        }
        /* swap */
        double* tr = ar; ar = br; br = tr;
        double* ti = ai; ai = bi; bi = ti;
        len = m;
        s *= r;
    }
    if (ar != xr) {
        memcpy(xr, ar, sizeof(double) * (size_t)n * (size_t)L);
        memcpy(xi, ai, sizeof(double) * (size_t)n * (size_t)L);
    }
}

/* ------------------------------------------------------------------------- */
/* 1-D real transforms on a batch [n][L]                                      */
/* ------------------------------------------------------------------------- */
typedef struct {
    double *r0, *i0, *r1, *i1, *r2, *i2; /* each of size (n+2)*L */
} work_t;

static void work_alloc(work_t* w, int nmax, int L) {
    size_t sz = sizeof(double) * (size_t)(2 * nmax + 4) * (size_t)L;
    w->r0 = (double*)malloc(sz); w->i0 = (double*)malloc(sz);
    w->r1 = (double*)malloc(sz); w->i1 = (double*)malloc(sz);
    w->r2 = (double*)malloc(sz); w->i2 = (double*)malloc(sz);
}
static void work_free(work_t* w) {
    free(w->r0); free(w->i0); free(w->r1); free(w->i1); free(w->r2); free(w->i2);
}

/* r2c: x[n][L] real -> X[k][L], k = 0..n/2 (outr/outi sized (n/2+1)*L) */
static void r2c_batch(int n, const double* x, double* outr, double* outi, int L, work_t* w) {
    if (n % 2 == 0 && n >= 2) {
        const int h = n / 2;
        cplan* P = cplan_get(h);
        cplan* Pn = cplan_get(n);
        for (int j = 0; j < h; ++j)
            for (int l = 0; l < L; ++l) {
                w->r0[(size_t)j * L + l] = x[(size_t)(2 * j) * L + l];
                w->i0[(size_t)j * L + l] = x[(size_t)(2 * j + 1) * L + l];
            }
        cfft_batch(P, w->r0, w->i0, w->r1, w->i1, L, -1);
        for (int k = 0; k <= h; ++k) {
            const int k1 = k % h, k2 = (h - k) % h;
            const double wr = Pn->wre[k % n], wi = Pn->wim[k % n];
            for (int l = 0; l < L; ++l) {
                double zr = w->r0[(size_t)k1 * L + l], zi = w->i0[(size_t)k1 * L + l];
                double cr = w->r0[(size_t)k2 * L + l], ci = -w->i0[(size_t)k2 * L + l];
                double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
                /* O = (Z - conj Z')/(2i) */
                double dr = zr - cr, di = zi - ci;
                double orr = 0.5 * di, oi = -0.5 * dr;
                outr[(size_t)k * L + l] = er + (wr * orr - wi * oi);
                outi[(size_t)k * L + l] = ei + (wr * oi + wi * orr);
            }
        }
    } else {
        cplan* P = cplan_get(n);
        for (size_t t = 0; t < (size_t)n * L; ++t) { w->r0[t] = x[t]; w->i0[t] = 0.0; }
        cfft_batch(P, w->r0, w->i0, w->r1, w->i1, L, -1);
        for (int k = 0; k <= n / 2; ++k)
            for (int l = 0; l < L; ++l) {
                outr[(size_t)k * L + l] = w->r0[(size_t)k * L + l];
                outi[(size_t)k * L + l] = w->i0[(size_t)k * L + l];
            }
    }
}

/* c2r: X[k][L], k = 0..n/2 -> y[n][L] real, unnormalised.  Imag of X[0], X[n/2] ignored. */
static void c2r_batch(int n, const double* inr, const double* ini, double* y, int L, work_t* w) {
    if (n % 2 == 0 && n >= 2) {
        const int h = n / 2;
        cplan* P = cplan_get(h);
        cplan* Pn = cplan_get(n);
        for (int k = 0; k < h; ++k) {
            const int kc = h - k;
            /* W_n^{-k} */
            const double wr = Pn->wre[k], wi = -Pn->wim[k];
            for (int l = 0; l < L; ++l) {
                double xr = inr[(size_t)k * L + l], xi = (k == 0) ? 0.0 : ini[(size_t)k * L + l];
                double cr = inr[(size_t)kc * L + l], ci = (kc == h) ? 0.0 : -ini[(size_t)kc * L + l];
                double er = xr + cr, ei = xi + ci;
                double dr = xr - cr, di = xi - ci;
                double orr = dr * wr - di * wi, oi = dr * wi + di * wr;
                /* Z = E + i O */
                w->r0[(size_t)k * L + l] = er - oi;
                w->i0[(size_t)k * L + l] = ei + orr;
            }
        }
        cfft_batch(P, w->r0, w->i0, w->r1, w->i1, L, +1);
        for (int j = 0; j < h; ++j)
            for (int l = 0; l < L; ++l) {
                y[(size_t)(2 * j) * L + l] = w->r0[(size_t)j * L + l];
                y[(size_t)(2 * j + 1) * L + l] = w->i0[(size_t)j * L + l];
            }
    } else {
        cplan* P = cplan_get(n);
        for (int k = 0; k < n; ++k) {
            int kk = k <= n / 2 ? k : n - k;
            double sg = k <= n / 2 ? 1.0 : -1.0;
            for (int l = 0; l < L; ++l) {
                w->r0[(size_t)k * L + l] = inr[(size_t)kk * L + l];
                w->i0[(size_t)k * L + l] = (kk == 0 || 2 * kk == n) ? 0.0 : sg * ini[(size_t)kk * L + l];
            }
        }
        cfft_batch(P, w->r0, w->i0, w->r1, w->i1, L, +1);
        for (size_t t = 0; t < (size_t)n * L; ++t) y[t] = w->r0[t];
    }
}

/* half-sample twiddles exp(-i pi k / (2n)), k < n, cached per n */
typedef struct hplan {
    int n;
    double *c, *s;
    struct hplan* next;
} hplan;
static hplan* g_hplans = NULL;
static hplan* hplan_get(int n) {
    hplan* p;
    for (p = __atomic_load_n(&g_hplans, __ATOMIC_ACQUIRE); p; p = p->next)
        if (p->n == n) return p;
#ifdef _OPENMP
#pragma omp critical(crysscft_shim_plan)
#endif
    {
        for (p = g_hplans; p; p = p->next)
            if (p->n == n) break;
        if (!p) {
            p = (hplan*)calloc(1, sizeof(hplan));
            p->n = n;
            p->c = (double*)malloc(sizeof(double) * (size_t)(n + 1));
            p->s = (double*)malloc(sizeof(double) * (size_t)(n + 1));
            for (int k = 0; k <= n; ++k) {
                long double a = SHIM_PI * (long double)k / (2.0L * (long double)n);
                p->c[k] = (double)cosl(a);
                p->s[k] = (double)sinl(a);
            }
            p->next = g_hplans;
            __atomic_store_n(&g_hplans, p, __ATOMIC_RELEASE);
        }
    }
    return p;
}

/* direct O(n^2) real-to-real for odd lengths (long double accumulation) */
static void r2r_direct(int n, int kind, double* x, int L) {
    double* y = (double*)malloc(sizeof(double) * (size_t)n * L);
    for (int k = 0; k < n; ++k)
        for (int l = 0; l < L; ++l) {
            long double acc = 0.0L;
            if (kind == FFTW_REDFT10) {
                for (int j = 0; j < n; ++j)
                    acc += 2.0L * x[(size_t)j * L + l] *
                           cosl(SHIM_PI * ((long double)j + 0.5L) * (long double)k / (long double)n);
            } else {
                acc = x[l];
                for (int j = 1; j < n; ++j)
                    acc += 2.0L * x[(size_t)j * L + l] *
                           cosl(SHIM_PI * (long double)j * ((long double)k + 0.5L) / (long double)n);
            }
            y[(size_t)k * L + l] = (double)acc;
        }
    memcpy(x, y, sizeof(double) * (size_t)n * L);
    free(y);
}

/* REDFT10 in place on x[n][L] */
static void dct2_batch(int n, double* x, int L, work_t* w) {
    if (n % 2 != 0) { r2r_direct(n, FFTW_REDFT10, x, L); return; }
    const int h = n / 2;
    hplan* H = hplan_get(n);
    double* v = w->r2;
    for (int j = 0; j < h; ++j)
        for (int l = 0; l < L; ++l) {
            v[(size_t)j * L + l] = x[(size_t)(2 * j) * L + l];
            v[(size_t)(n - 1 - j) * L + l] = x[(size_t)(2 * j + 1) * L + l];
        }
    double* Vr = w->i2;                      /* (h+1)*L */
    double* Vi = w->i2 + (size_t)(h + 1) * L; /* (h+1)*L */
    r2c_batch(n, v, Vr, Vi, L, w);
    for (int k = 0; k < n; ++k) {
        const int kk = k <= h ? k : n - k;
        const double sg = k <= h ? 1.0 : -1.0;
        const double c = H->c[k], s = H->s[k];
        for (int l = 0; l < L; ++l) {
            double vr = Vr[(size_t)kk * L + l], vi = sg * Vi[(size_t)kk * L + l];
            /* 2 Re(exp(-i pi k/2n) V) = 2 (c vr + s vi) */
            x[(size_t)k * L + l] = 2.0 * (c * vr + s * vi);
        }
    }
}

/* REDFT01 in place on x[n][L] */
static void dct3_batch(int n, double* x, int L, work_t* w) {
    if (n % 2 != 0) { r2r_direct(n, FFTW_REDFT01, x, L); return; }
    const int h = n / 2;
    hplan* H = hplan_get(n);
    double* Vr = w->i2;
    double* Vi = w->i2 + (size_t)(h + 1) * L;
    for (int k = 0; k <= h; ++k) {
        const double c = H->c[k], s = H->s[k];
        for (int l = 0; l < L; ++l) {
            double a = x[(size_t)k * L + l];
            double b = (k == 0) ? 0.0 : x[(size_t)(n - k) * L + l];
            /* (a - i b)(c + i s) */
            Vr[(size_t)k * L + l] = a * c + b * s;
            Vi[(size_t)k * L + l] = a * s - b * c;
        }
    }
    double* v = w->r2;
    c2r_batch(n, Vr, Vi, v, L, w);
    for (int j = 0; j < h; ++j)
        for (int l = 0; l < L; ++l) {
            x[(size_t)(2 * j) * L + l] = v[(size_t)j * L + l];
            x[(size_t)(2 * j + 1) * L + l] = v[(size_t)(n - 1 - j) * L + l];
        }
}

/* ------------------------------------------------------------------------- */
/* plans                                                                      */
/* ------------------------------------------------------------------------- */
enum { SHIM_R2C = 1, SHIM_C2R = 2, SHIM_R2R = 3 };

struct fftw_plan_s {
    int type;
    int n[3];
    long is[3], os[3]; /* strides in elements of the input / output type */
    void* in;
    void* out;
    int kind[3];
};

static fftw_plan make_plan(int type, const int n[3], const long is[3], const long os[3],
                           void* in, void* out) {
    fftw_plan p = (fftw_plan)calloc(1, sizeof(struct fftw_plan_s));
    p->type = type;
    for (int d = 0; d < 3; ++d) { p->n[d] = n[d]; p->is[d] = is[d]; p->os[d] = os[d]; }
    p->in = in;
    p->out = out;
    return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in,
                                 const int* inembed, int istride, int idist,
                                 fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags) {
    (void)idist; (void)odist; (void)flags;
    if (rank != 3 || howmany != 1) return NULL;
    int nn[3] = {n[0], n[1], n[2]};
    const int* ie = inembed ? inembed : n;
    int oe_def[3] = {n[0], n[1], n[2] / 2 + 1};
    const int* oe = onembed ? onembed : oe_def;
    long is[3] = {(long)ie[1] * ie[2] * istride, (long)ie[2] * istride, istride};
    long os[3] = {(long)oe[1] * oe[2] * ostride, (long)oe[2] * ostride, ostride};
    return make_plan(SHIM_R2C, nn, is, os, in, out);
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in,
                                 const int* inembed, int istride, int idist,
                                 double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags) {
    (void)idist; (void)odist; (void)flags;
    if (rank != 3 || howmany != 1) return NULL;
    int nn[3] = {n[0], n[1], n[2]};
    int ie_def[3] = {n[0], n[1], n[2] / 2 + 1};
    const int* ie = inembed ? inembed : ie_def;
    const int* oe = onembed ? onembed : n;
    long is[3] = {(long)ie[1] * ie[2] * istride, (long)ie[2] * istride, istride};
    long os[3] = {(long)oe[1] * oe[2] * ostride, (long)oe[2] * ostride, ostride};
    return make_plan(SHIM_C2R, nn, is, os, in, out);
}

fftw_plan fftw_plan_guru_dft_r2c(int rank, const fftw_iodim* dims, int howmany_rank,
                                 const fftw_iodim* howmany_dims, double* in, fftw_complex* out,
                                 unsigned flags) {
    (void)howmany_dims; (void)flags;
    if (rank != 3 || howmany_rank != 0) return NULL;
    int nn[3];
    long is[3], os[3];
    for (int d = 0; d < 3; ++d) { nn[d] = dims[d].n; is[d] = dims[d].is; os[d] = dims[d].os; }
    return make_plan(SHIM_R2C, nn, is, os, in, out);
}

fftw_plan fftw_plan_guru_dft_c2r(int rank, const fftw_iodim* dims, int howmany_rank,
                                 const fftw_iodim* howmany_dims, fftw_complex* in, double* out,
                                 unsigned flags) {
    (void)howmany_dims; (void)flags;
    if (rank != 3 || howmany_rank != 0) return NULL;
    int nn[3];
    long is[3], os[3];
    for (int d = 0; d < 3; ++d) { nn[d] = dims[d].n; is[d] = dims[d].is; os[d] = dims[d].os; }
    return make_plan(SHIM_C2R, nn, is, os, in, out);
}

fftw_plan fftw_plan_r2r_3d(int n0, int n1, int n2, double* in, double* out,
                           fftw_r2r_kind kind0, fftw_r2r_kind kind1, fftw_r2r_kind kind2,
                           unsigned flags) {
    (void)flags;
    int nn[3] = {n0, n1, n2};
    long is[3] = {(long)n1 * n2, n2, 1};
    fftw_plan p = make_plan(SHIM_R2R, nn, is, is, in, out);
    p->kind[0] = kind0; p->kind[1] = kind1; p->kind[2] = kind2;
    return p;
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

/* ------------------------------------------------------------------------- */
/* axis drivers on contiguous work arrays                                     */
/* ------------------------------------------------------------------------- */

/*
 * Complex transform along one axis of a contiguous complex array T (interleaved)
 * viewed as [outer][n][inner].
 */
static void complex_axis(double* T, long outer, int n, long inner, int sign) {
    const long nb_inner = (inner + SHIM_BATCH - 1) / SHIM_BATCH;
    const long total = outer * nb_inner;
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        work_t w;
        work_alloc(&w, n, SHIM_BATCH);
        cplan* P = cplan_get(n);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (long b = 0; b < total; ++b) {
            const long o = b / nb_inner;
            const long c0 = (b % nb_inner) * SHIM_BATCH;
            const int L = (int)((inner - c0) < SHIM_BATCH ? (inner - c0) : SHIM_BATCH);
            for (int j = 0; j < n; ++j) {
                const double* src = T + 2 * ((o * n + j) * inner + c0);
                for (int l = 0; l < L; ++l) {
                    w.r2[(size_t)j * L + l] = src[2 * l];
                    w.i2[(size_t)j * L + l] = src[2 * l + 1];
                }
            }
            cfft_batch(P, w.r2, w.i2, w.r1, w.i1, L, sign);
            for (int j = 0; j < n; ++j) {
                double* dst = T + 2 * ((o * n + j) * inner + c0);
                for (int l = 0; l < L; ++l) {
                    dst[2 * l] = w.r2[(size_t)j * L + l];
                    dst[2 * l + 1] = w.i2[(size_t)j * L + l];
                }
            }
        }
        work_free(&w);
    }
}

/* real-to-real transform along one axis of a contiguous real array R [outer][n][inner] */
static void r2r_axis(double* R, long outer, int n, long inner, int kind) {
    const long nb_inner = (inner + SHIM_BATCH - 1) / SHIM_BATCH;
    const long total = outer * nb_inner;
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        work_t w;
        work_alloc(&w, n, SHIM_BATCH);
        double* buf = (double*)malloc(sizeof(double) * (size_t)n * SHIM_BATCH);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (long b = 0; b < total; ++b) {
            const long o = b / nb_inner;
            const long c0 = (b % nb_inner) * SHIM_BATCH;
            const int L = (int)((inner - c0) < SHIM_BATCH ? (inner - c0) : SHIM_BATCH);
            for (int j = 0; j < n; ++j) {
                const double* src = R + (o * n + j) * inner + c0;
                for (int l = 0; l < L; ++l) buf[(size_t)j * L + l] = src[l];
            }
            if (kind == FFTW_REDFT10) dct2_batch(n, buf, L, &w);
            else dct3_batch(n, buf, L, &w);
            for (int j = 0; j < n; ++j) {
                double* dst = R + (o * n + j) * inner + c0;
                for (int l = 0; l < L; ++l) dst[l] = buf[(size_t)j * L + l];
            }
        }
        free(buf);
        work_free(&w);
    }
}

static void exec_r2c(const fftw_plan p) {
    const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    const int h = n2 / 2 + 1;
    const double* in = (const double*)p->in;
    double* out = (double*)p->out; /* interleaved complex */
    double* T = (double*)malloc(sizeof(double) * 2 * (size_t)n0 * n1 * h);
    /* last axis: r2c of each (j0, j1) line; batch SHIM_BATCH lines */
    const long lines = (long)n0 * n1;
    const long nb = (lines + SHIM_BATCH - 1) / SHIM_BATCH;
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        work_t w;
        work_alloc(&w, n2, SHIM_BATCH);
        double* buf = (double*)malloc(sizeof(double) * (size_t)n2 * SHIM_BATCH);
        double* Xr = (double*)malloc(sizeof(double) * (size_t)h * SHIM_BATCH);
        double* Xi = (double*)malloc(sizeof(double) * (size_t)h * SHIM_BATCH);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (long b = 0; b < nb; ++b) {
            const long l0 = b * SHIM_BATCH;
            const int L = (int)((lines - l0) < SHIM_BATCH ? (lines - l0) : SHIM_BATCH);
            for (int l = 0; l < L; ++l) {
                const long line = l0 + l;
                const long j0 = line / n1, j1 = line % n1;
                const double* src = in + j0 * p->is[0] + j1 * p->is[1];
                for (int j = 0; j < n2; ++j) buf[(size_t)j * L + l] = src[j * p->is[2]];
            }
            r2c_batch(n2, buf, Xr, Xi, L, &w);
            for (int l = 0; l < L; ++l) {
                double* dst = T + 2 * (size_t)(l0 + l) * h;
                for (int k = 0; k < h; ++k) {
                    dst[2 * k] = Xr[(size_t)k * L + l];
                    dst[2 * k + 1] = Xi[(size_t)k * L + l];
                }
            }
        }
        free(buf); free(Xr); free(Xi);
        work_free(&w);
    }
    complex_axis(T, n0, n1, h, -1);
    complex_axis(T, 1, n0, (long)n1 * h, -1);
    for (long j0 = 0; j0 < n0; ++j0)
        for (long j1 = 0; j1 < n1; ++j1)
            for (long k = 0; k < h; ++k) {
                const double* s = T + 2 * ((j0 * n1 + j1) * h + k);
                double* d = out + 2 * (j0 * p->os[0] + j1 * p->os[1] + k * p->os[2]);
                d[0] = s[0];
                d[1] = s[1];
            }
    free(T);
}

static void exec_c2r(const fftw_plan p) {
    const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    const int h = n2 / 2 + 1;
    const double* in = (const double*)p->in;
    double* out = (double*)p->out;
    double* T = (double*)malloc(sizeof(double) * 2 * (size_t)n0 * n1 * h);
    for (long j0 = 0; j0 < n0; ++j0)
        for (long j1 = 0; j1 < n1; ++j1)
            for (long k = 0; k < h; ++k) {
                const double* s = in + 2 * (j0 * p->is[0] + j1 * p->is[1] + k * p->is[2]);
                double* d = T + 2 * ((j0 * n1 + j1) * h + k);
                d[0] = s[0];
                d[1] = s[1];
            }
    complex_axis(T, 1, n0, (long)n1 * h, +1);
    complex_axis(T, n0, n1, h, +1);
    const long lines = (long)n0 * n1;
    const long nb = (lines + SHIM_BATCH - 1) / SHIM_BATCH;
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        work_t w;
        work_alloc(&w, n2, SHIM_BATCH);
        double* buf = (double*)malloc(sizeof(double) * (size_t)n2 * SHIM_BATCH);
        double* Xr = (double*)malloc(sizeof(double) * (size_t)h * SHIM_BATCH);
        double* Xi = (double*)malloc(sizeof(double) * (size_t)h * SHIM_BATCH);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (long b = 0; b < nb; ++b) {
            const long l0 = b * SHIM_BATCH;
            const int L = (int)((lines - l0) < SHIM_BATCH ? (lines - l0) : SHIM_BATCH);
            for (int l = 0; l < L; ++l) {
                const double* src = T + 2 * (size_t)(l0 + l) * h;
                for (int k = 0; k < h; ++k) {
                    Xr[(size_t)k * L + l] = src[2 * k];
                    Xi[(size_t)k * L + l] = src[2 * k + 1];
                }
            }
            c2r_batch(n2, Xr, Xi, buf, L, &w);
            for (int l = 0; l < L; ++l) {
                const long line = l0 + l;
                const long j0 = line / n1, j1 = line % n1;
                double* dst = out + j0 * p->os[0] + j1 * p->os[1];
                for (int j = 0; j < n2; ++j) dst[j * p->os[2]] = buf[(size_t)j * L + l];
            }
        }
        free(buf); free(Xr); free(Xi);
        work_free(&w);
    }
    free(T);
}

static void exec_r2r(const fftw_plan p) {
    const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    const size_t tot = (size_t)n0 * n1 * n2;
    double* R = (double*)malloc(sizeof(double) * tot);
    const double* src = (const double*)p->in;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (long i = 0; i < (long)tot; ++i) R[i] = src[i];
    r2r_axis(R, (long)n0 * n1, n2, 1, p->kind[2]);
    r2r_axis(R, n0, n1, n2, p->kind[1]);
    r2r_axis(R, 1, n0, (long)n1 * n2, p->kind[0]);
    double* dst = (double*)p->out;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (long i = 0; i < (long)tot; ++i) dst[i] = R[i];
    free(R);
}

void fftw_execute(const fftw_plan p) {
    if (!p) return;
    if (p->type == SHIM_R2C) exec_r2c(p);
    else if (p->type == SHIM_C2R) exec_c2r(p);
    else exec_r2r(p);
}

/* direct O(n^2) complex DFT in long double, for the shim's own tests */
void crysscft_shim_dft_1d_direct(int n, const double* in_re, const double* in_im,
                                 double* out_re, double* out_im, int sign) {
    for (int k = 0; k < n; ++k) {
        long double ar = 0.0L, ai = 0.0L;
        for (int j = 0; j < n; ++j) {
            long double a = (long double)sign * 2.0L * SHIM_PI *
                            (long double)(((long long)j * k) % n) / (long double)n;
            long double c = cosl(a), s = sinl(a);
            ar += in_re[j] * c - in_im[j] * s;
            ai += in_re[j] * s + in_im[j] * c;
        }
        out_re[k] = (double)ar;
        out_im[k] = (double)ai;
    }
}

int crysscft_shim_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
