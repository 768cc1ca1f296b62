/*
 * Oracle (test infrastructure only).  A small FP64 mixed-radix FFT that
 * implements the FFTW3 entry points declared in fftw3.h (the subset bound by
 * the reference at janus/fft/serial/fftw.pxd:3-43), so that the reference's
 * own Cython modules can be built and run in this image, which has no
 * libfftw3.  It follows the semantics FFTW documents for these calls:
 *
 *  - r2c is the unnormalised forward DFT (exponent sign -1) of a real
 *    row-major array; the output keeps n_last/2+1 complex values per row;
 *  - c2r is the unnormalised inverse DFT of a Hermitian half spectrum (the
 *    imaginary parts of the DC and, for even n_last, Nyquist terms of the
 *    last axis are ignored) and may overwrite its input;
 *  - when `in` and `out` alias (the in-place case the reference always uses,
 *    janus/fft/serial/_serial_fft.pyx:38-52), each real row is padded to
 *    2*(n_last/2+1) doubles, otherwise the real array is contiguous.
 *
 * Algorithm: Stockham autosort passes (radix 4, 2, 3, 5 with hand-written
 * butterflies, any other prime factor by a direct O(p^2) butterfly), twiddles
 * from a table computed in long double.  Real rows are transformed two at a
 * time through one complex FFT (z = a + i b).  Multi-dimensional transforms
 * are done axis by axis (last axis first for r2c, last axis last for c2r).
 * Single-threaded, like the reference's serial path.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* 1D complex plan                                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
    int n;
    int nf;
    int fac[64];
    double *tw; /* interleaved exp(-2 pi i t / n), t = 0..n-1 */
} cplan;

static int next_factor(int n) {
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (int p = 3; (long)p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

static cplan *cplan_create(int n) {
    cplan *p = (cplan *)calloc(1, sizeof(cplan));
    p->n = n;
    int m = n;
    p->nf = 0;
    while (m > 1) {
        int f = next_factor(m);
        p->fac[p->nf++] = f;
        m /= f;
    }
    p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int t = 0; t < n; ++t) {
        long double a = two_pi * (long double)t / (long double)n;
        p->tw[2 * t] = (double)cosl(a);
        p->tw[2 * t + 1] = (double)-sinl(a);
    }
    return p;
}

static void cplan_destroy(cplan *p) {
    if (!p) return;
    free(p->tw);
    free(p);
}

/* One Stockham pass of radix R over `batch` interleaved sequences held
 * side by side (element e of sequence b at x[2*(e*batch + b)]).
 * sign = -1 forward, +1 inverse. */
static void stockham_pass(const cplan *p, int R, int Ns, int sign,
                          const double *x, double *y, int batch) {
    const int n = p->n;
    const int nr = n / R;
    const int tstep = n / (Ns * R);
    double vr[64], vi[64];
    double *gr = NULL, *gi = NULL;
    if (R > 64) {
        gr = (double *)malloc(sizeof(double) * R);
        gi = (double *)malloc(sizeof(double) * R);
    }
    double *ar = R > 64 ? gr : vr, *ai = R > 64 ? gi : vi;
    double *or_ = NULL, *oi = NULL;
    if (R > 5 || R == 3 || R == 5) {
        or_ = (double *)malloc(sizeof(double) * R);
        oi = (double *)malloc(sizeof(double) * R);
    }
    for (int j = 0; j < nr; ++j) {
        const int k = j % Ns;
        const int base = (j / Ns) * Ns * R + k;
        for (int b = 0; b < batch; ++b) {
            for (int r = 0; r < R; ++r) {
                const double *src = x + 2 * ((size_t)(j + r * nr) * batch + b);
                double re = src[0], im = src[1];
                if (r > 0 && k > 0) {
                    int t = (k * r * tstep) % n;
                    double wr = p->tw[2 * t], wi = -sign * p->tw[2 * t + 1];
                    double tr = re * wr - im * wi;
                    im = re * wi + im * wr;
                    re = tr;
                }
                ar[r] = re;
                ai[r] = im;
            }
            if (R == 2) {
                double r0 = ar[0] + ar[1], i0 = ai[0] + ai[1];
                double r1 = ar[0] - ar[1], i1 = ai[0] - ai[1];
                ar[0] = r0; ai[0] = i0; ar[1] = r1; ai[1] = i1;
            } else if (R == 4) {
                double s0r = ar[0] + ar[2], s0i = ai[0] + ai[2];
                double d0r = ar[0] - ar[2], d0i = ai[0] - ai[2];
                double s1r = ar[1] + ar[3], s1i = ai[1] + ai[3];
                double d1r = ar[1] - ar[3], d1i = ai[1] - ai[3];
                /* rotate d1 by sign*i: (a+ib)*(sign i) = -sign b + i sign a */
                double rr = -sign * d1i, ri = sign * d1r;
                ar[0] = s0r + s1r; ai[0] = s0i + s1i;
                ar[2] = s0r - s1r; ai[2] = s0i - s1i;
                ar[1] = d0r + rr; ai[1] = d0i + ri;
                ar[3] = d0r - rr; ai[3] = d0i - ri;
            } else if (R == 3) {
                const double s3 = 0.86602540378443864676372317075294;
                double t1r = ar[1] + ar[2], t1i = ai[1] + ai[2];
                double t2r = ar[0] - 0.5 * t1r, t2i = ai[0] - 0.5 * t1i;
                double dr = ar[1] - ar[2], di = ai[1] - ai[2];
                /* t3 = sign * i * s3 * d */
                double t3r = -sign * s3 * di, t3i = sign * s3 * dr;
                ar[0] = ar[0] + t1r; ai[0] = ai[0] + t1i;
                ar[1] = t2r + t3r; ai[1] = t2i + t3i;
                ar[2] = t2r - t3r; ai[2] = t2i - t3i;
            } else if (R == 5) {
                const double c1 = 0.30901699437494742410229341718282;
                const double c2 = -0.80901699437494742410229341718282;
                const double s1 = 0.95105651629515357211643933337938;
                const double s2 = 0.58778525229247312916870595463907;
                double a1r = ar[1] + ar[4], a1i = ai[1] + ai[4];
                double b1r = ar[1] - ar[4], b1i = ai[1] - ai[4];
                double a2r = ar[2] + ar[3], a2i = ai[2] + ai[3];
                double b2r = ar[2] - ar[3], b2i = ai[2] - ai[3];
                double t1r = ar[0] + c1 * a1r + c2 * a2r;
                double t1i = ai[0] + c1 * a1i + c2 * a2i;
                double t2r = ar[0] + c2 * a1r + c1 * a2r;
                double t2i = ai[0] + c2 * a1i + c1 * a2i;
                double u1r = s1 * b1r + s2 * b2r, u1i = s1 * b1i + s2 * b2i;
                double u2r = s2 * b1r - s1 * b2r, u2i = s2 * b1i - s1 * b2i;
                ar[0] = ar[0] + a1r + a2r; ai[0] = ai[0] + a1i + a2i;
                /* V1 = t1 + sign*i*u1, V4 = t1 - sign*i*u1, same for 2/3 */
                ar[1] = t1r - sign * u1i; ai[1] = t1i + sign * u1r;
                ar[4] = t1r + sign * u1i; ai[4] = t1i - sign * u1r;
                ar[2] = t2r - sign * u2i; ai[2] = t2i + sign * u2r;
                ar[3] = t2r + sign * u2i; ai[3] = t2i - sign * u2r;
            } else if (R > 1) {
                /* direct DFT of prime size R with the n-point table */
                const int step = n / R;
                for (int q = 0; q < R; ++q) {
                    double sr = 0.0, si = 0.0;
                    for (int r = 0; r < R; ++r) {
                        int t = (int)(((long)r * q) % R) * step;
                        double wr = p->tw[2 * t], wi = -sign * p->tw[2 * t + 1];
                        sr += ar[r] * wr - ai[r] * wi;
                        si += ar[r] * wi + ai[r] * wr;
                    }
                    or_[q] = sr;
                    oi[q] = si;
                }
                memcpy(ar, or_, sizeof(double) * R);
                memcpy(ai, oi, sizeof(double) * R);
            }
            for (int r = 0; r < R; ++r) {
                double *dst = y + 2 * ((size_t)(base + r * Ns) * batch + b);
                dst[0] = ar[r];
                dst[1] = ai[r];
            }
        }
    }
    free(gr);
    free(gi);
    free(or_);
    free(oi);
}

/* In-place batched complex FFT: `batch` sequences of length n stored
 * element-major (element e of sequence b at data[2*(e*batch+b)]).
 * `work` must hold 2*n*batch doubles. */
static void cfft_batch(const cplan *p, int sign, double *data, double *work,
                       int batch) {
    double *x = data, *y = work;
    int Ns = 1;
    for (int f = 0; f < p->nf; ++f) {
        int R = p->fac[f];
        stockham_pass(p, R, Ns, sign, x, y, batch);
        Ns *= R;
        double *t = x;
        x = y;
        y = t;
    }
    if (x != data)
        memcpy(data, x, sizeof(double) * 2 * (size_t)p->n * batch);
}

/* ------------------------------------------------------------------------ */
/* multi-dimensional real plans                                             */
/* ------------------------------------------------------------------------ */

#define COL_BLOCK 16

struct fftw_plan_s {
    int rank;      /* 2 or 3 */
    int n[3];      /* logical sizes */
    int r2c;       /* 1: r2c, 0: c2r */
    double *real;  /* real array */
    double *cplx;  /* complex array (interleaved) */
    int inplace;
    cplan *axis[3];
};

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    return p;
}

void fftw_free(void *p) { free(p); }

double *fftw_alloc_real(size_t n) {
    return (double *)fftw_malloc(sizeof(double) * n);
}

fftw_complex *fftw_alloc_complex(size_t n) {
    return (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
}

static fftw_plan make_plan(int rank, const int *n, double *real, double *cplx,
                           int r2c) {
    fftw_plan p = (fftw_plan)calloc(1, sizeof(struct fftw_plan_s));
    p->rank = rank;
    for (int d = 0; d < rank; ++d) {
        p->n[d] = n[d];
        p->axis[d] = cplan_create(n[d]);
    }
    p->r2c = r2c;
    p->real = real;
    p->cplx = cplx;
    p->inplace = ((void *)real == (void *)cplx);
    return p;
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out,
                               unsigned flags) {
    (void)flags;
    int n[2] = {n0, n1};
    return make_plan(2, n, in, (double *)out, 1);
}

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out,
                               unsigned flags) {
    (void)flags;
    int n[2] = {n0, n1};
    return make_plan(2, n, out, (double *)in, 0);
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags) {
    (void)flags;
    int n[3] = {n0, n1, n2};
    return make_plan(3, n, in, (double *)out, 1);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags) {
    (void)flags;
    int n[3] = {n0, n1, n2};
    return make_plan(3, n, out, (double *)in, 0);
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    for (int d = 0; d < p->rank; ++d) cplan_destroy(p->axis[d]);
    free(p);
}

/* complex FFT along axis `ax` (not the last one) of the complex array
 * with dims (n[0], ..., n[rank-2], m) */
static void complex_axis(fftw_plan p, int ax, int sign, double *buf,
                         double *work) {
    const int rank = p->rank;
    const int m = p->n[rank - 1] / 2 + 1;
    long outer = 1, inner = m;
    for (int d = 0; d < ax; ++d) outer *= p->n[d];
    for (int d = ax + 1; d < rank - 1; ++d) inner *= p->n[d];
    const int len = p->n[ax];
    const cplan *cp = p->axis[ax];
    for (long o = 0; o < outer; ++o) {
        double *slab = p->cplx + 2 * (size_t)o * len * inner;
        for (long i0 = 0; i0 < inner; i0 += COL_BLOCK) {
            int nb = (int)((inner - i0) < COL_BLOCK ? (inner - i0) : COL_BLOCK);
            for (int e = 0; e < len; ++e)
                memcpy(buf + 2 * (size_t)e * nb,
                       slab + 2 * ((size_t)e * inner + i0),
                       sizeof(double) * 2 * nb);
            cfft_batch(cp, sign, buf, work, nb);
            for (int e = 0; e < len; ++e)
                memcpy(slab + 2 * ((size_t)e * inner + i0),
                       buf + 2 * (size_t)e * nb, sizeof(double) * 2 * nb);
        }
    }
}

static void exec_r2c(fftw_plan p) {
    const int rank = p->rank;
    const int n = p->n[rank - 1];
    const int m = n / 2 + 1;
    const long rstride = p->inplace ? 2L * m : n;
    long rows = 1;
    for (int d = 0; d < rank - 1; ++d) rows *= p->n[d];
    int maxlen = n;
    for (int d = 0; d < rank; ++d)
        if (p->n[d] > maxlen) maxlen = p->n[d];
    double *z = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (long r = 0; r < rows; r += 2) {
        const int pair = (r + 1 < rows);
        const double *a = p->real + r * rstride;
        const double *b = pair ? p->real + (r + 1) * rstride : NULL;
        for (int e = 0; e < n; ++e) {
            z[2 * e] = a[e];
            z[2 * e + 1] = pair ? b[e] : 0.0;
        }
        cfft_batch(p->axis[rank - 1], -1, z, w, 1);
        double *ca = p->cplx + 2 * r * m;
        double *cb = pair ? p->cplx + 2 * (r + 1) * m : NULL;
        for (int k = 0; k < m; ++k) {
            int kk = (n - k) % n;
            double pr = z[2 * k], pi = z[2 * k + 1];
            double qr = z[2 * kk], qi = -z[2 * kk + 1];
            ca[2 * k] = 0.5 * (pr + qr);
            ca[2 * k + 1] = 0.5 * (pi + qi);
            if (pair) {
                /* B = (P - Q) / (2i) */
                cb[2 * k] = 0.5 * (pi - qi);
                cb[2 * k + 1] = -0.5 * (pr - qr);
            }
        }
    }
    free(z);
    free(w);
    double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)maxlen * COL_BLOCK);
    double *work = (double *)malloc(sizeof(double) * 2 * (size_t)maxlen * COL_BLOCK);
    for (int ax = rank - 2; ax >= 0; --ax) complex_axis(p, ax, -1, buf, work);
    free(buf);
    free(work);
}

static void exec_c2r(fftw_plan p) {
    const int rank = p->rank;
    const int n = p->n[rank - 1];
    const int m = n / 2 + 1;
    const long rstride = p->inplace ? 2L * m : n;
    long rows = 1;
    for (int d = 0; d < rank - 1; ++d) rows *= p->n[d];
    int maxlen = n;
    for (int d = 0; d < rank; ++d)
        if (p->n[d] > maxlen) maxlen = p->n[d];
    double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)maxlen * COL_BLOCK);
    double *work = (double *)malloc(sizeof(double) * 2 * (size_t)maxlen * COL_BLOCK);
    for (int ax = 0; ax <= rank - 2; ++ax) complex_axis(p, ax, +1, buf, work);
    free(buf);
    free(work);
    double *z = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (long r = 0; r < rows; r += 2) {
        const int pair = (r + 1 < rows);
        const double *ca = p->cplx + 2 * r * m;
        const double *cb = pair ? p->cplx + 2 * (r + 1) * m : NULL;
        for (int k = 0; k < m; ++k) {
            double ar = ca[2 * k], ai = ca[2 * k + 1];
            double br = pair ? cb[2 * k] : 0.0, bi = pair ? cb[2 * k + 1] : 0.0;
            if (k == 0 || 2 * k == n) {
                ai = 0.0;
                bi = 0.0;
            }
            /* Z_k = A_k + i B_k */
            z[2 * k] = ar - bi;
            z[2 * k + 1] = ai + br;
            if (k > 0 && 2 * k != n) {
                /* Z_{n-k} = conj(A_k) + i conj(B_k) */
                int kk = n - k;
                z[2 * kk] = ar + bi;
                z[2 * kk + 1] = -ai + br;
            }
        }
        cfft_batch(p->axis[rank - 1], +1, z, w, 1);
        double *a = p->real + r * rstride;
        double *b = pair ? p->real + (r + 1) * rstride : NULL;
        for (int e = 0; e < n; ++e) {
            a[e] = z[2 * e];
            if (pair) b[e] = z[2 * e + 1];
        }
    }
    free(z);
    free(w);
}

void fftw_execute(const fftw_plan p) {
    if (!p) return;
    if (p->r2c)
        exec_r2c(p);
    else
        exec_c2r(p);
}
