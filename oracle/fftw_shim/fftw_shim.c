/*
 * FP64 FFTW3-API shim -- TEST INFRASTRUCTURE ONLY (part of the oracle).
 *
 * Implements the subset of FFTW3 the reference CPU path calls (see fftw3.h for
 * the list, the call sites and the semantics kept).  The algorithm is the
 * textbook mixed-radix Stockham auto-sort DFT:
 *
 *   for each radix r of n = r_1 r_2 ... r_s, with Ns = r_1 ... r_{t-1}:
 *     for j in [0, n/r):
 *       a_k = src[j + k n/r] * exp(sign 2 pi i (j mod Ns) k / (Ns r)),  k < r
 *       b   = DFT_r(a)
 *       dst[(j / Ns) Ns r + (j mod Ns) + q Ns] = b_q,                    q < r
 *
 * which leaves the result in natural order.  Twiddles are tabulated once per
 * plan as exp(sign 2 pi i m / n), m < n, from the FP64 libm cos/sin of the exact
 * angle, so every transform agrees with numpy's pocketfft to ~1e-15 relative.
 * Multi-dimensional transforms are successive 1D passes over gathered lines,
 * split across POSIX threads (fftw_plan_with_nthreads), which mirrors FFTW's
 * threaded planner for the purpose of CPU timing.
 */
#include "fftw3.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define SHIM_MAX_FACTORS 40

typedef struct {
    int n;
    int sign;
    int nf;
    int radix[SHIM_MAX_FACTORS];
    double *tw; /* 2n doubles: exp(sign * 2 pi i m / n) */
} line_plan;

enum { KIND_C2C = 0, KIND_R2C = 1, KIND_C2R = 2 };

struct gpe_shim_plan_s {
    int kind;
    int n[3];
    int sign;
    int nthreads;
    void *in;
    void *out;
    line_plan lp[3];      /* per-axis line plans (axis 2 full length n2) */
    double *scratch;      /* c2r: copy of the half spectrum */
};

static int g_nthreads = 1;

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }
void fftw_cleanup_threads(void) {}

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 64) != 0)
        return NULL;
    return p;
}
void fftw_free(void *p) { free(p); }

/* ----------------------------------------------------------------------------
 * 1D line plan
 * ------------------------------------------------------------------------- */
static void line_plan_init(line_plan *lp, int n, int sign) {
    lp->n    = n;
    lp->sign = sign;
    lp->nf   = 0;
    int m    = n;
    while (m % 4 == 0 && lp->nf < SHIM_MAX_FACTORS) {
        lp->radix[lp->nf++] = 4;
        m /= 4;
    }
    int p = 2;
    while (m > 1 && lp->nf < SHIM_MAX_FACTORS) {
        while (m % p == 0) {
            lp->radix[lp->nf++] = p;
            m /= p;
        }
        p = (p == 2) ? 3 : p + 2;
    }
    lp->tw = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < n; ++k) {
        double ang          = 2.0 * M_PI * (double)k / (double)n;
        lp->tw[2 * k]     = cos(ang);
        lp->tw[2 * k + 1] = (double)sign * sin(ang);
    }
}

static void line_plan_free(line_plan *lp) {
    free(lp->tw);
    lp->tw = NULL;
}

/* One Stockham stage of radix r from src to dst (complex interleaved). */
static void stage(const line_plan *lp, int r, int Ns, const double *src, double *dst) {
    const int n     = lp->n;
    const int nr    = n / r;
    const double *w = lp->tw;
    const int step  = n / (Ns * r); /* twiddle index step: jm*k*step */
    double ar[r], ai[r]; /* C99 VLAs: r is any prime factor of n */
    double br[r], bi[r];
    const double s = (double)lp->sign;
    for (int j = 0; j < nr; ++j) {
        const int jm = j % Ns;
        for (int k = 0; k < r; ++k) {
            double xr      = src[2 * (j + k * nr)];
            double xi      = src[2 * (j + k * nr) + 1];
            long t         = ((long)jm * k * step) % n;
            double wr      = w[2 * t];
            double wi      = w[2 * t + 1];
            ar[k]          = xr * wr - xi * wi;
            ai[k]          = xr * wi + xi * wr;
        }
        switch (r) {
        case 2:
            br[0] = ar[0] + ar[1];
            bi[0] = ai[0] + ai[1];
            br[1] = ar[0] - ar[1];
            bi[1] = ai[0] - ai[1];
            break;
        case 4: {
            double t0r = ar[0] + ar[2], t0i = ai[0] + ai[2];
            double t1r = ar[0] - ar[2], t1i = ai[0] - ai[2];
            double t2r = ar[1] + ar[3], t2i = ai[1] + ai[3];
            double t3r = ar[1] - ar[3], t3i = ai[1] - ai[3];
            /* multiply t3 by sign*i */
            double ur = -s * t3i, ui = s * t3r;
            br[0]     = t0r + t2r;
            bi[0]     = t0i + t2i;
            br[2]     = t0r - t2r;
            bi[2]     = t0i - t2i;
            br[1]     = t1r + ur;
            bi[1]     = t1i + ui;
            br[3]     = t1r - ur;
            bi[3]     = t1i - ui;
            break;
        }
        default: {
            /* generic r-point DFT using the plan's table: exp(sign 2 pi i kq/r) =
             * tw[(k q n/r) mod n] */
            for (int q = 0; q < r; ++q) {
                double sr = 0.0, si = 0.0;
                for (int k = 0; k < r; ++k) {
                    long t    = ((long)k * q % r) * nr;
                    double wr = w[2 * t], wi = w[2 * t + 1];
                    sr += ar[k] * wr - ai[k] * wi;
                    si += ar[k] * wi + ai[k] * wr;
                }
                br[q] = sr;
                bi[q] = si;
            }
            break;
        }
        }
        const int idxD = (j / Ns) * Ns * r + jm;
        for (int q = 0; q < r; ++q) {
            dst[2 * (idxD + q * Ns)]     = br[q];
            dst[2 * (idxD + q * Ns) + 1] = bi[q];
        }
    }
}

/* Transform x (2n doubles) in place; work is 2n doubles of scratch. */
static void line_fft(const line_plan *lp, double *x, double *work) {
    double *src = x, *dst = work;
    int Ns      = 1;
    for (int f = 0; f < lp->nf; ++f) {
        int r = lp->radix[f];
        stage(lp, r, Ns, src, dst);
        double *t = src;
        src       = dst;
        dst       = t;
        Ns *= r;
    }
    if (src != x)
        memcpy(x, src, sizeof(double) * 2 * (size_t)lp->n);
}

void gpe_shim_fft1d(int n, const double *in, double *out, int sign) {
    line_plan lp;
    line_plan_init(&lp, n, sign);
    double *work = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    memcpy(out, in, sizeof(double) * 2 * (size_t)n);
    line_fft(&lp, out, work);
    free(work);
    line_plan_free(&lp);
}

/* ----------------------------------------------------------------------------
 * Threaded axis passes over a complex 3D array of dims d0 x d1 x d2.
 * ------------------------------------------------------------------------- */
typedef struct {
    const line_plan *lp;
    double *data; /* complex interleaved, dims d[3] */
    int d[3];
    int axis;
    long first, last; /* line range */
} axis_job;

static void *axis_worker(void *arg) {
    axis_job *jb   = (axis_job *)arg;
    const int len  = jb->d[jb->axis];
    double *buf    = (double *)malloc(sizeof(double) * 2 * (size_t)len);
    double *work   = (double *)malloc(sizeof(double) * 2 * (size_t)len);
    const long d1  = jb->d[1], d2 = jb->d[2];
    for (long l = jb->first; l < jb->last; ++l) {
        long base, stride;
        if (jb->axis == 2) {
            base   = l * d2;
            stride = 1;
        } else if (jb->axis == 1) {
            long i = l / d2, k = l % d2;
            base   = i * d1 * d2 + k;
            stride = d2;
        } else {
            base   = l; /* l = j*d2 + k */
            stride = d1 * d2;
        }
        for (int t = 0; t < len; ++t) {
            buf[2 * t]     = jb->data[2 * (base + t * stride)];
            buf[2 * t + 1] = jb->data[2 * (base + t * stride) + 1];
        }
        line_fft(jb->lp, buf, work);
        for (int t = 0; t < len; ++t) {
            jb->data[2 * (base + t * stride)]     = buf[2 * t];
            jb->data[2 * (base + t * stride) + 1] = buf[2 * t + 1];
        }
    }
    free(buf);
    free(work);
    return NULL;
}

static void axis_pass(const line_plan *lp, double *data, const int d[3], int axis, int nthreads) {
    long nlines = (long)d[0] * d[1] * d[2] / d[axis];
    if (nthreads < 1)
        nthreads = 1;
    if (nthreads > nlines)
        nthreads = (int)(nlines > 0 ? nlines : 1);
    axis_job jobs[256];
    pthread_t th[256];
    if (nthreads > 256)
        nthreads = 256;
    for (int t = 0; t < nthreads; ++t) {
        jobs[t].lp    = lp;
        jobs[t].data  = data;
        jobs[t].d[0]  = d[0];
        jobs[t].d[1]  = d[1];
        jobs[t].d[2]  = d[2];
        jobs[t].axis  = axis;
        jobs[t].first = nlines * t / nthreads;
        jobs[t].last  = nlines * (t + 1) / nthreads;
    }
    if (nthreads == 1) {
        axis_worker(&jobs[0]);
        return;
    }
    for (int t = 1; t < nthreads; ++t)
        pthread_create(&th[t], NULL, axis_worker, &jobs[t]);
    axis_worker(&jobs[0]);
    for (int t = 1; t < nthreads; ++t)
        pthread_join(th[t], NULL);
}

/* ----------------------------------------------------------------------------
 * Real-axis passes (last axis) for r2c / c2r, threaded over lines.
 * ------------------------------------------------------------------------- */
typedef struct {
    const line_plan *lp;
    const double *rin;  /* r2c: real input n0*n1*n2 */
    double *cout;       /* r2c: half-spectrum output */
    const double *cin;  /* c2r: half-spectrum input (already transformed on axes 0,1) */
    double *rout;       /* c2r: real output */
    int n2;
    long first, last;
} real_job;

static void *r2c_worker(void *arg) {
    real_job *jb = (real_job *)arg;
    const int n2 = jb->n2, h = n2 / 2 + 1;
    double *buf  = (double *)malloc(sizeof(double) * 2 * (size_t)n2);
    double *work = (double *)malloc(sizeof(double) * 2 * (size_t)n2);
    for (long l = jb->first; l < jb->last; ++l) {
        for (int t = 0; t < n2; ++t) {
            buf[2 * t]     = jb->rin[l * n2 + t];
            buf[2 * t + 1] = 0.0;
        }
        line_fft(jb->lp, buf, work);
        memcpy(jb->cout + 2 * l * h, buf, sizeof(double) * 2 * (size_t)h);
    }
    free(buf);
    free(work);
    return NULL;
}

static void *c2r_worker(void *arg) {
    real_job *jb = (real_job *)arg;
    const int n2 = jb->n2, h = n2 / 2 + 1;
    double *buf  = (double *)malloc(sizeof(double) * 2 * (size_t)n2);
    double *work = (double *)malloc(sizeof(double) * 2 * (size_t)n2);
    for (long l = jb->first; l < jb->last; ++l) {
        const double *src = jb->cin + 2 * l * h;
        for (int k = 0; k < h; ++k) {
            buf[2 * k]     = src[2 * k];
            buf[2 * k + 1] = src[2 * k + 1];
        }
        for (int k = h; k < n2; ++k) {
            buf[2 * k]     = src[2 * (n2 - k)];
            buf[2 * k + 1] = -src[2 * (n2 - k) + 1];
        }
        line_fft(jb->lp, buf, work);
        for (int t = 0; t < n2; ++t)
            jb->rout[l * n2 + t] = buf[2 * t];
    }
    free(buf);
    free(work);
    return NULL;
}

static void real_pass(void *(*fn)(void *), real_job proto, long nlines, int nthreads) {
    if (nthreads < 1)
        nthreads = 1;
    if (nthreads > nlines)
        nthreads = (int)(nlines > 0 ? nlines : 1);
    if (nthreads > 256)
        nthreads = 256;
    real_job jobs[256];
    pthread_t th[256];
    for (int t = 0; t < nthreads; ++t) {
        jobs[t]       = proto;
        jobs[t].first = nlines * t / nthreads;
        jobs[t].last  = nlines * (t + 1) / nthreads;
    }
    if (nthreads == 1) {
        fn(&jobs[0]);
        return;
    }
    for (int t = 1; t < nthreads; ++t)
        pthread_create(&th[t], NULL, fn, &jobs[t]);
    fn(&jobs[0]);
    for (int t = 1; t < nthreads; ++t)
        pthread_join(th[t], NULL);
}

/* ----------------------------------------------------------------------------
 * Planner / executor
 * ------------------------------------------------------------------------- */
static fftw_plan plan_alloc(int kind, int n0, int n1, int n2, int sign, void *in, void *out) {
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->kind     = kind;
    p->n[0]     = n0;
    p->n[1]     = n1;
    p->n[2]     = n2;
    p->sign     = sign;
    p->nthreads = g_nthreads;
    p->in       = in;
    p->out      = out;
    line_plan_init(&p->lp[0], n0, sign);
    line_plan_init(&p->lp[1], n1, sign);
    line_plan_init(&p->lp[2], n2, sign);
    return p;
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags) {
    (void)flags;
    return plan_alloc(KIND_C2C, n0, n1, n2, sign, in, out);
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out,
                               unsigned flags) {
    (void)flags;
    return plan_alloc(KIND_R2C, n0, n1, n2, FFTW_FORWARD, in, out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out,
                               unsigned flags) {
    (void)flags;
    fftw_plan p  = plan_alloc(KIND_C2R, n0, n1, n2, FFTW_BACKWARD, in, out);
    p->scratch   = (double *)fftw_malloc(sizeof(double) * 2 * (size_t)n0 * n1 * (n2 / 2 + 1));
    return p;
}

void fftw_execute(const fftw_plan p) {
    const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    if (p->kind == KIND_C2C) {
        size_t bytes = sizeof(double) * 2 * (size_t)n0 * n1 * n2;
        if (p->out != p->in)
            memcpy(p->out, p->in, bytes);
        int d[3] = {n0, n1, n2};
        axis_pass(&p->lp[2], (double *)p->out, d, 2, p->nthreads);
        axis_pass(&p->lp[1], (double *)p->out, d, 1, p->nthreads);
        axis_pass(&p->lp[0], (double *)p->out, d, 0, p->nthreads);
    } else if (p->kind == KIND_R2C) {
        const int h   = n2 / 2 + 1;
        real_job jb;
        memset(&jb, 0, sizeof(jb));
        jb.lp   = &p->lp[2];
        jb.rin  = (const double *)p->in;
        jb.cout = (double *)p->out;
        jb.n2   = n2;
        real_pass(r2c_worker, jb, (long)n0 * n1, p->nthreads);
        int d[3] = {n0, n1, h};
        axis_pass(&p->lp[1], (double *)p->out, d, 1, p->nthreads);
        axis_pass(&p->lp[0], (double *)p->out, d, 0, p->nthreads);
    } else {
        const int h  = n2 / 2 + 1;
        size_t bytes = sizeof(double) * 2 * (size_t)n0 * n1 * h;
        memcpy(p->scratch, p->in, bytes);
        int d[3] = {n0, n1, h};
        axis_pass(&p->lp[0], p->scratch, d, 0, p->nthreads);
        axis_pass(&p->lp[1], p->scratch, d, 1, p->nthreads);
        real_job jb;
        memset(&jb, 0, sizeof(jb));
        jb.lp   = &p->lp[2];
        jb.cin  = p->scratch;
        jb.rout = (double *)p->out;
        jb.n2   = n2;
        real_pass(c2r_worker, jb, (long)n0 * n1, p->nthreads);
    }
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p)
        return;
    line_plan_free(&p->lp[0]);
    line_plan_free(&p->lp[1]);
    line_plan_free(&p->lp[2]);
    fftw_free(p->scratch);
    free(p);
}
