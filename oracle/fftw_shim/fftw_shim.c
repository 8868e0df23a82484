/*
 * FP64 3D complex DFT behind the FFTW-API subset declared in fftw3.h.
 * TEST INFRASTRUCTURE ONLY (CPU oracle and CPU baseline); never linked into
 * the GPU library.
 *
 * Algorithm (written from the mathematics, not from FFTW):
 *   - the 3D transform is three passes of 1D transforms, one per axis;
 *   - each pass gathers PS_LANES pencils into a lane-interleaved scratch block
 *     [n][PS_LANES] so every butterfly is a short vectorisable loop over lanes;
 *   - power-of-two lengths: iterative radix-2 decimation in time, input
 *     bit-reversed on gather, twiddles exp(-2 pi i k/n) tabulated in long double;
 *   - other lengths: Bluestein's chirp-z identity jk = (j^2 + k^2 - (k-j)^2)/2,
 *     i.e. a cyclic convolution of length m = 2^ceil(log2(2n-1)) done with the
 *     power-of-two transform; chirp angles use j^2 mod 2n so they stay exact.
 *   - pencil blocks are spread over OpenMP threads; the arithmetic on each
 *     pencil does not depend on the thread count, so results are bitwise
 *     reproducible for any thread count.
 */
#include "fftw3.h"

#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define PS_LANES 8

typedef struct {
    double re, im;
} cpx;

typedef struct eng1d {
    int n;
    int pow2;
    /* power of two */
    int *bitrev;  /* n entries */
    cpx *tw;      /* n/2 entries: exp(-2 pi i k / n) */
    /* Bluestein */
    int m;
    struct eng1d *sub; /* power-of-two engine of length m */
    cpx *chirp;        /* n entries: exp(-i pi (j^2 mod 2n) / n) (forward sign) */
    cpx *bhat_fwd;     /* m entries: DFT_m of conj(chirp) kernel, forward problem */
    cpx *bhat_bwd;     /* m entries: same for the backward problem */
} eng1d;

struct ps_shim_plan {
    int n[3];
    fftw_complex *in, *out;
    int sign;
    eng1d *e[3];
};

static int g_threads = 0;

void ps_shim_set_threads(int nthreads) { g_threads = nthreads > 0 ? nthreads : 0; }

int ps_shim_get_threads(void)
{
    if (g_threads > 0) return g_threads;
    const char *s = getenv("PS_SHIM_THREADS");
    if (s && atoi(s) > 0) return atoi(s);
    long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (int)c : 1;
}

static void *xalloc(size_t bytes)
{
    void *p = NULL;
    if (bytes == 0) bytes = 64;
    if (posix_memalign(&p, 64, bytes) != 0 || p == NULL) {
        fprintf(stderr, "fftw shim: out of memory (%zu bytes)\n", bytes);
        exit(EXIT_FAILURE);
    }
    return p;
}

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void eng_free(eng1d *e)
{
    if (!e) return;
    free(e->bitrev);
    free(e->tw);
    free(e->chirp);
    free(e->bhat_fwd);
    free(e->bhat_bwd);
    eng_free(e->sub);
    free(e);
}

static void fft_pow2_lanes(const eng1d *e, cpx *a, int sign);

static eng1d *eng_new(int n)
{
    eng1d *e = (eng1d *)calloc(1, sizeof(eng1d));
    e->n = n;
    e->pow2 = is_pow2(n);
    if (e->pow2) {
        int lg = 0;
        while ((1 << lg) < n) lg++;
        e->bitrev = (int *)xalloc(sizeof(int) * (size_t)n);
        for (int i = 0; i < n; i++) {
            int r = 0;
            for (int b = 0; b < lg; b++)
                if (i & (1 << b)) r |= 1 << (lg - 1 - b);
            e->bitrev[i] = r;
        }
        int h = n / 2 > 0 ? n / 2 : 1;
        e->tw = (cpx *)xalloc(sizeof(cpx) * (size_t)h);
        const long double two_pi = 6.283185307179586476925286766559005768L;
        for (int k = 0; k < h; k++) {
            long double ang = two_pi * (long double)k / (long double)n;
            e->tw[k].re = (double)cosl(ang);
            e->tw[k].im = (double)(-sinl(ang));
        }
        return e;
    }
    /* Bluestein */
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    e->m = m;
    e->sub = eng_new(m);
    e->chirp = (cpx *)xalloc(sizeof(cpx) * (size_t)n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int j = 0; j < n; j++) {
        long long q = ((long long)j * j) % (2LL * n);
        long double ang = pi * (long double)q / (long double)n;
        e->chirp[j].re = (double)cosl(ang);
        e->chirp[j].im = (double)(-sinl(ang));
    }
    /* kernel b_t = conj(c_t) for the problem with chirp c (forward: c = chirp,
     * backward: c = conj(chirp)); stored lane-broadcast-free as plain arrays. */
    for (int pass = 0; pass < 2; pass++) {
        cpx *bh = (cpx *)xalloc(sizeof(cpx) * (size_t)m * PS_LANES);
        memset(bh, 0, sizeof(cpx) * (size_t)m * PS_LANES);
        for (int t = 0; t < n; t++) {
            cpx c = e->chirp[t];
            if (pass == 1) c.im = -c.im;
            cpx b = {c.re, -c.im};
            for (int l = 0; l < PS_LANES; l++) {
                bh[(size_t)e->sub->bitrev[t] * PS_LANES + l] = b;
                if (t > 0) bh[(size_t)e->sub->bitrev[m - t] * PS_LANES + l] = b;
            }
        }
        fft_pow2_lanes(e->sub, bh, -1);
        cpx *flat = (cpx *)xalloc(sizeof(cpx) * (size_t)m);
        for (int k = 0; k < m; k++) flat[k] = bh[(size_t)k * PS_LANES];
        free(bh);
        if (pass == 0) e->bhat_fwd = flat;
        else e->bhat_bwd = flat;
    }
    return e;
}

/* In-place radix-2 DIT on PS_LANES interleaved pencils whose elements are
 * already in bit-reversed order: a[k*PS_LANES + lane]. */
static void fft_pow2_lanes(const eng1d *e, cpx *a, int sign)
{
    const int n = e->n;
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1;
        const int step = n / len;
        for (int base = 0; base < n; base += len) {
            for (int k = 0; k < half; k++) {
                const double wr = e->tw[k * step].re;
                const double wi = sign < 0 ? e->tw[k * step].im : -e->tw[k * step].im;
                cpx *u = a + (size_t)(base + k) * PS_LANES;
                cpx *v = a + (size_t)(base + k + half) * PS_LANES;
                for (int l = 0; l < PS_LANES; l++) {
                    const double vr = v[l].re * wr - v[l].im * wi;
                    const double vi = v[l].re * wi + v[l].im * wr;
                    const double ur = u[l].re, ui = u[l].im;
                    u[l].re = ur + vr;
                    u[l].im = ui + vi;
                    v[l].re = ur - vr;
                    v[l].im = ui - vi;
                }
            }
        }
    }
}

/* Transform PS_LANES interleaved pencils in natural order in `blk` (n rows),
 * using `work` (m*PS_LANES for Bluestein, n*PS_LANES otherwise) as scratch. */
static void fft_lanes(const eng1d *e, cpx *blk, cpx *work, int sign)
{
    const int n = e->n;
    if (e->pow2) {
        for (int k = 0; k < n; k++)
            memcpy(work + (size_t)e->bitrev[k] * PS_LANES, blk + (size_t)k * PS_LANES,
                   sizeof(cpx) * PS_LANES);
        fft_pow2_lanes(e, work, sign);
        memcpy(blk, work, sizeof(cpx) * (size_t)n * PS_LANES);
        return;
    }
    const int m = e->m;
    const eng1d *s = e->sub;
    memset(work, 0, sizeof(cpx) * (size_t)m * PS_LANES);
    for (int j = 0; j < n; j++) {
        cpx c = e->chirp[j];
        if (sign > 0) c.im = -c.im;
        cpx *dst = work + (size_t)s->bitrev[j] * PS_LANES;
        const cpx *src = blk + (size_t)j * PS_LANES;
        for (int l = 0; l < PS_LANES; l++) {
            dst[l].re = src[l].re * c.re - src[l].im * c.im;
            dst[l].im = src[l].re * c.im + src[l].im * c.re;
        }
    }
    fft_pow2_lanes(s, work, -1);
    const cpx *bh = sign < 0 ? e->bhat_fwd : e->bhat_bwd;
    /* pointwise product, then inverse DFT_m via bit-reversed gather */
    cpx *tmp = work + (size_t)m * PS_LANES; /* second half of the scratch */
    for (int k = 0; k < m; k++) {
        const cpx b = bh[k];
        const cpx *src = work + (size_t)k * PS_LANES;
        cpx *dst = tmp + (size_t)s->bitrev[k] * PS_LANES;
        for (int l = 0; l < PS_LANES; l++) {
            dst[l].re = src[l].re * b.re - src[l].im * b.im;
            dst[l].im = src[l].re * b.im + src[l].im * b.re;
        }
    }
    fft_pow2_lanes(s, tmp, +1);
    const double inv_m = 1.0 / (double)m;
    for (int k = 0; k < n; k++) {
        cpx c = e->chirp[k];
        if (sign > 0) c.im = -c.im;
        const cpx *src = tmp + (size_t)k * PS_LANES;
        cpx *dst = blk + (size_t)k * PS_LANES;
        for (int l = 0; l < PS_LANES; l++) {
            const double r = src[l].re * inv_m, i = src[l].im * inv_m;
            dst[l].re = r * c.re - i * c.im;
            dst[l].im = r * c.im + i * c.re;
        }
    }
}

/* 1D transforms along one axis of a row-major (n0,n1,n2) array.
 * The array is viewed as [outer][n][inner]; pencils are (outer, inner). */
static void axis_pass(cpx *data, long outer, int n, long inner, const eng1d *e, int sign)
{
    const long nblk_inner = (inner + PS_LANES - 1) / PS_LANES;
    const long nblocks = outer * nblk_inner;
    const size_t work_elems = (size_t)(e->pow2 ? n : 2 * e->m) * PS_LANES;
#pragma omp parallel num_threads(ps_shim_get_threads())
    {
        cpx *blk = (cpx *)xalloc(sizeof(cpx) * (size_t)n * PS_LANES);
        cpx *work = (cpx *)xalloc(sizeof(cpx) * work_elems);
#pragma omp for schedule(static)
        for (long b = 0; b < nblocks; b++) {
            const long o = b / nblk_inner;
            const long i0 = (b % nblk_inner) * PS_LANES;
            const int lanes = (int)((inner - i0) < PS_LANES ? (inner - i0) : PS_LANES);
            cpx *base = data + (size_t)o * n * inner + i0;
            for (int k = 0; k < n; k++) {
                const cpx *src = base + (size_t)k * inner;
                cpx *dst = blk + (size_t)k * PS_LANES;
                for (int l = 0; l < lanes; l++) dst[l] = src[l];
                for (int l = lanes; l < PS_LANES; l++) dst[l].re = dst[l].im = 0.0;
            }
            fft_lanes(e, blk, work, sign);
            for (int k = 0; k < n; k++) {
                cpx *dst = base + (size_t)k * inner;
                const cpx *src = blk + (size_t)k * PS_LANES;
                for (int l = 0; l < lanes; l++) dst[l] = src[l];
            }
        }
        free(blk);
        free(work);
    }
}

/* The contiguous axis: rows are gathered PS_LANES at a time (a small transpose). */
static void last_axis_pass(cpx *data, long rows, int n, const eng1d *e, int sign)
{
    const long nblocks = (rows + PS_LANES - 1) / PS_LANES;
    const size_t work_elems = (size_t)(e->pow2 ? n : 2 * e->m) * PS_LANES;
#pragma omp parallel num_threads(ps_shim_get_threads())
    {
        cpx *blk = (cpx *)xalloc(sizeof(cpx) * (size_t)n * PS_LANES);
        cpx *work = (cpx *)xalloc(sizeof(cpx) * work_elems);
#pragma omp for schedule(static)
        for (long b = 0; b < nblocks; b++) {
            const long r0 = b * PS_LANES;
            const int lanes = (int)((rows - r0) < PS_LANES ? (rows - r0) : PS_LANES);
            for (int l = 0; l < PS_LANES; l++) {
                const cpx *src = data + (size_t)(r0 + (l < lanes ? l : 0)) * n;
                for (int k = 0; k < n; k++) {
                    if (l < lanes) blk[(size_t)k * PS_LANES + l] = src[k];
                    else blk[(size_t)k * PS_LANES + l].re = blk[(size_t)k * PS_LANES + l].im = 0.0;
                }
            }
            fft_lanes(e, blk, work, sign);
            for (int l = 0; l < lanes; l++) {
                cpx *dst = data + (size_t)(r0 + l) * n;
                for (int k = 0; k < n; k++) dst[k] = blk[(size_t)k * PS_LANES + l];
            }
        }
        free(blk);
        free(work);
    }
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags)
{
    (void)flags;
    if (n0 <= 0 || n1 <= 0 || n2 <= 0) return NULL;
    struct ps_shim_plan *p = (struct ps_shim_plan *)calloc(1, sizeof(*p));
    p->n[0] = n0;
    p->n[1] = n1;
    p->n[2] = n2;
    p->in = in;
    p->out = out;
    p->sign = sign < 0 ? -1 : +1;
    for (int a = 0; a < 3; a++) {
        p->e[a] = NULL;
        for (int b = 0; b < a; b++)
            if (p->n[b] == p->n[a]) p->e[a] = p->e[b];
        if (!p->e[a]) p->e[a] = eng_new(p->n[a]);
    }
    return p;
}

void fftw_execute(const fftw_plan p)
{
    if (!p) return;
    const size_t total = (size_t)p->n[0] * p->n[1] * p->n[2];
    cpx *d = (cpx *)p->out;
    if (p->in != p->out) memcpy(p->out, p->in, sizeof(cpx) * total);
    last_axis_pass(d, (long)p->n[0] * p->n[1], p->n[2], p->e[2], p->sign);
    axis_pass(d, p->n[0], p->n[1], p->n[2], p->e[1], p->sign);
    axis_pass(d, 1, p->n[0], (long)p->n[1] * p->n[2], p->e[0], p->sign);
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    for (int a = 0; a < 3; a++) {
        int shared = 0;
        for (int b = 0; b < a; b++)
            if (p->e[b] == p->e[a]) shared = 1;
        if (!shared) eng_free(p->e[a]);
    }
    free(p);
}

void *fftw_malloc(size_t n) { return xalloc(n); }
void fftw_free(void *p) { free(p); }
fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)xalloc(n * sizeof(fftw_complex)); }
void fftw_cleanup(void) {}
