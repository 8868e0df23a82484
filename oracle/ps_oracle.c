/*
 * CPU oracle: FP64 restatement of polyspectrum's estimator.  TEST
 * INFRASTRUCTURE ONLY (see ps_oracle.h).  Compiled -std=c99, so GCC does not
 * contract a*b+c into FMA (-ffp-contract=off in ISO mode), exactly like the
 * reference build (common.mk:10).  Expressions whose rounding decides a
 * filter bit keep the reference's operation order; each such spot cites the
 * reference line.
 */
#include "ps_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_shim/fftw3.h"

typedef double _Complex cplx;

/* pi as the reference defines it (filter.c:19, kvectors.c:25). */
static double ref_pi(void) { return acos(-1.0); }

/* Lattice frequency of FFT index idx: filter.c:44-55 (idx = N/2 maps to -N/2). */
static int lattice_freq(int idx, int nbins) { return idx < nbins / 2 ? idx : idx - nbins; }

/* Squared radii of the 8 corners of the cell of half-width bw/2 around m,
 * folded into running min/max of squares (get_corners, filter.c:257-289:
 * corner order and a+b+c evaluation order kept). */
static void corners_fold(int mx, int my, int mz, double binwidth, double *min2, double *max2)
{
    const double x = (double)mx, y = (double)my, z = (double)mz;
    const double e = 0.5 * binwidth;
    const double xm = (x - e) * (x - e), xp = (x + e) * (x + e);
    const double ym = (y - e) * (y - e), yp = (y + e) * (y + e);
    const double zm = (z - e) * (z - e), zp = (z + e) * (z + e);
    double c[8];
    c[0] = xm + ym + zm;
    c[1] = xp + ym + zm;
    c[2] = xm + yp + zm;
    c[3] = xm + ym + zp;
    c[4] = xp + yp + zm;
    c[5] = xp + ym + zp;
    c[6] = xm + yp + zp;
    c[7] = xp + yp + zp;
    for (int q = 0; q < 8; q++) {
        if (c[q] > *max2) *max2 = c[q];
        if (c[q] < *min2) *min2 = c[q];
    }
}

/* get_corners as a call: takes and returns radii, squaring them on entry and
 * taking square roots on exit (filter.c:267-268, 287-288). */
static void corner_radii(int mx, int my, int mz, double binwidth, double *rmin, double *rmax)
{
    double min2 = (*rmin) * (*rmin);
    double max2 = (*rmax) * (*rmax);
    corners_fold(mx, my, mz, binwidth, &min2, &max2);
    *rmin = sqrt(min2);
    *rmax = sqrt(max2);
}

/* One filter bit.  kk = k/(2 pi)*L for the single-k kinds, (mmin, mmax) =
 * kmin/(2 pi)*L, kmax/(2 pi)*L for the range kinds. */
static int filter_bit(int kind, int mx, int my, int mz, double kk, double mmin, double mmax,
                      double binwidth)
{
    const double half = 0.5 * binwidth;
    switch (kind) {
    case ORA_SHELL_DEFAULT: { /* filter.c:57-59 */
        const double m = sqrt((double)(mx * mx + my * my + mz * mz));
        return fabs(kk - m) <= half;
    }
    case ORA_SHELL_RANGE: { /* filter.c:155-158 */
        const double m = sqrt((double)(mx * mx + my * my + mz * mz));
        const double below = mmin - m;
        const double above = m - mmax;
        return below <= half && above <= half;
    }
    case ORA_SHELL_WATKINSON: { /* filter.c:201-204 */
        double pmin = 1.e30, pmax = 0.;
        corner_radii(mx, my, mz, binwidth, &pmin, &pmax);
        return pmin <= kk && kk <= pmax;
    }
    case ORA_SHELL_WATKINSON_RANGE: { /* filter.c:243-246 */
        double pmin = 1.e30, pmax = 0.;
        corner_radii(mx, my, mz, binwidth, &pmin, &pmax);
        return (pmax >= mmax && pmin <= mmax) || (pmax <= mmax && pmin >= mmin) ||
               (pmax >= mmin && pmin <= mmin);
    }
    default:
        return 0;
    }
}

void ora_filter(int nbins, int kind, double k, double kmin, double kmax, double binwidth,
                double boxsize, unsigned char *out)
{
    const double pi = ref_pi();
    const double kk = k / (2. * pi) * boxsize;    /* filter.c:36, :180 */
    const double mmin = kmin / (2. * pi) * boxsize; /* filter.c:137, :223 */
    const double mmax = kmax / (2. * pi) * boxsize; /* filter.c:138, :224 */
    const size_t nn = (size_t)nbins;
    for (int i = 0; i < nbins; i++) {
        const int mx = lattice_freq(i, nbins);
        for (int j = 0; j < nbins; j++) {
            const int my = lattice_freq(j, nbins);
            unsigned char *row = out + ((size_t)i * nn + (size_t)j) * nn;
            for (int l = 0; l < nbins; l++)
                row[l] = (unsigned char)filter_bit(kind, mx, my, lattice_freq(l, nbins), kk, mmin,
                                                   mmax, binwidth);
        }
    }
}

void ora_filter_derived(int nbins, double k, double binwidth, double boxsize, unsigned char *out,
                        double *kmin, double *kmax)
{
    /* filter.c:78-114: the DEFAULT bit, and for every selected mode the
     * running (min, max) corner radius, visited in i, j, l order. */
    const double pi = ref_pi();
    const double kk = k / (2. * pi) * boxsize;
    double rmin = 1.e30, rmax = 0.;
    const size_t nn = (size_t)nbins;
    for (int i = 0; i < nbins; i++) {
        const int mx = lattice_freq(i, nbins);
        for (int j = 0; j < nbins; j++) {
            const int my = lattice_freq(j, nbins);
            unsigned char *row = out + ((size_t)i * nn + (size_t)j) * nn;
            for (int l = 0; l < nbins; l++) {
                const int mz = lattice_freq(l, nbins);
                const int bit = filter_bit(ORA_SHELL_DEFAULT, mx, my, mz, kk, 0., 0., binwidth);
                row[l] = (unsigned char)bit;
                if (bit) corner_radii(mx, my, mz, binwidth, &rmin, &rmax);
            }
        }
    }
    *kmin = rmin * 2. * pi / boxsize; /* filter.c:112-113 */
    *kmax = rmax * 2. * pi / boxsize;
}

/* k3 range of the closing leg from the ranges of legs 0 and 1
 * (calc_k3_min_and_max, filter.c:291-319). */
static void closing_leg_range(const double *k, double *kmin, double *kmax)
{
    const double c = (k[0] * k[0] + k[1] * k[1] - k[2] * k[2]) / (2. * k[0] * k[1]);
    const double a[8] = {kmin[0], kmin[0], kmax[0], kmax[0], k[0], kmax[0], k[0], kmin[0]};
    const double b[8] = {kmin[1], kmax[1], kmin[1], kmax[1], kmax[1], k[1], kmin[1], k[1]};
    double lo = 1.e30, hi = 0.;
    for (int q = 0; q < 8; q++) {
        const double t = a[q] * a[q] + b[q] * b[q] - 2. * a[q] * b[q] * c;
        if (t < lo) lo = t;
        if (t > hi) hi = t;
    }
    kmin[2] = sqrt(lo);
    kmax[2] = sqrt(hi);
}

static void *grab(size_t bytes)
{
    void *p = fftw_malloc(bytes);
    return p;
}

/* Leg filter as the reference selects it (polyspectrum.c:79-118, :179-218).
 * Returns 0, or -1 where the reference is undefined (DERIVED with n != 3:
 * calc_kn_min_and_max, filter.c:321-325, dereferences past a local pointer). */
static int leg_filter(int nbins, int leg, int n, const double *k, double *kmin, double *kmax,
                      double binwidth, int binning, double boxsize, unsigned char *mask)
{
    const int last = leg == n - 1;
    switch (binning) {
    case 1:
        if (!last) {
            ora_filter_derived(nbins, k[leg], binwidth, boxsize, mask, &kmin[leg], &kmax[leg]);
        } else {
            if (n != 3) return -1;
            closing_leg_range(k, kmin, kmax);
            ora_filter(nbins, ORA_SHELL_RANGE, 0., kmin[leg], kmax[leg], binwidth, boxsize, mask);
        }
        return 0;
    case 2:
        if (!last) ora_filter(nbins, ORA_SHELL_DEFAULT, k[leg], 0., 0., binwidth, boxsize, mask);
        else ora_filter(nbins, ORA_SHELL_RANGE, 0., kmin[leg], kmax[leg], binwidth, boxsize, mask);
        return 0;
    case 3:
        if (!last) ora_filter(nbins, ORA_SHELL_WATKINSON, k[leg], 0., 0., binwidth, boxsize, mask);
        else
            ora_filter(nbins, ORA_SHELL_WATKINSON_RANGE, 0., kmin[leg], kmax[leg], binwidth, boxsize,
                       mask);
        return 0;
    default:
        ora_filter(nbins, ORA_SHELL_DEFAULT, k[leg], 0., 0., binwidth, boxsize, mask);
        return 0;
    }
}

static void backward_dft(int nbins, cplx *in, cplx *out)
{
    fftw_plan p = fftw_plan_dft_3d(nbins, nbins, nbins, (fftw_complex *)in, (fftw_complex *)out,
                                   FFTW_BACKWARD, FFTW_ESTIMATE);
    fftw_execute(p);
    fftw_destroy_plan(p);
}

/* Shared leg loop of polyspectrum() and num_polygons(): running complex
 * products of I = IFFT[F] and (when dk != NULL) D = IFFT[F * dk]. */
static int leg_products(int nbins, const cplx *dk, int n, const double *k, double *kmin,
                        double *kmax, double binwidth, int binning, double boxsize,
                        cplx *prod_I, cplx *prod_D)
{
    const size_t total = (size_t)nbins * nbins * nbins;
    unsigned char *mask = (unsigned char *)malloc(total);
    cplx *filt = (cplx *)grab(sizeof(cplx) * total);
    cplx *field = (cplx *)grab(sizeof(cplx) * total);
    cplx *tmp = (cplx *)grab(sizeof(cplx) * total);
    int rc = 0;
    for (size_t q = 0; q < total; q++) {
        prod_I[q] = 1. + 0. * I; /* polyspectrum.c:57-61 */
        if (prod_D) prod_D[q] = 1. + 0. * I;
    }
    for (int leg = 0; leg < n && rc == 0; leg++) {
        rc = leg_filter(nbins, leg, n, k, kmin, kmax, binwidth, binning, boxsize, mask);
        if (rc) break;
        for (size_t q = 0; q < total; q++) filt[q] = mask[q] ? 1. + 0. * I : 0. + 0. * I;
        backward_dft(nbins, filt, field); /* generate_num_polygons, polyspectrum.c:41-49 */
        for (size_t q = 0; q < total; q++) prod_I[q] = prod_I[q] * field[q];
        if (prod_D) {
            /* generate_values_polygons, polyspectrum.c:24-38 */
            for (size_t q = 0; q < total; q++) tmp[q] = filt[q] * dk[q];
            backward_dft(nbins, tmp, field);
            for (size_t q = 0; q < total; q++) prod_D[q] = prod_D[q] * field[q];
        }
    }
    free(mask);
    fftw_free(filt);
    fftw_free(field);
    fftw_free(tmp);
    return rc;
}

static double real_sum(const cplx *a, size_t total)
{
    cplx s = 0. + 0. * I; /* sum_3D_fftw_array, utils_fftw.c:60-76 */
    for (size_t q = 0; q < total; q++) s += a[q];
    return creal(s);
}

double ora_polyspectrum(int nbins, const double *dk, int n, const double *k, double *kmin,
                        double *kmax, double binwidth, int binning, double boxsize,
                        double *sum_D, double *sum_I)
{
    const size_t total = (size_t)nbins * nbins * nbins;
    cplx *pI = (cplx *)grab(sizeof(cplx) * total);
    cplx *pD = (cplx *)grab(sizeof(cplx) * total);
    double result = NAN;
    if (leg_products(nbins, (const cplx *)dk, n, k, kmin, kmax, binwidth, binning, boxsize, pI,
                     pD) == 0) {
        const double sI = real_sum(pI, total);
        const double sD = real_sum(pD, total);
        const double volume = boxsize * boxsize * boxsize;
        result = pow(volume, n - 1) * pow(nbins, -n * 3) * sD / sI; /* polyspectrum.c:155 */
        if (sum_D) *sum_D = sD;
        if (sum_I) *sum_I = sI;
    }
    fftw_free(pI);
    fftw_free(pD);
    return result;
}

double ora_num_polygons(int nbins, int n, const double *k, double *kmin, double *kmax,
                        double binwidth, int binning, double boxsize)
{
    const size_t total = (size_t)nbins * nbins * nbins;
    cplx *pI = (cplx *)grab(sizeof(cplx) * total);
    double result = NAN;
    if (leg_products(nbins, NULL, n, k, kmin, kmax, binwidth, binning, boxsize, pI, NULL) == 0)
        result = real_sum(pI, total) / (double)(nbins * nbins * nbins); /* polyspectrum.c:247 */
    fftw_free(pI);
    return result;
}

int ora_forward(int nbins, int which, const void *dens, const void *xhii, int is_double,
                int use_only_phase, double *dk_out)
{
    const size_t total = (size_t)nbins * nbins * nbins;
    cplx *field = (cplx *)grab(sizeof(cplx) * total);
    const float *df = (const float *)dens, *xf = (const float *)xhii;
    const double *dd = (const double *)dens, *xd = (const double *)xhii;
#define VAL(pf, pd, q) (is_double ? (pd)[q] : (double)(pf)[q])
    for (size_t q = 0; q < total; q++) {
        double v;
        if (which == ORA_FIELD_DENS) v = VAL(df, dd, q);
        else if (which == ORA_FIELD_XHII) v = VAL(xf, xd, q);
        else v = VAL(df, dd, q) * (1. - VAL(xf, xd, q)); /* input_field.c:33 */
        field[q] = v + 0. * I;
    }
#undef VAL
    cplx *out = (cplx *)dk_out;
    fftw_plan p = fftw_plan_dft_3d(nbins, nbins, nbins, (fftw_complex *)field, (fftw_complex *)out,
                                   FFTW_FORWARD, FFTW_ESTIMATE); /* fft.c:32 */
    fftw_execute(p);
    fftw_destroy_plan(p);
    fftw_free(field);
    if (use_only_phase == 1) /* run.c:48-49 */
        for (size_t q = 0; q < total; q++) {
            const cplx v = out[q];
            out[q] = v / cabs(v); /* utils_fftw.c:89 */
        }
    return 0;
}

int ora_num_configs(const ora_params *p)
{
    if (p->n == 2) return p->num_values > 1 ? p->grid_size / 2 : 1;  /* kvectors.c:75-90 */
    if (p->n == 3) return p->equilateral == 1 ? p->num_values : (p->num_values > 1 ? p->num_values : 1);
    return -1; /* kvectors.c:60-64, :140-144: refused */
}

int ora_run(const ora_params *p, const void *dens, const void *xhii, int is_double, int first, int max_cfg,
            double *k_out, double *theta_out, double *B_out, double *npoly_out, double *kpoly_out,
            double *kmin_out, double *kmax_out)
{
    const double pi = ref_pi();
    const int n = p->n;
    const int nval = ora_num_configs(p);
    if (nval < 0 || n > 3) return -1;
    const int N = p->grid_size;
    /* kvectors.c:46-147 */
    double *kl = (double *)calloc((size_t)(nval > 2 ? nval : 2), sizeof(double));
    double *th = NULL;
    double kpoly[3] = {0., 0., 0.}, kpmin[3] = {0., 0., 0.}, kpmax[3] = {0., 0., 0.};
    if (n == 2) {
        if (p->num_values > 1) {
            for (int i = 0; i < nval; i++) kl[i] = 2. * pi / p->box_size * (double)(i + 1);
        } else {
            kl[0] = p->k1;
            kl[1] = p->k1; /* kvectors.c:89 writes k[1] of a length-1 array */
        }
        for (int i = 0; i < 2; i++) kpoly[i] = kpmin[i] = kpmax[i] = kl[i];
    } else {
        kpoly[0] = p->k1;
        kpoly[1] = p->k2;
        th = (double *)calloc((size_t)(nval > 1 ? nval : 1), sizeof(double));
        if (p->equilateral == 1) {
            const double kL = 2. * pi / p->box_size; /* kvectors.c:213-224 */
            for (int i = 0; i < nval; i++)
                kl[i] = kL * pow(p->grid_size / 2, (double)(i + 1) / (double)nval);
            th[0] = pi / 3.;
        } else if (p->num_values > 1) {
            for (int i = 0; i < nval; i++) { /* kvectors.c:172-198 */
                th[i] = pi * (double)i / (double)nval;
                const double c = cos(th[i]);
                kl[i] = sqrt(p->k1 * p->k1 + p->k2 * p->k2 - 2. * p->k1 * p->k2 * c);
            }
        } else {
            th[0] = p->theta;
            const double c = cos(p->theta);
            kl[0] = sqrt(p->k1 * p->k1 + p->k2 * p->k2 - 2. * p->k1 * p->k2 * c);
        }
    }
    const size_t total = (size_t)N * N * N;
    double *dk = (double *)grab(sizeof(double) * 2 * total);
    ora_forward(N, p->which_field, dens, xhii, is_double, p->use_only_phase, dk);
    const double L = (double)(float)p->box_size; /* grid.h:9 stores box_size as float */
    int written = 0;
    /* configurations [first, first + max_cfg) of the list; each one's ranges are
       set afresh inside the loop (run.c:56-84), so skipping earlier ones changes
       nothing */
    for (int i = first < 0 ? 0 : first; i < nval && written < max_cfg; i++) { /* run.c:56-107 */
        const int o = written;
        kpoly[n - 1] = kl[i];
        if (n == 2) kpoly[0] = kl[i];
        if (n == 3) {
            const int ti = p->equilateral == 1 ? 0 : i;
            if (p->equilateral == 1)
                for (int j = 0; j < n; j++) kpoly[j] = kl[i];
            if (p->kbinning >= 2) { /* kvectors.c:233-246 */
                const double cmin = fmin(1., cos(th[ti]) + 0.5 * p->dcos_theta);
                const double cmax = fmax(-1., cos(th[ti]) - 0.5 * p->dcos_theta);
                kpmin[n - 1] = sqrt(kpoly[0] * kpoly[0] + kpoly[1] * kpoly[1] -
                                    2. * kpoly[0] * kpoly[1] * cmin);
                kpmax[n - 1] = sqrt(kpoly[0] * kpoly[0] + kpoly[1] * kpoly[1] -
                                    2. * kpoly[0] * kpoly[1] * cmax);
            }
        }
        B_out[o] = ora_polyspectrum(N, dk, n, kpoly, kpmin, kpmax, p->kbinwidth, p->kbinning, L,
                                    NULL, NULL);
        npoly_out[o] = p->write_numpolygons == 1
                           ? ora_num_polygons(N, n, kpoly, kpmin, kpmax, p->kbinwidth, p->kbinning, L)
                           : 0.;
        k_out[o] = kl[i];
        theta_out[o] = th ? (p->equilateral == 1 ? th[0] : th[i]) : NAN;
        for (int j = 0; j < n; j++) {
            kpoly_out[o * n + j] = kpoly[j];
            kmin_out[o * n + j] = kpmin[j];
            kmax_out[o * n + j] = kpmax[j];
        }
        written++;
    }
    free(kl);
    free(th);
    fftw_free(dk);
    return written;
}
