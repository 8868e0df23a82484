/*
 * CPU oracle: a plain-C FP64 restatement of polyspectrum's FFT estimator.
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, and
 * only as the checker; the GPU product never links or calls it.
 *
 * Every function names the reference lines (annehutter/polyspectrum, paths
 * relative to the project root) whose arithmetic it restates.  The restatement
 * is pinned against the reference itself: oracle/Makefile builds the unmodified
 * reference sources against oracle/fftw_shim into oracle/_ref/, and
 * tests/test_oracle_cpu.py checks that both give bit-identical results; the
 * committed fixtures in tests/golden/ come from oracle/_ref.
 */
#ifndef PS_ORACLE_H
#define PS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* k-space filter kinds (src/filter.c) */
enum {
    ORA_SHELL_DEFAULT = 0,         /* construct_kfilter, filter.c:34-63 */
    ORA_SHELL_RANGE = 1,           /* construct_kfilter_with_kbinwidth, filter.c:130-162 */
    ORA_SHELL_WATKINSON = 2,       /* construct_kfilter_Watkinson, filter.c:178-208 */
    ORA_SHELL_WATKINSON_RANGE = 3  /* construct_kfilter_Watkinson_kn, filter.c:219-250 */
};

/* which field (src/input_field.c:40-81) */
enum { ORA_FIELD_DENS = 0, ORA_FIELD_XHII = 1, ORA_FIELD_XHI_DENS = 2 };

/* Evaluate one filter on the full N^3 lattice, row-major [i][j][l]; out = 0/1. */
void ora_filter(int nbins, int kind, double k, double kmin, double kmax, double binwidth,
                double boxsize, unsigned char *out);

/* DEFAULT filter plus the DERIVED k-range of its selected modes
 * (construct_kfilter_with_determining_kbinwidth, filter.c:78-114). */
void ora_filter_derived(int nbins, double k, double binwidth, double boxsize,
                        unsigned char *out, double *kmin, double *kmax);

/* Forward transform of the selected field (get_FT_field, input_field.c:40-81,
 * fft.c:19-37) and optional phase normalisation (utils_fftw.c:78-93).
 * dens/xhii are float (is_double=0) or double (is_double=1) N^3 arrays; the
 * output is N^3 interleaved (re,im) doubles. */
int ora_forward(int nbins, int which, const void *dens, const void *xhii, int is_double,
                int use_only_phase, double *dk_out);

/* polyspectrum(), polyspectrum.c:51-161, single process (local_n0 = N).
 * dk is N^3 interleaved complex.  kmin/kmax are in/out (DERIVED write-back).
 * sum_D / sum_I (may be NULL) receive Re(sum prod D) and Re(sum prod I). */
double ora_polyspectrum(int nbins, const double *dk, int n, const double *k, double *kmin,
                        double *kmax, double binwidth, int binning, double boxsize,
                        double *sum_D, double *sum_I);

/* num_polygons(), polyspectrum.c:163-252. */
double ora_num_polygons(int nbins, int n, const double *k, double *kmin, double *kmax,
                        double binwidth, int binning, double boxsize);

/* Parameters of one run (the [Grid]/[Polyspectrum] keys of confObj.c:39-105). */
typedef struct {
    int grid_size;
    double box_size;       /* as read from the ini file (double) */
    int which_field;       /* ORA_FIELD_* */
    int use_only_phase;    /* 1 = phase only; anything else = off (run.c:48) */
    int n;
    int equilateral;
    double k1, k2;
    int num_values;
    double theta;
    double kbinwidth;
    int kbinning;          /* 0 DEFAULT, 1 DERIVED, 2 GIVEN, 3 WATKINSON */
    double dcos_theta;
    int write_numpolygons;
} ora_params;

/* Number of configurations a run has (kvectors.c:46-147). <0 on refusal. */
int ora_num_configs(const ora_params *p);

/* The run.c:29-107 loop: forward transform, then for each configuration the
 * kpolygon bookkeeping of run.c:56-84, polyspectrum() and num_polygons().
 * Runs configurations [first, first + max_cfg) of the run's list.
 * Outputs (length max_cfg, or max_cfg*n for the per-leg arrays):
 *   k_out, theta_out (NaN where the run has no theta), B_out, npoly_out,
 *   kpoly_out / kmin_out / kmax_out: the kpolygon arrays after each config.
 * Returns the number of configurations written, <0 on error. */
int ora_run(const ora_params *p, const void *dens, const void *xhii, int is_double,
            int first, int max_cfg, double *k_out, double *theta_out, double *B_out, double *npoly_out,
            double *kpoly_out, double *kmin_out, double *kmax_out);

#ifdef __cplusplus
}
#endif

#endif
