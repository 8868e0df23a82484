/*
 * Harness around the UNMODIFIED reference sources (annehutter/polyspectrum
 * src/*.c minus main.c), built by oracle/Makefile into oracle/_ref/ against
 * the FFT shim.  TEST INFRASTRUCTURE ONLY.
 *
 * ref_run_ini() does what run() (src/run.c:29-125) does, with the reference's
 * own functions: readConfObj (confObj.c:131), read_params_to_kvectors
 * (kvectors.c:46), initGrid_with_values (grid.c:47), get_FT_field
 * (input_field.c:40, including the raw-file read of grid.c:122-228),
 * calc_phase_3D_fftw_array (utils_fftw.c:78), calc_k3min/calc_k3max
 * (kvectors.c:233-246), polyspectrum and num_polygons (polyspectrum.c:51,163).
 * Only the loop body of run.c:56-92 is repeated here, so that the results come
 * back as full-precision doubles instead of the %e text of run.c:128-222.
 */
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "fftw3.h"

#include "confObj.h"
#include "grid.h"
#include "input_field.h"
#include "kvectors.h"
#include "polyspectrum.h"
#include "utils_fftw.h"

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int ref_num_configs_ini(const char *ini)
{
    confObj_t sp = readConfObj((char *)ini);
    kvectors_t *kv = read_params_to_kvectors(sp);
    int nv = kv->numValues;
    deallocate_kvectors(kv);
    confObj_del(&sp);
    return nv;
}

/* Runs configurations [first, first+count) of the ini file's sweep (all of
 * them when count < 0).  Per-config outputs are indexed from 0.  Timings (s):
 * t_forward = get_FT_field + phase, t_configs = the polyspectrum/num_polygons
 * calls. */
int ref_run_ini(const char *ini, int first, int count, double *k_out, double *theta_out,
                double *B_out, double *npoly_out, double *kpoly_out, double *kmin_out,
                double *kmax_out, double *t_forward, double *t_configs)
{
    confObj_t sp = readConfObj((char *)ini);
    kvectors_t *kv = read_params_to_kvectors(sp);
    grid_t *g = initGrid_with_values(sp->grid_size);
    const int n = kv->n;

    double t0 = now_s();
    fftw_complex *ft = get_FT_field(g, sp);
    if (sp->calc_phases_only == 1) calc_phase_3D_fftw_array(g->nbins, g->local_n0, ft);
    double t1 = now_s();

    int last = kv->numValues;
    if (count >= 0 && first + count < last) last = first + count;
    int written = 0;
    for (int i = 0; i < last; i++) {
        /* run.c:59-84 */
        kv->kpolygon[n - 1] = kv->k[i];
        if (n == 2) kv->kpolygon[0] = kv->k[i];
        if (n == 3) {
            if (sp->equilateral == 1) {
                for (int j = 0; j < n; j++) kv->kpolygon[j] = kv->k[i];
                if (kv->kbinningCase >= 2) {
                    kv->kpolygonMin[n - 1] = calc_k3min(kv, 0);
                    kv->kpolygonMax[n - 1] = calc_k3max(kv, 0);
                }
            } else if (kv->kbinningCase >= 2) {
                kv->kpolygonMin[n - 1] = calc_k3min(kv, i);
                kv->kpolygonMax[n - 1] = calc_k3max(kv, i);
            }
        }
        if (i < first) continue; /* only the bookkeeping above carries state */
        const int o = i - first;
        /* run.c:87-91 */
        B_out[o] = polyspectrum(g->nbins, g->local_n0, g->local_0_start, ft, n, kv->kpolygon,
                                kv->kpolygonMin, kv->kpolygonMax, sp->kbinwidth,
                                kv->kbinningCase, g->box_size);
        npoly_out[o] = 0.;
        if (sp->write_numpolygons == 1)
            npoly_out[o] = num_polygons(g->nbins, g->local_n0, g->local_0_start, n, kv->kpolygon,
                                        kv->kpolygonMin, kv->kpolygonMax, sp->kbinwidth,
                                        kv->kbinningCase, g->box_size);
        k_out[o] = kv->k[i];
        theta_out[o] = kv->theta ? (sp->equilateral == 1 ? kv->theta[0] : kv->theta[i]) : 0. / 0.;
        for (int j = 0; j < n; j++) {
            kpoly_out[o * n + j] = kv->kpolygon[j];
            kmin_out[o * n + j] = kv->kpolygonMin[j];
            kmax_out[o * n + j] = kv->kpolygonMax[j];
        }
        written++;
    }
    double t2 = now_s();
    if (t_forward) *t_forward = t1 - t0;
    if (t_configs) *t_configs = t2 - t1;

    fftw_free(ft);
    deallocate_grid(g);
    deallocate_kvectors(kv);
    confObj_del(&sp);
    return written;
}
