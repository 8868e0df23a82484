/*
 * ps_run - command-line driver of the B200 polyspectrum estimator.
 *
 *   ps_run [--method batched|plain] [--device D] [--dry-run] [--exact] [--no-kappa] iniFile
 *
 * The reference's executable (src/main.c, src/run.c) rebuilt over the C-ABI of
 * include/ps_gpu.h: it reads the same ini file (the keys of confObj.c:39-105 in
 * the syntax of parse_ini.c:115-215), the same raw input grids (grid.c:122-228:
 * N^3 float, or double when *InputsInDoublePrecision = 1), prints the same
 * progress lines (run.c:33-108) and writes the same output file, with the same
 * name and format (run.c:128-222).  Where the reference exits with a message,
 * this exits with EXIT_FAILURE and the same message.  Beyond the reference:
 * unreadable or short input files and unwritable output files are reported
 * instead of being read or written through a NULL FILE*.
 *
 * --method batched (default) evaluates all configurations with
 * PS_FP32_BATCHED, --method plain with PS_FP64_PLAIN (the reference dataflow
 * in FP64).  --dry-run parses the ini file, generates the configurations and
 * prints them with the output file name, without reading the inputs or using
 * the GPU.
 */
#define _POSIX_C_SOURCE 200809L
#include <ctype.h>
#include <dirent.h>
#include <inttypes.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/ps_gpu.h"

#define MAXLEN 1024

/* ------------------------------------------------------------ ini file --- */
/* Sections and "key = value" lines (parse_ini.c:145-212): lines starting with
 * '#' and blank lines are skipped, a section name keeps only its alphanumeric
 * characters, a value runs from the first non-blank after '=' to the end of
 * the line minus trailing blanks (a trailing "# comment" stays part of it, as
 * there; numeric keys parse their leading number).  Lookups take the first
 * section of a name and the first key of a name inside it. */
typedef struct {
    int sec;
    char *key, *val;
} ini_key;

typedef struct {
    char **secs;
    int nsec;
    ini_key *keys;
    int nkey;
} ini_file;

static char *dup_range(const char *a, size_t n)
{
    char *s = malloc(n + 1);
    if (!s) return NULL;
    memcpy(s, a, n);
    s[n] = '\0';
    return s;
}

static void ini_free(ini_file *ini)
{
    for (int i = 0; i < ini->nsec; i++) free(ini->secs[i]);
    for (int i = 0; i < ini->nkey; i++) {
        free(ini->keys[i].key);
        free(ini->keys[i].val);
    }
    free(ini->secs);
    free(ini->keys);
    memset(ini, 0, sizeof(*ini));
}

/* 0 on success, -1 when the file cannot be opened, -2 on a malformed line
 * (reported as parse_ini.c:176,198 report it). */
static int ini_load(const char *path, ini_file *ini)
{
    memset(ini, 0, sizeof(*ini));
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char *line = NULL;
    size_t cap = 0;
    ssize_t len;
    int rc = 0;
    while ((len = getline(&line, &cap, f)) > 0) {
        size_t i = 0;
        while (line[i] == ' ' || line[i] == '\t') i++;
        if (i == (size_t)len - 1) line[0] = '\0';  /* only blanks before the last character */
        if (line[0] == '\0' || line[0] == '#') continue;
        if (line[0] == '[') {
            char name[MAXLEN];
            size_t n = 0;
            for (size_t p = 1; line[p] != '\0' && line[p] != ']'; p++)
                if (isalnum((unsigned char)line[p]) && n + 1 < sizeof(name)) name[n++] = line[p];
            if (n == 0) {
                fprintf(stderr, "Could not parse '%s'\n", line);
                rc = -2;
                break;
            }
            char **s = realloc(ini->secs, sizeof(char *) * (ini->nsec + 1));
            if (!s) { rc = -2; break; }
            ini->secs = s;
            ini->secs[ini->nsec++] = dup_range(name, n);
            continue;
        }
        if (ini->nsec == 0) continue;  /* keys before any section are ignored */
        size_t start = 0;
        while (line[start] == ' ' || line[start] == '\t') start++;
        size_t sep = start;
        while (line[sep] != '\0' && line[sep] != '=') sep++;
        int bad = sep == start || line[sep] == '\0';
        size_t vs = sep + 1;
        if (!bad) {
            while (line[vs] == ' ' || line[vs] == '\t') vs++;
            bad = line[vs] == '\0';
        }
        if (bad) {
            fprintf(stderr, "Could not parse '%s'\n", line);
            rc = -2;
            break;
        }
        size_t ke = sep;  /* one past the key's last character */
        while (ke > start && (line[ke - 1] == ' ' || line[ke - 1] == '\t')) ke--;
        size_t ve = strlen(line);
        while (ve > vs && (line[ve - 1] == ' ' || line[ve - 1] == '\t' || line[ve - 1] == '\n')) ve--;
        ini_key *k = realloc(ini->keys, sizeof(ini_key) * (ini->nkey + 1));
        if (!k) { rc = -2; break; }
        ini->keys = k;
        ini->keys[ini->nkey].sec = ini->nsec - 1;
        ini->keys[ini->nkey].key = dup_range(line + start, ke - start);
        ini->keys[ini->nkey].val = dup_range(line + vs, ve - vs);
        ini->nkey++;
    }
    free(line);
    fclose(f);
    if (rc) ini_free(ini);
    return rc;
}

/* value of key in section, NULL when absent; *sec_found tells which */
static const char *ini_get(const ini_file *ini, const char *sec, const char *key, int *sec_found)
{
    int s = -1;
    for (int i = 0; i < ini->nsec && s < 0; i++)
        if (strcmp(ini->secs[i], sec) == 0) s = i;
    if (sec_found) *sec_found = s >= 0;
    if (s < 0) return NULL;
    for (int i = 0; i < ini->nkey; i++)
        if (ini->keys[i].sec == s && strcmp(ini->keys[i].key, key) == 0) return ini->keys[i].val;
    return NULL;
}

static void fatal_key(const char *key, const char *sec)
{
    fprintf(stderr, "FATAL:  Could not get %s from section %s.\n", key, sec);  /* parse_ini.h:16-22 */
    exit(EXIT_FAILURE);
}

static int get_int(const ini_file *ini, const char *sec, const char *key)
{
    const char *v = ini_get(ini, sec, key, NULL);
    int32_t x;
    if (!v || sscanf(v, "%" SCNi32, &x) != 1) fatal_key(key, sec);
    return (int)x;
}

/* parse_ini_get_int32_ifavail: -1 when the key is absent from the section */
static int get_int_ifavail(const ini_file *ini, const char *sec, const char *key)
{
    int found = 0;
    const char *v = ini_get(ini, sec, key, &found);
    if (!found) fatal_key(key, sec);
    if (!v) return -1;
    int32_t x;
    if (sscanf(v, "%" SCNi32, &x) != 1) fatal_key(key, sec);
    return (int)x;
}

static double get_double(const ini_file *ini, const char *sec, const char *key)
{
    const char *v = ini_get(ini, sec, key, NULL);
    double x;
    if (!v || sscanf(v, "%lf", &x) != 1) fatal_key(key, sec);
    return x;
}

static char *get_string(const ini_file *ini, const char *sec, const char *key)
{
    const char *v = ini_get(ini, sec, key, NULL);
    if (!v) fatal_key(key, sec);
    return dup_range(v, strlen(v));
}

/* the keys of confObj_new (confObj.c:39-105), read in the same order */
typedef struct {
    int grid_size;
    double box_size;
    int gas_dp, ion_dp;
    char *density_file, *ion_file, *output_dir, *output_basename;
    int write_numpolygons;
    double h, omega_b, omega_m, omega_l, sigma8, Y;
    char *which_field;
    int calc_phases_only, n, equilateral;
    double k1, k2;
    int num_values;
    double theta, kbinwidth, dcosTheta;
    int kbinningCase;
} run_conf;

static void read_conf(const char *path, run_conf *c)
{
    ini_file ini;
    if (ini_load(path, &ini) != 0) {
        fprintf(stderr, "FATAL:  Could not open %s for reading.\n", path);  /* confObj.c:135-138 */
        exit(EXIT_FAILURE);
    }
    c->grid_size = get_int(&ini, "Grid", "gridsize");
    c->box_size = get_double(&ini, "Grid", "boxsize");
    c->gas_dp = get_int(&ini, "Grid", "gasInputsInDoublePrecision");
    c->ion_dp = get_int(&ini, "Grid", "ionInputsInDoublePrecision");
    c->density_file = get_string(&ini, "Grid", "densityFile");
    c->ion_file = get_string(&ini, "Grid", "ionFile");
    c->output_dir = get_string(&ini, "Output", "output_dir");
    c->output_basename = get_string(&ini, "Output", "output_basename");
    c->write_numpolygons = get_int(&ini, "Output", "write_numpolygons");
    c->h = get_double(&ini, "Cosmology", "hubble_h");
    c->omega_b = get_double(&ini, "Cosmology", "omega_b");
    c->omega_m = get_double(&ini, "Cosmology", "omega_m");
    c->omega_l = get_double(&ini, "Cosmology", "omega_l");
    c->sigma8 = get_double(&ini, "Cosmology", "sigma8");
    c->Y = get_double(&ini, "Cosmology", "Y");
    c->which_field = get_string(&ini, "Polyspectrum", "whichField");
    c->calc_phases_only = get_int_ifavail(&ini, "Polyspectrum", "useOnlyPhase");
    c->n = get_int(&ini, "Polyspectrum", "n");
    c->equilateral = get_int(&ini, "Polyspectrum", "equilateral");
    c->k1 = get_double(&ini, "Polyspectrum", "k1");
    c->k2 = get_double(&ini, "Polyspectrum", "k2");
    c->num_values = get_int(&ini, "Polyspectrum", "numValues");
    c->theta = get_double(&ini, "Polyspectrum", "theta");
    c->kbinwidth = get_double(&ini, "Polyspectrum", "kbinwidth");
    c->dcosTheta = get_double(&ini, "Polyspectrum", "cosThetaBinwidth");
    char *kb = get_string(&ini, "Polyspectrum", "kbinningCase");
    if (strcmp(kb, "DERIVED_BINNING") == 0) c->kbinningCase = PS_BIN_DERIVED;
    else if (strcmp(kb, "GIVEN_BINNING") == 0) c->kbinningCase = PS_BIN_GIVEN;
    else if (strcmp(kb, "WATKINSON") == 0) c->kbinningCase = PS_BIN_WATKINSON;
    else c->kbinningCase = PS_BIN_DEFAULT;
    free(kb);
    ini_free(&ini);
}

/* ------------------------------------------------------------ inputs ----- */
/* read_grid / read_grid_doubleprecision (grid.c:122-228): N^3 raw values */
/* An input grid file (read_grid, grid.c:122-228): it must hold n3 values of
   its precision; returns the first value (the reference's progress line
   prints the first value of the field).  The library then streams the file
   to the device (ps_gpu_set_field_files). */
static double check_raw(const char *path, size_t n3, int dp)
{
    const size_t es = dp ? sizeof(double) : sizeof(float);
    FILE *f = fopen(path, "rb");
    if (!f) {
        fprintf(stderr, "ps_run: cannot open input file %s\n", path);
        exit(EXIT_FAILURE);
    }
    double v = 0.0;
    size_t got = 0;
    if (dp) got = fread(&v, es, 1, f);
    else {
        float x = 0.f;
        got = fread(&x, es, 1, f);
        v = (double)x;
    }
    long long size = -1;
    if (fseek(f, 0, SEEK_END) == 0) size = (long long)ftell(f);
    fclose(f);
    const size_t have = size >= 0 ? (size_t)size / es : got;
    if (got != 1 || have < n3) {
        fprintf(stderr, "ps_run: %s holds %zu of the %zu values of the grid\n", path, have < n3 ? have : 0, n3);
        exit(EXIT_FAILURE);
    }
    return v;
}

/* ------------------------------------------------------------ output ----- */
/* file name of save_polyspectrum(_numpolygons) (run.c:128-150) */
static char *output_name(const run_conf *c)
{
    char ending[MAXLEN] = "";
    if (c->n == 2) snprintf(ending, sizeof(ending), "_ps.dat");
    else if (c->n == 3) {
        if (c->equilateral == 1) snprintf(ending, sizeof(ending), "_bs_equilateral.dat");
        else if (c->num_values == 1)
            snprintf(ending, sizeof(ending), "_bs_k_%4.2e_%4.2e_theta_%4.2e.dat", c->k1, c->k2, c->theta);
        else snprintf(ending, sizeof(ending), "_bs_k_%4.2e_%4.2e.dat", c->k1, c->k2);
    }
    const size_t len = strlen(c->output_dir) + 1 + strlen(c->output_basename) + strlen(ending) + 1;
    char *s = malloc(len);
    snprintf(s, len, "%s/%s%s", c->output_dir, c->output_basename, ending);
    return s;
}

static int write_output(const run_conf *c, const char *fname, int num, const double *theta, const double *k,
                        const double *B, const double *Np)
{
    FILE *f = fopen(fname, "wb");
    if (!f) return -1;
    const int wn = c->write_numpolygons == 1;
    if (c->n == 2 || c->equilateral == 1) {
        fprintf(f, "# k [h^-1 Mpc]\t Polyspectrum_%d(k)\n", c->n);
        for (int i = 0; i < num; i++) {
            if (wn) fprintf(f, "%e\t%e\t%e\n", k[i], B[i], Np[i]);
            else fprintf(f, "%e\t%e\n", k[i], B[i]);
        }
    } else if (c->n == 3) {
        fprintf(f, "# theta [rad]\t k [h^-1 Mpc]\t Polyspectrum_%d(k)\n", c->n);
        for (int i = 0; i < num; i++) {
            if (wn) fprintf(f, "%e\t%e\t%e\t%e\n", theta[i], k[i], B[i], Np[i]);
            else fprintf(f, "%e\t%e\t%e\n", theta[i], k[i], B[i]);
        }
    }
    return fclose(f) == 0 ? 0 : -1;
}

/* --exact: the same results at full precision ("%.17g": every double round-trips),
   one line per configuration with its legs as the estimator used them (a
   DERIVED closing leg with its computed range), written to <fname>.exact;
   the reference's file keeps "%e" (6 digits). */
static int write_exact(const run_conf *c, const char *fname, int num, const double *theta, const double *k,
                       const ps_cfg *cfgs, const double *B, const double *Np)
{
    const size_t len = strlen(fname) + 7;
    char *path = malloc(len);
    snprintf(path, len, "%s.exact", fname);
    FILE *f = fopen(path, "wb");
    free(path);
    if (!f) return -1;
    fprintf(f, "# n = %d; per configuration: theta [rad], k [h Mpc^-1], then (k_i kmin_i kmax_i) per leg, "
               "Polyspectrum_%d, Npolygons\n", c->n, c->n);
    for (int i = 0; i < num; i++) {
        fprintf(f, "%.17g\t%.17g", theta[i], k[i]);
        for (int l = 0; l < cfgs[i].n; l++)
            fprintf(f, "\t%.17g\t%.17g\t%.17g", cfgs[i].k[l], cfgs[i].kmin[l], cfgs[i].kmax[l]);
        fprintf(f, "\t%.17g\t%.17g\n", B[i], Np[i]);
    }
    return fclose(f) == 0 ? 0 : -1;
}

static void die_ps(const char *what, int rc)
{
    fprintf(stderr, "ps_run: %s: %s (%s)\n", what, ps_gpu_strerror(rc), ps_gpu_last_error());
    exit(EXIT_FAILURE);
}

static void usage(void)
{
    printf("ps_run: B200 polyspectrum estimator\n");
    printf("USAGE:\n");
    printf("ps_run [--method batched|plain] [--device D] [--dry-run] [--exact] [--no-kappa] iniFile\n");
    exit(EXIT_FAILURE);
}

int main(int argc, char **argv)
{
    const double t1 = (double)time(NULL);
    int method = PS_FP32_BATCHED, device = -1, dry = 0, exact = 0, kappa_on = 1;
    const char *ini_path = NULL;
    for (int a = 1; a < argc; a++) {
        if (strcmp(argv[a], "--method") == 0 && a + 1 < argc) {
            a++;
            if (strcmp(argv[a], "batched") == 0) method = PS_FP32_BATCHED;
            else if (strcmp(argv[a], "plain") == 0) method = PS_FP64_PLAIN;
            else usage();
        } else if (strcmp(argv[a], "--device") == 0 && a + 1 < argc) {
            device = atoi(argv[++a]);
        } else if (strcmp(argv[a], "--dry-run") == 0) {
            dry = 1;
        } else if (strcmp(argv[a], "--exact") == 0) {
            exact = 1;
        } else if (strcmp(argv[a], "--no-kappa") == 0) {
            kappa_on = 0;
        } else if (argv[a][0] == '-' || ini_path) {
            usage();
        } else {
            ini_path = argv[a];
        }
    }
    if (!ini_path) usage();

    run_conf c;
    read_conf(ini_path, &c);

    /* read_params_to_kvectors (kvectors.c:46-147) + run.c:56-84 */
    if (c.n < 2) {
        fprintf(stderr, "No valid input for n being the number of k-vectors, as their sum is unequal to zero: n>=2\n");
        exit(EXIT_FAILURE);
    }
    if (c.n > 3) {
        printf("Not implemented yet\n");
        exit(EXIT_FAILURE);
    }
    ps_run_params p = {c.grid_size, c.box_size, c.n, c.equilateral, c.k1, c.k2, c.num_values,
                       c.theta, c.kbinwidth, c.kbinningCase, c.dcosTheta};
    const int num = ps_make_configs(&p, NULL, 0, NULL, NULL);
    if (num < 0) die_ps("configuration list", num);
    ps_cfg *cfgs = calloc(num > 0 ? num : 1, sizeof(ps_cfg));
    double *kv = calloc(num > 0 ? num : 1, sizeof(double));
    double *th = calloc(num > 0 ? num : 1, sizeof(double));
    double *B = calloc(num > 0 ? num : 1, sizeof(double));
    double *Np = calloc(num > 0 ? num : 1, sizeof(double));
    if (!cfgs || !kv || !th || !B || !Np) {
        fprintf(stderr, "ps_run: no memory\n");
        exit(EXIT_FAILURE);
    }
    int rc = ps_make_configs(&p, cfgs, num, kv, th);
    if (rc < 0) die_ps("configuration list", rc);
    printf("kbinningCase = %d\n", c.kbinningCase);

    DIR *d = opendir(c.output_dir);
    if (!d) {
        fprintf(stderr, "Directory for output does not exist!\n");
        exit(EXIT_FAILURE);
    }
    closedir(d);
    char *fname = output_name(&c);

    if (dry) {
        for (int i = 0; i < num; i++) {
            printf("config %d: n=%d kbinningCase=%d kbinwidth=%.17g theta=%.17g k=%.17g legs", i, cfgs[i].n,
                   cfgs[i].kbinningCase, cfgs[i].kbinwidth, th[i], kv[i]);
            for (int l = 0; l < cfgs[i].n; l++)
                printf(" (%.17g %.17g %.17g)", cfgs[i].k[l], cfgs[i].kmin[l], cfgs[i].kmax[l]);
            printf("\n");
        }
        printf("FILENAME : %s\n", fname);
        return 0;
    }

    /* get_FT_field (input_field.c:40-81) */
    int which;
    if (strcmp(c.which_field, "DENS") == 0) which = PS_FIELD_DENS;
    else if (strcmp(c.which_field, "XHII") == 0) which = PS_FIELD_XHII;
    else if (strcmp(c.which_field, "XHI_DENS") == 0) which = PS_FIELD_XHI_DENS;
    else {
        printf("Option: %s\t", c.which_field);
        fflush(stdout);
        fprintf(stderr, "Not supported option. Please use 'DENS', 'XHII' or 'XHI_DENS'\n");
        exit(EXIT_FAILURE);
    }
    {
        /* the grid sizes the library's transforms take (ps_gpu_create refuses others) */
        static const int sizes[] = {16, 32, 48, 60, 64, 96, 128, 192, 256, 300, 320, 384, 512, 600, 1024};
        int ok = 0;
        for (size_t q = 0; q < sizeof(sizes) / sizeof(sizes[0]); q++) ok |= sizes[q] == c.grid_size;
        if (!ok) {
            fprintf(stderr, "ps_run: gridsize %d: supported are the powers of two 16..1024 and 48, 60, 96, 192, "
                            "300, 320, 384, 600\n", c.grid_size);
            exit(EXIT_FAILURE);
        }
    }
    printf("Option: %s\t", c.which_field);
    const size_t n3 = (size_t)c.grid_size * c.grid_size * c.grid_size;
    double v0 = 0.0;
    if (which == PS_FIELD_DENS) {
        v0 = check_raw(c.density_file, n3, c.gas_dp == 1);
    } else if (which == PS_FIELD_XHII) {
        v0 = check_raw(c.ion_file, n3, c.ion_dp == 1);
    } else {
        const double d0 = check_raw(c.density_file, n3, c.gas_dp == 1);
        v0 = d0 * (1. - check_raw(c.ion_file, n3, c.ion_dp == 1)); /* input_field.c:33 */
    }
    printf(" Mean value from FT is %e\nComputing FFT... ", v0);
    fflush(stdout);

    ps_gpu_ctx *ctx = NULL;
    rc = ps_gpu_create(&ctx, c.grid_size, (double)(float)c.box_size, method, device);  /* grid.h:9 */
    if (rc) die_ps("context", rc);
    rc = ps_gpu_set_field_files(ctx, which, which == PS_FIELD_XHII ? NULL : c.density_file, c.gas_dp == 1,
                                which == PS_FIELD_DENS ? NULL : c.ion_file, c.ion_dp == 1, c.calc_phases_only == 1);
    if (rc) die_ps("field", rc);
    printf("done.\n");

    double *kap = kappa_on ? (double *)malloc(sizeof(double) * (size_t)num) : NULL;
    if (kappa_on && !kap) {
        fprintf(stderr, "ps_run: no memory\n");
        exit(EXIT_FAILURE);
    }
    rc = ps_gpu_polyspectrum_batch(ctx, method, num, cfgs, B, Np, kap);
    if (rc) die_ps("polyspectrum", rc);
    /* The reference prints per configuration the imaginary over the real part of
     * both grid sums (polyspectrum.c:142), its rounding-health signal; here every
     * sum is real by construction, and the signal is the condition number of the
     * value sum, kappa = sum|terms| / |sum|: B is good to about kappa times the
     * method's unit roundoff. */
    const double eps = method == PS_FP64_PLAIN ? 1.1102230246251565e-16 : 5.9604644775390625e-08;
    for (int i = 0; i < num && kap; i++)
        printf("rank 0: kappa(sumValuesPolygons) = %e\t(relative error of B about %e)\n", kap[i], kap[i] * eps);
    for (int i = 0; i < num; i++) {  /* run.c:95-107 */
        if (c.n == 2) printf("k = %e\t P(k) = %e\t", kv[i], B[i]);
        if (c.n == 3)
            printf("k1 = %e\t k2 = %e\tk3 = %e\t B(k) = %e\t", cfgs[i].k[0], cfgs[i].k[1], kv[i], B[i]);
        if (c.write_numpolygons == 1) printf("Npolygons = %e\n", Np[i]);
        printf("\n");
    }
    printf("FILENAME : %s\n", fname);
    if (write_output(&c, fname, num, th, kv, B, Np) != 0) {
        fprintf(stderr, "ps_run: cannot write %s\n", fname);
        exit(EXIT_FAILURE);
    }
    if (exact && write_exact(&c, fname, num, th, kv, cfgs, B, Np) != 0) {
        fprintf(stderr, "ps_run: cannot write %s.exact\n", fname);
        exit(EXIT_FAILURE);
    }
    ps_gpu_finalize(ctx);
    free(fname);
    free(cfgs);
    free(kv);
    free(th);
    free(B);
    free(Np);
    free(kap);
    printf("Execution took %f s\n", (double)time(NULL) - t1);
    return 0;
}
