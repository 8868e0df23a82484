/*
 * ps_create_ini: writes a run's ini file from positional arguments, for
 * scripts that generate many runs (the reference's create_iniFile tool,
 * create_iniFile/src/main.c and main_withOptionPhase.c).  The file it writes
 * is what ps_run (and the reference executable) read.
 *
 *   ps_create_ini FILE gridsize boxsize gasDP ionDP densityFile ionFile
 *                 hubble_h omega_b omega_m omega_l sigma8 Y whichField
 *                 [useOnlyPhase] n equilateral k1 k2 numValues theta kbinwidth
 *                 kbinningCase cosThetaBinwidth output_dir output_basename
 *                 write_numpolygons
 *
 * 26 arguments: the layout of create_iniFile/src/main.c (no useOnlyPhase line);
 * 27 arguments: the layout of main_withOptionPhase.c (useOnlyPhase after
 * whichField).  Kept alike on purpose: argument order, the ini keys and their
 * order, the section names, the comments after values, and the number
 * formatting (reals parsed with atof into single precision, printed "%f"; the
 * reference stores them in float variables).  Any other argument count prints
 * the usage and exits with status 1 (the reference then writes through an
 * uninitialised file name).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static void usage(void)
{
    fprintf(stderr,
            "usage: ps_create_ini FILE gridsize boxsize gasInputsInDoublePrecision ionInputsInDoublePrecision\n"
            "       densityFile ionFile hubble_h omega_b omega_m omega_l sigma8 Y whichField [useOnlyPhase]\n"
            "       n equilateral k1 k2 numValues theta kbinwidth kbinningCase cosThetaBinwidth\n"
            "       output_dir output_basename write_numpolygons\n");
}

int main(int argc, char** argv)
{
    if (argc != 27 && argc != 28) {
        usage();
        return 1;
    }
    const int phase = argc == 28; /* useOnlyPhase given */
    int a = 1;
    const char* filename = argv[a++];
    const int gridsize = atoi(argv[a++]);
    const float boxsize = (float)atof(argv[a++]);
    const int gas_dp = atoi(argv[a++]);
    const int ion_dp = atoi(argv[a++]);
    const char* density_file = argv[a++];
    const char* ion_file = argv[a++];
    float cosmo[6]; /* hubble_h, omega_b, omega_m, omega_l, sigma8, Y */
    for (int q = 0; q < 6; q++) cosmo[q] = (float)atof(argv[a++]);
    const char* which_field = argv[a++];
    const int use_only_phase = phase ? atoi(argv[a++]) : 0;
    const int n = atoi(argv[a++]);
    const int equilateral = atoi(argv[a++]);
    const float k1 = (float)atof(argv[a++]);
    const float k2 = (float)atof(argv[a++]);
    const int num_values = atoi(argv[a++]);
    const float theta = (float)atof(argv[a++]);
    const float kbinwidth = (float)atof(argv[a++]);
    const char* kbinning_case = argv[a++];
    const float dcos_theta = (float)atof(argv[a++]);
    const char* output_dir = argv[a++];
    const char* output_basename = argv[a++];
    const int write_numpolygons = atoi(argv[a++]);

    FILE* f = fopen(filename, "wt");
    if (!f) {
        perror(filename);
        return 1;
    }
    static const char* const cosmo_keys[6] = {"hubble_h", "omega_b", "omega_m", "omega_l", "sigma8", "Y"};
    fprintf(f, "[Grid]\n");
    fprintf(f, "gridsize = %d\n", gridsize);
    fprintf(f, "boxsize = %f\t# in h^-1 Mpc\n", boxsize);
    fprintf(f, "gasInputsInDoublePrecision = %d\n", gas_dp);
    fprintf(f, "ionInputsInDoublePrecision = %d\n", ion_dp);
    fprintf(f, "densityFile = %s\n", density_file);
    fprintf(f, "ionFile = %s\n", ion_file);
    fprintf(f, "\n[Cosmology]\n");
    for (int q = 0; q < 6; q++) fprintf(f, "%s = %f\n", cosmo_keys[q], cosmo[q]);
    fprintf(f, "\n[Polyspectrum]\n");
    fprintf(f, "whichField = %s\n", which_field);
    fprintf(f, "# Possibilities: DENS, XHII, XHI_DENS\n");
    if (phase) fprintf(f, "useOnlyPhase = %d\n", use_only_phase);
    fprintf(f, "n = %d\n", n);
    fprintf(f, "equilateral = %d\n", equilateral);
    fprintf(f, "k1 = %f\t# in h Mpc^-1\n", k1);
    fprintf(f, "k2 = %f\t# in h Mpc^-1\n", k2);
    fprintf(f, "numValues = %d\n", num_values);
    fprintf(f, "theta = %f\n", theta);
    fprintf(f, "kbinwidth = %f\n", kbinwidth);
    fprintf(f, "kbinningCase = %s\n", kbinning_case);
    fprintf(f, "cosThetaBinwidth = %f\n", dcos_theta);
    fprintf(f, "\n[Output]\n");
    fprintf(f, "output_dir = %s\n", output_dir);
    fprintf(f, "output_basename = %s\n", output_basename);
    fprintf(f, "write_numpolygons = %d\n", write_numpolygons);
    if (fclose(f) != 0) {
        perror(filename);
        return 1;
    }
    return 0;
}
