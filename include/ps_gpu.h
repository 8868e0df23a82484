/*
 * ps_gpu.h - C-ABI of the B200 polyspectrum estimator (libpsgpu.so).
 *
 * Drop-in boundary for annehutter/polyspectrum's FFT estimator: the calls in
 * src/run.c that
 *   - build the transformed field     get_FT_field()            input_field.c:40  (run.c:47)
 *   - normalise it to phases          calc_phase_3D_fftw_array() utils_fftw.c:78 (run.c:48-49)
 *   - evaluate one configuration      polyspectrum()            polyspectrum.c:51 (run.c:87)
 *   - count its polygons              num_polygons()            polyspectrum.c:163 (run.c:91)
 *   - generate the k-configurations   read_params_to_kvectors() kvectors.c:46 + run.c:56-84
 * are replaced by the entry points below.  Host code stays C; every argument
 * is a plain pointer or scalar.  All functions return PS_OK (0) or a negative
 * PS_ERR_* status and never exit the process.
 *
 * Conventions
 *   - The context owns all device memory; host arrays stay owned by the caller
 *     and are read/written before the call returns.
 *   - One context per host thread; each context runs on its own CUDA stream.
 *   - Grids are N^3, row-major [i][j][l] as in the reference (filter.c:59),
 *     N a power of two in [16, 1024] or one of 48, 60, 96, 192, 300, 320, 384,
 *     600 (2^a 3^b 5^c; other sizes are refused with PS_ERR_UNSUPPORTED).
 *   - Transforms follow FFTW's unnormalised convention (fft.c:17).
 */
#ifndef PS_GPU_H
#define PS_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
#define PS_OK 0
#define PS_ERR_ARG (-1)          /* invalid argument                          */
#define PS_ERR_OOM (-2)          /* device or host allocation failed          */
#define PS_ERR_IO (-3)           /* file could not be read (short read)       */
#define PS_ERR_CUDA (-4)         /* CUDA runtime / kernel error               */
#define PS_ERR_TIMEOUT (-5)      /* a bounded device wait expired             */
#define PS_ERR_NONFINITE (-6)    /* non-finite input where finite is required */
#define PS_ERR_UNSUPPORTED (-7)  /* valid for the reference, not implemented  */
#define PS_ERR_UNDEFINED (-8)    /* the reference's behaviour is undefined    */

/* ---- estimator methods ----------------------------------------------------- */
/* PS_FP64_PLAIN: the reference dataflow in FP64, one configuration at a time:
 *   per leg one inverse transform of F*dk and one of F (polyspectrum.c:72-133),
 *   running products, grid sums, reference normalisation (polyspectrum.c:155).
 * PS_FP32_BATCHED: all configurations of a call planned together: shells are
 *   deduplicated, shared leg pairs are transformed once, closing legs of a
 *   shared pair are folded by Parseval's identity into one k-space pass, field
 *   transforms run in FP32 with FP64 accumulation, polygon counts are exact
 *   integers (counted by enumeration of leg pairs, or by FP64 transforms
 *   rounded per mode, see PS_PLAN_FFT_COUNTS). */
#define PS_FP64_PLAIN 1
#define PS_FP32_BATCHED 2

/* ---- field selection (input_field.c:40-81, confObj whichField) ------------- */
#define PS_FIELD_DENS 0     /* densityFile                                  */
#define PS_FIELD_XHII 1     /* ionFile                                      */
#define PS_FIELD_XHI_DENS 2 /* dens*(1 - xHII), input_field.c:22-37         */

/* ---- kbinningCase (confObj.c:98-105) ---------------------------------------- */
#define PS_BIN_DEFAULT 0
#define PS_BIN_DERIVED 1
#define PS_BIN_GIVEN 2
#define PS_BIN_WATKINSON 3

/* ---- where an input pointer lives ------------------------------------------ */
#define PS_MEM_HOST 0
#define PS_MEM_DEVICE 1

#define PS_MAX_LEGS 8

typedef struct ps_gpu_ctx ps_gpu_ctx;

/* One configuration: the arguments of polyspectrum() (polyspectrum.h:7) minus
 * the grid.  kmin/kmax are in/out exactly as there: DERIVED binning writes the
 * derived ranges of every leg back (polyspectrum.c:83, :89-93). */
typedef struct {
    int n;                      /* number of legs, 2..PS_MAX_LEGS            */
    int kbinningCase;           /* PS_BIN_*                                  */
    double kbinwidth;           /* in units of the fundamental mode          */
    double k[PS_MAX_LEGS];      /* leg lengths [h/Mpc]                       */
    double kmin[PS_MAX_LEGS];   /* in/out                                    */
    double kmax[PS_MAX_LEGS];   /* in/out                                    */
} ps_cfg;

/* Parameters of a run, the confObj keys that shape the configuration list
 * (confObj.h:24-58). */
typedef struct {
    int grid_size;
    double box_size;            /* as read from the ini file (double)        */
    int n;
    int equilateral;
    double k1, k2;
    int num_values;
    double theta;
    double kbinwidth;
    int kbinningCase;
    double dcosTheta;
} ps_run_params;

/* Create a context for an N^3 grid.  boxsize is the reference's grid box size
 * (grid.h:9 stores it as float: pass (double)(float)L).  methods is a mask of
 * PS_FP64_PLAIN | PS_FP32_BATCHED; the field spectra those methods need are
 * computed by ps_gpu_set_field.  device < 0 keeps the current device. */
int ps_gpu_create(ps_gpu_ctx **ctx, int nbins, double boxsize, int methods, int device);

/* Load a field and run the forward transform (+ optional phase normalisation):
 * replaces get_FT_field (input_field.c:40-81) and calc_phase_3D_fftw_array
 * (utils_fftw.c:78-93, run.c:48-49).  which selects the field as whichField
 * does; dens / xhii are N^3 float (is_double = 0) or double (is_double = 1)
 * arrays in host (PS_MEM_HOST) or device (PS_MEM_DEVICE) memory; the one a
 * field does not use may be NULL.  use_only_phase == 1 normalises every mode
 * to unit modulus; a zero mode becomes NaN as in the reference. */
int ps_gpu_set_field(ps_gpu_ctx *ctx, int which, const void *dens, const void *xhii,
                     int is_double, int mem, int use_only_phase);

/* ps_gpu_set_field reading the raw input grids from files, as read_grid does
 * (grid.c:122-228: N^3 float or double values in native byte order, the
 * gasInputsInDoublePrecision / ionInputsInDoublePrecision of the ini file):
 * each file streams through two 64 MiB page-locked buffers, the read of one
 * chunk overlapping the upload of the other, so no host copy of the grid is
 * made.  The path a field does not use may be NULL.  A float file beside a
 * double one is widened (exactly) on the device, as the reference's double
 * field holds it.  A missing or short file gives PS_ERR_IO. */
int ps_gpu_set_field_files(ps_gpu_ctx *ctx, int which, const char *dens_path, int dens_double,
                           const char *xhii_path, int xhii_double, int use_only_phase);

/* ps_gpu_create + ps_gpu_set_field for a single field (DENS slot). */
int ps_gpu_init(ps_gpu_ctx **ctx, int nbins, double boxsize, const void *field,
                int field_is_double, int use_only_phase, int methods);

/* One configuration with the context's first method: polyspectrum()
 * (polyspectrum.c:51-161) and num_polygons() (polyspectrum.c:163-252) in one
 * call.  B = V^(n-1) N^(-3n) Re sum prod D / Re sum prod I with V the cube of
 * the context's box size; Npoly = Re sum prod I / N^3. */
int ps_gpu_polyspectrum(ps_gpu_ctx *ctx, int n, const double *k, double *kmin, double *kmax,
                        double kbinwidth, int kbinningCase, double *B, double *Npoly);

/* nconf configurations with an explicit method (PS_FP64_PLAIN evaluates them
 * one by one; PS_FP32_BATCHED plans them together).  kappa_or_NULL receives a
 * condition number per configuration: sum |terms| / |sum terms| of the final
 * FP64 sum the method evaluates (grid sum or Parseval k-space sum). */
int ps_gpu_polyspectrum_batch(ps_gpu_ctx *ctx, int method, int nconf, ps_cfg *cfgs, double *B,
                              double *Npoly, double *kappa_or_NULL);

/* A batch prepared once and executed many times (for example once per field
 * of a simulation series).  Planning does all host work: legs are resolved to
 * shells and deduplicated, configurations are grouped, tables are uploaded and
 * scratch is sized; DERIVED k ranges and closing-leg shells are finished on the
 * device during execution.  Execution is stream work only, so with
 * PS_PLAN_GRAPH the first execution captures it into a CUDA graph that later
 * executions replay.  A plan belongs to the context it was created on and
 * uses the field most recently loaded into it.  PS_PLAN_KAPPA adds the
 * condition-number passes.  PS_FP64_PLAIN plans evaluate their configurations
 * one by one (no graph). */
#define PS_PLAN_GRAPH 1
#define PS_PLAN_KAPPA 2
/* PS_PLAN_AUTOTUNE: each pair group (configurations sharing two legs) runs its
 * transforms on an alias-free sub-grid; by default the smallest one, with this
 * flag the fastest of the smallest and up to two larger supported sizes, timed
 * at plan creation; the flag also times, per FP32 transform size the groups
 * use, the Y pass with its default thread layout against one with twice the
 * elements per thread (one radix pass fewer) and keeps the faster, and the
 * pair kernel (the per-row product of two inverse transforms, transformed
 * forward again) in its default layout, with one row transform live in
 * registers, and with twice the elements per thread, keeping the fastest,
 * and the 16-shell dot pass in its default geometry against twice the
 * elements per thread (timed on the group's whole field part).
 * Counts are identical either way; sums differ only by FP32 rounding.  Choices are
 * kept per context and can be exported / imported (ps_gpu_tune_export /
 * ps_gpu_tune_import) so later runs use the same sizes and layouts. */
#define PS_PLAN_AUTOTUNE 4
/* Polygon counts of a pair group whose shells are all r^2 intervals (DEFAULT,
 * GIVEN and DERIVED binning) are counted exactly in integers by default:
 * every leg pair (m_a, m_b), S_a reduced to orbit representatives under the
 * 48 axis permutations and sign flips, histogrammed by |m_a + m_b|^2 (wrapped
 * on the grid as the reference's cyclic sums wrap).  PS_PLAN_FFT_COUNTS
 * counts with FP64 transforms of the unit shells instead (the reference's
 * dataflow; WATKINSON shells always do).  Both give the same integers. */
#define PS_PLAN_FFT_COUNTS 8
typedef struct ps_gpu_plan ps_gpu_plan;
int ps_gpu_plan_create(ps_gpu_ctx *ctx, int method, int nconf, const ps_cfg *cfgs, int flags,
                       ps_gpu_plan **plan);
/* B, Npoly (and kappa when the plan has PS_PLAN_KAPPA) per configuration;
 * cfgs_out_or_NULL receives the configurations with DERIVED ranges written
 * back, as ps_gpu_polyspectrum_batch writes them. */
int ps_gpu_plan_execute(ps_gpu_ctx *ctx, ps_gpu_plan *plan, double *B, double *Npoly,
                        double *kappa_or_NULL, ps_cfg *cfgs_out_or_NULL);
/* Frees the plan (waits for its submissions).  Destroy plans before their
 * context; a plan that outlives its context holds no device memory and can
 * only be destroyed. */
void ps_gpu_plan_destroy(ps_gpu_plan *plan);

/* Asynchronous pipeline over a series of fields (no reference counterpart:
 * the reference runs one process per field).  ps_gpu_set_field_async is
 * ps_gpu_set_field without waiting: host arrays are copied on the context's
 * copy stream into one of two device staging slots, and the forward transform
 * is queued on the compute stream behind that copy.  ps_gpu_plan_submit queues
 * a PS_FP32_BATCHED plan execution behind it and the copy of its results to
 * a page-locked buffer of its own; they are unpacked into B, Npoly (and kappa,
 * cfgs_out) by the first later call on the context (ps_gpu_set_field_async,
 * ps_gpu_plan_submit, ps_gpu_synchronize) that finds the copy done, at the
 * latest by ps_gpu_synchronize; no host callback holds the streams.  So the
 * upload of field k+1 overlaps the configurations of field k.  Every pointer passed to
 * these two calls (inputs and outputs) must stay valid and the inputs
 * unchanged until ps_gpu_synchronize returns; host inputs overlap only when
 * they are page-locked (cudaHostAlloc / cudaHostRegister).  Errors detected on
 * the device during a submission are returned by ps_gpu_synchronize. */
int ps_gpu_set_field_async(ps_gpu_ctx *ctx, int which, const void *dens, const void *xhii,
                           int is_double, int mem, int use_only_phase);
/* Host XHI_DENS float inputs of a context created with PS_FP32_BATCHED alone
 * (ps_gpu_set_field and ps_gpu_set_field_async): host threads compose
 * dens*(1 - xHII), as input_field.c:33 computes it, for part of the rows into
 * a library-owned page-locked buffer, uploaded chunk by chunk at half the
 * PCIe bytes, while the other rows go up as they are (from page-locked
 * inputs only; pageable inputs are composed in full).  The split follows the
 * measured compose and copy rates.  Results are bit-identical to the
 * two-array upload.  ps_gpu_upload_bytes gives the host -> device bytes of
 * the last host field load (no reference counterpart). */
long long ps_gpu_upload_bytes(const ps_gpu_ctx *ctx);
/* Statistics of the last host field load: rows (N^2) and rows sent as they
 * are (rows_raw; the others were composed on host threads), host seconds
 * spent composing, device milliseconds of the raw rows' copies, the raw
 * fraction the next load will use, the host threads of the composition
 * ($PS_HOST_THREADS, default: the CPUs this process may run on less one; one
 * pool per process) and the host -> device bytes.  Zeros for loads that
 * compose nothing (device inputs, other fields).  No reference counterpart. */
typedef struct {
    long long rows, rows_raw, bytes;
    double compose_s, raw_copy_ms, next_raw_frac;
    int host_threads;
} ps_load_stats;
int ps_gpu_load_stats(const ps_gpu_ctx *ctx, ps_load_stats *out);
int ps_gpu_plan_submit(ps_gpu_ctx *ctx, ps_gpu_plan *plan, double *B, double *Npoly,
                       double *kappa_or_NULL, ps_cfg *cfgs_out_or_NULL);
int ps_gpu_synchronize(ps_gpu_ctx *ctx);

/* A PS_FP32_BATCHED plan execution queued on the context's stream with its
 * results left on the device (no copy, no host callback); ps_gpu_plan_results
 * waits for the stream and returns the results of the plan's latest
 * execution, as ps_gpu_plan_execute does.  For loops whose per-field results
 * are not needed on the host every time.  No reference counterpart. */
int ps_gpu_plan_launch(ps_gpu_ctx *ctx, ps_gpu_plan *plan);
/* Queues the parts of a PS_FP32_BATCHED plan's next execution that read no
 * field (the DERIVED k-ranges, the closing shells' tables and the exact
 * polygon counts) on the context's side stream, after the work already on
 * its stream.  The plan's next ps_gpu_plan_execute / _submit / _launch then
 * runs only the field parts on the stream, waiting for the prepared parts
 * where it reads them.  A field load queued between the two
 * (ps_gpu_set_field / _async) overlaps the prepared parts.  Every execution
 * still computes all of its results; a prepared execution's results are
 * identical to an unprepared one's.  No-op while per-kernel profiling is on,
 * or when already prepared.  No reference counterpart (run.c:98-120 loads
 * the field, then evaluates the configurations one after another). */
int ps_gpu_plan_prepare(ps_gpu_ctx *ctx, ps_gpu_plan *plan);
int ps_gpu_plan_results(ps_gpu_ctx *ctx, ps_gpu_plan *plan, double *B, double *Npoly,
                        double *kappa_or_NULL, ps_cfg *cfgs_out_or_NULL);
/* Queues, on the context's stream, a copy of the latest execution's results
 * into device memory dst (8 * nconf doubles): B and Npoly interleaved per
 * configuration (2 * nconf), then the DERIVED k-ranges, six per configuration
 * (kmin, kmax of legs 0, 1, 2; zeros for other binnings).  No wait: for an
 * exchange that stays on the device (an all-gather over ranks, the
 * counterpart of the reference's MPI reduction, polyspectrum.c:144-153). */
int ps_gpu_plan_results_device(ps_gpu_ctx *ctx, ps_gpu_plan *plan, double *dst);

/* The context's autotuned choices as text, one "grid N b_a b_b b_c M" line per
 * pair-group signature, one "pencil M alt" line (alt 0 or 1) per transform
 * size whose Y pass layout was timed and one "pair M v" line per FP32
 * transform size whose pair kernel variant was timed (v 0: the default, 1: one
 * row transform live in registers, 2: twice the elements per thread, one
 * radix pass fewer) and one "dot M alt" line per FP32 transform size whose
 * dot pass geometry was timed (alt 1: twice the elements per thread): writes
 * at most buflen bytes (NUL-terminated) and
 * returns the length of the whole text, or a negative status.  Import adds
 * the lines of such a text to the context's choices (unknown or malformed
 * lines: PS_ERR_ARG, nothing imported).  No reference counterpart. */
int ps_gpu_tune_export(ps_gpu_ctx *ctx, char *buf, int buflen);
int ps_gpu_tune_import(ps_gpu_ctx *ctx, const char *text);

/* Kernels the context has executed since its creation (a graph replay counts
 * the kernels in the graph); -1 for a NULL context. */
long long ps_gpu_launch_count(ps_gpu_ctx *ctx);

/* Gradient dB/d(delta) of one configuration with respect to the real input
 * field (the array the forward transform read), written to out as N^3 float
 * (out_is_double = 0) or double (1) in host or device memory (out_mem).  No
 * reference counterpart.  For a phase-only field (use_only_phase = 1) the
 * gradient goes through z/|z| and needs the modulus kept at loading
 * (ps_gpu_keep_modulus); without it PS_ERR_UNSUPPORTED.  The normalisation
 * needs the configuration's polygon count: when an earlier
 * ps_gpu_polyspectrum(_batch) call on this context evaluated the same
 * configuration with the same method, its count is reused (counts depend on
 * the shells only), else the call evaluates the configuration first. */
int ps_gpu_grad(ps_gpu_ctx *ctx, int method, int n, const double *k, const double *kmin,
                const double *kmax, double kbinwidth, int kbinningCase, void *out,
                int out_is_double, int out_mem);

/* Band-limited field spectrum: later loads (ps_gpu_set_field*) compute only
 * the modes whose three |components| are at most `band` (band < 0 or >= N/2:
 * all modes, the default).  Modes outside are left undefined, and every
 * computation that would read one returns PS_ERR_ARG, so results are the same
 * as with the full spectrum.  A plan's band (ps_gpu_plan_band: the largest
 * |component| of a mode any of its shells holds) is the narrowest band that
 * serves it.  No reference counterpart (the reference transforms all modes). */
int ps_gpu_set_spectrum_band(ps_gpu_ctx *ctx, int band);
int ps_gpu_plan_band(const ps_gpu_plan *plan);

/* With on != 0, later phase-only loads (use_only_phase = 1) also keep |X| per
 * mode of the field spectrum (one more real half-spectrum on the device), which
 * ps_gpu_grad needs to differentiate through z/|z| (utils_fftw.c:78-93).  No
 * reference counterpart. */
int ps_gpu_keep_modulus(ps_gpu_ctx *ctx, int on);

/* The configuration list of a run: read_params_to_kvectors (kvectors.c:46-147)
 * plus the per-configuration kpolygon bookkeeping of run.c:56-84.  Writes at
 * most max_cfg entries to cfgs (and the sweep values to k_out / theta_out,
 * NaN where the run has no theta; either may be NULL) and returns the number
 * of configurations, or a negative status (n < 2 or n > 3 are refused as
 * kvectors.c:60-64, :140-144 refuse them). */
int ps_make_configs(const ps_run_params *p, ps_cfg *cfgs, int max_cfg, double *k_out,
                    double *theta_out);

/* Use a caller-provided CUDA stream (cudaStream_t passed as void*); NULL
 * returns to the context's own stream. */
int ps_gpu_set_stream(ps_gpu_ctx *ctx, void *stream);

/* Device timing of the last ps_gpu_* compute call on the context, in ms
 * (CUDA events on the context's stream), and the number of kernels it launched. */
int ps_gpu_last_timing(ps_gpu_ctx *ctx, double *ms, long long *kernel_launches);

/* Per-kernel device timing.  When profiling is on, every kernel the context
 * launches is bracketed by CUDA events on the context's stream and charged,
 * with its algorithmic HBM bytes (the bytes its pass must read and write at
 * minimum), to its kernel family (FP64 instances of the transform kernels
 * as "<family>_f64"), one entry per transform size ("<family>@<size>").
 * ps_gpu_kernel_stats synchronises and
 * returns up to max families; the counters reset when profiling is switched
 * on.  No reference counterpart (the reference has only a total wall time,
 * main.c:38-82). */
typedef struct {
    char name[32];        /* kernel family                                  */
    long long launches;
    double ms;            /* summed device time                             */
    double bytes;         /* summed algorithmic bytes                       */
} ps_kernel_stat;
int ps_gpu_set_profiling(ps_gpu_ctx *ctx, int on);
int ps_gpu_kernel_stats(ps_gpu_ctx *ctx, ps_kernel_stat *out, int max);

/* Power spectrum P(k) (n = 2, DEFAULT binning, one shell per k) of a field
 * that is already in device memory, without allocating anything: for host
 * programs whose GPU memory belongs to another allocator (a framework's
 * caching pool that has reserved the device, a fixed real-time memory budget),
 * where a library may not call cudaMalloc of its own.  No counterpart in the
 * reference.  field_dev: N^3 float32 on the current device; N must be 16, 32
 * or 64, nshell 1..256, box size and kbinwidth positive and finite,
 * use_only_phase 0 or 1; anything else is rejected with PS_ERR_ARG.
 * Results equal those of ps_gpu_polyspectrum_batch (PS_FP32_BATCHED) on the
 * configurations {n=2, k = {k[s], k[s]}}: P[s] = B, Npoly[s] = exact count.
 * Its working memory is one fixed 8 MiB device array that every GPU loading
 * the library holds until exit; all calls on a device share it, so calls that
 * overlap on the GPU race.  The call reads its results back into P and Npoly
 * and synchronises `stream` (NULL: the legacy default stream) before it
 * returns.  The first call on a device resolves the array's address
 * (cudaGetSymbolAddress) and should come before any stream capture. */
int ps_gpu_power_spectrum_noalloc(int nbins, double boxsize, const float *field_dev,
                                  int use_only_phase, int nshell, const double *k,
                                  double kbinwidth, double *P, double *Npoly, void *stream);

/* Host-side fault injection for tests of the error paths (no reference
 * counterpart; the reference exit()s on these failures, grid.c:24,133,
 * utils.c:96).  spec "alloc:N", "read:N" or "launch:N" (comma-separated to arm
 * several): the Nth device or page-locked allocation, input-file read or
 * post-launch status check after this call fails once, with the status a
 * real failure returns (PS_ERR_OOM, PS_ERR_IO, PS_ERR_CUDA); "wait:N": the Nth
 * field transform staged by bulk copies waits on a barrier that cannot
 * complete, so its bounded wait (0.2 s) runs out and the load returns
 * PS_ERR_TIMEOUT.  No GPU fault is caused.  NULL or "" disarms.  $PS_FAULT arms the same way at the process's
 * first ps_gpu_create.  Malformed spec: PS_ERR_ARG. */
int ps_gpu_debug_fault(const char *spec);

void ps_gpu_finalize(ps_gpu_ctx *ctx);
const char *ps_gpu_strerror(int status);
/* Text of the last error on the calling thread (empty if none). */
const char *ps_gpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PS_GPU_H */
