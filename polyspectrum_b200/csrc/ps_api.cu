// libpsgpu: C-ABI, context, launch plumbing and the two estimator methods.
#include <math.h>
#include <sched.h>
#include <stdarg.h>

#include <cmath>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <atomic>
#include <functional>
#include <map>
#include <set>
#include <string>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/ps_gpu.h"
#include "ps_launch.cuh"
#include "ps_counts.cuh"

namespace ps {
PS_EXTERN_L3(float)
PS_EXTERN_L3(double)
}  // namespace ps

using namespace ps;

// =========================================================================
// errors
// =========================================================================
namespace {
thread_local char g_err[512] = {0};

int fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}
// Host-side fault injection, for tests of the error paths (no GPU fault is
// ever caused): once armed with "alloc:N", "read:N" or "launch:N" (a comma
// separated list arms several), the Nth device or page-locked allocation,
// input-file read or post-launch status check after arming fails once, with
// the status the real failure returns (PS_ERR_OOM, PS_ERR_IO, PS_ERR_CUDA);
// "wait:N" makes the Nth bulk-staged field transform's mbarrier expect 16
// bytes more than its copies bring, so its bounded wait runs out and the load
// returns PS_ERR_TIMEOUT (the copies themselves complete).
// Armed by ps_gpu_debug_fault, or by $PS_FAULT at the first ps_gpu_create.
enum FaultKind { FAULT_ALLOC = 0, FAULT_READ = 1, FAULT_LAUNCH = 2, FAULT_WAIT = 3, FAULT_KINDS = 4 };
std::atomic<long long> g_fault_at[FAULT_KINDS];
std::atomic<long long> g_fault_seen[FAULT_KINDS];

bool fault_hit(int kind)
{
    const long long at = g_fault_at[kind].load();
    if (at <= 0) return false;
    if (++g_fault_seen[kind] != at) return false;
    g_fault_at[kind] = 0;  // one shot
    return true;
}

int arm_faults(const char* spec)
{
    long long at[FAULT_KINDS] = {0, 0, 0, 0};
    static const char* names[FAULT_KINDS] = {"alloc", "read", "launch", "wait"};
    if (spec && *spec) {
        std::string txt(spec);
        size_t pos = 0;
        while (pos <= txt.size()) {
            size_t end = txt.find(',', pos);
            if (end == std::string::npos) end = txt.size();
            const std::string item = txt.substr(pos, end - pos);
            const size_t colon = item.find(':');
            int kind = -1;
            for (int q = 0; q < FAULT_KINDS && colon != std::string::npos; q++)
                if (item.compare(0, colon, names[q]) == 0 && colon == strlen(names[q])) kind = q;
            char* tail = nullptr;
            const long long n = kind >= 0 ? strtoll(item.c_str() + colon + 1, &tail, 10) : 0;
            if (kind < 0 || n <= 0 || !tail || *tail) return fail(PS_ERR_ARG, "fault spec '%s': want alloc:N, read:N, "
                                                                               "launch:N or wait:N, N >= 1", item.c_str());
            at[kind] = n;
            pos = end + 1;
        }
    }
    for (int q = 0; q < FAULT_KINDS; q++) {
        g_fault_seen[q] = 0;
        g_fault_at[q] = at[q];
    }
    return PS_OK;
}

// cudaGetLastError after launches, or the injected launch failure.
cudaError_t launch_status()
{
    if (fault_hit(FAULT_LAUNCH)) {
        cudaGetLastError();
        return cudaErrorLaunchFailure;
    }
    return cudaGetLastError();
}
}  // namespace

#define PS_CK(x)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (x);                                                                \
        if (e_ != cudaSuccess)                                                               \
            return fail(e_ == cudaErrorMemoryAllocation ? PS_ERR_OOM : PS_ERR_CUDA,          \
                        "%s: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__, __LINE__);  \
    } while (0)
#define PS_TRY(x)               \
    do {                        \
        int rc_ = (x);          \
        if (rc_ != PS_OK) return rc_; \
    } while (0)

#define PS_SWITCH_N(N, BODY)                       \
    switch (N) {                                   \
    case 16: { constexpr int NN = 16; BODY; } break;   \
    case 32: { constexpr int NN = 32; BODY; } break;   \
    case 64: { constexpr int NN = 64; BODY; } break;   \
    case 128: { constexpr int NN = 128; BODY; } break; \
    case 192: { constexpr int NN = 192; BODY; } break; \
    case 256: { constexpr int NN = 256; BODY; } break; \
    case 320: { constexpr int NN = 320; BODY; } break; \
    case 384: { constexpr int NN = 384; BODY; } break; \
    case 512: { constexpr int NN = 512; BODY; } break; \
    case 1024: { constexpr int NN = 1024; BODY; } break; \
    case 48: { constexpr int NN = 48; BODY; } break;   \
    case 60: { constexpr int NN = 60; BODY; } break;   \
    case 96: { constexpr int NN = 96; BODY; } break;   \
    case 300: { constexpr int NN = 300; BODY; } break; \
    case 600: { constexpr int NN = 600; BODY; } break; \
    default: return fail(PS_ERR_UNSUPPORTED, "grid size %d not supported", N); \
    }

// =========================================================================
// context
// =========================================================================
template <typename T> struct PrecBufs {
    V2<T>* tw = nullptr;    // W_N^m, m in [0, N): r2c / c2r pre- and post-processing
    V2<T>* twp = nullptr;   // Stockham table of the pencil transforms (length N)
    V2<T>* twr = nullptr;   // Stockham table of the row transforms (length N/2)
    V2<T>* twp_alt = nullptr;  // table of the alternative Y pass (PencilAlt), if N has one
    V2<T>* twr_alt = nullptr;  // row table of pair kernel variant 2 (PairVariants::ALT_RX), if N has one
    Tables<T> tables() const { return Tables<T>{twp, twr, tw, twp_alt, twr_alt}; }
    V2<T>* spec = nullptr;  // field spectrum, row stride S
    V2<T>* work = nullptr;  // work spectrum (band-limited strides <= S)
    V2<T>* work2 = nullptr; // second and third work spectra (pair groups; allocated on use)
    V2<T>* work3 = nullptr;
    V2<T>* hacc = nullptr;  // adjoint spectrum accumulator (allocated on use)
    T* ra = nullptr;        // real grids
    T* rb = nullptr;
    T* mod = nullptr;       // |X| of a phase-only field (ps_gpu_keep_modulus)
    int S = 0;
    bool have_spec = false;
    bool have_mod = false;
    // tables of smaller transform sizes (sub-grid products), made at plan time
    std::map<int, std::array<V2<T>*, 5>> sub;
};

// Host worker threads of the composition, one pool per process shared by
// every context: $PS_HOST_THREADS threads, else one per CPU this process may
// run on less one (left to the CUDA driver's threads and the caller), at most
// 64.  run(f) calls f(t) on every worker t and returns when all are done; jobs
// of different contexts (host threads) take turns.
struct HostPool {
    std::vector<std::thread> th;
    std::mutex m, turn;
    std::condition_variable cv, done_cv;
    std::function<void(size_t)> job;
    size_t gen = 0, pending = 0, n = 1;
    bool stop = false;
    static size_t default_threads()
    {
        const char* e = getenv("PS_HOST_THREADS");
        if (e && atoi(e) > 0) return (size_t)std::min(atoi(e), 64);
        cpu_set_t set;
        CPU_ZERO(&set);
        const int ncpu = sched_getaffinity(0, sizeof(set), &set) == 0 ? CPU_COUNT(&set) : 1;
        return (size_t)std::max(1, std::min(ncpu - 1, 64));
    }
    HostPool()
    {
        n = default_threads();
        for (size_t t = 1; t < n; t++)
            th.emplace_back([this, t]() {
                size_t seen = 0;
                for (;;) {
                    std::unique_lock<std::mutex> lk(m);
                    cv.wait(lk, [&]() { return stop || gen != seen; });
                    if (stop) return;
                    seen = gen;
                    const std::function<void(size_t)> f = job;
                    lk.unlock();
                    f(t);
                    lk.lock();
                    if (--pending == 0) done_cv.notify_one();
                }
            });
    }
    void run(const std::function<void(size_t)>& f)
    {
        std::lock_guard<std::mutex> one_job(turn);
        {
            std::lock_guard<std::mutex> lk(m);
            job = f;
            pending = n - 1;
            ++gen;
        }
        cv.notify_all();
        f(0);
        std::unique_lock<std::mutex> lk(m);
        done_cv.wait(lk, [&]() { return pending == 0; });
    }
    ~HostPool()
    {
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
        }
        cv.notify_all();
        for (auto& t : th) t.join();
    }
    // the process's pool, started on first use (never destroyed: its threads
    // sleep on a condition variable until the process exits)
    static HostPool& get()
    {
        static HostPool* pool = new HostPool();
        return *pool;
    }
};

// A plan execution queued by ps_gpu_plan_submit whose results are still on
// their way: the copy into `host` (page-locked, this submission's own) ends
// with `done`; the next call on the context that finds the event complete
// unpacks them into the caller's arrays.
struct PendingSubmit {
    const ps_gpu_plan* P;
    double* host;
    size_t host_len;
    cudaEvent_t done;
    double *B, *Np, *kappa;
    ps_cfg* cfgs_out;
};

struct ps_gpu_ctx {
    int N = 0;
    double L = 0.0;  // (double)(float) box size, grid.h:9
    int methods = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    // side lane: the count (FP64) parts of pair groups run on their own stream
    // with their own partial sums and shell table, concurrently with the field
    // (FP32) parts; ev_fork / ev_join order it inside a launch sequence
    cudaStream_t side_stream = nullptr;
    double* side_partials = nullptr;
    size_t side_partials_cap = 0;
    unsigned short* side_lut = nullptr;
    size_t side_lut_cap = 0;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // second field lane: the pair groups of a plan split over two streams (the
    // main one and this), each with its own FP32 work spectra, partial sums and
    // shell table, so the kernels of different groups overlap
    cudaStream_t lane2_stream = nullptr;
    double* lane2_partials = nullptr;
    size_t lane2_partials_cap = 0;
    unsigned short* lane2_lut = nullptr;
    size_t lane2_lut_cap = 0;
    V2<float>* lane2_work[3] = {nullptr, nullptr, nullptr};
    size_t lane2_work_cap = 0;  // elements of each
    cudaEvent_t ev_join2 = nullptr;
    PrecBufs<float> f;
    PrecBufs<double> d;
    double* partials = nullptr;
    size_t partials_cap = 0;
    double* dsums = nullptr;  // device scalars
    size_t dsums_cap = 0;
    Shell* dshells = nullptr;
    size_t dshells_cap = 0;
    unsigned long long* dminmax = nullptr;
    size_t dminmax_cap = 0;
    unsigned short* dlut = nullptr;  // r2 -> shell bitmask
    size_t dlut_cap = 0;
    // scratch buffers replaced by larger ones stay allocated until finalize:
    // a captured plan graph may still point at them
    std::vector<void*> retired;
    // autotuned transform size per pair-group signature (N, b_a, b_b, b_c)
    std::map<std::array<int, 4>, int> tune_grid;
    // autotuned Y pass geometry per FP32 transform size: 1 = the alternative
    // (PencilAlt: twice the elements per thread), 0 = the default
    std::map<int, int> pencil_alt;
    // autotuned pair kernel variant per FP32 transform size (PairVariants:
    // 0 the default, 1 one live row transform, 2 twice the elements per thread)
    std::map<int, int> pair_var;
    // autotuned FP32 dot pass geometry per transform size: 1 = PencilAlt
    std::map<int, int> dot_alt;
    bool capturing = false;  // inside a plan graph capture: no profiling events
    // host uploads: two staging slots of (dens, xhii), filled on copy_stream;
    // ev_copied[s] = slot s filled, ev_free[s] = its forward transform is done
    void* stage[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    size_t stage_bytes = 0;
    int slot = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
    // file uploads (ps_gpu_set_field_files): two page-locked chunk buffers,
    // ev_chunk[q] = the copy out of chunk buffer q is done
    void* pin[2] = {nullptr, nullptr};
    cudaEvent_t ev_chunk[2] = {nullptr, nullptr};
    // XHI_DENS composed on the host (FP32-only contexts): two page-locked field
    // buffers, ev_fpin[q] = the upload out of buffer q is done
    void* fpin[2] = {nullptr, nullptr};
    size_t fpin_bytes = 0;
    int fslot = 0;
    cudaEvent_t ev_fpin[2] = {nullptr, nullptr};
    size_t upload_bytes = 0;  // host -> device bytes of the last host field load
    // split of a host XHI_DENS load between raw rows (PCIe) and composed rows
    // (host threads): the raw fraction and the measured seconds per row
    double raw_frac = 0.3, t_comp_row = 0.0, t_up_row = 0.0;
    // statistics of the last host XHI_DENS load (ps_gpu_load_stats)
    long long load_rows = 0, load_rows_raw = 0;
    double load_compose_s = 0.0, load_raw_copy_ms = 0.0;
    // asynchronous submissions not yet unpacked, oldest first, and spare
    // page-locked result buffers / events for the next ones
    std::vector<PendingSubmit> pending;
    std::vector<std::pair<double*, size_t>> spare_host;
    std::vector<cudaEvent_t> spare_events;
    // polygon counts of configurations evaluated on this context (field
    // independent), keyed by method and configuration: ps_gpu_grad reuses them
    std::map<std::string, double> npoly_cache;
    cudaEvent_t ev_raw[2] = {nullptr, nullptr};
    std::atomic<int> async_err{0};  // status of submissions unpacked after their call returned
    int* dstatus = nullptr;  // device word: 1 when a kernel's bounded wait expired (PS_ERR_TIMEOUT)
    std::set<ps_gpu_plan*> plans;   // live plans (finalize releases their device memory)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    long long launches = 0;
    long long launches_total = 0;  // kernels executed since creation (graph replays included)
    int use_only_phase = 0;
    bool keep_modulus = false;  // phase-only loads keep |X| (phase-only adjoint)
    // field spectrum band: loads compute only modes whose |components| are at
    // most spec_band (-1: all); loaded_band is that of the field loaded last
    int spec_band = -1;
    int loaded_band = 0;
    bool field_set = false;
    // per-kernel profiling (ps_gpu_set_profiling)
    struct ProfRec {
        int kind, size;
        cudaEvent_t a, b;
        double bytes;
    };
    struct ProfAgg {
        double ms = 0.0, bytes = 0.0;
        long long n = 0;
    };
    bool prof_on = false;
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::map<std::pair<int, int>, ProfAgg> prof_agg;  // (family, transform size)
};

namespace {

int round_up(int a, int b) { return (a + b - 1) / b * b; }
// Grid sizes a context runs on: powers of two 16..1024 and 48, 60, 96, 192,
// 300, 320, 384, 600 (2^a 3^b 5^c; the reference's FFTW takes any N).
bool grid_size_ok(int n)
{
    for (int q : {16, 32, 48, 60, 64, 96, 128, 192, 256, 300, 320, 384, 512, 600, 1024})
        if (q == n) return true;
    return false;
}
double ref_pi() { return acos(-1.0); }  // filter.c:19

// Pencil-tile width (complex elements per row segment) of the pencil kernels.
template <typename T> int pw(int N)
{
    switch (N) {
    case 16: return PencilGeom<T, 16>::W;
    case 32: return PencilGeom<T, 32>::W;
    case 64: return PencilGeom<T, 64>::W;
    case 128: return PencilGeom<T, 128>::W;
    case 192: return PencilGeom<T, 192>::W;
    case 256: return PencilGeom<T, 256>::W;
    case 320: return PencilGeom<T, 320>::W;
    case 384: return PencilGeom<T, 384>::W;
    case 512: return PencilGeom<T, 512>::W;
    case 48: return PencilGeom<T, 48>::W;
    case 60: return PencilGeom<T, 60>::W;
    case 96: return PencilGeom<T, 96>::W;
    case 300: return PencilGeom<T, 300>::W;
    case 600: return PencilGeom<T, 600>::W;
    default: return PencilGeom<T, 1024>::W;
    }
}

template <typename T> int alloc_dev(T** p, size_t count)
{
    if (*p) return PS_OK;
    if (fault_hit(FAULT_ALLOC)) return fail(PS_ERR_OOM, "cudaMalloc of %zu bytes: injected failure", sizeof(T) * count);
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(PS_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", sizeof(T) * count,
                    cudaGetErrorString(e));
    }
    return PS_OK;
}

template <typename T> int init_prec(ps_gpu_ctx* c, PrecBufs<T>& b)
{
    const int N = c->N;
    b.S = round_up(N / 2 + 1, pw<T>(N));
    const size_t nspec = (size_t)N * N * b.S;
    const size_t nreal = (size_t)N * N * N;
    PS_TRY(alloc_dev(&b.tw, N));
    PS_TRY(alloc_dev(&b.twp, N));
    PS_TRY(alloc_dev(&b.twr, N / 2));
    {
        std::vector<V2<T>> hp(N), hr(N / 2), ha(N);
        PS_SWITCH_N(N, (L3<T, NN>::host_tables(hp.data(), hr.data())));
        PS_CK(cudaMemcpy(b.twp, hp.data(), sizeof(V2<T>) * N, cudaMemcpyHostToDevice));
        PS_CK(cudaMemcpy(b.twr, hr.data(), sizeof(V2<T>) * (N / 2), cudaMemcpyHostToDevice));
        bool has_alt = false;
        PS_SWITCH_N(N, (has_alt = L3<T, NN>::host_alt_table(ha.data())));
        if (has_alt) {
            PS_TRY(alloc_dev(&b.twp_alt, N));
            PS_CK(cudaMemcpy(b.twp_alt, ha.data(), sizeof(V2<T>) * N, cudaMemcpyHostToDevice));
        }
        bool has_pair_alt = false;
        PS_SWITCH_N(N, (has_pair_alt = L3<T, NN>::host_pair_alt_table(hr.data())));
        if (has_pair_alt) {
            PS_TRY(alloc_dev(&b.twr_alt, N / 2));
            PS_CK(cudaMemcpy(b.twr_alt, hr.data(), sizeof(V2<T>) * (N / 2), cudaMemcpyHostToDevice));
        }
    }
    PS_TRY(alloc_dev(&b.spec, nspec));
    PS_TRY(alloc_dev(&b.work, nspec));
    PS_TRY(alloc_dev(&b.ra, nreal));
    PS_TRY(alloc_dev(&b.rb, nreal));
    std::vector<V2<T>> h(N);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < N; m++) {
        const long double a = two_pi * (long double)m / (long double)N;
        h[m].x = (T)cosl(a);
        h[m].y = (T)(-sinl(a));
    }
    PS_CK(cudaMemcpy(b.tw, h.data(), sizeof(V2<T>) * N, cudaMemcpyHostToDevice));
    return PS_OK;
}

template <typename T> PrecBufs<T>& bufs(ps_gpu_ctx* c);

// Twiddle tables of an M-point transform (M <= N): the context's own for M = N,
// else made once (allocation: plan time only, never during graph capture).
template <typename T> int tables_for(ps_gpu_ctx* c, int M, Tables<T>* out)
{
    PrecBufs<T>& b = bufs<T>(c);
    if (M == c->N) {
        *out = b.tables();
        return PS_OK;
    }
    auto it = b.sub.find(M);
    if (it == b.sub.end()) {
        if (c->capturing) return fail(PS_ERR_ARG, "internal: tables of size %d not made before capture", M);
        std::array<V2<T>*, 5> t = {nullptr, nullptr, nullptr, nullptr, nullptr};
        std::vector<V2<T>> hp(M), hr(M / 2), h(M), ha(M), hr2(M / 2);
        const int N = M;
        PS_SWITCH_N(N, (L3<T, NN>::host_tables(hp.data(), hr.data())));
        bool has_alt = false, has_pair_alt = false;
        PS_SWITCH_N(N, (has_alt = L3<T, NN>::host_alt_table(ha.data())));
        PS_SWITCH_N(N, (has_pair_alt = L3<T, NN>::host_pair_alt_table(hr2.data())));
        const long double two_pi = 6.283185307179586476925286766559005768L;
        for (int m = 0; m < M; m++) {
            const long double a = two_pi * (long double)m / (long double)M;
            h[m].x = (T)cosl(a);
            h[m].y = (T)(-sinl(a));
        }
        int rc = alloc_dev(&t[0], M);
        if (rc == PS_OK) rc = alloc_dev(&t[1], M / 2);
        if (rc == PS_OK) rc = alloc_dev(&t[2], M);
        if (rc == PS_OK && has_alt) rc = alloc_dev(&t[3], M);
        if (rc == PS_OK && has_pair_alt) rc = alloc_dev(&t[4], M / 2);
        if (rc != PS_OK) {
            for (V2<T>* p : t) cudaFree(p);
            return rc;
        }
        b.sub[M] = t;
        PS_CK(cudaMemcpy(t[0], hp.data(), sizeof(V2<T>) * M, cudaMemcpyHostToDevice));
        PS_CK(cudaMemcpy(t[1], hr.data(), sizeof(V2<T>) * (M / 2), cudaMemcpyHostToDevice));
        PS_CK(cudaMemcpy(t[2], h.data(), sizeof(V2<T>) * M, cudaMemcpyHostToDevice));
        if (has_alt) PS_CK(cudaMemcpy(t[3], ha.data(), sizeof(V2<T>) * M, cudaMemcpyHostToDevice));
        if (has_pair_alt) PS_CK(cudaMemcpy(t[4], hr2.data(), sizeof(V2<T>) * (M / 2), cudaMemcpyHostToDevice));
        it = b.sub.find(M);
    }
    *out = Tables<T>{it->second[0], it->second[1], it->second[2], it->second[3], it->second[4]};
    return PS_OK;
}

template <typename T> void free_prec(PrecBufs<T>& b)
{
    for (auto& kv : b.sub)
        for (V2<T>* p : kv.second) cudaFree(p);
    b.sub.clear();
    cudaFree(b.tw);
    cudaFree(b.twp);
    cudaFree(b.twr);
    cudaFree(b.twp_alt);
    cudaFree(b.twr_alt);
    cudaFree(b.spec);
    cudaFree(b.work);
    cudaFree(b.work2);
    cudaFree(b.work3);
    cudaFree(b.hacc);
    cudaFree(b.mod);
    cudaFree(b.ra);
    cudaFree(b.rb);
    b = PrecBufs<T>();
}

template <typename T> int ensure_pair_bufs(ps_gpu_ctx* c, PrecBufs<T>& b)
{
    const size_t nspec = (size_t)c->N * c->N * b.S;
    PS_TRY(alloc_dev(&b.work2, nspec));
    PS_TRY(alloc_dev(&b.work3, nspec));
    return PS_OK;
}

int ensure_partials(ps_gpu_ctx* c, size_t n)
{
    if (n <= c->partials_cap) return PS_OK;
    if (c->partials) c->retired.push_back(c->partials);
    c->partials = nullptr;
    c->partials_cap = 0;
    PS_TRY(alloc_dev(&c->partials, n));
    c->partials_cap = n;
    return PS_OK;
}
int ensure_sums(ps_gpu_ctx* c, size_t n)
{
    if (n <= c->dsums_cap) return PS_OK;
    if (c->dsums) c->retired.push_back(c->dsums);
    c->dsums = nullptr;
    c->dsums_cap = 0;
    PS_TRY(alloc_dev(&c->dsums, n));
    c->dsums_cap = n;
    return PS_OK;
}
int ensure_shells(ps_gpu_ctx* c, size_t n)
{
    if (n <= c->dshells_cap) return PS_OK;
    if (c->dshells) c->retired.push_back(c->dshells);
    c->dshells = nullptr;
    c->dshells_cap = 0;
    PS_TRY(alloc_dev(&c->dshells, n));
    c->dshells_cap = n;
    return PS_OK;
}
int ensure_lut(ps_gpu_ctx* c, size_t n)
{
    if (n <= c->dlut_cap) return PS_OK;
    if (c->dlut) c->retired.push_back(c->dlut);
    c->dlut = nullptr;
    c->dlut_cap = 0;
    PS_TRY(alloc_dev(&c->dlut, n));
    c->dlut_cap = n;
    return PS_OK;
}
// While alive, the context's stream, partial sums and shell table are those
// of the side lane (every launch helper then works on the side lane).
// With per-kernel profiling on, everything stays on the main lane, so the
// events around each launch time that launch alone.
struct SideLane {
    ps_gpu_ctx* c;
    bool on;
    explicit SideLane(ps_gpu_ctx* cc, bool always = false) : c(cc), on(always || !cc->prof_on) { swap(); }
    ~SideLane() { swap(); }
    void swap()
    {
        if (!on) return;
        std::swap(c->stream, c->side_stream);
        std::swap(c->partials, c->side_partials);
        std::swap(c->partials_cap, c->side_partials_cap);
        std::swap(c->dlut, c->side_lut);
        std::swap(c->dlut_cap, c->side_lut_cap);
    }
};

// While alive, the context's stream, partial sums, shell table and FP32 work
// spectra are those of the second field lane (not while profiling: then
// everything runs on the main lane, one launch at a time).
struct Lane2 {
    ps_gpu_ctx* c;
    bool on;
    explicit Lane2(ps_gpu_ctx* cc, bool always = false) : c(cc), on(always || !cc->prof_on) { swap(); }
    ~Lane2() { swap(); }
    void swap()
    {
        if (!on) return;
        std::swap(c->stream, c->lane2_stream);
        std::swap(c->partials, c->lane2_partials);
        std::swap(c->partials_cap, c->lane2_partials_cap);
        std::swap(c->dlut, c->lane2_lut);
        std::swap(c->dlut_cap, c->lane2_lut_cap);
        std::swap(c->f.work, c->lane2_work[0]);
        std::swap(c->f.work2, c->lane2_work[1]);
        std::swap(c->f.work3, c->lane2_work[2]);
    }
};

// FP32 work spectra of the second lane, n elements each (replaced ones are
// retired: a captured graph may still point at them).
int ensure_lane2_work(ps_gpu_ctx* c, size_t n)
{
    if (n <= c->lane2_work_cap) return PS_OK;
    for (auto& p : c->lane2_work) {
        if (p) c->retired.push_back(p);
        p = nullptr;
    }
    c->lane2_work_cap = 0;
    for (auto& p : c->lane2_work) PS_TRY(alloc_dev(&p, n));
    c->lane2_work_cap = n;
    return PS_OK;
}

int ensure_minmax(ps_gpu_ctx* c, size_t n)
{
    if (n <= c->dminmax_cap) return PS_OK;
    if (c->dminmax) c->retired.push_back(c->dminmax);
    c->dminmax = nullptr;
    c->dminmax_cap = 0;
    PS_TRY(alloc_dev(&c->dminmax, n));
    c->dminmax_cap = n;
    return PS_OK;
}

// =========================================================================
// launch plumbing (runtime N -> template N)
// =========================================================================
template <typename T> PrecBufs<T>& bufs(ps_gpu_ctx* c);
template <> PrecBufs<float>& bufs<float>(ps_gpu_ctx* c) { return c->f; }
template <> PrecBufs<double>& bufs<double>(ps_gpu_ctx* c) { return c->d; }

// Y pass geometry of an M-point transform of precision T (autotuned choice).
template <typename T> int pencil_alt_of(const ps_gpu_ctx* c, int M)
{
    if (sizeof(T) != 4) return 0;
    const auto it = c->pencil_alt.find(M);
    return it == c->pencil_alt.end() ? 0 : it->second;
}

// Dot pass geometry of an M-point transform of precision T (autotuned choice).
template <typename T> int dot_alt_of(const ps_gpu_ctx* c, int M)
{
    if (sizeof(T) != 4) return 0;
    const auto it = c->dot_alt.find(M);
    return it == c->dot_alt.end() ? 0 : it->second;
}

// Pair kernel variant of an M-point transform of precision T (autotuned choice).
template <typename T> int pair_var_of(const ps_gpu_ctx* c, int M)
{
    if (sizeof(T) != 4) return 0;
    const auto it = c->pair_var.find(M);
    return it == c->pair_var.end() ? 0 : it->second;
}

}  // namespace

int ps::launch_fail(cudaError_t e, const char* what)
{
    return fail(e == cudaErrorMemoryAllocation ? PS_ERR_OOM : PS_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

namespace {

// ---------------------------------------------------------------- profiling
enum KernelFamily {
    KF_FWD_Z = 0, KF_PASS_Y, KF_FWD_X_STORE, KF_FWD_X_DOT, KF_INV_X, KF_INV_Z, KF_SUM, KF_DERIVED,
    KF_FINAL, KF_PAIR_Z, KF_LUT, KF_GRAD, KF_PAIR2, KF_PAIR_COUNTS, KF_COUNT
};
const char* const kFamilyName[KF_COUNT] = {"fwd_z_r2c", "pass_y", "fwd_x_store", "fwd_x_dot",
                                           "inv_x_masked", "inv_z_c2r", "sum_partials",
                                           "derived_range", "finalize", "pair_z", "shell_lut", "adjoint",
                                           "pair2_parseval", "pair_counts"};
// families of FP64 transform kernels are counted apart (name suffix _f64)
template <typename T> constexpr int fam(int kind) { return sizeof(T) == 8 ? kind + KF_COUNT : kind; }

int prof_fold(ps_gpu_ctx* c)
{
    if (c->prof.empty()) return PS_OK;
    PS_CK(cudaStreamSynchronize(c->stream));
    for (const auto& r : c->prof) {
        float ms = 0.f;
        PS_CK(cudaEventElapsedTime(&ms, r.a, r.b));
        ps_gpu_ctx::ProfAgg& g = c->prof_agg[{r.kind, r.size}];
        g.ms += ms;
        g.bytes += r.bytes;
        g.n += 1;
    }
    c->prof.clear();
    c->ev_used = 0;
    return PS_OK;
}

cudaEvent_t prof_event(ps_gpu_ctx* c)
{
    if (c->ev_used == c->ev_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_used++];
}

// Bracket one kernel launch: begin() before, end() after.
struct Prof {
    ps_gpu_ctx* c;
    cudaEvent_t a = nullptr;
    explicit Prof(ps_gpu_ctx* cc) : c(cc)
    {
        if (c->prof_on && !c->capturing) {
            if (c->prof.size() >= 4096) prof_fold(c);
            a = prof_event(c);
            if (a) cudaEventRecord(a, c->stream);
        }
    }
    // size: the transform size of the launch (0 for size-free kernels)
    void end(int kind, double bytes, int size = 0)
    {
        c->launches++;
        if (!c->capturing) c->launches_total++;
        if (!a) return;
        cudaEvent_t b = prof_event(c);
        if (!b) return;
        cudaEventRecord(b, c->stream);
        c->prof.push_back({kind, size, a, b, bytes});
    }
};

int sum_partials(ps_gpu_ctx* c, int nblocks, int ncols, double* out, int out_stride, const int* idx = nullptr)
{
    Prof pf(c);
    k_sum_partials<<<ncols, 1024, 0, c->stream>>>(c->partials, nblocks, out, out_stride, idx);
    pf.end(KF_SUM, 8.0 * nblocks * ncols);
    return PS_OK;
}

// Inverse X and Y passes of a shell-filtered spectrum into dst, band-limited to
// the shell: h < hb = min(band, N/2) + 1 columns, row stride *S_out.
// mode: LOAD_MASKED (F * field spectrum) or LOAD_UNIT (F).  M > 0 runs the
// transform on an M-grid (M < N, the shell's band below M/2): the same
// spectrum sampled on a coarser real-space grid.
template <typename T>
int c2r_xy(ps_gpu_ctx* c, int mode, const Shell* dshell, int band, V2<T>* dst, int* S_out, int* hb_out,
           int quad = 0, int M = 0)
{
    PrecBufs<T>& B = bufs<T>(c);
    const int N = M > 0 ? M : c->N;
    Tables<T> tb;
    PS_TRY(tables_for<T>(c, N, &tb));
    const int hb = std::min(band, N / 2) + 1;
    const int S = round_up(hb, pw<T>(N));
    const double V = sizeof(V2<T>), NN2 = (double)N * N;
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::inv_x(c->stream, B.spec, B.S, dst, S, mode, dshell, N / 2 + 1, tb, quad,
                                                c->N, 1))));
        const double q = quad ? (double)(N / 2 + 1) * (N / 2 + 1) / NN2 : 1.0;
        pf.end(fam<T>(KF_INV_X), q * NN2 * S * V + (mode == LOAD_MASKED ? NN2 * hb * V : 0.0), N);
    }
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::pass_y(c->stream, dst, S, true, tb, quad, std::min(band, N / 2), 0, NN,
                                                 pencil_alt_of<T>(c, N)))));
        const double q = quad ? (double)(N / 2 + 1) * (N / 2 + 1) / NN2 : 1.0;
        pf.end(fam<T>(KF_PASS_Y), 2.0 * q * NN2 * S * V, N);
    }
    *S_out = S;
    *hb_out = hb;
    return PS_OK;
}

// Inverse 3D transform of shell-filtered data with the real-space epilogue
// (store / multiply / reduce x^p * aux).  For reducing epilogues the grid sum
// lands in *dsum (device).
template <typename T>
int c2r_shell(ps_gpu_ctx* c, int mode, const Shell* dshell, int band, T* out, const T* aux, int epi,
              int power, double* dsum)
{
    PrecBufs<T>& B = bufs<T>(c);
    const int N = c->N;
    const bool reduce = epi >= EPI_MUL_REDUCE;
    if (reduce) PS_TRY(ensure_partials(c, (size_t)N * N));
    int S = 0, hb = 0, nb = 0;
    PS_TRY(c2r_xy<T>(c, mode, dshell, band, B.work, &S, &hb));
    const double V = sizeof(V2<T>), NN2 = (double)N * N;
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::inv_z(c->stream, B.work, S, hb, out, aux, epi, power, c->partials, B.tables(), &nb))));
        const double real = NN2 * N * sizeof(T);
        const double extra = (epi == EPI_STORE ? real : 0.0) + (epi == EPI_MUL_STORE ? 2.0 * real : 0.0) +
                             (epi == EPI_MUL_REDUCE ? real : 0.0);
        pf.end(fam<T>(KF_INV_Z), NN2 * hb * V + extra, N);
    }
    if (reduce) PS_TRY(sum_partials(c, nb, 1, dsum, 1));
    PS_CK(launch_status());
    return PS_OK;
}

// Spectrum of the real product of two band-limited inverse transforms (B may be
// NULL: square of A), rows kept to h < hout, forward Y pass done; into B.work3.
// M > 0: the inputs are M-grid transforms (c2r_xy with the same M).
template <typename T>
int pair_spectrum(ps_gpu_ctx* c, const V2<T>* A, int Sa, int hba, const V2<T>* Bq, int Sb, int hbb, int hout,
                  int* S_out, int quad = 0, int M = 0)
{
    PrecBufs<T>& B = bufs<T>(c);
    const int N = M > 0 ? M : c->N;
    Tables<T> tb;
    PS_TRY(tables_for<T>(c, N, &tb));
    const int S = round_up(hout, pw<T>(N));
    const double V = sizeof(V2<T>), NN2 = (double)N * N;
    const double q = quad ? (double)(N / 2 + 1) * (N / 2 + 1) / NN2 : 1.0;
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::pair_z(c->stream, A, Sa, hba, Bq, Sb, hbb, B.work3, S, hout, tb, quad,
                                                 pair_var_of<T>(c, N)))));
        pf.end(fam<T>(KF_PAIR_Z), q * NN2 * (hba + (Bq ? hbb : 0) + hout) * V, N);
    }
    {
        Prof pf(c);
        // rows |my| >= hout lie outside every shell the product is dotted with
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::pass_y(c->stream, B.work3, S, false, tb, quad, NN, 0, hout - 1,
                                                 pencil_alt_of<T>(c, N)))));
        pf.end(fam<T>(KF_PASS_Y), 2.0 * q * NN2 * S * V, N);
    }
    *S_out = S;
    return PS_OK;
}

// Forward transform of a real grid into B.work (row stride returned), rows
// truncated to h < hout.
template <typename T>
int r2c_work(ps_gpu_ctx* c, int kind, const void* a, const void* b, int hout, int* stride_out)
{
    PrecBufs<T>& B = bufs<T>(c);
    const int N = c->N;
    const int S = round_up(hout, pw<T>(N));
    const double V = sizeof(V2<T>), NN2 = (double)N * N;
    const double src_bytes = kind == SRC_T ? sizeof(T) : (kind == SRC_F32 ? 4.0 : kind == SRC_F64 ? 8.0 : kind == SRC_XHI_F32 ? 8.0 : 16.0);
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::fwd_z(c->stream, kind, a, b, B.work, S, hout, B.tables()))));
        pf.end(fam<T>(KF_FWD_Z), NN2 * N * src_bytes + NN2 * hout * V, N);
    }
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::pass_y(c->stream, B.work, S, false, B.tables()))));
        pf.end(fam<T>(KF_PASS_Y), 2.0 * NN2 * S * V, N);
    }
    *stride_out = S;
    return PS_OK;
}

// Forward field transform into B.spec (+ phase normalisation).
// split > 0 (FP32 XHI_DENS host loads): rows [0, split) hold dens in a and
// xHII in b, rows [split, N^2) the composed field in a (same offsets).
template <typename T> int forward_field(ps_gpu_ctx* c, int kind, const void* a, const void* b, size_t split = 0)
{
    PrecBufs<T>& B = bufs<T>(c);
    const int N = c->N;
    const int epi = c->use_only_phase == 1 ? SPEC_STORE_PHASE : SPEC_STORE;
    T* mod = nullptr;
    B.have_mod = false;
    if (epi == SPEC_STORE_PHASE && c->keep_modulus) {
        PS_TRY(alloc_dev(&B.mod, (size_t)N * N * B.S));
        mod = B.mod;
    }
    // band-limited spectrum: columns h <= band, rows and outputs |m| <= band
    const int band = (c->spec_band >= 0 && c->spec_band < N / 2) ? c->spec_band : N / 2;
    const int hcols = band + 1;
    const int ncols = std::min(B.S, round_up(hcols, pw<T>(N)));
    const double V = sizeof(V2<T>), NN2 = (double)N * N, H = hcols;
    const double src_bytes = kind == SRC_F32 ? 4.0 : kind == SRC_F64 ? 8.0 : kind == SRC_XHI_F32 ? 8.0 : 16.0;
    {
        Prof pf(c);
        if (split == 0) {
            const int extra = fault_hit(FAULT_WAIT) ? 16 : 0;
            PS_SWITCH_N(N, PS_TRY((L3<T, NN>::fwd_z(c->stream, kind, a, b, B.spec, B.S, hcols, B.tables(), -1, 0,
                                                    c->dstatus, extra))));
        } else {
            const size_t nr = (size_t)N * N;
            const float* af = (const float*)a;
            PS_SWITCH_N(N, PS_TRY((L3<T, NN>::fwd_z(c->stream, SRC_XHI_F32, af, b, B.spec, B.S, hcols, B.tables(),
                                                    -1, split, c->dstatus))));
            PS_SWITCH_N(N, PS_TRY((L3<T, NN>::fwd_z(c->stream, SRC_F32, af + split * N, nullptr,
                                                    B.spec + split * B.S, B.S, hcols, B.tables(), -1, nr - split,
                                                    c->dstatus))));
        }
        pf.end(fam<T>(KF_FWD_Z), NN2 * N * src_bytes + NN2 * H * V, N);
    }
    {
        Prof pf(c);
        // rows |my| > band are read by no later pass: not stored
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::pass_y(c->stream, B.spec, B.S, false, B.tables(), 0, NN, ncols,
                                                 band < N / 2 ? band : NN))));
        const double rows_out = band < N / 2 ? (double)N * (2 * band + 1) : NN2;
        pf.end(fam<T>(KF_PASS_Y), (NN2 + rows_out) * ncols * V, N);
    }
    {
        Prof pf(c);
        const double rows = band < N / 2 ? (double)N * (2 * band + 1) : NN2;
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::fwd_x(c->stream, B.spec, B.S, hcols, epi, B.spec, B.S, nullptr, 0,
                                                nullptr, 0, nullptr, 0, nullptr, B.tables(), nullptr, 1.0, 0, 0,
                                                0x7fffffff, mod, ncols, band < N / 2 ? band : NN))));
        pf.end(fam<T>(KF_FWD_X_STORE), rows * H * V + (band < N / 2 ? (double)(2 * band + 1) : (double)N) *
                                                         (2 * band + 1 < N ? 2 * band + 1 : N) * H * V, N);
    }
    c->loaded_band = band;
    PS_CK(launch_status());
    B.have_spec = true;
    B.have_mod = mod != nullptr;
    return PS_OK;
}

// Dot / count pass over a forward-transformed work buffer (stride S, band
// hvalid) for up to MAX_DOT_SHELLS shells per launch; results to dout[0..ns).
// hsh: host copies of the shells (decide whether an r2 bitmask table applies).
// M > 0: the buffer is an M-grid spectrum; dot sums are scaled by `weight`.
template <typename T>
int dot_pass(ps_gpu_ctx* c, V2<T>* data, int epi, int S, int hvalid, const Shell* dshells,
             const Shell* hsh, int ns, double* dout, int quad = 0, int M = 0, double weight = 1.0,
             const int* didx = nullptr)
{
    PrecBufs<T>& B = bufs<T>(c);
    const int N = M > 0 ? M : c->N;
    Tables<T> tb;
    PS_TRY(tables_for<T>(c, N, &tb));
    for (int s0 = 0; s0 < ns; s0 += MAX_DOT_SHELLS) {
        const int cnt = std::min(MAX_DOT_SHELLS, ns - s0);
        const size_t blocks = (size_t)N * (S / pw<T>(N));
        PS_TRY(ensure_partials(c, blocks * MAX_DOT_SHELLS));
        bool lut_ok = true;
        int lut_size = 0;
        long long r2max = 0;  // no mode of these shells lies outside |m|^2 <= r2max
        for (int q = s0; q < s0 + cnt; q++) {
            if (hsh[q].kind != SHELL_DEFAULT && hsh[q].kind != SHELL_RANGE) lut_ok = false;
            lut_size = std::max(lut_size, hsh[q].r2hi + 1);
            const long long b = std::min(hsh[q].band, N / 2);
            r2max = std::max(r2max, (hsh[q].kind == SHELL_DEFAULT || hsh[q].kind == SHELL_RANGE)
                                        ? (long long)hsh[q].r2hi : 3 * b * b);
        }
        const unsigned short* lut = nullptr;
        if (lut_ok) {
            PS_TRY(ensure_lut(c, (size_t)std::max(lut_size, 1)));
            Prof pf(c);
            if (lut_size > 0)
                k_shell_lut<<<(lut_size + 255) / 256, 256, 0, c->stream>>>(dshells + s0, cnt, lut_size, c->dlut);
            pf.end(KF_LUT, 2.0 * lut_size);
            lut = c->dlut;
        }
        int nb = 0;
        {
            Prof pf(c);
            PS_SWITCH_N(N, PS_TRY((L3<T, NN>::fwd_x(c->stream, data, S, hvalid, epi, nullptr, 0, B.spec, B.S,
                                                    dshells + s0, cnt, lut, lut_size, c->partials, tb, &nb,
                                                    weight, quad, c->N, (int)std::min<long long>(r2max, 0x7fffffff),
                                                    nullptr, 0, NN, dot_alt_of<T>(c, N)))));
            const double q = quad ? (double)(N / 2 + 1) * (N / 2 + 1) / ((double)N * N) : 1.0;
            pf.end(fam<T>(KF_FWD_X_DOT), q * N * N * hvalid * sizeof(V2<T>) * (epi == SPEC_DOT ? 2.0 : 1.0), N);
        }
        PS_TRY(didx ? sum_partials(c, nb, cnt, dout, 1, didx + s0) : sum_partials(c, nb, cnt, dout + s0, 1));
    }
    PS_CK(launch_status());
    return PS_OK;
}

// =========================================================================
// shells
// =========================================================================
struct ShellKey {
    int kind;
    double a, b, half;
    bool operator<(const ShellKey& o) const
    {
        return std::tie(kind, a, b, half) < std::tie(o.kind, o.a, o.b, o.half);
    }
};

int band_of(double r, int N)
{
    if (!(r >= 0.0) || !std::isfinite(r) || r >= (double)(N / 2)) return N / 2;
    return std::min(N / 2, (int)floor(r) + 2);
}

Shell make_shell(int kind, double k, double kmin, double kmax, double binwidth, double L, int N)
{
    const double pi = ref_pi();
    Shell s;
    memset(&s, 0, sizeof(s));
    s.kind = kind;
    s.half = 0.5 * binwidth;
    volatile double big = 1.e30;
    s.min2_init = big * big;
    s.kk = k / (2. * pi) * L;           // filter.c:36
    s.mmin = kmin / (2. * pi) * L;      // filter.c:137
    s.mmax = kmax / (2. * pi) * L;      // filter.c:138
    const double ah = fabs(s.half);
    double rb;
    switch (kind) {
    case SHELL_DEFAULT: rb = s.kk + ah; break;
    case SHELL_RANGE: rb = s.mmax + ah; break;
    case SHELL_WATKINSON: rb = s.kk + 1.7320508075688772 * ah + 1e-9; break;
    default: rb = std::max(s.mmin, s.mmax) + 1.7320508075688772 * ah + 1e-9; break;
    }
    s.band = band_of(rb, N);
    shell_r2_interval(s, N);
    if (kind == SHELL_DEFAULT || kind == SHELL_RANGE)  // |m_x| <= sqrt(r2) <= sqrt(r2hi)
        s.band = std::min(s.band, s.r2hi >= 0 ? (int)floor(sqrt((double)s.r2hi)) : 0);
    return s;
}

// Grid of k_derived_range: one thread per (mx, my) column for interval shells,
// per mode of the band cube otherwise.
int derived_blocks(const Shell& sh, int band)
{
    const long long side = 2 * band + 1;
    const long long total = (sh.kind == SHELL_DEFAULT || sh.kind == SHELL_RANGE) ? side * side
                                                                                : side * side * (band + 1);
    return (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148 * 16));
}

// DERIVED ranges (filter.c:78-114) of DEFAULT shells, computed on the device.
int derive_ranges(ps_gpu_ctx* c, const std::vector<Shell>& sh, std::vector<double>& kmin,
                  std::vector<double>& kmax)
{
    const int ns = (int)sh.size();
    kmin.assign(ns, 0.0);
    kmax.assign(ns, 0.0);
    if (!ns) return PS_OK;
    PS_TRY(ensure_shells(c, ns));
    PS_TRY(ensure_minmax(c, 2 * (size_t)ns));
    PS_CK(cudaMemcpyAsync(c->dshells, sh.data(), sizeof(Shell) * ns, cudaMemcpyHostToDevice, c->stream));
    std::vector<unsigned long long> init(2 * ns);
    for (int s = 0; s < ns; s++) {
        double m2 = sh[s].min2_init, z = 0.0;
        memcpy(&init[2 * s], &m2, 8);
        memcpy(&init[2 * s + 1], &z, 8);
    }
    PS_CK(cudaMemcpyAsync(c->dminmax, init.data(), 16 * (size_t)ns, cudaMemcpyHostToDevice, c->stream));
    const int N = c->N;
    for (int s = 0; s < ns; s++) {
        const int band = std::min(sh[s].band, N / 2);
        const int hmax = band;
        const int blocks = derived_blocks(sh[s], band);
        Prof pf(c);
        k_derived_range<<<blocks, 256, 0, c->stream>>>(N, c->dshells + s, hmax, c->dminmax + 2 * s);
        pf.end(KF_DERIVED, 0.0);
    }
    PS_CK(launch_status());
    PS_CK(cudaMemcpyAsync(init.data(), c->dminmax, 16 * (size_t)ns, cudaMemcpyDeviceToHost, c->stream));
    PS_CK(cudaStreamSynchronize(c->stream));
    const double pi = ref_pi();
    for (int s = 0; s < ns; s++) {
        double m2, x2;
        memcpy(&m2, &init[2 * s], 8);
        memcpy(&x2, &init[2 * s + 1], 8);
        const double rmin = sqrt(m2), rmax = sqrt(x2);
        kmin[s] = rmin * 2. * pi / c->L;  // filter.c:112-113
        kmax[s] = rmax * 2. * pi / c->L;
    }
    return PS_OK;
}

// calc_k3_min_and_max (filter.c:291-319), same operation order.
void closing_leg_range(const double* k, double* kmin, double* kmax)
{
    const double cth = (k[0] * k[0] + k[1] * k[1] - k[2] * k[2]) / (2. * k[0] * k[1]);
    const double a[8] = {kmin[0], kmin[0], kmax[0], kmax[0], k[0], kmax[0], k[0], kmin[0]};
    const double b[8] = {kmin[1], kmax[1], kmin[1], kmax[1], kmax[1], k[1], kmin[1], k[1]};
    double lo = 1.e30, hi = 0.;
    for (int q = 0; q < 8; q++) {
        const double t = a[q] * a[q] + b[q] * b[q] - 2. * a[q] * b[q] * cth;
        if (t < lo) lo = t;
        if (t > hi) hi = t;
    }
    kmin[2] = sqrt(lo);
    kmax[2] = sqrt(hi);
}

// Resolve every leg of every configuration to a shell (polyspectrum.c:79-118),
// running the DERIVED reductions on the device and writing the derived ranges
// back into the configurations.
int resolve_legs(ps_gpu_ctx* c, int nconf, ps_cfg* cfgs, std::vector<std::vector<Shell>>& legs)
{
    const int N = c->N;
    const double L = c->L;
    legs.assign(nconf, {});
    // pass 1: DEFAULT shells whose DERIVED range is needed
    std::map<ShellKey, int> dkey;
    std::vector<Shell> dsh;
    for (int q = 0; q < nconf; q++) {
        const ps_cfg& g = cfgs[q];
        if (g.n < 2 || g.n > PS_MAX_LEGS) return fail(PS_ERR_ARG, "config %d: n=%d out of range", q, g.n);
        if (g.kbinningCase == PS_BIN_DERIVED) {
            if (g.n != 3)
                return fail(PS_ERR_UNDEFINED,
                            "config %d: DERIVED binning with n=%d is undefined in the reference "
                            "(calc_kn_min_and_max, filter.c:321-325)", q, g.n);
            for (int l = 0; l < g.n - 1; l++) {
                ShellKey key{SHELL_DEFAULT, g.k[l], 0.0, 0.5 * g.kbinwidth};
                if (!dkey.count(key)) {
                    dkey[key] = (int)dsh.size();
                    dsh.push_back(make_shell(SHELL_DEFAULT, g.k[l], 0, 0, g.kbinwidth, L, N));
                }
            }
        }
    }
    std::vector<double> dmin, dmax;
    PS_TRY(derive_ranges(c, dsh, dmin, dmax));
    // pass 2: every leg
    for (int q = 0; q < nconf; q++) {
        ps_cfg& g = cfgs[q];
        const int n = g.n;
        auto& ls = legs[q];
        for (int l = 0; l < n; l++) {
            const bool last = l == n - 1;
            switch (g.kbinningCase) {
            case PS_BIN_DERIVED:
                if (!last) {
                    const int id = dkey[ShellKey{SHELL_DEFAULT, g.k[l], 0.0, 0.5 * g.kbinwidth}];
                    g.kmin[l] = dmin[id];
                    g.kmax[l] = dmax[id];
                    ls.push_back(dsh[id]);
                } else {
                    closing_leg_range(g.k, g.kmin, g.kmax);
                    ls.push_back(make_shell(SHELL_RANGE, 0, g.kmin[l], g.kmax[l], g.kbinwidth, L, N));
                }
                break;
            case PS_BIN_GIVEN:
                ls.push_back(last ? make_shell(SHELL_RANGE, 0, g.kmin[l], g.kmax[l], g.kbinwidth, L, N)
                                  : make_shell(SHELL_DEFAULT, g.k[l], 0, 0, g.kbinwidth, L, N));
                break;
            case PS_BIN_WATKINSON:
                ls.push_back(last ? make_shell(SHELL_WATKINSON_RANGE, 0, g.kmin[l], g.kmax[l],
                                               g.kbinwidth, L, N)
                                  : make_shell(SHELL_WATKINSON, g.k[l], 0, 0, g.kbinwidth, L, N));
                break;
            default:
                ls.push_back(make_shell(SHELL_DEFAULT, g.k[l], 0, 0, g.kbinwidth, L, N));
                break;
            }
        }
    }
    return PS_OK;
}

bool same_shell(const Shell& a, const Shell& b) { return memcmp(&a, &b, sizeof(Shell)) == 0; }

// =========================================================================
// finalisation: B = pow(V,n-1)*pow(N,-3n)*sumD/sumI (polyspectrum.c:155)
// =========================================================================
__global__ void k_finalize(int nconf, const double* __restrict__ coef, const double* __restrict__ sumD,
                           const double* __restrict__ sumI, double inv_n3, int count_mode,
                           double* __restrict__ out)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nconf) return;
    const double sD = sumD[q];
    double sI, np;
    if (count_mode) {  // sumI holds the exact polygon count
        np = sumI[q];
        sI = __dmul_rn(np, 1.0 / inv_n3);
    } else {
        sI = sumI[q];
        np = __dmul_rn(sI, inv_n3);
    }
    out[2 * q] = __ddiv_rn(__dmul_rn(coef[q], sD), sI);
    out[2 * q + 1] = count_mode ? np : __ddiv_rn(sI, 1.0 / inv_n3);
}

double norm_coef(double L, int N, int n)
{
    const double volume = L * L * L;
    return pow(volume, n - 1) * pow(N, -n * 3);
}

// =========================================================================
// method 1: plain FP64, reference dataflow
// =========================================================================
// A computation reaching modes of band `need` on a field loaded with a
// narrower spectrum band (ps_gpu_set_spectrum_band) is refused.
int check_band(const ps_gpu_ctx* c, int need)
{
    if (need > c->loaded_band)
        return fail(PS_ERR_ARG, "the field was loaded with spectrum band %d; this computation reaches modes of band %d",
                    c->loaded_band, need);
    return PS_OK;
}
int legs_band(const std::vector<Shell>& legs, int N)
{
    int b = 0;
    for (const Shell& sh : legs) b = std::max(b, std::min(sh.band, N / 2));
    return b;
}

// Key of a configuration's polygon count: the method and what selects the
// shells (DERIVED ranges are outputs, not inputs).
std::string npoly_key(int method, const ps_cfg& g)
{
    std::string k;
    auto add = [&](double v) { k.append(reinterpret_cast<const char*>(&v), sizeof(v)); };
    k.push_back((char)method);
    k.push_back((char)g.n);
    k.push_back((char)g.kbinningCase);
    add(g.kbinwidth);
    for (int l = 0; l < g.n && l < PS_MAX_LEGS; l++) {
        add(g.k[l]);
        if (g.kbinningCase != PS_BIN_DERIVED) {
            add(g.kmin[l]);
            add(g.kmax[l]);
        }
    }
    return k;
}

void remember_npoly(ps_gpu_ctx* c, int method, int nconf, const ps_cfg* in, const double* Np)
{
    if (c->npoly_cache.size() + (size_t)nconf > 4096) c->npoly_cache.clear();
    for (int q = 0; q < nconf; q++) c->npoly_cache[npoly_key(method, in[q])] = Np[q];
}

int plain_batch(ps_gpu_ctx* c, int nconf, ps_cfg* cfgs, double* B, double* Np, double* kappa)
{
    if (!c->d.have_spec) return fail(PS_ERR_ARG, "FP64 spectrum not available (methods mask)");
    std::vector<std::vector<Shell>> legs;
    const int N = c->N;
    PS_TRY(ensure_sums(c, 4 * (size_t)nconf + 8));
    PS_TRY(ensure_shells(c, PS_MAX_LEGS));
    std::vector<double> coef(nconf), habs(nconf, 0.0);
    for (int q = 0; q < nconf; q++) {
        PS_TRY(resolve_legs(c, 1, cfgs + q, legs));
        PS_TRY(check_band(c, legs_band(legs[0], N)));
        const int n = cfgs[q].n;
        PS_CK(cudaMemcpyAsync(c->dshells, legs[0].data(), sizeof(Shell) * n, cudaMemcpyHostToDevice,
                              c->stream));
        double* sD = c->dsums + q;
        double* sI = c->dsums + nconf + q;
        for (int pass = 0; pass < 2; pass++) {  // 0: D = IFFT[F dk], 1: I = IFFT[F]
            const int mode = pass == 0 ? LOAD_MASKED : LOAD_UNIT;
            double* prod = pass == 0 ? c->d.ra : c->d.rb;
            for (int l = 0; l < n; l++) {
                const int epi = l == 0 ? EPI_STORE : (l < n - 1 ? EPI_MUL_STORE : EPI_MUL_REDUCE);
                PS_TRY(c2r_shell<double>(c, mode, c->dshells + l, legs[0][l].band, prod, prod, epi, 1,
                                         pass == 0 ? sD : sI));
                if (kappa && pass == 0 && l == n - 1) {  // sum |prod D| for the condition number
                    double* sA = c->dsums + 3 * nconf + q;
                    PS_TRY(c2r_shell<double>(c, mode, c->dshells + l, legs[0][l].band, prod, prod,
                                             EPI_MUL_REDUCE_ABS, 1, sA));
                    PS_CK(cudaMemcpyAsync(&habs[q], sA, 8, cudaMemcpyDeviceToHost, c->stream));
                }
            }
        }
        coef[q] = norm_coef(c->L, N, n);
        // the host shell table is rewritten by the next config: keep order
        PS_CK(cudaStreamSynchronize(c->stream));
    }
    double* dcoef = c->dsums + 2 * nconf;
    PS_CK(cudaMemcpyAsync(dcoef, coef.data(), sizeof(double) * nconf, cudaMemcpyHostToDevice, c->stream));
    double* dout = nullptr;
    PS_TRY(alloc_dev(&dout, 2 * (size_t)nconf));
    const double inv_n3 = 1.0 / ((double)N * (double)N * (double)N);
    {
        Prof pf(c);
        k_finalize<<<(nconf + 127) / 128, 128, 0, c->stream>>>(nconf, dcoef, c->dsums, c->dsums + nconf,
                                                               inv_n3, 0, dout);
        pf.end(KF_FINAL, 0.0);
    }
    std::vector<double> h(2 * nconf);
    std::vector<double> hD(nconf);
    cudaError_t e1 = cudaMemcpyAsync(h.data(), dout, sizeof(double) * 2 * nconf, cudaMemcpyDeviceToHost,
                                     c->stream);
    if (e1 == cudaSuccess && kappa)
        e1 = cudaMemcpyAsync(hD.data(), c->dsums, sizeof(double) * nconf, cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e2 = cudaStreamSynchronize(c->stream);
    cudaFree(dout);
    PS_CK(e1);
    PS_CK(e2);
    for (int q = 0; q < nconf; q++) {
        B[q] = h[2 * q];
        Np[q] = h[2 * q + 1];
        if (kappa) kappa[q] = habs[q] / fabs(hD[q]);
    }
    return PS_OK;
}

// =========================================================================
// method 2: batched FP32 (FP64 counts)
// =========================================================================
struct Group {  // n=3 configurations sharing the leg pair (a, b)
    int a, b;
    std::vector<int> cfg;    // configuration indices
    std::vector<int> third;  // shell id of each configuration's remaining leg
};

// The closing leg of a DERIVED configuration: its RANGE shell follows from the
// device-derived ranges of legs 0 and 1 (calc_k3_min_and_max, filter.c:291-319).
struct ClosingDesc {
    int cfg;   // configuration (write-back row)
    int d0;    // derived-range slots of legs 0 and 1
    int d1;
    int slot;  // shell-table slot to fill
    int band;  // host upper bound of the shell's extent (launch geometry)
    int pad;
    double k0, k1, k2, half;
};

// kmin, kmax = sqrt(min / max corner^2) * 2 * PI / L (filter.c:112-113, same order)
__global__ void k_derive_finish(int nd, const unsigned long long* __restrict__ mm, double pi, double L,
                                double* __restrict__ kr)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nd) return;
    const double rmin = __dsqrt_rn(__longlong_as_double((long long)mm[2 * s]));
    const double rmax = __dsqrt_rn(__longlong_as_double((long long)mm[2 * s + 1]));
    kr[2 * s] = __ddiv_rn(__dmul_rn(__dmul_rn(rmin, 2.0), pi), L);
    kr[2 * s + 1] = __ddiv_rn(__dmul_rn(__dmul_rn(rmax, 2.0), pi), L);
}

__device__ __forceinline__ double k3_term(double a, double b, double c)  // a*a + b*b - 2.*a*b*c
{
    return __dsub_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(__dmul_rn(__dmul_rn(2.0, a), b), c));
}

// Closing-leg shells of DERIVED configurations (calc_k3_min_and_max, then
// construct_kfilter_with_kbinwidth's mmin/mmax), written into the shell table,
// and the derived k ranges of all three legs for the write-back.
__global__ void k_closing(int ncl, const ClosingDesc* __restrict__ cd, const double* __restrict__ kr,
                          Shell* __restrict__ table, double* __restrict__ wb, double pi, double L, int n,
                          double min2_init, int* __restrict__ err)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ncl) return;
    const ClosingDesc d = cd[q];
    const double kmin0 = kr[2 * d.d0], kmax0 = kr[2 * d.d0 + 1];
    const double kmin1 = kr[2 * d.d1], kmax1 = kr[2 * d.d1 + 1];
    const double k0 = d.k0, k1 = d.k1, k2 = d.k2;
    const double cth = __ddiv_rn(__dsub_rn(__dadd_rn(__dmul_rn(k0, k0), __dmul_rn(k1, k1)), __dmul_rn(k2, k2)),
                                 __dmul_rn(__dmul_rn(2.0, k0), k1));
    const double a[8] = {kmin0, kmin0, kmax0, kmax0, k0, kmax0, k0, kmin0};
    const double b[8] = {kmin1, kmax1, kmin1, kmax1, kmax1, k1, kmin1, k1};
    double lo = 1.e30, hi = 0.;
#pragma unroll
    for (int t = 0; t < 8; t++) {
        const double v = k3_term(a[t], b[t], cth);
        if (v < lo) lo = v;
        if (v > hi) hi = v;
    }
    const double kmin2 = __dsqrt_rn(lo), kmax2 = __dsqrt_rn(hi);
    Shell s;
    s.kind = SHELL_RANGE;
    s.band = d.band;
    s.kk = 0.0;
    s.half = d.half;
    s.min2_init = min2_init;
    const double twopi = __dmul_rn(2.0, pi);
    s.mmin = __dmul_rn(__ddiv_rn(kmin2, twopi), L);  // filter.c:137-138
    s.mmax = __dmul_rn(__ddiv_rn(kmax2, twopi), L);
    shell_r2_interval(s, n);
    // a band of N/2 holds every column; a narrower one must hold the whole shell
    if (s.r2hi >= 0 && d.band < n / 2 && (long long)s.r2hi > (long long)d.band * d.band) atomicExch(err, 1);
    table[d.slot] = s;
    double* w = wb + 6 * (size_t)d.cfg;
    w[0] = kmin0;
    w[1] = kmax0;
    w[2] = kmin1;
    w[3] = kmax1;
    w[4] = kmin2;
    w[5] = kmax2;
}

__global__ void k_copy_shells(int n, const int* __restrict__ src, const int* __restrict__ dst, Shell* table)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) table[dst[q]] = table[src[q]];
}

// leg-by-leg configurations hold grid sums: count = rint(sum / N^3), exact
// (the FP64 error is far below 1/2)
__global__ void k_round_counts(int n, const int* __restrict__ idx, double* __restrict__ sumI, double n3)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) sumI[idx[q]] = rint(sumI[idx[q]] / n3);
}


}  // namespace

// A batch prepared once: host planning, device tables and the launch sequence.
struct ps_gpu_plan {
    ps_gpu_ctx* ctx = nullptr;
    int method = 0, nconf = 0, flags = 0;
    std::vector<ps_cfg> cfgs;
    // the launch sequence (stream work only; every op enqueues on the
    // context's current stream), split by what each part reads:
    std::vector<std::function<int()>> ops;         // DERIVED k-ranges and closing shells
    std::vector<std::function<int()>> ops_counts;  // exact polygon counts per pair group (no field)
    std::vector<std::function<int()>> ops_groups;  // the pair groups' field parts (main or second lane)
    std::vector<std::function<int()>> ops_tail;    // n = 2 and leg-by-leg configurations, finalisation
    bool has_groups = false;
    std::vector<void*> owned;               // device buffers of this plan
    double* dres = nullptr;                 // B, Npoly per configuration
    double* dsumA = nullptr;                // sum |terms| (condition numbers)
    double* dsumD = nullptr;
    double* dwb = nullptr;                  // derived k ranges, 6 per configuration
    int* derr = nullptr;
    double* hres = nullptr;  // pinned host copy of dres | dwb | dsumA | dsumD | err
    std::vector<int> derived_cfgs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long graph_launches = 0;  // kernels in the captured graph
    int band = 0;                  // largest |component| of a mode the plan reads
    // ps_gpu_plan_prepare: the field-independent parts (ops, ops_counts) of
    // the next execution enqueued ahead on the side lane; ev_derived and
    // ev_counts mark their ends there
    bool prepared = false;
    cudaEvent_t ev_prep = nullptr, ev_derived = nullptr, ev_counts = nullptr;
    struct Part {  // one part captured as a graph (PS_PLAN_GRAPH)
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;
    } parts[4];  // derived, counts, groups, tail
};

namespace {

template <typename T> int plan_alloc(ps_gpu_plan* P, T** p, size_t count)
{
    *p = nullptr;
    PS_TRY(alloc_dev(p, count));
    P->owned.push_back(*p);
    return PS_OK;
}

template <typename T> int plan_upload(ps_gpu_plan* P, T** p, const std::vector<T>& h)
{
    PS_TRY(plan_alloc(P, p, std::max<size_t>(h.size(), 1)));
    if (!h.empty()) PS_CK(cudaMemcpy(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return PS_OK;
}

struct LegKey {
    int tag;  // 0: exact host shell (bytes), 1: DERIVED closing leg
    Shell sh;
    double k0, k1, k2, half;
    bool same(const LegKey& o) const
    {
        if (tag != o.tag) return false;
        if (tag == 0) return memcmp(&sh, &o.sh, sizeof(Shell)) == 0;
        return k0 == o.k0 && k1 == o.k1 && k2 == o.k2 && half == o.half;
    }
};

// Smallest transform size M (16 <= M <= N, one of the instantiated sizes) on which a pair
// group with leg bands ba, bb (largest |component| of a mode) and closing
// bands up to bc runs alias-free.  A triple m_a + m_b + m_c = 0 (mod M) with
// each component of |m_i| <= b_i and b_a + b_b + b_c < M is zero outright, so
// the cyclic sums over the M-grid and over the N-grid count the same triples
// (the reference's N-grid sums then have no aliased triples either); 2 b < M
// keeps every mode of a shell on its own M-grid index.  N when none fits.
const int kGridSizes[] = {16, 32, 64, 96, 128, 192, 256, 320, 384, 512, 1024};

int alias_free_grid(int N, int ba, int bb, int bc)
{
    const int bmax = std::max({ba, bb, bc});
    for (int M : kGridSizes)
        if (M < N && M > ba + bb + bc && M > 2 * bmax) return M;
    return N;
}

bool grid_supported(int M)
{
    for (int q : kGridSizes)
        if (q == M) return true;
    return false;
}

// Autotuning of a pair group's transform size: the alias-free minimum M0 and
// up to two larger supported sizes (<= N) are each run once to warm up, then
// timed over three runs with CUDA events on the context's stream; the fastest
// wins.  Every candidate gives the same counts and the same sums up to FP32
// rounding of the transforms.
int tune_grid(ps_gpu_ctx* c, const std::function<std::function<int()>(int)>& group_op, int M0, int* best)
{
    std::vector<int> cands;
    for (int q : kGridSizes)
        if (q >= M0 && q <= c->N && cands.size() < 3) cands.push_back(q);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PS_CK(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(PS_ERR_CUDA, "event creation failed");
    }
    float best_ms = 0.f;
    int rc = PS_OK;
    *best = M0;
    for (int M : cands) {
        if (M < c->N) {
            Tables<float> t32;
            Tables<double> t64;
            if ((rc = tables_for<float>(c, M, &t32)) != PS_OK || (rc = tables_for<double>(c, M, &t64)) != PS_OK) break;
        }
        const auto op = group_op(M);
        if ((rc = op()) != PS_OK) break;
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 3 && rc == PS_OK; r++) rc = op();
        cudaEventRecord(e1, c->stream);
        if (rc != PS_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "autotune timing failed");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (M == cands[0] || ms < best_ms) {
            best_ms = ms;
            *best = M;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// Autotuning of the FP32 Y pass geometry of an M-point transform: the
// default and the alternative (PencilAlt) each run once to warm up, then
// three times timed with CUDA events, in place on a scratch work spectrum of
// M planes of band-limited width; the faster is kept for the context.
int tune_pencil(ps_gpu_ctx* c, int M)
{
    if (c->pencil_alt.count(M)) return PS_OK;
    bool has_alt = false;
    {
        const int N = M;
        PS_SWITCH_N(N, (has_alt = L3<float, NN>::ALT > 0));
    }
    if (!has_alt || !c->f.work) {
        c->pencil_alt[M] = 0;
        return PS_OK;
    }
    Tables<float> tb;
    PS_TRY(tables_for<float>(c, M, &tb));
    const int S = std::min(c->f.S, round_up(M / 2 + 1, pw<float>(M)));
    if ((size_t)M * M * S > (size_t)c->N * c->N * c->f.S) {
        c->pencil_alt[M] = 0;
        return PS_OK;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PS_CK(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(PS_ERR_CUDA, "event creation failed");
    }
    float ms[2] = {0.f, 0.f};
    int rc = PS_OK;
    for (int alt = 0; alt < 2 && rc == PS_OK; alt++) {
        const int N = M;
        auto run = [&]() -> int {
            PS_SWITCH_N(N, PS_TRY((L3<float, NN>::pass_y(c->stream, c->f.work, S, true, tb, 0, NN, 0, NN, alt))));
            return PS_OK;
        };
        if ((rc = run()) != PS_OK) break;
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 3 && rc == PS_OK; r++) rc = run();
        cudaEventRecord(e1, c->stream);
        if (rc == PS_OK && cudaEventSynchronize(e1) != cudaSuccess) rc = fail(PS_ERR_CUDA, "autotune timing failed");
        if (rc == PS_OK) cudaEventElapsedTime(&ms[alt], e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == PS_OK) c->pencil_alt[M] = ms[1] < ms[0] ? 1 : 0;
    return rc;
}

// Autotuning of the FP32 pair kernel variant of an M-point transform
// (PairVariants: the default, one live row transform, twice the elements per
// thread): every variant the length has runs once to warm up, then three times
// timed with CUDA events, on legs of hva / hvb valid columns (hvb = 0: one leg
// squared) read from the start of a scratch work spectrum and products of hout
// columns written behind them; the fastest is kept for the context.  The
// variants compute the same transforms (their sums differ by FP32 rounding).
int tune_pair(ps_gpu_ctx* c, int M, int hva, int hvb, int hout)
{
    if (c->pair_var.count(M)) return PS_OK;
    int mask = 1;
    {
        const int N = M;
        PS_SWITCH_N(N, (mask = L3<float, NN>::pair_variants()));
    }
    const int w = pw<float>(M);
    const int Sa = round_up(std::max(hva, hvb), w), Sd = round_up(hout, w);
    const size_t need = (size_t)M * M * (size_t)(Sa + Sd);
    if (mask == 1 || !c->f.work || need > (size_t)c->N * c->N * c->f.S) {
        c->pair_var[M] = 0;
        return PS_OK;
    }
    Tables<float> tb;
    PS_TRY(tables_for<float>(c, M, &tb));
    const V2<float>* src = c->f.work;
    V2<float>* dst = c->f.work + (size_t)M * M * Sa;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PS_CK(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(PS_ERR_CUDA, "event creation failed");
    }
    float best_ms = 0.f;
    int best = 0, rc = PS_OK;
    for (int v = 0; v < 3 && rc == PS_OK; v++) {
        if (!((mask >> v) & 1)) continue;
        const int N = M;
        auto run = [&]() -> int {
            PS_SWITCH_N(N, PS_TRY((L3<float, NN>::pair_z(c->stream, src, Sa, hva, hvb > 0 ? src : nullptr, Sa, hvb,
                                                         dst, Sd, hout, tb, 0, v))));
            return PS_OK;
        };
        if ((rc = run()) != PS_OK) break;
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 3 && rc == PS_OK; r++) rc = run();
        cudaEventRecord(e1, c->stream);
        if (rc == PS_OK && cudaEventSynchronize(e1) != cudaSuccess) rc = fail(PS_ERR_CUDA, "autotune timing failed");
        float ms = 0.f;
        if (rc == PS_OK) cudaEventElapsedTime(&ms, e0, e1);
        if (rc == PS_OK && (v == 0 || ms < best_ms)) {
            best_ms = ms;
            best = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == PS_OK) c->pair_var[M] = best;
    return rc;
}

// Autotuning of the FP32 dot pass geometry of an M-point transform (the
// default against PencilAlt, twice the elements per thread): the group's
// whole field part (masked inverse transforms, pair kernel, forward Y pass,
// dot pass) runs once to warm up and three times timed with CUDA events in
// each geometry; the faster is kept for the context.  Both give the same sums
// up to FP32 rounding.
int tune_dot(ps_gpu_ctx* c, const std::function<int()>& group_field_op, int M)
{
    if (c->dot_alt.count(M)) return PS_OK;
    bool has_alt = false;
    {
        const int N = M;
        PS_SWITCH_N(N, (has_alt = L3<float, NN>::ALT > 0));
    }
    if (!has_alt) {
        c->dot_alt[M] = 0;
        return PS_OK;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PS_CK(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(PS_ERR_CUDA, "event creation failed");
    }
    float ms[2] = {0.f, 0.f};
    int rc = PS_OK;
    for (int alt = 0; alt < 2 && rc == PS_OK; alt++) {
        c->dot_alt[M] = alt;
        if ((rc = group_field_op()) != PS_OK) break;
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 3 && rc == PS_OK; r++) rc = group_field_op();
        cudaEventRecord(e1, c->stream);
        if (rc == PS_OK && cudaEventSynchronize(e1) != cudaSuccess) rc = fail(PS_ERR_CUDA, "autotune timing failed");
        if (rc == PS_OK) cudaEventElapsedTime(&ms[alt], e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == PS_OK) c->dot_alt[M] = ms[1] < ms[0] ? 1 : 0;
    else c->dot_alt.erase(M);
    return rc;
}

int sum_partials_n(ps_gpu_ctx* c, int nblocks, int ncols, double* out)
{
    return sum_partials(c, nblocks, ncols, out, 1);
}

int scatter_dev(ps_gpu_ctx* c, const double* src, const int* didx, int count, double* dst)
{
    Prof pf(c);
    k_scatter<<<(count + 127) / 128, 128, 0, c->stream>>>(src, didx, count, dst);
    pf.end(KF_SUM, 16.0 * count);
    return PS_OK;
}

// Plan of the batched method: everything host-side happens here; the ops only
// enqueue stream work (so a plan can be captured into a CUDA graph).
int plan_batched(ps_gpu_ctx* c, ps_gpu_plan* P)
{
    if (!(c->methods & PS_FP32_BATCHED)) return fail(PS_ERR_ARG, "batched method not enabled for this context");
    const int N = c->N;
    const double L = c->L;
    const int nconf = P->nconf;
    std::vector<ps_cfg>& cfgs = P->cfgs;
    const bool kappa = (P->flags & PS_PLAN_KAPPA) != 0;

    // ---- legs -> shells (DERIVED closing legs are completed on the device)
    std::vector<LegKey> uniq;
    std::vector<std::vector<int>> lid(nconf);
    std::vector<Shell> derived;  // DEFAULT shells whose DERIVED range is needed
    std::vector<ClosingDesc> closing;
    auto derived_slot = [&](const Shell& sh) {
        for (size_t q = 0; q < derived.size(); q++)
            if (memcmp(&derived[q], &sh, sizeof(Shell)) == 0) return (int)q;
        derived.push_back(sh);
        return (int)derived.size() - 1;
    };
    auto uniq_id = [&](const LegKey& k) {
        for (size_t u = 0; u < uniq.size(); u++)
            if (uniq[u].same(k)) return (int)u;
        uniq.push_back(k);
        return (int)uniq.size() - 1;
    };
    for (int q = 0; q < nconf; q++) {
        const ps_cfg& g = cfgs[q];
        if (g.n < 2 || g.n > PS_MAX_LEGS) return fail(PS_ERR_ARG, "config %d: n=%d out of range", q, g.n);
        if (g.kbinningCase == PS_BIN_DERIVED && g.n != 3)
            return fail(PS_ERR_UNDEFINED,
                        "config %d: DERIVED binning with n=%d is undefined in the reference "
                        "(calc_kn_min_and_max, filter.c:321-325)", q, g.n);
        for (int l = 0; l < g.n; l++) {
            const bool last = l == g.n - 1;
            LegKey key;
            memset(&key, 0, sizeof(key));
            switch (g.kbinningCase) {
            case PS_BIN_DERIVED:
                if (!last) {
                    key.sh = make_shell(SHELL_DEFAULT, g.k[l], 0, 0, g.kbinwidth, L, N);
                } else {
                    // host bound of the closing shell's radius: a derived kmax_i/kF is at most
                    // sqrt(r2hi_i) + sqrt(3)/2 bw (a corner of the selected voxel's cube), and
                    // k3^2 = a^2 + b^2 - 2ab cos(theta) <= a^2 + b^2 + 2ab max(1, |cos(theta)|)
                    const Shell s0 = make_shell(SHELL_DEFAULT, g.k[0], 0, 0, g.kbinwidth, L, N);
                    const Shell s1 = make_shell(SHELL_DEFAULT, g.k[1], 0, 0, g.kbinwidth, L, N);
                    const double e = 0.8660254037844387 * fabs(g.kbinwidth) + 1e-6;
                    const double r0 = (s0.r2hi >= 0 ? sqrt((double)s0.r2hi) : 0.0) + e;
                    const double r1 = (s1.r2hi >= 0 ? sqrt((double)s1.r2hi) : 0.0) + e;
                    const double cth = (g.k[0] * g.k[0] + g.k[1] * g.k[1] - g.k[2] * g.k[2]) / (2. * g.k[0] * g.k[1]);
                    const double cmax = std::isfinite(cth) ? std::max(1.0, fabs(cth)) : HUGE_VAL;
                    const double r3 = sqrt(r0 * r0 + r1 * r1 + 2.0 * r0 * r1 * cmax) * (1.0 + 1e-12);
                    key.tag = 1;
                    key.k0 = g.k[0];
                    key.k1 = g.k[1];
                    key.k2 = g.k[2];
                    key.half = 0.5 * g.kbinwidth;
                    key.sh.kind = SHELL_RANGE;
                    key.sh.band = band_of(r3 + fabs(0.5 * g.kbinwidth) + 1e-6, N);
                    key.sh.r2lo = 0;
                    // upper bound (table sizes only): a full band reaches the corner of the cube
                    key.sh.r2hi = key.sh.band < N / 2 ? key.sh.band * key.sh.band : 3 * (N / 2) * (N / 2);
                }
                break;
            case PS_BIN_GIVEN:
                key.sh = last ? make_shell(SHELL_RANGE, 0, g.kmin[l], g.kmax[l], g.kbinwidth, L, N)
                              : make_shell(SHELL_DEFAULT, g.k[l], 0, 0, g.kbinwidth, L, N);
                break;
            case PS_BIN_WATKINSON:
                key.sh = last ? make_shell(SHELL_WATKINSON_RANGE, 0, g.kmin[l], g.kmax[l], g.kbinwidth, L, N)
                              : make_shell(SHELL_WATKINSON, g.k[l], 0, 0, g.kbinwidth, L, N);
                break;
            default:
                key.sh = make_shell(SHELL_DEFAULT, g.k[l], 0, 0, g.kbinwidth, L, N);
                break;
            }
            lid[q].push_back(uniq_id(key));
        }
        if (g.kbinningCase == PS_BIN_DERIVED) {
            P->derived_cfgs.push_back(q);
            const int d0 = derived_slot(make_shell(SHELL_DEFAULT, g.k[0], 0, 0, g.kbinwidth, L, N));
            const int d1 = derived_slot(make_shell(SHELL_DEFAULT, g.k[1], 0, 0, g.kbinwidth, L, N));
            ClosingDesc d;
            memset(&d, 0, sizeof(d));
            d.cfg = q;
            d.d0 = d0;
            d.d1 = d1;
            d.slot = lid[q][2];
            d.band = uniq[lid[q][2]].sh.band;
            d.k0 = g.k[0];
            d.k1 = g.k[1];
            d.k2 = g.k[2];
            d.half = 0.5 * g.kbinwidth;
            closing.push_back(d);
        }
    }
    const int nu = (int)uniq.size();
    auto host_shell_of = [&](int u) -> const Shell& { return uniq[u].sh; };

    // ---- plan: pair groups (n = 3 sharing a leg pair), n = 2 (Parseval), the rest leg by leg
    std::vector<Group> groups;
    std::vector<int> direct, pairs2;
    {
        std::map<std::pair<int, int>, int> freq;
        for (int q = 0; q < nconf; q++)
            if (cfgs[q].n == 3) {
                const auto& v = lid[q];
                for (int x = 0; x < 3; x++)
                    for (int y = x + 1; y < 3; y++) freq[{std::min(v[x], v[y]), std::max(v[x], v[y])}]++;
            }
        std::map<std::pair<int, int>, int> gidx;
        for (int q = 0; q < nconf; q++) {
            const int n = cfgs[q].n;
            if (n == 2) { pairs2.push_back(q); continue; }
            if (n != 3) { direct.push_back(q); continue; }
            const auto& v = lid[q];
            int best = -1, bx = 0, by = 1;
            for (int x = 0; x < 3; x++)
                for (int y = x + 1; y < 3; y++) {
                    const int f = freq[{std::min(v[x], v[y]), std::max(v[x], v[y])}];
                    if (f > best) { best = f; bx = x; by = y; }
                }
            if (best < 2) { direct.push_back(q); continue; }
            const int z = 3 - bx - by;
            std::pair<int, int> key{std::min(v[bx], v[by]), std::max(v[bx], v[by])};
            auto it = gidx.find(key);
            if (it == gidx.end()) {
                gidx[key] = (int)groups.size();
                groups.push_back(Group{key.first, key.second, {}, {}});
                it = gidx.find(key);
            }
            groups[it->second].cfg.push_back(q);
            groups[it->second].third.push_back(v[z]);
        }
    }

    // ---- shell table: [unique shells][group closing lists][n=2 chunk tables]
    std::vector<Shell> table(nu);
    for (int u = 0; u < nu; u++) table[u] = host_shell_of(u);
    P->band = legs_band(table, N);
    std::vector<int> gofs(groups.size()), copy_src, copy_dst;
    for (size_t g = 0; g < groups.size(); g++) {
        gofs[g] = (int)table.size();
        for (int s : groups[g].third) {
            if (uniq[s].tag == 1) {  // filled on the device after k_closing
                copy_src.push_back(s);
                copy_dst.push_back((int)table.size());
            }
            table.push_back(host_shell_of(s));
        }
    }
    struct P2Chunk {
        int ofs, cnt, band, lut_size, idx_ofs;
        bool lut_ok;
    };
    std::vector<P2Chunk> p2;
    std::vector<int> idx_all;  // scatter indices (groups, then n=2 chunks)
    std::vector<int> gidx_ofs(groups.size());
    for (size_t g = 0; g < groups.size(); g++) {
        gidx_ofs[g] = (int)idx_all.size();
        for (int q : groups[g].cfg) idx_all.push_back(q);
    }
    for (size_t q0 = 0; q0 < pairs2.size(); q0 += MAX_DOT_SHELLS) {
        P2Chunk ch;
        ch.cnt = (int)std::min<size_t>(MAX_DOT_SHELLS, pairs2.size() - q0);
        ch.ofs = (int)table.size();
        ch.lut_ok = true;
        ch.band = 0;
        ch.lut_size = 0;
        for (int x = 0; x < ch.cnt; x++) {
            const Shell& sa = host_shell_of(lid[pairs2[q0 + x]][0]);
            const Shell& sb = host_shell_of(lid[pairs2[q0 + x]][1]);
            table.push_back(sa);
            table.push_back(sb);
            ch.band = std::max(ch.band, std::min(sa.band, sb.band));
            if (sa.kind > SHELL_RANGE || sb.kind > SHELL_RANGE) ch.lut_ok = false;
        }
        for (int x = 0; x < ch.cnt && ch.lut_ok; x++) {
            Shell iv = table[ch.ofs + 2 * x];
            iv.r2lo = std::max(table[ch.ofs + 2 * x].r2lo, table[ch.ofs + 2 * x + 1].r2lo);
            iv.r2hi = std::min(table[ch.ofs + 2 * x].r2hi, table[ch.ofs + 2 * x + 1].r2hi);
            ch.lut_size = std::max(ch.lut_size, iv.r2hi + 1);
            table.push_back(iv);
        }
        ch.idx_ofs = (int)idx_all.size();
        for (int x = 0; x < ch.cnt; x++) idx_all.push_back(pairs2[q0 + x]);
        p2.push_back(ch);
    }

    // ---- device buffers of the plan, scratch of the context sized up front
    Shell* dtable = nullptr;
    PS_TRY(plan_upload(P, &dtable, table));
    int* didx = nullptr;
    PS_TRY(plan_upload(P, &didx, idx_all));
    int *dcsrc = nullptr, *dcdst = nullptr, *dround = nullptr;
    PS_TRY(plan_upload(P, &dcsrc, copy_src));
    PS_TRY(plan_upload(P, &dcdst, copy_dst));
    PS_TRY(plan_upload(P, &dround, direct));
    ClosingDesc* dclose = nullptr;
    PS_TRY(plan_upload(P, &dclose, closing));
    const int nd = (int)derived.size();
    Shell* dderived = nullptr;
    PS_TRY(plan_upload(P, &dderived, derived));
    std::vector<unsigned long long> mm_init(2 * std::max(nd, 1), 0ull);
    for (int q = 0; q < nd; q++) memcpy(&mm_init[2 * q], &derived[q].min2_init, 8);
    unsigned long long *dmm_init = nullptr, *dmm = nullptr;
    PS_TRY(plan_upload(P, &dmm_init, mm_init));
    PS_TRY(plan_alloc(P, &dmm, mm_init.size()));
    double* dkr = nullptr;
    PS_TRY(plan_alloc(P, &dkr, 2 * (size_t)std::max(nd, 1)));
    std::vector<double> coef(nconf);
    for (int q = 0; q < nconf; q++) coef[q] = norm_coef(L, N, cfgs[q].n);
    double* dcoef = nullptr;
    PS_TRY(plan_upload(P, &dcoef, coef));
    const size_t gs = std::max<size_t>(nconf, 2 * MAX_DOT_SHELLS);
    double *sumD = nullptr, *sumI = nullptr, *sumA = nullptr, *gD = nullptr;  // gD: n = 2 chunk sums
    PS_TRY(plan_alloc(P, &sumD, nconf));
    PS_TRY(plan_alloc(P, &sumI, nconf));
    PS_TRY(plan_alloc(P, &sumA, nconf));
    PS_TRY(plan_alloc(P, &gD, gs));
    PS_TRY(plan_alloc(P, &P->dres, 2 * (size_t)nconf));
    PS_TRY(plan_alloc(P, &P->dwb, 6 * (size_t)nconf));
    PS_CK(cudaMemset(P->dwb, 0, 48 * (size_t)nconf));  // entries of non-DERIVED configurations stay 0
    PS_TRY(plan_alloc(P, &P->derr, 1));
    PS_CK(cudaMemset(P->derr, 0, sizeof(int)));
    if (fault_hit(FAULT_ALLOC) ||
        cudaHostAlloc((void**)&P->hres, (10 * (size_t)nconf + 1) * sizeof(double), cudaHostAllocDefault) !=
        cudaSuccess) {
        P->hres = nullptr;
        return fail(PS_ERR_OOM, "pinned result buffer of %d configurations", nconf);
    }
    P->dsumA = sumA;
    P->dsumD = sumD;
    if (!groups.empty()) {
        PS_TRY(ensure_pair_bufs(c, c->f));
        PS_TRY(ensure_pair_bufs(c, c->d));
    }
    {
        const size_t pen32 = (size_t)N * (c->f.S / pw<float>(N)), pen64 = (size_t)N * (c->d.S / pw<double>(N));
        const size_t np = std::max({(size_t)N * N, pen32 * MAX_DOT_SHELLS, pen64 * MAX_DOT_SHELLS,
                                    (size_t)148 * 8 * 2 * MAX_DOT_SHELLS});
        PS_TRY(ensure_partials(c, np));
        PS_TRY(ensure_lut(c, (size_t)3 * (N / 2) * (N / 2) + 2));
        if (!groups.empty()) {
            SideLane lane(c, true);  // the side lane's own scratch, profiling or not
            PS_TRY(ensure_partials(c, np));
            PS_TRY(ensure_lut(c, (size_t)3 * (N / 2) * (N / 2) + 2));
        }
    }
    const double n3 = (double)N * (double)N * (double)N;
    const double pi = ref_pi();
    volatile double big = 1.e30;
    const double min2_init = big * big;
    P->ops.clear();
    auto& ops = P->ops;

    // ---- DERIVED chain
    if (nd > 0) {
        ops.push_back([=]() {
            PS_CK(cudaMemcpyAsync(dmm, dmm_init, 16 * (size_t)nd, cudaMemcpyDeviceToDevice, c->stream));
            int blocks = 1;  // all shells in one launch, sized for the largest
            for (int q = 0; q < nd; q++)
                blocks = std::max(blocks, derived_blocks(derived[q], std::min(derived[q].band, N / 2)));
            {
                Prof pf(c);
                k_derived_ranges<<<dim3(blocks, nd), 256, 0, c->stream>>>(N, dderived, dmm);
                pf.end(KF_DERIVED, 0.0);
            }
            Prof pf(c);
            k_derive_finish<<<(nd + 127) / 128, 128, 0, c->stream>>>(nd, dmm, pi, L, dkr);
            pf.end(KF_DERIVED, 0.0);
            return PS_OK;
        });
    }
    if (!closing.empty()) {
        const int ncl = (int)closing.size();
        const int ncp = (int)copy_src.size();
        int* derr = P->derr;
        double* dwb = P->dwb;
        ops.push_back([=]() {
            Prof pf(c);
            k_closing<<<(ncl + 127) / 128, 128, 0, c->stream>>>(ncl, dclose, dkr, dtable, dwb, pi, L, N, min2_init,
                                                                derr);
            if (ncp > 0) k_copy_shells<<<(ncp + 127) / 128, 128, 0, c->stream>>>(ncp, dcsrc, dcdst, dtable);
            pf.end(KF_DERIVED, 0.0);
            return PS_OK;
        });
    }
    // ---- pair groups, split over the main and the second field lane
    bool prefix_done = false;
    std::vector<std::function<int()>> group_dop(groups.size()), group_iop(groups.size());
    std::vector<int> group_M(groups.size(), 0);
    std::vector<size_t> group_need(groups.size(), 0);
    for (size_t g = 0; g < groups.size(); g++) {
        const Group G = groups[g];
        const Shell sa = host_shell_of(G.a), sb = host_shell_of(G.b);
        int hmax = 0;
        for (int s : G.third) hmax = std::max(hmax, std::min(host_shell_of(s).band, N / 2));
        const int hout = hmax + 1;
        const int ng = (int)G.cfg.size();
        const int go = gofs[g], io = gidx_ofs[g];
        const Shell* hsh = table.data();  // host copy kept alive by the closure below
        std::vector<Shell> gtable(table.begin() + go, table.begin() + go + ng);
        // the group's transforms run on an M-grid on which no triple of its
        // modes aliases (scale of the product spectrum: (N/M)^3): the smallest
        // one, or the fastest candidate when autotuned
        const int ba = std::min(sa.band, N / 2), bb = std::min(sb.band, N / 2);
        // D part (FP32 field products) and I part (FP64 counts on the xy-quadrant:
        // unit filters are even in every axis) of the group on an M-grid
        auto d_part = [=](int M) -> std::function<int()> {
            const double wD = ((double)N / M) * ((double)N / M) * ((double)N / M);
            return [=]() {
                int Sa = 0, ha = 0, Sb = 0, hbb = 0, S = 0;
                PS_TRY(c2r_xy<float>(c, LOAD_MASKED, dtable + G.a, sa.band, c->f.work, &Sa, &ha, 0, M));
                if (G.a != G.b)
                    PS_TRY(c2r_xy<float>(c, LOAD_MASKED, dtable + G.b, sb.band, c->f.work2, &Sb, &hbb, 0, M));
                PS_TRY(pair_spectrum<float>(c, c->f.work, Sa, ha, G.a != G.b ? c->f.work2 : nullptr, Sb, hbb, hout,
                                            &S, 0, M));
                PS_TRY(dot_pass<float>(c, c->f.work3, SPEC_DOT, S, hout, dtable + go, gtable.data(), ng, sumD, 0, M,
                                       wD, didx + io));
                if (kappa)
                    PS_TRY(dot_pass<float>(c, c->f.work3, SPEC_DOT_ABS, S, hout, dtable + go, gtable.data(), ng, sumA,
                                           0, M, wD, didx + io));
                return PS_OK;
            };
        };
        // exact counts by enumeration when every shell of the group is an r^2
        // interval known on the host (closing shells may come from the DERIVED
        // chain: their intervals are read on the device); else FP64 transforms
        bool enum_counts = !(P->flags & PS_PLAN_FFT_COUNTS) && uniq[G.a].tag == 0 && uniq[G.b].tag == 0 &&
                           (sa.kind == SHELL_DEFAULT || sa.kind == SHELL_RANGE) &&
                           (sb.kind == SHELL_DEFAULT || sb.kind == SHELL_RANGE);
        for (int s3 : G.third) {
            const Shell& h3 = host_shell_of(s3);
            enum_counts = enum_counts && (h3.kind == SHELL_DEFAULT || h3.kind == SHELL_RANGE);
        }
        PairCountLists lists;
        if (enum_counts) enum_counts = pair_count_lists(sa, sb, N, &lists);
        int4* dreps = nullptr;
        short4* dmodes = nullptr;
        unsigned long long* dcounts = nullptr;
        if (enum_counts) {
            PS_TRY(plan_upload(P, &dreps, lists.reps));
            PS_TRY(plan_upload(P, &dmodes, lists.modes));
            PS_TRY(plan_alloc(P, &dcounts, (size_t)ng));
        }
        const int nrep = (int)lists.reps.size(), nmodes = (int)lists.modes.size();
        const int s_lo = lists.s_lo, nbins = lists.nbins;
        const bool wrap = lists.wrap;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        // one CTA of kCountThreads per SM over about eight work items each: the
        // count lane runs beside the field load and the field lanes, and one
        // histogram per SM leaves the rest of each SM's shared memory to their
        // passes
        const size_t csmem = kCountStageBytes + (size_t)nbins * sizeof(unsigned int);
        int cgrid = 1, rep_slice = kCountRepChunk;
        if (enum_counts) {
            // the shared-memory limit is a property of the kernel, not of a
            // launch (every group's launch, replayed from a graph too, must fit
            // under it): the largest histogram any group may have
            constexpr int kLimit = (int)(kCountStageBytes + kCountMaxBins * sizeof(unsigned int));
            PS_CK(cudaFuncSetAttribute(k_pair_counts<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLimit));
            PS_CK(cudaFuncSetAttribute(k_pair_counts<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLimit));
            const int nmc = (nmodes + kCountThreads * kCountBPT - 1) / (kCountThreads * kCountBPT);
            const int nrs = std::min(nrep, std::max(1, (8 * sms + nmc - 1) / nmc));
            rep_slice = std::min(kCountRepChunk, std::max(8, (nrep + nrs - 1) / nrs));
            const int nitems = nmc * ((nrep + rep_slice - 1) / rep_slice);
            cgrid = std::max(1, std::min(nitems, sms));
        }
        auto enum_part = [=]() -> int {
            PS_CK(cudaMemsetAsync(dcounts, 0, sizeof(unsigned long long) * ng, c->stream));
            Prof pf(c);
            if (wrap)
                k_pair_counts<true><<<cgrid, kCountThreads, csmem, c->stream>>>(
                    dreps, nrep, dmodes, nmodes, N, s_lo, nbins, rep_slice, dtable + go, ng, dcounts);
            else
                k_pair_counts<false><<<cgrid, kCountThreads, csmem, c->stream>>>(
                    dreps, nrep, dmodes, nmodes, N, s_lo, nbins, rep_slice, dtable + go, ng, dcounts);
            pf.end(KF_PAIR_COUNTS, 8.0 * nmodes + 16.0 * nrep);
            k_counts_out<<<(ng + 127) / 128, 128, 0, c->stream>>>(ng, dcounts, didx + io, sumI);
            PS_CK(launch_status());
            return PS_OK;
        };
        auto i_part = [=](int M) -> std::function<int()> {
            if (enum_counts) return enum_part;
            return [=]() {
                int Sa = 0, ha = 0, Sb = 0, hbb = 0, S = 0;
                PS_TRY(c2r_xy<double>(c, LOAD_UNIT, dtable + G.a, sa.band, c->d.work, &Sa, &ha, 1, M));
                if (G.a != G.b)
                    PS_TRY(c2r_xy<double>(c, LOAD_UNIT, dtable + G.b, sb.band, c->d.work2, &Sb, &hbb, 1, M));
                PS_TRY(pair_spectrum<double>(c, c->d.work, Sa, ha, G.a != G.b ? c->d.work2 : nullptr, Sb, hbb, hout,
                                             &S, 1, M));
                PS_TRY(dot_pass<double>(c, c->d.work3, SPEC_COUNT, S, hout, dtable + go, gtable.data(), ng, sumI, 1,
                                        M, 1.0, didx + io));
                return PS_OK;
            };
        };
        auto group_op = [=](int M) -> std::function<int()> {
            const auto dp = d_part(M), ip = i_part(M);
            return [=]() {
                PS_TRY(dp());
                return ip();
            };
        };
        int M = alias_free_grid(N, ba, bb, hmax);
        const std::array<int, 4> key = {N, ba, bb, hmax};
        auto known = c->tune_grid.find(key);
        if (known != c->tune_grid.end() && known->second >= M && known->second <= N && grid_supported(known->second)) {
            M = known->second;
        } else if (P->flags & PS_PLAN_AUTOTUNE) {
            if (!prefix_done) {  // the DERIVED chain fills the closing shells the candidates read
                for (auto& op : ops) PS_TRY(op());
                prefix_done = true;
            }
            PS_TRY(tune_grid(c, group_op, M, &M));
            c->tune_grid[key] = M;
        }
        if (M < N) {
            Tables<float> t32;
            Tables<double> t64;
            PS_TRY(tables_for<float>(c, M, &t32));
            PS_TRY(tables_for<double>(c, M, &t64));
        }
        if (P->flags & PS_PLAN_AUTOTUNE) {  // the FP32 pair kernel variant and dot pass geometry of this size
            PS_TRY(tune_pair(c, M, std::min(sa.band, M / 2) + 1, G.a != G.b ? std::min(sb.band, M / 2) + 1 : 0,
                             hout));
            if (!c->dot_alt.count(M)) {
                if (!prefix_done) {  // the DERIVED chain fills the closing shells the group reads
                    for (auto& op : ops) PS_TRY(op());
                    prefix_done = true;
                }
                PS_TRY(tune_dot(c, d_part(M), M));
            }
        }
        group_dop[g] = d_part(M);
        group_iop[g] = i_part(M);
        group_M[g] = M;
        {   // FP32 work spectra the group's field part writes on its M-grid
            const int w32 = pw<float>(M);
            const int s_ab = round_up(std::max(std::min(sa.band, M / 2), std::min(sb.band, M / 2)) + 1, w32);
            group_need[g] = (size_t)M * M * (size_t)std::max(s_ab, round_up(hout, w32));
        }
        (void)hsh;
    }
    if (P->flags & PS_PLAN_AUTOTUNE) {  // the FP32 Y pass geometry of the pair groups' transform sizes
        for (size_t g = 0; g < groups.size(); g++) PS_TRY(tune_pencil(c, group_M[g]));
    }
    // lanes: the groups by decreasing transform volume, each onto the less
    // loaded of the main and the second field lane (one lane when profiling
    // or with a single group)
    std::vector<int> group_lane(groups.size(), 0);
    if (groups.size() > 1) {
        std::vector<size_t> order(groups.size());
        for (size_t g = 0; g < groups.size(); g++) order[g] = g;
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t x, size_t y) { return group_M[x] > group_M[y]; });
        double load[2] = {0.0, 0.0};
        size_t need2 = 0;
        for (size_t g : order) {
            const int l = load[1] < load[0] ? 1 : 0;
            group_lane[g] = l;
            load[l] += (double)group_M[g] * group_M[g] * group_M[g];
            if (l == 1) need2 = std::max(need2, group_need[g]);
        }
        if (need2 > 0) {
            PS_TRY(ensure_lane2_work(c, need2));
            const size_t pen32 = (size_t)N * (c->f.S / pw<float>(N));
            const size_t np = std::max({(size_t)N * N, pen32 * MAX_DOT_SHELLS, (size_t)148 * 8 * 2 * MAX_DOT_SHELLS});
            Lane2 lane(c, true);  // the second lane's own scratch, profiling or not
            PS_TRY(ensure_partials(c, np));
            PS_TRY(ensure_lut(c, (size_t)3 * (N / 2) * (N / 2) + 2));
        }
    }
    // the groups' counts (run on the side lane) and field parts (main or
    // second lane); the lanes are forked and joined where the parts are enqueued
    P->has_groups = !groups.empty();
    for (size_t g = 0; g < groups.size(); g++) {
        const auto dop = group_dop[g];
        const bool second = group_lane[g] == 1;
        P->ops_counts.push_back(group_iop[g]);
        P->ops_groups.push_back([=]() {
            if (second) {
                Lane2 lane(c);
                return dop();
            }
            return dop();
        });
    }
    auto& tail = P->ops_tail;
    // ---- n = 2 (Parseval): one k-space pass per chunk
    for (const P2Chunk ch : p2) {
        tail.push_back([=]() {
            const unsigned short* lut = nullptr;
            if (ch.lut_ok) {
                Prof pf(c);
                if (ch.lut_size > 0)
                    k_shell_lut<<<(ch.lut_size + 255) / 256, 256, 0, c->stream>>>(dtable + ch.ofs + 2 * ch.cnt, ch.cnt,
                                                                                   ch.lut_size, c->dlut);
                pf.end(KF_LUT, 2.0 * ch.lut_size);
                lut = c->dlut;
            }
            const int b = std::min(ch.band, N / 2);
            const long long modes = (long long)(2 * b + 1) * (2 * b + 1) * (b + 1);
            const int blocks = (int)std::max<long long>(1, std::min<long long>((modes + 255) / 256, 148 * 8));
            {
                Prof pf(c);
                k_pair2_sums<float><<<blocks, 256, 0, c->stream>>>(N, c->f.spec, c->f.S, lut, ch.lut_size, dtable + ch.ofs,
                                                                   ch.cnt, b, c->partials);
                pf.end(KF_PAIR2, (double)modes * sizeof(V2<float>));
            }
            PS_TRY(sum_partials_n(c, blocks, 2 * MAX_DOT_SHELLS, gD));
            PS_TRY(scatter_dev(c, gD, didx + ch.idx_ofs, ch.cnt, sumD));
            PS_TRY(scatter_dev(c, gD + MAX_DOT_SHELLS, didx + ch.idx_ofs, ch.cnt, sumI));
            return PS_OK;
        });
    }
    // ---- leg by leg (singletons, n > 3): running products with powers
    for (int q : direct) {
        std::vector<std::pair<int, int>> up;  // (shell, multiplicity)
        for (int sidx : lid[q]) {
            bool found = false;
            for (auto& pr : up)
                if (pr.first == sidx) { pr.second++; found = true; }
            if (!found) up.push_back({sidx, 1});
        }
        std::vector<int> bands;
        for (auto& pr : up) bands.push_back(host_shell_of(pr.first).band);
        tail.push_back([=]() {
            const int r = (int)up.size();
            for (int pass = 0; pass < 2; pass++)
                for (int x = 0; x < r; x++) {
                    const int epi = r == 1 ? EPI_REDUCE : (x == 0 ? EPI_STORE : (x < r - 1 ? EPI_MUL_STORE : EPI_MUL_REDUCE));
                    if (pass == 0) {
                        PS_TRY(c2r_shell<float>(c, LOAD_MASKED, dtable + up[x].first, bands[x], c->f.ra, c->f.ra, epi,
                                                up[x].second, sumD + q));
                        if (kappa && x == r - 1)
                            PS_TRY(c2r_shell<float>(c, LOAD_MASKED, dtable + up[x].first, bands[x], c->f.ra, c->f.ra,
                                                    r == 1 ? EPI_REDUCE_ABS : EPI_MUL_REDUCE_ABS, up[x].second,
                                                    sumA + q));
                    } else {
                        PS_TRY(c2r_shell<double>(c, LOAD_UNIT, dtable + up[x].first, bands[x], c->d.ra, c->d.ra, epi,
                                                 up[x].second, sumI + q));
                    }
                }
            return PS_OK;
        });
    }
    if (!direct.empty()) {
        const int nr = (int)direct.size();
        tail.push_back([=]() {
            Prof pf(c);
            k_round_counts<<<(nr + 127) / 128, 128, 0, c->stream>>>(nr, dround, sumI, n3);
            pf.end(KF_FINAL, 0.0);
            return PS_OK;
        });
    }
    double* dres = P->dres;
    tail.push_back([=]() {
        Prof pf(c);
        k_finalize<<<(nconf + 127) / 128, 128, 0, c->stream>>>(nconf, dcoef, sumD, sumI, 1.0 / n3, 1, dres);
        pf.end(KF_FINAL, 0.0);
        PS_CK(launch_status());
        return PS_OK;
    });
    return PS_OK;
}

// The plan's parts (ps_gpu_plan::parts): 0 DERIVED chain, 1 counts, 2 the
// groups' field parts with the second lane forked and joined, 3 the tail.
enum PlanPart : int { PART_DERIVED = 0, PART_COUNTS = 1, PART_GROUPS = 2, PART_TAIL = 3 };

int enqueue_ops(const std::vector<std::function<int()>>& ops)
{
    for (auto& op : ops) PS_TRY(op());
    return PS_OK;
}

int enqueue_part(ps_gpu_ctx* c, ps_gpu_plan* P, int part)
{
    switch (part) {
    case PART_DERIVED:
        return enqueue_ops(P->ops);
    case PART_COUNTS:
        return enqueue_ops(P->ops_counts);
    case PART_GROUPS:
        if (P->has_groups && !c->prof_on) {
            PS_CK(cudaEventRecord(c->ev_fork, c->stream));
            PS_CK(cudaStreamWaitEvent(c->lane2_stream, c->ev_fork, 0));
        }
        PS_TRY(enqueue_ops(P->ops_groups));
        if (P->has_groups && !c->prof_on) {
            PS_CK(cudaEventRecord(c->ev_join2, c->lane2_stream));
            PS_CK(cudaStreamWaitEvent(c->stream, c->ev_join2, 0));
        }
        return PS_OK;
    default:
        return enqueue_ops(P->ops_tail);
    }
}

// The whole execution on the context's stream: the DERIVED chain, then the
// counts on the side lane beside the groups' field parts, then the tail.
int plan_enqueue(ps_gpu_ctx* c, ps_gpu_plan* P)
{
    if (P->prepared) {  // a prepared part may still write the plan's tables and counts
        PS_CK(cudaStreamWaitEvent(c->stream, P->ev_counts, 0));
        P->prepared = false;
    }
    PS_TRY(enqueue_part(c, P, PART_DERIVED));
    if (P->has_groups) {  // fork the side lane after the DERIVED chain the counts read
        PS_CK(cudaEventRecord(c->ev_fork, c->stream));
        PS_CK(cudaStreamWaitEvent(c->side_stream, c->ev_fork, 0));
        {
            SideLane lane(c);
            PS_TRY(enqueue_part(c, P, PART_COUNTS));
        }
        PS_TRY(enqueue_part(c, P, PART_GROUPS));
        PS_CK(cudaEventRecord(c->ev_join, c->side_stream));
        PS_CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    }
    return enqueue_part(c, P, PART_TAIL);
}

// Results of an executed batched plan: device -> pinned host copy (stream
// ordered), then unpacked on the host into the caller's arrays.
int plan_copy_results(ps_gpu_ctx* c, ps_gpu_plan* P, double* h)
{
    const size_t n = (size_t)P->nconf;
    PS_CK(cudaMemcpyAsync(h, P->dres, 16 * n, cudaMemcpyDeviceToHost, c->stream));
    PS_CK(cudaMemcpyAsync(h + 2 * n, P->dwb, 48 * n, cudaMemcpyDeviceToHost, c->stream));
    if (P->flags & PS_PLAN_KAPPA) {
        PS_CK(cudaMemcpyAsync(h + 8 * n, P->dsumA, 8 * n, cudaMemcpyDeviceToHost, c->stream));
        PS_CK(cudaMemcpyAsync(h + 9 * n, P->dsumD, 8 * n, cudaMemcpyDeviceToHost, c->stream));
    }
    PS_CK(cudaMemcpyAsync(h + 10 * n, P->derr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    return PS_OK;
}

// Host side of a finished execution whose results were copied to h (no CUDA calls).
int plan_unpack(const ps_gpu_plan* P, const double* h, double* B, double* Np, double* kappa, ps_cfg* cfgs_out)
{
    const int nconf = P->nconf;
    int err = 0;
    memcpy(&err, h + 10 * (size_t)nconf, sizeof(int));
    for (int q = 0; q < nconf; q++) {
        B[q] = h[2 * q];
        Np[q] = h[2 * q + 1];
        if (kappa) kappa[q] = P->cfgs[q].n == 2 ? 1.0 : h[8 * (size_t)nconf + q] / fabs(h[9 * (size_t)nconf + q]);
    }
    if (cfgs_out) {
        const double* wb = h + 2 * (size_t)nconf;
        for (int q = 0; q < nconf; q++) cfgs_out[q] = P->cfgs[q];
        for (int q : P->derived_cfgs) {
            for (int l = 0; l < 3; l++) {
                cfgs_out[q].kmin[l] = wb[6 * q + 2 * l];
                cfgs_out[q].kmax[l] = wb[6 * q + 2 * l + 1];
            }
        }
    }
    return err ? PS_ERR_CUDA : PS_OK;
}

int plan_finish(ps_gpu_ctx* c, ps_gpu_plan* P, double* B, double* Np, double* kappa, ps_cfg* cfgs_out)
{
    PS_TRY(plan_copy_results(c, P, P->hres));
    PS_CK(cudaStreamSynchronize(c->stream));
    if (plan_unpack(P, P->hres, B, Np, kappa, cfgs_out) != PS_OK)
        return fail(PS_ERR_CUDA, "internal: a derived shell exceeded its launch bound");
    return PS_OK;
}

// Unpacks the asynchronous submissions whose result copies are done, oldest
// first (with wait, all of them, waiting for each); their page-locked buffers
// and events go back to the context's spares.
int drain_pending(ps_gpu_ctx* c, bool wait)
{
    size_t k = 0;
    int rc = PS_OK;
    for (; k < c->pending.size(); k++) {
        PendingSubmit& j = c->pending[k];
        const cudaError_t e = wait ? cudaEventSynchronize(j.done) : cudaEventQuery(j.done);
        if (e == cudaErrorNotReady) break;
        if (e != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "asynchronous submission: %s", cudaGetErrorString(e));
            break;
        }
        if (plan_unpack(j.P, j.host, j.B, j.Np, j.kappa, j.cfgs_out) != PS_OK) {
            int expected = 0;
            c->async_err.compare_exchange_strong(expected, PS_ERR_CUDA);
        }
        c->spare_host.push_back({j.host, j.host_len});
        c->spare_events.push_back(j.done);
    }
    c->pending.erase(c->pending.begin(), c->pending.begin() + (long)k);
    return rc;
}

// Page-locked result buffer of at least len doubles and an event for one submission.
int submit_slot(ps_gpu_ctx* c, size_t len, double** host, cudaEvent_t* ev)
{
    *host = nullptr;
    for (size_t q = 0; q < c->spare_host.size(); q++)
        if (c->spare_host[q].second >= len) {
            *host = c->spare_host[q].first;
            c->spare_host.erase(c->spare_host.begin() + (long)q);
            break;
        }
    if (!*host) {
        if (fault_hit(FAULT_ALLOC) || cudaHostAlloc((void**)host, len * sizeof(double), cudaHostAllocDefault) != cudaSuccess) {
            *host = nullptr;
            return fail(PS_ERR_OOM, "page-locked result buffer of %zu doubles", len);
        }
    }
    if (!c->spare_events.empty()) {
        *ev = c->spare_events.back();
        c->spare_events.pop_back();
    } else if (cudaEventCreateWithFlags(ev, cudaEventDisableTiming) != cudaSuccess) {
        c->spare_host.push_back({*host, len});
        return fail(PS_ERR_CUDA, "event creation failed");
    }
    return PS_OK;
}

// Device and pinned memory of a plan (the plan object itself stays).
void plan_release(ps_gpu_plan* P)
{
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    P->exec = nullptr;
    P->graph = nullptr;
    for (auto& q : P->parts) {
        if (q.exec) cudaGraphExecDestroy(q.exec);
        if (q.graph) cudaGraphDestroy(q.graph);
        q = ps_gpu_plan::Part{};
    }
    for (cudaEvent_t* e : {&P->ev_prep, &P->ev_derived, &P->ev_counts}) {
        if (*e) cudaEventDestroy(*e);
        *e = nullptr;
    }
    P->prepared = false;
    P->ops_counts.clear();
    P->ops_groups.clear();
    P->ops_tail.clear();
    for (void* p : P->owned) cudaFree(p);
    P->owned.clear();
    if (P->hres) cudaFreeHost(P->hres);
    P->hres = nullptr;
    P->ops.clear();
}

void plan_free(ps_gpu_plan* P)
{
    if (!P) return;
    plan_release(P);
    delete P;
}

// Captures fn's stream work on the context's current stream into *g / *x
// (first use), then launches it there; kernels counted once per launch.
int capture_launch(ps_gpu_ctx* c, cudaGraph_t* g, cudaGraphExec_t* x, long long* nlaunch,
                   const std::function<int()>& fn)
{
    if (!*x) {
        c->capturing = true;
        const long long before = c->launches;
        cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            c->capturing = false;
            return fail(PS_ERR_CUDA, "cudaStreamBeginCapture: %s", cudaGetErrorString(e));
        }
        const int rc = fn();
        cudaGraph_t gr = nullptr;
        e = cudaStreamEndCapture(c->stream, &gr);
        c->capturing = false;
        if (rc != PS_OK) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
        }
        if (e != cudaSuccess) return fail(PS_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
        *g = gr;
        *nlaunch = c->launches - before;
        c->launches = before;
        PS_CK(cudaGraphInstantiate(x, gr, 0));
    }
    PS_CK(cudaGraphLaunch(*x, c->stream));
    c->launches += *nlaunch;
    c->launches_total += *nlaunch;
    return PS_OK;
}

// One part on the context's current stream: replayed from its graph
// (PS_PLAN_GRAPH) or enqueued launch by launch.
int run_part(ps_gpu_ctx* c, ps_gpu_plan* P, int part)
{
    if (!(P->flags & PS_PLAN_GRAPH)) return enqueue_part(c, P, part);
    ps_gpu_plan::Part& q = P->parts[part];
    return capture_launch(c, &q.graph, &q.exec, &q.launches, [=]() { return enqueue_part(c, P, part); });
}

// One execution of the plan on the context's stream.  After
// ps_gpu_plan_prepare: the groups' field parts wait for the prepared DERIVED
// chain, the tail for the prepared counts.  Else the whole sequence, replayed
// from one graph (PS_PLAN_GRAPH) or enqueued launch by launch.
int plan_run(ps_gpu_ctx* c, ps_gpu_plan* P)
{
    if (P->prepared) {
        P->prepared = false;
        PS_CK(cudaStreamWaitEvent(c->stream, P->ev_derived, 0));
        PS_TRY(run_part(c, P, PART_GROUPS));
        PS_CK(cudaStreamWaitEvent(c->stream, P->ev_counts, 0));
        return run_part(c, P, PART_TAIL);
    }
    if (!(P->flags & PS_PLAN_GRAPH)) return plan_enqueue(c, P);
    return capture_launch(c, &P->graph, &P->exec, &P->graph_launches, [=]() { return plan_enqueue(c, P); });
}

// Enqueues the field-independent parts of the plan's next execution (the
// DERIVED chain and the exact counts) on the side lane, after the work
// already on the context's stream.
int plan_prepare(ps_gpu_ctx* c, ps_gpu_plan* P)
{
    for (cudaEvent_t* e : {&P->ev_prep, &P->ev_derived, &P->ev_counts})
        if (!*e) PS_CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    PS_CK(cudaEventRecord(P->ev_prep, c->stream));
    PS_CK(cudaStreamWaitEvent(c->side_stream, P->ev_prep, 0));
    SideLane lane(c, true);
    PS_TRY(run_part(c, P, PART_DERIVED));
    PS_CK(cudaEventRecord(P->ev_derived, c->stream));
    PS_TRY(run_part(c, P, PART_COUNTS));
    PS_CK(cudaEventRecord(P->ev_counts, c->stream));
    P->prepared = true;
    return PS_OK;
}

int batched(ps_gpu_ctx* c, int nconf, ps_cfg* cfgs, double* B, double* Np, double* kappa)
{
    if (!c->f.have_spec) return fail(PS_ERR_ARG, "FP32 spectrum not available (methods mask)");
    ps_gpu_plan* P = new ps_gpu_plan();
    P->ctx = c;
    P->method = PS_FP32_BATCHED;
    P->nconf = nconf;
    P->flags = kappa ? PS_PLAN_KAPPA : 0;
    P->cfgs.assign(cfgs, cfgs + nconf);
    int rc = plan_batched(c, P);
    if (rc == PS_OK) rc = check_band(c, P->band);
    if (rc == PS_OK) rc = plan_enqueue(c, P);
    if (rc == PS_OK) rc = plan_finish(c, P, B, Np, kappa, cfgs);
    plan_free(P);
    return rc;
}

// =========================================================================
// adjoint: dB/d(delta) = c/sumI * c2r( sum_i F_i * FFT[prod_{j != i} D_j] )
// =========================================================================
template <typename T>
int grad_impl(ps_gpu_ctx* c, int n, const std::vector<Shell>& legs, double scale, void* out, int out_is_double,
              int out_mem)
{
    PrecBufs<T>& B = bufs<T>(c);
    const int N = c->N;
    const size_t nspec = (size_t)N * N * B.S;
    const size_t n3 = (size_t)N * N * N;
    PS_TRY(ensure_pair_bufs(c, B));
    PS_TRY(alloc_dev(&B.hacc, nspec));
    PS_TRY(ensure_shells(c, PS_MAX_LEGS));
    PS_CK(cudaMemcpyAsync(c->dshells, legs.data(), sizeof(Shell) * n, cudaMemcpyHostToDevice, c->stream));
    PS_CK(cudaMemsetAsync(B.hacc, 0, sizeof(V2<T>) * nspec, c->stream));
    int hb = 1;
    for (int l = 0; l < n; l++) hb = std::max(hb, std::min(legs[l].band, N / 2) + 1);
    if (n == 2) {
        Prof pf(c);
        k_grad_pair2<T><<<148 * 8, 256, 0, c->stream>>>(N, B.spec, B.S, c->dshells, B.hacc, B.S, hb);
        pf.end(fam<T>(KF_GRAD), 2.0 * N * N * hb * sizeof(V2<T>), N);
    } else {
        // leg i: FFT of the product of the other two legs, masked by F_i;
        // identical (mask, pair) terms are folded into one with a weight
        std::vector<std::pair<std::vector<int>, int>> terms;
        for (int i = 0; i < 3; i++) {
            std::vector<int> key = {i, (i + 1) % 3, (i + 2) % 3};
            if (key[1] > key[2]) std::swap(key[1], key[2]);
            bool found = false;
            for (auto& tm : terms) {
                const auto& k0 = tm.first;
                if (same_shell(legs[k0[0]], legs[key[0]]) &&
                    ((same_shell(legs[k0[1]], legs[key[1]]) && same_shell(legs[k0[2]], legs[key[2]])) ||
                     (same_shell(legs[k0[1]], legs[key[2]]) && same_shell(legs[k0[2]], legs[key[1]])))) {
                    tm.second++;
                    found = true;
                    break;
                }
            }
            if (!found) terms.push_back({key, 1});
        }
        for (const auto& tm : terms) {
            const int li = tm.first[0], la = tm.first[1], lb = tm.first[2];
            const bool same = same_shell(legs[la], legs[lb]);
            int Sa = 0, ha = 0, Sb = 0, hbb = 0, S = 0;
            PS_TRY(c2r_xy<T>(c, LOAD_MASKED, c->dshells + la, legs[la].band, B.work, &Sa, &ha));
            if (!same) PS_TRY(c2r_xy<T>(c, LOAD_MASKED, c->dshells + lb, legs[lb].band, B.work2, &Sb, &hbb));
            const int hout = std::min(legs[li].band, N / 2) + 1;
            PS_TRY(pair_spectrum<T>(c, B.work, Sa, ha, same ? nullptr : B.work2, Sb, hbb, hout, &S));
            Prof pf(c);
            PS_SWITCH_N(N, PS_TRY((L3<T, NN>::fwd_x(c->stream, B.work3, S, hout, SPEC_MASK_ADD, B.hacc, B.S, nullptr,
                                                    0, c->dshells + li, 1, nullptr, 0, nullptr, B.tables(),
                                                    nullptr, (double)tm.second))));
            pf.end(fam<T>(KF_GRAD), 3.0 * N * N * S * sizeof(V2<T>), N);
        }
    }
    if (c->use_only_phase == 1) {  // the field entered through z/|z|
        Prof pf(c);
        k_phase_adjoint<T><<<148 * 8, 256, 0, c->stream>>>((size_t)N * N, hb, B.hacc, B.S, B.spec, B.mod);
        pf.end(fam<T>(KF_GRAD), 4.0 * N * N * hb * sizeof(V2<T>), N);
    }
    // inverse transform of the accumulated spectrum into B.ra, then scale
    const int S = round_up(hb, pw<T>(N));
    int nb = 0;
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::inv_x(c->stream, B.hacc, B.S, B.work, S, LOAD_PLAIN, nullptr, hb, B.tables()))));
        pf.end(fam<T>(KF_INV_X), 2.0 * N * N * S * sizeof(V2<T>), N);
    }
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::pass_y(c->stream, B.work, S, true, B.tables()))));
        pf.end(fam<T>(KF_PASS_Y), 2.0 * N * N * S * sizeof(V2<T>), N);
    }
    {
        Prof pf(c);
        PS_SWITCH_N(N, PS_TRY((L3<T, NN>::inv_z(c->stream, B.work, S, hb, B.ra, nullptr, EPI_STORE, 1, nullptr,
                                                B.tables(), &nb))));
        pf.end(fam<T>(KF_INV_Z), (double)N * N * hb * sizeof(V2<T>) + (double)n3 * sizeof(T), N);
    }
    void* dst = out;
    void* stage = nullptr;
    const size_t out_bytes = n3 * (out_is_double ? 8 : 4);
    if (out_mem == PS_MEM_HOST) {
        PS_TRY(alloc_dev((unsigned char**)&stage, out_bytes));
        dst = stage;
    }
    {
        Prof pf(c);
        if (out_is_double)
            k_scale_out<T, double><<<148 * 8, 256, 0, c->stream>>>(B.ra, (double*)dst, n3, scale);
        else
            k_scale_out<T, float><<<148 * 8, 256, 0, c->stream>>>(B.ra, (float*)dst, n3, scale);
        pf.end(fam<T>(KF_GRAD), (double)n3 * (sizeof(T) + (out_is_double ? 8 : 4)), N);
    }
    cudaError_t e = launch_status();
    if (e == cudaSuccess && stage) {
        e = cudaMemcpyAsync(out, stage, out_bytes, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(stage);
    PS_CK(e);
    return PS_OK;
}

// PS_ERR_TIMEOUT (and the word cleared) when a kernel's bounded wait on this
// context's stream expired; call after the stream work it covers is done.
int check_status(ps_gpu_ctx* c)
{
    int h = 0;
    PS_CK(cudaMemcpyAsync(&h, c->dstatus, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PS_CK(cudaStreamSynchronize(c->stream));
    if (h) {
        PS_CK(cudaMemsetAsync(c->dstatus, 0, sizeof(int), c->stream));
        c->f.have_spec = c->d.have_spec = false;  // the field spectrum is incomplete
        c->field_set = false;
        return fail(PS_ERR_TIMEOUT, "a bulk copy into shared memory did not complete within its wait limit");
    }
    return PS_OK;
}

int timed_begin(ps_gpu_ctx* c)
{
    c->launches = 0;
    PS_CK(cudaEventRecord(c->ev0, c->stream));
    return PS_OK;
}
int timed_end(ps_gpu_ctx* c)
{
    PS_CK(cudaEventRecord(c->ev1, c->stream));
    PS_CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    PS_CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms = ms;
    return PS_OK;
}

// Field load (get_FT_field, input_field.c:40-81) as stream work: host arrays
// are copied on the copy stream into one of two staging slots, the forward
// transform waits for that copy on the compute stream, so the upload of the
// next field overlaps the work still queued on the current one.
int ensure_stage(ps_gpu_ctx* c, size_t bytes);
int transform_field(ps_gpu_ctx* c, const void* a, const void* b, int is_double, int use_only_phase, int s,
                    size_t split = 0);

// dens * (1 - xhii) rounded to float, each value exactly as the r2c loader
// computes it (double product and difference, input_field.c:33, then one
// rounding), on host threads.
void compose_xhi_dens(ps_gpu_ctx* c, const float* d, const float* x, float* out, size_t n)
{
    (void)c;
    HostPool& pool = HostPool::get();
    const size_t nt = pool.n, per = (n + nt - 1) / nt;
    pool.run([=](size_t t) {
        const size_t lo = std::min(n, t * per), hi = std::min(n, lo + per);
        for (size_t i = lo; i < hi; i++) out[i] = (float)((double)d[i] * (1.0 - (double)x[i]));
    });
}

// Host XHI_DENS field of an FP32-only context.  The first `split` rows go up
// as they are (dens and xHII, the copy engine starts on them at once) while
// host threads compose dens*(1 - xHII) of the other rows, chunk by chunk, into
// one of two page-locked buffers, each chunk uploaded as soon as it is done:
// composed rows cross PCIe at half the bytes, raw rows cost no host time, and
// the split is re-balanced after every load from the measured compose and
// copy rates (raw rows only from page-locked inputs).  Every composed value
// equals the r2c loader's, so the spectrum and all results are bit-identical
// to the two-array upload.
int load_xhi_dens_host(ps_gpu_ctx* c, const float* dens, const float* xhii, int use_only_phase)
{
    const int N = c->N;
    const size_t nr = (size_t)N * N, n3 = nr * N;
    const size_t bytes = n3 * sizeof(float);
    if (c->fpin_bytes < bytes) {
        for (int q = 0; q < 2; q++) {
            if (c->ev_fpin[q]) PS_CK(cudaEventSynchronize(c->ev_fpin[q]));
            if (c->fpin[q]) cudaFreeHost(c->fpin[q]);
            c->fpin[q] = nullptr;
        }
        c->fpin_bytes = 0;
        for (int q = 0; q < 2; q++)
            if (fault_hit(FAULT_ALLOC) || cudaHostAlloc(&c->fpin[q], bytes, cudaHostAllocDefault) != cudaSuccess) {
                c->fpin[q] = nullptr;
                return fail(PS_ERR_OOM, "page-locked field buffer of %zu bytes", bytes);
            }
        c->fpin_bytes = bytes;
    }
    for (int q = 0; q < 2; q++)
        if (!c->ev_fpin[q]) PS_CK(cudaEventCreateWithFlags(&c->ev_fpin[q], cudaEventDisableTiming));
    if (!c->ev_raw[0])
        for (int q = 0; q < 2; q++) PS_CK(cudaEventCreate(&c->ev_raw[q]));
    PS_TRY(ensure_stage(c, bytes));
    // raw rows only when both inputs are page-locked (a pageable copy would
    // hold the host thread until it is done)
    auto pinned = [](const void* p) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();  // the failed query's own error, not a kernel's
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    const bool raw_ok = pinned(dens) && pinned(xhii);
    constexpr size_t kAlign = 64;  // rows per split step (a multiple of every r2c row tile)
    size_t split = raw_ok ? (size_t)(c->raw_frac * (double)nr) / kAlign * kAlign : 0;
    split = std::min(split, nr);
    const int q = c->fslot;
    c->fslot ^= 1;
    PS_CK(cudaEventSynchronize(c->ev_fpin[q]));  // the upload that last read buffer q
    const int s = c->slot;
    c->slot ^= 1;
    PS_CK(cudaStreamWaitEvent(c->copy_stream, c->ev_free[s], 0));
    float* d0 = (float*)c->stage[s][0];
    float* d1 = (float*)c->stage[s][1];
    float* hp = (float*)c->fpin[q];
    if (split > 0) {
        PS_CK(cudaEventRecord(c->ev_raw[0], c->copy_stream));
        PS_CK(cudaMemcpyAsync(d0, dens, split * N * sizeof(float), cudaMemcpyHostToDevice, c->copy_stream));
        PS_CK(cudaMemcpyAsync(d1, xhii, split * N * sizeof(float), cudaMemcpyHostToDevice, c->copy_stream));
        PS_CK(cudaEventRecord(c->ev_raw[1], c->copy_stream));
    }
    const auto t0 = std::chrono::steady_clock::now();
    // composed rows in 8 uploads: each chunk's copy overlaps the next chunk's composition
    const size_t chunk = std::max<size_t>(kAlign, ((nr - split + 7) / 8 + kAlign - 1) / kAlign * kAlign);
    for (size_t r0 = split; r0 < nr; r0 += chunk) {
        const size_t r1 = std::min(nr, r0 + chunk);
        compose_xhi_dens(c, dens + r0 * N, xhii + r0 * N, hp + r0 * N, (r1 - r0) * N);
        PS_CK(cudaMemcpyAsync(d0 + r0 * N, hp + r0 * N, (r1 - r0) * N * sizeof(float), cudaMemcpyHostToDevice,
                              c->copy_stream));
    }
    const double t_comp = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    PS_CK(cudaEventRecord(c->ev_fpin[q], c->copy_stream));
    PS_CK(cudaEventRecord(c->ev_copied[s], c->copy_stream));
    PS_CK(cudaStreamWaitEvent(c->stream, c->ev_copied[s], 0));
    c->upload_bytes = (2 * split * N + (nr - split) * N) * sizeof(float);
    PS_TRY(transform_field(c, d0, split > 0 ? d1 : nullptr, 0, use_only_phase, s, split));
    // re-balance: with a composed rows at tc per row and every row's upload at
    // tu per float row (raw rows move two), the load takes about
    // max(tc (nr - split), tu (nr + split)); equal when split/nr = (tc - tu)/(tc + tu)
    c->load_rows = (long long)nr;
    c->load_rows_raw = (long long)split;
    c->load_compose_s = t_comp;
    c->load_raw_copy_ms = 0.0;
    if (raw_ok) {
        if (split < nr) c->t_comp_row = t_comp / (double)(nr - split);
        if (split > 0) {
            float ms = 0.f;
            if (cudaEventSynchronize(c->ev_raw[1]) == cudaSuccess &&
                cudaEventElapsedTime(&ms, c->ev_raw[0], c->ev_raw[1]) == cudaSuccess && ms > 0.f) {
                c->t_up_row = 1e-3 * ms / (2.0 * (double)split);
                c->load_raw_copy_ms = ms;
            }
        }
        if (c->t_comp_row > 0.0 && c->t_up_row > 0.0) {
            const double f = (c->t_comp_row - c->t_up_row) / (c->t_comp_row + c->t_up_row);
            c->raw_frac = std::min(0.95, std::max(0.0, f));
        }
    }
    return PS_OK;
}

int load_field(ps_gpu_ctx* c, int which, const void* dens, const void* xhii, int is_double, int mem,
               int use_only_phase)
{
    if (which < PS_FIELD_DENS || which > PS_FIELD_XHI_DENS) return fail(PS_ERR_ARG, "which=%d", which);
    if (mem != PS_MEM_HOST && mem != PS_MEM_DEVICE) return fail(PS_ERR_ARG, "mem=%d", mem);
    const void* a = which == PS_FIELD_XHII ? xhii : dens;
    const void* b = which == PS_FIELD_XHI_DENS ? xhii : nullptr;
    if (!a || (which == PS_FIELD_XHI_DENS && !b)) return fail(PS_ERR_ARG, "field pointer is NULL");
    const size_t n3 = (size_t)c->N * c->N * c->N;
    const size_t bytes = n3 * (is_double ? 8 : 4);
    int s = -1;
    c->load_rows = c->load_rows_raw = 0;
    c->load_compose_s = c->load_raw_copy_ms = 0.0;
    if (mem == PS_MEM_HOST && which == PS_FIELD_XHI_DENS && !is_double && c->methods == PS_FP32_BATCHED)
        return load_xhi_dens_host(c, (const float*)dens, (const float*)xhii, use_only_phase);
    if (mem == PS_MEM_HOST) {
        c->upload_bytes = bytes * (b ? 2 : 1);
        PS_TRY(ensure_stage(c, bytes));
        s = c->slot;
        c->slot ^= 1;
        PS_CK(cudaStreamWaitEvent(c->copy_stream, c->ev_free[s], 0));
        PS_CK(cudaMemcpyAsync(c->stage[s][0], a, bytes, cudaMemcpyHostToDevice, c->copy_stream));
        if (b) PS_CK(cudaMemcpyAsync(c->stage[s][1], b, bytes, cudaMemcpyHostToDevice, c->copy_stream));
        PS_CK(cudaEventRecord(c->ev_copied[s], c->copy_stream));
        PS_CK(cudaStreamWaitEvent(c->stream, c->ev_copied[s], 0));
        a = c->stage[s][0];
        if (b) b = c->stage[s][1];
    }
    return transform_field(c, a, b, is_double, use_only_phase, s);
}

// The forward transform of a loaded field (device arrays a, b), then slot s
// (if any) is released.
int transform_field(ps_gpu_ctx* c, const void* a, const void* b, int is_double, int use_only_phase, int s,
                    size_t split)
{
    const int kind = split ? SRC_F32 : b ? (is_double ? SRC_XHI_F64 : SRC_XHI_F32) : (is_double ? SRC_F64 : SRC_F32);
    c->use_only_phase = use_only_phase;
    c->f.have_spec = c->d.have_spec = false;
    if (c->methods & PS_FP32_BATCHED) PS_TRY(forward_field<float>(c, kind, a, b, split));
    if (c->methods & PS_FP64_PLAIN) PS_TRY(forward_field<double>(c, kind, a, b));
    if (s >= 0) PS_CK(cudaEventRecord(c->ev_free[s], c->stream));
    c->field_set = true;
    return PS_OK;
}

// Staging slots of at least `bytes` per array (device, two slots of two).
int ensure_stage(ps_gpu_ctx* c, size_t bytes)
{
    if (c->stage_bytes >= bytes) return PS_OK;
    // earlier uploads and the transforms reading them finish first
    PS_CK(cudaStreamSynchronize(c->copy_stream));
    PS_CK(cudaStreamSynchronize(c->stream));
    for (int q = 0; q < 2; q++)
        for (int r = 0; r < 2; r++) {
            cudaFree(c->stage[q][r]);
            c->stage[q][r] = nullptr;
        }
    c->stage_bytes = 0;
    for (int q = 0; q < 2; q++)
        for (int r = 0; r < 2; r++) PS_TRY(alloc_dev((unsigned char**)&c->stage[q][r], bytes));
    c->stage_bytes = bytes;
    return PS_OK;
}

constexpr size_t kFileChunk = (size_t)64 << 20;  // bytes per page-locked chunk buffer

static __global__ void k_widen(const float* __restrict__ in, double* __restrict__ out, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

// `bytes` of a raw file into device memory `dev` on the copy stream through
// the two chunk buffers: the read of one chunk overlaps the copy of the other.
int upload_file(ps_gpu_ctx* c, const char* path, size_t bytes, void* dev)
{
    FILE* f = fopen(path, "rb");
    if (!f) return fail(PS_ERR_IO, "cannot open %s", path);
    int rc = PS_OK, q = 0;
    for (size_t done = 0; done < bytes; q ^= 1) {
        const size_t len = std::min(kFileChunk, bytes - done);
        cudaError_t e = cudaEventSynchronize(c->ev_chunk[q]);  // chunk buffer q copied out
        if (e != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "chunk copy: %s", cudaGetErrorString(e));
            break;
        }
        const size_t got = fault_hit(FAULT_READ) ? 0 : fread(c->pin[q], 1, len, f);
        if (got != len) {
            rc = fail(PS_ERR_IO, "%s holds %zu of the %zu bytes of the grid", path, done + got, bytes);
            break;
        }
        e = cudaMemcpyAsync((unsigned char*)dev + done, c->pin[q], len, cudaMemcpyHostToDevice, c->copy_stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_chunk[q], c->copy_stream);
        if (e != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "chunk upload: %s", cudaGetErrorString(e));
            break;
        }
        done += len;
    }
    fclose(f);
    return rc;
}

}  // namespace

int ps::report_error(int code, const char* msg) { return fail(code, "%s", msg); }
Shell ps::host_shell(int kind, double k, double kmin, double kmax, double binwidth, double L, int N)
{
    return make_shell(kind, k, kmin, kmax, binwidth, L, N);
}
double ps::host_norm_coef(double L, int N, int n) { return norm_coef(L, N, n); }

// =========================================================================
// C-ABI
// =========================================================================
extern "C" {

const char* ps_gpu_strerror(int s)
{
    switch (s) {
    case PS_OK: return "ok";
    case PS_ERR_ARG: return "invalid argument";
    case PS_ERR_OOM: return "out of memory";
    case PS_ERR_IO: return "i/o error";
    case PS_ERR_CUDA: return "CUDA error";
    case PS_ERR_TIMEOUT: return "device wait timed out";
    case PS_ERR_NONFINITE: return "non-finite input";
    case PS_ERR_UNSUPPORTED: return "unsupported";
    case PS_ERR_UNDEFINED: return "undefined in the reference";
    default: return "unknown status";
    }
}

const char* ps_gpu_last_error(void) { return g_err; }

int ps_gpu_debug_fault(const char* spec) { g_err[0] = 0; return arm_faults(spec); }

int ps_gpu_create(ps_gpu_ctx** out, int nbins, double boxsize, int methods, int device)
{
    g_err[0] = 0;
    static std::once_flag env_faults;
    std::call_once(env_faults, []() {
        if (const char* e = getenv("PS_FAULT")) arm_faults(e);
    });
    if (!out) return fail(PS_ERR_ARG, "ctx pointer is NULL");
    *out = nullptr;
    if (!grid_size_ok(nbins))
        return fail(PS_ERR_UNSUPPORTED, "grid size %d: supported are the powers of two 16..1024 and 48, 60, 96, "
                                        "192, 300, 320, 384, 600", nbins);
    if (!(boxsize > 0.0) || !std::isfinite(boxsize)) return fail(PS_ERR_ARG, "box size must be positive");
    if (!(methods & (PS_FP64_PLAIN | PS_FP32_BATCHED)) || (methods & ~(PS_FP64_PLAIN | PS_FP32_BATCHED)))
        return fail(PS_ERR_ARG, "methods mask %d invalid", methods);
    int ndev = 0;
    PS_CK(cudaGetDeviceCount(&ndev));
    if (device >= ndev) return fail(PS_ERR_ARG, "device %d of %d", device, ndev);
    if (device >= 0) PS_CK(cudaSetDevice(device));
    ps_gpu_ctx* c = new ps_gpu_ctx();
    c->N = nbins;
    c->L = boxsize;
    c->methods = methods;
    cudaGetDevice(&c->device);
    int rc = PS_OK;
    do {
        if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "stream creation failed");
            break;
        }
        c->stream = c->own_stream;
        if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "event creation failed");
            break;
        }
        if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&c->lane2_stream, cudaStreamNonBlocking) != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "stream creation failed");
            break;
        }
        if (cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->ev_join2, cudaEventDisableTiming) != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "event creation failed");
            break;
        }
        bool ev_ok = true;
        for (int q = 0; q < 2; q++)
            ev_ok = ev_ok && cudaEventCreateWithFlags(&c->ev_copied[q], cudaEventDisableTiming) == cudaSuccess &&
                    cudaEventCreateWithFlags(&c->ev_free[q], cudaEventDisableTiming) == cudaSuccess;
        if (!ev_ok) {
            rc = fail(PS_ERR_CUDA, "event creation failed");
            break;
        }
        if ((rc = alloc_dev(&c->dstatus, 1)) != PS_OK) break;
        if (cudaMemset(c->dstatus, 0, sizeof(int)) != cudaSuccess) {
            rc = fail(PS_ERR_CUDA, "status word");
            break;
        }
        // the batched method transforms shells in FP32 and counts in FP64
        if (methods & PS_FP32_BATCHED) {
            if ((rc = init_prec(c, c->f)) != PS_OK) break;
            if ((rc = init_prec(c, c->d)) != PS_OK) break;
        }
        if ((methods & PS_FP64_PLAIN) && (rc = init_prec(c, c->d)) != PS_OK) break;
    } while (0);
    if (rc != PS_OK) {
        ps_gpu_finalize(c);
        return rc;
    }
    *out = c;
    return PS_OK;
}

int ps_gpu_set_field(ps_gpu_ctx* c, int which, const void* dens, const void* xhii, int is_double,
                     int mem, int use_only_phase)
{
    g_err[0] = 0;
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    PS_CK(cudaSetDevice(c->device));
    PS_TRY(timed_begin(c));
    PS_TRY(load_field(c, which, dens, xhii, is_double, mem, use_only_phase));
    PS_TRY(timed_end(c));
    return check_status(c);
}

int ps_gpu_set_field_async(ps_gpu_ctx* c, int which, const void* dens, const void* xhii, int is_double,
                           int mem, int use_only_phase)
{
    g_err[0] = 0;
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    PS_CK(cudaSetDevice(c->device));
    PS_TRY(drain_pending(c, false));
    return load_field(c, which, dens, xhii, is_double, mem, use_only_phase);
}

long long ps_gpu_upload_bytes(const ps_gpu_ctx* c) { return c ? (long long)c->upload_bytes : PS_ERR_ARG; }

int ps_gpu_load_stats(const ps_gpu_ctx* c, ps_load_stats* out)
{
    g_err[0] = 0;
    if (!c || !out) return fail(PS_ERR_ARG, "NULL argument");
    out->rows = c->load_rows;
    out->rows_raw = c->load_rows_raw;
    out->bytes = (long long)c->upload_bytes;
    out->compose_s = c->load_compose_s;
    out->raw_copy_ms = c->load_raw_copy_ms;
    out->next_raw_frac = c->raw_frac;
    out->host_threads = (int)HostPool::default_threads();
    return PS_OK;
}

int ps_gpu_set_field_files(ps_gpu_ctx* c, int which, const char* dens_path, int dens_double, const char* xhii_path,
                           int xhii_double, int use_only_phase)
{
    g_err[0] = 0;
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    if (which < PS_FIELD_DENS || which > PS_FIELD_XHI_DENS) return fail(PS_ERR_ARG, "which=%d", which);
    const bool use_d = which != PS_FIELD_XHII, use_x = which != PS_FIELD_DENS;
    if ((use_d && !dens_path) || (use_x && !xhii_path)) return fail(PS_ERR_ARG, "input file name is NULL");
    PS_CK(cudaSetDevice(c->device));
    PS_TRY(timed_begin(c));
    // the field's precision: double when any file it reads holds doubles (a
    // float file beside it is widened exactly on the device)
    const int dp = (use_d && dens_double) || (use_x && xhii_double);
    const size_t n3 = (size_t)c->N * c->N * c->N;
    PS_TRY(ensure_stage(c, n3 * (dp ? 8 : 4)));
    for (int q = 0; q < 2; q++) {
        if (!c->pin[q] && (fault_hit(FAULT_ALLOC) ||
                           cudaHostAlloc(&c->pin[q], kFileChunk, cudaHostAllocDefault) != cudaSuccess)) {
            c->pin[q] = nullptr;
            return fail(PS_ERR_OOM, "page-locked chunk buffer of %zu bytes", kFileChunk);
        }
        if (!c->ev_chunk[q]) PS_CK(cudaEventCreateWithFlags(&c->ev_chunk[q], cudaEventDisableTiming));
    }
    const int s = c->slot;
    c->slot ^= 1;
    PS_CK(cudaStreamWaitEvent(c->copy_stream, c->ev_free[s], 0));
    struct Input {
        const char* path;
        int is_double;
    };
    Input in[2];
    int nin = 0;
    if (which == PS_FIELD_XHII) in[nin++] = {xhii_path, xhii_double};
    else in[nin++] = {dens_path, dens_double};
    if (which == PS_FIELD_XHI_DENS) in[nin++] = {xhii_path, xhii_double};
    int rc = PS_OK;
    for (int r = 0; r < nin && rc == PS_OK; r++) {
        if (in[r].is_double || !dp) {
            rc = upload_file(c, in[r].path, n3 * (in[r].is_double ? 8 : 4), c->stage[s][r]);
        } else {
            // a float file of a double field: through the other slot's array (after
            // the transform that last read it), widened into this slot
            cudaError_t e = cudaStreamWaitEvent(c->copy_stream, c->ev_free[s ^ 1], 0);
            if (e != cudaSuccess) rc = fail(PS_ERR_CUDA, "%s", cudaGetErrorString(e));
            if (rc == PS_OK) rc = upload_file(c, in[r].path, n3 * 4, c->stage[s ^ 1][r]);
            if (rc == PS_OK) {
                k_widen<<<148 * 8, 256, 0, c->copy_stream>>>((const float*)c->stage[s ^ 1][r], (double*)c->stage[s][r],
                                                             n3);
                e = launch_status();
                if (e != cudaSuccess) rc = fail(PS_ERR_CUDA, "widen: %s", cudaGetErrorString(e));
            }
        }
    }
    if (rc != PS_OK) {
        cudaStreamSynchronize(c->copy_stream);  // no copy still reads a chunk buffer
        return rc;
    }
    PS_CK(cudaEventRecord(c->ev_copied[s], c->copy_stream));
    PS_CK(cudaStreamWaitEvent(c->stream, c->ev_copied[s], 0));
    PS_TRY(transform_field(c, c->stage[s][0], nin > 1 ? c->stage[s][1] : nullptr, dp, use_only_phase, s));
    PS_CK(cudaStreamSynchronize(c->copy_stream));
    PS_TRY(timed_end(c));
    return check_status(c);
}

int ps_gpu_init(ps_gpu_ctx** ctx, int nbins, double boxsize, const void* field, int field_is_double,
                int use_only_phase, int methods)
{
    PS_TRY(ps_gpu_create(ctx, nbins, boxsize, methods, -1));
    int rc = ps_gpu_set_field(*ctx, PS_FIELD_DENS, field, nullptr, field_is_double, PS_MEM_HOST,
                              use_only_phase);
    if (rc != PS_OK) {
        ps_gpu_finalize(*ctx);
        *ctx = nullptr;
    }
    return rc;
}

int ps_gpu_polyspectrum_batch(ps_gpu_ctx* c, int method, int nconf, ps_cfg* cfgs, double* B,
                              double* Npoly, double* kappa)
{
    g_err[0] = 0;
    if (!c || !cfgs || !B || !Npoly || nconf < 0) return fail(PS_ERR_ARG, "NULL argument");
    if (!c->field_set) return fail(PS_ERR_ARG, "no field loaded (ps_gpu_set_field)");
    if (nconf == 0) return PS_OK;
    if (method != PS_FP64_PLAIN && method != PS_FP32_BATCHED) return fail(PS_ERR_ARG, "method %d", method);
    if (!(c->methods & method)) return fail(PS_ERR_ARG, "method %d not enabled for this context", method);
    PS_CK(cudaSetDevice(c->device));
    PS_TRY(timed_begin(c));
    const std::vector<ps_cfg> in(cfgs, cfgs + nconf);
    int rc = method == PS_FP64_PLAIN ? plain_batch(c, nconf, cfgs, B, Npoly, kappa)
                                     : batched(c, nconf, cfgs, B, Npoly, kappa);
    if (rc != PS_OK) return rc;
    remember_npoly(c, method, nconf, in.data(), Npoly);
    return timed_end(c);
}

int ps_gpu_polyspectrum(ps_gpu_ctx* c, int n, const double* k, double* kmin, double* kmax,
                        double kbinwidth, int kbinningCase, double* B, double* Npoly)
{
    g_err[0] = 0;
    if (!c || !k || !kmin || !kmax || !B || !Npoly) return fail(PS_ERR_ARG, "NULL argument");
    if (n < 2 || n > PS_MAX_LEGS) return fail(PS_ERR_ARG, "n=%d out of range", n);
    ps_cfg g;
    memset(&g, 0, sizeof(g));
    g.n = n;
    g.kbinningCase = kbinningCase;
    g.kbinwidth = kbinwidth;
    for (int l = 0; l < n; l++) {
        g.k[l] = k[l];
        g.kmin[l] = kmin[l];
        g.kmax[l] = kmax[l];
    }
    const int method = (c->methods & PS_FP64_PLAIN) ? PS_FP64_PLAIN : PS_FP32_BATCHED;
    PS_TRY(ps_gpu_polyspectrum_batch(c, method, 1, &g, B, Npoly, nullptr));
    for (int l = 0; l < n; l++) {
        kmin[l] = g.kmin[l];
        kmax[l] = g.kmax[l];
    }
    return PS_OK;
}

int ps_gpu_grad(ps_gpu_ctx* c, int method, int n, const double* k, const double* kmin,
                const double* kmax, double kbinwidth, int kbinningCase, void* out, int out_is_double,
                int out_mem)
{
    g_err[0] = 0;
    if (!c || !k || !kmin || !kmax || !out) return fail(PS_ERR_ARG, "NULL argument");
    if (!c->field_set) return fail(PS_ERR_ARG, "no field loaded (ps_gpu_set_field)");
    if (method != PS_FP64_PLAIN && method != PS_FP32_BATCHED) return fail(PS_ERR_ARG, "method %d", method);
    if (!(c->methods & method)) return fail(PS_ERR_ARG, "method %d not enabled for this context", method);
    if (out_mem != PS_MEM_HOST && out_mem != PS_MEM_DEVICE) return fail(PS_ERR_ARG, "out_mem=%d", out_mem);
    if (n != 2 && n != 3)
        return fail(PS_ERR_UNSUPPORTED, "ps_gpu_grad: n=%d (the reference's configurations have n = 2 or 3)", n);
    if (c->use_only_phase == 1 && !(method == PS_FP64_PLAIN ? c->d.have_mod : c->f.have_mod))
        return fail(PS_ERR_UNSUPPORTED, "ps_gpu_grad: the field was loaded phase-only without its modulus; call "
                                        "ps_gpu_keep_modulus(ctx, 1) before loading it");
    PS_CK(cudaSetDevice(c->device));
    ps_cfg g;
    memset(&g, 0, sizeof(g));
    g.n = n;
    g.kbinningCase = kbinningCase;
    g.kbinwidth = kbinwidth;
    for (int l = 0; l < n; l++) {
        g.k[l] = k[l];
        g.kmin[l] = kmin[l];
        g.kmax[l] = kmax[l];
    }
    // the polygon count of the configuration (sum I = N^3 * Npoly): from an
    // earlier evaluation on this context (counts do not depend on the field),
    // else evaluated here
    double Np = 0.0;
    const auto known = c->npoly_cache.find(npoly_key(method, g));
    if (known != c->npoly_cache.end()) {
        Np = known->second;
    } else {
        ps_cfg g2 = g;
        double Bv = 0.0;
        int rc = method == PS_FP64_PLAIN ? plain_batch(c, 1, &g2, &Bv, &Np, nullptr)
                                         : batched(c, 1, &g2, &Bv, &Np, nullptr);
        if (rc != PS_OK) return rc;
        remember_npoly(c, method, 1, &g, &Np);
    }
    PS_TRY(timed_begin(c));
    std::vector<std::vector<Shell>> legs;
    PS_TRY(resolve_legs(c, 1, &g, legs));
    PS_TRY(check_band(c, legs_band(legs[0], c->N)));
    const double n3 = (double)c->N * (double)c->N * (double)c->N;
    const double scale = norm_coef(c->L, c->N, n) / (Np * n3);
    int rc = method == PS_FP64_PLAIN ? grad_impl<double>(c, n, legs[0], scale, out, out_is_double, out_mem)
                                     : grad_impl<float>(c, n, legs[0], scale, out, out_is_double, out_mem);
    if (rc != PS_OK) return rc;
    return timed_end(c);
}

int ps_make_configs(const ps_run_params* p, ps_cfg* cfgs, int max_cfg, double* k_out, double* theta_out)
{
    g_err[0] = 0;
    if (!p) return fail(PS_ERR_ARG, "params NULL");
    const double pi = ref_pi();
    const int n = p->n;
    if (n < 2) return fail(PS_ERR_ARG, "n must be >= 2 (kvectors.c:60-64)");
    if (n > 3) return fail(PS_ERR_UNSUPPORTED, "n > 3 not implemented in the reference (kvectors.c:140-144)");
    int nval;
    std::vector<double> kl, th;
    double kpoly[3] = {0, 0, 0}, kpmin[3] = {0, 0, 0}, kpmax[3] = {0, 0, 0};
    if (n == 2) {  // kvectors.c:75-96
        if (p->num_values > 1) {
            nval = p->grid_size / 2;
            kl.resize(std::max(nval, 2));
            for (int i = 0; i < nval; i++) kl[i] = 2. * pi / p->box_size * (double)(i + 1);
        } else {
            nval = 1;
            kl = {p->k1, p->k1};  // kvectors.c:88-89
        }
        for (int i = 0; i < 2; i++) kpoly[i] = kpmin[i] = kpmax[i] = kl[i];
    } else {  // kvectors.c:100-137
        kpoly[0] = p->k1;
        kpoly[1] = p->k2;
        if (p->equilateral == 1) {
            if (p->num_values <= 0) return fail(PS_ERR_ARG, "numValues must be > 0 (kvectors.c:107)");
            nval = p->num_values;
            kl.resize(nval);
            const double kL = 2. * pi / p->box_size;
            for (int i = 0; i < nval; i++) kl[i] = kL * pow(p->grid_size / 2, (double)(i + 1) / (double)nval);
            th = {pi / 3.};
        } else if (p->num_values > 1) {
            nval = p->num_values;
            kl.resize(nval);
            th.resize(nval);
            for (int i = 0; i < nval; i++) {
                th[i] = pi * (double)i / (double)nval;
                kl[i] = sqrt(p->k1 * p->k1 + p->k2 * p->k2 - 2. * p->k1 * p->k2 * cos(th[i]));
            }
        } else {
            nval = 1;
            th = {p->theta};
            kl = {sqrt(p->k1 * p->k1 + p->k2 * p->k2 - 2. * p->k1 * p->k2 * cos(p->theta))};
        }
    }
    for (int i = 0; i < nval && i < max_cfg; i++) {  // run.c:56-84
        kpoly[n - 1] = kl[i];
        if (n == 2) kpoly[0] = kl[i];
        if (n == 3) {
            const int ti = p->equilateral == 1 ? 0 : i;
            if (p->equilateral == 1)
                for (int j = 0; j < n; j++) kpoly[j] = kl[i];
            if (p->kbinningCase >= 2) {  // calc_k3min / calc_k3max, kvectors.c:233-246
                const double cmin = fmin(1., cos(th[ti]) + 0.5 * p->dcosTheta);
                const double cmax = fmax(-1., cos(th[ti]) - 0.5 * p->dcosTheta);
                kpmin[n - 1] = sqrt(kpoly[0] * kpoly[0] + kpoly[1] * kpoly[1] - 2. * kpoly[0] * kpoly[1] * cmin);
                kpmax[n - 1] = sqrt(kpoly[0] * kpoly[0] + kpoly[1] * kpoly[1] - 2. * kpoly[0] * kpoly[1] * cmax);
            }
        }
        if (cfgs) {
            ps_cfg& g = cfgs[i];
            memset(&g, 0, sizeof(g));
            g.n = n;
            g.kbinningCase = p->kbinningCase;
            g.kbinwidth = p->kbinwidth;
            for (int j = 0; j < n; j++) {
                g.k[j] = kpoly[j];
                g.kmin[j] = kpmin[j];
                g.kmax[j] = kpmax[j];
            }
        }
        if (k_out) k_out[i] = kl[i];
        if (theta_out) theta_out[i] = th.empty() ? NAN : (p->equilateral == 1 ? th[0] : th[i]);
    }
    return nval;
}

int ps_gpu_set_stream(ps_gpu_ctx* c, void* stream)
{
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return PS_OK;
}

int ps_gpu_last_timing(ps_gpu_ctx* c, double* ms, long long* launches)
{
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    if (ms) *ms = c->last_ms;
    if (launches) *launches = c->launches;
    return PS_OK;
}

int ps_gpu_plan_create(ps_gpu_ctx* c, int method, int nconf, const ps_cfg* cfgs, int flags, ps_gpu_plan** out)
{
    g_err[0] = 0;
    if (!c || !out || (nconf > 0 && !cfgs) || nconf < 0) return fail(PS_ERR_ARG, "NULL argument");
    *out = nullptr;
    if (method != PS_FP64_PLAIN && method != PS_FP32_BATCHED) return fail(PS_ERR_ARG, "method %d", method);
    if (!(c->methods & method)) return fail(PS_ERR_ARG, "method %d not enabled for this context", method);
    if (flags & ~(PS_PLAN_GRAPH | PS_PLAN_KAPPA | PS_PLAN_AUTOTUNE | PS_PLAN_FFT_COUNTS))
        return fail(PS_ERR_ARG, "flags %d", flags);
    PS_CK(cudaSetDevice(c->device));
    ps_gpu_plan* P = new ps_gpu_plan();
    P->ctx = c;
    P->method = method;
    P->nconf = nconf;
    P->flags = method == PS_FP32_BATCHED ? flags : (flags & PS_PLAN_KAPPA);
    P->cfgs.assign(cfgs, cfgs + nconf);
    if (method == PS_FP32_BATCHED && nconf > 0) {
        const int rc = plan_batched(c, P);
        if (rc != PS_OK) {
            plan_free(P);
            return rc;
        }
    }
    c->plans.insert(P);
    *out = P;
    return PS_OK;
}

int ps_gpu_plan_execute(ps_gpu_ctx* c, ps_gpu_plan* P, double* B, double* Npoly, double* kappa, ps_cfg* cfgs_out)
{
    g_err[0] = 0;
    if (!c || !P || !B || !Npoly) return fail(PS_ERR_ARG, "NULL argument");
    if (P->ctx != c) return fail(PS_ERR_ARG, "plan belongs to another context");
    if (!c->field_set) return fail(PS_ERR_ARG, "no field loaded (ps_gpu_set_field)");
    if (kappa && !(P->flags & PS_PLAN_KAPPA)) return fail(PS_ERR_ARG, "plan created without PS_PLAN_KAPPA");
    if (P->nconf == 0) return PS_OK;
    PS_CK(cudaSetDevice(c->device));
    PS_TRY(timed_begin(c));
    if (P->method == PS_FP64_PLAIN) {
        std::vector<ps_cfg> g = P->cfgs;
        PS_TRY(plain_batch(c, P->nconf, g.data(), B, Npoly, kappa));
        if (cfgs_out)
            for (int q = 0; q < P->nconf; q++) cfgs_out[q] = g[q];
    } else {
        if (!c->f.have_spec) return fail(PS_ERR_ARG, "FP32 spectrum not available");
        PS_TRY(check_band(c, P->band));
        if ((P->flags & PS_PLAN_GRAPH) && c->prof_on) PS_TRY(plan_enqueue(c, P));  // profiled: eager
        else PS_TRY(plan_run(c, P));
        PS_TRY(plan_finish(c, P, B, Npoly, kappa, cfgs_out));
    }
    return timed_end(c);
}

void ps_gpu_plan_destroy(ps_gpu_plan* P)
{
    if (!P) return;
    if (P->ctx) {
        cudaSetDevice(P->ctx->device);
        cudaStreamSynchronize(P->ctx->stream);       // submissions still reading it
        cudaStreamSynchronize(P->ctx->side_stream);  // and a prepared part still writing it
        drain_pending(P->ctx, true);            // and those not yet unpacked
        P->ctx->plans.erase(P);
    }
    plan_free(P);
}

int ps_gpu_plan_submit(ps_gpu_ctx* c, ps_gpu_plan* P, double* B, double* Npoly, double* kappa, ps_cfg* cfgs_out)
{
    g_err[0] = 0;
    if (!c || !P || !B || !Npoly) return fail(PS_ERR_ARG, "NULL argument");
    if (P->ctx != c) return fail(PS_ERR_ARG, "plan belongs to another context");
    if (P->method != PS_FP32_BATCHED)
        return fail(PS_ERR_UNSUPPORTED, "asynchronous submission needs a PS_FP32_BATCHED plan");
    if (!c->field_set) return fail(PS_ERR_ARG, "no field loaded (ps_gpu_set_field)");
    if (kappa && !(P->flags & PS_PLAN_KAPPA)) return fail(PS_ERR_ARG, "plan created without PS_PLAN_KAPPA");
    if (P->nconf == 0) return PS_OK;
    if (!c->f.have_spec) return fail(PS_ERR_ARG, "FP32 spectrum not available");
    PS_TRY(check_band(c, P->band));
    PS_CK(cudaSetDevice(c->device));
    if ((P->flags & PS_PLAN_GRAPH) && c->prof_on) PS_TRY(plan_enqueue(c, P));
    else PS_TRY(plan_run(c, P));
    const size_t len = 10 * (size_t)P->nconf + 1;
    double* h = nullptr;
    cudaEvent_t ev = nullptr;
    PS_TRY(submit_slot(c, len, &h, &ev));
    int rc = plan_copy_results(c, P, h);
    if (rc == PS_OK && cudaEventRecord(ev, c->stream) != cudaSuccess) rc = fail(PS_ERR_CUDA, "event record failed");
    if (rc != PS_OK) {
        cudaStreamSynchronize(c->stream);  // no copy still writes h
        c->spare_host.push_back({h, len});
        c->spare_events.push_back(ev);
        return rc;
    }
    c->pending.push_back(PendingSubmit{P, h, len, ev, B, Npoly, kappa, cfgs_out});
    return drain_pending(c, false);
}

int ps_gpu_plan_launch(ps_gpu_ctx* c, ps_gpu_plan* P)
{
    g_err[0] = 0;
    if (!c || !P) return fail(PS_ERR_ARG, "NULL argument");
    if (P->ctx != c) return fail(PS_ERR_ARG, "plan belongs to another context");
    if (P->method != PS_FP32_BATCHED)
        return fail(PS_ERR_UNSUPPORTED, "launching without read-back needs a PS_FP32_BATCHED plan");
    if (!c->field_set) return fail(PS_ERR_ARG, "no field loaded (ps_gpu_set_field)");
    if (P->nconf == 0) return PS_OK;
    if (!c->f.have_spec) return fail(PS_ERR_ARG, "FP32 spectrum not available");
    PS_TRY(check_band(c, P->band));
    PS_CK(cudaSetDevice(c->device));
    if ((P->flags & PS_PLAN_GRAPH) && c->prof_on) return plan_enqueue(c, P);
    return plan_run(c, P);
}

int ps_gpu_plan_prepare(ps_gpu_ctx* c, ps_gpu_plan* P)
{
    g_err[0] = 0;
    if (!c || !P) return fail(PS_ERR_ARG, "NULL argument");
    if (P->ctx != c) return fail(PS_ERR_ARG, "plan belongs to another context");
    if (P->method != PS_FP32_BATCHED) return fail(PS_ERR_UNSUPPORTED, "preparing needs a PS_FP32_BATCHED plan");
    if (P->nconf == 0 || c->prof_on || P->prepared) return PS_OK;  // profiled executions stay on one lane
    PS_CK(cudaSetDevice(c->device));
    return plan_prepare(c, P);
}

int ps_gpu_plan_results(ps_gpu_ctx* c, ps_gpu_plan* P, double* B, double* Npoly, double* kappa, ps_cfg* cfgs_out)
{
    g_err[0] = 0;
    if (!c || !P || !B || !Npoly) return fail(PS_ERR_ARG, "NULL argument");
    if (P->ctx != c) return fail(PS_ERR_ARG, "plan belongs to another context");
    if (P->method != PS_FP32_BATCHED) return fail(PS_ERR_UNSUPPORTED, "results of a PS_FP32_BATCHED plan only");
    if (kappa && !(P->flags & PS_PLAN_KAPPA)) return fail(PS_ERR_ARG, "plan created without PS_PLAN_KAPPA");
    if (P->nconf == 0) return PS_OK;
    PS_CK(cudaSetDevice(c->device));
    return plan_finish(c, P, B, Npoly, kappa, cfgs_out);
}

int ps_gpu_plan_results_device(ps_gpu_ctx* c, ps_gpu_plan* P, double* dst)
{
    g_err[0] = 0;
    if (!c || !P || !dst) return fail(PS_ERR_ARG, "NULL argument");
    if (P->ctx != c) return fail(PS_ERR_ARG, "plan belongs to another context");
    if (P->method != PS_FP32_BATCHED) return fail(PS_ERR_UNSUPPORTED, "results of a PS_FP32_BATCHED plan only");
    if (P->nconf == 0) return PS_OK;
    PS_CK(cudaSetDevice(c->device));
    const size_t n = (size_t)P->nconf;
    PS_CK(cudaMemcpyAsync(dst, P->dres, 16 * n, cudaMemcpyDeviceToDevice, c->stream));
    PS_CK(cudaMemcpyAsync(dst + 2 * n, P->dwb, 48 * n, cudaMemcpyDeviceToDevice, c->stream));
    return PS_OK;
}

int ps_gpu_synchronize(ps_gpu_ctx* c)
{
    g_err[0] = 0;
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    PS_CK(cudaSetDevice(c->device));
    PS_CK(cudaStreamSynchronize(c->copy_stream));
    PS_CK(cudaStreamSynchronize(c->stream));
    PS_TRY(drain_pending(c, true));
    PS_TRY(check_status(c));
    const int e = c->async_err.exchange(0);
    if (e != PS_OK) return fail(e, "internal: a derived shell exceeded its launch bound (asynchronous execution)");
    return PS_OK;
}

long long ps_gpu_launch_count(ps_gpu_ctx* c) { return c ? c->launches_total : -1; }

int ps_gpu_set_spectrum_band(ps_gpu_ctx* c, int band)
{
    g_err[0] = 0;
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    c->spec_band = band;
    return PS_OK;
}

int ps_gpu_plan_band(const ps_gpu_plan* P)
{
    g_err[0] = 0;
    if (!P) return fail(PS_ERR_ARG, "plan is NULL");
    if (P->method != PS_FP32_BATCHED) return P->ctx ? P->ctx->N / 2 : 0;
    return P->band;
}

int ps_gpu_keep_modulus(ps_gpu_ctx* c, int on)
{
    g_err[0] = 0;
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    c->keep_modulus = on != 0;
    return PS_OK;
}

int ps_gpu_tune_export(ps_gpu_ctx* c, char* buf, int buflen)
{
    g_err[0] = 0;
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    std::string t;
    char line[96];
    for (const auto& kv : c->tune_grid) {
        snprintf(line, sizeof(line), "grid %d %d %d %d %d\n", kv.first[0], kv.first[1], kv.first[2], kv.first[3],
                 kv.second);
        t += line;
    }
    for (const auto& kv : c->pencil_alt) {
        snprintf(line, sizeof(line), "pencil %d %d\n", kv.first, kv.second);
        t += line;
    }
    for (const auto& kv : c->pair_var) {
        snprintf(line, sizeof(line), "pair %d %d\n", kv.first, kv.second);
        t += line;
    }
    for (const auto& kv : c->dot_alt) {
        snprintf(line, sizeof(line), "dot %d %d\n", kv.first, kv.second);
        t += line;
    }
    if (buf && buflen > 0) {
        const size_t n = std::min(t.size(), (size_t)buflen - 1);
        memcpy(buf, t.data(), n);
        buf[n] = '\0';
    }
    return (int)t.size();
}

int ps_gpu_tune_import(ps_gpu_ctx* c, const char* text)
{
    g_err[0] = 0;
    if (!c || !text) return fail(PS_ERR_ARG, "NULL argument");
    std::map<std::array<int, 4>, int> add;
    std::map<int, int> add_pencil, add_pair, add_dot;
    const char* p = text;
    while (*p) {
        const char* e = strchr(p, '\n');
        const std::string ln(p, e ? (size_t)(e - p) : strlen(p));
        p = e ? e + 1 : p + ln.size();
        if (ln.find_first_not_of(" \t\r") == std::string::npos) continue;
        int n, ba, bb, bc, m, used = 0;
        if (sscanf(ln.c_str(), "pencil %d %d %n", &m, &n, &used) == 2 &&
            ln.find_first_not_of(" \t\r", used) == std::string::npos) {
            if (!grid_size_ok(m) || (n != 0 && n != 1))
                return fail(PS_ERR_ARG, "tune line out of range: '%s'", ln.c_str());
            add_pencil[m] = n;
            continue;
        }
        used = 0;
        if (sscanf(ln.c_str(), "pair %d %d %n", &m, &n, &used) == 2 &&
            ln.find_first_not_of(" \t\r", used) == std::string::npos) {
            if (!grid_size_ok(m) || n < 0 || n > 2)
                return fail(PS_ERR_ARG, "tune line out of range: '%s'", ln.c_str());
            add_pair[m] = n;
            continue;
        }
        used = 0;
        if (sscanf(ln.c_str(), "dot %d %d %n", &m, &n, &used) == 2 &&
            ln.find_first_not_of(" \t\r", used) == std::string::npos) {
            if (!grid_size_ok(m) || (n != 0 && n != 1))
                return fail(PS_ERR_ARG, "tune line out of range: '%s'", ln.c_str());
            add_dot[m] = n;
            continue;
        }
        used = 0;
        if (sscanf(ln.c_str(), "grid %d %d %d %d %d %n", &n, &ba, &bb, &bc, &m, &used) != 5 ||
            ln.find_first_not_of(" \t\r", used) != std::string::npos)
            return fail(PS_ERR_ARG, "tune line not understood: '%s'", ln.c_str());
        if (!grid_supported(m) || m > n || ba < 0 || bb < 0 || bc < 0)
            return fail(PS_ERR_ARG, "tune line out of range: '%s'", ln.c_str());
        add[{n, ba, bb, bc}] = m;
    }
    for (const auto& kv : add) c->tune_grid[kv.first] = kv.second;
    for (const auto& kv : add_pencil) c->pencil_alt[kv.first] = kv.second;
    for (const auto& kv : add_pair) c->pair_var[kv.first] = kv.second;
    for (const auto& kv : add_dot) c->dot_alt[kv.first] = kv.second;
    return PS_OK;
}

int ps_gpu_set_profiling(ps_gpu_ctx* c, int on)
{
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    PS_TRY(prof_fold(c));
    if (on && !c->prof_on) {
        c->prof_agg.clear();
    }
    c->prof_on = on != 0;
    return PS_OK;
}

int ps_gpu_kernel_stats(ps_gpu_ctx* c, ps_kernel_stat* out, int max)
{
    if (!c) return fail(PS_ERR_ARG, "ctx is NULL");
    PS_CK(cudaSetDevice(c->device));
    PS_TRY(prof_fold(c));
    int cnt = 0;
    for (const auto& kv : c->prof_agg) {
        const int q = kv.first.first, size = kv.first.second;
        if (out && cnt < max) {
            memset(&out[cnt], 0, sizeof(ps_kernel_stat));
            char sz[16] = "";
            if (size > 0) snprintf(sz, sizeof(sz), "@%d", size);
            snprintf(out[cnt].name, sizeof(out[cnt].name), "%s%s%s", kFamilyName[q % KF_COUNT],
                     q >= KF_COUNT ? "_f64" : "", sz);
            out[cnt].launches = kv.second.n;
            out[cnt].ms = kv.second.ms;
            out[cnt].bytes = kv.second.bytes;
        }
        cnt++;
    }
    return cnt;
}

void ps_gpu_finalize(ps_gpu_ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    drain_pending(c, true);
    for (auto& j : c->pending) {  // copies that failed: their buffers only
        cudaFreeHost(j.host);
        cudaEventDestroy(j.done);
    }
    for (auto& hb : c->spare_host) cudaFreeHost(hb.first);
    for (cudaEvent_t e : c->spare_events) cudaEventDestroy(e);
    for (ps_gpu_plan* P : c->plans) {  // plans outliving their context keep only their host part
        plan_release(P);
        P->ctx = nullptr;
    }
    c->plans.clear();
    free_prec(c->f);
    free_prec(c->d);
    cudaFree(c->partials);
    cudaFree(c->dstatus);
    cudaFree(c->dsums);
    cudaFree(c->dshells);
    cudaFree(c->dminmax);
    cudaFree(c->dlut);
    for (void* p : c->retired) cudaFree(p);
    for (int q = 0; q < 2; q++) {
        for (int r = 0; r < 2; r++) cudaFree(c->stage[q][r]);
        if (c->ev_copied[q]) cudaEventDestroy(c->ev_copied[q]);
        if (c->ev_free[q]) cudaEventDestroy(c->ev_free[q]);
        if (c->pin[q]) cudaFreeHost(c->pin[q]);
        if (c->ev_chunk[q]) cudaEventDestroy(c->ev_chunk[q]);
        if (c->fpin[q]) cudaFreeHost(c->fpin[q]);
        if (c->ev_fpin[q]) cudaEventDestroy(c->ev_fpin[q]);
        if (c->ev_raw[q]) cudaEventDestroy(c->ev_raw[q]);
    }
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->side_stream) {
        cudaStreamSynchronize(c->side_stream);
        cudaStreamDestroy(c->side_stream);
    }
    cudaFree(c->side_partials);
    cudaFree(c->side_lut);
    if (c->lane2_stream) {
        cudaStreamSynchronize(c->lane2_stream);
        cudaStreamDestroy(c->lane2_stream);
    }
    cudaFree(c->lane2_partials);
    cudaFree(c->lane2_lut);
    for (auto& p : c->lane2_work) cudaFree(p);
    if (c->ev_join2) cudaEventDestroy(c->ev_join2);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    delete c;
}

}  // extern "C"
