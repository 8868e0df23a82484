// ps_gpu_power_spectrum_noalloc: the power spectrum P(k) of a device-resident
// field without any device allocation.
//
// Who needs it: host programs whose GPU memory is owned by another allocator
// and may not be taken by a library behind its back - a framework's caching
// pool that has reserved the device's memory for itself, or a real-time or
// embedded host with a fixed, pre-planned memory budget - where a cudaMalloc
// of the library's own would fail or break that budget.  Everything the
// computation needs beyond the caller's input field and output arrays lives
// in one file-scope device array of fixed size, which the CUDA runtime
// reserves when it loads the library's device code.
//
// Limits and sharing:
//   * grids up to PS_NOALLOC_MAX_N^3 (64^3), at most PS_NOALLOC_MAX_SHELLS
//     shells per call; larger requests are rejected with PS_ERR_ARG;
//   * every GPU that loads the library holds the array (8 MiB) until exit;
//   * all calls on a device share the array and leave their data in it; calls
//     that overlap on the GPU (different streams, or host threads without
//     ordering between them) race on it - serialise them;
//   * the call copies its small tables from host memory, reads its results
//     back and synchronises `stream` before it returns;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.
#include <cmath>
#include <mutex>

#include "ps_launch.cuh"

namespace ps {
PS_EXTERN_L3(float)
PS_EXTERN_L3(double)
}  // namespace ps

using namespace ps;

#define PS_NOALLOC_MAX_N 64
#define PS_NOALLOC_MAX_SHELLS 256
#define PS_NOALLOC_SCRATCH_BYTES (8u << 20)

// The scratch memory of ps_gpu_power_spectrum_noalloc.  In host code this name
// is only a host-side stand-in: its device address comes from
// cudaGetSymbolAddress (noalloc_scratch_ptr below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[PS_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (set up once per device).
int noalloc_scratch_ptr(int dev, unsigned char** out)
{
    if (dev < 0 || dev >= kMaxDevices) return report_error(PS_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return launch_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                                                       "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev] = (unsigned char*)p;
    }
    *out = g_noalloc_ptr[dev];
    return PS_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// B = coef * sumD / (N^3 * count), Npoly = count = rint(sumI / N^3): the
// batched method's normalisation of leg-by-leg configurations.
__global__ void k_noalloc_finalize(int ns, double coef, double n3, const double* __restrict__ sums,
                                   double* __restrict__ out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const double cnt = rint(sums[ns + s] / n3);
    out[2 * s] = __ddiv_rn(__dmul_rn(coef, sums[s]), __dmul_rn(cnt, n3));
    out[2 * s + 1] = cnt;
}

template <int N>
int run_noalloc(cudaStream_t st, unsigned char* base, double L, const float* field, int phase, int ns,
                const double* k, double bw, double* P, double* Npoly)
{
    using V32 = float2;
    using V64 = double2;
    constexpr int W32 = PencilGeom<float, N>::W, W64 = PencilGeom<double, N>::W;
    constexpr int S32 = (N / 2 + 1 + W32 - 1) / W32 * W32;
    constexpr int S64 = (N / 2 + 1 + W64 - 1) / W64 * W64;
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += align256(bytes);
        return p;
    };
    V32* spec32 = (V32*)carve(sizeof(V32) * (size_t)N * N * S32);
    V32* work32 = (V32*)carve(sizeof(V32) * (size_t)N * N * S32);
    V64* work64 = (V64*)carve(sizeof(V64) * (size_t)N * N * S64);
    V32* tw32 = (V32*)carve(sizeof(V32) * N);
    V64* tw64 = (V64*)carve(sizeof(V64) * N);
    V32* twp32 = (V32*)carve(sizeof(V32) * N);
    V32* twr32 = (V32*)carve(sizeof(V32) * N / 2);
    V64* twp64 = (V64*)carve(sizeof(V64) * N);
    V64* twr64 = (V64*)carve(sizeof(V64) * N / 2);
    const Tables<float> tb32{twp32, twr32, tw32};
    const Tables<double> tb64{twp64, twr64, tw64};
    double* partials = (double*)carve(sizeof(double) * (size_t)N * N);
    double* sums = (double*)carve(sizeof(double) * 2 * PS_NOALLOC_MAX_SHELLS);
    double* out = (double*)carve(sizeof(double) * 2 * PS_NOALLOC_MAX_SHELLS);
    Shell* shells = (Shell*)carve(sizeof(Shell) * PS_NOALLOC_MAX_SHELLS);
    if (off > PS_NOALLOC_SCRATCH_BYTES) return report_error(PS_ERR_ARG, "no-alloc scratch too small");

    // twiddles and shells: host values (same expressions as the context's), copied in
    V32 h32[N];
    V64 h64[N];
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < N; m++) {
        const long double a = two_pi * (long double)m / (long double)N;
        h64[m] = V64{(double)cosl(a), (double)(-sinl(a))};
        h32[m] = V32{(float)cosl(a), (float)(-sinl(a))};
    }
    static thread_local Shell hs[PS_NOALLOC_MAX_SHELLS];
    for (int s = 0; s < ns; s++) hs[s] = host_shell(SHELL_DEFAULT, k[s], 0.0, 0.0, bw, L, N);
    V32 hp32[N], hr32[N / 2];
    V64 hp64[N], hr64[N / 2];
    L3<float, N>::host_tables(hp32, hr32);
    L3<double, N>::host_tables(hp64, hr64);
    PS_LCK(cudaMemcpyAsync(tw32, h32, sizeof(h32), cudaMemcpyHostToDevice, st));
    PS_LCK(cudaMemcpyAsync(tw64, h64, sizeof(h64), cudaMemcpyHostToDevice, st));
    PS_LCK(cudaMemcpyAsync(twp32, hp32, sizeof(hp32), cudaMemcpyHostToDevice, st));
    PS_LCK(cudaMemcpyAsync(twr32, hr32, sizeof(hr32), cudaMemcpyHostToDevice, st));
    PS_LCK(cudaMemcpyAsync(twp64, hp64, sizeof(hp64), cudaMemcpyHostToDevice, st));
    PS_LCK(cudaMemcpyAsync(twr64, hr64, sizeof(hr64), cudaMemcpyHostToDevice, st));
    PS_LCK(cudaMemcpyAsync(shells, hs, sizeof(Shell) * ns, cudaMemcpyHostToDevice, st));

    // forward transform of the field (get_FT_field + optional phase normalisation)
    PS_LTRY((L3<float, N>::fwd_z(st, SRC_F32, field, nullptr, spec32, S32, N / 2 + 1, tb32)));
    PS_LTRY((L3<float, N>::pass_y(st, spec32, S32, false, tb32)));
    PS_LTRY((L3<float, N>::fwd_x(st, spec32, S32, N / 2 + 1, phase == 1 ? SPEC_STORE_PHASE : SPEC_STORE,
                                 spec32, S32, nullptr, 0, nullptr, 0, nullptr, 0, nullptr, tb32, nullptr)));
    // per shell: sum_x D^2 (FP32 transform, FP64 sum) and sum_x I^2 (FP64)
    for (int s = 0; s < ns; s++) {
        const int hb = (hs[s].band < N / 2 ? hs[s].band : N / 2) + 1;
        const int Sd = (hb + W32 - 1) / W32 * W32, Si = (hb + W64 - 1) / W64 * W64;
        int nb = 0;
        PS_LTRY((L3<float, N>::inv_x(st, spec32, S32, work32, Sd, LOAD_MASKED, shells + s, N / 2 + 1, tb32)));
        PS_LTRY((L3<float, N>::pass_y(st, work32, Sd, true, tb32)));
        PS_LTRY((L3<float, N>::inv_z(st, work32, Sd, hb, nullptr, nullptr, EPI_REDUCE, 2, partials, tb32, &nb)));
        k_sum_partials<<<1, 1024, 0, st>>>(partials, nb, sums + s, 1, nullptr);
        PS_LTRY((L3<double, N>::inv_x(st, nullptr, S64, work64, Si, LOAD_UNIT, shells + s, N / 2 + 1, tb64)));
        PS_LTRY((L3<double, N>::pass_y(st, work64, Si, true, tb64)));
        PS_LTRY((L3<double, N>::inv_z(st, work64, Si, hb, nullptr, nullptr, EPI_REDUCE, 2, partials, tb64, &nb)));
        k_sum_partials<<<1, 1024, 0, st>>>(partials, nb, sums + ns + s, 1, nullptr);
    }
    const double n3 = (double)N * (double)N * (double)N;
    k_noalloc_finalize<<<(ns + 127) / 128, 128, 0, st>>>(ns, host_norm_coef(L, N, 2), n3, sums, out);
    PS_LCK(cudaGetLastError());
    static thread_local double hout[2 * PS_NOALLOC_MAX_SHELLS];
    PS_LCK(cudaMemcpyAsync(hout, out, sizeof(double) * 2 * ns, cudaMemcpyDeviceToHost, st));
    PS_LCK(cudaStreamSynchronize(st));
    for (int s = 0; s < ns; s++) {
        P[s] = hout[2 * s];
        Npoly[s] = hout[2 * s + 1];
    }
    return PS_OK;
}

}  // namespace

extern "C" int ps_gpu_power_spectrum_noalloc(int nbins, double boxsize, const float* field_dev,
                                             int use_only_phase, int nshell, const double* k,
                                             double kbinwidth, double* P, double* Npoly, void* stream)
{
    if (!field_dev || !k || !P || !Npoly) return report_error(PS_ERR_ARG, "NULL argument");
    if (nbins != 16 && nbins != 32 && nbins != 64)
        return report_error(PS_ERR_ARG, "ps_gpu_power_spectrum_noalloc: grid size must be 16, 32 or 64 "
                                        "(the fixed scratch holds at most 64^3)");
    if (nshell < 1 || nshell > PS_NOALLOC_MAX_SHELLS)
        return report_error(PS_ERR_ARG, "ps_gpu_power_spectrum_noalloc: 1..256 shells per call");
    if (!(boxsize > 0.0) || !std::isfinite(boxsize))
        return report_error(PS_ERR_ARG, "box size must be positive and finite");
    if (!(kbinwidth > 0.0) || !std::isfinite(kbinwidth))
        return report_error(PS_ERR_ARG, "kbinwidth must be positive and finite");
    if (use_only_phase != 0 && use_only_phase != 1) return report_error(PS_ERR_ARG, "use_only_phase must be 0 or 1");
    int dev = 0;
    PS_LCK(cudaGetDevice(&dev));
    unsigned char* base = nullptr;
    PS_LTRY(noalloc_scratch_ptr(dev, &base));
    cudaStream_t st = (cudaStream_t)stream;
    switch (nbins) {
    case 16: return run_noalloc<16>(st, base, boxsize, field_dev, use_only_phase, nshell, k, kbinwidth, P, Npoly);
    case 32: return run_noalloc<32>(st, base, boxsize, field_dev, use_only_phase, nshell, k, kbinwidth, P, Npoly);
    default: return run_noalloc<64>(st, base, boxsize, field_dev, use_only_phase, nshell, k, kbinwidth, P, Npoly);
    }
}
