// ps_kbench: per-kernel CUDA-event times of the hot passes on synthetic data,
// without a context: the forward transform of a 512^3 XHI_DENS field limited
// to band 164 (r2c rows, Y pass, phase-storing X pass), then the FP32 field
// part of one pair group on a 384-point alias-free sub-grid (leg bands 64 and
// 96, 16 closing shells up to band 161: two masked inverse X + Y passes, the
// pair kernel, the forward Y pass and the 16-shell dot pass) -- the shapes of
// the largest group of the 64-configuration 512^3 theta sweep.  About 2.7 GB
// on the device, so it is also the small case for full ncu captures of these
// kernels.  Values are synthetic (unit-modulus spectra, uniform real grids),
// so only times are meaningful.
//
//     python -m polyspectrum_b200.build --kbench
//     polyspectrum_b200/ps_kbench [reps]
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cmath>
#include <algorithm>
#include "ps_launch.cuh"
#include "ps_counts.cuh"

namespace ps {
int launch_fail(cudaError_t e, const char* what)
{
    fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    return 1;
}
template struct L3<float, 96>;
template struct L3<float, 128>;
template struct L3<float, 300>;
template struct L3<float, 320>;
template struct L3<float, 384>;
template struct L3<float, 512>;
}
using namespace ps;
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { fprintf(stderr, "%s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); exit(1);} } while (0)
#define LT(x) do { if ((x) != 0) { fprintf(stderr, "launch failed %s:%d\n", __FILE__, __LINE__); exit(1);} } while (0)

__global__ void k_fill(float2* p, size_t n, unsigned seed)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned h = (unsigned)i * 2654435761u ^ seed;
        h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
        const float a = 6.2831853f * (h & 0xffffff) / 16777216.0f;
        p[i] = make_float2(cosf(a), sinf(a));
    }
}
__global__ void k_fill_real(float* p, size_t n, unsigned seed)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned h = (unsigned)i * 2654435761u ^ seed;
        h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
        p[i] = (h & 0xffff) / 65536.0f;
    }
}
template <int M> Tables<float> make_tables()
{
    std::vector<float2> hp(M), hr(M / 2), h(M);
    L3<float, M>::host_tables(hp.data(), hr.data());
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < M; m++) {
        const long double a = two_pi * (long double)m / (long double)M;
        h[m].x = (float)cosl(a);
        h[m].y = (float)(-sinl(a));
    }
    float2 *a, *b, *c;
    CK(cudaMalloc(&a, M * 8)); CK(cudaMalloc(&b, M / 2 * 8)); CK(cudaMalloc(&c, M * 8));
    CK(cudaMemcpy(a, hp.data(), M * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b, hr.data(), M / 2 * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c, h.data(), M * 8, cudaMemcpyHostToDevice));
    return Tables<float>{a, b, c};
}
static int rup(int a, int b) { return (a + b - 1) / b * b; }

// Mean time of `reps` launches of the Y pass variant <M, INV, RX> over the
// pencils of data (stride S, ncols columns, input rows |my| <= jband, output
// rows |my| <= jout), with its own Stockham table.
template <int M, bool INV, int RX>
double time_pass_y(int reps, float2* data, int S, int ncols, int jband, int jout, const char* what)
{
    using G = PencilGeom<float, M, RX>;
    std::vector<float2> hp(M);
    transform_table<float2, M, G::R, G::TPF>(hp.data());
    float2* tw;
    CK(cudaMalloc(&tw, M * 8));
    CK(cudaMemcpy(tw, hp.data(), M * 8, cudaMemcpyHostToDevice));
    auto kern = k_pass_y<float, M, INV, RX>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, G::THREADS, G::SMEM));
    const unsigned blocks = (unsigned)(M * (ncols / G::W));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int it = 0; it < 3; it++) kern<<<blocks, G::THREADS, G::SMEM>>>(data, S, ncols, 0, jband, jout, tw);
    CK(cudaEventRecord(e0));
    for (int it = 0; it < reps; it++) kern<<<blocks, G::THREADS, G::SMEM>>>(data, S, ncols, 0, jband, jout, tw);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    CK(cudaGetLastError());
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    printf("pass_y %s@%d R=%d: %.4f ms  (%d threads, %d CTAs/SM)\n", what, M, G::R, ms / reps, G::THREADS, per_sm);
    CK(cudaFree(tw));
    return ms / reps;
}

// Row Stockham table of the pair kernel variant <M, RX>.
template <int M, int RX> float2* pair_row_table()
{
    using G = RowGeom<float, M, RX>;
    std::vector<float2> hr(M / 2);
    transform_table<float2, M / 2, G::R, G::TPF>(hr.data());
    float2* d;
    CK(cudaMalloc(&d, M / 2 * 8));
    CK(cudaMemcpy(d, hr.data(), M / 2 * 8, cudaMemcpyHostToDevice));
    return d;
}

// Mean time of `reps` launches of the pair kernel variant <M, RX, KEEP> on
// legs of bands ba, bb (arrays wa, wb of strides Sa, Sb) into w3 (stride S).
template <int M, int RX, bool KEEP>
double time_pair(int reps, const float2* wa, int Sa, int ba, const float2* wb, int Sb, int bb, float2* w3, int S,
                 int bc, const float2* twpp)
{
    using G = RowGeom<float, M, RX>;
    using PGm = PairGeom<float, M, RX, KEEP>;
    const float2* twr = pair_row_table<M, RX>();
    const size_t smem = PGm::smem(2, ba + 1, bb + 1);
    auto kern = k_pair_z<float, M, RX, KEEP>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 0, per_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, G::THREADS, smem));
    const int nrows = M * M, tiles = (nrows + G::WZ - 1) / G::WZ;
    const int grid = std::min(tiles, std::max(per_sm, 1) * sms);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int it = 0; it < 3; it++)
        kern<<<grid, G::THREADS, smem>>>(wa, Sa, ba + 1, wb, Sb, bb + 1, w3, S, bc + 1, nrows, twr, twpp);
    CK(cudaEventRecord(e0));
    for (int it = 0; it < reps; it++)
        kern<<<grid, G::THREADS, smem>>>(wa, Sa, ba + 1, wb, Sb, bb + 1, w3, S, bc + 1, nrows, twr, twpp);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    CK(cudaGetLastError());
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    printf("pair_z@%d R=%d keep=%d: %.4f ms  (%d threads, %d CTAs/SM, %zu B smem)\n", M, G::R, (int)KEEP,
           ms / reps, G::THREADS, per_sm, smem);
    CK(cudaFree((void*)twr));
    return ms / reps;
}

// Mean time of `reps` launches of the exact-count kernel <WRAP, BPT> on the
// lists L (closing shells dcl, ncl of them) with `grid` CTAs over work items
// of rep_slice representatives; the counts of the last launch go to hc.
template <bool WRAP, int BPT, int THREADS = kCountThreads>
double time_counts(int reps, const PairCountLists& L, const int4* dreps, const short4* dmodes, int N,
                   const Shell* dcl, int ncl, unsigned long long* dcounts, int rep_slice, bool one_wave,
                   std::vector<unsigned long long>& hc, bool max_ctas = false)
{
    const int nrep = (int)L.reps.size(), nb = (int)L.modes.size();
    rep_slice = std::max(1, std::min(rep_slice, kCountRepChunk));
    const size_t smem = kCountStageBytes + (size_t)L.nbins * sizeof(unsigned int);
    auto kern = k_pair_counts<WRAP, BPT, THREADS>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 0, per_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem));
    const int nmc = (nb + THREADS * BPT - 1) / (THREADS * BPT), nitems = nmc * ((nrep + rep_slice - 1) / rep_slice);
    const int grid = one_wave ? std::min(nitems, max_ctas ? sms : std::max(per_sm, 1) * sms) : nitems;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float total = 0.f;
    for (int it = 0; it < reps + 2; it++) {
        CK(cudaMemset(dcounts, 0, sizeof(unsigned long long) * ncl));
        CK(cudaEventRecord(e0));
        kern<<<grid, THREADS, smem>>>(dreps, nrep, dmodes, nb, N, L.s_lo, L.nbins, rep_slice, dcl, ncl, dcounts);
        CK(cudaEventRecord(e1));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (it >= 2) total += ms;
    }
    CK(cudaGetLastError());
    hc.assign(ncl, 0ull);
    CK(cudaMemcpy(hc.data(), dcounts, sizeof(unsigned long long) * ncl, cudaMemcpyDeviceToHost));
    printf("pair_counts wrap=%d BPT=%d threads=%d slice=%d %s: %.4f ms  (%d CTAs, %d CTAs/SM, %zu B smem)\n",
           (int)WRAP, BPT, THREADS, rep_slice, one_wave ? (max_ctas ? "one CTA per SM" : "one wave") : "one item per CTA",
           total / reps, grid, per_sm, smem);
    return total / reps;
}
struct Timer {
    std::vector<cudaEvent_t> ev; std::vector<double> acc; int k = 0;
    Timer(int n) : ev(n + 1), acc(n, 0.0) { for (auto& e : ev) CK(cudaEventCreate(&e)); }
    void start() { k = 0; CK(cudaEventRecord(ev[0])); }
    void lap() { CK(cudaEventRecord(ev[++k])); }
    void collect() { CK(cudaEventSynchronize(ev[k]));
        for (int q = 0; q < k; q++) { float ms; CK(cudaEventElapsedTime(&ms, ev[q], ev[q + 1])); acc[q] += ms; } }
};

int main(int argc, char** argv)
{
    const int reps = argc > 1 ? atoi(argv[1]) : 10;
    const int N = 512, SN = 272, hcols = 165, M = 384, ba = 64, bb = 96, bc = 161;
    const size_t n3 = (size_t)N * N * N;
    float *da, *db;
    float2* spec;
    CK(cudaMalloc(&da, n3 * 4)); CK(cudaMalloc(&db, n3 * 4));
    CK(cudaMalloc(&spec, (size_t)N * N * SN * 8));
    k_fill_real<<<1184, 256>>>(da, n3, 3u);
    k_fill_real<<<1184, 256>>>(db, n3, 5u);
    k_fill<<<1184, 256>>>(spec, (size_t)N * N * SN, 17u);
    const int Sa = rup(ba + 1, 16), Sb = rup(bb + 1, 16), S = rup(bc + 1, 16);
    float2 *wa, *wb, *w3;
    CK(cudaMalloc(&wa, (size_t)M * M * Sa * 8)); CK(cudaMalloc(&wb, (size_t)M * M * Sb * 8)); CK(cudaMalloc(&w3, (size_t)M * M * S * 8));
    Shell hs[2] = {};
    const int bands[2] = {ba, bb};
    for (int q = 0; q < 2; q++) { hs[q].kind = SHELL_RANGE; hs[q].band = bands[q]; hs[q].r2lo = (bands[q] - 2) * (bands[q] - 2); hs[q].r2hi = bands[q] * bands[q]; }
    Shell* dsh; CK(cudaMalloc(&dsh, sizeof(hs))); CK(cudaMemcpy(dsh, hs, sizeof(hs), cudaMemcpyHostToDevice));
    const int lut_size = bc * bc + 1;
    std::vector<unsigned short> lut(lut_size, 0);
    for (int c = 0; c < 16; c++) {
        const double r = 32 + (bc - 34) * (c + 0.5) / 16.0;
        for (int r2 = 0; r2 < lut_size; r2++) { const double s = std::sqrt((double)r2); if (s >= r - 2.5 && s <= r + 2.5) lut[r2] |= (unsigned short)(1u << c); }
    }
    unsigned short* dlut; CK(cudaMalloc(&dlut, lut_size * 2)); CK(cudaMemcpy(dlut, lut.data(), lut_size * 2, cudaMemcpyHostToDevice));
    double* partials; CK(cudaMalloc(&partials, (size_t)M * 64 * 16 * sizeof(double)));
    Tables<float> T5 = make_tables<512>(), T3 = make_tables<384>();
    using L5 = L3<float, 512>;
    using L4 = L3<float, 384>;
    const char* names[] = {"fwd_z@512 direct", "fwd_z@512 staged", "fwd_z@512 bulk", "pass_y@512", "fwd_x_store@512", "inv_x A@384", "pass_y A@384", "inv_x B@384",
                           "pass_y B@384", "pair_z@384", "pass_y fwd@384", "fwd_x_dot@384"};
    const int NK = 12;
    int* status;
    CK(cudaMalloc(&status, sizeof(int)));
    CK(cudaMemset(status, 0, sizeof(int)));
    Timer tm(NK);
    for (int it = 0; it < reps + 3; it++) {
        tm.start();
        LT(L5::fwd_z(0, SRC_XHI_F32, da, db, spec, SN, hcols, T5, 0)); tm.lap();
        LT(L5::fwd_z(0, SRC_XHI_F32, da, db, spec, SN, hcols, T5, 1)); tm.lap();
        LT(L5::fwd_z(0, SRC_XHI_F32, da, db, spec, SN, hcols, T5, 1, 0, status)); tm.lap();
        LT(L5::pass_y(0, spec, SN, false, T5, 0, N, 176)); tm.lap();
        LT(L5::fwd_x(0, spec, SN, hcols, SPEC_STORE_PHASE, spec, SN, nullptr, 0, nullptr, 0, nullptr, 0, nullptr, T5,
                     nullptr, 1.0, 0, 0, 0x7fffffff, nullptr, 176, 164)); tm.lap();
        LT(L4::inv_x(0, spec, SN, wa, Sa, LOAD_MASKED, dsh, M / 2 + 1, T3, 0, N, 1)); tm.lap();
        LT(L4::pass_y(0, wa, Sa, true, T3, 0, ba)); tm.lap();
        LT(L4::inv_x(0, spec, SN, wb, Sb, LOAD_MASKED, dsh + 1, M / 2 + 1, T3, 0, N, 1)); tm.lap();
        LT(L4::pass_y(0, wb, Sb, true, T3, 0, bb)); tm.lap();
        LT(L4::pair_z(0, wa, Sa, ba + 1, wb, Sb, bb + 1, w3, S, bc + 1, T3)); tm.lap();
        LT(L4::pass_y(0, w3, S, false, T3, 0, M, 0, bc)); tm.lap();
        int nb = 0;
        LT(L4::fwd_x(0, w3, S, bc + 1, SPEC_DOT, nullptr, 0, spec, SN, nullptr, 16, dlut, lut_size, partials, T3, &nb,
                     1.0, 0, N, lut_size - 1)); tm.lap();
        CK(cudaGetLastError());
        if (it == 2) { CK(cudaDeviceSynchronize()); tm.acc.assign(NK, 0.0); } else tm.collect();
    }
    CK(cudaDeviceSynchronize());
    for (int q = 0; q < NK; q++) printf("%-18s %.4f ms\n", names[q], tm.acc[q] / reps);
    int hstatus = 0;
    CK(cudaMemcpy(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost));
    if (hstatus) { fprintf(stderr, "bulk copy wait expired\n"); return 1; }

    // Y pass variants (elements per thread: the default and twice it)
    time_pass_y<384, true, 0>(reps, wb, Sb, Sb, bb, M, "inv B");
    time_pass_y<384, true, 24>(reps, wb, Sb, Sb, bb, M, "inv B");
    time_pass_y<384, false, 0>(reps, w3, S, S, M, bc, "fwd");
    time_pass_y<384, false, 24>(reps, w3, S, S, M, bc, "fwd");
    time_pass_y<512, false, 0>(reps, spec, SN, 176, N, N, "field");
    time_pass_y<512, false, 32>(reps, spec, SN, 176, N, N, "field");
    time_pass_y<512, false, 8>(reps, spec, SN, 176, N, N, "field");

    // pair kernel variants: the 384-point group above, and a 320-point group
    // (leg bands 52 and 77, closing band 128: the shapes of the third sweep)
    time_pair<384, 0, false>(reps, wa, Sa, ba, wb, Sb, bb, w3, S, bc, T3.twpp);
    time_pair<384, 0, true>(reps, wa, Sa, ba, wb, Sb, bb, w3, S, bc, T3.twpp);
    time_pair<384, 24, true>(reps, wa, Sa, ba, wb, Sb, bb, w3, S, bc, T3.twpp);
    {
        const int a2 = 52, b2 = 77, c2 = 128;
        const int Sa2 = rup(a2 + 1, 16), Sb2 = rup(b2 + 1, 16), S2 = rup(c2 + 1, 16);
        Tables<float> T2 = make_tables<320>();
        time_pair<320, 0, false>(reps, wa, Sa2, a2, wb, Sb2, b2, w3, S2, c2, T2.twpp);
        time_pair<320, 0, true>(reps, wa, Sa2, a2, wb, Sb2, b2, w3, S2, c2, T2.twpp);
        time_pair<320, 20, true>(reps, wa, Sa2, a2, wb, Sb2, b2, w3, S2, c2, T2.twpp);
        // the same group on a 300-point sub-grid (also alias-free: 52 + 77 + 128 < 300)
        Tables<float> T300 = make_tables<300>();
        time_pair<300, 0, false>(reps, wa, Sa2, a2, wb, Sb2, b2, w3, S2, c2, T300.twpp);
        time_pass_y<320, true, 0>(reps, wb, Sb2, Sb2, b2, 320, "inv B");
        time_pass_y<300, true, 0>(reps, wb, Sb2, Sb2, b2, 300, "inv B");
        time_pass_y<320, false, 0>(reps, w3, S2, S2, 320, c2, "fwd");
        time_pass_y<300, false, 0>(reps, w3, S2, S2, 300, c2, "fwd");
    }
    {
        // the smallest group of the sweep (leg bands 13 and 32, closing band 45)
        // on its 128-point grid and on a 96-point grid (13 + 32 + 45 < 96)
        const int a1 = 13, b1 = 32, c1 = 45;
        const int Sa1 = rup(a1 + 1, 16), Sb1 = rup(b1 + 1, 16), S1 = rup(c1 + 1, 16);
        Tables<float> T128 = make_tables<128>(), T96 = make_tables<96>();
        time_pair<128, 0, false>(reps, wa, Sa1, a1, wb, Sb1, b1, w3, S1, c1, T128.twpp);
        time_pair<96, 0, false>(reps, wa, Sa1, a1, wb, Sb1, b1, w3, S1, c1, T96.twpp);
        time_pass_y<128, true, 0>(reps, wb, Sb1, Sb1, b1, 128, "inv B");
        time_pass_y<96, true, 0>(reps, wb, Sb1, Sb1, b1, 96, "inv B");
        time_pass_y<128, false, 0>(reps, w3, S1, S1, 128, c1, "fwd");
        time_pass_y<96, false, 0>(reps, w3, S1, S1, 96, c1, "fwd");
    }
    {
        // exact polygon counts of the largest group: legs |m| in [63.5, 64.5]
        // and [95.5, 96.5], 16 closing shells covering |m| in [32, 161]
        const int NG = 512;
        auto shell = [](double lo, double hi) {
            Shell sh{};
            sh.kind = SHELL_DEFAULT;
            sh.r2lo = (int)std::ceil(lo * lo);
            sh.r2hi = (int)std::floor(hi * hi);
            sh.band = (int)std::ceil(hi);
            return sh;
        };
        const Shell sa = shell(63.5, 64.5), sb = shell(95.5, 96.5);
        std::vector<Shell> cl;
        for (int q = 0; q < 16; q++) cl.push_back(shell(32.0 + 8.0 * q, 32.0 + 8.0 * q + 16.0));
        PairCountLists L;
        if (!pair_count_lists(sa, sb, NG, &L)) { fprintf(stderr, "count lists refused\n"); return 1; }
        int4* dreps; short4* dmodes; Shell* dcl; unsigned long long* dcnt;
        CK(cudaMalloc(&dreps, L.reps.size() * sizeof(int4)));
        CK(cudaMalloc(&dmodes, L.modes.size() * sizeof(short4)));
        CK(cudaMalloc(&dcl, cl.size() * sizeof(Shell)));
        CK(cudaMalloc(&dcnt, cl.size() * sizeof(unsigned long long)));
        CK(cudaMemcpy(dreps, L.reps.data(), L.reps.size() * sizeof(int4), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dmodes, L.modes.data(), L.modes.size() * sizeof(short4), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dcl, cl.data(), cl.size() * sizeof(Shell), cudaMemcpyHostToDevice));
        printf("pair_counts lists: %zu representatives, %zu modes, %d bins, wrap %d\n", L.reps.size(), L.modes.size(),
               L.nbins, (int)L.wrap);
        const int nrep = (int)L.reps.size();
        std::vector<unsigned long long> ref, got;
        time_counts<true, 2>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, (nrep + 1) / 2, false, ref);
        auto check = [&](const std::vector<unsigned long long>& v) {
            if (v != ref) { fprintf(stderr, "pair_counts variant disagrees\n"); exit(1); }
        };
        time_counts<false, 2>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, (nrep + 1) / 2, false, got); check(got);
        time_counts<false, 4>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, (nrep + 2) / 3, false, got); check(got);
        for (int slice : {16, 32, 64, 128}) {
            time_counts<false, 2>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, slice, true, got); check(got);
            time_counts<false, 4>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, slice, true, got); check(got);
            time_counts<true, 2>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, slice, true, got); check(got);
        }
        time_counts<false, 1>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, 64, true, got); check(got);
        time_counts<false, 8>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, 64, true, got); check(got);
        // one CTA per SM (the library's grid: the count lane beside the field lanes)
        for (int slice : {32, 64, 128}) {
            time_counts<false, 4, 256>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, slice, true, got, true); check(got);
            time_counts<false, 4, 512>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, slice, true, got, true); check(got);
            time_counts<false, 2, 512>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, slice, true, got, true); check(got);
            time_counts<false, 4, 1024>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, slice, true, got, true); check(got);
        }
        time_counts<false, 4, 512>(reps, L, dreps, dmodes, NG, dcl, 16, dcnt, 64, true, got); check(got);
    }
    return 0;
}
