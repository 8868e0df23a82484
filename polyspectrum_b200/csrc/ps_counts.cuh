// Exact polygon counts of a pair group by enumeration in integers: the mode
// lists (host) and the histogram kernel.  Shared by the library and the
// stand-alone timing harness.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <vector>

#include "ps_common.cuh"

namespace ps {

// ------------------------------------------------------------------ exact pair counts
// Polygon counts of a pair group whose shells are all r^2 intervals, by
// enumeration in integers instead of FP64 transforms of unit shells:
//     count(c) = #{(m_a, m_b) in S_a x S_b : |w(m_a + m_b)|^2 in [r2lo_c, r2hi_c]},
// w = componentwise wrap into the grid's lattice frequencies [-N/2, N/2)
// (WRAP: only when a component can reach N/2; aliased triples are counted, as
// the reference's N-grid sums count them).  That is the number of triples
// m_a + m_b + m_c = 0 (mod N) with m_c in S_c (S_c = -S_c).  S_a enters as
// representatives of its orbits under the 48 axis permutations and sign
// flips with their orbit sizes as weights: S_b, the closing shells and |w(.)|^2
// are invariant under them.  The pairs are cut into work items (a chunk of
// THREADS BPT modes of S_b times a slice of rep_slice representatives); each CTA
// of a grid of resident CTAs takes items blockIdx.x, + gridDim.x, ... into
// its own histogram of |w(m_a + m_b)|^2 - s_lo over nbins bins in shared
// memory (integer atomics: the result does not depend on their order), so
// the clearing and the interval sums are paid once per CTA.  Each CTA then sums each closing shell's
// interval and adds it to counts[c].  Without WRAP the bin is
// |m_a|^2 - s_lo + |m_b|^2 + 2 m_a.m_b: the representatives are staged as
// (2x, 2y, 2z, weight) beside |m_a|^2 - s_lo, the modes keep |m_b|^2 (a large
// negative value for the idle slots past nb), so a pair costs three
// multiply-adds, an add and the range test before its atomic.
constexpr int kCountBPT = 4;
constexpr int kCountThreads = 1024;  // one CTA per SM: 32 warps to hide the atomics' latency
constexpr int kCountRepChunk = 512;  // largest rep_slice
constexpr size_t kCountStageBytes = kCountRepChunk * (sizeof(int4) + sizeof(int));
constexpr int kCountMaxBins = 44 * 1024;  // 176 KB of uint32 bins beside the staged representatives

template <bool WRAP, int BPT = kCountBPT, int THREADS = kCountThreads>
__global__ void __launch_bounds__(THREADS)
    k_pair_counts(const int4* __restrict__ reps, int nrep, const short4* __restrict__ modes, int nb, int n, int s_lo,
                  int nbins, int rep_slice, const Shell* __restrict__ closing, int ncl,
                  unsigned long long* __restrict__ counts)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int4* srep = reinterpret_cast<int4*>(smem_raw);
    int* snorm = reinterpret_cast<int*>(smem_raw + kCountRepChunk * sizeof(int4));
    unsigned int* hist = reinterpret_cast<unsigned int*>(smem_raw + kCountStageBytes);
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) hist[i] = 0u;
    const int half = n >> 1;
    constexpr int kChunk = THREADS * BPT;
    rep_slice = max(1, min(rep_slice, kCountRepChunk));  // the staging buffer's size
    const int nmc = (nb + kChunk - 1) / kChunk, nrs = (nrep + rep_slice - 1) / rep_slice;
    const int nitems = nmc * nrs;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int mc = item % nmc, r0 = (item / nmc) * rep_slice;
        const int cnt = min(rep_slice, nrep - r0);
        int bx[BPT], by[BPT], bz[BPT], bn[BPT];
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            const int idx = mc * kChunk + u * THREADS + (int)threadIdx.x;
            const bool valid = idx < nb;
            const short4 m = valid ? modes[idx] : short4{0, 0, 0, 0};
            bx[u] = m.x;
            by[u] = m.y;
            bz[u] = m.z;
            // idle slots: every bin index of theirs is negative (|.|^2 sums stay below 2^29)
            bn[u] = valid ? m.x * m.x + m.y * m.y + m.z * m.z : -(1 << 30);
        }
        __syncthreads();  // the previous item's representatives are no longer read
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
            const int4 a = reps[r0 + i];
            srep[i] = WRAP ? a : int4{2 * a.x, 2 * a.y, 2 * a.z, a.w};
            snorm[i] = a.x * a.x + a.y * a.y + a.z * a.z - s_lo;
        }
        __syncthreads();
#pragma unroll 2
        for (int r = 0; r < cnt; r++) {
            const int4 a = srep[r];
            const int an = snorm[r];
#pragma unroll
            for (int u = 0; u < BPT; u++) {
                int sb;
                if constexpr (WRAP) {
                    int qx = a.x + bx[u], qy = a.y + by[u], qz = a.z + bz[u];
                    qx += (qx < -half) * n - (qx >= half) * n;
                    qy += (qy < -half) * n - (qy >= half) * n;
                    qz += (qz < -half) * n - (qz >= half) * n;
                    sb = bn[u] < 0 ? -1 : qx * qx + qy * qy + qz * qz - s_lo;
                } else {
                    sb = an + bn[u] + a.x * bx[u] + a.y * by[u] + a.z * bz[u];
                }
                if ((unsigned)sb < (unsigned)nbins) atomicAdd(&hist[sb], (unsigned)a.w);
            }
        }
    }
    __syncthreads();
    // closing shell c: the bins of its interval (clamped to the histogram)
    const int lane = threadIdx.x & 31;
    for (int c = 0; c < ncl; c++) {
        const Shell sh = closing[c];
        const int lo = max(sh.r2lo - s_lo, 0), hi = min(sh.r2hi - s_lo, nbins - 1);
        unsigned long long v = 0ull;
        for (int i = lo + (int)threadIdx.x; i <= hi; i += blockDim.x) v += hist[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(&counts[c], v);
    }
}

// sumI[idx[c]] = counts[c] (exact integers, below 2^53)
static __global__ void k_counts_out(int n, const unsigned long long* __restrict__ counts, const int* __restrict__ idx,
                             double* __restrict__ sumI)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) sumI[idx[c]] = (double)counts[c];
}

// Mode lists of an exact pair count (k_pair_counts): the modes of S_b, the
// orbit representatives of S_a with their orbit sizes, the histogram range.
struct PairCountLists {
    std::vector<short4> modes;
    std::vector<int4> reps;
    int s_lo = 0, nbins = 0;
    bool wrap = false;
};

// Modes of an interval shell on the N-grid (lattice frequencies [-N/2, N/2)):
// per (x, y) column the z with r2lo <= x^2 + y^2 + z^2 <= r2hi.
inline std::vector<short4> interval_modes(const Shell& sh, int N)
{
    std::vector<short4> out;
    const int b = std::min(sh.band, N / 2);
    const int top = std::min(b, N / 2 - 1);
    if (sh.r2hi < 0 || sh.r2lo > sh.r2hi) return out;
    for (int x = -b; x <= top; x++)
        for (int y = -b; y <= top; y++) {
            const long long rest_hi = (long long)sh.r2hi - x * x - y * y;
            if (rest_hi < 0) continue;
            const long long rest_lo = (long long)sh.r2lo - x * x - y * y;
            int zmax = (int)sqrt((double)rest_hi);
            while ((long long)zmax * zmax > rest_hi) zmax--;
            while ((long long)(zmax + 1) * (zmax + 1) <= rest_hi) zmax++;
            int zmin = 0;
            if (rest_lo > 0) {
                zmin = (int)sqrt((double)rest_lo);
                while ((long long)zmin * zmin < rest_lo) zmin++;
                while (zmin > 0 && (long long)(zmin - 1) * (zmin - 1) >= rest_lo) zmin--;
            }
            for (int az = zmin; az <= zmax; az++) {
                if (az <= top) out.push_back(short4{(short)x, (short)y, (short)az, 0});
                if (az > 0 && az <= b) out.push_back(short4{(short)x, (short)y, (short)-az, 0});
            }
        }
    return out;
}

// Canonical member of a mode's orbit under axis permutations and sign flips
// on the N-grid: components |x| (as indices, -N/2 stays N/2 = -N/2), sorted.
inline std::array<int, 3> orbit_key(int x, int y, int z)
{
    std::array<int, 3> k = {std::abs(x), std::abs(y), std::abs(z)};
    std::sort(k.begin(), k.end());
    return k;
}

// The lists of a group with interval legs a, b on an N-grid; false when the
// enumeration does not apply (histogram too large for shared memory).
inline bool pair_count_lists(const Shell& sa, const Shell& sb, int N, PairCountLists* L)
{
    // host work O(b^2 + |S|); the enumeration itself |S_a| |S_b| / 48 pairs
    const double est = 4.0 * 3.14159 * (double)std::max(sa.r2hi, 1) * 4.0 * 3.14159 * (double)std::max(sb.r2hi, 1);
    if (std::max(sa.band, sb.band) > 300 || est / 48.0 > 4e10) return false;
    std::vector<short4> ma = interval_modes(sa, N), mb = interval_modes(sb, N);
    if ((double)ma.size() * (double)mb.size() / 48.0 > 4e9) return false;
    if (ma.size() > mb.size()) std::swap(ma, mb);  // representatives from the smaller shell
    std::map<std::array<int, 3>, int> orbits;
    for (const short4& m : ma) orbits[orbit_key(m.x, m.y, m.z)]++;
    L->reps.clear();
    for (const auto& kv : orbits) {
        // a representative as lattice frequencies (N/2 is the index of -N/2)
        int v[3];
        for (int q = 0; q < 3; q++) v[q] = kv.first[q] == N / 2 ? -(N / 2) : kv.first[q];
        L->reps.push_back(int4{v[0], v[1], v[2], kv.second});
    }
    L->modes = mb;
    const int bmax_a = std::min(sa.band, N / 2), bmax_b = std::min(sb.band, N / 2);
    L->wrap = bmax_a + bmax_b >= N / 2;
    const double ra_hi = sqrt((double)std::max(sa.r2hi, 0)), rb_hi = sqrt((double)std::max(sb.r2hi, 0));
    const double ra_lo = sqrt((double)std::max(sa.r2lo, 0)), rb_lo = sqrt((double)std::max(sb.r2lo, 0));
    double smax = (ra_hi + rb_hi) * (ra_hi + rb_hi);
    if (L->wrap) smax = std::min(smax, 3.0 * (N / 2) * (N / 2));
    const double dmin = L->wrap ? 0.0 : std::max({0.0, ra_lo - rb_hi, rb_lo - ra_hi});
    L->s_lo = std::max(0, (int)floor(dmin * dmin) - 1);
    const long long s_hi = (long long)ceil(smax) + 1;
    if (s_hi - L->s_lo + 1 > kCountMaxBins || ma.empty() || mb.empty()) return false;
    L->nbins = (int)(s_hi - L->s_lo + 1);
    return true;
}

}  // namespace ps
