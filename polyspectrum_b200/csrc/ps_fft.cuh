// In-CTA Stockham FFT of length N with R elements per thread.
//
// A transform of length N is done by TPF = N/R threads.  Thread t holds
// a[e] = x[t + TPF*e] ("canonical layout") on entry and X[t + TPF*e] on exit.
// Passes are radix-R (the last one may be a smaller radix, each thread then
// does R/Rp butterflies).  Pass p with radix Rp and span Ns (product of the
// previous radices) computes, for butterfly v in [0, N/Rp):
//     b_q = x[v + q*N/Rp] * W_{Ns*Rp}^{q*(v mod Ns)},  b = DFT_Rp(b),
//     y[(v/Ns)*Ns*Rp + (v mod Ns) + q*Ns] = b_q
// (the Stockham auto-sort form), so no bit reversal is ever needed and the
// last pass writes its outputs back into the registers it read, already in
// canonical layout.  Between passes the data goes through shared memory
// through an accessor (interleaved [pos][lane] for pencil passes, or one row
// per transform for the contiguous axis).
#pragma once

#include "ps_common.cuh"

namespace ps {

// cos(2 pi j / 32), j = 0..31: constants of the in-register butterflies.
__device__ __forceinline__ constexpr double cos32(int j)
{
    constexpr double c[8] = {1.0,
                             0.98078528040323044913,
                             0.92387953251128675613,
                             0.83146961230254523708,
                             0.70710678118654752440,
                             0.55557023301960222474,
                             0.38268343236508977173,
                             0.19509032201612826785};
    j &= 31;
    if (j <= 8) return j == 8 ? 0.0 : c[j];
    if (j <= 16) return -cos32(16 - j);
    return cos32(32 - j);
}

// W_R^k for the forward (e^{-}) or inverse (e^{+}) direction, applied to v.
template <int R, int K, bool INV, typename V> __device__ __forceinline__ V twiddle_const(V v)
{
    if constexpr (K == 0) {
        return v;
    } else if constexpr (4 * K == R) {
        return mul_mi<INV>(v);
    } else {
        using T = decltype(v.x);
        constexpr int j = K * (32 / R);
        const T c = (T)cos32(j);
        const T s = INV ? (T)cos32(j - 8) : (T)-cos32(j - 8);  // sin(2 pi j/32) = cos(2 pi (j-8)/32)
        return V{v.x * c - v.y * s, v.x * s + v.y * c};
    }
}

// Decimation-in-frequency DFT of length R in registers, natural order in and out.
template <int R, bool INV> struct Dft {
    template <typename V> static __device__ __forceinline__ void run(V* a)
    {
        constexpr int H = R / 2;
        V b[H], c[H];
        apply<0>(a, b, c);
        Dft<H, INV>::run(b);
        Dft<H, INV>::run(c);
#pragma unroll
        for (int k = 0; k < H; k++) {
            a[2 * k] = b[k];
            a[2 * k + 1] = c[k];
        }
    }
    template <int K, typename V> static __device__ __forceinline__ void apply(const V* a, V* b, V* c)
    {
        if constexpr (K < R / 2) {
            b[K] = cadd(a[K], a[K + R / 2]);
            c[K] = twiddle_const<R, K, INV>(csub(a[K], a[K + R / 2]));
            apply<K + 1>(a, b, c);
        }
    }
};
template <bool INV> struct Dft<1, INV> {
    template <typename V> static __device__ __forceinline__ void run(V*) {}
};

// Radix plan: passes of radix R while possible, then one pass of the remainder.
template <int N, int R> struct RadixPlan {
    __host__ __device__ static constexpr int count_full(int n) { return n >= R ? 1 + count_full(n / R) : 0; }
    __host__ __device__ static constexpr int rem_of(int n) { return n >= R ? rem_of(n / R) : n; }
    static constexpr int FULL = count_full(N);
    static constexpr int REM = rem_of(N);  // 1 if N is a power of R
    static constexpr int P = FULL + (REM > 1 ? 1 : 0);
    __host__ __device__ static constexpr int radix(int p) { return p < FULL ? R : REM; }
    __host__ __device__ static constexpr int span(int p)
    {
        int s = 1;
        for (int q = 0; q < p; q++) s *= radix(q);
        return s;
    }
    // offset of pass p's twiddles in the Stockham table (entries [k][q-1],
    // k < span(p), q in [1, radix(p))); the table has N - 1 entries in all
    __host__ __device__ static constexpr int tw_off(int p)
    {
        int o = 0;
        for (int q = 0; q < p; q++) o += span(q) * (radix(q) - 1);
        return o;
    }
    static_assert(R >= 2 && (R & (R - 1)) == 0, "radix must be a power of two");
    static_assert((N & (N - 1)) == 0 && N >= R, "length must be a power of two >= R");
};

// Elements per thread used for each transform length.
template <int N> struct DefaultRadix {
    static constexpr int value = N <= 16 ? N : (N == 32 || N == 64 || N == 128 || N == 512) ? 8 : 16;
};

// Synchronisation between passes: the whole CTA (pencil kernels, whose
// transforms span several warps), or only the threads of one row (row
// kernels): __syncwarp when a row lives in one warp, else a named barrier per
// row (ids 1..15; id 0 is __syncthreads').
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
template <int TPF> struct RowSync {
    int bar;         // named barrier id (TPF > 32)
    unsigned mask;   // this row's lanes (TPF <= 32)
    __device__ __forceinline__ void operator()() const
    {
        if constexpr (TPF <= 32) __syncwarp(mask);
        else asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(TPF) : "memory");
    }
};

// Stockham passes.  twt is the transform's twiddle table: for pass p, entry
// tw_off(p) + k*(Rp-1) + (q-1) = W_{Ns*Rp}^{q*k} (forward sign), so the lanes
// of a warp (consecutive k) read it with a stride of Rp-1 entries, which maps
// 8 (FP64) or 16 (FP32) consecutive lanes to distinct shared-memory banks.
template <typename V, int N, int R, bool INV, int P_ = 0, class Acc, class Sync>
__device__ __forceinline__ void fft_passes(V (&a)[R], int t, Acc& sm, const V* __restrict__ twt, const Sync& sync)
{
    using Plan = RadixPlan<N, R>;
    if constexpr (P_ < Plan::P) {
        constexpr int Rp = Plan::radix(P_);
        constexpr int Ns = Plan::span(P_);
        constexpr int BPT = R / Rp;
        constexpr int TPF = N / R;
        constexpr bool LAST = (P_ == Plan::P - 1);
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            V b[Rp];
#pragma unroll
            for (int q = 0; q < Rp; q++) b[q] = a[u + q * BPT];
            const int v = t + TPF * u;
            const int k = v & (Ns - 1);
            if constexpr (Ns > 1) {
                const V* tp = twt + Plan::tw_off(P_) + k * (Rp - 1);
#pragma unroll
                for (int q = 1; q < Rp; q++) {
                    V w = tp[q - 1];
                    if constexpr (INV) w.y = -w.y;
                    b[q] = cmul(b[q], w);
                }
            }
            Dft<Rp, INV>::run(b);
            if constexpr (LAST) {
#pragma unroll
                for (int q = 0; q < Rp; q++) a[u + q * BPT] = b[q];
            } else {
                const int j = (v / Ns) * Ns * Rp + k;
#pragma unroll
                for (int q = 0; q < Rp; q++) sm.st(j + q * Ns, b[q]);
            }
        }
        if constexpr (!LAST) {
            sync();
#pragma unroll
            for (int e = 0; e < R; e++) a[e] = sm.ld(t + TPF * e);
            sync();
            fft_passes<V, N, R, INV, P_ + 1>(a, t, sm, twt, sync);
        }
    }
}

// Host side: the Stockham table of RadixPlan<N, R> (forward sign), from
// exp(-2 pi i m / M) evaluated in long double.
template <typename V, int N, int R> inline void stockham_table(V* out)
{
    using Plan = RadixPlan<N, R>;
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int p = 0; p < Plan::P; p++) {
        const int Rp = Plan::radix(p), Ns = Plan::span(p);
        V* tp = out + Plan::tw_off(p);
        for (int k = 0; k < Ns; k++)
            for (int q = 1; q < Rp; q++) {
                const long double a = two_pi * (long double)(q * k) / (long double)(Ns * Rp);
                tp[k * (Rp - 1) + q - 1].x = (decltype(tp->x))cosl(a);
                tp[k * (Rp - 1) + q - 1].y = (decltype(tp->x))(-sinl(a));
            }
    }
}

// Shared-memory accessor for pencil passes: W transforms interleaved, element
// `pos` of transform `lane` at s[pos*W + lane] (conflict-free when W*sizeof(V)
// = 128 bytes, the tile width of one global row segment).
template <typename V, int W> struct SmemInterleaved {
    V* s;
    int lane;
    __device__ __forceinline__ void st(int pos, V v) { s[pos * W + lane] = v; }
    __device__ __forceinline__ V ld(int pos) const { return s[pos * W + lane]; }
};

// Shared-memory accessor for row passes: one row per transform, XOR-swizzled
// within 128-byte groups: element pos lives at pos ^ ((pos >> LB) & (G-1)),
// G = 2^LB elements per 128 bytes.  Stockham writes of stride Rp (and 2, 4
// interleaved runs) then hit G distinct bank groups per 128-byte wavefront,
// and reads of consecutive positions stay conflict-free.
template <typename V> struct SmemRow {
    static constexpr int LB = sizeof(V) == 16 ? 3 : 4;
    static constexpr int G = 1 << LB;
    V* s;
    __device__ __forceinline__ static int phys(int pos) { return pos ^ ((pos >> LB) & (G - 1)); }
    __device__ __forceinline__ void st(int pos, V v) { s[phys(pos)] = v; }
    __device__ __forceinline__ V ld(int pos) const { return s[phys(pos)]; }
};

}  // namespace ps
