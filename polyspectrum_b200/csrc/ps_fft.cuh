// In-CTA Stockham FFT of length N with R elements per thread.
//
// A transform of length N is done by TPF = N/R threads.  Thread t holds
// a[e] = x[t + TPF*e] ("canonical layout") on entry and X[t + TPF*e] on exit.
// N is a power of two, or 3 or 5 times one, for the register passes below;
// other lengths 2^a 3^b 5^c take the shared-memory passes (GenericPlan).  Passes are
// radix-R (for N = f 2^k, R = f 2^r: radix-2^r passes, one of a smaller power
// of two if needed, then one radix-R pass last); each thread does R/Rp
// butterflies per pass.  Pass p with radix Rp and span Ns (product of the
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

// cos(2 pi p / q) for integers p, q > 0, evaluated at compile time: the angle
// is folded into [0, pi/4] by the exact symmetries of cos and sin on the
// rational p/q, then summed as a Taylor series (13 terms; the remainder is
// below 1e-24 there).  For the radix-3 / radix-5 constants, whose angles are
// not multiples of pi/16.
__host__ __device__ constexpr double taylor_cos(double t)
{
    double term = 1.0, sum = 1.0;
    for (int i = 1; i <= 13; i++) {
        term *= -t * t / ((2.0 * i - 1.0) * (2.0 * i));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double taylor_sin(double t)
{
    double term = t, sum = t;
    for (int i = 1; i <= 13; i++) {
        term *= -t * t / ((2.0 * i) * (2.0 * i + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double cos_2pi(long long p, long long q)
{
    p %= q;
    if (p < 0) p += q;
    if (2 * p > q) p = q - p;                                  // cos(2pi(1-x)) = cos(2pi x)
    if (4 * p > q) return -cos_2pi(q - 2 * p, 2 * q);          // x > 1/4: -cos(2pi(1/2-x))
    if (8 * p > q) return taylor_sin(6.283185307179586477 * (double)(q - 4 * p) / (double)(4 * q));
    return taylor_cos(6.283185307179586477 * (double)p / (double)q);
}
__host__ __device__ constexpr double sin_2pi(long long p, long long q) { return cos_2pi(q - 4 * p, 4 * q); }

// W_R^k for the forward (e^{-}) or inverse (e^{+}) direction, applied to v.
template <int R, int K, bool INV, typename V> __device__ __forceinline__ V twiddle_const(V v)
{
    if constexpr (K == 0) {
        return v;
    } else if constexpr (4 * K == R) {
        return mul_mi<INV>(v);
    } else if constexpr (32 % R != 0) {
        using T = decltype(v.x);
        constexpr double cd = cos_2pi(K, R), sd = sin_2pi(K, R);
        const T c = (T)cd;
        const T s = INV ? (T)sd : (T)-sd;
        return V{v.x * c - v.y * s, v.x * s + v.y * c};
    } else {
        using T = decltype(v.x);
        constexpr int j = K * (32 / R);
        const T c = (T)cos32(j);
        const T s = INV ? (T)cos32(j - 8) : (T)-cos32(j - 8);  // sin(2 pi j/32) = cos(2 pi (j-8)/32)
        return V{v.x * c - v.y * s, v.x * s + v.y * c};
    }
}

// Decimation-in-frequency DFT of length R in registers, natural order in and
// out: even R splits into two halves, R = 3 and 5 are direct butterflies.
template <int R, bool INV> struct Dft {
    static_assert(R % 2 == 0, "odd DFT lengths other than 3 and 5 are not provided");
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
// y_k = sum_n a_n W_3^{nk}: y0 = a0 + s, y1,2 = a0 - s/2 -/+ i sin(2pi/3) d
// (forward), s = a1 + a2, d = a1 - a2; the inverse swaps the +/- i terms.
template <bool INV> struct Dft<3, INV> {
    template <typename V> static __device__ __forceinline__ void run(V* a)
    {
        using T = decltype(a[0].x);
        constexpr T s3 = (T)sin_2pi(1, 3);
        const V s = cadd(a[1], a[2]), d = csub(a[1], a[2]);
        const V t = V{a[0].x - (T)0.5 * s.x, a[0].y - (T)0.5 * s.y};
        const V u = V{-s3 * d.y, s3 * d.x};  // i sin(2pi/3) d
        a[0] = cadd(a[0], s);
        a[1] = INV ? cadd(t, u) : csub(t, u);
        a[2] = INV ? csub(t, u) : cadd(t, u);
    }
};
// Length 5: with t1 = a1 + a4, t2 = a2 + a3, d1 = a1 - a4, d2 = a2 - a3,
// y0 = a0 + t1 + t2, y1,4 = a0 + c1 t1 + c2 t2 -/+ i (s1 d1 + s2 d2),
// y2,3 = a0 + c2 t1 + c1 t2 -/+ i (s2 d1 - s1 d2) (forward signs),
// c_j = cos(2pi j/5), s_j = sin(2pi j/5).
template <bool INV> struct Dft<5, INV> {
    template <typename V> static __device__ __forceinline__ void run(V* a)
    {
        using T = decltype(a[0].x);
        constexpr T c1 = (T)cos_2pi(1, 5), c2 = (T)cos_2pi(2, 5);
        constexpr T s1 = (T)sin_2pi(1, 5), s2 = (T)sin_2pi(2, 5);
        const V t1 = cadd(a[1], a[4]), t2 = cadd(a[2], a[3]);
        const V d1 = csub(a[1], a[4]), d2 = csub(a[2], a[3]);
        const V r1 = V{a[0].x + c1 * t1.x + c2 * t2.x, a[0].y + c1 * t1.y + c2 * t2.y};
        const V r2 = V{a[0].x + c2 * t1.x + c1 * t2.x, a[0].y + c2 * t1.y + c1 * t2.y};
        const V p1 = V{s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y};
        const V p2 = V{s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y};
        const V i1 = V{-p1.y, p1.x}, i2 = V{-p2.y, p2.x};  // i p
        a[0] = cadd(a[0], cadd(t1, t2));
        a[1] = INV ? cadd(r1, i1) : csub(r1, i1);
        a[4] = INV ? csub(r1, i1) : cadd(r1, i1);
        a[2] = INV ? cadd(r2, i2) : csub(r2, i2);
        a[3] = INV ? csub(r2, i2) : cadd(r2, i2);
    }
};

// Radix plan.  R = f 2^r with f in {1, 3, 5} the odd part of N: passes of
// radix 2^r while possible, then one pass of the power-of-two remainder; for
// f > 1 these cover N / R and one radix-R pass (it carries the odd factor)
// comes last.  Every radix divides R.  With the odd pass last, every pass
// that goes through shared memory has a power-of-two radix and span, which
// the row layout (SmemRow) makes conflict-free.
template <int N, int R> struct RadixPlan {
    __host__ __device__ static constexpr int odd_of(int n) { return n % 2 ? n : odd_of(n / 2); }
    static constexpr int F = odd_of(R);
    static constexpr int R2 = R / F;                  // radix of the power-of-two passes
    static constexpr int TAIL = F > 1 ? 1 : 0;        // the radix-R pass of a mixed length
    static constexpr int N2 = N / (F > 1 ? R : 1);    // what the power-of-two passes cover
    __host__ __device__ static constexpr int count_full(int n) { return n >= R2 ? 1 + count_full(n / R2) : 0; }
    __host__ __device__ static constexpr int rem_of(int n) { return n >= R2 ? rem_of(n / R2) : n; }
    static constexpr int FULL = count_full(N2);
    static constexpr int REM = rem_of(N2);  // 1 if N2 is a power of R2
    static constexpr int NREM = REM > 1 ? 1 : 0;
    static constexpr int P = FULL + NREM + TAIL;
    __host__ __device__ static constexpr int radix(int p)
    {
        return p < FULL ? R2 : (p < FULL + NREM ? REM : R);
    }
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
    static_assert(F == 1 || F == 3 || F == 5, "radix must be 2^r, 3*2^r or 5*2^r");
    static_assert(R2 >= 2 || F > 1, "power-of-two radix must be >= 2");
    static_assert(N % R == 0 && odd_of(N) == F, "length must be R times a power of two");
    static_assert(F == 1 || R2 >= 2 || N == R, "mixed lengths need a power-of-two part in R");
};

// Elements per thread used for each register-plan length (3 2^k and 5 2^k:
// the odd factor times 2 or 4, 4 to 32 threads per transform).
template <int N> struct DefaultRadix {
    static constexpr int value = N == 24 ? 6 : N == 40 ? 10 : N == 48 ? 12 : N == 80 ? 20 : N == 96 ? 12
                               : N == 160 ? 20 : N == 192 ? 12 : N == 320 ? 20 : N == 384 ? 12
                               : N <= 16 ? N : (N == 32 || N == 64 || N == 128 || N == 512) ? 8 : 16;
};

// Thread layout of a transform of length L: R elements per thread, TPF
// threads per transform (a power of two, so rows pack whole warps).  Lengths
// whose odd part is 1, 3 or 5 use the register plan (TPF = L / R); the others
// ("ragged": 30, 60, 150, 300, 600, ...) take TPF threads with R = ceil(L/TPF)
// slots each, the last ones past L idle, and the shared-memory passes.
template <int L> struct LenKind {
    __host__ __device__ static constexpr int odd_of(int n) { return n % 2 ? n : odd_of(n / 2); }
    static constexpr bool RAGGED = !(odd_of(L) == 1 || odd_of(L) == 3 || odd_of(L) == 5);
    static constexpr int RAGGED_TPF = L <= 32 ? 4 : L <= 64 ? 8 : L <= 160 ? 16 : 32;
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
            const int k = v % Ns;
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
                for (int q = 0; q < Rp; q++) sm.template st<Rp, Ns>(j + q * Ns, b[q]);
            }
        }
        if constexpr (!LAST) {
            sync();
#pragma unroll
            for (int e = 0; e < R; e++) a[e] = sm.template ld<Rp, Ns>(t + TPF * e);
            sync();
            fft_passes<V, N, R, INV, P_ + 1>(a, t, sm, twt, sync);
        }
    }
}

// Pass sequence of lengths N = 2^a 3^b 5^c whose odd part does not fit one
// register pass ("ragged" transforms, e.g. 60, 150, 300, 600): radix-8 passes,
// one radix-4 or -2 pass for the rest of the power of two, then one radix-3
// pass per factor 3 and one radix-5 pass per factor 5.  Such transforms keep
// their data in shared memory between passes; each thread does the
// butterflies v = t, t + TPF, ... of a pass.
template <int N> struct GenericPlan {
    __host__ __device__ static constexpr int pow2_of(int n) { return n % 2 ? 1 : 2 * pow2_of(n / 2); }
    __host__ __device__ static constexpr int count_of(int n, int f) { return n % f ? 0 : 1 + count_of(n / f, f); }
    __host__ __device__ static constexpr int ilog2(int v) { return v > 1 ? 1 + ilog2(v / 2) : 0; }
    static constexpr int A = ilog2(pow2_of(N));
    static constexpr int B3 = count_of(N, 3), C5 = count_of(N, 5);
    static constexpr int P8 = A / 3, PR = A % 3 ? 1 : 0;
    static constexpr int P = P8 + PR + B3 + C5;
    __host__ __device__ static constexpr int radix(int p)
    {
        return p < P8 ? 8 : (p < P8 + PR ? (A % 3 == 2 ? 4 : 2) : (p < P8 + PR + B3 ? 3 : 5));
    }
    __host__ __device__ static constexpr int span(int p)
    {
        int s = 1;
        for (int q = 0; q < p; q++) s *= radix(q);
        return s;
    }
    __host__ __device__ static constexpr int tw_off(int p)
    {
        int o = 0;
        for (int q = 0; q < p; q++) o += span(q) * (radix(q) - 1);
        return o;
    }
    __host__ __device__ static constexpr int product()
    {
        int s = 1;
        for (int q = 0; q < P; q++) s *= radix(q);
        return s;
    }
    static_assert(product() == N, "length must be 2^a 3^b 5^c");
};

// Whether a transform of N elements over TPF threads with R elements each
// runs the register passes (RadixPlan; N = R * TPF with the odd part of N in
// R) or the shared-memory passes of GenericPlan.
template <int N, int R, int TPF> struct UseRegisterPlan {
    __host__ __device__ static constexpr int odd_of(int n) { return n % 2 ? n : odd_of(n / 2); }
    static constexpr bool value = R * TPF == N && odd_of(R) == odd_of(N) &&
                                  (odd_of(R) == 1 || odd_of(R) == 3 || odd_of(R) == 5) &&
                                  (odd_of(R) == 1 || R / odd_of(R) >= 2 || N == R);
};

// The passes of GenericPlan<N> on the transform held in shared memory behind
// `sm` (positions 0..N-1); each thread does butterflies t, t + TPF, ...
template <typename V, int N, int R, int TPF, bool INV, int P_ = 0, class Acc, class Sync>
__device__ __forceinline__ void generic_passes(Acc& sm, int t, const V* __restrict__ twt, const Sync& sync)
{
    using Plan = GenericPlan<N>;
    if constexpr (P_ < Plan::P) {
        constexpr int Rp = Plan::radix(P_);
        constexpr int Ns = Plan::span(P_);
        constexpr int NB = N / Rp;                   // butterflies of the pass
        constexpr int BPT = (NB + TPF - 1) / TPF;    // per thread (the last ones partly idle)
        V b[BPT][Rp];
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            const int v = t + TPF * u;
            if (v < NB) {
#pragma unroll
                for (int q = 0; q < Rp; q++) b[u][q] = sm.ld(v + q * NB);
            }
        }
        sync();
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            const int v = t + TPF * u;
            if (v < NB) {
                const int k = v % Ns;
                if constexpr (Ns > 1) {
                    const V* tp = twt + Plan::tw_off(P_) + k * (Rp - 1);
#pragma unroll
                    for (int q = 1; q < Rp; q++) {
                        V w = tp[q - 1];
                        if constexpr (INV) w.y = -w.y;
                        b[u][q] = cmul(b[u][q], w);
                    }
                }
                Dft<Rp, INV>::run(b[u]);
                const int j = (v / Ns) * Ns * Rp + k;
#pragma unroll
                for (int q = 0; q < Rp; q++) sm.st(j + q * Ns, b[u][q]);
            }
        }
        sync();
        generic_passes<V, N, R, TPF, INV, P_ + 1>(sm, t, twt, sync);
    }
}

// A transform of length N held by TPF threads, R elements each (canonical
// layout a[e] = x[t + TPF e]; with R * TPF > N the entries past N are not
// part of the transform and are left as they are).  Register passes when the
// length allows them, else shared-memory passes; either way the buffer behind
// `sm` holds N elements.
template <typename V, int N, int R, int TPF, bool INV, class Acc, class Sync>
__device__ __forceinline__ void fft_any(V (&a)[R], int t, Acc& sm, const V* __restrict__ twt, const Sync& sync)
{
    if constexpr (UseRegisterPlan<N, R, TPF>::value) {
        fft_passes<V, N, R, INV>(a, t, sm, twt, sync);
    } else {
#pragma unroll
        for (int e = 0; e < R; e++)
            if (t + TPF * e < N) sm.st(t + TPF * e, a[e]);
        sync();
        generic_passes<V, N, R, TPF, INV>(sm, t, twt, sync);
#pragma unroll
        for (int e = 0; e < R; e++)
            if (t + TPF * e < N) a[e] = sm.ld(t + TPF * e);
        sync();
    }
}

// Host side: the Stockham table of a pass plan (forward sign), from
// exp(-2 pi i m / M) evaluated in long double.
template <typename V, class Plan> inline void plan_table(V* out)
{
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
template <typename V, int N, int R> inline void stockham_table(V* out) { plan_table<V, RadixPlan<N, R>>(out); }
// the table of the transform fft_any<V, N, R, TPF> runs
template <typename V, int N, int R, int TPF> inline void transform_table(V* out)
{
    if constexpr (UseRegisterPlan<N, R, TPF>::value) plan_table<V, RadixPlan<N, R>>(out);
    else plan_table<V, GenericPlan<N>>(out);
}

// Shared-memory accessor for pencil passes: W transforms interleaved, element
// `pos` of transform `lane` at s[pos*W + lane] (conflict-free when W*sizeof(V)
// = 128 bytes, the tile width of one global row segment).
template <typename V, int W> struct SmemInterleaved {
    V* s;
    int lane;
    template <int Rp, int Ns> __device__ __forceinline__ void st(int pos, V v) { s[pos * W + lane] = v; }
    template <int Rp, int Ns> __device__ __forceinline__ V ld(int pos) const { return s[pos * W + lane]; }
    __device__ __forceinline__ void st(int pos, V v) { s[pos * W + lane] = v; }
    __device__ __forceinline__ V ld(int pos) const { return s[pos * W + lane]; }
};

// Shared-memory accessor for row passes: one row per transform, XOR-swizzled
// within blocks of G = 2^LB elements (128 bytes): element pos of block
// a = pos >> LB lives at pos ^ g(a).
//  * Exchange after a pass of radix Rp and span Ns (both powers of two): the
//    stores of one instruction put lane t at (t/Ns)*Ns*Rp + t%Ns + q*Ns.
//    When Ns*Rp < G the lanes that share an offset within their block differ
//    in a mod Rp, and g(a) = a*Ns moves them apart on the log2(Rp) bits that
//    q occupies; when Ns*Rp >= G they differ in a / K (K = Ns*Rp/G) and
//    g(a) = (a/K)*Ns does the same.  The loads that follow (consecutive
//    positions, one block per G lanes) stay conflict-free under any g.
//  * Elsewhere (r2c post-processing): g(a) = a.
template <typename V> struct SmemRow {
    static constexpr int LB = sizeof(V) == 16 ? 3 : 4;
    static constexpr int G = 1 << LB;
    V* s;
    __host__ __device__ static constexpr int ilog2(int v) { return v > 1 ? 1 + ilog2(v / 2) : 0; }
    template <int Rp, int Ns> __device__ __forceinline__ static int phys_x(int pos)
    {
        const int a = pos >> LB;
        if constexpr (Ns >= G || (Rp & (Rp - 1)) != 0 || (Ns & (Ns - 1)) != 0) {
            return pos ^ (a & (G - 1));
        } else if constexpr (Ns * Rp < G) {
            return pos ^ ((a * Ns) & (G - 1));
        } else {
            return pos ^ (((a >> ilog2(Ns * Rp / G)) * Ns) & (G - 1));
        }
    }
    __device__ __forceinline__ static int phys(int pos) { return pos ^ ((pos >> LB) & (G - 1)); }
    template <int Rp, int Ns> __device__ __forceinline__ void st(int pos, V v) { s[phys_x<Rp, Ns>(pos)] = v; }
    template <int Rp, int Ns> __device__ __forceinline__ V ld(int pos) const { return s[phys_x<Rp, Ns>(pos)]; }
    __device__ __forceinline__ void st(int pos, V v) { s[phys(pos)] = v; }
    __device__ __forceinline__ V ld(int pos) const { return s[phys(pos)]; }
};

}  // namespace ps
