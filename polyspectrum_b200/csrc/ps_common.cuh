// Common device types for the polyspectrum B200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ps {

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };
template <typename T> using V2 = typename Vec2<T>::type;

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return V{a.x + b.x, a.y + b.y}; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return V{a.x - b.x, a.y - b.y}; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b)
{
    return V{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename V> __device__ __forceinline__ V cconj(V a) { return V{a.x, -a.y}; }
// FP32 complex sums as one packed two-lane instruction each (add/sub .f32x2,
// sm_100): per lane the same IEEE round-to-nearest result as the scalar
// FADD, in half the issued instructions of the FFT butterflies.
__device__ __forceinline__ float2 cadd(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "add.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 csub(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "sub.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename V> __device__ __forceinline__ V mul_mi(V a)
{
    if constexpr (INV) return V{-a.y, a.x};
    else return V{a.y, -a.x};
}
template <typename V> __device__ __forceinline__ V czero() { return V{0, 0}; }

// ---------------------------------------------------------------------------
// Shell (k-space filter) descriptors.  The predicates restate the reference's
// filter functions (src/filter.c) with the same FP64 operation order; the
// intrinsics (__dadd_rn etc.) keep nvcc from contracting into FMA, so every
// filter bit equals the one the reference's -std=c99 build computes.
// ---------------------------------------------------------------------------
enum ShellKind : int {
    SHELL_DEFAULT = 0,         // construct_kfilter             filter.c:34-63
    SHELL_RANGE = 1,           // construct_kfilter_with_kbinwidth filter.c:130-162
    SHELL_WATKINSON = 2,       // construct_kfilter_Watkinson   filter.c:178-208
    SHELL_WATKINSON_RANGE = 3  // construct_kfilter_Watkinson_kn filter.c:219-250
};

struct Shell {
    int kind;
    int band;      // every selected mode has |m_x|,|m_y|,|m_z| <= band (host bound)
    int r2lo;      // DEFAULT / RANGE: selected <=> r2lo <= mx^2+my^2+mz^2 <= r2hi
    int r2hi;
    double kk;     // k/(2 pi)*L           (DEFAULT, WATKINSON)
    double mmin;   // kmin/(2 pi)*L        (RANGE kinds)
    double mmax;   // kmax/(2 pi)*L        (RANGE kinds)
    double half;   // 0.5*kbinwidth
    double min2_init;  // 1e30*1e30, the squared start value of get_corners (filter.c:201,267)
};

// Lattice frequency of FFT index idx (filter.c:44-55).
__device__ __forceinline__ int lattice_freq(int idx, int n) { return idx < (n >> 1) ? idx : idx - n; }

// get_corners (filter.c:257-289) on squared radii: min/max over the 8 corners
// of the cube of half-width e around m, folded into (min2, max2).
__device__ __forceinline__ void corners_fold(int mx, int my, int mz, double e, double& min2,
                                             double& max2)
{
    const double x = (double)mx, y = (double)my, z = (double)mz;
    const double xm = __dmul_rn(__dsub_rn(x, e), __dsub_rn(x, e));
    const double xp = __dmul_rn(__dadd_rn(x, e), __dadd_rn(x, e));
    const double ym = __dmul_rn(__dsub_rn(y, e), __dsub_rn(y, e));
    const double yp = __dmul_rn(__dadd_rn(y, e), __dadd_rn(y, e));
    const double zm = __dmul_rn(__dsub_rn(z, e), __dsub_rn(z, e));
    const double zp = __dmul_rn(__dadd_rn(z, e), __dadd_rn(z, e));
    const double c[8] = {__dadd_rn(__dadd_rn(xm, ym), zm), __dadd_rn(__dadd_rn(xp, ym), zm),
                         __dadd_rn(__dadd_rn(xm, yp), zm), __dadd_rn(__dadd_rn(xm, ym), zp),
                         __dadd_rn(__dadd_rn(xp, yp), zm), __dadd_rn(__dadd_rn(xp, ym), zp),
                         __dadd_rn(__dadd_rn(xm, yp), zp), __dadd_rn(__dadd_rn(xp, yp), zp)};
#pragma unroll
    for (int q = 0; q < 8; q++) {
        if (c[q] > max2) max2 = c[q];
        if (c[q] < min2) min2 = c[q];
    }
}

// The DEFAULT and RANGE predicates (filter.c:57-59, :155-158) depend on the
// integer r2 = mx^2+my^2+mz^2 only, through s = fl(sqrt(r2)), which is
// non-decreasing in r2; each is a conjunction of one condition that is
// monotone false->true in s and one that is monotone true->false (fl(a - s)
// is non-increasing in s).  So the selected r2 form one integer interval,
// found by binary search with the exact FP64 predicate (same operations as
// the reference, correctly rounded sqrt on host and device alike).
__host__ __device__ inline double exact_sqrt(double x)
{
#ifdef __CUDA_ARCH__
    return __dsqrt_rn(x);
#else
    return sqrt(x);
#endif
}
__host__ __device__ inline bool pred_lower(const Shell& s, int r2)  // monotone false -> true
{
    const double m = exact_sqrt((double)r2);
    return s.kind == SHELL_DEFAULT ? (s.kk - m <= s.half) : (s.mmin - m <= s.half);
}
__host__ __device__ inline bool pred_upper(const Shell& s, int r2)  // monotone true -> false
{
    const double m = exact_sqrt((double)r2);
    return s.kind == SHELL_DEFAULT ? (s.kk - m >= -s.half) : (m - s.mmax <= s.half);
}
// fabs(kk - m) <= half  <=>  -half <= fl(kk - m) <= half (fabs and negation are exact).
__host__ __device__ inline void shell_r2_interval(Shell& s, int n)
{
    if (s.kind != SHELL_DEFAULT && s.kind != SHELL_RANGE) {
        s.r2lo = 0;
        s.r2hi = 0x7fffffff;
        return;
    }
    const int r2max = 3 * (n / 2) * (n / 2);
    int lo = 0, hi = r2max + 1;  // first r2 with pred_lower (r2max+1: none)
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (pred_lower(s, mid)) hi = mid;
        else lo = mid + 1;
    }
    int a = -1, b = r2max;  // last r2 with pred_upper (-1: none)
    while (a < b) {
        const int mid = a + (b - a + 1) / 2;
        if (pred_upper(s, mid)) a = mid;
        else b = mid - 1;
    }
    s.r2lo = lo;
    s.r2hi = a;
}

__device__ __forceinline__ bool shell_bit(const Shell& s, int mx, int my, int mz)
{
    switch (s.kind) {
    case SHELL_DEFAULT:
    case SHELL_RANGE: {
        const int r2 = mx * mx + my * my + mz * mz;
        return r2 >= s.r2lo && r2 <= s.r2hi;
    }
    case SHELL_WATKINSON: {
        double min2 = s.min2_init, max2 = 0.0;
        corners_fold(mx, my, mz, s.half, min2, max2);
        const double pmin = __dsqrt_rn(min2), pmax = __dsqrt_rn(max2);
        return pmin <= s.kk && s.kk <= pmax;
    }
    case SHELL_WATKINSON_RANGE: {
        double min2 = s.min2_init, max2 = 0.0;
        corners_fold(mx, my, mz, s.half, min2, max2);
        const double pmin = __dsqrt_rn(min2), pmax = __dsqrt_rn(max2);
        return (pmax >= s.mmax && pmin <= s.mmax) || (pmax <= s.mmax && pmin >= s.mmin) ||
               (pmax >= s.mmin && pmin <= s.mmin);
    }
    default:
        return false;
    }
}

// Cheap necessary condition: outside the band cube nothing is selected.
__device__ __forceinline__ bool in_band(const Shell& s, int mx, int my, int mz)
{
    return abs(mx) <= s.band && abs(my) <= s.band && abs(mz) <= s.band;
}

// Bitmask of the shells (of ns <= 32) that select mode m; one out-of-line
// instance so the callers' unrolled loops stay small.
static __device__ __noinline__ unsigned shell_bits(const Shell* __restrict__ sh, int ns, int mx, int my, int mz)
{
    unsigned bits = 0u;
    for (int c = 0; c < ns; c++) {
        const Shell s = sh[c];
        if (in_band(s, mx, my, mz) && shell_bit(s, mx, my, mz)) bits |= 1u << c;
    }
    return bits;
}

// Half-spectrum weight: modes with 0 < h < N/2 stand for themselves and their
// Hermitian mirrors.
__device__ __forceinline__ int herm_weight(int h, int n) { return (h == 0 || h == (n >> 1)) ? 1 : 2; }

}  // namespace ps
