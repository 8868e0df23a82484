// 3D r2c / c2r pass kernels with fused loaders and epilogues.
//
// Layouts (row-major, i = axis 0, j = axis 1, l = axis 2 as in the reference's
// [i][j][l], filter.c:59):
//   real grid     x[(i*N + j)*N + l]
//   half spectrum X[(i*N + j)*S + h], h in [0, S), S >= band, S % W == 0;
//                 only h <= N/2 is spectrum, columns above hold don't-care data
//
// Inverse 3D transform (c2r, unnormalised like FFTW_BACKWARD, fft.c:52):
//   inv_x  : along i for every (j,h) pencil; loads through a shell filter
//   pass_y : along j for every (i,h) pencil, in place
//   inv_z  : c2r along l for every (i,j) row; epilogue stores / multiplies /
//            reduces the real field
// Forward 3D transform (r2c, unnormalised like FFTW_FORWARD, fft.c:32):
//   fwd_z  : r2c along l, loader composes the input field
//   pass_y : along j
//   fwd_x  : along i; epilogue stores the spectrum (optionally phase only) or
//            folds it into per-shell dot products
#pragma once

#include "ps_common.cuh"
#include "ps_fft.cuh"

namespace ps {

constexpr int MAX_DOT_SHELLS = 16;

// Pencils per CTA in the strided passes: one 128-byte segment of a row.
template <typename T> struct PencilWidth { static constexpr int value = 128 / (int)sizeof(V2<T>); };
// Rows per CTA in the contiguous-axis passes.
template <typename T, int N> struct RowsPerCta {
    static constexpr int NH = N / 2;
    static constexpr int TPF = NH / DefaultRadix<NH>::value;
    static constexpr int value = TPF >= 64 ? 4 : (TPF >= 16 ? 8 : (TPF >= 4 ? 16 : 32));
};

template <typename T, int N> struct PencilGeom {
    static constexpr int R = DefaultRadix<N>::value;
    static constexpr int TPF = N / R;
    static constexpr int W = PencilWidth<T>::value;
    static constexpr int THREADS = TPF * W;
    static constexpr size_t SMEM = (size_t)N * W * sizeof(V2<T>);
};
template <typename T, int N> struct RowGeom {
    static constexpr int NH = N / 2;
    static constexpr int R = DefaultRadix<NH>::value;
    static constexpr int TPF = NH / R;
    static constexpr int WZ = RowsPerCta<T, N>::value;
    static constexpr int THREADS = TPF * WZ;
    static constexpr int ROW = NH + NH / 32 + 2;  // padded row (>= NH+1)
    static constexpr size_t SMEM = (size_t)ROW * WZ * sizeof(V2<T>);
};

// ------------------------------------------------------------------ reductions
// Deterministic block sum: fixed shuffle tree, then warp partials in order.
template <int THREADS> __device__ __forceinline__ double block_sum(double v, double* red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    constexpr int NW = (THREADS + 31) / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
#pragma unroll 1
        for (int q = 0; q < NW; q++) s += red[q];
    }
    return s;
}

// ------------------------------------------------------------------ inverse X
enum InvLoad : int { LOAD_PLAIN = 0, LOAD_MASKED = 1, LOAD_UNIT = 2 };

template <typename T, int N>
__global__ void __launch_bounds__(PencilGeom<T, N>::THREADS)
    k_inv_x(const V2<T>* __restrict__ src, int src_stride, V2<T>* __restrict__ dst, int dst_stride,
            int mode, const Shell* __restrict__ shell_p, int hvalid, const V2<T>* __restrict__ tw)
{
    using G = PencilGeom<T, N>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemInterleaved<V, G::W> sm{reinterpret_cast<V*>(smem_raw), (int)(threadIdx.x % G::W)};
    const int w = threadIdx.x % G::W, t = threadIdx.x / G::W;
    const int tiles_per_row = dst_stride / G::W;
    const int j = blockIdx.x / tiles_per_row;
    const int h = (blockIdx.x % tiles_per_row) * G::W + w;
    const int my = lattice_freq(j, N);
    const int mz = h == N / 2 ? -(N / 2) : h;
    const bool col_ok = h < hvalid && h <= N / 2;
    Shell sh;
    if (mode != LOAD_PLAIN) sh = *shell_p;
    const bool pencil_live =
        col_ok && (mode == LOAD_PLAIN || (abs(my) <= sh.band && abs(mz) <= sh.band));
    // filter bits of this thread's R modes, one predicate instance (loop not unrolled)
    unsigned bits = 0u;
    if (pencil_live) {
        if (mode == LOAD_PLAIN) {
            bits = (1u << G::R) - 1u;
        } else {
#pragma unroll 1
            for (int e = 0; e < G::R; e++) {
                const int mx = lattice_freq(t + G::TPF * e, N);
                if (abs(mx) <= sh.band && shell_bit(sh, mx, my, mz)) bits |= 1u << e;
            }
        }
    }
    V a[G::R];
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int i = t + G::TPF * e;
        V v = czero<V>();
        if ((bits >> e) & 1u) {
            if (mode == LOAD_UNIT) v = V{(T)1, (T)0};
            else v = src[((size_t)i * N + j) * src_stride + h];
        }
        a[e] = v;
    }
    fft_passes<V, N, G::R, true, N>(a, t, sm, tw);
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int i = t + G::TPF * e;
        dst[((size_t)i * N + j) * dst_stride + h] = a[e];
    }
}

// ------------------------------------------------------------------ Y pass
template <typename T, int N, bool INV>
__global__ void __launch_bounds__(PencilGeom<T, N>::THREADS)
    k_pass_y(V2<T>* __restrict__ data, int stride, const V2<T>* __restrict__ tw)
{
    using G = PencilGeom<T, N>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemInterleaved<V, G::W> sm{reinterpret_cast<V*>(smem_raw), (int)(threadIdx.x % G::W)};
    const int w = threadIdx.x % G::W, t = threadIdx.x / G::W;
    const int tiles_per_plane = stride / G::W;
    const int i = blockIdx.x / tiles_per_plane;
    const int h = (blockIdx.x % tiles_per_plane) * G::W + w;
    V* base = data + (size_t)i * N * stride + h;
    V a[G::R];
#pragma unroll
    for (int e = 0; e < G::R; e++) a[e] = base[(size_t)(t + G::TPF * e) * stride];
    fft_passes<V, N, G::R, INV, N>(a, t, sm, tw);
#pragma unroll
    for (int e = 0; e < G::R; e++) base[(size_t)(t + G::TPF * e) * stride] = a[e];
}

// ------------------------------------------------------------------ inverse Z (c2r)
enum RealEpi : int {
    EPI_STORE = 0,      // out = x^p
    EPI_MUL_STORE = 1,  // out = x^p * aux   (aux may alias out)
    EPI_MUL_REDUCE = 2, // sum x^p * aux
    EPI_REDUCE = 3      // sum x^p
};

template <typename T> __device__ __forceinline__ T ipow(T x, int p)
{
    T r = x;
    for (int q = 1; q < p; q++) r *= x;
    return r;
}

template <typename T, int N>
__global__ void __launch_bounds__(RowGeom<T, N>::THREADS)
    k_inv_z(const V2<T>* __restrict__ src, int src_stride, int hvalid, T* out, const T* aux,
            int epi, int power, double* __restrict__ partials, const V2<T>* __restrict__ tw)
{
    using G = RowGeom<T, N>;
    using V = V2<T>;
    constexpr int NH = G::NH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[(G::THREADS + 31) / 32];
    const int w = threadIdx.x / G::TPF, t = threadIdx.x % G::TPF;
    V* srow = reinterpret_cast<V*>(smem_raw) + w * G::ROW;
    const size_t row = (size_t)blockIdx.x * G::WZ + w;
    const V* zr = src + row * src_stride;
    for (int hh = t; hh <= NH; hh += G::TPF) srow[hh] = hh < hvalid ? zr[hh] : czero<V>();
    __syncthreads();
    V a[G::R];
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int k = t + G::TPF * e;
        const V zk = srow[k];
        const V zm = cconj(srow[NH - k]);
        const V A = cadd(zk, zm);
        const V B = cmul(csub(zk, zm), cconj(tw[k]));  // exp(+2 pi i k / N)
        a[e] = V{A.x - B.y, A.y + B.x};
    }
    __syncthreads();
    SmemRow<V> sm{srow};
    fft_passes<V, NH, G::R, true, N>(a, t, sm, tw);
    double acc = 0.0;
    T* orow = out ? out + row * N : nullptr;
    const T* arow = aux ? aux + row * N : nullptr;
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int n2 = 2 * (t + G::TPF * e);
        T x0 = ipow(a[e].x, power), x1 = ipow(a[e].y, power);
        if (epi == EPI_STORE) {
            *reinterpret_cast<V*>(orow + n2) = V{x0, x1};
        } else if (epi == EPI_MUL_STORE) {
            const V q = *reinterpret_cast<const V*>(arow + n2);
            *reinterpret_cast<V*>(orow + n2) = V{x0 * q.x, x1 * q.y};
        } else if (epi == EPI_MUL_REDUCE) {
            const V q = *reinterpret_cast<const V*>(arow + n2);
            acc += (double)x0 * (double)q.x + (double)x1 * (double)q.y;
        } else {
            acc += (double)x0 + (double)x1;
        }
    }
    if (epi == EPI_MUL_REDUCE || epi == EPI_REDUCE) {
        const double s = block_sum<G::THREADS>(acc, red);
        if (threadIdx.x == 0) partials[blockIdx.x] = s;
    }
}

// ------------------------------------------------------------------ forward Z (r2c)
enum RealSrcKind : int {
    SRC_F32 = 0,       // a
    SRC_F64 = 1,       // a
    SRC_XHI_F32 = 2,   // (double)a * (1 - (double)b), input_field.c:33
    SRC_XHI_F64 = 3,
    SRC_T = 4          // array of the transform's own type
};

template <typename T>
__device__ __forceinline__ T load_real(int kind, const void* a, const void* b, size_t idx)
{
    switch (kind) {
    case SRC_F32:
        return (T)((const float*)a)[idx];
    case SRC_F64:
        return (T)((const double*)a)[idx];
    case SRC_XHI_F32: {
        const double d = (double)((const float*)a)[idx], x = (double)((const float*)b)[idx];
        return (T)__dmul_rn(d, __dsub_rn(1.0, x));
    }
    case SRC_XHI_F64: {
        const double d = ((const double*)a)[idx], x = ((const double*)b)[idx];
        return (T)__dmul_rn(d, __dsub_rn(1.0, x));
    }
    default:
        return ((const T*)a)[idx];
    }
}

template <typename T, int N>
__global__ void __launch_bounds__(RowGeom<T, N>::THREADS)
    k_fwd_z(int kind, const void* __restrict__ a_src, const void* __restrict__ b_src,
            V2<T>* __restrict__ dst, int dst_stride, int hout, const V2<T>* __restrict__ tw)
{
    using G = RowGeom<T, N>;
    using V = V2<T>;
    constexpr int NH = G::NH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = threadIdx.x / G::TPF, t = threadIdx.x % G::TPF;
    V* srow = reinterpret_cast<V*>(smem_raw) + w * G::ROW;
    const size_t row = (size_t)blockIdx.x * G::WZ + w;
    V a[G::R];
    if (kind == SRC_T) {
        const V* xr = reinterpret_cast<const V*>((const T*)a_src + row * N);
#pragma unroll
        for (int e = 0; e < G::R; e++) a[e] = xr[t + G::TPF * e];
    } else {
#pragma unroll
        for (int e = 0; e < G::R; e++) {
            const size_t n2 = row * N + 2 * (t + G::TPF * e);
            a[e] = V{load_real<T>(kind, a_src, b_src, n2), load_real<T>(kind, a_src, b_src, n2 + 1)};
        }
    }
    SmemRow<V> sm{srow};
    fft_passes<V, NH, G::R, false, N>(a, t, sm, tw);
    __syncthreads();
#pragma unroll
    for (int e = 0; e < G::R; e++) sm.st(t + G::TPF * e, a[e]);
    __syncthreads();
    V* xo = dst + row * dst_stride;
    const T half = (T)0.5;
    for (int k = t; k <= NH && k < hout; k += G::TPF) {
        const V yk = sm.ld(k & (NH - 1));
        const V ym = cconj(sm.ld((NH - k) & (NH - 1)));
        const V E = V{(yk.x + ym.x) * half, (yk.y + ym.y) * half};
        const V D = csub(yk, ym);
        const V O = V{D.y * half, -D.x * half};  // D / (2i)
        xo[k] = cadd(E, cmul(tw[k], O));
    }
}

// ------------------------------------------------------------------ forward X
enum SpecEpi : int {
    SPEC_STORE = 0,        // out = X
    SPEC_STORE_PHASE = 1,  // out = X / |X|  (utils_fftw.c:78-93)
    SPEC_DOT = 2,          // per shell c: sum_m w(h) F_c(m) Re(dk(m) conj(X(m)))
    SPEC_COUNT = 3,        // per shell c: sum_m w(h) F_c(m) rint(Re X(m) / N^3)
    SPEC_MASK_STORE = 4    // out = F(m) X(m)
};

template <typename T, int N>
__global__ void __launch_bounds__(PencilGeom<T, N>::THREADS)
    k_fwd_x(V2<T>* data, int stride, int hvalid, int epi, V2<T>* out, int out_stride,
            const V2<T>* __restrict__ dk, int dk_stride, const Shell* __restrict__ shells,
            int nshell, double* __restrict__ partials, const V2<T>* __restrict__ tw)
{
    using G = PencilGeom<T, N>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[(G::THREADS + 31) / 32];
    SmemInterleaved<V, G::W> sm{reinterpret_cast<V*>(smem_raw), (int)(threadIdx.x % G::W)};
    const int w = threadIdx.x % G::W, t = threadIdx.x / G::W;
    const int tiles_per_row = stride / G::W;
    const int j = blockIdx.x / tiles_per_row;
    const int h = (blockIdx.x % tiles_per_row) * G::W + w;
    const bool col_ok = h < hvalid && h <= N / 2;
    V a[G::R];
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int i = t + G::TPF * e;
        a[e] = data[((size_t)i * N + j) * stride + h];
    }
    fft_passes<V, N, G::R, false, N>(a, t, sm, tw);
    const int my = lattice_freq(j, N);
    const int mz = h == N / 2 ? -(N / 2) : h;
    if (epi == SPEC_STORE || epi == SPEC_STORE_PHASE || epi == SPEC_MASK_STORE) {
        unsigned keep = (1u << G::R) - 1u;
        if (epi == SPEC_MASK_STORE) {
            keep = 0u;
            const Shell sh = shells[0];
            if (col_ok) {
#pragma unroll 1
                for (int e = 0; e < G::R; e++) {
                    const int mx = lattice_freq(t + G::TPF * e, N);
                    if (in_band(sh, mx, my, mz) && shell_bit(sh, mx, my, mz)) keep |= 1u << e;
                }
            }
        }
        if (h >= out_stride) return;
#pragma unroll
        for (int e = 0; e < G::R; e++) {
            const int i = t + G::TPF * e;
            V v = a[e];
            if (epi == SPEC_STORE_PHASE) {
                if constexpr (sizeof(T) == 8) {
                    const double m = hypot(v.x, v.y);
                    v = V{v.x / m, v.y / m};
                } else {
                    const float m = hypotf(v.x, v.y);
                    v = V{v.x / m, v.y / m};
                }
            } else if (!((keep >> e) & 1u)) {
                v = czero<V>();
            }
            out[((size_t)i * N + j) * out_stride + h] = v;
        }
        return;
    }
    // SPEC_DOT / SPEC_COUNT: per-shell accumulation in FP64
    double acc[MAX_DOT_SHELLS];
#pragma unroll
    for (int c = 0; c < MAX_DOT_SHELLS; c++) acc[c] = 0.0;
    if (col_ok) {
        const double wgt = (double)herm_weight(h, N);
        const double inv_n3 = 1.0 / ((double)N * (double)N * (double)N);
#pragma unroll
        for (int e = 0; e < G::R; e++) {
            const int i = t + G::TPF * e;
            const unsigned sel = shell_bits(shells, nshell, lattice_freq(i, N), my, mz);
            if (sel) {
                double val;
                if (epi == SPEC_DOT) {
                    const V d = dk[((size_t)i * N + j) * dk_stride + h];
                    val = wgt * ((double)d.x * (double)a[e].x + (double)d.y * (double)a[e].y);
                } else {
                    val = wgt * rint((double)a[e].x * inv_n3);
                }
#pragma unroll
                for (int c = 0; c < MAX_DOT_SHELLS; c++)
                    if ((sel >> c) & 1u) acc[c] += val;
            }
        }
    }
#pragma unroll 1
    for (int c = 0; c < nshell; c++) {
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < MAX_DOT_SHELLS; q++)
            if (q == c) v = acc[q];
        const double s = block_sum<G::THREADS>(v, red);
        if (threadIdx.x == 0) partials[(size_t)c * gridDim.x + blockIdx.x] = s;
    }
}

// ------------------------------------------------------------------ final sums
// out[c] = sum_b partials[c*nblocks + b], fixed order (one CTA per column).
static __global__ void k_sum_partials(const double* __restrict__ partials, int nblocks, double* out,
                               int out_stride)
{
    __shared__ double red[32];
    const double* p = partials + (size_t)blockIdx.x * nblocks;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += p[b];
    s = block_sum<1024>(s, red);
    if (threadIdx.x == 0) out[(size_t)blockIdx.x * out_stride] = s;
}

// ------------------------------------------------------------------ DERIVED k-range
// min/max of squared corner radii over the DEFAULT-filter modes of a shell
// (construct_kfilter_with_determining_kbinwidth, filter.c:78-114).  The
// reference folds the running min/max through sqrt and back per voxel; for
// binary64 sqrt(fl(s*s)) = s, so that equals sqrt of the global min/max of the
// squared corners whatever the visiting order.  Non-negative doubles order
// like their bit patterns, so the fold is an integer atomicMin/atomicMax.
static __global__ void k_derived_range(int n, const Shell* __restrict__ shell_p, int hmax,
                                unsigned long long* minmax_bits)
{
    const Shell sh = *shell_p;
    const int band = min(sh.band, n / 2);
    const int side = 2 * band + 1;
    double min2 = sh.min2_init, max2 = 0.0;
    const long long total = (long long)side * side * (hmax + 1);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int hz = (int)(q % (hmax + 1));
        const long long r = q / (hmax + 1);
        const int mx = (int)(r / side) - band, my = (int)(r % side) - band;
        if (mx >= n / 2 || my >= n / 2 || mx < -(n / 2) || my < -(n / 2)) continue;
        const int mz = hz == n / 2 ? -(n / 2) : hz;
        if (shell_bit(sh, mx, my, mz)) corners_fold(mx, my, mz, sh.half, min2, max2);
    }
    // min2/max2 are non-negative (or the +huge start value)
    unsigned long long lo = __double_as_longlong(min2), hi = __double_as_longlong(max2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_down_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_down_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&minmax_bits[0], lo);
        atomicMax(&minmax_bits[1], hi);
    }
}

}  // namespace ps
