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
//   pair_z : c2r of two rows, product, r2c of the product (pair groups)
// Forward 3D transform (r2c, unnormalised like FFTW_FORWARD, fft.c:32):
//   fwd_z  : r2c along l, loader composes the input field
//   pass_y : along j
//   fwd_x  : along i; epilogue stores the spectrum (optionally phase only) or
//            folds it into per-shell dot products
//
// Every kernel stages the twiddle table W_N^m (m < N) in shared memory first;
// row kernels synchronise per row (warp or named barrier), pencil kernels per
// CTA (a pencil's threads span several warps).
#pragma once

#include "ps_common.cuh"
#include "ps_fft.cuh"

namespace ps {

constexpr int MAX_DOT_SHELLS = 16;

// Pencils per CTA in the strided passes: one 128-byte segment of a row.
template <typename T> struct PencilWidth { static constexpr int value = 128 / (int)sizeof(V2<T>); };

// Threads per pencil (strided-axis) transform: N / (register-plan radix),
// with radix 16 for FP32 at N = 512 so a CTA of 16 pencils is 512 threads;
// ragged lengths take LenKind's thread count (64 for FP64 pencils above 512).
template <typename T, int N> struct PencilThreads {
    static constexpr int value = LenKind<N>::RAGGED ? ((sizeof(T) == 8 && N > 512) ? 64 : LenKind<N>::RAGGED_TPF)
                               : N / ((sizeof(T) == 4 && N == 512) ? 16 : DefaultRadix<N>::value);
};
// RX > 0 overrides the elements per thread of a register-plan pencil length
// (pass variants with fewer, larger radix passes).
template <typename T, int N, int RX = 0> struct PencilGeom {
    static constexpr int TPF = RX > 0 && !LenKind<N>::RAGGED ? N / RX : PencilThreads<T, N>::value;
    static constexpr int R = (N + TPF - 1) / TPF;
    // element e of thread t is position t + TPF e of the transform; with
    // R * TPF > N (ragged lengths) the positions past N are idle slots
    static constexpr bool FULL = R * TPF == N;
    __device__ static constexpr bool live(int pos) { return FULL || pos < N; }
    // one 128-byte segment per row, whole warps per CTA, at most 512 threads
    // (so an epilogue keeps 16 FP64 accumulators in registers)
    static constexpr int W0 = PencilWidth<T>::value * TPF >= 32 ? PencilWidth<T>::value : 32 / TPF;
    static constexpr int W = W0 * TPF > 512 ? 512 / TPF : W0;
    static constexpr int THREADS = TPF * W;
    static constexpr size_t TW_BYTES = (size_t)N * sizeof(V2<T>);  // Stockham table (N-1 used)
    static constexpr size_t SMEM = TW_BYTES + (size_t)N * W * sizeof(V2<T>);
    // FP32 dot passes also stage the tile's field-spectrum pencils ([N][W],
    // interleaved like the exchange buffer) when that fits in shared memory
    static constexpr size_t DK_BYTES = (size_t)N * W * sizeof(V2<T>);
    static constexpr bool DK_SMEM = sizeof(T) == 4 && SMEM + DK_BYTES <= 227 * 1024;
    static constexpr size_t SMEM_DOT = SMEM + (DK_SMEM ? DK_BYTES : 0);
};

// The alternative pencil geometry of the FP32 Y pass for the larger
// register-plan lengths: twice the elements per thread, half the threads per
// pencil, one radix pass fewer (0: none).  Chosen per length by the plan
// autotuner against the default.
template <typename T, int N> struct PencilAlt {
    static constexpr int value = (sizeof(T) == 4 && !LenKind<N>::RAGGED && N >= 128 && N <= 512) ? 2 * PencilGeom<T, N>::R : 0;
};

// Elements per thread of the row (contiguous-axis) transforms of length NH:
// at most 32 threads per row (warp-synchronous) except FP64 rows of 512,
// which use radix 8 and 64 threads (two transforms must fit in registers).
template <typename T, int NH> struct RowRadix {
    static constexpr bool POW2 = (NH & (NH - 1)) == 0;
    // rows of 160 (320-point grids): radix 10 keeps two row transforms in
    // registers (radix 20 needed over 220 registers per thread)
    static constexpr int value = NH == 160 ? 10 : !POW2 ? DefaultRadix<NH>::value
                               : NH <= 16 ? NH : ((sizeof(T) == 4 && NH == 512) ? 16 : 8);
};
// RX > 0 overrides the elements per thread of a register-plan row length
// (the pair kernel's variants).
template <typename T, int N, int RX = 0> struct RowGeom {
    static constexpr int NH = N / 2;
    static constexpr int TPF = LenKind<NH>::RAGGED ? LenKind<NH>::RAGGED_TPF : NH / (RX > 0 ? RX : RowRadix<T, NH>::value);
    static constexpr int R = (NH + TPF - 1) / TPF;
    // element e of thread t is pair t + TPF e of the row; with R * TPF > NH
    // (ragged lengths) the pairs past NH are idle slots
    static constexpr bool FULL = R * TPF == NH;
    __device__ static constexpr bool live(int n) { return FULL || n < NH; }
    static constexpr int EPC = 16 / (int)sizeof(V2<T>);  // complex elements per 16-byte copy
    // rows per CTA (tile): up to 256 threads and 32 rows, and as many as fit
    // in 227 KB of shared memory with two double-buffered full-length inputs
    static constexpr int WZ0 = (256 / TPF) < 32 ? (256 / TPF) : 32;
    static constexpr size_t ROW_BYTES =
        (size_t)((NH < 16 ? NH : (NH + 15) / 16 * 16) + 4 * ((NH + 1 + EPC - 1) / EPC * EPC)) * sizeof(V2<T>);
    static constexpr int WZ_FIT = (int)((227 * 1024 - (size_t)(2 * NH + 2) * sizeof(V2<T>)) / ROW_BYTES);
    __host__ __device__ static constexpr int pow2_floor(int v) { return v >= 2 ? 2 * pow2_floor(v / 2) : 1; }
    // and a divisor of the N^2 rows, so whole tiles cover the grid
    __host__ __device__ static constexpr int pow2_dividing(int v, int cap) { return cap > 1 && v % cap ? pow2_dividing(v, cap / 2) : cap; }
    static constexpr int WZ = pow2_dividing(N * N, pow2_floor(WZ0 < WZ_FIT ? WZ0 : WZ_FIT));
    static constexpr int THREADS = TPF * WZ;
    // shared memory: row Stockham table [NH], pre/post twiddles W_N^k, k <= NH
    // [NH+2], per-row exchange buffers [WZ][NH], then the input stages
    static constexpr size_t TWR_OFF = 0;
    static constexpr size_t TWPP_OFF = TWR_OFF + (size_t)NH * sizeof(V2<T>);
    static constexpr size_t ROWBUF_OFF = TWPP_OFF + (size_t)(NH + 2) * sizeof(V2<T>);
    // row exchange buffers hold whole swizzle blocks of SmemRow (16 elements:
    // its XOR stays inside a block, which a ragged NH may end in the middle of)
    static constexpr int ROWBUF = NH < 16 ? NH : (NH + 15) / 16 * 16;
    static constexpr size_t STAGE_OFF = ROWBUF_OFF + (size_t)WZ * ROWBUF * sizeof(V2<T>);
    // input stage pitch (elements) for rows of hv valid entries
    __host__ __device__ static constexpr int pitch(int hv) { return (hv + EPC - 1) / EPC * EPC; }
    // dynamic shared memory of a kernel with `ninputs` double-buffered inputs
    __host__ __device__ static constexpr size_t smem(int ninputs, int hva, int hvb)
    {
        return STAGE_OFF + (size_t)2 * WZ * (pitch(hva) + (ninputs > 1 ? pitch(hvb) : 0)) * sizeof(V2<T>);
    }
    static_assert(TPF <= 32 || WZ <= 15, "one named barrier per row");
    static_assert(THREADS % 32 == 0, "whole warps per CTA");
    static_assert(smem(2, NH + 1, NH + 1) <= 227 * 1024, "row tile exceeds shared memory");
};

// Copy a twiddle table into shared memory (whole CTA).
template <typename V>
__device__ __forceinline__ V* stage_table(unsigned char* smem, const V* __restrict__ src, int n)
{
    V* dst = reinterpret_cast<V*>(smem);
    for (int q = threadIdx.x; q < n; q += blockDim.x) dst[q] = src[q];
    return dst;
}

// cp.async (16-byte, L2-only) copies global -> shared, grouped; the waits are
// the hardware's own (no polling loop in this code).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One level of a warp's recursive-halving sum of per-lane arrays: v[0..2H)
// -> v[0..H) holding, for lanes with (lane & O), the upper half plus the
// partner lane's upper half, else the lower halves.
template <int N2, int O> __device__ __forceinline__ void halve_sums(double* v, int lane)
{
    constexpr int H = N2 / 2;
    const bool up = (lane & O) != 0;
#pragma unroll
    for (int k = 0; k < H; k++) {
        const double keep = up ? v[k + H] : v[k];
        const double send = up ? v[k] : v[k + H];
        v[k] = keep + __shfl_xor_sync(0xffffffffu, send, O);
    }
}

// Stage WZ consecutive spectrum rows (first hv entries, rounded up to a
// 16-byte multiple, which stays inside the row stride ss) into `stage`
// (pitch P) with the whole CTA.
template <typename V, int WZ, int THREADS>
__device__ __forceinline__ void stage_rows(V* stage, int P, const V* __restrict__ src, size_t row0, int ss, int hv,
                                           int nrows = 0x7fffffff)
{
    constexpr int EPC = 16 / (int)sizeof(V);
    const int chunks = (hv + EPC - 1) / EPC;
    for (int c = threadIdx.x; c < WZ * chunks; c += THREADS) {
        const int w = c / chunks, q = c - w * chunks;
        if (row0 + w < (size_t)nrows) cp_async16(stage + w * P + q * EPC, src + (row0 + w) * ss + q * EPC);
    }
}

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
    k_inv_x(const V2<T>* __restrict__ src, int src_stride, int nsrc, V2<T>* __restrict__ dst, int dst_stride,
            int mode, const Shell* __restrict__ shell_p, int hvalid, int quad, int skip_dead,
            const V2<T>* __restrict__ tw_g)
{
    using G = PencilGeom<T, N>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tiles_per_row = dst_stride / G::W;
    // skip_dead: a filtered tile whose |my| exceeds the shell's band holds only
    // zeros and is not written (the inverse Y pass then treats those rows as
    // zero, its jband)
    if (skip_dead && mode != LOAD_PLAIN && abs(lattice_freq((int)(blockIdx.x / tiles_per_row), N)) > shell_p->band)
        return;
    const V* tw = stage_table<V>(smem_raw, tw_g, N);
    __syncthreads();
    SmemInterleaved<V, G::W> sm{reinterpret_cast<V*>(smem_raw + G::TW_BYTES), (int)(threadIdx.x % G::W)};
    const int w = threadIdx.x % G::W, t = threadIdx.x / G::W;
    // quad: pencils j <= N/2 only, outputs i <= N/2 only, stored [i][j][h] with
    // N/2+1 rows per plane (the unit filter is even in every axis).
    // nsrc: grid size of the source spectrum ([nsrc][nsrc][src_stride]); a mode
    // m of this N-grid is read at index m mod nsrc there (nsrc >= N, and the
    // shell's band is below N/2, so every selected mode has one home in both).
    const int nj = quad ? N / 2 + 1 : N;
    const int j = blockIdx.x / tiles_per_row;
    const int h = (blockIdx.x % tiles_per_row) * G::W + w;
    const int my = lattice_freq(j, N);
    const int mz = h == N / 2 ? -(N / 2) : h;
    const bool col_ok = h < hvalid && h <= N / 2;
    const size_t js = (size_t)(my < 0 ? my + nsrc : my);
    Shell sh;
    if (mode != LOAD_PLAIN) sh = *shell_p;
    const bool pencil_live =
        col_ok && (mode == LOAD_PLAIN || (abs(my) <= sh.band && abs(mz) <= sh.band));
    // filter bits of this thread's R modes, one predicate instance (loop not unrolled)
    unsigned bits = 0u;
    if (pencil_live) {
        if (mode == LOAD_PLAIN) {
#pragma unroll
            for (int e = 0; e < G::R; e++)
                if (G::live(t + G::TPF * e)) bits |= 1u << e;
        } else {
#pragma unroll 1
            for (int e = 0; e < G::R; e++) {
                if (!G::live(t + G::TPF * e)) continue;
                const int mx = lattice_freq(t + G::TPF * e, N);
                if (abs(mx) <= sh.band && shell_bit(sh, mx, my, mz)) bits |= 1u << e;
            }
        }
    }
    V a[G::R];
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int mx = lattice_freq(t + G::TPF * e, N);
        V v = czero<V>();
        if ((bits >> e) & 1u) {
            if (mode == LOAD_UNIT) v = V{(T)1, (T)0};
            else v = src[((size_t)(mx < 0 ? mx + nsrc : mx) * nsrc + js) * src_stride + h];
        }
        a[e] = v;
    }
    fft_any<V, N, G::R, G::TPF, true>(a, t, sm, tw, BlockSync{});
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int i = t + G::TPF * e;
        if (G::live(i) && (!quad || i <= N / 2)) dst[((size_t)i * nj + j) * dst_stride + h] = a[e];
    }
}

// ------------------------------------------------------------------ Y pass
template <typename T, int N, bool INV, int RX = 0>
__global__ void __launch_bounds__(PencilGeom<T, N, RX>::THREADS)
    k_pass_y(V2<T>* __restrict__ data, int stride, int ncols, int quad, int jband, int jout,
             const V2<T>* __restrict__ tw_g)
{
    using G = PencilGeom<T, N, RX>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = threadIdx.x % G::W, t = threadIdx.x / G::W;
    const int tiles_per_plane = ncols / G::W;  // columns h < ncols of rows of stride `stride`
    // quad: planes i <= N/2, rows j <= N/2 stored, row N-j read as row j
    // (data even in y)
    const int nj = quad ? N / 2 + 1 : N;
    const int i = blockIdx.x / tiles_per_plane;
    const int h = (blockIdx.x % tiles_per_plane) * G::W + w;
    V* base = data + (size_t)i * nj * stride + h;
    // jband < N/2: rows with |my| > jband are zero and not read (the inverse X
    // pass of a band-limited shell leaves them unwritten)
    V a[G::R];
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int j = t + G::TPF * e;
        const int jr = quad && j > N / 2 ? N - j : j;
        a[e] = G::live(j) && (jband >= N / 2 || abs(lattice_freq(j, N)) <= jband) ? base[(size_t)jr * stride]
                                                                                  : czero<V>();
    }
    const V* tw = stage_table<V>(smem_raw, tw_g, N);
    __syncthreads();
    SmemInterleaved<V, G::W> sm{reinterpret_cast<V*>(smem_raw + G::TW_BYTES), w};
    fft_any<V, N, G::R, G::TPF, INV>(a, t, sm, tw, BlockSync{});
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int j = t + G::TPF * e;
        // jout < N/2: rows with |my| > jout are read by no later pass and not stored
        if (G::live(j) && (!quad || j <= N / 2) && (jout >= N / 2 || abs(lattice_freq(j, N)) <= jout))
            base[(size_t)j * stride] = a[e];
    }
}

// ------------------------------------------------------------------ row helpers
// A CTA works on tiles of WZ consecutive (i,j) rows; row w of a tile is done
// by threads [w*TPF, (w+1)*TPF), which synchronise among themselves only.
template <typename T, int N, int RX = 0> struct RowCtx {
    using G = RowGeom<T, N, RX>;
    using V = V2<T>;
    int w, t;
    V* rowbuf;       // this row's exchange buffer [ROWBUF >= NH]
    const V* twr;    // Stockham table of the NH-point transform
    const V* twpp;   // W_N^k, k <= NH (r2c / c2r pre- and post-processing)
    RowSync<G::TPF> sync;
    // stage both tables (caller issues the __syncthreads that publishes them)
    __device__ __forceinline__ RowCtx(unsigned char* smem, const V* __restrict__ twr_g,
                                      const V* __restrict__ twpp_g)
    {
        twr = stage_table<V>(smem + G::TWR_OFF, twr_g, G::NH);
        twpp = stage_table<V>(smem + G::TWPP_OFF, twpp_g, G::NH + 1);
        w = threadIdx.x / G::TPF;
        t = threadIdx.x % G::TPF;
        rowbuf = reinterpret_cast<V*>(smem + G::ROWBUF_OFF) + w * G::ROWBUF;
        sync.bar = 1 + w;
        if constexpr (G::TPF >= 32) {
            sync.mask = 0xffffffffu;
        } else {
            const int base = (threadIdx.x & 31) / G::TPF * G::TPF;
            sync.mask = ((1u << G::TPF) - 1u) << base;
        }
    }
};

// c2r of one spectrum row held in shared memory (entries h < hv, zero above)
// into registers, canonical layout: a[e] = (x[2n], x[2n+1]), n = t + TPF*e.
template <typename T, int N, int RX = 0>
__device__ __forceinline__ void c2r_row(const V2<T>* zr, int hv, RowCtx<T, N, RX>& rc,
                                        V2<T> (&a)[RowGeom<T, N, RX>::R])
{
    using G = RowGeom<T, N, RX>;
    using V = V2<T>;
    constexpr int NH = G::NH;
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int k = rc.t + G::TPF * e;
        if (!G::live(k)) {
            a[e] = czero<V>();
            continue;
        }
        const V zk = k < hv ? zr[k] : czero<V>();
        const V zm = (NH - k) < hv ? cconj(zr[NH - k]) : czero<V>();
        const V A = cadd(zk, zm);
        const V B = cmul(csub(zk, zm), cconj(rc.twpp[k]));  // exp(+2 pi i k / N)
        a[e] = V{A.x - B.y, A.y + B.x};
    }
    SmemRow<V> sm{rc.rowbuf};
    fft_any<V, NH, G::R, G::TPF, true>(a, rc.t, sm, rc.twr, rc.sync);
    rc.sync();
}

// r2c of a real row held in registers (canonical pairs), writing h < hout.
template <typename T, int N, int RX = 0>
__device__ __forceinline__ void r2c_row(V2<T> (&a)[RowGeom<T, N, RX>::R], RowCtx<T, N, RX>& rc, V2<T>* __restrict__ xo,
                                        int hout)
{
    using G = RowGeom<T, N, RX>;
    using V = V2<T>;
    constexpr int NH = G::NH;
    SmemRow<V> sm{rc.rowbuf};
    fft_any<V, NH, G::R, G::TPF, false>(a, rc.t, sm, rc.twr, rc.sync);
    rc.sync();
#pragma unroll
    for (int e = 0; e < G::R; e++)
        if (G::live(rc.t + G::TPF * e)) sm.st(rc.t + G::TPF * e, a[e]);
    rc.sync();
    const T half = (T)0.5;
    for (int k = rc.t; k <= NH && k < hout; k += G::TPF) {
        const V yk = sm.ld(k == NH ? 0 : k);
        const V ym = cconj(sm.ld(k == 0 ? 0 : NH - k));
        const V E = V{(yk.x + ym.x) * half, (yk.y + ym.y) * half};
        const V D = csub(yk, ym);
        const V O = V{D.y * half, -D.x * half};  // D / (2i)
        xo[k] = cadd(E, cmul(rc.twpp[k], O));
    }
    rc.sync();
}

// ------------------------------------------------------------------ inverse Z (c2r)
enum RealEpi : int {
    EPI_STORE = 0,      // out = x^p
    EPI_MUL_STORE = 1,  // out = x^p * aux   (aux may alias out)
    EPI_MUL_REDUCE = 2, // sum x^p * aux
    EPI_REDUCE = 3,     // sum x^p
    EPI_MUL_REDUCE_ABS = 4,  // sum |x^p * aux|  (condition numbers)
    EPI_REDUCE_ABS = 5       // sum |x^p|
};

template <typename T> __device__ __forceinline__ T ipow(T x, int p)
{
    T r = x;
    for (int q = 1; q < p; q++) r *= x;
    return r;
}

// Persistent: CTA b handles tiles b, b + gridDim.x, ...; the next tile's rows
// are copied into the other stage buffer while the current one is computed.
template <typename T, int N>
__global__ void __launch_bounds__(RowGeom<T, N>::THREADS)
    k_inv_z(const V2<T>* __restrict__ src, int src_stride, int hvalid, T* out, const T* aux,
            int epi, int power, double* __restrict__ partials, const V2<T>* __restrict__ twr_g,
            const V2<T>* __restrict__ twpp_g)
{
    using G = RowGeom<T, N>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[(G::THREADS + 31) / 32];
    RowCtx<T, N> rc(smem_raw, twr_g, twpp_g);
    const int P = G::pitch(hvalid);
    V* stage = reinterpret_cast<V*>(smem_raw + G::STAGE_OFF);
    const int ntiles = N * N / G::WZ;
    int tile = blockIdx.x;
    if (tile < ntiles) stage_rows<V, G::WZ, G::THREADS>(stage, P, src, (size_t)tile * G::WZ, src_stride, hvalid);
    cp_async_commit();
    double acc = 0.0;
    for (int st = 0; tile < ntiles; tile += gridDim.x, st ^= 1) {
        const int next = tile + gridDim.x;
        if (next < ntiles)
            stage_rows<V, G::WZ, G::THREADS>(stage + (st ^ 1) * G::WZ * P, P, src, (size_t)next * G::WZ,
                                             src_stride, hvalid);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();
        const size_t row = (size_t)tile * G::WZ + rc.w;
        V a[G::R];
        c2r_row<T, N>(stage + st * G::WZ * P + rc.w * P, hvalid, rc, a);
        T* orow = out ? out + row * N : nullptr;
        const T* arow = aux ? aux + row * N : nullptr;
#pragma unroll
        for (int e = 0; e < G::R; e++) {
            if (!G::live(rc.t + G::TPF * e)) continue;
            const int n2 = 2 * (rc.t + G::TPF * e);
            T x0 = ipow(a[e].x, power), x1 = ipow(a[e].y, power);
            if (epi == EPI_STORE) {
                *reinterpret_cast<V*>(orow + n2) = V{x0, x1};
            } else if (epi == EPI_MUL_STORE) {
                const V q = *reinterpret_cast<const V*>(arow + n2);
                *reinterpret_cast<V*>(orow + n2) = V{x0 * q.x, x1 * q.y};
            } else if (epi == EPI_MUL_REDUCE) {
                const V q = *reinterpret_cast<const V*>(arow + n2);
                acc += (double)x0 * (double)q.x + (double)x1 * (double)q.y;
            } else if (epi == EPI_MUL_REDUCE_ABS) {
                const V q = *reinterpret_cast<const V*>(arow + n2);
                acc += fabs((double)x0 * (double)q.x) + fabs((double)x1 * (double)q.y);
            } else if (epi == EPI_REDUCE_ABS) {
                acc += fabs((double)x0) + fabs((double)x1);
            } else {
                acc += (double)x0 + (double)x1;
            }
        }
        __syncthreads();  // stage st is refilled two tiles later
    }
    if (epi >= EPI_MUL_REDUCE) {
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

// Real values 2n and 2n+1 of a row (ra, and rb for XHI_DENS), composed as
// load_real does, with one vector load per array.
template <typename T>
__device__ __forceinline__ V2<T> load_pair(int kind, const unsigned char* ra, const unsigned char* rb, int n)
{
    switch (kind) {
    case SRC_F32: {
        const float2 v = reinterpret_cast<const float2*>(ra)[n];
        return V2<T>{(T)v.x, (T)v.y};
    }
    case SRC_F64: {
        const double2 v = reinterpret_cast<const double2*>(ra)[n];
        return V2<T>{(T)v.x, (T)v.y};
    }
    case SRC_XHI_F32: {
        const float2 d = reinterpret_cast<const float2*>(ra)[n], x = reinterpret_cast<const float2*>(rb)[n];
        return V2<T>{(T)__dmul_rn((double)d.x, __dsub_rn(1.0, (double)x.x)),
                     (T)__dmul_rn((double)d.y, __dsub_rn(1.0, (double)x.y))};
    }
    default: {  // SRC_XHI_F64
        const double2 d = reinterpret_cast<const double2*>(ra)[n], x = reinterpret_cast<const double2*>(rb)[n];
        return V2<T>{(T)__dmul_rn(d.x, __dsub_rn(1.0, x.x)), (T)__dmul_rn(d.y, __dsub_rn(1.0, x.y))};
    }
    }
}

// One tile of WZ consecutive rows per CTA.  Two ways to bring the rows in:
//  * STAGED: the tile's input bytes (contiguous: WZ rows of N values per input
//    array) are copied to shared memory by cp.async (16-byte, L2-only) and the
//    loader reads its value pairs from there, so no register holds a load in
//    flight; FP32 rows of 512 then run four 256-thread CTAs per SM with up to
//    64 registers.  Needs 16-byte aligned inputs of 4- or 8-byte values.
//    With BULK the tile arrives by one bulk copy per input array
//    (cp.async.bulk through the TMA engine, completion counted on an mbarrier)
//    instead of one 16-byte cp.async per thread and chunk.  The wait on the
//    mbarrier is bounded (kBulkWaitNs of the global timer): past the limit the
//    kernel sets *status to 1, waits once more (bounded) for the copies and
//    returns without writing.  tx_extra > 0 (fault injection in tests) makes
//    the barrier expect more bytes than the copies bring, so the wait runs out.
//  * direct: all loads issued up front into registers (`vec`: one vector load
//    per value pair); FP32 rows of 512 are held to 32 registers so that eight
//    CTAs (every warp slot of the SM) keep their loads in flight.
constexpr unsigned long long kBulkWaitNs = 200000000ull;  // 0.2 s before a bulk copy counts as lost

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_try_wait_parity(unsigned bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return done != 0u;
}

template <typename T, int N, bool STAGED, bool BULK = false>
__global__ void __launch_bounds__(RowGeom<T, N>::THREADS,
                                  (sizeof(T) == 4 && N == 512) ? (STAGED ? 4 : 8) : 1)
    k_fwd_z(int kind, const void* __restrict__ a_src, const void* __restrict__ b_src,
            V2<T>* __restrict__ dst, int dst_stride, int hout, int vec, const V2<T>* __restrict__ twr_g,
            const V2<T>* __restrict__ twpp_g, int* __restrict__ status = nullptr, int tx_extra = 0)
{
    using G = RowGeom<T, N>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w0 = threadIdx.x / G::TPF, t0 = threadIdx.x % G::TPF;
    const size_t row = (size_t)blockIdx.x * G::WZ + w0;
    V a[G::R];
    if constexpr (STAGED) {
        const int eb = (kind == SRC_F32 || kind == SRC_XHI_F32) ? 4 : 8;
        const size_t tile_bytes = (size_t)G::WZ * N * eb;
        unsigned char* sa = smem_raw + G::STAGE_OFF;
        unsigned char* sb = sa + tile_bytes;
        const unsigned char* ga = reinterpret_cast<const unsigned char*>(a_src) + (size_t)blockIdx.x * tile_bytes;
        const unsigned char* gb =
            b_src ? reinterpret_cast<const unsigned char*>(b_src) + (size_t)blockIdx.x * tile_bytes : nullptr;
        __shared__ __align__(8) unsigned long long bar;  // BULK: completion of the tile's copies
        const unsigned bar_s = (unsigned)__cvta_generic_to_shared(&bar);
        if constexpr (BULK) {
            if (threadIdx.x == 0) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_s) : "memory");
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                const unsigned bytes = (unsigned)tile_bytes, total = bytes * (gb ? 2u : 1u) + (unsigned)tx_extra;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_s), "r"(total)
                             : "memory");
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             ::"r"((unsigned)__cvta_generic_to_shared(sa)), "l"(ga), "r"(bytes), "r"(bar_s)
                             : "memory");
                if (gb)
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                        ::"r"((unsigned)__cvta_generic_to_shared(sb)), "l"(gb), "r"(bytes), "r"(bar_s)
                        : "memory");
            }
        } else {
            for (size_t c = threadIdx.x; c < tile_bytes / 16; c += G::THREADS) {
                cp_async16(sa + 16 * c, ga + 16 * c);
                if (gb) cp_async16(sb + 16 * c, gb + 16 * c);
            }
            cp_async_commit();
        }
        RowCtx<T, N> rc(smem_raw, twr_g, twpp_g);  // tables staged while the copies fly
        if constexpr (BULK) {
            bool arrived = mbar_try_wait_parity(bar_s, 0u);
            for (const unsigned long long t0 = global_ns(); !arrived && global_ns() - t0 < kBulkWaitNs;)
                arrived = mbar_try_wait_parity(bar_s, 0u);
            if (!__syncthreads_and(arrived)) {  // the copy never completed: report, wait once more, leave
                if (threadIdx.x == 0 && status) atomicExch(status, 1);
                for (const unsigned long long t0 = global_ns(); !arrived && global_ns() - t0 < kBulkWaitNs;)
                    arrived = mbar_try_wait_parity(bar_s, 0u);
                return;
            }
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        const unsigned char* ra = sa + (size_t)w0 * N * eb;
        const unsigned char* rb = gb ? sb + (size_t)w0 * N * eb : nullptr;
#pragma unroll
        for (int e = 0; e < G::R; e++)
            a[e] = G::live(t0 + G::TPF * e) ? load_pair<T>(kind, ra, rb, t0 + G::TPF * e) : czero<V>();
        r2c_row<T, N>(a, rc, dst + row * dst_stride, hout);
    } else {
        if (kind == SRC_T) {
            const V* xr = reinterpret_cast<const V*>((const T*)a_src + row * N);
#pragma unroll
            for (int e = 0; e < G::R; e++) a[e] = G::live(t0 + G::TPF * e) ? xr[t0 + G::TPF * e] : czero<V>();
        } else if (vec) {
            // both values of a pair in one 8- or 16-byte load per array
            const int eb = (kind == SRC_F32 || kind == SRC_XHI_F32) ? 4 : 8;
            const unsigned char* ra = reinterpret_cast<const unsigned char*>(a_src) + row * N * eb;
            const unsigned char* rb = b_src ? reinterpret_cast<const unsigned char*>(b_src) + row * N * eb : nullptr;
#pragma unroll
            for (int e = 0; e < G::R; e++)
                a[e] = G::live(t0 + G::TPF * e) ? load_pair<T>(kind, ra, rb, t0 + G::TPF * e) : czero<V>();
        } else {
#pragma unroll
            for (int e = 0; e < G::R; e++) {
                const size_t n2 = row * N + 2 * (t0 + G::TPF * e);
                a[e] = G::live(t0 + G::TPF * e)
                           ? V{load_real<T>(kind, a_src, b_src, n2), load_real<T>(kind, a_src, b_src, n2 + 1)}
                           : czero<V>();
            }
        }
        RowCtx<T, N> rc(smem_raw, twr_g, twpp_g);
        __syncthreads();
        r2c_row<T, N>(a, rc, dst + row * dst_stride, hout);
    }
}

// ------------------------------------------------------------------ pair Z
// One (i,j) row of the product of two band-limited inverse transforms,
// transformed forward again: c2r(A) * c2r(B) -> r2c, all along l, so the real
// product D_a*D_b (or D_a^2 when B is NULL) never leaves the SM.  Output rows
// keep h < hout.  Persistent and double-buffered like k_inv_z.
//   RX   : elements per thread of the row transforms (0: RowRadix's choice)
//   KEEP : c2r(A)'s values wait in shared memory (each thread its own slots,
//          no synchronisation) while c2r(B) runs, so one row transform is
//          live in registers at a time instead of two
template <typename T, int N, int RX, bool KEEP> struct PairGeom {
    using G = RowGeom<T, N, RX>;
    // dynamic shared memory: the row kernels' layout, then the keep buffers
    __host__ __device__ static constexpr size_t smem(int ninputs, int hva, int hvb)
    {
        return G::smem(ninputs, hva, hvb) + (KEEP ? (size_t)G::WZ * G::ROWBUF * sizeof(V2<T>) : 0);
    }
    static constexpr bool FITS = smem(2, N / 2 + 1, N / 2 + 1) <= 227 * 1024;
};

// Pair kernel variants the plan autotuner times per FP32 transform size of
// register-plan rows from 128 to 512 points: 0 the default, 1 KEEP (one row
// transform live in registers), 2 KEEP with twice the default elements per
// thread (one radix pass fewer, half the threads per row).  KEEP_OK /
// ALT_RX (0: none) say which exist for a length.
template <typename T, int N> struct PairVariants {
    static constexpr bool REG = sizeof(T) == 4 && !LenKind<N / 2>::RAGGED && N >= 128 && N <= 512;
    static constexpr int RX2 = 2 * RowGeom<T, N>::R;
    static constexpr bool KEEP_OK = REG && PairGeom<T, N, 0, true>::FITS;
    static constexpr int ALT_RX = REG && (N / 2) % RX2 == 0 && (N / 2) / RX2 >= 4 ? RX2 : 0;
};

template <typename T, int N, int RX = 0, bool KEEP = false>
__global__ void __launch_bounds__(RowGeom<T, N, RX>::THREADS)
    k_pair_z(const V2<T>* __restrict__ srcA, int sa, int hva, const V2<T>* __restrict__ srcB, int sb,
             int hvb, V2<T>* __restrict__ dst, int ds, int hout, int nrows, const V2<T>* __restrict__ twr_g,
             const V2<T>* __restrict__ twpp_g)
{
    using G = RowGeom<T, N, RX>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RowCtx<T, N, RX> rc(smem_raw, twr_g, twpp_g);
    const bool two = srcB != nullptr;
    const int PA = G::pitch(hva), PB = two ? G::pitch(hvb) : 0;
    V* stA = reinterpret_cast<V*>(smem_raw + G::STAGE_OFF);
    V* stB = stA + 2 * G::WZ * PA;
    V* keep = stB + 2 * G::WZ * PB + rc.w * G::ROWBUF;  // KEEP: this row's slots
    const int ntiles = (nrows + G::WZ - 1) / G::WZ;
    int tile = blockIdx.x;
    if (tile < ntiles) {
        stage_rows<V, G::WZ, G::THREADS>(stA, PA, srcA, (size_t)tile * G::WZ, sa, hva, nrows);
        if (two) stage_rows<V, G::WZ, G::THREADS>(stB, PB, srcB, (size_t)tile * G::WZ, sb, hvb, nrows);
    }
    cp_async_commit();
    for (int st = 0; tile < ntiles; tile += gridDim.x, st ^= 1) {
        const int next = tile + gridDim.x;
        if (next < ntiles) {
            stage_rows<V, G::WZ, G::THREADS>(stA + (st ^ 1) * G::WZ * PA, PA, srcA, (size_t)next * G::WZ, sa, hva,
                                             nrows);
            if (two)
                stage_rows<V, G::WZ, G::THREADS>(stB + (st ^ 1) * G::WZ * PB, PB, srcB, (size_t)next * G::WZ, sb,
                                                 hvb, nrows);
        }
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();
        const size_t row = (size_t)tile * G::WZ + rc.w;
        if (row >= (size_t)nrows) {  // whole row group idle in the last tile
            __syncthreads();
            continue;
        }
        V a[G::R];
        c2r_row<T, N, RX>(stA + st * G::WZ * PA + rc.w * PA, hva, rc, a);
        if (two) {
            if constexpr (KEEP) {
#pragma unroll
                for (int e = 0; e < G::R; e++)
                    if (G::live(rc.t + G::TPF * e)) keep[rc.t + G::TPF * e] = a[e];
                c2r_row<T, N, RX>(stB + st * G::WZ * PB + rc.w * PB, hvb, rc, a);
#pragma unroll
                for (int e = 0; e < G::R; e++) {
                    const V q = G::live(rc.t + G::TPF * e) ? keep[rc.t + G::TPF * e] : czero<V>();
                    a[e] = V{a[e].x * q.x, a[e].y * q.y};
                }
            } else {
                V b[G::R];
                c2r_row<T, N, RX>(stB + st * G::WZ * PB + rc.w * PB, hvb, rc, b);
#pragma unroll
                for (int e = 0; e < G::R; e++) a[e] = V{a[e].x * b[e].x, a[e].y * b[e].y};
            }
        } else {
#pragma unroll
            for (int e = 0; e < G::R; e++) a[e] = V{a[e].x * a[e].x, a[e].y * a[e].y};
        }
        // the products sit in canonical layout as (x[2n], x[2n+1]): r2c input as is
        r2c_row<T, N, RX>(a, rc, dst + row * ds, hout);
        __syncthreads();
    }
}

// ------------------------------------------------------------------ forward X
enum SpecEpi : int {
    SPEC_STORE = 0,        // out = X
    SPEC_STORE_PHASE = 1,  // out = X / |X|  (utils_fftw.c:78-93)
    SPEC_DOT = 2,          // per shell c: sum_m w(h) F_c(m) Re(dk(m) conj(X(m)))
    SPEC_COUNT = 3,        // per shell c: sum_m w(h) F_c(m) rint(Re X(m) / N^3)
    SPEC_MASK_ADD = 4,     // out += weight * F(m) X(m) where F selects (adjoint)
    SPEC_DOT_ABS = 5       // as SPEC_DOT with |term| (condition numbers)
};

// DOT: true for the per-shell sum epilogues (SPEC_DOT, SPEC_COUNT,
// SPEC_DOT_ABS), false for the storing ones; the two are separate
// instantiations so the storing pass is not sized for the sums' registers.
// r2max (sums only): no shell of the launch holds a mode with |m|^2 > r2max,
// so a tile of pencils whose (my, mz) lie outside that ball is skipped.
// FP32 sums up to 384 points run two CTAs per SM (64 registers, a few bytes
// of spill: the 384-point pass 0.149 against 0.165 ms at one CTA per SM).
// RX > 0 (FP32 dot passes, autotuned): the alternative pencil geometry of
// PencilAlt, twice the elements per thread and one radix pass fewer.
template <typename T, int N, bool DOT, int RX = 0>
__global__ void __launch_bounds__(PencilGeom<T, N, RX>::THREADS,
                                  DOT ? (((sizeof(T) == 4 && N <= 384) || PencilGeom<T, N, RX>::THREADS <= 256) ? 2 : 1)
                                      : (sizeof(T) == 8 ? 1 : 2))
    k_fwd_x(V2<T>* data, int stride, int hvalid, int epi, V2<T>* out, int out_stride,
            const V2<T>* __restrict__ dk, int dk_stride, int ndk, const Shell* __restrict__ shells,
            int nshell, const unsigned short* __restrict__ lut, int lut_size, double weight, int quad,
            int r2max, double* __restrict__ partials, const V2<T>* __restrict__ tw_g, T* __restrict__ mod_out,
            int ncols, int jband)
{
    using G = PencilGeom<T, N, RX>;
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = threadIdx.x % G::W, t = threadIdx.x / G::W;
    // pencils of columns h < ncols (rows of stride `stride`); storing passes
    // with jband < N/2 (a band-limited field spectrum) skip the tiles whose
    // |my| exceeds it and write only modes with |mx| <= jband
    const int tiles_per_row = ncols / G::W;
    // quad (counts only): pencils j <= N/2 of data even in x and y stored
    // [i <= N/2][j <= N/2][h]; plane N-i read as plane i; interior j weigh 2
    const int nj = quad ? N / 2 + 1 : N;
    const int j = blockIdx.x / tiles_per_row;
    const int h = (blockIdx.x % tiles_per_row) * G::W + w;
    const bool col_ok = h < hvalid && h <= N / 2;
    const int my = lattice_freq(j, N);
    const int mz = h == N / 2 ? -(N / 2) : h;
    if constexpr (!DOT) {
        if (jband < N / 2 && abs(my) > jband) return;  // rows outside the field's band
    }
    const bool use_dk = epi == SPEC_DOT || epi == SPEC_DOT_ABS;
    const size_t jdk = (size_t)(my < 0 ? my + ndk : my);
    V* sdk = reinterpret_cast<V*>(smem_raw + G::SMEM);
    if constexpr (DOT) {
        // the whole tile outside every shell: no transform, zero partials
        const bool live = col_ok && my * my + mz * mz <= r2max;
        if (!__syncthreads_or(live)) {
            if (threadIdx.x < nshell) partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = 0.0;
            return;
        }
        if constexpr (G::DK_SMEM) {
            // field-spectrum pencils of the tile (128 bytes per x row, rows
            // that can hold a shell mode only) copied while the transform runs
            if (use_dk) {
                constexpr int EPC = 16 / (int)sizeof(V), CPR = G::W / EPC;
                const int h0 = (blockIdx.x % tiles_per_row) * G::W;
                const long long rest = (long long)r2max - (long long)my * my - (long long)h0 * h0;
                for (int c = threadIdx.x; c < N * CPR; c += G::THREADS) {
                    const int i = c / CPR, q = c - i * CPR;
                    const int mx = lattice_freq(i, N);
                    if ((long long)mx * mx <= rest)
                        cp_async16(sdk + i * G::W + q * EPC,
                                   dk + ((size_t)(mx < 0 ? mx + ndk : mx) * ndk + jdk) * dk_stride + h0 + q * EPC);
                }
            }
            cp_async_commit();
        }
    }
    V a[G::R];
#pragma unroll
    for (int e = 0; e < G::R; e++) {
        const int i = t + G::TPF * e;
        a[e] = G::live(i) ? data[((size_t)(quad && i > N / 2 ? N - i : i) * nj + j) * stride + h] : czero<V>();
    }
    // sums: the shell bits depend on indices only and are found before the
    // transform (16 bits per mode, two modes per register)
    unsigned bits2[(G::R + 1) / 2];
    if constexpr (DOT) {
#pragma unroll
        for (int e = 0; e < (G::R + 1) / 2; e++) bits2[e] = 0u;
#pragma unroll
        for (int e = 0; e < G::R; e++) {
            const int mx = lattice_freq(t + G::TPF * e, N);
            unsigned b = 0u;
            if (col_ok && G::live(t + G::TPF * e)) {
                if (lut) {
                    const int r2 = mx * mx + my * my + mz * mz;
                    b = r2 < lut_size ? (unsigned)__ldg(lut + r2) : 0u;
                } else {
                    b = shell_bits(shells, nshell, mx, my, mz);
                }
            }
            bits2[e / 2] |= (b & 0xffffu) << (16 * (e & 1));
        }
    }
    const V* tw = stage_table<V>(smem_raw, tw_g, N);
    __syncthreads();
    SmemInterleaved<V, G::W> sm{reinterpret_cast<V*>(smem_raw + G::TW_BYTES), w};
    fft_any<V, N, G::R, G::TPF, false>(a, t, sm, tw, BlockSync{});
    if constexpr (!DOT) {
        unsigned keep = (1u << G::R) - 1u;
        if (epi == SPEC_MASK_ADD) {
            keep = 0u;
            const Shell sh = shells[0];
            if (col_ok) {
#pragma unroll 1
                for (int e = 0; e < G::R; e++) {
                    if (!G::live(t + G::TPF * e)) continue;
                    const int mx = lattice_freq(t + G::TPF * e, N);
                    if (in_band(sh, mx, my, mz) && shell_bit(sh, mx, my, mz)) keep |= 1u << e;
                }
            }
        }
        if (h >= out_stride) return;
#pragma unroll
        for (int e = 0; e < G::R; e++) {
            const int i = t + G::TPF * e;
            if (!G::live(i)) continue;
            if (jband < N / 2 && abs(lattice_freq(i, N)) > jband) continue;
            V v = a[e];
            if (epi == SPEC_STORE_PHASE) {
                // mod_out (optional) keeps |X| for the phase-only adjoint
                T m;
                if constexpr (sizeof(T) == 8) {
                    m = hypot(v.x, v.y);
                    v = V{v.x / m, v.y / m};
                } else {
                    // FP32 spectra: one reciprocal square root when |v|^2 is a
                    // normal float, the overflow-safe quotient otherwise (a zero
                    // mode stays 0/0 = NaN, as utils_fftw.c:89 gives)
                    const float m2 = v.x * v.x + v.y * v.y;
                    if (m2 >= 1.17549435e-38f && m2 <= 3.40282347e38f) {
                        const float r = rsqrtf(m2);
                        v = V{v.x * r, v.y * r};
                        m = m2 * r;
                    } else {
                        m = hypotf(v.x, v.y);
                        v = V{v.x / m, v.y / m};
                    }
                }
                if (mod_out) mod_out[((size_t)i * N + j) * out_stride + h] = m;
            } else if (epi == SPEC_MASK_ADD) {
                if (!((keep >> e) & 1u)) continue;
                V* o = out + ((size_t)i * N + j) * out_stride + h;
                const V prev = *o;
                *o = V{prev.x + (T)weight * v.x, prev.y + (T)weight * v.y};
                continue;
            }
            out[((size_t)i * N + j) * out_stride + h] = v;
        }
    } else {
        // dk: field spectrum of an ndk-grid ([ndk][ndk][dk_stride], ndk >= N);
        // mode m of this grid sits at index m mod ndk there (shells lie below N/2).
        // Per-shell FP64 sums in registers, then one fixed-order reduction for
        // all shells at once (deterministic): warp xor-trees, per-warp rows in
        // shared memory, one thread per shell sums the rows in warp order.
        if constexpr (G::DK_SMEM) {
            cp_async_wait_all();
            __syncthreads();
        }
        // DOT sums carry `weight` (the (N_field / N)^3 of a sub-grid product spectrum)
        const double wgt =
            (double)(herm_weight(h, N) * (quad && j != 0 && j != N / 2 ? 2 : 1)) * (use_dk ? weight : 1.0);
        const double inv_n3 = 1.0 / ((double)N * (double)N * (double)N);
        // the 16 shells in two halves of 8 (8 FP64 accumulators live at a
        // time; a mode's term is formed once per half it has shells in).
        // Warp sums of a half by recursive halving: at lane offset o each lane
        // keeps half of its shells (the upper half when lane & o) and adds the
        // partner's copy of that half, so after offsets 16, 8, 4 lane l holds
        // shell c(l) = 4 b4 + 2 b3 + b2 of the half (b_k the lane bits), summed
        // over 8 lanes; offsets 2 and 1 complete it.
        static_assert(MAX_DOT_SHELLS == 16, "two halving trees of 8 shells");
        constexpr int NW = G::THREADS / 32;
        __shared__ double wsum[NW][MAX_DOT_SHELLS];
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            double acc[8];
#pragma unroll
            for (int c = 0; c < 8; c++) acc[c] = 0.0;
#pragma unroll
            for (int e = 0; e < G::R; e++) {
                const unsigned b = (bits2[e / 2] >> (16 * (e & 1) + 8 * half)) & 0xffu;
                if (b) {
                    double val;
                    if (use_dk) {
                        V d;
                        if constexpr (G::DK_SMEM) {
                            d = sdk[(t + G::TPF * e) * G::W + w];
                        } else {
                            const int mx = lattice_freq(t + G::TPF * e, N);
                            d = dk[((size_t)(mx < 0 ? mx + ndk : mx) * ndk + jdk) * dk_stride + h];
                        }
                        val = wgt * ((double)d.x * (double)a[e].x + (double)d.y * (double)a[e].y);
                    } else {
                        val = wgt * rint((double)a[e].x * inv_n3);
                    }
                    if (epi == SPEC_DOT_ABS) val = fabs(val);
#pragma unroll
                    for (int c = 0; c < 8; c++)
                        if ((b >> c) & 1u) acc[c] += val;
                }
            }
            halve_sums<8, 16>(acc, lane);
            halve_sums<4, 8>(acc, lane);
            halve_sums<2, 4>(acc, lane);
            acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], 2);
            acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], 1);
            if ((lane & 3) == 0) wsum[wid][8 * half + ((lane >> 2) & 7)] = acc[0];
        }
        __syncthreads();
        if (threadIdx.x < nshell) {
            double sum = 0.0;
#pragma unroll 1
            for (int q = 0; q < NW; q++) sum += wsum[q][threadIdx.x];
            partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = sum;
        }
    }
}

// Shell bitmask per r2 value (shells of the DEFAULT / RANGE kinds).
static __global__ void k_shell_lut(const Shell* __restrict__ shells, int ns, int size,
                                   unsigned short* __restrict__ lut)
{
    const int r2 = blockIdx.x * blockDim.x + threadIdx.x;
    if (r2 >= size) return;
    unsigned bits = 0u;
    for (int c = 0; c < ns; c++) bits |= (unsigned)(r2 >= shells[c].r2lo && r2 <= shells[c].r2hi) << c;
    lut[r2] = (unsigned short)bits;
}

// ------------------------------------------------------------------ adjoint helpers
// n = 2: dB/d(delta) needs L_a D_b + L_b D_a = IFFT[F_a FFT[D_b] + F_b FFT[D_a]]
// with FFT[D] = N^3 F dk (the inverse transform is unnormalised), i.e.
// IFFT[2 N^3 F_a F_b dk]; this writes that spectrum on the band h < hb (stride S).
template <typename T>
__global__ void k_grad_pair2(int n, const V2<T>* __restrict__ dk, int dks, const Shell* __restrict__ shells,
                             V2<T>* __restrict__ hacc, int S, int hb)
{
    const size_t total = (size_t)n * n * hb;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int h = (int)(q % hb);
        const size_t r = q / hb;
        const int j = (int)(r % n), i = (int)(r / n);
        const int mx = lattice_freq(i, n), my = lattice_freq(j, n), mz = h == n / 2 ? -(n / 2) : h;
        V2<T> v = czero<V2<T>>();
        if (h <= n / 2 && in_band(shells[0], mx, my, mz) && shell_bit(shells[0], mx, my, mz) &&
            in_band(shells[1], mx, my, mz) && shell_bit(shells[1], mx, my, mz)) {
            const V2<T> d = dk[r * dks + h];
            const T f = (T)(2.0 * (double)n * (double)n * (double)n);
            v = V2<T>{f * d.x, f * d.y};
        }
        hacc[r * S + h] = v;
    }
}

// Phase-only adjoint: the field enters through phi = z/|z| per mode, whose
// differential is (dz - phi Re(conj(phi) dz)) / |z|; its transpose maps the
// accumulated gradient spectrum H to (H - phi Re(conj(phi) H)) / |z| (in
// place, rows of the half spectrum, h < hb).  Modes with H = 0 stay 0.
template <typename T>
__global__ void k_phase_adjoint(size_t rows, int hb, V2<T>* __restrict__ hacc, int S,
                                const V2<T>* __restrict__ phi, const T* __restrict__ mod)
{
    const size_t total = rows * (size_t)hb;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const size_t r = q / hb, idx = r * S + q % hb;
        const V2<T> H = hacc[idx];
        if (H.x == (T)0 && H.y == (T)0) continue;
        const V2<T> u = phi[idx];
        const T m = mod[idx];
        const T p = u.x * H.x + u.y * H.y;  // Re(conj(phi) H)
        hacc[idx] = V2<T>{(H.x - u.x * p) / m, (H.y - u.y * p) / m};
    }
}

// out[x] = scale * in[x], converted to the output type.
template <typename T, typename O>
__global__ void k_scale_out(const T* __restrict__ in, O* __restrict__ out, size_t count, double scale)
{
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < count; q += (size_t)gridDim.x * blockDim.x)
        out[q] = (O)(scale * (double)in[q]);
}

// ------------------------------------------------------------------ n = 2 (Parseval)
// Per configuration c (legs a, b): S_D = N^3 sum_half w(h) F_a F_b |dk|^2 and
// the count sum_half w(h) F_a F_b (exact), over the band cube |m| <= band.
// The per-mode configuration bitmask comes from lut[r2] (interval shells) or
// from the shell pairs legs[2c], legs[2c+1].  Per-thread FP64 sums, one
// fixed-order reduction: partials[c] (sums) and partials[MAX + c] (counts).
template <typename T>
__global__ void __launch_bounds__(256)
    k_pair2_sums(int n, const V2<T>* __restrict__ dk, int dks, const unsigned short* __restrict__ lut, int lut_size,
                 const Shell* __restrict__ legs, int ncfg, int band, double* __restrict__ partials)
{
    double acc[MAX_DOT_SHELLS], cnt[MAX_DOT_SHELLS];
#pragma unroll
    for (int c = 0; c < MAX_DOT_SHELLS; c++) acc[c] = cnt[c] = 0.0;
    const int b = min(band, n / 2);
    const int side = 2 * b + 1;
    const long long total = (long long)side * side * (b + 1);
    const double n3 = (double)n * (double)n * (double)n;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int h = (int)(q % (b + 1));
        const long long r = q / (b + 1);
        const int mx = (int)(r / side) - b, my = (int)(r % side) - b;
        if (mx >= n / 2 || my >= n / 2) continue;  // +N/2 is the index of -N/2, visited as such
        const int mz = h == n / 2 ? -(n / 2) : h;
        unsigned bits = 0u;
        if (lut) {
            const int r2 = mx * mx + my * my + mz * mz;
            bits = r2 < lut_size ? (unsigned)__ldg(lut + r2) : 0u;
        } else {
            for (int c = 0; c < ncfg; c++) {
                const Shell& sa = legs[2 * c];
                const Shell& sb = legs[2 * c + 1];
                if (in_band(sa, mx, my, mz) && shell_bit(sa, mx, my, mz) && in_band(sb, mx, my, mz) &&
                    shell_bit(sb, mx, my, mz))
                    bits |= 1u << c;
            }
        }
        if (!bits) continue;
        const int i = mx < 0 ? mx + n : mx, j = my < 0 ? my + n : my;
        const V2<T> d = dk[((size_t)i * n + j) * dks + h];
        const double wgt = (double)herm_weight(h, n);
        const double val = wgt * n3 * ((double)d.x * (double)d.x + (double)d.y * (double)d.y);
#pragma unroll
        for (int c = 0; c < MAX_DOT_SHELLS; c++)
            if ((bits >> c) & 1u) {
                acc[c] += val;
                cnt[c] += wgt;
            }
    }
    __shared__ double wsum[8][2 * MAX_DOT_SHELLS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < MAX_DOT_SHELLS; c++) {
        double v = acc[c], u = cnt[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v += __shfl_xor_sync(0xffffffffu, v, o);
            u += __shfl_xor_sync(0xffffffffu, u, o);
        }
        if (lane == c) {
            wsum[wid][c] = v;
            wsum[wid][MAX_DOT_SHELLS + c] = u;
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * MAX_DOT_SHELLS) {
        double sum = 0.0;
#pragma unroll 1
        for (int q = 0; q < 8; q++) sum += wsum[q][threadIdx.x];
        partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = sum;
    }
}

// dst[idx[q]] = src[q]
static __global__ void k_scatter(const double* __restrict__ src, const int* __restrict__ idx, int count,
                                 double* __restrict__ dst)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < count) dst[idx[q]] = src[q];
}

// ------------------------------------------------------------------ final sums
// out[c] = sum_b partials[c*nblocks + b], fixed order (one CTA per column).
// Column c of the partial sums, summed in a fixed order, lands in
// out[c * out_stride], or in out[idx[c]] (the configuration it belongs to).
static __global__ void k_sum_partials(const double* __restrict__ partials, int nblocks, double* out,
                                      int out_stride, const int* __restrict__ idx)
{
    __shared__ double red[32];
    const double* p = partials + (size_t)blockIdx.x * nblocks;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += p[b];
    s = block_sum<1024>(s, red);
    if (threadIdx.x == 0) out[idx ? (size_t)idx[blockIdx.x] : (size_t)blockIdx.x * out_stride] = s;
}

// ------------------------------------------------------------------ DERIVED k-range
// min/max of squared corner radii over the DEFAULT-filter modes of a shell
// (construct_kfilter_with_determining_kbinwidth, filter.c:78-114).  The
// reference folds the running min/max through sqrt and back per voxel; for
// binary64 sqrt(fl(s*s)) = s, so that equals sqrt of the global min/max of the
// squared corners whatever the visiting order.  Non-negative doubles order
// like their bit patterns, so the fold is an integer atomicMin/atomicMax.
__device__ __forceinline__ int isqrt_floor(int v)  // floor(sqrt(v)), v >= 0
{
    int r = (int)sqrt((double)v);
    while (r * r > v) r--;
    while ((r + 1) * (r + 1) <= v) r++;
    return r;
}

// DERIVED range of one shell: min/max of the squared corner radii over its
// modes with |mz| <= hmax, folded into minmax_bits[0..1] (bit patterns of
// non-negative doubles order as integers).  The grid's x extent strides the
// shell's modes.
__device__ __forceinline__ void derived_range_body(int n, const Shell& sh, int hmax, unsigned long long* minmax_bits);

static __global__ void k_derived_range(int n, const Shell* __restrict__ shell_p, int hmax,
                                       unsigned long long* minmax_bits)
{
    derived_range_body(n, *shell_p, hmax, minmax_bits);
}

// nd shells in one launch: blockIdx.y selects the shell (hmax = its band, at
// most n/2); blocks past what a shell needs find no mode and fold nothing.
static __global__ void k_derived_ranges(int n, const Shell* __restrict__ shells, unsigned long long* minmax_bits)
{
    const Shell sh = shells[blockIdx.y];
    derived_range_body(n, sh, min(sh.band, n / 2), minmax_bits + 2 * blockIdx.y);
}

__device__ __forceinline__ void derived_range_body(int n, const Shell& sh, int hmax, unsigned long long* minmax_bits)
{
    const int band = min(sh.band, n / 2);
    const int side = 2 * band + 1;
    double min2 = sh.min2_init, max2 = 0.0;
    if (sh.kind == SHELL_DEFAULT || sh.kind == SHELL_RANGE) {
        // interval shells: one thread per (mx, my) column, mz over the exact
        // range r2lo <= mx^2 + my^2 + mz^2 <= r2hi (mz >= 0: the corner radii
        // of (mx, my, -mz) are those of (mx, my, mz))
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < side * side; q += gridDim.x * blockDim.x) {
            const int mx = q / side - band, my = q % side - band;
            if (mx >= n / 2 || my >= n / 2 || mx < -(n / 2) || my < -(n / 2)) continue;
            const int s = mx * mx + my * my;
            if (sh.r2hi < 0 || s > sh.r2hi) continue;
            int z0 = 0;
            if (sh.r2lo - s > 0) {
                z0 = isqrt_floor(sh.r2lo - s);
                if (z0 * z0 < sh.r2lo - s) z0++;
            }
            const int z1 = min(isqrt_floor(sh.r2hi - s), hmax);
            for (int hz = z0; hz <= z1; hz++)
                corners_fold(mx, my, hz == n / 2 ? -(n / 2) : hz, sh.half, min2, max2);
        }
    } else {
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
