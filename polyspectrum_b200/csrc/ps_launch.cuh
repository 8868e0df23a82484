// Launch wrappers of the pass kernels for one (precision, N), instantiated
// explicitly in ps_inst_f32.cu / ps_inst_f64.cu (and the *_mixed.cu units) so
// the heavy unrolled kernels compile in parallel translation units.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/ps_gpu.h"
#include "ps_kernels.cuh"

namespace ps {

int launch_fail(cudaError_t e, const char* what);
// Records a message for ps_gpu_last_error() and returns code.
int report_error(int code, const char* msg);
// Shell descriptor as the context builds it (filter.c expressions, host side).
Shell host_shell(int kind, double k, double kmin, double kmax, double binwidth, double L, int N);
// pow(V, n-1) * pow(N, -3n) with V = L^3 (polyspectrum.c:155).
double host_norm_coef(double L, int N, int n);

#define PS_LTRY(x)                \
    do {                          \
        int rc_ = (x);            \
        if (rc_ != 0) return rc_; \
    } while (0)
#define PS_LCK(x)                                        \
    do {                                                 \
        cudaError_t e_ = (x);                            \
        if (e_ != cudaSuccess) return launch_fail(e_, #x); \
    } while (0)

template <typename K> int set_smem(K kernel, size_t bytes)
{
    if (bytes > 48 * 1024)
        PS_LCK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return PS_OK;
}

// Grid of a persistent kernel: as many CTAs as fit on the device at once.
template <typename K> int persistent_grid(K kernel, int threads, size_t smem, int work_items, int* grid)
{
    int dev = 0, sms = 0, per_sm = 0;
    PS_LCK(cudaGetDevice(&dev));
    PS_LCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PS_LCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1) per_sm = 1;
    *grid = std::min(work_items, per_sm * sms);
    return PS_OK;
}

// Twiddle tables of one precision: twp = Stockham table of the pencil
// transforms (length N), twr = of the row transforms (length N/2), twpp =
// W_N^k for the r2c / c2r pre- and post-processing (k < N).
template <typename T> struct Tables {
    const V2<T>* twp;
    const V2<T>* twr;
    const V2<T>* twpp;
    const V2<T>* twp_alt = nullptr;  // Stockham table of the alternative Y pass (PencilAlt), if any
    const V2<T>* twr_alt = nullptr;  // row table of pair kernel variant 2 (PairVariants::ALT_RX), if any
};

template <typename T, int N> struct L3 {
    using V = V2<T>;
    using PG = PencilGeom<T, N>;
    using RG = RowGeom<T, N>;
    static int pencil_width() { return PG::W; }
    static constexpr int ALT = PencilAlt<T, N>::value;
    // host copy of the alternative Y pass's table (false: no alternative)
    static bool host_alt_table(V* twp_alt)
    {
        if constexpr (ALT > 0) {
            static_assert(PencilGeom<T, N, ALT>::W == PG::W, "same pencil tile width");
            transform_table<V, N, ALT, PencilGeom<T, N, ALT>::TPF>(twp_alt);
            return true;
        } else {
            (void)twp_alt;
            return false;
        }
    }
    static constexpr int PAIR_RX2 = PairVariants<T, N>::ALT_RX;
    // host copy of the row table of pair kernel variant 2 (false: no such variant)
    static bool host_pair_alt_table(V* twr_alt)
    {
        if constexpr (PAIR_RX2 > 0) {
            using G2 = RowGeom<T, N, PAIR_RX2>;
            transform_table<V, N / 2, G2::R, G2::TPF>(twr_alt);
            return true;
        } else {
            (void)twr_alt;
            return false;
        }
    }
    // the pair kernel variants this length has (PairVariants): bit v set = variant v runs
    static int pair_variants()
    {
        int m = 1;
        if constexpr (PairVariants<T, N>::KEEP_OK) m |= 2;
        if constexpr (PAIR_RX2 > 0) {
            if constexpr (PairGeom<T, N, PAIR_RX2, true>::FITS) m |= 4;
        }
        return m;
    }
    // host copies of the tables for this N
    static void host_tables(V* twp, V* twr)
    {
        transform_table<V, N, PG::R, PG::TPF>(twp);
        transform_table<V, N / 2, RG::R, RG::TPF>(twr);
    }
    // quad: the xy-quadrant layout of data even in x and y ([i <= N/2][j <= N/2][h])
    // nsrc: grid size of the source spectrum src (0: N; a larger field grid
    // when this N-grid holds a band-limited sub-grid transform)
    // skip_dead: tiles of all-zero pencils (|my| above the shell's band) are
    // left unwritten; the following pass_y must then be given that band
    static int inv_x(cudaStream_t st, const V* src, int ss, V* dst, int ds, int mode, const Shell* sh,
                     int hvalid, const Tables<T>& tb, int quad = 0, int nsrc = 0, int skip_dead = 0)
    {
        PS_LTRY(set_smem(k_inv_x<T, N>, PG::SMEM));
        const int nj = quad ? N / 2 + 1 : N;
        k_inv_x<T, N><<<(unsigned)(nj * (ds / PG::W)), PG::THREADS, PG::SMEM, st>>>(
            src, ss, nsrc > 0 ? nsrc : N, dst, ds, mode, sh, hvalid, quad, skip_dead, tb.twp);
        return PS_OK;
    }
    // jband < N/2: input rows with |my| > jband are zero and are not read
    // ncols (0: stride): only columns h < ncols, a multiple of the pencil width
    // jout < N/2: output rows with |my| > jout are not stored
    // alt: the alternative geometry (PencilAlt) when this length has one
    static int pass_y(cudaStream_t st, V* data, int stride, bool inv, const Tables<T>& tb, int quad = 0,
                      int jband = N, int ncols = 0, int jout = N, int alt = 0)
    {
        const int ni = quad ? N / 2 + 1 : N;
        const int nc = ncols > 0 ? ncols : stride;
        const unsigned blocks = (unsigned)(ni * (nc / PG::W));
        if constexpr (ALT > 0) {
            if (alt && tb.twp_alt) {
                using PA = PencilGeom<T, N, ALT>;
                if (inv) {
                    PS_LTRY(set_smem(k_pass_y<T, N, true, ALT>, PA::SMEM));
                    k_pass_y<T, N, true, ALT><<<blocks, PA::THREADS, PA::SMEM, st>>>(data, stride, nc, quad, jband, jout,
                                                                                     tb.twp_alt);
                } else {
                    PS_LTRY(set_smem(k_pass_y<T, N, false, ALT>, PA::SMEM));
                    k_pass_y<T, N, false, ALT><<<blocks, PA::THREADS, PA::SMEM, st>>>(data, stride, nc, quad, jband,
                                                                                      jout, tb.twp_alt);
                }
                return PS_OK;
            }
        }
        if (inv) {
            PS_LTRY(set_smem(k_pass_y<T, N, true>, PG::SMEM));
            k_pass_y<T, N, true><<<blocks, PG::THREADS, PG::SMEM, st>>>(data, stride, nc, quad, jband, jout, tb.twp);
        } else {
            PS_LTRY(set_smem(k_pass_y<T, N, false>, PG::SMEM));
            k_pass_y<T, N, false><<<blocks, PG::THREADS, PG::SMEM, st>>>(data, stride, nc, quad, jband, jout, tb.twp);
        }
        return PS_OK;
    }
    static int inv_z(cudaStream_t st, const V* src, int ss, int hvalid, T* out, const T* aux, int epi,
                     int power, double* partials, const Tables<T>& tb, int* nblocks)
    {
        const size_t smem = RG::smem(1, hvalid, 0);
        PS_LTRY(set_smem(k_inv_z<T, N>, RG::smem(1, N / 2 + 1, 0)));
        int grid = 0;
        PS_LTRY(persistent_grid(k_inv_z<T, N>, RG::THREADS, smem, N * N / RG::WZ, &grid));
        k_inv_z<T, N><<<grid, RG::THREADS, smem, st>>>(src, ss, hvalid, out, aux, epi, power, partials,
                                                       tb.twr, tb.twpp);
        if (nblocks) *nblocks = grid;
        return PS_OK;
    }
    // stage: 1 copies the input rows to shared memory first (k_fwd_z STAGED),
    // 0 loads them straight into registers, -1 picks staging when it applies
    // (16-byte aligned inputs of 4- or 8-byte values, tile fits shared memory)
    // nrows (0: all N^2): rows processed, from the row the pointers start at
    // (a multiple of the row tile RG::WZ)
    // status (non-NULL): stage by bulk copies (cp.async.bulk, one per input
    // array and tile) whose bounded wait sets *status to 1 if it expires
    static int fwd_z(cudaStream_t st, int kind, const void* a, const void* b, V* dst, int ds, int hout,
                     const Tables<T>& tb, int stage = -1, size_t nrows = 0, int* status = nullptr, int tx_extra = 0)
    {
        const bool two = kind == SRC_XHI_F32 || kind == SRC_XHI_F64;
        const size_t eb = (kind == SRC_F32 || kind == SRC_XHI_F32) ? 4 : 8;
        const uintptr_t addr = (uintptr_t)a | (two ? (uintptr_t)b : 0);
        const size_t smem_staged = RG::STAGE_OFF + (two ? 2 : 1) * (size_t)RG::WZ * N * eb;
        const bool can_stage = kind != SRC_T && addr % 16 == 0 && smem_staged <= 227 * 1024;
        const unsigned blocks = (unsigned)((nrows ? nrows : (size_t)N * N) / RG::WZ);
        if (blocks == 0) return PS_OK;
        if (stage != 0 && can_stage && status) {
            PS_LTRY(set_smem(k_fwd_z<T, N, true, true>, smem_staged));
            k_fwd_z<T, N, true, true><<<blocks, RG::THREADS, smem_staged, st>>>(kind, a, b, dst, ds, hout, 1, tb.twr,
                                                                                 tb.twpp, status, tx_extra);
            return PS_OK;
        }
        if (stage != 0 && can_stage) {
            PS_LTRY(set_smem(k_fwd_z<T, N, true>, smem_staged));
            k_fwd_z<T, N, true><<<blocks, RG::THREADS, smem_staged, st>>>(kind, a, b, dst, ds, hout, 1, tb.twr,
                                                                           tb.twpp);
            return PS_OK;
        }
        constexpr size_t smem = RG::STAGE_OFF;
        PS_LTRY(set_smem(k_fwd_z<T, N, false>, smem));
        const uintptr_t need = (kind == SRC_F32 || kind == SRC_XHI_F32) ? 8 : 16;  // float2 / double2
        const int vec = kind != SRC_T && (addr % need) == 0;
        k_fwd_z<T, N, false><<<blocks, RG::THREADS, smem, st>>>(kind, a, b, dst, ds, hout, vec, tb.twr, tb.twpp);
        return PS_OK;
    }
    template <int RX, bool KEEP>
    static int pair_z_v(cudaStream_t st, const V* a, int sa, int hva, const V* b, int sb, int hvb, V* dst, int ds,
                        int hout, const V* twr, const V* twpp, int quad)
    {
        using G = RowGeom<T, N, RX>;
        using PGm = PairGeom<T, N, RX, KEEP>;
        const size_t smem = PGm::smem(b ? 2 : 1, hva, hvb);
        PS_LTRY(set_smem(k_pair_z<T, N, RX, KEEP>, PGm::smem(2, N / 2 + 1, N / 2 + 1)));
        const int nrows = quad ? (N / 2 + 1) * (N / 2 + 1) : N * N;
        int grid = 0;
        PS_LTRY(persistent_grid(k_pair_z<T, N, RX, KEEP>, G::THREADS, smem, (nrows + G::WZ - 1) / G::WZ, &grid));
        k_pair_z<T, N, RX, KEEP><<<grid, G::THREADS, smem, st>>>(a, sa, hva, b, sb, hvb, dst, ds, hout, nrows, twr,
                                                                 twpp);
        return PS_OK;
    }
    // variant: the autotuned pair kernel variant (PairVariants; 0 the default,
    // and the default wherever the length lacks the one asked for)
    static int pair_z(cudaStream_t st, const V* a, int sa, int hva, const V* b, int sb, int hvb, V* dst,
                      int ds, int hout, const Tables<T>& tb, int quad = 0, int variant = 0)
    {
        if constexpr (PAIR_RX2 > 0) {
            if constexpr (PairGeom<T, N, PAIR_RX2, true>::FITS) {
                if (variant == 2 && tb.twr_alt && !quad)
                    return pair_z_v<PAIR_RX2, true>(st, a, sa, hva, b, sb, hvb, dst, ds, hout, tb.twr_alt, tb.twpp,
                                                    quad);
            }
        }
        if constexpr (PairVariants<T, N>::KEEP_OK) {
            if (variant == 1 && !quad)
                return pair_z_v<0, true>(st, a, sa, hva, b, sb, hvb, dst, ds, hout, tb.twr, tb.twpp, quad);
        }
        return pair_z_v<0, false>(st, a, sa, hva, b, sb, hvb, dst, ds, hout, tb.twr, tb.twpp, quad);
    }
    // ndk: grid size of the field spectrum dk (0: N); r2max: bound of the
    // launch's shells' |m|^2 for the sum epilogues (tiles outside are skipped)
    static int fwd_x(cudaStream_t st, V* data, int stride, int hvalid, int epi, V* out, int ostride,
                     const V* dk, int dks, const Shell* shells, int nshell, const unsigned short* lut,
                     int lut_size, double* partials, const Tables<T>& tb, int* nblocks, double weight = 1.0,
                     int quad = 0, int ndk = 0, int r2max = 0x7fffffff, T* mod_out = nullptr, int ncols = 0,
                     int jband = N, int alt = 0)
    {
        const int nj = quad ? N / 2 + 1 : N;
        const int nc = ncols > 0 ? ncols : stride;
        const unsigned blocks = (unsigned)(nj * (nc / PG::W));
        const bool dot = epi == SPEC_DOT || epi == SPEC_COUNT || epi == SPEC_DOT_ABS;
        if constexpr (ALT > 0) {  // alt: the dot pass in the alternative geometry (PencilAlt)
            if (dot && alt && tb.twp_alt) {
                using PA = PencilGeom<T, N, ALT>;
                PS_LTRY(set_smem(k_fwd_x<T, N, true, ALT>, PA::SMEM_DOT));
                k_fwd_x<T, N, true, ALT><<<blocks, PA::THREADS, PA::SMEM_DOT, st>>>(
                    data, stride, hvalid, epi, out, ostride, dk, dks, ndk > 0 ? ndk : N, shells, nshell, lut, lut_size,
                    weight, quad, r2max, partials, tb.twp_alt, mod_out, nc, jband);
                if (nblocks) *nblocks = (int)blocks;
                return PS_OK;
            }
        }
        if (dot) {
            PS_LTRY(set_smem(k_fwd_x<T, N, true>, PG::SMEM_DOT));
            k_fwd_x<T, N, true><<<blocks, PG::THREADS, PG::SMEM_DOT, st>>>(
                data, stride, hvalid, epi, out, ostride, dk, dks, ndk > 0 ? ndk : N, shells, nshell, lut, lut_size,
                weight, quad, r2max, partials, tb.twp, mod_out, nc, jband);
        } else {
            PS_LTRY(set_smem(k_fwd_x<T, N, false>, PG::SMEM));
            k_fwd_x<T, N, false><<<blocks, PG::THREADS, PG::SMEM, st>>>(
                data, stride, hvalid, epi, out, ostride, dk, dks, ndk > 0 ? ndk : N, shells, nshell, lut, lut_size,
                weight, quad, r2max, partials, tb.twp, mod_out, nc, jband);
        }
        if (nblocks) *nblocks = (int)blocks;
        return PS_OK;
    }
};

// Grid sizes.  Powers of two 16..1024, the 3 2^k / 5 2^k sizes of the
// alias-free sub-grids of pair groups (192, 320, 384), and further grid sizes
// 2^a 3^b 5^c a context may run on (48, 96: register plans; 60, 300, 600:
// shared-memory passes) - instantiated in two translation units per precision.
#define PS_INSTANTIATE_L3_POW2(T)     \
    template struct L3<T, 16>;        \
    template struct L3<T, 32>;        \
    template struct L3<T, 64>;        \
    template struct L3<T, 128>;       \
    template struct L3<T, 192>;       \
    template struct L3<T, 256>;       \
    template struct L3<T, 320>;       \
    template struct L3<T, 384>;       \
    template struct L3<T, 512>;       \
    template struct L3<T, 1024>;

#define PS_INSTANTIATE_L3_MIXED(T)    \
    template struct L3<T, 48>;        \
    template struct L3<T, 60>;        \
    template struct L3<T, 96>;        \
    template struct L3<T, 300>;       \
    template struct L3<T, 600>;

#define PS_EXTERN_L3(T)                  \
    extern template struct L3<T, 16>;    \
    extern template struct L3<T, 32>;    \
    extern template struct L3<T, 48>;    \
    extern template struct L3<T, 60>;    \
    extern template struct L3<T, 64>;    \
    extern template struct L3<T, 96>;    \
    extern template struct L3<T, 128>;   \
    extern template struct L3<T, 192>;   \
    extern template struct L3<T, 256>;   \
    extern template struct L3<T, 300>;   \
    extern template struct L3<T, 320>;   \
    extern template struct L3<T, 384>;   \
    extern template struct L3<T, 512>;   \
    extern template struct L3<T, 600>;   \
    extern template struct L3<T, 1024>;

}  // namespace ps
