// Launch wrappers of the pass kernels for one (precision, N), instantiated
// explicitly in ps_inst_f32.cu / ps_inst_f64.cu so the heavy unrolled kernels
// compile in parallel translation units.
#pragma once

#include <cuda_runtime.h>

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

template <typename T, int N> struct L3 {
    using V = V2<T>;
    using PG = PencilGeom<T, N>;
    using RG = RowGeom<T, N>;
    static int inv_x(cudaStream_t st, const V* src, int ss, V* dst, int ds, int mode, const Shell* sh,
                     int hvalid, const V* tw)
    {
        PS_LTRY(set_smem(k_inv_x<T, N>, PG::SMEM));
        k_inv_x<T, N><<<(unsigned)(N * (ds / PG::W)), PG::THREADS, PG::SMEM, st>>>(
            src, ss, dst, ds, mode, sh, hvalid, tw);
        return PS_OK;
    }
    static int pass_y(cudaStream_t st, V* data, int stride, bool inv, const V* tw)
    {
        const unsigned blocks = (unsigned)(N * (stride / PG::W));
        if (inv) {
            PS_LTRY(set_smem(k_pass_y<T, N, true>, PG::SMEM));
            k_pass_y<T, N, true><<<blocks, PG::THREADS, PG::SMEM, st>>>(data, stride, tw);
        } else {
            PS_LTRY(set_smem(k_pass_y<T, N, false>, PG::SMEM));
            k_pass_y<T, N, false><<<blocks, PG::THREADS, PG::SMEM, st>>>(data, stride, tw);
        }
        return PS_OK;
    }
    static int inv_z(cudaStream_t st, const V* src, int ss, int hvalid, T* out, const T* aux, int epi,
                     int power, double* partials, const V* tw, int* nblocks)
    {
        PS_LTRY(set_smem(k_inv_z<T, N>, RG::SMEM));
        const unsigned blocks = (unsigned)((size_t)N * N / RG::WZ);
        k_inv_z<T, N><<<blocks, RG::THREADS, RG::SMEM, st>>>(src, ss, hvalid, out, aux, epi,
                                                                    power, partials, tw);
        if (nblocks) *nblocks = (int)blocks;
        return PS_OK;
    }
    static int fwd_z(cudaStream_t st, int kind, const void* a, const void* b, V* dst, int ds, int hout,
                     const V* tw)
    {
        PS_LTRY(set_smem(k_fwd_z<T, N>, RG::SMEM));
        const unsigned blocks = (unsigned)((size_t)N * N / RG::WZ);
        k_fwd_z<T, N><<<blocks, RG::THREADS, RG::SMEM, st>>>(kind, a, b, dst, ds, hout, tw);
        return PS_OK;
    }
    static int fwd_x(cudaStream_t st, V* data, int stride, int hvalid, int epi, V* out, int ostride,
                     const V* dk, int dks, const Shell* shells, int nshell, double* partials,
                     const V* tw, int* nblocks)
    {
        PS_LTRY(set_smem(k_fwd_x<T, N>, PG::SMEM));
        const unsigned blocks = (unsigned)(N * (stride / PG::W));
        k_fwd_x<T, N><<<blocks, PG::THREADS, PG::SMEM, st>>>(
            data, stride, hvalid, epi, out, ostride, dk, dks, shells, nshell, partials, tw);
        if (nblocks) *nblocks = (int)blocks;
        return PS_OK;
    }
};


#define PS_INSTANTIATE_L3(T)          \
    template struct L3<T, 16>;        \
    template struct L3<T, 32>;        \
    template struct L3<T, 64>;        \
    template struct L3<T, 128>;       \
    template struct L3<T, 256>;       \
    template struct L3<T, 512>;       \
    template struct L3<T, 1024>;

#define PS_EXTERN_L3(T)                  \
    extern template struct L3<T, 16>;    \
    extern template struct L3<T, 32>;    \
    extern template struct L3<T, 64>;    \
    extern template struct L3<T, 128>;   \
    extern template struct L3<T, 256>;   \
    extern template struct L3<T, 512>;   \
    extern template struct L3<T, 1024>;

}  // namespace ps
