// fg_rspace.cu -- the R-space misfit of chi(k) rows and its gradient in one kernel (the loss of the reference's
// refinement, src/feffgpu/exafs/transform.py:104-145: windowed, k-weighted, zero-padded FFT restricted to the R window,
// then sum |chi_R - target_R|^2 / sum |target_R|^2).
//
// The transform restricted to the kept R points is a dense complex matrix F (NR, NK) built once by the host; one block
// per row evaluates chi_R = F x (a warp per R point, coalesced over k), the misfit and, in the same pass, its
// gradient dR/dx_k = 2/norm Re sum_m conj(d_m) F[m][k] (a thread per k, coalesced over k) -- so a refinement step
// needs no further launch for the loss's backward.  FP64, fixed-order sums.
#include <cuda_runtime.h>

#include "fg_launch.h"

namespace fg {
namespace {

constexpr int kThreads = 256;

__global__ void k_rspace(int NK, int NR, const double *__restrict__ rows, const double2 *__restrict__ F,
                         const double2 *__restrict__ target, double inv_norm, double *__restrict__ R,
                         double *__restrict__ grad)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double *x = reinterpret_cast<double *>(smem);                 // (NK) the row
    double2 *d = reinterpret_cast<double2 *>(x + ((NK + 1) & ~1));  // (NR) chi_R - target
    __shared__ double red[kThreads];
    const int64_t b = blockIdx.x;
    for (int k = threadIdx.x; k < NK; k += blockDim.x) x[k] = rows[b * NK + k];
    __syncthreads();
    // chi_R - target: one warp per R point, lanes over k (coalesced rows of F), a fixed-order shuffle reduction
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double s = 0.0;
    for (int m = warp; m < NR; m += nwarps) {
        const double2 *f = F + (int64_t)m * NK;
        double re = 0.0, im = 0.0;
        for (int k = lane; k < NK; k += 32) {
            const double2 v = f[k];
            re = fma(v.x, x[k], re);
            im = fma(v.y, x[k], im);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (lane == 0) {
            const double2 t = target[m];
            const double2 dm = make_double2(re - t.x, im - t.y);
            d[m] = dm;
            s = fma(dm.x, dm.x, fma(dm.y, dm.y, s));
        }
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) R[b] = red[0] * inv_norm;
    if (!grad) return;
    for (int k = threadIdx.x; k < NK; k += blockDim.x) {
        double g = 0.0;
        for (int m = 0; m < NR; ++m) {
            const double2 v = F[(int64_t)m * NK + k];
            g = fma(d[m].x, v.x, fma(d[m].y, v.y, g));          // Re(conj(d) F)
        }
        grad[b * NK + k] = 2.0 * inv_norm * g;
    }
}

}  // namespace
}  // namespace fg

using namespace fg;

extern "C" fg_status fg_rspace_misfit(int64_t B, int32_t NK, int32_t NR, const double *rows, const double *F,
                                      const double *target, double inv_norm, double *R, double *grad, void *stream)
{
    if (B < 0 || NK < 0 || NR < 0) return fail(FG_ERR_VALUE, "negative size");
    if (B == 0) return FG_OK;
    if (!rows || !F || !target || !R) return fail(FG_ERR_VALUE, "null argument");
    if (B > 0x7fffffffLL) return fail(FG_ERR_VALUE, "too many rows for one call");
    const size_t smem = (size_t)((NK + 1) & ~1) * sizeof(double) + (size_t)NR * sizeof(double2);
    if (smem > 200 * 1024) return fail(FG_ERR_VALUE, "NK and NR too large for one block's shared memory");
    if (smem > 48 * 1024) FG_CUDA(cudaFuncSetAttribute(k_rspace, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_rspace<<<(unsigned)B, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(
        NK, NR, rows, reinterpret_cast<const double2 *>(F), reinterpret_cast<const double2 *>(target), inv_norm, R,
        grad);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}
