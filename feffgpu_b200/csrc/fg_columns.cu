// fg_columns.cu -- FEFF's feffNNNN.dat columns of each path from its complex signal (the reference's
// genfmt.py:449-461, FEFF's fdtarr.f).
#include <algorithm>

#include "fg_kernels.cuh"

// FEFF's feffNNNN.dat columns of each path (the reference's genfmt.py:449-461, fdtarr.f): one warp per path, the
// amplitude and unwrapped phase of its signal, then per energy
//   mag = |cchi| |xk| reff^2 exp(2 reff / lambda) / red factor (in A), phase = phi - (2 Re phc unwrapped + l pi).
// cols (E, 4) per energy: |xk| (1/bohr), 2 / lambda (1/bohr), 1 / red factor, 2 Re phc unwrapped + l pi.
namespace fg {
namespace {
template <typename R>
__global__ void k_path_columns(int64_t B, int E, const C2<R> *__restrict__ cchi, const R *__restrict__ reff,
                               const double4 *__restrict__ cols, double *__restrict__ mag, double *__restrict__ phase)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double *amp = reinterpret_cast<double *>(smem) + (size_t)w * 2 * E;
    double *pha = amp + E;
    for (int64_t p = (int64_t)blockIdx.x * nw + w; p < B; p += (int64_t)gridDim.x * nw) {
        const C2<R> *c = cchi + p * E;
        amp_phase<R>(E, lane, [&](int e) { return c[e]; }, amp, pha);
        __syncwarp();
        const double rb = (double)reff[p] / kBohr;
        for (int e = lane; e < E; e += 32) {
            const double4 q = cols[e];
            const C2<R> v = c[e];
            const double a = sqrt((double)v.x * v.x + (double)v.y * v.y);
            mag[p * E + e] = a * q.x * rb * rb * exp(rb * q.y) * q.z * kBohr;
            phase[p * E + e] = pha[e] - q.w;
        }
        __syncwarp();
    }
}
}  // namespace
}  // namespace fg

using namespace fg;

extern "C" fg_status fg_path_columns(int64_t B, int32_t E, fg_precision prec, const void *cchi, const void *reff,
                                     const double *cols, double *mag, double *phase, void *stream)
{
    if (B < 0 || E < 1) return fail(FG_ERR_VALUE, "bad size");
    if (B == 0) return FG_OK;
    if (!cchi || !reff || !cols || !mag || !phase) return fail(FG_ERR_VALUE, "null argument");
    if (prec != FG_MIXED && prec != FG_FP64) return fail(FG_ERR_VALUE, "precision must be FG_MIXED or FG_FP64");
    const int warps = 4;
    const size_t smem = (size_t)warps * 2 * E * sizeof(double);
    if (smem > 200 * 1024) return fail(FG_ERR_VALUE, "too many energies");
    const int blocks = (int)std::min<int64_t>((B + warps - 1) / warps, 148 * 16);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (prec == FG_FP64) {
        if (smem > 48 * 1024) FG_CUDA(cudaFuncSetAttribute(k_path_columns<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_path_columns<double><<<blocks, 32 * warps, smem, st>>>(B, E, static_cast<const C2<double> *>(cchi),
                                                                 static_cast<const double *>(reff),
                                                                 reinterpret_cast<const double4 *>(cols), mag, phase);
    } else {
        if (smem > 48 * 1024) FG_CUDA(cudaFuncSetAttribute(k_path_columns<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_path_columns<float><<<blocks, 32 * warps, smem, st>>>(B, E, static_cast<const C2<float> *>(cchi),
                                                                static_cast<const float *>(reff),
                                                                reinterpret_cast<const double4 *>(cols), mag, phase);
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}
