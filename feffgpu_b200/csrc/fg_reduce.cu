// fg_reduce.cu -- the fused stage's batch check and its exact row sums: every weighted path term is added to its row as
// a fixed-point number of resolution 2^-64 (fixed_add, two 64-bit integer words per row entry), and the rows are read
// out once all paths are done.  Integer addition is associative, so the rows are exact sums of the rounded terms,
// bit for bit the same whatever the order in which paths finish, the launch shape or the GPU.
#include "fg_launch.h"

namespace fg {

namespace {
__global__ void k_validate(int64_t n, int nleg_max, int nrows, int nph1, const int *__restrict__ order,
                           const int *__restrict__ nleg, const int *__restrict__ row, const int64_t *__restrict__ ipots,
                           int *status)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int bad = 0;
    const int o = order[i];
    if (o < 0 || o >= n) bad |= kBadLayout;
    const int nl = nleg[i];
    if (nl < 2 || nl > nleg_max) bad |= kBadLayout;
    const int r = row[i];
    if (r < 0 || r >= nrows) bad |= kBadLayout;
    if (!(bad & kBadLayout))
        for (int j = 0; j < nl; ++j) {
            const int64_t v = ipots[i * nleg_max + j];
            if (v < 0 || v >= nph1) bad |= kBadIpot;
        }
    if (bad) atomicOr(status, bad);
}

// rows from the fixed-point sums: the low word's carry moved into the signed word in integers, then one value in FP64
__global__ void k_row_finish(int64_t count, const unsigned long long *__restrict__ racc, double *__restrict__ rows,
                             const int *status)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    unsigned long long lo = racc[count + i];
    const long long hi = (long long)(racc[i] + (lo >> 32));   // value * 2^32 (integer part), wraps modulo 2^64
    lo &= 0xffffffffull;
    const double v = (double)(hi >> 32) + ((double)(hi & 0xffffffffll) + (double)lo * 0x1p-32) * 0x1p-32;
    rows[i] = (status && *(volatile const int *)status) ? __longlong_as_double(0x7ff8000000000000ll) : v;
}
}  // namespace

fg_status launch_validate(const fg_paths *P, int nph1, int *status, cudaStream_t st)
{
    if (P->n > 0) {
        k_validate<<<(unsigned)((P->n + 255) / 256), 256, 0, st>>>(P->n, P->nleg_max, P->nrows, nph1, P->order,
                                                                   P->nleg, P->row, P->ipots, status);
        FG_CUDA(cudaGetLastError());
    }
    return FG_OK;
}

size_t row_sum_bytes(int nrows, int NK) { return align_up((size_t)2 * nrows * NK * sizeof(unsigned long long), 256); }

fg_status launch_row_finish(int64_t nrows, int NK, const unsigned long long *racc, double *rows, const int *status,
                            cudaStream_t st)
{
    const int64_t count = nrows * NK;
    if (count > 0) {
        k_row_finish<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(count, racc, rows, status);
        FG_CUDA(cudaGetLastError());
    }
    return FG_OK;
}

fg_status read_status(const int *status, cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    FG_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return FG_OK;
    int v = 0;
    FG_CUDA(cudaMemcpyAsync(&v, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (v & kBadIpot) return fail(FG_ERR_VALUE, "potential index outside 0..nph (the rows are NaN)");
    if (v & kBadRange)
        return fail(FG_ERR_VALUE, "a weighted path term is not finite or its magnitude is 2^31 or more (the rows are "
                                  "NaN)");
    if (v & kBadLayout)
        return fail(FG_ERR_VALUE, "malformed path batch: a launch-order entry, leg count or row is outside its range "
                                  "(the rows are NaN)");
    return FG_OK;
}

size_t fused_workspace(const fg_paths *P, int NK) { return kCounterBytes + row_sum_bytes(P->nrows, NK); }

}  // namespace fg

namespace fg {
// counter, per-path seeds of the chain adjoint (n x E complex, sized for FP64), per-path dL/dreff
size_t fused_bwd_workspace(const fg_paths *P, int, int E)
{
    return kCounterBytes + align_up((size_t)P->n * E * 2 * sizeof(double), 256) + align_up((size_t)P->n * sizeof(double), 256) +
           align_up((size_t)P->n * kGparStride * sizeof(double), 256);
}
size_t cchi_bwd_workspace(int64_t, int) { return kCounterBytes; }
}  // namespace fg

// ------------------------------------------------------------------------------------------------ FP32 FMA peak
namespace fg {
namespace {
__device__ float g_ffma_sink[256];   // keeps the chains live; written only if the sum hits an exact sentinel

__global__ void __launch_bounds__(256) k_ffma_peak(int iters, float seed)
{
    // 16 independent FMA chains per thread keep every FMA pipe busy; the result is stored so nothing is elided
    float a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = seed + 1e-3f * (threadIdx.x + i);
    const float m = 0.999999f, c = 1e-7f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 16; ++i) a[i] = fmaf(a[i], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 16; ++i) s += a[i];
    if (s == 12345.678f) g_ffma_sink[threadIdx.x] = s;
}
}  // namespace
}  // namespace fg

extern "C" fg_status fg_fp32_fma_peak(double *tflops, void *stream)
{
    if (!tflops) return fg::fail(FG_ERR_VALUE, "null argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    FG_CUDA(cudaGetDevice(&dev));
    FG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int per_sm = 0;
    FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fg::k_ffma_peak, 256, 0));
    const int blocks = sms * per_sm, iters = 20000;
    cudaEvent_t e0, e1;
    FG_CUDA(cudaEventCreate(&e0));
    FG_CUDA(cudaEventCreate(&e1));
    fg::k_ffma_peak<<<blocks, 256, 0, st>>>(iters / 10, 1.0f);  // warm-up
    cudaEventRecord(e0, st);
    fg::k_ffma_peak<<<blocks, 256, 0, st>>>(iters, 1.0f);
    cudaEventRecord(e1, st);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return fg::fail(FG_ERR_CUDA, cudaGetErrorString(err));
    *tflops = 2.0 * 16.0 * iters * (double)blocks * 256 / (ms * 1e-3) / 1e12;
    return FG_OK;
}

