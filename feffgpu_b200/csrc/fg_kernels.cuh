// fg_kernels.cuh -- forward kernels and their launches (included by the fg_inst_*.cu translation units).
#pragma once
#include <algorithm>
#include <string>

#include "fg_forward.cuh"
#include "fg_launch.h"

namespace fg {

template <typename R> __host__ __device__ constexpr size_t geo_bytes() { return (sizeof(WarpPath<R>) + 15) / 16 * 16; }

// Per-warp shared memory: the path state, the rotation tables of nsc legs and (fused kernels) the path's signal
// and unwrapped phase.
// The unwrapped phase of the fused kernel reuses the rotation tables' space once the energies are done.
template <typename R> __host__ __device__ inline size_t table_bytes(int L1, int nsc_max, int MM, int E, bool with_signal)
{
    const size_t d = align_up((size_t)nsc_max * (L1 + 1) * dstride(MM) * sizeof(R), 16);
    // with the signal: its unwrapped phase and amplitude (FP64) reuse the tables' space once the energies are done
    const size_t p = with_signal ? 2 * align_up((size_t)E * sizeof(double), 16) : 0;
    return d > p ? d : p;
}
// (fused kernel: then the signal and, with stage_t, the t-matrix staging tile of (L1 + 1) x 32 entries)
template <typename R> inline size_t warp_bytes(int L1, int nsc_max, int MM, int E, bool with_signal,
                                               bool stage_t = false)
{
    size_t b = geo_bytes<R>() + table_bytes<R>(L1, nsc_max, MM, E, with_signal);
    if (with_signal) b += align_up((size_t)E * sizeof(C2<R>), 16);
    if (with_signal && stage_t) b += (size_t)(L1 + 1) * 32 * sizeof(C2<R>);
    return b;
}

// EDGE 1..3: l_init + 1 of the edge (K/L1, L2/L3/M2/M3, M4/M5/N4/N5) at lambda orders 0..2; EDGE 4..6: the same
// edges at order 3.  MS and SS: the lambda kinds of multiple and single scattering (lamtab).
template <int EDGE> struct Kinds {
    static constexpr int EL = EDGE > 3 ? EDGE - 3 : EDGE;
    static constexpr int MS = EDGE > 3 ? 4 + EL : (EL == 1 ? 0 : 1);
    static constexpr int SS = EL + 1;
    static constexpr bool SS_SYM = SS == 2;      // the K-edge single-scattering set (flip-symmetric accumulation)
    static constexpr int MMMS = lamtab(MS).MM;
    static constexpr int MMSS = lamtab(SS).MM;
    static constexpr int MM = MMMS > MMSS ? MMMS : MMSS;
};

template <typename R, int EDGE>
__device__ __forceinline__ C2<R> path_energy(const WarpPath<R> &g, const R *dh, const Tables<R> &T, int e, int nleg,
                                             C2<R> *tst = nullptr)
{
    using K = Kinds<EDGE>;
    if (nleg == 2) {
        if constexpr (K::SS_SYM)
            return energy_ss_sym<R, K::SS>(g, dh, T, e);
        else
            return energy_ss_col<R, K::SS>(g, dh, T, e);
    }
    return energy_ms<R, K::MS>(g, dh, T, e, nleg, tst);
}

// One warp per path, grid-stride over the paths of one leg count: cchi (B, E) and reff (B).
template <typename R, int EDGE, typename CT>
__global__ void __launch_bounds__(256) k_cchi(Tables<R> T, const CT *__restrict__ coords,
                                               const int64_t *__restrict__ ipots, int64_t B, int nleg,
                                               C2<R> *__restrict__ out, R *__restrict__ reff, int *bad, size_t wbytes)
{
    using K = Kinds<EDGE>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned char *base = smem + (size_t)w * wbytes;
    WarpPath<R> &g = *reinterpret_cast<WarpPath<R> *>(base);
    R *dh = reinterpret_cast<R *>(base + geo_bytes<R>());
    const int E = T.E;
    const int MM = nleg == 2 ? K::MMSS : K::MMMS;
    for (int64_t p = (int64_t)blockIdx.x * nw + w; p < B; p += (int64_t)gridDim.x * nw) {
        path_setup<R, CT>(g, dh, T, coords + p * nleg * 3, ipots + p * nleg, nleg, lane, bad, MM);
        for (int e0 = first_chunk(E); e0 < E; e0 += 32) {
            const int e = e0 + lane;
            if (e >= 0 && e < E) out[p * E + e] = path_energy<R, EDGE>(g, dh, T, e, nleg);
        }
        if (lane == 0) reff[p] = (R)(g.reff * kBohr);
        __syncwarp();
    }
}

// Amplitude and unwrapped phase of one path's signal (stage.py:366-370, 380-384), one warp: differences brought
// into (-pi, pi] with round-half-even (torch.round) and summed in FP64.  amp may be null.
template <typename R, class Load, typename A = R>
__device__ __forceinline__ void amp_phase(int E, int lane, const Load &load, A *amp, double *pha)
{
    double carry = 0.0, prev_raw = 0.0;
    for (int e0 = 0; e0 < E; e0 += 32) {
        const int e = e0 + lane;
        double a = 0.0, ang = 0.0;
        if (e < E) {
            const C2<R> c = load(e);
            const double x = (double)c.x, y = (double)c.y;
            a = sqrt(x * x + y * y + 1e-30);
            ang = a >= 1e-16 ? atan2(y, x) : 0.0;
        }
        double prev = __shfl_up_sync(0xffffffffu, ang, 1);
        if (lane == 0) prev = prev_raw;
        double dlt = (e == 0 || e >= E) ? 0.0 : ang - prev;
        dlt -= 6.283185307179586 * rint(dlt / 6.283185307179586);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double v = __shfl_up_sync(0xffffffffu, dlt, o);
            if (lane >= o) dlt += v;
        }
        const double base = e0 == 0 ? __shfl_sync(0xffffffffu, ang, 0) : carry;
        const double u = base + dlt;
        if (e < E) {
            if (amp) amp[e] = (A)a;
            pha[e] = u;
        }
        carry = __shfl_sync(0xffffffffu, u, 31);
        prev_raw = __shfl_sync(0xffffffffu, ang, 31);
    }
}

// sin of an FP64 argument: FP64 for the plain form, FP64 range reduction then FP32 sine for the mixed form
template <typename R> __device__ __forceinline__ double sin_arg(double arg)
{
    if constexpr (sizeof(R) == 4) {
        arg -= 6.283185307179586 * rint(arg * 0.15915494309189535);
        return (double)sinf((float)arg);
    } else {
        return sin(arg);
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_chi_fine(int64_t B, int E, const C2<R> *__restrict__ cchi,
                                                   const R *__restrict__ reff, int NK, const R *__restrict__ q,
                                                   const R *__restrict__ S, const int *__restrict__ span,
                                                   R *__restrict__ chi, size_t wbytes)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    R *amp = reinterpret_cast<R *>(smem + (size_t)w * wbytes);
    double *pha = reinterpret_cast<double *>(smem + (size_t)w * wbytes + align_up((size_t)E * sizeof(R), 16));
    for (int64_t p = (int64_t)blockIdx.x * nw + w; p < B; p += (int64_t)gridDim.x * nw) {
        const C2<R> *c = cchi + p * E;
        amp_phase<R>(E, lane, [&](int e) { return c[e]; }, amp, pha);
        __syncwarp();
        const double rf = (double)reff[p];
        for (int k0 = 0; k0 < NK; k0 += 32) {
            const int k = k0 + lane;
            if (k < NK) {
                const int lo = span[2 * k], hi = span[2 * k + 1];
                double a = 0.0, ph = 0.0;
                for (int j = lo; j < hi; ++j) {
                    const double sv = (double)S[(size_t)k * E + j];
                    a += sv * (double)amp[j];
                    ph += sv * pha[j];
                }
                chi[p * NK + k] = (R)(a * sin_arg<R>(ph + 2.0 * (double)q[k] * rf));
            }
        }
        __syncwarp();
    }
}

struct PathsDev {
    int64_t n;
    int nleg_max;
    int nrows;
    const double *coords;
    const int64_t *ipots;
    const int *nleg;
    const double *deg;
    const double *sigma2;
    const int *order;
    const int *row;
};

// Fused forward: every path of the batch, all leg counts, from one work queue (costliest first); per path the
// signal at all E, its amplitude and unwrapped phase, and the weighted fine-grid terms
// deg exp(-2 sigma2 q^2) a(q) sin(phi(q) + 2 q reff), each added exactly to its row (fixed_add).  The batch's
// indices were checked by k_validate before the launch: with a malformed batch the kernel returns at once.
//
// MINB, the blocks of 128 threads per SM the registers are budgeted for, and stage_t, whether the t-matrix columns of
// a scatterer go through a shared-memory tile (asynchronous copies) or are read through L1, are tunable (FusedShape);
// neither changes a result bit.
template <typename R> struct FusedMinBlocks {
    static constexpr int def = sizeof(R) == 4 ? 2 : 1;   // measured fastest on B200 for the benchmark workloads
    static constexpr int alt = 3;                         // FP64 at 2 compiles as at 1 (255 registers fit two CTAs)
};
template <typename R, int EDGE, int MINB>
__global__ void __launch_bounds__(128, MINB)
    k_fused(Tables<R> T, PathsDev P, int NK, const double *__restrict__ q, const double *__restrict__ S,
            const int *__restrict__ span, unsigned long long *__restrict__ racc, C2<R> *__restrict__ cchi_save,
            double *__restrict__ reff_save, unsigned long long *counter, int *status, int nsc_max, size_t wbytes,
            int stage_t)
{
    using K = Kinds<EDGE>;
    extern __shared__ __align__(16) unsigned char smem[];
    if (*(volatile const int *)status & kBadLayout) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int E = T.E, L1 = T.L1;
    unsigned char *base = smem + (size_t)w * wbytes;
    WarpPath<R> &g = *reinterpret_cast<WarpPath<R> *>(base);
    R *dh = reinterpret_cast<R *>(base + geo_bytes<R>());
    C2<R> *cbuf = reinterpret_cast<C2<R> *>(base + geo_bytes<R>() + table_bytes<R>(L1, nsc_max, K::MM, E, true));
    C2<R> *tst = stage_t ? reinterpret_cast<C2<R> *>(reinterpret_cast<unsigned char *>(cbuf) +
                                                     align_up((size_t)E * sizeof(C2<R>), 16))
                         : nullptr;
    double *pha = reinterpret_cast<double *>(dh);   // the tables are dead once the path's energies are done
    double *amp = pha + align_up((size_t)E, 2);
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(counter, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= (unsigned long long)P.n) break;
        const int64_t p = P.order[t];
        const int nleg = P.nleg[p];
        path_setup<R, double>(g, dh, T, P.coords + p * P.nleg_max * 3, P.ipots + p * P.nleg_max, nleg, lane, status,
                              nleg == 2 ? K::MMSS : K::MMMS);
        for (int e0 = first_chunk(E); e0 < E; e0 += 32) {
            const int e = e0 + lane;
            if (e >= 0 && e < E) {
                const C2<R> v = path_energy<R, EDGE>(g, dh, T, e, nleg, tst);
                cbuf[e] = v;
                if (cchi_save) cchi_save[p * E + e] = v;
            }
        }
        __syncwarp();
        amp_phase<R>(E, lane, [&](int e) { return cbuf[e]; }, amp, pha);
        __syncwarp();
        const double rf = g.reff * kBohr, wdeg = P.deg[p], s2 = P.sigma2 ? P.sigma2[p] : 0.0;
        unsigned long long *acc_row = racc + (size_t)P.row[p] * NK;
        for (int k0 = 0; k0 < NK; k0 += 32) {
            const int k = k0 + lane;
            if (k < NK) {
                const int lo = span[2 * k], hi = span[2 * k + 1];
                double a = 0.0, ph = 0.0;
                for (int j = lo; j < hi; ++j) {
                    const double sv = S[(size_t)k * E + j];
                    a += sv * amp[j];
                    ph += sv * pha[j];
                }
                const double qk = q[k];
                const double damp = s2 != 0.0 ? exp(-2.0 * s2 * qk * qk) : 1.0;   // exact 1 without sigma^2
                const double v = wdeg * a * sin_arg<R>(ph + 2.0 * qk * rf) * damp;
                if (!fixed_add(acc_row + k, (size_t)P.nrows * NK, v)) atomicOr(status, kBadRange);
            }
        }
        if (lane == 0 && reff_save) reff_save[p] = rf;
        __syncwarp();
    }
}

template <typename KernelT>
inline fg_status grid_for(KernelT kern, int threads, size_t smem, int num_sms, int64_t work_warps, int &blocks)
{
    if (smem > 48 * 1024) FG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    FG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    if (per_sm < 1) return fail(FG_ERR_VALUE, "the kernel does not fit on an SM (shared memory " + std::to_string(smem) + " B)");
    const int64_t need = (work_warps + threads / 32 - 1) / (threads / 32);
    blocks = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)per_sm * num_sms));
    return FG_OK;
}

template <typename R, int EDGE>
fg_status Launch<R, EDGE>::cchi(const StageView &sv, const Tables<R> &T, int64_t B, int nleg, const void *coords,
                                int coords_f64, const int64_t *ipots, void *cchi, void *reff, int *bad, int warps,
                                cudaStream_t st)
{
    using K = Kinds<EDGE>;
    const int MM = nleg == 2 ? K::MMSS : K::MMMS;
    const size_t wb = warp_bytes<R>(sv.L1, nleg - 1, MM, sv.E, false);
    warps = fit_warps(warps, wb, sv.max_smem);
    const int threads = warps * 32;
    const size_t smem = wb * warps;
    int blocks = 0;
    if (coords_f64) {
        auto kern = k_cchi<R, EDGE, double>;
        if (fg_status rc = grid_for(kern, threads, smem, sv.num_sms, B, blocks)) return rc;
        timer_begin(st);
        kern<<<blocks, threads, smem, st>>>(T, static_cast<const double *>(coords), ipots, B, nleg,
                                            static_cast<C2<R> *>(cchi), static_cast<R *>(reff), bad, wb);
    } else {
        auto kern = k_cchi<R, EDGE, float>;
        if (fg_status rc = grid_for(kern, threads, smem, sv.num_sms, B, blocks)) return rc;
        timer_begin(st);
        kern<<<blocks, threads, smem, st>>>(T, static_cast<const float *>(coords), ipots, B, nleg,
                                            static_cast<C2<R> *>(cchi), static_cast<R *>(reff), bad, wb);
    }
    timer_end(st);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

template <typename R, int EDGE>
fg_status Launch<R, EDGE>::fused(const StageView &sv, const Tables<R> &T, const fg_paths *P, int NK, const double *q,
                                 const double *S, const int *span, double *rows, void *cchi_save, double *reff_save,
                                 unsigned char *ws, const FusedShape &shape, cudaStream_t st,
                                 unsigned long long *words)
{
    using K = Kinds<EDGE>;
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(ws);
    int *status = reinterpret_cast<int *>(ws + kStatusOffset);
    unsigned long long *racc = words ? words : reinterpret_cast<unsigned long long *>(ws + kCounterBytes);
    if (words) {
        FG_CUDA(cudaMemsetAsync(ws, 0, kCounterBytes, st));
        FG_CUDA(cudaMemsetAsync(words, 0, (size_t)2 * P->nrows * NK * sizeof(unsigned long long), st));
    } else {
        FG_CUDA(cudaMemsetAsync(ws, 0, kCounterBytes + row_sum_bytes(P->nrows, NK), st));
    }
    if (fg_status rc = launch_validate(P, sv.nph1, status, st)) return rc;
    if (P->n > 0) {
        const int nsc_max = P->nleg_max - 1;
        const size_t wb = warp_bytes<R>(sv.L1, nsc_max, K::MM, sv.E, true, shape.stage_t);
        const int warps = fit_warps(shape.warps > 4 ? 4 : shape.warps, wb, sv.max_smem);
        const int threads = warps * 32;
        auto kern = shape.regs_alt ? k_fused<R, EDGE, FusedMinBlocks<R>::alt> : k_fused<R, EDGE, FusedMinBlocks<R>::def>;
        int blocks = 0;
        if (fg_status rc = grid_for(kern, threads, wb * warps, sv.num_sms, P->n, blocks)) return rc;
        PathsDev pd{P->n, P->nleg_max, P->nrows, P->coords, P->ipots, P->nleg, P->deg, P->sigma2, P->order, P->row};
        timer_begin(st);
        kern<<<blocks, threads, wb * warps, st>>>(T, pd, NK, q, S, span, racc, static_cast<C2<R> *>(cchi_save),
                                                  reff_save, counter, status, nsc_max, wb, shape.stage_t ? 1 : 0);
        timer_end(st);
        FG_CUDA(cudaGetLastError());
    }
    if (!rows) return FG_OK;
    return launch_row_finish(P->nrows, NK, racc, rows, status, st);
}

template <typename R>
fg_status LaunchCommon<R>::chi_fine(const StageView &sv, int64_t B, const void *cchi, const void *reff, int NK,
                                    const void *q, const void *S, const int *span, void *chi, cudaStream_t st)
{
    const size_t wb = align_up((size_t)sv.E * sizeof(R), 16) + align_up((size_t)sv.E * sizeof(double), 16);
    const int warps = fit_warps(8, wb, sv.max_smem), threads = warps * 32;
    auto kern = k_chi_fine<R>;
    int blocks = 0;
    if (fg_status rc = grid_for(kern, threads, wb * warps, sv.num_sms, B, blocks)) return rc;
    kern<<<blocks, threads, wb * warps, st>>>(B, sv.E, static_cast<const C2<R> *>(cchi), static_cast<const R *>(reff),
                                              NK, static_cast<const R *>(q), static_cast<const R *>(S), span,
                                              static_cast<R *>(chi), wb);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

}  // namespace fg
