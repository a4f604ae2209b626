// fg_pairs.cu -- single scattering of whole configurations from tabulated two-leg signals (the reference's
// PairTables, src/feffgpu/exafs/forward.py:178-320): the histogram of absorber-neighbour distances on the tables'
// distance grid and the position gradient of the all-pairs single-scattering spectrum.
//
// A pair (absorber a, neighbour j) with 1e-6 < r^2 <= rmax^2 (minimum image in a cubic box or a general cell) has u = (r - r_min) / dr,
// i0 = clamp(floor(u), 0, nr - 2), f = clamp(u - i0, 0, 1) and adds 1 - f to bin i0 and f to bin i0 + 1 of the row of
// the neighbour's potential (forward.py:279-289).  The histogram is accumulated in fixed point (2^-32 units, 64-bit
// integer atomics, so the sum is exact and independent of the order of the adds: results repeat bit for bit), each
// pair adding exactly one unit in total; the spectrum is hist @ tables.  The gradient kernel gives each atom its own
// block that visits every pair the atom belongs to (as absorber and as neighbour) and reduces in a fixed order, so it
// needs no atomics either.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "fg_launch.h"

namespace fg {
namespace {

constexpr double kFix = 4294967296.0;   // 2^32 units per histogram count

__device__ __forceinline__ double wrapd(double r, double b) { return b > 0.0 ? r - b * rint(r / b) : r; }

struct PairGeom {
    double rx, ry, rz, r;
    bool ok;
};

// minimum image in a general cell (the reference's cell.py:26-35): f = rel inv(cell), rel = (f - round(f)) cell;
// c holds the cell (lattice vectors as rows, row-major) and then its inverse
__device__ __forceinline__ void wrap_celld(const double *__restrict__ c, double &x, double &y, double &z)
{
    const double *inv = c + 9;
    double f[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        f[j] = fma(z, inv[6 + j], fma(y, inv[3 + j], x * inv[j]));
        f[j] -= rint(f[j]);
    }
    x = fma(f[2], c[6], fma(f[1], c[3], f[0] * c[0]));
    y = fma(f[2], c[7], fma(f[1], c[4], f[0] * c[1]));
    z = fma(f[2], c[8], fma(f[1], c[5], f[0] * c[2]));
}

__device__ __forceinline__ PairGeom pair_geom(const double *pa, const double *pj, double box, const double *cell,
                                              double rmax2)
{
    PairGeom g;
    if (cell) {
        g.rx = pj[0] - pa[0];
        g.ry = pj[1] - pa[1];
        g.rz = pj[2] - pa[2];
        wrap_celld(cell, g.rx, g.ry, g.rz);
    } else {
        g.rx = wrapd(pj[0] - pa[0], box);
        g.ry = wrapd(pj[1] - pa[1], box);
        g.rz = wrapd(pj[2] - pa[2], box);
    }
    const double r2 = g.rx * g.rx + g.ry * g.ry + g.rz * g.rz;
    g.ok = r2 <= rmax2 && r2 > 1e-6;
    g.r = g.ok ? sqrt(r2) : 0.0;
    return g;
}

// One block per (copy, absorber): fixed-point histogram (nph + 1, nr) and the count of pairs below r_min.
__global__ void k_pair_hist(const double *__restrict__ pos, int64_t n, double box, const double *__restrict__ cell,
                            const int64_t *__restrict__ absorbers,
                            int A, const int32_t *__restrict__ ipot, int nph, double r_min, double dr, int nr,
                            double rmax, unsigned long long *__restrict__ hist, unsigned long long *__restrict__ nshort)
{
    const int64_t c = blockIdx.x / A, ai = blockIdx.x % A;
    const double *P = pos + c * n * 3;
    const int64_t a = absorbers ? absorbers[ai] : ai;
    const double *pa = P + 3 * a;
    const double rmax2 = rmax * rmax;
    unsigned long long s = 0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        const PairGeom g = pair_geom(pa, P + 3 * j, box, cell, rmax2);
        const int ip = ipot[j];
        if (!g.ok || ip < 0 || ip > nph) continue;   // potentials outside 0..nph are refused by the host
        if (g.r < r_min) ++s;
        const double u = (g.r - r_min) / dr;
        const double i0d = fmin(fmax(floor(u), 0.0), (double)(nr - 2));
        const double f = fmin(fmax(u - i0d, 0.0), 1.0);
        const unsigned long long qf = (unsigned long long)llrint(f * kFix);
        const int64_t row = (int64_t)ip * nr + (int64_t)i0d;
        atomicAdd(hist + row, (unsigned long long)kFix - qf);
        atomicAdd(hist + row + 1, qf);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(nshort, s);
}

// In place: fixed-point counts -> FP64.
__global__ void k_fixed_to_double(int64_t m, unsigned long long *__restrict__ h)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long v = h[i];
        reinterpret_cast<double *>(h)[i] = (double)v / kFix;
    }
}

// One block per (copy, atom i): gradient of sum_k g_k chi_k, chi = sum over every ordered pair of the interpolated
// table row / (C n), with D = T g (nph, nr) given.  The pair (i absorber, j neighbour) uses D of j's potential, the
// pair (j absorber, i neighbour) D of i's; both have the same distance and weight.  d weight / dr = 1 / dr where
// 0 <= u - i0 <= 1 (the clamp passes the gradient at its ends), else 0.
__global__ void k_pair_ss_grad(const double *__restrict__ pos, int64_t n, double box, const double *__restrict__ cell,
                               const int32_t *__restrict__ ipot,
                               int nph, const double *__restrict__ D, double r_min, double dr, int nr, double rmax,
                               double scale, double *__restrict__ grad)
{
    __shared__ double red[3][256];
    const int64_t c = blockIdx.x / n, i = blockIdx.x % n;
    const double *P = pos + c * n * 3;
    const double *pi = P + 3 * i;
    const double rmax2 = rmax * rmax;
    const int pi_pot = ipot[i];
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        if (j == i) continue;
        const PairGeom g = pair_geom(pi, P + 3 * j, box, cell, rmax2);
        if (!g.ok) continue;
        const double u = (g.r - r_min) / dr;
        const double i0d = fmin(fmax(floor(u), 0.0), (double)(nr - 2));
        const double t = u - i0d;
        if (t < 0.0 || t > 1.0) continue;
        const int i0 = (int)i0d;
        double s = 0.0;
        const int pj = ipot[j];
        if (pj >= 1 && pj <= nph) s += D[(int64_t)(pj - 1) * nr + i0 + 1] - D[(int64_t)(pj - 1) * nr + i0];
        if (pi_pot >= 1 && pi_pot <= nph) s += D[(int64_t)(pi_pot - 1) * nr + i0 + 1] - D[(int64_t)(pi_pot - 1) * nr + i0];
        // d/d pos_i of r_ij = -(pos_j - pos_i) / r
        const double k = -s * scale / (dr * g.r);
        gx += k * g.rx;
        gy += k * g.ry;
        gz += k * g.rz;
    }
    red[0][threadIdx.x] = gx;
    red[1][threadIdx.x] = gy;
    red[2][threadIdx.x] = gz;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; ++q) grad[(c * n + i) * 3 + q] = red[q][0];
}

}  // namespace
}  // namespace fg

using namespace fg;

extern "C" fg_status fg_pair_histogram(const double *pos, int32_t C, int64_t n, double box, const double *cell,
                                       const int64_t *absorbers,
                                       int32_t A, const int32_t *ipot, int32_t nph, double r_min, double dr, int32_t nr,
                                       double rmax, double *hist, uint64_t *n_short, void *stream)
{
    if (C < 0 || n < 0 || A < 0 || nph < 0) return fail(FG_ERR_VALUE, "negative size");
    if (nr < 2 || !(dr > 0.0) || !(rmax > 0.0)) return fail(FG_ERR_VALUE, "the distance grid needs nr >= 2, dr > 0, rmax > 0");
    if (!hist || !n_short) return fail(FG_ERR_VALUE, "null output");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t m = (int64_t)(nph + 1) * nr;
    FG_CUDA(cudaMemsetAsync(hist, 0, (size_t)m * sizeof(double), st));
    FG_CUDA(cudaMemsetAsync(n_short, 0, sizeof(uint64_t), st));
    const int64_t slots = absorbers ? A : n;
    if (C > 0 && slots > 0 && n > 0) {
        if (!pos || !ipot) return fail(FG_ERR_VALUE, "null argument");
        if ((int64_t)C * slots > 0x7fffffffLL) return fail(FG_ERR_VALUE, "too many copies x absorbers for one call");
        k_pair_hist<<<(unsigned)(C * slots), 128, 0, st>>>(pos, n, box, cell, absorbers, (int)slots, ipot, nph, r_min, dr,
                                                          nr, rmax, reinterpret_cast<unsigned long long *>(hist),
                                                          reinterpret_cast<unsigned long long *>(n_short));
        FG_CUDA(cudaGetLastError());
    }
    k_fixed_to_double<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, 4096)), 256, 0, st>>>(
        m, reinterpret_cast<unsigned long long *>(hist));
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

extern "C" fg_status fg_pair_ss_grad(const double *pos, int32_t C, int64_t n, double box, const double *cell,
                                     const int32_t *ipot,
                                     int32_t nph, const double *D, double r_min, double dr, int32_t nr, double rmax,
                                     double scale, double *grad, void *stream)
{
    if (C < 0 || n < 0 || nph < 0) return fail(FG_ERR_VALUE, "negative size");
    if (nr < 2 || !(dr > 0.0)) return fail(FG_ERR_VALUE, "the distance grid needs nr >= 2, dr > 0");
    if ((int64_t)C * n == 0) return FG_OK;
    if (!pos || !ipot || !D || !grad) return fail(FG_ERR_VALUE, "null argument");
    if ((int64_t)C * n > 0x7fffffffLL) return fail(FG_ERR_VALUE, "too many copies x atoms for one call");
    k_pair_ss_grad<<<(unsigned)(C * n), 256, 0, static_cast<cudaStream_t>(stream)>>>(pos, n, box, cell, ipot, nph, D, r_min,
                                                                                     dr, nr, rmax, scale, grad);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}
