// fg_geometry.cu -- the path geometry of GPUPathStage.geometry (the reference's stage.py:170-206): leg lengths ri,
// scattering angles beta and Euler sums eta of every leg, and its adjoint.  The arithmetic is leg_geometry's (the
// per-path setup of every kernel of the stage), FP64, with the reference's branch choices; the adjoint runs it on
// dual numbers, one coordinate direction per lane.
#include <algorithm>

#include "fg_kernels.cuh"

namespace fg {
namespace {
// One thread per path: coords (B, nleg, 3) bohr, absorber first; ri, beta, eta (B, nleg) for legs 1..nleg.
__global__ void k_path_geometry(int64_t B, int nleg, const double *__restrict__ coords, double *__restrict__ ri,
                                double *__restrict__ beta, double *__restrict__ eta)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < B; p += (int64_t)gridDim.x * blockDim.x) {
        const double *x = coords + p * nleg * 3;
        auto rat = [&](int i, double *o) {
            const int a = (i == 0 || i == nleg) ? 0 : i;
            o[0] = x[3 * a];
            o[1] = x[3 * a + 1];
            o[2] = x[3 * a + 2];
        };
        double alpha[kMaxLeg + 1], gamma[kMaxLeg + 1];
        for (int j = 1; j <= nleg; ++j) {
            const LegGeom lg = leg_geometry<double>(rat, j, nleg);
            ri[p * nleg + j - 1] = lg.ri;
            beta[p * nleg + j - 1] = lg.beta;
            alpha[j] = lg.alpha;
            gamma[j] = lg.gamma;
        }
        // eta_j = alpha_(j-1) + gamma_j with alpha_0 = alpha_nleg
        for (int j = 1; j <= nleg; ++j) eta[p * nleg + j - 1] = alpha[j == 1 ? nleg : j - 1] + gamma[j];
    }
}

// One warp per path, lane = 3 atom + component: dL/dcoords = sum_j dL/dri_j dri_j/dx + dL/dbeta_j ... + dL/deta_j
// deta_j/dx, each derivative along the lane's coordinate by dual numbers through leg_geometry.
__global__ void k_path_geometry_bwd(int64_t B, int nleg, const double *__restrict__ coords,
                                    const double *__restrict__ g_ri, const double *__restrict__ g_beta,
                                    const double *__restrict__ g_eta, double *__restrict__ grad)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t p = (int64_t)blockIdx.x * nw + w; p < B; p += (int64_t)gridDim.x * nw) {
        if (lane >= 3 * nleg) continue;
        const double *x = coords + p * nleg * 3;
        const int atom = lane / 3, comp = lane % 3;
        auto rat = [&](int i, Dual *o) {
            const int a = (i == 0 || i == nleg) ? 0 : i;
#pragma unroll
            for (int c = 0; c < 3; ++c) o[c] = Dual{x[3 * a + c], (a == atom && c == comp) ? 1.0 : 0.0};
        };
        Dual alpha_prev = leg_geometry<Dual>(rat, nleg, nleg).alpha;   // alpha_0 = alpha_nleg
        double out = 0.0;
        for (int j = 1; j <= nleg; ++j) {
            const LegGeomT<Dual> lg = leg_geometry<Dual>(rat, j, nleg);
            const int64_t o = p * nleg + j - 1;
            out += g_ri[o] * lg.ri.d + g_beta[o] * lg.beta.d + g_eta[o] * (alpha_prev.d + lg.gamma.d);
            alpha_prev = lg.alpha;
        }
        grad[p * nleg * 3 + lane] = out;
    }
}
}  // namespace
}  // namespace fg

using namespace fg;

extern "C" fg_status fg_path_geometry(int64_t B, int32_t nleg, const double *coords, double *ri, double *beta,
                                      double *eta, void *stream)
{
    if (B < 0 || nleg < 2 || nleg > kMaxLeg) return fail(FG_ERR_VALUE, "bad path shape (nleg 2..9)");
    if (B == 0) return FG_OK;
    if (!coords || !ri || !beta || !eta) return fail(FG_ERR_VALUE, "null argument");
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((B + 127) / 128, 148 * 16));
    k_path_geometry<<<blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(B, nleg, coords, ri, beta, eta);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

extern "C" fg_status fg_path_geometry_backward(int64_t B, int32_t nleg, const double *coords, const double *grad_ri,
                                               const double *grad_beta, const double *grad_eta, double *grad_coords,
                                               void *stream)
{
    if (B < 0 || nleg < 2 || nleg > kMaxLeg) return fail(FG_ERR_VALUE, "bad path shape (nleg 2..9)");
    if (B == 0) return FG_OK;
    if (!coords || !grad_ri || !grad_beta || !grad_eta || !grad_coords) return fail(FG_ERR_VALUE, "null argument");
    const int warps = 4;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((B + warps - 1) / warps, 148 * 16));
    k_path_geometry_bwd<<<blocks, 32 * warps, 0, static_cast<cudaStream_t>(stream)>>>(B, nleg, coords, grad_ri,
                                                                                       grad_beta, grad_eta,
                                                                                       grad_coords);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}
