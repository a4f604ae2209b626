// fg_launch.h -- host-side interface between the C ABI (fg_api.cu) and the kernel translation units
// (fg_inst_*.cu, one per precision and initial-state class, compiled in parallel).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "feffgpu_b200.h"
#include "fg_device.cuh"

namespace fg {

fg_status fail(fg_status s, const std::string &m);  // records the message for fg_last_error (fg_api.cu)

__host__ __device__ constexpr size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

constexpr size_t kCounterBytes = 256;   // head of every fused workspace: work-queue counters and flags
constexpr size_t kStatusOffset = 64;    // the int status word (kBadIpot | kBadLayout) within that head
constexpr int kGparStride = 32;         // per path in the fused backward's workspace: parameter gradients, frame

// What the launches need to know about a stage.
struct StageView {
    int E, L1, nph1, num_sms, ilinit;
    int max_smem;   // opt-in shared memory per block (bytes)
};

// Warps per block that fit the per-warp shared memory (at least 1; the launch reports a block that does not fit)
inline int fit_warps(int want, size_t per_warp, int max_smem)
{
    int w = want < 1 ? 1 : want;
    while (w > 1 && per_warp * (size_t)w > (size_t)max_smem) --w;
    return w;
}

// Launch shape of the fused forward kernel: warps per block (paths per CTA), the register budget (regs_alt: three
// blocks of 128 threads per SM instead of the default two in FP32, one in FP64) and whether the t-matrix columns of each scatterer are staged
// in a shared-memory tile (stage_t) or read through L1.  No shape changes a result bit.
struct FusedShape {
    int warps = 4;
    bool regs_alt = false;
    bool stage_t = false;
};

// Per precision R and initial-state class EDGE (l_init + 1 = 1, 2, 3: K/L1, L2/L3/M2/M3, M4/M5/N4/N5 edges).
template <typename R, int EDGE> struct Launch {
    static fg_status cchi(const StageView &sv, const Tables<R> &T, int64_t B, int nleg, const void *coords,
                          int coords_f64, const int64_t *ipots, void *cchi, void *reff, int *bad, int warps,
                          cudaStream_t st);
    // rows null: the exact sums are left in words (2 x nrows x NK, see fg_chi_reduce_words) instead of finished
    static fg_status fused(const StageView &sv, const Tables<R> &T, const fg_paths *P, int NK, const double *q,
                           const double *S, const int *span, double *rows, void *cchi_save, double *reff_save,
                           unsigned char *ws, const FusedShape &shape, cudaStream_t st,
                           unsigned long long *words = nullptr);
    static fg_status cchi_bwd(const StageView &sv, const Tables<R> &T, int64_t B, int nleg, const void *coords,
                              int coords_f64, const int64_t *ipots, const void *grad_cchi, const void *grad_reff,
                              void *grad_coords, unsigned char *ws, int warps, cudaStream_t st);
    static fg_status fused_bwd(const StageView &sv, const Tables<R> &T, const fg_paths *P, int NK, const double *q,
                               const double *S, const int *span, const int *tspan, const double *grad_rows,
                               const void *cchi_saved,
                               const double *reff_saved, double *grad_coords, double *grad_sigma2, unsigned char *ws,
                               int warps, cudaStream_t st);
};

// Precision-only launches (no lambda-set dependence).
template <typename R> struct LaunchCommon {
    static fg_status chi_fine(const StageView &sv, int64_t B, const void *cchi, const void *reff, int NK,
                              const void *q, const void *S, const int *span, void *chi, cudaStream_t st);
    static fg_status chi_fine_bwd(const StageView &sv, int64_t B, const void *cchi, const void *reff, int NK,
                                  const void *q, const void *S, const int *span, const int *tspan,
                                  const void *grad_chi, void *grad_cchi, void *grad_reff, cudaStream_t st);
};

// The fused calls' batch check (precision independent): every path's launch-order entry, leg count (2..nleg_max),
// row and potential indices; a bad one raises kBadLayout / kBadIpot in the status word (the per-path kernels then
// return at once on kBadLayout, and clamp potentials).
fg_status launch_validate(const fg_paths *P, int nph1, int *status, cudaStream_t st);

// Bytes of the exact row sums of nrows x NK (two 64-bit words per entry)
size_t row_sum_bytes(int nrows, int NK);

// Rows (nrows, NK) from the exact fixed-point sums (two word arrays of nrows * NK), NaN where the status is set
// (status may be null).
fg_status launch_row_finish(int64_t nrows, int NK, const unsigned long long *racc, double *rows, const int *status,
                            cudaStream_t st);

// The status word of a call's kernels (device int) turned into a return code: outside stream capture the call waits
// for its stream and reads the word (FG_ERR_VALUE with a message if a bit is set); under capture it returns FG_OK
// without waiting (the rows of a replay that meets a bad input are NaN).
fg_status read_status(const int *status, cudaStream_t st);

// The one-absorber path finder's device steps (fg_paths.cu).  candidates_one: the candidates of one absorber in atom
// order (cand_atom, cand_rel; n entries at most), their number in *nc and off = {0, nc}, the single-scattering partial
// paths (len, seq, slot) and absorbers[0] = absorber, with no host round trip; tmp_atom / tmp_rel (n rounded up to 256
// entries), bcnt and boff (n / 256 + 2) are scratch.  extend_count: children per partial path (k_extend's count
// pass) for min(P, *P_dev) parents when P_dev is given.  scan_counts: off[0] = 0, off[i + 1] = the inclusive sum of
// count[0..i] over min(P, *P_dev) entries, the sum in *total.
fg_status candidates_one(const float *pos, int64_t n, float box, const float *cell, int64_t absorber, float rmax,
                         int64_t *tmp_atom, float *tmp_rel, int32_t *bcnt, int64_t *boff, int64_t *cand_atom,
                         float *cand_rel, float *len, int32_t *seq, int32_t *slot, int64_t *off, int64_t *absorbers,
                         int64_t *nc, cudaStream_t st);
fg_status extend_count(int64_t P, const int64_t *P_dev, int32_t m, const int32_t *seq, const float *len,
                       const int32_t *slot, const int64_t *cand_off, const float *cand_rel, float two_r,
                       int32_t *count, cudaStream_t st);
fg_status scan_counts(int64_t P, const int64_t *P_dev, const int32_t *count, int64_t *off, int64_t *total,
                      cudaStream_t st);

// The path finder's description of B paths with a warp per path (fg_paths.cu), for a call on one absorber; paths with
// keep[b] == 0 are skipped (keep may be null); c1 (B, 3) and ip1 (B), when given, receive each path's first atom
// (for single scattering: the candidate) and its potential.
fg_status describe_paths_warp(int64_t B, int32_t nleg, const int32_t *seq, const int32_t *slot, const int64_t *cand_off,
                              const float *cand_rel, const int64_t *cand_atom, const int64_t *ipot_of,
                              const int64_t *absorbers, const fg_pf_tables *T, const uint8_t *keep, float *coords,
                              int64_t *ipots, int64_t *atoms, float *rtot, float *xport, int64_t *key, float *c1,
                              int64_t *ip1, cudaStream_t st);

// Events around the main kernel of a call when kernel timing is on (fg_set_kernel_timing)
void timer_begin(cudaStream_t st);
void timer_end(cudaStream_t st);

size_t fused_workspace(const fg_paths *P, int NK);
size_t fused_bwd_workspace(const fg_paths *P, int NK, int E);
size_t cchi_bwd_workspace(int64_t B, int nleg);

}  // namespace fg

#define FG_CUDA(call)                                                                                         \
    do {                                                                                                      \
        cudaError_t e_ = (call);                                                                              \
        if (e_ != cudaSuccess) return ::fg::fail(FG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
