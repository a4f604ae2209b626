/*
 * feffgpu_b200.h -- C ABI of the B200 path stage.
 *
 * The library evaluates the Rehr-Albers path stage of FEFF 8.5L (as nmarcella/feffGPU implements it in
 * src/feffgpu/stage.py:96-388) on an sm_100a GPU: per-path complex signals on the phase file's real-axis
 * energy grid, the fine-grid signal, and the degeneracy-weighted sum of paths into rows of chi(k), with the
 * hand-written adjoints of all three.
 *
 * Conventions shared by every entry point:
 *   - device pointers for arrays, host pointers for the phase description; no allocation on the caller's behalf
 *     beyond the stage's own tables (fg_stage_create) -- scratch memory is passed in as `workspace`;
 *   - `stream` is a cudaStream_t (NULL = the legacy default stream); every call is asynchronous on it;
 *   - coordinates are in angstrom, absorber first (translation invariant), shape (B, nleg, 3), row-major;
 *   - complex arrays are interleaved (re, im) of the precision's real type;
 *   - precision FG_MIXED: complex64 outputs (the reference's torch.complex64 mode), FP32 scattering-matrix chain,
 *     FP64 geometry, FP64 2kR + phase argument and FP64 cross-path sums; FG_FP64: complex128 throughout;
 *   - every entry point returns an fg_status; fg_last_error() gives a message for the calling thread.
 */
#ifndef FEFFGPU_B200_H
#define FEFFGPU_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FG_API __attribute__((visibility("default")))
#else
#define FG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fg_status {
    FG_OK = 0,
    FG_ERR_VALUE = 1,           /* bad argument: maps to ValueError (genfmt.py:151-152 raises it for lambda sets) */
    FG_ERR_NOT_IMPLEMENTED = 2, /* nsp != 1 (stage.py:99-100), icalc >= 10 (genfmt.py:123): NotImplementedError */
    FG_ERR_CUDA = 3,            /* a CUDA runtime error: RuntimeError */
    FG_ERR_WORKSPACE = 4        /* workspace too small: ValueError */
} fg_status;

typedef enum fg_precision { FG_MIXED = 0, FG_FP64 = 1 } fg_precision;

/* Phase tables of one FEFF phase file, host memory (src/feffgpu/pad.py:69-121, PhaseData).  Only the first
 * ne1 (real-axis) energies and spin 0 are read, as GPUPathStage does. */
typedef struct fg_phase_desc {
    int32_t ne1;          /* real-axis energies E */
    int32_t nph;          /* unique potentials 0..nph */
    int32_t ltot;         /* ph index offset: entry l + ltot holds l = -lmax0..lmax0 */
    int32_t nsp;          /* spin channels; only 1 is supported */
    int32_t ihole;        /* FEFF hole index (1 = K, 4 = L3, 9 = M5, ...) */
    int32_t iorder;       /* lambda-set order (GPUPathStage's iorder): 0..3, 2 by default; 4 and above exceed the
                           * rotation tables (FG_ERR_VALUE) */
    double edge;          /* edge energy (hartree), for xk */
    const int32_t *lmax0; /* (nph+1) partial waves stored per potential */
    const double *em;     /* (ne1) complex energies (hartree), interleaved */
    const double *eref;   /* (ne1) complex energy reference of spin 0, interleaved */
    const double *ph;     /* (ne1, 2*ltot+1, nph+1) complex phase shifts of spin 0, interleaved */
    const double *rkk;    /* (ne1, 8) complex reduced matrix elements of spin 0, interleaved */
} fg_phase_desc;

typedef struct fg_stage fg_stage;

typedef struct fg_stage_info {
    int32_t E;            /* energies of the stage (ne1) */
    int32_t L1;           /* largest lmax + 1 (GPUPathStage.L1, stage.py:105) */
    int32_t nph;
    int32_t kinit, ilinit;
    int32_t lamx_ss, laml0x_ss;   /* lambda-set sizes of two-leg paths */
    int32_t lamx_ms, laml0x_ms;   /* ... and of paths with two or more scatterers */
    int32_t device;
} fg_stage_info;

/* Build the device tables of one phase file on `device` (replaces GPUPathStage.__init__, stage.py:97-125).
 * Allocates the stage's tables (a few hundred KB) with cudaMalloc; fg_stage_destroy frees them. */
FG_API fg_status fg_stage_create(const fg_phase_desc *desc, int device, fg_stage **out);
FG_API void fg_stage_destroy(fg_stage *stage);
FG_API fg_status fg_stage_get_info(const fg_stage *stage, fg_stage_info *info);
/* lmax(ie, iph) as the stage uses it (pad.py:93-106), host output (E, nph+1). */
FG_API fg_status fg_stage_lmax(const fg_stage *stage, int32_t *lmax_out);
/* Real-axis momenta xk (E) in bohr^-1 (pad.py:111-115), host output. */
FG_API fg_status fg_stage_xk(const fg_stage *stage, double *xk_out);

/* Message of the last failed call on this thread ("" if none). */
FG_API const char *fg_last_error(void);

/* Per-path complex signal cchi (B, E) and effective half path length reff (B) in angstrom: replaces
 * GPUPathStage.cchi (stage.py:235-338).  coords (B, nleg, 3) as float (coords_f64 = 0) or double; ipots (B, nleg)
 * int64 with the absorber's potential first; 2 <= nleg <= 9.  cchi: complex64 (FG_MIXED) or complex128 (FG_FP64);
 * reff: float or double likewise.  ipots outside 0..nph are clamped and reported through *bad_ipot if non-NULL
 * (a device int32, left untouched when every index is valid). */
FG_API fg_status fg_cchi(const fg_stage *stage, fg_precision prec, int64_t B, int32_t nleg, const void *coords,
                  int32_t coords_f64, const int64_t *ipots, void *cchi, void *reff, int32_t *bad_ipot, void *stream);

/* Adjoint of fg_cchi: grad_coords (B, nleg, 3) = d(loss)/d(coords) from grad_cchi (B, E) complex with PyTorch's
 * convention d(loss)/d(Re) + i d(loss)/d(Im), and grad_reff (B) (may be NULL).  grad_coords has the precision's
 * real type.  Recomputes the per-leg scattering matrices (no forward state is kept).  `workspace` must hold
 * fg_cchi_backward_workspace(...) bytes.  Potential indices are clamped as in fg_cchi (which reports them). */
FG_API size_t fg_cchi_backward_workspace(const fg_stage *stage, int64_t B, int32_t nleg);
FG_API fg_status fg_cchi_backward(const fg_stage *stage, fg_precision prec, int64_t B, int32_t nleg, const void *coords,
                           int32_t coords_f64, const int64_t *ipots, const void *grad_cchi, const void *grad_reff,
                           void *grad_coords, void *workspace, size_t workspace_bytes, void *stream);

/* Fine-grid signal chi (B, NK) = a(q) sin(phi(q) + 2 q reff), with the amplitude and the unwrapped phase of cchi
 * interpolated by S (NK, E): replaces GPUPathStage.chi_fine (stage.py:372-388).  S is dense in the precision's
 * real type; span (NK, 2) int32 gives each row's non-zero column range [lo, hi) (the full row is always valid).
 * q (NK) and reff (B) have the precision's real type. */
FG_API fg_status fg_chi_fine(const fg_stage *stage, fg_precision prec, int64_t B, const void *cchi, const void *reff,
                      int32_t NK, const void *q, const void *S, const int32_t *span, void *chi, void *stream);
/* Adjoint of fg_chi_fine: grad_cchi (B, E) complex (PyTorch convention) and grad_reff (B) from grad_chi (B, NK).
 * tspan (E, 2) int32 gives each column's non-zero row range of S (the transposed interpolation). */
FG_API fg_status fg_chi_fine_backward(const fg_stage *stage, fg_precision prec, int64_t B, const void *cchi,
                               const void *reff, int32_t NK, const void *q, const void *S, const int32_t *span,
                               const int32_t *tspan, const void *grad_chi, void *grad_cchi, void *grad_reff,
                               void *stream);

/* A batch of paths with mixed leg counts for the fused stage (one persistent launch over every leg count). */
typedef struct fg_paths {
    int64_t n;               /* paths */
    int32_t nleg_max;        /* leg dimension of coords and ipots (<= 9) */
    int32_t nrows;           /* output rows */
    const double *coords;    /* (n, nleg_max, 3) angstrom, absorber first; legs past nleg[p] are ignored */
    const int64_t *ipots;    /* (n, nleg_max) */
    const int32_t *nleg;     /* (n) legs of each path, 2..nleg_max */
    const double *deg;       /* (n) degeneracy weight */
    const double *sigma2;    /* (n) per-path sigma^2 in A^2, or NULL (no damping) */
    const int32_t *row;      /* (n) output row of each path, 0..nrows-1 */
    const int32_t *order;    /* (n) launch order: a permutation of 0..n-1, costliest paths first */
} fg_paths;
/* The fused calls check the contents of these arrays on the device before their kernels read them: a launch-order
 * entry, leg count, row or potential index outside its range is never used to address memory; the call's rows become
 * NaN and, outside stream capture, the call waits for its stream and returns FG_ERR_VALUE naming the fault.  Under
 * stream capture it returns without waiting (a graph replay with such an input gives NaN rows).  Host pointers and
 * sizes are checked before any launch. */

/* Workspace of the fused calls: a work-queue counter and status word, and the rows' exact sums (2 x nrows x NK 64-bit
 * words; no per-path storage). */
FG_API size_t fg_chi_reduce_workspace(const fg_stage *stage, const fg_paths *paths, int32_t NK);

/* rows (nrows, NK) FP64 = sum over paths p of deg_p exp(-2 sigma2_p q^2) chi_p(q), chi_p from cchi and chi_fine
 * as above; every term is rounded to 2^-64 and summed exactly in 64-bit integers, so the rows do not depend on the
 * order in which paths are evaluated (deterministic, bit for bit); a term that is not finite or reaches 2^31 in
 * magnitude is an error.  Fuses GPUPathStage.cchi + chi_fine with the reduction
 * of the callers (chain.py:48-49, exafs/forward.py:162, md/spectrum.py:298).  q (NK), S (NK, E) and span as in
 * fg_chi_fine but always FP64.  If cchi_save (n, E complex of the precision) and reff_save (n, FP64) are non-NULL
 * the per-path signals are kept for fg_chi_reduce_backward.  Outside stream capture the call ends by waiting for
 * its stream (to read the status word of the checks above). */
FG_API fg_status fg_chi_reduce(const fg_stage *stage, fg_precision prec, const fg_paths *paths, int32_t NK, const double *q,
                        const double *S, const int32_t *span, double *rows, void *cchi_save, double *reff_save,
                        void *workspace, size_t workspace_bytes, void *stream);

/* fg_chi_reduce without the last step: the exact row sums are left in words (2 x nrows x NK 64-bit words, caller
 * owned, zeroed by the call): words[r * NK + k] the signed high word (the sum scaled by 2^32, integer part, modulo
 * 2^64) and words[nrows * NK + r * NK + k] the low word (the next 32 bits of every term, summed).  Words of partial
 * sums add exactly as 64-bit integers, so summing them over several GPUs (an integer all-reduce) and then calling
 * fg_rows_from_words gives rows bit for bit equal to one call over all the paths, whatever the number of GPUs or
 * the split.  The workspace needs only its 256-byte head.  No reference counterpart. */
FG_API fg_status fg_chi_reduce_words(const fg_stage *stage, fg_precision prec, const fg_paths *paths, int32_t NK,
                                     const double *q, const double *S, const int32_t *span, uint64_t *words,
                                     void *cchi_save, double *reff_save, void *workspace, size_t workspace_bytes,
                                     void *stream);
/* rows (nrows, NK) FP64 from words as fg_chi_reduce_words leaves them (or their integer sum over calls). */
FG_API fg_status fg_rows_from_words(int64_t nrows, int32_t NK, const uint64_t *words, double *rows, void *stream);

/* Scratch-free variant of fg_chi_reduce.  No counterpart in the reference: it exists for callers that must not
 * allocate device memory -- for example a host program whose GPU memory is handed out by an allocator it does not
 * control (a simulation code that reserves the whole device for its own pool at start-up) and so cannot provide
 * the workspace fg_chi_reduce asks for.  Instead of a caller workspace it uses an array compiled into the library,
 * FG_NOALLOC_SCRATCH_BYTES (32 MiB) on every GPU that loads the library, held until the process exits; a batch
 * whose fg_chi_reduce_workspace exceeds that (more than about 5,200 rows at 401 k points, whatever the number of
 * paths) is rejected with FG_ERR_VALUE (split it by rows).  It allocates
 * nothing: no cudaMalloc, no cudaFree, no allocating library call.  The first call with a given stage looks up the
 * array's device address with the stage's device current and keeps it in the stage; make that first call before any
 * stream capture.  A cudaDeviceReset invalidates every stage (its tables and this address): create new stages after
 * one.  All calls
 * share the array and it keeps the last call's contents (each call clears the queue counter it needs): calls whose
 * work overlaps on the GPU -- other streams, other host threads -- race on it and must be serialised by the caller.
 * Same inputs, checks and result as fg_chi_reduce; the per-path signals are not kept (no adjoint). */
#define FG_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
FG_API fg_status fg_chi_reduce_noalloc(const fg_stage *stage, fg_precision prec, const fg_paths *paths, int32_t NK,
                                       const double *q, const double *S, const int32_t *span, double *rows,
                                       void *stream);

/* Adjoint of fg_chi_reduce: grad_coords (n, nleg_max, 3) FP64 and grad_sigma2 (n) FP64 (may be NULL) from
 * grad_rows (nrows, NK), using the saved cchi and reff; tspan as in fg_chi_fine_backward.  No reference
 * counterpart for sigma^2 (a new input).  The batch is checked as in fg_chi_reduce (outside stream capture the call
 * waits for its stream and returns FG_ERR_VALUE on a bad index). */
FG_API size_t fg_chi_reduce_backward_workspace(const fg_stage *stage, const fg_paths *paths, int32_t NK);
FG_API fg_status fg_chi_reduce_backward(const fg_stage *stage, fg_precision prec, const fg_paths *paths, int32_t NK,
                                 const double *q, const double *S, const int32_t *span, const int32_t *tspan,
                                 const double *grad_rows,
                                 const void *cchi_saved, const double *reff_saved, double *grad_coords,
                                 double *grad_sigma2, void *workspace, size_t workspace_bytes, void *stream);

/* Device timing of the library's main kernel (the per-path kernel of each call), for profiling and autotuning:
 * while enabled, every call records CUDA events around its main kernel on the call's stream; fg_kernel_time_ms
 * waits for the last recorded end event and returns the elapsed milliseconds. */
FG_API fg_status fg_set_kernel_timing(int32_t enable);
FG_API fg_status fg_kernel_time_ms(float *ms);

/* Measured FP32 FMA throughput of this GPU (TFLOP/s): a calibration kernel of independent FFMA chains on every SM,
 * timed with CUDA events on `stream` (the roofline denominator of the FP32 CUDA-core kernels). */
FG_API fg_status fg_fp32_fma_peak(double *tflops, void *stream);

/* Launch tuning: warps per block (paths per CTA) of the persistent per-path kernels, forward and adjoint (1..8),
 * 0 = the built-in default.  fg_set_launch sets the process-wide default; fg_stage_set_launch overrides it for the
 * calls on one stage (what the autotuner sets per workload).  Shapes whose shared memory does not fit are
 * narrowed to the largest that fits.  No reference counterpart (the reference has no launch shapes to tune). */
FG_API fg_status fg_set_launch(int32_t fwd_warps, int32_t bwd_warps);
FG_API fg_status fg_stage_set_launch(fg_stage *stage, int32_t fwd_warps, int32_t bwd_warps);

/* Variant of the fused forward (fg_chi_reduce, fg_chi_reduce_noalloc) on one stage, for the autotuner: regs_alt = 1
 * budgets the registers for three blocks of 128 threads per SM (12 warps; the default budget is for two in FP32 and
 * one in FP64); stage_t = 1 copies each scatterer's t-matrix column into a shared-memory tile per warp (asynchronous
 * copies) instead of reading it through L1.  Both 0 (the default) are the fastest measured on B200 for the benchmark
 * workloads.  No variant changes a result bit.  No reference counterpart. */
FG_API fg_status fg_stage_set_fused_variant(fg_stage *stage, int32_t regs_alt, int32_t stage_t);

/* ---------------------------------------------------------------------------------------------- path finder
 * The enumeration of the reference's GPUPathFinder.enumerate (src/feffgpu/pathfinder.py:213-271; its _longer_paths,
 * :159-211, for five and more legs), batched over absorber slots; the host driver (feffgpu_b200/pathfinder.py)
 * strings the calls together and does the merges and the importance cut (pathfinder.py:102-157, 271-279).
 * Positions are FP32 Angstrom, as in the reference.  A path's atoms are stored as candidate-local indices of its
 * absorber slot (0..nc-1, nc = that slot's candidate count = the absorber itself). */

/* |f(beta)|, momentum and mean-free-path tables of the importance (pathfinder.py:43-65), device arrays. */
typedef struct fg_pf_tables {
    int32_t E;               /* energies of the tables (ne1) */
    int32_t nph1;            /* potentials */
    int32_t ik0;             /* first energy of the importance integral (0-based) */
    const float *fbeta;      /* (E, nph1, 81) |f(beta)| on cos(beta) = -1, -0.975, ..., 1 */
    const float *cksp;       /* (E) Re p, 1/A */
    const float *xlam;       /* (E) mean free path, A */
    const float *trap;       /* (E - ik0) trapezoid weights */
} fg_pf_tables;

/* Candidates (atoms within rmax of each absorber, the absorber excluded), in atom order, with the minimum image of
 * cell.py:26-35: cell == NULL: a cubic box of length box (box <= 0: a cluster); else cell holds 18 floats, the
 * periodic cell's lattice vectors as rows (3 x 3, row-major) and then its inverse, and box is ignored.  pos holds F
 * frames of n atoms (F n, 3); slot a belongs to frame a / per_frame and absorbers[a] is an atom index within that
 * frame.  offset == NULL: count (A) = candidates per slot.  Else offset (A + 1) is the exclusive scan of count and
 * cand_atom (total, frame-local atom indices), cand_rel (total, 3) are written.  pathfinder.py:219-224. */
FG_API fg_status fg_pf_candidates(const float *pos, int64_t n, float box, const float *cell,
                                  const int64_t *absorbers, int32_t A,
                                  int32_t per_frame, float rmax, int32_t *count, const int64_t *offset,
                                  int64_t *cand_atom, float *cand_rel, void *stream);
/* One level of growth: P partial paths of m atoms (seq (P, m), closed-so-far lengths len (P), slots (P)) get every
 * intermediate other than their last atom whose closed length fits two_r.  child_off == NULL: count (P) children
 * per partial path.  Else child_off (P) is the exclusive scan of count and the children (seq (C, m + 1), len, slot)
 * are written in parent order and intermediate order.  pathfinder.py:180-196. */
FG_API fg_status fg_pf_extend(int64_t P, int32_t m, const int32_t *seq, const float *len, const int32_t *slot,
                              const int64_t *cand_off, const float *cand_rel, float two_r, int32_t *count,
                              const int64_t *child_off, int32_t *child_seq, float *child_len, int32_t *child_slot,
                              void *stream);
/* keep (C) = 1 for the paths among C sequences of m atoms (last atom a candidate, not after its reverse), deg (C) =
 * 1 for a palindrome, else 2.  pathfinder.py:199-211. */
FG_API fg_status fg_pf_terminal(int64_t C, int32_t m, const int32_t *seq, const int32_t *slot, const int64_t *cand_off,
                                uint8_t *keep, float *deg, void *stream);
/* Per path of nleg legs (seq (B, nleg - 1)): coords (B, nleg, 3) relative to the absorber, ipots (B, nleg) (the
 * absorber 0, else ipot_of[atom]), atoms (B, nleg - 1) atom indices, closed length rtot (B); with T, the importance
 * xport (B) (pathfinder.py:75-100); with key and nleg > 2, the degeneracy key (B, 2 nleg): leg lengths and
 * cos(beta) rounded to 1e-3 in the lexicographically smaller direction (pathfinder.py:134-157). */
FG_API fg_status fg_pf_describe(int64_t B, int32_t nleg, const int32_t *seq, const int32_t *slot,
                                const int64_t *cand_off, const float *cand_rel, const int64_t *cand_atom,
                                const int64_t *ipot_of, const int64_t *absorbers, const fg_pf_tables *T,
                                float *coords, int64_t *ipots, int64_t *atoms, float *rtot, float *xport,
                                int64_t *key, void *stream);
/* Host: greedy windows of width eps over each segment [seg_off[s], seg_off[s+1]) of ascending lengths (the window
 * of FEFF's accidental-degeneracy merge, pathfinder.py:110-119); window ids restart at 0 per segment. */
FG_API fg_status fg_pf_windows(const float *sorted_len, const int64_t *seg_off, int64_t nseg, float eps,
                               int64_t *window);

/* The whole finder for one absorber in one call -- the reference's GPUPathFinder.enumerate (pathfinder.py:213-279),
 * which its front ends call once per absorber (exafs/forward.py:122-123, md/spectrum.py:275-277): candidates,
 * growth, description, the merges and the importance cut, with one synchronisation per growth level plus two.  pos
 * (n, 3) FP32 one frame on the device, box / cell as in fg_pf_candidates, ipot_of (n) on the device, T the
 * importance tables.  counts (10): kept paths per leg count (index nleg; -1 for a leg count the growth did not
 * reach), *ref the reference importance.  The paths stay in *result until fg_pf_result_gather copies those of one leg
 * count into caller arrays -- coords (B, nleg, 3) FP32, ipots (B, nleg), deg (B) FP32, xport (B) FP32, atoms
 * (B, nleg - 1) -- and fg_pf_result_destroy frees them (stream ordered).  The kept paths are those of the batched
 * entry points above, bit for bit.  Scratch comes from the library's own stream-ordered pool on the device. */
typedef struct fg_pf_result fg_pf_result;
FG_API fg_status fg_pf_enumerate_one(const float *pos, int64_t n, float box, const float *cell, int64_t absorber,
                                     const int64_t *ipot_of, const fg_pf_tables *T, float rmax, int32_t nlegmax,
                                     float critpw, int32_t merge_degenerate, fg_pf_result **result, int64_t *counts,
                                     float *ref, void *stream);
FG_API fg_status fg_pf_result_gather(fg_pf_result *result, int32_t nleg, float *coords, int64_t *ipots, float *deg,
                                     float *xport, int64_t *atoms, void *stream);
FG_API void fg_pf_result_destroy(fg_pf_result *result);

/* ---------------------------------------------------------------------------------------------- pair tables
 * Single scattering of whole configurations from tabulated two-leg signals (the reference's PairTables,
 * src/feffgpu/exafs/forward.py:178-320); the tables themselves are rows of fg_chi_reduce.  pos (C, n, 3) FP64
 * angstrom, C copies of n atoms; box: cubic length, <= 0 for a cluster; cell: NULL, or 18 doubles, the periodic
 * cell's lattice vectors as rows (3 x 3, row-major) and then its inverse (the minimum image of the reference's
 * cell.py:26-35; box is then ignored); ipot (n) int32 scatterer potential 0..nph
 * (0: never a neighbour in the spectrum); the distance grid r_min + dr i, i < nr. */

/* Histogram of absorber-neighbour distances (forward.py:248-289): every pair with 1e-6 < r^2 <= rmax^2 adds its
 * linear-interpolation weights to row ipot[j] of hist (nph + 1, nr) FP64; absorbers (A) atom indices, the same in
 * every copy, or NULL for every atom; n_short (device, 1) = pairs closer than r_min.  Deterministic: the weights are
 * summed in 2^-32 fixed point (exact, order-free), each pair adding exactly one. */
FG_API fg_status fg_pair_histogram(const double *pos, int32_t C, int64_t n, double box, const double *cell,
                                   const int64_t *absorbers, int32_t A, const int32_t *ipot, int32_t nph, double r_min, double dr, int32_t nr,
                                   double rmax, double *hist, uint64_t *n_short, void *stream);
/* Gradient (C, n, 3) of sum_k g_k chi_k with respect to pos, chi = scale * sum over every ordered pair of every
 * copy of the interpolated table row (PairTables.single_scattering, forward.py:303-319, with scale = 1 / (C n)),
 * given D = T g (nph, nr) FP64 (T the tables of potentials 1..nph).  One atom per block, fixed-order sums. */
FG_API fg_status fg_pair_ss_grad(const double *pos, int32_t C, int64_t n, double box, const double *cell,
                                 const int32_t *ipot, int32_t nph,
                                 const double *D, double r_min, double dr, int32_t nr, double rmax, double scale,
                                 double *grad, void *stream);

/* ---------------------------------------------------------------------------------------------- path columns
 * FEFF's feffNNNN.dat columns of B paths from their signals (replaces the reference's PathStage._columns,
 * genfmt.py:449-461, FEFF's fdtarr.f): mag (B, E) = |cchi| |xk| reff^2 exp(2 reff / lambda) / red factor in
 * angstrom, phase (B, E) = the unwrapped phase of cchi minus (2 Re phc unwrapped + l pi).  cchi (B, E) and reff (B,
 * angstrom) in the precision's types (as fg_cchi writes them); cols (E, 4) FP64 per energy: |xk| (1/bohr),
 * 2 / lambda (1/bohr), 1 / red factor, 2 Re phc unwrapped + l pi (GPUPathStage.columns builds it). */
FG_API fg_status fg_path_columns(int64_t B, int32_t E, fg_precision prec, const void *cchi, const void *reff,
                                 const double *cols, double *mag, double *phase, void *stream);

/* The path geometry of GPUPathStage.geometry (src/feffgpu/stage.py:170-206): coords (B, nleg, 3) FP64 in bohr,
 * absorber first -> ri, beta, eta (B, nleg) FP64 for legs 1..nleg (leg lengths in bohr, scattering angles, Euler sums
 * eta_j = alpha_(j-1) + gamma_j), with the reference's branch choices; the backward gives dL/dcoords (B, nleg, 3) from
 * dL/dri, dL/dbeta, dL/deta.  nleg 2..9. */
FG_API fg_status fg_path_geometry(int64_t B, int32_t nleg, const double *coords, double *ri, double *beta, double *eta,
                                  void *stream);
FG_API fg_status fg_path_geometry_backward(int64_t B, int32_t nleg, const double *coords, const double *grad_ri,
                                           const double *grad_beta, const double *grad_eta, double *grad_coords,
                                           void *stream);

/* ---------------------------------------------------------------------------------------------- R-space misfit
 * The loss of the refinement (src/feffgpu/exafs/transform.py:104-145): per row b of rows (B, NK) FP64,
 * R[b] = inv_norm * sum_m |(F x_b)_m - target_m|^2 with F (NR, NK) the windowed, k-weighted FFT restricted to the R
 * window (complex128, interleaved) and target (NR) complex128; with grad non-NULL also grad (B, NK) = dR[b]/dx_b.
 * One block per row, fixed-order FP64 sums. */
FG_API fg_status fg_rspace_misfit(int64_t B, int32_t NK, int32_t NR, const double *rows, const double *F,
                                  const double *target, double inv_norm, double *R, double *grad, void *stream);

/* ---------------------------------------------------------------------------------------------- multi-GPU split
 * Host: owner (n) = the rank of every path for a split over `world` ranks -- paths in order of decreasing cost (equal
 * costs in index order) each to the least-loaded rank (equal loads: the lowest rank).  The reference shards whole MD
 * frames across processes (src/feffgpu/parallel/__init__.py:78-133); this splits one path list by its cost. */
FG_API fg_status fg_shard_lpt(const double *cost, int64_t n, int32_t world, int32_t *owner);

#ifdef __cplusplus
}
#endif
#endif /* FEFFGPU_B200_H */
