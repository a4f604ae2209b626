// fg_paths.cu -- the path finder on the device (the reference's GPUPathFinder, src/feffgpu/pathfinder.py:159-279,
// itself FEFF's paths.f / pathsd.f / prcrit.f), batched over absorbers.
//
// A path of nleg legs is a sequence of nleg - 1 "intermediates" of its absorber: the candidates (atoms within rmax of
// the absorber, minimum image, the absorber excluded, in atom order) followed by the absorber itself.  Sequences grow
// one atom per level from the candidates: a child appends any intermediate other than its parent's last atom whose
// closed length (absorber -> sequence -> absorber) fits 2 rmax.  A sequence whose last atom is a candidate is a path;
// of a path and its reverse the lexicographically smaller is kept, with degeneracy 2, or 1 for a palindrome
// (pathfinder.py:233-271).  Children are written in parent order and, within a parent, in intermediate order, so the
// output order is the reference's (its enumeration is the same breadth-first order).
//
// Every length is FP32 and formed as the reference's FP32 arithmetic forms it: differences, squares and sums
// without contraction, correctly rounded square roots, lengths accumulated left to right.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "fg_launch.h"

namespace fg {
namespace {

constexpr int kNBeta = 40;   // cos(beta) grid of the importance table: 0.025 steps (pathfinder.py:23, 49-50)

__device__ __forceinline__ float len3(float x, float y, float z)
{
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}

// minimum image in a cubic box of length b (b <= 0: none), as rel - b * round(rel / b) without contraction
__device__ __forceinline__ float wrap1(float r, float b)
{
    return b > 0.f ? __fsub_rn(r, __fmul_rn(b, rintf(__fdiv_rn(r, b)))) : r;
}

// minimum image in a general periodic cell (cell.py:26-35 of the reference): f = rel inv(cell), rel = (f - round(f))
// cell, lattice vectors as the rows of cell; c holds the cell (row-major 3 x 3) and then its inverse
__device__ __forceinline__ void wrap_cell(const float *__restrict__ c, float &x, float &y, float &z)
{
    const float *inv = c + 9;
    float f[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        f[j] = fmaf(z, inv[6 + j], fmaf(y, inv[3 + j], x * inv[j]));
        f[j] -= rintf(f[j]);
    }
    x = fmaf(f[2], c[6], fmaf(f[1], c[3], f[0] * c[0]));
    y = fmaf(f[2], c[7], fmaf(f[1], c[4], f[0] * c[1]));
    z = fmaf(f[2], c[8], fmaf(f[1], c[5], f[0] * c[2]));
}

// ------------------------------------------------------------------------------------------------ candidates
// Whether atom i is a candidate of the absorber ab at (ax, ay, az), and its minimum-image position relative to it
__device__ __forceinline__ bool candidate(const float *__restrict__ pos, int64_t i, int64_t ab, float ax, float ay,
                                          float az, float box, const float *__restrict__ cell, float rmax, float &rx,
                                          float &ry, float &rz)
{
    if (cell) {
        rx = __fsub_rn(pos[3 * i], ax);
        ry = __fsub_rn(pos[3 * i + 1], ay);
        rz = __fsub_rn(pos[3 * i + 2], az);
        wrap_cell(cell, rx, ry, rz);
    } else {
        rx = wrap1(__fsub_rn(pos[3 * i], ax), box);
        ry = wrap1(__fsub_rn(pos[3 * i + 1], ay), box);
        rz = wrap1(__fsub_rn(pos[3 * i + 2], az), box);
    }
    return i != ab && len3(rx, ry, rz) <= rmax;
}

// One block per absorber slot.  count: number of candidates; with out != null the candidates are written in atom
// order at off[a] (ordered compaction: warp ballots, then the warps' counts in order).
template <bool WRITE>
__global__ void k_candidates(const float *__restrict__ pos_all, int64_t n, float box, const float *__restrict__ cell,
                             const int64_t *__restrict__ absorbers, int32_t per_frame, float rmax,
                             int32_t *__restrict__ count, const int64_t *__restrict__ off,
                             int64_t *__restrict__ cand_atom, float *__restrict__ cand_rel)
{
    __shared__ int warp_n[32];
    __shared__ int64_t base_s;
    const int a = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const float *pos = pos_all + (int64_t)(a / per_frame) * n * 3;   // the slot's frame
    const int64_t ab = absorbers[a];
    const float ax = pos[3 * ab], ay = pos[3 * ab + 1], az = pos[3 * ab + 2];
    if (threadIdx.x == 0) base_s = WRITE ? off[a] : 0;
    __syncthreads();
    int64_t total = 0;
    for (int64_t i0 = 0; i0 < n; i0 += blockDim.x) {
        const int64_t i = i0 + threadIdx.x;
        float rx = 0.f, ry = 0.f, rz = 0.f;
        const bool c = i < n && candidate(pos, i, ab, ax, ay, az, box, cell, rmax, rx, ry, rz);
        const unsigned m = __ballot_sync(0xffffffffu, c);
        if (lane == 0) warp_n[w] = __popc(m);
        __syncthreads();
        int before = 0, chunk = 0;
        for (int q = 0; q < nw; ++q) {
            if (q < w) before += warp_n[q];
            chunk += warp_n[q];
        }
        if (WRITE && c) {
            const int64_t o = base_s + total + before + __popc(m & ((1u << lane) - 1u));
            cand_atom[o] = i;
            cand_rel[3 * o] = rx;
            cand_rel[3 * o + 1] = ry;
            cand_rel[3 * o + 2] = rz;
        }
        total += chunk;
        __syncthreads();
    }
    if (!WRITE && threadIdx.x == 0) count[a] = (int32_t)total;
}

// The candidates of one absorber over many blocks, in two passes without a host round trip: block b compacts the
// candidates among atoms [b kCandChunk, (b + 1) kCandChunk) in atom order to the same offset of a scratch and counts
// them; after a scan of the counts (k_scan_counts) k_cand_place moves each block's run to its place, so the result is
// k_candidates' order.  A one-absorber call cannot fill the GPU with a block per absorber.
constexpr int kCandChunk = 256;

__global__ void __launch_bounds__(kCandChunk)
    k_cand_blocks(const float *__restrict__ pos, int64_t n, float box, const float *__restrict__ cell, int64_t ab,
                  float rmax, int64_t *__restrict__ tmp_atom, float *__restrict__ tmp_rel, int32_t *__restrict__ bcnt)
{
    __shared__ int warp_n[kCandChunk / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const float ax = pos[3 * ab], ay = pos[3 * ab + 1], az = pos[3 * ab + 2];
    const int64_t i = (int64_t)blockIdx.x * kCandChunk + threadIdx.x;
    float rx = 0.f, ry = 0.f, rz = 0.f;
    const bool c = i < n && candidate(pos, i, ab, ax, ay, az, box, cell, rmax, rx, ry, rz);
    const unsigned m = __ballot_sync(0xffffffffu, c);
    if (lane == 0) warp_n[w] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int q = 0; q < kCandChunk / 32; ++q) {
        if (q < w) before += warp_n[q];
        total += warp_n[q];
    }
    if (c) {
        const int64_t o = (int64_t)blockIdx.x * kCandChunk + before + __popc(m & ((1u << lane) - 1u));
        tmp_atom[o] = i;
        tmp_rel[3 * o] = rx;
        tmp_rel[3 * o + 1] = ry;
        tmp_rel[3 * o + 2] = rz;
    }
    if (threadIdx.x == 0) bcnt[blockIdx.x] = total;
}

// Block b's run to its place (boff: the scan of the block counts), with the single-scattering partial paths: length,
// sequence (the candidate itself) and slot 0.  Also off = {0, nc} and absorbers[0] = ab for the later kernels.
__global__ void __launch_bounds__(kCandChunk)
    k_cand_place(int64_t ab, const int64_t *__restrict__ tmp_atom, const float *__restrict__ tmp_rel,
                 const int32_t *__restrict__ bcnt, const int64_t *__restrict__ boff, int64_t nblocks,
                 int64_t *__restrict__ cand_atom, float *__restrict__ cand_rel, float *__restrict__ len,
                 int32_t *__restrict__ seq, int32_t *__restrict__ slot, int64_t *__restrict__ off,
                 int64_t *__restrict__ absorbers)
{
    const int64_t b = blockIdx.x;
    if (threadIdx.x < bcnt[b]) {
        const int64_t src = b * kCandChunk + threadIdx.x, o = boff[b] + threadIdx.x;
        const float x = tmp_rel[3 * src], y = tmp_rel[3 * src + 1], z = tmp_rel[3 * src + 2];
        cand_atom[o] = tmp_atom[src];
        cand_rel[3 * o] = x;
        cand_rel[3 * o + 1] = y;
        cand_rel[3 * o + 2] = z;
        len[o] = len3(x, y, z);
        seq[o] = (int32_t)o;
        slot[o] = 0;
    }
    if (b == 0 && threadIdx.x == 0) {
        off[0] = 0;
        off[1] = boff[nblocks];
        absorbers[0] = ab;
    }
}

// off[0] = 0, off[i + 1] = cnt[0] + ... + cnt[i] for i < P (P = min(P, *P_dev) when P_dev is given), and the sum in
// *total: one block, chunks of its width, warp scans carried across chunks.
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads)
    k_scan_counts(int64_t P, const int64_t *__restrict__ P_dev, const int32_t *__restrict__ cnt,
                  int64_t *__restrict__ off, int64_t *__restrict__ total)
{
    __shared__ long long warp_s[kScanThreads / 32];
    __shared__ long long carry_s;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (P_dev) P = min(P, *P_dev);
    if (threadIdx.x == 0) {
        off[0] = 0;
        carry_s = 0;
    }
    __syncthreads();
    for (int64_t i0 = 0; i0 < P; i0 += kScanThreads) {
        const int64_t i = i0 + threadIdx.x;
        long long x = i < P ? cnt[i] : 0;
        for (int d = 1; d < 32; d <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) warp_s[w] = x;
        __syncthreads();
        if (w == 0) {
            long long v = warp_s[lane];
            for (int d = 1; d < 32; d <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, v, d);
                if (lane >= d) v += y;
            }
            warp_s[lane] = v;
        }
        __syncthreads();
        const long long incl = carry_s + (w > 0 ? warp_s[w - 1] : 0) + x;
        if (i < P) off[i + 1] = incl;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry_s = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry_s;
}

// ------------------------------------------------------------------------------------------------ extension
struct Cands {
    const int64_t *off;     // (A + 1) candidate offsets per absorber slot
    const float *rel;       // (total, 3) relative positions
};

__device__ __forceinline__ void cand_xyz(const Cands &C, int64_t base, int nc, int j, float &x, float &y, float &z)
{
    if (j == nc) { x = y = z = 0.f; return; }   // the absorber
    const float *p = C.rel + 3 * (base + j);
    x = p[0]; y = p[1]; z = p[2];
}

// One warp per partial path; lanes walk the intermediates.  WRITE = false: count[p] children; true: write them at
// child_off[p] in intermediate order.
template <bool WRITE>
__global__ void k_extend(int64_t P, int m, const int32_t *__restrict__ seq, const float *__restrict__ len,
                         const int32_t *__restrict__ slot, Cands C, float two_r, int32_t *__restrict__ count,
                         const int64_t *__restrict__ child_off, int32_t *__restrict__ cseq, float *__restrict__ clen,
                         int32_t *__restrict__ cslot, const int64_t *__restrict__ P_dev = nullptr)
{
    if (P_dev) P = min(P, *P_dev);     // the parents' number where only the device knows it (P: its upper bound)
    const int lane = threadIdx.x & 31;
    const int64_t wg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwg = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t p = wg; p < P; p += nwg) {
        const int a = slot[p];
        const int64_t base = C.off[a];
        const int nc = (int)(C.off[a + 1] - base);
        const int last = seq[p * m + m - 1];
        float lx, ly, lz;
        cand_xyz(C, base, nc, last, lx, ly, lz);
        const float l0 = len[p];
        int64_t o = WRITE ? child_off[p] : 0;
        int cnt = 0;
        for (int j0 = 0; j0 <= nc; j0 += 32) {
            const int j = j0 + lane;
            bool ok = false;
            float tot = 0.f;
            if (j <= nc && j != last) {
                float x, y, z;
                cand_xyz(C, base, nc, j, x, y, z);
                tot = __fadd_rn(l0, len3(__fsub_rn(lx, x), __fsub_rn(ly, y), __fsub_rn(lz, z)));
                ok = __fadd_rn(tot, len3(x, y, z)) <= two_r;
            }
            const unsigned mask = __ballot_sync(0xffffffffu, ok);
            if (WRITE && ok) {
                const int64_t c = o + __popc(mask & ((1u << lane) - 1u));
                for (int q = 0; q < m; ++q) cseq[c * (m + 1) + q] = seq[p * m + q];
                cseq[c * (m + 1) + m] = j;
                clen[c] = tot;
                cslot[c] = a;
            }
            o += __popc(mask);
            cnt += __popc(mask);
        }
        if (!WRITE && lane == 0) count[p] = cnt;
    }
}

// Paths among the sequences: last atom a candidate, not after its reverse; deg 1 for a palindrome, else 2.
__global__ void k_terminal(int64_t Cn, int m, const int32_t *__restrict__ seq, const int32_t *__restrict__ slot,
                           const int64_t *__restrict__ off, uint8_t *__restrict__ keep, float *__restrict__ deg)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < Cn; c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t *s = seq + c * m;
        const int nc = (int)(off[slot[c] + 1] - off[slot[c]]);
        bool k = s[m - 1] != nc;
        int cmp = 0;
        for (int i = 0; i < m && cmp == 0; ++i) cmp = s[i] < s[m - 1 - i] ? -1 : (s[i] > s[m - 1 - i] ? 1 : 0);
        keep[c] = (k && cmp <= 0) ? 1 : 0;
        deg[c] = cmp == 0 ? 1.f : 2.f;
    }
}

// ------------------------------------------------------------------------------------------------ description
// One thread per path: coordinates (absorber at the origin), potentials, atom indices, closed length, the plane-wave
// importance (pathfinder.py:75-100) and, for nleg > 2, the degeneracy key (pathfinder.py:134-157).
__device__ __forceinline__ int indbet(float c)
{
    const float a = fabsf(c);
    float n = floorf(__fdiv_rn(a, 0.025f));
    if (__fsub_rn(a, __fmul_rn(n, 0.025f)) > 0.0125f) n = __fadd_rn(n, 1.f);
    if (c < 0.f) n = -n;
    int i = (int)n + kNBeta;
    return i < 0 ? 0 : (i > 2 * kNBeta ? 2 * kNBeta : i);
}

// Geometry of path b: its atoms' positions and potentials (written out when `write`), leg lengths, unit legs, closed
// length and the cosines of the scattering angles -- the arithmetic of the reference's FP32 description.
struct PathGeom {
    float px[kMaxLeg + 1], py[kMaxLeg + 1], pz[kMaxLeg + 1];
    int ip[kMaxLeg + 1];
    float ri[kMaxLeg], cb[kMaxLeg], rt;
};

__device__ __forceinline__ void path_geom(int64_t b, int nleg, const int32_t *__restrict__ seq,
                                          const int32_t *__restrict__ slot, const Cands &C,
                                          const int64_t *__restrict__ cand_atom, const int64_t *__restrict__ ipot_of,
                                          const int64_t *__restrict__ absorbers, bool write, float *__restrict__ coords,
                                          int64_t *__restrict__ ipots, int64_t *__restrict__ atoms,
                                          float *__restrict__ rtot_out, PathGeom &G)
{
    const int m = nleg - 1;
    const int a = slot[b];
    const int64_t base = C.off[a];
    const int nc = (int)(C.off[a + 1] - base);
    G.px[0] = G.py[0] = G.pz[0] = 0.f;
    G.ip[0] = 0;
    if (write) {
        coords[b * nleg * 3 + 0] = coords[b * nleg * 3 + 1] = coords[b * nleg * 3 + 2] = 0.f;
        ipots[b * nleg] = 0;
    }
    for (int q = 0; q < m; ++q) {
        const int j = seq[b * m + q];
        cand_xyz(C, base, nc, j, G.px[q + 1], G.py[q + 1], G.pz[q + 1]);
        const int64_t atom = j == nc ? absorbers[a] : cand_atom[base + j];
        G.ip[q + 1] = j == nc ? 0 : (int)ipot_of[atom];
        if (write) {
            atoms[b * m + q] = atom;
            ipots[b * nleg + q + 1] = G.ip[q + 1];
            coords[(b * nleg + q + 1) * 3 + 0] = G.px[q + 1];
            coords[(b * nleg + q + 1) * 3 + 1] = G.py[q + 1];
            coords[(b * nleg + q + 1) * 3 + 2] = G.pz[q + 1];
        }
    }
    // legs j = 0..nleg-1: atom j -> atom j+1 (atom nleg = the absorber)
    float ux[kMaxLeg], uy[kMaxLeg], uz[kMaxLeg];
    G.rt = 0.f;
    for (int j = 0; j < nleg; ++j) {
        const int k = j + 1 < nleg ? j + 1 : 0;
        const float dx = __fsub_rn(G.px[k], G.px[j]), dy = __fsub_rn(G.py[k], G.py[j]), dz = __fsub_rn(G.pz[k], G.pz[j]);
        G.ri[j] = len3(dx, dy, dz);
        G.rt = __fadd_rn(G.rt, G.ri[j]);
        const float r = fmaxf(G.ri[j], 1e-12f);
        ux[j] = __fdiv_rn(dx, r); uy[j] = __fdiv_rn(dy, r); uz[j] = __fdiv_rn(dz, r);
    }
    if (write) rtot_out[b] = G.rt;
    // cos(beta) at atom j+1 between leg j and leg j+1 (j = nleg - 1: at the absorber, last leg -> first leg)
    for (int j = 0; j < nleg; ++j) {
        const int k = j + 1 < nleg ? j + 1 : 0;
        G.cb[j] = __fadd_rn(__fadd_rn(__fmul_rn(ux[j], ux[k]), __fmul_rn(uy[j], uy[k])), __fmul_rn(uz[j], uz[k]));
    }
}

// |crit| trap of energy e, the term the importance sums over e (pathfinder.py:75-100)
__device__ __forceinline__ float importance_term(const PathGeom &G, int nleg, const int *ib, float cabs,
                                                 const fg_pf_tables &T, int e)
{
    const int m = nleg - 1;
    const float k = T.cksp[e];
    float crit = __fdiv_rn(cabs, __fmul_rn(G.ri[nleg - 1], k));
    for (int j = 0; j < m; ++j) {
        const float f = T.fbeta[((int64_t)e * T.nph1 + G.ip[j + 1]) * (2 * kNBeta + 1) + ib[j]];
        crit = __fdiv_rn(__fmul_rn(crit, f), __fmul_rn(G.ri[j], k));
    }
    crit = __fmul_rn(crit, expf(-__fdiv_rn(G.rt, T.xlam[e])));
    return __fmul_rn(fabsf(crit), T.trap[e - T.ik0]);
}

// forward key (ri..., cos...) and its reverse (ri reversed, cos of the scatterers reversed, the absorber's cos last),
// each rounded to 1e-3; the lexicographically smaller one (pathfinder.py:134-157)
__device__ __forceinline__ void path_key(const PathGeom &G, int nleg, int64_t *__restrict__ key)
{
    int64_t kf[2 * kMaxLeg], kr[2 * kMaxLeg];
    for (int j = 0; j < nleg; ++j) {
        kf[j] = (int64_t)rintf(__fmul_rn(G.ri[j], 1000.f));
        kf[nleg + j] = (int64_t)rintf(__fmul_rn(G.cb[j], 1000.f));
        kr[j] = (int64_t)rintf(__fmul_rn(G.ri[nleg - 1 - j], 1000.f));
    }
    for (int j = 0; j < nleg - 1; ++j) kr[nleg + j] = (int64_t)rintf(__fmul_rn(G.cb[nleg - 2 - j], 1000.f));
    kr[2 * nleg - 1] = kf[2 * nleg - 1];
    int cmp = 0;
    for (int j = 0; j < 2 * nleg && cmp == 0; ++j) cmp = kr[j] < kf[j] ? -1 : (kr[j] > kf[j] ? 1 : 0);
    for (int j = 0; j < 2 * nleg; ++j) key[j] = cmp < 0 ? kr[j] : kf[j];
}

// One thread per path: coordinates (absorber at the origin), potentials, atom indices, closed length, the plane-wave
// importance (pathfinder.py:75-100) and, for nleg > 2, the degeneracy key (pathfinder.py:134-157).
__global__ void k_describe(int64_t B, int nleg, const int32_t *__restrict__ seq, const int32_t *__restrict__ slot,
                           Cands C, const int64_t *__restrict__ cand_atom, const int64_t *__restrict__ ipot_of,
                           const int64_t *__restrict__ absorbers, fg_pf_tables T, float *__restrict__ coords,
                           int64_t *__restrict__ ipots, int64_t *__restrict__ atoms, float *__restrict__ rtot_out,
                           float *__restrict__ xport, int64_t *__restrict__ key)
{
    const int m = nleg - 1;
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x) {
        PathGeom G;
        path_geom(b, nleg, seq, slot, C, cand_atom, ipot_of, absorbers, true, coords, ipots, atoms, rtot_out, G);
        if (xport) {
            int ib[kMaxLeg];
            for (int j = 0; j < m; ++j) ib[j] = indbet(G.cb[j]);
            const float cabs = fmaxf(fabsf(G.cb[nleg - 1]), 0.3f);
            float s = 0.f;
            for (int e = T.ik0; e < T.E; ++e) s = __fadd_rn(s, importance_term(G, nleg, ib, cabs, T, e));
            xport[b] = s;
        }
        if (key && nleg > 2) path_key(G, nleg, key + b * 2 * nleg);
    }
}

// The same description, one warp per path (a few thousand paths of one absorber would leave most of the GPU idle
// with a thread each): the lanes form the importance's per-energy terms, one lane sums them in energy order -- the
// thread-per-path kernel's order, so the importance is bit for bit the same.  Paths whose keep flag is 0 (sequences
// that are not paths) are skipped.
constexpr int kDescribeWarps = 4;
__global__ void __launch_bounds__(32 * kDescribeWarps)
    k_describe_warp(int64_t B, int nleg, const int32_t *__restrict__ seq, const int32_t *__restrict__ slot, Cands C,
                    const int64_t *__restrict__ cand_atom, const int64_t *__restrict__ ipot_of,
                    const int64_t *__restrict__ absorbers, fg_pf_tables T, const uint8_t *__restrict__ keep,
                    float *__restrict__ coords, int64_t *__restrict__ ipots, int64_t *__restrict__ atoms,
                    float *__restrict__ rtot_out, float *__restrict__ xport, int64_t *__restrict__ key,
                    float *__restrict__ c1, int64_t *__restrict__ ip1)
{
    extern __shared__ float terms_all[];                       // (kDescribeWarps, E)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float *terms = terms_all + (size_t)w * T.E;
    const int m = nleg - 1;
    for (int64_t b = (int64_t)blockIdx.x * kDescribeWarps + w; b < B; b += (int64_t)gridDim.x * kDescribeWarps) {
        if (keep && !keep[b]) continue;                        // warp-uniform
        PathGeom G;
        path_geom(b, nleg, seq, slot, C, cand_atom, ipot_of, absorbers, lane == 0, coords, ipots, atoms, rtot_out, G);
        if (lane == 0 && c1) {
            c1[3 * b] = G.px[1];
            c1[3 * b + 1] = G.py[1];
            c1[3 * b + 2] = G.pz[1];
        }
        if (lane == 0 && ip1) ip1[b] = G.ip[1];
        if (xport) {
            int ib[kMaxLeg];
            for (int j = 0; j < m; ++j) ib[j] = indbet(G.cb[j]);
            const float cabs = fmaxf(fabsf(G.cb[nleg - 1]), 0.3f);
            for (int e = T.ik0 + lane; e < T.E; e += 32) terms[e] = importance_term(G, nleg, ib, cabs, T, e);
            __syncwarp();
            if (lane == 0) {
                float s = 0.f;
                for (int e = T.ik0; e < T.E; ++e) s = __fadd_rn(s, terms[e]);
                xport[b] = s;
            }
            __syncwarp();
        }
        if (lane == 0 && key && nleg > 2) path_key(G, nleg, key + b * 2 * nleg);
    }
}

int grid_of(int64_t work, int per_block)
{
    const int64_t g = (work + per_block - 1) / per_block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

}  // namespace
}  // namespace fg

using namespace fg;

extern "C" fg_status fg_pf_candidates(const float *pos, int64_t n, float box, const float *cell,
                                      const int64_t *absorbers, int32_t A,
                                      int32_t per_frame, float rmax, int32_t *count, const int64_t *offset,
                                      int64_t *cand_atom, float *cand_rel, void *stream)
{
    if (n < 0 || A < 0 || per_frame < 1) return fail(FG_ERR_VALUE, "negative size");
    if (A == 0) return FG_OK;
    if (!pos || !absorbers) return fail(FG_ERR_VALUE, "null argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // a block per absorber slot; a few slots (one absorber's call) get wide blocks so that the scan over the atoms
    // is short (the compaction is ordered by warps, so the result does not depend on the width)
    const int threads = A < 64 ? 1024 : 256;
    if (!offset) {
        if (!count) return fail(FG_ERR_VALUE, "null count");
        k_candidates<false><<<A, threads, 0, st>>>(pos, n, box, cell, absorbers, per_frame, rmax, count, nullptr,
                                                   nullptr, nullptr);
    } else {
        if (!cand_atom || !cand_rel) return fail(FG_ERR_VALUE, "null output");
        k_candidates<true><<<A, threads, 0, st>>>(pos, n, box, cell, absorbers, per_frame, rmax, nullptr, offset,
                                                  cand_atom, cand_rel);
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

extern "C" fg_status fg_pf_extend(int64_t P, int32_t m, const int32_t *seq, const float *len, const int32_t *slot,
                                  const int64_t *cand_off, const float *cand_rel, float two_r, int32_t *count,
                                  const int64_t *child_off, int32_t *child_seq, float *child_len, int32_t *child_slot,
                                  void *stream)
{
    if (P < 0 || m < 1 || m + 1 > kMaxLeg - 1) return fail(FG_ERR_VALUE, "bad partial-path shape");
    if (P == 0) return FG_OK;
    if (!seq || !len || !slot || !cand_off || !cand_rel) return fail(FG_ERR_VALUE, "null argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Cands C{cand_off, cand_rel};
    const int blocks = grid_of(P * 32, 256);
    if (!child_off) {
        if (!count) return fail(FG_ERR_VALUE, "null count");
        k_extend<false><<<blocks, 256, 0, st>>>(P, m, seq, len, slot, C, two_r, count, nullptr, nullptr, nullptr,
                                                nullptr);
    } else {
        if (!child_seq || !child_len || !child_slot) return fail(FG_ERR_VALUE, "null output");
        k_extend<true><<<blocks, 256, 0, st>>>(P, m, seq, len, slot, C, two_r, nullptr, child_off, child_seq, child_len,
                                               child_slot);
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

extern "C" fg_status fg_pf_terminal(int64_t C, int32_t m, const int32_t *seq, const int32_t *slot,
                                    const int64_t *cand_off, uint8_t *keep, float *deg, void *stream)
{
    if (C < 0 || m < 1) return fail(FG_ERR_VALUE, "bad shape");
    if (C == 0) return FG_OK;
    if (!seq || !slot || !cand_off || !keep || !deg) return fail(FG_ERR_VALUE, "null argument");
    k_terminal<<<grid_of(C, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(C, m, seq, slot, cand_off, keep, deg);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

extern "C" fg_status fg_pf_describe(int64_t B, int32_t nleg, const int32_t *seq, const int32_t *slot,
                                    const int64_t *cand_off, const float *cand_rel, const int64_t *cand_atom,
                                    const int64_t *ipot_of, const int64_t *absorbers, const fg_pf_tables *T,
                                    float *coords, int64_t *ipots, int64_t *atoms, float *rtot, float *xport,
                                    int64_t *key, void *stream)
{
    if (B < 0 || nleg < 2 || nleg > kMaxLeg) return fail(FG_ERR_VALUE, "bad path shape");
    if (B == 0) return FG_OK;
    if (!seq || !slot || !cand_off || !cand_rel || !cand_atom || !ipot_of || !absorbers || !coords || !ipots ||
        !atoms || !rtot || (xport && !T))
        return fail(FG_ERR_VALUE, "null argument");
    fg_pf_tables t{};
    if (T) {
        t = *T;
        if (t.E < 1 || t.nph1 < 1 || t.ik0 < 0 || t.ik0 >= t.E || !t.fbeta || !t.cksp || !t.xlam || !t.trap)
            return fail(FG_ERR_VALUE, "incomplete importance tables");
    }
    k_describe<<<grid_of(B, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        B, nleg, seq, slot, Cands{cand_off, cand_rel}, cand_atom, ipot_of, absorbers, t, coords, ipots, atoms, rtot,
        xport, key);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

namespace fg {
fg_status candidates_one(const float *pos, int64_t n, float box, const float *cell, int64_t absorber, float rmax,
                         int64_t *tmp_atom, float *tmp_rel, int32_t *bcnt, int64_t *boff, int64_t *cand_atom,
                         float *cand_rel, float *len, int32_t *seq, int32_t *slot, int64_t *off, int64_t *absorbers,
                         int64_t *nc, cudaStream_t st)
{
    const int64_t G = (n + kCandChunk - 1) / kCandChunk;
    if (G > INT32_MAX) return fail(FG_ERR_VALUE, "too many atoms");
    k_cand_blocks<<<(unsigned)G, kCandChunk, 0, st>>>(pos, n, box, cell, absorber, rmax, tmp_atom, tmp_rel, bcnt);
    FG_CUDA(cudaGetLastError());
    k_scan_counts<<<1, kScanThreads, 0, st>>>(G, nullptr, bcnt, boff, nc);
    FG_CUDA(cudaGetLastError());
    k_cand_place<<<(unsigned)G, kCandChunk, 0, st>>>(absorber, tmp_atom, tmp_rel, bcnt, boff, G, cand_atom, cand_rel,
                                                     len, seq, slot, off, absorbers);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

fg_status extend_count(int64_t P, const int64_t *P_dev, int32_t m, const int32_t *seq, const float *len,
                       const int32_t *slot, const int64_t *cand_off, const float *cand_rel, float two_r,
                       int32_t *count, cudaStream_t st)
{
    if (P <= 0) return FG_OK;
    k_extend<false><<<grid_of(P * 32, 256), 256, 0, st>>>(P, m, seq, len, slot, Cands{cand_off, cand_rel}, two_r,
                                                          count, nullptr, nullptr, nullptr, nullptr, P_dev);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

fg_status scan_counts(int64_t P, const int64_t *P_dev, const int32_t *count, int64_t *off, int64_t *total,
                      cudaStream_t st)
{
    k_scan_counts<<<1, kScanThreads, 0, st>>>(P, P_dev, count, off, total);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

fg_status describe_paths_warp(int64_t B, int32_t nleg, const int32_t *seq, const int32_t *slot, const int64_t *cand_off,
                              const float *cand_rel, const int64_t *cand_atom, const int64_t *ipot_of,
                              const int64_t *absorbers, const fg_pf_tables *T, const uint8_t *keep, float *coords,
                              int64_t *ipots, int64_t *atoms, float *rtot, float *xport, int64_t *key, float *c1,
                              int64_t *ip1, cudaStream_t st)
{
    if (B == 0) return FG_OK;
    const fg_pf_tables t = *T;
    const size_t smem = (size_t)kDescribeWarps * t.E * sizeof(float);
    if (smem > 48 * 1024) FG_CUDA(cudaFuncSetAttribute(k_describe_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)smem));
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((B + kDescribeWarps - 1) / kDescribeWarps, 148 * 16));
    k_describe_warp<<<blocks, 32 * kDescribeWarps, smem, st>>>(B, nleg, seq, slot, Cands{cand_off, cand_rel}, cand_atom,
                                                                ipot_of, absorbers, t, keep, coords, ipots, atoms,
                                                                rtot, xport, key, c1, ip1);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}
}  // namespace fg

extern "C" fg_status fg_pf_windows(const float *sorted_len, const int64_t *seg_off, int64_t nseg, float eps,
                                   int64_t *window)
{
    if (nseg < 0 || !seg_off || (nseg > 0 && (!sorted_len || !window))) return fail(FG_ERR_VALUE, "null argument");
    // greedy windows of width eps over each segment's ascending lengths (pathfinder.py:110-119)
    for (int64_t s = 0; s < nseg; ++s) {
        const int64_t lo = seg_off[s], hi = seg_off[s + 1];
        int64_t i = lo, w = 0;
        while (i < hi) {
            const float edge = sorted_len[i] + eps;
            const int64_t j = std::max<int64_t>(std::lower_bound(sorted_len + i, sorted_len + hi, edge) - sorted_len,
                                                i + 1);
            for (int64_t q = i; q < j; ++q) window[q] = w;
            ++w;
            i = j;
        }
    }
    return FG_OK;
}
