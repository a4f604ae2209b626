// fg_pf_one.cu -- the path finder for one absorber, driven from the host in C++ (the reference's front ends call the
// finder once per absorber: src/feffgpu/exafs/forward.py:122-123, md/spectrum.py:275-277).  The kernels are the
// batched finder's (fg_paths.cu); what changes is the driver: one call runs candidates, growth, description, merges
// and importance cut with two synchronisations (the numbers of candidates and of three-leg sequences; the result
// fields) plus one per growth level past three legs, instead of a Python sequence of small torch operations whose
// launch and dispatch latency dominated a call of a few hundred paths.  The merges and the cut run
// on the host in FP32 with the arithmetic and order of the batched path (and so of the reference, pathfinder.py:
// 102-157, 271-279), so the kept paths are bit for bit those of fg_pf_* driven by feffgpu_b200/pathfinder.py.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "fg_launch.h"

namespace fg {
namespace {

// The finder's own stream-ordered memory pool per device: its scratch comes and goes with every call, so the pool
// keeps up to 1 GiB reserved between calls instead of returning it to the driver at each synchronisation (the
// device's default pool, and its settings, are left alone).
constexpr int kMaxDevices = 128;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};

fg_status finder_pool(cudaMemPool_t *out)
{
    int dev = 0;
    FG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(FG_ERR_VALUE, "device index out of range");
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pool[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        FG_CUDA(cudaMemPoolCreate(&g_pool[dev], &props));
        uint64_t keep = uint64_t(1) << 30;
        FG_CUDA(cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    *out = g_pool[dev];
    return FG_OK;
}

// Device scratch of one call, stream-ordered from the finder's pool and handed out from a few large blocks (a call
// needs about thirty arrays; one pool allocation each cost more host time than the kernels that fill them).  Two
// regions: `get` for arrays that stay on the device, `get_host` for the fields the host reads after the last
// synchronisation, which so lie in a few contiguous blocks that are copied to the host in one copy each.
struct Scratch {
    struct Block {
        unsigned char *base = nullptr;
        size_t used = 0, cap = 0;
    };
    static constexpr size_t kBlock = size_t(4) << 20;
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    std::vector<Block> dev, host;
    fg_status take(std::vector<Block> &region, size_t bytes, void **out)
    {
        bytes = align_up(std::max<size_t>(bytes, 1), 256);
        if (region.empty() || region.back().cap - region.back().used < bytes) {
            if (!pool)
                if (fg_status rc = finder_pool(&pool)) return rc;
            Block b;
            b.cap = std::max(bytes, kBlock);
            void *p = nullptr;
            FG_CUDA(cudaMallocFromPoolAsync(&p, b.cap, pool, st));
            b.base = static_cast<unsigned char *>(p);
            region.push_back(b);
        }
        Block &b = region.back();
        *out = b.base + b.used;
        b.used += bytes;
        return FG_OK;
    }
    template <typename T> fg_status get(size_t count, T **out)
    {
        void *p = nullptr;
        if (fg_status rc = take(dev, count * sizeof(T), &p)) return rc;
        *out = static_cast<T *>(p);
        return FG_OK;
    }
    template <typename T> fg_status get_host(size_t count, T **out)
    {
        void *p = nullptr;
        if (fg_status rc = take(host, count * sizeof(T), &p)) return rc;
        *out = static_cast<T *>(p);
        return FG_OK;
    }
    void release()
    {
        for (const Block &b : dev) cudaFreeAsync(b.base, st);
        for (const Block &b : host) cudaFreeAsync(b.base, st);
        dev.clear();
        host.clear();
    }
};

// The kept paths of one leg count into the caller's arrays: path b of the output is described path idx[b], with the
// degeneracy deg_k[b] of the merges
__global__ void k_gather_paths(int64_t B, int nleg, const int64_t *__restrict__ idx, const float *__restrict__ deg_k,
                               const float *__restrict__ c_in, const int64_t *__restrict__ ip_in,
                               const float *__restrict__ x_in, const int64_t *__restrict__ at_in,
                               float *__restrict__ coords, int64_t *__restrict__ ipots, float *__restrict__ deg,
                               float *__restrict__ xport, int64_t *__restrict__ atoms)
{
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const int64_t j = idx[b];
    for (int q = 0; q < 3 * nleg; ++q) coords[b * 3 * nleg + q] = c_in[j * 3 * nleg + q];
    for (int q = 0; q < nleg; ++q) ipots[b * nleg + q] = ip_in[j * nleg + q];
    for (int q = 0; q < nleg - 1; ++q) atoms[b * (nleg - 1) + q] = at_in[j * (nleg - 1) + q];
    xport[b] = x_in[j];
    deg[b] = deg_k[b];
}

// indices that sort v ascending, equal values in index order (numpy's argsort(kind="stable"))
template <typename T> std::vector<int64_t> stable_argsort(const std::vector<T> &v)
{
    std::vector<int64_t> o(v.size());
    std::iota(o.begin(), o.end(), int64_t(0));
    std::stable_sort(o.begin(), o.end(), [&](int64_t a, int64_t b) { return v[a] < v[b]; });
    return o;
}

// numpy.unique(rows, axis=0, return_inverse=True)[1]: the rank of each row among the distinct rows in lexicographic
// order; rows of width w, row i at keys[i * w]
std::vector<int64_t> unique_inverse(const std::vector<int64_t> &keys, int64_t n, int w, int64_t *groups)
{
    std::vector<int64_t> o(n);
    std::iota(o.begin(), o.end(), int64_t(0));
    auto less = [&](int64_t a, int64_t b) {
        return std::lexicographical_compare(keys.begin() + a * w, keys.begin() + (a + 1) * w, keys.begin() + b * w,
                                            keys.begin() + (b + 1) * w);
    };
    std::stable_sort(o.begin(), o.end(), less);
    std::vector<int64_t> inv(n);
    int64_t g = -1;
    for (int64_t i = 0; i < n; ++i) {
        if (i == 0 || less(o[i - 1], o[i])) ++g;
        inv[o[i]] = g;
    }
    *groups = g + 1;
    return inv;
}

}  // namespace
}  // namespace fg

using namespace fg;

// One leg count of the result: its device arrays (all paths described, before the cut) and the kept indices.
struct fg_pf_leg {
    int nleg = 0;
    int64_t nb = 0;                     // paths described
    float *coords = nullptr;            // (nb, nleg, 3)
    int64_t *ipots = nullptr, *atoms = nullptr;
    float *rtot = nullptr, *xport = nullptr, *deg = nullptr;
    int64_t *key = nullptr;
    uint8_t *keep = nullptr;            // terminal flags (nleg > 2), null for single scattering
    std::vector<int64_t> kept;          // indices into the described paths
    std::vector<float> kept_deg;        // degeneracies of the kept paths
    const int64_t *d_kept = nullptr;    // the same two on the device
    const float *d_kept_deg = nullptr;
};

struct fg_pf_result {
    Scratch scratch;
    std::vector<fg_pf_leg> legs;
    float ref = 1.f;
};

namespace {
// pinned staging for the device -> host copies of one call (per host thread, grown as needed)
struct Pinned {
    void *p = nullptr;
    size_t n = 0;
    ~Pinned()
    {
        if (p) cudaFreeHost(p);
    }
};
thread_local Pinned t_pinned;

fg_status pinned(size_t bytes, unsigned char **out)
{
    if (t_pinned.n < bytes) {
        if (t_pinned.p) cudaFreeHost(t_pinned.p);
        t_pinned.p = nullptr;
        t_pinned.n = 0;
        const size_t want = std::max<size_t>(bytes, size_t(1) << 20);
        FG_CUDA(cudaMallocHost(&t_pinned.p, want));
        t_pinned.n = want;
    }
    *out = static_cast<unsigned char *>(t_pinned.p);
    return FG_OK;
}

constexpr int64_t kPartialLimit = 30000000;   // partial paths per absorber (the reference's limit, pathfinder.py:25)

// The merges and the importance cut of one absorber (the host side of feffgpu_b200/pathfinder.py's one-absorber
// path, itself pathfinder.py:102-157, 271-279 of the reference), FP32 throughout in the same operation order.
struct LegHost {
    int nleg;
    int64_t nb;                            // terminal paths
    std::vector<int64_t> idx;              // their indices among the described sequences
    std::vector<float> xport, deg, rtot;   // per terminal path
    std::vector<int64_t> key;              // (nb, 2 nleg) when keyed
};

void merge_and_cut(std::vector<LegHost> &L, int64_t cnt, const std::vector<float> &c1, const std::vector<int64_t> &ip1,
                   bool merge, float critpw, std::vector<fg_pf_leg> &legs, float &ref_out)
{
    LegHost &ss = L[0];
    const int64_t nb2 = ss.nb;
    std::vector<float> d(nb2);
    for (int64_t i = 0; i < nb2; ++i) {
        const float x = c1[3 * i], y = c1[3 * i + 1], z = c1[3 * i + 2];
        d[i] = std::sqrt(x * x + y * y + z * z);
    }
    float ref = 1.f;
    std::vector<int64_t> rep(nb2);
    std::iota(rep.begin(), rep.end(), int64_t(0));
    std::vector<float> ss_deg = ss.deg;
    auto first_min = [](const std::vector<float> &v, const std::vector<int64_t> &at) {
        int64_t best = 0;
        for (int64_t i = 1; i < (int64_t)at.size(); ++i)
            if (v[at[i]] < v[at[best]]) best = i;
        return best;
    };
    if (!merge || nb2 == 0) {
        if (nb2 && cnt > 0) ref = ss.xport[rep[first_min(d, rep)]];
    }
    if (merge && nb2) {
        // greedy 1e-3 A windows over the sorted closed lengths of every path
        std::vector<float> all;
        for (const LegHost &l : L) all.insert(all.end(), l.rtot.begin(), l.rtot.end());
        const std::vector<int64_t> o = stable_argsort(all);
        std::vector<float> sr(all.size());
        for (size_t i = 0; i < all.size(); ++i) sr[i] = all[o[i]];
        std::vector<int64_t> seg{0, (int64_t)sr.size()}, win_sorted(sr.size()), win(sr.size());
        fg_pf_windows(sr.data(), seg.data(), 1, 1e-3f, win_sorted.data());
        for (size_t i = 0; i < sr.size(); ++i) win[o[i]] = win_sorted[i];
        const std::vector<int64_t> od = stable_argsort(d);
        std::vector<int64_t> keys((size_t)nb2 * 3);
        for (int64_t i = 0; i < nb2; ++i) {
            keys[3 * i] = (int64_t)std::nearbyint(d[od[i]] * 1000.f);
            keys[3 * i + 1] = ip1[od[i]];
            keys[3 * i + 2] = win[od[i]];
        }
        int64_t G = 0;
        const std::vector<int64_t> inv = unique_inverse(keys, nb2, 3, &G);
        std::vector<int64_t> firstp(G, nb2);
        std::vector<float> gcount(G, 0.f);
        for (int64_t i = 0; i < nb2; ++i) {
            firstp[inv[i]] = std::min(firstp[inv[i]], i);
            gcount[inv[i]] += 1.f;
        }
        const std::vector<int64_t> go = stable_argsort(firstp);
        rep.assign(G, 0);
        ss_deg.assign(G, 0.f);
        for (int64_t g = 0; g < G; ++g) {
            rep[g] = od[firstp[go[g]]];
            ss_deg[g] = gcount[go[g]];
        }
        const int64_t f = first_min(d, rep);
        ref = ss.xport[rep[f]] * ss_deg[f];
    }
    ref_out = ref;
    legs.resize(L.size());
    for (size_t li = 0; li < L.size(); ++li) {
        const LegHost &l = L[li];
        std::vector<int64_t> idx;
        std::vector<float> dg;
        if (l.nleg == 2) {
            idx = rep;
            dg = ss_deg;
        } else {
            idx.resize(l.nb);
            std::iota(idx.begin(), idx.end(), int64_t(0));
            dg = l.deg;
        }
        std::vector<float> dtot = dg;
        if (l.nleg > 2 && merge && l.nb && cnt > 1) {
            int64_t G = 0;
            const std::vector<int64_t> inv = unique_inverse(l.key, l.nb, 2 * l.nleg, &G);
            std::vector<float> tot(G, 0.f);
            for (int64_t i = 0; i < l.nb; ++i) tot[inv[i]] += dg[i];
            for (int64_t i = 0; i < l.nb; ++i) dtot[i] = tot[inv[i]];
        }
        fg_pf_leg &out = legs[li];
        out.nleg = l.nleg;
        out.kept.clear();
        out.kept_deg.clear();
        for (size_t i = 0; i < idx.size(); ++i) {
            const float frac = 100.f * dtot[i] * l.xport[idx[i]] / ref;
            if (frac >= critpw) {
                out.kept.push_back(l.idx[idx[i]]);
                out.kept_deg.push_back(dg[i]);
            }
        }
    }
}
}  // namespace

extern "C" fg_status fg_pf_enumerate_one(const float *pos, int64_t n, float box, const float *cell, int64_t absorber,
                                         const int64_t *ipot_of, const fg_pf_tables *T, float rmax, int32_t nlegmax,
                                         float critpw, int32_t merge, fg_pf_result **out, int64_t *counts, float *ref,
                                         void *stream)
{
    if (!pos || !ipot_of || !T || !out || !counts || !ref) return fail(FG_ERR_VALUE, "null argument");
    if (n < 1 || absorber < 0 || absorber >= n) return fail(FG_ERR_VALUE, "absorber outside the atoms");
    if (nlegmax < 2 || nlegmax > kMaxLeg) return fail(FG_ERR_VALUE, "nlegmax must be 2..9");
    *out = nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fg_pf_result *r = new fg_pf_result();
    r->scratch.st = st;
    Scratch &S = r->scratch;
    auto bail = [&](fg_status rc) {
        S.release();
        delete r;
        return rc;
    };
#define FG_TRY(x)                            \
    do {                                     \
        if (fg_status rc_ = (x)) return bail(rc_); \
    } while (0)
    auto cuda = [&](cudaError_t e, const char *what) -> fg_status {
        return e == cudaSuccess ? FG_OK : fail(FG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    unsigned char *hp = nullptr;
    // Candidates and the first level's child counts without a host round trip (sized by the atom count, an upper
    // bound of the candidates'), then one synchronisation for both numbers.
    const int64_t G = (n + 255) / 256;
    int64_t *d_ab = nullptr, *d_off = nullptr, *d_counts = nullptr, *tmp_atom = nullptr, *boff = nullptr;
    int64_t *cand_atom = nullptr, *d_coff = nullptr;
    int32_t *bcnt = nullptr, *seq = nullptr, *slot = nullptr, *cc = nullptr;
    float *tmp_rel = nullptr, *cand_rel = nullptr, *len = nullptr;
    FG_TRY(S.get(1, &d_ab));
    FG_TRY(S.get(2, &d_off));
    FG_TRY(S.get(2, &d_counts));
    FG_TRY(S.get(G * 256, &tmp_atom));
    FG_TRY(S.get(G * 256 * 3, &tmp_rel));
    FG_TRY(S.get(G, &bcnt));
    FG_TRY(S.get(G + 1, &boff));
    FG_TRY(S.get(n, &cand_atom));
    FG_TRY(S.get(3 * n, &cand_rel));
    FG_TRY(S.get(n, &seq));
    FG_TRY(S.get(n, &slot));
    FG_TRY(S.get(n, &len));
    FG_TRY(candidates_one(pos, n, box, cell, absorber, rmax, tmp_atom, tmp_rel, bcnt, boff, cand_atom, cand_rel, len,
                          seq, slot, d_off, d_ab, d_counts, st));
    const float two_r = 2.f * rmax;
    if (nlegmax > 2) {
        FG_TRY(S.get(n, &cc));
        FG_TRY(S.get(n + 1, &d_coff));
        FG_TRY(extend_count(n, d_counts, 1, seq, len, slot, d_off, cand_rel, two_r, cc, st));
        FG_TRY(scan_counts(n, d_counts, cc, d_coff, d_counts + 1, st));
    } else {
        FG_TRY(cuda(cudaMemsetAsync(d_counts + 1, 0, sizeof(int64_t), st), "memset"));
    }
    FG_TRY(pinned(64, &hp));
    FG_TRY(cuda(cudaMemcpyAsync(hp, d_counts, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, st), "copy"));
    FG_TRY(cuda(cudaStreamSynchronize(st), "synchronize"));
    int64_t counts_h[2];
    std::memcpy(counts_h, hp, sizeof(counts_h));
    const int64_t nc = counts_h[0];
    // a warp per path; sequences that are not paths (terminal flag 0) are skipped.  The single-scattering call also
    // writes each candidate's position and potential (c1, ip1) for the merges.
    float *c1_dev = nullptr;
    int64_t *ip1_dev = nullptr;
    auto describe = [&](fg_pf_leg &l, const int32_t *s, const int32_t *sl, bool want_key) -> fg_status {
        const int64_t B = l.nb;
        if (fg_status rc = S.get(B * l.nleg * 3, &l.coords)) return rc;
        if (fg_status rc = S.get(B * l.nleg, &l.ipots)) return rc;
        if (fg_status rc = S.get(B * (l.nleg - 1), &l.atoms)) return rc;
        if (fg_status rc = S.get_host(B, &l.rtot)) return rc;
        if (fg_status rc = S.get_host(B, &l.xport)) return rc;
        if (want_key)
            if (fg_status rc = S.get_host(B * 2 * l.nleg, &l.key)) return rc;
        if (l.nleg == 2) {
            if (fg_status rc = S.get_host(B * 3, &c1_dev)) return rc;
            if (fg_status rc = S.get_host(B, &ip1_dev)) return rc;
        }
        return describe_paths_warp(B, l.nleg, s, sl, d_off, cand_rel, cand_atom, ipot_of, d_ab, T, l.keep, l.coords,
                                   l.ipots, l.atoms, l.rtot, l.xport, l.key, l.nleg == 2 ? c1_dev : nullptr,
                                   l.nleg == 2 ? ip1_dev : nullptr, st);
    };
    std::vector<fg_pf_leg> &legs = r->legs;
    legs.reserve(kMaxLeg);
    legs.emplace_back();
    legs[0].nleg = 2;
    legs[0].nb = nc;
    FG_TRY(describe(legs[0], seq, slot, false));
    // growth, one level per extra leg; past the first, one synchronisation per level (the number of children sizes
    // the next)
    int64_t P = nc > 1 ? nc : 0;     // multiple scattering needs two candidates (pathfinder.py:237, 243, 262)
    for (int m = 1; m <= nlegmax - 2 && P > 0; ++m) {
        int64_t Cn = counts_h[1];
        if (m > 1) {
            FG_TRY(S.get(P, &cc));
            FG_TRY(S.get(P + 1, &d_coff));
            FG_TRY(extend_count(P, nullptr, m, seq, len, slot, d_off, cand_rel, two_r, cc, st));
            FG_TRY(scan_counts(P, nullptr, cc, d_coff, d_counts + 1, st));
            FG_TRY(cuda(cudaMemcpyAsync(hp, d_counts + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "copy"));
            FG_TRY(cuda(cudaStreamSynchronize(st), "synchronize"));
            std::memcpy(&Cn, hp, sizeof(int64_t));
        }
        if (Cn > kPartialLimit || Cn * (4 * (m + 2) + 8) > (int64_t(8) << 30))
            return bail(fail(FG_ERR_VALUE, std::to_string(Cn) + " partial paths of " + std::to_string(m + 2) +
                                               " legs: lower the path cutoff or the largest number of legs"));
        if (Cn == 0) break;
        int32_t *cseq = nullptr, *cslot = nullptr;
        float *clen = nullptr;
        FG_TRY(S.get(Cn * (m + 1), &cseq));
        FG_TRY(S.get(Cn, &cslot));
        FG_TRY(S.get(Cn, &clen));
        FG_TRY(fg_pf_extend(P, m, seq, len, slot, d_off, cand_rel, two_r, nullptr, d_coff, cseq, clen, cslot, stream));
        fg_pf_leg l;
        l.nleg = m + 2;
        l.nb = Cn;
        FG_TRY(S.get_host(Cn, &l.keep));
        FG_TRY(S.get_host(Cn, &l.deg));
        FG_TRY(fg_pf_terminal(Cn, m + 1, cseq, cslot, d_off, l.keep, l.deg, stream));
        FG_TRY(describe(l, cseq, cslot, merge != 0));
        legs.push_back(l);
        seq = cseq;
        slot = cslot;
        len = clen;
        P = Cn;
    }
    // the fields the merges and the cut read: one copy per block of the host region, through pinned memory
    size_t bytes = 0;
    std::vector<size_t> at_block(S.host.size());
    for (size_t i = 0; i < S.host.size(); ++i) {
        at_block[i] = bytes;
        bytes += align_up(S.host[i].used, 256);
    }
    FG_TRY(pinned(bytes, &hp));
    for (size_t i = 0; i < S.host.size(); ++i)
        FG_TRY(cuda(cudaMemcpyAsync(hp + at_block[i], S.host[i].base, S.host[i].used, cudaMemcpyDeviceToHost, st),
                    "copy"));
    FG_TRY(cuda(cudaStreamSynchronize(st), "synchronize"));
    // the host copy of a device pointer of the host region
    auto on_host = [&](const void *d) -> const unsigned char * {
        if (!d) return nullptr;
        const unsigned char *p = static_cast<const unsigned char *>(d);
        for (size_t i = 0; i < S.host.size(); ++i)
            if (p >= S.host[i].base && p < S.host[i].base + S.host[i].used) return hp + at_block[i] + (p - S.host[i].base);
        return nullptr;
    };
    std::vector<LegHost> H(legs.size());
    for (size_t i = 0; i < legs.size(); ++i) {
        const fg_pf_leg &l = legs[i];
        LegHost &h = H[i];
        h.nleg = l.nleg;
        if (l.nb == 0) continue;
        const float *xp = reinterpret_cast<const float *>(on_host(l.xport));
        const float *rt = reinterpret_cast<const float *>(on_host(l.rtot));
        const float *dg = reinterpret_cast<const float *>(on_host(l.deg));
        const uint8_t *kp = on_host(l.keep);
        const int64_t *ky = reinterpret_cast<const int64_t *>(on_host(l.key));
        for (int64_t j = 0; j < l.nb; ++j) {
            if (kp && !kp[j]) continue;              // not a path (ends at the absorber, or after its reverse)
            h.idx.push_back(j);
            h.xport.push_back(xp[j]);
            h.rtot.push_back(rt[j]);
            h.deg.push_back(dg ? dg[j] : 1.f);
            if (ky) h.key.insert(h.key.end(), ky + j * 2 * l.nleg, ky + (j + 1) * 2 * l.nleg);
        }
        h.nb = (int64_t)h.idx.size();
    }
    std::vector<float> c1(nc * 3);
    std::vector<int64_t> ip1(nc);
    if (nc > 0) {
        std::memcpy(c1.data(), on_host(c1_dev), c1.size() * sizeof(float));
        std::memcpy(ip1.data(), on_host(ip1_dev), ip1.size() * sizeof(int64_t));
    }
    std::vector<fg_pf_leg> kept;
    merge_and_cut(H, nc, c1, ip1, merge != 0, critpw, kept, r->ref);
    for (int i = 0; i <= kMaxLeg; ++i) counts[i] = -1;
    size_t nkept = 0;
    for (size_t i = 0; i < legs.size(); ++i) {
        legs[i].kept = std::move(kept[i].kept);
        legs[i].kept_deg = std::move(kept[i].kept_deg);
        counts[legs[i].nleg] = (int64_t)legs[i].kept.size();
        nkept += legs[i].kept.size();
    }
    // every leg's kept indices, then their degeneracies, to the device in one copy
    std::vector<int64_t> packed(2 * nkept);
    int64_t *d_packed = nullptr;
    FG_TRY(S.get(packed.size(), &d_packed));
    size_t o = 0;
    for (fg_pf_leg &l : legs) {
        std::copy(l.kept.begin(), l.kept.end(), packed.begin() + o);
        float *dg = reinterpret_cast<float *>(packed.data() + nkept + o);
        std::copy(l.kept_deg.begin(), l.kept_deg.end(), dg);
        l.d_kept = d_packed + o;
        l.d_kept_deg = reinterpret_cast<const float *>(d_packed + nkept + o);
        o += l.kept.size();
    }
    if (nkept)
        FG_TRY(cuda(cudaMemcpyAsync(d_packed, packed.data(), packed.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                                    st), "copy"));
    *ref = r->ref;
    *out = r;
    return FG_OK;
#undef FG_TRY
}

extern "C" fg_status fg_pf_result_gather(fg_pf_result *r, int32_t nleg, float *coords, int64_t *ipots, float *deg,
                                         float *xport, int64_t *atoms, void *stream)
{
    if (!r) return fail(FG_ERR_VALUE, "null result");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (fg_pf_leg &l : r->legs) {
        if (l.nleg != nleg) continue;
        const int64_t B = (int64_t)l.kept.size();
        if (B == 0) return FG_OK;
        if (!coords || !ipots || !deg || !xport || !atoms) return fail(FG_ERR_VALUE, "null output");
        k_gather_paths<<<(unsigned)((B + 127) / 128), 128, 0, st>>>(B, nleg, l.d_kept, l.d_kept_deg, l.coords, l.ipots,
                                                                   l.xport, l.atoms, coords, ipots, deg, xport, atoms);
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    return fail(FG_ERR_VALUE, "no paths of " + std::to_string(nleg) + " legs in the result");
}

extern "C" void fg_pf_result_destroy(fg_pf_result *r)
{
    if (!r) return;
    r->scratch.release();
    delete r;
}
