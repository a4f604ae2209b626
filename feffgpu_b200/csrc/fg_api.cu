// fg_api.cu -- the C ABI of include/feffgpu_b200.h: stage tables, argument checks and dispatch to the kernel units.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "feffgpu_b200.h"
#include "fg_launch.h"

using namespace fg;
using cd = std::complex<double>;

// ================================================================================================ errors and launch
namespace {
thread_local std::string g_err;
int g_fwd_warps = 4;
int g_bwd_warps = 4;
}  // namespace

fg_status fg::fail(fg_status s, const std::string &m)
{
    g_err = m;
    return s;
}

// ================================================================================================ the stage
struct fg_stage {
    int device = 0, E = 0, nph = 0, nph1 = 0, ltot = 0, ihole = 0, iorder = 2, kinit = 0, ilinit = 0, L1 = 0;
    int nterm = 0, term_l[2] = {0, 0};
    int num_sms = 148;
    int max_smem = 227 * 1024;
    int fwd_warps = 0, bwd_warps = 0;   // launch shape of this stage's calls, 0 = the process default
    int fused_regs_alt = 0, fused_stage_t = 0;   // the fused forward's register budget and t-matrix staging
    // device address of the no-allocation scratch in this stage's context, looked up by its first
    // fg_chi_reduce_noalloc call (a device reset invalidates the stage, and with it this address)
    void *noalloc_scratch = nullptr;
    std::mutex noalloc_mu;
    std::vector<int> lmax_host;     // (E, nph1)
    std::vector<double> xk_host;    // (E)
    Tables<float> tf{};
    Tables<double> td{};
    std::vector<void *> bufs;
};

namespace {
// hole index -> (kappa, l) of the initial state (COMMON/setkap.f; genfmt.py:22-38)
bool hole_kappa(int ihole, int &kinit, int &linit)
{
    struct H { int k, l; std::initializer_list<int> holes; };
    const H tab[] = {{-1, 0, {1, 2, 5, 10, 17, 24, 27}}, {1, 1, {3, 6, 11, 18, 25, 30}}, {-2, 1, {4, 7, 12, 19, 26}},
                     {2, 2, {8, 13, 20, 27}}, {-3, 2, {9, 14, 21, 28}}, {3, 3, {15, 22}}, {-4, 3, {16, 23}}};
    for (const H &h : tab)
        for (int v : h.holes)
            if (v == ihole) { kinit = h.k; linit = h.l; return true; }
    return false;
}

// final-state channels and the spin-traced diagonal of bmat, ipol = 0, le2 = 0 (MATH/bcoef.f; genfmt.py:230-264)
void final_state(int kinit, int lind[9], double bdiag[9])
{
    for (int i = 0; i < 9; ++i) { lind[i] = -1; bdiag[i] = 0.0; }
    for (int k = -1; k <= 1; ++k) {
        int kap = k == 0 ? -(kinit + k) : kinit + k;
        int l = kap > 0 ? kap : -kap - 1;
        lind[k + 2] = l > 4 ? -1 : l;
    }
    // the quadrupole channels (k + 6) stay off: le2 = 0
    for (int k = 1; k <= 3; ++k)
        if (lind[k] >= 0) bdiag[k] = -2.0 * 0.5 / (2 * lind[k] + 1.0) / 3.0;
}

// Legendre normalisation xnlm(il, im), il, im 1-based (snlm.f; genfmt.py:41-53)
double xnlm_of(int il, int im)
{
    if (im < 1 || im > il) return 0.0;
    const double afac = 1.0 / 64.0;
    const int l = il - 1, m = im - 1;
    // flg(i) = i! afac^i
    auto flg = [&](int i) { double f = 1.0; for (int q = 1; q <= i; ++q) f *= q * afac; return f; };
    return std::sqrt((2 * l + 1) * flg(l - m) / flg(l + m)) * std::pow(afac, m);
}

template <typename T> fg_status upload(fg_stage *s, const std::vector<T> &v, const T **out)
{
    void *p = nullptr;
    FG_CUDA(cudaMalloc(&p, std::max<size_t>(v.size(), 1) * sizeof(T)));
    s->bufs.push_back(p);
    if (!v.empty()) FG_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    *out = static_cast<const T *>(p);
    return FG_OK;
}

template <typename R> fg_status build_tables(fg_stage *s, Tables<R> &T, const std::vector<cd> &tl,
                                             const std::vector<cd> &ck, const std::vector<cd> &dk,
                                             const std::vector<cd> &wt, const std::vector<double> &xfac,
                                             const std::vector<double> &xn, const std::vector<double> &rc,
                                             const std::vector<int> &lmax_t)
{
    T.E = s->E; T.nph1 = s->nph1; T.L1 = s->L1; T.nterm = s->nterm;
    T.term_l[0] = s->term_l[0]; T.term_l[1] = s->term_l[1];
    auto cvt = [](const std::vector<cd> &v) {
        std::vector<C2<R>> o(v.size());
        for (size_t i = 0; i < v.size(); ++i) o[i] = C2<R>{(R)v[i].real(), (R)v[i].imag()};
        return o;
    };
    std::vector<double2> dkv(dk.size());
    for (size_t i = 0; i < dk.size(); ++i) dkv[i] = make_double2(dk[i].real(), dk[i].imag());
    fg_status st;
    if ((st = upload(s, cvt(tl), &T.tl))) return st;
    if ((st = upload(s, cvt(ck), &T.ck))) return st;
    if ((st = upload(s, dkv, &T.dk))) return st;
    if ((st = upload(s, cvt(wt), &T.wt))) return st;
    if ((st = upload(s, xfac, &T.xfac))) return st;
    if ((st = upload(s, xn, &T.xnlm))) return st;
    if ((st = upload(s, rc, &T.rc))) return st;
    if ((st = upload(s, lmax_t, &T.lmax))) return st;
    T.MMd = 3;
    T.nlam = s->iorder == 0 ? 1 : (s->iorder == 1 ? 3 : (s->iorder == 3 ? 10 : 6));
    return FG_OK;
}
}  // namespace

extern "C" const char *fg_last_error(void) { return g_err.c_str(); }

// ------------------------------------------------------------------------------------------------ kernel timing
namespace {
bool g_timing = false;
int g_timing_dev = -1;
cudaEvent_t g_ev0 = nullptr, g_ev1 = nullptr;
bool g_recorded = false;
}  // namespace

void fg::timer_begin(cudaStream_t st)
{
    if (!g_timing) return;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != g_timing_dev) {
        if (g_ev0) { cudaEventDestroy(g_ev0); cudaEventDestroy(g_ev1); }
        cudaEventCreate(&g_ev0);
        cudaEventCreate(&g_ev1);
        g_timing_dev = dev;
    }
    cudaEventRecord(g_ev0, st);
}

void fg::timer_end(cudaStream_t st)
{
    if (!g_timing || !g_ev1) return;
    cudaEventRecord(g_ev1, st);
    g_recorded = true;
}

extern "C" fg_status fg_set_kernel_timing(int32_t enable)
{
    g_timing = enable != 0;
    return FG_OK;
}

extern "C" fg_status fg_kernel_time_ms(float *ms)
{
    if (!ms) return fail(FG_ERR_VALUE, "null argument");
    if (!g_recorded) return fail(FG_ERR_VALUE, "no timed kernel yet (enable fg_set_kernel_timing first)");
    FG_CUDA(cudaEventSynchronize(g_ev1));
    FG_CUDA(cudaEventElapsedTime(ms, g_ev0, g_ev1));
    return FG_OK;
}

extern "C" fg_status fg_set_launch(int32_t fwd_warps, int32_t bwd_warps)
{
    if (fwd_warps < 0 || fwd_warps > 8 || bwd_warps < 0 || bwd_warps > 8) return fail(FG_ERR_VALUE, "warps must be 0..8");
    g_fwd_warps = fwd_warps ? fwd_warps : 4;
    g_bwd_warps = bwd_warps ? bwd_warps : 4;
    return FG_OK;
}

extern "C" fg_status fg_stage_set_launch(fg_stage *s, int32_t fwd_warps, int32_t bwd_warps)
{
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (fwd_warps < 0 || fwd_warps > 8 || bwd_warps < 0 || bwd_warps > 8) return fail(FG_ERR_VALUE, "warps must be 0..8");
    s->fwd_warps = fwd_warps;
    s->bwd_warps = bwd_warps;
    return FG_OK;
}

extern "C" fg_status fg_stage_set_fused_variant(fg_stage *s, int32_t regs_alt, int32_t stage_t)
{
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if ((regs_alt != 0 && regs_alt != 1) || (stage_t != 0 && stage_t != 1))
        return fail(FG_ERR_VALUE, "regs_alt and stage_t must be 0 or 1");
    s->fused_regs_alt = regs_alt;
    s->fused_stage_t = stage_t;
    return FG_OK;
}

extern "C" fg_status fg_stage_create(const fg_phase_desc *d, int device, fg_stage **out)
{
    g_err.clear();
    if (!d || !out) return fail(FG_ERR_VALUE, "null argument");
    *out = nullptr;
    if (d->nsp != 1) return fail(FG_ERR_NOT_IMPLEMENTED, "spin-dependent phase files are not ported");
    if (d->iorder >= 10) return fail(FG_ERR_NOT_IMPLEMENTED, "icalc >= 10 not ported");
    if (d->iorder < 0 || d->iorder > 3)
        return fail(FG_ERR_VALUE, "iorder " + std::to_string(d->iorder) +
                                      ": the lambda set exceeds the rotation tables (|m| <= 3)");
    if (d->ne1 < 2 || d->nph < 0 || d->ltot < 0 || !d->lmax0 || !d->em || !d->eref || !d->ph || !d->rkk)
        return fail(FG_ERR_VALUE, "incomplete phase description");
    fg_stage *s = new fg_stage();
    s->device = device;
    s->E = d->ne1; s->nph = d->nph; s->nph1 = d->nph + 1; s->ltot = d->ltot; s->ihole = d->ihole; s->iorder = d->iorder;
    int linit = 0;
    if (!hole_kappa(d->ihole, s->kinit, linit)) { delete s; return fail(FG_ERR_VALUE, "invalid hole number"); }
    s->ilinit = linit + 1;
    if (s->ilinit > 3) {
        delete s;
        return fail(FG_ERR_NOT_IMPLEMENTED, "initial states with l > 2 need |m| > 3 rotation matrices (not built)");
    }
    const int E = s->E, nph1 = s->nph1, nl = 2 * d->ltot + 1;
    auto ph = [&](int ie, int l, int ip) {
        const double *p = d->ph + 2 * (((size_t)ie * nl + (l + d->ltot)) * nph1 + ip);
        return cd(p[0], p[1]);
    };
    // lmax (pad.py:93-106)
    s->lmax_host.assign((size_t)E * nph1, 0);
    int lmx = 0;
    for (int ip = 0; ip < nph1; ++ip) {
        if (d->lmax0[ip] > d->ltot || d->lmax0[ip] < 0) { delete s; return fail(FG_ERR_VALUE, "lmax0 exceeds ltot"); }
        for (int ie = 0; ie < E; ++ie) {
            int lm = 0;
            for (int l = d->lmax0[ip]; l >= 0; --l) {
                lm = l;
                if (std::abs(std::sin(ph(ie, l, ip))) > 1.0e-7) break;
            }
            s->lmax_host[(size_t)ie * nph1 + ip] = lm;
            lmx = std::max(lmx, lm);
        }
    }
    s->L1 = lmx + 1;
    const int L1 = s->L1;
    // xk, ck (pad.py:111-121)
    s->xk_host.resize(E);
    std::vector<cd> ck(E), dk(E);
    for (int ie = 0; ie < E; ++ie) {
        const double e = d->em[2 * ie] - d->edge;
        s->xk_host[ie] = (e > 0 ? 1.0 : (e < 0 ? -1.0 : 0.0)) * std::sqrt(std::fabs(2 * e));
        ck[ie] = std::sqrt(2.0 * (cd(d->em[2 * ie], d->em[2 * ie + 1]) - cd(d->eref[2 * ie], d->eref[2 * ie + 1])));
        dk[ie] = ck[ie] - s->xk_host[ie];
    }
    // j-averaged t-matrix (stage.py:111-118), layout (ip, il, e)
    std::vector<cd> tl((size_t)nph1 * (L1 + 1) * E);
    const cd twoi(0.0, 2.0);
    for (int ip = 0; ip < nph1; ++ip)
        for (int il = 1; il <= L1; ++il)
            for (int ie = 0; ie < E; ++ie) {
                const int ll = il - 1;
                const cd tm = (std::exp(twoi * ph(ie, -ll, ip)) - 1.0) / twoi;
                const cd tp = (std::exp(twoi * ph(ie, ll, ip)) - 1.0) / twoi;
                tl[((size_t)ip * (L1 + 1) + il) * E + ie] = tm * double(ll + 1) + tp * double(ll);
            }
    // final-state terms (bcoef + mmtr: bmati is diagonal in k, so terms group by the channel's l)
    int lind[9];
    double bdiag[9];
    final_state(s->kinit, lind, bdiag);
    std::vector<cd> wt;
    for (int k = 1; k <= 8; ++k) {
        if (lind[k] < 0) continue;
        int t = 0;
        while (t < s->nterm && s->term_l[t] != lind[k]) ++t;
        if (t == s->nterm) {
            s->term_l[s->nterm++] = lind[k];
            wt.resize((size_t)s->nterm * E, cd(0, 0));
        }
        for (int ie = 0; ie < E; ++ie) {
            const cd r(d->rkk[2 * (ie * 8 + k - 1)], d->rkk[2 * (ie * 8 + k - 1) + 1]);
            wt[(size_t)t * E + ie] += bdiag[k] * r * r;
        }
    }
    // the kernels unroll the termination's partial waves up to il = l_init + 2 (LamTab::IT) and its terms up to one
    // from an s level, two otherwise (LamTab::NT)
    bool terms_ok = s->nterm <= (s->ilinit == 1 ? 1 : 2);
    for (int t = 0; t < s->nterm; ++t) terms_ok = terms_ok && s->term_l[t] + 1 <= s->ilinit + 1;
    if (!terms_ok) {
        delete s;
        return fail(FG_ERR_VALUE, "final-state terms outside l_init +- 1");
    }
    // xnlm, xfac (folded Legendre factors), recursion coefficients of d^l
    const int XR = std::max(L1 + 2, 6);
    std::vector<double> xn((size_t)XR * 8, 0.0), xfac((size_t)XR * 49, 0.0), rc((size_t)(L1 + 1) * 49 * 3, 0.0);
    for (int il = 1; il < XR; ++il)
        for (int im = 1; im <= std::min(il, 5); ++im) xn[il * 8 + im] = xnlm_of(il, im);
    for (int il = 1; il < XR; ++il)
        for (int m1 = -3; m1 <= 3; ++m1)
            for (int m2 = -3; m2 <= 3; ++m2) {
                const int a1 = std::abs(m1), a2 = std::abs(m2);
                if (a1 >= il || a2 >= il) continue;
                const double x1 = xnlm_of(il, a1 + 1), x2 = xnlm_of(il, a2 + 1);
                xfac[(size_t)il * 49 + (m1 + 3) * 7 + m2 + 3] = (a1 & 1 ? -x1 : x1) / x2;
            }
    for (int lm = 1; lm <= L1; ++lm)
        for (int m = -3; m <= 3; ++m)
            for (int n = -3; n <= 3; ++n) {
                const double l = lm;
                const double p = ((l + 1) * (l + 1) - m * m) * ((l + 1) * (l + 1) - n * n);
                double den = l * std::sqrt(std::max(p, 0.0));
                if (den == 0.0) den = 1.0;
                const double a1 = l * l - m * m, a2 = l * l - n * n;
                double *q = &rc[(((size_t)lm * 7 + m + 3) * 7 + n + 3) * 3];
                q[0] = (2 * l + 1) * l * (l + 1) / den;
                q[1] = (2 * l + 1) * m * n / den;
                q[2] = (l + 1) * std::sqrt(std::max(a1, 0.0) * std::max(a2, 0.0)) / den;
            }
    // then the seed coefficients of Wigner's explicit sum for l <= 3 (wigner_small), [l][m + 3][n + 3][k]: the
    // same IEEE operations (a correctly rounded square root and division of exact factorial products) as the sum
    // formed them term by term on the device
    {
        const size_t seed0 = (size_t)(L1 + 1) * 49 * 3;
        rc.resize(seed0 + (size_t)4 * 49 * 8, 0.0);
        const double fct[8] = {1, 1, 2, 6, 24, 120, 720, 5040};
        for (int l = 0; l <= 3; ++l)
            for (int m = -l; m <= l; ++m)
                for (int n = -l; n <= l; ++n) {
                    const double pref = std::sqrt(fct[l + m] * fct[l - m] * fct[l + n] * fct[l - n]);
                    for (int k = 0; k <= 2 * l; ++k) {
                        const int a = l + n - k, b = k, c = m - n + k, d = l - m - k;
                        if (a < 0 || b < 0 || c < 0 || d < 0) continue;
                        double term = pref / (fct[a] * fct[b] * fct[c] * fct[d]);
                        if ((m - n + k) & 1) term = -term;
                        rc[seed0 + (((size_t)l * 7 + m + 3) * 7 + n + 3) * 8 + k] = term;
                    }
                }
    }
    // lmax on the device as (ip, e)
    std::vector<int> lmax_t((size_t)nph1 * E);
    for (int ip = 0; ip < nph1; ++ip)
        for (int ie = 0; ie < E; ++ie) lmax_t[(size_t)ip * E + ie] = s->lmax_host[(size_t)ie * nph1 + ip];

    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) { delete s; return fail(FG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce)); }
    cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&s->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    fg_status st = build_tables<float>(s, s->tf, tl, ck, dk, wt, xfac, xn, rc, lmax_t);
    if (!st) st = build_tables<double>(s, s->td, tl, ck, dk, wt, xfac, xn, rc, lmax_t);
    if (st) { fg_stage_destroy(s); return st; }
    *out = s;
    return FG_OK;
}

extern "C" void fg_stage_destroy(fg_stage *s)
{
    if (!s) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (void *p : s->bufs) cudaFree(p);
    cudaSetDevice(prev);
    delete s;
}

extern "C" fg_status fg_stage_get_info(const fg_stage *s, fg_stage_info *info)
{
    if (!s || !info) return fail(FG_ERR_VALUE, "null argument");
    info->E = s->E; info->L1 = s->L1; info->nph = s->nph; info->kinit = s->kinit; info->ilinit = s->ilinit;
    const LamTab ss = lamtab(s->ilinit + 1), ms = lamtab(s->ilinit == 1 ? 0 : 1);
    info->lamx_ss = ss.N; info->laml0x_ss = ss.N0; info->lamx_ms = ms.N; info->laml0x_ms = ms.N0;
    info->device = s->device;
    return FG_OK;
}

extern "C" fg_status fg_stage_lmax(const fg_stage *s, int32_t *out)
{
    if (!s || !out) return fail(FG_ERR_VALUE, "null argument");
    std::copy(s->lmax_host.begin(), s->lmax_host.end(), out);
    return FG_OK;
}

extern "C" fg_status fg_stage_xk(const fg_stage *s, double *out)
{
    if (!s || !out) return fail(FG_ERR_VALUE, "null argument");
    std::copy(s->xk_host.begin(), s->xk_host.end(), out);
    return FG_OK;
}


// ================================================================================================ dispatch
namespace {

fg_status set_device(const fg_stage *s)
{
    FG_CUDA(cudaSetDevice(s->device));
    return FG_OK;
}

int fwd_warps(const fg_stage *s) { return s->fwd_warps ? s->fwd_warps : g_fwd_warps; }
int bwd_warps(const fg_stage *s) { return s->bwd_warps ? s->bwd_warps : g_bwd_warps; }
FusedShape fused_shape(const fg_stage *s)
{
    FusedShape f;
    f.warps = fwd_warps(s);
    f.regs_alt = s->fused_regs_alt != 0;
    f.stage_t = s->fused_stage_t != 0;
    return f;
}

StageView view(const fg_stage *s) { return StageView{s->E, s->L1, s->nph1, s->num_sms, s->ilinit, s->max_smem}; }

// Calls F::template run<R, EDGE>(tables) for the stage's precision and initial-state class.
// The kernels of the stage's edge class (l_init + 1) and lambda order (EDGE + 3 at order 3)
template <class F> fg_status by_kind(const fg_stage *s, fg_precision prec, F &&f)
{
    const int edge = (s->ilinit < 1 ? 1 : (s->ilinit > 3 ? 3 : s->ilinit)) + (s->iorder == 3 ? 3 : 0);
    if (prec == FG_FP64) {
        switch (edge) {
        case 1: return f(Launch<double, 1>{}, s->td);
        case 2: return f(Launch<double, 2>{}, s->td);
        case 3: return f(Launch<double, 3>{}, s->td);
        case 4: return f(Launch<double, 4>{}, s->td);
        case 5: return f(Launch<double, 5>{}, s->td);
        default: return f(Launch<double, 6>{}, s->td);
        }
    }
    if (prec != FG_MIXED) return fail(FG_ERR_VALUE, "precision must be FG_MIXED or FG_FP64");
    switch (edge) {
    case 1: return f(Launch<float, 1>{}, s->tf);
    case 2: return f(Launch<float, 2>{}, s->tf);
    case 3: return f(Launch<float, 3>{}, s->tf);
    case 4: return f(Launch<float, 4>{}, s->tf);
    case 5: return f(Launch<float, 5>{}, s->tf);
    default: return f(Launch<float, 6>{}, s->tf);
    }
}

// Host-side checks of a batch's sizes and pointers; k_validate checks the contents (indices) on the device and
// reports through the call's status word.
fg_status check_paths(const fg_paths *P)
{
    if (!P) return fail(FG_ERR_VALUE, "null paths");
    if (P->n < 0 || P->nrows < 0) return fail(FG_ERR_VALUE, "negative size");
    if (P->nleg_max < 2 || P->nleg_max > kMaxLeg) return fail(FG_ERR_VALUE, "nleg_max must be 2..9");
    if (P->n > 0 && (!P->coords || !P->ipots || !P->nleg || !P->deg || !P->order || !P->row))
        return fail(FG_ERR_VALUE, "null array in paths");
    if (P->n > 0 && P->nrows == 0) return fail(FG_ERR_VALUE, "paths but no rows");
    if (P->n > 0x7fffffff) return fail(FG_ERR_VALUE, "at most 2^31-1 paths per call");
    return FG_OK;
}

}  // namespace

extern "C" fg_status fg_cchi(const fg_stage *s, fg_precision prec, int64_t B, int32_t nleg, const void *coords,
                             int32_t coords_f64, const int64_t *ipots, void *cchi, void *reff, int32_t *bad_ipot,
                             void *stream)
{
    g_err.clear();
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (nleg < 2 || nleg > kMaxLeg) return fail(FG_ERR_VALUE, "nleg must be 2..9");
    if (B < 0) return fail(FG_ERR_VALUE, "negative batch");
    if (B == 0) return FG_OK;
    if (!coords || !ipots || !cchi || !reff) return fail(FG_ERR_VALUE, "null array");
    if (fg_status rc = set_device(s)) return rc;
    const StageView sv = view(s);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return by_kind(s, prec, [&](auto L, const auto &T) {
        return decltype(L)::cchi(sv, T, B, nleg, coords, coords_f64, ipots, cchi, reff, bad_ipot, fwd_warps(s), st);
    });
}

extern "C" size_t fg_cchi_backward_workspace(const fg_stage *s, int64_t B, int32_t nleg)
{
    if (!s || B < 0 || nleg < 2 || nleg > kMaxLeg) return 0;
    return cchi_bwd_workspace(B, nleg);
}

extern "C" fg_status fg_cchi_backward(const fg_stage *s, fg_precision prec, int64_t B, int32_t nleg,
                                      const void *coords, int32_t coords_f64, const int64_t *ipots,
                                      const void *grad_cchi, const void *grad_reff, void *grad_coords,
                                      void *workspace, size_t workspace_bytes, void *stream)
{
    g_err.clear();
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (nleg < 2 || nleg > kMaxLeg) return fail(FG_ERR_VALUE, "nleg must be 2..9");
    if (B < 0) return fail(FG_ERR_VALUE, "negative batch");
    if (B == 0) return FG_OK;
    if (!coords || !ipots || !grad_cchi || !grad_coords) return fail(FG_ERR_VALUE, "null array");
    const size_t need = cchi_bwd_workspace(B, nleg);
    if (need && (!workspace || workspace_bytes < need))
        return fail(FG_ERR_WORKSPACE, "workspace needs " + std::to_string(need) + " bytes");
    if (fg_status rc = set_device(s)) return rc;
    const StageView sv = view(s);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return by_kind(s, prec, [&](auto L, const auto &T) {
        return decltype(L)::cchi_bwd(sv, T, B, nleg, coords, coords_f64, ipots, grad_cchi, grad_reff, grad_coords,
                                     static_cast<unsigned char *>(workspace), bwd_warps(s), st);
    });
}

extern "C" fg_status fg_chi_fine(const fg_stage *s, fg_precision prec, int64_t B, const void *cchi, const void *reff,
                                 int32_t NK, const void *q, const void *S, const int32_t *span, void *chi, void *stream)
{
    g_err.clear();
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (B < 0 || NK < 0) return fail(FG_ERR_VALUE, "negative size");
    if (B == 0 || NK == 0) return FG_OK;
    if (!cchi || !reff || !q || !S || !span || !chi) return fail(FG_ERR_VALUE, "null array");
    if (fg_status rc = set_device(s)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (prec == FG_FP64) return LaunchCommon<double>::chi_fine(view(s), B, cchi, reff, NK, q, S, span, chi, st);
    if (prec != FG_MIXED) return fail(FG_ERR_VALUE, "precision must be FG_MIXED or FG_FP64");
    return LaunchCommon<float>::chi_fine(view(s), B, cchi, reff, NK, q, S, span, chi, st);
}

extern "C" fg_status fg_chi_fine_backward(const fg_stage *s, fg_precision prec, int64_t B, const void *cchi,
                                          const void *reff, int32_t NK, const void *q, const void *S,
                                          const int32_t *span, const int32_t *tspan, const void *grad_chi,
                                          void *grad_cchi, void *grad_reff, void *stream)
{
    g_err.clear();
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (B < 0 || NK < 0) return fail(FG_ERR_VALUE, "negative size");
    if (B == 0) return FG_OK;
    if (!cchi || !reff || !q || !S || !span || !tspan || !grad_chi || !grad_cchi || !grad_reff)
        return fail(FG_ERR_VALUE, "null array");
    if (fg_status rc = set_device(s)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (prec == FG_FP64)
        return LaunchCommon<double>::chi_fine_bwd(view(s), B, cchi, reff, NK, q, S, span, tspan, grad_chi, grad_cchi,
                                                  grad_reff, st);
    if (prec != FG_MIXED) return fail(FG_ERR_VALUE, "precision must be FG_MIXED or FG_FP64");
    return LaunchCommon<float>::chi_fine_bwd(view(s), B, cchi, reff, NK, q, S, span, tspan, grad_chi, grad_cchi,
                                             grad_reff, st);
}

extern "C" size_t fg_chi_reduce_workspace(const fg_stage *s, const fg_paths *P, int32_t NK)
{
    if (!s || !P || NK < 0) return 0;
    return fused_workspace(P, NK);
}

extern "C" fg_status fg_chi_reduce(const fg_stage *s, fg_precision prec, const fg_paths *P, int32_t NK,
                                   const double *q, const double *S, const int32_t *span, double *rows,
                                   void *cchi_save, double *reff_save, void *workspace, size_t workspace_bytes,
                                   void *stream)
{
    g_err.clear();
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (fg_status rc = check_paths(P)) return rc;
    if (NK < 0) return fail(FG_ERR_VALUE, "negative NK");
    if (NK == 0 || P->nrows == 0) return FG_OK;
    if (!q || !S || !span || !rows) return fail(FG_ERR_VALUE, "null array");
    const size_t need = fused_workspace(P, NK);
    if (!workspace || workspace_bytes < need)
        return fail(FG_ERR_WORKSPACE, "workspace needs " + std::to_string(need) + " bytes");
    if (fg_status rc = set_device(s)) return rc;
    const StageView sv = view(s);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (fg_status rc = by_kind(s, prec, [&](auto L, const auto &T) {
            return decltype(L)::fused(sv, T, P, NK, q, S, span, rows, cchi_save, reff_save,
                                      static_cast<unsigned char *>(workspace), fused_shape(s), st);
        }))
        return rc;
    return read_status(reinterpret_cast<const int *>(static_cast<unsigned char *>(workspace) + kStatusOffset), st);
}

extern "C" fg_status fg_chi_reduce_words(const fg_stage *s, fg_precision prec, const fg_paths *P, int32_t NK,
                                         const double *q, const double *S, const int32_t *span, uint64_t *words,
                                         void *cchi_save, double *reff_save, void *workspace, size_t workspace_bytes,
                                         void *stream)
{
    g_err.clear();
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (fg_status rc = check_paths(P)) return rc;
    if (NK < 0) return fail(FG_ERR_VALUE, "negative NK");
    if (NK == 0 || P->nrows == 0) return FG_OK;
    if (!q || !S || !span || !words) return fail(FG_ERR_VALUE, "null array");
    if (!workspace || workspace_bytes < kCounterBytes)
        return fail(FG_ERR_WORKSPACE, "workspace needs " + std::to_string(kCounterBytes) + " bytes");
    if (fg_status rc = set_device(s)) return rc;
    const StageView sv = view(s);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (fg_status rc = by_kind(s, prec, [&](auto L, const auto &T) {
            return decltype(L)::fused(sv, T, P, NK, q, S, span, nullptr, cchi_save, reff_save,
                                      static_cast<unsigned char *>(workspace), fused_shape(s), st,
                                      reinterpret_cast<unsigned long long *>(words));
        }))
        return rc;
    return read_status(reinterpret_cast<const int *>(static_cast<unsigned char *>(workspace) + kStatusOffset), st);
}

extern "C" fg_status fg_rows_from_words(int64_t nrows, int32_t NK, const uint64_t *words, double *rows, void *stream)
{
    if (nrows < 0 || NK < 0) return fail(FG_ERR_VALUE, "bad size");
    if (nrows == 0 || NK == 0) return FG_OK;
    if (!words || !rows) return fail(FG_ERR_VALUE, "null array");
    return launch_row_finish(nrows, NK, reinterpret_cast<const unsigned long long *>(words), rows, nullptr,
                             static_cast<cudaStream_t>(stream));
}

extern "C" size_t fg_chi_reduce_backward_workspace(const fg_stage *s, const fg_paths *P, int32_t NK)
{
    if (!s || !P || NK < 0) return 0;
    return fused_bwd_workspace(P, NK, s->E);
}

extern "C" fg_status fg_chi_reduce_backward(const fg_stage *s, fg_precision prec, const fg_paths *P, int32_t NK,
                                            const double *q, const double *S, const int32_t *span,
                                            const int32_t *tspan, const double *grad_rows, const void *cchi_saved,
                                            const double *reff_saved, double *grad_coords, double *grad_sigma2,
                                            void *workspace, size_t workspace_bytes, void *stream)
{
    g_err.clear();
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (fg_status rc = check_paths(P)) return rc;
    if (NK < 0) return fail(FG_ERR_VALUE, "negative NK");
    if (P->n == 0) return FG_OK;
    if (!q || !S || !span || !tspan || !grad_rows || !cchi_saved || !reff_saved || !grad_coords)
        return fail(FG_ERR_VALUE, "null array");
    const size_t need = fused_bwd_workspace(P, NK, s->E);
    if (need && (!workspace || workspace_bytes < need))
        return fail(FG_ERR_WORKSPACE, "workspace needs " + std::to_string(need) + " bytes");
    if (fg_status rc = set_device(s)) return rc;
    const StageView sv = view(s);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (fg_status rc = by_kind(s, prec, [&](auto L, const auto &T) {
            return decltype(L)::fused_bwd(sv, T, P, NK, q, S, span, tspan, grad_rows, cchi_saved, reff_saved,
                                          grad_coords, grad_sigma2, static_cast<unsigned char *>(workspace),
                                          bwd_warps(s), st);
        }))
        return rc;
    return read_status(reinterpret_cast<const int *>(static_cast<unsigned char *>(workspace) + kStatusOffset), st);
}

// ------------------------------------------------------------------------------------------------ no-allocation variant
// The scratch of fg_chi_reduce_noalloc: a fixed array in the library's device image (one per GPU that loads it).
// In host code the name is only a host-side stand-in; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[FG_NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of g_noalloc_scratch in the context of stage s, whose device must be current: looked up once per
// stage (a stage belongs to one device and one context; a device reset invalidates the stage with its tables, so a
// stage created after a reset looks the address up again).
fg_status noalloc_scratch(fg_stage *s, void **out)
{
    std::lock_guard<std::mutex> lock(s->noalloc_mu);
    if (!s->noalloc_scratch) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(FG_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        s->noalloc_scratch = p;
    }
    *out = s->noalloc_scratch;
    return FG_OK;
}
}  // namespace

extern "C" fg_status fg_chi_reduce_noalloc(const fg_stage *s, fg_precision prec, const fg_paths *P, int32_t NK,
                                           const double *q, const double *S, const int32_t *span, double *rows,
                                           void *stream)
{
    g_err.clear();
    if (!s) return fail(FG_ERR_VALUE, "null stage");
    if (fg_status rc = check_paths(P)) return rc;
    if (NK < 0) return fail(FG_ERR_VALUE, "negative NK");
    if (NK == 0 || P->nrows == 0) return FG_OK;
    if (!q || !S || !span || !rows) return fail(FG_ERR_VALUE, "null array");
    const size_t need = fused_workspace(P, NK);
    if (need > FG_NOALLOC_SCRATCH_BYTES)
        return fail(FG_ERR_VALUE, "fg_chi_reduce_noalloc: this batch needs " + std::to_string(need) +
                                      " bytes of scratch, the library's fixed scratch holds " +
                                      std::to_string((size_t)FG_NOALLOC_SCRATCH_BYTES) + " bytes; split it by rows");
    if (fg_status rc = set_device(s)) return rc;
    void *ws = nullptr;
    if (fg_status rc = noalloc_scratch(const_cast<fg_stage *>(s), &ws)) return rc;
    const StageView sv = view(s);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (fg_status rc = by_kind(s, prec, [&](auto L, const auto &T) {
            return decltype(L)::fused(sv, T, P, NK, q, S, span, rows, nullptr, nullptr,
                                      static_cast<unsigned char *>(ws), fused_shape(s), st);
        }))
        return rc;
    return read_status(reinterpret_cast<const int *>(static_cast<unsigned char *>(ws) + kStatusOffset), st);
}
