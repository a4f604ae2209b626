// fg_adjoint.cuh -- the hand-written adjoint of the path stage (reverse mode, recomputing the per-leg matrices).
//
// Per path (one warp) and energy (one lane), with the upstream gradient gbar = dL/dRe(cchi) + i dL/dIm(cchi):
//   dL = Re(conj(gbar) dcchi),  cchi = ptrac cfac,  ptrac = Tr(T F_nsc ... F_1).
// Multiple scattering: sweep 1 forms every F~_k (the forward's partial-wave loop) and stores F~_k and the prefix
// products P_k = F_k ... F_1 P_0 in per-lane local memory; the termination is differentiated with P_nsc and gives the
// start of the suffix R_nsc = [T 0]; sweep 2 runs k = nsc .. 1: the orbit weights Wh (dL/dF~_k folded over the flip
// symmetry) from M_k = P_(k-1) R_k, the Euler-angle derivative d/deta_(k+1) = -i sum_a m_a (P_k R_k)(a, a), the
// update R_(k-1) = R_k F_k, and one partial-wave loop that contracts the derivatives of F~_k against Wh:
//   d/drho_(k+1), d/drho_k  from the spherical-wave factors themselves (dc_j/drho = -i z ((j - 1) c_j + j c_(j+1))),
//   d/dbeta_k               through d'(beta) (a second rotation table).
// Single scattering differentiates its one matrix the same way, with tangent recursions of the spherical waves.
// The termination's parameters (rho_1, rho_nleg, beta_nleg, eta_1) are differentiated with P_nsc, and cfac gives
// d/dri_j = cfac (i (ck - xk) - 1/ri_j).  The per-energy gradients of (ri, beta, eta) are summed over the energies
// (lane accumulators, then a fixed-order warp reduction) and carried to the coordinates by forward-mode dual numbers
// through the geometry (one coordinate direction per lane), with the reference's branch choices
// (stage.py:148-206 under torch autograd).
#pragma once
#include <type_traits>

#include "fg_kernels.cuh"

namespace fg {

// ------------------------------------------------------------------------------------------------ setup
// Rotation tables D^(k) and their derivatives d/dbeta D^(k) for k = 1..nsc (one recursion for both; path_setup
// then skips its own pass) and the termination's d/dbeta d^{l_t}(beta_nleg).
template <typename R>
__device__ void adj_setup(const WarpPath<R> &g, R *dh, R *dhd, R (*dterm_db)[49], const Tables<R> &T, int nleg,
                          int lane, int MM)
{
    const int nsc = nleg - 1;
    const int NC = ncanon(MM), DS = dstride(MM), L1 = T.L1;
    for (int task = lane; task < nsc * NC; task += 32) {
        const int k = task / NC + 1, r = task % NC;
        int m1, m2;
        canon_mn(MM, r, m1, m2);
        const double b = g.beta[k];
        const double c = cos(b), s = sin(b), c2 = cos(0.5 * b), s2 = sin(0.5 * b);
        const size_t o = (size_t)(k - 1) * (L1 + 1) * DS + r;
        R *out = dh + o, *outd = dhd + o;
        const double *xf = T.xfac + (m1 + 3) * 7 + (m2 + 3);
        double dm1 = 0.0, d0 = 0.0, em1 = 0.0, e0 = 0.0;   // d and d/dbeta at l-2, l-1
        const int lseed = min(L1, 4);
        for (int l = 0; l < lseed; ++l) {             // l <= 3: Wigner's explicit sum
            const double dl = wigner_small(l, m1, m2, c2, s2, seed_table(T));
            const double el = wigner_small_dbeta(l, m1, m2, c2, s2, seed_table(T));
            const double x = xf[(size_t)(l + 1) * 49];
            out[(size_t)(l + 1) * DS] = (R)(dl * x);
            outd[(size_t)(l + 1) * DS] = (R)(el * x);
            dm1 = d0; d0 = dl;
            em1 = e0; e0 = el;
        }
        // the three-term recursion, unrolled so that the coefficient loads issue ahead of the dependent steps
#pragma unroll 4
        for (int l = lseed; l < L1; ++l) {
            const double *q = T.rc + (((size_t)(l - 1) * 7 + (m1 + 3)) * 7 + (m2 + 3)) * 3;
            const double f = fma(q[0], c, -q[1]);
            const double dl = fma(f, d0, -q[2] * dm1);
            const double el = fma(f, e0, fma(-q[0] * s, d0, -q[2] * em1));
            const double x = xf[(size_t)(l + 1) * 49];
            out[(size_t)(l + 1) * DS] = (R)(dl * x);
            outd[(size_t)(l + 1) * DS] = (R)(el * x);
            dm1 = d0; d0 = dl;
            em1 = e0; e0 = el;
        }
    }
    for (int task = lane; task < T.nterm * 49; task += 32) {
        const int t = task / 49, m1 = (task % 49) / 7 - 3, m2 = task % 7 - 3;
        const double b = g.beta[nleg];
        dterm_db[t][task % 49] = (R)wigner_small_dbeta(T.term_l[t], m1, m2, cos(0.5 * b), sin(0.5 * b),
                                                        seed_table(T));
    }
}

// ------------------------------------------------------------------------------------------------ termination
// c[il][im] and dc/drho of one leg for il <= ITM with the truncation of GPUPathStage._clm (see clm_small)
template <typename R, int ITM, int NCOL>
__device__ __forceinline__ void clm_small_t(C2<R> z, int lxp1, C2<R> (&c)[ITM + 1][NCOL + 1],
                                            C2<R> (&dc)[ITM + 1][NCOL + 1])
{
    const C2<R> dz = cmul(C2<R>{R(0), R(-1)}, cmul(z, z));   // dz/drho = -i z^2
    C2<R> pv[NCOL + 1], cv[NCOL + 1], dpv[NCOL + 1], dcv[NCOL + 1];
#pragma unroll
    for (int j = 0; j <= NCOL; ++j) {
        pv[j] = cv[j] = dpv[j] = dcv[j] = cz<R>();
        c[0][j] = dc[0][j] = cz<R>();
    }
    pv[1] = cv[1] = C2<R>{R(1), R(0)};
#pragma unroll
    for (int il = 1; il <= ITM; ++il) {
#pragma unroll
        for (int j = 0; j <= NCOL; ++j) {
            const bool keep = (il <= lxp1) || (j == 1 && il <= 2);
            c[il][j] = keep ? cv[j] : cz<R>();
            dc[il][j] = keep ? dcv[j] : cz<R>();
        }
        const R w = R(2 * il - 1);
        const C2<R> wz = cscl(z, w), wdz = cscl(dz, w);
        C2<R> nv[NCOL + 1], dnv[NCOL + 1];
        nv[0] = dnv[0] = cz<R>();
#pragma unroll
        for (int j = 1; j <= NCOL; ++j) {
            const C2<R> sv = j > 1 ? cadd(cv[j], cv[j - 1]) : cv[j];
            const C2<R> dsv = j > 1 ? cadd(dcv[j], dcv[j - 1]) : dcv[j];
            nv[j] = cfms(wz, sv, pv[j]);
            dnv[j] = cfms(wdz, sv, cfms(wz, dsv, dpv[j]));
        }
#pragma unroll
        for (int j = 1; j <= NCOL; ++j) {
            pv[j] = cv[j]; cv[j] = nv[j];
            dpv[j] = dcv[j]; dcv[j] = dnv[j];
        }
    }
}

// G1_t (gam of leg 1), G2_t ((2l+1) gamtl of leg nleg) for the final-state entries and their rho-derivatives
template <typename R, int KIND> struct TermLegs {
    static constexpr LamTab L = lamtab(KIND);
    C2<R> G1[2][L.N0], G2[2][L.N0], dG1[2][L.N0], dG2[2][L.N0];
};

template <typename R, int KIND>
__device__ __forceinline__ void term_legs(const WarpPath<R> &g, const Tables<R> &T, int e, int nleg, C2<R> ck,
                                          TermLegs<R, KIND> &tl)
{
    constexpr LamTab L = lamtab(KIND);
    // columns up to |m| + n + 1 of leg 1 (CI) and n + 1 of leg nleg (CO) enter
    constexpr int N0 = L.N0, ITM = L.IT, CI = L.CI, CO = L.CO;
    const int E = T.E;
    const int la = T.lmax[g.ip[0] * E + e], l1 = T.lmax[g.ip[1] * E + e], ln = T.lmax[g.ip[nleg - 1] * E + e];
    C2<R> c1[ITM + 1][CI + 1], cn[ITM + 1][CO + 1], d1[ITM + 1][CI + 1], dn[ITM + 1][CO + 1];
    clm_small_t<R, ITM, CI>(zfac(cscl(ck, (R)g.ri[1])), max(la, l1) + 1, c1, d1);
    clm_small_t<R, ITM, CO>(zfac(cscl(ck, (R)g.ri[nleg])), max(ln, la) + 1, cn, dn);
    for (int t = 0; t < lamtab(KIND).NT && t < T.nterm; ++t) {
        const int il = T.term_l[t] + 1;
#pragma unroll
        for (int i = 0; i < N0; ++i) {
            const int am = L.m[i] < 0 ? -L.m[i] : L.m[i];
            const bool ok = am + 1 <= il;
            const int imn = am + L.n[i] + 1, in = L.n[i] + 1;
            C2<R> a1 = cz<R>(), an = cz<R>(), b1 = cz<R>(), bn = cz<R>();
#pragma unroll
            for (int q = 1; q <= ITM; ++q)
                if (q == il) {
                    a1 = c1[q][imn]; b1 = d1[q][imn];
                    an = cn[q][in]; bn = dn[q][in];
                }
            const R xn = (R)T.xnlm[il * 8 + am + 1];
            const R f1 = (ok && imn <= il) ? ((am & 1) ? -xn : xn) : R(0);
            const R f2 = ok ? (R)(2 * il - 1) / xn : R(0);
            tl.G1[t][i] = cscl(a1, f1); tl.dG1[t][i] = cscl(b1, f1);
            tl.G2[t][i] = cscl(an, f2); tl.dG2[t][i] = cscl(bn, f2);
        }
    }
}

// ------------------------------------------------------------------------------------------------ streaming dF
// Per partial wave: accumulate F~_k (canonical entries) and contract dF_k with the weights Wh (per canonical entry:
// sum over its flip orbit of sign * e^{-i eta m1} * M[b][a]) for the derivatives along rho_in, rho_out, beta_k.
template <typename R, int KIND, int NR, int NC>
__device__ __forceinline__ void accumulate_f_adj(C2<R> (&acc)[RepTab<KIND, NR, NC>().n],
                                                 const C2<R> (&Wh)[RepTab<KIND, NR, NC>().n], const R *dhk,
                                                 const R *dhdk, const C2<R> *tlk, int E, int ilx, C2<R> z_in,
                                                 C2<R> z_out, C2<R> &g_in, C2<R> &g_out, C2<R> &g_beta)
{
    constexpr RepTab<KIND, NR, NC> RT{};
    constexpr LamTab L = lamtab(KIND);
    constexpr int DS = dstride(L.MM);
    constexpr int NCAN = ncanon(L.MM);
    constexpr int CI = L.CI, CO = L.CO;
#pragma unroll
    for (int r = 0; r < RT.n; ++r) acc[r] = cz<R>();
    const C2<R> dz_in = cmul(C2<R>{R(0), R(-1)}, cmul(z_in, z_in));
    const C2<R> dz_out = cmul(C2<R>{R(0), R(-1)}, cmul(z_out, z_out));
    C2<R> pi[CI + 1], ci[CI + 1], po[CO + 1], co[CO + 1];
    C2<R> dpi[CI + 1], dci[CI + 1], dpo[CO + 1], dco[CO + 1];
#pragma unroll
    for (int j = 0; j <= CI; ++j) pi[j] = ci[j] = dpi[j] = dci[j] = cz<R>();
#pragma unroll
    for (int j = 0; j <= CO; ++j) po[j] = co[j] = dpo[j] = dco[j] = cz<R>();
    pi[1] = ci[1] = po[1] = co[1] = C2<R>{R(1), R(0)};
    C2<R> gi = cz<R>(), go = cz<R>(), gb = cz<R>();
    for (int il = 1; il <= ilx; ++il) {
        const C2<R> t = tlk[(size_t)il * E];
        const R *dr = dhk + (size_t)il * DS;
        const R *ddr = dhdk + (size_t)il * DS;
        R d[NCAN], dd[NCAN];
#pragma unroll
        for (int q = 0; q < NCAN; ++q) { d[q] = dr[q]; dd[q] = ddr[q]; }
        C2<R> tco[CO + 1], tdco[CO + 1];
#pragma unroll
        for (int j = 1; j <= CO; ++j) { tco[j] = cmul(t, co[j]); tdco[j] = cmul(t, dco[j]); }
        // X[ci][co] = sum Wh D, Y[ci][co] = sum Wh D'
        C2<R> X[CI + 1][CO + 1], Y[CI + 1][CO + 1];
#pragma unroll
        for (int a = 0; a <= CI; ++a)
#pragma unroll
            for (int b = 0; b <= CO; ++b) X[a][b] = Y[a][b] = cz<R>();
#pragma unroll
        for (int r = 0; r < RT.n; ++r) {
            acc[r] = cfmr(cmul(ci[RT.ci[r]], tco[RT.co[r]]), d[RT.d[r]], acc[r]);
            X[RT.ci[r]][RT.co[r]] = cfmr(Wh[r], d[RT.d[r]], X[RT.ci[r]][RT.co[r]]);
            Y[RT.ci[r]][RT.co[r]] = cfmr(Wh[r], dd[RT.d[r]], Y[RT.ci[r]][RT.co[r]]);
        }
#pragma unroll
        for (int a = 1; a <= CI; ++a) {
            C2<R> v = cz<R>();
#pragma unroll
            for (int b = 1; b <= CO; ++b) {
                v = cfma(X[a][b], tco[b], v);
                gb = cfma(Y[a][b], cmul(ci[a], tco[b]), gb);
            }
            gi = cfma(dci[a], v, gi);
        }
#pragma unroll
        for (int b = 1; b <= CO; ++b) {
            C2<R> v = cz<R>();
#pragma unroll
            for (int a = 1; a <= CI; ++a) v = cfma(X[a][b], ci[a], v);
            go = cfma(tdco[b], v, go);
        }
        // next partial wave, values and rho-tangents
        const R w = R(2 * il - 1);
        const C2<R> wi = cscl(z_in, w), wo = cscl(z_out, w), wdi = cscl(dz_in, w), wdo = cscl(dz_out, w);
        C2<R> ni[CI + 1], no[CO + 1], dni[CI + 1], dno[CO + 1];
#pragma unroll
        for (int j = 1; j <= CI; ++j) {
            const C2<R> sv = j > 1 ? cadd(ci[j], ci[j - 1]) : ci[j];
            const C2<R> dsv = j > 1 ? cadd(dci[j], dci[j - 1]) : dci[j];
            ni[j] = cfms(wi, sv, pi[j]);
            dni[j] = cfms(wdi, sv, cfms(wi, dsv, dpi[j]));
        }
#pragma unroll
        for (int j = 1; j <= CO; ++j) {
            const C2<R> sv = j > 1 ? cadd(co[j], co[j - 1]) : co[j];
            const C2<R> dsv = j > 1 ? cadd(dco[j], dco[j - 1]) : dco[j];
            no[j] = cfms(wo, sv, po[j]);
            dno[j] = cfms(wdo, sv, cfms(wo, dsv, dpo[j]));
        }
#pragma unroll
        for (int j = 1; j <= CI; ++j) { pi[j] = ci[j]; ci[j] = ni[j]; dpi[j] = dci[j]; dci[j] = dni[j]; }
#pragma unroll
        for (int j = 1; j <= CO; ++j) { po[j] = co[j]; co[j] = no[j]; dpo[j] = dco[j]; dco[j] = dno[j]; }
    }
    g_in = gi;
    g_out = go;
    g_beta = gb;
}

// -i z v: the factor of the rho-derivative of the spherical-wave factors
template <typename R> __device__ __forceinline__ C2<R> mi_z(C2<R> z, C2<R> v)
{
    const C2<R> zv = pmul(z, v);
    return C2<R>{zv.y, -zv.x};
}

// The contraction part of accumulate_f_adj alone (F~_k itself is known from the first sweep): per partial wave the
// weighted sums along rho_in, rho_out and beta_k.  The rho-derivatives of the spherical-wave factors come from the
// factors themselves: column j (m = j - 1) of c(z), z = -i / rho, obeys dc_j/drho = -i z ((j - 1) c_j + j c_(j+1))
// (checked against finite differences of the recursion), so one more column of the value recursion replaces the
// tangent recursions and their state (forward + backward of the benchmark batch 262 -> 257 ms on B200).  Every complex
// operation of the loop runs as FP32-pair instructions.  (The single-scattering adjoints below keep the tangent
// recursions: two-leg paths are a small share of any batch.)
template <typename R, int KIND, int NR, int NC>
__device__ __forceinline__ void contract_f_adj(const C2<R> (&Wh)[RepTab<KIND, NR, NC>().n], const R *dhk,
                                                        const R *dhdk, const C2<R> *tlk, int E, int ilx, C2<R> z_in,
                                                        C2<R> z_out, C2<R> &g_in, C2<R> &g_out, C2<R> &g_beta)
{
    constexpr RepTab<KIND, NR, NC> RT{};
    constexpr LamTab L = lamtab(KIND);
    constexpr int DS = dstride(L.MM);
    constexpr int NCAN = ncanon(L.MM);
    constexpr int CI = L.CI, CO = L.CO;
    C2<R> pi[CI + 2], ci[CI + 2], po[CO + 2], co[CO + 2];
#pragma unroll
    for (int j = 0; j <= CI + 1; ++j) pi[j] = ci[j] = cz<R>();
#pragma unroll
    for (int j = 0; j <= CO + 1; ++j) po[j] = co[j] = cz<R>();
    pi[1] = ci[1] = po[1] = co[1] = C2<R>{R(1), R(0)};
    C2<R> gi = cz<R>(), go = cz<R>(), gb = cz<R>();
    C2<R> t1 = tlk[E], t2 = ilx >= 2 ? tlk[(size_t)2 * E] : cz<R>();
    for (int il = 1; il <= ilx; ++il) {
        const C2<R> t = t1;
        t1 = t2;
        if (il + 2 <= ilx) t2 = tlk[(size_t)(il + 2) * E];
        R d[NCAN], dd[NCAN];
        load_row<R, NCAN>(dhk + (size_t)il * DS, d);
        load_row<R, NCAN>(dhdk + (size_t)il * DS, dd);
        C2<R> tco[CO + 1], tdco[CO + 1];
#pragma unroll
        for (int j = 1; j <= CO; ++j) {
            tco[j] = pmul(t, co[j]);
            tdco[j] = pmul(t, mi_z(z_out, pfmr(co[j], R(j - 1), cscl(co[j + 1], R(j)))));
        }
        C2<R> X[CI + 1][CO + 1], Y[CI + 1][CO + 1];
#pragma unroll
        for (int a = 0; a <= CI; ++a)
#pragma unroll
            for (int b = 0; b <= CO; ++b) X[a][b] = Y[a][b] = cz<R>();
#pragma unroll
        for (int r = 0; r < RT.n; ++r) {
            X[RT.ci[r]][RT.co[r]] = pfmr(Wh[r], d[RT.d[r]], X[RT.ci[r]][RT.co[r]]);
            Y[RT.ci[r]][RT.co[r]] = pfmr(Wh[r], dd[RT.d[r]], Y[RT.ci[r]][RT.co[r]]);
        }
#pragma unroll
        for (int a = 1; a <= CI; ++a) {
            C2<R> v = cz<R>(), y = cz<R>();
#pragma unroll
            for (int b = 1; b <= CO; ++b) {
                v = pfma(X[a][b], tco[b], v);
                y = pfma(Y[a][b], tco[b], y);
            }
            gi = pfma(mi_z(z_in, pfmr(ci[a], R(a - 1), cscl(ci[a + 1], R(a)))), v, gi);
            gb = pfma(ci[a], y, gb);
        }
#pragma unroll
        for (int b = 1; b <= CO; ++b) {
            C2<R> v = cz<R>();
#pragma unroll
            for (int a = 1; a <= CI; ++a) v = pfma(X[a][b], ci[a], v);
            go = pfma(tdco[b], v, go);
        }
        const R w = R(2 * il - 1);
        const C2<R> wi = cscl(z_in, w), wo = cscl(z_out, w);
        C2<R> ni[CI + 2], no[CO + 2];
#pragma unroll
        for (int j = 1; j <= CI + 1; ++j) ni[j] = pfms(wi, j > 1 ? padd(ci[j], ci[j - 1]) : ci[j], pi[j]);
#pragma unroll
        for (int j = 1; j <= CO + 1; ++j) no[j] = pfms(wo, j > 1 ? padd(co[j], co[j - 1]) : co[j], po[j]);
#pragma unroll
        for (int j = 1; j <= CI + 1; ++j) { pi[j] = ci[j]; ci[j] = ni[j]; }
#pragma unroll
        for (int j = 1; j <= CO + 1; ++j) { po[j] = co[j]; co[j] = no[j]; }
    }
    g_in = gi;
    g_out = go;
    g_beta = gb;
}

// Weights of the contraction: Wh[r] = sum over the orbit of r of sign * ph(m_a) * M(b, a), and the same with an
// extra -i m_a for the Euler-angle derivative.  M(b, a) is given as a functor.
template <typename R, int KIND, int NR, int NC, int MM, class MF>
__device__ __forceinline__ void orbit_weights(const MF &M, const C2<R> (&ph)[2 * MM + 1],
                                              C2<R> (&Wh)[RepTab<KIND, NR, NC>().n],
                                              C2<R> (&We)[RepTab<KIND, NR, NC>().n])
{
    constexpr RepTab<KIND, NR, NC> RT{};
    constexpr LamTab L = lamtab(KIND);
#pragma unroll
    for (int r = 0; r < RT.n; ++r) Wh[r] = We[r] = cz<R>();
#pragma unroll
    for (int a = 0; a < NR; ++a)
#pragma unroll
        for (int b = 0; b < NC; ++b) {
            const C2<R> v = cmul(ph[L.m[a] + MM], M(b, a));
            const C2<R> sv = RT.sg[a][b] > 0 ? v : cscl(v, R(-1));
            Wh[RT.rep[a][b]] = cadd(Wh[RT.rep[a][b]], sv);
            // -i m_a sv
            We[RT.rep[a][b]] = cadd(We[RT.rep[a][b]], C2<R>{sv.y * R(L.m[a]), -sv.x * R(L.m[a])});
        }
}

// Per-lane gradient accumulators of one path: dL/d(ri_j), dL/d(beta_j), dL/d(eta_j), j = 1..nleg (bohr, rad).
struct ParGrad {
    double ri[kMaxLeg + 1], beta[kMaxLeg + 1], eta[kMaxLeg + 1];
};

// Termination contribution with P (the full chain, N0 x N0): ptrac and the gradients along eta_1, beta_nleg,
// rho_1, rho_nleg (each times s, real part taken by the caller).  Rows a_lo <= a < a_hi only.  With Tm (row
// stride ldt; in local memory) non-null it also receives the termination matrix itself, as term_matrix forms it.
template <typename R, int KIND, class PF>
__device__ __forceinline__ C2<R> term_adj(const WarpPath<R> &g, const R (*dterm_db)[49], const Tables<R> &T, int e,
                                          const TermLegs<R, KIND> &tl, const PF &P, C2<R> &g_eta1, C2<R> &g_betan,
                                          C2<R> &g_rho1, C2<R> &g_rhon, C2<R> *Tm = nullptr, int ldt = 0,
                                          int a_lo = 0, int a_hi = kLamTot)
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N0 = L.N0, MM = L.MM;
    C2<R> ph1[2 * MM + 1];
    phase_powers<R, MM>(g.phs[1], ph1);
    C2<R> ptrac = cz<R>();
    for (int t = 0; t < T.nterm; ++t) {
        const C2<R> W = T.wt[t * T.E + e];
        C2<R> s = cz<R>(), se = cz<R>(), sb = cz<R>(), s1 = cz<R>(), sn = cz<R>();
#pragma unroll
        for (int a = 0; a < N0; ++a) {
            if (a < a_lo || a >= a_hi) continue;
            const C2<R> wf = cmul(W, cmul(ph1[L.m[a] + MM], tl.G1[t][a]));
            C2<R> x = cz<R>(), xb = cz<R>(), xn = cz<R>();
#pragma unroll
            for (int b = 0; b < N0; ++b) {
                const int di = (L.m[a] + 3) * 7 + L.m[b] + 3;
                const C2<R> p = P(b, a);
                const C2<R> gd = cscl(tl.G2[t][b], g.dterm[t][di]);
                x = cfma(gd, p, x);
                xb = cfma(cscl(tl.G2[t][b], dterm_db[t][di]), p, xb);
                xn = cfma(cscl(tl.dG2[t][b], g.dterm[t][di]), p, xn);
                if (Tm) Tm[a * ldt + b] = t == 0 ? cmul(wf, gd) : cfma(wf, gd, Tm[a * ldt + b]);
            }
            const C2<R> f = ph1[L.m[a] + MM];
            const C2<R> v = cmul(cmul(f, tl.G1[t][a]), x);
            s = cadd(s, v);
            se = cadd(se, C2<R>{v.y * R(L.m[a]), -v.x * R(L.m[a])});
            sb = cfma(cmul(f, tl.G1[t][a]), xb, sb);
            s1 = cfma(cmul(f, tl.dG1[t][a]), x, s1);
            sn = cfma(cmul(f, tl.G1[t][a]), xn, sn);
        }
        ptrac = cfma(W, s, ptrac);
        g_eta1 = cfma(W, se, g_eta1);
        g_betan = cfma(W, sb, g_betan);
        g_rho1 = cfma(W, s1, g_rho1);
        g_rhon = cfma(W, sn, g_rhon);
    }
    return ptrac;
}

// Termination matrix rows T[a][b] (a, b < N0), as termination() forms them
template <typename R, int KIND>
__device__ __forceinline__ void term_matrix(const WarpPath<R> &g, const Tables<R> &T, int e,
                                            const TermLegs<R, KIND> &tl, C2<R> (&Tm)[lamtab(KIND).N0][lamtab(KIND).N0])
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N0 = L.N0, MM = L.MM;
    C2<R> ph1[2 * MM + 1];
    phase_powers<R, MM>(g.phs[1], ph1);
#pragma unroll
    for (int a = 0; a < N0; ++a)
#pragma unroll
        for (int b = 0; b < N0; ++b) Tm[a][b] = cz<R>();
    for (int t = 0; t < T.nterm; ++t) {
        const C2<R> W = T.wt[t * T.E + e];
#pragma unroll
        for (int a = 0; a < N0; ++a) {
            const C2<R> f = cmul(W, cmul(ph1[L.m[a] + MM], tl.G1[t][a]));
#pragma unroll
            for (int b = 0; b < N0; ++b)
                Tm[a][b] = cfma(f, cscl(tl.G2[t][b], g.dterm[t][(L.m[a] + 3) * 7 + L.m[b] + 3]), Tm[a][b]);
        }
    }
}

// Adds Re(s * dcfac/dri) = Re(s * cfac... ) terms: dL/dri_j += Re(conj(gbar) cchi (i dk - 1/ri_j)).
template <typename R>
__device__ __forceinline__ void cfac_grad(const WarpPath<R> &g, const Tables<R> &T, int e, int nleg, C2<R> gbar,
                                          C2<R> cchi, ParGrad &pg)
{
    const double2 dk = T.dk[e];
    // conj(gbar) cchi
    const double ax = (double)gbar.x * cchi.x + (double)gbar.y * cchi.y;
    const double ay = (double)gbar.x * cchi.y - (double)gbar.y * cchi.x;
    // times i dk = (-dk.y, dk.x)
    const double re_idk = ax * (-dk.y) - ay * dk.x;
    for (int j = 1; j <= nleg; ++j) pg.ri[j] += re_idk - ax / g.ri[j];
}

// ------------------------------------------------------------------------------------------------ one energy
// Multiple scattering (nleg >= 3).  Adds this energy's parameter gradients into pg.  Every scattering matrix is
// handled as a full lamx x lamx matrix (one code path for the first, middle and last matrices): the first matrix's
// columns beyond laml0x meet the zero rows of P_0 (the lamx x laml0x identity) and the last matrix's rows beyond
// laml0x meet the zero columns of R_nsc = [T 0].  Sweep 1 keeps every F~_k and P_k in per-lane local memory, so that
// sweep 2's partial-wave loop carries only the contraction.  The small matrix products between the partial-wave
// loops run as rolled loops over one index of the local-memory operand: the per-energy code then stays within the
// instruction cache (the unrolled products made the kernel several times larger than its two hot loops); their
// complex multiply-adds are FP32-pair instructions (3 % faster; in the forward's register-resident chain product the
// pairing measured slower and is not used).  Keeping only every second or third prefix and recomputing the others
// from F~_k (1.5-2.3 KB instead of 3.7 KB of local memory per lane) measured 1-3 % slower on B200: the local memory is
// not what bounds this kernel.
//
// MASK: the stage's lambda order is below 2 (T.nlam < N); a separate instantiation, so that the order-2 code carries
// none of the masking (with it inline the order-2 adjoint measured 4 % slower).
template <typename R, int KIND, bool MASK = false>
__device__ void energy_ms_adj(const WarpPath<R> &g, const R *dh, const R *dhd, const R (*dterm_db)[49],
                              const Tables<R> &T, int e, int nleg, C2<R> gbar, ParGrad &pg)
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N = L.N, N0 = L.N0, MM = L.MM, DS = dstride(MM);
    constexpr RepTab<KIND, N, N> RT{};
    const int E = T.E, nsc = nleg - 1;
    const size_t dleg = (size_t)(T.L1 + 1) * DS, tlip = (size_t)(T.L1 + 1) * E;
    const C2<R> ck = T.ck[e];
    if (fabs((double)ck.x) + fabs((double)ck.y) <= 1e-16) return;
    auto add_re = [](double &acc, C2<R> s, C2<R> v) { acc += (double)s.x * v.x - (double)s.y * v.y; };
    const C2<R> cf = cfac(g, T, e, nleg, ck);
    const C2<R> sd = cmul(C2<R>{gbar.x, -gbar.y}, cf);      // s = conj(gbar) cfac: dL = Re(s dptrac)
    const C2<R> sck = cmul(sd, ck);
    // per-lane local memory: F~_k (k = 1..nsc), P_k = F_k ... F_1 P_0 (k = 0..nsc), R_k.  (Measured on B200: loading
    // the next column while the current one is in use, or forming P_0 on the fly instead of storing it, is slower.)
    C2<R> Fst[kMaxLeg - 1][RT.n];
    C2<R> Pst[kMaxLeg][N][N0];
    C2<R> Rst[N0][N];
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
        for (int b = 0; b < N0; ++b) Pst[0][a][b] = a == b ? C2<R>{R(1), R(0)} : cz<R>();
    // sweep 1
    for (int k = 1; k <= nsc; ++k) {
        C2<R> acc[RT.n];
        const int ip = g.ip[k];
        accumulate_f<R, KIND, N, N>(acc, dh + (k - 1) * dleg, T.tl + ip * tlip + e, E, T.lmax[ip * E + e] + 1,
                                    zfac(cscl(ck, (R)g.ri[k + 1])), zfac(cscl(ck, (R)g.ri[k])));
        if constexpr (MASK) mask_lambda<R, KIND, N, N>(acc, T.nlam);
#pragma unroll
        for (int r = 0; r < RT.n; ++r) Fst[k - 1][r] = acc[r];
        C2<R> ph[2 * MM + 1];
        phase_powers<R, MM>(g.phs[k + 1], ph);
        // P_k = e^{-i eta_(k+1) m} F~_k P_(k-1), one column of P at a time
#pragma unroll 1
        for (int b = 0; b < N0; ++b) {
            C2<R> col[N];
#pragma unroll
            for (int c = 0; c < N; ++c) col[c] = Pst[k - 1][c][b];
#pragma unroll
            for (int a = 0; a < N; ++a) {
                C2<R> s = cz<R>();
#pragma unroll
                for (int c = 0; c < N; ++c) {
                    const C2<R> f = acc[RT.rep[a][c]];
                    s = RT.sg[a][c] > 0 ? pfma(f, col[c], s) : pfms(f, col[c], s);
                }
                Pst[k][a][b] = cmul(ph[L.m[a] + MM], s);
            }
        }
    }
    // the termination with P_nsc: its own gradients, ptrac and cfac's gradient
    TermLegs<R, KIND> tl;
    term_legs<R, KIND>(g, T, e, nleg, ck, tl);
    {
        C2<R> ge1 = cz<R>(), gbn = cz<R>(), gr1 = cz<R>(), grn = cz<R>();
        // sweep 2 starts from R_nsc = [T 0] (laml0x x lamx): term_adj writes T into the first columns
#pragma unroll
        for (int a = 0; a < N0; ++a)
#pragma unroll
            for (int b = N0; b < N; ++b) Rst[a][b] = cz<R>();
        const C2<R> ptrac = term_adj<R, KIND>(g, dterm_db, T, e, tl, [&](int b, int a) { return Pst[nsc][b][a]; },
                                              ge1, gbn, gr1, grn, &Rst[0][0], N);
        add_re(pg.eta[1], sd, ge1);
        add_re(pg.beta[nleg], sd, gbn);
        add_re(pg.ri[1], sck, gr1);
        add_re(pg.ri[nleg], sck, grn);
        cfac_grad(g, T, e, nleg, gbar, cmul(ptrac, cf), pg);
    }
    // sweep 2, k = nsc .. 1 with R_k = T F_nsc ... F_(k+1) and M_k = P_(k-1) R_k
    for (int k = nsc; k >= 1; --k) {
        C2<R> ph[2 * MM + 1];
        phase_powers<R, MM>(g.phs[k + 1], ph);
        // Wh[r] = sum over the flip orbit of r of sign * e^{-i eta m_a} M(b, a), M(b, a) = sum_c P_(k-1)(b, c)
        // R_k(c, a), one c at a time.  The Euler-angle derivative needs no weights of its own: with F_k = Phi F~_k,
        // d ptrac / d eta_(k+1) = Tr(R_k (-i m) F_k P_(k-1)) = -i sum_a m_a (P_k R_k)(a, a), and P_k is stored.
        C2<R> Wh[RT.n];
        {
#pragma unroll
            for (int r = 0; r < RT.n; ++r) Wh[r] = cz<R>();
#pragma unroll 1
            for (int c = 0; c < N0; ++c) {
                C2<R> pc[N], rr[N];
#pragma unroll
                for (int b = 0; b < N; ++b) pc[b] = Pst[k - 1][b][c];
#pragma unroll
                for (int a = 0; a < N; ++a) rr[a] = cmul(ph[L.m[a] + MM], Rst[c][a]);
#pragma unroll
                for (int a = 0; a < N; ++a)
#pragma unroll
                    for (int b = 0; b < N; ++b) {
                        const int r = RT.rep[a][b];
                        Wh[r] = RT.sg[a][b] > 0 ? pfma(pc[b], rr[a], Wh[r]) : pfms(pc[b], rr[a], Wh[r]);
                    }
            }
            if constexpr (MASK) mask_lambda<R, KIND, N, N>(Wh, T.nlam);   // entries outside the set are constants
            C2<R> tm = cz<R>();                     // sum_a m_a (P_k R_k)(a, a)
#pragma unroll 1
            for (int c = 0; c < N0; ++c)
#pragma unroll
                for (int a = 0; a < N; ++a)
                    if (L.m[a] != 0) tm = pfma(cscl(Pst[k][a][c], R(L.m[a])), Rst[c][a], tm);
            add_re(pg.eta[k + 1], sd, C2<R>{tm.y, -tm.x});   // -i tm
        }
        if (k > 1) {
            // R_(k-1) = R_k F_k with F_k(c, b) = e^{-i eta m_c} sign F~_k[rep(c, b)], one row of R at a time
            C2<R> f[RT.n];
#pragma unroll
            for (int r = 0; r < RT.n; ++r) f[r] = Fst[k - 1][r];
#pragma unroll 1
            for (int a = 0; a < N0; ++a) {
                C2<R> row[N];
#pragma unroll
                for (int c = 0; c < N; ++c) row[c] = cmul(Rst[a][c], ph[L.m[c] + MM]);
#pragma unroll
                for (int b = 0; b < N; ++b) {
                    C2<R> v = cz<R>();
#pragma unroll
                    for (int c = 0; c < N; ++c)
                        v = RT.sg[c][b] > 0 ? pfma(row[c], f[RT.rep[c][b]], v) : pfms(row[c], f[RT.rep[c][b]], v);
                    Rst[a][b] = v;
                }
            }
        }
        C2<R> gi, go, gb;
        const int ip = g.ip[k];
        contract_f_adj<R, KIND, N, N>(Wh, dh + (k - 1) * dleg, dhd + (k - 1) * dleg, T.tl + ip * tlip + e, E,
                                      T.lmax[ip * E + e] + 1, zfac(cscl(ck, (R)g.ri[k + 1])),
                                      zfac(cscl(ck, (R)g.ri[k])), gi, go, gb);
        add_re(pg.ri[k + 1], sck, gi);
        add_re(pg.ri[k], sck, go);
        add_re(pg.beta[k], sd, gb);
    }
}

// Single scattering, K edge (flip-symmetric six-entry set): T first, then one sweep over F_1 with M = T.
template <typename R, int KIND>
__device__ void energy_ss_sym_adj(const WarpPath<R> &g, const R *dh, const R *dhd, const R (*dterm_db)[49],
                                  const Tables<R> &T, int e, C2<R> gbar, ParGrad &pg)
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N = L.N, N0 = L.N0, MM = L.MM;
    const int E = T.E;
    const size_t tlip = (size_t)(T.L1 + 1) * E;
    const C2<R> ck = T.ck[e];
    if (fabs((double)ck.x) + fabs((double)ck.y) <= 1e-16) return;
    TermLegs<R, KIND> tl;
    term_legs<R, KIND>(g, T, e, 2, ck, tl);
    C2<R> Tm[N0][N0];
    term_matrix<R, KIND>(g, T, e, tl, Tm);
    const C2<R> cf = cfac(g, T, e, 2, ck);
    const C2<R> sd = cmul(C2<R>{gbar.x, -gbar.y}, cf);
    const C2<R> sck = cmul(sd, ck);
    auto add_re = [](double &acc, C2<R> s, C2<R> v) { acc += (double)s.x * v.x - (double)s.y * v.y; };
    constexpr RepTab<KIND, N, N0> RT{};
    C2<R> ph[2 * MM + 1];
    phase_powers<R, MM>(g.phs[2], ph);
    C2<R> Wh[RT.n], We[RT.n];
    orbit_weights<R, KIND, N, N0, MM>([&](int b, int a) { return Tm[b][a]; }, ph, Wh, We);
    C2<R> acc[RT.n];
    C2<R> gi, go, gb;
    const int ip = g.ip[1];
    accumulate_f_adj<R, KIND, N, N0>(acc, Wh, dh, dhd, T.tl + ip * tlip + e, E, T.lmax[ip * E + e] + 1,
                                     zfac(cscl(ck, (R)g.ri[2])), zfac(cscl(ck, (R)g.ri[1])), gi, go, gb);
    C2<R> ge = cz<R>();
#pragma unroll
    for (int r = 0; r < RT.n; ++r) ge = cfma(acc[r], We[r], ge);
    add_re(pg.ri[2], sck, gi);
    add_re(pg.ri[1], sck, go);
    add_re(pg.beta[1], sd, gb);
    add_re(pg.eta[2], sd, ge);
    C2<R> ge1 = cz<R>(), gbn = cz<R>(), gr1 = cz<R>(), grn = cz<R>();
    const C2<R> ptrac = term_adj<R, KIND>(
        g, dterm_db, T, e, tl,
        [&](int b, int a) {
            const C2<R> v = RT.sg[b][a] > 0 ? acc[RT.rep[b][a]] : cscl(acc[RT.rep[b][a]], R(-1));
            return cmul(ph[L.m[b] + MM], v);
        },
        ge1, gbn, gr1, grn);
    add_re(pg.eta[1], sd, ge1);
    add_re(pg.beta[2], sd, gbn);
    add_re(pg.ri[1], sck, gr1);
    add_re(pg.ri[2], sck, grn);
    cfac_grad(g, T, e, 2, gbar, cmul(ptrac, cf), pg);
}

// Single scattering at L and M edges: one column of F at a time (as energy_ss_col), each with its own sweep.
template <typename R, int KIND>
__device__ void energy_ss_col_adj(const WarpPath<R> &g, const R *dh, const R *dhd, const R (*dterm_db)[49],
                                  const Tables<R> &T, int e, C2<R> gbar, ParGrad &pg)
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N = L.N, MM = L.MM, DS = dstride(MM), CI = L.CI, CO = L.CO;
    const int E = T.E;
    const size_t tlip = (size_t)(T.L1 + 1) * E;
    const C2<R> ck = T.ck[e];
    if (fabs((double)ck.x) + fabs((double)ck.y) <= 1e-16) return;
    TermLegs<R, KIND> tl;
    term_legs<R, KIND>(g, T, e, 2, ck, tl);
    const C2<R> cf = cfac(g, T, e, 2, ck);
    const C2<R> sd = cmul(C2<R>{gbar.x, -gbar.y}, cf);
    const C2<R> sck = cmul(sd, ck);
    auto add_re = [](double &acc, C2<R> s, C2<R> v) { acc += (double)s.x * v.x - (double)s.y * v.y; };
    const int ip = g.ip[1];
    const C2<R> *tlk = T.tl + ip * tlip + e;
    const int ilx = T.lmax[ip * E + e] + 1;
    const C2<R> z_in = zfac(cscl(ck, (R)g.ri[2])), z_out = zfac(cscl(ck, (R)g.ri[1]));
    const C2<R> dz_in = cmul(C2<R>{R(0), R(-1)}, cmul(z_in, z_in));
    const C2<R> dz_out = cmul(C2<R>{R(0), R(-1)}, cmul(z_out, z_out));
    C2<R> ph[2 * MM + 1], ph1[2 * MM + 1];
    phase_powers<R, MM>(g.phs[2], ph);
    phase_powers<R, MM>(g.phs[1], ph1);
    C2<R> ptrac = cz<R>();
#pragma unroll 1
    for (int col = 0; col < N; ++col) {
        int m2 = 0, n2 = 0;
#pragma unroll
        for (int q = 0; q < N; ++q)
            if (q == col) { m2 = L.m[q]; n2 = L.n[q]; }
        // the termination row T[col][a] weights column col of F: W[a] = ph(m_a) T[col][a]
        C2<R> Trow[N];
#pragma unroll
        for (int a = 0; a < N; ++a) Trow[a] = cz<R>();
        for (int t = 0; t < T.nterm; ++t) {
            const C2<R> W = T.wt[t * E + e];
            C2<R> g1 = cz<R>();
#pragma unroll
            for (int q = 0; q < N; ++q)
                if (q == col) g1 = cmul(W, cmul(ph1[L.m[q] + MM], tl.G1[t][q]));
#pragma unroll
            for (int a = 0; a < N; ++a)
                Trow[a] = cfma(g1, cscl(tl.G2[t][a], g.dterm[t][(m2 + 3) * 7 + L.m[a] + 3]), Trow[a]);
        }
        C2<R> acc[N];
#pragma unroll
        for (int a = 0; a < N; ++a) acc[a] = cz<R>();
        C2<R> pi[CI + 1], ci[CI + 1], po[CO + 1], co[CO + 1], dpi[CI + 1], dci[CI + 1], dpo[CO + 1], dco[CO + 1];
#pragma unroll
        for (int j = 0; j <= CI; ++j) pi[j] = ci[j] = dpi[j] = dci[j] = cz<R>();
#pragma unroll
        for (int j = 0; j <= CO; ++j) po[j] = co[j] = dpo[j] = dco[j] = cz<R>();
        pi[1] = ci[1] = po[1] = co[1] = C2<R>{R(1), R(0)};
        C2<R> gi = cz<R>(), go = cz<R>(), gb = cz<R>();
        for (int il = 1; il <= ilx; ++il) {
            const C2<R> t = tlk[(size_t)il * E];
            const R *dr = dh + (size_t)il * DS;
            const R *ddr = dhd + (size_t)il * DS;
            C2<R> tco = cz<R>(), tdco = cz<R>();
#pragma unroll
            for (int j = 1; j <= CO; ++j)
                if (j == n2 + 1) { tco = cmul(t, co[j]); tdco = cmul(t, dco[j]); }
#pragma unroll
            for (int a = 0; a < N; ++a) {
                const int m1 = L.m[a];
                const int am = m1 < 0 ? -m1 : m1;
                const bool can = canonical(m1, m2);
                const int idx = can ? dcanon(MM, m1, m2) : dcanon(MM, -m1, -m2);
                R dv = dr[idx], ddv = ddr[idx];
                if (!can && ((m1 - m2) & 1)) { dv = -dv; ddv = -ddv; }
                const int cidx = am + L.n[a] + 1;
                const C2<R> u = cmul(ci[cidx], tco);
                acc[a] = cfmr(u, dv, acc[a]);
                const C2<R> w = cmul(ph[m1 + MM], Trow[a]);
                gi = cfma(cscl(w, dv), cmul(dci[cidx], tco), gi);
                go = cfma(cscl(w, dv), cmul(ci[cidx], tdco), go);
                gb = cfma(cscl(w, ddv), u, gb);
            }
            const R wt = R(2 * il - 1);
            const C2<R> wi = cscl(z_in, wt), wo = cscl(z_out, wt), wdi = cscl(dz_in, wt), wdo = cscl(dz_out, wt);
            C2<R> ni[CI + 1], no[CO + 1], dni[CI + 1], dno[CO + 1];
#pragma unroll
            for (int j = 1; j <= CI; ++j) {
                const C2<R> sv = j > 1 ? cadd(ci[j], ci[j - 1]) : ci[j];
                const C2<R> dsv = j > 1 ? cadd(dci[j], dci[j - 1]) : dci[j];
                ni[j] = cfms(wi, sv, pi[j]);
                dni[j] = cfms(wdi, sv, cfms(wi, dsv, dpi[j]));
            }
#pragma unroll
            for (int j = 1; j <= CO; ++j) {
                const C2<R> sv = j > 1 ? cadd(co[j], co[j - 1]) : co[j];
                const C2<R> dsv = j > 1 ? cadd(dco[j], dco[j - 1]) : dco[j];
                no[j] = cfms(wo, sv, po[j]);
                dno[j] = cfms(wdo, sv, cfms(wo, dsv, dpo[j]));
            }
#pragma unroll
            for (int j = 1; j <= CI; ++j) { pi[j] = ci[j]; ci[j] = ni[j]; dpi[j] = dci[j]; dci[j] = dni[j]; }
#pragma unroll
            for (int j = 1; j <= CO; ++j) { po[j] = co[j]; co[j] = no[j]; dpo[j] = dco[j]; dco[j] = dno[j]; }
        }
        C2<R> ge = cz<R>();
#pragma unroll
        for (int a = 0; a < N; ++a) {
            const C2<R> v = cmul(cmul(ph[L.m[a] + MM], Trow[a]), acc[a]);
            ge = cadd(ge, C2<R>{v.y * R(L.m[a]), -v.x * R(L.m[a])});
        }
        add_re(pg.ri[2], sck, gi);
        add_re(pg.ri[1], sck, go);
        add_re(pg.beta[1], sd, gb);
        add_re(pg.eta[2], sd, ge);
        // the termination row col with column col of F as P(b, col)
        C2<R> ge1 = cz<R>(), gbn = cz<R>(), gr1 = cz<R>(), grn = cz<R>();
        ptrac = cadd(ptrac, term_adj<R, KIND>(
                                g, dterm_db, T, e, tl, [&](int b, int) { return cmul(ph[L.m[b] + MM], acc[b]); }, ge1,
                                gbn, gr1, grn, nullptr, 0, col, col + 1));
        add_re(pg.eta[1], sd, ge1);
        add_re(pg.beta[2], sd, gbn);
        add_re(pg.ri[1], sck, gr1);
        add_re(pg.ri[2], sck, grn);
    }
    cfac_grad(g, T, e, 2, gbar, cmul(ptrac, cf), pg);
}

template <typename R, int EDGE, bool MASK = false>
__device__ __forceinline__ void path_energy_adj(const WarpPath<R> &g, const R *dh, const R *dhd,
                                                const R (*dterm_db)[49], const Tables<R> &T, int e, int nleg,
                                                C2<R> gbar, ParGrad &pg)
{
    using K = Kinds<EDGE>;
    if (nleg == 2) {
        if constexpr (K::SS_SYM)
            energy_ss_sym_adj<R, K::SS>(g, dh, dhd, dterm_db, T, e, gbar, pg);
        else
            energy_ss_col_adj<R, K::SS>(g, dh, dhd, dterm_db, T, e, gbar, pg);
        return;
    }
    energy_ms_adj<R, K::MS, MASK>(g, dh, dhd, dterm_db, T, e, nleg, gbar, pg);
}

// ------------------------------------------------------------------------------------------------ kernels
template <typename R> struct AdjShared {
    R dterm_db[2][49];
    double gpar[3 * (kMaxLeg + 1)];
    double cg[9 * kMaxLeg];            // coordinate-gradient contributions per (leg, atom slot, component)
};

template <typename R> __host__ __device__ constexpr size_t adj_head_bytes()
{
    return geo_bytes<R>() + (sizeof(AdjShared<R>) + 15) / 16 * 16;
}

template <typename R> inline size_t adj_warp_bytes(int L1, int nsc_max, int MM)
{
    return adj_head_bytes<R>() + 2 * align_up((size_t)nsc_max * (L1 + 1) * dstride(MM) * sizeof(R), 16);
}

// ------------------------------------------------------------------------------------------------ frames
// FEFF's Euler angles of a leg along z are undefined: trig's small-vector branch (stage.py:148-157) makes them
// constants, so their derivatives there are not those of the path signal, and near the axis they are large terms
// that cancel.  The signal is invariant under a rotation of the whole path, so a path with a leg within
// asin(kAxialSin) of the z axis is differentiated in a rotated frame whose z axis is the candidate axis farthest
// from every leg (for any nine legs some candidate keeps at least about 18 degrees from all of them), and its
// coordinate gradient is rotated back.  Every other path keeps the identity frame and its results are unchanged.
// The candidates: a golden-angle spiral over the upper hemisphere, away from low-index lattice directions.
constexpr double kAxialSin = 0.1;
constexpr int kFrames = 8;

__device__ __forceinline__ void frame_axis(int c, double &ux, double &uy, double &uz)
{
    constexpr double U[kFrames][3] = {
        {0.39843402527945515, 0.1600486234699024, 0.903125},   {-0.54971449428963837, 0.2067028885692874, 0.809375},
        {0.31602489695350588, -0.62290378380655709, 0.715625}, {0.21048585883560078, 0.75429913668599635, 0.621875},
        {-0.72079234200148334, -0.44893472140949026, 0.528125}, {0.88543036946101195, -0.16532217096063032, 0.434375},
        {-0.56492954713603705, 0.75155120660382946, 0.340625}, {-0.093899422019386392, -0.96448723833932881, 0.246875}};
    ux = U[c][0]; uy = U[c][1]; uz = U[c][2];
}

// Rotation Q of frame f (1..kFrames) taking its axis u to z (Rodrigues about u x z): x' = Q x.
__device__ __forceinline__ void frame_matrix(int f, double (&Q)[3][3])
{
    double ux, uy, uz;
    frame_axis(f - 1, ux, uy, uz);
    const double s = sqrt(ux * ux + uy * uy), c = uz, kx = uy / s, ky = -ux / s, t = 1.0 - c;
    Q[0][0] = c + t * kx * kx; Q[0][1] = t * kx * ky;     Q[0][2] = s * ky;
    Q[1][0] = t * kx * ky;     Q[1][1] = c + t * ky * ky; Q[1][2] = -s * kx;
    Q[2][0] = -s * ky;         Q[2][1] = s * kx;          Q[2][2] = c;
}

// Warp-uniform frame of a path: 0 (identity) unless a leg lies within asin(kAxialSin) of z, else the candidate whose
// smallest sin(angle to a leg) is largest.  Lane j (1..nleg) holds leg j, x_j - x_(j-1) (x_nleg = x_0).
template <typename R> __device__ int choose_frame(const WarpPath<R> &g, int nleg, int lane)
{
    double vx = 0.0, vy = 0.0, vz = 0.0, r2 = 0.0;
    if (lane >= 1 && lane <= nleg) {
        const int a = lane == nleg ? 0 : lane, b = lane - 1;
        vx = g.xyz[a][0] - g.xyz[b][0]; vy = g.xyz[a][1] - g.xyz[b][1]; vz = g.xyz[a][2] - g.xyz[b][2];
        r2 = vx * vx + vy * vy + vz * vz;
    }
    auto warp_min = [](double v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        return v;
    };
    // sin^2 of the angle between the leg and axis u; lanes without a leg, and legs of zero length, do not constrain
    auto sin2 = [&](double ux, double uy, double uz) {
        if (r2 <= 0.0) return 1.0;
        const double d = ux * vx + uy * vy + uz * vz;
        return 1.0 - d * d / r2;
    };
    if (warp_min(sin2(0.0, 0.0, 1.0)) >= kAxialSin * kAxialSin) return 0;
    int best = 1;
    double best_s = -1.0;
    for (int c = 0; c < kFrames; ++c) {
        double ux, uy, uz;
        frame_axis(c, ux, uy, uz);
        const double s = warp_min(sin2(ux, uy, uz));
        if (s > best_s) { best_s = s; best = c + 1; }
    }
    return best;
}

// Rotates the path's atoms into frame f and recomputes the Euler angles and phases (leg lengths, scattering angles
// and so the rotation tables are invariant and kept).
template <typename R> __device__ void reframe_path(WarpPath<R> &g, int nleg, int lane, int f)
{
    double Q[3][3];
    frame_matrix(f, Q);
    if (lane < nleg) {
        const double x = g.xyz[lane][0], y = g.xyz[lane][1], z = g.xyz[lane][2];
#pragma unroll
        for (int i = 0; i < 3; ++i) g.xyz[lane][i] = Q[i][0] * x + Q[i][1] * y + Q[i][2] * z;
    }
    __syncwarp();
    if (lane >= 1 && lane <= nleg) {
        auto rat = [&](int i, double *o) {
            const int a = (i == 0 || i == nleg) ? 0 : i;
            o[0] = g.xyz[a][0]; o[1] = g.xyz[a][1]; o[2] = g.xyz[a][2];
        };
        const LegGeom lg = leg_geometry<double>(rat, lane, nleg);
        g.alpha[lane] = lg.alpha;
        g.gamma[lane] = lg.gamma;
    }
    __syncwarp();
    if (lane >= 1 && lane <= nleg) {
        const double eta = g.alpha[lane == 1 ? nleg : lane - 1] + g.gamma[lane];
        double s, c;
        sincos(eta, &s, &c);
        g.phs[lane] = C2<R>{(R)c, (R)(-s)};
    }
    __syncwarp();
}

// The coordinate gradient held one component per lane (lane = 3 atom + component) rotated from frame f back to the
// original frame: g = Q^T g'.
__device__ __forceinline__ double unframe_grad(double gc, int lane, int f)
{
    double Q[3][3];
    frame_matrix(f, Q);
    const int a = lane / 3, c = lane % 3;
    const double g0 = __shfl_sync(0xffffffffu, gc, min(3 * a, 31));
    const double g1 = __shfl_sync(0xffffffffu, gc, min(3 * a + 1, 31));
    const double g2 = __shfl_sync(0xffffffffu, gc, min(3 * a + 2, 31));
    return Q[0][c] * g0 + Q[1][c] * g1 + Q[2][c] * g2;
}

// Geometry adjoint: dL/dcoords (nleg, 3) of one path from the reduced parameter gradients in gpar (bohr units),
// returned one coordinate direction per lane (lane = 3 atom + component).  Leg j's geometry reads three atoms (j,
// j + 1, j - 1; the absorber for 0 and nleg), so each (leg, atom slot, component) is one dual-number evaluation of
// leg_geometry seeded along that coordinate: 9 nleg tasks spread over the warp (three rounds for eight legs) instead
// of nleg + 1 evaluations in sequence on every lane.  Leg j's parameters enter the loss as gpar_ri[j] ri_j +
// gpar_beta[j] beta_j + gpar_eta[j] gamma_j + gpar_eta[j'] alpha_j with j' = j + 1 (1 for j = nleg:
// eta_1 = alpha_nleg + gamma_1).  The contributions pass through cg (9 kMaxLeg doubles of the warp's shared memory)
// and each lane sums those of its coordinate in a fixed order (leg, then slot).
__device__ __forceinline__ double coord_grad(const double (*xyz)[3], const double *gpar, double *cg, int nleg,
                                             int lane)
{
    const double inv = 1.0 / kBohr;
    auto amap = [nleg](int x) { return (x == 0 || x == nleg) ? 0 : x; };
    // the atom in slot s of leg j (leg_geometry's i, ip1, im1) and whether an earlier slot holds the same atom
    auto slot_atom = [&](int j, int s, bool &dup) {
        const int i = j == nleg ? 0 : j, ip1 = j == nleg ? 1 : j + 1, im1 = j - 1;
        const int a0 = amap(i), a1 = amap(ip1), a2 = amap(im1);
        dup = (s == 1 && a1 == a0) || (s == 2 && (a2 == a0 || a2 == a1));
        return s == 0 ? a0 : (s == 1 ? a1 : a2);
    };
    for (int task = lane; task < 9 * nleg; task += 32) {
        const int j = task / 9 + 1, s = (task % 9) / 3, comp = task % 3;
        bool dup;
        const int atom = slot_atom(j, s, dup);
        double v = 0.0;
        if (!dup) {
            auto rat = [&](int i, Dual *o) {
                const int a = amap(i);
#pragma unroll
                for (int c = 0; c < 3; ++c) o[c] = Dual{xyz[a][c], (a == atom && c == comp) ? inv : 0.0};
            };
            const LegGeomT<Dual> lg = leg_geometry<Dual>(rat, j, nleg);
            const int jn = j == nleg ? 1 : j + 1;
            v = gpar[j] * lg.ri.d + gpar[(kMaxLeg + 1) + j] * lg.beta.d + gpar[2 * (kMaxLeg + 1) + j] * lg.gamma.d +
                gpar[2 * (kMaxLeg + 1) + jn] * lg.alpha.d;
        }
        cg[task] = v;
    }
    __syncwarp();
    double out = 0.0;
    if (lane < 3 * nleg) {
        const int atom = lane / 3, comp = lane % 3;
        for (int j = 1; j <= nleg; ++j)
#pragma unroll
            for (int s = 0; s < 3; ++s) {
                bool dup;
                if (slot_atom(j, s, dup) == atom && !dup) out += cg[(j - 1) * 9 + 3 * s + comp];
            }
    }
    __syncwarp();
    return out;
}

// The adjoint over a set of paths: per path the seeds gbar (E, complex) and dL/dreff (A), out dL/dcoords.
// Paths come from `order` (or are 0..B-1), coordinates/ipots with a row stride of `stride` legs.
// SPLIT: the coordinate gradient is k_coord_grad's (the fused backward); the kernel hands over each path's parameter
// gradients and frame in gpar_out and carries none of that code.
template <typename R, int EDGE, typename CT, bool MASK = false, bool SPLIT = false>
__global__ void __launch_bounds__(128) k_adjoint(Tables<R> T, const CT *__restrict__ coords,
                                                  const int64_t *__restrict__ ipots, int stride,
                                                  const int *__restrict__ nlegs, int nleg_uniform, int64_t B,
                                                  const int *__restrict__ order, const C2<R> *__restrict__ gbar,
                                                  const double *__restrict__ greff_d, const R *__restrict__ greff_r,
                                                  R *__restrict__ gout_r, double *__restrict__ gout_d,
                                                  unsigned long long *counter, int *status, int nsc_max, size_t wbytes,
                                                  double *__restrict__ gpar_out)
{
    using K = Kinds<EDGE>;
    extern __shared__ __align__(16) unsigned char smem[];
    if (*(volatile const int *)status & kBadLayout) return;     // a batch that k_validate refused
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int E = T.E, L1 = T.L1;
    unsigned char *base = smem + (size_t)w * wbytes;
    WarpPath<R> &g = *reinterpret_cast<WarpPath<R> *>(base);
    AdjShared<R> &as = *reinterpret_cast<AdjShared<R> *>(base + geo_bytes<R>());
    const size_t dsz = align_up((size_t)nsc_max * (L1 + 1) * dstride(K::MM) * sizeof(R), 16);
    R *dh = reinterpret_cast<R *>(base + adj_head_bytes<R>());
    R *dhd = reinterpret_cast<R *>(base + adj_head_bytes<R>() + dsz);
    for (;;) {
        unsigned long long tk = 0;
        if (lane == 0) tk = atomicAdd(counter, 1ull);
        tk = __shfl_sync(0xffffffffu, tk, 0);
        if (tk >= (unsigned long long)B) break;
        const int64_t p = order ? order[tk] : (int64_t)tk;
        const int nleg = nlegs ? nlegs[p] : nleg_uniform;
        const int MM = nleg == 2 ? K::MMSS : K::MMMS;
        path_setup<R, CT>(g, dh, T, coords + p * stride * 3, ipots + p * stride, nleg, lane, status, MM, false);
        adj_setup<R>(g, dh, dhd, as.dterm_db, T, nleg, lane, MM);
        __syncwarp();
        const int frame = choose_frame<R>(g, nleg, lane);
        if (frame) reframe_path<R>(g, nleg, lane, frame);
        ParGrad pg;
        for (int j = 0; j <= kMaxLeg; ++j) pg.ri[j] = pg.beta[j] = pg.eta[j] = 0.0;
        for (int e0 = first_chunk(E); e0 < E; e0 += 32) {
            const int e = e0 + lane;
            if (e >= 0 && e < E)
                path_energy_adj<R, EDGE, MASK>(g, dh, dhd, as.dterm_db, T, e, nleg, gbar[p * E + e], pg);
        }
        // fixed-order warp reduction of the per-lane sums
        for (int j = 1; j <= nleg; ++j) {
            double v[3] = {pg.ri[j], pg.beta[j], pg.eta[j]};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
            }
            if (lane == 0) {
                as.gpar[j] = v[0];
                as.gpar[(kMaxLeg + 1) + j] = v[1];
                as.gpar[2 * (kMaxLeg + 1) + j] = v[2];
            }
        }
        __syncwarp();
        if (lane == 0) {
            // reff (A) = BOHR sum ri (bohr) / 2
            const double gr = greff_d ? greff_d[p] : (greff_r ? (double)greff_r[p] : 0.0);
            for (int j = 1; j <= nleg; ++j) as.gpar[j] += gr * kBohr * 0.5;
        }
        __syncwarp();
        if constexpr (SPLIT) {
            // the coordinate gradient is k_coord_grad's: hand over the parameter gradients and the frame
            double *o = gpar_out + p * kGparStride;
            for (int i = lane; i < 3 * (kMaxLeg + 1); i += 32) o[i] = as.gpar[i];
            if (lane == 0) o[3 * (kMaxLeg + 1)] = (double)frame;
        } else {
            double gc = coord_grad(g.xyz, as.gpar, as.cg, nleg, lane);
            if (frame) gc = unframe_grad(gc, lane, frame);
            if (lane < 3 * stride) {
                const int64_t o = p * stride * 3 + lane;
                const double v = lane < 3 * nleg ? gc : 0.0;
                if (gout_d) gout_d[o] = v;
                else gout_r[o] = (R)v;
            }
        }
        __syncwarp();
    }
}

// The coordinate gradient of the fused backward as a kernel of its own (a warp per path, four per CTA): the paths'
// parameter gradients and frames come from k_adjoint through gpar (kGparStride doubles per path), the atoms from the
// batch, rotated into the path's frame exactly as reframe_path rotates them; then coord_grad and the rotation back,
// as k_adjoint does inline for the drop-in cchi backward.  Inside k_adjoint this per-path code ran at 8 warps per SM
// between long energy loops; here it runs at 20 (96 registers), and the split k_adjoint carries none of it: forward +
// backward of the path-finder batch on B200 219.3 -> 216.8 ms, gradients bit-identical.
template <typename CT>
__global__ void __launch_bounds__(128) k_coord_grad(const CT *__restrict__ coords, int stride,
                                                     const int *__restrict__ nlegs, int nleg_uniform, int64_t B,
                                                     const double *__restrict__ gpar, double *__restrict__ gout,
                                                     const int *status)
{
    __shared__ double s_xyz[4][kMaxLeg][3], s_gpar[4][3 * (kMaxLeg + 1)], s_cg[4][9 * kMaxLeg];
    if (*(volatile const int *)status & kBadLayout) return;     // a batch that k_validate refused
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t p = (int64_t)blockIdx.x * 4 + w; p < B; p += (int64_t)gridDim.x * 4) {
        const int nleg = nlegs ? nlegs[p] : nleg_uniform;
        const double *gp = gpar + p * kGparStride;
        for (int i = lane; i < nleg * 3; i += 32) s_xyz[w][i / 3][i % 3] = (double)coords[p * stride * 3 + i] / kBohr;
        for (int i = lane; i < 3 * (kMaxLeg + 1); i += 32) s_gpar[w][i] = gp[i];
        const int frame = (int)gp[3 * (kMaxLeg + 1)];
        __syncwarp();
        if (frame) {
            double Q[3][3];
            frame_matrix(frame, Q);
            if (lane < nleg) {
                const double x = s_xyz[w][lane][0], y = s_xyz[w][lane][1], z = s_xyz[w][lane][2];
#pragma unroll
                for (int i = 0; i < 3; ++i) s_xyz[w][lane][i] = Q[i][0] * x + Q[i][1] * y + Q[i][2] * z;
            }
            __syncwarp();
        }
        double gc = coord_grad(s_xyz[w], s_gpar[w], s_cg[w], nleg, lane);
        if (frame) gc = unframe_grad(gc, lane, frame);
        if (lane < 3 * stride) gout[p * stride * 3 + lane] = lane < 3 * nleg ? gc : 0.0;
        __syncwarp();
    }
}

// Fine-grid adjoint (stage.py:372-388 differentiated): per path, from upstream weights G(q) on the fine grid, the
// seeds gbar(e) = dL/dRe(cchi) + i dL/dIm(cchi), dL/dreff (A) and, with per-path sigma2, dL/dsigma2.
// mode 0: G = grad_chi[p][q] (chi_fine's adjoint); mode 1: G = grad_rows[row[p]][q] deg[p] exp(-2 sigma2 q^2)
// (the fused sum's adjoint).  Interpolation transposed with the column ranges tspan of S.
template <typename R>
__global__ void __launch_bounds__(256) k_fine_adjoint(int64_t B, int E, int NK, int mode,
                                                       const C2<R> *__restrict__ cchi, const R *__restrict__ reff_r,
                                                       const double *__restrict__ reff_d, const R *__restrict__ q_r,
                                                       const double *__restrict__ q_d, const R *__restrict__ S_r,
                                                       const double *__restrict__ S_d, const int *__restrict__ span,
                                                       const int *__restrict__ tspan, const R *__restrict__ gchi,
                                                       const double *__restrict__ grows, const int *__restrict__ row,
                                                       const double *__restrict__ deg,
                                                       const double *__restrict__ sigma2, C2<R> *__restrict__ gbar,
                                                       R *__restrict__ greff_r, double *__restrict__ greff_d,
                                                       double *__restrict__ gsig, int *status, size_t wbytes)
{
    extern __shared__ __align__(16) unsigned char smem[];
    if (status && (*(volatile const int *)status & kBadLayout)) return;   // a batch that k_validate refused
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned char *base = smem + (size_t)w * wbytes;
    double *amp = reinterpret_cast<double *>(base);        // FP64, as the forward forms it
    double *pha = reinterpret_cast<double *>(base + align_up((size_t)E * 8, 16));
    double *dA = reinterpret_cast<double *>(base + 2 * align_up((size_t)E * 8, 16));
    double *dP = dA + NK;
    auto Sv = [&](int k, int j) { return S_d ? S_d[(size_t)k * E + j] : (double)S_r[(size_t)k * E + j]; };
    for (int64_t p = (int64_t)blockIdx.x * nw + w; p < B; p += (int64_t)gridDim.x * nw) {
        const C2<R> *c = cchi + p * E;
        amp_phase<R>(E, lane, [&](int e) { return c[e]; }, amp, pha);
        __syncwarp();
        const double rf = reff_d ? reff_d[p] : (double)reff_r[p];
        const double s2 = (mode == 1 && sigma2) ? sigma2[p] : 0.0;
        const double wd = mode == 1 ? deg[p] : 1.0;
        const double *gr = mode == 1 ? grows + (int64_t)row[p] * NK : nullptr;
        double g_reff = 0.0, g_s2 = 0.0;
        for (int k0 = 0; k0 < NK; k0 += 32) {
            const int k = k0 + lane;
            double da = 0.0, dp = 0.0;
            if (k < NK) {
                const int lo = span[2 * k], hi = span[2 * k + 1];
                double a = 0.0, ph = 0.0;
                for (int j = lo; j < hi; ++j) {
                    const double sv = Sv(k, j);
                    a += sv * (double)amp[j];
                    ph += sv * pha[j];
                }
                const double qk = q_d ? q_d[k] : (double)q_r[k];
                const double damp = s2 != 0.0 ? exp(-2.0 * s2 * qk * qk) : 1.0;
                const double G = (mode == 1 ? gr[k] * wd : (double)gchi[p * NK + k]) * damp;
                const double arg = ph + 2.0 * qk * rf;
                const double sn = sin_arg<R>(arg), cs = sin_arg<R>(arg + 1.5707963267948966);
                da = G * sn;
                dp = G * a * cs;
                g_reff += dp * 2.0 * qk;
                g_s2 += G * a * sn * (-2.0 * qk * qk);
                dA[k] = da;
                dP[k] = dp;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g_reff += __shfl_xor_sync(0xffffffffu, g_reff, o);
            g_s2 += __shfl_xor_sync(0xffffffffu, g_s2, o);
        }
        __syncwarp();
        for (int e0 = 0; e0 < E; e0 += 32) {
            const int e = e0 + lane;
            if (e < E) {
                const int lo = tspan[2 * e], hi = tspan[2 * e + 1];
                double ga = 0.0, gp = 0.0;
                for (int k = lo; k < hi; ++k) {
                    const double sv = Sv(k, e);
                    ga += sv * dA[k];
                    gp += sv * dP[k];
                }
                const C2<R> cv = c[e];
                const double x = (double)cv.x, y = (double)cv.y;
                const double a = sqrt(x * x + y * y + 1e-30);
                double gx = ga * x / a, gy = ga * y / a;
                if (a >= 1e-16) {
                    const double r2 = x * x + y * y;
                    gx += gp * (-y) / r2;
                    gy += gp * x / r2;
                }
                gbar[p * E + e] = C2<R>{(R)gx, (R)gy};
            }
        }
        if (lane == 0) {
            if (greff_d) greff_d[p] = g_reff;
            if (greff_r) greff_r[p] = (R)g_reff;
            if (gsig) gsig[p] = g_s2;
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------------------ launches
template <typename R, int EDGE, typename CT>
fg_status launch_adjoint(const StageView &sv, const Tables<R> &T, const CT *coords, const int64_t *ipots, int stride,
                         const int *nlegs, int nleg_uniform, int nsc_max, int64_t B, const int *order,
                         const C2<R> *gbar, const double *greff_d, const R *greff_r, R *gout_r, double *gout_d,
                         unsigned long long *counter, int *status, int warps, cudaStream_t st,
                         double *gpar_out = nullptr)
{
    using K = Kinds<EDGE>;
    const size_t wb = adj_warp_bytes<R>(sv.L1, nsc_max, K::MM);
    warps = fit_warps(warps, wb, sv.max_smem);
    const int threads = warps * 32;
    auto kern = k_adjoint<R, EDGE, CT, false>;
    if constexpr (K::MS <= 1)                       // orders 0 and 1 restrict the order-2 sets
        if (T.nlam < lamtab(K::MS).N) kern = k_adjoint<R, EDGE, CT, true>;
    if constexpr (std::is_same<CT, double>::value)  // the fused backward (FP64 coordinates) splits
        if (gpar_out) {
            kern = k_adjoint<R, EDGE, CT, false, true>;
            if constexpr (K::MS <= 1)
                if (T.nlam < lamtab(K::MS).N) kern = k_adjoint<R, EDGE, CT, true, true>;
        }
    int blocks = 0;
    if (fg_status rc = grid_for(kern, threads, wb * warps, sv.num_sms, B, blocks)) return rc;
    timer_begin(st);
    kern<<<blocks, threads, wb * warps, st>>>(T, coords, ipots, stride, nlegs, nleg_uniform, B, order, gbar, greff_d,
                                              greff_r, gout_r, gout_d, counter, status, nsc_max, wb, gpar_out);
    timer_end(st);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

template <typename R>
fg_status launch_fine_adjoint(const StageView &sv, int64_t B, int NK, int mode, const void *cchi, const R *reff_r,
                              const double *reff_d, const R *q_r, const double *q_d, const R *S_r, const double *S_d,
                              const int *span, const int *tspan, const R *gchi, const double *grows, const int *row,
                              const double *deg, const double *sigma2, C2<R> *gbar, R *greff_r,
                              double *greff_d, double *gsig, int *status, cudaStream_t st)
{
    const size_t wb = 2 * align_up((size_t)sv.E * 8, 16) + align_up((size_t)NK * 16, 16);
    const int warps = fit_warps(4, wb, sv.max_smem), threads = warps * 32;
    auto kern = k_fine_adjoint<R>;
    int blocks = 0;
    if (fg_status rc = grid_for(kern, threads, wb * warps, sv.num_sms, B, blocks)) return rc;
    kern<<<blocks, threads, wb * warps, st>>>(B, sv.E, NK, mode, static_cast<const C2<R> *>(cchi), reff_r, reff_d, q_r,
                                              q_d, S_r, S_d, span, tspan, gchi, grows, row, deg, sigma2, gbar,
                                              greff_r, greff_d, gsig, status, wb);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

template <typename R, int EDGE>
fg_status Launch<R, EDGE>::cchi_bwd(const StageView &sv, const Tables<R> &T, int64_t B, int nleg, const void *coords,
                                    int coords_f64, const int64_t *ipots, const void *grad_cchi, const void *grad_reff,
                                    void *grad_coords, unsigned char *ws, int warps, cudaStream_t st)
{
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(ws);
    int *status = reinterpret_cast<int *>(ws + kStatusOffset);
    const C2<R> *gb = static_cast<const C2<R> *>(grad_cchi);
    const R *gr = static_cast<const R *>(grad_reff);
    FG_CUDA(cudaMemsetAsync(ws, 0, kCounterBytes, st));
    if (coords_f64)
        return launch_adjoint<R, EDGE, double>(sv, T, static_cast<const double *>(coords), ipots, nleg, nullptr, nleg,
                                               nleg - 1, B, nullptr, gb, nullptr, gr, static_cast<R *>(grad_coords),
                                               nullptr, counter, status, warps, st);
    return launch_adjoint<R, EDGE, float>(sv, T, static_cast<const float *>(coords), ipots, nleg, nullptr, nleg,
                                          nleg - 1, B, nullptr, gb, nullptr, gr, static_cast<R *>(grad_coords),
                                          nullptr, counter, status, warps, st);
}

template <typename R, int EDGE>
fg_status Launch<R, EDGE>::fused_bwd(const StageView &sv, const Tables<R> &T, const fg_paths *P, int NK,
                                     const double *q, const double *S, const int *span, const int *tspan,
                                     const double *grad_rows, const void *cchi_saved, const double *reff_saved,
                                     double *grad_coords, double *grad_sigma2, unsigned char *ws, int warps,
                                     cudaStream_t st)
{
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(ws);
    int *status = reinterpret_cast<int *>(ws + kStatusOffset);
    C2<R> *gbar = reinterpret_cast<C2<R> *>(ws + kCounterBytes);
    double *greff = reinterpret_cast<double *>(ws + kCounterBytes + align_up((size_t)P->n * sv.E * sizeof(C2<double>), 256));
    double *gpar = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(greff) +
                                              align_up((size_t)P->n * sizeof(double), 256));
    FG_CUDA(cudaMemsetAsync(ws, 0, kCounterBytes, st));
    if (P->n == 0) return FG_OK;
    if (fg_status rc = launch_validate(P, sv.nph1, status, st)) return rc;
    if (fg_status rc = launch_fine_adjoint<R>(sv, P->n, NK, 1, cchi_saved, nullptr, reff_saved, nullptr, q, nullptr, S,
                                              span, tspan, nullptr, grad_rows, P->row, P->deg, P->sigma2,
                                              gbar, nullptr, greff, grad_sigma2, status, st))
        return rc;
    if (fg_status rc = launch_adjoint<R, EDGE, double>(sv, T, P->coords, P->ipots, P->nleg_max, P->nleg, 0,
                                                       P->nleg_max - 1, P->n, P->order, gbar, greff, nullptr, nullptr,
                                                       grad_coords, counter, status, warps, st, gpar))
        return rc;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((P->n + 3) / 4, (int64_t)sv.num_sms * 16));
    k_coord_grad<double><<<blocks, 128, 0, st>>>(P->coords, P->nleg_max, P->nleg, 0, P->n, gpar, grad_coords, status);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

template <typename R>
fg_status LaunchCommon<R>::chi_fine_bwd(const StageView &sv, int64_t B, const void *cchi, const void *reff, int NK,
                                        const void *q, const void *S, const int *span, const int *tspan,
                                        const void *grad_chi, void *grad_cchi, void *grad_reff, cudaStream_t st)
{
    return launch_fine_adjoint<R>(sv, B, NK, 0, cchi, static_cast<const R *>(reff), nullptr, static_cast<const R *>(q),
                                  nullptr, static_cast<const R *>(S), nullptr, span, tspan,
                                  static_cast<const R *>(grad_chi), nullptr, nullptr, nullptr, nullptr,
                                  static_cast<C2<R> *>(grad_cchi), static_cast<R *>(grad_reff), nullptr, nullptr,
                                  nullptr, st);
}

}  // namespace fg
