// fg_forward.cuh -- the per-path setup and the per-energy path signal (forward).
//
// Reference algorithm: GPUPathStage.cchi (src/feffgpu/stage.py:235-338), itself the batched form of FEFF's GENFMT
// (src/feffgpu/genfmt.py:395-447).  The formulation here is register-resident and streams over the partial waves:
//
//   F_k[l1, l2] = e^{-i eta_{k+1} m1} sum_il D^(k)[il, m1, m2] c_{k+1}[il, |m1|+n1+1] t_il(e, ipot_k) c_k[il, n2+1]
//
// with D^(k)[il, m1, m2] = d^{il-1}_{m1 m2}(beta_k) xnlm(il,|m1|+1) (-1)^|m1| / xnlm(il,|m2|+1) (the Legendre
// normalisations of gam and gamtl folded into the per-path rotation table), c_j the spherical-wave factors of leg
// j (sclmz) advanced one partial wave per step, and only the flip-canonical (m1, m2) entries accumulated.
#pragma once
#include "fg_device.cuh"

namespace fg {

// Per-warp shared state of the path being evaluated.
template <typename R> struct WarpPath {
    double xyz[kMaxLeg][3];        // atoms of the path, bohr, absorber first
    double ri[kMaxLeg + 1];        // leg lengths, 1..nleg (bohr)
    double beta[kMaxLeg + 1];
    double alpha[kMaxLeg + 1];
    double gamma[kMaxLeg + 1];
    double reff;                   // bohr
    C2<R> phs[kMaxLeg + 1];        // e^{-i eta_j}
    int ip[kMaxLeg + 1];           // potential of atom j (0 and nleg: the absorber)
    R dterm[2][49];                // d^{l_t}_{m1 m2}(beta_nleg), [m1+3][m2+3]
};

template <typename R, int MM> __host__ __device__ constexpr size_t dh_floats(int L1, int nsc)
{
    return (size_t)nsc * (L1 + 1) * dstride(MM);
}

// (m1, m2) of canonical index r
__device__ __forceinline__ void canon_mn(int MM, int r, int &m1, int &m2)
{
    if (r <= MM) { m1 = 0; m2 = r; return; }
    r -= MM + 1;
    m1 = 1 + r / (2 * MM + 1);
    m2 = r % (2 * MM + 1) - MM;
}

// Warp-cooperative setup of one path: geometry (FP64), Euler phases, rotation tables of legs 1..nsc (unless
// tables is false: the adjoint forms them with their derivatives) and the termination's rotation matrices.
// coords: (nleg, 3) angstrom (float or double), ipots: (nleg).
template <typename R, typename CT>
__device__ void path_setup(WarpPath<R> &g, R *dh, const Tables<R> &T, const CT *coords, const int64_t *ipots,
                           int nleg, int lane, int *bad_ipot, int MM, bool tables = true)
{
    const int nsc = nleg - 1;
    for (int i = lane; i < nleg * 3; i += 32) g.xyz[i / 3][i % 3] = (double)coords[i] / kBohr;
    if (lane <= nleg) {
        int64_t v = ipots[(lane == 0 || lane == nleg) ? 0 : lane];
        if (v < 0 || v >= T.nph1) {
            if (bad_ipot) atomicOr(bad_ipot, kBadIpot);
            v = v < 0 ? 0 : T.nph1 - 1;
        }
        g.ip[lane] = (int)v;
    }
    __syncwarp();
    if (lane >= 1 && lane <= nleg) {
        auto rat = [&](int i, double *o) {
            const int a = (i == 0 || i == nleg) ? 0 : i;
            o[0] = g.xyz[a][0]; o[1] = g.xyz[a][1]; o[2] = g.xyz[a][2];
        };
        LegGeom lg = leg_geometry<double>(rat, lane, nleg);
        g.ri[lane] = lg.ri; g.beta[lane] = lg.beta; g.alpha[lane] = lg.alpha; g.gamma[lane] = lg.gamma;
    }
    __syncwarp();
    if (lane >= 1 && lane <= nleg) {
        const double eta = g.alpha[lane == 1 ? nleg : lane - 1] + g.gamma[lane];
        double s, c;
        sincos(eta, &s, &c);
        g.phs[lane] = C2<R>{(R)c, (R)(-s)};
    }
    if (lane == 0) {
        double r = 0.0;
        for (int j = 1; j <= nleg; ++j) r += g.ri[j];
        g.reff = 0.5 * r;
    }
    // rotation tables D^(k), k = 1..nsc, il = 1..L1
    const int NC = ncanon(MM), DS = dstride(MM), L1 = T.L1;
    for (int task = lane; tables && task < nsc * NC; task += 32) {
        const int k = task / NC + 1, r = task % NC;
        int m1, m2;
        canon_mn(MM, r, m1, m2);
        const double b = g.beta[k];
        const double c = cos(b), c2 = cos(0.5 * b), s2 = sin(0.5 * b);
        R *out = dh + (size_t)(k - 1) * (L1 + 1) * DS + r;
        const double *xf = T.xfac + (m1 + 3) * 7 + (m2 + 3);
        double dm1 = 0.0, d0 = 0.0;
        const int lseed = min(L1, 4);
        for (int l = 0; l < lseed; ++l) {             // l <= 3: Wigner's explicit sum
            const double dl = wigner_small(l, m1, m2, c2, s2, seed_table(T));
            out[(size_t)(l + 1) * DS] = (R)(dl * xf[(size_t)(l + 1) * 49]);
            dm1 = d0;
            d0 = dl;
        }
        // the three-term recursion: its coefficient loads do not depend on it, so the unrolled trips issue them
        // ahead of the dependent multiply-adds
#pragma unroll 4
        for (int l = lseed; l < L1; ++l) {
            const double *q = T.rc + (((size_t)(l - 1) * 7 + (m1 + 3)) * 7 + (m2 + 3)) * 3;
            const double dl = fma(fma(q[0], c, -q[1]), d0, -q[2] * dm1);
            out[(size_t)(l + 1) * DS] = (R)(dl * xf[(size_t)(l + 1) * 49]);
            dm1 = d0;
            d0 = dl;
        }
    }
    // termination rotation matrices at the absorber (beta_nleg), l_t <= 3
    for (int task = lane; task < T.nterm * 49; task += 32) {
        const int t = task / 49, m1 = (task % 49) / 7 - 3, m2 = task % 7 - 3;
        const double b = g.beta[nleg];
        g.dterm[t][task % 49] = (R)wigner_small(T.term_l[t], m1, m2, cos(0.5 * b), sin(0.5 * b), seed_table(T));
    }
    __syncwarp();
}

// A rotation-table row (NCAN entries of a 16-byte aligned row) with vector loads
template <typename R, int NCAN> __device__ __forceinline__ void load_row(const R *row, R (&d)[NCAN])
{
    if constexpr (sizeof(R) == 4) {
        const float4 *v = reinterpret_cast<const float4 *>(row);
#pragma unroll
        for (int i = 0; i < (NCAN + 3) / 4; ++i) {
            const float4 x = v[i];
            if (4 * i + 0 < NCAN) d[4 * i + 0] = x.x;
            if (4 * i + 1 < NCAN) d[4 * i + 1] = x.y;
            if (4 * i + 2 < NCAN) d[4 * i + 2] = x.z;
            if (4 * i + 3 < NCAN) d[4 * i + 3] = x.w;
        }
    } else {
        const double2 *v = reinterpret_cast<const double2 *>(row);
#pragma unroll
        for (int i = 0; i < (NCAN + 1) / 2; ++i) {
            const double2 x = v[i];
            if (2 * i + 0 < NCAN) d[2 * i + 0] = x.x;
            if (2 * i + 1 < NCAN) d[2 * i + 1] = x.y;
        }
    }
}

// ------------------------------------------------------------------------------------------------ streaming F
// Accumulates the canonical entries of F~_k (before the Euler phase) for rows lam1 < NR, columns lam2 < NC.
// Scatterer k, gam leg k+1 (rho_in), gamtl leg k (rho_out), partial waves il = 1..ilx.  UNR unrolls the partial-wave
// loop (two steps per trip rotate the recursion's registers instead of copying them: 6 % faster for the forward
// kernel on B200; the adjoint's first sweep, under its higher register pressure, is faster rolled).  The products
// and the accumulation run as FP32-pair instructions (4.6 % faster on B200); the recursion stays scalar (pairing it
// measured slower).
template <typename R, int KIND, int NR, int NC, int UNR = 1>
__device__ __forceinline__ void accumulate_f(C2<R> (&acc)[RepTab<KIND, NR, NC>().n], const R *dhk,
                                             const C2<R> *tlk, int tstride, int ilx, C2<R> z_in, C2<R> z_out)
{
    constexpr RepTab<KIND, NR, NC> RT{};
    constexpr LamTab L = lamtab(KIND);
    constexpr int DS = dstride(L.MM);
    constexpr int NCAN = ncanon(L.MM);
    constexpr int CI = L.CI, CO = L.CO;
#pragma unroll
    for (int r = 0; r < RT.n; ++r) acc[r] = cz<R>();
    // spherical-wave recursion state: columns 1..CI of the gam leg, 1..CO of the gamtl leg; c[0][1] = 1 makes the
    // uniform step c[il+1][im] = c[il-1][im] - (2il-1) z (c[il][im] + c[il][im-1]) give FEFF's seeds
    C2<R> pi[CI + 1], ci[CI + 1], po[CO + 1], co[CO + 1];
#pragma unroll
    for (int j = 0; j <= CI; ++j) { pi[j] = cz<R>(); ci[j] = cz<R>(); }
#pragma unroll
    for (int j = 0; j <= CO; ++j) { po[j] = cz<R>(); co[j] = cz<R>(); }
    pi[1] = C2<R>{R(1), R(0)};
    ci[1] = C2<R>{R(1), R(0)};
    po[1] = C2<R>{R(1), R(0)};
    co[1] = C2<R>{R(1), R(0)};
    // t-matrix of the next two partial waves in flight (the table is read from L2)
    C2<R> t1 = tlk[tstride], t2 = ilx >= 2 ? tlk[(size_t)2 * tstride] : cz<R>();
#pragma unroll UNR
    for (int il = 1; il <= ilx; ++il) {
        const C2<R> t = t1;
        t1 = t2;
        if (il + 2 <= ilx) t2 = tlk[(size_t)(il + 2) * tstride];
        R d[NCAN];
        load_row<R, NCAN>(dhk + (size_t)il * DS, d);
        C2<R> tco[CO + 1];
#pragma unroll
        for (int j = 1; j <= CO; ++j) tco[j] = pmul(t, co[j]);
#pragma unroll
        for (int r = 0; r < RT.n; ++r) acc[r] = pfmr(pmul(ci[RT.ci[r]], tco[RT.co[r]]), d[RT.d[r]], acc[r]);
        // next partial wave
        const R w = R(2 * il - 1);
        const C2<R> wi = cscl(z_in, w), wo = cscl(z_out, w);
        C2<R> ni[CI + 1], no[CO + 1];
        ni[1] = cfms(wi, ci[1], pi[1]);
#pragma unroll
        for (int j = 2; j <= CI; ++j) ni[j] = cfms(wi, cadd(ci[j], ci[j - 1]), pi[j]);
        no[1] = cfms(wo, co[1], po[1]);
#pragma unroll
        for (int j = 2; j <= CO; ++j) no[j] = cfms(wo, cadd(co[j], co[j - 1]), po[j]);
#pragma unroll
        for (int j = 1; j <= CI; ++j) { pi[j] = ci[j]; ci[j] = ni[j]; }
#pragma unroll
        for (int j = 1; j <= CO; ++j) { po[j] = co[j]; co[j] = no[j]; }
    }
}

// e^{-i eta m} for m = -MM..MM from e^{-i eta}
template <typename R, int MM> __device__ __forceinline__ void phase_powers(C2<R> e1, C2<R> (&ph)[2 * MM + 1])
{
    ph[MM] = C2<R>{R(1), R(0)};
    C2<R> p = e1;
#pragma unroll
    for (int m = 1; m <= MM; ++m) {
        ph[MM + m] = p;
        ph[MM - m] = cconj(p);
        p = cmul(p, e1);
    }
}

// ------------------------------------------------------------------------------------------------ spherical waves
// c[il][im] of one leg for il <= ITM, with GPUPathStage._clm's truncation (stage.py:209-232): entries beyond the
// leg's partial-wave limit lxp1 vanish except c[1][1] = 1 and c[2][1] = 1 - z.
template <typename R, int ITM, int NCOL>
__device__ __forceinline__ void clm_small(C2<R> z, int lxp1, C2<R> (&c)[ITM + 1][NCOL + 1])
{
    C2<R> pv[NCOL + 1], cv[NCOL + 1];
#pragma unroll
    for (int j = 0; j <= NCOL; ++j) { pv[j] = cz<R>(); cv[j] = cz<R>(); c[0][j] = cz<R>(); }
    pv[1] = C2<R>{R(1), R(0)};
    cv[1] = C2<R>{R(1), R(0)};
#pragma unroll
    for (int il = 1; il <= ITM; ++il) {
#pragma unroll
        for (int j = 0; j <= NCOL; ++j) {
            const bool keep = (il <= lxp1) || (j == 1 && il <= 2);
            c[il][j] = keep ? cv[j] : cz<R>();
        }
        const C2<R> w = cscl(z, R(2 * il - 1));
        C2<R> nv[NCOL + 1];
        nv[0] = cz<R>();
        nv[1] = cfms(w, cv[1], pv[1]);
#pragma unroll
        for (int j = 2; j <= NCOL; ++j) nv[j] = cfms(w, cadd(cv[j], cv[j - 1]), pv[j]);
#pragma unroll
        for (int j = 1; j <= NCOL; ++j) { pv[j] = cv[j]; cv[j] = nv[j]; }
    }
}

// ------------------------------------------------------------------------------------------------ termination
// Tr(T Q) with the termination matrix of mmtrxi/mmtr (genfmt.py:346-392; stage.py:318-335): gam from leg 1,
// (2l+1)-weighted gamtl from leg nleg, d^{l}(beta_nleg), the final-state weights and e^{-i eta_1 m1}.
// Q(b, a) returns entry (b, a) of the chain product for a, b < N0.
// Only the rows a_lo <= a < a_hi of T enter (the single-scattering column path passes one row at a time).
template <typename R, int KIND, class QF>
__device__ __forceinline__ C2<R> termination(const WarpPath<R> &g, const Tables<R> &T, int e, int nleg, C2<R> ck,
                                             const QF &Q, int a_lo = 0, int a_hi = kLamTot)
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N0 = L.N0, MM = L.MM;
    // columns up to |m| + n + 1 of leg 1 (CI) and n + 1 of leg nleg (CO) enter
    constexpr int ITM = L.IT, CI = L.CI, CO = L.CO;
    const int E = T.E;
    const int la = T.lmax[g.ip[0] * E + e], l1 = T.lmax[g.ip[1] * E + e], ln = T.lmax[g.ip[nleg - 1] * E + e];
    const int lx1 = max(la, l1) + 1, lxn = max(ln, la) + 1;
    const C2<R> r1 = cscl(ck, (R)g.ri[1]), rn = cscl(ck, (R)g.ri[nleg]);
    C2<R> c1[ITM + 1][CI + 1], cn[ITM + 1][CO + 1];
    clm_small<R, ITM, CI>(zfac(r1), lx1, c1);
    clm_small<R, ITM, CO>(zfac(rn), lxn, cn);
    C2<R> ph1[2 * MM + 1];
    phase_powers<R, MM>(g.phs[1], ph1);
    C2<R> ptrac = cz<R>();
    for (int t = 0; t < lamtab(KIND).NT && t < T.nterm; ++t) {
        const int il = T.term_l[t] + 1;
        const C2<R> W = T.wt[t * E + e];
        C2<R> G1[N0], G2[N0];
#pragma unroll
        for (int i = 0; i < N0; ++i) {
            const int am = L.m[i] < 0 ? -L.m[i] : L.m[i];
            const bool ok = am + 1 <= il;
            const int imn = am + L.n[i] + 1, in = L.n[i] + 1;
            C2<R> cv1 = cz<R>(), cvn = cz<R>();
#pragma unroll
            for (int q = 1; q <= ITM; ++q)
                if (q == il) { cv1 = c1[q][imn]; cvn = cn[q][in]; }
            const R xn = (R)T.xnlm[il * 8 + am + 1];
            const R f1 = (am & 1) ? -xn : xn;
            const R f2 = ok ? (R)(2 * il - 1) / xn : R(0);
            G1[i] = (ok && imn <= il) ? cscl(cv1, f1) : cz<R>();
            G2[i] = cscl(cvn, f2);
        }
        C2<R> s = cz<R>();
#pragma unroll
        for (int a = 0; a < N0; ++a) {
            if (a < a_lo || a >= a_hi) continue;
            C2<R> x = cz<R>();
#pragma unroll
            for (int b = 0; b < N0; ++b) x = cfma(cscl(G2[b], g.dterm[t][(L.m[a] + 3) * 7 + L.m[b] + 3]), Q(b, a), x);
            s = cfma(cmul(ph1[L.m[a] + MM], G1[a]), x, s);
        }
        ptrac = cfma(W, s, ptrac);
    }
    return ptrac;
}

// cfac = exp(i (sum rho - 2 xk reff)) / prod rho = exp(2 i reff (ck - xk)) / (ck^nleg prod ri) (stage.py:336-337),
// the argument in FP64.
template <typename R>
__device__ __forceinline__ C2<R> cfac(const WarpPath<R> &g, const Tables<R> &T, int e, int nleg, C2<R> ck)
{
    const double2 dk = T.dk[e];
    const double r2 = 2.0 * g.reff;
    double ph = r2 * dk.x;
    const double mag = exp(-r2 * dk.y);
    C2<R> prho = C2<R>{R(1), R(0)};
    for (int j = 1; j <= nleg; ++j) prho = cmul(prho, cscl(ck, (R)g.ri[j]));
    C2<R> ex;
    if constexpr (sizeof(R) == 4) {
        ph = ph - 6.283185307179586 * rint(ph * 0.15915494309189535);
        float s, c;
        sincosf((float)ph, &s, &c);
        ex = C2<R>{(R)(mag * c), (R)(mag * s)};
    } else {
        double s, c;
        sincos(ph, &s, &c);
        ex = C2<R>{(R)(mag * c), (R)(mag * s)};
    }
    return cmul(ex, cinv(prho));
}

// ------------------------------------------------------------------------------------------------ one energy
// Paths with two or more scatterers (nleg >= 3).  Every scattering matrix is accumulated as a full lamx x lamx
// matrix -- the first matrix's columns beyond laml0x and the last one's rows beyond laml0x are computed and not
// used -- so that one unrolled loop serves the whole chain: measured on B200 the smaller instruction footprint
// outweighs the extra entries (57.4 vs 62.4 ms for the 2e5-path benchmark launch).
// One lane's t-matrix column t(ip, l, e), l = 1..ilx, into its column of a warp's staging tile (row stride 32
// entries), by asynchronous copies to shared memory; the lane waits for its own copies only.
template <typename R>
__device__ __forceinline__ void stage_t_column(C2<R> *tile_col, const C2<R> *tg, int E, int ilx)
{
    for (int il = 1; il <= ilx; ++il) {
        const unsigned s = (unsigned)__cvta_generic_to_shared(tile_col + il * 32);
        if constexpr (sizeof(C2<R>) == 8)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(tg + (size_t)il * E) : "memory");
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(tg + (size_t)il * E) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// tst: the warp's t-matrix staging tile ((L1 + 1) x 32 entries, shared memory) or null to read the table through L1.
template <typename R, int KIND>
__device__ C2<R> energy_ms(const WarpPath<R> &g, const R *dh, const Tables<R> &T, int e, int nleg,
                           C2<R> *tst = nullptr)
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N = L.N, N0 = L.N0, MM = L.MM, DS = dstride(MM);
    constexpr RepTab<KIND, N, N> RT{};
    const int E = T.E, nsc = nleg - 1;
    const size_t dleg = (size_t)(T.L1 + 1) * DS, tlip = (size_t)(T.L1 + 1) * E;
    const C2<R> ck = T.ck[e];
    if (fabs((double)ck.x) + fabs((double)ck.y) <= 1e-16) return cz<R>();
    C2<R> P[N][N0];
    for (int k = 1; k <= nsc; ++k) {
        C2<R> acc[RT.n];
        const int ip = g.ip[k];
        const int ilx = T.lmax[ip * E + e] + 1;
        const C2<R> *tk = T.tl + ip * tlip + e;
        int tstride = E;
        if (tst) {
            C2<R> *col = tst + (threadIdx.x & 31);
            stage_t_column<R>(col, tk, E, ilx);
            tk = col;
            tstride = 32;
        }
        accumulate_f<R, KIND, N, N, sizeof(R) == 4 ? 2 : 1>(acc, dh + (k - 1) * dleg, tk, tstride, ilx,
                                                           zfac(cscl(ck, (R)g.ri[k + 1])), zfac(cscl(ck, (R)g.ri[k])));
        mask_lambda<R, KIND, N, N>(acc, T.nlam);
        C2<R> ph[2 * MM + 1];
        phase_powers<R, MM>(g.phs[k + 1], ph);
        C2<R> Pn[N][N0];
#pragma unroll
        for (int a = 0; a < N; ++a)
#pragma unroll
            for (int b = 0; b < N0; ++b) {
                C2<R> s = cz<R>();
                if (k == 1) {
                    s = RT.sg[a][b] > 0 ? acc[RT.rep[a][b]] : cscl(acc[RT.rep[a][b]], R(-1));
                } else if (sizeof(R) == 8 || a < N0 || k < nsc) {
                    // the termination reads rows < N0 of the last product only (skipping the others: 1.2 % faster
                    // in FP32 on B200, 0.7 % slower in FP64, where it is not done)
#pragma unroll
                    for (int c = 0; c < N; ++c) {
                        const C2<R> f = acc[RT.rep[a][c]];
                        s = RT.sg[a][c] > 0 ? cfma(f, P[c][b], s) : cfms(f, P[c][b], s);
                    }
                }
                Pn[a][b] = cmul(ph[L.m[a] + MM], s);
            }
#pragma unroll
        for (int a = 0; a < N; ++a)
#pragma unroll
            for (int b = 0; b < N0; ++b) P[a][b] = Pn[a][b];
    }
    const C2<R> ptrac = termination<R, KIND>(g, T, e, nleg, ck, [&](int b, int a) { return P[b][a]; });
    return cmul(ptrac, cfac(g, T, e, nleg, ck));
}
// Single scattering (nleg = 2), K edge: the six-entry set, flip-symmetric accumulation.
template <typename R, int KIND>
__device__ C2<R> energy_ss_sym(const WarpPath<R> &g, const R *dh, const Tables<R> &T, int e)
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N = L.N, N0 = L.N0, MM = L.MM;
    const int E = T.E;
    const size_t tlip = (size_t)(T.L1 + 1) * E;
    const C2<R> ck = T.ck[e];
    if (fabs((double)ck.x) + fabs((double)ck.y) <= 1e-16) return cz<R>();
    constexpr RepTab<KIND, N, N0> RT{};
    C2<R> acc[RT.n];
    const int ip = g.ip[1];
    accumulate_f<R, KIND, N, N0, sizeof(R) == 4 ? 2 : 1>(acc, dh, T.tl + ip * tlip + e, E, T.lmax[ip * E + e] + 1,
                                 zfac(cscl(ck, (R)g.ri[2])), zfac(cscl(ck, (R)g.ri[1])));
    C2<R> ph[2 * MM + 1];
    phase_powers<R, MM>(g.phs[2], ph);
    const C2<R> ptrac = termination<R, KIND>(g, T, e, 2, ck, [&](int b, int a) {
        const C2<R> v = RT.sg[b][a] > 0 ? acc[RT.rep[b][a]] : cscl(acc[RT.rep[b][a]], R(-1));
        return cmul(ph[L.m[b] + MM], v);
    });
    return cmul(ptrac, cfac(g, T, e, 2, ck));
}

// Single scattering at L and M edges (fifteen-entry sets): one column of F at a time, each with its own sweep
// over the partial waves, so that the accumulators stay in registers.
template <typename R, int KIND>
__device__ C2<R> energy_ss_col(const WarpPath<R> &g, const R *dh, const Tables<R> &T, int e)
{
    constexpr LamTab L = lamtab(KIND);
    constexpr int N = L.N, MM = L.MM, DS = dstride(MM), CI = L.CI, CO = L.CO;
    const int E = T.E;
    const size_t tlip = (size_t)(T.L1 + 1) * E;
    const C2<R> ck = T.ck[e];
    if (fabs((double)ck.x) + fabs((double)ck.y) <= 1e-16) return cz<R>();
    const int ip = g.ip[1];
    const C2<R> *tlk = T.tl + ip * tlip + e;
    const int ilx = T.lmax[ip * E + e] + 1;
    const C2<R> z_in = zfac(cscl(ck, (R)g.ri[2])), z_out = zfac(cscl(ck, (R)g.ri[1]));
    C2<R> ph[2 * MM + 1];
    phase_powers<R, MM>(g.phs[2], ph);
    C2<R> ptrac = cz<R>();
#pragma unroll 1
    for (int col = 0; col < N; ++col) {
        int m2 = 0, n2 = 0;
#pragma unroll
        for (int q = 0; q < N; ++q)
            if (q == col) { m2 = L.m[q]; n2 = L.n[q]; }
        C2<R> acc[N];
#pragma unroll
        for (int a = 0; a < N; ++a) acc[a] = cz<R>();
        C2<R> pi[CI + 1], ci[CI + 1], po[CO + 1], co[CO + 1];
#pragma unroll
        for (int j = 0; j <= CI; ++j) { pi[j] = cz<R>(); ci[j] = cz<R>(); }
#pragma unroll
        for (int j = 0; j <= CO; ++j) { po[j] = cz<R>(); co[j] = cz<R>(); }
        pi[1] = ci[1] = po[1] = co[1] = C2<R>{R(1), R(0)};
        for (int il = 1; il <= ilx; ++il) {
            const C2<R> t = tlk[(size_t)il * E];
            const R *dr = dh + (size_t)il * DS;
            C2<R> tco = cz<R>();
#pragma unroll
            for (int j = 1; j <= CO; ++j)
                if (j == n2 + 1) tco = cmul(t, co[j]);
#pragma unroll
            for (int a = 0; a < N; ++a) {
                const int m1 = L.m[a];
                const int am = m1 < 0 ? -m1 : m1;
                const bool can = canonical(m1, m2);
                const int idx = can ? dcanon(MM, m1, m2) : dcanon(MM, -m1, -m2);
                R dv = dr[idx];
                if (!can && ((m1 - m2) & 1)) dv = -dv;
                acc[a] = cfmr(cmul(ci[am + L.n[a] + 1], tco), dv, acc[a]);
            }
            const R w = R(2 * il - 1);
            const C2<R> wi = cscl(z_in, w), wo = cscl(z_out, w);
            C2<R> ni[CI + 1], no[CO + 1];
            ni[1] = cfms(wi, ci[1], pi[1]);
#pragma unroll
            for (int j = 2; j <= CI; ++j) ni[j] = cfms(wi, cadd(ci[j], ci[j - 1]), pi[j]);
            no[1] = cfms(wo, co[1], po[1]);
#pragma unroll
            for (int j = 2; j <= CO; ++j) no[j] = cfms(wo, cadd(co[j], co[j - 1]), po[j]);
#pragma unroll
            for (int j = 1; j <= CI; ++j) { pi[j] = ci[j]; ci[j] = ni[j]; }
#pragma unroll
            for (int j = 1; j <= CO; ++j) { po[j] = co[j]; co[j] = no[j]; }
        }
        // column col of Q = F: contributes sum_b T[col, b] Q[b, col]
        ptrac = cadd(ptrac, termination<R, KIND>(
                                g, T, e, 2, ck, [&](int b, int) { return cmul(ph[L.m[b] + MM], acc[b]); }, col, col + 1));
    }
    return cmul(ptrac, cfac(g, T, e, 2, ck));
}

}  // namespace fg
