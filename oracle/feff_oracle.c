/*
 * feff_oracle.c -- TEST INFRASTRUCTURE, not part of the product.
 *
 * A plain-C, FP64 restatement of the reference's path stage (FEFF 8.5L GENFMT as ported in nmarcella/feffGPU),
 * used only as the checker by the tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.
 * Nothing in feffgpu_b200/ links or calls it.
 *
 * One path at a time, one energy at a time, as the literal port does:
 *   geometry            src/feffgpu/genfmt.py:56-112   (trig, arg, pathgeom; ipol = 0), with the scattering
 *                       angle of src/feffgpu/stage.py:189-200
 *   lambda sets         src/feffgpu/genfmt.py:115-153  (setlam)
 *   normalisation       src/feffgpu/genfmt.py:41-53    (snlm)
 *   final-state coeffs  src/feffgpu/genfmt.py:230-264  (bcoef, unpolarised)
 *   hole -> kappa       src/feffgpu/genfmt.py:22-38    (setkap)
 *   spherical waves     src/feffgpu/genfmt.py:207-227  (sclmz)
 *   scattering matrix   src/feffgpu/genfmt.py:306-344  (fmtrxi)
 *   termination         src/feffgpu/genfmt.py:346-392  (mmtrxi, mmtr)
 *   path signal         src/feffgpu/genfmt.py:395-445  (chain product, trace, cfac)
 *   j-averaged t-matrix src/feffgpu/stage.py:111-118
 * Rotation matrices: the three-term recursion in l of src/feffgpu/stage.py:41-93 (wigner_d_small), not the
 * Edmonds recursion of genfmt.py:156-204 (rot3i).  Measured against a 80-digit evaluation of Wigner's sum at
 * beta = 2.1, rot3i's FP64 error grows to 2e-9 at l = 30, 1e-6 at l = 40 and 9e-5 at l = 47, the three-term
 * recursion stays below 1e-15; phase files reach l = 47 (the W set), so the stable form is the checker.
 *
 * Build: oracle/Makefile (gcc -O2 -pthread -shared -fPIC); paths are spread over POSIX threads.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <stdatomic.h>

#define MTOT 4
#define NTOT 2
#define LAMTOT 15
#define MMAX 3           /* |m| of the rotation matrices kept (stage.py:23) */
#define ND (2 * MMAX + 1)
#define EPS 1.0e-16
#define BOHR 0.52917721067

typedef double complex cplx;

/* Phase tables as the path stage sees them (first E = ne1 energies of the phase file). */
typedef struct {
    int E;              /* real-axis energies */
    int nph;            /* potentials 0..nph */
    int ltot;           /* ph index offset: l + ltot */
    int ihole;
    int iorder;
    const int32_t *lmax; /* (E, nph+1): largest l with a non-negligible phase shift */
    const double *ph;    /* (E, 2*ltot+1, nph+1) complex, interleaved re/im */
    const double *xk;    /* (E) real momentum relative to the edge, bohr^-1 */
    const double *ck;    /* (E) complex momentum, interleaved */
    const double *rkk;   /* (E, 8) complex reduced matrix elements, interleaved */
} fo_phase;

/* ---------------------------------------------------------------- small tables */

static int setkap(int ihole, int *kinit, int *linit)
{
    /* genfmt.py:22-38 */
    static const int k1[] = {1, 2, 5, 10, 17, 24, 27}, k2[] = {3, 6, 11, 18, 25, 30}, k3[] = {4, 7, 12, 19, 26},
                     k4[] = {8, 13, 20, 27}, k5[] = {9, 14, 21, 28}, k6[] = {15, 22}, k7[] = {16, 23};
#define IN(a) for (size_t i_ = 0; i_ < sizeof(a) / sizeof(a[0]); ++i_) if (a[i_] == ihole)
    IN(k1) { *kinit = -1; *linit = 0; return 0; }
    IN(k2) { *kinit = 1; *linit = 1; return 0; }
    IN(k3) { *kinit = -2; *linit = 1; return 0; }
    IN(k4) { *kinit = 2; *linit = 2; return 0; }
    IN(k5) { *kinit = -3; *linit = 2; return 0; }
    IN(k6) { *kinit = 3; *linit = 3; return 0; }
    IN(k7) { *kinit = -4; *linit = 3; return 0; }
#undef IN
    return -1;
}

/* xnlm[il][im], 1-based, il <= lmaxp1, im <= min(mmaxp1, il) (genfmt.py:41-53) */
static void snlm(int lmaxp1, int mmaxp1, double *xnlm /* (lmaxp1+1) x (mmaxp1+1) */)
{
    const double afac = 1.0 / 64.0;
    double flg[211];
    flg[0] = 1.0;
    flg[1] = afac;
    for (int i = 2; i < 211; ++i) flg[i] = flg[i - 1] * i * afac;
    memset(xnlm, 0, sizeof(double) * (lmaxp1 + 1) * (mmaxp1 + 1));
    for (int il = 1; il <= lmaxp1; ++il)
        for (int im = 1; im <= (mmaxp1 < il ? mmaxp1 : il); ++im) {
            int l = il - 1, m = im - 1;
            xnlm[il * (mmaxp1 + 1) + im] = sqrt((2 * l + 1) * flg[l - m] / flg[l + m]) * pow(afac, m);
        }
}

/* lind[1..8] (-1 = unphysical) and the spin-traced diagonal bdiag[1..8], ipol = 0, le2 = 0 (genfmt.py:230-264) */
static void bcoef(int kinit, int lind[9], double bdiag[9])
{
    const int lx = 4, le2 = 0;
    for (int i = 0; i < 9; ++i) { lind[i] = 0; bdiag[i] = 0.0; }
    for (int k = -1; k <= 1; ++k) {
        int kap = kinit + k;
        if (k == 0) kap = -kap;
        int lkap = kap > 0 ? kap : abs(kap) - 1;
        if (lkap > lx) lkap = -1;
        lind[k + 2] = lkap;
    }
    for (int k = -2; k <= 2; ++k) {
        int jkap = abs(kinit) + k;
        if (jkap <= 0) jkap = 0;
        int kap = jkap;
        if (kinit < 0 && abs(k) != 1) kap = -jkap;
        if (kinit > 0 && abs(k) == 1) kap = -jkap;
        int lkap = kap > 0 ? kap : -kap - 1;
        if (lkap > lx || le2 == 0 || (le2 == 1 && abs(k) == 2)) lkap = -1;
        lind[k + 6] = lkap;
    }
    for (int k = 1; k <= 8; ++k) {
        if (lind[k] < 0) continue;
        int i2 = (le2 == 2 && k > 3) ? 5 : 3;
        double v = 0.5 / (2 * lind[k] + 1.0) / i2;
        bdiag[k] = 2.0 * (k <= 3 ? -v : v);   /* trace over the two spin projections */
    }
}

typedef struct {
    int mlam[LAMTOT + 1], nlam[LAMTOT + 1];
    int lamx, laml0x, mmaxp1, nmax;
} lamset;

/* genfmt.py:115-153 */
static int setlam(int iorder, int nsc, int ilinit, lamset *L)
{
    int mmax, nmax, iord;
    if (nsc == 1) {
        mmax = nmax = ilinit;
        iord = 2 * nmax + mmax;
    } else if (iorder < 10) {
        iord = iorder; mmax = iorder; nmax = iorder / 2;
    } else {
        return -2;
    }
    int m0[LAMTOT], n0[LAMTOT], cnt = 0, filled = 0;
    for (int n = 0; n <= nmax && !filled; ++n)
        for (int m = 0; m <= mmax; ++m) {
            if (2 * n + m > iord) continue;
            if (cnt >= LAMTOT) { filled = 1; break; }
            m0[cnt] = -m; n0[cnt] = n; ++cnt;
            if (m == 0) continue;
            if (cnt >= LAMTOT) { filled = 1; break; }
            m0[cnt] = m; n0[cnt] = n; ++cnt;
        }
    L->lamx = cnt;
    int k = 1;
    for (int i = 0; i < cnt; ++i)
        if (n0[i] <= ilinit && abs(m0[i]) <= ilinit) { L->mlam[k] = m0[i]; L->nlam[k] = n0[i]; ++k; }
    L->laml0x = k - 1;
    for (int i = 0; i < cnt; ++i)
        if (!(n0[i] <= ilinit && abs(m0[i]) <= ilinit)) { L->mlam[k] = m0[i]; L->nlam[k] = n0[i]; ++k; }
    L->mlam[0] = L->nlam[0] = 0;
    int mx = 0, nx = 0;
    for (int i = 1; i <= cnt; ++i) {
        if (L->mlam[i] + 1 > mx) mx = L->mlam[i] + 1;
        if (L->nlam[i] > nx) nx = L->nlam[i];
    }
    L->mmaxp1 = mx;
    L->nmax = nx;
    if (nx > NTOT || mx > MTOT + 1) return -1;
    return 0;
}

/* ---------------------------------------------------------------- geometry (genfmt.py:56-112) */

static void trig(const double v[3], double *ct, double *st, double *cp, double *sp)
{
    double x = v[0], y = v[1], z = v[2];
    double r = sqrt(x * x + y * y + z * z), rxy = sqrt(x * x + y * y);
    if (r < 1e-6) { *ct = 1.0; *st = 0.0; } else { *ct = z / r; *st = rxy / r; }
    if (rxy < 1e-6) { *cp = (*ct >= 0) ? 1.0 : -1.0; *sp = 0.0; } else { *cp = x / rxy; *sp = y / rxy; }
}

static double arg_fi(double x, double y, double fi)
{
    if (fabs(x) < 1e-6) x = 0.0;
    if (fabs(y) < 1e-6) y = 0.0;
    return (x == 0.0 && y == 0.0) ? fi : atan2(y, x);
}

/* rat[j][3], j = 0..nleg (rat[0] = absorber copy, rat[nleg] = absorber); ri, beta 1..nleg; eta 0..nleg+1 */
static void pathgeom(double (*rat)[3], int nleg, double *ri, double *beta, double *eta)
{
    int nsc = nleg - 1;
    double alpha[16], gamma[16];
    for (int j = 0; j < nleg + 2; ++j) { ri[j] = beta[j] = eta[j] = alpha[j] = gamma[j] = 0.0; }
    for (int j = 1; j <= nleg; ++j) {
        int i, ip1, im1;
        if (j == nsc + 1) { i = 0; ip1 = 1; im1 = nsc; } else { i = j; ip1 = j + 1; im1 = j - 1; }
        double a[3], b[3];
        for (int c = 0; c < 3; ++c) { a[c] = rat[ip1][c] - rat[i][c]; b[c] = rat[i][c] - rat[im1][c]; }
        double ctp, stp, cpp, spp, ct, st, cp, sp;
        trig(a, &ctp, &stp, &cpp, &spp);
        trig(b, &ct, &st, &cp, &sp);
        double cppp = cp * cpp + sp * spp, sppp = spp * cp - cpp * sp;
        double phi = atan2(sp, cp), phip = atan2(spp, cpp);
        /* alph = -(st ctp - ct stp cppp - i stp sppp), gamm = -(st ctp cppp - ct stp + i st sppp) */
        double ax = -(st * ctp - ct * stp * cppp), ay = stp * sppp;
        double gx = -(st * ctp * cppp - ct * stp), gy = -st * sppp;
        double bb = ct * ctp + st * stp * cppp;
        if (bb > 1.0) bb = 1.0;
        if (bb < -1.0) bb = -1.0;
        double a_j = arg_fi(ax, ay, phip - phi);
        double g_j = arg_fi(gx, gy, 0.0);
        /* beta = atan2(|u1 x u2|, u1.u2) as stage.py:189-200 computes it; genfmt.py:104's acos(b) loses accuracy
         * near 0 and pi (FEFF's 6-decimal path coordinates make collinear legs 1e-7 rad off straight) */
        double u1[3] = {st * cp, st * sp, ct}, u2[3] = {stp * cpp, stp * spp, ctp};
        double wx = u1[1] * u2[2] - u1[2] * u2[1], wy = u1[2] * u2[0] - u1[0] * u2[2], wz = u1[0] * u2[1] - u1[1] * u2[0];
        beta[j] = atan2(sqrt(wx * wx + wy * wy + wz * wz + 1e-30), bb);
        alpha[j] = M_PI - g_j;
        gamma[j] = M_PI - a_j;
        ri[j] = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    }
    alpha[0] = alpha[nleg];
    for (int j = 1; j <= nleg; ++j) eta[j] = alpha[j - 1] + gamma[j];
}

/* ---------------------------------------------------------------- rotation matrices */

static double fact(int n) { double f = 1.0; for (int i = 2; i <= n; ++i) f *= i; return f; }

/* Wigner's explicit sum for the l = 3 seeds with |m| or |n| = 3 (stage.py:26-38) */
static double wigner_explicit(double beta, int l, int m, int n)
{
    double c2 = cos(beta / 2), s2 = sin(beta / 2), out = 0.0;
    double pref = sqrt(fact(l + m) * fact(l - m) * fact(l + n) * fact(l - n));
    for (int k = 0; k <= 2 * l; ++k) {
        int a = l + n - k, b = k, c = m - n + k, d = l - m - k;
        if (a < 0 || b < 0 || c < 0 || d < 0) continue;
        double coef = (((m - n + k) & 1) ? -1.0 : 1.0) * pref / (fact(a) * fact(b) * fact(c) * fact(d));
        out += coef * pow(c2, 2 * l + n - m - 2 * k) * pow(s2, m - n + 2 * k);
    }
    return out;
}

/* d[l][m+MMAX][n+MMAX], l = 0..lmax (stage.py:41-93: closed forms at l = 1, 2, explicit |m| = 3 seeds at l = 3,
 * three-term recursion in l otherwise) */
static void wigner_d(double beta, int lmax, double *d /* (lmax+1) * ND * ND */)
{
    const int o = MMAX;
    double c = cos(beta), s = sin(beta), c2 = cos(beta / 2), s2 = sin(beta / 2);
    memset(d, 0, sizeof(double) * (lmax + 1) * ND * ND);
#define D(l, m, n) d[((l) * ND + (m) + o) * ND + (n) + o]
    D(0, 0, 0) = 1.0;
    if (lmax >= 1) {
        D(1, 1, 1) = c2 * c2;
        D(1, 1, 0) = -s / sqrt(2.0);
        D(1, 1, -1) = s2 * s2;
        D(1, 0, 1) = s / sqrt(2.0);
        D(1, 0, 0) = c;
        D(1, 0, -1) = -s / sqrt(2.0);
        D(1, -1, 1) = s2 * s2;
        D(1, -1, 0) = s / sqrt(2.0);
        D(1, -1, -1) = c2 * c2;
    }
    if (lmax >= 2) {
        struct { int m, n; double v; } t[9] = {
            {2, 2, pow(c2, 4)}, {2, 1, -(1 + c) / 2 * s}, {2, 0, sqrt(3.0 / 8.0) * s * s}, {2, -1, -(1 - c) / 2 * s},
            {2, -2, pow(s2, 4)}, {1, 1, (1 + c) / 2 * (2 * c - 1)}, {1, 0, -sqrt(1.5) * s * c},
            {1, -1, (1 - c) / 2 * (2 * c + 1)}, {0, 0, (3 * c * c - 1) / 2}};
        for (int i = 0; i < 9; ++i) {
            int m = t[i].m, n = t[i].n;
            double v = t[i].v, sg = ((m - n) & 1) ? -1.0 : 1.0;
            D(2, m, n) = v;
            D(2, n, m) = sg * v;
            D(2, -m, -n) = sg * v;
            D(2, -n, -m) = v;
        }
    }
    for (int l = 2; l < lmax; ++l) {
        for (int m = -MMAX; m <= MMAX; ++m)
            for (int n = -MMAX; n <= MMAX; ++n) {
                double a1 = (double)l * l - m * m, a2 = (double)l * l - n * n;
                double a = (l + 1) * sqrt((a1 > 0 ? a1 : 0) * (a2 > 0 ? a2 : 0));
                double b = (2 * l + 1) * (l * (l + 1) * c - m * n);
                double p = ((double)(l + 1) * (l + 1) - m * m) * ((double)(l + 1) * (l + 1) - n * n);
                double den = l * sqrt(p > 0 ? p : 0);
                if (den == 0.0) den = 1.0;
                D(l + 1, m, n) = (b * D(l, m, n) - a * D(l - 1, m, n)) / den;
            }
        if (l + 1 == 3)
            for (int m = -3; m <= 3; ++m)
                for (int n = -3; n <= 3; ++n)
                    if (abs(m) == 3 || abs(n) == 3) D(3, m, n) = wigner_explicit(beta, 3, m, n);
    }
#undef D
}

/* ---------------------------------------------------------------- spherical-wave factors (genfmt.py:207-227) */

#define NCM (MTOT + NTOT + 2)
static void sclmz(cplx rho, int lmaxp1, int mmaxp1, int ldim, cplx *clmi /* ldim x NCM */)
{
    for (int i = 0; i < ldim * NCM; ++i) clmi[i] = 0;
#define C(il, im) clmi[(il) * NCM + (im)]
    cplx z = -I / rho, cmm = 1.0;
    C(1, 1) = 1.0;
    C(2, 1) = C(1, 1) - z;
    int lmax = lmaxp1 - 1;
    for (int il = 2; il <= lmax; ++il) C(il + 1, 1) = C(il - 1, 1) - z * (2 * il - 1) * C(il, 1);
    int mmxp1 = mmaxp1 < lmaxp1 ? mmaxp1 : lmaxp1;
    for (int im = 2; im <= mmxp1; ++im) {
        int m = im - 1, imp1 = im + 1;
        cmm = -cmm * (2 * m - 1) * z;
        C(im, im) = cmm;
        C(imp1, im) = cmm * (2 * m + 1) * (1.0 - im * z);
        for (int il = imp1; il <= lmax; ++il) {
            int l = il - 1;
            C(il + 1, im) = C(l, im) - (2 * l + 1) * z * (C(il, im) + C(il, m));
        }
    }
#undef C
}

/* ---------------------------------------------------------------- one path */

typedef struct {
    const fo_phase *P;
    int L1;            /* largest lmax + 1 over the energies and potentials */
    int ldim;          /* il dimension of the c and d arrays */
    int kinit, ilinit;
    int lind[9];
    double bdiag[9];
    double *xnlm;      /* ldim x (MTOT+2) */
    cplx *tl;          /* (E, L1+1, nph+1) j-averaged t-matrix, il = l+1 */
} ctx;

#define XN(il, im) C->xnlm[(il) * (MTOT + 2) + (im)]

static void path_cchi(const ctx *C, int nleg, const double *coords, const int64_t *ipots, double *out, double *reff_out,
                      double *dwork, cplx *cwork)
{
    const fo_phase *P = C->P;
    const int E = P->E, nsc = nleg - 1, nph1 = P->nph + 1, ldim = C->ldim;
    double rat[16][3];
    for (int c = 0; c < 3; ++c) {
        for (int j = 1; j < nleg; ++j) rat[j][c] = coords[j * 3 + c] / BOHR;
        rat[nleg][c] = coords[c] / BOHR;
        rat[0][c] = coords[c] / BOHR;
    }
    int ipot[16];
    for (int j = 1; j < nleg; ++j) ipot[j] = (int)ipots[j];
    ipot[nleg] = (int)ipots[0];
    ipot[0] = ipot[nleg];
    double ri[16], beta[16], eta[16];
    pathgeom(rat, nleg, ri, beta, eta);
    double reff = 0.0;
    for (int j = 1; j <= nleg; ++j) reff += ri[j];
    reff /= 2;
    *reff_out = reff * BOHR;

    lamset L;
    setlam(P->iorder, nsc, C->ilinit, &L);
    const int lamx = L.lamx, laml0x = L.laml0x, mnmxp1 = L.mmaxp1 + L.nmax;

    /* d^l(beta_j) for every leg, l = 0..L1-1 */
    double *dl = dwork;   /* (nleg+1) x L1 x ND x ND */
    const size_t dsz = (size_t)C->L1 * ND * ND;
    for (int j = 1; j <= nleg; ++j) wigner_d(beta[j], C->L1 - 1, dl + j * dsz);
#define DL(j, il, m1, m2) dl[(j) * dsz + (((il) - 1) * ND + (m1) + MMAX) * ND + (m2) + MMAX]

    cplx *clmi = cwork;                                   /* (nleg+1) x ldim x NCM */
    cplx *gam = clmi + (nleg + 1) * ldim * NCM;          /* ldim x (MTOT+2) x (NTOT+2) */
    cplx *gamtl = gam + ldim * (MTOT + 2) * (NTOT + 2);
    cplx *fm = gamtl + ldim * (MTOT + 2) * (NTOT + 2);   /* (LAMTOT+1)^2 x (nleg+1) */
#define CL(j, il, im) clmi[((j) * ldim + (il)) * NCM + (im)]
#define G(a, il, im, in) a[((il) * (MTOT + 2) + (im)) * (NTOT + 2) + (in)]
#define FM(l1, l2, k) fm[(((k) * (LAMTOT + 1)) + (l1)) * (LAMTOT + 1) + (l2)]

    int valid_lo = 99, valid_hi = -1;
    for (int k = 1; k <= 8; ++k)
        if (C->lind[k] >= 0) {
            if (C->lind[k] < valid_lo) valid_lo = C->lind[k];
            if (C->lind[k] > valid_hi) valid_hi = C->lind[k];
        }
    const int lxx = MTOT < C->ilinit ? MTOT : C->ilinit;

    for (int ie = 0; ie < E; ++ie) {
        cplx ck = P->ck[2 * ie] + I * P->ck[2 * ie + 1];
        out[2 * ie] = out[2 * ie + 1] = 0.0;
        if (cabs(ck) <= EPS) continue;
        cplx rho[16];
        for (int j = 1; j <= nleg; ++j) rho[j] = ck * ri[j];
        for (int ileg = 1; ileg <= nleg; ++ileg) {
            int isc0 = ileg > 1 ? ileg - 1 : nleg;
            int la = P->lmax[ie * nph1 + ipot[isc0]] + 1, lb = P->lmax[ie * nph1 + ipot[ileg]] + 1;
            int lxp1 = la > lb ? la : lb;
            int mnp1 = lxp1 < mnmxp1 ? lxp1 : mnmxp1;
            sclmz(rho[ileg], lxp1, mnp1, ldim, &CL(ileg, 0, 0));
        }
        memset(fm, 0, sizeof(cplx) * (LAMTOT + 1) * (LAMTOT + 1) * (nleg + 1));

        /* fmtrxi (genfmt.py:306-344) for the pairs (ileg, ilegp) = (2,1), (nleg, nleg-1), (ilegp+1, ilegp) */
        for (int pass = 0; pass < nleg - 1; ++pass) {
            int ileg, ilegp, lam1x, lam2x;
            if (pass == 0) { ileg = 2; ilegp = 1; lam1x = lamx; lam2x = laml0x; }
            else if (pass == 1) { ileg = nleg; ilegp = nleg - 1; lam1x = laml0x; lam2x = lamx; }
            else { ilegp = pass; ileg = pass + 1; lam1x = lamx; lam2x = lamx; }
            const int ip = ipot[ilegp];
            const int ilx = P->lmax[ie * nph1 + ip] + 1;
            memset(gam, 0, sizeof(cplx) * ldim * (MTOT + 2) * (NTOT + 2));
            memset(gamtl, 0, sizeof(cplx) * ldim * (MTOT + 2) * (NTOT + 2));
            const int lmx = lam1x > lam2x ? lam1x : lam2x;
            for (int il = 1; il <= ilx; ++il) {
                cplx t = C->tl[((size_t)ie * (C->L1 + 1) + il) * nph1 + ip];
                for (int lam = 1; lam <= lmx; ++lam) {
                    int m = L.mlam[lam];
                    if (m < 0) continue;
                    int im = m + 1;
                    if (im > il) continue;
                    int in = L.nlam[lam] + 1, imn = in + m;
                    if (lam <= lam1x)
                        G(gam, il, im, in) = imn <= il ? XN(il, im) * ((m & 1) ? -1.0 : 1.0) * CL(ileg, il, imn) : 0;
                    if (lam <= lam2x) G(gamtl, il, im, in) = t / XN(il, im) * CL(ilegp, il, in);
                }
            }
            for (int l1 = 1; l1 <= lam1x; ++l1) {
                int m1 = L.mlam[l1], in1 = L.nlam[l1] + 1, iam1 = abs(m1) + 1;
                for (int l2 = 1; l2 <= lam2x; ++l2) {
                    int m2 = L.mlam[l2], in2 = L.nlam[l2] + 1, iam2 = abs(m2) + 1;
                    int imn1 = iam1 + in1 - 1;
                    int ilmin = iam1;
                    if (iam2 > ilmin) ilmin = iam2;
                    if (imn1 > ilmin) ilmin = imn1;
                    if (in2 > ilmin) ilmin = in2;
                    cplx ct = 0;
                    for (int il = ilmin; il <= ilx; ++il) {
                        if (abs(m1) >= il || abs(m2) >= il) continue;
                        ct += G(gam, il, iam1, in1) * G(gamtl, il, iam2, in2) * DL(ilegp, il, m1, m2);
                    }
                    if (eta[ileg] != 0.0) ct *= cexp(-I * eta[ileg] * m1);
                    FM(l1, l2, ilegp) = ct;
                }
            }
            if (nleg == 2) break;
        }

        /* chain product: pmat = f(nleg,nleg-1) ... f(3,2) f(2,1) (genfmt.py:437-439) */
        cplx pm[LAMTOT + 1][LAMTOT + 1], tmp[LAMTOT + 1][LAMTOT + 1];
        for (int a = 1; a <= lamx; ++a)
            for (int b = 1; b <= laml0x; ++b) pm[a][b] = FM(a, b, 1);
        for (int isc = 2; isc < nleg; ++isc) {
            for (int a = 1; a <= lamx; ++a)
                for (int b = 1; b <= laml0x; ++b) {
                    cplx s = 0;
                    for (int c = 1; c <= lamx; ++c) s += FM(a, c, isc) * pm[c][b];
                    tmp[a][b] = s;
                }
            for (int a = 1; a <= lamx; ++a)
                for (int b = 1; b <= laml0x; ++b) pm[a][b] = tmp[a][b];
        }

        /* termination (mmtrxi + mmtr, genfmt.py:346-392): gam from leg 1, gamtl (2l+1) from leg nleg,
         * d(beta_nleg); bmati is diagonal in k, so the double sum over (k1, k2) keeps k1 = k2 */
        memset(gam, 0, sizeof(cplx) * ldim * (MTOT + 2) * (NTOT + 2));
        memset(gamtl, 0, sizeof(cplx) * ldim * (MTOT + 2) * (NTOT + 2));
        for (int il = valid_lo + 1; il <= valid_hi + 1; ++il) {
            double tt = 2 * il - 1;
            for (int lam = 1; lam <= laml0x; ++lam) {
                int m = L.mlam[lam];
                if (m < 0) continue;
                int im = m + 1;
                if (im > il) continue;
                int in = L.nlam[lam] + 1, imn = in + m;
                G(gam, il, im, in) = imn <= il ? XN(il, im) * ((m & 1) ? -1.0 : 1.0) * CL(1, il, imn) : 0;
                G(gamtl, il, im, in) = tt / XN(il, im) * CL(nleg, il, in);
            }
        }
        cplx ptrac = 0;
        for (int l1 = 1; l1 <= laml0x; ++l1) {
            int m1 = L.mlam[l1], in1 = L.nlam[l1] + 1, iam1 = abs(m1) + 1;
            for (int l2 = 1; l2 <= laml0x; ++l2) {
                int m2 = L.mlam[l2], in2 = L.nlam[l2] + 1, iam2 = abs(m2) + 1;
                cplx f = 0;
                if (abs(m1) <= lxx && abs(m2) <= lxx)
                    for (int k = 1; k <= 8; ++k) {
                        int lk = C->lind[k] + 1;
                        if (lk <= 0 || iam1 > lk || iam2 > lk) continue;
                        cplx r = P->rkk[2 * (ie * 8 + k - 1)] + I * P->rkk[2 * (ie * 8 + k - 1) + 1];
                        double dd = (abs(m1) < lk && abs(m2) < lk) ? DL(nleg, lk, m1, m2) : 0.0;
                        f += C->bdiag[k] * dd * r * r * G(gam, lk, iam1, in1) * G(gamtl, lk, iam2, in2);
                    }
                f *= cexp(-I * eta[1] * m1);
                ptrac += f * pm[l2][l1];
            }
        }
        cplx srho = 0, prho = 1;
        for (int j = 1; j <= nleg; ++j) { srho += rho[j]; prho *= rho[j]; }
        cplx cfac = cexp(I * (srho - 2 * P->xk[ie] * reff)) / prho;
        cplx cc = ptrac * cfac;
        out[2 * ie] = creal(cc);
        out[2 * ie + 1] = cimag(cc);
    }
#undef DL
#undef CL
#undef G
#undef FM
}

/* ---------------------------------------------------------------- public entry points */

typedef struct {
    const ctx *C;
    int nleg;
    int64_t B;
    const double *coords;
    const int64_t *ipots;
    double *cchi, *reff;
    atomic_long next;
} work;

/* Paths are handed out four at a time from a shared counter. */
static void *worker(void *arg)
{
    work *W = (work *)arg;
    const ctx *C = W->C;
    const int nleg = W->nleg, E = C->P->E;
    const size_t dsz = (size_t)(nleg + 1) * C->L1 * ND * ND;
    const size_t csz = (size_t)(nleg + 1) * C->ldim * NCM + 2 * (size_t)C->ldim * (MTOT + 2) * (NTOT + 2) +
                       (size_t)(LAMTOT + 1) * (LAMTOT + 1) * (nleg + 1);
    double *dw = (double *)malloc(sizeof(double) * dsz);
    cplx *cw = (cplx *)malloc(sizeof(cplx) * csz);
    for (;;) {
        long b0 = atomic_fetch_add(&W->next, 4);
        if (b0 >= W->B) break;
        for (long b = b0; b < b0 + 4 && b < W->B; ++b)
            path_cchi(C, nleg, W->coords + b * nleg * 3, W->ipots + b * nleg, W->cchi + 2 * b * E, W->reff + b, dw, cw);
    }
    free(dw);
    free(cw);
    return NULL;
}

/* Status: 0 ok, -1 invalid argument, -2 not implemented (icalc >= 10, bad hole). */
int fo_cchi(const fo_phase *P, int nleg, int64_t B, const double *coords /* (B, nleg, 3) A */,
            const int64_t *ipots /* (B, nleg) */, double *cchi /* (B, E) complex */, double *reff /* (B) A */,
            int nthreads)
{
    if (!P || nleg < 2 || nleg > 9 || B < 0) return -1;
    ctx C;
    C.P = P;
    if (setkap(P->ihole, &C.kinit, &C.ilinit)) return -2;
    C.ilinit += 1;
    lamset Lt;
    if (setlam(P->iorder, nleg - 1, C.ilinit, &Lt) == -2) return -2;
    const int nph1 = P->nph + 1;
    int lm = 0;
    for (int i = 0; i < P->E * nph1; ++i)
        if (P->lmax[i] > lm) lm = P->lmax[i];
    C.L1 = lm + 1;
    C.ldim = C.L1 + 2 > 6 ? C.L1 + 2 : 6;
    bcoef(C.kinit, C.lind, C.bdiag);
    C.xnlm = (double *)malloc(sizeof(double) * C.ldim * (MTOT + 2));
    snlm(C.ldim - 1, MTOT + 1, C.xnlm);
    C.tl = (cplx *)calloc((size_t)P->E * (C.L1 + 1) * nph1, sizeof(cplx));
    const int nl = 2 * P->ltot + 1;
    for (int ie = 0; ie < P->E; ++ie)
        for (int il = 1; il <= C.L1; ++il)
            for (int ip = 0; ip < nph1; ++ip) {
                int ll = il - 1;
                const double *pm = P->ph + 2 * (((size_t)ie * nl + (P->ltot - ll)) * nph1 + ip);
                const double *pp = P->ph + 2 * (((size_t)ie * nl + (P->ltot + ll)) * nph1 + ip);
                cplx dm = pm[0] + I * pm[1], dp = pp[0] + I * pp[1];
                cplx tm = (cexp(2 * I * dm) - 1) / (2 * I), tp = (cexp(2 * I * dp) - 1) / (2 * I);
                C.tl[((size_t)ie * (C.L1 + 1) + il) * nph1 + ip] = tm * (ll + 1) + tp * ll;
            }
    work W = {&C, nleg, B, coords, ipots, cchi, reff, 0};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    int started = 0;
    for (int t = 1; t < nthreads; ++t)
        if (pthread_create(&th[t], NULL, worker, &W) == 0) ++started; else break;
    worker(&W);
    for (int t = 1; t <= started; ++t) pthread_join(th[t], NULL);
    free(C.xnlm);
    free(C.tl);
    return 0;
}

/* The lambda set of a path with nsc scatterers (for the tests' bookkeeping). */
int fo_lambda(int ihole, int iorder, int nsc, int *mlam, int *nlam, int *sizes /* lamx, laml0x, mmaxp1, nmax */)
{
    int kinit, linit;
    if (setkap(ihole, &kinit, &linit)) return -2;
    lamset L;
    int rc = setlam(iorder, nsc, linit + 1, &L);
    if (rc) return rc;
    for (int i = 0; i <= L.lamx; ++i) { mlam[i] = L.mlam[i]; nlam[i] = L.nlam[i]; }
    sizes[0] = L.lamx; sizes[1] = L.laml0x; sizes[2] = L.mmaxp1; sizes[3] = L.nmax;
    return 0;
}

/* d^l_{mn}(beta), l = 0..lmax, |m|,|n| <= 3 (for the tests). */
void fo_wigner_d(double beta, int lmax, double *d) { wigner_d(beta, lmax, d); }

/* Leg lengths (A), angles and Euler sums of one path (for the tests). */
void fo_geometry(int nleg, const double *coords, double *ri, double *beta, double *eta)
{
    double rat[16][3];
    for (int c = 0; c < 3; ++c) {
        for (int j = 1; j < nleg; ++j) rat[j][c] = coords[j * 3 + c] / BOHR;
        rat[nleg][c] = rat[0][c] = coords[c] / BOHR;
    }
    double r[16], b[16], e[16];
    pathgeom(rat, nleg, r, b, e);
    for (int j = 0; j < nleg; ++j) { ri[j] = r[j + 1] * BOHR; beta[j] = b[j + 1]; eta[j] = e[j + 1]; }
}
