// fg_device.cuh -- device-side building blocks of the B200 path stage.
//
// Work decomposition: one warp owns one path at a time; its lanes own 32 consecutive energies of the phase file's
// real-axis grid and loop over the grid in chunks of 32.  Everything that depends on the path only (leg geometry,
// rotation matrices, Euler phases) is computed once per path by the warp into its own shared-memory slice; the
// energy-dependent work (spherical-wave recursions, scattering matrices, chain product, termination, cfac) runs
// per lane in registers.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace fg {

constexpr double kBohr = 0.52917721067;   // pad.py:13
constexpr int kMaxLeg = 9;                 // pathfinder.py:26 (NLEG_MAX)
constexpr int kLamTot = 15;                // genfmt.py:18

// Bits of the status word the per-path kernels raise (atomicOr) instead of reading out of bounds: a potential index
// outside 0..nph (clamped, as the reference's tables would raise IndexError), and a malformed batch layout (a path
// index, leg count, summation index or chunk offset outside its range; that path or term is skipped).
constexpr int kBadIpot = 1;
constexpr int kBadLayout = 2;
constexpr int kBadRange = 4;    // a weighted path term not finite or beyond the exact row sums' range (|v| >= 2^31)

// The fused stage's row sums: per path and k point the term is added to its row exactly, as a fixed-point number of
// resolution 2^-64 held in two 64-bit integer sums: a signed word of resolution 2^-32 (its additions wrap modulo
// 2^64, which leaves the final sum exact whenever the row itself is below 2^31) and a low word of the next 32 bits
// (non-negative, below 2^32 per term, so up to 2^31 terms cannot overflow it).  Integer addition is associative,
// so the rows do not depend on the order in which paths finish, the launch shape or the GPU.  (Measured on B200:
// 45.80 ms against 45.99 for per-path terms in memory summed in a fixed order afterwards on the 189,419-path benchmark
// batch, 137.5 against 149.1 ms on the 4.2e6-path MD batch, and no workspace beyond the rows.)
// Adds v to the fixed-point sum whose two words are a[0] and a[stride]; false (nothing added) if v is not finite or
// |v| >= 2^31.
__device__ __forceinline__ bool fixed_add(unsigned long long *a, size_t stride, double v)
{
    if (!(fabs(v) < 2147483648.0)) return false;
    const double x = v * 4294967296.0;                  // exact: v * 2^32, |x| < 2^63
    const double hi = floor(x);
    const double lo = rint((x - hi) * 4294967296.0);    // the next 32 bits, 0 <= lo <= 2^32; rounding below 2^-64
    atomicAdd(a, (unsigned long long)(long long)hi);
    atomicAdd(a + stride, (unsigned long long)lo);
    return true;
}

// ------------------------------------------------------------------------------------------------ complex helpers
template <typename R> struct C2 { R x, y; };

template <typename R> __device__ __forceinline__ C2<R> cz() { return C2<R>{R(0), R(0)}; }
template <typename R> __device__ __forceinline__ C2<R> cadd(C2<R> a, C2<R> b) { return C2<R>{a.x + b.x, a.y + b.y}; }
template <typename R> __device__ __forceinline__ C2<R> csub(C2<R> a, C2<R> b) { return C2<R>{a.x - b.x, a.y - b.y}; }
template <typename R> __device__ __forceinline__ C2<R> cmul(C2<R> a, C2<R> b)
{
    return C2<R>{fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x)};
}
template <typename R> __device__ __forceinline__ C2<R> cscl(C2<R> a, R r) { return C2<R>{a.x * r, a.y * r}; }
template <typename R> __device__ __forceinline__ C2<R> cconj(C2<R> a) { return C2<R>{a.x, -a.y}; }
// acc + a b
template <typename R> __device__ __forceinline__ C2<R> cfma(C2<R> a, C2<R> b, C2<R> acc)
{
    return C2<R>{fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y))};
}
// acc - a b
template <typename R> __device__ __forceinline__ C2<R> cfms(C2<R> a, C2<R> b, C2<R> acc)
{
    return C2<R>{fma(-a.x, b.x, fma(a.y, b.y, acc.x)), fma(-a.x, b.y, fma(-a.y, b.x, acc.y))};
}
// acc + a r
template <typename R> __device__ __forceinline__ C2<R> cfmr(C2<R> a, R r, C2<R> acc)
{
    return C2<R>{fma(a.x, r, acc.x), fma(a.y, r, acc.y)};
}
// acc + conj(a) b
template <typename R> __device__ __forceinline__ C2<R> cfmac(C2<R> a, C2<R> b, C2<R> acc)
{
    return C2<R>{fma(a.x, b.x, fma(a.y, b.y, acc.x)), fma(a.x, b.y, fma(-a.y, b.x, acc.y))};
}
template <typename R> __device__ __forceinline__ C2<R> cinv(C2<R> a)
{
    R d = R(1) / fma(a.x, a.x, a.y * a.y);
    return C2<R>{a.x * d, -a.y * d};
}
// Packed forms for the partial-wave loops: in FP32 each complex operation is issued as FP32-pair instructions
// (sm_100 FFMA2 / FMUL2 / FADD2, both components in one instruction); the broadcast and rotated operand pairs
// (a.x a.x), (a.y a.y), (-b.y b.x) are shared by the loops' repeated operands.  FP64 keeps the scalar forms.
__device__ __forceinline__ float2 pk(C2<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ C2<float> upk(float2 a) { return C2<float>{a.x, a.y}; }
__device__ __forceinline__ float2 bcast(float r) { return make_float2(r, r); }
__device__ __forceinline__ float2 rot(C2<float> b) { return make_float2(-b.y, b.x); }   // i b
// a b
template <typename R> __device__ __forceinline__ C2<R> pmul(C2<R> a, C2<R> b)
{
    if constexpr (sizeof(R) == 4)
        return upk(__ffma2_rn(bcast(a.y), rot(b), __fmul2_rn(bcast(a.x), pk(b))));
    else
        return cmul(a, b);
}
// acc + a r
template <typename R> __device__ __forceinline__ C2<R> pfmr(C2<R> a, R r, C2<R> acc)
{
    if constexpr (sizeof(R) == 4)
        return upk(__ffma2_rn(pk(a), bcast(r), pk(acc)));
    else
        return cfmr(a, r, acc);
}
// acc + a b
template <typename R> __device__ __forceinline__ C2<R> pfma(C2<R> a, C2<R> b, C2<R> acc)
{
    if constexpr (sizeof(R) == 4)
        return upk(__ffma2_rn(bcast(a.y), rot(b), __ffma2_rn(bcast(a.x), pk(b), pk(acc))));
    else
        return cfma(a, b, acc);
}
// acc - a b
template <typename R> __device__ __forceinline__ C2<R> pfms(C2<R> a, C2<R> b, C2<R> acc)
{
    if constexpr (sizeof(R) == 4)
        return upk(__ffma2_rn(bcast(-a.y), rot(b), __ffma2_rn(bcast(-a.x), pk(b), pk(acc))));
    else
        return cfms(a, b, acc);
}
template <typename R> __device__ __forceinline__ C2<R> padd(C2<R> a, C2<R> b)
{
    if constexpr (sizeof(R) == 4)
        return upk(__fadd2_rn(pk(a), pk(b)));
    else
        return cadd(a, b);
}

// -i / rho, the argument of FEFF's spherical-wave factors (genfmt.py:210)
template <typename R> __device__ __forceinline__ C2<R> zfac(C2<R> rho)
{
    R d = R(1) / fma(rho.x, rho.x, rho.y * rho.y);
    return C2<R>{-rho.y * d, -rho.x * d};
}

// ------------------------------------------------------------------------------------------------ lambda sets
// The lambda index sets of setlam (genfmt.py:115-153) in the order setlam leaves them: the laml0x entries that
// reach the final state lead.  kind 0: K edge, two or more scatterers; 1: L and M edges, two or more scatterers
// (iorder 2 gives the same six entries, all of them within the final state); 2/3/4: single scattering at K/L/M
// edges (mmax = nmax = l_init + 1, FEFF's LAMTOT = 15 truncates the M set); 5/6/7: two or more scatterers at
// iorder 3 (ten entries) at K/L/M edges.  Orders 0 and 1 use kinds 0 and 1 restricted to their first 3 and 1
// entries (mask_lambda).
struct LamTab {
    int N, N0, MM, CI, CO;
    int IT;                     // largest il = l + 1 of a final-state term: l_init + 2 (K and L1: 2, L2/L3: 3, M: 4)
    int NT;                     // distinct final-state l: 1 from an s level (K, L1), 2 otherwise (l_init +- 1)
    int m[kLamTot], n[kLamTot];
};

__host__ __device__ constexpr LamTab lamtab(int kind)
{
    LamTab t{};
    if (kind == 0 || kind == 1 || kind == 2) {
        const int mK[6] = {0, -1, 1, 0, -2, 2}, nK[6] = {0, 0, 0, 1, 0, 0};
        const int mL[6] = {0, -1, 1, -2, 2, 0}, nL[6] = {0, 0, 0, 0, 0, 1};
        const int mS[6] = {0, -1, 1, 0, -1, 1}, nS[6] = {0, 0, 0, 1, 1, 1};
        t.N = 6;
        t.N0 = kind == 0 ? 4 : 6;
        for (int i = 0; i < 6; ++i) {
            t.m[i] = kind == 0 ? mK[i] : (kind == 1 ? mL[i] : mS[i]);
            t.n[i] = kind == 0 ? nK[i] : (kind == 1 ? nL[i] : nS[i]);
        }
    } else if (kind >= 5 && kind <= 7) {
        // multiple scattering at order 3 (setlam, genfmt.py:115-153: m = 0, +-1, +-2, +-3 with n = 0 and m = 0, +-1
        // with n = 1), the entries within the final state of edge l_init + 1 = kind - 4 (n, |m| <= l_init + 1) first
        const int m0[10] = {0, -1, 1, -2, 2, -3, 3, 0, -1, 1}, n0[10] = {0, 0, 0, 0, 0, 0, 0, 1, 1, 1};
        const int il = kind - 4;
        int c = 0;
        for (int pass = 0; pass < 2; ++pass) {
            for (int i = 0; i < 10; ++i) {
                const int am = m0[i] < 0 ? -m0[i] : m0[i];
                const bool first = n0[i] <= il && am <= il;
                if (first == (pass == 0)) { t.m[c] = m0[i]; t.n[c] = n0[i]; ++c; }
            }
            if (pass == 0) t.N0 = c;
        }
        t.N = 10;
    } else {
        const int mmax = kind == 3 ? 2 : 3;
        int c = 0;
        for (int n = 0; n <= mmax && c < kLamTot; ++n)
            for (int m = 0; m <= mmax && c < kLamTot; ++m) {
                if (2 * n + m > 3 * (kind - 1)) continue;
                t.m[c] = -m; t.n[c] = n; ++c;
                if (m == 0 || c >= kLamTot) continue;
                t.m[c] = m; t.n[c] = n; ++c;
            }
        t.N = c;
        t.N0 = c;
    }
    t.IT = (kind == 0 || kind == 2 || kind == 5) ? 2 : ((kind == 3 || kind == 6) ? 3 : 4);
    t.NT = (kind == 0 || kind == 2 || kind == 5) ? 1 : 2;
    t.MM = 0; t.CI = 0; t.CO = 0;
    for (int i = 0; i < t.N; ++i) {
        int am = t.m[i] < 0 ? -t.m[i] : t.m[i];
        if (am > t.MM) t.MM = am;
        if (am + t.n[i] + 1 > t.CI) t.CI = am + t.n[i] + 1;
        if (t.n[i] + 1 > t.CO) t.CO = t.n[i] + 1;
    }
    return t;
}

__host__ __device__ constexpr bool canonical(int m1, int m2) { return m1 > 0 || (m1 == 0 && m2 >= 0); }
// Canonical (m1, m2) pairs are stored; d_{-m1,-m2} = (-1)^(m1-m2) d_{m1,m2} gives the others.
__host__ __device__ constexpr int dcanon(int MM, int m1, int m2)
{
    return m1 == 0 ? m2 : (MM + 1) + (m1 - 1) * (2 * MM + 1) + (m2 + MM);
}
// First energy of a path's loop over chunks of 32 energies (a lane per energy).  When E is not a multiple of 32 the
// partial chunk comes first, over the lowest energies, whose partial-wave limits are the smallest, rather than last,
// over the highest and most expensive: its idle lanes then wait on the cheapest chunk (for E = 401 the chunks are
// -15..16, 17..48, ..., 369..400).
__host__ __device__ constexpr int first_chunk(int E) { return (E % 32) ? (E % 32) - 32 : 0; }
__host__ __device__ constexpr int ncanon(int MM) { return (MM + 1) + MM * (2 * MM + 1); }
// Row stride of the rotation tables: the canonical entries rounded up to a 16-byte multiple of FP32 (and of FP64)
// so rows load as float4 / double2 (28 for MM = 3 instead of a 32-entry row: less shared memory per warp, more of
// the unified L1 left as cache for the t-matrix tables, whose hit rate the forward kernel is sensitive to).
__host__ __device__ constexpr int dstride(int MM) { return (ncanon(MM) + 3) & ~3; }

// Representatives of the scattering-matrix entries (lam1 < NR, lam2 < NC) under the flip (m1, m2) -> (-m1, -m2):
// the pre-phase matrix obeys F~[flip] = (-1)^(m1-m2) F~ because the spherical-wave factors depend on |m| only and
// the rotation matrix has that symmetry; only canonical entries are accumulated.
template <int KIND, int NR, int NC> struct RepTab {
    int n;
    int a[kLamTot * kLamTot], b[kLamTot * kLamTot], d[kLamTot * kLamTot], ci[kLamTot * kLamTot],
        co[kLamTot * kLamTot];
    int rep[kLamTot][kLamTot], sg[kLamTot][kLamTot];
    __host__ __device__ constexpr RepTab() : n(0), a{}, b{}, d{}, ci{}, co{}, rep{}, sg{}
    {
        const LamTab L = lamtab(KIND);
        for (int i = 0; i < NR; ++i)
            for (int j = 0; j < NC; ++j)
                if (canonical(L.m[i], L.m[j])) {
                    const int am = L.m[i] < 0 ? -L.m[i] : L.m[i];
                    a[n] = i; b[n] = j; d[n] = dcanon(L.MM, L.m[i], L.m[j]);
                    ci[n] = am + L.n[i] + 1; co[n] = L.n[j] + 1;
                    rep[i][j] = n; sg[i][j] = 1;
                    ++n;
                }
        for (int i = 0; i < NR; ++i)
            for (int j = 0; j < NC; ++j)
                if (!canonical(L.m[i], L.m[j])) {
                    int fi = 0, fj = 0;
                    for (int k = 0; k < L.N; ++k) {
                        if (L.m[k] == -L.m[i] && L.n[k] == L.n[i]) fi = k;
                        if (L.m[k] == -L.m[j] && L.n[k] == L.n[j]) fj = k;
                    }
                    rep[i][j] = rep[fi][fj];
                    sg[i][j] = ((L.m[i] - L.m[j]) & 1) ? -1 : 1;
                }
    }
};

// The multiple-scattering lambda set of a lower order (setlam, genfmt.py:115-153): iorder 1 keeps (m, n) = (0, 0),
// (-1, 0), (1, 0) and iorder 0 (0, 0), the first 3 and 1 entries of the order-2 sets here, a flip-closed subset.
// A scattering matrix (or its adjoint weights) restricted to it: the canonical entries with a row or column beyond
// the first nlam are zero, so the chain product, the termination and the trace are those of the smaller set.
template <typename R, int KIND, int NR, int NC>
__device__ __forceinline__ void mask_lambda(C2<R> (&acc)[RepTab<KIND, NR, NC>().n], int nlam)
{
    constexpr RepTab<KIND, NR, NC> RT{};
    if (nlam >= NR && nlam >= NC) return;
#pragma unroll
    for (int r = 0; r < RT.n; ++r)
        if (RT.a[r] >= nlam || RT.b[r] >= nlam) acc[r] = C2<R>{R(0), R(0)};
}

// ------------------------------------------------------------------------------------------------ stage tables
// Device tables of one phase file (built by fg_stage_create).
template <typename R> struct Tables {
    int E, nph1, L1, nterm, MMd;
    int term_l[2];              // l of the termination terms (distinct final-state l of bcoef, genfmt.py:230)
    int nlam;                   // multiple-scattering lambda entries of the stage's order: 6 (iorder 2), 3 (1), 1 (0)
    const C2<R> *tl;            // (nph1, L1+1, E) j-averaged t-matrix, index il = l + 1 (stage.py:111-118)
    const int *lmax;            // (nph1, E)
    const C2<R> *ck;            // (E) complex momentum, bohr^-1
    const double2 *dk;          // (E) ck - xk in FP64 (the cfac argument, stage.py:336-337)
    const C2<R> *wt;            // (nterm, E) sum over k with lind_k = l of bdiag_k rkk_k^2 (mmtrxi, genfmt.py:378)
    const double *xfac;         // (L1+2, 7, 7) xnlm(il,|m1|+1) (-1)^|m1| / xnlm(il,|m2|+1), 0 where |m| >= il
    const double *xnlm;         // (L1+2, 8) Legendre normalisation, snlm (genfmt.py:41-53)
    const double *rc;           // (L1+1, 7, 7, 3) three-term recursion coefficients for d^{l+1} (stage.py:80-86),
                                // then the (4, 7, 7, 8) seed coefficients of wigner_small (seed_table)
};

// ------------------------------------------------------------------------------------------------ geometry
// Forward-mode dual number (value, derivative along one direction): the adjoint differentiates the geometry by
// running it once per coordinate direction, one direction per lane.
struct Dual {
    double v, d;
};
__device__ __forceinline__ double val(double x) { return x; }
__device__ __forceinline__ double val(Dual x) { return x.v; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual{-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return Dual{q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator*(double a, Dual b) { return Dual{a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return Dual{a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return Dual{a - b.v, -b.d}; }
__device__ __forceinline__ Dual sqrt(Dual a)
{
    const double r = ::sqrt(a.v);
    return Dual{r, r > 0.0 ? a.d / (2.0 * r) : 0.0};
}
__device__ __forceinline__ Dual atan2(Dual y, Dual x)
{
    const double den = x.v * x.v + y.v * y.v;
    return Dual{::atan2(y.v, x.v), den > 0.0 ? (x.v * y.d - y.v * x.d) / den : 0.0};
}
// keep the math library's overloads visible beside the Dual ones
using ::atan2;
using ::sqrt;

template <typename S> __device__ __forceinline__ S cst(double v);
template <> __device__ __forceinline__ double cst<double>(double v) { return v; }
template <> __device__ __forceinline__ Dual cst<Dual>(double v) { return Dual{v, 0.0}; }

// trig.f, as stage.py:148-157 and genfmt.py:56-69; the small-vector branches are constants (zero derivative)
template <typename S>
__device__ __forceinline__ void trig(S x, S y, S z, S &ct, S &st, S &cp, S &sp)
{
    const S r = sqrt(x * x + y * y + z * z), rxy = sqrt(x * x + y * y);
    const bool sr = val(r) < 1e-6, sxy = val(rxy) < 1e-6;
    ct = sr ? cst<S>(1.0) : z / r;
    st = sr ? cst<S>(0.0) : rxy / r;
    cp = sxy ? cst<S>(val(ct) < 0 ? -1.0 : 1.0) : x / rxy;
    sp = sxy ? cst<S>(0.0) : y / rxy;
}

// arg with FEFF's 1e-6 thresholds (stage.py:160-168): a component below the threshold counts as zero (and has
// no derivative), both zero gives fi
template <typename S> __device__ __forceinline__ S arg_fi(S x, S y, S fi)
{
    x = fabs(val(x)) < 1e-6 ? cst<S>(0.0) : x;
    y = fabs(val(y)) < 1e-6 ? cst<S>(0.0) : y;
    return (val(x) == 0.0 && val(y) == 0.0) ? fi : atan2(y, x);
}

// Leg j (1-based) of a path: length (bohr), scattering angle beta and the Euler angles alpha, gamma
// (pathgeom, stage.py:170-206).  rat(i, o) writes atom i in bohr; atom 0 and atom nleg are the absorber.
template <typename S> struct LegGeomT { S ri, beta, alpha, gamma; };
using LegGeom = LegGeomT<double>;

template <typename S, class Rat> __device__ __forceinline__ LegGeomT<S> leg_geometry(const Rat &rat, int j, int nleg)
{
    const int nsc = nleg - 1;
    int i, ip1, im1;
    if (j == nsc + 1) { i = 0; ip1 = 1; im1 = nsc; } else { i = j; ip1 = j + 1; im1 = j - 1; }
    S ai[3], bi[3], ci[3];
    rat(i, ai); rat(ip1, bi); rat(im1, ci);
    S ctp, stp, cpp, spp, ct, st, cp, sp;
    trig<S>(bi[0] - ai[0], bi[1] - ai[1], bi[2] - ai[2], ctp, stp, cpp, spp);
    trig<S>(ai[0] - ci[0], ai[1] - ci[1], ai[2] - ci[2], ct, st, cp, sp);
    const S cppp = cp * cpp + sp * spp, sppp = spp * cp - cpp * sp;
    const S phi = atan2(sp, cp), phip = atan2(spp, cpp);
    const S ax = -(st * ctp - ct * stp * cppp), ay = stp * sppp;
    S b = ct * ctp + st * stp * cppp;
    if (val(b) > 1.0) b = cst<S>(1.0);          // clamp: no derivative outside [-1, 1]
    if (val(b) < -1.0) b = cst<S>(-1.0);
    const S u1x = st * cp, u1y = st * sp, u1z = ct, u2x = stp * cpp, u2y = stp * spp, u2z = ctp;
    const S wx = u1y * u2z - u1z * u2y, wy = u1z * u2x - u1x * u2z, wz = u1x * u2y - u1y * u2x;
    const S sb2 = wx * wx + wy * wy + wz * wz;
    const S gx = -(st * ctp * cppp - ct * stp), gy = -st * sppp;
    const S a_j = arg_fi<S>(ax, ay, phip - phi);
    const S g_j = arg_fi<S>(gx, gy, cst<S>(0.0));
    LegGeomT<S> g;
    g.alpha = M_PI - g_j;
    g.gamma = M_PI - a_j;
    g.beta = atan2(sqrt(sb2 + cst<S>(1e-30)), b);
    const S dx = ai[0] - ci[0], dy = ai[1] - ci[1], dz = ai[2] - ci[2];
    g.ri = sqrt(dx * dx + dy * dy + dz * dz);
    return g;
}

// ------------------------------------------------------------------------------------------------ rotation matrices
// d^l_{mn}(beta) for l <= 3 from Wigner's explicit sum (the seeds; stage.py:26-38 and the closed forms of
// stage.py:52-76 are its l = 1, 2 cases): sum over k of w_k c2^pc s2^ps, pc = 2l + n - m - 2k, ps = m - n + 2k, with
// the signed coefficients w_k = (-1)^(m-n+k) sqrt((l+m)!(l-m)!(l+n)!(l-n)!) / ((l+n-k)! k! (m-n+k)! (l-m-k)!) read
// from the stage's seed table ws (seed_table; built on the host by the same IEEE operations).  k runs over the terms
// whose factorial arguments are all >= 0.
__device__ __forceinline__ double wigner_small(int l, int m, int n, double c2, double s2, const double *ws)
{
    if (l > 3 || abs(m) > l || abs(n) > l) return 0.0;      // the table holds l <= 3 (final states l_t <= 3)
    const double *w = ws + ((l * 7 + m + 3) * 7 + n + 3) * 8;
    double out = 0.0;
    for (int k = max(0, n - m); k <= min(l + n, l - m); ++k) {
        const int pc = 2 * l + n - m - 2 * k, ps = m - n + 2 * k;
        double pw = 1.0;
        for (int q = 0; q < pc; ++q) pw *= c2;
        for (int q = 0; q < ps; ++q) pw *= s2;
        out += w[k] * pw;
    }
    return out;
}

// d/dbeta of d^l_{mn}(beta) for l <= 3 (the derivative of the half-angle powers of Wigner's sum)
__device__ __forceinline__ double wigner_small_dbeta(int l, int m, int n, double c2, double s2, const double *ws)
{
    if (l > 3 || abs(m) > l || abs(n) > l) return 0.0;      // the table holds l <= 3 (final states l_t <= 3)
    const double *w = ws + ((l * 7 + m + 3) * 7 + n + 3) * 8;
    double out = 0.0;
    for (int k = max(0, n - m); k <= min(l + n, l - m); ++k) {
        const int pc = 2 * l + n - m - 2 * k, ps = m - n + 2 * k;
        // d/dbeta c2^pc s2^ps = (ps c2^(pc+1) s2^(ps-1) - pc c2^(pc-1) s2^(ps+1)) / 2
        double t1 = 0.0, t2 = 0.0;
        if (ps > 0) {
            double pw = 1.0;
            for (int q = 0; q < pc + 1; ++q) pw *= c2;
            for (int q = 0; q < ps - 1; ++q) pw *= s2;
            t1 = ps * pw;
        }
        if (pc > 0) {
            double pw = 1.0;
            for (int q = 0; q < pc - 1; ++q) pw *= c2;
            for (int q = 0; q < ps + 1; ++q) pw *= s2;
            t2 = pc * pw;
        }
        out += w[k] * 0.5 * (t1 - t2);
    }
    return out;
}

// The seed coefficients, stored after the recursion coefficients in the rc buffer: (4, 7, 7, 8) doubles indexed
// [l][m + 3][n + 3][k].
template <typename R> __device__ __forceinline__ const double *seed_table(const Tables<R> &T)
{
    return T.rc + (size_t)(T.L1 + 1) * 49 * 3;
}

}  // namespace fg
