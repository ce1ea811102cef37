// pm_pair.cu -- K2 (mixed precision) and K9 (FP64) cell-pair force kernels.
//
// Enumeration (both kernels): one warp per work item (cell A, neighbour delta
// k), k = 0 being A with itself.  The delta list is the reference's
// (CellListEnumerator<Periodic, Cubic>::initialize,
// topology/CellListEnumerator_periodicBoundaries.h:37-108), and a pair of
// cells (A, B = A + delta mod grid) is visited only when B >= A in linear
// order, exactly as the enumerator's next() (:157-179) does.  Inside the same
// cell, pairs i < j (slot order = ascending original index).  So every
// unordered atom pair is tested exactly once, like NonbondedCutoffForce::
// doEvaluate (forces/NonbondedCutoffForce.h:85-109).
//
// Inside an item, lane l holds i-atom l of A in registers; the j-atoms of B
// are staged in shared memory (float4 position + charge, int4 meta) and
// rotated: at step t lane l pairs with j = (l + t) mod 32, so every lane
// touches a different j and the j-force accumulator of that j in shared
// memory without atomics.  i-forces stay in registers.  At the end of a
// chunk each atom's partial force is rounded once to int64 fixed point and
// added with an integer atomic -- the total force is independent of order.
//
// Per pair (OneAtomPair::doOneAtomPair / OneAtomPairTwo::doOneAtomPair,
// forces/OneAtomPair.h:127-188, forces/OneAtomPairTwo.h:131-199):
//   cutoff test r^2 > rc^2 -> skip (rc = largest switching cutoff);
//   exclusion check only for atoms of the same molecule (FULL -> skip,
//   MODIFIED -> A14/B14 and coulombScalingFactor);
//   potentials, switching F = F S - E dS, E = E S when any switch modifies;
//   f_i -= d F, f_j += d F (d = x_j - x_i), energies into the LJ / Coulomb
//   slots, virial addVirial(d F, d) (base/ScalarStructure.cpp:41-62).
//
// Mixed precision: distances from FP32 cell-relative coordinates plus a
// per-delta FP32 cell offset; a pair whose FP32 r^2 lies within a relative
// guard band of a cutoff is re-decided in FP64 with the reference's own
// minimalDifference arithmetic on the original positions, so the pair set is
// the reference's bit for bit.  Potentials and switching in FP32; energies
// and virial summed in FP64 per lane.
//
// FP64 kernel: every pair through the reference's minimalDifference on the
// FP64 positions, reference operation order throughout.
#include <algorithm>

#include "pm_kernels.h"
#include "../../include/pmgpu.h"

#include "pm_adjoint_math.cuh"

namespace pm {

// ------------------------------------------------------------------ combos
struct Combo { int n, p0, s0, p1, s1; };
#define LJ PMGPU_POT_LENNARD_JONES
#define CO PMGPU_POT_COULOMB
#define EW PMGPU_POT_EWALD_REAL
#define NP PMGPU_POT_NONE
#define SCUT PMGPU_SW_CUTOFF
#define SC1 PMGPU_SW_C1
#define SC2 PMGPU_SW_C2
#define SSH PMGPU_SW_SHIFT
#define SUN PMGPU_SW_UNIVERSAL
#define LJT PMGPU_POT_LENNARD_JONES_TABLE
#define COT PMGPU_POT_COULOMB_TABLE
#define EWT PMGPU_POT_EWALD_REAL_TABLE
// The registered periodic OneAtomPair[Two] templates
// (factories/registerForceExemplarsCutoff.cpp:36-137) plus the fused
// LennardJones Coulomb -switchingFunction C2 -switchingFunction C2.  A table
// potential's own switching function is inside its table; the pair applies
// UniversalSwitchingFunction to it (combos 17-24).
static const Combo kCombos[] = {
    {1, CO, SC1, NP, SUN}, {1, CO, SC2, NP, SUN}, {1, CO, SCUT, NP, SUN}, {1, CO, SSH, NP, SUN},
    {1, EW, SCUT, NP, SUN}, {1, LJ, SC1, NP, SUN}, {1, LJ, SC2, NP, SUN}, {1, LJ, SCUT, NP, SUN},
    {1, LJ, SSH, NP, SUN},
    {2, LJ, SC1, EW, SCUT}, {2, LJ, SC1, CO, SSH}, {2, LJ, SC2, CO, SC1}, {2, LJ, SC2, EW, SCUT},
    {2, LJ, SC2, CO, SCUT}, {2, LJ, SC2, CO, SSH}, {2, LJ, SCUT, EW, SCUT}, {2, LJ, SC2, CO, SC2},
    {1, LJT, SUN, NP, SUN}, {1, COT, SUN, NP, SUN}, {1, EWT, SUN, NP, SUN},
    {2, LJ, SC1, EWT, SUN}, {2, LJ, SC2, EWT, SUN}, {2, LJ, SCUT, EWT, SUN},
    {2, LJT, SUN, EWT, SUN}, {2, LJT, SUN, COT, SUN},
};
constexpr int kNumCombos = sizeof(kCombos) / sizeof(kCombos[0]);

__host__ __device__ constexpr bool pot_table(int p) { return p == LJT || p == COT || p == EWT; }
// the ScalarStructure slot of a potential's energy
__host__ __device__ constexpr bool pot_lj_slot(int p) { return p == LJ || p == LJT; }

int pair_combo_id(int n_terms, const int* pot, const int* sw)
{
    // a table term's sw is the tabulated switching function
    const int s0 = pot_table(pot[0]) ? SUN : sw[0];
    const int s1 = n_terms > 1 && pot_table(pot[1]) ? SUN : (n_terms > 1 ? sw[1] : SUN);
    for (int k = 0; k < kNumCombos; ++k) {
        const Combo& c = kCombos[k];
        if (c.n != n_terms) continue;
        if (c.p0 == pot[0] && c.s0 == s0 && (n_terms == 1 || (c.p1 == pot[1] && c.s1 == s1)))
            return k;
    }
    return -1;
}

__host__ __device__ constexpr bool sw_modifies(int s) { return s == SC1 || s == SC2 || s == SSH; }
__host__ __device__ constexpr bool pot_r2(int p) { return p == LJ || p == CO; }
// the pair's rough cutoff test runs when a switching function is used or the
// potential has its own cutoff (OneAtomPair.h:141, OneAtomPairTwo.h:145)
__host__ __device__ constexpr bool term_cut(int p, int s) { return s != SUN || pot_table(p); }

// ---------------------------------------------------------------- shared
struct ItemGeom {
    int a, b;           // cell indices
    int same;
    float ox, oy, oz;   // FP32 offset of cell B's image relative to A
    int valid;
};

__device__ __forceinline__ ItemGeom decode_item(const PairArgs& p, int item)
{
    ItemGeom g;
    const CellGrid& cg = p.grid;
    int nd1 = p.nd + 1;
    g.a = item / nd1;
    int k = item - g.a * nd1;
    g.valid = 0;
    if (k == 0) {
        g.b = g.a; g.same = 1; g.ox = g.oy = g.oz = 0.f;
    } else {
        int4 d = p.deltas[k - 1];
        int ax = g.a / (cg.ny * cg.nz), ay = (g.a / cg.nz) % cg.ny, az = g.a % cg.nz;
        int bx = ((ax + d.x) % cg.nx + cg.nx) % cg.nx;
        int by = ((ay + d.y) % cg.ny + cg.ny) % cg.ny;
        int bz = ((az + d.z) % cg.nz + cg.nz) % cg.nz;
        g.b = (bx * cg.ny + by) * cg.nz + bz;
        g.same = 0;
        float4 o = p.doff[k - 1];
        g.ox = o.x; g.oy = o.y; g.oz = o.z;
        if (g.b < g.a) return g;
    }
    g.valid = 1;
    return g;
}

// ExclusionTable::check for a pair of the same molecule; returns the class
__device__ __forceinline__ int excl_class(const PairArgs& p, int oi, int oj)
{
    return excl_lookup(p.xfull, p.xmod, p.xrow, p.xent, oi, oj);
}

// ---------------------------------------------------------------- FP32 math
// FP32 hi part and remainder of a double constant
#define PM_HI(x) ((float)(x))
#define PM_LO(x) ((float)((x) - (double)(float)(x)))

// e^-x for x >= 0 as 2^(-x log2 e) on the hardware base-2 exponential
// (ex2.approx: relative error ~2^-22); the rounding of the scaled argument
// adds |x| log2(e) 2^-24 relative, the same order as the rounding of x itself
__device__ __forceinline__ float exp_neg(float x)
{
    float y;
    const float a = x * -1.4426950408889634f;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
    return y;
}

// 1/x: the hardware approximation and one Newton-Raphson step
// (y' = y + y (1 - x y)), faithful to ~1 ulp for normal x
__device__ __forceinline__ float rcp_nr(float x)
{
    float y = __fdividef(1.0f, x);
    float e = fmaf(-x, y, 1.0f);
    return fmaf(y, e, y);
}

__device__ __forceinline__ float poly5f(float ar)
{
    // poly5 (base/mathutilities.cpp:29-40), Abramowitz & Stegun 7.1.26.  The
    // coefficients are the same for every pair, so their FP32 rounding is
    // compensated (hi + lo) instead of biasing the real-space Ewald sum.
    const double E1 = 0.254829592, E2 = -0.284496736, E3 = 1.421413741,
                 E4 = -1.453152027, E5 = 1.061405429, PP = 0.3275911;
    float t = rcp_nr(fmaf(PM_HI(PP), ar, fmaf(PM_LO(PP), ar, 1.0f)));
    // each remainder is added after the O(1) partial result it corrects
    float h = fmaf(t, PM_HI(E5), PM_HI(E4)) + fmaf(t, PM_LO(E5), PM_LO(E4));
    h = fmaf(t, h, PM_HI(E3)) + PM_LO(E3);
    h = fmaf(t, h, PM_HI(E2)) + PM_LO(E2);
    h = fmaf(t, h, PM_HI(E1)) + PM_LO(E1);
    return t * h;
}

// qq is the compensated charge product (hi*hi exact inside the FMA plus the
// hi*lo cross terms), so the FP32 rounding of each atom's charge cancels
template <int POT>
__device__ __forceinline__ void pot_f32(const PairArgs& p, const TermF& t, float r2, float rd2, float rinv,
                                        float qq, int ti, int tj, int excl, float& e, float& f)
{
    if (POT == LJ) {
        const float4* tab = excl == PMGPU_EXCL_MODIFIED ? p.ljm : p.ljn;
        float4 par = __ldg(tab + (ti * p.n_types + tj));   // A_hi, B_hi, A_lo, B_lo
        float r6 = rd2 * rd2 * rd2;
        float r12 = r6 * r6;
        float r6B = fmaf(par.y, r6, par.w * r6);
        float r12A = fmaf(par.x, r12, par.z * r12);
        e = r12A - r6B;
        f = (12.0f * r12A - 6.0f * r6B) * rd2;
    } else if (POT == CO) {
        e = qq * rinv;
        e = excl == PMGPU_EXCL_MODIFIED ? e * p.csf : e;
        f = e * rd2;
    } else if (POT == EW) {
        qq = (p.csfd != 1.0 && excl == PMGPU_EXCL_MODIFIED) ? qq * p.csf : qq;
        float r = r2 * rinv;
        float ar = fmaf(t.alpha, r, t.alpha_lo * r);     // compensated alpha
        float ex = qq * exp_neg(ar * ar);
        e = poly5f(ar) * ex * rinv;
        f = fmaf(t.two_alpha_pi, ex, fmaf(t.two_alpha_pi_lo, ex, e)) * rinv * rinv;
    } else if (pot_table(POT)) {
        // LookUpTableBase::index on the FP32 r^2 (its top exponent and PRE
        // mantissa bits pick the entry) and the cubic of ::interpolate
        // (base/LookUpTableBase.h:243-272) in FP32 on the FP32 copy of the
        // table; out of range -> the first / last entry with dt = 0
        const unsigned u = __float_as_uint(r2);
        int k = (int)(u >> t.tab_shift) * t.tab_step - t.tab_first;
        const bool clamp = k < 0 || k > t.tab_last;
        k = k < 0 ? 0 : (k > t.tab_last ? t.tab_last : k);
        const float dt = clamp ? 0.f : r2 - __uint_as_float(u & ~((1u << t.tab_shift) - 1u));
        const float4* T = reinterpret_cast<const float4*>(t.tab + k);
        float a, b, c, d;
        if (POT == LJT) {
            // A part and B part of the entry; compensated A, B
            const float4* tab = excl == PMGPU_EXCL_MODIFIED ? p.ljm : p.ljn;
            const float4 par = __ldg(tab + (ti * p.n_types + tj));   // A_hi, B_hi, A_lo, B_lo
            const float4 ta = __ldg(T), tb = __ldg(T + 1);
            a = fmaf(par.x, ta.x, par.z * ta.x) + fmaf(par.y, tb.x, par.w * tb.x);
            b = fmaf(par.x, ta.y, par.z * ta.y) + fmaf(par.y, tb.y, par.w * tb.y);
            c = fmaf(par.x, ta.z, par.z * ta.z) + fmaf(par.y, tb.z, par.w * tb.z);
            d = fmaf(par.x, ta.w, par.z * ta.w) + fmaf(par.y, tb.w, par.w * tb.w);
        } else {
            const float q = (p.csfd != 1.0 && excl == PMGPU_EXCL_MODIFIED) ? qq * p.csf : qq;
            const float4 tc = __ldg(T);
            a = tc.x * q; b = tc.y * q; c = tc.z * q; d = tc.w * q;
        }
        e = fmaf(fmaf(fmaf(dt, d, c), dt, b), dt, a);
        f = -2.0f * fmaf(fmaf(3.0f * dt, d, 2.0f * c), dt, b);
    } else {
        e = 0.f; f = 0.f;
    }
}

// switching functions as selects (no branches: the two pair evaluations of
// a lane interleave)
template <int SW>
__device__ __forceinline__ void sw_f32(const TermF& t, float r2, float rinv, bool inside, float& v, float& d)
{
    if (SW == SC2) {
        const float c2 = t.cut2 - r2;
        const float c4 = c2 * (t.s2 + 2.0f * r2);
        const float c24 = c2 * c4;
        const float dd = c2 * c2 - c4;
        const bool out = r2 > t.cut2, mid = r2 >= t.on2;
        v = out ? 0.f : (mid ? fmaf(t.s1, c24, t.s1_lo * c24) : 1.f);
        d = (out || !mid) ? 0.f : fmaf(t.s3, dd, t.s3_lo * dd);
    } else if (SW == SC1) {
        const float dist = r2 * rinv;
        const float in = fmaf(-r2, t.c1_05_3, t.c1_15_1) + fmaf(-r2, t.c1_05_3_lo, t.c1_15_1_lo);
        const bool out = r2 > t.cut2;
        v = out ? 0.f : fmaf(-dist, in, 1.0f);
        d = out ? 0.f : fmaf(dist, t.c1_15_3, -t.c1_15_1 * rinv) + fmaf(dist, t.c1_15_3_lo, -t.c1_15_1_lo * rinv);
    } else if (SW == SSH) {
        const float x = fmaf(-r2, t.sh_a, 1.0f) - r2 * t.sh_a_lo;
        const bool out = r2 > t.cut2;
        v = out ? 0.f : x * x;
        d = out ? 0.f : fmaf(t.sh_b, x, t.sh_b_lo * x);
    } else if (SW == SCUT) {
        d = 0.f;
        v = inside ? 1.f : 0.f;
    } else {
        v = 1.f; d = 0.f;
    }
}

// exact FP64 squared distance of two atoms (reference minimalDifference)
__device__ __forceinline__ double exact_d2(const PairArgs& p, int oi, int oj)
{
    const double* pi = p.pos + 3 * (size_t)oi;
    const double* pj = p.pos + 3 * (size_t)oj;
    double dx, dy, dz;
    return pbc_min_diff(p.pbc, pi[0], pi[1], pi[2], pj[0], pj[1], pj[2], dx, dy, dz);
}


// ---------------------------------------------------------------- FP64 math
template <int POT>
__device__ __forceinline__ void pot_f64(const PairArgs& p, const TermD& t, double d2, double rd2,
                                        double qi, double qj, int ti, int tj, int excl, double& e, double& f)
{
    if (POT == LJ) {
        // LennardJonesForce::operator() (forces/LennardJonesForce.h:37-74)
        double4 par = p.ljd[(size_t)ti * p.n_types + tj];
        double A = excl == PMGPU_EXCL_MODIFIED ? par.z : par.x;
        double B = excl == PMGPU_EXCL_MODIFIED ? par.w : par.y;
        double r6 = rd2 * rd2 * rd2;
        double r12 = r6 * r6;
        double r6B = B * r6;
        double r12A = A * r12;
        e = r12A - r6B;
        f = 12.0 * r12A * rd2 - 6.0 * r6B * rd2;
    } else if (POT == CO) {
        // CoulombForce::operator() (forces/CoulombForce.h:41-57)
        e = qi * qj * sqrt(rd2);
        if (excl == PMGPU_EXCL_MODIFIED) e *= p.csfd;
        f = e * rd2;
    } else if (POT == EW) {
        // CoulombEwaldRealForce::operator() (forces/CoulombEwaldRealForce.h:45-73)
        double qq = qi * qj;
        if (p.csfd != 1.0 && excl == PMGPU_EXCL_MODIFIED) qq *= p.csfd;
        double r = sqrt(d2);
        double rr = 1.0 / r;
        double ar = t.alpha * r;
        double ex = qq * exp(-ar * ar);
        const double E1 = 0.254829592, E2 = -0.284496736, E3 = 1.421413741,
                     E4 = -1.453152027, E5 = 1.061405429, PP = 0.3275911;
        double tt = 1.0 / (1.0 + PP * ar);
        double poly = tt * (E1 + tt * (E2 + tt * (E3 + tt * (E4 + tt * E5))));
        e = poly * ex * rr;
        f = ((e + t.two_alpha_pi * ex) * rr * rr);
    } else if (pot_table(POT)) {
        // LookUpTableBase::index / ::interpolate (base/LookUpTableBase.h:243-272)
        // with LennardJonesTableForce::operator() (forces/LennardJonesTableForce.h:81-101),
        // CoulombTableForce::operator() (CoulombTableForce.h:83-108) and
        // CoulombEwaldRealTableForce::operator() (CoulombEwaldRealTableForce.h:85-107)
        const long long u = __double_as_longlong(d2);
        long long k = (u >> t.tab_shift) * t.tab_step - t.tab_first;
        double dt = 0.0;
        if (k < 0) k = 0;
        else if (k > t.tab_last) k = t.tab_last;
        else dt = d2 - __longlong_as_double(u & ~((1ll << t.tab_shift) - 1ll));
        const double4* T = reinterpret_cast<const double4*>(t.tab + k);
        double a, b, c, d;
        if (POT == LJT) {
            const double4 par = p.ljd[(size_t)ti * p.n_types + tj];
            const double A = excl != PMGPU_EXCL_MODIFIED ? par.x : par.z;
            const double B = excl != PMGPU_EXCL_MODIFIED ? par.y : par.w;
            const double4 ta = T[0], tb = T[1];
            a = ta.x * A + tb.x * B;
            b = ta.y * A + tb.y * B;
            c = ta.z * A + tb.z * B;
            d = ta.w * A + tb.w * B;
        } else {
            const double q = qi * qj * ((p.csfd != 1.0 && excl == PMGPU_EXCL_MODIFIED) ? p.csfd : 1.0);
            const double4 tc = T[0];
            a = tc.x * q; b = tc.y * q; c = tc.z * q; d = tc.w * q;
        }
        e = ((dt * d + c) * dt + b) * dt + a;
        f = -2.0 * ((3.0 * dt * d + 2.0 * c) * dt + b);
    } else {
        e = 0.0; f = 0.0;
    }
}

template <int SW>
__device__ __forceinline__ void sw_f64(const TermD& t, double d2, double& v, double& d)
{
    if (SW == SC2) {           // C2SwitchingFunction.h:64-82
        d = 0.0;
        if (d2 > t.cut2) v = 0.0;
        else if (d2 >= t.on2) {
            double c2 = t.cut2 - d2;
            double c4 = c2 * (t.s2 + 2.0 * d2);
            v = t.s1 * (c2 * c4);
            d = t.s3 * (c2 * c2 - c4);
        } else v = 1.0;
    } else if (SW == SC1) {    // C1SwitchingFunction.h:64-75
        if (d2 > t.cut2) { v = 0.0; d = 0.0; return; }
        double dist = sqrt(d2);
        v = 1.0 - dist * (t.c1_15_1 - d2 * t.c1_05_3);
        d = -t.c1_15_1 / dist + dist * t.c1_15_3;
    } else if (SW == SSH) {    // ShiftSwitchingFunction.h
        if (d2 > t.cut2) { v = 0.0; d = 0.0; return; }
        double x = (1.0 - d2 * t.sh_a);
        v = x * x;
        d = t.sh_b * x;
    } else if (SW == SCUT) {   // CutoffSwitchingFunction.h:64-68
        d = 0.0;
        v = (d2 > t.cut2 ? 0.0 : 1.0);
    } else {
        v = 1.0; d = 0.0;
    }
}

#include "pm_pair_mixed.cuh"
#include "pm_pair_col.cuh"

template <int NT, int P0, int S0, int P1, int S1>
__global__ void __launch_bounds__(128) k_pair_fp64(PairArgs p)
{
    constexpr bool kMod = sw_modifies(S0) || (NT > 1 && sw_modifies(S1));
    constexpr bool kUse = term_cut(P0, S0) || (NT > 1 && term_cut(P1, S1));
    constexpr bool kR2 = pot_r2(P0) || (NT > 1 && pot_r2(P1));
    __shared__ double4 sjp[4][32];
    __shared__ int4 sjm[4][32];
    __shared__ double4 sjf[4][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int warps_total = gridDim.x * 4;
    const int n_items = p.grid.ncell * (p.nd + 1);
    double acc[kERec];
    for (int k = 0; k < kERec; ++k) acc[k] = 0.0;

    for (int item = blockIdx.x * 4 + w; item < n_items; item += warps_total) {
        ItemGeom g = decode_item(p, item);
        if (!g.valid) continue;
        int sa = p.start[g.a], ea = p.start[g.a + 1];
        int sb = p.start[g.b], eb = p.start[g.b + 1];
        if (sa == ea || sb == eb) continue;
        for (int ia = sa; ia < ea; ia += 32) {
            int i = ia + lane;
            bool vi = i < ea;
            double4 pi = vi ? p.spos64[i] : make_double4(0, 0, 0, 0);
            int4 mi = vi ? p.smeta[i] : make_int4(-1, 0, -2, 0);
            double fix = 0.0, fiy = 0.0, fiz = 0.0;
            for (int jb = g.same ? ia : sb; jb < eb; jb += 32) {
                int j = jb + lane;
                bool vj = j < eb;
                sjp[w][lane] = vj ? p.spos64[j] : make_double4(0, 0, 0, 0);
                sjm[w][lane] = vj ? p.smeta[j] : make_int4(-1, 0, -3, 0);
                sjf[w][lane] = make_double4(0, 0, 0, 0);
                __syncwarp();
                int nj = min(32, eb - jb);
                bool diag = g.same && jb == ia;
                for (int t = 0; t < 32; ++t) {
                    int jl = (lane + t) & 31;
                    bool ok = vi && jl < nj && (!diag || jb + jl > i);
                    if (!ok) continue;
                    double4 pj = sjp[w][jl];
                    double dx, dy, dz;
                    double d2 = pbc_min_diff(p.pbc, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
                    if (kUse && d2 > p.cut2d) continue;
                    int4 mj = sjm[w][jl];
                    int excl = PMGPU_EXCL_NONE;
                    if (mi.z == mj.z) {
                        excl = excl_class(p, mi.x, mj.x);
                        if (excl == PMGPU_EXCL_FULL) continue;
                    }
                    double rd2 = kR2 ? 1.0 / d2 : 1.0;
                    double e0, f0, e1 = 0.0, f1 = 0.0;
                    pot_f64<P0>(p, p.td[0], d2, rd2, pi.w, pj.w, mi.y, mj.y, excl, e0, f0);
                    if (NT > 1) pot_f64<P1>(p, p.td[1], d2, rd2, pi.w, pj.w, mi.y, mj.y, excl, e1, f1);
                    if (kMod) {
                        double sv, sd;
                        sw_f64<S0>(p.td[0], d2, sv, sd);
                        f0 = f0 * sv - e0 * sd;
                        e0 = e0 * sv;
                        if (NT > 1) {
                            sw_f64<S1>(p.td[1], d2, sv, sd);
                            f1 = f1 * sv - e1 * sd;
                            e1 = e1 * sv;
                        }
                    }
                    if (pot_lj_slot(P0)) acc[0] += e0; else acc[1] += e0;
                    if (NT > 1) { if (pot_lj_slot(P1)) acc[0] += e1; else acc[1] += e1; }
                    double ft = NT > 1 ? (f0 + f1) : f0;
                    double fx = dx * ft, fy = dy * ft, fz = dz * ft;
                    fix -= fx; fiy -= fy; fiz -= fz;
                    double4 aj = sjf[w][jl];
                    aj.x += fx; aj.y += fy; aj.z += fz;
                    sjf[w][jl] = aj;
                    if (p.virial) {
                        double xy = fx * dy, xz = fx * dz, yz = fy * dz;
                        acc[2] += fx * dx; acc[3] += xy; acc[4] += xz;
                        acc[5] += xy; acc[6] += fy * dy; acc[7] += yz;
                        acc[8] += xz; acc[9] += yz; acc[10] += fz * dz;
                    }
                    if (p.rec_pairs) {
                        unsigned long long k = atomicAdd(p.rec_count, 1ull);
                        if ((long long)k < p.rec_cap) {
                            p.rec_pairs[2 * k] = min(mi.x, mj.x);
                            p.rec_pairs[2 * k + 1] = max(mi.x, mj.x);
                        }
                    }
                }
                __syncwarp();
                if (vj) {
                    double4 fj = sjf[w][lane];
                    fixed_add3(p.facc + 3 * (size_t)j, fj.x, fj.y, fj.z, p.scale, p.status);
                }
                __syncwarp();
            }
            if (vi) fixed_add3(p.facc + 3 * (size_t)i, fix, fiy, fiz, p.scale, p.status);
        }
    }
    block_reduce_store<4>(acc, p.erec, p.erec_stride, blockIdx.x);
}

// Molecular virial of a cutoff force (OneAtomPair.h:174-181,
// OneAtomPairTwo.h:185-192): every pair of atoms of different molecules inside
// the cutoff adds its FP64 pair force against the minimal difference of the
// two molecules' positions (ScalarStructure::addVirial(f, diff, comDiff),
// base/ScalarStructure.cpp:90-132), and against the pair vector to the
// inter-molecular atomic virial.  The cell pairs and the arithmetic of
// k_pair_fp64; a pair of one molecule adds to neither tensor (exclusions act
// only within a molecule, so none applies here).  No forces, no energies.
template <int NT, int P0, int S0, int P1, int S1>
__global__ void __launch_bounds__(128) k_pair_molvir(PairArgs p)
{
    constexpr bool kMod = sw_modifies(S0) || (NT > 1 && sw_modifies(S1));
    constexpr bool kUse = term_cut(P0, S0) || (NT > 1 && term_cut(P1, S1));
    constexpr bool kR2 = pot_r2(P0) || (NT > 1 && pot_r2(P1));
    __shared__ double4 sjp[4][32];
    __shared__ int2 sjm[4][32];       // type, molecule
    __shared__ double4 sjc[4][32];    // the molecule's position
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int warps_total = gridDim.x * 4;
    const int n_items = p.grid.ncell * (p.nd + 1);
    double acc[kMRec];
    for (int k = 0; k < kMRec; ++k) acc[k] = 0.0;

    for (int item = blockIdx.x * 4 + w; item < n_items; item += warps_total) {
        ItemGeom g = decode_item(p, item);
        if (!g.valid) continue;
        int sa = p.start[g.a], ea = p.start[g.a + 1];
        int sb = p.start[g.b], eb = p.start[g.b + 1];
        if (sa == ea || sb == eb) continue;
        for (int ia = sa; ia < ea; ia += 32) {
            int i = ia + lane;
            bool vi = i < ea;
            double4 pi = vi ? p.spos64[i] : make_double4(0, 0, 0, 0);
            int4 mi = vi ? p.smeta[i] : make_int4(-1, 0, -2, 0);
            double cix = 0.0, ciy = 0.0, ciz = 0.0;
            if (vi) {
                const double* c = p.molpos + 3 * (size_t)mi.z;
                cix = c[0]; ciy = c[1]; ciz = c[2];
            }
            for (int jb = g.same ? ia : sb; jb < eb; jb += 32) {
                int j = jb + lane;
                bool vj = j < eb;
                sjp[w][lane] = vj ? p.spos64[j] : make_double4(0, 0, 0, 0);
                int4 mj4 = vj ? p.smeta[j] : make_int4(-1, 0, -3, 0);
                sjm[w][lane] = make_int2(mj4.y, mj4.z);
                if (vj) {
                    const double* c = p.molpos + 3 * (size_t)mj4.z;
                    sjc[w][lane] = make_double4(c[0], c[1], c[2], 0.0);
                }
                __syncwarp();
                int nj = min(32, eb - jb);
                bool diag = g.same && jb == ia;
                for (int t = 0; t < 32; ++t) {
                    int jl = (lane + t) & 31;
                    bool ok = vi && jl < nj && (!diag || jb + jl > i);
                    if (!ok) continue;
                    const int2 mj = sjm[w][jl];
                    if (mj.y == mi.z) continue;
                    double4 pj = sjp[w][jl];
                    double dx, dy, dz;
                    double d2 = pbc_min_diff(p.pbc, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
                    if (kUse && d2 > p.cut2d) continue;
                    double rd2 = kR2 ? 1.0 / d2 : 1.0;
                    double e0, f0, e1 = 0.0, f1 = 0.0;
                    pot_f64<P0>(p, p.td[0], d2, rd2, pi.w, pj.w, mi.y, mj.x, PMGPU_EXCL_NONE, e0, f0);
                    if (NT > 1) pot_f64<P1>(p, p.td[1], d2, rd2, pi.w, pj.w, mi.y, mj.x, PMGPU_EXCL_NONE, e1, f1);
                    if (kMod) {
                        double sv, sd;
                        sw_f64<S0>(p.td[0], d2, sv, sd);
                        f0 = f0 * sv - e0 * sd;
                        if (NT > 1) {
                            sw_f64<S1>(p.td[1], d2, sv, sd);
                            f1 = f1 * sv - e1 * sd;
                        }
                    }
                    double ft = NT > 1 ? (f0 + f1) : f0;
                    double fx = dx * ft, fy = dy * ft, fz = dz * ft;
                    const double4 cj = sjc[w][jl];
                    double cx, cy, cz;
                    pbc_min_diff(p.pbc, cix, ciy, ciz, cj.x, cj.y, cj.z, cx, cy, cz);
                    add_outer(acc, fx, fy, fz, cx, cy, cz);
                    add_outer(acc + 9, fx, fy, fz, dx, dy, dz);
                }
                __syncwarp();
            }
        }
    }
    block_reduce_store_n<4, kMRec>(acc, p.mrec, p.mrec_stride, blockIdx.x);
}

// K10 over the cell list: the backward pass of a cutoff force's pair terms
// (pm_adjoint.cu's per-pair math) over the forward kernels' cell pairs, each
// unordered pair once (the pair set of k_pair_fp64, exact FP64 minimal image
// and cutoff decision).  Per pair: dE/dq~ to both atoms, dE/dA, dE/dB split
// between (t_i, t_j) and (t_j, t_i), (H v)_i += c and (H v)_j -= c with
// c = F u + 2 F' (d.u) d, u = v_j - v_i, and the energies.  i outputs in
// registers, j outputs in shared memory per chunk; both added to the
// atom-order outputs with FP64 atomics.  The LJ table gradient goes through
// a small per-thread cache of type-pair sums (a thread's i atom keeps its
// type, and a few type pairs carry most pairs), flushed to shared or global
// memory on eviction and at the end: the table's few entries would otherwise
// take every pair's atomics on the same addresses.
constexpr int kAdjSmemTypes = 32;
constexpr int kLjCache = 4;

struct LjCache {
    long long key[kLjCache];
    double a[kLjCache], b[kLjCache];
    int next;
};

__device__ __forceinline__ void lj_cache_add(LjCache& c, long long key, double pa, double pb, double* tab)
{
#pragma unroll
    for (int s = 0; s < kLjCache; ++s)
        if (c.key[s] == key) { c.a[s] += pa; c.b[s] += pb; return; }
    // evict round robin
    const int v = c.next;
    c.next = (c.next + 1) % kLjCache;
#pragma unroll
    for (int s = 0; s < kLjCache; ++s)
        if (s == v) {
            if (c.key[s] >= 0) { atomicAdd(tab + c.key[s], c.a[s]); atomicAdd(tab + c.key[s] + 1, c.b[s]); }
            c.key[s] = key; c.a[s] = pa; c.b[s] = pb;
        }
}

template <typename R>
__global__ void __launch_bounds__(128) k_pair_adjoint_cells(PairArgs p, AdjArgs aa)
{
    __shared__ double4 sjp[4][32];
    __shared__ int4 sjm[4][32];
    __shared__ double sjv[4][32][3];
    __shared__ double sjdq[4][32];
    __shared__ double sjhv[4][32][3];
    __shared__ double s_lj[kAdjSmemTypes * kAdjSmemTypes * 4];
    const bool lj_smem = aa.dlj && aa.n_types <= kAdjSmemTypes;
    if (lj_smem)
        for (int k = threadIdx.x; k < aa.n_types * aa.n_types * 4; k += blockDim.x) s_lj[k] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int warps_total = gridDim.x * 4;
    const int n_items = p.grid.ncell * (p.nd + 1);
    double el = 0.0, ec = 0.0;
    double* lj_tab = lj_smem ? s_lj : aa.dlj;
    LjCache cache;
#pragma unroll
    for (int k = 0; k < kLjCache; ++k) { cache.key[k] = -1; cache.a[k] = 0.0; cache.b[k] = 0.0; }
    cache.next = 0;
    for (int item = blockIdx.x * 4 + w; item < n_items; item += warps_total) {
        ItemGeom g = decode_item(p, item);
        if (!g.valid) continue;
        int sa = p.start[g.a], ea = p.start[g.a + 1];
        int sb = p.start[g.b], eb = p.start[g.b + 1];
        if (sa == ea || sb == eb) continue;
        for (int ia = sa; ia < ea; ia += 32) {
            int i = ia + lane;
            bool vi = i < ea;
            double4 pi = vi ? p.spos64[i] : make_double4(0, 0, 0, 0);
            int4 mi = vi ? p.smeta[i] : make_int4(-1, 0, -2, 0);
            double vix = 0.0, viy = 0.0, viz = 0.0;
            if (vi && aa.v) {
                vix = aa.v[3 * (size_t)mi.x]; viy = aa.v[3 * (size_t)mi.x + 1]; viz = aa.v[3 * (size_t)mi.x + 2];
            }
            double dqi = 0.0, hix = 0.0, hiy = 0.0, hiz = 0.0;
            for (int jb = g.same ? ia : sb; jb < eb; jb += 32) {
                int j = jb + lane;
                bool vj = j < eb;
                sjp[w][lane] = vj ? p.spos64[j] : make_double4(0, 0, 0, 0);
                int4 mj4 = vj ? p.smeta[j] : make_int4(-1, 0, -3, 0);
                sjm[w][lane] = mj4;
                for (int c = 0; c < 3; ++c) {
                    sjv[w][lane][c] = (vj && aa.v) ? aa.v[3 * (size_t)mj4.x + c] : 0.0;
                    sjhv[w][lane][c] = 0.0;
                }
                sjdq[w][lane] = 0.0;
                __syncwarp();
                int nj = min(32, eb - jb);
                bool diag = g.same && jb == ia;
                for (int t = 0; t < 32; ++t) {
                    int jl = (lane + t) & 31;
                    bool ok = vi && jl < nj && (!diag || jb + jl > i);
                    if (!ok) continue;
                    double4 pj = sjp[w][jl];
                    double dx, dy, dz;
                    double a = pbc_min_diff(p.pbc, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
                    if (aa.use_cut && a > aa.cut2d) continue;
                    int4 mj = sjm[w][jl];
                    int excl = PMGPU_EXCL_NONE;
                    if (mi.z == mj.z) {
                        excl = excl_class(p, mi.x, mj.x);
                        if (excl == PMGPU_EXCL_FULL) continue;
                    }
                    const double4 par = aa.ljd[(size_t)mi.y * aa.n_types + mj.y];
                    R F, F1, pqq, pA, pB;
                    adj_pair<R>(aa, a, pi.w, pj.w, par, excl, 1.0, F, F1, pqq, pA, pB, el, ec);
                    dqi += (double)pqq * pj.w;
                    sjdq[w][jl] += (double)pqq * pi.w;
                    if (aa.v) {
                        const double ux = sjv[w][jl][0] - vix, uy = sjv[w][jl][1] - viy, uz = sjv[w][jl][2] - viz;
                        const double du = dx * ux + dy * uy + dz * uz;
                        const double fF = (double)F, t2 = 2.0 * (double)F1 * du;
                        const double cx = fF * ux + t2 * dx, cy = fF * uy + t2 * dy, cz = fF * uz + t2 * dz;
                        hix += cx; hiy += cy; hiz += cz;
                        sjhv[w][jl][0] -= cx; sjhv[w][jl][1] -= cy; sjhv[w][jl][2] -= cz;
                    }
                    if (aa.dlj && (pA != 0 || pB != 0)) {
                        const int mo = excl == PMGPU_EXCL_MODIFIED ? 2 : 0;
                        const long long k1 = ((long long)mi.y * aa.n_types + mj.y) * 4 + mo;
                        const long long k2 = ((long long)mj.y * aa.n_types + mi.y) * 4 + mo;
                        lj_cache_add(cache, k1, 0.5 * (double)pA, 0.5 * (double)pB, lj_tab);
                        lj_cache_add(cache, k2, 0.5 * (double)pA, 0.5 * (double)pB, lj_tab);
                    }
                }
                __syncwarp();
                if (vj) {
                    const int oj = mj4.x;
                    if (aa.dq && sjdq[w][lane] != 0.0) atomicAdd(aa.dq + oj, sjdq[w][lane]);
                    if (aa.hv)
                        for (int c = 0; c < 3; ++c)
                            if (sjhv[w][lane][c] != 0.0) atomicAdd(aa.hv + 3 * (size_t)oj + c, sjhv[w][lane][c]);
                }
                __syncwarp();
            }
            if (vi) {
                if (aa.dq && dqi != 0.0) atomicAdd(aa.dq + mi.x, dqi);
                if (aa.hv) {
                    if (hix != 0.0) atomicAdd(aa.hv + 3 * (size_t)mi.x, hix);
                    if (hiy != 0.0) atomicAdd(aa.hv + 3 * (size_t)mi.x + 1, hiy);
                    if (hiz != 0.0) atomicAdd(aa.hv + 3 * (size_t)mi.x + 2, hiz);
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kLjCache; ++k)
        if (cache.key[k] >= 0) {
            atomicAdd(lj_tab + cache.key[k], cache.a[k]);
            atomicAdd(lj_tab + cache.key[k] + 1, cache.b[k]);
        }
    if (aa.energy) {
        for (int o = 16; o > 0; o >>= 1) {
            el += __shfl_xor_sync(0xffffffffu, el, o);
            ec += __shfl_xor_sync(0xffffffffu, ec, o);
        }
        if (lane == 0) {
            if (el != 0.0) atomicAdd(aa.energy, el);
            if (ec != 0.0) atomicAdd(aa.energy + 1, ec);
        }
    }
    if (lj_smem) {
        __syncthreads();
        for (int k = threadIdx.x; k < aa.n_types * aa.n_types * 4; k += blockDim.x)
            if (s_lj[k] != 0.0) atomicAdd(aa.dlj + k, s_lj[k]);
    }
}

int launch_pair_adjoint_cells(const PairArgs& p, const AdjArgs& a, int fp64, int blocks, cudaStream_t s,
                              long long* launches)
{
    if (fp64) k_pair_adjoint_cells<double><<<blocks, 128, 0, s>>>(p, a);
    else k_pair_adjoint_cells<float><<<blocks, 128, 0, s>>>(p, a);
    *launches += 1;
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------- launch
long long plist_estimate(int n_atoms, const CellGrid& g, int nh)
{
    // every i-supercluster against every cluster of its half shell, at the
    // mean cell occupancy plus one partial cluster, with 50% slack for uneven
    // cells
    double per_cell = (double)n_atoms / (kCluster * (double)g.ncell) + 1.0;
    double supers = (double)n_atoms / (kCluster * kSuper) + g.ncell;
    return (long long)(1.5 * supers * (nh + 1) * per_cell) + 4096;
}

long long chunk_estimate(int n_atoms, const CellGrid& g, int nh, int chunk)
{
    return plist_estimate(n_atoms, g, nh) / chunk + (long long)n_atoms / (kCluster * kSuper) + g.ncell + 1024;
}

int pair_blocks(const CellGrid& g, int nd)
{
    long long items = (long long)g.ncell * (nd + 1);
    long long b = (items + 3) / 4;
    long long cap = 148 * 16;
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

template <template <int, int, int, int, int> class K>
struct Dispatch;

#define PM_COMBO_SWITCH(KERNEL)                                                                        \
    switch (combo) {                                                                                   \
    case 0: KERNEL<1, CO, SC1, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                               \
    case 1: KERNEL<1, CO, SC2, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                               \
    case 2: KERNEL<1, CO, SCUT, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                              \
    case 3: KERNEL<1, CO, SSH, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                               \
    case 4: KERNEL<1, EW, SCUT, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                              \
    case 5: KERNEL<1, LJ, SC1, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                               \
    case 6: KERNEL<1, LJ, SC2, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                               \
    case 7: KERNEL<1, LJ, SCUT, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                              \
    case 8: KERNEL<1, LJ, SSH, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                               \
    case 9: KERNEL<2, LJ, SC1, EW, SCUT><<<blocks, 128, 0, s>>>(a); break;                              \
    case 10: KERNEL<2, LJ, SC1, CO, SSH><<<blocks, 128, 0, s>>>(a); break;                              \
    case 11: KERNEL<2, LJ, SC2, CO, SC1><<<blocks, 128, 0, s>>>(a); break;                              \
    case 12: KERNEL<2, LJ, SC2, EW, SCUT><<<blocks, 128, 0, s>>>(a); break;                             \
    case 13: KERNEL<2, LJ, SC2, CO, SCUT><<<blocks, 128, 0, s>>>(a); break;                             \
    case 14: KERNEL<2, LJ, SC2, CO, SSH><<<blocks, 128, 0, s>>>(a); break;                              \
    case 15: KERNEL<2, LJ, SCUT, EW, SCUT><<<blocks, 128, 0, s>>>(a); break;                            \
    case 16: KERNEL<2, LJ, SC2, CO, SC2><<<blocks, 128, 0, s>>>(a); break;                              \
    case 17: KERNEL<1, LJT, SUN, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                             \
    case 18: KERNEL<1, COT, SUN, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                             \
    case 19: KERNEL<1, EWT, SUN, NP, SUN><<<blocks, 128, 0, s>>>(a); break;                             \
    case 20: KERNEL<2, LJ, SC1, EWT, SUN><<<blocks, 128, 0, s>>>(a); break;                             \
    case 21: KERNEL<2, LJ, SC2, EWT, SUN><<<blocks, 128, 0, s>>>(a); break;                             \
    case 22: KERNEL<2, LJ, SCUT, EWT, SUN><<<blocks, 128, 0, s>>>(a); break;                            \
    case 23: KERNEL<2, LJT, SUN, EWT, SUN><<<blocks, 128, 0, s>>>(a); break;                            \
    case 24: KERNEL<2, LJT, SUN, COT, SUN><<<blocks, 128, 0, s>>>(a); break;                            \
    default: return (int)cudaErrorInvalidValue;                                                        \
    }

// one full wave of the mixed kernel (persistent warps take chunks of work)
template <int NT, int P0, int S0, int P1, int S1, bool WRAP>
static int run_mixed_w(const PairArgs& a, cudaStream_t s, long long* launches)
{
    static int sms = 0, per_sm = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_mixed<NT, P0, S0, P1, S1, WRAP>, 128, 0);
        if (sms <= 0) sms = 148;
        if (per_sm <= 0) per_sm = 1;
    }
    // a tuned number of resident blocks per SM (fewer leave room for the PME
    // kernels running beside it), else the occupancy limit
    const int bps = a.blocks_per_sm > 0 ? std::min(per_sm, a.blocks_per_sm) : per_sm;
    const int blocks = sms * bps;
    launch_pdl(k_pair_mixed<NT, P0, S0, P1, S1, WRAP>, blocks, 128, 0, s, a);
    *launches += 1;
    return (int)cudaGetLastError();
}

template <int NT, int P0, int S0, int P1, int S1>
static int run_mixed(const PairArgs& a, cudaStream_t s, long long* launches)
{
    return a.wrap ? run_mixed_w<NT, P0, S0, P1, S1, true>(a, s, launches)
                  : run_mixed_w<NT, P0, S0, P1, S1, false>(a, s, launches);
}

int launch_cluster_list(const PairArgs& a, cudaStream_t s, long long* launches)
{
    // one warp per cell and block of 32 half-shell cells
    long long warps = (long long)a.grid.ncell * ((a.nh + 1 + 31) / 32);
    int lb = (int)((warps + 3) / 4);
    launch_pdl(k_cluster_list, lb > 0 ? lb : 1, 128, 0, s, a);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_pair_mixed(const PairArgs& a, int combo, cudaStream_t s, long long* launches)
{
    switch (combo) {
#define PM_MIXED_CASE(ID, ...) case ID: return run_mixed<__VA_ARGS__>(a, s, launches);
    PM_MIXED_CASE(0, 1, CO, SC1, NP, SUN)
    PM_MIXED_CASE(1, 1, CO, SC2, NP, SUN)
    PM_MIXED_CASE(2, 1, CO, SCUT, NP, SUN)
    PM_MIXED_CASE(3, 1, CO, SSH, NP, SUN)
    PM_MIXED_CASE(4, 1, EW, SCUT, NP, SUN)
    PM_MIXED_CASE(5, 1, LJ, SC1, NP, SUN)
    PM_MIXED_CASE(6, 1, LJ, SC2, NP, SUN)
    PM_MIXED_CASE(7, 1, LJ, SCUT, NP, SUN)
    PM_MIXED_CASE(8, 1, LJ, SSH, NP, SUN)
    PM_MIXED_CASE(9, 2, LJ, SC1, EW, SCUT)
    PM_MIXED_CASE(10, 2, LJ, SC1, CO, SSH)
    PM_MIXED_CASE(11, 2, LJ, SC2, CO, SC1)
    PM_MIXED_CASE(12, 2, LJ, SC2, EW, SCUT)
    PM_MIXED_CASE(13, 2, LJ, SC2, CO, SCUT)
    PM_MIXED_CASE(14, 2, LJ, SC2, CO, SSH)
    PM_MIXED_CASE(15, 2, LJ, SCUT, EW, SCUT)
    PM_MIXED_CASE(16, 2, LJ, SC2, CO, SC2)
    PM_MIXED_CASE(17, 1, LJT, SUN, NP, SUN)
    PM_MIXED_CASE(18, 1, COT, SUN, NP, SUN)
    PM_MIXED_CASE(19, 1, EWT, SUN, NP, SUN)
    PM_MIXED_CASE(20, 2, LJ, SC1, EWT, SUN)
    PM_MIXED_CASE(21, 2, LJ, SC2, EWT, SUN)
    PM_MIXED_CASE(22, 2, LJ, SCUT, EWT, SUN)
    PM_MIXED_CASE(23, 2, LJT, SUN, EWT, SUN)
    PM_MIXED_CASE(24, 2, LJT, SUN, COT, SUN)
#undef PM_MIXED_CASE
    default: return (int)cudaErrorInvalidValue;
    }
}

int launch_near_energy(const PairArgs& a, int combo, int n_atoms, cudaStream_t s, long long* launches)
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    // about 26 near pairs per atom in water, one per thread; at most one
    // resident wave (16 blocks per SM; the kernel is grid-stride)
    long long want = (30LL * n_atoms + 127) / 128;
    const int blocks = (int)std::max(1LL, std::min<long long>(want, 16LL * sms));
    PM_COMBO_SWITCH(k_near_energy)
    *launches += 1;
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------- column path
long long col_list_estimate(int n_atoms, const ColGrid& g, double volume, double cutoff)
{
    // half of the 4-atom j-clusters within the cutoff plus 1.5 column sides
    // of each i-cluster, with 30% slack
    const double rho = volume > 0.0 ? n_atoms / volume : 0.0;
    const double r = cutoff + 1.5 * std::max(g.sx, g.sy);
    const double per = rho * (4.0 / 3.0) * 3.14159265358979 * r * r * r / 8.0;
    const double icl = (double)n_atoms / kCluster + g.ncol + 1;
    return (long long)(1.3 * icl * per) + 4096;
}

long long col_chunk_estimate(long long entries, int n_atoms, const ColGrid& g, int chunk)
{
    return entries / std::max(1, chunk) + (long long)n_atoms / kCluster + g.ncol + 1024;
}

int launch_col_list(const PairArgs& a, cudaStream_t s, long long* launches)
{
    const int blocks = std::max(1, (a.icl_cap + 3) / 4);    // one warp per i-cluster
    launch_pdl(k_col_list, blocks, 128, 0, s, a);
    *launches += 1;
    return (int)cudaGetLastError();
}

template <int NT, int P0, int S0, int P1, int S1>
static int run_col(const PairArgs& a, cudaStream_t s, long long* launches)
{
    static int sms = 0, per_sm = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_col<NT, P0, S0, P1, S1>, 128, 0);
        if (sms <= 0) sms = 148;
        if (per_sm <= 0) per_sm = 1;
    }
    const int bps = a.blocks_per_sm > 0 ? std::min(per_sm, a.blocks_per_sm) : per_sm;
    launch_pdl(k_pair_col<NT, P0, S0, P1, S1>, sms * bps, 128, 0, s, a);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_pair_col(const PairArgs& a, int combo, cudaStream_t s, long long* launches)
{
    switch (combo) {
#define PM_COL_CASE(ID, ...) case ID: return run_col<__VA_ARGS__>(a, s, launches);
    PM_COL_CASE(0, 1, CO, SC1, NP, SUN)
    PM_COL_CASE(1, 1, CO, SC2, NP, SUN)
    PM_COL_CASE(2, 1, CO, SCUT, NP, SUN)
    PM_COL_CASE(3, 1, CO, SSH, NP, SUN)
    PM_COL_CASE(4, 1, EW, SCUT, NP, SUN)
    PM_COL_CASE(5, 1, LJ, SC1, NP, SUN)
    PM_COL_CASE(6, 1, LJ, SC2, NP, SUN)
    PM_COL_CASE(7, 1, LJ, SCUT, NP, SUN)
    PM_COL_CASE(8, 1, LJ, SSH, NP, SUN)
    PM_COL_CASE(9, 2, LJ, SC1, EW, SCUT)
    PM_COL_CASE(10, 2, LJ, SC1, CO, SSH)
    PM_COL_CASE(11, 2, LJ, SC2, CO, SC1)
    PM_COL_CASE(12, 2, LJ, SC2, EW, SCUT)
    PM_COL_CASE(13, 2, LJ, SC2, CO, SCUT)
    PM_COL_CASE(14, 2, LJ, SC2, CO, SSH)
    PM_COL_CASE(15, 2, LJ, SCUT, EW, SCUT)
    PM_COL_CASE(16, 2, LJ, SC2, CO, SC2)
    PM_COL_CASE(17, 1, LJT, SUN, NP, SUN)
    PM_COL_CASE(18, 1, COT, SUN, NP, SUN)
    PM_COL_CASE(19, 1, EWT, SUN, NP, SUN)
    PM_COL_CASE(20, 2, LJ, SC1, EWT, SUN)
    PM_COL_CASE(21, 2, LJ, SC2, EWT, SUN)
    PM_COL_CASE(22, 2, LJ, SCUT, EWT, SUN)
    PM_COL_CASE(23, 2, LJT, SUN, EWT, SUN)
    PM_COL_CASE(24, 2, LJT, SUN, COT, SUN)
#undef PM_COL_CASE
    default: return (int)cudaErrorInvalidValue;
    }
}

template <int NT, int P0, int S0, int P1, int S1>
static int run_col_batch(const BatchPairArgs& b, cudaStream_t s, long long* launches)
{
    static int sms = 0, per_sm = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_col_batch<NT, P0, S0, P1, S1>, 128, 0);
        if (sms <= 0) sms = 148;
        if (per_sm <= 0) per_sm = 1;
    }
    k_pair_col_batch<NT, P0, S0, P1, S1><<<sms * per_sm, 128, 0, s>>>(b);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_pair_col_batch(const BatchPairArgs& b, int combo, cudaStream_t s, long long* launches)
{
    if (b.n < 1 || b.n > kBatchPairMax) return (int)cudaErrorInvalidValue;
    switch (combo) {
#define PM_COLB_CASE(ID, ...) case ID: return run_col_batch<__VA_ARGS__>(b, s, launches);
    PM_COLB_CASE(0, 1, CO, SC1, NP, SUN)
    PM_COLB_CASE(1, 1, CO, SC2, NP, SUN)
    PM_COLB_CASE(2, 1, CO, SCUT, NP, SUN)
    PM_COLB_CASE(3, 1, CO, SSH, NP, SUN)
    PM_COLB_CASE(4, 1, EW, SCUT, NP, SUN)
    PM_COLB_CASE(5, 1, LJ, SC1, NP, SUN)
    PM_COLB_CASE(6, 1, LJ, SC2, NP, SUN)
    PM_COLB_CASE(7, 1, LJ, SCUT, NP, SUN)
    PM_COLB_CASE(8, 1, LJ, SSH, NP, SUN)
    PM_COLB_CASE(9, 2, LJ, SC1, EW, SCUT)
    PM_COLB_CASE(10, 2, LJ, SC1, CO, SSH)
    PM_COLB_CASE(11, 2, LJ, SC2, CO, SC1)
    PM_COLB_CASE(12, 2, LJ, SC2, EW, SCUT)
    PM_COLB_CASE(13, 2, LJ, SC2, CO, SCUT)
    PM_COLB_CASE(14, 2, LJ, SC2, CO, SSH)
    PM_COLB_CASE(15, 2, LJ, SCUT, EW, SCUT)
    PM_COLB_CASE(16, 2, LJ, SC2, CO, SC2)
    PM_COLB_CASE(17, 1, LJT, SUN, NP, SUN)
    PM_COLB_CASE(18, 1, COT, SUN, NP, SUN)
    PM_COLB_CASE(19, 1, EWT, SUN, NP, SUN)
    PM_COLB_CASE(20, 2, LJ, SC1, EWT, SUN)
    PM_COLB_CASE(21, 2, LJ, SC2, EWT, SUN)
    PM_COLB_CASE(22, 2, LJ, SCUT, EWT, SUN)
    PM_COLB_CASE(23, 2, LJT, SUN, EWT, SUN)
    PM_COLB_CASE(24, 2, LJT, SUN, COT, SUN)
#undef PM_COLB_CASE
    default: return (int)cudaErrorInvalidValue;
    }
}

int launch_near_energy_col(const PairArgs& a, int combo, int n_atoms, cudaStream_t s, long long* launches)
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    long long want = (30LL * n_atoms + 127) / 128;
    const int blocks = (int)std::max(1LL, std::min<long long>(want, 16LL * sms));
    PM_COMBO_SWITCH(k_near_energy_col)
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_pair_fp64(const PairArgs& a, int combo, int blocks, cudaStream_t s, long long* launches)
{
    PM_COMBO_SWITCH(k_pair_fp64)
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_pair_molvir(const PairArgs& a, int combo, int blocks, cudaStream_t s, long long* launches)
{
    PM_COMBO_SWITCH(k_pair_molvir)
    *launches += 1;
    return (int)cudaGetLastError();
}

}  // namespace pm
