// pm_adjoint_math.cuh -- per-pair math of the backward pass (K10), shared by
// the all-pairs kernel (pm_adjoint.cu) and the cell-list kernel (pm_pair.cu).
#pragma once

#include "pm_kernels.h"
#include "../../include/pmgpu.h"

namespace pm {

// value, first and second derivative w.r.t. a = r^2 of a switching function
// (the reference's switchingDeriv is 2 S'(a))
template <typename R>
__device__ __forceinline__ void switch_a(int sw, const TermD& t, double a_exact, R a, R& s, R& s1, R& s2)
{
    s = 1; s1 = 0; s2 = 0;
    if (sw == PMGPU_SW_C2) {                 // C2SwitchingFunction.h:64-82
        if (a_exact > t.cut2) { s = 0; return; }
        if (a_exact < t.on2) return;
        const R c2 = (R)t.cut2 - a;
        const R sp = (R)t.s2 + 2 * a;
        s = (R)t.s1 * c2 * c2 * sp;
        s1 = (R)t.s1 * (2 * c2 * c2 - 2 * c2 * sp);
        s2 = (R)t.s1 * (2 * sp - 8 * c2);
    } else if (sw == PMGPU_SW_C1) {          // C1SwitchingFunction.h:64-75
        if (a_exact > t.cut2) { s = 0; return; }
        const R r = sqrt(a);
        s = 1 - r * ((R)t.c1_15_1 - a * (R)t.c1_05_3);
        s1 = -(R)0.5 * (R)t.c1_15_1 / r + (R)1.5 * (R)t.c1_05_3 * r;
        s2 = (R)0.25 * (R)t.c1_15_1 / (r * a) + (R)0.75 * (R)t.c1_05_3 / r;
    } else if (sw == PMGPU_SW_SHIFT) {       // ShiftSwitchingFunction.h
        if (a_exact > t.cut2) { s = 0; return; }
        const R x = 1 - a * (R)t.sh_a;
        s = x * x;
        s1 = -2 * (R)t.sh_a * x;
        s2 = 2 * (R)t.sh_a * (R)t.sh_a;
    } else if (sw == PMGPU_SW_CUTOFF) {      // CutoffSwitchingFunction.h:64-68
        s = a_exact > t.cut2 ? 0 : 1;
    }
}

// One term of a pair: energy e, force factor f (F_j = d f), f' = df/da and
// the partials of e w.r.t. the charge product (per unit q~_i q~_j) and the LJ
// A, B entries.  LJ and Coulomb are exact derivatives of their energies; the
// Ewald real term differentiates the reference's force expression
// (CoulombEwaldRealForce.h:45-73: poly5 energy, exact-erfc-derivative force).
template <typename R>
__device__ __forceinline__ void term_raw(int pot, const TermD& t, R a, R qq, R A, R B, R kappa,
                                         R& e, R& e1, R& f, R& f1, R& pqq, R& pA, R& pB)
{
    e = e1 = f = f1 = pqq = pA = pB = 0;
    const R ia = 1 / a;
    if (pot == PMGPU_POT_LENNARD_JONES) {
        const R a3 = ia * ia * ia, a6 = a3 * a3;
        e = A * a6 - B * a3;
        e1 = (-6 * A * a6 + 3 * B * a3) * ia;
        const R e2 = (42 * A * a6 - 12 * B * a3) * ia * ia;
        f = -2 * e1;
        f1 = -2 * e2;
        pA = a6;
        pB = -a3;
    } else if (pot == PMGPU_POT_COULOMB) {
        const R phi = kappa * sqrt(ia);
        e = qq * phi;
        e1 = -(R)0.5 * e * ia;
        f = e * ia;
        f1 = -(R)1.5 * e * ia * ia;
        pqq = phi;
    } else if (pot == PMGPU_POT_EWALD_REAL) {
        const R E1 = (R)0.254829592, E2 = (R)-0.284496736, E3 = (R)1.421413741, E4 = (R)-1.453152027,
                E5 = (R)1.061405429, PP = (R)0.3275911;
        const R al = (R)t.alpha, c = (R)t.two_alpha_pi;
        const R r = sqrt(a), ir = 1 / r;
        const R x = al * r;
        const R ex = exp(-x * x);
        const R tt = 1 / (1 + PP * x);
        const R H = E1 + tt * (E2 + tt * (E3 + tt * (E4 + tt * E5)));
        const R Hp = E2 + tt * (2 * E3 + tt * (3 * E4 + tt * 4 * E5));
        const R P = tt * H;
        const R Pp = -PP * tt * tt * (H + tt * Hp);            // dP/dx
        const R unit = kappa * P * ex * ir;                     // energy per unit qq
        const R unit1 = kappa * ex * ir * (Pp * x * (R)0.5 * ia - al * al * P - P * (R)0.5 * ia);
        e = qq * unit;
        e1 = qq * unit1;
        const R g = e + c * qq * kappa * ex;                    // f = g / a
        const R g1 = e1 - c * qq * kappa * al * al * ex;
        f = g * ia;
        f1 = g1 * ia - g * ia * ia;
        pqq = unit;
    }
}

__device__ __forceinline__ bool adj_table(int pot)
{
    return pot == PMGPU_POT_LENNARD_JONES_TABLE || pot == PMGPU_POT_COULOMB_TABLE ||
           pot == PMGPU_POT_EWALD_REAL_TABLE;
}

// A table potential: in each interval the table is a cubic in a = r^2
// (LookUpTableBase::interpolate, base/LookUpTableBase.h:266-272), so its
// value, de/da and d^2e/da^2 come from the same coefficients; f = -2 de/da
// is the reference's force.  Inside an interval the derivatives are exact;
// the table is C1 across intervals (value and gradient match), its second
// derivative is piecewise linear.  Per unit q~_i q~_j (Coulomb tables, the
// 1-4 factor in kappa) or per unit A and B (LennardJonesTable).
__device__ __forceinline__ void term_table(int pot, const TermD& t, double a, double qq, double A, double B,
                                           double kappa, double& e, double& e1, double& f, double& f1,
                                           double& pqq, double& pA, double& pB)
{
    const long long u = __double_as_longlong(a);
    long long k = (u >> t.tab_shift) * t.tab_step - t.tab_first;
    double dt = 0.0;
    if (k < 0) k = 0;
    else if (k > t.tab_last) k = t.tab_last;
    else dt = a - __longlong_as_double(u & ~((1ll << t.tab_shift) - 1ll));
    const double* T = t.tab + k;
    auto cubic = [dt](const double* c, double& v, double& v1, double& v2) {
        v = ((dt * c[3] + c[2]) * dt + c[1]) * dt + c[0];
        v1 = (3.0 * dt * c[3] + 2.0 * c[2]) * dt + c[1];
        v2 = 6.0 * dt * c[3] + 2.0 * c[2];
    };
    double v, v1, v2;
    pqq = pA = pB = 0.0;
    if (pot == PMGPU_POT_LENNARD_JONES_TABLE) {
        double w, w1, w2;
        cubic(T, v, v1, v2);
        cubic(T + 4, w, w1, w2);
        e = A * v + B * w;
        e1 = A * v1 + B * w1;
        f1 = -2.0 * (A * v2 + B * w2);
        pA = v;
        pB = w;
    } else {
        cubic(T, v, v1, v2);
        e = qq * kappa * v;
        e1 = qq * kappa * v1;
        f1 = -2.0 * qq * kappa * v2;
        pqq = kappa * v;
    }
    f = -2.0 * e1;
}

// The terms of one pair at a = |d|^2 (exact FP64 a for the switch and
// table decisions, R math): the switched force factor F (F_j = d F), its
// derivative F1 = dF/da, the energy's partials per unit charge product (pqq)
// and per unit LJ A and B (pA, pB), and the LJ / Coulomb energies (el, ec,
// +=, scaled by wgt).
template <typename R>
__device__ __forceinline__ void adj_pair(const AdjArgs& p, double a, double qi, double qj, double4 par, int excl,
                                         double wgt, R& F, R& F1, R& pqq, R& pA, R& pB, double& el, double& ec)
{
    const R ar = (R)a;
    const R qq = (R)(qi * qj);
    const bool mod = excl == PMGPU_EXCL_MODIFIED;
    const R A = (R)(mod ? par.z : par.x), B = (R)(mod ? par.w : par.y);
    const R kappa = (R)(mod ? p.csf : 1.0);
    F = 0; F1 = 0; pqq = 0; pA = 0; pB = 0;
    for (int t = 0; t < p.n_terms; ++t) {
        const TermD& td = p.td[t];
        R e, e1, f, f1, q1, a1, b1;
        const bool tab = adj_table(td.pot);
        if (tab) {
            // FP64 look-up whatever R; the table's switch is inside it
            double de, de1, df, df1, dq1, da1, db1;
            term_table(td.pot, td, a, qi * qj, mod ? par.z : par.x, mod ? par.w : par.y, mod ? p.csf : 1.0, de, de1,
                       df, df1, dq1, da1, db1);
            e = (R)de; e1 = (R)de1; f = (R)df; f1 = (R)df1; q1 = (R)dq1; a1 = (R)da1; b1 = (R)db1;
        } else {
            term_raw<R>(td.pot, td, ar, qq, A, B, kappa, e, e1, f, f1, q1, a1, b1);
        }
        R sv = 1, s1 = 0, s2 = 0;
        if (p.modify && !tab) switch_a<R>(td.sw, td, a, ar, sv, s1, s2);
        F += f * sv - 2 * e * s1;
        F1 += f1 * sv + f * s1 - 2 * e1 * s1 - 2 * e * s2;
        pqq += q1 * sv;
        pA += a1 * sv;
        pB += b1 * sv;
        if (td.pot == PMGPU_POT_LENNARD_JONES || td.pot == PMGPU_POT_LENNARD_JONES_TABLE)
            el += wgt * (double)(e * sv);
        else ec += wgt * (double)(e * sv);
    }
}

}  // namespace pm
