// pm_adjoint.cu -- K10: backward pass of the nonbonded pair terms.
//
// For the pair terms of a force (the OneAtomPair[Two] potentials and
// switches of the cutoff path, or all pairs without a cutoff), one kernel
// recomputes every pair -- nothing of the forward evaluation is stored -- and
// accumulates
//   dE/dq~_i        gradient of the energy w.r.t. the scaled charges,
//   dE/dA, dE/dB    w.r.t. the Lennard-Jones table entries (A, B, A14, B14
//                   of the pair's type pair, each pair split evenly between
//                   (t_i, t_j) and (t_j, t_i)),
//   (H v)_i         the Hessian-vector product: the force Jacobian applied to
//                   a displacement v, with the blocks of integrators/
//                   Hessian.cpp:456-623 (ReducedHessLennardJones.cpp:7-51,
//                   ReducedHessCoulomb.cpp:8-43, C2SwitchingFunction::hessian
//                   C2SwitchingFunction.cpp:45-53): per pair
//                   K = -(F I + 2 F'(a) d d^T), a = |d|^2, F the switched
//                   force factor (F_j = d F), added as K to the ii and jj
//                   blocks and -K to the ij blocks.
// Every ordered pair (i, j != i) is visited by the thread of i, so each atom
// accumulates only its own outputs (no per-pair atomics except the LJ table).
// The cutoff decision and the minimal image are exact FP64 (as in the forward
// kernels); the pair math runs in R = double or float.

#include "pm_kernels.h"
#include "../../include/pmgpu.h"

namespace pm {

namespace {

constexpr int kTile = 128;
constexpr int kSmemTypes = 32;       // LJ table gradient staged in shared memory below this

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
struct TermOut {
    double e, f, f1, pqq, pA, pB;
};

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

template <typename R>
__global__ void __launch_bounds__(kTile) k_pair_adjoint(AdjArgs p)
{
    __shared__ double s_pos[kTile][3];
    __shared__ double s_q[kTile];
    __shared__ int s_type[kTile], s_mol[kTile];
    __shared__ double s_v[kTile][3];
    __shared__ double s_lj[kSmemTypes * kSmemTypes * 4];
    const bool lj_smem = p.dlj && p.n_types <= kSmemTypes;
    if (lj_smem)
        for (int k = threadIdx.x; k < p.n_types * p.n_types * 4; k += kTile) s_lj[k] = 0.0;
    const int i = blockIdx.x * kTile + threadIdx.x;
    const int j0 = blockIdx.y * kTile;
    {
        const int j = j0 + threadIdx.x;
        if (j < p.n) {
            for (int c = 0; c < 3; ++c) {
                s_pos[threadIdx.x][c] = p.pos[3 * (size_t)j + c];
                s_v[threadIdx.x][c] = p.v ? p.v[3 * (size_t)j + c] : 0.0;
            }
            s_q[threadIdx.x] = p.q[j];
            s_type[threadIdx.x] = p.type[j];
            s_mol[threadIdx.x] = p.mol[j];
        }
    }
    __syncthreads();
    double dq = 0.0, hv[3] = {0.0, 0.0, 0.0}, el = 0.0, ec = 0.0;
    double fi[3] = {0.0, 0.0, 0.0}, vir[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double hd[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};   // the ii block of the dense Hessian
    if (i < p.n) {
        const double xi = p.pos[3 * (size_t)i], yi = p.pos[3 * (size_t)i + 1], zi = p.pos[3 * (size_t)i + 2];
        const double qi = p.q[i];
        const int ti = p.type[i], mi = p.mol[i];
        double vi[3] = {0.0, 0.0, 0.0};
        if (p.v) for (int c = 0; c < 3; ++c) vi[c] = p.v[3 * (size_t)i + c];
        const int jn = min(kTile, p.n - j0);
        for (int jj = 0; jj < jn; ++jj) {
            const int j = j0 + jj;
            if (j == i) continue;
            double dx, dy, dz, a;
            if (p.periodic) {
                a = pbc_min_diff(p.pbc, xi, yi, zi, s_pos[jj][0], s_pos[jj][1], s_pos[jj][2], dx, dy, dz);
            } else {   // vacuum: plain difference
                dx = dsub(s_pos[jj][0], xi); dy = dsub(s_pos[jj][1], yi); dz = dsub(s_pos[jj][2], zi);
                a = dnorm2(dx, dy, dz);
            }
            if (p.use_cut && a > p.cut2d) continue;
            int excl = PMGPU_EXCL_NONE;
            if (mi == s_mol[jj]) {
                excl = excl_lookup(p.xfull, p.xmod, p.xrow, p.xent, i, j);
                if (excl == PMGPU_EXCL_FULL) continue;
            }
            const R ar = (R)a;
            const R qq = (R)(qi * s_q[jj]);
            const double4 par = p.ljd[(size_t)ti * p.n_types + s_type[jj]];
            const bool mod = excl == PMGPU_EXCL_MODIFIED;
            const R A = (R)(mod ? par.z : par.x), B = (R)(mod ? par.w : par.y);
            const R kappa = (R)(mod ? p.csf : 1.0);
            R F = 0, F1 = 0, pqq = 0, pA = 0, pB = 0;
            for (int t = 0; t < p.n_terms; ++t) {
                const TermD& td = p.td[t];
                R e, e1, f, f1, q1, a1, b1;
                const bool tab = adj_table(td.pot);
                if (tab) {
                    // FP64 look-up whatever R; the table's switch is inside it
                    double de, de1, df, df1, dq1, da1, db1;
                    term_table(td.pot, td, a, qi * s_q[jj], mod ? par.z : par.x, mod ? par.w : par.y,
                               mod ? p.csf : 1.0, de, de1, df, df1, dq1, da1, db1);
                    e = (R)de; e1 = (R)de1; f = (R)df; f1 = (R)df1; q1 = (R)dq1; a1 = (R)da1; b1 = (R)db1;
                } else {
                    term_raw<R>(td.pot, td, ar, qq, A, B, kappa, e, e1, f, f1, q1, a1, b1);
                }
                R s = 1, s1 = 0, s2 = 0;
                if (p.modify && !tab) switch_a<R>(td.sw, td, a, ar, s, s1, s2);
                F += f * s - 2 * e * s1;
                F1 += f1 * s + f * s1 - 2 * e1 * s1 - 2 * e * s2;
                pqq += q1 * s;
                pA += a1 * s;
                pB += b1 * s;
                if (td.pot == PMGPU_POT_LENNARD_JONES || td.pot == PMGPU_POT_LENNARD_JONES_TABLE)
                    el += 0.5 * (double)(e * s);
                else ec += 0.5 * (double)(e * s);
            }
            dq += (double)pqq * s_q[jj];
            if (p.facc) {   // F_i = -d F; the pair's virial d (x) d F, half per ordered pair
                const double fd = (double)F;
                fi[0] -= dx * fd; fi[1] -= dy * fd; fi[2] -= dz * fd;
                if (p.virial) {
                    const double h = 0.5 * fd;
                    vir[0] += h * dx * dx; vir[1] += h * dx * dy; vir[2] += h * dx * dz;
                    vir[3] += h * dy * dy; vir[4] += h * dy * dz; vir[5] += h * dz * dz;
                }
            }
            if (p.v) {
                // (H v)_i += -K (v_j - v_i),  K = -(F I + 2 F' d d^T)
                const double ux = s_v[jj][0] - vi[0], uy = s_v[jj][1] - vi[1], uz = s_v[jj][2] - vi[2];
                const double du = dx * ux + dy * uy + dz * uz;
                const double two_f1 = 2.0 * (double)F1;
                hv[0] += (double)F * ux + two_f1 * du * dx;
                hv[1] += (double)F * uy + two_f1 * du * dy;
                hv[2] += (double)F * uz + two_f1 * du * dz;
            }
            if (p.hess) {
                // H_ij = F I + 2 F' d d^T (the HVP's block above); H_ii = -sum_j H_ij.
                // Row block i belongs to this thread: no other thread writes H_ij.
                const double fF = (double)F, t2 = 2.0 * (double)F1;
                const double d[3] = {dx, dy, dz};
                const size_t ld = 3 * (size_t)p.n;
                double* row = p.hess + 3 * (size_t)i * ld + 3 * (size_t)j;
#pragma unroll
                for (int ra = 0; ra < 3; ++ra)
#pragma unroll
                    for (int cb = 0; cb < 3; ++cb) {
                        const double b = (ra == cb ? fF : 0.0) + t2 * d[ra] * d[cb];
                        row[ra * ld + cb] += b;
                        hd[3 * ra + cb] -= b;
                    }
            }
            if (p.dlj && (pA != 0 || pB != 0)) {
                const size_t k = ((size_t)ti * p.n_types + s_type[jj]) * 4 + (mod ? 2 : 0);
                if (lj_smem) {
                    atomicAdd(s_lj + k, 0.5 * (double)pA);
                    atomicAdd(s_lj + k + 1, 0.5 * (double)pB);
                } else {
                    atomicAdd(p.dlj + k, 0.5 * (double)pA);
                    atomicAdd(p.dlj + k + 1, 0.5 * (double)pB);
                }
            }
        }
        if (p.dq && dq != 0.0) atomicAdd(p.dq + i, dq);
        if (p.hess) {   // the diagonal block sums over the j tiles of other blocks too
            const size_t ld = 3 * (size_t)p.n;
            for (int ra = 0; ra < 3; ++ra)
                for (int cb = 0; cb < 3; ++cb)
                    if (hd[3 * ra + cb] != 0.0) atomicAdd(p.hess + (3 * (size_t)i + ra) * ld + 3 * (size_t)i + cb,
                                                          hd[3 * ra + cb]);
        }
        if (p.hv)
            for (int c = 0; c < 3; ++c)
                if (hv[c] != 0.0) atomicAdd(p.hv + 3 * (size_t)i + c, hv[c]);
        if (p.energy) {
            if (el != 0.0) atomicAdd(p.energy, el);
            if (ec != 0.0) atomicAdd(p.energy + 1, ec);
        }
        if (p.facc) fixed_add3(p.facc + 3 * (size_t)i, fi[0], fi[1], fi[2], p.scale, p.status);
    }
    if (p.erec) {
        double acc[kERec] = {el, ec, vir[0], vir[1], vir[2], vir[1], vir[3], vir[4], vir[2], vir[4], vir[5]};
        block_reduce_store<kTile / 32>(acc, p.erec, p.erec_stride, blockIdx.y * gridDim.x + blockIdx.x);
    }
    if (lj_smem) {
        __syncthreads();
        for (int k = threadIdx.x; k < p.n_types * p.n_types * 4; k += kTile)
            if (s_lj[k] != 0.0) atomicAdd(p.dlj + k, s_lj[k]);
    }
}

}  // namespace

int adjoint_blocks(int n)
{
    const int t = (n + kTile - 1) / kTile;
    return t * t;
}

int launch_pair_adjoint(const AdjArgs& a, int fp64, cudaStream_t s, long long* launches)
{
    if (a.n <= 0) return 0;
    const int t = (a.n + kTile - 1) / kTile;
    dim3 grid(t, t);
    if (fp64) k_pair_adjoint<double><<<grid, kTile, 0, s>>>(a);
    else k_pair_adjoint<float><<<grid, kTile, 0, s>>>(a);
    *launches += 1;
    return (int)cudaGetLastError();
}

}  // namespace pm
