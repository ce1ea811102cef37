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

#include "pm_adjoint_math.cuh"

namespace pm {

namespace {

constexpr int kTile = 128;
constexpr int kSmemTypes = 32;       // LJ table gradient staged in shared memory below this

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
            const double4 par = p.ljd[(size_t)ti * p.n_types + s_type[jj]];
            const bool mod = excl == PMGPU_EXCL_MODIFIED;
            R F, F1, pqq, pA, pB;
            adj_pair<R>(p, a, qi, s_q[jj], par, excl, 0.5, F, F1, pqq, pA, pB, el, ec);
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
