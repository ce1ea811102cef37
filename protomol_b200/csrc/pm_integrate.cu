// pm_integrate.cu -- the kick / drift updates of the Leapfrog integrator on
// device-resident positions, velocities and forces.
//
// LeapfrogIntegrator::run(n) (integrators/LeapfrogIntegrator.cpp:107-120)
// without modifiers is
//   doHalfKickdoDrift   v += F h 0.5 / m;  x += v h           (:47-68)
//   calculateForces
//   n - 1 times:  doKickdoDrift   v += F h / m;  x += v h    (:70-101)
//                 calculateForces
//   doHalfKick          v += F h' / m,  h' = 0.5 dt / T      (StandardIntegrator.cpp:83-96)
// with h = dt / T (Constant::INV_TIMEFACTOR, base/pmconstants.cpp:48-49)
// and m the atom's mass.  The products and sums below keep the reference's
// operation order and are not contracted into FMAs, so a step is the
// reference's step bit for bit given the same forces.
#include "pm_kernels.h"

namespace pm {

namespace {

__global__ void __launch_bounds__(256) k_leapfrog(int n, const double* __restrict__ mass,
                                                  double* __restrict__ pos, double* __restrict__ vel,
                                                  const double* __restrict__ force, double h, double hk, int mode)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double m = mass[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const size_t k = 3 * (size_t)i + c;
        double v = vel[k];
        const double f = force[k];
        if (mode == kLeapfrogFirst)            // (F * h) * 0.5 / m
            v = __dadd_rn(v, __ddiv_rn(__dmul_rn(__dmul_rn(f, h), 0.5), m));
        else                                   // F * h / m  (h = dt/T, or h' for the last half kick)
            v = __dadd_rn(v, __ddiv_rn(__dmul_rn(f, hk), m));
        vel[k] = v;
        if (mode != kLeapfrogLast) pos[k] = __dadd_rn(pos[k], __dmul_rn(v, h));
    }
}

// the drift alone (STSIntegrator::doDrift, STSIntegrator.cpp:64-69:
// positions.intoWeightedAdd(h, velocities), x += v h)
__global__ void __launch_bounds__(256) k_drift(int n, double* __restrict__ pos, const double* __restrict__ vel,
                                               double h)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const size_t k = 3 * (size_t)i + c;
        pos[k] = __dadd_rn(pos[k], __dmul_rn(vel[k], h));
    }
}

constexpr int kConsThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();                    // red is reused from the previous call
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
    return t;
}

// the caller's cluster loop bounds
__device__ __forceinline__ void cluster_range(const ConsArgs& a, int c, int& b, int& e)
{
    b = a.cl_start[c];
    e = a.cl_start[c + 1];
}

// ModifierMetaShake::calcError: mean of |  |x2 - x1|^2 - r0^2 | / (2 r0^2)
__device__ double shake_error(const ConsArgs& a, double* red)
{
    double s = 0.0;
    for (int c = threadIdx.x; c < a.n_clusters; c += blockDim.x) {
        int b, e;
        cluster_range(a, c, b, e);
        for (int k = b; k < e; ++k) {
            const int2 p = a.atoms[k];
            const double* x1 = a.pos + 3 * (size_t)p.x;
            const double* x2 = a.pos + 3 * (size_t)p.y;
            const double dx = x2[0] - x1[0], dy = x2[1] - x1[1], dz = x2[2] - x1[2];
            const double r2 = a.rest[k] * a.rest[k];
            s += fabs(dx * dx + dy * dy + dz * dz - r2) / (2.0 * r2);
        }
    }
    return block_sum(s, red) / a.n_cons;
}

// ModifierMetaRattle::calcError: mean of | (x1 - x2) . (v1 - v2) |
__device__ double rattle_error(const ConsArgs& a, double* red)
{
    double s = 0.0;
    for (int c = threadIdx.x; c < a.n_clusters; c += blockDim.x) {
        int b, e;
        cluster_range(a, c, b, e);
        for (int k = b; k < e; ++k) {
            const int2 p = a.atoms[k];
            const double* x1 = a.pos + 3 * (size_t)p.x;
            const double* x2 = a.pos + 3 * (size_t)p.y;
            const double* v1 = a.vel + 3 * (size_t)p.x;
            const double* v2 = a.vel + 3 * (size_t)p.y;
            s += fabs((x1[0] - x2[0]) * (v1[0] - v2[0]) + (x1[1] - x2[1]) * (v1[1] - v2[1]) +
                      (x1[2] - x2[2]) * (v1[2] - v2[2]));
        }
    }
    return block_sum(s, red) / a.n_cons;
}

// One SHAKE sweep of constraint k (ModifierShake.cpp:33-80), every product and
// sum rounded on its own in the reference's order
__device__ __forceinline__ void shake_one(const ConsArgs& a, int k)
{
    const int2 p = a.atoms[k];
    double* x1 = a.pos + 3 * (size_t)p.x;
    double* x2 = a.pos + 3 * (size_t)p.y;
    double* v1 = a.vel + 3 * (size_t)p.x;
    double* v2 = a.vel + 3 * (size_t)p.y;
    const double* l1 = a.last + 3 * (size_t)p.x;
    const double* l2 = a.last + 3 * (size_t)p.y;
    const double r0 = a.rest[k];
    double pab[3], rab[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        pab[c] = __dsub_rn(x1[c], x2[c]);
        rab[c] = __dsub_rn(l1[c], l2[c]);
    }
    const double pabsq = __dadd_rn(__dadd_rn(__dmul_rn(pab[0], pab[0]), __dmul_rn(pab[1], pab[1])),
                                   __dmul_rn(pab[2], pab[2]));
    const double rabsq = __dmul_rn(r0, r0);
    const double diffsq = __dsub_rn(rabsq, pabsq);
    const double rpab = __dadd_rn(__dadd_rn(__dmul_rn(rab[0], pab[0]), __dmul_rn(rab[1], pab[1])),
                                  __dmul_rn(rab[2], pab[2]));
    const double rM1 = __ddiv_rn(1.0, a.mass[p.x]);
    const double rM2 = __ddiv_rn(1.0, a.mass[p.y]);
    const double gab = __ddiv_rn(diffsq, __dmul_rn(__dmul_rn(2.0, __dadd_rn(rM1, rM2)), rpab));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double dp = __dmul_rn(rab[c], gab);
        x1[c] = __dadd_rn(x1[c], __dmul_rn(dp, rM1));
        x2[c] = __dsub_rn(x2[c], __dmul_rn(dp, rM2));
        dp = __ddiv_rn(dp, a.dt);
        v1[c] = __dadd_rn(v1[c], __dmul_rn(dp, rM1));
        v2[c] = __dsub_rn(v2[c], __dmul_rn(dp, rM2));
    }
}

// One RATTLE update of constraint k (ModifierRattle.cpp:31-67); its virial
// term (2 dp) (x) rab into vir
__device__ __forceinline__ void rattle_one(const ConsArgs& a, int k, double* vir)
{
    const int2 p = a.atoms[k];
    const double* x1 = a.pos + 3 * (size_t)p.x;
    const double* x2 = a.pos + 3 * (size_t)p.y;
    double* v1 = a.vel + 3 * (size_t)p.x;
    double* v2 = a.vel + 3 * (size_t)p.y;
    const double rM1 = __ddiv_rn(1.0, a.mass[p.x]);
    const double rM2 = __ddiv_rn(1.0, a.mass[p.y]);
    double rab[3], vab[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        rab[c] = __dsub_rn(x1[c], x2[c]);
        vab[c] = __dsub_rn(v1[c], v2[c]);
    }
    const double rabsq = __dadd_rn(__dadd_rn(__dmul_rn(rab[0], rab[0]), __dmul_rn(rab[1], rab[1])),
                                   __dmul_rn(rab[2], rab[2]));
    const double rvab = __dadd_rn(__dadd_rn(__dmul_rn(rab[0], vab[0]), __dmul_rn(rab[1], vab[1])),
                                  __dmul_rn(rab[2], vab[2]));
    const double gab = __ddiv_rn(-rvab, __dmul_rn(__dmul_rn(a.dt, __dadd_rn(rM1, rM2)), rabsq));
    double dp[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        dp[c] = __dmul_rn(rab[c], gab);
        const double ddt = __dmul_rn(dp[c], a.dt);
        v1[c] = __dadd_rn(v1[c], __dmul_rn(ddt, rM1));
        v2[c] = __dsub_rn(v2[c], __dmul_rn(ddt, rM2));
    }
    if (vir) {
        const double fx = 2.0 * dp[0], fy = 2.0 * dp[1], fz = 2.0 * dp[2];
        const double xy = fx * rab[1], xz = fx * rab[2], yz = fy * rab[2];
        vir[0] += fx * rab[0]; vir[1] += xy; vir[2] += xz;
        vir[3] += xy; vir[4] += fy * rab[1]; vir[5] += yz;
        vir[6] += xz; vir[7] += yz; vir[8] += fz * rab[2];
    }
}

__global__ void __launch_bounds__(kConsThreads) k_shake(ConsArgs a)
{
    __shared__ double red[kConsThreads / 32];
    double err = shake_error(a, red);
    int iter = 0;
    while (err > a.eps) {
        for (int c = threadIdx.x; c < a.n_clusters; c += blockDim.x) {
            int b, e;
            cluster_range(a, c, b, e);
            for (int k = b; k < e; ++k) shake_one(a, k);
        }
        err = shake_error(a, red);    // each thread reads only its own clusters' atoms until here
        if (++iter > a.max_iter) {
            if (threadIdx.x == 0) atomicAdd(a.hits, 1);
            break;
        }
    }
}

__global__ void __launch_bounds__(kConsThreads) k_rattle(ConsArgs a)
{
    __shared__ double red[kConsThreads / 32];
    double vir[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double err = rattle_error(a, red);
    int iter = 0;
    while (err > a.eps) {
        for (int c = threadIdx.x; c < a.n_clusters; c += blockDim.x) {
            int b, e;
            cluster_range(a, c, b, e);
            for (int k = b; k < e; ++k) rattle_one(a, k, a.virial ? vir : nullptr);
        }
        err = rattle_error(a, red);
        if (++iter > a.max_iter) {
            if (threadIdx.x == 0) atomicAdd(a.hits, 1);
            break;
        }
    }
    if (a.virial)
        for (int k = 0; k < 9; ++k) {
            const double t = block_sum(vir[k], red);
            if (threadIdx.x == 0) a.virial[k] += t;
        }
}

}  // namespace

int launch_leapfrog(int n, const double* mass, double* pos, double* vel, const double* force, double h, double hk,
                    int mode, cudaStream_t s, long long* launches)
{
    if (n <= 0) return 0;
    if (mode == kLeapfrogDrift) k_drift<<<(n + 255) / 256, 256, 0, s>>>(n, pos, vel, h);
    else k_leapfrog<<<(n + 255) / 256, 256, 0, s>>>(n, mass, pos, vel, force, h, hk, mode);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_shake(const ConsArgs& a, cudaStream_t s, long long* launches)
{
    if (a.n_cons <= 0) return 0;
    k_shake<<<1, kConsThreads, 0, s>>>(a);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_rattle(const ConsArgs& a, cudaStream_t s, long long* launches)
{
    if (a.n_cons <= 0) return 0;
    k_rattle<<<1, kConsThreads, 0, s>>>(a);
    *launches += 1;
    return (int)cudaGetLastError();
}

}  // namespace pm
