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

}  // namespace

int launch_leapfrog(int n, const double* mass, double* pos, double* vel, const double* force, double h, double hk,
                    int mode, cudaStream_t s, long long* launches)
{
    if (n <= 0) return 0;
    k_leapfrog<<<(n + 255) / 256, 256, 0, s>>>(n, mass, pos, vel, force, h, hk, mode);
    *launches += 1;
    return (int)cudaGetLastError();
}

}  // namespace pm
