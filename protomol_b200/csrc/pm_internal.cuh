// pm_internal.cuh -- shared device structures and helpers of libpmgpu.
//
// Layout in HBM (per system):
//   positions      FP64 AoS, 3N (caller's order)            24 B/atom
//   spos           float4 per cell-sorted atom: x, y, z relative to the
//                  atom's cell corner, scaled charge        16 B/atom
//   smeta          int4 per cell-sorted atom: original index, LJ type,
//                  molecule, 0                              16 B/atom
//   facc           int64 fixed-point forces, 3 per sorted atom (scale 2^32
//                  for mixed precision, 2^40 for FP64)      24 B/atom
//   cell_start     CSR offsets of the cell-sorted order, ncell + 1 ints
//   PME grid       int64 fixed-point charge grid (spread), complex
//                  half-spectrum K_x*K_y*(K_z/2+1) (FFT), real grid (gather)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>

namespace pm {

constexpr int kMaxDeltas = 1024;
constexpr int kExclWindow = 32;        // exclusion bitmask window (index delta 1..32)
constexpr double kScaleMixed = 4294967296.0;        // 2^32
constexpr double kScaleFp64 = 1099511627776.0;      // 2^40
constexpr double kFixedLimit = 4.0e18;               // |value * scale| bound before int64 overflow

// status bits written by kernels
constexpr int kStatusOverflow = 1;
constexpr int kStatusOutOfGrid = 2;
constexpr int kStatusListFull = 4;     // cluster-pair list or chunk capacity exceeded
constexpr int kStatusColumns = 8;      // a column or cluster the column path cannot take (use the cell path)
constexpr int kStatusListStale = 16;   // an atom moved more than half the pair list's skin since it was built

// FP64 constants of PeriodicBoundaryConditions::set
// (topology/PeriodicBoundaryConditions.cpp:40-77), orthogonal box.
struct Pbc {
    double e1x, e2y, e3z;       // box edge lengths (e1.x, e2.y, e3.z)
    double e1rx, e2ry, e3rz;    // inverse basis components used by rint()
    double hx, hy, hz;          // myH = max - min
    double h2x, h2y, h2z;       // myH2 = myH * 0.5
    double d;                   // myD = min(Li/2)^2
    double ox, oy, oz;          // origin
    double dx, dy, dz;          // origin - min (buildCellLists delta)
};

// Cell grid of CubicCellManager::initialize + ArrayCellListStructure
// (topology/CubicCellManager.cpp:25-42, ArrayCellListStructure.cpp:24-93).
struct CellGrid {
    int nx, ny, nz, ncell;
    double csx, csy, csz;       // myRealCellSize
    double rcsx, rcsy, rcsz;    // myRealRCellSize
};

// ---- programmatic dependent launch ----------------------------------------
// The kernels of one evaluation's critical path are launched with
// programmatic stream serialization: a kernel's blocks may be scheduled while
// the previous kernel's last blocks finish, and wait here (griddepcontrol.wait,
// sm_90+) until that kernel has completed and its memory is visible.  For a
// kernel launched without the attribute the wait returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

#ifdef __CUDACC__
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
#endif

// ---- exact FP64 arithmetic in the reference's operation order ------------
// (no FMA contraction: every product and sum rounded on its own)
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dnorm2(double x, double y, double z)
{
    return dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z));
}

// PeriodicBoundaryConditions::minimalDifference(c1, c2, distSquared)
// (topology/PeriodicBoundaryConditions.h:76-118), orthogonal branch.
__device__ __forceinline__ double pbc_min_diff(const Pbc& b, double x1, double y1, double z1,
                                               double x2, double y2, double z2,
                                               double& dx, double& dy, double& dz)
{
    dx = dsub(x2, x1); dy = dsub(y2, y1); dz = dsub(z2, z1);
    double d2 = dnorm2(dx, dy, dz);
    if (d2 > b.d) {
        if (dx < -b.h2x) dx = dadd(dx, b.hx); else if (dx > b.h2x) dx = dsub(dx, b.hx);
        if (dy < -b.h2y) dy = dadd(dy, b.hy); else if (dy > b.h2y) dy = dsub(dy, b.hy);
        if (dz < -b.h2z) dz = dadd(dz, b.hz); else if (dz > b.h2z) dz = dsub(dz, b.hz);
        d2 = dnorm2(dx, dy, dz);
        if (d2 > b.d) {
            dx = dsub(dx, dmul(b.e1x, rint(dmul(b.e1rx, dx))));
            dy = dsub(dy, dmul(b.e2y, rint(dmul(b.e2ry, dy))));
            dz = dsub(dz, dmul(b.e3z, rint(dmul(b.e3rz, dz))));
            d2 = dnorm2(dx, dy, dz);
        }
    }
    return d2;
}

// PeriodicBoundaryConditions::minimalPosition (PeriodicBoundaryConditions.h:120-150)
__device__ __forceinline__ void pbc_min_pos(const Pbc& b, double x, double y, double z,
                                            double& rx, double& ry, double& rz)
{
    double dx = dsub(x, b.ox), dy = dsub(y, b.oy), dz = dsub(z, b.oz);
    if (!(dnorm2(dx, dy, dz) <= b.d)) {
        if (dx < -b.h2x) dx = dadd(dx, b.hx); else if (dx > b.h2x) dx = dsub(dx, b.hx);
        if (dy < -b.h2y) dy = dadd(dy, b.hy); else if (dy > b.h2y) dy = dsub(dy, b.hy);
        if (dz < -b.h2z) dz = dadd(dz, b.hz); else if (dz > b.h2z) dz = dsub(dz, b.hz);
        if (!(dnorm2(dx, dy, dz) <= b.d)) {
            dx = dsub(dx, dmul(b.e1x, rint(dmul(b.e1rx, dx))));
            dy = dsub(dy, dmul(b.e2y, rint(dmul(b.e2ry, dy))));
            dz = dsub(dz, dmul(b.e3z, rint(dmul(b.e3rz, dz))));
        }
    }
    rx = dx; ry = dy; rz = dz;
}

// ---- exclusions --------------------------------------------------------------
// ExclusionTable::check (topology/ExclusionTable.h:130-146) for a pair of the
// same molecule: bit masks of the index deltas 1..kExclWindow per atom, then
// a CSR of (partner, class) sorted by partner; returns the class.
__device__ __forceinline__ int excl_lookup(const uint32_t* xfull, const uint32_t* xmod, const int* xrow,
                                           const int2* xent, int oi, int oj)
{
    int lo = min(oi, oj), hi = max(oi, oj);
    int dl = hi - lo;
    if (dl <= 0) return 0;                       // PMGPU_EXCL_NONE
    if (dl <= kExclWindow) {
        uint32_t bit = 1u << (dl - 1);
        if (__ldg(xfull + lo) & bit) return 2;    // PMGPU_EXCL_FULL
        if (__ldg(xmod + lo) & bit) return 1;     // PMGPU_EXCL_MODIFIED
        return 0;
    }
    int b = __ldg(xrow + lo), e = __ldg(xrow + lo + 1);
    while (b < e) {   // binary search on partner index
        int m = (b + e) >> 1;
        int2 v = xent[m];
        if (v.x == hi) return v.y;
        if (v.x < hi) b = m + 1; else e = m;
    }
    return 0;
}

// ---- fixed-point force accumulation ---------------------------------------
// Each contribution is rounded to an int64 multiple of 1/scale and added with
// an integer atomic, so the total is independent of summation order.
__device__ __forceinline__ void fixed_add(unsigned long long* slot, double v, double scale, int* status)
{
    double s = v * scale;
    if (!(fabs(s) < kFixedLimit)) {   // also catches NaN
        atomicOr(status, kStatusOverflow);
        return;
    }
    long long q = __double2ll_rn(s);
    if (q != 0) atomicAdd(slot, (unsigned long long)q);
}

__device__ __forceinline__ void fixed_add3(unsigned long long* base, double x, double y, double z,
                                           double scale, int* status)
{
    fixed_add(base + 0, x, scale, status);
    fixed_add(base + 1, y, scale, status);
    fixed_add(base + 2, z, scale, status);
}

// ---- energy / virial partial records ---------------------------------------
// 11 components: LENNARDJONES, COULOMB, VIRIALXX..VIRIALZZ.  Records are
// stored component-major: component k of record r at erec[k * stride + r],
// so the final reduction reads each component contiguously.
constexpr int kERec = 11;

template <int NW>
__device__ __forceinline__ void block_reduce_store(double (&v)[kERec], double* erec, int stride, int rec)
{
    // warp reduce
    for (int k = 0; k < kERec; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    __shared__ double red[NW][kERec];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < kERec; ++k) red[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < kERec) {
        double s = 0.0;
        for (int q = 0; q < NW; ++q) s += red[q][threadIdx.x];
        erec[(size_t)threadIdx.x * stride + rec] = s;
    }
}

// one record per warp, no block barrier (warps of a block finish unevenly)
__device__ __forceinline__ void warp_reduce_store(double (&v)[kERec], double* erec, int stride, int rec)
{
    for (int k = 0; k < kERec; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    int lane = threadIdx.x & 31;
    if (lane < kERec) {
        double s = v[0];
#pragma unroll
        for (int k = 1; k < kERec; ++k) if (lane == k) s = v[k];
        erec[(size_t)lane * stride + rec] = s;
    }
}

// ---- molecular virial records -------------------------------------------
// 18 components: MOLVIRIALXX..MOLVIRIALZZ, then the atomic virial of the
// pairs between different molecules (VIRIALXX..VIRIALZZ), component-major
// like the energy records
constexpr int kMRec = 18;

// ScalarStructure::addVirial / addMolVirial (base/ScalarStructure.cpp:41-88):
// the tensor f (x) d with the upper triangle mirrored
__device__ __forceinline__ void add_outer(double* v, double fx, double fy, double fz, double dx, double dy,
                                          double dz)
{
    const double xy = fx * dy, xz = fx * dz, yz = fy * dz;
    v[0] += fx * dx; v[1] += xy; v[2] += xz;
    v[3] += xy; v[4] += fy * dy; v[5] += yz;
    v[6] += xz; v[7] += yz; v[8] += fz * dz;
}

template <int NW, int N>
__device__ __forceinline__ void block_reduce_store_n(double (&v)[N], double* rec, int stride, int r)
{
    for (int k = 0; k < N; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    __shared__ double red[NW][N];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < N; ++k) red[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < N) {
        double s = 0.0;
        for (int q = 0; q < NW; ++q) s += red[q][threadIdx.x];
        rec[(size_t)threadIdx.x * stride + r] = s;
    }
}

}  // namespace pm
