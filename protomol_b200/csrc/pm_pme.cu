// pm_pme.cu -- K3 spread, K4/K5 3-D FFT with the fused reciprocal
// convolution, K6 gather and K7 Ewald correction of the particle-mesh Ewald
// force (NonbondedPMEwaldSystemForce, forces/NonbondedPMEwaldSystemForce.h).
//
// Grid conventions follow Grid<BSpline> (base/Grid.h): grid coordinate
// u = x K / L (no origin shift) wrapped into [0, K) by repeated +-K, base
// index floor(u) - (P-1)/2 + K, weights BSpline::set(u - floor(u))
// (base/BSpline.cpp:64-117); reciprocal energy and virial as
// Grid::scalarSum (base/Grid.h:276-389) summed over the full spectrum; the
// convolved grid is the real part of the unnormalised inverse transform;
// forces as Grid::interpolateForce (base/Grid.h:193-228).
//
// The complex-to-complex ZFFT of the reference (base/fft.c, FFTComplex.cpp)
// is replaced by a real-to-complex transform: z lines r2c into the half
// spectrum K_x * K_y * (K_z/2 + 1), then complex passes along y and x.  The
// x pass is fused with the convolution: a CTA transforms a tile of x-lines
// forward, multiplies by theta(m) while summing energy and virial in FP64,
// transforms back and writes once.  Each pass is one read and one write of
// the half spectrum, with the lines staged in shared memory and transformed
// there by a mixed-radix (4, 2, 3, 5, generic) Stockham FFT.
//
// Mixed precision: the charge grid is accumulated in int64 fixed point
// (deterministic), the FFT and gather run in FP32.  FP64: double grid with
// FP64 atomics, FP64 FFT and gather.
#include <algorithm>

#include "pm_kernels.h"
#include "../../include/pmgpu.h"

namespace pm {

template <typename R> struct Cx;
template <> struct Cx<float> { typedef float2 T; };
template <> struct Cx<double> { typedef double2 T; };

template <typename C> __device__ __forceinline__ C cmul(C a, C b)
{
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cconj_if(C a, bool c) { if (c) a.y = -a.y; return a; }

// Stockham plan of one line length: radices (4 first, then 2, 3, 5, 7: the
// reference's FFT handles the same factors) and, per stage, the sizes the kernel divides by
// (exact multiply-high reciprocals: every index here is below 2^15) and the
// twiddle stride n / (Ns R)
struct FftPlan {
    int n;
    int nrad;
    int rad[16];
    int m[16];                 // n / R
    int ns[16];                // product of the earlier radices
    unsigned m_rcp[16];        // ceil(2^32 / m)
    unsigned ns_rcp[16];       // ceil(2^32 / ns)
    int tws[16];               // n / (ns R)
};

__device__ __forceinline__ int fdiv(int x, unsigned rcp) { return (int)__umulhi((unsigned)x, rcp); }

// the table's n-th roots exp(-2 pi i k / n), conjugated for sign > 0
template <typename C>
__device__ __forceinline__ C tw_at(const C* tw, int k, int sign)
{
    C w = tw[k];
    if (sign > 0) w.y = -w.y;
    return w;
}

// RAD-point DFT of v in registers, exp(sign 2 pi i jk / RAD)
template <typename C, typename R, int RAD>
__device__ __forceinline__ void dft_fixed(C (&v)[RAD], int sign, const C* tw, int n)
{
    if (RAD == 2) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    } else if (RAD == 4) {
        C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        C c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        C di; di.x = -sign * d.y; di.y = sign * d.x;          // d * (sign i)
        v[0] = cadd(a, c); v[2] = csub(a, c);
        v[1] = cadd(b, di); v[3] = csub(b, di);
    } else if (RAD == 3) {
        const R c1 = (R)-0.5, s1 = (R)0.86602540378443864676 * (R)sign;
        C a = v[0], b = v[1], c = v[2];
        C t; t.x = b.x + c.x; t.y = b.y + c.y;
        C m; m.x = a.x + c1 * t.x; m.y = a.y + c1 * t.y;
        C d; d.x = -s1 * (b.y - c.y); d.y = s1 * (b.x - c.x);
        v[0].x = a.x + t.x; v[0].y = a.y + t.y;
        v[1] = cadd(m, d); v[2] = csub(m, d);
    } else if (RAD == 5) {
        const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
        const R s1 = (R)0.95105651629515357212 * (R)sign, s2 = (R)0.58778525229247312917 * (R)sign;
        C a = v[0];
        C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        C u1 = csub(v[1], v[4]), u2 = csub(v[2], v[3]);
        C m1; m1.x = a.x + c1 * t1.x + c2 * t2.x; m1.y = a.y + c1 * t1.y + c2 * t2.y;
        C m2; m2.x = a.x + c2 * t1.x + c1 * t2.x; m2.y = a.y + c2 * t1.y + c1 * t2.y;
        C n1; n1.x = -(s1 * u1.y + s2 * u2.y); n1.y = s1 * u1.x + s2 * u2.x;
        C n2; n2.x = -(s2 * u1.y - s1 * u2.y); n2.y = s2 * u1.x - s1 * u2.x;
        v[0].x = a.x + t1.x + t2.x; v[0].y = a.y + t1.y + t2.y;
        v[1] = cadd(m1, n1); v[4] = csub(m1, n1);
        v[2] = cadd(m2, n2); v[3] = csub(m2, n2);
    } else {
        // 7: direct DFT with the roots exp(sign 2 pi i jk / RAD) = table[(jk mod RAD) n / RAD]
        C out[RAD];
#pragma unroll
        for (int k = 0; k < RAD; ++k) {
            C s = v[0];
#pragma unroll
            for (int j = 1; j < RAD; ++j) s = cadd(s, cmul(v[j], tw_at(tw, ((j * k) % RAD) * (n / RAD), sign)));
            out[k] = s;
        }
#pragma unroll
        for (int k = 0; k < RAD; ++k) v[k] = out[k];
    }
}

// one Stockham stage of radix RAD over `lines` lines (stride ld) in shared memory
template <typename C, typename R, int RAD>
__device__ __forceinline__ void fft_stage(const C* a, C* b, int lines, int ld, const FftPlan& pl, int s,
                                          const C* tw, int sign)
{
    const int m = pl.m[s], Ns = pl.ns[s], tws = pl.tws[s];
    for (int idx = threadIdx.x; idx < lines * m; idx += blockDim.x) {
        const int line = m > 1 ? fdiv(idx, pl.m_rcp[s]) : idx;
        const int j = idx - line * m;
        const int jq = Ns > 1 ? fdiv(j, pl.ns_rcp[s]) : j;
        const int k = j - jq * Ns;
        const C* in = a + line * ld;
        C* out = b + line * ld;
        C v[RAD];
#pragma unroll
        for (int r = 0; r < RAD; ++r) v[r] = in[j + r * m];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < RAD; ++r) v[r] = cmul(v[r], tw_at(tw, k * r * tws, sign));   // k r < Ns RAD
        }
        dft_fixed<C, R, RAD>(v, sign, tw, pl.n);
        const int base = jq * Ns * RAD + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) out[base + r * Ns] = v[r];
    }
}

// Stockham FFT of `lines` lines of length pl.n in shared memory (a -> b ->
// a ...), exp(sign 2 pi i jk / n), unnormalised; returns the buffer holding
// the result.  tw: the n-th roots, staged in shared memory by the caller.
template <typename C, typename R>
__device__ C* fft_lines(C* a, C* b, int lines, int ld, const FftPlan& pl, const C* tw, int sign)
{
    for (int s = 0; s < pl.nrad; ++s) {
        switch (pl.rad[s]) {
        case 2: fft_stage<C, R, 2>(a, b, lines, ld, pl, s, tw, sign); break;
        case 3: fft_stage<C, R, 3>(a, b, lines, ld, pl, s, tw, sign); break;
        case 4: fft_stage<C, R, 4>(a, b, lines, ld, pl, s, tw, sign); break;
        case 5: fft_stage<C, R, 5>(a, b, lines, ld, pl, s, tw, sign); break;
        default: fft_stage<C, R, 7>(a, b, lines, ld, pl, s, tw, sign); break;
        }
        __syncthreads();
        C* t = a; a = b; b = t;
    }
    return a;
}

// ------------------------------------------------------------------ spread
__device__ __forceinline__ double wrap_grid(double x, int K)
{
    // while (x < 0.0) x += K; while (x >= K) x -= K;  (bounded: positions
    // more than 64 boxes away are reduced with floor first)
    if (!(fabs(x) < 64.0 * K)) x = x - (double)K * floor(x / (double)K);
    int it = 0;
    while (x < 0.0 && it < 256) { x += K; ++it; }
    while (x >= (double)K && it < 512) { x -= K; ++it; }
    return x;
}

template <typename R>
__device__ __forceinline__ void bspline4(R w, R* th, R* dth, int order)
{
    // BSpline::set (base/BSpline.cpp:64-117) for any order >= 3
    th[order - 1] = (R)0;
    th[1] = w;
    th[0] = (R)1 - w;
    for (int k = 2; k < order - 1; k++) {
        R div = (R)1 / (R)k;
        th[k] = div * w * th[k - 1];
        for (int j = 1; j < k; j++)
            th[k - j] = div * ((w + (R)j) * th[k - j - 1] + ((R)(k + 1 - j) - w) * th[k - j]);
        th[0] = div * ((R)1 - w) * th[0];
    }
    dth[0] = -th[0];
    for (int j = 1; j <= order - 1; j++) dth[j] = th[j - 1] - th[j];
    R div = (R)1 / (R)(order - 1);
    th[order - 1] = div * w * th[order - 2];
    for (int j = 1; j < order - 1; j++)
        th[order - 1 - j] = div * ((w + (R)j) * th[order - j - 2] + ((R)(order - j) - w) * th[order - 1 - j]);
    th[0] = div * ((R)1 - w) * th[0];
}

constexpr int kMaxOrder = 12;

template <typename R>
__device__ __forceinline__ void grid_point(const PmeArgs& a, int atom, int& i0, int& j0, int& k0,
                                           R* tx, R* dtx, R* ty, R* dty, R* tz, R* dtz)
{
    double x = wrap_grid(a.pos[3 * (size_t)atom] * a.hxr, a.kx);
    double y = wrap_grid(a.pos[3 * (size_t)atom + 1] * a.hyr, a.ky);
    double z = wrap_grid(a.pos[3 * (size_t)atom + 2] * a.hzr, a.kz);
    int ix = (int)x, iy = (int)y, iz = (int)z;
    i0 = ix + a.offx; j0 = iy + a.offy; k0 = iz + a.offz;
    if (a.order == 2) {
        R wx = (R)(x - ix), wy = (R)(y - iy), wz = (R)(z - iz);
        tx[1] = wx; tx[0] = (R)1 - wx; dtx[1] = 1; dtx[0] = -1;
        ty[1] = wy; ty[0] = (R)1 - wy; dty[1] = 1; dty[0] = -1;
        tz[1] = wz; tz[0] = (R)1 - wz; dtz[1] = 1; dtz[0] = -1;
    } else {
        bspline4<R>((R)(x - ix), tx, dtx, a.order);
        bspline4<R>((R)(y - iy), ty, dty, a.order);
        bspline4<R>((R)(z - iz), tz, dtz, a.order);
    }
}

template <typename R>
__global__ void k_spread(PmeArgs a)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n) return;
    int atom = a.sorted ? a.sorted[s] : s;
    R tx[kMaxOrder], dtx[kMaxOrder], ty[kMaxOrder], dty[kMaxOrder], tz[kMaxOrder], dtz[kMaxOrder];
    int i0, j0, k0;
    grid_point<R>(a, atom, i0, j0, k0, tx, dtx, ty, dty, tz, dtz);
    // the charge multiplies in FP64: every atom of a type shares its charge,
    // so an FP32-rounded charge would scale the whole grid systematically
    const double qs = a.q[atom] * a.qscale;
    const int P = a.order;
    for (int i = 0; i < P; i++) {
        int i1 = (i + i0) % a.kx;
        for (int j = 0; j < P; j++) {
            R ab = tx[i] * ty[j];
            int j1 = (j + j0) % a.ky;
            size_t row = ((size_t)i1 * a.ky + j1) * a.kz;
            for (int k = 0; k < P; k++) {
                int k1 = (k + k0) % a.kz;
                R v = ab * tz[k];
                // int64 fixed point: deterministic, order-independent grid sums
                long long qv = __double2ll_rn(qs * (double)v);
                if (qv) atomicAdd((unsigned long long*)(a.qgrid + row + k1), (unsigned long long)qv);
            }
        }
    }
}

// ------------------------------------------------------------------ FFT passes
constexpr int kModeZR2C = 0, kModeY = 1, kModeXConv = 2, kModeZC2R = 3;
// forward x transform and Grid::scalarSum's energy / virial only (no
// convolution written back, no inverse): the FP64 energy of a mixed force
constexpr int kModeXEnergy = 4;

struct PassArgs {
    PmeArgs a;
    FftPlan plan;
    int lines;        // lines per CTA
    int ld;           // smem line stride
    int sign;
    int tw_off;
    int erec_off;
    int store_energy;  // kModeXConv: write the energy / virial records
};

template <typename R, int MODE>
__global__ void __launch_bounds__(256, 2) k_fft_pass(PassArgs pa)
{
    pdl_wait();
    typedef typename Cx<R>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* buf0 = (C*)smem_raw;
    C* buf1 = buf0 + pa.lines * pa.ld;
    const PmeArgs& a = pa.a;
    const FftPlan& pl = pa.plan;
    const int n = pl.n;
    // the n-th roots of this axis in shared memory (read by every stage);
    // the barrier after the line loads below covers them
    C* stw = buf1 + pa.lines * pa.ld;
    {
        const C* gtw = (const C*)a.tw + pa.tw_off;
        for (int k = threadIdx.x; k < n; k += blockDim.x) stw[k] = gtw[k];
    }
    const C* tw = stw;
    C* cg = (C*)a.cgrid;
    int L = pa.lines;
    double acc[kERec];
    for (int k = 0; k < kERec; ++k) acc[k] = 0.0;

    if (MODE == kModeZR2C || MODE == kModeZC2R) {
        // lines along z (contiguous); CTA handles L consecutive (x, y) lines
        int nlines = a.kx * a.ky;
        int l0 = blockIdx.x * L;
        int nl = min(L, nlines - l0);
        if (MODE == kModeZR2C) {
            for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
                int l = idx / n, z = idx - l * n;
                size_t g = (size_t)(l0 + l) * a.kz + z;
                R v = (R)((double)a.qgrid[g] * (1.0 / a.qscale));
                C c; c.x = v; c.y = 0;
                buf0[l * pa.ld + z] = c;
            }
        } else {
            for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
                int l = idx / n, z = idx - l * n;
                C c;
                if (z < a.kzh) c = cg[(size_t)(l0 + l) * a.kzh + z];
                else { c = cg[(size_t)(l0 + l) * a.kzh + (n - z)]; c.y = -c.y; }
                buf0[l * pa.ld + z] = c;
            }
        }
        __syncthreads();
        C* r = fft_lines<C, R>(buf0, buf1, nl, pa.ld, pl, tw, pa.sign);
        if (MODE == kModeZR2C) {
            for (int idx = threadIdx.x; idx < nl * a.kzh; idx += blockDim.x) {
                int l = idx / a.kzh, z = idx - l * a.kzh;
                cg[(size_t)(l0 + l) * a.kzh + z] = r[l * pa.ld + z];
            }
        } else {
            R* rg = (R*)a.rgrid;
            for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
                int l = idx / n, z = idx - l * n;
                rg[(size_t)(l0 + l) * a.kz + z] = r[l * pa.ld + z].x;
            }
        }
        return;
    }

    // lines along y (fixed x) or x (fixed y): tile of L consecutive zh
    int ntile = (a.kzh + L - 1) / L;
    int outer = blockIdx.x / ntile;         // x for Y pass, y for X pass
    int zh0 = (blockIdx.x - outer * ntile) * L;
    int nl = min(L, a.kzh - zh0);
    size_t stride, base;
    if (MODE == kModeY) { stride = a.kzh; base = (size_t)outer * a.ky * a.kzh + zh0; }
    else { stride = (size_t)a.ky * a.kzh; base = (size_t)outer * a.kzh + zh0; }
    for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
        int e = idx / nl, l = idx - e * nl;     // consecutive threads: consecutive zh
        buf0[l * pa.ld + e] = cg[base + e * stride + l];
    }
    __syncthreads();
    C* r = fft_lines<C, R>(buf0, buf1, nl, pa.ld, pl, tw, pa.sign);
    if (MODE == kModeXConv || MODE == kModeXEnergy) {
        // theta(m) multiply + energy / virial (Grid::scalarSum) on the
        // forward-transformed x-lines, then the inverse x transform
        int y = outer;
        int y0 = y <= a.ky / 2 ? y : y - a.ky;
        double my = y0 * a.lr;
        double by = a.bfac[a.kx + y], ey = a.efac[a.kx + y];
        for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
            int l = idx / n, x = idx - l * n;
            int z = zh0 + l;
            int x0 = x <= a.kx / 2 ? x : x - a.kx;
            double mx = x0 * a.wr, mz = z * a.hr;
            C& c = r[l * pa.ld + x];
            if (x == 0 && y == 0 && z == 0) { c.x = 0; c.y = 0; continue; }
            double m2 = mx * mx + my * my + mz * mz;
            double theta = a.bfac[x] * by * a.bfac[a.kx + a.ky + z] * a.efac[x] * ey *
                           a.efac[a.kx + a.ky + z] * a.piVr / m2;
            double qv = (double)c.x * (double)c.x + (double)c.y * (double)c.y;
            double e = qv * theta;
            if (z > 0 && (z != a.kz / 2 || (a.kz & 1))) e *= 2.0;
            acc[1] += e;
            if (a.virial) {
                double v = 2.0 * (1.0 / m2 + a.fac);
                acc[2] += e * (1.0 - v * mx * mx); acc[3] -= e * (v * mx * my); acc[4] -= e * (v * mx * mz);
                acc[6] += e * (1.0 - v * my * my); acc[7] -= e * (v * my * mz);
                acc[10] += e * (1.0 - v * mz * mz);
            }
            if (MODE == kModeXConv) {
                c.x = (R)(c.x * theta);
                c.y = (R)(c.y * theta);
            }
        }
        if (MODE == kModeXConv) {
            __syncthreads();
            C* other = (r == buf0) ? buf1 : buf0;
            r = fft_lines<C, R>(r, other, nl, pa.ld, pl, tw, +1);
        }
    }
    if (MODE != kModeXEnergy) {
        for (int idx = threadIdx.x; idx < nl * n; idx += blockDim.x) {
            int e = idx / nl, l = idx - e * nl;
            cg[base + e * stride + l] = r[l * pa.ld + e];
        }
    }
    if ((MODE == kModeXConv && pa.store_energy) || MODE == kModeXEnergy) {
        for (int k = 0; k < kERec; ++k) acc[k] *= 0.5;
        acc[5] = acc[3]; acc[8] = acc[4]; acc[9] = acc[7];
        block_reduce_store<8>(acc, a.erec, a.erec_stride, pa.erec_off + blockIdx.x);
    }
}

// ------------------------------------------------------------------ gather
template <typename R>
__global__ void k_gather(PmeArgs a)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n) return;
    int atom = a.sorted ? a.sorted[s] : s;
    R tx[kMaxOrder], dtx[kMaxOrder], ty[kMaxOrder], dty[kMaxOrder], tz[kMaxOrder], dtz[kMaxOrder];
    int i0, j0, k0;
    grid_point<R>(a, atom, i0, j0, k0, tx, dtx, ty, dty, tz, dtz);
    const R* g = (const R*)a.rgrid;
    R fx = 0, fy = 0, fz = 0;
    const int P = a.order;
    for (int i = 0; i < P; i++) {
        int i1 = (i + i0) % a.kx;
        for (int j = 0; j < P; j++) {
            int j1 = (j + j0) % a.ky;
            R xij = dtx[i] * ty[j], yij = tx[i] * dty[j], zij = tx[i] * ty[j];
            size_t row = ((size_t)i1 * a.ky + j1) * a.kz;
            for (int k = 0; k < P; k++) {
                int k1 = (k + k0) % a.kz;
                R term = g[row + k1];
                fx -= term * xij * tz[k];
                fy -= term * yij * tz[k];
                fz -= term * zij * dtz[k];
            }
        }
    }
    double q = a.q[atom];
    // cell-sorted slot, or the atom itself when neither map is given
    int slot = a.sorted ? s : (a.slot_of ? a.slot_of[atom] : atom);
    fixed_add3(a.facc + 3 * (size_t)slot, (double)fx * a.hxr * q, (double)fy * a.hyr * q,
               (double)fz * a.hzr * q, a.scale, a.status);
}

// dE_recip/dq~_i: the convolved grid interpolated at the atom (the gather
// above without the derivative), so that E_recip = 1/2 sum_i q~_i phi_i
template <typename R>
__global__ void k_gather_potential(PmeArgs a, double* phi)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n) return;
    int atom = a.sorted ? a.sorted[s] : s;
    R tx[kMaxOrder], dtx[kMaxOrder], ty[kMaxOrder], dty[kMaxOrder], tz[kMaxOrder], dtz[kMaxOrder];
    int i0, j0, k0;
    grid_point<R>(a, atom, i0, j0, k0, tx, dtx, ty, dty, tz, dtz);
    const R* g = (const R*)a.rgrid;
    double acc = 0.0;
    const int P = a.order;
    for (int i = 0; i < P; i++) {
        int i1 = (i + i0) % a.kx;
        for (int j = 0; j < P; j++) {
            int j1 = (j + j0) % a.ky;
            R ab = tx[i] * ty[j];
            size_t row = ((size_t)i1 * a.ky + j1) * a.kz;
            R sum = 0;
            for (int k = 0; k < P; k++) sum += g[row + (k + k0) % a.kz] * tz[k];
            acc += (double)(ab * sum);
        }
    }
    phi[atom] += acc;
}

static void make_plan(int n, FftPlan& p)
{
    p.n = n;
    p.nrad = 0;
    int m = n;
    // radix 4 rather than 8: a radix-8 butterfly (measured) carried ten times
    // the reciprocal-energy error of the radix-4 chain on the same grids
    const int radices[5] = {4, 2, 3, 5, 7};
    for (int r : radices)
        while (m % r == 0 && p.nrad < 16) { p.rad[p.nrad++] = r; m /= r; }
    if (m > 1) { p.nrad = -1; return; }   // a prime factor above 7: unsupported
    int ns = 1;
    for (int s = 0; s < p.nrad; ++s) {
        const int r = p.rad[s];
        p.m[s] = n / r;
        p.ns[s] = ns;
        // ceil(2^32 / d); d = 1 is handled without a division in the kernel
        p.m_rcp[s] = p.m[s] > 1 ? (unsigned)((0x100000000ull + p.m[s] - 1) / p.m[s]) : 0u;
        p.ns_rcp[s] = ns > 1 ? (unsigned)((0x100000000ull + ns - 1) / ns) : 0u;
        p.tws[s] = n / (ns * r);
        ns *= r;
    }
}

// ---- order-P kernels with the order known at compile time (P = 4, the
// default): spline weights and grid indices in registers, every index
// wrapped once per axis (i0 + p lies in [K - 1, 2K + 1] for P = 4)
template <typename R, int P>
__device__ __forceinline__ void bspline_fixed(R w, R (&th)[P], R (&dth)[P])
{
    // BSpline::set (base/BSpline.cpp:64-117), the recurrences of bspline4
    th[P - 1] = (R)0;
    th[1] = w;
    th[0] = (R)1 - w;
#pragma unroll
    for (int k = 2; k < P - 1; k++) {
        const R div = (R)1 / (R)k;
        th[k] = div * w * th[k - 1];
#pragma unroll
        for (int j = 1; j < k; j++)
            th[k - j] = div * ((w + (R)j) * th[k - j - 1] + ((R)(k + 1 - j) - w) * th[k - j]);
        th[0] = div * ((R)1 - w) * th[0];
    }
    dth[0] = -th[0];
#pragma unroll
    for (int j = 1; j <= P - 1; j++) dth[j] = th[j - 1] - th[j];
    const R div = (R)1 / (R)(P - 1);
    th[P - 1] = div * w * th[P - 2];
#pragma unroll
    for (int j = 1; j < P - 1; j++)
        th[P - 1 - j] = div * ((w + (R)j) * th[P - j - 2] + ((R)(P - j) - w) * th[P - 1 - j]);
    th[0] = div * ((R)1 - w) * th[0];
}

__device__ __forceinline__ int wrap_index(int v, int K)
{
    v = v >= K ? v - K : v;
    return v >= K ? v - K : v;
}

template <typename R, int P>
__device__ __forceinline__ void grid_point_p(const PmeArgs& a, int atom, int (&ix)[P], int (&iy)[P], int (&iz)[P],
                                             R (&tx)[P], R (&dtx)[P], R (&ty)[P], R (&dty)[P], R (&tz)[P],
                                             R (&dtz)[P])
{
    const double x = wrap_grid(a.pos[3 * (size_t)atom] * a.hxr, a.kx);
    const double y = wrap_grid(a.pos[3 * (size_t)atom + 1] * a.hyr, a.ky);
    const double z = wrap_grid(a.pos[3 * (size_t)atom + 2] * a.hzr, a.kz);
    const int x0 = (int)x, y0 = (int)y, z0 = (int)z;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        ix[p] = wrap_index(x0 + a.offx + p, a.kx);
        iy[p] = wrap_index(y0 + a.offy + p, a.ky);
        iz[p] = wrap_index(z0 + a.offz + p, a.kz);
    }
    bspline_fixed<R, P>((R)(x - x0), tx, dtx);
    bspline_fixed<R, P>((R)(y - y0), ty, dty);
    bspline_fixed<R, P>((R)(z - z0), tz, dtz);
}

template <typename R, int P>
__global__ void __launch_bounds__(128) k_spread_p(PmeArgs a)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n) return;
    const int atom = a.sorted ? a.sorted[s] : s;
    R tx[P], dtx[P], ty[P], dty[P], tz[P], dtz[P];
    int ix[P], iy[P], iz[P];
    grid_point_p<R, P>(a, atom, ix, iy, iz, tx, dtx, ty, dty, tz, dtz);
    // the charge multiplies in FP64 (see k_spread)
    const double qs = a.q[atom] * a.qscale;
#pragma unroll
    for (int i = 0; i < P; i++)
#pragma unroll
        for (int j = 0; j < P; j++) {
            const R ab = tx[i] * ty[j];
            unsigned long long* row = (unsigned long long*)a.qgrid + ((size_t)ix[i] * a.ky + iy[j]) * a.kz;
#pragma unroll
            for (int k = 0; k < P; k++) {
                const long long qv = __double2ll_rn(qs * (double)(ab * tz[k]));
                if (qv) atomicAdd(row + iz[k], (unsigned long long)qv);
            }
        }
}

template <typename R, int P>
__global__ void __launch_bounds__(128) k_gather_p(PmeArgs a)
{
    pdl_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n) return;
    const int atom = a.sorted ? a.sorted[s] : s;
    R tx[P], dtx[P], ty[P], dty[P], tz[P], dtz[P];
    int ix[P], iy[P], iz[P];
    grid_point_p<R, P>(a, atom, ix, iy, iz, tx, dtx, ty, dty, tz, dtz);
    const R* g = (const R*)a.rgrid;
    R fx = 0, fy = 0, fz = 0;
#pragma unroll
    for (int i = 0; i < P; i++)
#pragma unroll
        for (int j = 0; j < P; j++) {
            const R xij = dtx[i] * ty[j], yij = tx[i] * dty[j], zij = tx[i] * ty[j];
            const R* row = g + ((size_t)ix[i] * a.ky + iy[j]) * a.kz;
#pragma unroll
            for (int k = 0; k < P; k++) {
                const R term = row[iz[k]];
                fx -= term * xij * tz[k];
                fy -= term * yij * tz[k];
                fz -= term * zij * dtz[k];
            }
        }
    const double q = a.q[atom];
    const int slot = a.sorted ? s : (a.slot_of ? a.slot_of[atom] : atom);
    fixed_add3(a.facc + 3 * (size_t)slot, (double)fx * a.hxr * q, (double)fy * a.hyr * q,
               (double)fz * a.hzr * q, a.scale, a.status);
}

// The reciprocal term's molecular virial (reciprocalTerm,
// forces/NonbondedPMEwaldSystemForce.h:903-924): every atom's reciprocal force
// (interpolateForce, recomputed from the convolved grid as k_gather does)
// against the minimal difference from the atom's minimal position to its
// molecule's position (Darden et al., J. Chem. Phys. 103, 8577); one record
// (kMRec, the atomic part zero) per block of 128 atoms
template <typename R>
__global__ void __launch_bounds__(128) k_gather_molvir(PmeArgs a)
{
    double acc[kMRec];
#pragma unroll
    for (int k = 0; k < kMRec; ++k) acc[k] = 0.0;
    const int atom = blockIdx.x * blockDim.x + threadIdx.x;
    if (atom < a.n) {
        R tx[kMaxOrder], dtx[kMaxOrder], ty[kMaxOrder], dty[kMaxOrder], tz[kMaxOrder], dtz[kMaxOrder];
        int i0, j0, k0;
        grid_point<R>(a, atom, i0, j0, k0, tx, dtx, ty, dty, tz, dtz);
        const R* g = (const R*)a.rgrid;
        R fx = 0, fy = 0, fz = 0;
        const int P = a.order;
        for (int i = 0; i < P; i++) {
            int i1 = (i + i0) % a.kx;
            for (int j = 0; j < P; j++) {
                int j1 = (j + j0) % a.ky;
                R xij = dtx[i] * ty[j], yij = tx[i] * dty[j], zij = tx[i] * ty[j];
                size_t row = ((size_t)i1 * a.ky + j1) * a.kz;
                for (int k = 0; k < P; k++) {
                    int k1 = (k + k0) % a.kz;
                    R term = g[row + k1];
                    fx -= term * xij * tz[k];
                    fy -= term * yij * tz[k];
                    fz -= term * zij * dtz[k];
                }
            }
        }
        const double q = a.q[atom];
        const double fix = (double)fx * a.hxr * q, fiy = (double)fy * a.hyr * q, fiz = (double)fz * a.hzr * q;
        double rx, ry, rz, mx, my, mz;
        pbc_min_pos(a.pbc, a.pos[3 * (size_t)atom], a.pos[3 * (size_t)atom + 1], a.pos[3 * (size_t)atom + 2],
                    rx, ry, rz);
        const double* c = a.molpos + 3 * (size_t)a.mol[atom];
        pbc_min_diff(a.pbc, rx, ry, rz, c[0], c[1], c[2], mx, my, mz);
        add_outer(acc, fix, fiy, fiz, mx, my, mz);
    }
    block_reduce_store_n<4, kMRec>(acc, a.mrec, a.mrec_stride, blockIdx.x);
}

int pme_molvir_blocks(int n) { return n > 0 ? (n + 127) / 128 : 0; }

// ---- Hessian-vector product of the reciprocal energy ----------------------
// E = 1/2 sum_g Q(g) phi(g), phi = G * Q (the convolution of the FFT stage),
// Q(g) = sum_i q~_i W_i(g), W_i the B-spline weights of atom i.  With
// dQ(g) = sum_j q~_j grad W_j(g) . v_j and dphi = G * dQ:
//   (H v)_i = q~_i sum_g [(grad grad W_i(g)) v_i] phi(g) + q~_i sum_g grad W_i(g) dphi(g).
// The second derivatives of the B-spline along each axis come from the
// order P - 2 spline (M_P'' = M_{P-2}(u) - 2 M_{P-2}(u - 1) + M_{P-2}(u - 2)).
template <typename R>
__device__ __forceinline__ void bspline_second(R w, R (&d2)[kMaxOrder], int order)
{
    // u[2 + j] holds the order P - 2 spline value t[j]; two zero pads below
    // and zeros above make d2[j] = t[j - 2] - 2 t[j - 1] + t[j] a plain stencil
    R u[kMaxOrder + 2];
#pragma unroll
    for (int j = 0; j < kMaxOrder + 2; ++j) u[j] = (R)0;
    u[2] = (R)1;
    // raise the order-1 spline to order P - 2 (the recurrence of bspline4)
    for (int k = 1; k < order - 2; k++) {
        const R div = (R)1 / (R)k;
        u[2 + k] = div * w * u[2 + k - 1];
        for (int j = 1; j < k; j++)
            u[2 + k - j] = div * ((w + (R)j) * u[2 + k - j - 1] + ((R)(k + 1 - j) - w) * u[2 + k - j]);
        u[2] = div * ((R)1 - w) * u[2];
    }
#pragma unroll
    for (int j = 0; j < kMaxOrder; ++j) d2[j] = u[j] - (R)2 * u[j + 1] + u[j + 2];
}

// dQ: every atom's weights differentiated along its displacement v_j
template <typename R>
__global__ void __launch_bounds__(128) k_spread_dir(PmeArgs a)
{
    const int atom = blockIdx.x * blockDim.x + threadIdx.x;
    if (atom >= a.n) return;
    R tx[kMaxOrder], dtx[kMaxOrder], ty[kMaxOrder], dty[kMaxOrder], tz[kMaxOrder], dtz[kMaxOrder];
    int i0, j0, k0;
    grid_point<R>(a, atom, i0, j0, k0, tx, dtx, ty, dty, tz, dtz);
    const double* v = a.dir + 3 * (size_t)atom;
    const double qs = a.q[atom] * a.qscale;
    const R vx = (R)(v[0] * a.hxr), vy = (R)(v[1] * a.hyr), vz = (R)(v[2] * a.hzr);
    const int P = a.order;
    for (int i = 0; i < P; i++) {
        const int i1 = (i + i0) % a.kx;
        for (int j = 0; j < P; j++) {
            const int j1 = (j + j0) % a.ky;
            const R cxy = vx * dtx[i] * ty[j] + vy * tx[i] * dty[j];
            const R txy = tx[i] * ty[j];
            const size_t row = ((size_t)i1 * a.ky + j1) * a.kz;
            for (int k = 0; k < P; k++) {
                const R w = cxy * tz[k] + vz * txy * dtz[k];
                const long long qv = __double2ll_rn(qs * (double)w);
                if (qv) atomicAdd((unsigned long long*)(a.qgrid + row + (k + k0) % a.kz), (unsigned long long)qv);
            }
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(128) k_gather_hvp(PmeArgs a)
{
    const int atom = blockIdx.x * blockDim.x + threadIdx.x;
    if (atom >= a.n) return;
    R tx[kMaxOrder], dtx[kMaxOrder], ty[kMaxOrder], dty[kMaxOrder], tz[kMaxOrder], dtz[kMaxOrder];
    R ddx[kMaxOrder], ddy[kMaxOrder], ddz[kMaxOrder];
    int i0, j0, k0;
    grid_point<R>(a, atom, i0, j0, k0, tx, dtx, ty, dty, tz, dtz);
    {
        const double x = wrap_grid(a.pos[3 * (size_t)atom] * a.hxr, a.kx);
        const double y = wrap_grid(a.pos[3 * (size_t)atom + 1] * a.hyr, a.ky);
        const double z = wrap_grid(a.pos[3 * (size_t)atom + 2] * a.hzr, a.kz);
        bspline_second<R>((R)(x - (int)x), ddx, a.order);
        bspline_second<R>((R)(y - (int)y), ddy, a.order);
        bspline_second<R>((R)(z - (int)z), ddz, a.order);
    }
    const R* phi = (const R*)a.rgrid;
    const R* dphi = (const R*)a.rgrid_d;
    const double* v = a.dir + 3 * (size_t)atom;
    const R hx = (R)a.hxr, hy = (R)a.hyr, hz = (R)a.hzr;
    const R vx = (R)v[0], vy = (R)v[1], vz = (R)v[2];
    // second-derivative sums S_ab = sum phi d2W/dx_a dx_b / (h_a h_b), gradient sums G_a
    R sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0, gx = 0, gy = 0, gz = 0;
    const int P = a.order;
    for (int i = 0; i < P; i++) {
        const int i1 = (i + i0) % a.kx;
        for (int j = 0; j < P; j++) {
            const int j1 = (j + j0) % a.ky;
            const size_t row = ((size_t)i1 * a.ky + j1) * a.kz;
            for (int k = 0; k < P; k++) {
                const size_t g = row + (k + k0) % a.kz;
                const R p = phi[g], d = dphi[g];
                sxx += p * ddx[i] * ty[j] * tz[k];
                syy += p * tx[i] * ddy[j] * tz[k];
                szz += p * tx[i] * ty[j] * ddz[k];
                sxy += p * dtx[i] * dty[j] * tz[k];
                sxz += p * dtx[i] * ty[j] * dtz[k];
                syz += p * tx[i] * dty[j] * dtz[k];
                gx += d * dtx[i] * ty[j] * tz[k];
                gy += d * tx[i] * dty[j] * tz[k];
                gz += d * tx[i] * ty[j] * dtz[k];
            }
        }
    }
    const double q = a.q[atom];
    const double hxx = (double)(hx * hx * sxx), hyy = (double)(hy * hy * syy), hzz = (double)(hz * hz * szz);
    const double hxy = (double)(hx * hy * sxy), hxz = (double)(hx * hz * sxz), hyz = (double)(hy * hz * syz);
    const double ox = q * (hxx * vx + hxy * vy + hxz * vz + (double)(hx * gx));
    const double oy = q * (hxy * vx + hyy * vy + hyz * vz + (double)(hy * gy));
    const double oz = q * (hxz * vx + hyz * vy + hzz * vz + (double)(hz * gz));
    double* o = a.hv + 3 * (size_t)atom;
    o[0] += ox; o[1] += oy; o[2] += oz;
}

static int run_energy64(const PmeArgs& a0, cudaStream_t s, long long* launches, int* erec_used);

template <typename R>
static int run_reciprocal(const PmeArgs& a, cudaStream_t s, long long* launches, int* erec_used, int stage)
{
    typedef typename Cx<R>::T C;
    int nb = (a.n + 127) / 128;
    size_t nreal = (size_t)a.kx * a.ky * a.kz;
    *erec_used = 0;
    if (stage == kStageSpread) {
        cudaMemsetAsync(a.qgrid, 0, sizeof(long long) * nreal, s);
        if (a.n > 0) {
            // with the FP64 energy transform (large grids, see run_energy64)
            // the B-spline weights are FP64 too: FP32 weights (~1e-7 each)
            // move the reciprocal energy by ~1.5e-7, which the FP32
            // transform's own rounding happened to offset on small grids
            // (measured at 64^3: 1.0e-3 and -1.0e-3 of 6,974 kcal/mol); the
            // spread is bound by its 64 integer atomics per atom either way
            if (a.cgrid64) {
                if (a.order == 4) k_spread_p<double, 4><<<nb, 128, 0, s>>>(a);
                else k_spread<double><<<nb, 128, 0, s>>>(a);
            } else {
                if (a.order == 4) k_spread_p<R, 4><<<nb, 128, 0, s>>>(a);
                else k_spread<R><<<nb, 128, 0, s>>>(a);
            }
            *launches += 1;
        }
        return (int)cudaGetLastError();
    }
    if (stage == kStageGather) {
        if (a.n > 0) {
            if (a.order == 4) launch_pdl(k_gather_p<R, 4>, nb, 128, 0, s, a);
            else k_gather<R><<<nb, 128, 0, s>>>(a);
            *launches += 1;
        }
        if (sizeof(R) == 4 && a.cgrid64 && !a.energy64_apart) {
            int e = (int)cudaGetLastError();
            if (e) return e;
            return run_energy64(a, s, launches, erec_used);
        }
        return (int)cudaGetLastError();
    }
    if (stage == kStageEnergy64) {
        if (sizeof(R) == 4 && a.cgrid64) return run_energy64(a, s, launches, erec_used);
        return 0;
    }
    if (stage == kStageMolvir) {
        if (a.n > 0) { k_gather_molvir<R><<<nb, 128, 0, s>>>(a); *launches += 1; }
        return (int)cudaGetLastError();
    }
    if (stage == kStageSpreadDir) {
        cudaMemsetAsync(a.qgrid, 0, sizeof(long long) * nreal, s);
        if (a.n > 0) { k_spread_dir<R><<<nb, 128, 0, s>>>(a); *launches += 1; }
        return (int)cudaGetLastError();
    }
    if (stage == kStageHvpGather) {
        if (a.n > 0) { k_gather_hvp<R><<<nb, 128, 0, s>>>(a); *launches += 1; }
        return (int)cudaGetLastError();
    }
    if (stage == kStagePotential) {   // a.facc holds the double phi[N] output here
        if (a.n > 0) { k_gather_potential<R><<<nb, 128, 0, s>>>(a, (double*)a.facc); *launches += 1; }
        return (int)cudaGetLastError();
    }

    FftPlan px, py, pz;
    make_plan(a.kx, px); make_plan(a.ky, py); make_plan(a.kz, pz);
    if (px.nrad < 0 || py.nrad < 0 || pz.nrad < 0) return (int)cudaErrorInvalidValue;
    const int threads = 256;
    // z lines per block: up to 16 KB of line data and twice the tuned line
    // count of the strided passes (fewer lines: more, smaller blocks, for
    // small grids that are latency-bound)
    const int zmax = a.fft_lines > 0 ? 2 * std::min(a.fft_lines, 16) : 32;
    auto lines_for = [zmax](int n) {
        int l = (16384 / (int)sizeof(C)) / n;
        l = std::min(l, zmax);
        return l < 1 ? 1 : (l > 32 ? 32 : l);
    };
    // z r2c
    {
        PassArgs pa; pa.a = a; pa.plan = pz; pa.lines = lines_for(a.kz); pa.ld = a.kz + 1; pa.sign = -1;
        pa.tw_off = a.twz; pa.erec_off = 0;
        int blocks = (a.kx * a.ky + pa.lines - 1) / pa.lines;
        size_t sm = (2 * (size_t)pa.lines * pa.ld + (size_t)pa.plan.n) * sizeof(C);
        launch_pdl(k_fft_pass<R, kModeZR2C>, blocks, threads, sm, s, pa);
    }
    // lines per CTA for the strided passes: 16 (128 B coalesced rows for
    // float2) unless two line buffers would exceed ~200 KB of shared memory
    const int max_lines = a.fft_lines > 0 ? std::min(a.fft_lines, 16) : 16;
    auto tile_for = [max_lines](int n) {
        int t = (200 * 1024) / (2 * (n + 1) * (int)sizeof(C));
        return t < 1 ? 1 : (t > max_lines ? max_lines : t);
    };
    int tile = tile_for(a.ky);
    // y forward
    {
        PassArgs pa; pa.a = a; pa.plan = py; pa.lines = tile; pa.ld = a.ky + 1; pa.sign = -1;
        pa.tw_off = a.twy; pa.erec_off = 0;
        int blocks = a.kx * ((a.kzh + tile - 1) / tile);
        size_t sm = (2 * (size_t)pa.lines * pa.ld + (size_t)pa.plan.n) * sizeof(C);
        launch_pdl(k_fft_pass<R, kModeY>, blocks, threads, sm, s, pa);
    }
    // x forward + convolution + x inverse
    int xtile = tile_for(a.kx);
    int xblocks = a.ky * ((a.kzh + xtile - 1) / xtile);
    {
        PassArgs pa; pa.a = a; pa.plan = px; pa.lines = xtile; pa.ld = a.kx + 1; pa.sign = -1;
        pa.tw_off = a.twx; pa.erec_off = 0; pa.store_energy = a.cgrid64 ? 0 : 1;
        size_t sm = (2 * (size_t)pa.lines * pa.ld + (size_t)pa.plan.n) * sizeof(C);
        launch_pdl(k_fft_pass<R, kModeXConv>, xblocks, threads, sm, s, pa);
    }
    // y inverse
    {
        PassArgs pa; pa.a = a; pa.plan = py; pa.lines = tile; pa.ld = a.ky + 1; pa.sign = +1;
        pa.tw_off = a.twy; pa.erec_off = 0;
        int blocks = a.kx * ((a.kzh + tile - 1) / tile);
        size_t sm = (2 * (size_t)pa.lines * pa.ld + (size_t)pa.plan.n) * sizeof(C);
        launch_pdl(k_fft_pass<R, kModeY>, blocks, threads, sm, s, pa);
    }
    // z c2r
    {
        PassArgs pa; pa.a = a; pa.plan = pz; pa.lines = lines_for(a.kz); pa.ld = a.kz + 1; pa.sign = +1;
        pa.tw_off = a.twz; pa.erec_off = 0;
        int blocks = (a.kx * a.ky + pa.lines - 1) / pa.lines;
        size_t sm = (2 * (size_t)pa.lines * pa.ld + (size_t)pa.plan.n) * sizeof(C);
        launch_pdl(k_fft_pass<R, kModeZC2R>, blocks, threads, sm, s, pa);
    }
    *launches += 5;
    *erec_used = a.cgrid64 ? 0 : xblocks;
    return (int)cudaGetLastError();
}

// The FP64 forward transform of the charge grid (z r2c, y, x) with the
// energy and virial of Grid::scalarSum, for a mixed-precision force: its
// energy records replace those of the FP32 convolution pass.  Same passes,
// FP64 twiddles, a double2 half spectrum of its own.
static int run_energy64(const PmeArgs& a0, cudaStream_t s, long long* launches, int* erec_used)
{
    typedef double2 C;
    PmeArgs a = a0;
    a.cgrid = a0.cgrid64;
    a.tw = a0.tw64;
    FftPlan px, py, pz;
    make_plan(a.kx, px); make_plan(a.ky, py); make_plan(a.kz, pz);
    if (px.nrad < 0 || py.nrad < 0 || pz.nrad < 0) return (int)cudaErrorInvalidValue;
    const int threads = 256;
    const int zmax = a.fft_lines > 0 ? 2 * std::min(a.fft_lines, 16) : 32;
    int zl = std::min((16384 / (int)sizeof(C)) / a.kz, zmax);
    zl = zl < 1 ? 1 : (zl > 32 ? 32 : zl);
    const int max_lines = a.fft_lines > 0 ? std::min(a.fft_lines, 16) : 16;
    auto tile_for = [max_lines](int n) {
        int t = (200 * 1024) / (2 * (n + 1) * (int)sizeof(C));
        return t < 1 ? 1 : (t > max_lines ? max_lines : t);
    };
    {
        PassArgs pa; pa.a = a; pa.plan = pz; pa.lines = zl; pa.ld = a.kz + 1; pa.sign = -1;
        pa.tw_off = a.twz; pa.erec_off = 0; pa.store_energy = 0;
        int blocks = (a.kx * a.ky + pa.lines - 1) / pa.lines;
        size_t sm = (2 * (size_t)pa.lines * pa.ld + (size_t)pa.plan.n) * sizeof(C);
        launch_pdl(k_fft_pass<double, kModeZR2C>, blocks, threads, sm, s, pa);
    }
    const int tile = tile_for(a.ky);
    {
        PassArgs pa; pa.a = a; pa.plan = py; pa.lines = tile; pa.ld = a.ky + 1; pa.sign = -1;
        pa.tw_off = a.twy; pa.erec_off = 0; pa.store_energy = 0;
        int blocks = a.kx * ((a.kzh + tile - 1) / tile);
        size_t sm = (2 * (size_t)pa.lines * pa.ld + (size_t)pa.plan.n) * sizeof(C);
        launch_pdl(k_fft_pass<double, kModeY>, blocks, threads, sm, s, pa);
    }
    const int xtile = tile_for(a.kx);
    const int xblocks = a.ky * ((a.kzh + xtile - 1) / xtile);
    {
        PassArgs pa; pa.a = a; pa.plan = px; pa.lines = xtile; pa.ld = a.kx + 1; pa.sign = -1;
        pa.tw_off = a.twx; pa.erec_off = 0; pa.store_energy = 1;
        size_t sm = (2 * (size_t)pa.lines * pa.ld + (size_t)pa.plan.n) * sizeof(C);
        launch_pdl(k_fft_pass<double, kModeXEnergy>, xblocks, threads, sm, s, pa);
    }
    *launches += 3;
    *erec_used = xblocks;
    return (int)cudaGetLastError();
}

int launch_pme_reciprocal(const PmeArgs& a, int fp64, cudaStream_t s, long long* launches,
                          double* erec_base, int* erec_used, int stage)
{
    PmeArgs b = a;
    b.erec = erec_base;
    return fp64 ? run_reciprocal<double>(b, s, launches, erec_used, stage)
                : run_reciprocal<float>(b, s, launches, erec_used, stage);
}

// The FFT passes stage two line buffers in dynamic shared memory; allow the
// opt-in maximum (less the kernel's static shared memory, or the attribute is
// refused) once per device, so that launches (also inside graph capture)
// need no attribute calls.
template <typename K>
static void allow_dynamic_smem(K kernel, int optin)
{
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

void pme_init_attributes()
{
    static unsigned long long done = 0;   // one bit per device
    int dev = 0, mx = 48 * 1024;
    cudaGetDevice(&dev);
    if (dev < 64 && (done >> dev) & 1ull) return;
    cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    allow_dynamic_smem(k_fft_pass<float, kModeZR2C>, mx);
    allow_dynamic_smem(k_fft_pass<float, kModeY>, mx);
    allow_dynamic_smem(k_fft_pass<float, kModeXConv>, mx);
    allow_dynamic_smem(k_fft_pass<float, kModeZC2R>, mx);
    allow_dynamic_smem(k_fft_pass<double, kModeZR2C>, mx);
    allow_dynamic_smem(k_fft_pass<double, kModeY>, mx);
    allow_dynamic_smem(k_fft_pass<double, kModeXConv>, mx);
    allow_dynamic_smem(k_fft_pass<double, kModeZC2R>, mx);
    allow_dynamic_smem(k_fft_pass<double, kModeXEnergy>, mx);
    cudaGetLastError();   // a refused attribute surfaces at the launch that needs it
    if (dev < 64) done |= 1ull << dev;
}

// ------------------------------------------------------------------ correction
// correctionTerm (forces/NonbondedPMEwaldSystemForce.h:942-981), FP64, over
// the exclusion table (FULL and MODIFIED pairs, molecules not consulted).
__global__ void k_pme_correction(CorrArgs a)
{
    double acc[kERec];
    for (int k = 0; k < kERec; ++k) acc[k] = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // point self energy and charged-system term (initialize, :604-628),
        // the latter also on the virial diagonal (evaluate, :296-301)
        acc[1] = a.const_energy;
        if (a.virial) acc[2] = acc[6] = acc[10] = a.const_virial;
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n_excl; k += gridDim.x * blockDim.x) {
        int2 pr = a.pairs[k];
        const double* p1 = a.pos + 3 * (size_t)pr.x;
        const double* p2 = a.pos + 3 * (size_t)pr.y;
        double rx, ry, rz;
        double r2 = pbc_min_diff(a.pbc, p1[0], p1[1], p1[2], p2[0], p2[1], p2[2], rx, ry, rz);
        double qq = a.q[pr.x] * a.q[pr.y];
        if (a.cls[k] == PMGPU_EXCL_MODIFIED) qq *= 1 - a.csf;
        double r = sqrt(r2);
        double rr = 1 / r;
        double e = erf(a.alpha * r) * rr;
        acc[1] -= qq * e;
        double f = (qq * (a.two_alpha_pi * exp(-a.alpha2 * r2) - e) * rr * rr);
        double fx = rx * f, fy = ry * f, fz = rz * f;
        const int si = a.slot_of ? a.slot_of[pr.x] : pr.x, sj = a.slot_of ? a.slot_of[pr.y] : pr.y;
        fixed_add3(a.facc + 3 * (size_t)si, -fx, -fy, -fz, a.scale, a.status);
        fixed_add3(a.facc + 3 * (size_t)sj, fx, fy, fz, a.scale, a.status);
        if (a.virial) {
            double xy = fx * ry, xz = fx * rz, yz = fy * rz;
            acc[2] += fx * rx; acc[3] += xy; acc[4] += xz;
            acc[5] += xy; acc[6] += fy * ry; acc[7] += yz;
            acc[8] += xz; acc[9] += yz; acc[10] += fz * rz;
        }
    }
    block_reduce_store<8>(acc, a.erec, a.erec_stride, blockIdx.x);
}

// dE_correction/dq~: each exclusion pair's -kappa q~_i q~_j erf(alpha r)/r
// (kappa = 1, or 1 - csf for MODIFIED) differentiated w.r.t. both charges
__global__ void k_pme_correction_adjoint(CorrArgs a, double* dq)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n_excl; k += gridDim.x * blockDim.x) {
        int2 pr = a.pairs[k];
        const double* p1 = a.pos + 3 * (size_t)pr.x;
        const double* p2 = a.pos + 3 * (size_t)pr.y;
        double rx, ry, rz;
        double r2 = pbc_min_diff(a.pbc, p1[0], p1[1], p1[2], p2[0], p2[1], p2[2], rx, ry, rz);
        double kappa = a.cls[k] == PMGPU_EXCL_MODIFIED ? 1 - a.csf : 1.0;
        double r = sqrt(r2);
        double e = kappa * erf(a.alpha * r) / r;
        atomicAdd(dq + pr.x, -e * a.q[pr.y]);
        atomicAdd(dq + pr.y, -e * a.q[pr.x]);
    }
}

// H v of the correction term: each excluded pair's energy
// U(r) = -kappa q~_a q~_b erf(alpha r) / r (correctionTerm,
// NonbondedPMEwaldSystemForce.h:942-981) gives the block
// K = U''(r) u u^T + U'(r) / r (I - u u^T), u = d / r, d = r_b - r_a, added as
// (H v)_a += K (v_a - v_b), (H v)_b += K (v_b - v_a)
__global__ void k_pme_correction_hvp(CorrArgs a, const double* v, double* hv)
{
    const double sqpi = 1.7724538509055160273;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n_excl; k += gridDim.x * blockDim.x) {
        const int2 pr = a.pairs[k];
        const double* p1 = a.pos + 3 * (size_t)pr.x;
        const double* p2 = a.pos + 3 * (size_t)pr.y;
        double dx, dy, dz;
        const double r2 = pbc_min_diff(a.pbc, p1[0], p1[1], p1[2], p2[0], p2[1], p2[2], dx, dy, dz);
        const double kappa = a.cls[k] == PMGPU_EXCL_MODIFIED ? 1 - a.csf : 1.0;
        const double c = -kappa * a.q[pr.x] * a.q[pr.y];
        const double r = sqrt(r2), ir = 1.0 / r;
        const double er = erf(a.alpha * r), ex = exp(-a.alpha2 * r2);
        const double g = 2.0 * a.alpha / sqpi * ex;          // d erf(alpha r) / dr
        // f = erf(alpha r) / r, f' and f''
        const double f1 = g * ir - er * ir * ir;
        const double f2 = -2.0 * a.alpha2 * r * g * ir - 2.0 * g * ir * ir + 2.0 * er * ir * ir * ir;
        const double U1 = c * f1, U2 = c * f2;
        const double ux = dx * ir, uy = dy * ir, uz = dz * ir;
        const double wx = v[3 * (size_t)pr.x] - v[3 * (size_t)pr.y];
        const double wy = v[3 * (size_t)pr.x + 1] - v[3 * (size_t)pr.y + 1];
        const double wz = v[3 * (size_t)pr.x + 2] - v[3 * (size_t)pr.y + 2];
        const double uw = ux * wx + uy * wy + uz * wz;
        const double t = U1 * ir;
        const double kx = (U2 - t) * uw * ux + t * wx;
        const double ky = (U2 - t) * uw * uy + t * wy;
        const double kz = (U2 - t) * uw * uz + t * wz;
        atomicAdd(hv + 3 * (size_t)pr.x, kx); atomicAdd(hv + 3 * (size_t)pr.x + 1, ky);
        atomicAdd(hv + 3 * (size_t)pr.x + 2, kz);
        atomicAdd(hv + 3 * (size_t)pr.y, -kx); atomicAdd(hv + 3 * (size_t)pr.y + 1, -ky);
        atomicAdd(hv + 3 * (size_t)pr.y + 2, -kz);
    }
}

int launch_pme_correction_hvp(const CorrArgs& a, const double* v, double* hv, cudaStream_t s, long long* launches)
{
    if (a.n_excl <= 0) return 0;
    int blocks = (a.n_excl + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_pme_correction_hvp<<<blocks, 256, 0, s>>>(a, v, hv);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_pme_correction_adjoint(const CorrArgs& a, double* dq, cudaStream_t s, long long* launches)
{
    if (a.n_excl <= 0) return 0;
    int blocks = (a.n_excl + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_pme_correction_adjoint<<<blocks, 256, 0, s>>>(a, dq);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_pme_correction(const CorrArgs& a, cudaStream_t s, long long* launches, int* blocks_used)
{
    int blocks = (a.n_excl + 255) / 256;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_pme_correction<<<blocks, 256, 0, s>>>(a);
    *launches += 1;
    *blocks_used = blocks;
    return (int)cudaGetLastError();
}

// ------------------------------------------------------------------ real space with images
// realTerm (forces/NonbondedPMEwaldSystemForce.h:658-768) for boxes with an
// edge <= 2 rc, where the lattice (buildLatticeVectors,
// topology/PeriodicBoundaryConditions.cpp:80-111) holds images besides
// (0, 0, 0): for every unordered pair i < j and every atom with itself
// (whose (0, 0, 0) image is excluded), the minimal difference plus each
// lattice vector, inside the cutoff (Cutoff switching: no modification).  A
// FULL exclusion removes the first image only and a MODIFIED one scales the
// first image only, as the reference's loop resets the class after it.  One
// warp per atom i, lanes over j >= i; FP64 in the reference's operation
// order, forces in fixed point.
__global__ void __launch_bounds__(256) k_pme_real_lattice(RealLatArgs a)
{
    double acc[kERec];
#pragma unroll
    for (int k = 0; k < kERec; ++k) acc[k] = 0.0;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    const double E1 = 0.254829592, E2 = -0.284496736, E3 = 1.421413741, E4 = -1.453152027, E5 = 1.061405429,
                 PP = 0.3275911;
    for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < a.n; i += warps) {
        const double xi = a.pos[3 * (size_t)i], yi = a.pos[3 * (size_t)i + 1], zi = a.pos[3 * (size_t)i + 2];
        const double qi = a.q[i];
        const int mi = a.mol[i];
        double fix = 0.0, fiy = 0.0, fiz = 0.0;
        for (int j = i + lane; j < a.n; j += 32) {
            double mx, my, mz;
            pbc_min_diff(a.pbc, xi, yi, zi, a.pos[3 * (size_t)j], a.pos[3 * (size_t)j + 1], a.pos[3 * (size_t)j + 2],
                         mx, my, mz);
            int excl = a.mol[j] == mi ? excl_lookup(a.xfull, a.xmod, a.xrow, a.xent, i, j) : PMGPU_EXCL_NONE;
            if (i == j) excl = PMGPU_EXCL_FULL;
            const double qj = a.q[j];
            double fjx = 0.0, fjy = 0.0, fjz = 0.0;
            for (int k = 0; k < a.n_lattice; ++k) {
                if (excl == PMGPU_EXCL_FULL) { excl = PMGPU_EXCL_NONE; continue; }
                const double4 L = a.lattice[k];
                const double rx = dadd(mx, L.x), ry = dadd(my, L.y), rz = dadd(mz, L.z);
                const double r2 = dnorm2(rx, ry, rz);
                if (r2 > a.rc2) continue;
                const double r = sqrt(r2);
                double qq = qi * qj;
                if (excl == PMGPU_EXCL_MODIFIED) qq *= a.csf;
                const double rr = 1.0 / r;
                const double ar = a.alpha * r;
                const double e = qq * exp(-ar * ar);
                const double t = 1.0 / (1.0 + PP * ar);
                const double energy = t * (E1 + t * (E2 + t * (E3 + t * (E4 + t * E5)))) * e * rr;
                const double force = (energy + a.two_alpha_pi * e) * rr * rr;
                acc[1] += energy;
                const double fx = rx * force, fy = ry * force, fz = rz * force;
                fix -= fx; fiy -= fy; fiz -= fz;
                fjx += fx; fjy += fy; fjz += fz;
                if (a.virial) {
                    const double xy = fx * ry, xz = fx * rz, yz = fy * rz;
                    acc[2] += fx * rx; acc[3] += xy; acc[4] += xz;
                    acc[5] += xy; acc[6] += fy * ry; acc[7] += yz;
                    acc[8] += xz; acc[9] += yz; acc[10] += fz * rz;
                }
                excl = PMGPU_EXCL_NONE;
            }
            if (fjx != 0.0 || fjy != 0.0 || fjz != 0.0)
                fixed_add3(a.facc + 3 * (size_t)j, fjx, fjy, fjz, a.scale, a.status);
        }
        for (int o = 16; o > 0; o >>= 1) {
            fix += __shfl_xor_sync(FULL, fix, o);
            fiy += __shfl_xor_sync(FULL, fiy, o);
            fiz += __shfl_xor_sync(FULL, fiz, o);
        }
        if (lane == 0) fixed_add3(a.facc + 3 * (size_t)i, fix, fiy, fiz, a.scale, a.status);
    }
    block_reduce_store<8>(acc, a.erec, a.erec_stride, blockIdx.x);
}

// realTerm's molecular virial (NonbondedPMEwaldSystemForce.h:750-757): every
// image of a pair of atoms of different molecules inside the cutoff adds its
// force against the minimal difference of the molecules' positions, and
// against the image vector to the inter-molecular atomic virial.  The loop
// and arithmetic of k_pme_real_lattice (pairs of one molecule skipped: they
// add to neither tensor); no forces, no energies.
__global__ void __launch_bounds__(256) k_pme_real_lattice_molvir(RealLatArgs a)
{
    double acc[kMRec];
#pragma unroll
    for (int k = 0; k < kMRec; ++k) acc[k] = 0.0;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    const double E1 = 0.254829592, E2 = -0.284496736, E3 = 1.421413741, E4 = -1.453152027, E5 = 1.061405429,
                 PP = 0.3275911;
    for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < a.n; i += warps) {
        const double xi = a.pos[3 * (size_t)i], yi = a.pos[3 * (size_t)i + 1], zi = a.pos[3 * (size_t)i + 2];
        const double qi = a.q[i];
        const int mi = a.mol[i];
        const double* ci = a.molpos + 3 * (size_t)mi;
        for (int j = i + 1 + lane; j < a.n; j += 32) {
            const int mj = a.mol[j];
            if (mj == mi) continue;
            double mx, my, mz, cx, cy, cz;
            pbc_min_diff(a.pbc, xi, yi, zi, a.pos[3 * (size_t)j], a.pos[3 * (size_t)j + 1], a.pos[3 * (size_t)j + 2],
                         mx, my, mz);
            const double* cj = a.molpos + 3 * (size_t)mj;
            pbc_min_diff(a.pbc, ci[0], ci[1], ci[2], cj[0], cj[1], cj[2], cx, cy, cz);
            const double qq = qi * a.q[j];
            for (int k = 0; k < a.n_lattice; ++k) {
                const double4 L = a.lattice[k];
                const double rx = dadd(mx, L.x), ry = dadd(my, L.y), rz = dadd(mz, L.z);
                const double r2 = dnorm2(rx, ry, rz);
                if (r2 > a.rc2) continue;
                const double r = sqrt(r2);
                const double rr = 1.0 / r;
                const double ar = a.alpha * r;
                const double e = qq * exp(-ar * ar);
                const double t = 1.0 / (1.0 + PP * ar);
                const double energy = t * (E1 + t * (E2 + t * (E3 + t * (E4 + t * E5)))) * e * rr;
                const double force = (energy + a.two_alpha_pi * e) * rr * rr;
                const double fx = rx * force, fy = ry * force, fz = rz * force;
                add_outer(acc, fx, fy, fz, cx, cy, cz);
                add_outer(acc + 9, fx, fy, fz, rx, ry, rz);
            }
        }
    }
    block_reduce_store_n<8, kMRec>(acc, a.mrec, a.mrec_stride, blockIdx.x);
}

int launch_pme_real_lattice_molvir(const RealLatArgs& a, cudaStream_t s, long long* launches, int* blocks_used)
{
    int blocks = (a.n + 7) / 8;
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_pme_real_lattice_molvir<<<blocks, 256, 0, s>>>(a);
    *launches += 1;
    *blocks_used = blocks;
    return (int)cudaGetLastError();
}

int launch_pme_real_lattice(const RealLatArgs& a, cudaStream_t s, long long* launches, int* blocks_used)
{
    int blocks = (a.n + 7) / 8;                  // one warp per atom, 8 warps per block
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_pme_real_lattice<<<blocks, 256, 0, s>>>(a);
    *launches += 1;
    *blocks_used = blocks;
    return (int)cudaGetLastError();
}

// ------------------------------------------------------------------ finalize
__global__ void __launch_bounds__(256) k_finalize(FinArgs a)
{
    pdl_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double v[kERec];
#pragma unroll
    for (int k = 0; k < kERec; ++k) v[k] = 0.0;
    if (s < a.n) {
        const int i = a.sorted ? a.sorted[s] : s;   // no cell-sorted order: atom order
        // the atom's total force, added to the output once (so that an
        // output that already holds forces gets one rounding per component)
        double fp[3] = {0.0, 0.0, 0.0}, ft[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (a.f32) fp[c] = (double)(long long)a.f32[3 * (size_t)s + c] * (1.0 / kScaleMixed);
            double f = fp[c];
            if (a.f32p) f += (double)(long long)a.f32p[3 * (size_t)s + c] * (1.0 / kScaleMixed);
            if (a.f40) f += (double)(long long)a.f40[3 * (size_t)s + c] * (1.0 / kScaleFp64);
            if (a.a32) f += (double)(long long)a.a32[3 * (size_t)i + c] * (1.0 / kScaleMixed);
            if (a.a40) f += (double)(long long)a.a40[3 * (size_t)i + c] * (1.0 / kScaleFp64);
            ft[c] = f;
        }
        if (a.pair_virial & 1) {
            // the cell-relative position the FP32 pair vectors were formed from
            const float4 h = a.spos[s], l = a.slo[s];
            const double p[3] = {(double)h.x + (double)l.x, (double)h.y + (double)l.y, (double)h.z + (double)l.z};
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) v[2 + 3 * r + c] = p[r] * fp[c];
        }
        if (a.c32) {
            // column-cluster pair forces, per slot; their virial from the
            // fixed-point position the pair vectors were formed from
            // slot_of is whole only when the column binning completed (a
            // refused system is redone on the cell layout); never read past c32
            const int sl = min(max(a.c_slot_of[i], 0), a.c_slots - 1);
            double fc[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                fc[c] = (double)(long long)a.c32[3 * (size_t)sl + c] * (1.0 / kScaleMixed);
                ft[c] += fc[c];
            }
            if (a.pair_virial & 2) {
                // position relative to its i-cluster's origin (the first atom)
                const int4 q = a.cq[sl], o = a.corg[sl >> 3];
                const double p[3] = {(double)(int)((unsigned)q.x - (unsigned)o.x) * a.cscale[0],
                                     (double)(int)((unsigned)q.y - (unsigned)o.y) * a.cscale[1],
                                     (double)(int)((unsigned)q.z - (unsigned)o.z) * a.cscale[2]};
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) v[2 + 3 * r + c] += p[r] * fc[c];
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) a.fout[3 * (size_t)i + c] += ft[c];
    }
    if (a.pair_virial) block_reduce_store<8>(v, a.erec, a.erec_stride, blockIdx.x);
}

int launch_finalize(const FinArgs& a, cudaStream_t s, long long* launches, int* records)
{
    *records = 0;
    if (a.n <= 0) return 0;
    const int blocks = (a.n + 255) / 256;
    launch_pdl(k_finalize, blocks, 256, 0, s, a);
    *launches += 1;
    if (a.pair_virial) *records = blocks;
    return (int)cudaGetLastError();
}

// deterministic sum of energy records: block k sums component k (contiguous)
__global__ void k_energy_reduce(const double* erec, int stride, int nrec, const unsigned long long* efix,
                                double* out)
{
    pdl_wait();
    int k = blockIdx.x;
    const double* c = erec + (size_t)k * stride;
    double s = 0.0;
    for (int r = threadIdx.x; r < nrec; r += blockDim.x) s += c[r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double part[8];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) part[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += part[q];
        if (efix) t += (double)(long long)efix[k] * (1.0 / 4294967296.0);
        out[k] += t;
    }
}

// block k < 9: molecular virial component k; block 9 + k: the
// inter-molecular atomic virial component k (only without the atomic virial)
__global__ void k_molvir_finish(MolvirFinish f)
{
    const int k = blockIdx.x;
    const bool mol = k < 9;
    if (!mol && f.virial) return;
    const double* c = f.mrec + (size_t)k * f.mstride;
    double s = 0.0;
    for (int r = threadIdx.x; r < f.nmrec; r += blockDim.x) s += c[r];
    if (mol)
        for (int g = 0; g < f.nranges; ++g) {
            const double* e = f.erec + (size_t)(2 + k) * f.estride + f.range_first[g];
            for (int r = threadIdx.x; r < f.range_count[g]; r += blockDim.x) s += e[r];
        }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double part[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) part[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += part[q];
        f.out[mol ? 11 + k : 2 + (k - 9)] += t;
    }
}

int launch_molvir_finish(const MolvirFinish& f, cudaStream_t s, long long* launches)
{
    k_molvir_finish<<<kMRec, 256, 0, s>>>(f);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_energy_reduce(const double* erec, int stride, int nrec, const unsigned long long* efix,
                         double* out, cudaStream_t s, long long* launches)
{
    launch_pdl(k_energy_reduce, kERec, 256, 0, s, erec, stride, nrec, efix, out);
    *launches += 1;
    return (int)cudaGetLastError();
}

}  // namespace pm
