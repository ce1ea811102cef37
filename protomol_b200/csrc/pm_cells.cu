// pm_cells.cu -- K1: cell binning by counting sort, three launches.
//
// The cell of atom i is buildCellLists' (topology/buildCellLists.cpp:11-38),
// bit for bit: floor((origin - min + minimalPosition(x_i)) *
// (1 / realCellSize)) in FP64 in the reference's operation order
// (CubicCellManager::findCell, topology/CubicCellManager.h:61-64).  Instead
// of the reference's linked lists the atoms are counting-sorted into CSR cell
// ranges.  Inside a cell they are ordered by the Morton key of their position
// on an 8x8x8 sub-grid of the cell, ties by original index, so that every run
// of 8 consecutive slots is a compact cluster.  The within-cutoff pair set
// does not depend on this order (the pair kernels visit every pair of the
// reference's cell pairs once).
//
//   k_bin_count    cell, key and count of every atom; the last block to
//                  finish (a done counter, no waiting) scans the counts into
//                  the cell starts and the cluster starts
//   k_bin_scatter  atom -> a slot of its cell's range; the counts are
//                  decremented back to zero, so no memset precedes the next
//                  binning (the counts are zeroed once when the grid is set)
//   k_bin_cells    one warp per cell: the order inside the cell, the sorted
//                  arrays (compensated FP32 coordinates and charge, metadata,
//                  FP64 position and charge) and the cell's cluster boxes
//
// Roofline: latency-bound at 10^4 atoms, HBM-bound at 10^6; per atom it reads
// 24 B position + 8 B charge + 8 B type/molecule and writes 16 + 16 + 16 + 32
// B of sorted data and 8 B of index arrays.
#include "pm_kernels.h"

namespace pm {

namespace {

constexpr int kBinThreads = 256;
constexpr int kCellStage = 128;      // atoms of a cell ordered in shared memory (larger: from global)

__device__ __forceinline__ void bin_cell_of(const Pbc& b, const CellGrid& g, double x, double y, double z,
                                            int& cx, int& cy, int& cz, double& vx, double& vy, double& vz)
{
    double mx, my, mz;
    pbc_min_pos(b, x, y, z, mx, my, mz);
    // delta + minimalPosition(x)  (Vector3D operator+)
    vx = dadd(b.dx, mx);
    vy = dadd(b.dy, my);
    vz = dadd(b.dz, mz);
    cx = (int)floor(dmul(vx, g.rcsx));
    cy = (int)floor(dmul(vy, g.rcsy));
    cz = (int)floor(dmul(vz, g.rcsz));
}

// Single-block exclusive scans of the per-cell atom counts (-> start) and
// cluster counts ceil(count / 8) (-> cstart), by the calling block.
__device__ void scan_counts(const int* counts, int* start, int* cstart, int ncell)
{
    __shared__ int part[kBinThreads], cpart[kBinThreads];
    const int t = threadIdx.x;
    const int per = (ncell + blockDim.x - 1) / blockDim.x;
    const int b = min(ncell, t * per), e = min(ncell, b + per);
    int s = 0, cs = 0;
    for (int k = b; k < e; ++k) {
        const int c = __ldcg(counts + k);          // device-scope atomics: read at L2
        s += c;
        cs += (c + kCluster - 1) / kCluster;
    }
    part[t] = s;
    cpart[t] = cs;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {     // Hillis-Steele inclusive scan
        const int v = t >= o ? part[t - o] : 0;
        const int cv = t >= o ? cpart[t - o] : 0;
        __syncthreads();
        part[t] += v;
        cpart[t] += cv;
        __syncthreads();
    }
    int run = part[t] - s, crun = cpart[t] - cs;
    for (int k = b; k < e; ++k) {
        const int c = __ldcg(counts + k);
        start[k] = run;
        cstart[k] = crun;
        run += c;
        crun += (c + kCluster - 1) / kCluster;
    }
    if (t == blockDim.x - 1) { start[ncell] = part[t]; cstart[ncell] = cpart[t]; }
}

__global__ void __launch_bounds__(kBinThreads) k_bin_count(BinArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const CellGrid& g = a.grid;
    if (i < a.n) {
        int cx, cy, cz;
        double vx, vy, vz;
        bin_cell_of(a.pbc, g, a.pos[3 * i], a.pos[3 * i + 1], a.pos[3 * i + 2], cx, cy, cz, vx, vy, vz);
        a.cell3[3 * i] = cx;
        a.cell3[3 * i + 1] = cy;
        a.cell3[3 * i + 2] = cz;
        if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) {
            // The reference stores such an atom outside its cell array (an
            // atom exactly on the +L/2 face); here it is filed under its
            // periodic image and the event is reported.
            atomicOr(a.status, kStatusOutOfGrid);
            cx = ((cx % g.nx) + g.nx) % g.nx;
            cy = ((cy % g.ny) + g.ny) % g.ny;
            cz = ((cz % g.nz) + g.nz) % g.nz;
        }
        const int c = (cx * g.ny + cy) * g.nz + cz;
        a.cell_lin[i] = c;
        // Morton key of the position inside the cell on an 8x8x8 sub-grid
        const int qx = min(7, max(0, (int)(dmul(vx - (double)cx * g.csx, g.rcsx) * 8.0)));
        const int qy = min(7, max(0, (int)(dmul(vy - (double)cy * g.csy, g.rcsy) * 8.0)));
        const int qz = min(7, max(0, (int)(dmul(vz - (double)cz * g.csz, g.rcsz) * 8.0)));
        int key = 0;
#pragma unroll
        for (int bit = 2; bit >= 0; --bit)
            key = (key << 3) | (((qx >> bit) & 1) << 2) | (((qy >> bit) & 1) << 1) | ((qz >> bit) & 1);
        a.skey[i] = key;
        atomicAdd(a.counts + c, 1);
    }
    // the last block to finish scans the counts (no block waits for another)
    __shared__ bool last;
    __threadfence();                                        // this thread's counts before the done count
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(a.done, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    scan_counts(a.counts, a.start, a.cstart, g.ncell);
}

__global__ void __launch_bounds__(kBinThreads) k_bin_scatter(BinArgs a)
{
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int c = a.cell_lin[i];
    // fills the cell's range from its end; the count returns to zero
    a.tmp[a.start[c] + atomicSub(a.counts + c, 1) - 1] = i;
}

// the sorted-slot data of atom i at slot dst; returns the FP32 (hi)
// cell-relative position
__device__ __forceinline__ float3 write_atom(const BinArgs& a, int i, int dst)
{
    a.sorted[dst] = i;
    a.slot_of[i] = dst;
    const CellGrid& g = a.grid;
    int cx, cy, cz;
    double vx, vy, vz;
    const double x = a.pos[3 * i], y = a.pos[3 * i + 1], z = a.pos[3 * i + 2];
    bin_cell_of(a.pbc, g, x, y, z, cx, cy, cz, vx, vy, vz);
    // coordinates relative to the corner of the unwrapped cell; an atom filed
    // under its periodic image (cx = nx) lands just below that image's corner
    const double rx = vx - (double)cx * g.csx;
    const double ry = vy - (double)cy * g.csy;
    const double rz = vz - (double)cz * g.csz;
    const double qi = a.q[i];
    // compensated FP32: value = hi + lo to ~2^-48 relative, so that the
    // rounding of an atom's coordinates or charge does not bias all of its
    // pair terms the same way
    const float hx = (float)rx, hy = (float)ry, hz = (float)rz, hq = (float)qi;
    a.spos[dst] = make_float4(hx, hy, hz, hq);
    a.slo[dst] = make_float4((float)(rx - (double)hx), (float)(ry - (double)hy), (float)(rz - (double)hz),
                             (float)(qi - (double)hq));
    a.smeta[dst] = make_int4(i, a.type[i], a.mol[i], 0);
    if (a.spos64) a.spos64[dst] = make_double4(x, y, z, qi);
    return make_float3(hx, hy, hz);
}

__device__ __forceinline__ bool key_before(int kj, int ij, int ki, int ii)
{
    return kj < ki || (kj == ki && ij < ii);
}

__global__ void __launch_bounds__(128) k_bin_cells(BinArgs a)
{
    pdl_wait();
    __shared__ int s_idx[4][kCellStage], s_key[4][kCellStage];
    __shared__ float s_px[4][kCellStage], s_py[4][kCellStage], s_pz[4][kCellStage];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int c = blockIdx.x * 4 + w;                       // one warp per cell
    if (c >= a.grid.ncell) return;                          // warp-uniform
    const int b = a.start[c], m = a.start[c + 1] - b;
    const bool staged = m <= kCellStage;
    if (staged) {
        for (int k = lane; k < m; k += 32) {
            const int i = a.tmp[b + k];
            s_idx[w][k] = i;
            s_key[w][k] = a.skey[i];
        }
        __syncwarp();
    }
    // rank = the atoms of the cell before this one in (key, index) order
    for (int k = lane; k < m; k += 32) {
        const int i = staged ? s_idx[w][k] : a.tmp[b + k];
        const int ki = staged ? s_key[w][k] : a.skey[i];
        int rank = 0;
        if (staged) {
            for (int j = 0; j < m; ++j) rank += key_before(s_key[w][j], s_idx[w][j], ki, i);
        } else {
            for (int j = 0; j < m; ++j) {
                const int o = a.tmp[b + j];
                rank += key_before(a.skey[o], o, ki, i);
            }
        }
        const float3 h = write_atom(a, i, b + rank);
        if (staged) { s_px[w][rank] = h.x; s_py[w][rank] = h.y; s_pz[w][rank] = h.z; }
    }
    __syncwarp();                                           // this warp's writes are visible to it
    // the cell's clusters: runs of 8 slots
    const int cl0 = a.cstart[c], ncl = (m + kCluster - 1) / kCluster;
    for (int q = lane; q < ncl; q += 32) {
        const int cl = cl0 + q;
        if (cl >= a.ncl_cap) break;
        float4 lo = make_float4(3e38f, 3e38f, 3e38f, 0.f), hi = make_float4(-3e38f, -3e38f, -3e38f, 0.f);
        const int r1 = min(m, (q + 1) * kCluster);
        for (int r = q * kCluster; r < r1; ++r) {
            float x, y, z;
            if (staged) {
                x = s_px[w][r]; y = s_py[w][r]; z = s_pz[w][r];
            } else {
                const float4 p = a.spos[b + r];
                x = p.x; y = p.y; z = p.z;
            }
            lo.x = fminf(lo.x, x); lo.y = fminf(lo.y, y); lo.z = fminf(lo.z, z);
            hi.x = fmaxf(hi.x, x); hi.y = fmaxf(hi.y, y); hi.z = fmaxf(hi.z, z);
        }
        a.cbox[2 * cl] = lo;
        a.cbox[2 * cl + 1] = hi;
        a.ccell[cl] = c;
    }
}

// ---------------------------------------------------------------- K1c
// Column clusters of the mixed pair path.  Every atom's position becomes an
// unsigned 32-bit fixed-point coordinate of the periodic box,
// round(frac((x - min) / L) 2^32) per axis, so that the wrapped int32
// difference of two atoms is their minimal-image displacement in units of
// L / 2^32 with no rounding at all; the atoms are counting-sorted into the
// columns of an x-y grid and ordered by z inside a column (ties by index).
// Slot 8 c + k holds atom k of i-cluster c; a column's last cluster is
// padded (original index -1).  The reference cell of every atom is computed
// here too (bit-exact, for pmgpu_get_cells).

__device__ __forceinline__ unsigned fix32(double u)
{
    const double f = u - floor(u);                        // [0, 1)
    return (unsigned)(__double2ull_rn(f * 4294967296.0) & 0xffffffffull);
}

__global__ void __launch_bounds__(kBinThreads) k_col_count(ColBinArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const ColGrid& g = a.g;
    if (i < a.n) {
        const double x = a.pos[3 * i], y = a.pos[3 * i + 1], z = a.pos[3 * i + 2];
        int cx, cy, cz;
        double vx, vy, vz;
        bin_cell_of(a.pbc, a.grid, x, y, z, cx, cy, cz, vx, vy, vz);
        a.cell3[3 * i] = cx;
        a.cell3[3 * i + 1] = cy;
        a.cell3[3 * i + 2] = cz;
        if (cx < 0 || cy < 0 || cz < 0 || cx >= a.grid.nx || cy >= a.grid.ny || cz >= a.grid.nz)
            atomicOr(a.status, kStatusOutOfGrid);
        const unsigned qx = fix32((x - g.mnx) / g.lx);
        const unsigned qy = fix32((y - g.mny) / g.ly);
        const unsigned qz = fix32((z - g.mnz) / g.lz);
        a.qfix[3 * i] = qx;
        a.qfix[3 * i + 1] = qy;
        a.qfix[3 * i + 2] = qz;
        const int kx = (int)(((unsigned long long)qx * (unsigned)g.ncx) >> 32);
        const int ky = (int)(((unsigned long long)qy * (unsigned)g.ncy) >> 32);
        const int c = kx * g.ncy + ky;
        a.col[i] = c;
        atomicAdd(a.counts + c, 1);
    }
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(a.done, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    scan_counts(a.counts, a.colstart, a.ccstart, g.ncol);
}

__global__ void __launch_bounds__(kBinThreads) k_col_scatter(ColBinArgs a)
{
    pdl_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int c = a.col[i];
    a.tmp[a.colstart[c] + atomicSub(a.counts + c, 1) - 1] = i;
}

constexpr int kColStage = 2048;      // atoms of a column ordered in shared memory
constexpr int kColThreads = 128;

// one block per column: z order (a bitonic sort of the (z, index) keys in
// shared memory), slot data, padding, cluster boxes and the clusters' virial
// origins.  The sorted atoms' fixed-point coordinates and the j-cluster boxes
// stay in shared memory for the box passes (no global round trips there).
__global__ void __launch_bounds__(kColThreads) k_col_sort(ColBinArgs a)
{
    pdl_wait();
    // [0, 8K): order; [8K, 32K): sort keys, then the atoms' coordinates;
    // [32K, 48K): the j-cluster boxes
    __shared__ __align__(16) unsigned char s_raw[4 * kColStage + 12 * kColStage + 16 * kColStage / 2];
    int* s_ord = reinterpret_cast<int*>(s_raw);
    unsigned long long* s_key = reinterpret_cast<unsigned long long*>(s_raw + 4 * kColStage);
    unsigned* s_qf = reinterpret_cast<unsigned*>(s_raw + 4 * kColStage);
    float4* s_jb = reinterpret_cast<float4*>(s_raw + 16 * kColStage);
    const int t = threadIdx.x;
    const ColGrid& g = a.g;
    const int c = blockIdx.x;
    const int b = a.colstart[c], m = a.colstart[c + 1] - b;
    const int cl0 = a.ccstart[c], ncl = (m + 7) / 8;
    if (m > kColStage || cl0 + ncl > a.ncl_cap) {            // block-uniform: the cell layout takes this system
        if (t == 0) atomicOr(a.status, kStatusColumns);
        return;
    }
    int n2 = 32;                                            // keys padded to a power of two
    while (n2 < m) n2 <<= 1;
    for (int k = t; k < n2; k += kColThreads) {
        unsigned long long key = ~0ull;
        if (k < m) {
            const int i = a.tmp[b + k];
            key = ((unsigned long long)a.qfix[3 * i + 2] << 32) | (unsigned)i;
        }
        s_key[k] = key;
    }
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = t; i < n2; i += kColThreads) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long u = s_key[i], v = s_key[ixj];
                    if (((i & k) == 0) ? (u > v) : (u < v)) { s_key[i] = v; s_key[ixj] = u; }
                }
            }
            __syncthreads();
        }
    for (int k = t; k < m; k += kColThreads) s_ord[k] = (int)(s_key[k] & 0xffffffffull);
    __syncthreads();                                        // the keys' space becomes the coordinates'
    const size_t slot0 = 8 * (size_t)cl0;
    for (int r = t; r < 8 * ncl; r += kColThreads) {
        const bool valid = r < m;
        const int i = s_ord[valid ? r : (r & ~7)];          // padding: the cluster's first atom's place
        const double qi = a.q[i];
        const float qh = valid ? (float)qi : 0.f;
        const float ql = valid ? (float)(qi - (double)qh) : 0.f;
        const unsigned fx = a.qfix[3 * i], fy = a.qfix[3 * i + 1], fz = a.qfix[3 * i + 2];
        const int4 qv = make_int4((int)fx, (int)fy, (int)fz, __float_as_int(qh));
        a.cq[slot0 + r] = qv;
        a.cm[slot0 + r] = valid ? make_int4(i, a.type[i], a.mol[i], __float_as_int(ql)) : make_int4(-1, 0, -2, 0);
        if (valid) {
            a.slot_of[i] = (int)(slot0 + r);
            s_qf[3 * r] = fx; s_qf[3 * r + 1] = fy; s_qf[3 * r + 2] = fz;
        }
        if ((r & 7) == 0) a.corg[cl0 + (r >> 3)] = make_int4(qv.x, qv.y, qv.z, 0);
    }
    __syncthreads();
    // boxes of the j-clusters (4 slots each, the halves of the i-clusters)
    // and of the i-clusters; an empty half gets a box beyond every window
    const double kx = g.lx * (1.0 / 4294967296.0), ky = g.ly * (1.0 / 4294967296.0), kz = g.lz * (1.0 / 4294967296.0);
    for (int q = t; q < 2 * ncl; q += kColThreads) {
        const int r0 = 4 * q, r1 = min(m, r0 + 4);
        // empty: lo.w = 1, both corners at +3e38 (the z order of the column's
        // boxes stays monotone, and no window reaches it)
        float4 lo = make_float4(3e38f, 3e38f, 3e38f, 1.f), hi = make_float4(3e38f, 3e38f, 3e38f, 0.f);
        if (r0 < r1) { lo.w = 0.f; hi = make_float4(-3e38f, -3e38f, -3e38f, 0.f); }
        for (int r = r0; r < r1; ++r) {
            const float x = (float)(s_qf[3 * r] * kx), y = (float)(s_qf[3 * r + 1] * ky),
                        z = (float)(s_qf[3 * r + 2] * kz);
            lo.x = fminf(lo.x, x); lo.y = fminf(lo.y, y); lo.z = fminf(lo.z, z);
            hi.x = fmaxf(hi.x, x); hi.y = fmaxf(hi.y, y); hi.z = fmaxf(hi.z, z);
        }
        const size_t jc = 2 * (size_t)cl0 + q;
        a.jbox[2 * jc] = lo;
        a.jbox[2 * jc + 1] = hi;
        s_jb[2 * q] = lo;
        s_jb[2 * q + 1] = hi;
    }
    __syncthreads();
    for (int q = t; q < ncl; q += kColThreads) {
        const float4 l0 = s_jb[4 * q], h0 = s_jb[4 * q + 1];
        const float4 l1 = s_jb[4 * q + 2], h1 = s_jb[4 * q + 3];
        const bool e1 = l1.w != 0.f;                        // empty second half
        a.ibox[2 * (cl0 + q)] = e1 ? l0 : make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.f);
        a.ibox[2 * (cl0 + q) + 1] = e1 ? h0 : make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.f);
        a.ccol[cl0 + q] = c;
    }
    // the column's z index for the list kernel's window searches: per bin
    // edge z_b = b L_z / kZBins the first j-cluster whose box ends at or
    // above z_b, and the first whose box starts above it (both corners are
    // monotone along the column; empty halves sit at +3e38, at the end)
    const float binw = g.lzf / kZBins;
    int* zi = a.zidx + (size_t)c * kZIndex;
    for (int b = t; b <= kZBins; b += kColThreads) {
        const float zb = b * binw;
        int lo = 0, hi = 2 * ncl;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s_jb[2 * mid + 1].z < zb) lo = mid + 1; else hi = mid;
        }
        int lo2 = 0, hi2 = 2 * ncl;
        while (lo2 < hi2) {
            const int mid = (lo2 + hi2) >> 1;
            if (s_jb[2 * mid].z > zb) hi2 = mid; else lo2 = mid + 1;
        }
        zi[b] = 2 * cl0 + lo;
        zi[kZBins + 1 + b] = 2 * cl0 + lo2;
    }
}

// K0: range blockIdx.y set to zero, grid-stride
__global__ void __launch_bounds__(kBinThreads) k_zero(ZeroRanges z)
{
    unsigned* p = z.p[blockIdx.y];
    const long long n = z.words[blockIdx.y];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = 0u;
}

__global__ void __launch_bounds__(kBinThreads) k_col_refresh(ColBinArgs a, double half_skin2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const ColGrid& g = a.g;
    const double x = a.pos[3 * i], y = a.pos[3 * i + 1], z = a.pos[3 * i + 2];
    int cx, cy, cz;
    double vx, vy, vz;
    bin_cell_of(a.pbc, a.grid, x, y, z, cx, cy, cz, vx, vy, vz);
    a.cell3[3 * i] = cx;
    a.cell3[3 * i + 1] = cy;
    a.cell3[3 * i + 2] = cz;
    const unsigned qx = fix32((x - g.mnx) / g.lx), qy = fix32((y - g.mny) / g.ly), qz = fix32((z - g.mnz) / g.lz);
    // the displacement since the build, from the build-time fixed point
    const double ux = (double)(int)(qx - a.qfix[3 * i]) * (g.lx * (1.0 / 4294967296.0));
    const double uy = (double)(int)(qy - a.qfix[3 * i + 1]) * (g.ly * (1.0 / 4294967296.0));
    const double uz = (double)(int)(qz - a.qfix[3 * i + 2]) * (g.lz * (1.0 / 4294967296.0));
    if (ux * ux + uy * uy + uz * uz > half_skin2) atomicOr(a.status, kStatusListStale);
    const int sl = a.slot_of[i];
    const int4 old = a.cq[sl];
    a.cq[sl] = make_int4((int)qx, (int)qy, (int)qz, old.w);
}

}  // namespace

int launch_zero(const ZeroRanges& z, cudaStream_t s, long long* launches)
{
    if (z.count <= 0) return 0;
    long long most = 0;
    for (int r = 0; r < z.count; ++r) most = std::max(most, z.words[r]);
    const int blocks = (int)std::max(1LL, std::min<long long>((most + 4 * kBinThreads - 1) / (4 * kBinThreads), 4 * 148));
    k_zero<<<dim3(blocks, z.count), kBinThreads, 0, s>>>(z);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_col_refresh(const ColBinArgs& a, double half_skin, cudaStream_t s, long long* launches)
{
    if (a.n <= 0) return 0;
    const int nb = (a.n + kBinThreads - 1) / kBinThreads;
    k_col_refresh<<<nb, kBinThreads, 0, s>>>(a, half_skin * half_skin);
    *launches += 1;
    return (int)cudaGetLastError();
}

int launch_col_bin(const ColBinArgs& a, cudaStream_t s, long long* launches)
{
    // half-size blocks: the atoms' FP64 conversions are latency-bound, and
    // twice the blocks spread them over more SMs
    const int tb = kBinThreads / 2;
    const int nb = a.n > 0 ? (a.n + tb - 1) / tb : 1;
    k_col_count<<<nb, tb, 0, s>>>(a);
    *launches += 1;
    if (a.n > 0) {
        launch_pdl(k_col_scatter, nb, tb, 0, s, a);
        launch_pdl(k_col_sort, a.g.ncol, kColThreads, 0, s, a);
        *launches += 2;
    }
    return (int)cudaGetLastError();
}

int launch_bin(const BinArgs& a, cudaStream_t s, long long* launches)
{
    // k_bin_count runs even without atoms: its last block writes the (zero)
    // cell starts
    const int nb = a.n > 0 ? (a.n + kBinThreads - 1) / kBinThreads : 1;
    k_bin_count<<<nb, kBinThreads, 0, s>>>(a);
    *launches += 1;
    if (a.n > 0) {
        launch_pdl(k_bin_scatter, nb, kBinThreads, 0, s, a);
        launch_pdl(k_bin_cells, (a.grid.ncell + 3) / 4, 128, 0, s, a);
        *launches += 2;
    }
    return (int)cudaGetLastError();
}

}  // namespace pm
