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

}  // namespace

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
