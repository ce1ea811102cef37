// pm_cells.cu -- K1: cell binning by counting sort.
//
// Reproduces buildCellLists (topology/buildCellLists.cpp:11-38) bit for bit:
// the cell of atom i is floor((origin - min + minimalPosition(x_i)) *
// (1 / realCellSize)) evaluated in FP64 in the reference's operation order
// (CubicCellManager::findCell, topology/CubicCellManager.h:61-64).  Instead of
// the reference's linked lists (atoms pushed in reverse index order, so each
// list is in ascending index order) the atoms are counting-sorted into CSR
// cell ranges, ascending original index within a cell -- the same order the
// reference walks a cell list in.
//
// Roofline: HBM-bound; per atom it reads 24 B position + 8 B charge + 8 B
// type/molecule and writes 16 B spos + 16 B smeta + 12 B index arrays.
#include "pm_kernels.h"

namespace pm {

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

__global__ void k_bin_assign(BinArgs a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const CellGrid& g = a.grid;
    int cx, cy, cz;
    double vx, vy, vz;
    bin_cell_of(a.pbc, g, a.pos[3 * i], a.pos[3 * i + 1], a.pos[3 * i + 2], cx, cy, cz, vx, vy, vz);
    a.cell3[3 * i] = cx;
    a.cell3[3 * i + 1] = cy;
    a.cell3[3 * i + 2] = cz;
    if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz) {
        // The reference stores such an atom outside its cell array (an atom
        // exactly on the +L/2 face); here it is filed under its periodic
        // image and the event is reported.
        atomicOr(a.status, kStatusOutOfGrid);
        cx = ((cx % g.nx) + g.nx) % g.nx;
        cy = ((cy % g.ny) + g.ny) % g.ny;
        cz = ((cz % g.nz) + g.nz) % g.nz;
    }
    int c = (cx * g.ny + cy) * g.nz + cz;
    a.cell_lin[i] = c;
    // Morton key of the position inside the cell on an 8x8x8 sub-grid: runs
    // of 8 consecutive atoms in key order form compact clusters
    int qx = min(7, max(0, (int)(dmul(vx - (double)cx * g.csx, g.rcsx) * 8.0)));
    int qy = min(7, max(0, (int)(dmul(vy - (double)cy * g.csy, g.rcsy) * 8.0)));
    int qz = min(7, max(0, (int)(dmul(vz - (double)cz * g.csz, g.rcsz) * 8.0)));
    int key = 0;
#pragma unroll
    for (int b = 2; b >= 0; --b)
        key = (key << 3) | (((qx >> b) & 1) << 2) | (((qy >> b) & 1) << 1) | ((qz >> b) & 1);
    a.skey[i] = key;
    atomicAdd(a.counts + c, 1);
}

// Single-block exclusive scans of the per-cell atom counts (-> start) and
// cluster counts ceil(count / 8) (-> cstart); ncell <= a few 1e5.
__global__ void k_bin_scan(const int* counts, int* start, int* cstart, int ncell)
{
    __shared__ int part[1024], cpart[1024];
    int t = threadIdx.x;
    int per = (ncell + blockDim.x - 1) / blockDim.x;
    int b = t * per, e = min(ncell, b + per);
    int s = 0, cs = 0;
    for (int k = b; k < e; ++k) { s += counts[k]; cs += (counts[k] + kCluster - 1) / kCluster; }
    part[t] = s;
    cpart[t] = cs;
    __syncthreads();
    // Hillis-Steele inclusive scan over the per-thread sums
    for (int o = 1; o < blockDim.x; o <<= 1) {
        int v = t >= o ? part[t - o] : 0;
        int cv = t >= o ? cpart[t - o] : 0;
        __syncthreads();
        part[t] += v;
        cpart[t] += cv;
        __syncthreads();
    }
    int run = part[t] - s, crun = cpart[t] - cs;
    for (int k = b; k < e; ++k) {
        start[k] = run;
        cstart[k] = crun;
        run += counts[k];
        crun += (counts[k] + kCluster - 1) / kCluster;
    }
    if (t == blockDim.x - 1) { start[ncell] = part[t]; cstart[ncell] = cpart[t]; }
}

// Bounding box (FP32 cell-relative, hi parts) and cell of every 8-atom
// cluster; one thread per cluster (the cell by binary search of cstart).
__global__ void k_cluster_box(BinArgs a)
{
    int cl = blockIdx.x * blockDim.x + threadIdx.x;
    int ncl = a.cstart[a.grid.ncell];
    if (cl >= ncl || cl >= a.ncl_cap) return;
    int lo_c = 0, hi_c = a.grid.ncell;        // last cell with cstart <= cl
    while (hi_c - lo_c > 1) {
        int m = (lo_c + hi_c) >> 1;
        if (a.cstart[m] <= cl) lo_c = m; else hi_c = m;
    }
    int c = lo_c;
    int s = a.start[c] + (cl - a.cstart[c]) * kCluster;
    int e = min(a.start[c + 1], s + kCluster);
    float4 lo = make_float4(3e38f, 3e38f, 3e38f, 0.f), hi = make_float4(-3e38f, -3e38f, -3e38f, 0.f);
    for (int k = s; k < e; ++k) {
        float4 p = a.spos[k];
        lo.x = fminf(lo.x, p.x); lo.y = fminf(lo.y, p.y); lo.z = fminf(lo.z, p.z);
        hi.x = fmaxf(hi.x, p.x); hi.y = fmaxf(hi.y, p.y); hi.z = fmaxf(hi.z, p.z);
    }
    a.cbox[2 * cl] = lo;
    a.cbox[2 * cl + 1] = hi;
    a.ccell[cl] = c;
}

__global__ void k_bin_scatter(BinArgs a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    int c = a.cell_lin[i];
    int slot = a.start[c] + atomicAdd(a.fill + c, 1);
    a.tmp[slot] = i;
}

// Deterministic order inside a cell: by cell-relative z, ties by original
// index (the rank of an atom is the number of atoms of its cell before it),
// so that consecutive runs of 8 atoms form compact z-slabs (clusters).
// Also writes the FP32 cell-relative coordinates of the mixed kernels.
__global__ void k_bin_finish(BinArgs a)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n) return;
    int i = a.tmp[s];
    int c = a.cell_lin[i];
    int b = a.start[c], e = a.start[c + 1];
    int ki = a.skey[i];
    int rank = 0;
    for (int k = b; k < e; ++k) {
        int o = a.tmp[k];
        int ko = a.skey[o];
        rank += (ko < ki) || (ko == ki && o < i);
    }
    int dst = b + rank;
    a.sorted[dst] = i;
    a.slot_of[i] = dst;
    const CellGrid& g = a.grid;
    int cx, cy, cz;
    double vx, vy, vz;
    double x = a.pos[3 * i], y = a.pos[3 * i + 1], z = a.pos[3 * i + 2];
    bin_cell_of(a.pbc, g, x, y, z, cx, cy, cz, vx, vy, vz);
    // coordinates relative to the corner of the unwrapped cell; an atom filed
    // under its periodic image (cx = nx) lands just below that image's corner
    double rx = vx - (double)cx * g.csx;
    double ry = vy - (double)cy * g.csy;
    double rz = vz - (double)cz * g.csz;
    double qi = a.q[i];
    // compensated FP32: value = hi + lo to ~2^-48 relative, so that the
    // rounding of an atom's coordinates or charge does not bias all of its
    // pair terms the same way
    float hx = (float)rx, hy = (float)ry, hz = (float)rz, hq = (float)qi;
    a.spos[dst] = make_float4(hx, hy, hz, hq);
    a.slo[dst] = make_float4((float)(rx - (double)hx), (float)(ry - (double)hy), (float)(rz - (double)hz),
                             (float)(qi - (double)hq));
    a.smeta[dst] = make_int4(i, a.type[i], a.mol[i], 0);
    if (a.spos64) a.spos64[dst] = make_double4(x, y, z, qi);
}

int launch_bin(const BinArgs& a, cudaStream_t s, long long* launches)
{
    int nb = (a.n + 255) / 256;
    cudaMemsetAsync(a.counts, 0, sizeof(int) * a.grid.ncell, s);
    cudaMemsetAsync(a.fill, 0, sizeof(int) * a.grid.ncell, s);
    if (a.n > 0) {
        k_bin_assign<<<nb, 256, 0, s>>>(a);
    }
    k_bin_scan<<<1, 1024, 0, s>>>(a.counts, a.start, a.cstart, a.grid.ncell);
    if (a.n > 0) {
        k_bin_scatter<<<nb, 256, 0, s>>>(a);
        k_bin_finish<<<nb, 256, 0, s>>>(a);
        k_cluster_box<<<(a.ncl_cap + 127) / 128, 128, 0, s>>>(a);
    }
    *launches += a.n > 0 ? 5 : 1;
    return (int)cudaGetLastError();
}

}  // namespace pm
