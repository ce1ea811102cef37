// pm_pair_mixed.cuh -- K2: mixed-precision cluster-pair force kernels
// (included by pm_pair.cu, which provides the helpers).
//
// Clusters: inside a reference cell the atoms are ordered by the Morton key of
// their position on an 8x8x8 sub-grid of the cell (k_bin_cells), so every run
// of 8 consecutive atoms is a compact cluster with a bounding box (also
// k_bin_cells).  Up to four consecutive clusters of a cell form an
// i-supercluster (32 atoms).
//
// K2a k_cluster_list: one warp per cell and block of 32 half-shell cells.
// For each i-supercluster of the cell it lists every j-cluster of those
// cells of the half shell -- the cell itself (j-clusters >= the
// supercluster's first) and the positive half of the reference's
// neighbour-cell deltas, which covers every unordered cell pair once (in the
// small-grid mode, where a periodic image can occur twice among the deltas,
// the reference's list with its B > A rule) -- whose bounding box comes within
// the cutoff (plus the FP32 guard band) of at least one of the supercluster's
// cluster boxes, with a 4-bit mask of those i-clusters.  A warp's entries of
// a supercluster are contiguous and cut into chunks of p.chunk entries.  The
// interacting pair set is the reference's: only the order in which a pair's
// two atoms are visited differs, and forces are accumulated in
// order-independent fixed point.
//
// K2b k_pair_mixed: warps take chunks from a work counter.  A warp stages the
// chunk's 32 i-atoms in shared memory; for every entry it loads the j-cluster
// once (lane l holds j-atoms l / 8 and l / 8 + 4) and runs the 8x8 tiles of
// the masked i-clusters, i-atom l % 8 per lane: two independent pair
// evaluations per lane and tile, computed without branches (masked by
// selects) so that they interleave.  The next entry's j-atoms are fetched
// while the current one is computed.  j-forces are reduce-scattered over the
// 8 lanes of a j-atom once per entry (7 shuffles for 6 values) and added with
// one integer atomic per lane; i-forces stay in registers for the chunk.
// Energies are summed in FP64 over the chunk.  Every chunk's partials are
// rounded to int64 fixed point and summed as integers, so all results are
// independent of the order of the list and of the chunk-to-warp assignment.
//
// Near pairs (FP32 r^2 < near2, 5 A): on water their energies reach ~30
// kcal/mol each while the total is a ~1e-3 cancellation of the sum of |e|,
// so their FP32 rounding is nearly all of the energy error (1.8e-7 of |E_LJ|
// + |E_C| on the 14,281-atom box with FP32 energies everywhere).  K2b leaves
// their energies out and queues the pairs per warp in shared memory, then
// appends the queue to the near-pair list once per chunk (one atomic); K2c
// (k_near_energy) evaluates their energies in FP64 with the FP64 kernel's
// arithmetic, one pair per thread, each rounded to fixed point on its own.
// Their forces stay FP32.
//
// Virial: with the whole-cell offsets o of the half shell, the pair vector is
// d = (p_j + o) - p_i with p the atom's position relative to its cell
// corner, so sum_pairs d (x) f = sum_atoms p (x) F_pair + sum_entries o (x)
// F_entry, F_entry the entry's total force on its j-cluster.  The kernel adds
// the second sum (three FP64 products per lane and entry), the finalize kernel
// the first from the fixed-point pair forces.  In the small-grid mode (per-pair
// minimal image) the virial is summed per pair.

constexpr float kFarAway = 1.0e4f;   // position of the padding lanes of partial clusters
constexpr int kSuper = 4;            // clusters per i-supercluster
constexpr int kNearCap = 512;        // near pairs a warp queues for FP64 energies

// ---------------------------------------------------------------- K2a: list
__device__ __forceinline__ bool box_near(const float4& ilo, const float4& ihi, const float4& jlo, const float4& jhi,
                                         float ox, float oy, float oz, float lim)
{
    float bx = fmaxf(0.f, fmaxf((jlo.x + ox) - ihi.x, ilo.x - (jhi.x + ox)));
    float by = fmaxf(0.f, fmaxf((jlo.y + oy) - ihi.y, ilo.y - (jhi.y + oy)));
    float bz = fmaxf(0.f, fmaxf((jlo.z + oz) - ihi.z, ilo.z - (jhi.z + oz)));
    return bx * bx + by * by + bz * bz <= lim;
}

// entry: x = first j slot, y = (delta + 1) | nj << 16 | imask << 24
__device__ __forceinline__ int entry_y(int k, int nj, unsigned imask)
{
    return (k + 1) | (nj << 16) | (int)(imask << 24);
}

// the lane's candidate cell of the half shell (k = -1: the cell itself)
struct Cand {
    int k, jb, je, sb, eb, cb0;
    float ox, oy, oz;
};

__device__ __forceinline__ Cand candidate(const PairArgs& p, int A, int ax, int ay, int az, int ic0, int ca1, int k)
{
    const CellGrid& cg = p.grid;
    Cand c;
    c.k = k; c.jb = 0; c.je = 0; c.ox = c.oy = c.oz = 0.f;
    int B = A;
    if (k < 0) {
        c.jb = ic0; c.je = ca1;
    } else if (k < p.nh) {
        int4 d = p.hdeltas[k];
        int bx = ((ax + d.x) % cg.nx + cg.nx) % cg.nx;
        int by = ((ay + d.y) % cg.ny + cg.ny) % cg.ny;
        int bz = ((az + d.z) % cg.nz + cg.nz) % cg.nz;
        B = (bx * cg.ny + by) * cg.nz + bz;
        if (!(p.half_rule && B <= A)) {
            c.jb = p.cstart[B]; c.je = p.cstart[B + 1];
            float4 o = p.hoff[k];
            c.ox = o.x; c.oy = o.y; c.oz = o.z;
        }
    }
    c.sb = p.start[B]; c.eb = p.start[B + 1]; c.cb0 = p.cstart[B];
    return c;
}

// mask of the supercluster's i-clusters whose box comes near j-cluster jc
__device__ __forceinline__ unsigned near_mask(const PairArgs& p, const Cand& c, int jc, const float4 (&ilo)[kSuper],
                                              const float4 (&ihi)[kSuper], int nsc, int ic0, float lim)
{
    const float4 jlo = p.cbox[2 * jc], jhi = p.cbox[2 * jc + 1];
    unsigned m = 0u;
#pragma unroll
    for (int q = 0; q < kSuper; ++q)
        if (q < nsc && (c.k >= 0 || jc >= ic0 + q) &&
            (p.wrap || box_near(ilo[q], ihi[q], jlo, jhi, c.ox, c.oy, c.oz, lim)))
            m |= 1u << q;
    return m;
}

__global__ void __launch_bounds__(128) k_cluster_list(PairArgs p)
{
    pdl_wait();
    // one warp per (cell, block of 32 half-shell cells): the warp's entries of
    // a supercluster are contiguous and cut into their own chunks
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const CellGrid& cg = p.grid;
    const int nkb = (p.nh + 1 + 31) / 32;                    // slot 0: the cell itself
    const int A = gw / nkb;
    if (A >= cg.ncell) return;                               // warp-uniform
    const int k = (gw - A * nkb) * 32 + lane - 1;
    const int ca0 = p.cstart[A], ca1 = p.cstart[A + 1];
    const int sa = p.start[A], ea = p.start[A + 1];
    const int ax = A / (cg.ny * cg.nz), ay = (A / cg.nz) % cg.ny, az = A % cg.nz;
    // tiles farther apart than this (FP32 box distance^2) hold no pair
    const float lim = p.cut2f * (1.0f + 8.0f * p.guard) + 1e-3f;
    for (int ic0 = ca0; ic0 < ca1; ic0 += kSuper) {
        const int nsc = min(kSuper, ca1 - ic0);
        const int ifirst = sa + (ic0 - ca0) * kCluster;
        const int nit = min(kSuper * kCluster, ea - ifirst);
        float4 ilo[kSuper], ihi[kSuper];
#pragma unroll
        for (int q = 0; q < kSuper; ++q) {
            const int ic = min(ic0 + q, ca1 - 1);
            ilo[q] = p.cbox[2 * ic]; ihi[q] = p.cbox[2 * ic + 1];
        }
        const Cand c = candidate(p, A, ax, ay, az, ic0, ca1, k);
        // the masks of the first 8 j-clusters are kept (4 bits each) for the
        // writing pass; a cell with more clusters recomputes the rest
        int cnt = 0;
        unsigned kept = 0u;
        for (int jc = c.jb; jc < c.je; ++jc) {
            const unsigned m = near_mask(p, c, jc, ilo, ihi, nsc, ic0, lim);
            if (jc - c.jb < 8) kept |= m << (4 * (jc - c.jb));
            cnt += m ? 1 : 0;
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int ne = __shfl_sync(FULL, incl, 31);
        if (ne == 0) continue;
        const int nch = (ne + p.chunk - 1) / p.chunk;
        int b0 = 0, b1 = 0;
        if (lane == 0) {
            b0 = atomicAdd(p.plist_count, ne);
            b1 = atomicAdd(p.chunk_count, nch);
            if (b0 + ne > p.plist_cap) { atomicOr(p.status, kStatusListFull); atomicMax(p.plist_need, b0 + ne); }
            if (b1 + nch > p.chunk_cap) { atomicOr(p.status, kStatusListFull); atomicMax(p.chunk_need, b1 + nch); }
        }
        const int ebase = __shfl_sync(FULL, b0, 0), cbase = __shfl_sync(FULL, b1, 0);
        int w = ebase + incl - cnt;
        for (int jc = c.jb; jc < c.je && cnt > 0; ++jc) {
            const unsigned m = jc - c.jb < 8 ? (kept >> (4 * (jc - c.jb))) & 0xfu
                                             : near_mask(p, c, jc, ilo, ihi, nsc, ic0, lim);
            if (!m) continue;
            if (w < p.plist_cap) {
                const int jfirst = c.sb + (jc - c.cb0) * kCluster;
                p.plist[w] = make_int2(jfirst, entry_y(c.k, min(kCluster, c.eb - jfirst), m));
            }
            ++w;
        }
        // chunk descriptors: {first i slot, i atoms, first entry, entries}
        for (int t = lane; t < nch; t += 32)
            if (cbase + t < p.chunk_cap && ebase + ne <= p.plist_cap)
                p.chunks[cbase + t] = make_int4(ifirst, nit, ebase + t * p.chunk, min(p.chunk, ne - t * p.chunk));
    }
}

// ---------------------------------------------------------------- K2b: pairs
struct JAtom {
    float4 p, l;     // FP32 hi / lo of the cell-relative position and charge
    int4 m;          // original index, LJ type, molecule
};

__device__ __forceinline__ void load_atom(const PairArgs& p, int slot, bool valid, float far, JAtom& a)
{
    if (valid) {
        a.p = p.spos[slot]; a.l = p.slo[slot]; a.m = p.smeta[slot];
    } else {   // padding: far away, no charge, type 0, no molecule
        a.p = make_float4(far, far, far, 0.f); a.l = make_float4(0.f, 0.f, 0.f, 0.f);
        a.m = make_int4(-1, 0, -2, 0);
    }
}

struct PairGeo {
    float dx, dy, dz, r2;
    bool act, in0, in1;
    bool near, same;             // inside a cutoff's guard band; the same molecule
    int excl;
};

// geometry and the FP32 within-cutoff decision of one pair; the two rare
// cases -- a distance inside a cutoff's guard band (exact FP64 decision) and
// a pair of one molecule (the exclusion class) -- are only flagged here and
// resolved by resolve_rare, which a warp enters only when one of its lanes
// holds such a pair
template <int NT, int S0, int S1, bool WRAP>
__device__ __forceinline__ PairGeo pair_geo(const PairArgs& p, const JAtom& ia, const JAtom& ja,
                                            float ox, float oy, float oz, float olx, float oly, float olz,
                                            bool valid)
{
    PairGeo g;
    const float g_lo = 1.0f - p.guard, g_hi = 1.0f + p.guard;
    const float t0c2 = p.tf[0].cut2, t1c2 = NT > 1 ? p.tf[1].cut2 : 0.f;
    // every rounding depends on both atoms; the lo parts restore the
    // coordinates and the cell offset to ~2^-48
    float dx = ((ja.p.x - ia.p.x) + ox) + ((ja.l.x - ia.l.x) + olx);
    float dy = ((ja.p.y - ia.p.y) + oy) + ((ja.l.y - ia.l.y) + oly);
    float dz = ((ja.p.z - ia.p.z) + oz) + ((ja.l.z - ia.l.z) + olz);
    if (WRAP) {
        float kx = rintf(dx * p.ilx), ky = rintf(dy * p.ily), kz = rintf(dz * p.ilz);
        dx = fmaf(-p.lx, kx, fmaf(-p.lx_lo, kx, dx));
        dy = fmaf(-p.ly, ky, fmaf(-p.ly_lo, ky, dy));
        dz = fmaf(-p.lz, kz, fmaf(-p.lz_lo, kz, dz));
    }
    float r2 = dx * dx + dy * dy + dz * dz;
    bool far = r2 > p.cut2f * g_hi;
    bool near = !far && r2 >= p.cut2f * g_lo;
    if (S0 == SCUT && t0c2 != p.cut2f) near |= (r2 >= t0c2 * g_lo && r2 <= t0c2 * g_hi);
    if (NT > 1 && S1 == SCUT && t1c2 != p.cut2f) near |= (r2 >= t1c2 * g_lo && r2 <= t1c2 * g_hi);
    g.near = near && valid;
    g.in0 = r2 <= t0c2;
    g.in1 = NT > 1 ? r2 <= t1c2 : false;
    g.act = valid && !far;
    g.same = ia.m.z == ja.m.z;
    g.excl = PMGPU_EXCL_NONE;
    g.dx = dx; g.dy = dy; g.dz = dz; g.r2 = r2;
    return g;
}

__device__ __forceinline__ bool is_rare(const PairGeo& g) { return g.near || (g.act && g.same); }

// the exact FP64 decision inside the guard band, then the exclusion class of
// a pair of one molecule (ExclusionTable::check)
template <int NT>
__device__ __forceinline__ void resolve_rare(const PairArgs& p, PairGeo& g, const JAtom& ia, const JAtom& ja)
{
    if (g.near) {
        const double d2 = exact_d2(p, ia.m.x, ja.m.x);
        g.act = !(d2 > p.cut2d);                  // near implies a valid pair
        g.in0 = !(d2 > p.td[0].cut2);
        g.in1 = NT > 1 ? !(d2 > p.td[1].cut2) : false;
    }
    if (g.act && g.same) {
        g.excl = excl_class(p, ia.m.x, ja.m.x);
        if (g.excl == PMGPU_EXCL_FULL) g.act = false;
    }
}

// 1/sqrt(x) and 1/x: the hardware approximation and one Newton-Raphson step
// (y' = y + y (1 - x y^2) / 2, y' = y + y (1 - x y)), faithful to ~1 ulp, for
// the normal positive arguments of the pair kernel
__device__ __forceinline__ float rsqrt_nr(float x)
{
    float y = rsqrtf(x);
    float e = fmaf(-x * y, y, 1.0f);
    return fmaf(0.5f * y, e, y);
}

// the OneAtomPair[Two] terms of one pair (OneAtomPairTwo.h doOneAtomPair:
// both switches are applied when either modifies): scalar force factor
// (F_j = d * ft) and energies, zero for an inactive pair
template <int NT, int P0, int S0, int P1, int S1>
__device__ __forceinline__ void pair_math(const PairArgs& p, const PairGeo& g, const JAtom& ia, const JAtom& ja,
                                          float& ft, float& el, float& ec)
{
    constexpr bool kMod = sw_modifies(S0) || (NT > 1 && sw_modifies(S1));
    const float r2 = g.act ? g.r2 : 1.0f;         // keeps inactive lanes finite
    float rinv = rsqrt_nr(r2);
    float rd2 = rinv * rinv;
    float qq = fmaf(ia.p.w, ja.p.w, fmaf(ia.p.w, ja.l.w, ia.l.w * ja.p.w));
    float e0, f0, e1 = 0.f, f1 = 0.f;
    pot_f32<P0>(p, p.tf[0], r2, rd2, rinv, qq, ia.m.y, ja.m.y, g.excl, e0, f0);
    if (NT > 1) pot_f32<P1>(p, p.tf[1], r2, rd2, rinv, qq, ia.m.y, ja.m.y, g.excl, e1, f1);
    if (kMod) {
        float sv, sd;
        sw_f32<S0>(p.tf[0], r2, rinv, g.in0, sv, sd);
        f0 = f0 * sv - e0 * sd;
        e0 = e0 * sv;
        if (NT > 1) {
            sw_f32<S1>(p.tf[1], r2, rinv, g.in1, sv, sd);
            f1 = f1 * sv - e1 * sd;
            e1 = e1 * sv;
        }
    }
    float l = 0.f, c = 0.f;
    if (pot_lj_slot(P0)) l += e0; else c += e0;
    if (NT > 1) { if (pot_lj_slot(P1)) l += e1; else c += e1; }
    ft = g.act ? f0 + f1 : 0.f;
    el = g.act ? l : 0.f;
    ec = g.act ? c : 0.f;
}

// FP64 energies of one pair of sorted slots, the FP64 kernel's arithmetic
// (pot_f64, sw_f64) on the raw positions and charges (spos64) and the exact
// minimal image: the FP64 kernel's value of the pair
template <int NT, int P0, int S0, int P1, int S1>
__device__ __forceinline__ void pair_energy_f64(const PairArgs& p, int si, int sj, int excl, double& el, double& ec)
{
    constexpr bool kMod = sw_modifies(S0) || (NT > 1 && sw_modifies(S1));
    const double4 pi = p.spos64[si], pj = p.spos64[sj];
    const int ti = p.smeta[si].y, tj = p.smeta[sj].y;
    double dx, dy, dz;
    const double d2 = pbc_min_diff(p.pbc, pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, dx, dy, dz);
    const double rd2 = 1.0 / d2;
    double e0, f0, e1 = 0.0, f1 = 0.0;
    pot_f64<P0>(p, p.td[0], d2, rd2, pi.w, pj.w, ti, tj, excl, e0, f0);
    if (NT > 1) pot_f64<P1>(p, p.td[1], d2, rd2, pi.w, pj.w, ti, tj, excl, e1, f1);
    if (kMod) {
        double sv, sd;
        sw_f64<S0>(p.td[0], d2, sv, sd);
        e0 *= sv;
        if (NT > 1) {
            sw_f64<S1>(p.td[1], d2, sv, sd);
            e1 *= sv;
        }
    }
    el += (pot_lj_slot(P0) ? e0 : 0.0) + (NT > 1 && pot_lj_slot(P1) ? e1 : 0.0);
    ec += (!pot_lj_slot(P0) ? e0 : 0.0) + (NT > 1 && !pot_lj_slot(P1) ? e1 : 0.0);
}

// the warp's queued near pairs -> the near-pair list (called by the whole
// warp); a full list sets the capacity status and the size it needs
__device__ __forceinline__ void append_near(const PairArgs& p, const int2* q, int nq, int lane)
{
    const unsigned FULL = 0xffffffffu;
    __syncwarp();                                    // the other lanes' entries are visible
    int base = 0;
    if (lane == 0) base = atomicAdd(p.near_count, nq);
    base = __shfl_sync(FULL, base, 0);
    if (base <= p.near_cap - nq) {
        for (int k = lane; k < nq; k += 32) p.near[base + k] = q[k];
    } else if (lane == 0) {
        atomicOr(p.status, kStatusListFull);
        atomicMax(p.near_need, base + nq);
    }
    __syncwarp();                                    // the queue is refilled next
}

// int64 fixed-point add of one FP32 value (value * 2^32 is exact in FP32)
__device__ __forceinline__ void fixed_addf(unsigned long long* slot, float v, int* status)
{
    float s = v * 4294967296.0f;
    if (!(fabsf(s) < 4.0e18f)) { atomicOr(status, kStatusOverflow); return; }
    long long q = __float2ll_rn(s);
    if (q != 0) atomicAdd(slot, (unsigned long long)q);
}

// FP64 partial -> int64 fixed point (scale 2^32)
__device__ __forceinline__ long long fixed_of(double v, bool& bad)
{
    double s = v * 4294967296.0;
    bad |= !(fabs(s) < 4.0e18);
    return __double2ll_rn(s);
}

// sum over the 4 lanes of an i-atom (lanes il + 8 jg), scattered: lane
// (il, jg) ends with component jg of i-atom il (component 3 is zero)
__device__ __forceinline__ float i_reduce_scatter(float fx, float fy, float fz, int jg)
{
    const unsigned FULL = 0xffffffffu;
    const bool hb = (jg >> 1) & 1, lb = jg & 1;
    float k0 = (hb ? fz : fx) + __shfl_xor_sync(FULL, hb ? fx : fz, 16);     // component 2 hb
    float k1 = (hb ? 0.f : fy) + __shfl_xor_sync(FULL, hb ? fy : 0.f, 16);   // component 2 hb + 1
    return (lb ? k1 : k0) + __shfl_xor_sync(FULL, lb ? k0 : k1, 8);
}

// sum over the 8 lanes il of a jg of (a.x, a.y, a.z, b.x, b.y, b.z, 0, 0),
// scattered: lane il ends with value il
__device__ __forceinline__ float j_reduce_scatter(float ax, float ay, float az, float bx, float by, float bz, int il)
{
    const unsigned FULL = 0xffffffffu;
    const bool b2 = (il >> 2) & 1, b1 = (il >> 1) & 1, b0 = il & 1;
    float w0 = (b2 ? by : ax) + __shfl_xor_sync(FULL, b2 ? ax : by, 4);
    float w1 = (b2 ? bz : ay) + __shfl_xor_sync(FULL, b2 ? ay : bz, 4);
    float w2 = (b2 ? 0.f : az) + __shfl_xor_sync(FULL, b2 ? az : 0.f, 4);
    float w3 = (b2 ? 0.f : bx) + __shfl_xor_sync(FULL, b2 ? bx : 0.f, 4);
    // w[k] = value k + 4 b2
    float u0 = (b1 ? w2 : w0) + __shfl_xor_sync(FULL, b1 ? w0 : w2, 2);
    float u1 = (b1 ? w3 : w1) + __shfl_xor_sync(FULL, b1 ? w1 : w3, 2);
    // u[k] = value k + 2 b1 + 4 b2
    return (b0 ? u1 : u0) + __shfl_xor_sync(FULL, b0 ? u0 : u1, 1);
}

template <int NT, int P0, int S0, int P1, int S1, bool WRAP>
__global__ void __launch_bounds__(128, 4) k_pair_mixed(PairArgs p)
{
    pdl_wait();
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, il = lane & 7, jg = lane >> 3;
    __shared__ float4 s_p[4][kSuper * kCluster], s_l[4][kSuper * kCluster];
    __shared__ int4 s_m[4][kSuper * kCluster];
    __shared__ int2 s_near[4][kNearCap];
    __shared__ unsigned long long s_e[kERec];
    if (threadIdx.x < kERec) s_e[threadIdx.x] = 0ull;
    __syncthreads();
    // per-lane int64 sums over the chunks: LJ, Coulomb, and the lane's virial
    // column (shift form: W[0..2][c]; per-pair form: xx xy xz yy yz zz)
    long long acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool bad = false;
    const int nchunks = (*p.status & kStatusListFull) ? 0 : min(*p.chunk_count, p.chunk_cap);
    const int comp = il < 3 ? il : il - 3;           // j-force component held after the reduce-scatter
    const int jsel = il < 3 ? 0 : 4;                 // j-atom jg or jg + 4

    while (true) {
        int ch = 0;
        if (lane == 0) ch = atomicAdd(p.chunk_next, 1);
        ch = __shfl_sync(FULL, ch, 0);
        if (ch >= nchunks) break;
        const int4 cd = p.chunks[ch];
        {
            JAtom a;
            load_atom(p, cd.x + lane, lane < cd.y, kFarAway, a);
            s_p[w][lane] = a.p; s_l[w][lane] = a.l; s_m[w][lane] = a.m;
        }
        __syncwarp();
        // i-forces of the four i-clusters; the loop over them below is not
        // unrolled (one copy of the pair code keeps the instruction cache
        // warm), so the registers rotate: fi[0] is always the current cluster
        float fi[kSuper][3];
#pragma unroll
        for (int q = 0; q < kSuper; ++q) fi[q][0] = fi[q][1] = fi[q][2] = 0.f;
        double el = 0.0, ec = 0.0;
        int nq = 0;                                // queued near pairs
        double wv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};

        const int e_end = cd.z + cd.w;
        int2 ent = p.plist[cd.z];
        int2 ent_next = cd.z + 1 < e_end ? p.plist[cd.z + 1] : ent;
        JAtom ja, jb;
        {
            const int nj = (ent.y >> 16) & 0xff;
            load_atom(p, ent.x + jg, jg < nj, -kFarAway, ja);
            load_atom(p, ent.x + jg + 4, jg + 4 < nj, -kFarAway, jb);
        }
        for (int e = cd.z; e < e_end; ++e) {
            if (nq > kNearCap - 2 * kSuper * 32) {         // room for one more entry
                append_near(p, s_near[w], nq, lane);
                nq = 0;
            }
            const int2 cur = ent;
            const JAtom ca = ja, cb = jb;
            if (e + 1 < e_end) {                   // software pipeline
                ent = ent_next;
                const int nj = (ent.y >> 16) & 0xff;
                load_atom(p, ent.x + jg, jg < nj, -kFarAway, ja);
                load_atom(p, ent.x + jg + 4, jg + 4 < nj, -kFarAway, jb);
                if (e + 2 < e_end) ent_next = p.plist[e + 2];
            }
            const int k = (cur.y & 0xffff) - 1;
            const int nj = (cur.y >> 16) & 0xff;
            const unsigned imask = (unsigned)cur.y >> 24;
            float ox = 0.f, oy = 0.f, oz = 0.f, olx = 0.f, oly = 0.f, olz = 0.f;
            if (k >= 0) {
                const float4 o = p.hoff[k], ol = p.hoff_lo[k];
                ox = o.x; oy = o.y; oz = o.z; olx = ol.x; oly = ol.y; olz = ol.z;
            }
            float fax = 0.f, fay = 0.f, faz = 0.f, fbx = 0.f, fby = 0.f, fbz = 0.f;
            bool entry_math = false;                       // warp-uniform: a tile of this entry ran the math
#pragma unroll 1
            for (int q = 0; q < kSuper; ++q) {
                if (imask & (1u << q)) {                   // warp-uniform
                    const int s = q * kCluster + il;
                    JAtom ia;
                    ia.p = s_p[w][s]; ia.l = s_l[w][s]; ia.m = s_m[w][s];
                    const bool vi = s < cd.y;
                    const bool diag = k < 0 && cur.x == cd.x + q * kCluster;   // i-cluster with itself
                    const bool va = vi && jg < nj && (!diag || jg > il);
                    const bool vb = vi && jg + 4 < nj && (!diag || jg + 4 > il);
                    PairGeo ga = pair_geo<NT, S0, S1, WRAP>(p, ia, ca, ox, oy, oz, olx, oly, olz, va);
                    PairGeo gb = pair_geo<NT, S0, S1, WRAP>(p, ia, cb, ox, oy, oz, olx, oly, olz, vb);
                    if (__any_sync(FULL, is_rare(ga) || is_rare(gb))) {   // warp-uniform, rare
                        resolve_rare<NT>(p, ga, ia, ca);
                        resolve_rare<NT>(p, gb, ia, cb);
                    }
                    // the math only for the 8x4 half-tiles (j-atoms 0-3 and
                    // 4-7, spatially separate halves of the cluster) that hold a
                    // pair inside the cutoff: about 40% of them hold none
                    const bool any_a = __any_sync(FULL, ga.act), any_b = __any_sync(FULL, gb.act);
                    if (!(any_a || any_b)) goto next_cluster;
                    entry_math = true;
                    float fta = 0.f, ela = 0.f, eca = 0.f, ftb = 0.f, elb = 0.f, ecb = 0.f;
                    if (any_a && any_b) {
                        pair_math<NT, P0, S0, P1, S1>(p, ga, ia, ca, fta, ela, eca);
                        pair_math<NT, P0, S0, P1, S1>(p, gb, ia, cb, ftb, elb, ecb);
                    } else {
                        float ft, e1, e2;
                        pair_math<NT, P0, S0, P1, S1>(p, any_a ? ga : gb, ia, any_a ? ca : cb, ft, e1, e2);
                        if (any_a) { fta = ft; ela = e1; eca = e2; } else { ftb = ft; elb = e1; ecb = e2; }
                    }
                    const float x1 = ga.dx * fta, y1 = ga.dy * fta, z1 = ga.dz * fta;
                    const float x2 = gb.dx * ftb, y2 = gb.dy * ftb, z2 = gb.dz * ftb;
                    fi[0][0] -= x1 + x2; fi[0][1] -= y1 + y2; fi[0][2] -= z1 + z2;
                    fax += x1; fay += y1; faz += z1; fbx += x2; fby += y2; fbz += z2;
                    // near pairs: queued for FP64 energies in place of the FP32 ones
                    {
                        const bool na = ga.act && ga.r2 < p.near2, nb = gb.act && gb.r2 < p.near2;   // near2 = 0: none
                        if (__any_sync(FULL, na || nb)) {
                            const unsigned ba = __ballot_sync(FULL, na), bb = __ballot_sync(FULL, nb);
                            const unsigned lt = (1u << lane) - 1u;
                            const int si = cd.x + q * kCluster + il, sj = cur.x + jg;
                            if (na) {
                                s_near[w][nq + __popc(ba & lt)] =
                                    make_int2(si, sj | (ga.excl == PMGPU_EXCL_MODIFIED ? 1 << 30 : 0));
                                ela = 0.f; eca = 0.f;
                            }
                            nq += __popc(ba);
                            if (nb) {
                                s_near[w][nq + __popc(bb & lt)] =
                                    make_int2(si, (sj + 4) | (gb.excl == PMGPU_EXCL_MODIFIED ? 1 << 30 : 0));
                                elb = 0.f; ecb = 0.f;
                            }
                            nq += __popc(bb);
                        }
                    }
                    el += (double)(ela + elb);
                    ec += (double)(eca + ecb);
                    if (WRAP && p.virial) {
                        wv[0] += (double)fmaf(x1, ga.dx, x2 * gb.dx);
                        wv[1] += (double)fmaf(x1, ga.dy, x2 * gb.dy);
                        wv[2] += (double)fmaf(x1, ga.dz, x2 * gb.dz);
                        wv[3] += (double)fmaf(y1, ga.dy, y2 * gb.dy);
                        wv[4] += (double)fmaf(y1, ga.dz, y2 * gb.dz);
                        wv[5] += (double)fmaf(z1, ga.dz, z2 * gb.dz);
                    }
                    if (p.rec_pairs) {                      // diagnostic pair recording
#pragma unroll
                        for (int t = 0; t < 2; ++t) {
                            const PairGeo& g = t ? gb : ga;
                            const JAtom& j = t ? cb : ca;
                            if (g.act) {
                                unsigned long long r = atomicAdd(p.rec_count, 1ull);
                                if ((long long)r < p.rec_cap) {
                                    p.rec_pairs[2 * r] = min(ia.m.x, j.m.x);
                                    p.rec_pairs[2 * r + 1] = max(ia.m.x, j.m.x);
                                }
                            }
                        }
                    }
                }
              next_cluster:
                // rotate: the next cluster's forces become fi[0]
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float t = fi[0][c];
                    fi[0][c] = fi[1][c]; fi[1][c] = fi[2][c]; fi[2][c] = fi[3][c]; fi[3][c] = t;
                }
            }
            // j-forces: lane il ends with component comp of j-atom jg + jsel
            // (nothing to add when no tile of the entry held a pair)
            if (entry_math) {
                const float v = j_reduce_scatter(fax, fay, faz, fbx, fby, fbz, il);
                if (il < 6 && jg + jsel < nj && v != 0.f)
                    fixed_addf(p.facc + 3 * (size_t)(cur.x + jg + jsel) + comp, v, p.status);
                if (!WRAP && p.virial && il < 6 && k >= 0) {   // o (x) F_entry, column comp
                    const double4 o64 = p.hoff64[k];
                    wv[0] = fma(o64.x, (double)v, wv[0]);
                    wv[1] = fma(o64.y, (double)v, wv[1]);
                    wv[2] = fma(o64.z, (double)v, wv[2]);
                }
            }
        }
        // chunk end: i-forces, then the chunk's partials in fixed point
#pragma unroll
        for (int q = 0; q < kSuper; ++q) {
            const float v = i_reduce_scatter(fi[q][0], fi[q][1], fi[q][2], jg);
            const int s = q * kCluster + il;
            if (jg < 3 && s < cd.y && v != 0.f) fixed_addf(p.facc + 3 * (size_t)(cd.x + s) + jg, v, p.status);
        }
        if (nq > 0) append_near(p, s_near[w], nq, lane);
        acc[0] += fixed_of(el, bad);
        acc[1] += fixed_of(ec, bad);
        if (p.virial) {
#pragma unroll
            for (int t = 0; t < 6; ++t) acc[2 + t] += fixed_of(wv[t], bad);
        }
        __syncwarp();                                      // s_p is reused by the next chunk
    }
    if (bad) atomicOr(p.status, kStatusOverflow);
    // warp sums into shared int64 slots, then one atomic per block and component
#pragma unroll
    for (int t = 0; t < 2; ++t)
        for (int o = 16; o > 0; o >>= 1) acc[t] += __shfl_xor_sync(FULL, acc[t], o);
    if (lane == 0) {
        atomicAdd(&s_e[0], (unsigned long long)acc[0]);
        atomicAdd(&s_e[1], (unsigned long long)acc[1]);
    }
    if (p.virial) {
        if (WRAP) {
            // per-pair form: xx xy xz yy yz zz
#pragma unroll
            for (int t = 2; t < 8; ++t)
                for (int o = 16; o > 0; o >>= 1) acc[t] += __shfl_xor_sync(FULL, acc[t], o);
            if (lane == 0) {
                const int slot[6] = {2, 3, 4, 6, 7, 10};
#pragma unroll
                for (int t = 0; t < 6; ++t) atomicAdd(&s_e[slot[t]], (unsigned long long)acc[2 + t]);
                atomicAdd(&s_e[5], (unsigned long long)acc[3]);    // yx = xy
                atomicAdd(&s_e[8], (unsigned long long)acc[4]);    // zx = xz
                atomicAdd(&s_e[9], (unsigned long long)acc[6]);    // zy = yz
            }
        } else if (il < 6) {
            // shift form: the lane holds W[a][comp] for a = x, y, z
#pragma unroll
            for (int a = 0; a < 3; ++a) atomicAdd(&s_e[2 + 3 * a + comp], (unsigned long long)acc[2 + a]);
        }
    }
    __syncthreads();
    if (threadIdx.x < kERec && s_e[threadIdx.x] != 0ull) atomicAdd(p.efix + threadIdx.x, s_e[threadIdx.x]);
}

// K2c: the FP64 energies of the near pairs the mixed pair kernel listed (it
// left their FP32 energies out).  Each pair's energies are rounded to int64
// fixed point on their own, so the sums do not depend on the list's order.
template <int NT, int P0, int S0, int P1, int S1>
__global__ void __launch_bounds__(128) k_near_energy(PairArgs p)
{
    const unsigned FULL = 0xffffffffu;
    __shared__ long long s_acc[2][4];
    if (*p.status & kStatusListFull) return;               // block-uniform
    const int n = min(*p.near_count, p.near_cap);
    long long al = 0, ac = 0;
    bool bad = false;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int2 e = p.near[k];
        double el = 0.0, ec = 0.0;
        pair_energy_f64<NT, P0, S0, P1, S1>(p, e.x, e.y & 0x3fffffff,
                                            (e.y >> 30) ? PMGPU_EXCL_MODIFIED : PMGPU_EXCL_NONE, el, ec);
        al += fixed_of(el, bad);
        ac += fixed_of(ec, bad);
    }
    if (bad) atomicOr(p.status, kStatusOverflow);
    for (int o = 16; o > 0; o >>= 1) {
        al += __shfl_xor_sync(FULL, al, o);
        ac += __shfl_xor_sync(FULL, ac, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { s_acc[0][w] = al; s_acc[1][w] = ac; }
    __syncthreads();
    if (threadIdx.x < 2) {
        long long t = s_acc[threadIdx.x][0] + s_acc[threadIdx.x][1] + s_acc[threadIdx.x][2] + s_acc[threadIdx.x][3];
        if (t != 0) atomicAdd(p.efix + threadIdx.x, (unsigned long long)t);
    }
}
