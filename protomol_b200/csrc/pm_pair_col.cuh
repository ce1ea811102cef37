// pm_pair_col.cuh -- K2a' / K2b' / K2c': the mixed-precision pair force over
// column clusters (included by pm_pair.cu after pm_pair_mixed.cuh, whose
// helpers it shares).
//
// Layout (K1c, pm_cells.cu): every atom holds an unsigned 32-bit fixed-point
// coordinate of the periodic box per axis, q = round(frac((x - min) / L) 2^32).
// The int32 difference of two atoms' coordinates is then their minimal-image
// displacement in units of L / 2^32, exactly: no cell offset and no rounding
// shared by the pairs of an atom or of a cell pair enters the pair vector.
// The only roundings are the conversion of that integer to FP32 and its
// product with the FP32 hi + lo of L / 2^32, both unbiased, so the FP32 pair
// energies carry no systematic error into the sums (cell-relative FP32
// coordinates with FP32 cell offsets lose the offsets' and the atoms' FP32
// remainders in the last addition, a bias of ~1e-8 of every distance).
//
// Clusters: the atoms of one column of an x-y grid (~4 A side), sorted by z,
// cut into runs of 8 (i-clusters); each half of an i-cluster is a 4-atom
// j-cluster.  A warp's tile is one i-cluster against one j-cluster: 8 x 4
// pairs, one per lane (lane l: i-atom l % 8, j-atom l / 8).
//
// K2a' k_col_list: one warp per i-cluster, one lane per candidate column of
// the half neighbourhood.  A j-cluster is listed when its bounding box, in
// the periodic image the column and the z window select, comes within the
// cutoff (plus the FP32 guard band) of the i-cluster's box.  Every unordered
// pair of atoms is visited once: a pair of columns from the one whose offset
// to the other is in the positive half (ox > 0, or ox = 0 < oy), the own
// column from the own cluster on, and in the own cluster (diag tiles) only
// j > i.  The box edges are more
// than (2 rx + 1) columns wide and the z windows shorter than the box, so no
// j-cluster is reached twice, and every pair inside the cutoff lies in the
// tile's image (t, the entry's shift), which the virial's shift form needs.
//
// K2b' k_pair_col: persistent warps over chunks of one i-cluster's entries,
// two tiles per iteration.  i-forces stay in registers for the chunk;
// j-forces are reduce-scattered over the 8 lanes of a j-atom and added in
// int64 fixed point.  The exact FP64 decisions near a cutoff, the exclusion
// classes, the near pairs' FP64 energies and the fixed-point sums are those
// of K2b.
//
// Virial in the shift form, with each atom's position taken from its
// i-cluster's origin O_c (the cluster's first atom), so that the lever arm
// of the per-atom term is a cluster's size, not the box's:
// sum_pairs d (x) f = sum_atoms (x - O_c(a)) (x) F + sum_tiles o (x) F_tile,
// o = O_c(j) - O_c(i) + t L.  The finalize kernel adds the first sum from
// the fixed-point positions and forces; the list kernel stores each tile's
// o in FP32 (a rounding of the tile's own) and the pair kernel sums o (x)
// F_tile in FP64.

__device__ __forceinline__ int col_entry_y(int tx, int ty, int tz, bool diag)
{
    return (tx + 1) | ((ty + 1) << 2) | ((tz + 1) << 4) | ((diag ? 1 : 0) << 6);
}

// the j-cluster range [jb, je) of column colj's image tz whose boxes may meet
// the window [zlo, zhi] (in the box frame): j-boxes are sorted by z in a
// column (both corners monotone), so the column's z index gives a start at
// or before each end of the range, and a short forward scan finds it
__device__ __forceinline__ int2 col_zrange(const PairArgs& p, int colj, int jb, int je, float zlo, float zhi,
                                           float sz)
{
    const float plo = zlo - sz, phi = zhi - sz;          // the window in the column's frame [0, L)
    if (phi < 0.f || plo >= p.cg.lzf) return make_int2(jb, 0);
    const int* zi = p.zidx + (size_t)colj * kZIndex;
    const float inv = kZBins / p.cg.lzf;
    // first j-cluster ending at or above plo, from the bin edge one below
    // plo's (the FP32 bin of plo may round up by one)
    const int b0 = plo <= 0.f ? 0 : max(0, min(kZBins, (int)(plo * inv)) - 1);
    int lo = max(jb, __ldg(zi + b0));
    while (lo < je && p.jbox[2 * lo + 1].z < plo) ++lo;
    // first j-cluster starting above phi, likewise from one bin edge below
    const int b1 = max(0, min(kZBins, (int)(phi * inv)) - 1);
    int lo2 = max(lo, __ldg(zi + kZBins + 1 + b1));
    while (lo2 < je && p.jbox[2 * lo2].z <= phi) ++lo2;
    return make_int2(lo, lo2 - lo);
}

constexpr int kColStageEntries = 512;    // entries of one i-cluster staged in shared memory
constexpr int kEnergyFlush = 8;          // pair-kernel iterations per FP32 energy partial sum

// The list of i-cluster ic (one warp): every candidate column of the half
// neighbourhood -- the column offsets (ox, oy) with ox > 0 or ox = 0 < oy,
// and the own column from the own cluster on -- in rounds of 32, one lane per
// column (x-y gap, z window, the j-cluster ranges of its z images), then the
// round's j-clusters flattened over the lanes for the box tests.  Entries
// are written in a fixed order to out[0 .. cap); returns how many there are
// (also when more than cap).
__device__ int col_gather(const PairArgs& p, int ic, int col_i, const float4& ilo, const float4& ihi,
                          const int4& Oi, float lim, int4* out, int cap, int4 (*s_part)[3], int* s_pre)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const ColGrid& g = p.cg;
    const double ux = g.lx * (1.0 / 4294967296.0), uy = g.ly * (1.0 / 4294967296.0), uz = g.lz * (1.0 / 4294967296.0);
    const int nyo = 2 * g.ry + 1;
    const int ncand = (g.rx + 1) * nyo;                  // ox = 0 .. rx
    const int cxi = col_i / g.ncy, cyi = col_i % g.ncy;
    int ne = 0;
    for (int k0 = 0; k0 < ncand; k0 += 32) {
        const int k = k0 + lane;
        int cnt = 0;
        int4 part[3];
#pragma unroll
        for (int z = 0; z < 3; ++z) part[z] = make_int4(0, 0, 0, 0);
        const int ox = k / nyo, oy = k % nyo - g.ry;
        if (k < ncand && (ox > 0 || oy >= 0)) {
            int jx = cxi + ox, jy = cyi + oy, tx = 0, ty = 0;
            if (jx >= g.ncx) { jx -= g.ncx; tx = 1; }
            if (jy < 0) { jy += g.ncy; ty = -1; } else if (jy >= g.ncy) { jy -= g.ncy; ty = 1; }
            const int colj = jx * g.ncy + jy;
            const float sx = tx * g.lxf, sy = ty * g.lyf;
            const float x0 = jx * g.sx + sx, y0 = jy * g.sy + sy;
            const float gx = fmaxf(0.f, fmaxf(x0 - ihi.x, ilo.x - (x0 + g.sx)));
            const float gy = fmaxf(0.f, fmaxf(y0 - ihi.y, ilo.y - (y0 + g.sy)));
            const float rem = lim - (gx * gx + gy * gy);
            if (rem >= 0.f) {
                const float wz = sqrtf(rem);
                const bool own = ox == 0 && oy == 0;
                const int jb = own ? 2 * ic : 2 * p.ccstart[colj];
                const int je = 2 * p.ccstart[colj + 1];
#pragma unroll
                for (int z = 0; z < 3; ++z) {
                    const int tz = z - 1;
                    const int2 r = col_zrange(p, colj, jb, je, ilo.z - wz, ihi.z + wz, tz * g.lzf);
                    part[z] = make_int4(r.x, r.y, col_entry_y(tx, ty, tz, false) | (own ? 1 << 7 : 0), 0);
                    cnt += r.y;
                }
            }
        }
#pragma unroll
        for (int z = 0; z < 3; ++z) s_part[lane][z] = part[z];
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        s_pre[lane + 1] = incl;
        if (lane == 0) s_pre[0] = 0;
        __syncwarp();
        const int total = __shfl_sync(FULL, incl, 31);
        for (int f0 = 0; f0 < total; f0 += 32) {
            const int f = f0 + lane;
            bool take = false;
            int4 ent = make_int4(0, 0, 0, 0);
            if (f < total) {
                int lo = 0, hi = 32;                      // owner lane: s_pre[o] <= f < s_pre[o + 1]
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (s_pre[mid] <= f) lo = mid; else hi = mid;
                }
                int u = f - s_pre[lo];
                int4 pt = s_part[lo][0];
                if (u >= pt.y) { u -= pt.y; pt = s_part[lo][1]; if (u >= pt.y) { u -= pt.y; pt = s_part[lo][2]; } }
                const int jc = pt.x + u;
                const int fl = pt.z & 0x3f;
                const float sx = ((fl & 3) - 1) * g.lxf, sy = (((fl >> 2) & 3) - 1) * g.lyf,
                            sz = (((fl >> 4) & 3) - 1) * g.lzf;
                const float4 jl = p.jbox[2 * jc], jh = p.jbox[2 * jc + 1];
                const float bx = fmaxf(0.f, fmaxf((jl.x + sx) - ihi.x, ilo.x - (jh.x + sx)));
                const float by = fmaxf(0.f, fmaxf((jl.y + sy) - ihi.y, ilo.y - (jh.y + sy)));
                const float bz = fmaxf(0.f, fmaxf((jl.z + sz) - ihi.z, ilo.z - (jh.z + sz)));
                take = bx * bx + by * by + bz * bz <= lim;
                if (take) {
                    // the tile's virial offset O_c(j) - O_c(i) + t L, exact in
                    // fixed point, then FP32 (a rounding of its own per tile)
                    const bool diag = (pt.z >> 7) && (jc >> 1) == ic;
                    const int4 Oj = p.corg[jc >> 1];
                    const long long qx = (long long)(unsigned)Oj.x - (long long)(unsigned)Oi.x +
                                         (long long)((fl & 3) - 1) * 4294967296LL;
                    const long long qy = (long long)(unsigned)Oj.y - (long long)(unsigned)Oi.y +
                                         (long long)(((fl >> 2) & 3) - 1) * 4294967296LL;
                    const long long qz = (long long)(unsigned)Oj.z - (long long)(unsigned)Oi.z +
                                         (long long)(((fl >> 4) & 3) - 1) * 4294967296LL;
                    ent = make_int4(jc | ((fl | (diag ? 1 << 6 : 0)) << 25), __float_as_int((float)((double)qx * ux)),
                                    __float_as_int((float)((double)qy * uy)), __float_as_int((float)((double)qz * uz)));
                }
            }
            const unsigned b = __ballot_sync(FULL, take);
            const int at = ne + __popc(b & ((1u << lane) - 1u));
            if (take && at < cap) out[at] = ent;
            ne += __popc(b);
        }
        __syncwarp();                                     // s_part / s_pre are rewritten next round
    }
    return ne;
}

__global__ void __launch_bounds__(128) k_col_list(PairArgs p)
{
    pdl_wait();
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __shared__ int4 s_ent[4][kColStageEntries];
    __shared__ int4 s_part[4][32][3];                    // per lane and z image: {first j, count, flags, 0}
    __shared__ int s_pre[4][33];
    const int ic = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    if (ic >= p.icl_cap) return;                                 // warp-uniform
    // a refused system leaves a mark in the list's need count, which a
    // reused list keeps (the status word starts at zero every evaluation)
    if (*p.status & kStatusColumns) {
        if (ic == 0 && lane == 0) atomicMax(p.plist_need, 1);
        return;
    }
    const ColGrid& g = p.cg;
    if (ic >= p.ccstart[g.ncol]) return;
    const int col_i = p.ccol[ic];
    const float4 ilo = p.ibox[2 * ic], ihi = p.ibox[2 * ic + 1];
    if (ihi.z - ilo.z > g.zext) {                                // a tile's image could be ambiguous
        if (lane == 0) { atomicOr(p.status, kStatusColumns); atomicMax(p.plist_need, 1); }
        return;
    }
    const int4 Oi = p.corg[ic];
    // a reused list holds the pairs within the cutoff plus the skin
    const float rl = sqrtf(p.cut2f) + p.list_skin;
    const float lim = rl * rl * (1.0f + 8.0f * p.guard) + 1e-3f;
    const int ne = col_gather(p, ic, col_i, ilo, ihi, Oi, lim, s_ent[w], kColStageEntries, s_part[w], s_pre[w]);
    if (ne == 0) return;
    const int nch = (ne + p.chunk - 1) / p.chunk;
    int b0 = 0, b1 = 0;
    if (lane == 0) {
        // the entries take two int2 places each of the list buffer (plist_cap
        // and plist_need count int2)
        b0 = atomicAdd(p.plist_count, ne);
        b1 = atomicAdd(p.chunk_count, nch);
        if (2 * (b0 + ne) > p.plist_cap) { atomicOr(p.status, kStatusListFull); atomicMax(p.plist_need, 2 * (b0 + ne)); }
        if (b1 + nch > p.chunk_cap) { atomicOr(p.status, kStatusListFull); atomicMax(p.chunk_need, b1 + nch); }
    }
    const int ebase = __shfl_sync(FULL, b0, 0), cbase = __shfl_sync(FULL, b1, 0);
    if (2 * (ebase + ne) > p.plist_cap || cbase + nch > p.chunk_cap) return;   // warp-uniform
    if (ne <= kColStageEntries) {
        for (int t = lane; t < ne; t += 32) p.clist[ebase + t] = s_ent[w][t];
    } else {                                              // more than the staging holds: list again, into place
        col_gather(p, ic, col_i, ilo, ihi, Oi, lim, p.clist + ebase, ne, s_part[w], s_pre[w]);
    }
    for (int t = lane; t < nch; t += 32)
        p.chunks[cbase + t] = make_int4(ic, 0, ebase + t * p.chunk, min(p.chunk, ne - t * p.chunk));
}

// geometry and the FP32 within-cutoff decision of one pair of the 8 x 4 tile
template <int NT, int S0, int S1>
__device__ __forceinline__ PairGeo col_geo(const PairArgs& p, const int4& pi, const int4& pj, bool valid,
                                           int mol_i, int mol_j)
{
    PairGeo g;
    const float g_lo = 1.0f - p.guard, g_hi = 1.0f + p.guard;
    const float t0c2 = p.tf[0].cut2, t1c2 = NT > 1 ? p.tf[1].cut2 : 0.f;
    // minimal image in fixed point, exact; one rounding to FP32, then the
    // compensated unit L / 2^32
    const float qx = (float)(int)((unsigned)pj.x - (unsigned)pi.x);
    const float qy = (float)(int)((unsigned)pj.y - (unsigned)pi.y);
    const float qz = (float)(int)((unsigned)pj.z - (unsigned)pi.z);
    const float dx = fmaf(qx, p.cg.sch[0], qx * p.cg.scl[0]);
    const float dy = fmaf(qy, p.cg.sch[1], qy * p.cg.scl[1]);
    const float dz = fmaf(qz, p.cg.sch[2], qz * p.cg.scl[2]);
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const bool far = r2 > p.cut2f * g_hi;
    bool near = !far && r2 >= p.cut2f * g_lo;
    if (S0 == SCUT && t0c2 != p.cut2f) near |= (r2 >= t0c2 * g_lo && r2 <= t0c2 * g_hi);
    if (NT > 1 && S1 == SCUT && t1c2 != p.cut2f) near |= (r2 >= t1c2 * g_lo && r2 <= t1c2 * g_hi);
    g.near = near && valid;
    g.in0 = r2 <= t0c2;
    g.in1 = NT > 1 ? r2 <= t1c2 : false;
    g.act = valid && !far;
    g.same = mol_i == mol_j;
    g.excl = PMGPU_EXCL_NONE;
    g.dx = dx; g.dy = dy; g.dz = dz; g.r2 = r2;
    return g;
}

// the tile of one list entry, decoded, with its j-atom for this lane
struct ColTile {
    int jc;                      // j-cluster
    bool diag;
    float ox, oy, oz;            // virial offset
    int4 P, M;                   // j-atom: fixed-point position + charge hi; original index, type, molecule, charge lo
};

// the tile of entry c (has: the entry exists), with its j-atom for lane jj
__device__ __forceinline__ void col_tile_of(const PairArgs& p, const int4& c, bool has, int jj, ColTile& t)
{
    t.jc = c.x & 0x1ffffff;
    t.diag = has && (((unsigned)c.x >> 31) & 1u);
    t.ox = __int_as_float(c.y); t.oy = __int_as_float(c.z); t.oz = __int_as_float(c.w);
    if (has) {                                   // read-only during the pair kernel
        t.P = __ldg(p.cq + 4 * (size_t)t.jc + jj);
        t.M = __ldg(p.cm + 4 * (size_t)t.jc + jj);
    } else {
        t.P = make_int4(0, 0, 0, 0);
        t.M = make_int4(-1, 0, -2, 0);
    }
}

template <bool SH>
__device__ __forceinline__ int4 col_entry(const int4* ents, int e, int e_end)
{
    if (e >= e_end) return make_int4(0, 0, 0, 0);
    return SH ? ents[e] : __ldg(ents + e);
}

__device__ __forceinline__ JAtom col_atom(const int4& P, const int4& M)
{
    JAtom a;
    a.p = make_float4(0.f, 0.f, 0.f, __int_as_float(P.w));
    a.l = make_float4(0.f, 0.f, 0.f, __int_as_float(M.w));
    a.m = make_int4(M.x, M.y, M.z, 0);
    return a;
}

// One i-cluster's run of list entries [e_begin, e_end) of ents (the global
// list, or entries in shared memory: SH), two tiles per iteration: the tile
// loop of K2b'.  Adds the j-forces and, at the end, the i-forces; queues the
// near pairs (flushed at the end) and adds the run's energies and tile virial
// to the lane's int64 sums acc.
template <bool SH, int NT, int P0, int S0, int P1, int S1>
__device__ __forceinline__ void col_run(const PairArgs& p, int ic, const int4* ents, int e_begin, int e_end,
                                        int2* s_near, long long (&acc)[5], bool& bad)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, il = lane & 7, jj = lane >> 3;
    // after the reduce-scatter lane il (< 6) holds component il % 3 of the
    // j-force of tile A's (il < 3) or tile B's (il >= 3) j-atom jj
    const bool holds = il < 6, onB = il >= 3;
    const int comp = il < 3 ? il : il - 3;
    const int si = 8 * ic + il;
    const int4 Pi = p.cq[si], Mi = p.cm[si];
    const JAtom ia = col_atom(Pi, Mi);
    const bool vi = Mi.x >= 0;
    float fix = 0.f, fiy = 0.f, fiz = 0.f;
    double el = 0.0, ec = 0.0;
    // the far pairs' FP32 energies summed over up to kEnergyFlush
    // iterations in FP32, then into the FP64 sums
    float elf = 0.f, ecf = 0.f;
    int nacc = 0;
    double wv[3] = {0.0, 0.0, 0.0};
    int nq = 0;
    // software pipeline: the entries two iterations ahead, the j-atoms of
    // the next iteration's tiles one ahead
    ColTile nA, nB;
    col_tile_of(p, col_entry<SH>(ents, e_begin, e_end), true, jj, nA);
    col_tile_of(p, col_entry<SH>(ents, e_begin + 1, e_end), e_begin + 1 < e_end, jj, nB);
    int4 qA = col_entry<SH>(ents, e_begin + 2, e_end), qB = col_entry<SH>(ents, e_begin + 3, e_end);
    for (int e = e_begin; e < e_end; e += 2) {
        if (nq > kNearCap - 64) {                  // room for one more pair of tiles
            append_near(p, s_near, nq, lane);
            nq = 0;
        }
        const ColTile tA = nA, tB = nB;
        const bool hasB = e + 1 < e_end;           // warp-uniform
        if (e + 2 < e_end) {
            col_tile_of(p, qA, true, jj, nA);
            col_tile_of(p, qB, e + 3 < e_end, jj, nB);
            qA = col_entry<SH>(ents, e + 4, e_end);
            qB = col_entry<SH>(ents, e + 5, e_end);
        }
        const JAtom ja = col_atom(tA.P, tA.M), jb = col_atom(tB.P, tB.M);
        const bool va = vi && ja.m.x >= 0 && (!tA.diag || 4 * (tA.jc & 1) + jj > il);
        const bool vb = hasB && vi && jb.m.x >= 0 && (!tB.diag || 4 * (tB.jc & 1) + jj > il);
        PairGeo ga = col_geo<NT, S0, S1>(p, Pi, tA.P, va, ia.m.z, ja.m.z);
        PairGeo gb = col_geo<NT, S0, S1>(p, Pi, tB.P, vb, ia.m.z, jb.m.z);
        if (__any_sync(FULL, is_rare(ga) || is_rare(gb))) {   // warp-uniform, rare
            resolve_rare<NT>(p, ga, ia, ja);
            resolve_rare<NT>(p, gb, ia, jb);
        }
        const bool any_a = __any_sync(FULL, ga.act), any_b = __any_sync(FULL, gb.act);
        if (!(any_a || any_b)) continue;
        float fta = 0.f, ela = 0.f, eca = 0.f, ftb = 0.f, elb = 0.f, ecb = 0.f;
        if (any_a && any_b) {
            pair_math<NT, P0, S0, P1, S1>(p, ga, ia, ja, fta, ela, eca);
            pair_math<NT, P0, S0, P1, S1>(p, gb, ia, jb, ftb, elb, ecb);
        } else {
            float ft, e1, e2;
            pair_math<NT, P0, S0, P1, S1>(p, any_a ? ga : gb, ia, any_a ? ja : jb, ft, e1, e2);
            if (any_a) { fta = ft; ela = e1; eca = e2; } else { ftb = ft; elb = e1; ecb = e2; }
        }
        const float xa = ga.dx * fta, ya = ga.dy * fta, za = ga.dz * fta;
        const float xb = gb.dx * ftb, yb = gb.dy * ftb, zb = gb.dz * ftb;
        fix -= xa + xb; fiy -= ya + yb; fiz -= za + zb;
        // near pairs: queued (original indices) for FP64 energies in place of the FP32 ones
        {
            const bool na = ga.act && ga.r2 < p.near2, nb = gb.act && gb.r2 < p.near2;   // near2 = 0: none
            if (__any_sync(FULL, na || nb)) {
                const unsigned ba = __ballot_sync(FULL, na), bb = __ballot_sync(FULL, nb);
                const unsigned lt = (1u << lane) - 1u;
                if (na) {
                    s_near[nq + __popc(ba & lt)] =
                        make_int2(ia.m.x, ja.m.x | (ga.excl == PMGPU_EXCL_MODIFIED ? 1 << 30 : 0));
                    ela = 0.f; eca = 0.f;
                }
                nq += __popc(ba);
                if (nb) {
                    s_near[nq + __popc(bb & lt)] =
                        make_int2(ia.m.x, jb.m.x | (gb.excl == PMGPU_EXCL_MODIFIED ? 1 << 30 : 0));
                    elb = 0.f; ecb = 0.f;
                }
                nq += __popc(bb);
            }
        }
        elf += ela + elb;
        ecf += eca + ecb;
        if (++nacc == kEnergyFlush) {
            el += (double)elf;
            ec += (double)ecf;
            elf = 0.f; ecf = 0.f; nacc = 0;
        }
        // j-forces of both tiles: lane il < 6 ends with one component
        const float v = j_reduce_scatter(xa, ya, za, xb, yb, zb, il);
        if (holds && v != 0.f)
            fixed_addf(p.facc + 3 * (4 * (size_t)(onB ? tB.jc : tA.jc) + jj) + comp, v, p.status);
        if (p.virial && holds) {                       // o (x) F_tile, column comp
            const float ox = onB ? tB.ox : tA.ox, oy = onB ? tB.oy : tA.oy, oz = onB ? tB.oz : tA.oz;
            wv[0] += (double)(ox * v);
            wv[1] += (double)(oy * v);
            wv[2] += (double)(oz * v);
        }
        if (p.rec_pairs) {                             // diagnostic pair recording
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const PairGeo& g = t ? gb : ga;
                const JAtom& j = t ? jb : ja;
                if (g.act) {
                    const unsigned long long r = atomicAdd(p.rec_count, 1ull);
                    if ((long long)r < p.rec_cap) {
                        p.rec_pairs[2 * r] = min(ia.m.x, j.m.x);
                        p.rec_pairs[2 * r + 1] = max(ia.m.x, j.m.x);
                    }
                }
            }
        }
    }
    el += (double)elf;
    ec += (double)ecf;
    // chunk end: i-forces (lanes jj = 0, 1, 2 hold component jj of i-atom il)
    const float vi3 = i_reduce_scatter(fix, fiy, fiz, jj);
    if (jj < 3 && vi && vi3 != 0.f) fixed_addf(p.facc + 3 * (size_t)si + jj, vi3, p.status);
    if (nq > 0) append_near(p, s_near, nq, lane);
    acc[0] += fixed_of(el, bad);
    acc[1] += fixed_of(ec, bad);
    if (p.virial) {
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[2 + a] += fixed_of(wv[a], bad);
    }
    __syncwarp();
}

// Two 8 x 4 tiles (consecutive entries A and B of the chunk) per iteration:
// two independent pair evaluations per lane interleave, and the per-tile
// work -- votes, the j-force reduce-scatter of both tiles in one (7 shuffles
// for 6 values), the fixed-point adds, the virial offsets, the energy sums --
// is shared by the two.
template <int NT, int P0, int S0, int P1, int S1>
__global__ void __launch_bounds__(128, 5) k_pair_col(PairArgs p)
{
    pdl_wait();
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, il = lane & 7, jj = lane >> 3;
    __shared__ int2 s_near[4][kNearCap];
    __shared__ unsigned long long s_e[kERec];
    if (threadIdx.x < kERec) s_e[threadIdx.x] = 0ull;
    __syncthreads();
    // per-lane int64 sums over the chunks: LJ, Coulomb, and the tile-offset
    // virial W[0..2][comp] of the lanes that hold a j-force component
    long long acc[5] = {0, 0, 0, 0, 0};
    bool bad = false;
    // an incomplete list (capacity exceeded or the system refused, also when
    // it was built by an earlier evaluation and is reused) runs no pair
    const bool list_bad = (*p.status & (kStatusListFull | kStatusColumns)) || *p.plist_need != 0 || *p.chunk_need != 0;
    if (list_bad && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(p.status, kStatusListFull);
    const int nchunks = list_bad ? 0 : min(*p.chunk_count, p.chunk_cap);
    // lane il (< 6) holds component il % 3 of a j-force (col_run)
    const bool holds = il < 6;
    const int comp = il < 3 ? il : il - 3;
    while (true) {
        int ch = 0;
        if (lane == 0) ch = atomicAdd(p.chunk_next, 1);
        ch = __shfl_sync(FULL, ch, 0);
        if (ch >= nchunks) break;
        const int4 cd = p.chunks[ch];
        col_run<false, NT, P0, S0, P1, S1>(p, cd.x, p.clist, cd.z, cd.z + cd.w, s_near[w], acc, bad);
    }
    if (bad) atomicOr(p.status, kStatusOverflow);
#pragma unroll
    for (int t = 0; t < 2; ++t)
        for (int o = 16; o > 0; o >>= 1) acc[t] += __shfl_xor_sync(FULL, acc[t], o);
    if (lane == 0) {
        atomicAdd(&s_e[0], (unsigned long long)acc[0]);
        atomicAdd(&s_e[1], (unsigned long long)acc[1]);
    }
    if (p.virial) {
        // W[a][comp]: sum over the four j-atom groups (xor 8, 16; lanes that
        // hold no component carry zeros), then lanes 0-5 of the first group
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            acc[2 + a] += __shfl_xor_sync(FULL, acc[2 + a], 8);
            acc[2 + a] += __shfl_xor_sync(FULL, acc[2 + a], 16);
        }
        if (holds && jj == 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a) atomicAdd(&s_e[2 + 3 * a + comp], (unsigned long long)acc[2 + a]);
        }
    }
    __syncthreads();
    if (threadIdx.x < kERec && s_e[threadIdx.x] != 0ull) atomicAdd(p.efix + threadIdx.x, s_e[threadIdx.x]);
}

// The lanes' int64 sums (acc) of one system into its energy words, at once
// (the batch kernel: the warp leaves the system)
__device__ __forceinline__ void col_warp_sums(const PairArgs& p, long long (&acc)[5], bool& bad)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, il = lane & 7, jj = lane >> 3;
    const int comp = il < 3 ? il : il - 3;
    if (bad && lane == 0) atomicOr(p.status, kStatusOverflow);
    bad = __any_sync(FULL, bad) && false;
#pragma unroll
    for (int t = 0; t < 2; ++t)
        for (int o = 16; o > 0; o >>= 1) acc[t] += __shfl_xor_sync(FULL, acc[t], o);
    if (lane == 0) {
        if (acc[0] != 0) atomicAdd(p.efix + 0, (unsigned long long)acc[0]);
        if (acc[1] != 0) atomicAdd(p.efix + 1, (unsigned long long)acc[1]);
    }
    if (p.virial) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            acc[2 + a] += __shfl_xor_sync(FULL, acc[2 + a], 8);
            acc[2 + a] += __shfl_xor_sync(FULL, acc[2 + a], 16);
        }
        if (il < 6 && jj == 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
                if (acc[2 + a] != 0) atomicAdd(p.efix + 2 + 3 * a + comp, (unsigned long long)acc[2 + a]);
        }
    }
#pragma unroll
    for (int t = 0; t < 5; ++t) acc[t] = 0;
}

// K11: the column-path pair kernels of a batch's members as one persistent
// launch over (member, chunk) work items.  Every member's list was built by
// its own K2a' launch before this one.  Each block prefix-sums the members'
// chunk counts in shared memory (a member whose list is incomplete counts
// none and is marked as K2b' marks it); a warp takes items from one counter,
// copies its member's arguments into shared memory when the member changes,
// runs the chunk (col_run, the K2b' tile loop) and adds its sums to the
// member's energy words when it leaves the member.  Nothing waits on
// another launch: the graph orders this one after every member's list.
template <int NT, int P0, int S0, int P1, int S1>
__global__ void __launch_bounds__(128, 4) k_pair_col_batch(BatchPairArgs b)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __shared__ int2 s_near[4][kNearCap];
    __shared__ int s_pre[kBatchPairMax + 1];
    __shared__ PairArgs s_args[4];
    if (threadIdx.x == 0) {
        int t = 0;
        for (int m = 0; m < b.n; ++m) {
            const PairArgs& p = b.args[m];
            s_pre[m] = t;
            const bool list_bad = (*p.status & (kStatusListFull | kStatusColumns)) || *p.plist_need != 0 ||
                                  *p.chunk_need != 0;
            if (list_bad && blockIdx.x == 0) atomicOr(p.status, kStatusListFull);
            t += list_bad ? 0 : min(*p.chunk_count, p.chunk_cap);
        }
        s_pre[b.n] = t;
    }
    __syncthreads();
    const int total = s_pre[b.n];
    long long acc[5] = {0, 0, 0, 0, 0};
    bool bad = false;
    int cur = -1;
    const PairArgs& p = s_args[w];
    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(b.next, 1);
        item = __shfl_sync(FULL, item, 0);
        if (item >= total) break;
        int lo = 0, hi = b.n;                         // the member: s_pre[lo] <= item < s_pre[lo + 1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_pre[mid] <= item) lo = mid; else hi = mid;
        }
        if (lo != cur) {
            if (cur >= 0) col_warp_sums(p, acc, bad);
            __syncwarp();
            const int* src = reinterpret_cast<const int*>(b.args + lo);
            int* dst = reinterpret_cast<int*>(&s_args[w]);
            for (int i = lane; i < (int)(sizeof(PairArgs) / sizeof(int)); i += 32) dst[i] = src[i];
            __syncwarp();
            cur = lo;
        }
        const int4 cd = p.chunks[item - s_pre[lo]];
        col_run<false, NT, P0, S0, P1, S1>(p, cd.x, p.clist, cd.z, cd.z + cd.w, s_near[w], acc, bad);
    }
    if (cur >= 0) col_warp_sums(p, acc, bad);
}

// FP64 energies of one pair of atoms by original index: the FP64 kernel's
// arithmetic (pot_f64, sw_f64) on the raw positions and the exact minimal
// image
template <int NT, int P0, int S0, int P1, int S1>
__device__ __forceinline__ void pair_energy_f64_orig(const PairArgs& p, int oi, int oj, int excl, double& el,
                                                     double& ec)
{
    constexpr bool kMod = sw_modifies(S0) || (NT > 1 && sw_modifies(S1));
    const double* pi = p.pos + 3 * (size_t)oi;
    const double* pj = p.pos + 3 * (size_t)oj;
    double dx, dy, dz;
    const double d2 = pbc_min_diff(p.pbc, pi[0], pi[1], pi[2], pj[0], pj[1], pj[2], dx, dy, dz);
    const double rd2 = 1.0 / d2;
    const double qi = p.qorig[oi], qj = p.qorig[oj];
    const int ti = p.torig[oi], tj = p.torig[oj];
    double e0, f0, e1 = 0.0, f1 = 0.0;
    pot_f64<P0>(p, p.td[0], d2, rd2, qi, qj, ti, tj, excl, e0, f0);
    if (NT > 1) pot_f64<P1>(p, p.td[1], d2, rd2, qi, qj, ti, tj, excl, e1, f1);
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

// K2c': the FP64 energies of the near pairs K2b' listed (original indices),
// each rounded to int64 fixed point on its own
template <int NT, int P0, int S0, int P1, int S1>
__global__ void __launch_bounds__(128) k_near_energy_col(PairArgs p)
{
    const unsigned FULL = 0xffffffffu;
    __shared__ long long s_acc[2][4];
    if (*p.status & (kStatusListFull | kStatusColumns)) return;   // block-uniform
    const int n = min(*p.near_count, p.near_cap);
    long long al = 0, ac = 0;
    bool bad = false;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int2 e = p.near[k];
        double el = 0.0, ec = 0.0;
        pair_energy_f64_orig<NT, P0, S0, P1, S1>(p, e.x, e.y & 0x3fffffff,
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
        const long long t = s_acc[threadIdx.x][0] + s_acc[threadIdx.x][1] + s_acc[threadIdx.x][2] + s_acc[threadIdx.x][3];
        if (t != 0) atomicAdd(p.efix + threadIdx.x, (unsigned long long)t);
    }
}
