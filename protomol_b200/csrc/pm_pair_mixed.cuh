// pm_pair_mixed.cuh -- K2: mixed-precision cell-pair force kernel on 8x8
// cluster tiles (included by pm_pair.cu, which provides the helpers).
//
// Clusters: inside a reference cell the atoms are ordered by the Morton key of
// their position on an 8x8x8 sub-grid of the cell (k_bin_finish), so every run
// of 8 consecutive atoms is a compact cluster with a bounding box
// (k_cluster_box).
//
// Work item = (cell A, batch of 8 deltas of the half shell), one warp.  The
// half shell is the positive half of the reference's delta list, which covers
// every unordered pair of cells exactly once and gives every cell the same
// work (in the small-grid mode, where a periodic image can occur twice among
// the deltas, it is the reference's list with its B > A rule); batch 0 also
// holds the cell A with itself.  The interacting pair set is the reference's
// in both cases: only the order in which a pair's two atoms are visited
// differs, and forces are accumulated in order-independent fixed point.
//
// The warp stages A's atoms (up to 32 = 4 clusters at a time) in shared
// memory.  For every cell B of the batch and every j-cluster of B it loads the
// j-cluster once (lane l holds j-atom l / 8, then l / 8 + 4), tests the
// j-cluster box against the 4 i-cluster boxes and runs the surviving 8x8
// tiles: lane l pairs i-atom l % 8 of an i-cluster with its j-atom.  So one
// j-cluster load serves up to four tiles, i-forces stay in registers for the
// whole item (4 clusters x 3), j-forces are summed over the 8 lanes of a j
// once per j-cluster step.  Forces are rounded to int64 fixed point once per
// atom and item / j-cluster and added with integer atomics.

constexpr int kBatch = 8;    // deltas per work item

template <int NT, int P0, int S0, int P1, int S1>
__device__ __forceinline__ void pair_f32(const PairArgs& p, const float4& pi, const float4& li, const int4& mi,
                                         const float4& pj, const float4& lj, const int4& mj,
                                         float ox, float oy, float oz, float olx, float oly, float olz,
                                         float& fx, float& fy, float& fz, double& el, double& ec,
                                         float (&vir)[6])
{
    constexpr bool kMod = sw_modifies(S0) || (NT > 1 && sw_modifies(S1));
    constexpr bool kUse = S0 != SUN || (NT > 1 && S1 != SUN);
    const float g_lo = 1.0f - p.guard, g_hi = 1.0f + p.guard;
    const float t0c2 = p.tf[0].cut2, t1c2 = NT > 1 ? p.tf[1].cut2 : 0.f;
    // every rounding depends on both atoms; the lo parts restore the
    // coordinates and the cell offset to ~2^-48
    float dx = ((pj.x - pi.x) + ox) + ((lj.x - li.x) + olx);
    float dy = ((pj.y - pi.y) + oy) + ((lj.y - li.y) + oly);
    float dz = ((pj.z - pi.z) + oz) + ((lj.z - li.z) + olz);
    if (p.wrap) {
        float kx = rintf(dx * p.ilx), ky = rintf(dy * p.ily), kz = rintf(dz * p.ilz);
        dx = fmaf(-p.lx, kx, fmaf(-p.lx_lo, kx, dx));
        dy = fmaf(-p.ly, ky, fmaf(-p.ly_lo, ky, dy));
        dz = fmaf(-p.lz, kz, fmaf(-p.lz_lo, kz, dz));
    }
    float r2 = dx * dx + dy * dy + dz * dz;
    if (kUse && r2 > p.cut2f * g_hi) return;                // far outside: the common case
    bool near = r2 >= p.cut2f * g_lo;
    if (S0 == SCUT && t0c2 != p.cut2f) near |= (r2 >= t0c2 * g_lo && r2 <= t0c2 * g_hi);
    if (NT > 1 && S1 == SCUT && t1c2 != p.cut2f) near |= (r2 >= t1c2 * g_lo && r2 <= t1c2 * g_hi);
    bool in_pair, in0, in1;
    if (near) {
        double d2 = exact_d2(p, mi.x, mj.x);
        in_pair = !(d2 > p.cut2d);
        in0 = !(d2 > p.td[0].cut2);
        in1 = NT > 1 ? !(d2 > p.td[1].cut2) : false;
    } else {
        in_pair = true;
        in0 = !(r2 > t0c2);
        in1 = NT > 1 ? !(r2 > t1c2) : false;
    }
    if (kUse && !in_pair) return;
    int excl = PMGPU_EXCL_NONE;
    if (mi.z == mj.z) {
        excl = excl_class(p, mi.x, mj.x);
        if (excl == PMGPU_EXCL_FULL) return;
    }
    float rinv = __frsqrt_rn(r2);            // correctly rounded: unbiased
    float rd2 = rinv * rinv;
    float qq = fmaf(pi.w, pj.w, fmaf(pi.w, lj.w, li.w * pj.w));
    float e0, f0, e1 = 0.f, f1 = 0.f;
    pot_f32<P0>(p, p.tf[0], r2, rd2, rinv, qq, mi.y, mj.y, excl, e0, f0);
    if (NT > 1) pot_f32<P1>(p, p.tf[1], r2, rd2, rinv, qq, mi.y, mj.y, excl, e1, f1);
    if (kMod) {
        float sv, sd;
        sw_f32<S0>(p.tf[0], r2, rinv, in0, sv, sd);
        f0 = f0 * sv - e0 * sd;
        e0 = e0 * sv;
        if (NT > 1) {
            sw_f32<S1>(p.tf[1], r2, rinv, in1, sv, sd);
            f1 = f1 * sv - e1 * sd;
            e1 = e1 * sv;
        }
    }
    if (P0 == LJ) el += (double)e0; else ec += (double)e0;
    if (NT > 1) { if (P1 == LJ) el += (double)e1; else ec += (double)e1; }
    float ft = NT > 1 ? f0 + f1 : f0;
    fx = dx * ft; fy = dy * ft; fz = dz * ft;
    if (p.virial) {
        vir[0] = fmaf(fx, dx, vir[0]); vir[1] = fmaf(fx, dy, vir[1]); vir[2] = fmaf(fx, dz, vir[2]);
        vir[3] = fmaf(fy, dy, vir[3]); vir[4] = fmaf(fy, dz, vir[4]); vir[5] = fmaf(fz, dz, vir[5]);
    }
    if (p.rec_pairs) {
        unsigned long long k = atomicAdd(p.rec_count, 1ull);
        if ((long long)k < p.rec_cap) {
            p.rec_pairs[2 * k] = min(mi.x, mj.x);
            p.rec_pairs[2 * k + 1] = max(mi.x, mj.x);
        }
    }
}

__device__ __forceinline__ bool box_near(const float4& ilo, const float4& ihi, const float4& jlo, const float4& jhi,
                                         float ox, float oy, float oz, float lim)
{
    float bx = fmaxf(0.f, fmaxf((jlo.x + ox) - ihi.x, ilo.x - (jhi.x + ox)));
    float by = fmaxf(0.f, fmaxf((jlo.y + oy) - ihi.y, ilo.y - (jhi.y + oy)));
    float bz = fmaxf(0.f, fmaxf((jlo.z + oz) - ihi.z, ilo.z - (jhi.z + oz)));
    return bx * bx + by * by + bz * bz <= lim;
}

template <int NT, int P0, int S0, int P1, int S1>
__global__ void __launch_bounds__(128, 5) k_pair_mixed(PairArgs p)
{
    __shared__ float4 sip[4][32];
    __shared__ float4 sil[4][32];
    __shared__ int4 sim[4][32];
    __shared__ float4 sib[4][8];
    __shared__ double wvir[4][6];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int il = lane & 7, jg = lane >> 3;
    const int warps_total = gridDim.x * 4;
    const CellGrid& cg = p.grid;
    const int nbatch = (p.nh + 1 + kBatch - 1) / kBatch;   // slot 0: the cell itself
    const int n_items = cg.ncell * nbatch;
    // tiles farther apart than this (FP32 box distance^2) hold no pair
    const float box_lim = p.cut2f * (1.0f + 8.0f * p.guard) + 1e-3f;
    if (lane < 6) wvir[w][lane] = 0.0;
    __syncwarp();
    double el = 0.0, ec = 0.0;

    for (int item = blockIdx.x * 4 + w; item < n_items; item += warps_total) {
        const int A = item / nbatch;
        const int batch = item - A * nbatch;
        const int sa = p.start[A], ea = p.start[A + 1];
        if (sa == ea) continue;
        const int ca0 = p.cstart[A];
        const int nca = p.cstart[A + 1] - ca0;
        const int ax = A / (cg.ny * cg.nz), ay = (A / cg.nz) % cg.ny, az = A % cg.nz;
        // A's clusters in chunks of 4 (32 atoms)
        for (int c0 = 0; c0 < nca; c0 += 4) {
            const int ncc = min(4, nca - c0);
            {
                int s = sa + c0 * kCluster + lane;
                bool v = s < ea && lane < ncc * kCluster;
                sip[w][lane] = v ? p.spos[s] : make_float4(0.f, 0.f, 0.f, 0.f);
                sil[w][lane] = v ? p.slo[s] : make_float4(0.f, 0.f, 0.f, 0.f);
                sim[w][lane] = v ? p.smeta[s] : make_int4(-1, 0, -2, 0);
                if (lane < 2 * ncc) sib[w][lane] = p.cbox[2 * (ca0 + c0) + lane];
            }
            __syncwarp();
            float fi[4][3];
#pragma unroll
            for (int c = 0; c < 4; ++c) fi[c][0] = fi[c][1] = fi[c][2] = 0.f;
            float vir[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            // the cells of this batch (k = -1: A itself)
            for (int kk = 0; kk < kBatch; ++kk) {
                const int k = batch * kBatch + kk - 1;
                if (k >= p.nh) break;
                int B = A;
                float ox = 0.f, oy = 0.f, oz = 0.f, olx = 0.f, oly = 0.f, olz = 0.f;
                if (k >= 0) {
                    int4 d = p.hdeltas[k];
                    int bx = ((ax + d.x) % cg.nx + cg.nx) % cg.nx;
                    int by = ((ay + d.y) % cg.ny + cg.ny) % cg.ny;
                    int bz = ((az + d.z) % cg.nz + cg.nz) % cg.nz;
                    B = (bx * cg.ny + by) * cg.nz + bz;
                    if (p.half_rule && B <= A) continue;
                    float4 o = p.hoff[k], ol = p.hoff_lo[k];
                    ox = o.x; oy = o.y; oz = o.z; olx = ol.x; oly = ol.y; olz = ol.z;
                }
                const bool self = k < 0;
                const int sb = p.start[B], eb = p.start[B + 1];
                const int cb0 = p.cstart[B];
                const int ncb = p.cstart[B + 1] - cb0;
                for (int jc = self ? c0 : 0; jc < ncb; ++jc) {
                    const float4 jlo = p.cbox[2 * (cb0 + jc)], jhi = p.cbox[2 * (cb0 + jc) + 1];
                    unsigned imask = 0u;
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (c < ncc && (!self || jc >= c0 + c) &&
                            (p.wrap || box_near(sib[w][2 * c], sib[w][2 * c + 1], jlo, jhi, ox, oy, oz, box_lim)))
                            imask |= 1u << c;
                    if (!imask) continue;
                    const int jbase = sb + jc * kCluster;
                    const int nj = min(kCluster, eb - jbase);
#pragma unroll
                    for (int step = 0; step < 2; ++step) {
                        const int jl = jg + 4 * step;
                        const int jslot = jbase + jl;
                        const bool vj = jl < nj;
                        float4 pj = make_float4(0.f, 0.f, 0.f, 0.f), lj = pj;
                        int4 mj = make_int4(-1, 0, -3, 0);
                        if (vj) { pj = p.spos[jslot]; lj = p.slo[jslot]; mj = p.smeta[jslot]; }
                        float fjx = 0.f, fjy = 0.f, fjz = 0.f;
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            if (!(imask & (1u << c))) continue;
                            const int islot = sa + (c0 + c) * kCluster + il;
                            const bool ok = vj && islot < ea && sim[w][c * kCluster + il].x >= 0 &&
                                            (!(self && jc == c0 + c) || jslot > islot);
                            if (!ok) continue;
                            float fx = 0.f, fy = 0.f, fz = 0.f;
                            pair_f32<NT, P0, S0, P1, S1>(p, sip[w][c * kCluster + il], sil[w][c * kCluster + il],
                                                         sim[w][c * kCluster + il], pj, lj, mj, ox, oy, oz,
                                                         olx, oly, olz, fx, fy, fz, el, ec, vir);
                            fi[c][0] -= fx; fi[c][1] -= fy; fi[c][2] -= fz;
                            fjx += fx; fjy += fy; fjz += fz;
                        }
                        // j-force: sum over the 8 lanes of this j (lanes 8 jg .. 8 jg + 7)
#pragma unroll
                        for (int o = 1; o < 8; o <<= 1) {
                            fjx += __shfl_xor_sync(0xffffffffu, fjx, o);
                            fjy += __shfl_xor_sync(0xffffffffu, fjy, o);
                            fjz += __shfl_xor_sync(0xffffffffu, fjz, o);
                        }
                        if (il == 0 && vj && (fjx != 0.f || fjy != 0.f || fjz != 0.f))
                            fixed_add3(p.facc + 3 * (size_t)jslot, fjx, fjy, fjz, p.scale, p.status);
                    }
                }
            }
            // i-forces: sum over the 4 lanes of an i (lanes il, il + 8, il + 16, il + 24)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
#pragma unroll
                for (int o = 8; o < 32; o <<= 1) {
                    fi[c][0] += __shfl_xor_sync(0xffffffffu, fi[c][0], o);
                    fi[c][1] += __shfl_xor_sync(0xffffffffu, fi[c][1], o);
                    fi[c][2] += __shfl_xor_sync(0xffffffffu, fi[c][2], o);
                }
                const int islot = sa + (c0 + c) * kCluster + il;
                if (lane < 8 && c < ncc && islot < ea && (fi[c][0] != 0.f || fi[c][1] != 0.f || fi[c][2] != 0.f))
                    fixed_add3(p.facc + 3 * (size_t)islot, fi[c][0], fi[c][1], fi[c][2], p.scale, p.status);
            }
            if (p.virial) {
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    float v = vir[c];
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    if (lane == 0) wvir[w][c] += (double)v;
                }
            }
            __syncwarp();
        }
    }
    __syncwarp();
    double acc[kERec];
    acc[0] = el; acc[1] = ec;
    acc[2] = lane == 0 ? wvir[w][0] : 0.0; acc[3] = lane == 0 ? wvir[w][1] : 0.0;
    acc[4] = lane == 0 ? wvir[w][2] : 0.0; acc[6] = lane == 0 ? wvir[w][3] : 0.0;
    acc[7] = lane == 0 ? wvir[w][4] : 0.0; acc[10] = lane == 0 ? wvir[w][5] : 0.0;
    acc[5] = acc[3]; acc[8] = acc[4]; acc[9] = acc[7];
    warp_reduce_store(acc, p.erec, p.erec_stride, blockIdx.x * 4 + w);
}
