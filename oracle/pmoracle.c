/*
 * pmoracle.c -- CPU restatement of ProtoMol 2.1's nonbonded force path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker; see pmoracle.h).
 *
 * Parity is pinned against the reference itself: oracle/ref builds the
 * reference's own NonbondedCutoffSystemForce / NonbondedPMEwaldSystemForce
 * from its sources into oracle/_ref, and the tests compare this file's output
 * with it (bit-exact for the cell assignment and pair set, <= 1e-12 relative
 * for forces, energies and virial; the FFT differs from the reference's
 * vendored ZFFT only by rounding).
 *
 * Build: gcc -O2 -ffp-contract=off -fPIC -shared pmoracle.c -lm
 */
#include "pmoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>

/* base/pmconstants.cpp */
#define PMO_EPSILON 1.0e-14
#define PMO_PI 3.14159265358979323846
#define PMO_MAX_INT_2 (INT_MAX / 2)

/* ------------------------------------------------------------------ vectors */
typedef struct { double x, y, z; } v3;

static v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 vadd(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vsub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vmul(v3 a, double w) { return mk(a.x * w, a.y * w, a.z * w); }
static v3 vdiv(v3 a, double w) { return mk(a.x / w, a.y / w, a.z / w); }
static double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double vnorm2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
/* Vector3D::operator^ (base/Vector3D.h:103-106) */
static v3 vcross(v3 a, v3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static v3 vload(const double* p) { return mk(p[0], p[1], p[2]); }

/* ------------------------------------------- PeriodicBoundaryConditions */
typedef struct {
    v3 e1, e2, e3, origin, e1r, e2r, e3r, min, max, H, H2;
    double D, V;
    int orth;
} pbc_t;

/* PeriodicBoundaryConditions::set (topology/PeriodicBoundaryConditions.cpp:40-77) */
static void pbc_set(pbc_t* b, const double* box)
{
    v3 e1 = vload(box), e2 = vload(box + 3), e3 = vload(box + 6), o = vload(box + 9);
    b->e1 = e1; b->e2 = e2; b->e3 = e3; b->origin = o;
    b->V = fabs(vdot(vcross(e1, e2), e3));
    b->orth = !(e1.y != 0.0 || e1.z != 0.0 || e2.x != 0.0 || e2.z != 0.0 || e3.x != 0.0 || e3.y != 0.0);
    v3 a1 = vcross(e2, e3); b->e1r = vdiv(a1, vdot(e1, a1));
    v3 a2 = vcross(e3, e1); b->e2r = vdiv(a2, vdot(e2, a2));
    v3 a3 = vcross(e1, e2); b->e3r = vdiv(a3, vdot(e3, a3));
    v3 s = vadd(vadd(e1, e2), e3);
    v3 a = vsub(o, vmul(s, 0.5));
    v3 c = vadd(o, vmul(s, 0.5));
    b->min = mk(fmin(a.x, c.x), fmin(a.y, c.y), fmin(a.z, c.z));
    b->max = mk(fmax(a.x, c.x), fmax(a.y, c.y), fmax(a.z, c.z));
    double dx = (e1.x * 0.5) * (e1.x * 0.5);
    double dy = (e2.y * 0.5) * (e2.y * 0.5);
    double dz = (e3.z * 0.5) * (e3.z * 0.5);
    b->D = dx < (dy < dz ? dy : dz) ? dx : (dy < dz ? dy : dz);
    b->H = vsub(b->max, b->min);
    b->H2 = vmul(b->H, 0.5);
}

/* minimalDifference(c1, c2, distSquared) (PeriodicBoundaryConditions.h:76-118) */
static v3 pbc_min_diff(const pbc_t* b, v3 c1, v3 c2, double* d2)
{
    v3 d = vsub(c2, c1);
    if (b->orth) {
        *d2 = vnorm2(d);
        if (*d2 > b->D) {
            if (d.x < -b->H2.x) d.x += b->H.x; else if (d.x > b->H2.x) d.x -= b->H.x;
            if (d.y < -b->H2.y) d.y += b->H.y; else if (d.y > b->H2.y) d.y -= b->H.y;
            if (d.z < -b->H2.z) d.z += b->H.z; else if (d.z > b->H2.z) d.z -= b->H.z;
            *d2 = vnorm2(d);
            if (*d2 > b->D) {
                d.x -= b->e1.x * rint(b->e1r.x * d.x);
                d.y -= b->e2.y * rint(b->e2r.y * d.y);
                d.z -= b->e3.z * rint(b->e3r.z * d.z);
                *d2 = vnorm2(d);
            }
        }
    } else {
        v3 t = vadd(vadd(vmul(b->e1, rint(vdot(b->e1r, d))), vmul(b->e2, rint(vdot(b->e2r, d)))),
                    vmul(b->e3, rint(vdot(b->e3r, d))));
        d = vsub(d, t);
        *d2 = vnorm2(d);
    }
    return d;
}

/* minimalPosition (PeriodicBoundaryConditions.h:120-150) */
static v3 pbc_min_pos(const pbc_t* b, v3 c)
{
    v3 d = vsub(c, b->origin);
    if (b->orth) {
        if (vnorm2(d) <= b->D) return d;
        if (d.x < -b->H2.x) d.x += b->H.x; else if (d.x > b->H2.x) d.x -= b->H.x;
        if (d.y < -b->H2.y) d.y += b->H.y; else if (d.y > b->H2.y) d.y -= b->H.y;
        if (d.z < -b->H2.z) d.z += b->H.z; else if (d.z > b->H2.z) d.z -= b->H.z;
        if (vnorm2(d) <= b->D) return d;
        return vsub(d, mk(b->e1.x * rint(b->e1r.x * d.x), b->e2.y * rint(b->e2r.y * d.y),
                          b->e3.z * rint(b->e3r.z * d.z)));
    }
    v3 t = vadd(vadd(vmul(b->e1, rint(vdot(b->e1r, d))), vmul(b->e2, rint(vdot(b->e2r, d)))),
                vmul(b->e3, rint(vdot(b->e3r, d))));
    return vsub(d, t);
}

/* --------------------------------------------------------- cell lists */
typedef struct {
    int nx, ny, nz;
    v3 rcs;                 /* myRealRCellSize */
    v3 cs;                  /* myRealCellSize */
    int* head;              /* first atom per cell, -1 empty */
    int* next;              /* cellListNext per atom */
    int* cell;              /* 3N cell coordinates */
    int out_of_grid;
    int maxNX, maxNY, maxNZ, nx1, ny1, nz1, maxNX1, maxNY1, maxNZ1;
} cells_t;

static void cells_free(cells_t* c)
{
    free(c->head); free(c->next); free(c->cell);
}

/* CubicCellManager::initialize (CubicCellManager.cpp:25-42) +
 * ArrayCellListStructure::initialize (ArrayCellListStructure.cpp:24-93) +
 * buildCellLists (buildCellLists.cpp:11-38). */
static void cells_build(cells_t* c, const pbc_t* b, const pmo_system* s)
{
    v3 d = vsub(b->max, b->min);
    double cell = s->cell_size;
    c->cs = mk(d.x / fmax(1.0, floor(d.x / cell)), d.y / fmax(1.0, floor(d.y / cell)),
               d.z / fmax(1.0, floor(d.z / cell)));
    c->rcs = mk(1.0 / c->cs.x, 1.0 / c->cs.y, 1.0 / c->cs.z);
    int nx = (int)floor(d.x / c->cs.x + PMO_EPSILON);
    int ny = (int)floor(d.y / c->cs.y + PMO_EPSILON);
    int nz = (int)floor(d.z / c->cs.z + PMO_EPSILON);
    c->nx = nx < 1 ? 1 : nx; c->ny = ny < 1 ? 1 : ny; c->nz = nz < 1 ? 1 : nz;
    int max2 = PMO_MAX_INT_2;
    c->maxNX = max2 - max2 % c->nx; c->maxNY = max2 - max2 % c->ny; c->maxNZ = max2 - max2 % c->nz;
    c->nx1 = -c->nx / 2; c->ny1 = -c->ny / 2; c->nz1 = -c->nz / 2;
    c->maxNX1 = c->maxNX - c->nx1; c->maxNY1 = c->maxNY - c->ny1; c->maxNZ1 = c->maxNZ - c->nz1;
    size_t ncell = (size_t)c->nx * c->ny * c->nz;
    c->head = (int*)malloc(ncell * sizeof(int));
    for (size_t k = 0; k < ncell; ++k) c->head[k] = -1;
    c->next = (int*)malloc((size_t)s->n_atoms * sizeof(int));
    c->cell = (int*)malloc((size_t)s->n_atoms * 3 * sizeof(int));
    c->out_of_grid = 0;
    v3 delta = vsub(b->origin, b->min);
    for (int i = s->n_atoms - 1; i >= 0; --i) {
        v3 p = vadd(delta, pbc_min_pos(b, vload(s->pos + 3 * i)));
        /* CubicCellManager::findCell (CubicCellManager.h:61-64) */
        int cx = (int)floor(p.x * c->rcs.x), cy = (int)floor(p.y * c->rcs.y), cz = (int)floor(p.z * c->rcs.z);
        c->cell[3 * i] = cx; c->cell[3 * i + 1] = cy; c->cell[3 * i + 2] = cz;
        if (cx < 0 || cy < 0 || cz < 0 || cx >= c->nx || cy >= c->ny || cz >= c->nz) {
            /* The reference writes outside its cell array here (undefined);
             * the restatement files the atom under the periodic image. */
            c->out_of_grid++;
            cx = ((cx % c->nx) + c->nx) % c->nx;
            cy = ((cy % c->ny) + c->ny) % c->ny;
            cz = ((cz % c->nz) + c->nz) % c->nz;
        }
        size_t k = ((size_t)cx * c->ny + cy) * c->nz + cz;
        c->next[i] = c->head[k];
        c->head[k] = i;
    }
}

typedef struct { int x, y, z; } cell3;

static int cell_less(const void* a, const void* b)
{
    const cell3* p = (const cell3*)a; const cell3* q = (const cell3*)b;
    if (p->x != q->x) return p->x < q->x ? -1 : 1;
    if (p->y != q->y) return p->y < q->y ? -1 : 1;
    if (p->z != q->z) return p->z < q->z ? -1 : 1;
    return 0;
}

/* Neighbour-delta list of CellListEnumerator<Periodic, Cubic>::initialize
 * (CellListEnumerator_periodicBoundaries.h:37-108): closest-approach test,
 * deduplicated modulo the grid with basisCell, sorted lexicographically. */
static int build_deltas(const cells_t* c, double cutoff, cell3** out)
{
    double cutoff2 = cutoff * cutoff;
    int nx = (int)(cutoff / c->cs.x + 1.0 + PMO_EPSILON);
    int ny = (int)(cutoff / c->cs.y + 1.0 + PMO_EPSILON);
    int nz = (int)(cutoff / c->cs.z + 1.0 + PMO_EPSILON);
    int n0 = nx < c->nx ? nx : c->nx, n1 = ny < c->ny ? ny : c->ny, n2 = nz < c->nz ? nz : c->nz;
    double xx = c->cs.x * c->cs.x, yy = c->cs.y * c->cs.y, zz = c->cs.z * c->cs.z;
    int cap = (2 * n0 + 1) * (2 * n1 + 1) * (2 * n2 + 1) + 1;
    cell3* seen = (cell3*)malloc(sizeof(cell3) * cap);
    cell3* list = (cell3*)malloc(sizeof(cell3) * cap);
    int nseen = 0, nlist = 0;
    seen[nseen++] = (cell3){0, 0, 0};
    for (int k = -n0; k <= n0; k++) {
        int x = abs(k) - 1; if (x < 0) x = 0;
        double d0 = x * x * xx;
        for (int l = -n1; l <= n1; l++) {
            int y = abs(l) - 1; if (y < 0) y = 0;
            double d1 = d0 + y * y * yy;
            for (int m = -n2; m <= n2; m++) {
                int z = abs(m) - 1; if (z < 0) z = 0;
                if (d1 + z * z * zz < cutoff2) {
                    cell3 md = {(k + c->maxNX1) % c->nx + c->nx1, (l + c->maxNY1) % c->ny + c->ny1,
                                (m + c->maxNZ1) % c->nz + c->nz1};
                    int found = 0;
                    for (int t = 0; t < nseen; ++t)
                        if (seen[t].x == md.x && seen[t].y == md.y && seen[t].z == md.z) { found = 1; break; }
                    if (!found) { seen[nseen++] = md; list[nlist++] = md; }
                }
            }
        }
    }
    free(seen);
    qsort(list, nlist, sizeof(cell3), cell_less);
    *out = list;
    return nlist;
}

/* ------------------------------------------------------------ exclusions */
typedef struct { long long key; int cls; } excl_entry;

static int excl_cmp(const void* a, const void* b)
{
    long long x = ((const excl_entry*)a)->key, y = ((const excl_entry*)b)->key;
    return x < y ? -1 : (x > y ? 1 : 0);
}

typedef struct { excl_entry* e; int n; } excl_t;

static void excl_build(excl_t* t, const pmo_system* s)
{
    t->n = s->n_excl;
    t->e = (excl_entry*)malloc(sizeof(excl_entry) * (t->n > 0 ? t->n : 1));
    for (int k = 0; k < t->n; ++k) {
        int a = s->excl[3 * k], b = s->excl[3 * k + 1];
        if (a > b) { int tmp = a; a = b; b = tmp; }
        t->e[k].key = (long long)a * 2147483648LL + b;
        t->e[k].cls = s->excl_check ? s->excl_check[k] : s->excl[3 * k + 2];
    }
    qsort(t->e, t->n, sizeof(excl_entry), excl_cmp);
}

/* ExclusionTable::check (topology/ExclusionTable.h:130-146) */
static int excl_check(const excl_t* t, int a, int b)
{
    if (b < a) { int tmp = a; a = b; b = tmp; }
    excl_entry k = {(long long)a * 2147483648LL + b, 0};
    excl_entry* f = (excl_entry*)bsearch(&k, t->e, t->n, sizeof(excl_entry), excl_cmp);
    return f ? f->cls : PMO_EXCL_NONE;
}

/* ---------------------------------------------------------- potentials */
/* poly5 (base/mathutilities.cpp:29-40), Abramowitz & Stegun 7.1.26 */
double pmo_poly5(double ar)
{
    const double E1 = 0.254829592, E2 = -0.284496736, E3 = 1.421413741,
                 E4 = -1.453152027, E5 = 1.061405429, PP = 0.3275911;
    double t = 1.0 / (1.0 + PP * ar);
    return ((t) * (E1 + (t) * (E2 + (t) * (E3 + (t) * (E4 + (t) * E5)))));
}

typedef struct {
    int pot, sw;
    /* switching constants */
    double cut, cut2, on2, s1, s2, s3;         /* C2 */
    double c1_15_1, c1_05_3, c1_15_3;           /* C1 */
    double sh_c_2, sh_4c_2;                      /* Shift */
    int use, modify;
    double alpha, two_alpha_pi;                 /* EwaldReal */
    /* table potentials: LookUpTableBase's table and hashing constants */
    double* tab;
    long long tab_first, tab_last;
    int tab_step, tab_shift;
} term_t;

static void term_switch(const term_t* t, double d2, double* value, double* deriv);

static int is_table(int pot)
{
    return pot == PMO_POT_LJ_TABLE || pot == PMO_POT_COULOMB_TABLE || pot == PMO_POT_EWALD_REAL_TABLE;
}

/* ---- look-up tables (base/LookUpTableBase.h) ---- */
/* lowerboundExp2 (base/mathutilities.cpp:43-51) */
static double lowerbound_exp2(double r)
{
    double res = 1.0;
    while (res < r) res *= 2.0;
    while (res > r) res /= 2.0;
    return res;
}

static long long dbits(double x) { long long u; memcpy(&u, &x, 8); return u; }
static double dfrombits(long long u) { double x; memcpy(&x, &u, 8); return x; }

/* LookUpTableBase::expn: the biased binary exponent of lowerboundExp2(a) */
static long long lut_expn(double a) { return dbits(lowerbound_exp2(a)) >> 52; }

/* power<n> for the negative powers the tabulated functions use
 * (base/mathutilities.h:72-94: square(power<n/2>) * power<n - 2 (n/2)>,
 * C++ division truncating towards zero) */
static double pw_m1(double x) { return 1. / x; }
static double pw_m2(double x) { double y = pw_m1(x); return (y * y) * 1; }
static double pw_m3(double x) { double y = pw_m1(x); return (y * y) * pw_m1(x); }
static double pw_m4(double x) { double y = pw_m2(x); return (y * y) * 1; }
static double pw_m6(double x) { double y = pw_m3(x); return (y * y) * 1; }
static double pw_m7(double x) { double y = pw_m3(x); return (y * y) * pw_m1(x); }
static double pw_m8(double x) { double y = pw_m4(x); return (y * y) * 1; }
static double pw_m12(double x) { double y = pw_m6(x); return (y * y) * 1; }
static double pw_m14(double x) { double y = pw_m7(x); return (y * y) * 1; }

/* LookUpValues::assign of the three table potentials, lookUpExp = 2 (the
 * table variable r is r^2, r1 = sqrt(r)):
 * forces/LennardJonesTableForceBase.h:35-45, CoulombTableForceBase.h:33-39,
 * CoulombEwaldRealTableForceBase.h:36-43 */
static void lut_assign(int pot, double alpha, double r, double r1, double v, double d, double* val)
{
    if (pot == PMO_POT_LJ_TABLE) {
        double e = pw_m12(r1);
        double f = 12.0 * pw_m14(r1);
        val[0] = e * v;
        val[1] = -0.5 * (f * v - e * d);
        e = -pw_m6(r1);
        f = -6.0 * pw_m8(r1);
        val[4] = e * v;
        val[5] = -0.5 * (f * v - e * d);
    } else if (pot == PMO_POT_COULOMB_TABLE) {
        double e = pw_m1(r1);
        double f = pw_m3(r1);
        val[0] = e * v;
        val[1] = -0.5 * (f * v - e * d);
    } else {
        double r2 = r;
        double e = erfc(alpha * r1) / r1;
        double f = (e + 2.0 * alpha / sqrt(PMO_PI) * exp(-alpha * alpha * r2)) / r2;
        val[0] = e * v;
        val[1] = -0.5 * (f * v - e * d);
    }
}

/* LookUpTableBase(from = 0.1, to = rc^2, lookUpExp = 2, ...) constructor
 * (base/LookUpTableBase.h:115-205) with the precision the registered
 * templates use: PRE = 7 for LennardJonesTable, 6 for the Coulomb tables
 * (factories/registerForceExemplarsCutoff.cpp:47-48,58,69).  The tabulated
 * switching function is sw_term's. */
static long long lut_build(int pot, const term_t* sw_term, double alpha, double to, double* out, long long cap,
                           long long* first, long long* last, int* step, int* shift)
{
    const int pre = pot == PMO_POT_LJ_TABLE ? 7 : 6;
    const int n = 1 << pre;
    const int stp = (pot == PMO_POT_LJ_TABLE ? 2 : 1) * 4;
    double from = 0.1;
    const long long octaves = lut_expn(to) + 1 - lut_expn(from);
    const long long size = (octaves * n + 1) * stp;
    if (out == NULL || size > cap) return size;
    *shift = 52 - pre;
    *first = (dbits(lowerbound_exp2(from)) >> *shift) * stp;
    *last = octaves * n * stp;
    *step = stp;
    from = lowerbound_exp2(from);
    for (long long i = 0; i < size / stp; ++i) {
        double base = from * (double)(1 << (i / n));
        double del = base / (double)n;
        double r = base + del * (double)(i % n);
        double r1 = sqrt(r);
        double v, d;
        term_switch(sw_term, r, &v, &d);
        lut_assign(pot, alpha, r, r1, v, d, out + i * stp);
        for (int j = 0; j < stp; j += 4) { out[2 + i * stp + j] = 0.0; out[3 + i * stp + j] = 0.0; }
        if (i > 0) {
            double x = from * (double)(1 << ((i - 1) / n)) / (double)n;
            double* t = out + (i - 1) * stp;
            for (int j = 0; j < stp; j += 4) {
                double v1 = t[0 + j], g1 = t[1 + j], v2 = t[0 + stp + j], g2 = t[1 + stp + j];
                double c = (3.0 * (v2 - v1) - x * (2.0 * g1 + g2)) / (x * x);
                double dd = (-2.0 * (v2 - v1) + x * (g1 + g2)) / (x * x * x);
                for (int k = 0; k < 2; ++k) {
                    double dv = (v1 - v2) + ((dd * x + c) * x + g1) * x;
                    double dg = (g1 - g2) + (3.0 * dd * x + 2.0 * c) * x;
                    c -= (3.0 * dv - x * dg) / (x * x);
                    dd -= (-2.0 * dv + x * dg) / (x * x * x);
                }
                t[2 + j] = c;
                t[3 + j] = dd;
            }
        }
    }
    return size;
}

/* LookUpTableBase::index and ::interpolate (base/LookUpTableBase.h:243-272):
 * the entry from the top bits of r^2's representation, the remainder dt */
static void lut_index(const term_t* t, double r2, long long* i, double* dt)
{
    long long u = dbits(r2);
    *i = (u >> t->tab_shift) * t->tab_step - t->tab_first;
    *dt = 0.0;
    if (*i < 0) *i = 0;
    else if (*i > t->tab_last) *i = t->tab_last;
    else *dt = r2 - dfrombits(u & ~((1LL << t->tab_shift) - 1LL));
}

static void lut_interpolate(double a, double b, double c, double d, double dt, double* energy, double* force)
{
    *energy = ((dt * d + c) * dt + b) * dt + a;
    *force = -2.0 * ((3.0 * dt * d + 2.0 * c) * dt + b);
}

static void term_init(term_t* t, int pot, int sw, double on, double cut, double alpha)
{
    memset(t, 0, sizeof(*t));
    t->pot = pot; t->sw = sw; t->cut = cut; t->cut2 = cut * cut;
    t->use = sw != PMO_SW_UNIVERSAL;
    t->modify = (sw == PMO_SW_C1 || sw == PMO_SW_C2 || sw == PMO_SW_SHIFT);
    if (sw == PMO_SW_C2) {
        /* C2SwitchingFunction.cpp:15-23 */
        double d = cut * cut - on * on;
        t->on2 = on * on;
        t->s1 = 1.0 / (d * d * d);
        t->s2 = cut * cut - 3.0 * on * on;
        t->s3 = 4.0 / (d * d * d);
    } else if (sw == PMO_SW_C1) {
        /* C1SwitchingFunction.cpp:18-25 */
        t->c1_15_1 = 1.5 / cut;
        t->c1_05_3 = 0.5 / (cut * cut * cut);
        t->c1_15_3 = 1.5 / (cut * cut * cut);
    } else if (sw == PMO_SW_SHIFT) {
        /* ShiftSwitchingFunction.cpp */
        t->sh_c_2 = 1.0 / (cut * cut);
        t->sh_4c_2 = -4.0 / (cut * cut);
    }
    t->alpha = alpha;
    t->two_alpha_pi = 2.0 * alpha / sqrt(PMO_PI);
    if (is_table(pot)) {
        /* the pair applies UniversalSwitchingFunction and tests the table's
         * cutoff (Cutoff<true>, forces/oneAtomContraints.h:24-31;
         * OneAtomPair.h:141) */
        long long n = lut_build(pot, t, alpha, t->cut2, NULL, 0, NULL, NULL, NULL, NULL);
        t->tab = (double*)malloc(sizeof(double) * (size_t)n);
        lut_build(pot, t, alpha, t->cut2, t->tab, n, &t->tab_first, &t->tab_last, &t->tab_step, &t->tab_shift);
        t->sw = PMO_SW_UNIVERSAL;
        t->use = 1;
        t->modify = 0;
    }
}

long long pmo_lookup_table(int pot, int sw, double switchon, double cutoff, double alpha,
                           double* table, long long cap)
{
    if (!is_table(pot)) return -1;
    term_t t;
    term_init(&t, PMO_POT_NONE, sw, switchon, cutoff, alpha);
    long long first, last;
    int step, shift;
    return lut_build(pot, &t, alpha, t.cut2, table, cap, &first, &last, &step, &shift);
}

/* Switching functions: value and derivOverD as in the reference operator()s. */
static void term_switch(const term_t* t, double d2, double* value, double* deriv)
{
    switch (t->sw) {
    case PMO_SW_C2:   /* C2SwitchingFunction.h:64-82 */
        *deriv = 0.0;
        if (d2 > t->cut2) { *value = 0.0; }
        else if (d2 >= t->on2) {
            double c2 = t->cut2 - d2;
            double c4 = c2 * (t->s2 + 2.0 * d2);
            *value = t->s1 * (c2 * c4);
            *deriv = t->s3 * (c2 * c2 - c4);
        } else { *value = 1.0; }
        break;
    case PMO_SW_C1: { /* C1SwitchingFunction.h:64-75 */
        if (d2 > t->cut2) { *value = 0.0; *deriv = 0.0; return; }
        double dist = sqrt(d2);
        *value = 1.0 - dist * (t->c1_15_1 - d2 * t->c1_05_3);
        *deriv = -t->c1_15_1 / dist + dist * t->c1_15_3;
        break; }
    case PMO_SW_SHIFT: { /* ShiftSwitchingFunction.h */
        if (d2 > t->cut2) { *value = 0.0; *deriv = 0.0; return; }
        double x = (1.0 - d2 * t->sh_c_2);
        *value = x * x;
        *deriv = t->sh_4c_2 * x;
        break; }
    case PMO_SW_CUTOFF: /* CutoffSwitchingFunction.h:64-68 */
        *deriv = 0;
        *value = (d2 > t->cut2 ? 0.0 : 1.0);
        break;
    default:            /* UniversalSwitchingFunction */
        *value = 1.0; *deriv = 0.0;
    }
}

static int pot_dist_r2(int pot) { return pot == PMO_POT_LJ || pot == PMO_POT_COULOMB; }

static void term_potential(const term_t* t, const pmo_system* s, int i, int j, int excl,
                           double d2, double rd2, double* energy, double* force)
{
    if (t->pot == PMO_POT_LJ) {
        /* LennardJonesForce::operator() (forces/LennardJonesForce.h:37-74) */
        const double* p = s->lj + 4 * ((size_t)s->type[i] * s->n_types + s->type[j]);
        double A, B;
        if (excl != PMO_EXCL_MODIFIED) { A = p[0]; B = p[1]; } else { A = p[2]; B = p[3]; }
        double r6 = rd2 * rd2 * rd2;
        double r12 = r6 * r6;
        double r6B = B * r6;
        double r12A = A * r12;
        *energy = r12A - r6B;
        *force = 12.0 * r12A * rd2 - 6.0 * r6B * rd2;
    } else if (t->pot == PMO_POT_COULOMB) {
        /* CoulombForce::operator() (forces/CoulombForce.h:41-57) */
        *energy = s->q[i] * s->q[j] * sqrt(rd2);
        if (excl == PMO_EXCL_MODIFIED) *energy *= s->csf;
        *force = *energy * rd2;
    } else if (t->pot == PMO_POT_EWALD_REAL) {
        /* CoulombEwaldRealForce::operator() (forces/CoulombEwaldRealForce.h:45-73) */
        double qq = s->q[i] * s->q[j];
        if (s->csf != 1.0 && excl == PMO_EXCL_MODIFIED) qq *= s->csf;
        double r = sqrt(d2);
        double rr = 1.0 / r;
        double ar = t->alpha * r;
        double e = qq * exp(-ar * ar);
        *energy = pmo_poly5(ar) * e * rr;
        *force = ((*energy + t->two_alpha_pi * e) * rr * rr);
    } else if (t->pot == PMO_POT_LJ_TABLE) {
        /* LennardJonesTableForce::operator() (forces/LennardJonesTableForce.h:81-101) */
        const double* p = s->lj + 4 * ((size_t)s->type[i] * s->n_types + s->type[j]);
        double A = (excl != PMO_EXCL_MODIFIED ? p[0] : p[2]);
        double B = (excl != PMO_EXCL_MODIFIED ? p[1] : p[3]);
        long long k;
        double dt;
        lut_index(t, d2, &k, &dt);
        const double* T = t->tab + k;
        double a = T[0] * A + T[4] * B;
        double b = T[1] * A + T[5] * B;
        double c = T[2] * A + T[6] * B;
        double d = T[3] * A + T[7] * B;
        lut_interpolate(a, b, c, d, dt, energy, force);
    } else if (t->pot == PMO_POT_COULOMB_TABLE || t->pot == PMO_POT_EWALD_REAL_TABLE) {
        /* CoulombTableForce::operator() (forces/CoulombTableForce.h:83-108),
         * CoulombEwaldRealTableForce::operator() (CoulombEwaldRealTableForce.h:85-107) */
        double q = s->q[i] * s->q[j] * ((s->csf != 1.0 && excl == PMO_EXCL_MODIFIED) ? s->csf : 1.0);
        long long k;
        double dt;
        lut_index(t, d2, &k, &dt);
        const double* T = t->tab + k;
        lut_interpolate(T[0] * q, T[1] * q, T[2] * q, T[3] * q, dt, energy, force);
    } else {
        *energy = 0.0; *force = 0.0;
    }
}

/* ScalarStructure::addVirial (base/ScalarStructure.cpp:41-62) */
static void add_virial(double* v, v3 f, v3 d)
{
    double xy = f.x * d.y, xz = f.x * d.z, yz = f.y * d.z;
    v[0] += f.x * d.x; v[1] += xy; v[2] += xz;
    v[3] += xy; v[4] += f.y * d.y; v[5] += yz;
    v[6] += xz; v[7] += yz; v[8] += f.z * d.z;
}

typedef struct {
    const pmo_system* s;
    const pbc_t* b;
    const excl_t* ex;
    term_t t[2];
    int n_terms;
    double cut2;
    int any_r2, any_modify;
    double* f;
    pmo_result* r;
    int* pairs; long long cap;
    int vacuum;
} pair_ctx;

/* minimalDifference of the two molecules' positions (OneAtomPair.h:178-179):
 * minimal image, or the plain difference in vacuum */
static v3 mol_diff(const pair_ctx* c, int mi, int mj)
{
    v3 a = vload(c->s->mol_pos + 3 * (size_t)mi), b = vload(c->s->mol_pos + 3 * (size_t)mj);
    if (c->vacuum) return vsub(b, a);
    double d2;
    return pbc_min_diff(c->b, a, b, &d2);
}

/* OneAtomPair::doOneAtomPair (forces/OneAtomPair.h:127-188) and
 * OneAtomPairTwo::doOneAtomPair (forces/OneAtomPairTwo.h:131-199). */
static void one_atom_pair(pair_ctx* c, int i, int j)
{
    const pmo_system* s = c->s;
    double d2;
    v3 diff;
    if (c->vacuum) { diff = vsub(vload(s->pos + 3 * j), vload(s->pos + 3 * i)); d2 = vnorm2(diff); }
    else diff = pbc_min_diff(c->b, vload(s->pos + 3 * i), vload(s->pos + 3 * j), &d2);
    int use = c->t[0].use || (c->n_terms > 1 && c->t[1].use);
    if (use && d2 > c->cut2) return;
    int same = s->mol[i] == s->mol[j];
    int excl = same ? excl_check(c->ex, i, j) : PMO_EXCL_NONE;
    if (excl == PMO_EXCL_FULL) return;
    double rd2 = c->any_r2 ? 1.0 / d2 : 1.0;
    double e[2] = {0, 0}, f[2] = {0, 0};
    for (int k = 0; k < c->n_terms; ++k)
        term_potential(&c->t[k], s, i, j, excl, d2, rd2, &e[k], &f[k]);
    if (c->any_modify) {
        for (int k = 0; k < c->n_terms; ++k) {
            double sv, sd;
            term_switch(&c->t[k], d2, &sv, &sd);
            f[k] = f[k] * sv - e[k] * sd;
            e[k] = e[k] * sv;
        }
    }
    for (int k = 0; k < c->n_terms; ++k) {
        if (c->t[k].pot == PMO_POT_LJ || c->t[k].pot == PMO_POT_LJ_TABLE) c->r->lennard_jones += e[k];
        else c->r->coulomb += e[k];
    }
    double ftot = c->n_terms > 1 ? (f[0] + f[1]) : f[0];
    v3 fij = vmul(diff, ftot);
    double* fi = c->f + 3 * i;
    double* fj = c->f + 3 * j;
    fi[0] -= fij.x; fi[1] -= fij.y; fi[2] -= fij.z;
    fj[0] += fij.x; fj[1] += fij.y; fj[2] += fij.z;
    if (!same && s->mol_pos) {
        /* ScalarStructure::addVirial(force, diff, comDiff)
         * (base/ScalarStructure.cpp:90-132): atomic and molecular virial */
        add_virial(c->r->virial, fij, diff);
        add_virial(c->r->mol_virial, fij, mol_diff(c, s->mol[i], s->mol[j]));
    } else if (!s->no_virial) {
        add_virial(c->r->virial, fij, diff);
    }
    if (c->pairs && c->r->n_pairs < c->cap) {
        c->pairs[2 * c->r->n_pairs] = i < j ? i : j;
        c->pairs[2 * c->r->n_pairs + 1] = i < j ? j : i;
    }
    c->r->n_pairs++;
}

static void pair_ctx_init(pair_ctx* c, const pmo_system* s, const pmo_cutoff_params* p)
{
    memset(c, 0, sizeof(*c));
    c->s = s;
    c->n_terms = p->n_terms;
    double cut2 = 0.0;
    for (int k = 0; k < p->n_terms; ++k) {
        term_init(&c->t[k], p->pot[k], p->sw[k], p->switchon[k], p->sw_cutoff[k], p->alpha[k]);
        /* Cutoff<>::cutoff: the switching function's cutoff^2; the pair test
         * uses the larger one (OneAtomPairTwo.h:48) */
        if (c->t[k].cut2 > cut2) cut2 = c->t[k].cut2;
        if (pot_dist_r2(p->pot[k])) c->any_r2 = 1;
        if (c->t[k].modify) c->any_modify = 1;
    }
    c->cut2 = cut2;
}

static void pair_ctx_free(pair_ctx* c)
{
    for (int k = 0; k < 2; ++k) { free(c->t[k].tab); c->t[k].tab = NULL; }
}

int pmo_molecular_centers(const pmo_system* s, const double* mass, double* centers)
{
    int nm = 0;
    for (int i = 0; i < s->n_atoms; ++i)
        if (s->mol[i] + 1 > nm) nm = s->mol[i] + 1;
    /* per molecule: center, Kahan compensation, sum of masses, atoms seen */
    double* acc = (double*)calloc(8 * (size_t)nm, sizeof(double));
    for (int i = 0; i < s->n_atoms; ++i) {
        double* a = acc + 8 * (size_t)s->mol[i];
        double m = mass ? mass[i] : 1.0;
        v3 x = vmul(vload(s->pos + 3 * i), m);
        if (a[7] == 0.0) {
            a[0] = x.x; a[1] = x.y; a[2] = x.z;
            a[6] = m;
        } else {
            v3 center = mk(a[0], a[1], a[2]), tempC = mk(a[3], a[4], a[5]);
            a[6] += m;
            v3 tempY = vsub(x, tempC);
            v3 tempT = vadd(center, tempY);
            tempC = vsub(vsub(tempT, center), tempY);
            a[0] = tempT.x; a[1] = tempT.y; a[2] = tempT.z;
            a[3] = tempC.x; a[4] = tempC.y; a[5] = tempC.z;
        }
        a[7] += 1.0;
    }
    for (int m = 0; m < nm; ++m) {
        const double* a = acc + 8 * (size_t)m;
        if (a[7] == 0.0) { centers[3 * m] = centers[3 * m + 1] = centers[3 * m + 2] = 0.0; continue; }
        v3 c = vdiv(mk(a[0], a[1], a[2]), a[6]);
        centers[3 * m] = c.x; centers[3 * m + 1] = c.y; centers[3 * m + 2] = c.z;
    }
    free(acc);
    return nm;
}

/* ModifierMetaShake::calcError (integrators/ModifierMetaShake.cpp) */
static double shake_error(int n_cons, const int* atoms, const double* rest, const double* pos)
{
    double error = 0;
    for (int i = 0; i < n_cons; i++) {
        v3 d = vsub(vload(pos + 3 * atoms[2 * i + 1]), vload(pos + 3 * atoms[2 * i]));
        double r2 = rest[i] * rest[i];
        error += fabs(vnorm2(d) - r2) / (2.0 * r2);
    }
    return error / n_cons;
}

int pmo_shake(int n_cons, const int* atoms, const double* rest, const double* mass, int n_atoms,
              double* pos, double* vel, double* last, double dt, double eps, int max_iter)
{
    if (n_cons <= 0) return 0;
    double error = shake_error(n_cons, atoms, rest, pos);
    int iter = 0;
    while (error > eps) {
        for (int i = 0; i < n_cons; i++) {
            int a1 = atoms[2 * i], a2 = atoms[2 * i + 1];
            v3 pab = vsub(vload(pos + 3 * a1), vload(pos + 3 * a2));
            double pabsq = vnorm2(pab);
            double rabsq = rest[i] * rest[i];
            double diffsq = rabsq - pabsq;
            v3 rab = vsub(vload(last + 3 * a1), vload(last + 3 * a2));
            double rpab = vdot(rab, pab);
            double rM1 = 1 / mass[a1];
            double rM2 = 1 / mass[a2];
            double gab = diffsq / (2 * (rM1 + rM2) * rpab);
            v3 dp = vmul(rab, gab);
            v3 p1 = vadd(vload(pos + 3 * a1), vmul(dp, rM1));
            v3 p2 = vsub(vload(pos + 3 * a2), vmul(dp, rM2));
            pos[3 * a1] = p1.x; pos[3 * a1 + 1] = p1.y; pos[3 * a1 + 2] = p1.z;
            pos[3 * a2] = p2.x; pos[3 * a2 + 1] = p2.y; pos[3 * a2 + 2] = p2.z;
            dp = vdiv(dp, dt);
            v3 w1 = vadd(vload(vel + 3 * a1), vmul(dp, rM1));
            v3 w2 = vsub(vload(vel + 3 * a2), vmul(dp, rM2));
            vel[3 * a1] = w1.x; vel[3 * a1 + 1] = w1.y; vel[3 * a1 + 2] = w1.z;
            vel[3 * a2] = w2.x; vel[3 * a2 + 1] = w2.y; vel[3 * a2 + 2] = w2.z;
        }
        error = shake_error(n_cons, atoms, rest, pos);
        iter++;
        if (iter > max_iter) break;
    }
    memcpy(last, pos, sizeof(double) * 3 * (size_t)n_atoms);
    return iter;
}

/* ModifierMetaRattle::calcError (integrators/ModifierMetaRattle.cpp) */
static double rattle_error(int n_cons, const int* atoms, const double* pos, const double* vel)
{
    double error = 0;
    for (int i = 0; i < n_cons; i++) {
        int a1 = atoms[2 * i], a2 = atoms[2 * i + 1];
        v3 vab = vsub(vload(vel + 3 * a1), vload(vel + 3 * a2));
        v3 rab = vsub(vload(pos + 3 * a1), vload(pos + 3 * a2));
        error += fabs(vdot(rab, vab));
    }
    return error / n_cons;
}

int pmo_rattle(int n_cons, const int* atoms, const double* rest, const double* mass,
               const double* pos, double* vel, double dt, double eps, int max_iter, double* virial)
{
    (void)rest;
    if (n_cons <= 0) return 0;
    double error = rattle_error(n_cons, atoms, pos, vel);
    int iter = 0;
    while (error > eps) {
        for (int i = 0; i < n_cons; i++) {
            int a1 = atoms[2 * i], a2 = atoms[2 * i + 1];
            double rM1 = 1 / mass[a1];
            double rM2 = 1 / mass[a2];
            v3 rab = vsub(vload(pos + 3 * a1), vload(pos + 3 * a2));
            double rabsq = vnorm2(rab);
            v3 vab = vsub(vload(vel + 3 * a1), vload(vel + 3 * a2));
            double rvab = vdot(rab, vab);
            double gab = -rvab / (dt * (rM1 + rM2) * rabsq);
            v3 dp = vmul(rab, gab);
            v3 w1 = vadd(vload(vel + 3 * a1), vmul(vmul(dp, dt), rM1));
            v3 w2 = vsub(vload(vel + 3 * a2), vmul(vmul(dp, dt), rM2));
            vel[3 * a1] = w1.x; vel[3 * a1 + 1] = w1.y; vel[3 * a1 + 2] = w1.z;
            vel[3 * a2] = w2.x; vel[3 * a2 + 1] = w2.y; vel[3 * a2 + 2] = w2.z;
            if (virial) add_virial(virial, vmul(dp, 2), rab);
        }
        error = rattle_error(n_cons, atoms, pos, vel);
        iter++;
        if (iter > max_iter) break;
    }
    return iter;
}

int pmo_cell_assign(const pmo_system* s, int* cells, int* dims)
{
    pbc_t b; pbc_set(&b, s->box);
    cells_t c; cells_build(&c, &b, s);
    memcpy(cells, c.cell, sizeof(int) * 3 * (size_t)s->n_atoms);
    dims[0] = c.nx; dims[1] = c.ny; dims[2] = c.nz;
    int oog = c.out_of_grid;
    cells_free(&c);
    return oog;
}

/* NonbondedCutoffSystemForce::evaluate (NonbondedCutoffSystemForce.h:63-74)
 * -> NonbondedCutoffForce::doEvaluate (NonbondedCutoffForce.h:85-109) with
 * the periodic enumerator's next() order (CellListEnumerator_periodicBoundaries.h:157-179). */
int pmo_cutoff_force(const pmo_system* s, const pmo_cutoff_params* p,
                     double* forces, pmo_result* r, int* pairs, long long cap)
{
    pbc_t b; pbc_set(&b, s->box);
    cells_t c; cells_build(&c, &b, s);
    excl_t ex; excl_build(&ex, s);
    cell3* deltas = NULL;
    int nd = build_deltas(&c, p->algo_cutoff, &deltas);
    pair_ctx pc; pair_ctx_init(&pc, s, p);
    pc.b = &b; pc.ex = &ex; pc.f = forces; pc.r = r; pc.pairs = pairs; pc.cap = cap;
    r->out_of_grid += c.out_of_grid;
    int ncell = c.nx * c.ny * c.nz;
    for (int A = 0; A < ncell; ++A) {
        if (c.head[A] < 0) continue;
        /* the same cell: j after i in the list */
        for (int i = c.head[A]; i != -1; i = c.next[i])
            for (int j = c.next[i]; j != -1; j = c.next[j])
                one_atom_pair(&pc, i, j);
        int ax = A / (c.ny * c.nz), ay = (A / c.nz) % c.ny, az = A % c.nz;
        for (int k = 0; k < nd; ++k) {
            /* findPeriodic (ArrayCellListStructure.h:108-122) */
            int bx = (ax + deltas[k].x + c.maxNX) % c.nx;
            int by = (ay + deltas[k].y + c.maxNY) % c.ny;
            int bz = (az + deltas[k].z + c.maxNZ) % c.nz;
            int B = (bx * c.ny + by) * c.nz + bz;
            if (c.head[B] < 0 || B < A) continue;
            for (int i = c.head[A]; i != -1; i = c.next[i])
                for (int j = c.head[B]; j != -1; j = c.next[j])
                    one_atom_pair(&pc, i, j);
        }
    }
    free(deltas);
    free(ex.e);
    cells_free(&c);
    pair_ctx_free(&pc);
    return 0;
}

/* NonbondedSimpleFullSystemForce::doEvaluate (NonbondedSimpleFullSystemForce.h:160-190),
 * unblocked i < j order, vacuum boundary conditions. */
int pmo_simple_full_force(const pmo_system* s, const pmo_cutoff_params* p,
                          double* forces, pmo_result* r)
{
    excl_t ex; excl_build(&ex, s);
    pair_ctx pc; pair_ctx_init(&pc, s, p);
    pc.ex = &ex; pc.f = forces; pc.r = r; pc.vacuum = 1;
    for (int i = 0; i < s->n_atoms; ++i)
        for (int j = i + 1; j < s->n_atoms; ++j)
            one_atom_pair(&pc, i, j);
    free(ex.e);
    pair_ctx_free(&pc);
    return 0;
}

/* -------------------------------------------------------------------- FFT */
/* Mixed-radix recursive complex DFT (unnormalised), out-of-place on strided
 * input: X[k] = sum_j x[j] exp(sign 2 pi i j k / n).  Plays the role of the
 * vendored ZFFT (base/fft.c zfft3d) used by FFTComplex::forward/backward. */
static void dft_rec(const double* in, int stride, double* out, int n, int sign)
{
    if (n == 1) { out[0] = in[0]; out[1] = in[1]; return; }
    int p = 2;
    while (n % p) ++p;           /* smallest prime factor */
    int m = n / p;
    double* sub = (double*)malloc(sizeof(double) * 2 * n);
    for (int r = 0; r < p; ++r)
        dft_rec(in + 2 * (size_t)r * stride, stride * p, sub + 2 * r * m, m, sign);
    for (int k = 0; k < n; ++k) {
        double re = 0.0, im = 0.0;
        for (int r = 0; r < p; ++r) {
            double ang = sign * 2.0 * PMO_PI * (double)r * (double)k / (double)n;
            double c = cos(ang), sn = sin(ang);
            const double* x = sub + 2 * (r * m + k % m);
            re += x[0] * c - x[1] * sn;
            im += x[0] * sn + x[1] * c;
        }
        out[2 * k] = re; out[2 * k + 1] = im;
    }
    free(sub);
}

int pmo_fft3d(double* data, int nx, int ny, int nz, int sign)
{
    int nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
    double* in = (double*)malloc(sizeof(double) * 2 * nmax);
    double* out = (double*)malloc(sizeof(double) * 2 * nmax);
    /* along z (contiguous) */
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            double* line = data + 2 * ((size_t)x * ny + y) * nz;
            dft_rec(line, 1, out, nz, sign);
            memcpy(line, out, sizeof(double) * 2 * nz);
        }
    /* along y */
    for (int x = 0; x < nx; ++x)
        for (int z = 0; z < nz; ++z) {
            for (int y = 0; y < ny; ++y) {
                double* e = data + 2 * (((size_t)x * ny + y) * nz + z);
                in[2 * y] = e[0]; in[2 * y + 1] = e[1];
            }
            dft_rec(in, 1, out, ny, sign);
            for (int y = 0; y < ny; ++y) {
                double* e = data + 2 * (((size_t)x * ny + y) * nz + z);
                e[0] = out[2 * y]; e[1] = out[2 * y + 1];
            }
        }
    /* along x */
    for (int y = 0; y < ny; ++y)
        for (int z = 0; z < nz; ++z) {
            for (int x = 0; x < nx; ++x) {
                double* e = data + 2 * (((size_t)x * ny + y) * nz + z);
                in[2 * x] = e[0]; in[2 * x + 1] = e[1];
            }
            dft_rec(in, 1, out, nx, sign);
            for (int x = 0; x < nx; ++x) {
                double* e = data + 2 * (((size_t)x * ny + y) * nz + z);
                e[0] = out[2 * x]; e[1] = out[2 * x + 1];
            }
        }
    free(in); free(out);
    return 0;
}

/* -------------------------------------------------------------------- PME */
/* BSpline::set (base/BSpline.cpp:64-117) */
static void bspline_set(int order, double w, double* theta, double* dtheta)
{
    if (order == 1) { theta[0] = 1; dtheta[0] = 0; return; }
    if (order == 2) { theta[1] = w; theta[0] = 1.0 - w; dtheta[1] = 1; dtheta[0] = -1; return; }
    theta[order - 1] = 0.0;
    theta[1] = w;
    theta[0] = 1.0 - w;
    for (int k = 2; k < order - 1; k++) {
        double div = 1.0 / k;
        theta[k] = div * w * theta[k - 1];
        for (int j = 1; j < k; j++)
            theta[k - j] = div * ((w + j) * theta[k - j - 1] + (k + 1 - j - w) * theta[k - j]);
        theta[0] = div * (1 - w) * theta[0];
    }
    dtheta[0] = -theta[0];
    for (int j = 1; j <= order - 1; j++)
        dtheta[j] = theta[j - 1] - theta[j];
    double div = 1.0 / (order - 1.0);
    theta[order - 1] = div * w * theta[order - 2];
    for (int j = 1; j < order - 1; j++)
        theta[order - 1 - j] = div * ((w + j) * theta[order - j - 2] + (order - j - w) * theta[order - 1 - j]);
    theta[0] = div * (1 - w) * theta[0];
}

/* Grid::dftmod (base/Grid.h:650-665) */
static void dftmod(int order, int n, const double* interp, double* mod)
{
    for (unsigned int i = 0; i < (unsigned)n; i++) {
        double sumCos = 0.0, sumSin = 0.0;
        for (unsigned int j = 0; j < (unsigned)order; j++) {
            double x = PMO_PI * 2.0 * i * j / (double)n;
            sumCos += interp[j] * cos(x);
            sumSin += interp[j] * sin(x);
        }
        mod[i] = 1.0 / (sumCos * sumCos + sumSin * sumSin);
    }
}

/* NonbondedPMEwaldSystemForce::evaluate (NonbondedPMEwaldSystemForce.h:271-349)
 * with initialize (:499-648), correctionTerm (:942-981), realTerm (:658-768),
 * reciprocalTerm (:879-932) and the Grid<BSpline> members (base/Grid.h). */
int pmo_pme_force(const pmo_system* s, const pmo_pme_params* p, double* forces, pmo_result* r)
{
    pbc_t b; pbc_set(&b, s->box);
    if (!b.orth) return -1;
    int N = s->n_atoms;
    double LX = b.e1.x, LY = b.e2.y, LZ = b.e3.z, V = b.V;
    double alpha = p->alpha, rc = p->cutoff;
    if (alpha <= 0.0) {
        alpha = 1.0;
        while (erfc(alpha * rc) / rc >= p->accuracy) alpha *= 2.0;
        double low = 0., high = alpha;
        for (unsigned int i = 0; i < 100; ++i) {
            alpha = 0.5 * (low + high);
            if (erfc(alpha * rc) / rc >= p->accuracy) low = alpha; else high = alpha;
        }
    }
    r->alpha = alpha;
    double alpha2 = alpha * alpha;
    double two_alpha_pi = 2.0 * alpha / sqrt(PMO_PI);
    double rc2 = rc * rc;

    double self = 0.0, charged = 0.0;
    if (p->correction) {
        double q = 0.0;
        for (int i = 0; i < N; i++) q += s->q[i] * s->q[i];
        self = -q * alpha / sqrt(PMO_PI);
        q = 0.0;
        for (int i = 0; i < N; i++) q += s->q[i];
        if (fabs(q * 0.00268283) > 1.0e-5) charged = -PMO_PI / (2.0 * V * alpha2) * q * q;
    }

    double intra = 0.0;
    if (p->correction) {
        for (int k = 0; k < s->n_excl; k++) {
            int a1 = s->excl[3 * k], a2 = s->excl[3 * k + 1], cls = s->excl[3 * k + 2];
            double rSquared;
            v3 rij = pbc_min_diff(&b, vload(s->pos + 3 * a1), vload(s->pos + 3 * a2), &rSquared);
            double qq = s->q[a1] * s->q[a2];
            if (cls == PMO_EXCL_MODIFIED) qq *= 1 - s->csf;
            double rr_ = sqrt(rSquared);
            double rr = 1 / rr_;
            double e = erf(alpha * rr_) * rr;
            intra -= qq * e;
            v3 fij = vmul(rij, (qq * (two_alpha_pi * exp(-alpha2 * rSquared) - e) * rr * rr));
            double* f1 = forces + 3 * a1; double* f2 = forces + 3 * a2;
            f1[0] -= fij.x; f1[1] -= fij.y; f1[2] -= fij.z;
            f2[0] += fij.x; f2[1] += fij.y; f2[2] += fij.z;
            if (!s->no_virial) add_virial(r->virial, fij, rij);
        }
        if (!s->no_virial) { r->virial[0] += charged; r->virial[4] += charged; r->virial[8] += charged; }
    }

    double ereal = 0.0;
    if (p->real) {
        /* realTerm: cell pairs x lattice images (buildLatticeVectors,
         * PeriodicBoundaryConditions.cpp:80-110), Cutoff switching. */
        cells_t c; cells_build(&c, &b, s);
        excl_t ex; excl_build(&ex, s);
        cell3* deltas = NULL;
        int nd = build_deltas(&c, rc, &deltas);
        /* lattice vectors with |L| <= 2 rc, sorted by norm, (0,0,0) first */
        int bK = (int)floor(rc / fabs(LX) + 1.0), bL = (int)floor(rc / fabs(LY) + 1.0),
            bM = (int)floor(rc / fabs(LZ) + 1.0);
        int cap = (2 * bK + 1) * (2 * bL + 1) * (2 * bM + 1);
        double* lat = (double*)malloc(sizeof(double) * 3 * cap);
        double* nrm = (double*)malloc(sizeof(double) * cap);
        int nl = 0;
        for (int k = -bK; k <= bK; k++)
            for (int l = -bL; l <= bL; l++)
                for (int m = -bM; m <= bM; m++)
                    if (k != 0 || l != 0 || m != 0) {
                        v3 co = vadd(vadd(vmul(b.e1, k), vmul(b.e2, l)), vmul(b.e3, m));
                        if (sqrt(vnorm2(co)) <= 2 * rc) {
                            lat[3 * nl] = co.x; lat[3 * nl + 1] = co.y; lat[3 * nl + 2] = co.z;
                            nrm[nl] = vnorm2(co); nl++;
                        }
                    }
        /* stable insertion sort by norm (std::sort is not stable, but the
         * reference's comparator only orders by norm; equal-norm images give
         * equal contributions up to summation order) */
        for (int a = 1; a < nl; ++a) {
            double kn = nrm[a]; double kv[3] = {lat[3 * a], lat[3 * a + 1], lat[3 * a + 2]};
            int z = a - 1;
            while (z >= 0 && nrm[z] > kn) {
                nrm[z + 1] = nrm[z]; memcpy(lat + 3 * (z + 1), lat + 3 * z, sizeof(double) * 3); z--;
            }
            nrm[z + 1] = kn; memcpy(lat + 3 * (z + 1), kv, sizeof(double) * 3);
        }
        int ntot = nl + 1;
        double* L = (double*)malloc(sizeof(double) * 3 * ntot);
        L[0] = L[1] = L[2] = 0.0;
        memcpy(L + 3, lat, sizeof(double) * 3 * nl);
        free(lat); free(nrm);
        term_t cutsw; term_init(&cutsw, PMO_POT_NONE, PMO_SW_CUTOFF, 0, rc, alpha);
        int ncell = c.nx * c.ny * c.nz;
        for (int A = 0; A < ncell; ++A) {
            if (c.head[A] < 0) continue;
            int ax = A / (c.ny * c.nz), ay = (A / c.nz) % c.ny, az = A % c.nz;
            for (int kd = -1; kd < nd; ++kd) {
                int B = A;
                if (kd >= 0) {
                    int bx = (ax + deltas[kd].x + c.maxNX) % c.nx;
                    int by = (ay + deltas[kd].y + c.maxNY) % c.ny;
                    int bz = (az + deltas[kd].z + c.maxNZ) % c.nz;
                    B = (bx * c.ny + by) * c.nz + bz;
                    if (c.head[B] < 0 || B < A) continue;
                }
                int notSame = B != A;
                for (int i = c.head[A]; i != -1; i = c.next[i]) {
                    double qi = s->q[i];
                    v3 ri = vload(s->pos + 3 * i), fi = mk(0, 0, 0);
                    int mi = s->mol[i];
                    for (int j = notSame ? c.head[B] : i; j != -1; j = c.next[j]) {
                        double d2dummy;
                        v3 rijMin = pbc_min_diff(&b, ri, vload(s->pos + 3 * j), &d2dummy);
                        int mj = s->mol[j];
                        double qj = s->q[j];
                        int same = mi == mj;
                        int excl = same ? excl_check(&ex, i, j) : PMO_EXCL_NONE;
                        if (i == j) excl = PMO_EXCL_FULL;
                        for (int k = 0; k < ntot; k++) {
                            if (excl == PMO_EXCL_FULL) { excl = PMO_EXCL_NONE; continue; }
                            v3 rij = vadd(rijMin, vload(L + 3 * k));
                            double rSquared = vnorm2(rij);
                            if (rSquared > rc2) continue;
                            double rr_ = sqrt(rSquared);
                            double qq = qi * qj;
                            if (excl == PMO_EXCL_MODIFIED) qq *= s->csf;
                            double rr = 1.0 / rr_;
                            double ar = alpha * rr_;
                            double e = qq * exp(-ar * ar);
                            double energy = pmo_poly5(ar) * e * rr;
                            double force = ((energy + two_alpha_pi * e) * rr * rr);
                            double sv, sd;
                            term_switch(&cutsw, rSquared, &sv, &sd);
                            force = force * sv - energy * sd;
                            energy = energy * sv;
                            ereal += energy;
                            v3 fij = vmul(rij, force);
                            fi = vsub(fi, fij);
                            double* fj = forces + 3 * j;
                            fj[0] += fij.x; fj[1] += fij.y; fj[2] += fij.z;
                            if (!same && s->mol_pos) {
                                /* realTerm (NonbondedPMEwaldSystemForce.h:750-757) */
                                add_virial(r->virial, fij, rij);
                                double dd;
                                add_virial(r->mol_virial, fij,
                                           pbc_min_diff(&b, vload(s->mol_pos + 3 * (size_t)mi),
                                                        vload(s->mol_pos + 3 * (size_t)mj), &dd));
                            } else if (!s->no_virial) {
                                add_virial(r->virial, fij, rij);
                            }
                            excl = PMO_EXCL_NONE;
                        }
                    }
                    forces[3 * i] += fi.x; forces[3 * i + 1] += fi.y; forces[3 * i + 2] += fi.z;
                }
            }
        }
        free(L); free(deltas); free(ex.e); cells_free(&c);
    }

    double erecip = 0.0;
    if (p->reciprocal) {
        /* Grid::initialize (base/Grid.h:557-648) */
        int NX = p->grid[0], NY = p->grid[1], NZ = p->grid[2], P = p->order;
        int offX = -(P - 1) / 2 + NX, offY = -(P - 1) / 2 + NY, offZ = -(P - 1) / 2 + NZ;
        double Wr = 1.0 / LX, Lr = 1.0 / LY, Hr = 1.0 / LZ;
        double Vg = LX * LY * LZ;
        double HXr = NX / LX, HYr = NY / LY, HZr = NZ / LZ;
        double fac = PMO_PI * PMO_PI / (alpha * alpha);
        double* expX = (double*)malloc(sizeof(double) * NX);
        double* expY = (double*)malloc(sizeof(double) * NY);
        double* expZ = (double*)malloc(sizeof(double) * NZ);
        for (unsigned i = 0; i < (unsigned)NX; i++) {
            int i0 = i <= (unsigned)NX / 2 ? (int)i : (int)i - NX;
            expX[i] = exp(-fac * ((i0 * Wr) * (i0 * Wr)));
        }
        for (unsigned j = 0; j < (unsigned)NY; j++) {
            int j0 = j <= (unsigned)NY / 2 ? (int)j : (int)j - NY;
            expY[j] = exp(-fac * ((j0 * Lr) * (j0 * Lr)));
        }
        for (unsigned k = 0; k <= (unsigned)NZ / 2; k++) {
            int k0 = (int)k;
            expZ[k] = exp(-fac * ((k0 * Hr) * (k0 * Hr)));
        }
        double* th0 = (double*)malloc(sizeof(double) * P);
        double* dth0 = (double*)malloc(sizeof(double) * P);
        bspline_set(P, 0.0, th0, dth0);
        double* modX = (double*)malloc(sizeof(double) * NX);
        double* modY = (double*)malloc(sizeof(double) * NY);
        double* modZ = (double*)malloc(sizeof(double) * NZ);
        dftmod(P, NX, th0, modX); dftmod(P, NY, th0, modY); dftmod(P, NZ, th0, modZ);

        size_t ng = (size_t)NX * NY * NZ;
        double* Q = (double*)calloc(2 * ng, sizeof(double));
        int* ipos = (int*)malloc(sizeof(int) * 3 * N);
        double* th = (double*)malloc(sizeof(double) * 6 * P * (size_t)N);
        /* anterpolateCharge (base/Grid.h:138-190) */
        for (int a = 0; a < N; a++) {
            double q = s->q[a];
            double x = s->pos[3 * a] * HXr, y = s->pos[3 * a + 1] * HYr, z = s->pos[3 * a + 2] * HZr;
            while (x < 0.0) x += NX;
            while (x >= (unsigned)NX) x -= NX;
            while (y < 0.0) y += NY;
            while (y >= (unsigned)NY) y -= NY;
            while (z < 0.0) z += NZ;
            while (z >= (unsigned)NZ) z -= NZ;
            int ix = (int)x, iy = (int)y, iz = (int)z;
            int i0 = ix + offX, j0 = iy + offY, k0 = iz + offZ;
            ipos[3 * a] = i0; ipos[3 * a + 1] = j0; ipos[3 * a + 2] = k0;
            double* tx = th + 6 * P * (size_t)a;
            double *dtx = tx + P, *ty = tx + 2 * P, *dty = tx + 3 * P, *tz = tx + 4 * P, *dtz = tx + 5 * P;
            bspline_set(P, x - ix, tx, dtx);
            bspline_set(P, y - iy, ty, dty);
            bspline_set(P, z - iz, tz, dtz);
            for (int i = 0; i < P; i++) {
                double aa = q * tx[i];
                int i1 = (i + i0) % NX;
                for (int j = 0; j < P; j++) {
                    double ab = aa * ty[j];
                    int j1 = (j + j0) % NY;
                    for (int k = 0; k < P; k++) {
                        int k1 = (k + k0) % NZ;
                        Q[2 * (((size_t)i1 * NY + j1) * NZ + k1)] += ab * tz[k];
                    }
                }
            }
        }
        pmo_fft3d(Q, NX, NY, NZ, -1);
        /* scalarSum (base/Grid.h:276-389) */
        double energy = 0.0, vxx = 0.0, vxy = 0.0, vxz = 0.0, vyy = 0.0, vyz = 0.0, vzz = 0.0;
        double piVr = 1.0 / (PMO_PI * Vg);
        for (unsigned i = 0; i < (unsigned)NX; i++) {
            int i0 = i <= (unsigned)NX / 2 ? (int)i : (int)i - NX;
            double mi = i0 * Wr;
            double ex = expX[i] * piVr;
            for (unsigned j = 0; j < (unsigned)NY; j++) {
                int j0 = j <= (unsigned)NY / 2 ? (int)j : (int)j - NY;
                double mXY = modX[i] * modY[j];
                double mj = j0 * Lr;
                double mij = mi * mi + mj * mj;
                double exy = ex * expY[j];
                for (unsigned k = (i != 0 || j != 0 ? 0 : 1); k <= (unsigned)NZ / 2; k++) {
                    int k0 = (int)k;
                    double mk_ = k0 * Hr;
                    double m2 = mij + mk_ * mk_;
                    double theta = mXY * modZ[k] * exy * expZ[k] / m2;
                    double* w0 = Q + 2 * (((size_t)i * NY + j) * NZ + k);
                    double qv = w0[0] * w0[0] + w0[1] * w0[1];
                    double e = qv * theta;
                    double v = 2.0 * (1.0 / m2 + fac);
                    if (k > 0 && ((k != (unsigned)NZ / 2) || (NZ & 1))) {
                        e *= 2.0;
                        double* w = Q + 2 * ((((size_t)(NX - i) % NX) * NY + (NY - j) % NY) * NZ + (NZ - k) % NZ);
                        w[0] *= theta; w[1] *= theta;
                    }
                    energy += e;
                    vxx += e * (1.0 - v * mi * mi);
                    vxy -= e * (v * mi * mj);
                    vxz -= e * (v * mi * mk_);
                    vyy += e * (1.0 - v * mj * mj);
                    vyz -= e * (v * mj * mk_);
                    vzz += e * (1.0 - v * mk_ * mk_);
                    w0[0] *= theta; w0[1] *= theta;
                }
            }
        }
        Q[0] = 0.0; Q[1] = 0.0;
        double vrec[9] = {vxx * 0.5, vxy * 0.5, vxz * 0.5, vxy * 0.5, vyy * 0.5, vyz * 0.5,
                          vxz * 0.5, vyz * 0.5, vzz * 0.5};
        /* scalarSum's atomic and molecular virial (base/Grid.h:366-387); the
         * sums themselves are taken only when virial() is on (:341-349), so
         * without it the molecular virial gets zero here */
        if (!s->no_virial)
            for (int k = 0; k < 9; ++k) r->virial[k] += vrec[k];
        if (s->mol_pos && !s->no_virial)
            for (int k = 0; k < 9; ++k) r->mol_virial[k] += vrec[k];
        erecip = energy * 0.5;
        pmo_fft3d(Q, NX, NY, NZ, +1);
        /* interpolateForce (base/Grid.h:193-228) */
        for (int a = 0; a < N; a++) {
            int i0 = ipos[3 * a], j0 = ipos[3 * a + 1], k0 = ipos[3 * a + 2];
            double fx = 0.0, fy = 0.0, fz = 0.0;
            double* tx = th + 6 * P * (size_t)a;
            double *dtx = tx + P, *ty = tx + 2 * P, *dty = tx + 3 * P, *tz = tx + 4 * P, *dtz = tx + 5 * P;
            for (int i = 0; i < P; i++) {
                int i1 = (i + i0) % NX;
                for (int j = 0; j < P; j++) {
                    int j1 = (j + j0) % NY;
                    double xij = dtx[i] * ty[j];
                    double yij = tx[i] * dty[j];
                    double zij = tx[i] * ty[j];
                    for (int k = 0; k < P; k++) {
                        int k1 = (k + k0) % NZ;
                        double term = Q[2 * (((size_t)i1 * NY + j1) * NZ + k1)];
                        fx -= term * xij * tz[k];
                        fy -= term * yij * tz[k];
                        fz -= term * zij * dtz[k];
                    }
                }
            }
            double q = s->q[a];
            v3 fi = mk(fx * HXr * q, fy * HYr * q, fz * HZr * q);
            forces[3 * a] += fi.x;
            forces[3 * a + 1] += fi.y;
            forces[3 * a + 2] += fi.z;
            if (s->mol_pos) {
                /* reciprocalTerm (NonbondedPMEwaldSystemForce.h:905-924): the
                 * atom's reciprocal force against its offset from the
                 * molecule's position (Darden et al., J. Chem. Phys. 103, 8577) */
                double dd;
                v3 ria = pbc_min_pos(&b, vload(s->pos + 3 * a));
                v3 mri = pbc_min_diff(&b, ria, vload(s->mol_pos + 3 * (size_t)s->mol[a]), &dd);
                add_virial(r->mol_virial, fi, mri);
            }
        }
        free(expX); free(expY); free(expZ); free(th0); free(dth0);
        free(modX); free(modY); free(modZ); free(Q); free(ipos); free(th);
    }

    double e = ereal + erecip + intra + 0.0 + self + charged;
    r->coulomb += e;
    r->e_real += ereal; r->e_recip += erecip; r->e_intra += intra;
    r->e_self += self; r->e_charged += charged;
    return 0;
}

/* ------------------------------------------------------------ Hessian */
/* Switching-function Hessians (C2SwitchingFunction.cpp:45-53,
 * C1SwitchingFunction.cpp:39-49): the matrix is s_i I + s_r rr^T. */
static void switch_hessian(const term_t* t, double a, double* s_i, double* s_r)
{
    if (t->sw == PMO_SW_C2) {
        double tm1 = t->cut2 - t->on2;
        double tm2 = tm1 * tm1 * tm1;
        *s_i = 12.0 * (a - t->cut2) * (a - t->on2) / tm2;
        *s_r = 24.0 * (2.0 * a - t->cut2 - t->on2) / tm2;
    } else {   /* C1 */
        double r = sqrt(a);
        double tm1 = 1.5 / (t->cut * r);
        double tm2 = 1.5 / (t->cut * t->cut * t->cut) * r;
        *s_i = -tm1 + tm2;
        *s_r = (tm1 + tm2) / a;
    }
}

/* Dense Hessian of the pair terms as integrators/Hessian.cpp:456-623 builds
 * it: for every pair i < j that is not FULL-excluded, with rij the minimal
 * difference, ReducedHessLennardJones (forces/ReducedHessLennardJones.cpp:7-51)
 * or ReducedHessCoulomb (forces/ReducedHessCoulomb.cpp:8-43) gives
 *   H = (tm1 I + tm2 rr) S + Shess E_raw - 2 F_raw S' rr
 * (E_raw, F_raw and Shess only where 0 < S < 1), added to the ii and jj
 * blocks and subtracted from the ij and ji blocks.  H: 3N x 3N, +=.
 * Returns -1 for terms Hessian.cpp has no block for (Ewald real; switches
 * other than Universal, C1, C2). */
int pmo_pair_hessian(const pmo_system* s, const pmo_cutoff_params* p, int vacuum, double* H)
{
    pair_ctx pc;
    pair_ctx_init(&pc, s, p);
    for (int k = 0; k < p->n_terms; ++k) {
        int bad = (pc.t[k].pot != PMO_POT_LJ && pc.t[k].pot != PMO_POT_COULOMB) ||
                  (pc.t[k].sw != PMO_SW_UNIVERSAL && pc.t[k].sw != PMO_SW_C1 && pc.t[k].sw != PMO_SW_C2);
        if (bad) { pair_ctx_free(&pc); return -1; }
    }
    pbc_t b;
    if (!vacuum) pbc_set(&b, s->box);
    excl_t ex; excl_build(&ex, s);
    const size_t n3 = 3 * (size_t)s->n_atoms;
    for (int i = 0; i < s->n_atoms; ++i)
        for (int j = i + 1; j < s->n_atoms; ++j) {
            int excl = s->mol[i] == s->mol[j] ? excl_check(&ex, i, j) : PMO_EXCL_NONE;
            if (excl == PMO_EXCL_FULL) continue;
            double a;
            v3 r;
            if (vacuum) { r = vsub(vload(s->pos + 3 * j), vload(s->pos + 3 * i)); a = vnorm2(r); }
            else r = pbc_min_diff(&b, vload(s->pos + 3 * i), vload(s->pos + 3 * j), &a);
            double rr[3] = {r.x, r.y, r.z};
            double hi = 0.0, hr = 0.0;   /* H = hi I + hr rr^T */
            for (int k = 0; k < p->n_terms; ++k) {
                const term_t* t = &pc.t[k];
                double sv = 1.0, sd = 0.0, shi = 0.0, shr = 0.0, e = 0.0, f = 0.0;
                if (t->sw != PMO_SW_UNIVERSAL) {
                    term_switch(t, a, &sv, &sd);
                    if (sv > 0.0 && sv < 1.0) {
                        term_potential(t, s, i, j, excl, a, 1.0 / a, &e, &f);
                        switch_hessian(t, a, &shi, &shr);
                    }
                }
                double ti, tr;
                if (t->pot == PMO_POT_LJ) {
                    const double* lp = s->lj + 4 * ((size_t)s->type[i] * s->n_types + s->type[j]);
                    double A = excl == PMO_EXCL_MODIFIED ? lp[2] : lp[0];
                    double B = excl == PMO_EXCL_MODIFIED ? lp[3] : lp[1];
                    double a4 = a * a * a * a, a5 = a4 * a, a7 = a4 * a * a * a, a8 = a4 * a4;
                    ti = 6 * B / a4 - 12 * A / a7;
                    tr = -48 * B / a5 + 168 * A / a8;
                } else {
                    double csf = excl == PMO_EXCL_MODIFIED ? s->csf : 1.0;
                    double tm1 = -csf * s->q[i] * s->q[j] / a / sqrt(a);
                    ti = tm1;
                    tr = -3.0 / a * tm1;
                }
                hi += ti * sv + shi * e;
                hr += tr * sv + shr * e - 2.0 * f * sd;
            }
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) {
                    double v = (l == m ? hi : 0.0) + hr * rr[l] * rr[m];
                    H[(3 * (size_t)i + l) * n3 + 3 * (size_t)i + m] += v;
                    H[(3 * (size_t)j + l) * n3 + 3 * (size_t)j + m] += v;
                    H[(3 * (size_t)i + l) * n3 + 3 * (size_t)j + m] -= v;
                    H[(3 * (size_t)j + l) * n3 + 3 * (size_t)i + m] -= v;
                }
        }
    free(ex.e);
    return 0;
}
