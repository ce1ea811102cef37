// pmgpu_api.cu -- the C ABI (include/pmgpu.h) over the libpmgpu kernels.
//
// Host-side set-up follows the reference's constructors and initialize()
// methods (cited per function); everything per evaluation runs on the
// system's CUDA stream.  No CPU fallback: a missing or failing device is an
// error status.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/pmgpu.h"
#include "pm_kernels.h"

using namespace pm;

static const double kPi = 3.14159265358979323846;   // Constant::M_PI (base/pmconstants.cpp:56)
static const double kEpsilon = 1.0e-14;              // Constant::EPSILON (base/pmconstants.cpp:45)
// status word, list count and need, chunk count and need, work counter, pad,
// then 11 int64 energy/virial sums
static const size_t kSmallBytes = 64 + 8 * kERec;
// the evaluation's output slots: pmgpu_energies_mol (LJ, Coulomb, virial,
// molecular virial)
static const int kEOut = 20;

// evaluation phases timed in profiling mode (pmgpu_phase_times)
enum { kPhaseBin = 0, kPhasePair, kPhaseCorrection, kPhaseSpread, kPhaseFft, kPhaseGather, kPhaseFinalize,
       kPhaseList, kPhaseEnergy64, kNumPhases };

struct ProfMark {
    int phase;
    cudaEvent_t b, e;
};

struct GraphKey {
    std::vector<long long> ids;
    const void* pos = nullptr;
    const void* fout = nullptr;
    const void* energy = nullptr;
    unsigned flags = 0;
    int box_version = -1, topo_version = -1, buf_version = -1;
    int reuse = 0;                     // the evaluation keeps the pair list of an earlier one
    bool operator==(const GraphKey& o) const
    {
        return ids == o.ids && pos == o.pos && fout == o.fout && energy == o.energy && flags == o.flags &&
               box_version == o.box_version && topo_version == o.topo_version && buf_version == o.buf_version &&
               reuse == o.reuse;
    }
};

static long long g_next_force_id = 1;

struct pmgpu_system {
    int device = 0;
    cudaStream_t stream = nullptr;
    // PME runs on a second, higher-priority stream beside the pair kernels
    // (forked after binning, joined before finalize)
    cudaStream_t side = nullptr;
    // two more branches of the PME work: the correction term, and the FP64
    // energy transform of a mixed force (both beside the FP32 FFT chain)
    cudaStream_t side2 = nullptr, side3 = nullptr;
    cudaEvent_t ev_spread = nullptr, ev_e64 = nullptr, ev_corr = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_pair = nullptr, ev_near = nullptr;   // the last near-pair energies on the side stream
    std::string err;
    long long launches = 0;
    // topology
    int n = 0, t = 0, e = 0;
    double csf = 1.0;
    std::vector<double> q;
    std::vector<int> excl_pairs, excl_cls;
    double* d_q = nullptr;
    int* d_type = nullptr;
    int* d_mol = nullptr;
    int n_mol = 0;                     // molecule ids 0 .. n_mol - 1
    // GenericTopology::molecules[m].position (pmgpu_set_molecule_positions),
    // read by the molecular virial; records of its kernels (kMRec)
    double* d_molpos = nullptr;
    bool molpos_set = false;
    double* d_mrec = nullptr;
    int mrec_cap = 0;
    // bond constraints of the resident Leapfrog (pmgpu_set_constraints):
    // clusters of constraints sharing atoms, SHAKE's last positions
    int n_cons = 0, n_ccl = 0;
    int* d_cl_start = nullptr;
    int2* d_cons_atoms = nullptr;
    double* d_cons_rest = nullptr;
    double* d_cons_last = nullptr;
    int* d_cons_hits = nullptr;
    double shake_eps = 0.0, rattle_eps = 0.0;
    int shake_iter = 0, rattle_iter = 0;
    float4* d_ljn = nullptr;
    float4* d_ljm = nullptr;
    double4* d_ljd = nullptr;
    uint32_t* d_xfull = nullptr;
    uint32_t* d_xmod = nullptr;
    int* d_xrow = nullptr;
    int2* d_xent = nullptr;
    int2* d_epairs = nullptr;
    int* d_ecls = nullptr;
    // box
    bool box_set = false;
    int box_version = 0;
    double box[12];
    double cell_size = 0.0;
    Pbc pbc;
    CellGrid grid;
    // per-evaluation buffers
    double* d_pos = nullptr;
    double* d_fout = nullptr;
    double* d_energy = nullptr;        // kEOut
    double* h_energy = nullptr;        // pinned kEOut
    int* h_status = nullptr;           // pinned: the status word, copied back with the results
    unsigned long long* d_facc32 = nullptr;   // mixed (2^32): 3N pair forces + 3N other (d_facc32p)
    unsigned long long* d_facc32p = nullptr;
    unsigned long long* d_facc40 = nullptr;   // FP64 (2^40)
    // PME forces in atom order (PME needs no binning, so it runs beside it):
    // 3N mixed (2^32) then 3N FP64 (2^40)
    unsigned long long* d_faccA = nullptr;
    int* d_cell_lin = nullptr;
    int* d_cell3 = nullptr;
    int* d_counts = nullptr;
    int* d_start = nullptr;
    int* d_cstart = nullptr;
    float4* d_cbox = nullptr;
    int cbox_cap = 0;
    int* d_ccell = nullptr;
    int* d_skey = nullptr;
    int* d_tmp = nullptr;
    int* d_sorted = nullptr;
    int* d_slot = nullptr;
    float4* d_spos = nullptr;
    float4* d_slo = nullptr;
    int4* d_smeta = nullptr;
    double4* d_spos64 = nullptr;
    // small per-evaluation scratch, zeroed by one memset: status word,
    // cluster-pair list and chunk counters, int64 energy/virial sums
    void* d_small = nullptr;
    int* d_status = nullptr;
    int* d_plist_count = nullptr;
    int* d_plist_need = nullptr;
    int* d_chunk_count = nullptr;
    int* d_chunk_need = nullptr;
    int* d_chunk_next = nullptr;
    unsigned long long* d_efix = nullptr;
    // cluster-pair list and chunks of the mixed kernel
    int2* d_plist = nullptr;
    long long plist_cap = 0;
    long long plist_need = 0;          // reported by the last evaluation that overflowed
    int4* d_chunks = nullptr;
    long long chunk_cap = 0;
    long long chunk_need = 0;
    int2* d_near = nullptr;            // near pairs of the mixed kernels (FP64 energies)
    long long near_cap = 0;
    long long near_need = 0;
    int ncell_cap = 0;
    double* d_erec = nullptr;
    int erec_cap = 0;
    // column-cluster path of the mixed pair forces: the grid of the box
    // (col_set_grid), per-atom and per-slot buffers; disabled for good when a
    // column or cluster exceeded the path's limits (the cell path takes over)
    ColGrid cg;
    bool col_grid = false;
    bool col_grid_stale = true;        // box or atom count changed since col_set_grid
    bool col_disabled = false;
    bool col_just_disabled = false;
    bool eval_use_col = false;         // the evaluation being enqueued uses the column path
    // reused pair lists (pmgpu_set_pair_list): the column list built with the
    // cutoff plus a skin is kept for rebuild_every evaluations while no atom
    // moves more than half the skin
    double list_skin = 0.0;
    int list_every = 1;
    bool list_valid = false;
    bool list_just_invalidated = false;
    int evals_since_build = 0;
    std::vector<long long> list_ids;   // the forces the list was built for
    long long list_builds = 0;
    bool eval_reuse = false;           // the evaluation being enqueued reuses the list
    int last_layout = 0;               // pmgpu_pair_layout of the last evaluation with mixed cutoff forces
    ColGrid eval_cg;                   // its grid with the reach of its cutoffs
    unsigned* d_qfix = nullptr;
    int* d_colid = nullptr;
    int* d_ctmp = nullptr;
    int* d_cslot = nullptr;
    int* d_ccounts = nullptr;
    int* d_colstart = nullptr;
    int* d_ccstart = nullptr;
    int* d_zidx = nullptr;          // z index of every column's j-clusters (kZIndex ints per column)
    int col_ncol_cap = 0;
    int4* d_cq = nullptr;
    int4* d_cm = nullptr;
    float4* d_ibox = nullptr;
    float4* d_jbox = nullptr;
    int* d_ccol = nullptr;
    int4* d_corg = nullptr;
    unsigned long long* d_facc32c = nullptr;
    int col_ncl_cap = 0;
    double* d_acc0 = nullptr;          // 3N: the caller's force accumulator as pmgpu_evaluate received it
    double* h_fbuf = nullptr;          // pinned 3N: the forces' copy back for a pageable accumulator
    bool binned = false;
    std::set<pmgpu_force*> forces;     // live forces made on this system
    int topo_version = 0;
    int buf_version = 0;               // bumped when a per-evaluation buffer moves
    pmgpu_tuning tuning = {16, 0, 16, 1, 0, 0.0};   // launch shapes (pmgpu_set_tuning, pmgpu_autotune)
    // CUDA graphs of the last few distinct evaluations (force groups,
    // buffers, flags), replayed when the key matches; the least recently
    // used is replaced (a multiple-time-step integrator alternates groups)
    bool use_graphs = true;
    struct GraphEntry {
        GraphKey key;
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;
        unsigned long long last_use = 0;
    };
    std::vector<GraphEntry> graphs;
    unsigned long long graph_clock = 0;
    // profiling
    bool profiling = false;
    std::vector<cudaEvent_t> prof_pool;
    size_t prof_next = 0;
    std::vector<ProfMark> prof_marks;
    double prof_ms[kNumPhases] = {0};
    long long prof_evals = 0;
};

struct pmgpu_force {
    pmgpu_system* sys = nullptr;
    long long id = g_next_force_id++;   // never reused (graph keys)
    int kind = 0;   // 0 cutoff, 1 PME
    int precision = 0;
    pmgpu_cutoff_params cp;
    pmgpu_pme_params pp;
    // cutoff
    int combo = -1;
    int box_version = -1;
    int topo_version = -1;           // PME: the self and charged-system terms depend on the charges
    int nd = 0;
    int4* d_deltas = nullptr;
    float4* d_doff = nullptr;
    int4* d_hdeltas = nullptr;      // half shell of the mixed kernel
    float4* d_hoff = nullptr;
    float4* d_hoff_lo = nullptr;
    double4* d_hoff64 = nullptr;
    int nh = 0;
    int half_rule = 0;
    int wrap = 0;
    TermF tf[2];
    TermD td[2];
    double* d_tab64[2] = {nullptr, nullptr};   // look-up tables of table potentials
    float* d_tab32[2] = {nullptr, nullptr};
    double cut2 = 0.0;
    // PME
    double alpha = 0.0;
    int kzh = 0;
    long long* d_qgrid = nullptr;
    void* d_cgrid = nullptr;
    void* d_rgrid = nullptr;
    void* d_tw = nullptr;
    // Hessian-vector product: the grids of the directional-derivative charges
    // (allocated by the first pmgpu_adjoint with v)
    long long* d_hq = nullptr;
    void* d_hc = nullptr;
    void* d_hr = nullptr;
    void* d_cgrid64 = nullptr;      // mixed: FP64 half spectrum and twiddles of the energy transform
    void* d_tw64 = nullptr;
    double* d_bfac = nullptr;
    double* d_efac = nullptr;
    double self_energy = 0.0, charged_energy = 0.0;
    int twx = 0, twy = 0, twz = 0;
    // -real: the real-space term as an internal CoulombEwaldReal / Cutoff
    // pair force (owned by this force, evaluated before it) when every box
    // edge exceeds 2 Rc; otherwise realTerm's lattice images (k_pme_real_lattice)
    pmgpu_force* real_sub = nullptr;
    double4* d_lattice = nullptr;
    int n_lattice = 0;
};

// PMEwald -real in a box with an edge <= 2 Rc: buildLatticeVectors gives
// images besides (0, 0, 0), so realTerm is the lattice kernel, not the pair force
static bool pme_needs_lattice(const pmgpu_force* f)
{
    if (f->kind != 1 || !f->pp.real || !f->sys->box_set) return false;
    const double* b = f->sys->box;
    const double rc2 = 2.0 * f->pp.cutoff;
    return !(std::fabs(b[0]) > rc2 && std::fabs(b[4]) > rc2 && std::fabs(b[8]) > rc2);
}

// ------------------------------------------------------------------ helpers
static int fail(pmgpu_system* s, int code, const std::string& msg)
{
    if (s) s->err = msg;
    return code;
}

static int cuda_fail(pmgpu_system* s, cudaError_t e, const char* where)
{
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    if (s) s->err = m;
    return e == cudaErrorMemoryAllocation ? PMGPU_ERR_NOMEM : PMGPU_ERR_CUDA;
}

#define CK(call, where)                                         \
    do {                                                        \
        cudaError_t _e = (call);                                \
        if (_e != cudaSuccess) return cuda_fail(sys, _e, where); \
    } while (0)

template <typename T>
static cudaError_t dalloc(T** p, size_t count)
{
    if (*p) { cudaFree(*p); *p = nullptr; }
    if (count == 0) count = 1;
    return cudaMalloc((void**)p, sizeof(T) * count);
}

template <typename T>
static void dfree(T*& p)
{
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// ------------------------------------------------------------------ context
extern "C" int pmgpu_system_create(int device, pmgpu_system** out)
{
    if (!out) return PMGPU_ERR_ARG;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= device || device < 0) return PMGPU_ERR_CUDA;
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return PMGPU_ERR_CUDA;
    pmgpu_system* sys = new pmgpu_system();
    sys->device = device;
    e = cudaStreamCreateWithFlags(&sys->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete sys; return PMGPU_ERR_CUDA; }
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&sys->side, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&sys->side2, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaStreamCreateWithPriority(&sys->side3, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&sys->ev_spread, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sys->ev_e64, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sys->ev_corr, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sys->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sys->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sys->ev_pair, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&sys->ev_near, cudaEventDisableTiming) != cudaSuccess) {
        cudaStreamDestroy(sys->stream);
        delete sys;
        return PMGPU_ERR_CUDA;
    }
    if (cudaMalloc(&sys->d_small, kSmallBytes) != cudaSuccess ||
        cudaMalloc((void**)&sys->d_energy, sizeof(double) * kEOut) != cudaSuccess ||
        cudaMallocHost((void**)&sys->h_energy, sizeof(double) * kEOut) != cudaSuccess ||
        cudaMallocHost((void**)&sys->h_status, sizeof(int)) != cudaSuccess) {
        delete sys;
        return PMGPU_ERR_NOMEM;
    }
    sys->d_status = (int*)sys->d_small;
    sys->d_plist_count = sys->d_status + 1;
    sys->d_plist_need = sys->d_status + 2;
    sys->d_chunk_count = sys->d_status + 3;
    sys->d_chunk_need = sys->d_status + 4;
    sys->d_chunk_next = sys->d_status + 5;
    sys->d_efix = (unsigned long long*)((char*)sys->d_small + 64);   // ints 8..15: binning
    *out = sys;
    return PMGPU_OK;
}

static void free_atom_buffers(pmgpu_system* s)
{
    dfree(s->d_q); dfree(s->d_type); dfree(s->d_mol); dfree(s->d_ljn); dfree(s->d_ljm); dfree(s->d_ljd);
    dfree(s->d_molpos); s->molpos_set = false;
    dfree(s->d_slo); dfree(s->d_skey);
    dfree(s->d_xfull); dfree(s->d_xmod); dfree(s->d_xrow); dfree(s->d_xent);
    dfree(s->d_epairs); dfree(s->d_ecls);
    dfree(s->d_pos); dfree(s->d_fout); dfree(s->d_facc32); dfree(s->d_facc40); dfree(s->d_faccA);
    s->d_facc32p = nullptr;   // second half of d_facc32
    dfree(s->d_cell_lin); dfree(s->d_cell3); dfree(s->d_tmp); dfree(s->d_sorted); dfree(s->d_slot);
    dfree(s->d_spos); dfree(s->d_smeta); dfree(s->d_spos64);
    dfree(s->d_qfix); dfree(s->d_colid); dfree(s->d_ctmp); dfree(s->d_cslot);
}

static void free_col_buffers(pmgpu_system* s)
{
    dfree(s->d_ccounts); dfree(s->d_colstart); dfree(s->d_ccstart); dfree(s->d_zidx);
    dfree(s->d_cq); dfree(s->d_cm); dfree(s->d_ibox); dfree(s->d_jbox); dfree(s->d_ccol); dfree(s->d_facc32c);
    dfree(s->d_corg);
    s->col_ncol_cap = 0;
    s->col_ncl_cap = 0;
}

static void free_force(pmgpu_force* f);

extern "C" int pmgpu_system_destroy(pmgpu_system* sys)
{
    if (!sys) return PMGPU_OK;
    cudaSetDevice(sys->device);
    cudaStreamSynchronize(sys->stream);
    // forces still alive belong to this system: release them too
    std::set<pmgpu_force*> live;
    live.swap(sys->forces);
    for (pmgpu_force* f : live) free_force(f);
    for (auto& g : sys->graphs) cudaGraphExecDestroy(g.exec);
    sys->graphs.clear();
    for (cudaEvent_t e : sys->prof_pool) cudaEventDestroy(e);
    free_atom_buffers(sys);
    free_col_buffers(sys);
    dfree(sys->d_counts); dfree(sys->d_start); dfree(sys->d_erec); dfree(sys->d_mrec);
    dfree(sys->d_cl_start); dfree(sys->d_cons_atoms); dfree(sys->d_cons_rest); dfree(sys->d_cons_last);
    dfree(sys->d_cons_hits);
    dfree(sys->d_small); dfree(sys->d_energy);
    dfree(sys->d_cstart); dfree(sys->d_cbox); dfree(sys->d_ccell); dfree(sys->d_plist); dfree(sys->d_chunks);
    dfree(sys->d_near);
    if (sys->h_energy) cudaFreeHost(sys->h_energy);
    if (sys->h_status) cudaFreeHost(sys->h_status);
    dfree(sys->d_acc0);
    if (sys->h_fbuf) cudaFreeHost(sys->h_fbuf);
    cudaEventDestroy(sys->ev_fork);
    cudaEventDestroy(sys->ev_join);
    cudaEventDestroy(sys->ev_pair);
    cudaEventDestroy(sys->ev_near);
    cudaEventDestroy(sys->ev_spread);
    cudaEventDestroy(sys->ev_e64);
    cudaEventDestroy(sys->ev_corr);
    cudaStreamDestroy(sys->side2);
    cudaStreamDestroy(sys->side3);
    cudaStreamDestroy(sys->side);
    cudaStreamDestroy(sys->stream);
    delete sys;
    return PMGPU_OK;
}

extern "C" int pmgpu_last_error(pmgpu_system* sys, char* buf, int len)
{
    if (!buf || len <= 0) return PMGPU_ERR_ARG;
    std::string m = sys ? sys->err : std::string("no system");
    snprintf(buf, (size_t)len, "%s", m.c_str());
    return PMGPU_OK;
}

extern "C" void* pmgpu_stream(pmgpu_system* sys) { return sys ? (void*)sys->stream : nullptr; }

extern "C" int pmgpu_set_profiling(pmgpu_system* sys, int enable)
{
    if (!sys) return PMGPU_ERR_ARG;
    cudaSetDevice(sys->device);
    CK(cudaStreamSynchronize(sys->stream), "sync");
    sys->profiling = enable != 0;
    sys->prof_marks.clear();
    sys->prof_next = 0;
    for (int k = 0; k < kNumPhases; ++k) sys->prof_ms[k] = 0.0;
    sys->prof_evals = 0;
    return PMGPU_OK;
}

extern "C" int pmgpu_phase_times(pmgpu_system* sys, double* ms, int n, long long* evals)
{
    if (!sys || !ms || n <= 0) return PMGPU_ERR_ARG;
    cudaSetDevice(sys->device);
    CK(cudaStreamSynchronize(sys->stream), "sync");
    long long bins = 0;
    for (const ProfMark& m : sys->prof_marks) {
        float t = 0.f;
        if (m.e && cudaEventElapsedTime(&t, m.b, m.e) == cudaSuccess) sys->prof_ms[m.phase] += t;
        if (m.phase == kPhaseBin) ++bins;
    }
    sys->prof_evals += bins;
    sys->prof_marks.clear();
    sys->prof_next = 0;
    for (int k = 0; k < n && k < kNumPhases; ++k) ms[k] = sys->prof_ms[k];
    for (int k = kNumPhases; k < n; ++k) ms[k] = 0.0;
    if (evals) *evals = sys->prof_evals;
    return PMGPU_OK;
}
extern "C" long long pmgpu_launch_count(pmgpu_system* sys) { return sys ? sys->launches : 0; }

// the outcome of the evaluations up to now from their status word st (read
// after the stream has drained)
static int status_result(pmgpu_system* sys, int st)
{
    if (st & kStatusOverflow)
        return fail(sys, PMGPU_ERR_OVERFLOW, "non-finite or out-of-range force (fixed-point range exceeded)");
    if (st & kStatusColumns) {
        // a column held more atoms, or an i-cluster spanned more of the box
        // height, than the column path takes: the cell-cluster path from now on
        if (!sys->col_disabled) {
            sys->col_disabled = true;
            sys->col_just_disabled = true;
            sys->buf_version++;
        }
        sys->list_valid = false;
        return fail(sys, PMGPU_ERR_CAPACITY, "column clusters out of range (the cell-cluster path is used next)");
    }
    if (st & kStatusListStale) {
        sys->list_valid = false;
        sys->list_just_invalidated = true;
        return fail(sys, PMGPU_ERR_CAPACITY, "an atom moved more than half the pair list's skin since the list was "
                                             "built (it is rebuilt at the next evaluation)");
    }
    if (st & kStatusListFull) {
        // list need, chunk count, chunk need, work counter, near count, near need
        int need[6] = {0, 0, 0, 0, 0, 0};
        CK(cudaMemcpy(need, sys->d_plist_need, sizeof(need), cudaMemcpyDeviceToHost), "status");
        sys->plist_need = std::max<long long>(sys->plist_need, need[0]);
        sys->chunk_need = std::max<long long>(sys->chunk_need, need[2]);
        sys->near_need = std::max<long long>(sys->near_need, need[5]);
        sys->list_valid = false;
        return fail(sys, PMGPU_ERR_CAPACITY, "cluster-pair list capacity exceeded (grown for the next evaluation)");
    }
    return PMGPU_OK;
}

extern "C" int pmgpu_synchronize(pmgpu_system* sys)
{
    if (!sys) return PMGPU_ERR_ARG;
    cudaSetDevice(sys->device);
    CK(cudaStreamSynchronize(sys->stream), "synchronize");
    int st = 0;
    CK(cudaMemcpy(&st, sys->d_status, sizeof(int), cudaMemcpyDeviceToHost), "status");
    return status_result(sys, st);
}

// ------------------------------------------------------------------ topology
extern "C" int pmgpu_set_topology(pmgpu_system* sys, int n_atoms, const double* scaled_charge,
                                  const int* type, const int* molecule, int n_types,
                                  const double* lj_table, int n_excl, const int* excl_pairs,
                                  const int* excl_class, const int* excl_check_class,
                                  double coulomb_scaling_factor)
{
    if (!sys) return PMGPU_ERR_ARG;
    if (n_atoms < 0 || n_types < 0 || n_excl < 0) return fail(sys, PMGPU_ERR_ARG, "negative size");
    if (n_atoms > 0 && (!scaled_charge || !type || !molecule)) return fail(sys, PMGPU_ERR_ARG, "null atom array");
    if (n_types > 0 && !lj_table) return fail(sys, PMGPU_ERR_ARG, "null Lennard-Jones table");
    if (n_excl > 0 && (!excl_pairs || !excl_class)) return fail(sys, PMGPU_ERR_ARG, "null exclusion array");
    int n_mol = 0;
    for (int i = 0; i < n_atoms; ++i) {
        if (type[i] < 0 || type[i] >= n_types) return fail(sys, PMGPU_ERR_ARG, "atom type out of range");
        if (molecule[i] < 0) return fail(sys, PMGPU_ERR_ARG, "negative molecule id");
        n_mol = std::max(n_mol, molecule[i] + 1);
    }
    cudaSetDevice(sys->device);
    CK(cudaStreamSynchronize(sys->stream), "set_topology");
    free_atom_buffers(sys);
    sys->topo_version++;
    for (auto& g : sys->graphs) cudaGraphExecDestroy(g.exec);
    sys->graphs.clear();
    if (n_atoms != sys->n) sys->n_cons = 0;   // constraints name atoms of the previous topology
    sys->n = n_atoms; sys->t = n_types; sys->e = n_excl; sys->csf = coulomb_scaling_factor;
    sys->n_mol = n_mol;
    sys->q.assign(scaled_charge, scaled_charge + n_atoms);
    sys->binned = false;
    int n = n_atoms;
    CK(dalloc(&sys->d_q, n), "alloc"); CK(dalloc(&sys->d_type, n), "alloc"); CK(dalloc(&sys->d_mol, n), "alloc");
    CK(cudaMemcpy(sys->d_q, scaled_charge, sizeof(double) * n, cudaMemcpyHostToDevice), "copy");
    CK(cudaMemcpy(sys->d_type, type, sizeof(int) * n, cudaMemcpyHostToDevice), "copy");
    CK(cudaMemcpy(sys->d_mol, molecule, sizeof(int) * n, cudaMemcpyHostToDevice), "copy");
    // Lennard-Jones table (LennardJonesParameterTable, T x T)
    size_t tt = (size_t)n_types * n_types;
    // FP32 hi/lo pairs: a type pair's A and B are shared by many atom pairs,
    // so their rounding must not bias the Lennard-Jones sum
    std::vector<float4> ljn(tt), ljm(tt);
    std::vector<double4> ljd(tt);
    auto hilo = [](double v, float& h, float& l) { h = (float)v; l = (float)(v - (double)h); };
    for (size_t k = 0; k < tt; ++k) {
        const double* p = lj_table + 4 * k;
        float ah, al, bh, bl;
        hilo(p[0], ah, al); hilo(p[1], bh, bl);
        ljn[k] = make_float4(ah, bh, al, bl);
        hilo(p[2], ah, al); hilo(p[3], bh, bl);
        ljm[k] = make_float4(ah, bh, al, bl);
        ljd[k] = make_double4(p[0], p[1], p[2], p[3]);
    }
    CK(dalloc(&sys->d_ljn, tt), "alloc"); CK(dalloc(&sys->d_ljm, tt), "alloc"); CK(dalloc(&sys->d_ljd, tt), "alloc");
    CK(cudaMemcpy(sys->d_ljn, ljn.data(), sizeof(float4) * tt, cudaMemcpyHostToDevice), "copy");
    CK(cudaMemcpy(sys->d_ljm, ljm.data(), sizeof(float4) * tt, cudaMemcpyHostToDevice), "copy");
    CK(cudaMemcpy(sys->d_ljd, ljd.data(), sizeof(double4) * tt, cudaMemcpyHostToDevice), "copy");
    // exclusions: check() classes as window bit masks (index delta 1..32) and
    // a CSR list for larger deltas (ExclusionTable's lowDeltas / highDeltas)
    std::vector<uint32_t> xfull(n, 0u), xmod(n, 0u);
    std::vector<std::vector<int2>> far(n);
    sys->excl_pairs.assign(2 * (size_t)n_excl, 0);
    sys->excl_cls.assign(n_excl, 0);
    for (int k = 0; k < n_excl; ++k) {
        int a = excl_pairs[2 * k], b = excl_pairs[2 * k + 1];
        if (a < 0 || b < 0 || a >= n || b >= n || a == b) return fail(sys, PMGPU_ERR_ARG, "bad exclusion pair");
        if (a > b) std::swap(a, b);
        int tcls = excl_class[k];
        int ccls = excl_check_class ? excl_check_class[k] : tcls;
        sys->excl_pairs[2 * k] = a; sys->excl_pairs[2 * k + 1] = b;
        sys->excl_cls[k] = tcls;
        int d = b - a;
        if (d <= kExclWindow) {
            uint32_t bit = 1u << (d - 1);
            xfull[a] &= ~bit; xmod[a] &= ~bit;
            if (ccls == PMGPU_EXCL_FULL) xfull[a] |= bit;
            else if (ccls == PMGPU_EXCL_MODIFIED) xmod[a] |= bit;
        } else {
            far[a].push_back(make_int2(b, ccls));
        }
    }
    std::vector<int> xrow(n + 1, 0);
    std::vector<int2> xent;
    for (int a = 0; a < n; ++a) {
        std::sort(far[a].begin(), far[a].end(), [](int2 u, int2 v) { return u.x < v.x; });
        xrow[a] = (int)xent.size();
        for (auto& v : far[a]) xent.push_back(v);
    }
    xrow[n] = (int)xent.size();
    CK(dalloc(&sys->d_xfull, n), "alloc"); CK(dalloc(&sys->d_xmod, n), "alloc");
    CK(dalloc(&sys->d_xrow, n + 1), "alloc"); CK(dalloc(&sys->d_xent, xent.size()), "alloc");
    CK(cudaMemcpy(sys->d_xfull, xfull.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice), "copy");
    CK(cudaMemcpy(sys->d_xmod, xmod.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice), "copy");
    CK(cudaMemcpy(sys->d_xrow, xrow.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice), "copy");
    if (!xent.empty())
        CK(cudaMemcpy(sys->d_xent, xent.data(), sizeof(int2) * xent.size(), cudaMemcpyHostToDevice), "copy");
    CK(dalloc(&sys->d_epairs, n_excl), "alloc"); CK(dalloc(&sys->d_ecls, n_excl), "alloc");
    if (n_excl) {
        CK(cudaMemcpy(sys->d_epairs, sys->excl_pairs.data(), sizeof(int) * 2 * n_excl, cudaMemcpyHostToDevice), "copy");
        CK(cudaMemcpy(sys->d_ecls, sys->excl_cls.data(), sizeof(int) * n_excl, cudaMemcpyHostToDevice), "copy");
    }
    // per-evaluation atom buffers
    CK(dalloc(&sys->d_pos, 3 * (size_t)n), "alloc"); CK(dalloc(&sys->d_fout, 3 * (size_t)n), "alloc");
    CK(dalloc(&sys->d_facc32, 6 * (size_t)n), "alloc"); CK(dalloc(&sys->d_facc40, 3 * (size_t)n), "alloc");
    CK(dalloc(&sys->d_faccA, 6 * (size_t)n), "alloc");
    sys->d_facc32p = sys->d_facc32 + 3 * (size_t)n;
    CK(dalloc(&sys->d_cell_lin, n), "alloc"); CK(dalloc(&sys->d_cell3, 3 * (size_t)n), "alloc");
    CK(dalloc(&sys->d_tmp, n), "alloc"); CK(dalloc(&sys->d_sorted, n), "alloc"); CK(dalloc(&sys->d_slot, n), "alloc");
    CK(dalloc(&sys->d_spos, n), "alloc"); CK(dalloc(&sys->d_smeta, n), "alloc"); CK(dalloc(&sys->d_spos64, n), "alloc");
    CK(dalloc(&sys->d_slo, n), "alloc"); CK(dalloc(&sys->d_skey, n), "alloc");
    CK(dalloc(&sys->d_qfix, 3 * (size_t)n), "alloc"); CK(dalloc(&sys->d_colid, n), "alloc");
    CK(dalloc(&sys->d_ctmp, n), "alloc"); CK(dalloc(&sys->d_cslot, n), "alloc");
    CK(cudaMemset(sys->d_cslot, 0, sizeof(int) * (size_t)std::max(n, 1)), "memset");
    sys->col_ncl_cap = 0;   // slot arrays depend on N and the column grid: sized at evaluation
    sys->col_grid_stale = true;
    sys->list_valid = false;
    sys->cbox_cap = 0;   // cluster boxes depend on N and the cell grid: sized at evaluation
    CK(dalloc(&sys->d_acc0, 3 * (size_t)std::max(n, 1)), "alloc");
    if (sys->h_fbuf) cudaFreeHost(sys->h_fbuf);
    sys->h_fbuf = nullptr;
    CK(cudaMallocHost((void**)&sys->h_fbuf, sizeof(double) * 3 * (size_t)std::max(n, 1)), "host alloc");
    return PMGPU_OK;
}

// ------------------------------------------------------------------ box
// Column grid of the column-cluster pair path for the box: columns of ~4 A
// in x and y (narrower when a column would hold more than ~384 atoms at the
// box's mean density), fixed point L / 2^32 per axis.  The reach and the
// eligibility depend on the cutoff (col_reach).
static int col_set_grid(pmgpu_system* sys)
{
    ColGrid& g = sys->cg;
    memset(&g, 0, sizeof(g));
    const double lx = sys->box[0], ly = sys->box[4], lz = sys->box[8];
    g.lx = lx; g.ly = ly; g.lz = lz;
    g.mnx = sys->box[9] - 0.5 * lx; g.mny = sys->box[10] - 0.5 * ly; g.mnz = sys->box[11] - 0.5 * lz;
    const double rho = sys->n > 0 ? sys->n / (lx * ly * lz) : 0.0;
    double side = 4.0;
    if (rho * side * side * lz > 384.0) side = std::sqrt(384.0 / (rho * lz));
    g.ncx = std::max(1, (int)std::floor(lx / side));
    g.ncy = std::max(1, (int)std::floor(ly / side));
    sys->col_grid = (long long)g.ncx * g.ncy <= (1 << 22);
    if (!sys->col_grid) return PMGPU_OK;
    g.ncol = g.ncx * g.ncy;
    g.sx = (float)(lx / g.ncx); g.sy = (float)(ly / g.ncy);
    g.lxf = (float)lx; g.lyf = (float)ly; g.lzf = (float)lz;
    const double L[3] = {lx, ly, lz};
    for (int a = 0; a < 3; ++a) {
        const double u = L[a] / 4294967296.0;
        g.sch[a] = (float)u;
        g.scl[a] = (float)(u - (double)g.sch[a]);
    }
    if (g.ncol > sys->col_ncol_cap) {
        CK(dalloc(&sys->d_ccounts, g.ncol), "alloc");
        CK(dalloc(&sys->d_colstart, g.ncol + 1), "alloc");
        CK(dalloc(&sys->d_ccstart, g.ncol + 1), "alloc");
        CK(dalloc(&sys->d_zidx, (size_t)g.ncol * kZIndex), "alloc");
        sys->col_ncol_cap = g.ncol;
    }
    // the binning returns the counts to zero; they start there
    CK(cudaMemsetAsync(sys->d_ccounts, 0, sizeof(int) * (size_t)g.ncol, sys->stream), "memset");
    return PMGPU_OK;
}

// Reach of the column list for a pair test at cutoff rc, and whether the
// column path applies: no column may be reached through two offsets, and the
// z windows (an i-cluster's extent plus twice the list radius) must be
// shorter than the box, so that every pair inside the cutoff lies in its
// tile's image
static bool col_reach(const pmgpu_system* sys, double rc, ColGrid& g)
{
    if (!sys->col_grid || sys->col_disabled) return false;
    g = sys->cg;
    const double rl = std::sqrt(rc * rc * (1.0 + 8.0 * 2.0e-5) + 1e-3);
    g.rx = (int)std::ceil(rl / g.sx) + 1;
    g.ry = (int)std::ceil(rl / g.sy) + 1;
    if (2 * g.rx + 1 > g.ncx || 2 * g.ry + 1 > g.ncy) return false;
    const double zext = g.lz - 2.0 * rl - 0.5;
    if (!(zext > 1.0)) return false;
    g.zext = (float)zext;
    return true;
}

extern "C" int pmgpu_set_box(pmgpu_system* sys, const double* e1, const double* e2, const double* e3,
                             const double* origin, double cell_size)
{
    if (!sys || !e1 || !e2 || !e3 || !origin) return PMGPU_ERR_ARG;
    if (!(cell_size > 0.0)) return fail(sys, PMGPU_ERR_ARG, "Cubic cellmanager: cutoff > 0");
    bool orth = !(e1[1] != 0.0 || e1[2] != 0.0 || e2[0] != 0.0 || e2[2] != 0.0 || e3[0] != 0.0 || e3[1] != 0.0);
    if (!orth) return fail(sys, PMGPU_ERR_UNSUPPORTED, "only orthogonal periodic boxes are supported");
    if (!(e1[0] > 0.0 && e2[1] > 0.0 && e3[2] > 0.0)) return fail(sys, PMGPU_ERR_ARG, "box edges must be positive");
    cudaSetDevice(sys->device);
    CK(cudaStreamSynchronize(sys->stream), "set_box");
    for (int k = 0; k < 3; ++k) {
        sys->box[k] = e1[k]; sys->box[3 + k] = e2[k]; sys->box[6 + k] = e3[k]; sys->box[9 + k] = origin[k];
    }
    sys->cell_size = cell_size;
    // PeriodicBoundaryConditions::set (topology/PeriodicBoundaryConditions.cpp:40-77)
    Pbc& b = sys->pbc;
    double ex = e1[0], ey = e2[1], ez = e3[2];
    b.e1x = ex; b.e2y = ey; b.e3z = ez;
    // myE1r = (e2 x e3) / e1.(e2 x e3): for an orthogonal box the x component
    double a1x = e2[1] * e3[2] - e2[2] * e3[1];
    b.e1rx = a1x / (e1[0] * a1x + e1[1] * (e2[2] * e3[0] - e2[0] * e3[2]) + e1[2] * (e2[0] * e3[1] - e2[1] * e3[0]));
    double a2y = e3[2] * e1[0] - e3[0] * e1[2];
    b.e2ry = a2y / (e2[0] * (e3[1] * e1[2] - e3[2] * e1[1]) + e2[1] * a2y + e2[2] * (e3[0] * e1[1] - e3[1] * e1[0]));
    double a3z = e1[0] * e2[1] - e1[1] * e2[0];
    b.e3rz = a3z / (e3[0] * (e1[1] * e2[2] - e1[2] * e2[1]) + e3[1] * (e1[2] * e2[0] - e1[0] * e2[2]) + e3[2] * a3z);
    double sx = (e1[0] + e2[0]) + e3[0], sy = (e1[1] + e2[1]) + e3[1], sz = (e1[2] + e2[2]) + e3[2];
    double ax = origin[0] - sx * 0.5, ay = origin[1] - sy * 0.5, az = origin[2] - sz * 0.5;
    double cx = origin[0] + sx * 0.5, cy = origin[1] + sy * 0.5, cz = origin[2] + sz * 0.5;
    double mnx = std::min(ax, cx), mny = std::min(ay, cy), mnz = std::min(az, cz);
    double mxx = std::max(ax, cx), mxy = std::max(ay, cy), mxz = std::max(az, cz);
    double dx = (ex * 0.5) * (ex * 0.5), dy = (ey * 0.5) * (ey * 0.5), dz = (ez * 0.5) * (ez * 0.5);
    b.d = std::min(dx, std::min(dy, dz));
    b.hx = mxx - mnx; b.hy = mxy - mny; b.hz = mxz - mnz;
    b.h2x = b.hx * 0.5; b.h2y = b.hy * 0.5; b.h2z = b.hz * 0.5;
    b.ox = origin[0]; b.oy = origin[1]; b.oz = origin[2];
    b.dx = origin[0] - mnx; b.dy = origin[1] - mny; b.dz = origin[2] - mnz;
    // CubicCellManager::initialize + ArrayCellListStructure::initialize
    CellGrid& g = sys->grid;
    double hx = mxx - mnx, hy = mxy - mny, hz = mxz - mnz;
    g.csx = hx / std::max(1.0, std::floor(hx / cell_size));
    g.csy = hy / std::max(1.0, std::floor(hy / cell_size));
    g.csz = hz / std::max(1.0, std::floor(hz / cell_size));
    g.rcsx = 1.0 / g.csx; g.rcsy = 1.0 / g.csy; g.rcsz = 1.0 / g.csz;
    g.nx = std::max(1, (int)std::floor(hx / g.csx + kEpsilon));
    g.ny = std::max(1, (int)std::floor(hy / g.csy + kEpsilon));
    g.nz = std::max(1, (int)std::floor(hz / g.csz + kEpsilon));
    long long nc = (long long)g.nx * g.ny * g.nz;
    if (nc > (1ll << 28)) return fail(sys, PMGPU_ERR_ARG, "simulation box / cell size ratio too big");
    g.ncell = (int)nc;
    if (g.ncell > sys->ncell_cap) {
        CK(dalloc(&sys->d_counts, g.ncell), "alloc");
        CK(dalloc(&sys->d_start, g.ncell + 1), "alloc"); CK(dalloc(&sys->d_cstart, g.ncell + 1), "alloc");
        sys->ncell_cap = g.ncell;
    }
    // the binning leaves the counts at zero; they start there
    CK(cudaMemsetAsync(sys->d_counts, 0, sizeof(int) * (size_t)g.ncell, sys->stream), "memset");
    sys->col_grid_stale = true;
    sys->list_valid = false;
    sys->box_set = true;
    sys->box_version++;
    sys->binned = false;
    return PMGPU_OK;
}

// ------------------------------------------------------------------ forces
static bool pot_is_table(int pot)
{
    return pot == PMGPU_POT_LENNARD_JONES_TABLE || pot == PMGPU_POT_COULOMB_TABLE ||
           pot == PMGPU_POT_EWALD_REAL_TABLE;
}

// the switching functions a table can hold, value and derivOverD
// (C2SwitchingFunction.h:64-82, CutoffSwitchingFunction.h:64-68,
// ShiftSwitchingFunction.h)
static void host_switch(const TermD& t, double r2, double& v, double& d)
{
    if (t.sw == PMGPU_SW_C2) {
        d = 0.0;
        if (r2 > t.cut2) v = 0.0;
        else if (r2 >= t.on2) {
            double c2 = t.cut2 - r2;
            double c4 = c2 * (t.s2 + 2.0 * r2);
            v = t.s1 * (c2 * c4);
            d = t.s3 * (c2 * c2 - c4);
        } else v = 1.0;
    } else if (t.sw == PMGPU_SW_SHIFT) {
        if (r2 > t.cut2) { v = 0.0; d = 0.0; return; }
        double x = 1.0 - r2 * t.sh_a;
        v = x * x;
        d = t.sh_b * x;
    } else if (t.sw == PMGPU_SW_CUTOFF) {
        d = 0.0;
        v = r2 > t.cut2 ? 0.0 : 1.0;
    } else {
        v = 1.0; d = 0.0;
    }
}

static double lowerbound_exp2(double r)      // base/mathutilities.cpp:43-51
{
    double res = 1.0;
    while (res < r) res *= 2.0;
    while (res > r) res /= 2.0;
    return res;
}

static long long dbits(double x) { long long u; memcpy(&u, &x, 8); return u; }

// square(power<n/2>(x)) * power<n - 2 (n/2)>(x) for the negative powers of
// the tabulated functions (base/mathutilities.h:72-94)
static double ipow_neg(double x, int n)
{
    if (n == -1) return 1. / x;
    if (n == 0) return 1;
    double h = ipow_neg(x, n / 2);
    return (h * h) * ipow_neg(x, n - 2 * (n / 2));
}

// The look-up table of a table potential: LookUpTableBase(0.1, rc^2, 2,
// LookUpValues, swf) (base/LookUpTableBase.h:115-205) with PRE 7 for
// LennardJonesTable and 6 for the Coulomb tables (the registered templates,
// factories/registerForceExemplarsCutoff.cpp:47-48,58,69), the values of
// LookUpValues::assign (forces/LennardJonesTableForceBase.h:35-45,
// CoulombTableForceBase.h:33-39, CoulombEwaldRealTableForceBase.h:36-43) and
// the Hermite coefficients with their two refinement steps, in FP64 and the
// reference's operation order, so the table is the reference's bit for bit.
static std::vector<double> build_lookup_table(int pot, const TermD& sw, double alpha, int& pre, int& step,
                                              long long& first, long long& last)
{
    pre = pot == PMGPU_POT_LENNARD_JONES_TABLE ? 7 : 6;
    step = (pot == PMGPU_POT_LENNARD_JONES_TABLE ? 2 : 1) * 4;
    const int n = 1 << pre;
    double from = 0.1;
    const long long octaves = (dbits(lowerbound_exp2(sw.cut2)) >> 52) + 1 - (dbits(lowerbound_exp2(from)) >> 52);
    const long long entries = octaves * n + 1;
    std::vector<double> t((size_t)(entries * step), 0.0);
    first = (dbits(lowerbound_exp2(from)) >> (52 - pre)) * step;
    last = (entries - 1) * step;
    from = lowerbound_exp2(from);
    for (long long i = 0; i < entries; ++i) {
        double base = from * (double)(1 << (i / n));
        double del = base / (double)n;
        double r = base + del * (double)(i % n);
        double r1 = std::sqrt(r);
        double v, d;
        host_switch(sw, r, v, d);
        double* val = t.data() + i * step;
        if (pot == PMGPU_POT_LENNARD_JONES_TABLE) {
            double e = ipow_neg(r1, -12), f = 12.0 * ipow_neg(r1, -14);
            val[0] = e * v;
            val[1] = -0.5 * (f * v - e * d);
            e = -ipow_neg(r1, -6); f = -6.0 * ipow_neg(r1, -8);
            val[4] = e * v;
            val[5] = -0.5 * (f * v - e * d);
        } else if (pot == PMGPU_POT_COULOMB_TABLE) {
            double e = ipow_neg(r1, -1), f = ipow_neg(r1, -3);
            val[0] = e * v;
            val[1] = -0.5 * (f * v - e * d);
        } else {
            double r2 = r;
            double e = std::erfc(alpha * r1) / r1;
            double f = (e + 2.0 * alpha / std::sqrt(kPi) * std::exp(-alpha * alpha * r2)) / r2;
            val[0] = e * v;
            val[1] = -0.5 * (f * v - e * d);
        }
        if (i == 0) continue;
        const double x = from * (double)(1 << ((i - 1) / n)) / (double)n;
        double* pv = t.data() + (i - 1) * step;
        for (int j = 0; j < step; j += 4) {
            const double v1 = pv[j], g1 = pv[j + 1], v2 = pv[j + step], g2 = pv[j + 1 + step];
            double c = (3.0 * (v2 - v1) - x * (2.0 * g1 + g2)) / (x * x);
            double dd = (-2.0 * (v2 - v1) + x * (g1 + g2)) / (x * x * x);
            for (int it = 0; it < 2; ++it) {
                double dv = (v1 - v2) + ((dd * x + c) * x + g1) * x;
                double dg = (g1 - g2) + (3.0 * dd * x + 2.0 * c) * x;
                c -= (3.0 * dv - x * dg) / (x * x);
                dd -= (-2.0 * dv + x * dg) / (x * x * x);
            }
            pv[j + 2] = c;
            pv[j + 3] = dd;
        }
    }
    return t;
}

// uploads a table potential's table (FP64 and its FP32 rounding) and sets
// the terms' look-up constants
static cudaError_t table_setup(pmgpu_force* f, int k)
{
    int pre = 0, step = 0;
    long long first = 0, last = 0;
    std::vector<double> t = build_lookup_table(f->td[k].pot, f->td[k], f->td[k].alpha, pre, step, first, last);
    std::vector<float> t32(t.size());
    for (size_t i = 0; i < t.size(); ++i) t32[i] = (float)t[i];
    cudaError_t e = dalloc(&f->d_tab64[k], t.size());
    if (e == cudaSuccess) e = dalloc(&f->d_tab32[k], t.size());
    if (e == cudaSuccess) e = cudaMemcpy(f->d_tab64[k], t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(f->d_tab32[k], t32.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    TermD& d = f->td[k];
    d.tab = f->d_tab64[k]; d.tab_step = step; d.tab_first = first; d.tab_last = (int)last; d.tab_shift = 52 - pre;
    TermF& g = f->tf[k];
    uint32_t ub;
    const float from32 = 0.0625f;            // lowerboundExp2(0.1)
    memcpy(&ub, &from32, 4);
    g.tab = f->d_tab32[k]; g.tab_step = step; g.tab_shift = 23 - pre;
    g.tab_first = (int)(ub >> g.tab_shift) * step; g.tab_last = (int)last;
    return cudaSuccess;
}

static void term_setup(const pmgpu_cutoff_params* p, int k, TermF& f, TermD& d)
{
    memset(&f, 0, sizeof(f));
    memset(&d, 0, sizeof(d));
    d.pot = f.pot = p->pot[k];
    d.sw = f.sw = p->sw[k];
    double c = p->cutoff[k], on = p->switchon[k];
    d.cut2 = c * c;
    if (d.sw == PMGPU_SW_C2) {       // C2SwitchingFunction.cpp:15-23
        double q = c * c - on * on;
        d.on2 = on * on;
        d.s1 = 1.0 / (q * q * q);
        d.s2 = c * c - 3.0 * on * on;
        d.s3 = 4.0 / (q * q * q);
    } else if (d.sw == PMGPU_SW_C1) { // C1SwitchingFunction.cpp:18-25
        d.c1_15_1 = 1.5 / c;
        d.c1_05_3 = 0.5 / (c * c * c);
        d.c1_15_3 = 1.5 / (c * c * c);
    } else if (d.sw == PMGPU_SW_SHIFT) {
        d.sh_a = 1.0 / (c * c);
        d.sh_b = -4.0 / (c * c);
    }
    d.alpha = p->alpha[k];
    d.two_alpha_pi = 2.0 * d.alpha / std::sqrt(kPi);   // CoulombEwaldRealForce.cpp:17-21
    f.cut2 = (float)d.cut2; f.on2 = (float)d.on2; f.s1 = (float)d.s1; f.s2 = (float)d.s2; f.s3 = (float)d.s3;
    f.c1_15_1 = (float)d.c1_15_1; f.c1_05_3 = (float)d.c1_05_3; f.c1_15_3 = (float)d.c1_15_3;
    f.sh_a = (float)d.sh_a; f.sh_b = (float)d.sh_b;
    f.alpha = (float)d.alpha; f.two_alpha_pi = (float)d.two_alpha_pi;
    f.alpha_lo = (float)(d.alpha - (double)f.alpha);
    f.two_alpha_pi_lo = (float)(d.two_alpha_pi - (double)f.two_alpha_pi);
    f.s1_lo = (float)(d.s1 - (double)f.s1);
    f.s3_lo = (float)(d.s3 - (double)f.s3);
    f.c1_15_1_lo = (float)(d.c1_15_1 - (double)f.c1_15_1);
    f.c1_05_3_lo = (float)(d.c1_05_3 - (double)f.c1_05_3);
    f.c1_15_3_lo = (float)(d.c1_15_3 - (double)f.c1_15_3);
    f.sh_a_lo = (float)(d.sh_a - (double)f.sh_a);
    f.sh_b_lo = (float)(d.sh_b - (double)f.sh_b);
}

extern "C" int pmgpu_cutoff_create(pmgpu_system* sys, const pmgpu_cutoff_params* p, pmgpu_force** out)
{
    if (!sys || !p || !out) return PMGPU_ERR_ARG;
    *out = nullptr;
    if (p->n_terms < 1 || p->n_terms > 2) return fail(sys, PMGPU_ERR_ARG, "n_terms must be 1 or 2");
    if (p->precision != PMGPU_PRECISION_MIXED && p->precision != PMGPU_PRECISION_FP64)
        return fail(sys, PMGPU_ERR_ARG, "unknown precision");
    for (int k = 0; k < p->n_terms; ++k) {
        if (p->sw[k] == PMGPU_SW_C2 && !(p->switchon[k] >= 0.0 && p->cutoff[k] > 0.0 && p->switchon[k] < p->cutoff[k]))
            return fail(sys, PMGPU_ERR_ARG, "C2 switching function: 0 <= switchon < cutoff");
        if (p->sw[k] != PMGPU_SW_UNIVERSAL && !(p->cutoff[k] > 0.0))
            return fail(sys, PMGPU_ERR_ARG, "switching function cutoff > 0");
        if ((p->pot[k] == PMGPU_POT_EWALD_REAL || p->pot[k] == PMGPU_POT_EWALD_REAL_TABLE) && !(p->alpha[k] > 0.0))
            return fail(sys, PMGPU_ERR_ARG, "CoulombEwaldReal -alpha > 0");
        // the tabulated switching functions of the registered table templates
        const int pk = p->pot[k], sk = p->sw[k];
        if ((pk == PMGPU_POT_LENNARD_JONES_TABLE && sk != PMGPU_SW_C2) ||
            (pk == PMGPU_POT_COULOMB_TABLE && sk != PMGPU_SW_CUTOFF && sk != PMGPU_SW_SHIFT) ||
            (pk == PMGPU_POT_EWALD_REAL_TABLE && sk != PMGPU_SW_CUTOFF))
            return fail(sys, PMGPU_ERR_UNSUPPORTED, "table potential with a switching function not registered for it");
    }
    if (!(p->algorithm_cutoff > 0.0)) return fail(sys, PMGPU_ERR_ARG, "NonbondedCutoff -cutoff > 0");
    int combo = pair_combo_id(p->n_terms, p->pot, p->sw);
    if (combo < 0) return fail(sys, PMGPU_ERR_UNSUPPORTED, "force combination not registered for periodic boundaries");
    pmgpu_force* f = new pmgpu_force();
    f->sys = sys;
    f->kind = 0;
    f->precision = p->precision;
    f->cp = *p;
    f->combo = combo;
    double c2 = 0.0;
    for (int k = 0; k < p->n_terms; ++k) {
        term_setup(p, k, f->tf[k], f->td[k]);
        // Cutoff<>::cutoff of each term is its switching function's cutoff^2,
        // a table potential's the tabulated one's; the pair test uses the
        // largest (OneAtomPairTwo.h:48)
        c2 = std::max(c2, f->td[k].cut2);
        if (pot_is_table(p->pot[k])) {
            cudaSetDevice(sys->device);
            cudaError_t e = table_setup(f, k);
            if (e != cudaSuccess) {
                free_force(f);
                return cuda_fail(sys, e, "look-up table");
            }
        }
    }
    f->cut2 = c2;
    sys->forces.insert(f);
    *out = f;
    return PMGPU_OK;
}

extern "C" long long pmgpu_lookup_table(int pot, int sw, double switchon, double cutoff, double alpha,
                                        double* table, long long cap)
{
    if (!pot_is_table(pot) || !(cutoff > 0.0) || cap < 0) return -1;
    if ((pot == PMGPU_POT_LENNARD_JONES_TABLE && !(sw == PMGPU_SW_C2 && switchon >= 0.0 && switchon < cutoff)) ||
        (pot == PMGPU_POT_COULOMB_TABLE && sw != PMGPU_SW_CUTOFF && sw != PMGPU_SW_SHIFT) ||
        (pot == PMGPU_POT_EWALD_REAL_TABLE && (sw != PMGPU_SW_CUTOFF || !(alpha > 0.0))))
        return -1;
    pmgpu_cutoff_params p;
    memset(&p, 0, sizeof(p));
    p.n_terms = 1; p.pot[0] = pot; p.sw[0] = sw; p.switchon[0] = switchon; p.cutoff[0] = cutoff; p.alpha[0] = alpha;
    TermF f;
    TermD d;
    term_setup(&p, 0, f, d);
    int pre = 0, step = 0;
    long long first = 0, last = 0;
    std::vector<double> t = build_lookup_table(pot, d, alpha, pre, step, first, last);
    if (table) memcpy(table, t.data(), sizeof(double) * (size_t)std::min<long long>(cap, (long long)t.size()));
    return (long long)t.size();
}

// NonbondedSimpleFullSystemForce with VacuumBoundaryConditions
// (forces/NonbondedSimpleFullSystemForce.h:165-182,
// factories/registerForceExemplarsSimpleFull.cpp:88-152): every pair once, no
// minimal image, the OneAtomPair[Two] potentials and switches
extern "C" int pmgpu_full_create(pmgpu_system* sys, const pmgpu_cutoff_params* p, pmgpu_force** out)
{
    if (!sys || !p || !out) return PMGPU_ERR_ARG;
    *out = nullptr;
    if (p->n_terms < 1 || p->n_terms > 2) return fail(sys, PMGPU_ERR_ARG, "n_terms must be 1 or 2");
    if (p->precision != PMGPU_PRECISION_MIXED && p->precision != PMGPU_PRECISION_FP64)
        return fail(sys, PMGPU_ERR_ARG, "unknown precision");
    for (int k = 0; k < p->n_terms; ++k) {
        if (p->pot[k] < PMGPU_POT_LENNARD_JONES || p->pot[k] > PMGPU_POT_EWALD_REAL)
            return fail(sys, PMGPU_ERR_ARG, "unknown potential");
        if (p->sw[k] == PMGPU_SW_C2 && !(p->switchon[k] >= 0.0 && p->cutoff[k] > 0.0 && p->switchon[k] < p->cutoff[k]))
            return fail(sys, PMGPU_ERR_ARG, "C2 switching function: 0 <= switchon < cutoff");
        if (p->sw[k] != PMGPU_SW_UNIVERSAL && !(p->cutoff[k] > 0.0))
            return fail(sys, PMGPU_ERR_ARG, "switching function cutoff > 0");
        if (p->pot[k] == PMGPU_POT_EWALD_REAL && !(p->alpha[k] > 0.0))
            return fail(sys, PMGPU_ERR_ARG, "CoulombEwaldReal -alpha > 0");
    }
    pmgpu_force* f = new pmgpu_force();
    f->sys = sys;
    f->kind = 2;
    f->precision = p->precision;
    f->cp = *p;
    double c2 = 0.0;
    for (int k = 0; k < p->n_terms; ++k) {
        term_setup(p, k, f->tf[k], f->td[k]);
        c2 = std::max(c2, f->td[k].cut2);
    }
    f->cut2 = c2;
    sys->forces.insert(f);
    *out = f;
    return PMGPU_OK;
}

// the recompute kernel's arguments for a pair force (cutoff or vacuum)
static void adj_pair_args(pmgpu_system* sys, pmgpu_force* f, AdjArgs& a)
{
    memset(&a, 0, sizeof(a));
    a.n = sys->n; a.pos = sys->d_pos; a.q = sys->d_q; a.type = sys->d_type; a.mol = sys->d_mol;
    a.pbc = sys->pbc; a.periodic = f->kind == 2 ? 0 : 1;
    a.xfull = sys->d_xfull; a.xmod = sys->d_xmod; a.xrow = sys->d_xrow; a.xent = sys->d_xent;
    a.ljd = sys->d_ljd; a.n_types = sys->t;
    a.n_terms = f->cp.n_terms; a.td[0] = f->td[0]; a.td[1] = f->td[1];
    bool mod = false, use = false;
    for (int t = 0; t < f->cp.n_terms; ++t) {
        const int sw = f->cp.sw[t];
        mod |= sw == PMGPU_SW_C1 || sw == PMGPU_SW_C2 || sw == PMGPU_SW_SHIFT;
        use |= sw != PMGPU_SW_UNIVERSAL;
    }
    a.modify = mod ? 1 : 0; a.use_cut = use ? 1 : 0; a.cut2d = f->cut2; a.csf = sys->csf;
    a.status = sys->d_status;
}

// Neighbour-delta list of CellListEnumerator<Periodic, Cubic>::initialize
// (topology/CellListEnumerator_periodicBoundaries.h:37-108).
static void build_deltas(const CellGrid& g, double cutoff, std::vector<int4>& out, int& reach_ok)
{
    double cutoff2 = cutoff * cutoff;
    int nx = (int)(cutoff / g.csx + 1.0 + kEpsilon);
    int ny = (int)(cutoff / g.csy + 1.0 + kEpsilon);
    int nz = (int)(cutoff / g.csz + 1.0 + kEpsilon);
    int n0 = std::min(nx, g.nx), n1 = std::min(ny, g.ny), n2 = std::min(nz, g.nz);
    reach_ok = (g.nx >= 2 * nx + 1) && (g.ny >= 2 * ny + 1) && (g.nz >= 2 * nz + 1);
    int max2 = 2147483647 / 2;
    int maxNX = max2 - max2 % g.nx, maxNY = max2 - max2 % g.ny, maxNZ = max2 - max2 % g.nz;
    int nx1 = -g.nx / 2, ny1 = -g.ny / 2, nz1 = -g.nz / 2;
    int maxNX1 = maxNX - nx1, maxNY1 = maxNY - ny1, maxNZ1 = maxNZ - nz1;
    double xx = g.csx * g.csx, yy = g.csy * g.csy, zz = g.csz * g.csz;
    struct C3 { int x, y, z; bool operator<(const C3& o) const { return x != o.x ? x < o.x : (y != o.y ? y < o.y : z < o.z); } };
    std::set<C3> seen;
    std::vector<C3> list;
    seen.insert(C3{0, 0, 0});
    for (int k = -n0; k <= n0; k++) {
        int x = std::abs(k) - 1; if (x < 0) x = 0;
        double d0 = x * x * xx;
        for (int l = -n1; l <= n1; l++) {
            int y = std::abs(l) - 1; if (y < 0) y = 0;
            double d1 = d0 + y * y * yy;
            for (int m = -n2; m <= n2; m++) {
                int z = std::abs(m) - 1; if (z < 0) z = 0;
                if (d1 + z * z * zz < cutoff2) {
                    C3 md{(k + maxNX1) % g.nx + nx1, (l + maxNY1) % g.ny + ny1, (m + maxNZ1) % g.nz + nz1};
                    if (seen.insert(md).second) list.push_back(md);
                }
            }
        }
    }
    std::sort(list.begin(), list.end());
    out.clear();
    for (auto& c : list) out.push_back(make_int4(c.x, c.y, c.z, 0));
}

static int prepare_cutoff(pmgpu_force* f)
{
    pmgpu_system* sys = f->sys;
    if (f->box_version == sys->box_version) return PMGPU_OK;
    std::vector<int4> deltas;
    int reach_ok = 0;
    build_deltas(sys->grid, f->cp.algorithm_cutoff, deltas, reach_ok);
    if ((int)deltas.size() > kMaxDeltas) return fail(sys, PMGPU_ERR_ARG, "cutoff / cell size ratio too large");
    std::vector<float4> off(deltas.size());
    for (size_t k = 0; k < deltas.size(); ++k)
        off[k] = make_float4((float)(deltas[k].x * sys->grid.csx), (float)(deltas[k].y * sys->grid.csy),
                             (float)(deltas[k].z * sys->grid.csz), 0.f);
    f->nd = (int)deltas.size();
    f->wrap = reach_ok ? 0 : 1;
    CK(dalloc(&f->d_deltas, deltas.size()), "alloc");
    CK(dalloc(&f->d_doff, deltas.size()), "alloc");
    if (!deltas.empty()) {
        CK(cudaMemcpy(f->d_deltas, deltas.data(), sizeof(int4) * deltas.size(), cudaMemcpyHostToDevice), "copy");
        CK(cudaMemcpy(f->d_doff, off.data(), sizeof(float4) * off.size(), cudaMemcpyHostToDevice), "copy");
    }
    // half shell of the mixed kernel: when every delta of the reach is a
    // distinct cell (reach_ok), the lexicographically positive half of the
    // (symmetric) delta list visits each unordered cell pair exactly once;
    // otherwise the reference's list with its B > A rule
    std::vector<int4> hd;
    for (const int4& d : deltas)
        if (!reach_ok || d.x > 0 || (d.x == 0 && (d.y > 0 || (d.y == 0 && d.z > 0)))) hd.push_back(d);
    std::vector<float4> ho(hd.size()), hl(hd.size());
    std::vector<double4> h64(hd.size());
    for (size_t k = 0; k < hd.size(); ++k) {
        double o[3] = {hd[k].x * sys->grid.csx, hd[k].y * sys->grid.csy, hd[k].z * sys->grid.csz};
        float h[3], l[3];
        for (int c = 0; c < 3; ++c) { h[c] = (float)o[c]; l[c] = (float)(o[c] - (double)h[c]); }
        ho[k] = make_float4(h[0], h[1], h[2], 0.f);
        hl[k] = make_float4(l[0], l[1], l[2], 0.f);
        // the offset the FP32 pair vectors carry (hi + lo), for the virial
        h64[k] = make_double4((double)h[0] + (double)l[0], (double)h[1] + (double)l[1],
                              (double)h[2] + (double)l[2], 0.0);
    }
    f->nh = (int)hd.size();
    f->half_rule = reach_ok ? 0 : 1;
    CK(dalloc(&f->d_hdeltas, hd.size()), "alloc");
    CK(dalloc(&f->d_hoff, hd.size()), "alloc");
    CK(dalloc(&f->d_hoff_lo, hd.size()), "alloc");
    CK(dalloc(&f->d_hoff64, hd.size()), "alloc");
    if (!hd.empty()) {
        CK(cudaMemcpy(f->d_hdeltas, hd.data(), sizeof(int4) * hd.size(), cudaMemcpyHostToDevice), "copy");
        CK(cudaMemcpy(f->d_hoff, ho.data(), sizeof(float4) * ho.size(), cudaMemcpyHostToDevice), "copy");
        CK(cudaMemcpy(f->d_hoff_lo, hl.data(), sizeof(float4) * hl.size(), cudaMemcpyHostToDevice), "copy");
        CK(cudaMemcpy(f->d_hoff64, h64.data(), sizeof(double4) * h64.size(), cudaMemcpyHostToDevice), "copy");
    }
    f->box_version = sys->box_version;
    return PMGPU_OK;
}

// Grid::dftmod (base/Grid.h:650-665) of the order-P B-spline at w = 0
static void dftmod(int order, int n, std::vector<double>& mod)
{
    std::vector<double> th(order), dth(order);
    // BSpline::set(0.0) (base/BSpline.cpp:64-117)
    double w = 0.0;
    if (order == 2) { th[1] = w; th[0] = 1.0 - w; }
    else {
        th[order - 1] = 0.0; th[1] = w; th[0] = 1.0 - w;
        for (int k = 2; k < order - 1; k++) {
            double div = 1.0 / k;
            th[k] = div * w * th[k - 1];
            for (int j = 1; j < k; j++)
                th[k - j] = div * ((w + j) * th[k - j - 1] + (k + 1 - j - w) * th[k - j]);
            th[0] = div * (1 - w) * th[0];
        }
        double div = 1.0 / (order - 1.0);
        th[order - 1] = div * w * th[order - 2];
        for (int j = 1; j < order - 1; j++)
            th[order - 1 - j] = div * ((w + j) * th[order - j - 2] + (order - j - w) * th[order - 1 - j]);
        th[0] = div * (1 - w) * th[0];
    }
    mod.resize(n);
    for (unsigned int i = 0; i < (unsigned)n; i++) {
        double sc = 0.0, ss = 0.0;
        for (unsigned int j = 0; j < (unsigned)order; j++) {
            double x = kPi * 2.0 * i * j / (double)n;
            sc += th[j] * std::cos(x);
            ss += th[j] * std::sin(x);
        }
        mod[i] = 1.0 / (sc * sc + ss * ss);
    }
}

// grid sizes of prime factors 2, 3, 5 and 7 (the reference's FFT, base/fft.c
// fftfact_, handles the same: radices 2, 3, 4, 5, 7)
static bool smooth_ok(int n)
{
    int m = n;
    for (int f : {2, 3, 5, 7})
        while (m > 1 && m % f == 0) m /= f;
    return m == 1;
}

extern "C" int pmgpu_pme_create(pmgpu_system* sys, const pmgpu_pme_params* p, pmgpu_force** out)
{
    if (!sys || !p || !out) return PMGPU_ERR_ARG;
    *out = nullptr;
    // NonbondedPMEwaldSystemForce::doMake validation (:1099-1139)
    std::string err;
    if (p->order < 2 || (p->order % 2) != 0) err += "PMEwald order (=" + std::to_string(p->order) + ") > 1 and even.";
    if (p->grid[0] < p->order || p->grid[1] < p->order || p->grid[2] < p->order)
        err += "PMEwald force: order <= nx, ny, nz.";
    if (!(p->cutoff > 0.0)) err += "PMEwald cutoff > 0.";
    if (!(p->accuracy > 0.0)) err += "PMEwald accuracy > 0.";
    if (!err.empty()) return fail(sys, PMGPU_ERR_ARG, " force PMEwald :" + err);
    if (p->order > 12) return fail(sys, PMGPU_ERR_UNSUPPORTED, "PME order > 12");
    // the (real, reciprocal, correction) sets of the registered exemplars
    // (factories/registerForceExemplarsFastElectrostatic.cpp:50-55)
    if (!(p->real || p->reciprocal || p->correction) || (p->real && p->reciprocal && !p->correction))
        return fail(sys, PMGPU_ERR_UNSUPPORTED, "PMEwald: no registered exemplar with these terms");
    for (int k = 0; k < 3; ++k)
        if (!smooth_ok(p->grid[k]) || p->grid[k] > 4096)
            return fail(sys, PMGPU_ERR_UNSUPPORTED, "PME grid size needs prime factors 2, 3, 5, 7 and <= 4096");
    if (p->precision != PMGPU_PRECISION_MIXED && p->precision != PMGPU_PRECISION_FP64)
        return fail(sys, PMGPU_ERR_ARG, "unknown precision");
    if (!sys->box_set || sys->n == 0 && sys->q.empty()) {
        // allowed: tables are built lazily at the first evaluation
    }
    pmgpu_force* f = new pmgpu_force();
    f->sys = sys;
    f->kind = 1;
    f->precision = p->precision;
    f->pp = *p;
    // alpha: bisection of erfc(alpha Rc)/Rc = accuracy (:564-586)
    double alpha = p->alpha, rc = p->cutoff;
    if (alpha <= 0.0) {
        alpha = 1.0;
        while (std::erfc(alpha * rc) / rc >= p->accuracy) alpha *= 2.0;
        double low = 0., high = alpha;
        for (unsigned int i = 0; i < 100; ++i) {
            alpha = 0.5 * (low + high);
            if (std::erfc(alpha * rc) / rc >= p->accuracy) low = alpha; else high = alpha;
        }
    }
    f->alpha = alpha;
    if (p->real) {
        // realTerm (:658-768) with only the zero lattice vector (every box
        // edge > 2 Rc, checked at evaluation) is the CoulombEwaldReal pair
        // force with a Cutoff switch at Rc: same pair set, exclusions (FULL
        // skipped, MODIFIED scaled by csf), poly5 energy and force
        pmgpu_cutoff_params cp;
        memset(&cp, 0, sizeof(cp));
        cp.n_terms = 1;
        cp.pot[0] = PMGPU_POT_EWALD_REAL; cp.sw[0] = PMGPU_SW_CUTOFF;
        cp.cutoff[0] = rc; cp.alpha[0] = alpha; cp.algorithm_cutoff = rc;
        cp.precision = p->precision;
        pmgpu_force* sub = nullptr;
        int r = pmgpu_cutoff_create(sys, &cp, &sub);
        if (r) { delete f; return r; }
        sys->forces.erase(sub);
        f->real_sub = sub;
    }
    sys->forces.insert(f);
    *out = f;
    return PMGPU_OK;
}

static int prepare_pme(pmgpu_force* f)
{
    pmgpu_system* sys = f->sys;
    if (f->box_version == sys->box_version && f->topo_version == sys->topo_version) return PMGPU_OK;
    const pmgpu_pme_params& p = f->pp;
    f->n_lattice = 0;
    if (pme_needs_lattice(f)) {
        // PeriodicBoundaryConditions::buildLatticeVectors(Rc)
        // (topology/PeriodicBoundaryConditions.cpp:80-111): k, l, m up to
        // floor(Rc / L + 1), |v| <= 2 Rc, sorted by norm, (0, 0, 0) first
        // (NonbondedPMEwaldSystemForce.h:630-631)
        const double rc = p.cutoff, lx = sys->box[0], ly = sys->box[4], lz = sys->box[8];
        const int bk = (int)std::floor(rc / std::fabs(lx) + 1.0), bl = (int)std::floor(rc / std::fabs(ly) + 1.0),
                  bm = (int)std::floor(rc / std::fabs(lz) + 1.0);
        std::vector<double4> lat;
        for (int k = -bk; k <= bk; k++)
            for (int l = -bl; l <= bl; l++)
                for (int m = -bm; m <= bm; m++)
                    if (k != 0 || l != 0 || m != 0) {
                        const double x = lx * k, y = ly * l, z = lz * m;
                        const double n2 = x * x + y * y + z * z;
                        if (std::sqrt(n2) <= 2 * rc) lat.push_back(make_double4(x, y, z, n2));
                    }
        std::stable_sort(lat.begin(), lat.end(), [](const double4& a, const double4& b) { return a.w < b.w; });
        lat.insert(lat.begin(), make_double4(0.0, 0.0, 0.0, 0.0));
        CK(dalloc(&f->d_lattice, lat.size()), "alloc");
        CK(cudaMemcpy(f->d_lattice, lat.data(), sizeof(double4) * lat.size(), cudaMemcpyHostToDevice), "copy");
        f->n_lattice = (int)lat.size();
    }
    int kx = p.grid[0], ky = p.grid[1], kz = p.grid[2];
    f->kzh = kz / 2 + 1;
    double LX = sys->box[0], LY = sys->box[4], LZ = sys->box[8];
    double alpha = f->alpha;
    double fac = kPi * kPi / (alpha * alpha);
    // exp tables and B-spline moduli (Grid::initialize, base/Grid.h:557-648)
    std::vector<double> ex(kx), ey(ky), ez(f->kzh);
    for (unsigned i = 0; i < (unsigned)kx; i++) {
        int i0 = i <= (unsigned)kx / 2 ? (int)i : (int)i - kx;
        double m = i0 * (1.0 / LX);
        ex[i] = std::exp(-fac * (m * m));
    }
    for (unsigned j = 0; j < (unsigned)ky; j++) {
        int j0 = j <= (unsigned)ky / 2 ? (int)j : (int)j - ky;
        double m = j0 * (1.0 / LY);
        ey[j] = std::exp(-fac * (m * m));
    }
    for (int k = 0; k < f->kzh; k++) {
        double m = k * (1.0 / LZ);
        ez[k] = std::exp(-fac * (m * m));
    }
    std::vector<double> mx, my, mz;
    dftmod(p.order, kx, mx); dftmod(p.order, ky, my); dftmod(p.order, kz, mz);
    std::vector<double> bf, ef;
    bf.insert(bf.end(), mx.begin(), mx.end()); bf.insert(bf.end(), my.begin(), my.end());
    bf.insert(bf.end(), mz.begin(), mz.begin() + f->kzh);
    ef.insert(ef.end(), ex.begin(), ex.end()); ef.insert(ef.end(), ey.begin(), ey.end());
    ef.insert(ef.end(), ez.begin(), ez.end());
    CK(dalloc(&f->d_bfac, bf.size()), "alloc"); CK(dalloc(&f->d_efac, ef.size()), "alloc");
    CK(cudaMemcpy(f->d_bfac, bf.data(), sizeof(double) * bf.size(), cudaMemcpyHostToDevice), "copy");
    CK(cudaMemcpy(f->d_efac, ef.data(), sizeof(double) * ef.size(), cudaMemcpyHostToDevice), "copy");
    // twiddles exp(-2 pi i k / n) per axis
    f->twx = 0; f->twy = kx; f->twz = kx + ky;
    int ntw = kx + ky + kz;
    std::vector<double> tw(2 * (size_t)ntw);
    int ns[3] = {kx, ky, kz};
    int offs[3] = {f->twx, f->twy, f->twz};
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < ns[a]; ++k) {
            long double ang = 2.0L * 3.141592653589793238462643383279502884L * k / ns[a];
            tw[2 * (offs[a] + k)] = (double)cosl(ang);
            tw[2 * (offs[a] + k) + 1] = (double)-sinl(ang);
        }
    size_t nreal = (size_t)kx * ky * kz, nhalf = (size_t)kx * ky * f->kzh;
    if (f->precision == PMGPU_PRECISION_FP64) {
        CK(dalloc((double2**)&f->d_tw, ntw), "alloc");
        CK(cudaMemcpy(f->d_tw, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice), "copy");
        CK(dalloc((double2**)&f->d_cgrid, nhalf), "alloc");
        CK(dalloc((double**)&f->d_rgrid, nreal), "alloc");
        CK(dalloc(&f->d_qgrid, nreal), "alloc");
    } else {
        std::vector<float> twf(tw.size());
        for (size_t k = 0; k < tw.size(); ++k) twf[k] = (float)tw[k];
        CK(dalloc((float2**)&f->d_tw, ntw), "alloc");
        CK(cudaMemcpy(f->d_tw, twf.data(), sizeof(float) * twf.size(), cudaMemcpyHostToDevice), "copy");
        CK(dalloc((float2**)&f->d_cgrid, nhalf), "alloc");
        CK(dalloc((float**)&f->d_rgrid, nreal), "alloc");
        CK(dalloc(&f->d_qgrid, nreal), "alloc");
        // the reciprocal energy and virial from FP64 B-spline weights and an
        // FP64 forward transform of the fixed-point charge grid; the FP32
        // chain gives the forces.  With the FP32 weights and transform the
        // reciprocal energy is off by ~1e-3 kcal/mol per 10^4 atoms, which
        // reaches the total energy of water boxes (a near cancellation of
        // the real-space, reciprocal and self terms): 2.5e-7 of the total on
        // a 9,000-atom box at 45^3, 5.9e-7 on 1,000,000 atoms at 216^3.
        CK(dalloc((double2**)&f->d_tw64, ntw), "alloc");
        CK(cudaMemcpy(f->d_tw64, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice), "copy");
        CK(dalloc((double2**)&f->d_cgrid64, nhalf), "alloc");
    }
    // point self energy and charged-system term (:604-628)
    double V = std::fabs(sys->box[0] * sys->box[4] * sys->box[8]);
    double q2 = 0.0, q1 = 0.0;
    for (int i = 0; i < sys->n; ++i) q2 += sys->q[i] * sys->q[i];
    for (int i = 0; i < sys->n; ++i) q1 += sys->q[i];
    f->self_energy = p.correction ? -q2 * alpha / std::sqrt(kPi) : 0.0;
    f->charged_energy = 0.0;
    if (p.correction && std::fabs(q1 * 0.00268283) > 1.0e-5)
        f->charged_energy = -kPi / (2.0 * V * (alpha * alpha)) * q1 * q1;
    f->box_version = sys->box_version;
    f->topo_version = sys->topo_version;
    return PMGPU_OK;
}

static void free_force(pmgpu_force* f)
{
    if (f->real_sub) free_force(f->real_sub);
    dfree(f->d_deltas); dfree(f->d_doff); dfree(f->d_qgrid); dfree(f->d_lattice);
    dfree(f->d_hdeltas); dfree(f->d_hoff); dfree(f->d_hoff_lo); dfree(f->d_hoff64);
    if (f->d_cgrid) cudaFree(f->d_cgrid);
    if (f->d_rgrid) cudaFree(f->d_rgrid);
    if (f->d_tw) cudaFree(f->d_tw);
    if (f->d_cgrid64) cudaFree(f->d_cgrid64);
    if (f->d_tw64) cudaFree(f->d_tw64);
    dfree(f->d_hq);
    if (f->d_hc) cudaFree(f->d_hc);
    if (f->d_hr) cudaFree(f->d_hr);
    dfree(f->d_bfac); dfree(f->d_efac);
    for (int k = 0; k < 2; ++k) { dfree(f->d_tab64[k]); dfree(f->d_tab32[k]); }
    delete f;
}

extern "C" int pmgpu_force_destroy(pmgpu_force* f)
{
    if (!f) return PMGPU_OK;
    pmgpu_system* sys = f->sys;
    cudaSetDevice(sys->device);
    cudaStreamSynchronize(sys->stream);
    sys->forces.erase(f);
    free_force(f);
    return PMGPU_OK;
}

extern "C" int pmgpu_pme_alpha(pmgpu_force* f, double* alpha)
{
    if (!f || !alpha || f->kind != 1) return PMGPU_ERR_ARG;
    *alpha = f->alpha;
    return PMGPU_OK;
}

// ------------------------------------------------------------------ evaluate
static int bin(pmgpu_system* sys, const double* d_pos)
{
    BinArgs a;
    a.skey = sys->d_skey; a.cstart = sys->d_cstart; a.cbox = sys->d_cbox; a.ccell = sys->d_ccell;
    a.ncl_cap = sys->cbox_cap;
    a.n = sys->n; a.pos = d_pos; a.q = sys->d_q; a.type = sys->d_type; a.mol = sys->d_mol;
    a.pbc = sys->pbc; a.grid = sys->grid;
    a.cell_lin = sys->d_cell_lin; a.cell3 = sys->d_cell3; a.counts = sys->d_counts; a.done = sys->d_status + 8;
    a.start = sys->d_start; a.tmp = sys->d_tmp; a.sorted = sys->d_sorted; a.slot_of = sys->d_slot;
    a.spos = sys->d_spos; a.slo = sys->d_slo; a.smeta = sys->d_smeta; a.spos64 = sys->d_spos64;
    a.status = sys->d_status;
    int e = launch_bin(a, sys->stream, &sys->launches);
    if (e) return cuda_fail(sys, (cudaError_t)e, "binning");
    sys->binned = true;
    return PMGPU_OK;
}

// K1c: the column-cluster layout of the positions (and the reference cell of
// every atom, as bin() gives it)
static int col_bin(pmgpu_system* sys, const double* d_pos)
{
    ColBinArgs a;
    memset(&a, 0, sizeof(a));
    a.n = sys->n; a.pos = d_pos; a.q = sys->d_q; a.type = sys->d_type; a.mol = sys->d_mol;
    a.pbc = sys->pbc; a.grid = sys->grid; a.cell3 = sys->d_cell3;
    a.g = sys->eval_cg;
    a.qfix = sys->d_qfix; a.col = sys->d_colid; a.counts = sys->d_ccounts; a.done = sys->d_status + 9;
    a.colstart = sys->d_colstart; a.ccstart = sys->d_ccstart; a.tmp = sys->d_ctmp; a.zidx = sys->d_zidx;
    a.cq = sys->d_cq; a.cm = sys->d_cm; a.slot_of = sys->d_cslot;
    a.ibox = sys->d_ibox; a.jbox = sys->d_jbox; a.ccol = sys->d_ccol; a.ncl_cap = sys->col_ncl_cap;
    a.corg = sys->d_corg;
    a.status = sys->d_status;
    int e = launch_col_bin(a, sys->stream, &sys->launches);
    if (e) return cuda_fail(sys, (cudaError_t)e, "column binning");
    sys->binned = true;
    return PMGPU_OK;
}

// between rebuilds of a reused list: the current positions into the slots
static int col_refresh(pmgpu_system* sys, const double* d_pos)
{
    ColBinArgs a;
    memset(&a, 0, sizeof(a));
    a.n = sys->n; a.pos = d_pos; a.pbc = sys->pbc; a.grid = sys->grid; a.cell3 = sys->d_cell3;
    a.g = sys->eval_cg; a.qfix = sys->d_qfix; a.cq = sys->d_cq; a.slot_of = sys->d_cslot; a.status = sys->d_status;
    int e = launch_col_refresh(a, 0.5 * sys->list_skin, sys->stream, &sys->launches);
    if (e) return cuda_fail(sys, (cudaError_t)e, "pair list refresh");
    sys->binned = true;
    return PMGPU_OK;
}

// the column-path members of the pair arguments
static void fill_col_args(pmgpu_system* sys, PairArgs& a)
{
    a.cq = sys->d_cq; a.cm = sys->d_cm; a.ibox = sys->d_ibox; a.jbox = sys->d_jbox;
    a.ccstart = sys->d_ccstart; a.ccol = sys->d_ccol; a.icl_cap = sys->col_ncl_cap; a.corg = sys->d_corg;
    a.zidx = sys->d_zidx;
    a.clist = (int4*)sys->d_plist;          // entries of two int2 places each (plist_cap counts int2)
    a.cg = sys->eval_cg;
    a.qorig = sys->d_q; a.torig = sys->d_type;
    a.facc = sys->d_facc32c;
    a.list_skin = sys->list_every > 1 ? (float)sys->list_skin : 0.0f;
}

// The pair kernels a force runs in this evaluation: the FP64 ones for an
// FP64 force, and for a mixed cutoff force when the tuning asks for them
// (fp64_pairs: no cluster list and no near-pair pass, the shorter launch
// chain that is faster on systems of a few hundred atoms)
// internal evaluation flags (never a caller's): the evaluation's energy
// output (kFlagZeroOut), and its force output too (kFlagZeroForces), start at
// zero, set by the graph's zero kernel (pmgpu_evaluate's own buffers)
constexpr unsigned kFlagZeroOut = 1u << 30;
constexpr unsigned kFlagZeroForces = 1u << 29;
constexpr unsigned kFlagsInternal = kFlagZeroOut | kFlagZeroForces;

static inline bool pairs64(const pmgpu_system* sys, const pmgpu_force* f)
{
    return f->precision == PMGPU_PRECISION_FP64 || (f->kind == 0 && sys->tuning.fp64_pairs);
}

static void fill_pair_args(pmgpu_system* sys, pmgpu_force* f, const double* d_pos, PairArgs& a)
{
    memset(&a, 0, sizeof(a));
    a.start = sys->d_start; a.spos = sys->d_spos; a.slo = sys->d_slo; a.smeta = sys->d_smeta;
    a.spos64 = sys->d_spos64; a.cstart = sys->d_cstart; a.cbox = sys->d_cbox;
    a.pos = d_pos;
    a.xfull = sys->d_xfull; a.xmod = sys->d_xmod; a.xrow = sys->d_xrow; a.xent = sys->d_xent;
    a.ljn = sys->d_ljn; a.ljm = sys->d_ljm; a.ljd = sys->d_ljd; a.n_types = sys->t;
    a.deltas = f->d_deltas; a.doff = f->d_doff; a.nd = f->nd;
    a.hdeltas = f->d_hdeltas; a.hoff = f->d_hoff; a.hoff_lo = f->d_hoff_lo; a.nh = f->nh;
    a.half_rule = f->half_rule; a.ccell = sys->d_ccell; a.ncl_cap = sys->cbox_cap;
    a.plist = sys->d_plist; a.plist_cap = (int)sys->plist_cap;
    a.chunks = sys->d_chunks; a.chunk_cap = (int)sys->chunk_cap;
    a.near = sys->d_near; a.near_cap = (int)sys->near_cap;
    a.chunk = sys->tuning.chunk_entries; a.blocks_per_sm = sys->tuning.pair_blocks_per_sm;
    a.near_count = sys->d_status + 6; a.near_need = sys->d_status + 7;
    a.plist_count = sys->d_plist_count; a.plist_need = sys->d_plist_need;
    a.chunk_count = sys->d_chunk_count; a.chunk_need = sys->d_chunk_need; a.chunk_next = sys->d_chunk_next;
    a.hoff64 = f->d_hoff64; a.efix = sys->d_efix;
    a.grid = sys->grid; a.pbc = sys->pbc; a.wrap = f->wrap;
    a.lx_lo = (float)(sys->box[0] - (double)(float)sys->box[0]);
    a.ly_lo = (float)(sys->box[4] - (double)(float)sys->box[4]);
    a.lz_lo = (float)(sys->box[8] - (double)(float)sys->box[8]);
    a.erec_stride = sys->erec_cap;
    a.lx = (float)sys->box[0]; a.ly = (float)sys->box[4]; a.lz = (float)sys->box[8];
    a.ilx = (float)(1.0 / sys->box[0]); a.ily = (float)(1.0 / sys->box[4]); a.ilz = (float)(1.0 / sys->box[8]);
    a.n_terms = f->cp.n_terms;
    a.tf[0] = f->tf[0]; a.tf[1] = f->tf[1]; a.td[0] = f->td[0]; a.td[1] = f->td[1];
    a.cut2f = (float)f->cut2; a.cut2d = f->cut2;
    a.guard = 2.0e-5f;
    // the energies of pairs closer than 5 A are recomputed in FP64: they hold
    // nearly all of the FP32 energy rounding (|e| up to ~30 kcal/mol each on
    // water, where the total is a ~1e-3 cancellation of the sum of |e|)
    a.near2 = sys->d_near ? 25.0f : 0.0f;
    a.csf = (float)sys->csf; a.csfd = sys->csf;
    a.status = sys->d_status;
    // mixed forces on whole-cell shifts go to the pair accumulator (their
    // virial is completed from it at finalize), the small-grid mode to the other
    if (pairs64(sys, f)) { a.facc = sys->d_facc40; a.scale = kScaleFp64; }
    else { a.facc = f->wrap ? sys->d_facc32p : sys->d_facc32; a.scale = kScaleMixed; }
}

static int ensure_erec(pmgpu_system* sys, int need)
{
    if (need <= sys->erec_cap) return PMGPU_OK;
    int cap = std::max(need, 2 * sys->erec_cap);
    CK(dalloc(&sys->d_erec, (size_t)cap * kERec), "alloc");
    sys->erec_cap = cap;
    sys->buf_version++;          // a captured graph holds the old buffer
    return PMGPU_OK;
}

// energy records one cutoff force writes
static int pair_records(pmgpu_system* sys, pmgpu_force* f)
{
    // the mixed kernel sums energies in fixed point (d_efix), no records
    if (f->kind == 2) return adjoint_blocks(sys->n);
    return pairs64(sys, f) ? pair_blocks(sys->grid, f->nd) : 0;
}

// upper bound of the energy records of the fused x pass (one per CTA, at
// least one x-line per CTA)
static int pme_xblocks(const pmgpu_force* f) { return f->pp.grid[1] * f->kzh; }

// Everything that allocates or copies synchronously: force tables, buffer
// capacities.  Runs before an evaluation is enqueued (or captured).
static int eval_prepare(pmgpu_system* sys, int nf, pmgpu_force* const* forces, unsigned flags)
{
    if (nf < 0 || (nf > 0 && !forces)) return fail(sys, PMGPU_ERR_ARG, "bad force list");
    bool periodic = false;
    for (int k = 0; k < nf; ++k) periodic |= forces[k] && forces[k]->kind != 2;
    if (periodic && !sys->box_set) return fail(sys, PMGPU_ERR_STATE, "box not set (pmgpu_set_box)");
    int need = 1;
    for (int k = 0; k < nf; ++k) {
        pmgpu_force* f = forces[k];
        if (!f || f->sys != sys) return fail(sys, PMGPU_ERR_ARG, "force belongs to another system");
        int r = f->kind == 0 ? prepare_cutoff(f) : (f->kind == 1 ? prepare_pme(f) : PMGPU_OK);
        if (r) return r;
        if (f->kind != 1) need += pair_records(sys, f);
        else need += pme_xblocks(f) + 2 * 148 * 4;    // FFT energy, correction, lattice real space
    }
    need += (sys->n + 255) / 256;   // finalize: pair virial records
    int r = ensure_erec(sys, need);
    if (r) return r;
    if (flags & PMGPU_FLAG_MOLECULAR_VIRIAL) {
        // the molecule positions come from the caller (GenericTopology::
        // molecules[m].position, set by the integrator or front end)
        if (!sys->molpos_set)
            return fail(sys, PMGPU_ERR_STATE, "molecular virial without molecule positions (pmgpu_set_molecule_positions)");
        int mneed = 1, n_pme = 0;
        for (int k = 0; k < nf; ++k) {
            pmgpu_force* f = forces[k];
            if (f->kind == 2)
                return fail(sys, PMGPU_ERR_UNSUPPORTED, "molecular virial of an all-pairs (vacuum) force");
            if (f->kind == 0) mneed += pair_blocks(sys->grid, f->nd);
            if (f->kind == 1) {
                ++n_pme;
                if (f->pp.real && pme_needs_lattice(f)) mneed += 148 * 4;
                if (f->pp.reciprocal) mneed += pme_molvir_blocks(sys->n);
            }
        }
        if (n_pme > 4) return fail(sys, PMGPU_ERR_UNSUPPORTED, "molecular virial with more than 4 PME forces");
        if (mneed > sys->mrec_cap) {
            int cap = std::max(mneed, 2 * sys->mrec_cap);
            CK(dalloc(&sys->d_mrec, (size_t)cap * kMRec), "alloc");
            sys->mrec_cap = cap;
            sys->buf_version++;
        }
    }
    // clusters: at most N / 8 full ones plus one partial per cell
    int ncl = sys->n / kCluster + sys->grid.ncell + 1;
    if (ncl > sys->cbox_cap) {
        CK(dalloc(&sys->d_cbox, 2 * (size_t)ncl), "alloc");
        CK(dalloc(&sys->d_ccell, (size_t)ncl), "alloc");
        sys->cbox_cap = ncl;
        sys->buf_version++;
    }
    // the column-cluster path takes the mixed cutoff forces of the group when
    // none of them is in the small-grid mode and the box suits the largest
    // of their cutoffs; otherwise the cell-cluster path takes them all
    sys->eval_use_col = false;
    {
        double rc2 = 0.0;
        bool any = false, ok = true;
        for (int k = 0; k < nf; ++k)
            if (forces[k]->kind == 0 && !pairs64(sys, forces[k])) {
                any = true;
                ok = ok && !forces[k]->wrap;
                rc2 = std::max(rc2, forces[k]->cut2);
            }
        if (any && ok) {
            if (sys->col_grid_stale) {
                int rg = col_set_grid(sys);
                if (rg) return rg;
                sys->col_grid_stale = false;
            }
            ColGrid g;
            if (col_reach(sys, std::sqrt(rc2) + sys->list_skin, g)) {
                sys->eval_use_col = true;
                sys->eval_cg = g;
            }
        }
    }
    long long lneed = 0, cneed = 0;
    if (sys->eval_use_col) {
        const ColGrid& g = sys->eval_cg;
        const int icl = sys->n / kCluster + g.ncol + 1;
        if (icl > sys->col_ncl_cap) {
            const size_t slots = (size_t)kCluster * icl;
            CK(dalloc(&sys->d_cq, slots), "alloc"); CK(dalloc(&sys->d_cm, slots), "alloc");
            CK(dalloc(&sys->d_ibox, 2 * (size_t)icl), "alloc"); CK(dalloc(&sys->d_jbox, 4 * (size_t)icl), "alloc");
            CK(dalloc(&sys->d_ccol, (size_t)icl), "alloc"); CK(dalloc(&sys->d_facc32c, 3 * slots), "alloc");
            CK(dalloc(&sys->d_corg, (size_t)icl), "alloc");
            sys->col_ncl_cap = icl;
            sys->buf_version++;
        }
        double rc2 = 0.0;
        for (int k = 0; k < nf; ++k)
            if (forces[k]->kind == 0 && !pairs64(sys, forces[k])) rc2 = std::max(rc2, forces[k]->cut2);
        const long long entries = col_list_estimate(sys->n, g, g.lx * g.ly * g.lz, std::sqrt(rc2) + sys->list_skin);
        lneed = 2 * entries;                  // int4 entries in the int2 list buffer
        cneed = col_chunk_estimate(entries, sys->n, g, sys->tuning.chunk_entries);
    } else {
        for (int k = 0; k < nf; ++k)
            if (forces[k]->kind == 0 && !pairs64(sys, forces[k])) {
                lneed = std::max(lneed, plist_estimate(sys->n, sys->grid, forces[k]->nh));
                cneed = std::max(cneed, chunk_estimate(sys->n, sys->grid, forces[k]->nh, sys->tuning.chunk_entries));
            }
    }
    if (lneed > 0) {
        lneed = std::max(lneed, sys->plist_need + sys->plist_need / 4);
        cneed = std::max(cneed, sys->chunk_need + sys->chunk_need / 4);
        if (lneed > INT_MAX || cneed > INT_MAX)
            return fail(sys, PMGPU_ERR_CAPACITY, "cluster-pair list above 2^31 entries");
        if (lneed > sys->plist_cap) {
            CK(dalloc(&sys->d_plist, (size_t)lneed), "alloc");
            sys->plist_cap = lneed;
            sys->buf_version++;
        }
        if (cneed > sys->chunk_cap) {
            CK(dalloc(&sys->d_chunks, (size_t)cneed), "alloc");
            sys->chunk_cap = cneed;
            sys->buf_version++;
        }
        // near pairs (< 5 A): ~26 per atom in water
        long long nneed = std::max(30LL * sys->n + 4096, sys->near_need + sys->near_need / 4);
        if (nneed > INT_MAX / 2) return fail(sys, PMGPU_ERR_CAPACITY, "near-pair list above 2^30 entries");
        if (nneed > sys->near_cap) {
            CK(dalloc(&sys->d_near, (size_t)nneed), "alloc");
            sys->near_cap = nneed;
            sys->buf_version++;
        }
    }
    pme_init_attributes();
    return PMGPU_OK;
}

static cudaEvent_t prof_event(pmgpu_system* sys)
{
    if (sys->prof_next == sys->prof_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        sys->prof_pool.push_back(e);
    }
    return sys->prof_pool[sys->prof_next++];
}

// CUDA-event timing of one phase of an evaluation (profiling mode only)
static int prof_begin(pmgpu_system* sys, int phase)
{
    if (!sys->profiling) return -1;
    ProfMark m;
    m.phase = phase;
    m.b = prof_event(sys);
    m.e = nullptr;
    cudaEventRecord(m.b, sys->stream);
    sys->prof_marks.push_back(m);
    return (int)sys->prof_marks.size() - 1;
}

static void prof_end(pmgpu_system* sys, int m)
{
    if (m < 0) return;
    sys->prof_marks[m].e = prof_event(sys);
    cudaEventRecord(sys->prof_marks[m].e, sys->stream);
}

// One evaluation's enqueue, in parts, so that a batch can run its members'
// column-path pair kernels as one launch between them: run_begin (memsets,
// the PME branch, binning, all-pairs forces), run_cutoffs (the cutoff
// forces in order; with may_defer, the first column-path mixed force stops
// after its list, its arguments left in dargs), run_resume (that force's
// near pairs after the batch's pair kernel, the remaining cutoff forces,
// run_end) and run_end (molecular virial, PME join, finalize, energy
// reduction).  Only asynchronous work on the system's stream (capturable
// in a graph).
struct EvalRun {
    pmgpu_system* sys = nullptr;
    int nf = 0;
    pmgpu_force* const* forces = nullptr;
    const double* d_pos = nullptr;
    double* d_fout = nullptr;
    double* d_energy = nullptr;
    unsigned flags = 0;
    int virial = 0;
    bool molvir = false;
    int mused = 0;                      // molecular virial records
    MolvirFinish mf;
    bool use32 = false, use40 = false;
    size_t n3 = 0;
    int mbin = -1;
    bool any_cut = false, any_pme = false, any_full = false;
    bool use_col = false, mixed_cells = false, cell_sort = false, mv_bin = false;
    bool fork = false;                  // PME on the side stream beside the pair kernels
    bool near_on_side = false;
    int used = 0;                       // energy records
    int last_mixed = -1;                // the last mixed cutoff force (its near pairs may go to the side stream)
    int lists = 0;
    int pair_virial = 0, col_virial = 0;
    int k_next = 0;                     // the next force run_cutoffs looks at
    int deferred = -1;                  // the force whose pair kernel a batch runs
    PairArgs dargs;                     // its arguments
};

// the names of one evaluation's state (EvalRun) inside its parts
#define PM_EVAL_RUN_NAMES(R)                                                                              \
    [[maybe_unused]] pmgpu_system* sys = (R).sys;                                                        \
    [[maybe_unused]] const int nf = (R).nf;                                                              \
    [[maybe_unused]] pmgpu_force* const* forces = (R).forces;                                            \
    [[maybe_unused]] const double* d_pos = (R).d_pos;                                                    \
    [[maybe_unused]] double* d_fout = (R).d_fout;                                                        \
    [[maybe_unused]] double* d_energy = (R).d_energy;                                                    \
    [[maybe_unused]] int& virial = (R).virial;                                                           \
    [[maybe_unused]] bool& molvir = (R).molvir;                                                          \
    [[maybe_unused]] int& mused = (R).mused;                                                             \
    [[maybe_unused]] MolvirFinish& mf = (R).mf;                                                          \
    [[maybe_unused]] bool& use32 = (R).use32;                                                            \
    [[maybe_unused]] bool& use40 = (R).use40;                                                            \
    [[maybe_unused]] size_t& n3 = (R).n3;                                                                \
    [[maybe_unused]] bool& any_cut = (R).any_cut;                                                        \
    [[maybe_unused]] bool& any_pme = (R).any_pme;                                                        \
    [[maybe_unused]] bool& any_full = (R).any_full;                                                      \
    [[maybe_unused]] bool& use_col = (R).use_col;                                                        \
    [[maybe_unused]] bool& mixed_cells = (R).mixed_cells;                                                \
    [[maybe_unused]] bool& cell_sort = (R).cell_sort;                                                    \
    [[maybe_unused]] bool& mv_bin = (R).mv_bin;                                                          \
    [[maybe_unused]] bool& fork = (R).fork;                                                              \
    [[maybe_unused]] bool& near_on_side = (R).near_on_side;                                              \
    [[maybe_unused]] int& used = (R).used;                                                               \
    [[maybe_unused]] int& last_mixed = (R).last_mixed;                                                   \
    [[maybe_unused]] int& lists = (R).lists;                                                             \
    [[maybe_unused]] int& pair_virial = (R).pair_virial;                                                 \
    [[maybe_unused]] int& col_virial = (R).col_virial;                                                   \
    [[maybe_unused]] cudaStream_t s = sys->stream;                                                       \
    [[maybe_unused]] int r = PMGPU_OK;

// PME: reads only positions and charges and accumulates in atom order.
// Beside the pair kernels (branches = true) the correction term and the
// FP64 energy transform of a mixed force run on branches of their own,
// joined back into ps at the end.
static int run_pme(EvalRun& R, cudaStream_t ps, bool branches)
{
    PM_EVAL_RUN_NAMES(R)
        bool corr_branch = false, e64_branch = false;
        for (int k = 0; k < nf; ++k) {
            pmgpu_force* f = forces[k];
            if (f->kind != 1) continue;
            const bool fp64 = pairs64(sys, f);
            unsigned long long* facc = fp64 ? sys->d_faccA + n3 : sys->d_faccA;
            const double scale = fp64 ? kScaleFp64 : kScaleMixed;
            const pmgpu_pme_params& p = f->pp;
            if (p.correction) {
                CorrArgs c;
                c.n_excl = sys->e; c.pairs = sys->d_epairs; c.cls = sys->d_ecls; c.pos = d_pos; c.q = sys->d_q;
                c.slot_of = nullptr; c.pbc = sys->pbc; c.alpha = f->alpha; c.alpha2 = f->alpha * f->alpha;
                c.two_alpha_pi = 2.0 * f->alpha / std::sqrt(kPi); c.csf = sys->csf;
                c.facc = facc; c.scale = scale; c.erec = sys->d_erec + used; c.erec_stride = sys->erec_cap;
                c.status = sys->d_status;
                c.virial = virial;
                c.const_energy = f->self_energy + f->charged_energy;
                c.const_virial = f->charged_energy;
                int b = 0;
                int m = prof_begin(sys, kPhaseCorrection);
                cudaStream_t cs = ps;
                if (branches && !corr_branch) {
                    CK(cudaEventRecord(sys->ev_corr, ps), "fork");
                    CK(cudaStreamWaitEvent(sys->side3, sys->ev_corr, 0), "fork");
                    corr_branch = true;
                }
                if (corr_branch) cs = sys->side3;
                int e = launch_pme_correction(c, cs, &sys->launches, &b);
                if (e) return cuda_fail(sys, (cudaError_t)e, "PME correction");
                prof_end(sys, m);
                used += b;
            }
            if (p.real && f->n_lattice > 0) {
                RealLatArgs la;
                memset(&la, 0, sizeof(la));
                la.n = sys->n; la.pos = d_pos; la.q = sys->d_q; la.mol = sys->d_mol;
                la.xfull = sys->d_xfull; la.xmod = sys->d_xmod; la.xrow = sys->d_xrow; la.xent = sys->d_xent;
                la.pbc = sys->pbc; la.lattice = f->d_lattice; la.n_lattice = f->n_lattice;
                la.rc2 = f->pp.cutoff * f->pp.cutoff; la.alpha = f->alpha;
                la.two_alpha_pi = 2.0 * f->alpha / std::sqrt(kPi); la.csf = sys->csf;
                la.facc = facc; la.scale = scale; la.erec = sys->d_erec + used; la.erec_stride = sys->erec_cap;
                la.status = sys->d_status; la.virial = virial;
                int b = 0;
                int m = prof_begin(sys, kPhasePair);
                int e = launch_pme_real_lattice(la, ps, &sys->launches, &b);
                if (e) return cuda_fail(sys, (cudaError_t)e, "PME real space (lattice images)");
                prof_end(sys, m);
                used += b;
                if (molvir) {
                    la.molpos = sys->d_molpos; la.mrec = sys->d_mrec + mused; la.mrec_stride = sys->mrec_cap;
                    e = launch_pme_real_lattice_molvir(la, ps, &sys->launches, &b);
                    if (e) return cuda_fail(sys, (cudaError_t)e, "PME real space molecular virial");
                    mused += b;
                }
            }
            if (p.reciprocal) {
                PmeArgs a;
                memset(&a, 0, sizeof(a));
                a.n = sys->n; a.pos = d_pos; a.q = sys->d_q; a.sorted = nullptr; a.slot_of = nullptr;
                a.kx = p.grid[0]; a.ky = p.grid[1]; a.kz = p.grid[2]; a.kzh = f->kzh; a.order = p.order;
                double LX = sys->box[0], LY = sys->box[4], LZ = sys->box[8];
                a.hxr = p.grid[0] / LX; a.hyr = p.grid[1] / LY; a.hzr = p.grid[2] / LZ;
                a.offx = -(p.order - 1) / 2 + p.grid[0];
                a.offy = -(p.order - 1) / 2 + p.grid[1];
                a.offz = -(p.order - 1) / 2 + p.grid[2];
                a.qgrid = f->d_qgrid; a.cgrid = f->d_cgrid; a.rgrid = f->d_rgrid; a.tw = f->d_tw;
                a.cgrid64 = fp64 ? nullptr : f->d_cgrid64; a.tw64 = f->d_tw64;
                a.twx = f->twx; a.twy = f->twy; a.twz = f->twz;
                a.bfac = f->d_bfac; a.efac = f->d_efac;
                a.piVr = 1.0 / (kPi * (LX * LY * LZ));
                a.fac = kPi * kPi / (f->alpha * f->alpha);
                a.wr = 1.0 / LX; a.lr = 1.0 / LY; a.hr = 1.0 / LZ;
                a.facc = facc; a.scale = scale; a.qscale = kScaleFp64; a.erec_stride = sys->erec_cap;
                a.status = sys->d_status; a.virial = virial; a.fft_lines = sys->tuning.fft_lines;
                a.mol = sys->d_mol; a.molpos = sys->d_molpos; a.pbc = sys->pbc;
                a.mrec = sys->d_mrec; a.mrec_stride = sys->mrec_cap;
                const bool e64 = branches && a.cgrid64 != nullptr && !e64_branch;
                // profiling times the FP64 energy transform as a phase of its own
                const bool e64_timed = sys->profiling && a.cgrid64 != nullptr;
                a.energy64_apart = (e64 || e64_timed) ? 1 : 0;
                const int phases[3] = {kPhaseSpread, kPhaseFft, kPhaseGather};
                const int stages[3] = {kStageSpread, kStageFft, kStageGather};
                for (int st = 0; st < 3; ++st) {
                    int m = prof_begin(sys, phases[st]);
                    int u = 0;
                    int e = launch_pme_reciprocal(a, fp64 ? 1 : 0, ps, &sys->launches,
                                                  sys->d_erec + used, &u, stages[st]);
                    if (e) return cuda_fail(sys, (cudaError_t)e, "PME reciprocal");
                    // scalarSum's records: its tensor is the molecular virial's too
                    if (molvir && u > 0) {
                        mf.range_first[mf.nranges] = used;
                        mf.range_count[mf.nranges++] = u;
                    }
                    used += u;
                    prof_end(sys, m);
                    if (st == 2 && e64_timed) {
                        int me = prof_begin(sys, kPhaseEnergy64);
                        int ue = 0;
                        e = launch_pme_reciprocal(a, 0, ps, &sys->launches, sys->d_erec + used, &ue, kStageEnergy64);
                        if (e) return cuda_fail(sys, (cudaError_t)e, "PME energy transform");
                        if (molvir && ue > 0) {
                            mf.range_first[mf.nranges] = used;
                            mf.range_count[mf.nranges++] = ue;
                        }
                        used += ue;
                        prof_end(sys, me);
                    }
                    if (st == 2 && molvir) {
                        PmeArgs am = a;
                        am.mrec = sys->d_mrec + mused;
                        int um = 0;
                        e = launch_pme_reciprocal(am, fp64 ? 1 : 0, ps, &sys->launches, nullptr, &um, kStageMolvir);
                        if (e) return cuda_fail(sys, (cudaError_t)e, "PME reciprocal molecular virial");
                        mused += pme_molvir_blocks(sys->n);
                    }
                    if (st == 0 && e64) {
                        // the FP64 energy transform reads only the charge grid:
                        // from the spread on, beside the FP32 transform and gather
                        CK(cudaEventRecord(sys->ev_spread, ps), "fork");
                        CK(cudaStreamWaitEvent(sys->side2, sys->ev_spread, 0), "fork");
                        u = 0;
                        e = launch_pme_reciprocal(a, 0, sys->side2, &sys->launches, sys->d_erec + used, &u,
                                                  kStageEnergy64);
                        if (e) return cuda_fail(sys, (cudaError_t)e, "PME energy transform");
                        if (molvir && u > 0) {
                            mf.range_first[mf.nranges] = used;
                            mf.range_count[mf.nranges++] = u;
                        }
                        used += u;
                        e64_branch = true;
                    }
                }
            }
        }
        if (corr_branch) {
            CK(cudaEventRecord(sys->ev_corr, sys->side3), "join");
            CK(cudaStreamWaitEvent(ps, sys->ev_corr, 0), "join");
        }
        if (e64_branch) {
            CK(cudaEventRecord(sys->ev_e64, sys->side2), "join");
            CK(cudaStreamWaitEvent(ps, sys->ev_e64, 0), "join");
        }
        return PMGPU_OK;
}

// the near pairs' FP64 energies of cutoff force k after its pair kernel
static int run_near(EvalRun& R, int k, const PairArgs& a, bool fp64, bool col)
{
    PM_EVAL_RUN_NAMES(R)
    pmgpu_force* f = forces[k];
    if (fp64 || !(a.near2 > 0.0f)) return PMGPU_OK;
    // the last cutoff force's near-pair energies (needed only by the energy
    // reduction) run on the side stream, after PME, beside finalize; earlier
    // forces' before the next list reuses the buffer
    cudaStream_t ns = s;
    if (fork && k == last_mixed) {
        CK(cudaEventRecord(sys->ev_pair, s), "event");
        CK(cudaStreamWaitEvent(sys->side, sys->ev_pair, 0), "event");
        ns = sys->side;
    }
    int e = col ? launch_near_energy_col(a, f->combo, sys->n, ns, &sys->launches)
                : launch_near_energy(a, f->combo, sys->n, ns, &sys->launches);
    if (e) return cuda_fail(sys, (cudaError_t)e, "near-pair energies");
    if (ns != s) {
        CK(cudaEventRecord(sys->ev_near, sys->side), "event");
        near_on_side = true;
    }
    return PMGPU_OK;
}

static int run_begin(EvalRun& R)
{
    PM_EVAL_RUN_NAMES(R)
    const unsigned flags = R.flags;
    virial = (flags & PMGPU_FLAG_VIRIAL) ? 1 : 0;
    molvir = (flags & PMGPU_FLAG_MOLECULAR_VIRIAL) != 0;
    mused = 0;
    memset(&mf, 0, sizeof(mf));
    use32 = use40 = false;
    for (int k = 0; k < nf; ++k) (pairs64(sys, forces[k]) ? use40 : use32) = true;
    n3 = 3 * (size_t)sys->n;
    R.mbin = prof_begin(sys, kPhaseBin);
    // the evaluation's counters and accumulators start at zero: one launch
    // for all of them (k_zero) instead of a memset node each
    ZeroRanges zr;
    memset(&zr, 0, sizeof(zr));
    auto zero = [&zr](void* p, size_t bytes) {
        zr.p[zr.count] = static_cast<unsigned*>(p);
        zr.words[zr.count++] = (long long)(bytes / sizeof(unsigned));
    };
    if (sys->eval_reuse) {
        // the list's counts (ints 1-4) stay; the status, the work counter,
        // the near-pair counts, the binning counters and the sums start at zero
        zero(sys->d_small, sizeof(int));
        zero((char*)sys->d_small + 5 * sizeof(int), kSmallBytes - 5 * sizeof(int));
    } else {
        zero(sys->d_small, kSmallBytes);
    }
    any_cut = any_pme = any_full = false;
    bool atom_mixed = false, atom_fp64 = false;        // PME / all-pairs forces of each precision
    for (int k = 0; k < nf; ++k) {
        any_cut |= forces[k]->kind == 0;
        any_pme |= forces[k]->kind == 1;
        any_full |= forces[k]->kind == 2;
        if (forces[k]->kind != 0) (pairs64(sys, forces[k]) ? atom_fp64 : atom_mixed) = true;
    }
    use_col = sys->eval_use_col;
    // the cell-ordered mixed accumulators serve the cell path's mixed cutoff
    // forces only; the atom-ordered ones (mixed half, FP64 half) PME and the
    // all-pairs forces of that precision
    mixed_cells = false;
    for (int k = 0; k < nf; ++k)
        if (forces[k]->kind == 0 && !pairs64(sys, forces[k]) && !use_col) mixed_cells = true;
    if (mixed_cells) zero(sys->d_facc32, 2 * sizeof(unsigned long long) * n3);
    if (use40) zero(sys->d_facc40, sizeof(unsigned long long) * n3);
    if (atom_mixed) zero(sys->d_faccA, sizeof(unsigned long long) * n3);
    if (atom_fp64) zero(sys->d_faccA + n3, sizeof(unsigned long long) * n3);
    for (int k = 0; k < nf; ++k)
        if (forces[k]->kind == 0 && forces[k]->precision != PMGPU_PRECISION_FP64)
            sys->last_layout = pairs64(sys, forces[k]) ? PMGPU_LAYOUT_FP64
                             : (use_col ? PMGPU_LAYOUT_COLUMNS : PMGPU_LAYOUT_CELLS);
    if (use_col) zero(sys->d_facc32c, sizeof(unsigned long long) * 3 * kCluster * (size_t)sys->col_ncl_cap);
    if (flags & kFlagZeroOut) zero(d_energy, sizeof(double) * kEOut);
    if (flags & kFlagZeroForces) zero(d_fout, sizeof(double) * n3);
    {
        int e = launch_zero(zr, s, &sys->launches);
        if (e) return cuda_fail(sys, (cudaError_t)e, "zero");
    }
    // the cell-sorted order: for the FP64 cutoff forces, and for the mixed
    // ones when the column path does not take them
    cell_sort = false;
    for (int k = 0; k < nf; ++k)
        if (forces[k]->kind == 0 && (pairs64(sys, forces[k]) || !use_col)) cell_sort = true;
    // the molecular virial kernels of the cutoff forces read the cell-sorted
    // order too (binned for them alone on the column path)
    mv_bin = molvir && any_cut && !cell_sort;
    used = 0;
    // with cutoff forces too, PME runs on the side stream from the start,
    // beside binning, the list and the pair kernels, and is joined before
    // finalize (not while profiling, which times every phase alone)
    fork = any_cut && any_pme && !sys->profiling && sys->tuning.pme_concurrent;
    if (fork) {
        CK(cudaEventRecord(sys->ev_fork, s), "fork");
        CK(cudaStreamWaitEvent(sys->side, sys->ev_fork, 0), "fork");
        r = run_pme(R, sys->side, true);
        if (r) return r;
        CK(cudaEventRecord(sys->ev_join, sys->side), "join");
    }
    if (cell_sort || mv_bin) {
        r = bin(sys, d_pos);
        if (r) return r;
    }
    if (use_col) {
        r = sys->eval_reuse ? col_refresh(sys, d_pos) : col_bin(sys, d_pos);
        if (r) return r;
    }
    prof_end(sys, R.mbin);
    // vacuum all-pairs forces: the recompute kernel in forward mode, forces in
    // atom order like PME
    for (int k = 0; k < nf; ++k) {
        pmgpu_force* f = forces[k];
        if (f->kind != 2) continue;
        const bool fp64 = pairs64(sys, f);
        AdjArgs a;
        adj_pair_args(sys, f, a);
        a.pos = d_pos;
        a.facc = fp64 ? sys->d_faccA + n3 : sys->d_faccA;
        a.scale = fp64 ? kScaleFp64 : kScaleMixed;
        a.erec = sys->d_erec + used; a.erec_stride = sys->erec_cap; a.virial = virial;
        int m = prof_begin(sys, kPhasePair);
        int e = launch_pair_adjoint(a, fp64 ? 1 : 0, s, &sys->launches);
        if (e) return cuda_fail(sys, (cudaError_t)e, "all-pairs force");
        prof_end(sys, m);
        used += pair_records(sys, f);
    }
    last_mixed = -1;
    for (int k = 0; k < nf; ++k)
        if (forces[k]->kind == 0 && !pairs64(sys, forces[k])) last_mixed = k;
    near_on_side = false;
    lists = 0;
    pair_virial = col_virial = 0;
    R.k_next = 0;
    R.deferred = -1;
    return PMGPU_OK;
}

static int run_cutoffs(EvalRun& R, bool may_defer)
{
    PM_EVAL_RUN_NAMES(R)
    for (int k = R.k_next; k < nf; ++k) {
        R.k_next = k + 1;
        pmgpu_force* f = forces[k];
        if (f->kind != 0) continue;
        const bool fp64 = pairs64(sys, f);
        const bool col = !fp64 && use_col;
        if (!fp64 && !col && !f->wrap && virial) pair_virial = 1;
        if (col && virial) col_virial = 1;
        PairArgs a;
        fill_pair_args(sys, f, d_pos, a);
        if (col) fill_col_args(sys, a);
        a.virial = virial;
        a.erec = sys->d_erec + used;
        if (!fp64 && !(col && sys->eval_reuse)) {
            // list count and need, chunk count and need, work counter
            if (lists++ > 0) CK(cudaMemsetAsync(sys->d_plist_count, 0, 6 * sizeof(int), s), "memset");
            int ml = prof_begin(sys, kPhaseList);
            int e = col ? launch_col_list(a, s, &sys->launches) : launch_cluster_list(a, s, &sys->launches);
            if (e) return cuda_fail(sys, (cudaError_t)e, "cluster-pair list");
            prof_end(sys, ml);
        }
        if (may_defer && col && !sys->eval_reuse) {
            // a batch runs this pair kernel with its other members' (run_resume)
            R.deferred = k;
            R.dargs = a;
            return PMGPU_OK;
        }
        int m = prof_begin(sys, kPhasePair);
        int e = fp64 ? launch_pair_fp64(a, f->combo, pair_blocks(sys->grid, f->nd), s, &sys->launches)
                     : (col ? launch_pair_col(a, f->combo, s, &sys->launches)
                            : launch_pair_mixed(a, f->combo, s, &sys->launches));
        if (e) return cuda_fail(sys, (cudaError_t)e, "pair kernel");
        r = run_near(R, k, a, fp64, col);
        if (r) return r;
        prof_end(sys, m);
        used += pair_records(sys, f);
    }
    return PMGPU_OK;
}

static int run_end(EvalRun& R)
{
    PM_EVAL_RUN_NAMES(R)
    if (molvir) {
        // the cutoff forces' molecular virial over the cell-sorted order
        for (int k = 0; k < nf; ++k) {
            pmgpu_force* f = forces[k];
            if (f->kind != 0) continue;
            PairArgs a;
            fill_pair_args(sys, f, d_pos, a);
            a.molpos = sys->d_molpos; a.mrec = sys->d_mrec + mused; a.mrec_stride = sys->mrec_cap;
            const int blocks = pair_blocks(sys->grid, f->nd);
            int e = launch_pair_molvir(a, f->combo, blocks, s, &sys->launches);
            if (e) return cuda_fail(sys, (cudaError_t)e, "molecular virial");
            mused += blocks;
        }
    }
    if (fork) {
        CK(cudaStreamWaitEvent(s, sys->ev_join, 0), "join");
    } else if (any_pme) {
        r = run_pme(R, s, false);
        if (r) return r;
    }
    int mfin = prof_begin(sys, kPhaseFinalize);
    if (use32 || use40) {
        FinArgs fa;
        memset(&fa, 0, sizeof(fa));
        fa.n = sys->n;
        // the slot-ordered accumulators exist only with the cell-sorted order
        fa.f32 = mixed_cells ? sys->d_facc32 : nullptr;
        fa.f32p = mixed_cells ? sys->d_facc32p : nullptr;
        fa.f40 = use40 && cell_sort ? sys->d_facc40 : nullptr;
        if (use_col) {
            fa.c32 = sys->d_facc32c; fa.c_slot_of = sys->d_cslot; fa.cq = sys->d_cq;
            fa.c_slots = kCluster * sys->col_ncl_cap;
            fa.corg = sys->d_corg;
            fa.cscale[0] = sys->eval_cg.lx / 4294967296.0;
            fa.cscale[1] = sys->eval_cg.ly / 4294967296.0;
            fa.cscale[2] = sys->eval_cg.lz / 4294967296.0;
        }
        for (int k = 0; k < nf; ++k)
            if (forces[k]->kind != 0) {
                if (pairs64(sys, forces[k])) fa.a40 = sys->d_faccA + n3;
                else fa.a32 = sys->d_faccA;
            }
        fa.sorted = cell_sort ? sys->d_sorted : nullptr; fa.spos = sys->d_spos; fa.slo = sys->d_slo;
        fa.pair_virial = pair_virial | (col_virial << 1);
        fa.fout = d_fout;
        fa.erec = sys->d_erec + used; fa.erec_stride = sys->erec_cap;
        int rec = 0;
        int e = launch_finalize(fa, s, &sys->launches, &rec);
        if (e) return cuda_fail(sys, (cudaError_t)e, "finalize");
        used += rec;
    }
    if (nf > 0) {
        if (near_on_side) CK(cudaStreamWaitEvent(s, sys->ev_near, 0), "join");
        int e = launch_energy_reduce(sys->d_erec, sys->erec_cap, used, sys->d_efix, d_energy, s, &sys->launches);
        if (e) return cuda_fail(sys, (cudaError_t)e, "energy reduce");
        if (molvir) {
            mf.mrec = sys->d_mrec; mf.mstride = sys->mrec_cap; mf.nmrec = mused;
            mf.erec = sys->d_erec; mf.estride = sys->erec_cap;
            mf.virial = virial; mf.out = d_energy;
            e = launch_molvir_finish(mf, s, &sys->launches);
            if (e) return cuda_fail(sys, (cudaError_t)e, "molecular virial");
        }
    }
    prof_end(sys, mfin);
    return PMGPU_OK;
}

static int run_resume(EvalRun& R)
{
    const int k = R.deferred;
    R.deferred = -1;
    int r = run_near(R, k, R.dargs, false, true);
    if (r) return r;
    R.used += pair_records(R.sys, R.forces[k]);
    r = run_cutoffs(R, false);
    if (r) return r;
    return run_end(R);
}

static void run_init(EvalRun& R, pmgpu_system* sys, int nf, pmgpu_force* const* forces, const double* d_pos,
                     double* d_fout, double* d_energy, unsigned flags)
{
    R = EvalRun();
    R.sys = sys; R.nf = nf; R.forces = forces; R.d_pos = d_pos; R.d_fout = d_fout; R.d_energy = d_energy;
    R.flags = flags;
}

static int eval_enqueue(pmgpu_system* sys, int nf, pmgpu_force* const* forces, const double* d_pos,
                        double* d_fout, double* d_energy, unsigned flags)
{
    EvalRun R;
    run_init(R, sys, nf, forces, d_pos, d_fout, d_energy, flags);
    int r = run_begin(R);
    if (r) return r;
    r = run_cutoffs(R, false);
    if (r) return r;
    return run_end(R);
}

// prepare, then enqueue -- replaying a captured CUDA graph when the same
// forces run on the same buffers again (the evaluation is one graph launch)
static int eval_core(pmgpu_system* sys, int nf_in, pmgpu_force* const* forces_in, const double* d_pos,
                     double* d_fout, double* d_energy, unsigned flags)
{
    // a PME force with -real brings its real-space pair force along (boxes
    // whose edges all exceed 2 Rc; in smaller ones its lattice kernel runs)
    std::vector<pmgpu_force*> all;
    for (int k = 0; k < nf_in; ++k) {
        if (!forces_in || !forces_in[k]) return fail(sys, PMGPU_ERR_ARG, "bad force list");
        if (forces_in[k]->real_sub && !pme_needs_lattice(forces_in[k])) all.push_back(forces_in[k]->real_sub);
        all.push_back(forces_in[k]);
    }
    const int nf = (int)all.size();
    pmgpu_force* const* forces = all.data();
    int r = eval_prepare(sys, nf, forces, flags);
    if (r) return r;
    // a reused pair list: the column path with one mixed cutoff force (its
    // list is the system's only one), a rebuild period above one, a list
    // built for these forces, still valid and younger than the period
    std::vector<long long> ids;
    int n_mixed_cut = 0;
    for (int k = 0; k < nf; ++k) {
        ids.push_back(forces[k]->id);
        if (forces[k]->kind == 0 && !pairs64(sys, forces[k])) ++n_mixed_cut;
    }
    const bool can_reuse = sys->eval_use_col && sys->list_every > 1 && n_mixed_cut == 1;
    sys->eval_reuse = can_reuse && sys->list_valid && sys->list_ids == ids && sys->evals_since_build < sys->list_every;
    auto note_list = [&]() {
        if (!sys->eval_use_col || n_mixed_cut == 0) return;
        if (sys->eval_reuse) {
            sys->evals_since_build++;
        } else {
            sys->list_builds++;
            sys->list_valid = can_reuse;
            sys->list_ids = ids;
            sys->evals_since_build = 1;
        }
    };
    if (sys->profiling || !sys->use_graphs) {
        r = eval_enqueue(sys, nf, forces, d_pos, d_fout, d_energy, flags);
        if (!r) note_list();
        return r;
    }
    GraphKey key;
    key.ids = ids;
    key.reuse = sys->eval_reuse ? 1 : 0;
    key.pos = d_pos; key.fout = d_fout; key.energy = d_energy; key.flags = flags;
    key.box_version = sys->box_version; key.topo_version = sys->topo_version; key.buf_version = sys->buf_version;
    cudaStream_t s = sys->stream;
    pmgpu_system::GraphEntry* hit = nullptr;
    for (auto& g : sys->graphs)
        if (g.key == key) { hit = &g; break; }
    if (!hit) {
        const size_t kGraphCache = 4;
        long long l0 = sys->launches;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "graph capture");
        r = eval_enqueue(sys, nf, forces, d_pos, d_fout, d_energy, flags);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (r) { if (graph) cudaGraphDestroy(graph); return r; }
        if (e != cudaSuccess) return cuda_fail(sys, e, "graph capture");
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_fail(sys, e, "graph instantiate");
        if (sys->graphs.size() >= kGraphCache) {    // replace the least recently used
            auto lru = sys->graphs.begin();
            for (auto it = sys->graphs.begin(); it != sys->graphs.end(); ++it)
                if (it->last_use < lru->last_use) lru = it;
            cudaGraphExecDestroy(lru->exec);
            sys->graphs.erase(lru);
        }
        pmgpu_system::GraphEntry g;
        g.key = key;
        g.exec = exec;
        g.launches = sys->launches - l0;
        sys->launches = l0;
        sys->graphs.push_back(g);
        hit = &sys->graphs.back();
    }
    hit->last_use = ++sys->graph_clock;
    CK(cudaGraphLaunch(hit->exec, s), "graph launch");
    sys->launches += hit->launches;
    note_list();
    return PMGPU_OK;
}

extern "C" int pmgpu_evaluate_device(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces,
                                     const double* d_positions, double* d_forces_accum,
                                     double* d_energies, unsigned flags)
{
    if (!sys || !d_positions || !d_forces_accum || !d_energies) return PMGPU_ERR_ARG;
    cudaSetDevice(sys->device);
    // without PMGPU_FLAG_VIRIAL every kernel adds zero to the virial slots
    return eval_core(sys, n_forces, forces, d_positions, d_forces_accum, d_energies, flags & ~kFlagsInternal);
}

extern "C" int pmgpu_evaluate(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces,
                              const double* positions, double* forces_accum,
                              pmgpu_energies* energies, unsigned flags)
{
    if (!sys || !positions || !forces_accum || !energies) return PMGPU_ERR_ARG;
    cudaSetDevice(sys->device);
    if (sys->n == 0 && sys->q.empty() && sys->d_pos == nullptr) return fail(sys, PMGPU_ERR_STATE, "topology not set");
    size_t n3 = 3 * (size_t)sys->n;
    cudaStream_t s = sys->stream;
    const size_t fbytes = sizeof(double) * n3;
    CK(cudaMemcpyAsync(sys->d_pos, positions, fbytes, cudaMemcpyHostToDevice, s), "H2D positions");
    // A page-locked accumulator goes to the device, the evaluation adds to it
    // there and the sum comes back in its place (no pass over it on the
    // host); a pageable one stays on the host (two pageable copies cost more
    // than the addition) and receives the forces from a pinned buffer.
    cudaPointerAttributes pa;
    const bool pinned = cudaPointerGetAttributes(&pa, forces_accum) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();                          // a pageable pointer may leave an error on older drivers
    if (pinned) CK(cudaMemcpyAsync(sys->d_acc0, forces_accum, fbytes, cudaMemcpyHostToDevice, s), "H2D forces");
    const unsigned zflags = pinned ? kFlagZeroOut : (kFlagZeroOut | kFlagZeroForces);
    int r = PMGPU_OK;
    // a second attempt only when the cluster-pair list outgrew its estimate
    // (the first attempt recorded the size it needs)
    for (int attempt = 0; attempt < 2; ++attempt) {
        // the energies are zeroed inside the evaluation's graph; the status
        // word comes back with the results (one wait, no second round trip)
        if (pinned) CK(cudaMemcpyAsync(sys->d_fout, sys->d_acc0, fbytes, cudaMemcpyDeviceToDevice, s), "copy forces");
        r = eval_core(sys, n_forces, forces, sys->d_pos, sys->d_fout, sys->d_energy,
                      (flags & ~kFlagsInternal) | zflags);
        if (r) break;
        CK(cudaMemcpyAsync(pinned ? forces_accum : sys->h_fbuf, sys->d_fout, fbytes, cudaMemcpyDeviceToHost, s),
           "D2H forces");
        CK(cudaMemcpyAsync(sys->h_energy, sys->d_energy, sizeof(double) * kEOut, cudaMemcpyDeviceToHost, s), "D2H energies");
        CK(cudaMemcpyAsync(sys->h_status, sys->d_status, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H status");
        sys->col_just_disabled = false;
        sys->list_just_invalidated = false;
        CK(cudaStreamSynchronize(s), "synchronize");
        r = status_result(sys, *sys->h_status);
        if (!(r == PMGPU_ERR_CAPACITY && (sys->plist_need > sys->plist_cap || sys->chunk_need > sys->chunk_cap ||
                                          sys->near_need > sys->near_cap || sys->col_just_disabled ||
                                          sys->list_just_invalidated)))
            break;
    }
    if (r) {
        // a failed evaluation leaves the caller's accumulator as it was
        const int r0 = r;
        if (pinned && cudaMemcpyAsync(forces_accum, sys->d_acc0, fbytes, cudaMemcpyDeviceToHost, s) == cudaSuccess)
            cudaStreamSynchronize(s);
        return r0;
    }
    if (!pinned)
        for (size_t k = 0; k < n3; ++k) forces_accum[k] += sys->h_fbuf[k];
    energies->lennard_jones += sys->h_energy[0];
    energies->coulomb += sys->h_energy[1];
    // with the molecular virial alone the atomic slots hold the
    // inter-molecular pairs' part (ScalarStructure::addVirial(f, d, comDiff))
    if (flags & (PMGPU_FLAG_VIRIAL | PMGPU_FLAG_MOLECULAR_VIRIAL))
        for (int k = 0; k < 9; ++k) energies->virial[k] += sys->h_energy[2 + k];
    if (flags & PMGPU_FLAG_MOLECULAR_VIRIAL) {
        pmgpu_energies_mol* em = reinterpret_cast<pmgpu_energies_mol*>(energies);
        for (int k = 0; k < 9; ++k) em->molecular_virial[k] += sys->h_energy[11 + k];
    }
    return PMGPU_OK;
}

extern "C" int pmgpu_set_molecule_positions(pmgpu_system* sys, int n_molecules, const double* positions)
{
    if (!sys || !positions) return PMGPU_ERR_ARG;
    if (sys->n == 0 && sys->q.empty()) return fail(sys, PMGPU_ERR_STATE, "topology not set");
    if (n_molecules != sys->n_mol)
        return fail(sys, PMGPU_ERR_ARG, "one position per molecule of the topology is needed");
    cudaSetDevice(sys->device);
    if (!sys->d_molpos) {
        CK(dalloc(&sys->d_molpos, 3 * (size_t)std::max(n_molecules, 1)), "alloc");
        sys->buf_version++;
    }
    // stream-ordered: the next evaluation reads these positions
    if (n_molecules > 0)
        CK(cudaMemcpyAsync(sys->d_molpos, positions, sizeof(double) * 3 * (size_t)n_molecules,
                           cudaMemcpyHostToDevice, sys->stream), "H2D molecule positions");
    sys->molpos_set = true;
    return PMGPU_OK;
}

// ------------------------------------------------------------------ diagnostics
extern "C" int pmgpu_pair_layout(pmgpu_system* sys) { return sys ? sys->last_layout : 0; }

extern "C" int pmgpu_set_pair_list(pmgpu_system* sys, double skin, int rebuild_every)
{
    if (!sys) return PMGPU_ERR_ARG;
    if (!(skin >= 0.0 && skin <= 10.0) || rebuild_every < 1) return fail(sys, PMGPU_ERR_ARG, "skin 0..10 A, period >= 1");
    sys->list_skin = rebuild_every > 1 ? skin : 0.0;
    sys->list_every = rebuild_every;
    sys->list_valid = false;
    sys->buf_version++;                // graphs captured for another list
    return PMGPU_OK;
}

extern "C" long long pmgpu_pair_list_builds(pmgpu_system* sys) { return sys ? sys->list_builds : 0; }

extern "C" int pmgpu_get_cells(pmgpu_system* sys, int* cells, int* dims)
{
    if (!sys || !cells || !dims) return PMGPU_ERR_ARG;
    if (!sys->binned) return fail(sys, PMGPU_ERR_STATE, "no evaluation yet");
    cudaSetDevice(sys->device);
    CK(cudaStreamSynchronize(sys->stream), "sync");
    CK(cudaMemcpy(cells, sys->d_cell3, sizeof(int) * 3 * (size_t)sys->n, cudaMemcpyDeviceToHost), "copy");
    dims[0] = sys->grid.nx; dims[1] = sys->grid.ny; dims[2] = sys->grid.nz;
    return PMGPU_OK;
}

extern "C" int pmgpu_get_pairs(pmgpu_system* sys, pmgpu_force* f, const double* positions,
                               long long* count, int* pairs, long long cap)
{
    if (!sys || !f || !positions || !count || (cap > 0 && !pairs)) return PMGPU_ERR_ARG;
    if (pme_needs_lattice(f))
        return fail(sys, PMGPU_ERR_UNSUPPORTED, "pair recording of PMEwald -real with lattice images");
    if (f->kind != 0 && f->real_sub) f = f->real_sub;   // PME -real: its real-space pairs
    if (f->kind != 0) return fail(sys, PMGPU_ERR_UNSUPPORTED, "pair recording is for cutoff forces");
    if (!sys->box_set) return fail(sys, PMGPU_ERR_STATE, "box not set");
    cudaSetDevice(sys->device);
    int r = eval_prepare(sys, 1, &f, 0);
    if (r) return r;
    cudaStream_t s = sys->stream;
    size_t n3 = 3 * (size_t)sys->n;
    CK(cudaMemcpyAsync(sys->d_pos, positions, sizeof(double) * n3, cudaMemcpyHostToDevice, s), "H2D");
    CK(cudaMemsetAsync(sys->d_small, 0, kSmallBytes, s), "memset");
    CK(cudaMemsetAsync(sys->d_facc32, 0, 2 * sizeof(unsigned long long) * n3, s), "memset");
    CK(cudaMemsetAsync(sys->d_facc40, 0, sizeof(unsigned long long) * n3, s), "memset");
    bool fp64 = pairs64(sys, f);
    const bool col = !fp64 && sys->eval_use_col;          // eval_prepare decided for this force alone
    if (f->precision != PMGPU_PRECISION_FP64)
        sys->last_layout = fp64 ? PMGPU_LAYOUT_FP64 : (col ? PMGPU_LAYOUT_COLUMNS : PMGPU_LAYOUT_CELLS);
    if (col) {
        CK(cudaMemsetAsync(sys->d_facc32c, 0, sizeof(unsigned long long) * 3 * kCluster * (size_t)sys->col_ncl_cap, s),
           "memset");
        r = col_bin(sys, sys->d_pos);
    } else {
        r = bin(sys, sys->d_pos);
    }
    if (r) return r;
    r = ensure_erec(sys, std::max(1, pair_records(sys, f)));
    if (r) return r;
    int* d_pairs = nullptr;
    unsigned long long* d_count = nullptr;
    long long dcap = cap > 0 ? cap : 1;
    CK(cudaMalloc((void**)&d_pairs, sizeof(int) * 2 * (size_t)dcap), "alloc");
    CK(cudaMalloc((void**)&d_count, sizeof(unsigned long long)), "alloc");
    CK(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s), "memset");
    PairArgs a;
    fill_pair_args(sys, f, sys->d_pos, a);
    if (col) fill_col_args(sys, a);
    a.near2 = 0.0f;                                    // recording only: no near-pair list
    a.erec = sys->d_erec;
    a.rec_pairs = d_pairs; a.rec_count = d_count; a.rec_cap = dcap;
    int e = fp64 ? launch_pair_fp64(a, f->combo, pair_blocks(sys->grid, f->nd), s, &sys->launches)
                 : (col ? launch_col_list(a, s, &sys->launches) : launch_cluster_list(a, s, &sys->launches));
    if (!e && !fp64) e = col ? launch_pair_col(a, f->combo, s, &sys->launches)
                             : launch_pair_mixed(a, f->combo, s, &sys->launches);
    unsigned long long cnt = 0;
    int st = 0;
    if (!e) e = (int)cudaMemcpyAsync(&cnt, d_count, sizeof(cnt), cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaMemcpyAsync(&st, sys->d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!e) e = (int)cudaStreamSynchronize(s);
    if (!e && (st & (kStatusListFull | kStatusColumns))) {
        // the list did not fit (or the column path refused the system): the
        // recording is incomplete; the next call runs with the grown buffers
        cudaFree(d_pairs);
        cudaFree(d_count);
        (void)pmgpu_synchronize(sys);                  // records the sizes needed (and its message)
        return PMGPU_ERR_CAPACITY;
    }
    if (!e && cnt > 0 && cap > 0)
        e = (int)cudaMemcpy(pairs, d_pairs, sizeof(int) * 2 * (size_t)std::min<long long>(cnt, cap), cudaMemcpyDeviceToHost);
    cudaFree(d_pairs);
    cudaFree(d_count);
    if (e) return cuda_fail(sys, (cudaError_t)e, "pair recording");
    *count = (long long)cnt;
    if ((long long)cnt > cap) return fail(sys, PMGPU_ERR_CAPACITY, "pair capacity too small");
    return PMGPU_OK;
}

// ------------------------------------------------------------------ allocation-free PME reciprocal
// pmgpu_pme_reciprocal_static: the PME reciprocal-space term (spread, FFT
// with the convolution, gather) in mixed precision, on scratch memory that
// the library reserves statically in every GPU that loads it, so that the
// call itself never allocates.  The kernels are the ones the PME force uses.
//
// Layout of the scratch (each part 256-byte aligned):
//   charge grid   int64  x kStaticGrid
//   half spectrum float2 x kStaticHalf
//   real grid     float  x kStaticGrid
//   forces        int64  x 3 kStaticAtoms (fixed point, 2^32)
//   identity      int    x kStaticAtoms (atom order = slot order)
//   records       double x 11 kStaticRecords (energy/virial per FFT block)
//   twiddles      float2 x 3 kStaticAxis
//   moduli, exp   double x 3 kStaticAxis each
//   status        int
namespace {
constexpr int kStaticAtoms = 65536;
constexpr int kStaticGrid = 64 * 64 * 64;
constexpr int kStaticHalf = 3 * 65536;
constexpr int kStaticAxis = 1024;
constexpr int kStaticRecords = 8192;

constexpr size_t st_align(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kOffQgrid = 0;
constexpr size_t kOffCgrid = kOffQgrid + st_align(sizeof(long long) * kStaticGrid);
constexpr size_t kOffRgrid = kOffCgrid + st_align(sizeof(float2) * kStaticHalf);
constexpr size_t kOffFacc = kOffRgrid + st_align(sizeof(float) * kStaticGrid);
constexpr size_t kOffIdent = kOffFacc + st_align(sizeof(unsigned long long) * 3 * kStaticAtoms);
constexpr size_t kOffErec = kOffIdent + st_align(sizeof(int) * kStaticAtoms);
constexpr size_t kOffTw = kOffErec + st_align(sizeof(double) * kERec * kStaticRecords);
constexpr size_t kOffBfac = kOffTw + st_align(sizeof(float2) * 3 * kStaticAxis);
constexpr size_t kOffEfac = kOffBfac + st_align(sizeof(double) * 3 * kStaticAxis);
constexpr size_t kOffStatus = kOffEfac + st_align(sizeof(double) * 3 * kStaticAxis);
constexpr size_t kStaticBytes = kOffStatus + 256;   // about 8.4 MB
}  // namespace

// The scratch itself.  In host code this name is only a stand-in for the
// device symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_pme_scratch[kStaticBytes];

__global__ void k_static_identity(int* ident, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ident[i] = i;
}

// Device address of the scratch on the current device, looked up (and the
// identity map filled) on the first call per device.
static std::mutex g_static_mutex;
static std::map<int, unsigned char*> g_static_base;

static int static_scratch(int device, unsigned char** base)
{
    std::lock_guard<std::mutex> lock(g_static_mutex);
    auto it = g_static_base.find(device);
    if (it != g_static_base.end()) { *base = it->second; return PMGPU_OK; }
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_pme_scratch) != cudaSuccess || !ptr) return PMGPU_ERR_CUDA;
    unsigned char* b = (unsigned char*)ptr;
    k_static_identity<<<(kStaticAtoms + 255) / 256, 256>>>((int*)(b + kOffIdent), kStaticAtoms);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return PMGPU_ERR_CUDA;
    g_static_base[device] = b;
    *base = b;
    return PMGPU_OK;
}

extern "C" int pmgpu_pme_reciprocal_static(int device, int n_atoms, const double* d_positions,
                                           const double* d_scaled_charges, const double box[3], const int grid[3],
                                           int order, double alpha, double* d_forces_accum, double* d_energies,
                                           unsigned flags, void* stream)
{
    if (!box || !grid || !d_forces_accum || !d_energies) return PMGPU_ERR_ARG;
    if (n_atoms < 0 || (n_atoms > 0 && (!d_positions || !d_scaled_charges))) return PMGPU_ERR_ARG;
    if (order < 2 || order % 2 != 0 || order > 12) return PMGPU_ERR_ARG;
    if (!(alpha > 0.0) || !(box[0] > 0.0) || !(box[1] > 0.0) || !(box[2] > 0.0)) return PMGPU_ERR_ARG;
    const int kx = grid[0], ky = grid[1], kz = grid[2];
    if (kx < order || ky < order || kz < order) return PMGPU_ERR_ARG;
    // the FFT's radices, as pmgpu_pme_create checks them
    if (!smooth_ok(kx) || !smooth_ok(ky) || !smooth_ok(kz)) return PMGPU_ERR_UNSUPPORTED;
    const int kzh = kz / 2 + 1;
    // the sizes the static scratch holds
    if (n_atoms > kStaticAtoms || kx > kStaticAxis || ky > kStaticAxis || kz > kStaticAxis ||
        (long long)kx * ky * kz > kStaticGrid || (long long)kx * ky * kzh > kStaticHalf ||
        (long long)ky * kzh > kStaticRecords)
        return PMGPU_ERR_CAPACITY;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return PMGPU_ERR_CUDA;
    unsigned char* base = nullptr;
    int r = static_scratch(device, &base);
    if (r) { cudaSetDevice(prev); return r; }
    cudaStream_t s = (cudaStream_t)stream;
    const double LX = box[0], LY = box[1], LZ = box[2];
    const double fac = kPi * kPi / (alpha * alpha);
    // exp tables, B-spline moduli and twiddles, as for the PME force
    std::vector<double> ef, bf;
    for (int i = 0; i < kx; i++) { double m = (i <= kx / 2 ? i : i - kx) / LX; ef.push_back(std::exp(-fac * m * m)); }
    for (int j = 0; j < ky; j++) { double m = (j <= ky / 2 ? j : j - ky) / LY; ef.push_back(std::exp(-fac * m * m)); }
    for (int k = 0; k < kzh; k++) { double m = k / LZ; ef.push_back(std::exp(-fac * m * m)); }
    std::vector<double> mx, my, mz;
    dftmod(order, kx, mx); dftmod(order, ky, my); dftmod(order, kz, mz);
    bf.insert(bf.end(), mx.begin(), mx.end()); bf.insert(bf.end(), my.begin(), my.end());
    bf.insert(bf.end(), mz.begin(), mz.begin() + kzh);
    std::vector<float> tw;
    const int ns[3] = {kx, ky, kz};
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < ns[a]; ++k) {
            long double ang = 2.0L * 3.141592653589793238462643383279502884L * k / ns[a];
            tw.push_back((float)cosl(ang));
            tw.push_back((float)-sinl(ang));
        }
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    ok(cudaMemcpyAsync(base + kOffEfac, ef.data(), sizeof(double) * ef.size(), cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(base + kOffBfac, bf.data(), sizeof(double) * bf.size(), cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(base + kOffTw, tw.data(), sizeof(float) * tw.size(), cudaMemcpyHostToDevice, s));
    // what must start at zero: status and the fixed-point forces (the
    // charge grid is cleared by the spread stage itself)
    ok(cudaMemsetAsync(base + kOffStatus, 0, sizeof(int), s));
    if (n_atoms > 0) ok(cudaMemsetAsync(base + kOffFacc, 0, sizeof(unsigned long long) * 3 * (size_t)n_atoms, s));
    PmeArgs a;
    memset(&a, 0, sizeof(a));
    a.n = n_atoms; a.pos = d_positions; a.q = d_scaled_charges;
    a.sorted = (const int*)(base + kOffIdent); a.slot_of = (const int*)(base + kOffIdent);
    a.kx = kx; a.ky = ky; a.kz = kz; a.kzh = kzh; a.order = order;
    a.hxr = kx / LX; a.hyr = ky / LY; a.hzr = kz / LZ;
    a.offx = -(order - 1) / 2 + kx; a.offy = -(order - 1) / 2 + ky; a.offz = -(order - 1) / 2 + kz;
    a.qgrid = (long long*)(base + kOffQgrid); a.cgrid = base + kOffCgrid; a.rgrid = base + kOffRgrid;
    a.tw = base + kOffTw; a.twx = 0; a.twy = kx; a.twz = kx + ky;
    a.bfac = (const double*)(base + kOffBfac); a.efac = (const double*)(base + kOffEfac);
    a.piVr = 1.0 / (kPi * (LX * LY * LZ)); a.fac = fac;
    a.wr = 1.0 / LX; a.lr = 1.0 / LY; a.hr = 1.0 / LZ;
    a.facc = (unsigned long long*)(base + kOffFacc); a.scale = kScaleMixed; a.qscale = kScaleFp64;
    a.erec_stride = kStaticRecords; a.status = (int*)(base + kOffStatus);
    a.virial = (flags & PMGPU_FLAG_VIRIAL) ? 1 : 0;
    pme_init_attributes();
    long long launches = 0;
    int records = 0;
    double* erec = (double*)(base + kOffErec);
    const int stages[3] = {kStageSpread, kStageFft, kStageGather};
    for (int st = 0; st < 3 && e == cudaSuccess; ++st) {
        int u = 0;
        ok((cudaError_t)launch_pme_reciprocal(a, 0, s, &launches, erec + records, &u, stages[st]));
        records += u;
    }
    if (e == cudaSuccess) {
        FinArgs fa;
        memset(&fa, 0, sizeof(fa));
        fa.n = n_atoms; fa.f32p = a.facc; fa.sorted = a.sorted; fa.fout = d_forces_accum;
        int rec = 0;
        ok((cudaError_t)launch_finalize(fa, s, &launches, &rec));
    }
    if (e == cudaSuccess) ok((cudaError_t)launch_energy_reduce(erec, kStaticRecords, records, nullptr, d_energies, s, &launches));
    ok(cudaStreamSynchronize(s));
    int st = 0;
    ok(cudaMemcpy(&st, base + kOffStatus, sizeof(int), cudaMemcpyDeviceToHost));
    cudaSetDevice(prev);
    if (e != cudaSuccess) return PMGPU_ERR_CUDA;
    return (st & kStatusOverflow) ? PMGPU_ERR_OVERFLOW : PMGPU_OK;
}

// ------------------------------------------------------------------ batches
// Many independent systems evaluated by one CUDA graph launch: each member's
// evaluation (its forces on its device buffers) is captured on the member's
// own streams, all branching from and joining back into the batch's stream,
// so the small systems of a batch run concurrently and fill the GPU.
struct pmgpu_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr;
    cudaEvent_t ev_pairs = nullptr;           // the members' one pair launch has run
    int pair_launch = 1;                      // 1: the column-path pair kernels as one launch (K11)
    PairArgs* d_args = nullptr;               // the members' pair arguments for that launch
    size_t args_cap = 0;
    int* d_next = nullptr;                    // its work counters, one per combination of terms
    struct Member {
        pmgpu_system* sys;
        std::vector<pmgpu_force*> forces;    // -real expanded
        const double* pos;
        double* fout;
        double* energy;
        unsigned flags;
        cudaEvent_t done;
        cudaEvent_t listed;                  // its list is built (before the one pair launch)
    };
    std::vector<Member> members;
    std::vector<GraphKey> keys;               // of the captured graph
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> member_launches;   // kernels per member in the graph
    std::string err;
};

static int batch_fail(pmgpu_batch* b, int code, const std::string& msg)
{
    b->err = msg;
    return code;
}

extern "C" int pmgpu_batch_create(int device, pmgpu_batch** out)
{
    if (!out) return PMGPU_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return PMGPU_ERR_CUDA;
    pmgpu_batch* b = new pmgpu_batch();
    b->device = device;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_start, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_pairs, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc((void**)&b->d_next, 32 * sizeof(int)) != cudaSuccess) {
        delete b;
        return PMGPU_ERR_CUDA;
    }
    *out = b;
    return PMGPU_OK;
}

extern "C" int pmgpu_batch_destroy(pmgpu_batch* b)
{
    if (!b) return PMGPU_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (auto& m : b->members) {
        cudaEventDestroy(m.done);
        cudaEventDestroy(m.listed);
    }
    cudaEventDestroy(b->ev_start);
    cudaEventDestroy(b->ev_pairs);
    cudaFree(b->d_args);
    cudaFree(b->d_next);
    cudaStreamDestroy(b->stream);
    delete b;
    return PMGPU_OK;
}

extern "C" int pmgpu_batch_add(pmgpu_batch* b, pmgpu_system* sys, int n_forces, pmgpu_force* const* forces,
                               const double* d_positions, double* d_forces_accum, double* d_energies,
                               unsigned flags)
{
    if (!b || !sys || n_forces < 1 || !forces || !d_positions || !d_forces_accum || !d_energies)
        return PMGPU_ERR_ARG;
    if (sys->device != b->device) return batch_fail(b, PMGPU_ERR_ARG, "system on another device");
    pmgpu_batch::Member m;
    m.sys = sys; m.pos = d_positions; m.fout = d_forces_accum; m.energy = d_energies;
    m.flags = flags & ~kFlagsInternal;
    for (int k = 0; k < n_forces; ++k) {
        if (!forces[k] || forces[k]->sys != sys) return batch_fail(b, PMGPU_ERR_ARG, "force of another system");
        if (forces[k]->real_sub && !pme_needs_lattice(forces[k])) m.forces.push_back(forces[k]->real_sub);
        m.forces.push_back(forces[k]);
    }
    cudaSetDevice(b->device);
    if (cudaEventCreateWithFlags(&m.done, cudaEventDisableTiming) != cudaSuccess) return PMGPU_ERR_CUDA;
    if (cudaEventCreateWithFlags(&m.listed, cudaEventDisableTiming) != cudaSuccess) {
        cudaEventDestroy(m.done);
        return PMGPU_ERR_CUDA;
    }
    b->members.push_back(m);
    return PMGPU_OK;
}

extern "C" int pmgpu_batch_evaluate(pmgpu_batch* b)
{
    if (!b) return PMGPU_ERR_ARG;
    if (b->members.empty()) return PMGPU_OK;
    cudaSetDevice(b->device);
    std::vector<GraphKey> keys;
    for (auto& m : b->members) {
        if (m.sys->profiling) return batch_fail(b, PMGPU_ERR_STATE, "a member system is in profiling mode");
        int r = eval_prepare(m.sys, (int)m.forces.size(), m.forces.data(), m.flags);
        if (r) return batch_fail(b, r, m.sys->err);
        GraphKey k;
        for (pmgpu_force* f : m.forces) k.ids.push_back(f->id);
        k.pos = m.pos; k.fout = m.fout; k.energy = m.energy; k.flags = m.flags;
        k.box_version = m.sys->box_version; k.topo_version = m.sys->topo_version;
        k.buf_version = m.sys->buf_version;
        keys.push_back(k);
    }
    if (!(b->exec && keys == b->keys)) {
        if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
        std::vector<long long> l0;
        for (auto& m : b->members) l0.push_back(m.sys->launches);
        // the one pair launch (K11) takes the members' column-path mixed
        // cutoff forces when every member is its own system
        const size_t nm = b->members.size();
        bool one_launch = b->pair_launch == 1 && nm <= (size_t)kBatchPairMax;
        for (size_t i = 0; i < nm && one_launch; ++i)
            for (size_t j = 0; j < i; ++j)
                if (b->members[i].sys == b->members[j].sys) one_launch = false;
        if (one_launch && nm > b->args_cap) {
            cudaFree(b->d_args);
            b->d_args = nullptr;
            b->args_cap = 0;
            if (cudaMalloc((void**)&b->d_args, nm * sizeof(PairArgs)) != cudaSuccess)
                return batch_fail(b, PMGPU_ERR_CUDA, "batch pair arguments");
            b->args_cap = nm;
        }
        std::vector<EvalRun> runs(nm);
        std::vector<size_t> deferred;
        std::vector<PairArgs> hargs;
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return batch_fail(b, PMGPU_ERR_CUDA, "batch graph capture");
        int r = PMGPU_OK;
        cudaError_t e = cudaEventRecord(b->ev_start, b->stream);
        for (size_t k = 0; k < nm && r == PMGPU_OK && e == cudaSuccess; ++k) {
            auto& m = b->members[k];
            e = cudaStreamWaitEvent(m.sys->stream, b->ev_start, 0);
            if (e != cudaSuccess) break;
            run_init(runs[k], m.sys, (int)m.forces.size(), m.forces.data(), m.pos, m.fout, m.energy, m.flags);
            r = run_begin(runs[k]);
            if (!r) r = run_cutoffs(runs[k], one_launch);
            if (!r && runs[k].deferred < 0) r = run_end(runs[k]);
            if (r) { b->err = m.sys->err; break; }
            if (runs[k].deferred >= 0) {
                deferred.push_back(k);
                e = cudaEventRecord(m.listed, m.sys->stream);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, m.listed, 0);
            } else {
                e = cudaEventRecord(m.done, m.sys->stream);
            }
        }
        if (r == PMGPU_OK && e == cudaSuccess && !deferred.empty()) {
            // one persistent launch per combination of terms over the members'
            // chunks, then every deferred member resumes after it
            std::vector<int> combos;
            for (size_t k : deferred) {
                const int c = runs[k].forces[runs[k].deferred]->combo;
                if (std::find(combos.begin(), combos.end(), c) == combos.end()) combos.push_back(c);
            }
            for (size_t g = 0; g < combos.size() && e == cudaSuccess && r == PMGPU_OK; ++g) {
                const size_t off = hargs.size();
                for (size_t k : deferred)
                    if (runs[k].forces[runs[k].deferred]->combo == combos[g]) hargs.push_back(runs[k].dargs);
                e = cudaMemsetAsync(b->d_next + g, 0, sizeof(int), b->stream);
                if (e != cudaSuccess) break;
                BatchPairArgs ba;
                ba.args = b->d_args + off;
                ba.n = (int)(hargs.size() - off);
                ba.next = b->d_next + g;
                e = (cudaError_t)launch_pair_col_batch(ba, combos[g], b->stream, &b->members[deferred[0]].sys->launches);
            }
            if (e == cudaSuccess) e = cudaEventRecord(b->ev_pairs, b->stream);
            for (size_t i = 0; i < deferred.size() && e == cudaSuccess && r == PMGPU_OK; ++i) {
                auto& m = b->members[deferred[i]];
                e = cudaStreamWaitEvent(m.sys->stream, b->ev_pairs, 0);
                if (e != cudaSuccess) break;
                r = run_resume(runs[deferred[i]]);
                if (r) { b->err = m.sys->err; break; }
                e = cudaEventRecord(m.done, m.sys->stream);
            }
        }
        for (size_t k = 0; k < nm && r == PMGPU_OK && e == cudaSuccess; ++k)
            e = cudaStreamWaitEvent(b->stream, b->members[k].done, 0);
        cudaGraph_t graph = nullptr;
        cudaError_t ec = cudaStreamEndCapture(b->stream, &graph);
        if (r || e != cudaSuccess || ec != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            for (size_t k = 0; k < b->members.size(); ++k) b->members[k].sys->launches = l0[k];
            return r ? r : batch_fail(b, PMGPU_ERR_CUDA, std::string("batch graph capture: ") +
                                          cudaGetErrorString(e != cudaSuccess ? e : ec));
        }
        e = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            return batch_fail(b, PMGPU_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e));
        }
        // the one pair launch reads the members' arguments from device memory
        if (!hargs.empty()) {
            e = cudaMemcpy(b->d_args, hargs.data(), hargs.size() * sizeof(PairArgs), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
                return batch_fail(b, PMGPU_ERR_CUDA, std::string("batch pair arguments: ") + cudaGetErrorString(e));
            }
        }
        b->member_launches.clear();
        for (size_t k = 0; k < b->members.size(); ++k) {
            b->member_launches.push_back(b->members[k].sys->launches - l0[k]);
            b->members[k].sys->launches = l0[k];
        }
        b->keys = keys;
    }
    cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
    if (e != cudaSuccess) return batch_fail(b, PMGPU_ERR_CUDA, std::string("batch graph launch: ") + cudaGetErrorString(e));
    for (size_t k = 0; k < b->members.size(); ++k) b->members[k].sys->launches += b->member_launches[k];
    return PMGPU_OK;
}

extern "C" int pmgpu_batch_set_pair_launch(pmgpu_batch* b, int one_launch)
{
    if (!b || (one_launch != 0 && one_launch != 1)) return PMGPU_ERR_ARG;
    if (b->pair_launch != one_launch && b->exec) {
        cudaSetDevice(b->device);
        cudaStreamSynchronize(b->stream);
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
        b->keys.clear();
    }
    b->pair_launch = one_launch;
    return PMGPU_OK;
}

extern "C" int pmgpu_batch_synchronize(pmgpu_batch* b)
{
    if (!b) return PMGPU_ERR_ARG;
    cudaSetDevice(b->device);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, PMGPU_ERR_CUDA, cudaGetErrorString(e));
    // the members' status words: the first failure is reported
    for (size_t k = 0; k < b->members.size(); ++k) {
        int r = pmgpu_synchronize(b->members[k].sys);
        if (r) return batch_fail(b, r, "member " + std::to_string(k) + ": " + b->members[k].sys->err);
    }
    return PMGPU_OK;
}

extern "C" int pmgpu_batch_last_error(pmgpu_batch* b, char* buf, int len)
{
    if (!b || !buf || len <= 0) return PMGPU_ERR_ARG;
    snprintf(buf, (size_t)len, "%s", b->err.c_str());
    return PMGPU_OK;
}

extern "C" void* pmgpu_batch_stream(pmgpu_batch* b) { return b ? (void*)b->stream : nullptr; }

// ------------------------------------------------------------------ tuning
static bool tuning_valid(const pmgpu_tuning& t)
{
    return t.chunk_entries >= 4 && t.chunk_entries <= 64 && t.pair_blocks_per_sm >= 0 &&
           t.pair_blocks_per_sm <= 8 && t.fft_lines >= 1 && t.fft_lines <= 16 &&
           (t.pme_concurrent == 0 || t.pme_concurrent == 1) && (t.fp64_pairs == 0 || t.fp64_pairs == 1);
}

static void apply_tuning(pmgpu_system* sys, const pmgpu_tuning& t)
{
    sys->tuning = t;
    sys->buf_version++;                  // the captured graph holds the old launch shapes
}

extern "C" int pmgpu_get_tuning(pmgpu_system* sys, pmgpu_tuning* out)
{
    if (!sys || !out) return PMGPU_ERR_ARG;
    *out = sys->tuning;
    return PMGPU_OK;
}

extern "C" int pmgpu_set_tuning(pmgpu_system* sys, const pmgpu_tuning* t)
{
    if (!sys || !t) return PMGPU_ERR_ARG;
    if (!tuning_valid(*t)) return fail(sys, PMGPU_ERR_ARG, "tuning value out of range");
    apply_tuning(sys, *t);
    return PMGPU_OK;
}

// coordinate search over the five launch parameters: each is tried at its
// candidate values with the others at the best so far, two sweeps; time(t)
// measures one candidate in ms per evaluation
constexpr int kFp64PairsMaxAtoms = 4096;     // largest system the autotuner offers fp64_pairs

template <class TimeFn>
static int tune_search(pmgpu_tuning start, bool has_pme, bool has_pairs, bool try_fp64, TimeFn time,
                       pmgpu_tuning* best)
{
    double best_ms = 0.0;
    int r = time(start, &best_ms);
    if (r) return r;
    pmgpu_tuning b = start;
    const int chunks[3] = {8, 16, 32}, bps[3] = {0, 3, 2}, lines[3] = {16, 8, 4}, conc[2] = {1, 0},
              f64[2] = {0, 1};
    for (int sweep = 0; sweep < 2; ++sweep) {
        for (int param = 0; param < 5; ++param) {
            if ((param == 0 || param == 1 || param == 4) && !has_pairs) continue;
            if (param == 4 && !try_fp64) continue;
            if ((param == 2 || param == 3) && !has_pme) continue;
            if (param == 3 && !has_pairs) continue;
            const int nv = param >= 3 ? 2 : 3;
            for (int v = 0; v < nv; ++v) {
                pmgpu_tuning t = b;
                int* slot = param == 0 ? &t.chunk_entries : param == 1 ? &t.pair_blocks_per_sm
                          : param == 2 ? &t.fft_lines : param == 3 ? &t.pme_concurrent : &t.fp64_pairs;
                const int val = param == 0 ? chunks[v] : param == 1 ? bps[v] : param == 2 ? lines[v]
                              : param == 3 ? conc[v] : f64[v];
                if (*slot == val) continue;
                *slot = val;
                double ms = 0.0;
                r = time(t, &ms);
                if (r) return r;
                if (ms < best_ms) { best_ms = ms; b = t; }
            }
        }
    }
    b.ms_per_eval = best_ms;
    *best = b;
    return PMGPU_OK;
}

static void force_kinds(int nf, pmgpu_force* const* forces, bool& has_pme, bool& has_pairs)
{
    has_pme = has_pairs = false;
    for (int k = 0; k < nf; ++k) {
        if (forces[k]->kind == 1 && forces[k]->pp.reciprocal) has_pme = true;
        if ((forces[k]->kind == 0 && forces[k]->precision != PMGPU_PRECISION_FP64) ||
            (forces[k]->kind == 1 && forces[k]->real_sub))
            has_pairs = true;
    }
}

extern "C" int pmgpu_autotune(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces, const double* positions,
                              unsigned flags, int evals, pmgpu_tuning* best)
{
    if (!sys || n_forces <= 0 || !forces || !positions || evals < 1 || !best) return PMGPU_ERR_ARG;
    if (sys->profiling) return fail(sys, PMGPU_ERR_STATE, "autotune in profiling mode");
    cudaSetDevice(sys->device);
    flags &= ~kFlagsInternal;
    int r = eval_prepare(sys, n_forces, forces, flags);
    if (r) return r;
    cudaStream_t s = sys->stream;
    const size_t n3 = 3 * (size_t)sys->n;
    CK(cudaMemcpyAsync(sys->d_pos, positions, sizeof(double) * n3, cudaMemcpyHostToDevice, s), "H2D positions");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0), "event");
    if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return cuda_fail(sys, cudaErrorUnknown, "event"); }
    auto time = [&](const pmgpu_tuning& t, double* ms) -> int {
        apply_tuning(sys, t);
        // two warm-up evaluations; a second round when they outgrew a list
        // (the chunk count depends on the tuning; eval_core grows it)
        for (int attempt = 0; attempt < 2; ++attempt) {
            int q = PMGPU_OK;
            for (int w = 0; w < 2 && q == PMGPU_OK; ++w)
                q = eval_core(sys, n_forces, forces, sys->d_pos, sys->d_fout, sys->d_energy, flags);
            if (q) return q;
            q = pmgpu_synchronize(sys);
            if (q == PMGPU_OK) break;
            if (q != PMGPU_ERR_CAPACITY || attempt == 1) return q;
        }
        cudaEventRecord(e0, s);
        for (int k = 0; k < evals; ++k) {
            int q = eval_core(sys, n_forces, forces, sys->d_pos, sys->d_fout, sys->d_energy, flags);
            if (q) return q;
        }
        cudaEventRecord(e1, s);
        int q = pmgpu_synchronize(sys);
        if (q) return q;
        float el = 0.f;
        cudaEventElapsedTime(&el, e0, e1);
        *ms = el / evals;
        return PMGPU_OK;
    };
    bool has_pme = false, has_pairs = false;
    force_kinds(n_forces, forces, has_pme, has_pairs);
    pmgpu_tuning b;
    // the FP64 pair kernels can win only on a few thousand atoms or fewer,
    // where an evaluation is a chain of launch latencies; on larger systems
    // they are not timed (a disturbed timing could not pick them)
    r = tune_search(sys->tuning, has_pme, has_pairs, sys->n <= kFp64PairsMaxAtoms, time, &b);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r) return r;
    apply_tuning(sys, b);
    *best = b;
    return PMGPU_OK;
}

extern "C" int pmgpu_batch_autotune(pmgpu_batch* b, int evals, pmgpu_tuning* best)
{
    if (!b || evals < 1 || !best) return PMGPU_ERR_ARG;
    if (b->members.empty()) return batch_fail(b, PMGPU_ERR_STATE, "empty batch");
    cudaSetDevice(b->device);
    bool has_pme = false, has_pairs = false;
    for (auto& m : b->members) {
        bool p1 = false, p2 = false;
        force_kinds((int)m.forces.size(), m.forces.data(), p1, p2);
        has_pme = has_pme || p1;
        has_pairs = has_pairs || p2;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess) return batch_fail(b, PMGPU_ERR_CUDA, "event");
    if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return batch_fail(b, PMGPU_ERR_CUDA, "event"); }
    auto time = [&](const pmgpu_tuning& t, double* ms) -> int {
        for (auto& m : b->members) apply_tuning(m.sys, t);
        for (int attempt = 0; attempt < 2; ++attempt) {
            int q = PMGPU_OK;
            for (int w = 0; w < 2 && q == PMGPU_OK; ++w) q = pmgpu_batch_evaluate(b);
            if (q) return q;
            q = pmgpu_batch_synchronize(b);
            if (q == PMGPU_OK) break;
            if (q != PMGPU_ERR_CAPACITY || attempt == 1) return q;
        }
        cudaEventRecord(e0, b->stream);
        for (int k = 0; k < evals; ++k) {
            int q = pmgpu_batch_evaluate(b);
            if (q) return q;
        }
        cudaEventRecord(e1, b->stream);
        int q = pmgpu_batch_synchronize(b);
        if (q) return q;
        float el = 0.f;
        cudaEventElapsedTime(&el, e0, e1);
        *ms = el / evals;
        return PMGPU_OK;
    };
    pmgpu_tuning t;
    // one tuning for every member: the FP64 pair kernels are not a candidate
    int r = tune_search(b->members[0].sys->tuning, has_pme, has_pairs, false, time, &t);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r) return r;
    for (auto& m : b->members) apply_tuning(m.sys, t);
    *best = t;
    return PMGPU_OK;
}

// ------------------------------------------------------------------ dense Hessian
static const int kHessianMaxAtoms = 8192;    // 3N x 3N doubles: 4.8 GB at the limit

extern "C" int pmgpu_hessian(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces_in, const double* positions,
                             double* hessian)
{
    if (!sys || !positions || !hessian || n_forces < 1 || !forces_in) return PMGPU_ERR_ARG;
    cudaSetDevice(sys->device);
    std::vector<pmgpu_force*> fl;
    for (int k = 0; k < n_forces; ++k) {
        if (!forces_in[k] || forces_in[k]->sys != sys) return fail(sys, PMGPU_ERR_ARG, "bad force list");
        if (pme_needs_lattice(forces_in[k]))
            return fail(sys, PMGPU_ERR_UNSUPPORTED, "the Hessian of PMEwald -real with lattice images is not available");
        if (forces_in[k]->real_sub) fl.push_back(forces_in[k]->real_sub);
        if (forces_in[k]->kind == 1 && (forces_in[k]->pp.reciprocal || forces_in[k]->pp.correction))
            return fail(sys, PMGPU_ERR_UNSUPPORTED, "the Hessian of the PME reciprocal / correction terms is not "
                                                    "available (the real-space pairs are)");
        if (forces_in[k]->kind != 1) fl.push_back(forces_in[k]);
    }
    if (sys->n > kHessianMaxAtoms) return fail(sys, PMGPU_ERR_CAPACITY, "dense Hessian above 8192 atoms");
    int r = eval_prepare(sys, (int)fl.size(), fl.data(), 0);
    if (r) return r;
    const size_t n3 = 3 * (size_t)sys->n, nh = n3 * n3;
    cudaStream_t s = sys->stream;
    double* d_h = nullptr;
    cudaError_t e = dalloc(&d_h, nh);
    auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    ok(cudaMemcpyAsync(sys->d_pos, positions, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
    ok(cudaMemsetAsync(d_h, 0, sizeof(double) * nh, s));
    for (pmgpu_force* f : fl) {
        AdjArgs a;
        adj_pair_args(sys, f, a);
        a.hess = d_h;
        ok((cudaError_t)launch_pair_adjoint(a, f->precision == PMGPU_PRECISION_FP64 ? 1 : 0, s, &sys->launches));
    }
    std::vector<double> out(e == cudaSuccess ? nh : 0);
    if (e == cudaSuccess) ok(cudaMemcpyAsync(out.data(), d_h, sizeof(double) * nh, cudaMemcpyDeviceToHost, s));
    ok(cudaStreamSynchronize(s));
    dfree(d_h);
    if (e != cudaSuccess) return cuda_fail(sys, e, "Hessian");
    for (size_t k = 0; k < nh; ++k) hessian[k] += out[k];
    return PMGPU_OK;
}

// ------------------------------------------------------------------ leapfrog
static const double kInvTimeFactor = 0.02045482828087295;   // Constant::INV_TIMEFACTOR (base/pmconstants.cpp:49)
static const double kTimeFactor = 48.88821290839616;        // Constant::TIMEFACTOR (base/pmconstants.cpp:48)

extern "C" int pmgpu_leapfrog_run(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces, const double* d_mass,
                                  double* d_positions, double* d_velocities, double* d_forces, double* d_energies,
                                  double timestep, int n_steps, unsigned flags)
{
    if (!sys || n_forces <= 0 || !forces || !d_mass || !d_positions || !d_velocities || !d_forces || !d_energies)
        return PMGPU_ERR_ARG;
    if (!(timestep > 0.0) || n_steps < 0) return fail(sys, PMGPU_ERR_ARG, "timestep must be positive, steps >= 0");
    // the molecule positions move with the atoms: the caller's per-step evaluation sets them
    if (flags & PMGPU_FLAG_MOLECULAR_VIRIAL)
        return fail(sys, PMGPU_ERR_UNSUPPORTED, "molecular virial inside a resident run");
    if (n_steps == 0) return PMGPU_OK;
    cudaSetDevice(sys->device);
    cudaStream_t s = sys->stream;
    const size_t n3 = 3 * (size_t)sys->n;
    const double h = timestep * kInvTimeFactor;              // getTimestep() * Constant::INV_TIMEFACTOR
    const double hk = 0.5 * timestep * kInvTimeFactor;       // doHalfKick's step
    // SHAKE as a post-drift modifier, RATTLE as a post-step modifier
    // (applications/protomol-app/protomol.cpp:553-577)
    const bool shake = sys->n_cons > 0 && sys->shake_eps > 0.0 && sys->shake_iter > 0;
    const bool rattle = sys->n_cons > 0 && sys->rattle_eps > 0.0 && sys->rattle_iter > 0;
    ConsArgs ca;
    memset(&ca, 0, sizeof(ca));
    ca.n_cons = sys->n_cons; ca.n_clusters = sys->n_ccl; ca.cl_start = sys->d_cl_start; ca.atoms = sys->d_cons_atoms;
    ca.rest = sys->d_cons_rest; ca.mass = d_mass; ca.pos = d_positions; ca.vel = d_velocities;
    ca.last = sys->d_cons_last; ca.dt = timestep / kTimeFactor; ca.hits = sys->d_cons_hits;
    auto do_shake = [&]() -> int {
        ConsArgs a = ca;
        a.eps = sys->shake_eps; a.max_iter = sys->shake_iter;
        int e = launch_shake(a, s, &sys->launches);
        if (e) return cuda_fail(sys, (cudaError_t)e, "SHAKE");
        // ModifierShake stores the positions it leaves for the next sweep's bond vectors
        CK(cudaMemcpyAsync(sys->d_cons_last, d_positions, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s), "copy");
        return PMGPU_OK;
    };
    auto do_rattle = [&]() -> int {
        ConsArgs a = ca;
        a.eps = sys->rattle_eps; a.max_iter = sys->rattle_iter;
        a.virial = (flags & PMGPU_FLAG_VIRIAL) ? d_energies + 2 : nullptr;
        int e = launch_rattle(a, s, &sys->launches);
        return e ? cuda_fail(sys, (cudaError_t)e, "RATTLE") : PMGPU_OK;
    };
    // ModifierMetaRattleShake::doInitialize: the last positions start as the positions
    if (shake)
        CK(cudaMemcpyAsync(sys->d_cons_last, d_positions, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s), "copy");
    for (int step = 0; step < n_steps; ++step) {
        if (step > 0 && rattle) {
            // doKickdoDrift with a post-step modifier: half kick, RATTLE, half
            // kick, drift (LeapfrogIntegrator.cpp:72-83)
            int e = launch_leapfrog(sys->n, d_mass, d_positions, d_velocities, d_forces, h, hk, kLeapfrogLast, s,
                                    &sys->launches);
            if (e) return cuda_fail(sys, (cudaError_t)e, "leapfrog half kick");
            int r = do_rattle();
            if (r) return r;
            e = launch_leapfrog(sys->n, d_mass, d_positions, d_velocities, d_forces, h, hk, kLeapfrogLast, s,
                                &sys->launches);
            if (e) return cuda_fail(sys, (cudaError_t)e, "leapfrog half kick");
            e = launch_leapfrog(sys->n, d_mass, d_positions, d_velocities, d_forces, h, h, kLeapfrogDrift, s,
                                &sys->launches);
            if (e) return cuda_fail(sys, (cudaError_t)e, "leapfrog drift");
        } else {
            int e = launch_leapfrog(sys->n, d_mass, d_positions, d_velocities, d_forces, h, h,
                                    step == 0 ? kLeapfrogFirst : kLeapfrogMiddle, s, &sys->launches);
            if (e) return cuda_fail(sys, (cudaError_t)e, "leapfrog step");
        }
        if (shake) {
            int r = do_shake();
            if (r) return r;
        }
        // calculateForces: forces and energies cleared, then evaluated
        CK(cudaMemsetAsync(d_forces, 0, sizeof(double) * n3, s), "memset");
        CK(cudaMemsetAsync(d_energies, 0, sizeof(double) * kERec, s), "memset");
        int r = eval_core(sys, n_forces, forces, d_positions, d_forces, d_energies, flags);
        if (r) return r;
    }
    int e = launch_leapfrog(sys->n, d_mass, d_positions, d_velocities, d_forces, h, hk, kLeapfrogLast, s,
                            &sys->launches);
    if (e) return cuda_fail(sys, (cudaError_t)e, "leapfrog half kick");
    if (rattle) {
        int r = do_rattle();
        if (r) return r;
    }
    return PMGPU_OK;
}

extern "C" int pmgpu_set_constraints(pmgpu_system* sys, int n_constraints, const int* atoms, const double* rest_length,
                                     double shake_epsilon, int shake_max_iter, double rattle_epsilon,
                                     int rattle_max_iter)
{
    if (!sys || n_constraints < 0 || (n_constraints > 0 && (!atoms || !rest_length))) return PMGPU_ERR_ARG;
    const int n = sys->n;
    for (int k = 0; k < n_constraints; ++k) {
        const int a = atoms[2 * k], b = atoms[2 * k + 1];
        if (a < 0 || b < 0 || a >= n || b >= n || a == b) return fail(sys, PMGPU_ERR_ARG, "constraint atom out of range");
        if (!(rest_length[k] > 0.0)) return fail(sys, PMGPU_ERR_ARG, "constraint rest length must be positive");
    }
    cudaSetDevice(sys->device);
    CK(cudaStreamSynchronize(sys->stream), "set_constraints");
    // clusters: connected components of the constraint graph, ordered by
    // their first constraint, each keeping the list order
    std::vector<int> parent(n);
    for (int i = 0; i < n; ++i) parent[i] = i;
    auto find = [&](int x) {
        while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
        return x;
    };
    for (int k = 0; k < n_constraints; ++k) {
        const int ra = find(atoms[2 * k]), rb = find(atoms[2 * k + 1]);
        if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
    }
    std::vector<int> cluster_of_root(n, -1), order, start;
    std::vector<std::vector<int>> members;
    for (int k = 0; k < n_constraints; ++k) {
        const int root = find(atoms[2 * k]);
        if (cluster_of_root[root] < 0) {
            cluster_of_root[root] = (int)members.size();
            members.emplace_back();
        }
        members[cluster_of_root[root]].push_back(k);
    }
    std::vector<int2> ca;
    std::vector<double> cr;
    start.push_back(0);
    for (const auto& m : members) {
        for (int k : m) {
            ca.push_back(make_int2(atoms[2 * k], atoms[2 * k + 1]));
            cr.push_back(rest_length[k]);
        }
        start.push_back((int)ca.size());
    }
    dfree(sys->d_cl_start); dfree(sys->d_cons_atoms); dfree(sys->d_cons_rest); dfree(sys->d_cons_last);
    sys->n_cons = 0; sys->n_ccl = 0;
    if (n_constraints > 0) {
        CK(dalloc(&sys->d_cl_start, start.size()), "alloc");
        CK(dalloc(&sys->d_cons_atoms, ca.size()), "alloc");
        CK(dalloc(&sys->d_cons_rest, cr.size()), "alloc");
        CK(dalloc(&sys->d_cons_last, 3 * (size_t)n), "alloc");
        CK(cudaMemcpy(sys->d_cl_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice), "copy");
        CK(cudaMemcpy(sys->d_cons_atoms, ca.data(), sizeof(int2) * ca.size(), cudaMemcpyHostToDevice), "copy");
        CK(cudaMemcpy(sys->d_cons_rest, cr.data(), sizeof(double) * cr.size(), cudaMemcpyHostToDevice), "copy");
    }
    if (!sys->d_cons_hits) {
        CK(dalloc(&sys->d_cons_hits, 1), "alloc");
        CK(cudaMemset(sys->d_cons_hits, 0, sizeof(int)), "memset");
    }
    sys->n_cons = n_constraints;
    sys->n_ccl = (int)members.size();
    sys->shake_eps = shake_epsilon; sys->shake_iter = shake_max_iter;
    sys->rattle_eps = rattle_epsilon; sys->rattle_iter = rattle_max_iter;
    return PMGPU_OK;
}

extern "C" long long pmgpu_constraint_limit_hits(pmgpu_system* sys)
{
    if (!sys || !sys->d_cons_hits) return 0;
    cudaSetDevice(sys->device);
    if (cudaStreamSynchronize(sys->stream) != cudaSuccess) return -1;
    int h = 0;
    if (cudaMemcpy(&h, sys->d_cons_hits, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return h;
}

extern "C" int pmgpu_impulse_run(pmgpu_system* sys, int n_slow, pmgpu_force* const* slow, int n_fast,
                                 pmgpu_force* const* fast, const double* d_mass, double* d_positions,
                                 double* d_velocities, double* d_slow_forces, double* d_fast_forces,
                                 double* d_slow_energies, double* d_fast_energies, double timestep, int cyclelength,
                                 int n_steps, unsigned flags)
{
    if (!sys || n_slow <= 0 || !slow || n_fast <= 0 || !fast || !d_mass || !d_positions || !d_velocities ||
        !d_slow_forces || !d_fast_forces || !d_slow_energies || !d_fast_energies)
        return PMGPU_ERR_ARG;
    if (!(timestep > 0.0) || cyclelength < 1 || n_steps < 0)
        return fail(sys, PMGPU_ERR_ARG, "timestep must be positive, cyclelength >= 1, steps >= 0");
    if (flags & PMGPU_FLAG_MOLECULAR_VIRIAL)
        return fail(sys, PMGPU_ERR_UNSUPPORTED, "molecular virial inside a resident run");
    cudaSetDevice(sys->device);
    cudaStream_t s = sys->stream;
    const size_t n3 = 3 * (size_t)sys->n;
    // MTSIntegrator::getTimestep = cyclelength * the inner timestep; doHalfKick's step
    const double h_half = 0.5 * ((double)cyclelength * timestep) * kInvTimeFactor;
    for (int step = 0; step < n_steps; ++step) {
        int e = launch_leapfrog(sys->n, d_mass, d_positions, d_velocities, d_slow_forces, 0.0, h_half,
                                kLeapfrogLast, s, &sys->launches);     // doHalfKick (a kick, no drift)
        if (e) return cuda_fail(sys, (cudaError_t)e, "impulse half kick");
        int r = pmgpu_leapfrog_run(sys, n_fast, fast, d_mass, d_positions, d_velocities, d_fast_forces,
                                   d_fast_energies, timestep, cyclelength, flags);   // doDriftOrNextIntegrator
        if (r) return r;
        CK(cudaMemsetAsync(d_slow_forces, 0, sizeof(double) * n3, s), "memset");    // calculateForces
        CK(cudaMemsetAsync(d_slow_energies, 0, sizeof(double) * kERec, s), "memset");
        r = eval_core(sys, n_slow, slow, d_positions, d_slow_forces, d_slow_energies, flags);
        if (r) return r;
        e = launch_leapfrog(sys->n, d_mass, d_positions, d_velocities, d_slow_forces, 0.0, h_half,
                            kLeapfrogLast, s, &sys->launches);         // doHalfKick
        if (e) return cuda_fail(sys, (cudaError_t)e, "impulse half kick");
    }
    return PMGPU_OK;
}

// ------------------------------------------------------------------ adjoint
static void adj_pme_args(pmgpu_system* sys, pmgpu_force* f, PmeArgs& a)
{
    const pmgpu_pme_params& p = f->pp;
    memset(&a, 0, sizeof(a));
    a.n = sys->n; a.pos = sys->d_pos; a.q = sys->d_q;
    a.kx = p.grid[0]; a.ky = p.grid[1]; a.kz = p.grid[2]; a.kzh = f->kzh; a.order = p.order;
    double LX = sys->box[0], LY = sys->box[4], LZ = sys->box[8];
    a.hxr = p.grid[0] / LX; a.hyr = p.grid[1] / LY; a.hzr = p.grid[2] / LZ;
    a.offx = -(p.order - 1) / 2 + p.grid[0];
    a.offy = -(p.order - 1) / 2 + p.grid[1];
    a.offz = -(p.order - 1) / 2 + p.grid[2];
    a.qgrid = f->d_qgrid; a.cgrid = f->d_cgrid; a.rgrid = f->d_rgrid; a.tw = f->d_tw;
    a.twx = f->twx; a.twy = f->twy; a.twz = f->twz;
    a.bfac = f->d_bfac; a.efac = f->d_efac;
    a.piVr = 1.0 / (kPi * (LX * LY * LZ));
    a.fac = kPi * kPi / (f->alpha * f->alpha);
    a.wr = 1.0 / LX; a.lr = 1.0 / LY; a.hr = 1.0 / LZ;
    a.qscale = kScaleFp64; a.erec_stride = sys->erec_cap;
    a.status = sys->d_status;
}

extern "C" int pmgpu_adjoint(pmgpu_system* sys, int n_forces, pmgpu_force* const* forces_in, const double* positions,
                             const double* v, double* dE_dq, double* dE_dlj, double* hv, double* energies)
{
    if (!sys || !positions || n_forces < 1 || !forces_in) return PMGPU_ERR_ARG;
    cudaSetDevice(sys->device);
    std::vector<pmgpu_force*> fl;
    for (int k = 0; k < n_forces; ++k) {
        if (!forces_in[k] || forces_in[k]->sys != sys) return fail(sys, PMGPU_ERR_ARG, "bad force list");
        if (pme_needs_lattice(forces_in[k]))
            return fail(sys, PMGPU_ERR_UNSUPPORTED, "the backward pass of PMEwald -real with lattice images is not "
                                                    "available");
        if (forces_in[k]->real_sub) fl.push_back(forces_in[k]->real_sub);
        fl.push_back(forces_in[k]);
    }
    if (hv && !v) return fail(sys, PMGPU_ERR_ARG, "Hessian-vector product needs v");
    int r = eval_prepare(sys, (int)fl.size(), fl.data(), 0);
    if (r) return r;
    if (hv)
        for (pmgpu_force* f : fl) {
            if (f->kind != 1 || !f->pp.reciprocal || f->d_hq) continue;
            // the second set of grids of the reciprocal H v (dQ, its spectrum, dphi)
            const size_t nreal = (size_t)f->pp.grid[0] * f->pp.grid[1] * f->pp.grid[2];
            const size_t nhalf = (size_t)f->pp.grid[0] * f->pp.grid[1] * f->kzh;
            const bool f64 = f->precision == PMGPU_PRECISION_FP64;
            CK(dalloc(&f->d_hq, nreal), "alloc");
            if (f64) {
                CK(dalloc((double2**)&f->d_hc, nhalf), "alloc");
                CK(dalloc((double**)&f->d_hr, nreal), "alloc");
            } else {
                CK(dalloc((float2**)&f->d_hc, nhalf), "alloc");
                CK(dalloc((float**)&f->d_hr, nreal), "alloc");
            }
        }
    const int n = sys->n, T = sys->t;
    cudaStream_t s = sys->stream;
    size_t n3 = 3 * (size_t)n;
    double *d_v = nullptr, *d_dq = nullptr, *d_lj = nullptr, *d_hv = nullptr, *d_e = nullptr;
    auto cleanup = [&]() { dfree(d_v); dfree(d_dq); dfree(d_lj); dfree(d_hv); dfree(d_e); };
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    ok(cudaMemcpyAsync(sys->d_pos, positions, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
    ok(cudaMemsetAsync(sys->d_small, 0, kSmallBytes, s));
    ok(dalloc(&d_dq, (size_t)n)); ok(dalloc(&d_lj, (size_t)T * T * 4)); ok(dalloc(&d_e, 2));
    if (hv) { ok(dalloc(&d_v, n3)); ok(dalloc(&d_hv, n3)); }
    if (e == cudaSuccess) {
        ok(cudaMemsetAsync(d_dq, 0, sizeof(double) * n, s));
        ok(cudaMemsetAsync(d_lj, 0, sizeof(double) * T * T * 4, s));
        ok(cudaMemsetAsync(d_e, 0, sizeof(double) * 2, s));
        if (hv) {
            ok(cudaMemcpyAsync(d_v, v, sizeof(double) * n3, cudaMemcpyHostToDevice, s));
            ok(cudaMemsetAsync(d_hv, 0, sizeof(double) * n3, s));
        }
    }
    if (e != cudaSuccess) { cleanup(); return cuda_fail(sys, e, "adjoint setup"); }
    // cutoff forces run over the cell list of the positions (the forward
    // kernels' cell-sorted order)
    bool any_cut = false;
    for (pmgpu_force* f : fl) any_cut |= f->kind == 0;
    if (any_cut) {
        r = bin(sys, sys->d_pos);
        if (r) { cleanup(); return r; }
    }
    std::vector<double> host_dq(n, 0.0);
    for (pmgpu_force* f : fl) {
        const bool fp64 = f->precision == PMGPU_PRECISION_FP64;
        if (f->kind == 0 || f->kind == 2) {
            AdjArgs a;
            adj_pair_args(sys, f, a);
            a.v = d_v; a.dq = d_dq; a.dlj = d_lj; a.hv = d_hv; a.energy = d_e;
            if (f->kind == 0) {
                PairArgs pa;
                fill_pair_args(sys, f, sys->d_pos, pa);
                ok((cudaError_t)launch_pair_adjoint_cells(pa, a, fp64 ? 1 : 0, pair_blocks(sys->grid, f->nd), s,
                                                          &sys->launches));
            } else {
                ok((cudaError_t)launch_pair_adjoint(a, fp64 ? 1 : 0, s, &sys->launches));
            }
        } else {
            const pmgpu_pme_params& p = f->pp;
            if (p.reciprocal) {
                PmeArgs a;
                adj_pme_args(sys, f, a);
                a.scale = fp64 ? kScaleFp64 : kScaleMixed;
                const int stages[3] = {kStageSpread, kStageFft, kStagePotential};
                for (int st = 0; st < 3 && e == cudaSuccess; ++st) {
                    int u = 0;
                    a.facc = (unsigned long long*)d_dq;   // phi output of the potential stage
                    ok((cudaError_t)launch_pme_reciprocal(a, fp64 ? 1 : 0, s, &sys->launches, sys->d_erec, &u,
                                                          stages[st]));
                }
                if (hv && e == cudaSuccess) {
                    // dQ along v, its convolution dphi, then the two gathers (rgrid holds phi)
                    PmeArgs b = a;
                    b.qgrid = f->d_hq; b.cgrid = f->d_hc; b.rgrid = f->d_hr; b.dir = d_v;
                    const int hstages[2] = {kStageSpreadDir, kStageFft};
                    for (int st = 0; st < 2 && e == cudaSuccess; ++st) {
                        int u = 0;
                        ok((cudaError_t)launch_pme_reciprocal(b, fp64 ? 1 : 0, s, &sys->launches, sys->d_erec, &u,
                                                              hstages[st]));
                    }
                    PmeArgs c = a;
                    c.rgrid_d = f->d_hr; c.dir = d_v; c.hv = d_hv;
                    int u = 0;
                    ok((cudaError_t)launch_pme_reciprocal(c, fp64 ? 1 : 0, s, &sys->launches, sys->d_erec, &u,
                                                          kStageHvpGather));
                }
            }
            if (p.correction) {
                CorrArgs c;
                memset(&c, 0, sizeof(c));
                c.n_excl = sys->e; c.pairs = sys->d_epairs; c.cls = sys->d_ecls; c.pos = sys->d_pos; c.q = sys->d_q;
                c.pbc = sys->pbc; c.alpha = f->alpha; c.alpha2 = f->alpha * f->alpha; c.csf = sys->csf;
                ok((cudaError_t)launch_pme_correction_adjoint(c, d_dq, s, &sys->launches));
                if (hv) ok((cudaError_t)launch_pme_correction_hvp(c, d_v, d_hv, s, &sys->launches));
                // point self energy -alpha/sqrt(pi) sum q~^2 and the charged-system term
                // -pi/(2 V alpha^2) (sum q~)^2 (initialize, :604-628), differentiated
                double q1 = 0.0;
                for (int i = 0; i < n; ++i) q1 += sys->q[i];
                const double V = std::fabs(sys->box[0] * sys->box[4] * sys->box[8]);
                const double charged = std::fabs(q1 * 0.00268283) > 1.0e-5
                                           ? -kPi / (V * f->alpha * f->alpha) * q1 : 0.0;
                for (int i = 0; i < n; ++i) host_dq[i] += -2.0 * f->alpha / std::sqrt(kPi) * sys->q[i] + charged;
            }
        }
    }
    std::vector<double> out_dq(n), out_lj((size_t)T * T * 4), out_hv(hv ? n3 : 0), out_e(2);
    ok(cudaMemcpyAsync(out_dq.data(), d_dq, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(out_lj.data(), d_lj, sizeof(double) * out_lj.size(), cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(out_e.data(), d_e, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
    if (hv) ok(cudaMemcpyAsync(out_hv.data(), d_hv, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
    ok(cudaStreamSynchronize(s));
    cleanup();
    if (e != cudaSuccess) return cuda_fail(sys, e, "adjoint");
    if (dE_dq) for (int i = 0; i < n; ++i) dE_dq[i] += out_dq[i] + host_dq[i];
    if (dE_dlj) for (size_t k = 0; k < out_lj.size(); ++k) dE_dlj[k] += out_lj[k];
    if (hv) for (size_t k = 0; k < n3; ++k) hv[k] += out_hv[k];
    if (energies) { energies[0] += out_e[0]; energies[1] += out_e[1]; }
    return PMGPU_OK;
}
