// Host orchestration and C ABI (include/esp_b200.h).
//
// A batch plans N independent systems: it resolves each system's mesh and
// PSWF parameters, builds the tables (host FP64 for the 1D pieces, GPU FP64
// for the influence function), lays out all particle / mesh / spectrum
// arrays back to back, and precomputes the work-item lists every stage
// launches over. A single-system context (esp_ctx) is a batch of one: the
// reference's ESPForceComputeGPU (src/ESPForceComputeGPU.cc:47-448) maps to
// esp_create + esp_compute.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include <cuda.h>

#include "esp_b200.h"
#include "esp_host_util.h"
#include "esp_kernels.h"
#include "esp_md.h"
#include "esp_tables.h"

using namespace espb;

namespace {
thread_local std::string g_err;
}  // namespace

namespace espb {

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

double kappa_required(double target) {
    const double lt[] = {-3, -4, -5, -6, -7, -8};
    const double kv[] = {11.5, 14.0, 18.5, 22.0, 26.0, 30.0};
    double l = std::log10(std::max(1e-9, std::min(1e-2, target)));
    if (l >= lt[0]) return kv[0];
    for (int i = 0; i < 5; ++i)
        if (l >= lt[i + 1]) {
            double f = (l - lt[i]) / (lt[i + 1] - lt[i]);
            return kv[i] + f * (kv[i + 1] - kv[i]);
        }
    return kv[5];
}

double split_c_for_spacing(double rcut, double h) {
    // 0.93 kappa_N, rounded to 0.5: the measured optimum against FP64 Ewald
    // at P = 8, h = r_c / 6
    const double c = std::round(2.0 * 0.93 * M_PI * rcut / h) * 0.5;
    return std::max(2.0, std::min(60.0, c));
}

uint32_t radix_plan(int n) {
    std::vector<int> r;
    int m = n;
    int twos = 0;
    while (m % 2 == 0) {
        m /= 2;
        ++twos;
    }
    while (twos >= 2) {
        r.push_back(4);
        twos -= 2;
    }
    if (twos) r.push_back(2);
    while (m % 3 == 0) {
        r.push_back(3);
        m /= 3;
    }
    while (m % 5 == 0) {
        r.push_back(5);
        m /= 5;
    }
    if (m != 1 || r.size() > 8) return 0;
    uint32_t code = 0;
    for (size_t i = 0; i < r.size(); ++i) code |= (uint32_t)r[i] << (4 * i);
    return code;
}

// (PX, PP) pitches of the interpolation tile. A group of G lanes serves one
// particle (lane c reads stencil plane oz + c) and K = 32 / G groups share a
// warp. With the plane pitch PP = K (mod 32) a group's lanes fall in the bank
// class of its row start, and with the row pitch PX a multiple of K that
// class is the particle's x origin mod K; the kernel orders particles so the
// K groups of a warp have distinct classes (conflict-free reads).
void choose_pitch(int P, int E, int& PX, int& PP) {
    // interpolation region pitches: plane pitch = K (mod 32), so the G lanes
    // of a particle read G banks K apart; row pitch = 1 (mod K), so the bank
    // class of a particle is (ox + oy) mod K, close to uniform over a tile
    const int G = P <= 4 ? 4 : (P <= 8 ? 8 : 16);
    const int K = 32 / G;
    PX = E;
    while (PX % K != 1) ++PX;
    PP = E * PX;
    while (PP % 32 != K) ++PP;
}

int build_param_set(double c, double cw, int P, int D, double rcut, PsetHost& h, ParamSet& d, double tol) {
    try {
        h.split.build(c, tol);
        h.win.build(P, cw, D);
    } catch (const std::exception& ex) {
        return fail(ESP_ERR_INVALID, ex.what());
    }
    h.rcut = rcut;
    if (h.split.qv.size() > (size_t)MAX_QC)
        return fail(ESP_ERR_UNSUPPORTED, "split polynomial needs more than 32 coefficients");
    d = ParamSet{};
    for (int a = 0; a < P; ++a)
        for (int j = 0; j <= D; ++j) d.wcoef[a * (MAX_D + 1) + j] = (float)h.win.coef[(size_t)a * (D + 1) + j];
    d.nq = (int)h.split.qv.size();
    for (int j = 0; j < d.nq; ++j) d.qv[j] = (float)h.split.qv[j];
    for (int j = 1; j < d.nq; ++j) d.dqv[j - 1] = (float)(2.0 * j * h.split.qv[j]);
    d.rcut = (float)rcut;
    d.rcut2 = (float)(rcut * rcut);
    d.inv_rcut = (float)(1.0 / rcut);
    d.two_inv_rcut3 = (float)(2.0 / (rcut * rcut * rcut));
    d.self_coef = -0.5 * h.split.lambda0 * INV_4PI_D / rcut;
    d.bg_coef = -0.25 * rcut * rcut * h.split.m2;
    d.rcut_d = rcut;
    return 0;
}

void interp_box(int E, int& BX, int& BY) {
    BX = E + 3;
    while (BX % 8 != 4) ++BX;
    BY = E | 1;
}

bool encode_phi_map(void* map, float* base, int nxp, int nyp, int nzp, int BX, int BY, int BZ) {
    typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static EncodeTiled fn = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(f);
        looked_up = true;
    }
    if (!fn) return false;
    // 16-byte rules of the tensor map: base, strides and the box's inner extent
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (nxp & 3) || (BX & 3) || BX > 256 || BY > 256 || BZ > 256)
        return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nxp, (cuuint64_t)nyp, (cuuint64_t)nzp};
    const cuuint64_t strides[2] = {(cuuint64_t)nxp * 4, (cuuint64_t)nxp * nyp * 4};
    const cuuint32_t box[3] = {(cuuint32_t)BX, (cuuint32_t)BY, (cuuint32_t)BZ};
    const cuuint32_t estr[3] = {1, 1, 1};
    return fn(reinterpret_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void influence_inputs(const SysDev& S, const PsetHost& h, double Lx, double Ly, double Lz, double rcut,
                      std::vector<double>& w1d, std::vector<double>& tq, std::vector<double>& wq) {
    w1d.assign(S.nx + S.ny + S.nz, 0.0);
    const int nn[3] = {S.nx, S.ny, S.nz};
    const double L[3] = {Lx, Ly, Lz};
    int o = 0;
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < nn[d]; ++i) {
            const int f = (i < (nn[d] + 1) / 2) ? i : nn[d] - i;
            w1d[o++] = h.win.fourier(2.0 * M_PI * f / nn[d]);
        }
    double kmax2 = 0;
    for (int d = 0; d < 3; ++d) {
        const double k = M_PI * nn[d] / L[d];
        kmax2 += k * k;
    }
    const double kap_max = std::sqrt(kmax2) * rcut;
    const int nq = std::max(48, std::min(320, (int)(0.6 * kap_max) + 40));
    gauss_legendre01(nq, tq, wq);
    for (int j = 0; j < nq; ++j) wq[j] *= h.split.pro.psi(tq[j]) / h.split.pro.int01;
}

}  // namespace espb

namespace {

// Per-stage CUDA-event timing on the launching stream. Records are queued
// without synchronising; read() synchronises once and sums the elapsed
// times (used by benchmarks to time kernels inside their timed region).
struct StageTimer {
    bool on = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> stage;
    int used = 0;
    double ms[ESP_N_STAGES] = {0};
    long long count[ESP_N_STAGES] = {0};
    int cur = -1;
    ~StageTimer() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    void collect() {
        if (used == 0) return;
        cudaEventSynchronize(ev[2 * used - 1]);
        for (int i = 0; i < used; ++i) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) {
                ms[stage[i]] += t;
                count[stage[i]] += 1;
            }
        }
        used = 0;
    }
    void begin(int id, cudaStream_t st) {
        if (!on) return;
        if (used * 2 + 2 > (int)ev.size()) {
            if (ev.size() >= 8192) {
                collect();
            } else {
                for (int k = 0; k < 256; ++k) {
                    cudaEvent_t e;
                    cudaEventCreate(&e);
                    ev.push_back(e);
                }
                stage.resize(ev.size() / 2);
            }
        }
        cur = id;
        cudaEventRecord(ev[2 * used], st);
    }
    void end(cudaStream_t st) {
        if (!on || cur < 0) return;
        cudaEventRecord(ev[2 * used + 1], st);
        stage[used] = cur;
        ++used;
        cur = -1;
    }
    void reset() {
        for (int k = 0; k < ESP_N_STAGES; ++k) {
            ms[k] = 0;
            count[k] = 0;
        }
    }
};

}  // namespace

struct esp_batch {
    esp_params prm{};
    int P = 8, T = 8, D = 10, tpp = 8, PX = 0, PP = 0;
    int nsys = 0, totN = 0, n_tiles = 0;
    std::vector<int> N;
    std::vector<double> box;
    std::vector<int> mesh;
    std::vector<SysDev> sd;
    std::vector<PsetHost> psh;
    std::vector<ParamSet> psd;
    std::vector<double> c_split, c_win;
    int n_chunks = 0, n_pchunks = 0, n_x = 0, n_y = 0, n_z = 0;
    DevAlloc mem;
    // device
    SysDev* d_sys = nullptr;
    ParamSet* d_pset = nullptr;
    int2 *d_chunks = nullptr, *d_pchunks = nullptr;
    int* d_tile_sys = nullptr;
    uint32_t *d_tcount = nullptr, *d_tstart = nullptr;
    float4 *d_posq = nullptr, *d_trec = nullptr, *d_srec = nullptr;
    uint32_t *d_rel = nullptr, *d_key = nullptr, *d_perm_u = nullptr, *d_perm = nullptr, *d_srel = nullptr;
    double* d_rho = nullptr;
    float2 *d_spec = nullptr, *d_gtab = nullptr, *d_tw = nullptr;
    float* d_phi = nullptr;
    int4 *d_x = nullptr, *d_y = nullptr, *d_z = nullptr;
    int2 *d_p = nullptr, *d_s = nullptr;
    int n_p = 0, n_s = 0, smem_plane = 0, smem_slab = 0;
    double *d_acc = nullptr, *d_energy = nullptr, *d_virial = nullptr;
    // TMA-staged interpolation: tensor maps of the halo-padded potential mesh
    // (one per system, NULL when unavailable), the box, the kernels' error word
    CUtensorMap* d_tmaps = nullptr;
    int tma_bx = 0, tma_by = 0;
    int* d_kerr = nullptr;  // [kernel error word, tile-queue counter]
    // cell grids of the neighbour-list builds (allocated on first use): one
    // for HOOMD-layout lists, one for the library's pair list (whose rows
    // are indexed by the slots of its own build)
    struct CellGrid {
        DevAlloc mem;
        double rlist = -1;
        int n_cells = 0, cap = -1;  // cap: row capacity the rows' offsets (nl_off) were laid out for
        std::vector<CellDev> h_cells;
        CellDev* d_cells = nullptr;
        int* d_cell_sys = nullptr;
        uint32_t *d_ckey = nullptr, *d_ccount = nullptr, *d_cstart = nullptr, *d_cperm = nullptr,
                 *d_slot2idx = nullptr, *d_idx2slot = nullptr;
        float4 *d_wpos = nullptr, *d_cpos = nullptr;
        int* d_overflow = nullptr;  // [flag, largest row] of the last build
    } cg_nl, cg_pl;
    int setup_cells(CellGrid& g, double rlist, int cap);
    NlistArgs nlist_args(CellGrid& g, const float* pos4, double rlist, int cap) const;
    // the library's pair list: rows by cell-sorted slot, and the
    // slot-ordered positions the bin stage writes for it
    DevAlloc plmem;
    uint32_t *d_pl_head = nullptr, *d_pl_nn = nullptr, *d_pl_nl = nullptr;
    float4* d_spos = nullptr;
    int pl_cap = 0;
    bool pl_ready = false, pl_pending = false, pl_overflow = false;
    int* h_pl_ovf = nullptr;  // page-locked copy of the last build's [flag, largest row]
    cudaEvent_t pl_ev = nullptr;
    PairList pl{};
    int build_pairlist(cudaStream_t st, const float* pos4, double rlist, int cap);
    // the last HOOMD-layout build: its overflow flag is read lazily as well
    // (page-locked copy + event); compute and md_run check it when handed
    // the rows it wrote
    int* h_nl_ovf = nullptr;
    cudaEvent_t nl_ev = nullptr;
    bool nl_pending = false, nl_overflow = false;
    const unsigned *nl_last_head = nullptr, *nl_last_nl = nullptr;
    int nlist_check(bool wait, int* needed);
    // ESP_ERR_OVERFLOW when the last pair-list build overflowed; without
    // `wait` an unfinished build counts as fine (checked again next time)
    int pairlist_check(bool wait, int* needed);
    // second stream for the concurrent pair term, its force array and the
    // fork/join events (created at plan time, kept across re-plans)
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    float4* d_fsr = nullptr;
    // FP64 mode: tables, records, spectrum and work lists
    bool f64 = false;
    DevAlloc mem64;
    double4 *d_posq64 = nullptr, *d_trec64 = nullptr, *d_srec64 = nullptr;
    double *d_w64 = nullptr, *d_q64 = nullptr, *d_phi64 = nullptr;
    double2 *d_tw64 = nullptr, *d_cbuf = nullptr, *d_gtab64 = nullptr;
    int2 *d_pch64 = nullptr, *d_xl = nullptr, *d_yl = nullptr, *d_zl = nullptr;
    int n_pch64 = 0, n_xl = 0, n_yl = 0, n_zl = 0, nq64 = 0;
    int plan64(const std::vector<float2>& tw, long long g_total);
    int compute_f64(cudaStream_t st, const double* pos4, const double* q, const unsigned* head, const unsigned* nn,
                    const unsigned* nl, double* force4, double* energy, double* virial, int flags);
    // rigid (O, H, H) molecules of the MD harness (SETTLE / RATTLE)
    DevAlloc rgmem;
    int4* d_mols = nullptr;   // {system, first atom, molecules} per SETTLE_CHUNK molecules
    int2* d_rskip = nullptr;  // per system: local range of the molecules' atoms
    double2* d_geo = nullptr; // (d_OH, d_HH)
    int n_mols = 0;           // work items
    double r_doh = 0, r_dhh = 0;
    int set_rigid(const int* first, const int* count, double d_oh, double d_hh);
    int nve1(cudaStream_t st, void* pos4, void* vel4, const void* force4, double dt, bool f64);
    int nve2(cudaStream_t st, const void* pos4, void* vel4, const void* force4, double dt, bool f64);
    // excluded pairs (caller-owned device arrays), applied by every
    // long-range evaluation
    const uint32_t* ex_n = nullptr;
    const uint32_t* ex_list = nullptr;
    int ex_pitch = 0;

    StageTimer timer;
    struct GraphKey {
        const void *pos, *vel, *q, *head, *nn, *nl, *force, *energy, *virial;
        double dt;
        bool with_energy;
        bool f64 = false;                               // md_run_f64 steps
        double lj_eps = 0, lj_sigma = 0, lj_rcut = 0;   // md_run_f64's Lennard-Jones term (sigma 0: none)
        bool operator==(const GraphKey& o) const {
            return pos == o.pos && vel == o.vel && q == o.q && head == o.head && nn == o.nn && nl == o.nl &&
                   force == o.force && energy == o.energy && virial == o.virial && dt == o.dt &&
                   with_energy == o.with_energy && f64 == o.f64 && lj_eps == o.lj_eps && lj_sigma == o.lj_sigma &&
                   lj_rcut == o.lj_rcut;
        }
    };
    // captured MD steps, one per distinct set of caller pointers; a few
    // entries so that a caller alternating between buffer sets (uploads of
    // the next batch overlapping this one) does not recapture every call.
    // The least recently used entry is replaced.
    static constexpr int N_GRAPHS = 8;
    struct GraphEntry {
        GraphKey key{};
        cudaGraphExec_t exec = nullptr;
        unsigned long long used = 0;
    } graphs[N_GRAPHS];
    unsigned long long graph_tick = 0;
    void drop_graphs() {
        for (GraphEntry& g : graphs)
            if (g.exec) {
                cudaGraphExecDestroy(g.exec);
                g.exec = nullptr;
            }
    }
    ~esp_batch() {
        drop_graphs();
        if (st2) {
            cudaStreamSynchronize(st2);
            cudaStreamDestroy(st2);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (pl_ev) {
            cudaEventSynchronize(pl_ev);
            cudaEventDestroy(pl_ev);
        }
        if (h_pl_ovf) cudaFreeHost(h_pl_ovf);
        if (nl_ev) {
            cudaEventSynchronize(nl_ev);
            cudaEventDestroy(nl_ev);
        }
        if (h_nl_ovf) cudaFreeHost(h_nl_ovf);
    }

    LaunchArgs args() const;
    int plan(const esp_params& p, int ns, const int* N_, const double* boxes, const int* mesh_);
    int md_run(cudaStream_t st, float* pos4, float* vel4, const float* q, const unsigned* head, const unsigned* nn,
               const unsigned* nl, float* force4, double* energy, double* virial, int nsteps, double dt,
               int use_graph);
    int md_run_f64(cudaStream_t st, double* pos4, double* vel4, const double* q, const unsigned* head,
                   const unsigned* nn, const unsigned* nl, double* force4, double* energy, double* virial, int nsteps,
                   double dt, double lj_eps, double lj_sigma, double lj_rcut, int use_graph);
    // nsteps calls of step(with_energy), with_energy on the last; with
    // use_graph each form is captured once per key (st is swapped for the
    // capture stream while step runs) and replayed
    int run_steps(cudaStream_t& st, GraphKey key, const std::function<int(bool)>& step, int nsteps, bool use_graph);
    // want_energy = false (MD steps whose energies are overwritten by the
    // next step) leaves the pair energies out of force.w and energy
    // virial_pp / external: HOOMD's per-particle virial (6 x pitch floats)
    // and the terms no particle owns (7 doubles per system), both optional
    int compute(cudaStream_t st, const float* pos4, const float* q, const unsigned* head, const unsigned* nn,
                const unsigned* nl, float* force4, double* energy, double* virial, int flags,
                bool want_energy = true, float* virial_pp = nullptr, int vpp_pitch = 0,
                double* external = nullptr);
    int spread_only(cudaStream_t st, const float* pos4, const float* q, double* rho_out);
    int build_nlist(cudaStream_t st, const float* pos4, double rlist, int cap, unsigned* head, unsigned* nn,
                    unsigned* nl);
    int info(int s, esp_info* out) const;
    int autotune(cudaStream_t st, const float* pos4, const float* q, const unsigned* head, const unsigned* nn,
                 const unsigned* nl, int flags, int reps, esp_params* chosen, double* trial_ms, int max_trials);
};

int esp_batch::plan(const esp_params& p, int ns, const int* N_, const double* boxes, const int* mesh_) {
    mem.release();
    mem64.release();
    f64 = false;
    if (p.precision != ESP_FP32 && p.precision != ESP_FP64) return fail(ESP_ERR_INVALID, "precision must be ESP_FP32 or ESP_FP64");
    // the neighbour-list cell grids and the pair list depend only on the
    // systems (particle counts, boxes): a re-plan of the same systems (the
    // autotuner's candidates) keeps them
    const bool same_systems = ns == nsys && std::equal(N_, N_ + ns, N.begin()) &&
                              std::equal(boxes, boxes + 3 * ns, box.begin());
    if (!same_systems) {
        rgmem.release();
        n_mols = 0;
        d_mols = nullptr;
        d_rskip = nullptr;
        cg_nl.mem.release();
        cg_nl.rlist = -1;
        cg_pl.mem.release();
        cg_pl.rlist = -1;
        plmem.release();
        pl_cap = 0;
        pl_ready = pl_pending = pl_overflow = false;
        nl_last_head = nl_last_nl = nullptr;
        nl_pending = nl_overflow = false;
    }
    prm = p;
    if (ns <= 0) return fail(ESP_ERR_INVALID, "number of systems must be positive");
    if (p.order < 2 || p.order > MAX_P) return fail(ESP_ERR_UNSUPPORTED, "order must be in [2, 12]");
    if (p.interp_mode < 0 || p.interp_mode > 2) return fail(ESP_ERR_INVALID, "interp_mode must be 0, 1 or 2");
    if (!(p.rcut > 0)) return fail(ESP_ERR_INVALID, "rcut must be positive");
    if (p.alpha != 0.0) return fail(ESP_ERR_UNSUPPORTED, "Debye screening (alpha != 0) is not supported");
    if (p.kappa < 0 || p.window_c < 0) return fail(ESP_ERR_INVALID, "kappa and window_c must be >= 0");
    P = p.order;
    nsys = ns;
    N.assign(N_, N_ + ns);
    box.assign(boxes, boxes + 3 * ns);
    mesh.assign(3 * ns, 0);
    tpp = p.threads_per_particle ? p.threads_per_particle : 4;  // the tuned choice on the mixed batch
    if (tpp != 4 && tpp != 8 && tpp != 16 && tpp != 32)
        return fail(ESP_ERR_UNSUPPORTED, "threads_per_particle must be 4, 8, 16 or 32");
    const double target = p.target_error > 0 ? p.target_error : 1e-5;
    const double kreq = kappa_required(target);
    // default tile: extended region E = T + P - 1 = 16 (the dense spreading
    // kernel's register column and a 16^3 interpolation tile)
    T = p.tile > 0 ? p.tile : std::max(1, 17 - P);
    if (T > 64) return fail(ESP_ERR_UNSUPPORTED, "tile edge must be <= 64");
    totN = 0;
    for (int s = 0; s < ns; ++s) {
        if (N[s] < 0) return fail(ESP_ERR_INVALID, "negative particle count");
        if (N[s] >= (1 << 26)) return fail(ESP_ERR_UNSUPPORTED, "at most 2^26 - 1 particles per system");
        for (int d = 0; d < 3; ++d) {
            const double L = box[3 * s + d];
            if (!(L > 0)) return fail(ESP_ERR_INVALID, "box lengths must be positive");
            if (2.0 * p.rcut > L) return fail(ESP_ERR_INVALID, "rcut must not exceed half the box");
            int n = mesh_ ? mesh_[3 * s + d] : 0;
            if (n <= 0 && d == 0 && p.nx > 0) n = p.nx;
            if (n <= 0 && d == 1 && p.ny > 0) n = p.ny;
            if (n <= 0 && d == 2 && p.nz > 0) n = p.nz;
            if (n <= 0) {
                const double h = M_PI * p.rcut / kreq;
                n = smooth235(std::max(P, (int)std::ceil(L / h)));
            }
            if (n < P || n < 4 || n > FFT_MAX_N || radix_plan(n) == 0)
                return fail(ESP_ERR_UNSUPPORTED, "mesh size " + std::to_string(n) +
                                                     " must be 2/3/5-smooth, >= order and <= 256");
            if (T > n) T = n;
            mesh[3 * s + d] = n;
        }
        totN += N[s];
    }
    D = p.window_degree > 0 ? p.window_degree
                            : (p.precision == ESP_FP64 ? std::max(P + 2, 9) : default_window_degree(P));
    if (D > MAX_D) return fail(ESP_ERR_UNSUPPORTED, "window degree must be <= 15");
    // parameter sets
    std::map<std::tuple<double, double>, int> pmap;
    psh.clear();
    psd.clear();
    c_split.assign(ns, 0);
    c_win.assign(ns, 0);
    std::vector<int> sys_pset(ns);
    // One split per batch: the coarsest mesh sets c, so every system shares
    // the pair-term polynomial (kernel-parameter resident) and the finer
    // meshes are only more accurate.
    double hmax_all = 0;
    for (int s = 0; s < ns; ++s)
        for (int d = 0; d < 3; ++d) hmax_all = std::max(hmax_all, box[3 * s + d] / mesh[3 * s + d]);
    for (int s = 0; s < ns; ++s) {
        const double c = p.kappa > 0 ? std::max(2.0, std::min(60.0, p.kappa * p.rcut))
                                     : split_c_for_spacing(p.rcut, hmax_all);
        const double cw = p.window_c > 0 ? p.window_c : 2.2 * P;
        c_split[s] = c;
        c_win[s] = cw;
        auto key = std::make_tuple(c, cw);
        auto it = pmap.find(key);
        if (it == pmap.end()) {
            PsetHost h;
            ParamSet d;
            // the FP64 mode fits the split polynomial to 1e-12; for FP32 a 3e-8
            // fit is below the FP32 evaluation's own rounding (~1e-7) and
            // saves a term per pair
            const int rc = build_param_set(c, cw, P, D, p.rcut, h, d, p.precision == ESP_FP64 ? 1e-12 : 3e-8);
            if (rc) return rc;
            it = pmap.emplace(key, (int)psh.size()).first;
            psh.push_back(std::move(h));
            psd.push_back(d);
        }
        sys_pset[s] = it->second;
    }
    // twiddles
    std::map<int, int> twoff;
    std::vector<float2> tw;
    auto twid = [&](int n) {
        auto it = twoff.find(n);
        if (it != twoff.end()) return it->second;
        const int off = (int)tw.size();
        for (int t = 0; t < n; ++t) {
            const double a = -2.0 * M_PI * t / n;
            tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        }
        twoff[n] = off;
        return off;
    };
    // system descriptors, influence-table sharing
    sd.assign(ns, SysDev{});
    std::map<std::tuple<int, double, double, double, int, int, int>, long long> gmap;
    long long m_off = 0, s_off = 0, g_off = 0, mp_off = 0;
    int p_off = 0, t_off = 0;
    std::vector<int> g_first;  // system that owns each distinct table
    for (int s = 0; s < ns; ++s) {
        SysDev& S = sd[s];
        S.N = N[s];
        S.p_off = p_off;
        S.nx = mesh[3 * s];
        S.ny = mesh[3 * s + 1];
        S.nz = mesh[3 * s + 2];
        S.nxh = S.nx / 2 + 1;
        S.m_off = m_off;
        S.s_off = s_off;
        S.ntx = (S.nx + T - 1) / T;
        S.nty = (S.ny + T - 1) / T;
        S.ntz = (S.nz + T - 1) / T;
        S.t_off = t_off;
        S.nxp = halo_extent(S.nx, T, P, true);
        S.nyp = halo_extent(S.ny, T, P, false);
        S.nzp = halo_extent(S.nz, T, P, false);
        S.mp_off = mp_off;
        S.Lx = (float)box[3 * s];
        S.Ly = (float)box[3 * s + 1];
        S.Lz = (float)box[3 * s + 2];
        S.inv_Lx = 1.0f / S.Lx;
        S.inv_Ly = 1.0f / S.Ly;
        S.inv_Lz = 1.0f / S.Lz;
        S.gxd = S.nx / box[3 * s];
        S.gyd = S.ny / box[3 * s + 1];
        S.gzd = S.nz / box[3 * s + 2];
        S.Lxd = box[3 * s];
        S.Lyd = box[3 * s + 1];
        S.Lzd = box[3 * s + 2];
        S.V = box[3 * s] * box[3 * s + 1] * box[3 * s + 2];
        S.pset = sys_pset[s];
        S.twx = twid(S.nx);
        S.twy = twid(S.ny);
        S.twz = twid(S.nz);
        S.radx = radix_plan(S.nx);
        S.rady = radix_plan(S.ny);
        S.radz = radix_plan(S.nz);
        auto gk = std::make_tuple(S.pset, box[3 * s], box[3 * s + 1], box[3 * s + 2], S.nx, S.ny, S.nz);
        auto it = gmap.find(gk);
        if (it == gmap.end()) {
            it = gmap.emplace(gk, g_off).first;
            g_first.push_back(s);
            g_off += (long long)S.nz * S.ny * S.nxh;
        }
        S.g_off = it->second;
        p_off += N[s];
        m_off += (long long)S.nx * S.ny * S.nz;
        mp_off += ((long long)S.nxp * S.nyp * S.nzp + 31) & ~31LL;  // 128-byte aligned systems
        s_off += (long long)S.nz * S.ny * S.nxh;
        t_off += S.ntx * S.nty * S.ntz;
    }
    n_tiles = t_off;
    // work lists
    std::vector<int2> chunks, pchunks;
    const int ppb = 256 / tpp;
    std::vector<int> tile_sys(n_tiles);
    std::vector<int4> xi, yi, zi;
    std::vector<int2> pi, si;
    smem_plane = 0;
    smem_slab = 0;
    for (int s = 0; s < ns; ++s) {
        const SysDev& S = sd[s];
        for (int i = 0; i < S.N; i += 256) chunks.push_back(make_int2(s, S.p_off + i));
        for (int i = 0; i < S.N; i += ppb) pchunks.push_back(make_int2(s, S.p_off + i));
        for (int t = 0; t < S.ntx * S.nty * S.ntz; ++t) tile_sys[S.t_off + t] = s;
        // whole planes / slabs in shared memory when they fit, else per-line passes
        const int sp = fft_plane_smem(S.nx, S.ny), ss = fft_slab_smem(S.nx, S.nz);
        if (sp <= FFT_SMEM_MAX && p.fft_mode == 0) {
            smem_plane = std::max(smem_plane, sp);
            for (int z = 0; z < S.nz; ++z) pi.push_back(make_int2(s, z));
        } else {
            for (int z = 0; z < S.nz; ++z)
                for (int y0 = 0; y0 < S.ny; y0 += 2 * FFT_B_X) xi.push_back(make_int4(s, z, y0, 0));
            for (int z = 0; z < S.nz; ++z)
                for (int k0 = 0; k0 < S.nxh; k0 += FFT_B_YZ) yi.push_back(make_int4(s, z, k0, 0));
        }
        if (ss <= FFT_SMEM_MAX && p.fft_mode == 0) {
            smem_slab = std::max(smem_slab, ss);
            for (int y = 0; y < S.ny; ++y) si.push_back(make_int2(s, y));
        } else {
            for (int y = 0; y < S.ny; ++y)
                for (int k0 = 0; k0 < S.nxh; k0 += FFT_B_YZ) zi.push_back(make_int4(s, y, k0, 0));
        }
    }
    // FFT work in decreasing size (longest processing time first): the
    // largest planes and slabs of an uneven batch start first instead of
    // forming the launch's tail
    auto plane_cost = [&](const int2& it) { return (long long)sd[it.x].nx * sd[it.x].ny; };
    auto slab_cost = [&](const int2& it) { return (long long)sd[it.x].nx * sd[it.x].nz; };
    std::stable_sort(pi.begin(), pi.end(), [&](const int2& a, const int2& b) { return plane_cost(a) > plane_cost(b); });
    std::stable_sort(si.begin(), si.end(), [&](const int2& a, const int2& b) { return slab_cost(a) > slab_cost(b); });
    auto line_cost = [&](const int4& it) { return (long long)std::max({sd[it.x].nx, sd[it.x].ny, sd[it.x].nz}); };
    for (auto* v : {&xi, &yi, &zi})
        std::stable_sort(v->begin(), v->end(), [&](const int4& a, const int4& b) { return line_cost(a) > line_cost(b); });
    n_p = (int)pi.size();
    n_s = (int)si.size();
    n_chunks = (int)chunks.size();
    n_pchunks = (int)pchunks.size();
    n_x = (int)xi.size();
    n_y = (int)yi.size();
    n_z = (int)zi.size();
    choose_pitch(P, T + P - 1, PX, PP);
    // allocate
    int rc = 0;
    if ((rc = mem.get(d_sys, ns)) || (rc = mem.get(d_pset, psd.size())) || (rc = mem.get(d_chunks, chunks.size())) ||
        (rc = mem.get(d_pchunks, pchunks.size())) || (rc = mem.get(d_tile_sys, n_tiles)) ||
        (rc = mem.get(d_tcount, n_tiles)) || (rc = mem.get(d_tstart, n_tiles + 1)) || (rc = mem.get(d_posq, totN)) ||
        (rc = mem.get(d_trec, totN)) || (rc = mem.get(d_srec, totN)) || (rc = mem.get(d_rel, totN)) ||
        (rc = mem.get(d_key, totN)) || (rc = mem.get(d_perm_u, totN)) || (rc = mem.get(d_perm, totN)) ||
        (rc = mem.get(d_srel, totN)) || (rc = mem.get(d_rho, m_off)) || (rc = mem.get(d_phi, mp_off)) ||
        (rc = mem.get(d_spec, s_off)) || (rc = mem.get(d_gtab, g_off)) || (rc = mem.get(d_tw, tw.size())) ||
        (rc = mem.get(d_x, xi.size())) || (rc = mem.get(d_y, yi.size())) || (rc = mem.get(d_z, zi.size())) ||
        (rc = mem.get(d_p, pi.size())) || (rc = mem.get(d_s, si.size())) ||
        (rc = mem.get(d_acc, (size_t)ns * ACC_STRIDE)) || (rc = mem.get(d_energy, ns)) ||
        (rc = mem.get(d_virial, (size_t)ns * 6)) || (rc = mem.get(d_fsr, totN)) || (rc = mem.get(d_kerr, 2)))
        return rc;
    ESPB_CK(cudaMemset(d_kerr, 0, 2 * sizeof(int)));
    // tensor maps for the TMA-staged interpolation (supports 5..8; the
    // cp.async form otherwise or when any map cannot be encoded)
    d_tmaps = nullptr;
    interp_box(T + P - 1, tma_bx, tma_by);
    if ((p.interp_mode == 0 || p.interp_mode == 2) && P >= 5 && P <= 8) {
        std::vector<CUtensorMap> maps(ns);
        bool ok = true;
        for (int s = 0; s < ns && ok; ++s) {
            const SysDev& S = sd[s];
            ok = encode_phi_map(&maps[s], d_phi + S.mp_off, S.nxp, S.nyp, S.nzp, tma_bx, tma_by, T + P - 1);
        }
        if (ok) {
            if ((rc = mem.get(d_tmaps, ns))) return rc;
            ESPB_CK(cudaMemcpy(d_tmaps, maps.data(), ns * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
        }
    }
    if (!st2) {
        ESPB_CK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
        ESPB_CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        ESPB_CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    }
    ESPB_CK(cudaMemcpy(d_sys, sd.data(), ns * sizeof(SysDev), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_pset, psd.data(), psd.size() * sizeof(ParamSet), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_chunks, chunks.data(), chunks.size() * sizeof(int2), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_pchunks, pchunks.data(), pchunks.size() * sizeof(int2), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_tile_sys, tile_sys.data(), n_tiles * sizeof(int), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_x, xi.data(), xi.size() * sizeof(int4), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_y, yi.data(), yi.size() * sizeof(int4), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_z, zi.data(), zi.size() * sizeof(int4), cudaMemcpyHostToDevice));
    if (!pi.empty()) ESPB_CK(cudaMemcpy(d_p, pi.data(), pi.size() * sizeof(int2), cudaMemcpyHostToDevice));
    if (!si.empty()) ESPB_CK(cudaMemcpy(d_s, si.data(), si.size() * sizeof(int2), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemset(d_tcount, 0, n_tiles * sizeof(uint32_t)));
    ESPB_CK(cudaMemset(d_rho, 0, (size_t)std::max<long long>(m_off, 1) * sizeof(double)));
    drop_graphs();
    {
        // kernel attributes are set here, outside any stream capture
        LaunchArgs a = args();
        a.configure_only = 1;
        // a tile whose kernels need more shared memory than a CTA can have
        // is refused here (the attribute call fails with an invalid value)
        if (launch_spread(a, 0) != cudaSuccess || launch_interp(a, 0) != cudaSuccess) {
            cudaGetLastError();
            return fail(ESP_ERR_UNSUPPORTED, "tile edge " + std::to_string(T) + " with support " + std::to_string(P) +
                                                 ": its extended region needs more shared memory than a CTA has; "
                                                 "use a smaller tile");
        }
        ESPB_CK(launch_fft(a, 0));
    }
    f64 = p.precision == ESP_FP64;
    if (f64) {
        if ((rc = plan64(tw, g_off))) return rc;
    }
    // influence tables (FP64 on the GPU)
    for (int s : g_first) {
        const SysDev& S = sd[s];
        const PsetHost& h = psh[S.pset];
        std::vector<double> w1d, tq, wq;
        influence_inputs(S, h, box[3 * s], box[3 * s + 1], box[3 * s + 2], p.rcut, w1d, tq, wq);
        const int nq = (int)tq.size();
        double *d_w1d = nullptr, *d_tq = nullptr, *d_wq = nullptr;
        ESPB_CK(cudaMalloc(&d_w1d, w1d.size() * sizeof(double)));
        ESPB_CK(cudaMalloc(&d_tq, nq * sizeof(double)));
        ESPB_CK(cudaMalloc(&d_wq, nq * sizeof(double)));
        ESPB_CK(cudaMemcpy(d_w1d, w1d.data(), w1d.size() * sizeof(double), cudaMemcpyHostToDevice));
        ESPB_CK(cudaMemcpy(d_tq, tq.data(), nq * sizeof(double), cudaMemcpyHostToDevice));
        ESPB_CK(cudaMemcpy(d_wq, wq.data(), nq * sizeof(double), cudaMemcpyHostToDevice));
        cudaError_t e = launch_influence(S, d_w1d, d_tq, d_wq, nq, p.rcut, 1e-14, d_gtab, 0);
        if (e == cudaSuccess && f64) e = launch_influence64(S, d_w1d, d_tq, d_wq, nq, p.rcut, 1e-14, d_gtab64, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        cudaFree(d_w1d);
        cudaFree(d_tq);
        cudaFree(d_wq);
        if (e != cudaSuccess) return fail(ESP_ERR_CUDA, std::string("influence build: ") + cudaGetErrorString(e));
    }
    return 0;
}

// FP64 tables (window and split coefficients in double, twiddles from FP64
// angles), FP64 records and spectrum, and the FP64 work lists: 32 particles
// per pair chunk, four x row pairs or y/z lines per FFT item.
int esp_batch::plan64(const std::vector<float2>& tw, long long g_total) {
    const PsetHost& h = psh[0];
    std::vector<double> w64(h.win.coef.begin(), h.win.coef.end());
    std::vector<double> q64(h.split.qv.begin(), h.split.qv.end());
    nq64 = (int)q64.size();
    std::vector<double2> tw64(tw.size());
    for (const SysDev& S : sd)
        for (int d = 0; d < 3; ++d) {
            const int n = d == 0 ? S.nx : (d == 1 ? S.ny : S.nz);
            const int off = d == 0 ? S.twx : (d == 1 ? S.twy : S.twz);
            for (int t = 0; t < n; ++t) {
                const double a = -2.0 * M_PI * t / n;
                tw64[off + t] = make_double2(std::cos(a), std::sin(a));
            }
        }
    std::vector<int2> pch, xl, yl, zl;
    long long M = 0;
    for (int s = 0; s < nsys; ++s) {
        const SysDev& S = sd[s];
        for (int i = 0; i < S.N; i += 32) pch.push_back(make_int2(s, S.p_off + i));
        // half spectrum: x row pairs, then nxh columns for the y and z lines
        const long long lx = (long long)((S.ny + 1) / 2) * S.nz, ly = (long long)S.nxh * S.nz,
                        lz = (long long)S.nxh * S.ny;
        for (long long l = 0; l < lx; l += 4) xl.push_back(make_int2(s, (int)l));
        for (long long l = 0; l < ly; l += 4) yl.push_back(make_int2(s, (int)l));
        for (long long l = 0; l < lz; l += 4) zl.push_back(make_int2(s, (int)l));
        M += (long long)S.nx * S.ny * S.nz;
    }
    n_pch64 = (int)pch.size();
    n_xl = (int)xl.size();
    n_yl = (int)yl.size();
    n_zl = (int)zl.size();
    int rc = 0;
    if ((rc = mem64.get(d_posq64, totN)) || (rc = mem64.get(d_trec64, totN)) || (rc = mem64.get(d_srec64, totN)) ||
        (rc = mem64.get(d_w64, w64.size())) || (rc = mem64.get(d_q64, q64.size())) || (rc = mem64.get(d_phi64, M)) ||
        (rc = mem64.get(d_tw64, tw64.size())) || (rc = mem64.get(d_cbuf, M)) || (rc = mem64.get(d_gtab64, g_total)) ||
        (rc = mem64.get(d_pch64, pch.size())) || (rc = mem64.get(d_xl, xl.size())) || (rc = mem64.get(d_yl, yl.size())) ||
        (rc = mem64.get(d_zl, zl.size())))
        return rc;
    ESPB_CK(cudaMemcpy(d_w64, w64.data(), w64.size() * sizeof(double), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_q64, q64.data(), q64.size() * sizeof(double), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_tw64, tw64.data(), tw64.size() * sizeof(double2), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_pch64, pch.data(), pch.size() * sizeof(int2), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_xl, xl.data(), xl.size() * sizeof(int2), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_yl, yl.data(), yl.size() * sizeof(int2), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_zl, zl.data(), zl.size() * sizeof(int2), cudaMemcpyHostToDevice));
    if (launch64_configure(P, T) != cudaSuccess) {
        cudaGetLastError();
        return fail(ESP_ERR_UNSUPPORTED, "tile edge " + std::to_string(T) + " with support " + std::to_string(P) +
                                             ": the FP64 tile kernels need more shared memory than a CTA has; "
                                             "use a smaller tile");
    }
    return 0;
}

int esp_batch::compute_f64(cudaStream_t st, const double* pos4, const double* q, const unsigned* head,
                           const unsigned* nn, const unsigned* nl, double* force4, double* energy, double* virial,
                           int flags) {
    if (!f64) return fail(ESP_ERR_UNSUPPORTED, "context planned for FP32: create it with precision ESP_FP64");
    if (!pos4 || !q || !force4) return fail(ESP_ERR_INVALID, "null position, charge or force pointer");
    if (!(flags & ESP_ALL)) return fail(ESP_ERR_INVALID, "flags select no term");
    if ((flags & ESP_SHORT_RANGE) && (!head || !nn || !nl))
        return fail(ESP_ERR_INVALID, "short-range term needs the neighbour list");
    Launch64 b;
    b.a = args();
    LaunchArgs& a = b.a;
    if (energy) a.energy = energy;
    if (virial) a.virial = virial;
    a.want_virial = virial != nullptr;
    a.nl_head = head;
    a.nl_n = nn;
    a.nl_list = nl;
    a.ex_n = ex_n;
    a.ex_list = ex_list;
    a.ex_pitch = ex_pitch;
    b.long_range = flags & ESP_LONG_RANGE;
    b.short_range = flags & ESP_SHORT_RANGE;
    a.add_bg = b.long_range ? 1 : 0;
    b.pos_in = reinterpret_cast<const double4*>(pos4);
    b.q_in = q;
    b.posq = d_posq64;
    b.trec = d_trec64;
    b.srec = d_srec64;
    b.force = reinterpret_cast<double4*>(force4);
    b.wcoef = d_w64;
    b.qv = d_q64;
    b.nq = nq64;
    b.tw = d_tw64;
    b.cbuf = d_cbuf;
    b.phi = d_phi64;
    b.gtab = d_gtab64;
    b.pchunks = d_pch64;
    b.n_pchunks = n_pch64;
    b.xl = d_xl;
    b.yl = d_yl;
    b.zl = d_zl;
    b.n_xl = n_xl;
    b.n_yl = n_yl;
    b.n_zl = n_zl;
    ESPB_CK(cudaMemsetAsync(d_acc, 0, (size_t)nsys * ACC_STRIDE * sizeof(double), st));
    ESPB_CK(launch64_eval(b, st));
    if (!b.long_range)  // the bin stage counted particles per tile; clear for the next call
        ESPB_CK(cudaMemsetAsync(d_tcount, 0, (size_t)n_tiles * sizeof(uint32_t), st));
    ESPB_CK(launch_finalize(a, st));
    return 0;
}

LaunchArgs esp_batch::args() const {
    LaunchArgs a;
    a.sys = d_sys;
    a.psets = d_pset;
    a.nsys = nsys;
    a.P = P;
    a.T = T;
    a.D = D;
    a.PX = PX;
    a.PP = PP;
    a.tpp = tpp;
    // one split per batch (plan() guarantees a single parameter set)
    a.nq = psd[0].nq;
    for (int c = 0; c < MAX_QC; ++c) {
        a.pc.q[c] = c < psd[0].nq ? psd[0].qv[c] : 0.f;
        a.pc.d[c] = c < psd[0].nq - 1 ? psd[0].dqv[c] : 0.f;
    }
    a.chunks = d_chunks;
    a.n_chunks = n_chunks;
    a.pchunks = d_pchunks;
    a.n_pchunks = n_pchunks;
    a.tile_sys = d_tile_sys;
    a.n_tiles = n_tiles;
    a.tile_count = d_tcount;
    a.tile_start = d_tstart;
    a.posq = d_posq;
    a.trec = d_trec;
    a.rel = d_rel;
    a.key = d_key;
    a.perm_u = d_perm_u;
    a.perm = d_perm;
    a.srec = d_srec;
    a.srel = d_srel;
    a.rho = d_rho;
    a.spec = d_spec;
    a.phi = d_phi;
    a.gtab = d_gtab;
    a.tw = d_tw;
    a.xitems = d_x;
    a.n_xitems = n_x;
    a.yitems = d_y;
    a.n_yitems = n_y;
    a.zitems = d_z;
    a.n_zitems = n_z;
    a.pitems = d_p;
    a.n_pitems = n_p;
    a.sitems = d_s;
    a.n_sitems = n_s;
    a.smem_plane = smem_plane;
    a.smem_slab = smem_slab;
    a.acc = d_acc;
    a.energy = d_energy;
    a.virial = d_virial;
    a.tmaps = d_tmaps;
    a.tma_bx = tma_bx;
    a.tma_by = tma_by;
    a.kerr = d_kerr;
    // interp_mode 2: the persistent TMA kernel fed from a tile queue (its counter)
    a.queue = prm.interp_mode == 2 ? d_kerr + 1 : nullptr;
    a.nmax_x = a.nmax_y = a.nmax_z = 1;
    for (const SysDev& S : sd) {
        a.nmax_x = std::max(a.nmax_x, S.nx);
        a.nmax_y = std::max(a.nmax_y, S.ny);
        a.nmax_z = std::max(a.nmax_z, S.nz);
    }
    return a;
}

int esp_batch::compute(cudaStream_t st, const float* pos4, const float* q, const unsigned* head, const unsigned* nn,
                       const unsigned* nl, float* force4, double* energy, double* virial, int flags,
                       bool want_energy, float* virial_pp, int vpp_pitch, double* external) {
    if (f64) return fail(ESP_ERR_UNSUPPORTED, "context planned for FP64: use esp_compute_f64");
    if (!pos4 || !q || !force4) return fail(ESP_ERR_INVALID, "null position, charge or force pointer");
    if (!(flags & ESP_ALL)) return fail(ESP_ERR_INVALID, "flags select no term");
    // no neighbour list given: the short-range term runs over the library's pair list
    const bool use_pl = !head && !nn && !nl;
    if ((flags & ESP_SHORT_RANGE) && !use_pl && (!head || !nn || !nl))
        return fail(ESP_ERR_INVALID, "short-range term needs the neighbour list (head, n_neigh, nlist)");
    if ((flags & ESP_SHORT_RANGE) && use_pl && !pl_ready)
        return fail(ESP_ERR_INVALID, "no neighbour list given and no pair list built (esp_batch_build_pairlist)");
    LaunchArgs a = args();
    if ((flags & ESP_SHORT_RANGE) && use_pl) a.plist = &pl;
    a.pos_in = reinterpret_cast<const float4*>(pos4);
    a.q_in = q;
    a.force = reinterpret_cast<float4*>(force4);
    if (energy) a.energy = energy;
    if (virial) a.virial = virial;
    if (virial_pp && vpp_pitch < totN) return fail(ESP_ERR_INVALID, "virial pitch below the particle count");
    a.want_virial = virial != nullptr || virial_pp != nullptr || external != nullptr;
    a.want_energy = (want_energy || a.want_virial) ? 1 : 0;
    a.virial_pp = virial_pp;
    a.vpp_pitch = vpp_pitch;
    a.external = external;
    if (virial_pp) ESPB_CK(cudaMemsetAsync(virial_pp, 0, (size_t)6 * vpp_pitch * sizeof(float), st));
    a.nl_head = head;
    a.nl_n = nn;
    a.nl_list = nl;
    const bool lr = flags & ESP_LONG_RANGE, sr = flags & ESP_SHORT_RANGE;
    a.accumulate = lr ? 1 : 0;
    a.add_bg = lr ? 1 : 0;
    ESPB_CK(cudaMemsetAsync(d_acc, 0, (size_t)nsys * ACC_STRIDE * sizeof(double), st));
    timer.begin(ESP_STAGE_BIN, st);
    ESPB_CK(launch_bin(a, st));
    timer.end(st);
    // The pair term needs only the wrapped positions of the bin stage: with
    // both terms requested it runs on a second stream, into its own force
    // array, concurrently with spread -> FFT -> interpolation (whose kernels
    // leave issue slots idle), and is added before the totals. Stage timing
    // keeps the sequential order so that per-stage times stay separable.
    // (not with a per-particle virial: the pair and exclusion kernels both add to it)
    const bool fork = lr && sr && !timer.on && d_fsr && !virial_pp;
    if (fork) {
        ESPB_CK(cudaEventRecord(ev_fork, st));
        ESPB_CK(cudaStreamWaitEvent(st2, ev_fork, 0));
        LaunchArgs ap = a;
        ap.force = d_fsr;
        ap.accumulate = 0;
        ESPB_CK(launch_pair(ap, st2));
        ESPB_CK(cudaEventRecord(ev_join, st2));
    }
    if (lr) {
        timer.begin(ESP_STAGE_SORT, st);
        ESPB_CK(launch_sort(a, st));
        timer.end(st);
        timer.begin(ESP_STAGE_SPREAD, st);
        ESPB_CK(launch_spread(a, st));
        timer.end(st);
        timer.begin(ESP_STAGE_FFT, st);
        ESPB_CK(launch_fft(a, st));
        timer.end(st);
        timer.begin(ESP_STAGE_INTERP, st);
        ESPB_CK(launch_interp(a, st));
        timer.end(st);
        if (ex_n) {
            a.ex_n = ex_n;
            a.ex_list = ex_list;
            a.ex_pitch = ex_pitch;
            ESPB_CK(launch_exclusions(a, st));
        }
    } else {
        // bin counted particles per tile; clear the histogram for the next call
        ESPB_CK(cudaMemsetAsync(d_tcount, 0, (size_t)n_tiles * sizeof(uint32_t), st));
    }
    if (fork) {
        ESPB_CK(cudaStreamWaitEvent(st, ev_join, 0));
        ESPB_CK(launch_add_forces(a.chunks, a.n_chunks, a.sys, d_fsr, a.force, st));
    } else if (sr) {
        timer.begin(ESP_STAGE_PAIR, st);
        ESPB_CK(launch_pair(a, st));
        timer.end(st);
    }
    ESPB_CK(launch_finalize(a, st));
    return 0;
}

int esp_batch::md_run(cudaStream_t st, float* pos4, float* vel4, const float* q, const unsigned* head,
                      const unsigned* nn, const unsigned* nl, float* force4, double* energy, double* virial, int nsteps,
                      double dt, int use_graph) {
    if (nsteps < 0) return fail(ESP_ERR_INVALID, "negative step count");
    if (!pos4 || !vel4 || !q || !force4) return fail(ESP_ERR_INVALID, "null pointer");
    if (!(head && nn && nl) && (head || nn || nl || !pl_ready))
        return fail(ESP_ERR_INVALID, "md_run needs the neighbour list (head, n_neigh, nlist) or a built pair list");
    {
        int rc = !head ? pairlist_check(false, nullptr)
                       : (head == nl_last_head && nl == nl_last_nl ? nlist_check(false, nullptr) : 0);
        if (rc) return rc;
    }
    // Every step overwrites the energies (force.w, energy) of the previous
    // one, so only the last step evaluates the pair energies.
    auto step = [&](bool with_energy) -> int {
        timer.begin(ESP_STAGE_NVE, st);
        int rc = nve1(st, pos4, vel4, force4, dt, false);
        timer.end(st);
        if (rc) return rc;
        rc = compute(st, pos4, q, head, nn, nl, force4, energy, virial, ESP_ALL, with_energy);
        if (rc) return rc;
        timer.begin(ESP_STAGE_NVE, st);
        rc = nve2(st, pos4, vel4, force4, dt, false);
        timer.end(st);
        return rc;
    };
    const GraphKey key{pos4, vel4, q, head, nn, nl, force4, energy, virial, dt, false};
    return run_steps(st, key, step, nsteps, use_graph && !timer.on);
}

int esp_batch::md_run_f64(cudaStream_t st, double* pos4, double* vel4, const double* q, const unsigned* head,
                          const unsigned* nn, const unsigned* nl, double* force4, double* energy, double* virial,
                          int nsteps, double dt, double lj_eps, double lj_sigma, double lj_rcut, int use_graph) {
    if (!f64) return fail(ESP_ERR_UNSUPPORTED, "context planned for FP32: create it with precision ESP_FP64");
    if (nsteps < 0) return fail(ESP_ERR_INVALID, "negative step count");
    if (!pos4 || !vel4 || !q || !force4 || !head || !nn || !nl)
        return fail(ESP_ERR_INVALID, "md_run_f64 needs positions, velocities, charges, forces and the neighbour list");
    const bool lj = lj_sigma > 0;
    if (lj && !(lj_rcut > 0)) return fail(ESP_ERR_INVALID, "Lennard-Jones r_cut must be positive");
    if (head == nl_last_head && nl == nl_last_nl) {
        const int rc = nlist_check(false, nullptr);
        if (rc) return rc;
    }
    auto step = [&](bool) -> int {
        int rc = nve1(st, pos4, vel4, force4, dt, true);
        if (rc) return rc;
        rc = compute_f64(st, pos4, q, head, nn, nl, force4, energy, virial, ESP_ALL);
        if (rc) return rc;
        if (lj)
            ESPB_CK(launch_lj(d_chunks, n_chunks, d_sys, pos4, head, nn, nl, lj_eps, lj_sigma, lj_rcut, force4, energy,
                              true, st));
        return nve2(st, pos4, vel4, force4, dt, true);
    };
    GraphKey key{pos4, vel4, q, head, nn, nl, force4, energy, virial, dt, false};
    key.f64 = true;
    key.lj_eps = lj ? lj_eps : 0.0;
    key.lj_sigma = lj ? lj_sigma : 0.0;
    key.lj_rcut = lj ? lj_rcut : 0.0;
    return run_steps(st, key, step, nsteps, use_graph != 0);
}

int esp_batch::run_steps(cudaStream_t& st, GraphKey key, const std::function<int(bool)>& step, int nsteps,
                         bool use_graph) {
    if (!use_graph) {
        for (int k = 0; k < nsteps; ++k) {
            int rc = step(k == nsteps - 1);
            if (rc) return rc;
        }
        return 0;
    }
    // one captured step per (key, energy or not)
    auto graph_for = [&](bool with_energy, cudaGraphExec_t& out) -> int {
        key.with_energy = with_energy;
        GraphEntry* ge = nullptr;
        for (GraphEntry& g : graphs)
            if (g.exec && g.key == key) ge = &g;
        if (!ge) {
            ge = &graphs[0];
            for (GraphEntry& g : graphs)
                if (!g.exec || g.used < ge->used) {
                    ge = &g;
                    if (!g.exec) break;
                }
            if (ge->exec) {
                cudaGraphExecDestroy(ge->exec);
                ge->exec = nullptr;
            }
            cudaStream_t cs = nullptr;
            ESPB_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
            int rc = 0;
            if (e == cudaSuccess) {
                cudaStream_t saved = st;
                st = cs;
                rc = step(with_energy);
                st = saved;
                cudaError_t e2 = cudaStreamEndCapture(cs, &g);
                if (e == cudaSuccess) e = e2;
            }
            cudaStreamDestroy(cs);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&ge->exec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                ge->exec = nullptr;
                return fail(ESP_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            }
            ge->key = key;
        }
        ge->used = ++graph_tick;
        out = ge->exec;
        return 0;
    };
    if (nsteps == 0) return 0;
    cudaGraphExec_t g_last = nullptr, g_mid = nullptr;
    int rc = 0;
    if (nsteps > 1 && (rc = graph_for(false, g_mid))) return rc;
    if ((rc = graph_for(true, g_last))) return rc;
    for (int k = 0; k + 1 < nsteps; ++k) ESPB_CK(cudaGraphLaunch(g_mid, st));
    ESPB_CK(cudaGraphLaunch(g_last, st));
    return 0;
}

int esp_batch::spread_only(cudaStream_t st, const float* pos4, const float* q, double* rho_out) {
    if (!pos4 || !q || !rho_out) return fail(ESP_ERR_INVALID, "null pointer");
    long long M = 0;
    for (const SysDev& S : sd) M += (long long)S.nx * S.ny * S.nz;
    ESPB_CK(cudaMemsetAsync(rho_out, 0, (size_t)M * sizeof(double), st));
    ESPB_CK(cudaMemsetAsync(d_acc, 0, (size_t)nsys * ACC_STRIDE * sizeof(double), st));
    LaunchArgs a = args();
    a.pos_in = reinterpret_cast<const float4*>(pos4);
    a.q_in = q;
    a.rho = rho_out;
    ESPB_CK(launch_bin(a, st));
    ESPB_CK(launch_sort(a, st));
    ESPB_CK(launch_spread(a, st));
    return 0;
}

int esp_batch::setup_cells(CellGrid& g, double rlist, int cap) {
    if (rlist == g.rlist) {
        if (cap == g.cap) return 0;
        // same cells, new row capacity: HOOMD-layout rows of system s start at p_off * cap
        for (int s = 0; s < nsys; ++s) g.h_cells[s].nl_off = (long long)sd[s].p_off * cap;
        ESPB_CK(cudaMemcpy(g.d_cells, g.h_cells.data(), nsys * sizeof(CellDev), cudaMemcpyHostToDevice));
        g.cap = cap;
        return 0;
    }
    g.mem.release();
    g.rlist = -1;
    g.cap = -1;
    g.h_cells.assign(nsys, CellDev{});
    std::vector<int> cell_sys;
    int c_off = 0;
    long long nl_off = 0;
    for (int s = 0; s < nsys; ++s) {
        CellDev& C = g.h_cells[s];
        int nc[3];
        for (int d = 0; d < 3; ++d) {
            if (2.0 * rlist > box[3 * s + d]) return fail(ESP_ERR_INVALID, "rlist must not exceed half the box");
            nc[d] = std::max(1, (int)std::floor(box[3 * s + d] / rlist));
        }
        C.ncx = nc[0];
        C.ncy = nc[1];
        C.ncz = nc[2];
        C.inv_wx = (float)(nc[0] / box[3 * s]);
        C.inv_wy = (float)(nc[1] / box[3 * s + 1]);
        C.inv_wz = (float)(nc[2] / box[3 * s + 2]);
        C.c_off = c_off;
        C.nl_off = nl_off;
        for (int c = 0; c < nc[0] * nc[1] * nc[2]; ++c) cell_sys.push_back(s);
        c_off += nc[0] * nc[1] * nc[2];
        nl_off += (long long)N[s] * cap;
    }
    g.n_cells = c_off;
    int rc = 0;
    if ((rc = g.mem.get(g.d_cells, nsys)) || (rc = g.mem.get(g.d_cell_sys, g.n_cells)) ||
        (rc = g.mem.get(g.d_ckey, totN)) || (rc = g.mem.get(g.d_ccount, g.n_cells)) ||
        (rc = g.mem.get(g.d_cstart, g.n_cells + 1)) || (rc = g.mem.get(g.d_cperm, totN)) ||
        (rc = g.mem.get(g.d_slot2idx, totN)) || (rc = g.mem.get(g.d_idx2slot, totN)) ||
        (rc = g.mem.get(g.d_wpos, totN)) ||
        (rc = g.mem.get(g.d_cpos, totN)) || (rc = g.mem.get(g.d_overflow, 2)))
        return rc;
    ESPB_CK(cudaMemcpy(g.d_cells, g.h_cells.data(), nsys * sizeof(CellDev), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(g.d_cell_sys, cell_sys.data(), g.n_cells * sizeof(int), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemset(g.d_ccount, 0, g.n_cells * sizeof(uint32_t)));
    g.rlist = rlist;
    g.cap = cap;
    return 0;
}

NlistArgs esp_batch::nlist_args(CellGrid& g, const float* pos4, double rlist, int cap) const {
    NlistArgs a;
    a.chunks = d_chunks;
    a.n_chunks = n_chunks;
    a.sys = d_sys;
    a.cells = g.d_cells;
    a.cell_sys = g.d_cell_sys;
    a.n_cells = g.n_cells;
    a.total = totN;
    a.pos = reinterpret_cast<const float4*>(pos4);
    a.ckey = g.d_ckey;
    a.ccount = g.d_ccount;
    a.cstart = g.d_cstart;
    a.perm_u = g.d_cperm;
    a.slot2idx = g.d_slot2idx;
    a.idx2slot = g.d_idx2slot;
    a.wpos = g.d_wpos;
    a.cpos = g.d_cpos;
    a.rlist2 = (float)(rlist * rlist);
    a.cap = cap;
    a.overflow = g.d_overflow;
    a.ex_n = ex_n;
    a.ex_list = ex_list;
    a.ex_pitch = ex_pitch;
    return a;
}

int esp_batch::build_nlist(cudaStream_t st, const float* pos4, double rlist, int cap, unsigned* head, unsigned* nn,
                           unsigned* nl) {
    if (!(rlist > 0) || cap <= 0) return fail(ESP_ERR_INVALID, "rlist and cap must be positive");
    if (!pos4 || !head || !nn || !nl) return fail(ESP_ERR_INVALID, "null pointer");
    if ((double)totN * cap >= 4294967296.0)
        return fail(ESP_ERR_UNSUPPORTED, "HOOMD-layout rows address 32-bit offsets: totN * cap must be below 2^32");
    int rc = setup_cells(cg_nl, rlist, cap);
    if (rc) return rc;
    NlistArgs a = nlist_args(cg_nl, pos4, rlist, cap);
    a.head = head;
    a.nn = nn;
    a.nl = nl;
    if (!h_nl_ovf) ESPB_CK(cudaHostAlloc((void**)&h_nl_ovf, 2 * sizeof(int), cudaHostAllocDefault));
    if (!nl_ev) ESPB_CK(cudaEventCreateWithFlags(&nl_ev, cudaEventDisableTiming));
    // HOOMD-layout rows: head[i] = first entry of system s + local i * cap
    timer.begin(ESP_STAGE_NLIST, st);
    ESPB_CK(launch_nlist(a, st));
    timer.end(st);
    // the overflow flag is read lazily (esp_batch_nlist_check, or the next
    // compute / md_run over these rows): no host synchronisation here
    ESPB_CK(cudaMemcpyAsync(h_nl_ovf, cg_nl.d_overflow, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    ESPB_CK(cudaEventRecord(nl_ev, st));
    nl_last_head = head;
    nl_last_nl = nl;
    nl_pending = true;
    nl_overflow = false;
    return 0;
}

int esp_batch::nlist_check(bool wait, int* needed) {
    if (!nl_ev || !h_nl_ovf) return fail(ESP_ERR_INVALID, "no neighbour list has been built (esp_batch_build_nlist)");
    if (nl_pending) {
        if (wait) {
            ESPB_CK(cudaEventSynchronize(nl_ev));
        } else {
            const cudaError_t q = cudaEventQuery(nl_ev);
            if (q == cudaErrorNotReady) return 0;
            if (q != cudaSuccess)
                return fail(ESP_ERR_CUDA, std::string("neighbour-list build: ") + cudaGetErrorString(q));
        }
        nl_pending = false;
        nl_overflow = h_nl_ovf[0] != 0;
    }
    if (needed) *needed = h_nl_ovf[1];
    if (nl_overflow)
        return fail(ESP_ERR_OVERFLOW, "neighbour-list row capacity exceeded (largest row " +
                                          std::to_string(h_nl_ovf[1]) + "); n_neigh holds the needed counts");
    return 0;
}

int esp_batch::build_pairlist(cudaStream_t st, const float* pos4, double rlist, int cap) {
    if (!(rlist > 0) || cap <= 0) return fail(ESP_ERR_INVALID, "rlist and cap must be positive");
    if (!pos4) return fail(ESP_ERR_INVALID, "null position pointer");
    if (f64) return fail(ESP_ERR_UNSUPPORTED, "the library's pair list serves the FP32 path");
    if ((double)totN * cap >= 4294967296.0) return fail(ESP_ERR_UNSUPPORTED, "pair list of 2^32 entries or more");
    int rc = setup_cells(cg_pl, rlist, cap);
    if (rc) return rc;
    if (pl_cap != cap) {
        plmem.release();
        pl_cap = 0;
        if ((rc = plmem.get(d_pl_nl, (size_t)totN * cap)) || (rc = plmem.get(d_pl_head, totN)) ||
            (rc = plmem.get(d_pl_nn, totN)) || (rc = plmem.get(d_spos, totN)))
            return rc;
        pl_cap = cap;
        drop_graphs();  // captured steps hold the previous arrays
    }
    if (!h_pl_ovf) ESPB_CK(cudaHostAlloc((void**)&h_pl_ovf, 2 * sizeof(int), cudaHostAllocDefault));
    if (!pl_ev) ESPB_CK(cudaEventCreateWithFlags(&pl_ev, cudaEventDisableTiming));
    NlistArgs a = nlist_args(cg_pl, pos4, rlist, cap);
    a.head = d_pl_head;
    a.nn = d_pl_nn;
    a.nl = d_pl_nl;
    a.sorted = true;
    timer.begin(ESP_STAGE_NLIST, st);
    ESPB_CK(launch_nlist(a, st));
    timer.end(st);
    // the overflow flag is read lazily: no host synchronisation here
    ESPB_CK(cudaMemcpyAsync(h_pl_ovf, cg_pl.d_overflow, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    ESPB_CK(cudaEventRecord(pl_ev, st));
    pl.slot2idx = cg_pl.d_slot2idx;
    pl.idx2slot = cg_pl.d_idx2slot;
    pl.spos = d_spos;
    pl.head = d_pl_head;
    pl.nn = d_pl_nn;
    pl.nl = d_pl_nl;
    pl.cap = cap;
    pl_ready = true;
    pl_pending = true;
    pl_overflow = false;
    return 0;
}

int esp_batch::pairlist_check(bool wait, int* needed) {
    if (!pl_ready) return fail(ESP_ERR_INVALID, "no pair list has been built (esp_batch_build_pairlist)");
    if (pl_pending) {
        if (wait) {
            ESPB_CK(cudaEventSynchronize(pl_ev));
        } else {
            const cudaError_t q = cudaEventQuery(pl_ev);
            if (q == cudaErrorNotReady) return 0;
            if (q != cudaSuccess) return fail(ESP_ERR_CUDA, std::string("pair-list build: ") + cudaGetErrorString(q));
        }
        pl_pending = false;
        pl_overflow = h_pl_ovf[0] != 0;
    }
    if (needed) *needed = h_pl_ovf[1];
    if (pl_overflow) {
        return fail(ESP_ERR_OVERFLOW, "pair-list row capacity exceeded (largest row " + std::to_string(h_pl_ovf[1]) +
                                          "); rebuild with a larger cap");
    }
    return 0;
}

int esp_batch::set_rigid(const int* first, const int* count, double d_oh, double d_hh) {
    rgmem.release();
    n_mols = 0;
    d_mols = nullptr;
    d_rskip = nullptr;
    drop_graphs();  // captured steps hold the previous molecule list
    if (!first || !count) return 0;
    if (!(d_oh > 0) || !(d_hh > 0) || d_hh >= 2.0 * d_oh)
        return fail(ESP_ERR_INVALID, "rigid water needs 0 < d_hh < 2 d_oh");
    std::vector<int4> mols;
    std::vector<int2> skip(nsys);
    for (int s = 0; s < nsys; ++s) {
        if (count[s] < 0 || first[s] < 0 || (long long)first[s] + 3LL * count[s] > N[s])
            return fail(ESP_ERR_INVALID, "rigid molecules outside system " + std::to_string(s));
        for (int m = 0; m < count[s]; m += SETTLE_CHUNK)
            mols.push_back(make_int4(s, sd[s].p_off + first[s] + 3 * m, std::min(SETTLE_CHUNK, count[s] - m), 0));
        skip[s] = make_int2(first[s], first[s] + 3 * count[s]);
    }
    int rc = 0;
    if ((rc = rgmem.get(d_mols, mols.size())) || (rc = rgmem.get(d_rskip, nsys)) || (rc = rgmem.get(d_geo, 1)))
        return rc;
    const double2 geo = make_double2(d_oh, d_hh);
    ESPB_CK(cudaMemcpy(d_geo, &geo, sizeof(double2), cudaMemcpyHostToDevice));
    if (!mols.empty()) ESPB_CK(cudaMemcpy(d_mols, mols.data(), mols.size() * sizeof(int4), cudaMemcpyHostToDevice));
    ESPB_CK(cudaMemcpy(d_rskip, skip.data(), nsys * sizeof(int2), cudaMemcpyHostToDevice));
    n_mols = (int)mols.size();
    r_doh = d_oh;
    r_dhh = d_hh;
    return 0;
}

int esp_batch::nve1(cudaStream_t st, void* pos4, void* vel4, const void* force4, double dt, bool is64) {
    const int2* skip = n_mols ? d_rskip : nullptr;
    if (is64)
        ESPB_CK(launch_nve64(1, d_chunks, n_chunks, d_sys, reinterpret_cast<double4*>(pos4),
                             reinterpret_cast<double4*>(vel4), reinterpret_cast<const double4*>(force4), dt, st, skip));
    else
        ESPB_CK(launch_nve1(d_chunks, n_chunks, d_sys, reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(vel4),
                            reinterpret_cast<const float4*>(force4), (float)dt, st, skip));
    if (n_mols) ESPB_CK(launch_settle1(d_mols, n_mols, d_sys, pos4, vel4, force4, dt, d_geo, is64, st));
    return 0;
}

int esp_batch::nve2(cudaStream_t st, const void* pos4, void* vel4, const void* force4, double dt, bool is64) {
    if (is64)
        ESPB_CK(launch_nve64(2, d_chunks, n_chunks, d_sys, nullptr, reinterpret_cast<double4*>(vel4),
                             reinterpret_cast<const double4*>(force4), dt, st));
    else
        ESPB_CK(launch_nve2(d_chunks, n_chunks, d_sys, reinterpret_cast<float4*>(vel4),
                            reinterpret_cast<const float4*>(force4), (float)dt, st));
    if (n_mols) ESPB_CK(launch_settle2(d_mols, n_mols, d_sys, pos4, vel4, is64, st));
    return 0;
}

int esp_batch::autotune(cudaStream_t st, const float* pos4, const float* q, const unsigned* head,
                        const unsigned* nn, const unsigned* nl, int flags, int reps, esp_params* chosen,
                        double* trial_ms, int max_trials) {
    if (f64) return fail(ESP_ERR_UNSUPPORTED, "the autotuner times the FP32 path");
    if (reps < 1) return fail(ESP_ERR_INVALID, "reps must be positive");
    const std::vector<int> Nv = N;
    const std::vector<double> boxv = box;
    const std::vector<int> meshv = mesh;  // candidates keep the meshes (and so the accuracy)
    esp_params cur = prm;
    cur.tile = T;
    cur.threads_per_particle = tpp;
    float* d_force = nullptr;
    double* d_e = nullptr;
    ESPB_CK(cudaMalloc(&d_force, (size_t)std::max(totN, 1) * 16));
    ESPB_CK(cudaMalloc(&d_e, (size_t)nsys * sizeof(double)));
    cudaEvent_t e0, e1;
    ESPB_CK(cudaEventCreate(&e0));
    ESPB_CK(cudaEventCreate(&e1));
    int ntrial = 0;
    auto run = [&](const esp_params& c, double& ms) -> int {
        int rc = plan(c, (int)Nv.size(), Nv.data(), boxv.data(), meshv.data());
        if (rc) return rc;
        if ((rc = compute(st, pos4, q, head, nn, nl, d_force, d_e, nullptr, flags))) return rc;  // warm-up
        ESPB_CK(cudaEventRecord(e0, st));
        for (int k = 0; k < reps; ++k)
            if ((rc = compute(st, pos4, q, head, nn, nl, d_force, d_e, nullptr, flags))) return rc;
        ESPB_CK(cudaEventRecord(e1, st));
        ESPB_CK(cudaEventSynchronize(e1));
        float t = 0.f;
        ESPB_CK(cudaEventElapsedTime(&t, e0, e1));
        ms = t / reps;
        if (trial_ms && ntrial < max_trials) trial_ms[ntrial] = ms;
        ++ntrial;
        return 0;
    };
    int rc = 0;
    double best_ms = 0;
    esp_params best = cur;
    if ((rc = run(cur, best_ms))) goto done;
    {
        // pair lanes per particle
        for (int t : {4, 8, 16}) {
            if (t == best.threads_per_particle) continue;
            esp_params c = best;
            c.threads_per_particle = t;
            double ms = 0;
            if ((rc = run(c, ms))) goto done;
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
        // tile edge: the 16^3 tensor-core tile and two smaller dense tiles
        const int Tdef = std::max(1, 17 - P);
        for (int t : {Tdef - 1, Tdef - 2}) {
            if (t < 2 || t == best.tile) continue;
            esp_params c = best;
            c.tile = t;
            double ms = 0;
            if ((rc = run(c, ms))) goto done;
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
        // FFT pass form
        {
            esp_params c = best;
            c.fft_mode = best.fft_mode ? 0 : 1;
            double ms = 0;
            if ((rc = run(c, ms))) goto done;
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
        // TMA interpolation: one CTA per tile, or persistent CTAs on a tile queue
        if (P >= 5 && P <= 8 && (best.interp_mode == 0 || best.interp_mode == 2)) {
            esp_params c = best;
            c.interp_mode = best.interp_mode == 0 ? 2 : 0;
            double ms = 0;
            if ((rc = run(c, ms))) goto done;
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    }
done:
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_force);
    cudaFree(d_e);
    if (rc) return rc;
    if ((rc = plan(best, (int)Nv.size(), Nv.data(), boxv.data(), meshv.data()))) return rc;
    if (chosen) *chosen = best;
    return 0;
}

int esp_batch::info(int s, esp_info* out) const {
    if (!out || s < 0 || s >= nsys) return fail(ESP_ERR_INVALID, "bad system index or null info");
    const SysDev& S = sd[s];
    const PsetHost& h = psh[S.pset];
    out->nx = S.nx;
    out->ny = S.ny;
    out->nz = S.nz;
    out->order = P;
    out->tile = T;
    out->window_degree = D;
    out->c_split = c_split[s];
    out->c_window = c_win[s];
    out->rcut = h.rcut;
    out->lambda0 = h.split.lambda0;
    out->m2 = h.split.m2;
    out->split_fit_err = h.split.fit_err;
    out->window_fit_err = h.win.fit_err;
    out->device_bytes = mem.bytes + cg_nl.mem.bytes + cg_pl.mem.bytes + plmem.bytes;
    return 0;
}

struct esp_ctx {
    esp_params prm{};
    double L[3] = {0, 0, 0};
    int N = -1;
    bool dirty = true;
    esp_batch b;
};

extern "C" {

int esp_params_default(esp_params* p) {
    if (!p) return fail(ESP_ERR_INVALID, "null params");
    std::memset(p, 0, sizeof(*p));
    p->order = 8;
    p->rcut = 3.0;
    p->n_table = 512;
    p->target_error = 1e-5;
    return 0;
}

const char* esp_last_error(void) { return g_err.c_str(); }

int esp_create(const esp_params* p, double Lx, double Ly, double Lz, int N, esp_ctx** out) {
    if (!p || !out) return fail(ESP_ERR_INVALID, "null argument");
    *out = nullptr;
    esp_ctx* c = new esp_ctx();
    c->prm = *p;
    c->L[0] = Lx;
    c->L[1] = Ly;
    c->L[2] = Lz;
    c->N = N;
    int rc = c->b.plan(c->prm, 1, &c->N, c->L, nullptr);
    if (rc) {
        delete c;
        return rc;
    }
    c->dirty = false;
    *out = c;
    return 0;
}

int esp_set_params(esp_ctx* c, const esp_params* p) {
    if (!c || !p) return fail(ESP_ERR_INVALID, "null argument");
    c->prm = *p;
    c->dirty = true;
    return 0;
}

int esp_set_box(esp_ctx* c, double Lx, double Ly, double Lz) {
    if (!c) return fail(ESP_ERR_INVALID, "null context");
    c->L[0] = Lx;
    c->L[1] = Ly;
    c->L[2] = Lz;
    c->dirty = true;
    return 0;
}

int esp_invalidate(esp_ctx* c) {
    if (!c) return fail(ESP_ERR_INVALID, "null context");
    c->dirty = true;
    return 0;
}

int esp_compute(esp_ctx* c, void* stream, const float* pos4, const float* charge, int N, const unsigned* head,
                const unsigned* n_neigh, const unsigned* nlist, float* force4, double* energy, double* virial6,
                int flags) {
    if (!c) return fail(ESP_ERR_INVALID, "null context");
    if (N < 0) return fail(ESP_ERR_INVALID, "negative particle count");
    if (N != c->N || c->dirty) {
        c->N = N;
        int rc = c->b.plan(c->prm, 1, &c->N, c->L, nullptr);
        if (rc) return rc;
        c->dirty = false;
    }
    if (N == 0) {
        cudaStream_t st = (cudaStream_t)stream;
        if (energy) ESPB_CK(cudaMemsetAsync(energy, 0, sizeof(double), st));
        if (virial6) ESPB_CK(cudaMemsetAsync(virial6, 0, 6 * sizeof(double), st));
        return 0;
    }
    return c->b.compute((cudaStream_t)stream, pos4, charge, head, n_neigh, nlist, force4, energy, virial6, flags);
}

int esp_compute_hoomd(esp_ctx* c, void* stream, const float* pos4, const float* charge, int N, const unsigned* head,
                      const unsigned* n_neigh, const unsigned* nlist, float* force4, float* virial_pp,
                      int virial_pitch, double* external7, int flags) {
    if (!c) return fail(ESP_ERR_INVALID, "null context");
    if (N <= 0) return fail(ESP_ERR_INVALID, "particle count must be positive");
    if (!virial_pp || !external7) return fail(ESP_ERR_INVALID, "null virial or external-term pointer");
    if (N != c->N || c->dirty) {
        c->N = N;
        int rc = c->b.plan(c->prm, 1, &c->N, c->L, nullptr);
        if (rc) return rc;
        c->dirty = false;
    }
    return c->b.compute((cudaStream_t)stream, pos4, charge, head, n_neigh, nlist, force4, nullptr, nullptr, flags,
                        true, virial_pp, virial_pitch, external7);
}

int esp_compute_f64(esp_ctx* c, void* stream, const double* pos4, const double* charge, int N, const unsigned* head,
                    const unsigned* n_neigh, const unsigned* nlist, double* force4, double* energy, double* virial6,
                    int flags) {
    if (!c) return fail(ESP_ERR_INVALID, "null context");
    if (N < 0) return fail(ESP_ERR_INVALID, "negative particle count");
    if (N != c->N || c->dirty) {
        c->N = N;
        int rc = c->b.plan(c->prm, 1, &c->N, c->L, nullptr);
        if (rc) return rc;
        c->dirty = false;
    }
    if (N == 0) {
        cudaStream_t st = (cudaStream_t)stream;
        if (energy) ESPB_CK(cudaMemsetAsync(energy, 0, sizeof(double), st));
        if (virial6) ESPB_CK(cudaMemsetAsync(virial6, 0, 6 * sizeof(double), st));
        return 0;
    }
    return c->b.compute_f64((cudaStream_t)stream, pos4, charge, head, n_neigh, nlist, force4, energy, virial6, flags);
}

int esp_get_info(const esp_ctx* c, esp_info* info) {
    if (!c) return fail(ESP_ERR_INVALID, "null context");
    return c->b.info(0, info);
}

int esp_destroy(esp_ctx* c) {
    delete c;
    return 0;
}

int esp_spread(esp_ctx* c, void* stream, const float* pos4, const float* charge, int N, double* rho) {
    if (!c) return fail(ESP_ERR_INVALID, "null context");
    if (N <= 0) return fail(ESP_ERR_INVALID, "particle count must be positive");
    if (N != c->N || c->dirty) {
        c->N = N;
        int rc = c->b.plan(c->prm, 1, &c->N, c->L, nullptr);
        if (rc) return rc;
        c->dirty = false;
    }
    return c->b.spread_only((cudaStream_t)stream, pos4, charge, rho);
}

int esp_get_sort(const esp_ctx* c, void* stream, unsigned* key, unsigned* perm) {
    if (!c || !key || !perm) return fail(ESP_ERR_INVALID, "null argument");
    const int N = c->b.totN;
    cudaStream_t st = (cudaStream_t)stream;
    ESPB_CK(cudaMemcpyAsync(key, c->b.d_key, N * sizeof(unsigned), cudaMemcpyDeviceToDevice, st));
    ESPB_CK(cudaMemcpyAsync(perm, c->b.d_perm, N * sizeof(unsigned), cudaMemcpyDeviceToDevice, st));
    return 0;
}

int esp_get_potential(const esp_ctx* c, void* stream, float* phi) {
    if (!c || !phi) return fail(ESP_ERR_INVALID, "null argument");
    const SysDev& S = c->b.sd[0];
    // the interior of the halo-padded mesh, plane by plane
    for (int z = 0; z < S.nz; ++z)
        ESPB_CK(cudaMemcpy2DAsync(phi + (size_t)z * S.ny * S.nx, (size_t)S.nx * sizeof(float),
                                  c->b.d_phi + S.mp_off + (size_t)z * S.nyp * S.nxp, (size_t)S.nxp * sizeof(float),
                                  (size_t)S.nx * sizeof(float), S.ny, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return 0;
}

int esp_batch_create(const esp_params* p, int nsys, const int* N, const double* boxes, const int* mesh,
                     esp_batch** out) {
    if (!p || !N || !boxes || !out) return fail(ESP_ERR_INVALID, "null argument");
    *out = nullptr;
    esp_batch* b = new esp_batch();
    int rc = b->plan(*p, nsys, N, boxes, mesh);
    if (rc) {
        delete b;
        return rc;
    }
    *out = b;
    return 0;
}

int esp_batch_compute(esp_batch* b, void* stream, const float* pos4, const float* charge, const unsigned* head,
                      const unsigned* n_neigh, const unsigned* nlist, float* force4, double* energy, double* virial6,
                      int flags) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    if ((flags & ESP_SHORT_RANGE) && !head && !n_neigh && !nlist && b->pl_ready) {
        int rc = b->pairlist_check(false, nullptr);
        if (rc) return rc;
    }
    if ((flags & ESP_SHORT_RANGE) && head && head == b->nl_last_head && nlist == b->nl_last_nl) {
        int rc = b->nlist_check(false, nullptr);
        if (rc) return rc;
    }
    return b->compute((cudaStream_t)stream, pos4, charge, head, n_neigh, nlist, force4, energy, virial6, flags);
}

int esp_batch_build_pairlist(esp_batch* b, void* stream, const float* pos4, double rlist, int cap) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->build_pairlist((cudaStream_t)stream, pos4, rlist, cap);
}

int esp_batch_device_errors(esp_batch* b, int* flags) {
    if (!b || !flags) return fail(ESP_ERR_INVALID, "null argument");
    ESPB_CK(cudaDeviceSynchronize());
    ESPB_CK(cudaMemcpy(flags, b->d_kerr, sizeof(int), cudaMemcpyDeviceToHost));
    ESPB_CK(cudaMemset(b->d_kerr, 0, sizeof(int)));
    return 0;
}

int esp_batch_pairlist_check(esp_batch* b, int* needed_cap) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->pairlist_check(true, needed_cap);
}

int esp_batch_compute_f64(esp_batch* b, void* stream, const double* pos4, const double* charge, const unsigned* head,
                          const unsigned* n_neigh, const unsigned* nlist, double* force4, double* energy,
                          double* virial6, int flags) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->compute_f64((cudaStream_t)stream, pos4, charge, head, n_neigh, nlist, force4, energy, virial6, flags);
}

int esp_batch_autotune(esp_batch* b, void* stream, const float* pos4, const float* charge, const unsigned* head,
                       const unsigned* n_neigh, const unsigned* nlist, int flags, int reps, esp_params* chosen,
                       double* trial_ms, int max_trials) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->autotune((cudaStream_t)stream, pos4, charge, head, n_neigh, nlist, flags, reps, chosen, trial_ms,
                       max_trials);
}

int esp_batch_get_info(const esp_batch* b, int sys, esp_info* info) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->info(sys, info);
}

int esp_batch_total_particles(const esp_batch* b) { return b ? b->totN : -1; }

int esp_batch_destroy(esp_batch* b) {
    delete b;
    return 0;
}

int esp_batch_set_exclusions(esp_batch* b, const unsigned* n_ex, const unsigned* ex_list, int ex_pitch) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    if (n_ex && (!ex_list || ex_pitch <= 0)) return fail(ESP_ERR_INVALID, "exclusion list needs ex_list and ex_pitch > 0");
    b->ex_n = n_ex;
    b->ex_list = n_ex ? ex_list : nullptr;
    b->ex_pitch = n_ex ? ex_pitch : 0;
    b->drop_graphs();  // captured steps hold the previous pointers
    return 0;
}

int esp_set_exclusions(esp_ctx* c, const unsigned* n_ex, const unsigned* ex_list, int ex_pitch) {
    if (!c) return fail(ESP_ERR_INVALID, "null context");
    return esp_batch_set_exclusions(&c->b, n_ex, ex_list, ex_pitch);
}

int esp_batch_md_run(esp_batch* b, void* stream, float* pos4, float* vel4, const float* charge, const unsigned* head,
                     const unsigned* n_neigh, const unsigned* nlist, float* force4, double* energy, double* virial6,
                     int nsteps, double dt, int use_graph) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->md_run((cudaStream_t)stream, pos4, vel4, charge, head, n_neigh, nlist, force4, energy, virial6, nsteps,
                     dt, use_graph);
}

int esp_batch_md_run_f64(esp_batch* b, void* stream, double* pos4, double* vel4, const double* charge,
                         const unsigned* head, const unsigned* n_neigh, const unsigned* nlist, double* force4,
                         double* energy, double* virial6, int nsteps, double dt, double lj_epsilon, double lj_sigma,
                         double lj_r_cut, int use_graph) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->md_run_f64((cudaStream_t)stream, pos4, vel4, charge, head, n_neigh, nlist, force4, energy, virial6,
                         nsteps, dt, lj_epsilon, lj_sigma, lj_r_cut, use_graph);
}

int esp_batch_set_timing(esp_batch* b, int on) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    b->timer.collect();
    b->timer.reset();
    b->timer.on = on != 0;
    return 0;
}

int esp_batch_stage_times(esp_batch* b, double* ms, long long* counts) {
    if (!b || !ms) return fail(ESP_ERR_INVALID, "null argument");
    b->timer.collect();
    for (int k = 0; k < ESP_N_STAGES; ++k) {
        ms[k] = b->timer.ms[k];
        if (counts) counts[k] = b->timer.count[k];
    }
    b->timer.reset();
    return 0;
}

int esp_pswf_eval_pairs(void* stream, int n, const double* rsq, const double* qiqj, double rcut, int n_segs,
                        const double* screen, const double* dscreen, const double* r_lo, const double* dr_inv,
                        double* force_divr, double* pair_eng, int* evaluated) {
    if (n < 0 || n_segs <= 0) return fail(ESP_ERR_INVALID, "bad sizes");
    if (n > 0 && (!rsq || !qiqj || !screen || !dscreen || !r_lo || !dr_inv || !force_divr || !pair_eng || !evaluated))
        return fail(ESP_ERR_INVALID, "null pointer");
    ESPB_CK(launch_pswf_eval_pairs(n, rsq, qiqj, rcut, n_segs, screen, dscreen, r_lo, dr_inv, force_divr, pair_eng,
                                   evaluated, (cudaStream_t)stream));
    return 0;
}

int esp_batch_build_nlist(esp_batch* b, void* stream, const float* pos4, double rlist, int cap, unsigned* head,
                          unsigned* n_neigh, unsigned* nlist) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->build_nlist((cudaStream_t)stream, pos4, rlist, cap, head, n_neigh, nlist);
}

int esp_batch_nlist_check(esp_batch* b, int* needed_cap) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->nlist_check(true, needed_cap);
}

int esp_batch_nve_step1(esp_batch* b, void* stream, float* pos4, float* vel4, const float* force4, double dt) {
    if (!b || !pos4 || !vel4 || !force4) return fail(ESP_ERR_INVALID, "null argument");
    return b->nve1((cudaStream_t)stream, pos4, vel4, force4, dt, false);
}

int esp_batch_lj(esp_batch* b, void* stream, const float* pos4, const unsigned* head, const unsigned* n_neigh,
                 const unsigned* nlist, double epsilon, double sigma, double r_cut, float* force4, double* energy) {
    if (!b || !pos4 || !head || !n_neigh || !nlist || !force4) return fail(ESP_ERR_INVALID, "null argument");
    if (!(sigma > 0) || !(r_cut > 0)) return fail(ESP_ERR_INVALID, "sigma and r_cut must be positive");
    ESPB_CK(launch_lj(b->d_chunks, b->n_chunks, b->d_sys, pos4, head, n_neigh, nlist, epsilon, sigma, r_cut, force4,
                      energy, false, (cudaStream_t)stream));
    return 0;
}

int esp_batch_lj_f64(esp_batch* b, void* stream, const double* pos4, const unsigned* head, const unsigned* n_neigh,
                     const unsigned* nlist, double epsilon, double sigma, double r_cut, double* force4,
                     double* energy) {
    if (!b || !pos4 || !head || !n_neigh || !nlist || !force4) return fail(ESP_ERR_INVALID, "null argument");
    if (!(sigma > 0) || !(r_cut > 0)) return fail(ESP_ERR_INVALID, "sigma and r_cut must be positive");
    ESPB_CK(launch_lj(b->d_chunks, b->n_chunks, b->d_sys, pos4, head, n_neigh, nlist, epsilon, sigma, r_cut, force4,
                      energy, true, (cudaStream_t)stream));
    return 0;
}

int esp_batch_nve_step1_f64(esp_batch* b, void* stream, double* pos4, double* vel4, const double* force4, double dt) {
    if (!b || !pos4 || !vel4 || !force4) return fail(ESP_ERR_INVALID, "null argument");
    return b->nve1((cudaStream_t)stream, pos4, vel4, force4, dt, true);
}

int esp_batch_nve_step2_f64(esp_batch* b, void* stream, const double* pos4, double* vel4, const double* force4,
                            double dt) {
    if (!b || !vel4 || !force4) return fail(ESP_ERR_INVALID, "null argument");
    if (b->n_mols && !pos4) return fail(ESP_ERR_INVALID, "rigid molecules need the positions");
    return b->nve2((cudaStream_t)stream, pos4, vel4, force4, dt, true);
}

int esp_batch_nve_step2(esp_batch* b, void* stream, const float* pos4, float* vel4, const float* force4, double dt) {
    if (!b || !vel4 || !force4) return fail(ESP_ERR_INVALID, "null argument");
    if (b->n_mols && !pos4) return fail(ESP_ERR_INVALID, "rigid molecules need the positions");
    return b->nve2((cudaStream_t)stream, pos4, vel4, force4, dt, false);
}

int esp_batch_set_rigid_water(esp_batch* b, const int* first, const int* count, double d_oh, double d_hh) {
    if (!b) return fail(ESP_ERR_INVALID, "null batch");
    return b->set_rigid(first, count, d_oh, d_hh);
}

}  // extern "C"

// ============================================================================
// No-allocation spreading (esp_spread_noalloc).
//
// For callers that cannot allocate device memory (an engine whose pool
// allocator owns all of the device memory, or a step that must not call
// cudaFree because it synchronises the device): bin + sort + spreading of
// one system with every work array carved out of one file-scope scratch
// array of fixed size. The kernels are the ones esp_spread launches; only
// where their work arrays live differs.
// ============================================================================
#include <mutex>

namespace {

constexpr int NA_MAX_N = ESP_SPREAD_NOALLOC_MAX_N;
constexpr int NA_MAX_TILES = ESP_SPREAD_NOALLOC_MAX_TILES;
static_assert(NA_MAX_N % 256 == 0, "particle limit must be a whole number of 256-particle chunks");
constexpr size_t na_round(size_t b) { return (b + 255) & ~(size_t)255; }

// Byte offsets of the work arrays inside the scratch array (256-byte aligned).
constexpr size_t NA_SYS = 0;
constexpr size_t NA_PSET = NA_SYS + na_round(sizeof(SysDev));
constexpr size_t NA_CHUNKS = NA_PSET + na_round(sizeof(ParamSet));
constexpr size_t NA_TILE_SYS = NA_CHUNKS + na_round(sizeof(int2) * (NA_MAX_N / 256));
constexpr size_t NA_TCOUNT = NA_TILE_SYS + na_round(sizeof(int) * NA_MAX_TILES);
constexpr size_t NA_TSTART = NA_TCOUNT + na_round(sizeof(uint32_t) * NA_MAX_TILES);
constexpr size_t NA_ACC = NA_TSTART + na_round(sizeof(uint32_t) * (NA_MAX_TILES + 1));
constexpr size_t NA_POSQ = NA_ACC + na_round(sizeof(double) * ACC_STRIDE);
constexpr size_t NA_TREC = NA_POSQ + sizeof(float4) * NA_MAX_N;
constexpr size_t NA_SREC = NA_TREC + sizeof(float4) * NA_MAX_N;
constexpr size_t NA_REL = NA_SREC + sizeof(float4) * NA_MAX_N;
constexpr size_t NA_SREL = NA_REL + sizeof(uint32_t) * NA_MAX_N;
constexpr size_t NA_KEY = NA_SREL + sizeof(uint32_t) * NA_MAX_N;
constexpr size_t NA_PERM_U = NA_KEY + sizeof(uint32_t) * NA_MAX_N;
constexpr size_t NA_PERM = NA_PERM_U + sizeof(uint32_t) * NA_MAX_N;
constexpr size_t NA_BYTES = NA_PERM + sizeof(uint32_t) * NA_MAX_N;  // 2,280,448 bytes
static_assert(NA_BYTES <= (size_t)3 << 20, "scratch must stay a few MB");

// The scratch itself. In host code this name is only a handle for
// cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) unsigned char g_na_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
unsigned char* g_na_base[NA_MAX_DEVICES] = {};
void* g_na_ctx[NA_MAX_DEVICES] = {};

// The driver context current on this thread (cuCtxGetCurrent through the
// runtime's driver entry point, so the library needs no link to libcuda).
void* na_current_context() {
    typedef int (*GetCurrent)(void**);
    static GetCurrent fn = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<GetCurrent>(f);
        looked_up = true;
    }
    void* ctx = nullptr;
    if (fn) fn(&ctx);
    return ctx;
}

// Set-up per device, with that device current: the scratch array's device
// address and the spreading kernels' shared-memory limits. Done on the first
// call on a device, and again when the device's context has changed since
// (after cudaDeviceReset the old address is no longer valid).
int na_setup(unsigned char** base) {
    int dev = 0;
    ESPB_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) return fail(ESP_ERR_UNSUPPORTED, "device index above 63");
    ESPB_CK(cudaSetDevice(dev));  // makes the device's primary context current
    void* ctx = na_current_context();
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_base[dev] || g_na_ctx[dev] != ctx) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_na_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(ESP_ERR_CUDA, std::string("cudaGetSymbolAddress of the spreading scratch: ") +
                                          cudaGetErrorString(e));
        for (int P = 2; P <= MAX_P; ++P) {
            LaunchArgs a;
            a.configure_only = 1;
            a.P = P;
            a.T = 17 - P;  // extended region of 16: the tensor-core and dense kernels
            ESPB_CK(launch_spread(a, 0));
        }
        g_na_base[dev] = static_cast<unsigned char*>(ptr);
        g_na_ctx[dev] = ctx;
    }
    *base = g_na_base[dev];
    return 0;
}

// Window coefficients per (P, c_w, D), built once on the host.
int na_param_set(int P, double cw, int D, ParamSet* out) {
    static std::mutex mu;
    static std::map<std::tuple<int, double, int>, ParamSet> cache;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(P, cw, D);
    auto it = cache.find(key);
    if (it == cache.end()) {
        Window win;
        try {
            win.build(P, cw, D);
        } catch (const std::exception& ex) {
            return fail(ESP_ERR_INVALID, ex.what());
        }
        ParamSet d{};
        for (int a = 0; a < P; ++a)
            for (int j = 0; j <= D; ++j) d.wcoef[a * (MAX_D + 1) + j] = (float)win.coef[(size_t)a * (D + 1) + j];
        it = cache.emplace(key, d).first;
    }
    *out = it->second;
    return 0;
}

// Writes the system descriptor, window coefficients and work lists into the
// scratch, and clears what the bin kernel accumulates into (tile counts and
// the charge sums): the scratch keeps the previous call's contents.
__global__ void k_na_prepare(SysDev S, ParamSet ps, SysDev* sys, ParamSet* pset, int2* chunks, int n_chunks,
                             int* tile_sys, uint32_t* tile_count, int n_tiles, double* acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        *sys = S;
        *pset = ps;
    }
    if (i < n_chunks) chunks[i] = make_int2(0, 256 * i);
    if (i < n_tiles) {
        tile_sys[i] = 0;
        tile_count[i] = 0u;
    }
    if (i < ACC_STRIDE) acc[i] = 0.0;
}

}  // namespace

extern "C" int esp_spread_noalloc(void* stream, const esp_params* p, double Lx, double Ly, double Lz,
                                  const float* pos4, const float* charge, int N, double* rho) {
    if (!p || !pos4 || !charge || !rho) return fail(ESP_ERR_INVALID, "null argument");
    if (N <= 0) return fail(ESP_ERR_INVALID, "particle count must be positive");
    if (N > NA_MAX_N)
        return fail(ESP_ERR_UNSUPPORTED, "esp_spread_noalloc: N = " + std::to_string(N) +
                                             " exceeds its fixed scratch limit of " + std::to_string(NA_MAX_N) +
                                             " particles (esp_spread has no such limit)");
    const int P = p->order;
    if (P < 2 || P > MAX_P) return fail(ESP_ERR_UNSUPPORTED, "order must be in [2, 12]");
    if (p->precision != ESP_FP32 && p->precision != ESP_FP64)
        return fail(ESP_ERR_INVALID, "precision must be ESP_FP32 or ESP_FP64");
    const double L[3] = {Lx, Ly, Lz};
    const int n[3] = {p->nx, p->ny, p->nz};
    int T = p->tile > 0 ? p->tile : 17 - P;
    for (int d = 0; d < 3; ++d) {
        if (!(L[d] > 0)) return fail(ESP_ERR_INVALID, "box lengths must be positive");
        if (n[d] <= 0) return fail(ESP_ERR_INVALID, "esp_spread_noalloc needs an explicit mesh (nx, ny, nz > 0)");
        if (n[d] < std::max(P, 4) || n[d] > FFT_MAX_N)
            return fail(ESP_ERR_UNSUPPORTED, "mesh size " + std::to_string(n[d]) + " must be in [max(order, 4), 256]");
        T = std::min(T, n[d]);
    }
    if (T + P - 1 > 16) return fail(ESP_ERR_UNSUPPORTED, "esp_spread_noalloc needs tile + order - 1 <= 16");
    const int nt[3] = {(n[0] + T - 1) / T, (n[1] + T - 1) / T, (n[2] + T - 1) / T};
    const long long n_tiles = (long long)nt[0] * nt[1] * nt[2];
    if (n_tiles > NA_MAX_TILES)
        return fail(ESP_ERR_UNSUPPORTED, "esp_spread_noalloc: " + std::to_string(n_tiles) +
                                             " tiles exceed its fixed scratch limit of " +
                                             std::to_string(NA_MAX_TILES));
    // the window of esp_create for the same parameters (FP64 contexts fit it
    // to a higher degree); the spreading itself runs the FP32 kernels
    const int D = p->window_degree > 0 ? p->window_degree
                                       : (p->precision == ESP_FP64 ? std::max(P + 2, 9) : default_window_degree(P));
    if (D > MAX_D) return fail(ESP_ERR_UNSUPPORTED, "window degree must be <= 15");
    if (p->window_c < 0) return fail(ESP_ERR_INVALID, "window_c must be >= 0");
    const double cw = p->window_c > 0 ? p->window_c : 2.2 * P;

    ParamSet ps;
    int rc = na_param_set(P, cw, D, &ps);
    if (rc) return rc;
    SysDev S{};
    S.N = N;
    S.nx = n[0];
    S.ny = n[1];
    S.nz = n[2];
    S.nxh = n[0] / 2 + 1;
    S.ntx = nt[0];
    S.nty = nt[1];
    S.ntz = nt[2];
    S.Lx = (float)Lx;
    S.Ly = (float)Ly;
    S.Lz = (float)Lz;
    S.inv_Lx = 1.0f / S.Lx;
    S.inv_Ly = 1.0f / S.Ly;
    S.inv_Lz = 1.0f / S.Lz;
    S.gxd = n[0] / Lx;
    S.gyd = n[1] / Ly;
    S.gzd = n[2] / Lz;
    S.Lxd = Lx;
    S.Lyd = Ly;
    S.Lzd = Lz;
    S.V = Lx * Ly * Lz;

    unsigned char* base = nullptr;
    if ((rc = na_setup(&base))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int n_chunks = (N + 255) / 256;
    LaunchArgs a;
    a.sys = reinterpret_cast<SysDev*>(base + NA_SYS);
    a.psets = reinterpret_cast<ParamSet*>(base + NA_PSET);
    a.nsys = 1;
    a.P = P;
    a.T = T;
    a.D = D;
    a.chunks = reinterpret_cast<int2*>(base + NA_CHUNKS);
    a.n_chunks = n_chunks;
    a.tile_sys = reinterpret_cast<int*>(base + NA_TILE_SYS);
    a.n_tiles = (int)n_tiles;
    a.tile_count = reinterpret_cast<uint32_t*>(base + NA_TCOUNT);
    a.tile_start = reinterpret_cast<uint32_t*>(base + NA_TSTART);
    a.acc = reinterpret_cast<double*>(base + NA_ACC);
    a.posq = reinterpret_cast<float4*>(base + NA_POSQ);
    a.trec = reinterpret_cast<float4*>(base + NA_TREC);
    a.srec = reinterpret_cast<float4*>(base + NA_SREC);
    a.rel = reinterpret_cast<uint32_t*>(base + NA_REL);
    a.srel = reinterpret_cast<uint32_t*>(base + NA_SREL);
    a.key = reinterpret_cast<uint32_t*>(base + NA_KEY);
    a.perm_u = reinterpret_cast<uint32_t*>(base + NA_PERM_U);
    a.perm = reinterpret_cast<uint32_t*>(base + NA_PERM);
    a.pos_in = reinterpret_cast<const float4*>(pos4);
    a.q_in = charge;
    a.rho = rho;

    const int n_prep = std::max(std::max(n_chunks, (int)n_tiles), (int)ACC_STRIDE);
    ESPB_CK(cudaMemsetAsync(rho, 0, (size_t)n[0] * n[1] * n[2] * sizeof(double), st));
    k_na_prepare<<<(n_prep + 255) / 256, 256, 0, st>>>(S, ps, const_cast<SysDev*>(a.sys),
                                                       const_cast<ParamSet*>(a.psets), const_cast<int2*>(a.chunks),
                                                       n_chunks, const_cast<int*>(a.tile_sys), a.tile_count,
                                                       (int)n_tiles, a.acc);
    ESPB_CK(cudaGetLastError());
    ESPB_CK(launch_bin(a, st));
    ESPB_CK(launch_sort(a, st));
    ESPB_CK(launch_spread(a, st));
    return 0;
}
