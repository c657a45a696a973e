// Continuous-batching request server (esp_server_*, include/esp_b200.h).
//
// Every request is one independent system (rock-salt lattice, water box, ...)
// that needs a neighbour list, one evaluation and a few NVE steps. The
// server keeps one set of device arenas, allocated once from the HBM budget:
// particle arrays (positions, velocities, forces, charges, bin records,
// sorted records, neighbour-list heads), mesh arrays (charge mesh,
// potential, half spectrum), influence tables, tile counters and one
// neighbour-list pool. An admitted request owns ranges of these arenas (its
// footprint) and a slot in the system-descriptor table, so the batched
// kernels of the batch path serve it unchanged: a round launches each stage
// once over the work lists of all admitted systems. Requests that arrive
// while others run are admitted at the next round boundary, in arrival
// order, while their ranges fit; finished requests release their ranges in
// stream order.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include <cuda.h>

#include "esp_b200.h"
#include "esp_host_util.h"
#include "esp_kernels.h"
#include "esp_md.h"
#include "esp_tables.h"

namespace espb {
namespace {

__global__ void k_fill_int(int* __restrict__ p, int n, int v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// First-fit allocator of [0, cap) in units; aligned offsets and lengths.
struct RangeAlloc {
    long long cap = 0;
    std::map<long long, long long> free_;  // start -> length
    std::map<long long, long long> used_;  // start -> length
    void init(long long c) {
        cap = c;
        free_.clear();
        used_.clear();
        if (c > 0) free_[0] = c;
    }
    long long alloc(long long n, long long align) {
        n = (n + align - 1) / align * align;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            const long long fs = it->first, fl = it->second;
            const long long s = (fs + align - 1) / align * align;
            if (s + n > fs + fl) continue;
            free_.erase(it);
            if (s > fs) free_[fs] = s - fs;
            if (s + n < fs + fl) free_[s + n] = fs + fl - (s + n);
            used_[s] = n;
            return s;
        }
        return -1;
    }
    void release(long long s) {
        auto u = used_.find(s);
        if (u == used_.end()) return;
        long long n = u->second;
        used_.erase(u);
        auto nx = free_.lower_bound(s);
        if (nx != free_.end() && nx->first == s + n) {
            n += nx->second;
            free_.erase(nx);
        }
        auto pv = free_.lower_bound(s);
        if (pv != free_.begin()) {
            --pv;
            if (pv->first + pv->second == s) {
                pv->second += n;
                return;
            }
        }
        free_[s] = n;
    }
    long long high() const { return used_.empty() ? 0 : used_.rbegin()->first + used_.rbegin()->second; }
};

// Page-locked staging of one round's host-to-device uploads.
struct Staging {
    char* buf = nullptr;
    size_t cap = 0, used = 0;
    cudaEvent_t ev = nullptr;  // recorded after the last copy out of buf
    bool pending = false;
    ~Staging() {
        if (buf) cudaFreeHost(buf);
        if (ev) cudaEventDestroy(ev);
    }
};

// Bytes per particle of the particle arena: pos, vel, force, posq, trec,
// wpos, srec (float4) and charge, rel, key, perm_u, head, n_neigh, ckey,
// srel, perm (4 bytes).
constexpr long long PARTICLE_BYTES = 7 * 16 + 9 * 4;
constexpr long long MESH_BYTES = 8 + 4 + 8;  // rho (double), phi (float), half spectrum (float2)
constexpr int MAX_CELLS_AXIS = 40;
constexpr int MAX_PSETS = 16;

struct Request {
    esp_request r{};
    long long id = 0;
    int state = 0;
    double t_arrival = 0, t_admit = -1, t_done = -1;
    int slot = -1;
    long long p_off = -1, m_off = -1, t_off = -1, nl_off = -1;
    int mesh[3] = {0, 0, 0};
    int ntile[3] = {0, 0, 0};
    int cap = 0, pset = 0;
    int geo = -1;  // rigid water: index into the geometry table, else -1
    int steps_done = 0;
    bool evaluated = false;
    long long footprint = 0;
    std::tuple<int, double, double, double, int, int, int> gkey;
};

struct GEntry {
    long long off = 0, len = 0;
    int refs = 0;
    long long last_use = 0;
};

struct Round {
    cudaEvent_t ev = nullptr;
    std::vector<Request*> fin;
    int* ovf = nullptr;  // page-locked, one flag per finishing request
};

}  // namespace
}  // namespace espb

using namespace espb;

struct esp_server {
    // configuration
    esp_params prm{};
    int P = 8, T = 9, D = 10, tpp = 8, PX = 0, PP = 0;
    int max_slots = 0, max_particles = 0;
    double c_split = 0, c_win = 0, kreq = 0;
    int dev = 0;
    cudaStream_t st = nullptr;

    // parameter sets (one per distinct cutoff, all with the same split c)
    std::vector<double> pset_rcut;
    std::vector<PsetHost> psh;
    std::vector<ParamSet> psd;
    PairCoef pc{};
    int nq = 0;

    // twiddles for every 2/3/5-smooth length <= FFT_MAX_N
    std::vector<int> tw_off;

    // arenas
    DevAlloc mem;
    long long P_cap = 0, M_cap = 0, G_cap = 0, T_cap = 0, NL_cap = 0, C_cap = 0;
    RangeAlloc palloc, malloc_, galloc, talloc, nlalloc;
    std::vector<int> free_slots;
    SysDev* d_sys = nullptr;
    ParamSet* d_pset = nullptr;
    CellDev* d_cells = nullptr;
    int* d_cell_sys = nullptr;
    float4 *d_pos = nullptr, *d_vel = nullptr, *d_force = nullptr, *d_posq = nullptr, *d_trec = nullptr,
           *d_srec = nullptr, *d_wpos = nullptr, *d_cpos = nullptr;
    float* d_q = nullptr;
    uint32_t *d_rel = nullptr, *d_key = nullptr, *d_perm_u = nullptr, *d_perm = nullptr, *d_srel = nullptr,
             *d_head = nullptr, *d_nn = nullptr, *d_ckey = nullptr, *d_cperm = nullptr,
             *d_ccount = nullptr, *d_cstart = nullptr, *d_nl = nullptr;
    int* d_tile_sys = nullptr;
    uint32_t *d_tcount = nullptr, *d_tstart = nullptr;
    double* d_rho = nullptr;
    float* d_phi = nullptr;
    float2 *d_spec = nullptr, *d_gtab = nullptr, *d_tw = nullptr;
    double *d_acc = nullptr, *d_energy = nullptr, *d_infl = nullptr;
    int* d_ovf = nullptr;  // per slot: [overflow flag, longest row] of its neighbour-list build
    int2 *d_chunks = nullptr, *d_pchunks = nullptr, *d_mdchunks = nullptr, *d_nlchunks = nullptr;
    int2 *d_pitems = nullptr, *d_sitems = nullptr;
    int4 *d_xitems = nullptr, *d_yitems = nullptr, *d_zitems = nullptr;
    // rigid water (SETTLE): per-slot atom range the plain integrator skips,
    // per-round work items, and the (d_OH, d_HH) geometries seen so far
    int2* d_rskip = nullptr;
    int4* d_ritems = nullptr;
    // TMA-staged interpolation: one tensor map per slot (its halo-padded
    // potential range), the box, the kernels' error word
    CUtensorMap* d_tmaps = nullptr;
    bool use_tma = false;
    int tma_bx = 0, tma_by = 0;
    int* d_kerr = nullptr;  // [kernel error word, tile-queue counter]
    double2* d_geo = nullptr;
    std::vector<double2> geos;
    static constexpr int MAX_GEOS = 16;
    long long ritem_cap = 0;
    long long chunk_cap = 0, pchunk_cap = 0;
    static constexpr long long ITEM_CAP = 1 << 20;

    // influence-table cache
    std::map<std::tuple<int, double, double, double, int, int, int>, GEntry> gcache;
    long long gclock = 0;

    // requests and scheduling
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::vector<std::unique_ptr<Request>> reqs;
    std::deque<Request*> pending;
    std::vector<Request*> active;
    std::deque<Round> inflight;
    std::vector<cudaEvent_t> ev_pool;
    Staging stage[2];
    int stage_idx = 0;
    bool started = false, stop = false;
    std::chrono::steady_clock::time_point t0;
    std::thread worker;
    std::atomic<int> error_code{0};
    std::string error_msg;
    esp_server_stats stats{};  // guarded by mu
    std::atomic<long long> n_rounds{0}, n_builds{0}, n_hits{0};
    long long bytes_active = 0;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    int init(const esp_server_config& cfg);
    void run();
    int admit(Request* q, Staging& sg);
    int launch_round(Staging& sg);
    void retire(bool block);
    void release(Request* q);
    void fail_all(int code);
    int upload(Staging& sg, void* dst, const void* src, size_t bytes);
    cudaEvent_t get_event();
    int influence(Request* q, const SysDev& S, Staging& sg);
};

// ---------------------------------------------------------------------------
// set-up
// ---------------------------------------------------------------------------
int esp_server::init(const esp_server_config& cfg) {
    prm = cfg.params;
    P = prm.order;
    if (P < 2 || P > MAX_P) return fail(ESP_ERR_UNSUPPORTED, "order must be in [2, 12]");
    if (prm.alpha != 0.0) return fail(ESP_ERR_UNSUPPORTED, "Debye screening (alpha != 0) is not supported");
    if (cfg.max_systems < 1 || cfg.max_systems > 4096) return fail(ESP_ERR_INVALID, "max_systems must be in [1, 4096]");
    if (cfg.max_particles < 1) return fail(ESP_ERR_INVALID, "max_particles must be positive");
    if (cfg.hbm_budget < (256LL << 20)) return fail(ESP_ERR_INVALID, "hbm_budget must be at least 256 MB");
    max_slots = cfg.max_systems;
    max_particles = cfg.max_particles;
    tpp = prm.threads_per_particle ? prm.threads_per_particle : 4;
    if (tpp != 4 && tpp != 8 && tpp != 16 && tpp != 32)
        return fail(ESP_ERR_UNSUPPORTED, "threads_per_particle must be 4, 8, 16 or 32");
    T = prm.tile > 0 ? prm.tile : std::max(1, 17 - P);
    if (T > 64) return fail(ESP_ERR_UNSUPPORTED, "tile edge must be <= 64");
    D = prm.window_degree > 0 ? prm.window_degree : default_window_degree(P);
    if (D > MAX_D) return fail(ESP_ERR_UNSUPPORTED, "window degree must be <= 15");
    kreq = kappa_required(prm.target_error > 0 ? prm.target_error : 1e-5);
    // the split bandwidth of a system meshed at exactly h = pi r_c / kappa_N;
    // it does not depend on r_c, so every request shares one split
    c_split = split_c_for_spacing(1.0, M_PI / kreq);
    c_win = prm.window_c > 0 ? prm.window_c : 2.2 * P;
    choose_pitch(P, T + P - 1, PX, PP);
    ESPB_CK(cudaGetDevice(&dev));
    ESPB_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));

    // arena capacities from the budget (the neighbour-list pool is indexed
    // by 32-bit row offsets)
    const double B = (double)cfg.hbm_budget;
    P_cap = std::max<long long>(2LL * max_particles, (long long)(0.10 * B / PARTICLE_BYTES));
    P_cap = std::min<long long>(P_cap, 1LL << 30);
    M_cap = (long long)(0.22 * B / MESH_BYTES);
    G_cap = (long long)(0.08 * B / 8);
    NL_cap = std::min<long long>((long long)(0.58 * B / 4), (1LL << 32) - 1024);
    T_cap = std::max<long long>(4096, M_cap / 512);
    C_cap = (long long)MAX_CELLS_AXIS * MAX_CELLS_AXIS * MAX_CELLS_AXIS;
    palloc.init(P_cap);
    malloc_.init(M_cap);
    galloc.init(G_cap);
    talloc.init(T_cap);
    nlalloc.init(NL_cap);
    for (int s = max_slots - 1; s >= 0; --s) free_slots.push_back(s);

    // twiddles
    std::vector<float2> tw;
    tw_off.assign(FFT_MAX_N + 1, -1);
    for (int n = 2; n <= FFT_MAX_N; ++n) {
        if (radix_plan(n) == 0) continue;
        tw_off[n] = (int)tw.size();
        for (int t = 0; t < n; ++t) {
            const double a = -2.0 * M_PI * t / n;
            tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        }
    }
    chunk_cap = P_cap / 256 + max_slots + 16;
    pchunk_cap = P_cap / 8 + max_slots + 16;  // 256 / tpp >= 8 particles per chunk
    ritem_cap = P_cap / (3 * SETTLE_CHUNK) + max_slots + 16;
    int rc = 0;
    if ((rc = mem.get(d_sys, max_slots)) || (rc = mem.get(d_pset, MAX_PSETS)) || (rc = mem.get(d_cells, max_slots)) ||
        (rc = mem.get(d_cell_sys, C_cap)) || (rc = mem.get(d_pos, P_cap)) || (rc = mem.get(d_vel, P_cap)) ||
        (rc = mem.get(d_force, P_cap)) || (rc = mem.get(d_posq, P_cap)) || (rc = mem.get(d_trec, P_cap)) ||
        (rc = mem.get(d_srec, P_cap)) || (rc = mem.get(d_wpos, P_cap)) || (rc = mem.get(d_q, P_cap)) ||
        (rc = mem.get(d_rel, P_cap)) || (rc = mem.get(d_key, P_cap)) || (rc = mem.get(d_perm_u, P_cap)) ||
        (rc = mem.get(d_perm, P_cap)) || (rc = mem.get(d_srel, P_cap)) || (rc = mem.get(d_head, P_cap)) ||
        (rc = mem.get(d_nn, P_cap)) || (rc = mem.get(d_ckey, P_cap)) || (rc = mem.get(d_cperm, max_particles)) ||
        (rc = mem.get(d_cpos, max_particles)) ||
        (rc = mem.get(d_ccount, C_cap)) || (rc = mem.get(d_cstart, C_cap + 1)) || (rc = mem.get(d_nl, NL_cap)) ||
        (rc = mem.get(d_tile_sys, T_cap)) || (rc = mem.get(d_tcount, T_cap)) || (rc = mem.get(d_tstart, T_cap + 1)) ||
        (rc = mem.get(d_rho, M_cap)) || (rc = mem.get(d_phi, M_cap)) || (rc = mem.get(d_spec, M_cap)) ||
        (rc = mem.get(d_gtab, G_cap)) || (rc = mem.get(d_tw, tw.size())) ||
        (rc = mem.get(d_acc, (size_t)max_slots * ACC_STRIDE)) || (rc = mem.get(d_energy, max_slots)) ||
        (rc = mem.get(d_infl, 3 * FFT_MAX_N + 2 * 320)) || (rc = mem.get(d_ovf, 2 * max_slots)) ||
        (rc = mem.get(d_chunks, chunk_cap)) || (rc = mem.get(d_pchunks, pchunk_cap)) ||
        (rc = mem.get(d_mdchunks, chunk_cap)) || (rc = mem.get(d_nlchunks, (max_particles + 255) / 256)) ||
        (rc = mem.get(d_pitems, ITEM_CAP)) || (rc = mem.get(d_sitems, ITEM_CAP)) || (rc = mem.get(d_xitems, ITEM_CAP)) ||
        (rc = mem.get(d_yitems, ITEM_CAP)) || (rc = mem.get(d_zitems, ITEM_CAP)) ||
        (rc = mem.get(d_rskip, max_slots)) || (rc = mem.get(d_ritems, ritem_cap)) || (rc = mem.get(d_geo, MAX_GEOS)) ||
        (rc = mem.get(d_tmaps, max_slots)) || (rc = mem.get(d_kerr, 2)))
        return rc;
    ESPB_CK(cudaMemset(d_kerr, 0, 2 * sizeof(int)));
    interp_box(T + P - 1, tma_bx, tma_by);
    use_tma = (prm.interp_mode == 0 || prm.interp_mode == 2) && P >= 5 && P <= 8;
    stats.arena_bytes = mem.bytes;
    ESPB_CK(cudaMemcpy(d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
    // counters that the kernels leave at zero, and meshes the inverse FFT pass
    // leaves cleared
    ESPB_CK(cudaMemset(d_tcount, 0, T_cap * sizeof(uint32_t)));
    ESPB_CK(cudaMemset(d_ccount, 0, C_cap * sizeof(uint32_t)));
    ESPB_CK(cudaMemset(d_rho, 0, M_cap * sizeof(double)));
    ESPB_CK(cudaMemset(d_tile_sys, 0, T_cap * sizeof(int)));
    {
        std::vector<SysDev> idle(max_slots);
        for (SysDev& S : idle) S.V = 1.0;
        ESPB_CK(cudaMemcpy(d_sys, idle.data(), max_slots * sizeof(SysDev), cudaMemcpyHostToDevice));
    }
    {
        LaunchArgs a;
        a.configure_only = 1;
        a.P = P;
        a.T = T;
        a.D = D;
        a.PX = PX;
        a.PP = PP;
        a.tma_bx = tma_bx;
        a.tma_by = tma_by;
        ESPB_CK(launch_spread(a, 0));
        ESPB_CK(launch_interp(a, 0));
        ESPB_CK(launch_fft(a, 0));
    }
    for (Staging& s : stage) {
        s.cap = 8 << 20;
        ESPB_CK(cudaHostAlloc((void**)&s.buf, s.cap, cudaHostAllocDefault));
        ESPB_CK(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
    }
    ESPB_CK(cudaDeviceSynchronize());
    t0 = std::chrono::steady_clock::now();
    worker = std::thread([this] { run(); });
    return 0;
}

cudaEvent_t esp_server::get_event() {
    if (!ev_pool.empty()) {
        cudaEvent_t e = ev_pool.back();
        ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
}

int esp_server::upload(Staging& sg, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return 0;
    const size_t need = (sg.used + bytes + 255) & ~(size_t)255;
    if (need > sg.cap) {
        // grow: wait until every copy out of the old buffer has run
        ESPB_CK(cudaStreamSynchronize(st));
        size_t cap = sg.cap;
        while (cap < need) cap *= 2;
        char* nb = nullptr;
        ESPB_CK(cudaHostAlloc((void**)&nb, cap, cudaHostAllocDefault));
        cudaFreeHost(sg.buf);
        sg.buf = nb;
        sg.cap = cap;
        sg.used = 0;
    }
    char* p = sg.buf + sg.used;
    std::memcpy(p, src, bytes);
    sg.used = (sg.used + bytes + 255) & ~(size_t)255;
    sg.pending = true;
    ESPB_CK(cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, st));
    return 0;
}

// ---------------------------------------------------------------------------
// admission
// ---------------------------------------------------------------------------
int esp_server::influence(Request* q, const SysDev& S, Staging& sg) {
    std::vector<double> w1d, tq, wq;
    influence_inputs(S, psh[q->pset], q->r.Lx, q->r.Ly, q->r.Lz, pset_rcut[q->pset], w1d, tq, wq);
    std::vector<double> buf(3 * FFT_MAX_N + 2 * 320, 0.0);
    std::copy(w1d.begin(), w1d.end(), buf.begin());
    std::copy(tq.begin(), tq.end(), buf.begin() + 3 * FFT_MAX_N);
    std::copy(wq.begin(), wq.end(), buf.begin() + 3 * FFT_MAX_N + 320);
    int rc = upload(sg, d_infl, buf.data(), buf.size() * sizeof(double));
    if (rc) return rc;
    ESPB_CK(launch_influence(S, d_infl, d_infl + 3 * FFT_MAX_N, d_infl + 3 * FFT_MAX_N + 320, (int)tq.size(),
                             pset_rcut[q->pset], 1e-14, d_gtab, st));
    return 0;
}

// Returns 0 when admitted, 1 when the request must wait for memory, or a
// negative ESP_ERR code when it can never run.
int esp_server::admit(Request* q, Staging& sg) {
    const esp_request& r = q->r;
    // parameter set of this cutoff
    int ps = -1;
    for (size_t i = 0; i < pset_rcut.size(); ++i)
        if (pset_rcut[i] == r.rcut) ps = (int)i;
    if (ps < 0) {
        if ((int)pset_rcut.size() >= MAX_PSETS) return fail(ESP_ERR_UNSUPPORTED, "more than 16 distinct cutoffs");
        PsetHost h;
        ParamSet d;
        int rc = build_param_set(c_split, c_win, P, D, r.rcut, h, d, 3e-8);
        if (rc) return rc;
        ps = (int)pset_rcut.size();
        pset_rcut.push_back(r.rcut);
        psh.push_back(std::move(h));
        psd.push_back(d);
        if (ps == 0) {
            nq = d.nq;
            for (int c = 0; c < MAX_QC; ++c) {
                pc.q[c] = c < d.nq ? d.qv[c] : 0.f;
                pc.d[c] = c < d.nq - 1 ? d.dqv[c] : 0.f;
            }
        }
        rc = upload(sg, d_pset + ps, &psd[ps], sizeof(ParamSet));
        if (rc) return rc;
    }
    q->pset = ps;
    // mesh, tiles and footprint
    const double L[3] = {r.Lx, r.Ly, r.Lz};
    const double h = M_PI * r.rcut / kreq;
    long long M = 1, ntiles = 1;
    for (int d = 0; d < 3; ++d) {
        const int n = smooth235(std::max(P, (int)std::ceil(L[d] / h)));
        if (n > FFT_MAX_N || radix_plan(n) == 0) return fail(ESP_ERR_UNSUPPORTED, "request mesh above 256 per axis");
        if (n < T) return fail(ESP_ERR_UNSUPPORTED, "request mesh smaller than the tile edge");
        q->mesh[d] = n;
        q->ntile[d] = (n + T - 1) / T;
        M *= n;
        ntiles *= q->ntile[d];
    }
    const long long G = (long long)q->mesh[2] * q->mesh[1] * (q->mesh[0] / 2 + 1);
    // mesh arena units: the halo-padded potential mesh is the largest of the
    // three arrays sharing the range (charge mesh, potential, half spectrum)
    const long long Mp = std::max(M, (long long)halo_extent(q->mesh[0], T, P, true) * halo_extent(q->mesh[1], T, P, false) *
                                         halo_extent(q->mesh[2], T, P, false));
    const double rlist = r.rcut + r.skin;
    int cap = r.nlist_cap;
    if (cap <= 0) {
        const double dens = r.N / (r.Lx * r.Ly * r.Lz);
        cap = (int)std::ceil(1.6 * 4.18879 * rlist * rlist * rlist * dens) + 32;
    }
    cap = (cap + 3) & ~3;
    q->cap = cap;
    const long long NL = (long long)r.N * cap;
    if (r.N > P_cap / 2 || Mp > M_cap || ntiles > T_cap || NL > NL_cap || G > G_cap)
        return fail(ESP_ERR_UNSUPPORTED, "request larger than the server arenas");
    if (free_slots.empty()) return 1;
    // influence table: shared with earlier requests of the same box and mesh
    q->gkey = std::make_tuple(ps, r.Lx, r.Ly, r.Lz, q->mesh[0], q->mesh[1], q->mesh[2]);
    auto git = gcache.find(q->gkey);
    bool build_g = false;
    if (git == gcache.end()) {
        long long off = galloc.alloc(G, 64);
        while (off < 0) {
            // evict the least recently used unreferenced table
            auto victim = gcache.end();
            for (auto it = gcache.begin(); it != gcache.end(); ++it)
                if (it->second.refs == 0 && (victim == gcache.end() || it->second.last_use < victim->second.last_use))
                    victim = it;
            if (victim == gcache.end()) break;
            galloc.release(victim->second.off);
            gcache.erase(victim);
            off = galloc.alloc(G, 64);
        }
        if (off < 0) return 1;
        GEntry e;
        e.off = off;
        e.len = G;
        git = gcache.emplace(q->gkey, e).first;
        build_g = true;
    }
    q->p_off = palloc.alloc(r.N, 256);
    q->m_off = q->p_off >= 0 ? malloc_.alloc(Mp, 64) : -1;
    q->t_off = q->m_off >= 0 ? talloc.alloc(ntiles, 1) : -1;
    q->nl_off = q->t_off >= 0 ? nlalloc.alloc(NL, 64) : -1;
    if (q->nl_off < 0) {
        if (q->p_off >= 0) palloc.release(q->p_off);
        if (q->m_off >= 0) malloc_.release(q->m_off);
        if (q->t_off >= 0) talloc.release(q->t_off);
        q->p_off = q->m_off = q->t_off = q->nl_off = -1;
        if (build_g) {
            galloc.release(git->second.off);
            gcache.erase(git);
        }
        return 1;
    }
    git->second.refs++;
    git->second.last_use = ++gclock;
    q->slot = free_slots.back();
    free_slots.pop_back();
    q->footprint = (long long)r.N * PARTICLE_BYTES + Mp * MESH_BYTES + ntiles * 12 + NL * 4 + (build_g ? G * 8 : 0);

    // system descriptor
    SysDev S{};
    S.N = r.N;
    S.p_off = (int)q->p_off;
    S.nx = q->mesh[0];
    S.ny = q->mesh[1];
    S.nz = q->mesh[2];
    S.nxh = S.nx / 2 + 1;
    S.m_off = q->m_off;
    S.s_off = q->m_off;
    S.g_off = git->second.off;
    S.ntx = q->ntile[0];
    S.nty = q->ntile[1];
    S.ntz = q->ntile[2];
    S.t_off = (int)q->t_off;
    S.nxp = halo_extent(S.nx, T, P, true);
    S.nyp = halo_extent(S.ny, T, P, false);
    S.nzp = halo_extent(S.nz, T, P, false);
    S.mp_off = q->m_off;
    if (use_tma) {
        CUtensorMap map;
        if (!encode_phi_map(&map, d_phi + S.mp_off, S.nxp, S.nyp, S.nzp, tma_bx, tma_by, T + P - 1))
            use_tma = false;  // the cp.async staging from now on
        else {
            int rcm = upload(sg, d_tmaps + q->slot, &map, sizeof(CUtensorMap));
            if (rcm) return rcm;
        }
    }
    S.Lx = (float)r.Lx;
    S.Ly = (float)r.Ly;
    S.Lz = (float)r.Lz;
    S.inv_Lx = 1.0f / S.Lx;
    S.inv_Ly = 1.0f / S.Ly;
    S.inv_Lz = 1.0f / S.Lz;
    S.gxd = S.nx / r.Lx;
    S.gyd = S.ny / r.Ly;
    S.gzd = S.nz / r.Lz;
    S.Lxd = r.Lx;
    S.Lyd = r.Ly;
    S.Lzd = r.Lz;
    S.V = r.Lx * r.Ly * r.Lz;
    S.pset = ps;
    S.twx = tw_off[S.nx];
    S.twy = tw_off[S.ny];
    S.twz = tw_off[S.nz];
    S.radx = radix_plan(S.nx);
    S.rady = radix_plan(S.ny);
    S.radz = radix_plan(S.nz);
    int rc = upload(sg, d_sys + q->slot, &S, sizeof(SysDev));
    if (rc) return rc;
    // rigid water: geometry index and the atoms the plain integrator skips
    q->geo = -1;
    if (r.rigid_doh > 0) {
        for (size_t g = 0; g < geos.size(); ++g)
            if (geos[g].x == r.rigid_doh && geos[g].y == r.rigid_dhh) q->geo = (int)g;
        if (q->geo < 0) {
            if ((int)geos.size() >= MAX_GEOS) return fail(ESP_ERR_UNSUPPORTED, "more than 16 rigid-water geometries");
            q->geo = (int)geos.size();
            geos.push_back(make_double2(r.rigid_doh, r.rigid_dhh));
            if ((rc = upload(sg, d_geo + q->geo, &geos.back(), sizeof(double2)))) return rc;
        }
    }
    const int2 skip = make_int2(0, q->geo >= 0 ? r.N : 0);
    if ((rc = upload(sg, d_rskip + q->slot, &skip, sizeof(int2)))) return rc;
    // inputs (caller's host memory) and tile owner table
    ESPB_CK(cudaMemcpyAsync(d_pos + q->p_off, r.pos4, (size_t)r.N * 16, cudaMemcpyHostToDevice, st));
    ESPB_CK(cudaMemcpyAsync(d_q + q->p_off, r.charge, (size_t)r.N * 4, cudaMemcpyHostToDevice, st));
    if (r.vel4) ESPB_CK(cudaMemcpyAsync(d_vel + q->p_off, r.vel4, (size_t)r.N * 16, cudaMemcpyHostToDevice, st));
    k_fill_int<<<(int)((ntiles + 255) / 256), 256, 0, st>>>(d_tile_sys + q->t_off, (int)ntiles, q->slot);
    ESPB_CK(cudaGetLastError());
    if (build_g) {
        rc = influence(q, S, sg);
        if (rc) return rc;
        n_builds++;
    } else {
        n_hits++;
    }
    // neighbour list (cell list of this system alone)
    CellDev C{};
    int nc[3];
    for (int d = 0; d < 3; ++d) {
        if (2.0 * rlist > L[d]) return fail(ESP_ERR_INVALID, "rcut + skin must not exceed half the box");
        nc[d] = std::min(MAX_CELLS_AXIS, std::max(1, (int)std::floor(L[d] / rlist)));
    }
    C.ncx = nc[0];
    C.ncy = nc[1];
    C.ncz = nc[2];
    C.inv_wx = (float)(nc[0] / r.Lx);
    C.inv_wy = (float)(nc[1] / r.Ly);
    C.inv_wz = (float)(nc[2] / r.Lz);
    C.c_off = 0;
    C.nl_off = q->nl_off;
    const int ncell = nc[0] * nc[1] * nc[2];
    std::vector<int2> ch;
    for (int i = 0; i < r.N; i += 256) ch.push_back(make_int2(q->slot, (int)q->p_off + i));
    if ((rc = upload(sg, d_cells + q->slot, &C, sizeof(CellDev))) || (rc = upload(sg, d_nlchunks, ch.data(), ch.size() * sizeof(int2))))
        return rc;
    k_fill_int<<<(ncell + 255) / 256, 256, 0, st>>>(d_cell_sys, ncell, q->slot);
    ESPB_CK(cudaGetLastError());
    NlistArgs na;
    na.chunks = d_nlchunks;
    na.n_chunks = (int)ch.size();
    na.sys = d_sys;
    na.cells = d_cells;
    na.cell_sys = d_cell_sys;
    na.n_cells = ncell;
    na.total = r.N;
    na.pos = d_pos;
    na.ckey = d_ckey;
    na.ccount = d_ccount;
    na.cstart = d_cstart;
    na.perm_u = d_cperm;
    na.wpos = d_wpos;
    na.cpos = d_cpos;
    na.rlist2 = (float)(rlist * rlist);
    na.cap = cap;
    na.head = d_head;
    na.nn = d_nn;
    na.nl = d_nl;
    na.overflow = d_ovf + 2 * q->slot;  // [flag, longest row] of this slot's build
    ESPB_CK(launch_nlist(na, st));
    q->steps_done = 0;
    q->evaluated = false;
    bytes_active += q->footprint;
    return 0;
}

void esp_server::release(Request* q) {
    palloc.release(q->p_off);
    malloc_.release(q->m_off);
    talloc.release(q->t_off);
    nlalloc.release(q->nl_off);
    auto git = gcache.find(q->gkey);
    if (git != gcache.end()) git->second.refs--;
    free_slots.push_back(q->slot);
    bytes_active -= q->footprint;
}

// ---------------------------------------------------------------------------
// one round: every admitted system advances by one evaluation
// ---------------------------------------------------------------------------
int esp_server::launch_round(Staging& sg) {
    std::vector<int2> chunks, pchunks, mdchunks, pit, sit;
    std::vector<int4> xit, yit, zit, ritems;
    const int ppb = 256 / tpp;
    int nmax[3] = {4, 4, 4};
    int smem_plane = 0, smem_slab = 0;
    for (Request* q : active) {
        const int s = q->slot, N = q->r.N, po = (int)q->p_off;
        for (int i = 0; i < N; i += 256) chunks.push_back(make_int2(s, po + i));
        for (int i = 0; i < N; i += ppb) pchunks.push_back(make_int2(s, po + i));
        if (q->evaluated) {
            for (int i = 0; i < N; i += 256) mdchunks.push_back(make_int2(s, po + i));
            if (q->geo >= 0)
                for (int m = 0; m < N / 3; m += SETTLE_CHUNK)
                    ritems.push_back(make_int4(s, po + 3 * m, std::min(SETTLE_CHUNK, N / 3 - m), q->geo));
        }
        const int nx = q->mesh[0], ny = q->mesh[1], nz = q->mesh[2], nxh = nx / 2 + 1;
        nmax[0] = std::max(nmax[0], nx);
        nmax[1] = std::max(nmax[1], ny);
        nmax[2] = std::max(nmax[2], nz);
        const int sp = fft_plane_smem(nx, ny), ss = fft_slab_smem(nx, nz);
        if (sp <= FFT_SMEM_MAX) {
            smem_plane = std::max(smem_plane, sp);
            for (int z = 0; z < nz; ++z) pit.push_back(make_int2(s, z));
        } else {
            for (int z = 0; z < nz; ++z)
                for (int y0 = 0; y0 < ny; y0 += 2 * FFT_B_X) xit.push_back(make_int4(s, z, y0, 0));
            for (int z = 0; z < nz; ++z)
                for (int k0 = 0; k0 < nxh; k0 += FFT_B_YZ) yit.push_back(make_int4(s, z, k0, 0));
        }
        if (ss <= FFT_SMEM_MAX) {
            smem_slab = std::max(smem_slab, ss);
            for (int y = 0; y < ny; ++y) sit.push_back(make_int2(s, y));
        } else {
            for (int y = 0; y < ny; ++y)
                for (int k0 = 0; k0 < nxh; k0 += FFT_B_YZ) zit.push_back(make_int4(s, y, k0, 0));
        }
    }
    if ((long long)chunks.size() > chunk_cap || (long long)pchunks.size() > pchunk_cap ||
        (long long)pit.size() > ITEM_CAP || (long long)sit.size() > ITEM_CAP || (long long)xit.size() > ITEM_CAP ||
        (long long)yit.size() > ITEM_CAP || (long long)zit.size() > ITEM_CAP || (long long)ritems.size() > ritem_cap)
        return fail(ESP_ERR_UNSUPPORTED, "work lists exceed their buffers");
    int rc = 0;
    if ((rc = upload(sg, d_chunks, chunks.data(), chunks.size() * sizeof(int2))) ||
        (rc = upload(sg, d_pchunks, pchunks.data(), pchunks.size() * sizeof(int2))) ||
        (rc = upload(sg, d_mdchunks, mdchunks.data(), mdchunks.size() * sizeof(int2))) ||
        (rc = upload(sg, d_pitems, pit.data(), pit.size() * sizeof(int2))) ||
        (rc = upload(sg, d_sitems, sit.data(), sit.size() * sizeof(int2))) ||
        (rc = upload(sg, d_xitems, xit.data(), xit.size() * sizeof(int4))) ||
        (rc = upload(sg, d_yitems, yit.data(), yit.size() * sizeof(int4))) ||
        (rc = upload(sg, d_zitems, zit.data(), zit.size() * sizeof(int4))) ||
        (rc = upload(sg, d_ritems, ritems.data(), ritems.size() * sizeof(int4))))
        return rc;
    LaunchArgs a;
    a.pc = pc;
    a.nq = nq;
    a.sys = d_sys;
    a.psets = d_pset;
    a.nsys = max_slots;
    a.P = P;
    a.T = T;
    a.D = D;
    a.PX = PX;
    a.PP = PP;
    a.tpp = tpp;
    a.accumulate = 1;
    a.chunks = d_chunks;
    a.n_chunks = (int)chunks.size();
    a.pchunks = d_pchunks;
    a.n_pchunks = (int)pchunks.size();
    a.tile_sys = d_tile_sys;
    a.n_tiles = (int)talloc.high();
    a.tile_count = d_tcount;
    a.tile_start = d_tstart;
    a.pos_in = d_pos;
    a.q_in = d_q;
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
    a.pitems = d_pitems;
    a.n_pitems = (int)pit.size();
    a.sitems = d_sitems;
    a.n_sitems = (int)sit.size();
    a.xitems = d_xitems;
    a.n_xitems = (int)xit.size();
    a.yitems = d_yitems;
    a.n_yitems = (int)yit.size();
    a.zitems = d_zitems;
    a.n_zitems = (int)zit.size();
    a.smem_plane = smem_plane;
    a.smem_slab = smem_slab;
    a.nmax_x = nmax[0];
    a.nmax_y = nmax[1];
    a.nmax_z = nmax[2];
    a.force = d_force;
    a.acc = d_acc;
    a.energy = d_energy;
    a.virial = nullptr;
    a.tmaps = use_tma ? d_tmaps : nullptr;
    a.tma_bx = tma_bx;
    a.tma_by = tma_by;
    a.kerr = d_kerr;
    // interp_mode 2: the persistent TMA kernel fed from a tile queue (its counter)
    a.queue = prm.interp_mode == 2 ? d_kerr + 1 : nullptr;
    a.want_virial = 0;
    a.add_bg = 1;
    a.nl_head = d_head;
    a.nl_n = d_nn;
    a.nl_list = d_nl;
    const float dt = active.empty() ? 0.f : (float)active[0]->r.dt;
    // NVE first half for the systems past their first evaluation; systems
    // of one round share dt (checked at submit)
    ESPB_CK(launch_nve1(d_mdchunks, (int)mdchunks.size(), d_sys, d_pos, d_vel, d_force, dt, st, d_rskip));
    ESPB_CK(launch_settle1(d_ritems, (int)ritems.size(), d_sys, d_pos, d_vel, d_force, dt, d_geo, false, st));
    ESPB_CK(cudaMemsetAsync(d_acc, 0, (size_t)max_slots * ACC_STRIDE * sizeof(double), st));
    ESPB_CK(launch_bin(a, st));
    ESPB_CK(launch_sort(a, st));
    ESPB_CK(launch_spread(a, st));
    ESPB_CK(launch_fft(a, st));
    ESPB_CK(launch_interp(a, st));
    ESPB_CK(launch_pair(a, st));
    ESPB_CK(launch_finalize(a, st));
    ESPB_CK(launch_nve2(d_mdchunks, (int)mdchunks.size(), d_sys, d_vel, d_force, dt, st));
    ESPB_CK(launch_settle2(d_ritems, (int)ritems.size(), d_sys, d_pos, d_vel, false, st));
    n_rounds++;

    Round rd;
    std::vector<Request*> keep;
    for (Request* q : active) {
        if (q->evaluated) q->steps_done++;
        q->evaluated = true;
        if (q->steps_done >= q->r.nsteps) rd.fin.push_back(q);
        else keep.push_back(q);
    }
    if (!rd.fin.empty()) {
        // one page-locked flag per finishing request, inside this round's staging
        const size_t need = ((sg.used + rd.fin.size() * sizeof(int) + 255) & ~(size_t)255);
        if (need > sg.cap) {
            ESPB_CK(cudaStreamSynchronize(st));
            char* nb = nullptr;
            size_t cap = sg.cap * 2;
            while (cap < need) cap *= 2;
            ESPB_CK(cudaHostAlloc((void**)&nb, cap, cudaHostAllocDefault));
            cudaFreeHost(sg.buf);
            sg.buf = nb;
            sg.cap = cap;
            sg.used = 0;
        }
        rd.ovf = reinterpret_cast<int*>(sg.buf + sg.used);
        sg.used = (sg.used + rd.fin.size() * sizeof(int) + 255) & ~(size_t)255;
    }
    for (size_t k = 0; k < rd.fin.size(); ++k) {
        Request* q = rd.fin[k];
        const esp_request& r = q->r;
        const size_t n = (size_t)r.N;
        if (r.out_pos4) ESPB_CK(cudaMemcpyAsync(r.out_pos4, d_pos + q->p_off, n * 16, cudaMemcpyDeviceToHost, st));
        if (r.out_vel4) ESPB_CK(cudaMemcpyAsync(r.out_vel4, d_vel + q->p_off, n * 16, cudaMemcpyDeviceToHost, st));
        if (r.out_force4) ESPB_CK(cudaMemcpyAsync(r.out_force4, d_force + q->p_off, n * 16, cudaMemcpyDeviceToHost, st));
        if (r.out_energy) ESPB_CK(cudaMemcpyAsync(r.out_energy, d_energy + q->slot, 8, cudaMemcpyDeviceToHost, st));
        ESPB_CK(cudaMemcpyAsync(rd.ovf + k, d_ovf + 2 * q->slot, sizeof(int), cudaMemcpyDeviceToHost, st));
        release(q);  // later uploads into these ranges are stream-ordered after the copies above
    }
    active.swap(keep);
    rd.ev = get_event();
    ESPB_CK(cudaEventRecord(rd.ev, st));
    sg.pending = true;
    inflight.push_back(std::move(rd));
    return 0;
}

void esp_server::retire(bool block) {
    while (!inflight.empty()) {
        Round& rd = inflight.front();
        cudaError_t e = block ? cudaEventSynchronize(rd.ev) : cudaEventQuery(rd.ev);
        if (e == cudaErrorNotReady) return;
        const double t = now();
        {
            std::lock_guard<std::mutex> lk(mu);
            for (size_t k = 0; k < rd.fin.size(); ++k) {
                Request* q = rd.fin[k];
                if (e != cudaSuccess) {
                    q->state = ESP_ERR_CUDA;
                    stats.failed++;
                } else if (rd.ovf && rd.ovf[k]) {
                    q->state = ESP_ERR_OVERFLOW;
                    stats.failed++;
                } else {
                    q->state = 2;
                    stats.completed++;
                    stats.particle_steps += (long long)q->r.N * std::max(q->r.nsteps, 1);
                }
                q->t_done = t;
            }
        }
        done_cv.notify_all();
        ev_pool.push_back(rd.ev);
        inflight.pop_front();
        block = false;
        if (e != cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            error_msg = std::string("server stream: ") + cudaGetErrorString(e);
            error_code = ESP_ERR_CUDA;
        }
    }
}

void esp_server::fail_all(int code) {
    std::lock_guard<std::mutex> lk(mu);
    for (auto& q : reqs)
        if (q->state == 0 || q->state == 1) {
            q->state = code;
            q->t_done = now();
            stats.failed++;
        }
    pending.clear();
    active.clear();
    done_cv.notify_all();
}

void esp_server::run() {
    cudaSetDevice(dev);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            for (;;) {
                if (stop) return;
                const bool busy = !active.empty() || !inflight.empty();
                const double t = now();
                const bool arrived = started && !pending.empty() && pending.front()->t_arrival <= t;
                if (busy || arrived) break;
                if (started && !pending.empty())
                    cv.wait_for(lk, std::chrono::duration<double>(pending.front()->t_arrival - t));
                else
                    cv.wait(lk);
            }
        }
        if (error_code) {
            retire(true);
            fail_all(error_code);
            continue;
        }
        // this round's staging buffer: its previous uploads must have run
        Staging& sg = stage[stage_idx];
        if (sg.pending) {
            cudaEventSynchronize(sg.ev);
            sg.pending = false;
        }
        retire(false);
        sg.used = 0;
        // admit arrived requests in arrival order while they fit
        for (;;) {
            Request* q = nullptr;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (!started || pending.empty() || pending.front()->t_arrival > now()) break;
                q = pending.front();
            }
            if (!active.empty() && q->r.dt != active[0]->r.dt) break;  // one dt per round
            int rc = admit(q, sg);
            if (rc == 1 && active.empty() && inflight.empty())
                rc = fail(ESP_ERR_ALLOC, "request does not fit the empty server arenas");
            if (rc == 1) break;  // waits for memory or a slot
            std::lock_guard<std::mutex> lk(mu);
            pending.pop_front();
            if (rc < 0) {
                q->state = rc;
                q->t_done = now();
                stats.failed++;
                done_cv.notify_all();
                continue;
            }
            q->state = 1;
            q->t_admit = now();
            active.push_back(q);
            stats.max_active = std::max(stats.max_active, (int)active.size());
            stats.peak_bytes = std::max(stats.peak_bytes, bytes_active);
        }
        if (!active.empty()) {
            const int rc = launch_round(sg);
            if (rc) {
                std::lock_guard<std::mutex> lk(mu);
                error_msg = esp_last_error();
                error_code = rc;
            }
        }
        if (sg.pending) cudaEventRecord(sg.ev, st);
        stage_idx ^= 1;
        if (active.empty() && !inflight.empty()) retire(true);
        while (inflight.size() > 2) retire(true);
    }
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int esp_server_create(const esp_server_config* cfg, esp_server** out) {
    if (!cfg || !out) return fail(ESP_ERR_INVALID, "null argument");
    *out = nullptr;
    auto* s = new esp_server();
    const int rc = s->init(*cfg);
    if (rc) {
        const std::string msg = esp_last_error();
        esp_server_destroy(s);
        return fail(rc, msg);
    }
    *out = s;
    return 0;
}

int esp_server_submit(esp_server* s, const esp_request* r, long long* id) {
    if (!s || !r) return fail(ESP_ERR_INVALID, "null argument");
    if (r->N <= 0 || r->N > s->max_particles) return fail(ESP_ERR_INVALID, "N must be in [1, max_particles]");
    if (!(r->Lx > 0 && r->Ly > 0 && r->Lz > 0)) return fail(ESP_ERR_INVALID, "box lengths must be positive");
    if (!(r->rcut > 0) || r->skin < 0) return fail(ESP_ERR_INVALID, "rcut must be positive and skin >= 0");
    if (r->nsteps < 0) return fail(ESP_ERR_INVALID, "negative step count");
    if (r->nsteps > 0 && (!r->vel4 || !(r->dt > 0))) return fail(ESP_ERR_INVALID, "NVE steps need velocities and dt > 0");
    if (!r->pos4 || !r->charge) return fail(ESP_ERR_INVALID, "null input pointer");
    if (r->rigid_doh > 0 && (r->N % 3 != 0 || !(r->rigid_dhh > 0) || r->rigid_dhh >= 2.0 * r->rigid_doh))
        return fail(ESP_ERR_INVALID, "rigid water needs N = 3 x molecules and 0 < d_hh < 2 d_oh");
    std::lock_guard<std::mutex> lk(s->mu);
    // an arrival already in the past counts from now; the queue stays in
    // arrival order because the clock only moves forward
    double t_arr = std::max(0.0, r->arrival);
    if (s->started) t_arr = std::max(t_arr, s->now());
    if (!s->pending.empty() && t_arr < s->pending.back()->t_arrival)
        return fail(ESP_ERR_INVALID, "arrival times must not decrease");
    auto q = std::make_unique<Request>();
    q->r = *r;
    q->id = (long long)s->reqs.size();
    q->t_arrival = t_arr;
    s->pending.push_back(q.get());
    s->reqs.push_back(std::move(q));
    s->stats.submitted++;
    if (id) *id = s->reqs.back()->id;
    s->cv.notify_all();
    return 0;
}

int esp_server_start(esp_server* s) {
    if (!s) return fail(ESP_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->started) {
        s->t0 = std::chrono::steady_clock::now();
        s->started = true;
    }
    s->cv.notify_all();
    return 0;
}

int esp_server_status(esp_server* s, long long id, esp_request_status* out) {
    if (!s || !out) return fail(ESP_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || id >= (long long)s->reqs.size()) return fail(ESP_ERR_INVALID, "unknown request id");
    const Request& q = *s->reqs[id];
    out->state = q.state;
    out->t_arrival = q.t_arrival;
    out->t_admit = q.t_admit;
    out->t_done = q.t_done;
    out->nx = q.mesh[0];
    out->ny = q.mesh[1];
    out->nz = q.mesh[2];
    out->footprint = q.footprint;
    return 0;
}

int esp_server_wait_all(esp_server* s, double timeout_s) {
    if (!s) return fail(ESP_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    for (;;) {
        if (s->stats.completed + s->stats.failed >= s->stats.submitted) break;
        if (s->done_cv.wait_until(lk, deadline) == std::cv_status::timeout &&
            s->stats.completed + s->stats.failed < s->stats.submitted)
            return fail(ESP_ERR_INVALID, "timed out waiting for requests");
    }
    if (s->error_code) return fail(s->error_code, s->error_msg);
    return 0;
}

int esp_server_get_stats(esp_server* s, esp_server_stats* out) {
    if (!s || !out) return fail(ESP_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->rounds = s->n_rounds;
    out->influence_builds = s->n_builds;
    out->influence_hits = s->n_hits;
    return 0;
}

int esp_server_destroy(esp_server* s) {
    if (!s) return 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    if (s->st) {
        cudaStreamSynchronize(s->st);
        for (Round& rd : s->inflight) cudaEventDestroy(rd.ev);
        for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
        cudaStreamDestroy(s->st);
    }
    delete s;
    return 0;
}

}  // extern "C"
