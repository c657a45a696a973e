/*
 * esp_b200.h -- C ABI of the Blackwell (sm_100a) ESP electrostatics path.
 *
 * ESP = Ewald Summation with Prolates: the long-range Coulomb part on a
 * mesh (PSWF spreading, 3D FFT, influence multiply, inverse FFT,
 * interpolation) plus the short-range EvaluatorPairPSWF term over a
 * neighbour list. Units follow the reference: E = q_i q_j / (4 pi r).
 *
 * Conventions (all entry points):
 *  - plain pointers and sizes only; device pointers are CUDA device memory
 *    owned by the caller; `stream` is a cudaStream_t passed as void*;
 *  - positions are float4 per particle laid out as 4 floats (x, y, z, w),
 *    w ignored (HOOMD keeps the type there), any periodic image;
 *  - forces are written as 4 floats per particle: fx, fy, fz, per-particle
 *    energy (the Scalar4 output contract of HOOMD's ForceCompute::m_force);
 *  - neighbour lists use HOOMD's layout: the neighbours of particle i are
 *    nlist[head[i] + k], k < n_neigh[i], full (both i-j and j-i) lists;
 *  - virial: 6 doubles xx, xy, xz, yy, yz, zz with W_ab = -dE/d eps_ab;
 *  - every call returns 0 on success or a negative ESP_ERR_* code and
 *    throws nothing; esp_last_error() gives the message. Calls are
 *    asynchronous on `stream` and not thread-safe per context.
 *
 * The reference interfaces each entry point replaces are cited per call
 * (paths relative to the reference repository slweng0321/ESP_HOOMD).
 */
#ifndef ESP_B200_H_
#define ESP_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

#define ESP_OK 0
#define ESP_ERR_INVALID (-1)     /* bad argument */
#define ESP_ERR_CUDA (-2)        /* CUDA runtime error */
#define ESP_ERR_ALLOC (-3)       /* device allocation failed */
#define ESP_ERR_UNSUPPORTED (-4) /* parameter outside the supported set */
#define ESP_ERR_OVERFLOW (-5)    /* neighbour list capacity exceeded */

/* precision of a context (esp_params.precision) */
#define ESP_FP32 0 /* FP32 bulk arithmetic, FP64 reductions (esp_compute) */
#define ESP_FP64 1 /* every stage in FP64 (esp_compute_f64) */

/* compute flags */
#define ESP_LONG_RANGE 1  /* mesh part + self + background (esp.Spectral) */
#define ESP_SHORT_RANGE 2 /* pair part over the neighbour list (esp.Local) */
#define ESP_ALL 3

typedef struct esp_ctx esp_ctx;
typedef struct esp_batch esp_batch;

/* Parameters. Mirrors ESPForceCompute::setParams(nx, ny, nz, order, kappa,
 * rcut, alpha, n_table) of src/ESPForceCompute.h:99-106, plus the knobs of
 * the runtime table generator that replaces src/PSWF_Coeffs.h:24-27. */
typedef struct esp_params {
    int nx, ny, nz;      /* mesh; 0 = chosen from target_error */
    int order;           /* PSWF support P in grid points, 2..12 */
    double kappa;        /* split bandwidth in 1/length: c = kappa * rcut; 0 = auto */
    double rcut;         /* real-space cutoff r_c (> 0) */
    double alpha;        /* Debye screening; only 0 is supported */
    int n_table;         /* segments of the introspection table */
    double target_error; /* relative RMS force error the auto choices aim at */
    double window_c;     /* window bandwidth c_w; 0 = auto */
    int window_degree;   /* window polynomial degree; 0 = auto */
    int tile;            /* tile edge in mesh cells; 0 = auto (tile + order - 1 = 16); a tile whose
                            extended region needs more shared memory than a CTA has is refused at
                            create with ESP_ERR_UNSUPPORTED */
    int threads_per_particle; /* pair kernel lanes per particle: 4, 8, 16, 32; 0 = 4 */
    int precision;       /* ESP_FP32 (default) or ESP_FP64 */
    int fft_mode;        /* 0: whole planes/slabs in shared memory where they fit; 1: per-line passes */
    int interp_mode;     /* 0: the potential tile staged by TMA, one CTA per tile (supports 5..8);
                            1: cp.async staging; 2: TMA, persistent CTAs fed from a tile queue with
                            the next tile's box in flight (supports 5..8) */
} esp_params;

/* Resolved configuration of a context or of one system of a batch. */
typedef struct esp_info {
    int nx, ny, nz, order, tile, window_degree;
    double c_split, c_window, rcut;
    double lambda0, m2;      /* Q(0) and int_0^1 psi t^2 / int_0^1 psi */
    double split_fit_err, window_fit_err;
    long long device_bytes;  /* device memory held by the context */
} esp_info;

/* Fill `p` with defaults (order 8, rcut 3.0, target 1e-5, everything else auto). */
int esp_params_default(esp_params* p);

/* Message of the last failed call on this thread (ctx may be NULL). */
const char* esp_last_error(void);

/* ---------------------------------------------------------------- single system
 * Replaces ESPForceComputeGPU (src/ESPForceComputeGPU.h:55-131): the
 * constructor + initializeFFT() + setupCoeffs() (src/ESPForceComputeGPU.cc:47-214,
 * src/ESPForceCompute.cc:179-198). Orthorhombic box Lx, Ly, Lz. */
int esp_create(const esp_params* p, double Lx, double Ly, double Lz, int N, esp_ctx** out);

/* ESPForceCompute::setParams (src/ESPForceCompute.cc:71-89): new parameters,
 * tables rebuilt on the next compute. */
int esp_set_params(esp_ctx* ctx, const esp_params* p);

/* Box change (HOOMD box resize); re-plans the influence table. */
int esp_set_box(esp_ctx* ctx, double Lx, double Ly, double Lz);

/* ESPForceCompute::invalidate (src/ESPForceCompute.h:120): rebuild all
 * tables on the next compute. */
int esp_invalidate(esp_ctx* ctx);

/* One evaluation: ESPForceCompute::computeForces (src/ESPForceCompute.cc:96-127)
 * with its GPU stages (src/ESPForceComputeGPU.cu:206-373) when
 * flags & ESP_LONG_RANGE, and PotentialPairGPU<EvaluatorPairPSWF>
 * (src/module.cc:79, src/EvaluatorPairPSWF.h:274-295) when
 * flags & ESP_SHORT_RANGE. Overwrites force[4N]; writes energy[1] and
 * virial[6] (device doubles, may be NULL). The neighbour-list pointers may
 * be NULL without ESP_SHORT_RANGE. */
int esp_compute(esp_ctx* ctx, void* stream, const float* pos4, const float* charge, int N,
                const unsigned* head, const unsigned* n_neigh, const unsigned* nlist,
                float* force4, double* energy, double* virial6, int flags);

/* One evaluation written in the output contract of HOOMD's ForceCompute, as
 * the reference's ESPForceCompute fills it (src/ESPForceCompute.cc:96-127):
 * force4 as esp_compute (m_force: force and per-particle energy, the mesh,
 * self and pair terms); virial_pp[k * virial_pitch + i], k = xx, xy, xz, yy,
 * yz, zz (m_virial, device floats, virial_pitch >= N): particle i's half of
 * the virial of its pairs (short-range term and exclusion corrections);
 * external7 (device doubles) = {E_ext, W_ext xx, xy, xz, yy, yz, zz}
 * (m_external_energy, m_external_virial): the terms no particle owns -- the
 * neutralising background energy and the k-space virial plus the
 * background's. Sum_i force4[i].w + E_ext and sum_i virial_pp + W_ext are the
 * totals esp_compute returns. */
int esp_compute_hoomd(esp_ctx* ctx, void* stream, const float* pos4, const float* charge, int N,
                      const unsigned* head, const unsigned* n_neigh, const unsigned* nlist, float* force4,
                      float* virial_pp, int virial_pitch, double* external7, int flags);

/* FP64 evaluation (contexts created with precision ESP_FP64), for HOOMD
 * double builds: positions and forces are 4 doubles per particle (Scalar4 =
 * double4), charges doubles; otherwise as esp_compute. Every stage runs in
 * FP64 (split polynomial fitted to 1e-12), the path for accuracy targets
 * below the FP32 floor (~1e-7 relative RMS force error). */
int esp_compute_f64(esp_ctx* ctx, void* stream, const double* pos4, const double* charge, int N,
                    const unsigned* head, const unsigned* n_neigh, const unsigned* nlist,
                    double* force4, double* energy, double* virial6, int flags);

int esp_get_info(const esp_ctx* ctx, esp_info* info);
int esp_destroy(esp_ctx* ctx);

/* Excluded pairs: the input of ESPForceComputeGPU::fixExclusionsGPU
 * (src/ESPForceComputeGPU.cc:390-420) and its kernel
 * (src/ESPForceComputeGPU.cu:391-471), HOOMD's NeighborList exclusion arrays.
 * Particle i excludes ex_list[i * ex_pitch + k], k < n_ex[i] (device arrays,
 * indices local to the system, every pair listed from both sides). Every
 * later long-range evaluation removes the mesh's interaction of these pairs
 * (force, energy, virial) at any distance; the neighbour list given to the
 * short-range term must leave them out, as HOOMD's does (lists built by
 * esp_batch_build_nlist / esp_batch_build_pairlist while exclusions are set
 * do). The arrays stay owned by the caller and must stay valid while set;
 * n_ex = NULL clears. */
int esp_set_exclusions(esp_ctx* ctx, const unsigned* n_ex, const unsigned* ex_list, int ex_pitch);

/* Stage outputs, for validation of single stages (no reference
 * counterpart: the reference exposes only the final forces).
 * esp_spread: bin + sort + spreading of (pos4, charge) into the caller's
 * FP64 charge mesh rho[nz*ny*nx] (x fastest; zeroed first), the charge
 * assignment of src/ESPForceComputeGPU.cu:206-272.
 * esp_get_sort: tile key of every particle (key[N], input order) and the
 * stable permutation (perm[N], sorted slot -> particle) of the last call.
 * esp_get_potential: the potential mesh phi[nz*ny*nx] of the last
 * long-range evaluation. */
int esp_spread(esp_ctx* ctx, void* stream, const float* pos4, const float* charge, int N, double* rho);
int esp_get_sort(const esp_ctx* ctx, void* stream, unsigned* key, unsigned* perm);
int esp_get_potential(const esp_ctx* ctx, void* stream, float* phi);

/* No-allocation charge spreading. No counterpart in the reference.
 * Some callers cannot allocate device memory: an MD engine that hands all of
 * its device memory to its own pool allocator, or a time step that must not
 * call cudaFree (which synchronises the whole device) in the middle of a
 * run. esp_create/esp_spread allocate their work arrays with cudaMalloc, so
 * such callers cannot use them. esp_spread_noalloc does the same bin + sort +
 * spreading into the caller's FP64 charge mesh rho[nz*ny*nx] (x fastest;
 * zeroed first) with no context: its work arrays live in one fixed-size
 * scratch array inside the library (2.2 MB, held on every GPU that
 * loads the library until the process exits), and it calls no allocating
 * CUDA or library routine.
 *  - Limits: 1 <= N <= ESP_SPREAD_NOALLOC_MAX_N particles and at most
 *    ESP_SPREAD_NOALLOC_MAX_TILES tiles; larger inputs are rejected with
 *    ESP_ERR_UNSUPPORTED (use esp_spread for them).
 *  - Parameters: p->order, p->window_c, p->window_degree, p->tile and
 *    p->precision (ESP_FP32 or ESP_FP64; it selects the default window
 *    degree, as in esp_create) as in esp_create; the mesh p->nx, p->ny, p->nz
 *    must be given (no automatic choice), each in [max(order, 4), 256];
 *    tile + order - 1 <= 16.
 *  - The first call on a device (per device, with that device current) looks
 *    up the scratch array's device address and sets the spreading kernels'
 *    shared-memory limits; make that first call before any stream capture.
 *    The set-up is redone when the device's context changes (for example
 *    after cudaDeviceReset), on the next call.
 *  - Every call on a device shares the one scratch array: calls whose work
 *    overlaps on the GPU (different streams, or different host threads,
 *    without ordering between them) race and give wrong meshes. Calls
 *    ordered on one stream are safe.
 * Results equal esp_spread's for the same parameters and mesh, up to the
 * order of FP64 atomic additions. */
#define ESP_SPREAD_NOALLOC_MAX_N 32768
#define ESP_SPREAD_NOALLOC_MAX_TILES 4096
int esp_spread_noalloc(void* stream, const esp_params* p, double Lx, double Ly, double Lz, const float* pos4,
                       const float* charge, int N, double* rho);

/* ---------------------------------------------------------------- batches
 * Many independent systems evaluated by one launch per stage (no reference
 * counterpart; the reference evaluates one HOOMD system per ForceCompute).
 * System s holds N[s] particles at offset sum_{r<s} N[r] of the
 * concatenated arrays; boxes[3s..3s+2] its box; mesh[3s..] its mesh or
 * NULL for automatic meshes. Neighbour indices are local to each system;
 * head[] values index the concatenated nlist array. energy[nsys],
 * virial[6*nsys]. */
int esp_batch_create(const esp_params* p, int nsys, const int* N, const double* boxes, const int* mesh,
                     esp_batch** out);
int esp_batch_compute(esp_batch* b, void* stream, const float* pos4, const float* charge, const unsigned* head,
                      const unsigned* n_neigh, const unsigned* nlist, float* force4, double* energy,
                      double* virial6, int flags);
int esp_batch_compute_f64(esp_batch* b, void* stream, const double* pos4, const double* charge, const unsigned* head,
                          const unsigned* n_neigh, const unsigned* nlist, double* force4, double* energy,
                          double* virial6, int flags);
/* Autotuner (no reference counterpart; the reference's Autotuner<1> only
 * picks block sizes, src/ESPForceComputeGPU.cc:52-61): times `reps`
 * evaluations (flags as esp_batch_compute) of candidate plans on the given
 * inputs with CUDA events on `stream` -- pair lanes per particle (4, 8, 16),
 * tile edge (the 16^3 tensor-core tile and smaller dense tiles), FFT pass form
 * (whole planes/slabs in shared memory or per-line passes), TMA interpolation
 * form (one CTA per tile or persistent CTAs on a tile queue) -- by coordinate
 * descent, keeps the fastest plan (same meshes and accuracy) and writes its
 * parameters to `chosen` (may be NULL) and the per-candidate times (ms per
 * evaluation, up to `max_trials`) to `trial_ms` (may be NULL). Synchronises
 * `stream`; allocates like esp_batch_create. */
int esp_batch_autotune(esp_batch* b, void* stream, const float* pos4, const float* charge, const unsigned* head,
                       const unsigned* n_neigh, const unsigned* nlist, int flags, int reps, esp_params* chosen,
                       double* trial_ms, int max_trials);
int esp_batch_get_info(const esp_batch* b, int sys, esp_info* info);
/* Error word of the batch's kernels since the last call (no reference
 * counterpart): bit 0 -- a TMA-staged interpolation tile waited longer than
 * its bound for its potential box and was skipped (results invalid).
 * Synchronises the device, then clears the word. */
int esp_batch_device_errors(esp_batch* b, int* flags);
int esp_batch_total_particles(const esp_batch* b);
int esp_batch_destroy(esp_batch* b);
/* Exclusions of a batch, as esp_set_exclusions: rows by the particle's index
 * in the concatenated arrays, excluded indices local to its system. */
int esp_batch_set_exclusions(esp_batch* b, const unsigned* n_ex, const unsigned* ex_list, int ex_pitch);

/* ---------------------------------------------------------------- evaluator
 * EvaluatorPairPSWF::evalForceAndEnergy (src/EvaluatorPairPSWF.h:274-295)
 * with detail::pswf_eval_L (src/EvaluatorPairPSWF.h:113-143) over n pairs,
 * reading a PSWF_Coeffs.h-layout segment table (src/PSWF_Coeffs.h:29-30,
 * 4130, 8229, 8915): screen/dscreen [5*n_segs], r_lo/dr_inv [n_segs]. All
 * arrays are device doubles; evaluated[i] is the evaluator's return value.
 * energy_shift is not applied (the reference's V_cut is 0). */
int esp_pswf_eval_pairs(void* stream, int n, const double* rsq, const double* qiqj, double rcut, int n_segs,
                        const double* screen, const double* dscreen, const double* r_lo, const double* dr_inv,
                        double* force_divr, double* pair_eng, int* evaluated);

/* ---------------------------------------------------------------- MD harness
 * The pieces HOOMD would supply (neighbour list, NVE integrator), for
 * standalone runs and benchmarks. Neighbour list: cell list from the
 * particle positions, full list of all pairs with r < rlist (rlist at most
 * half the smallest box edge), fixed row capacity `cap` (head[i] = offset of
 * system s + local i * cap; totN * cap below 2^32). Does not synchronise: a
 * row longer than cap keeps its first cap entries, n_neigh holds the true
 * counts, and the overflow is reported (ESP_ERR_OVERFLOW) by
 * esp_batch_nlist_check, which waits for the build and writes the longest
 * row of an overflowing build to *needed_cap (0 when no row overflowed; may
 * be NULL), and by the first esp_batch_compute /
 * esp_batch_md_run over these rows that finds the build finished. Results
 * computed over an overflowed list are invalid; rebuild with a larger cap. */
int esp_batch_build_nlist(esp_batch* b, void* stream, const float* pos4, double rlist, int cap, unsigned* head,
                          unsigned* n_neigh, unsigned* nlist);
int esp_batch_nlist_check(esp_batch* b, int* needed_cap);

/* Pair list owned by the library: the short-range term's neighbour list
 * when the library builds it (the reference takes HOOMD's NeighborList,
 * src/module.cc:73-79; this replaces that list for standalone and batched
 * runs). Lists all pairs with r < rlist of pos4 (rlist at most half the
 * smallest box edge) on a cell grid of edge >= rlist, in cell order: rows
 * indexed by the build's cell-sorted slot, entries slots, so that a row's
 * neighbours are neighbours in memory (each evaluation's bin stage writes
 * the slot-ordered positions they are read from). esp_batch_compute and
 * esp_batch_md_run called with head = n_neigh = nlist = NULL run the
 * short-range term over the last list built. `cap` is the row capacity
 * (totN * cap below 2^32). Does not synchronise: overflow is reported as for
 * esp_batch_build_nlist, by esp_batch_pairlist_check and by the first
 * esp_batch_compute / esp_batch_md_run over the list that finds the build
 * finished. */
int esp_batch_build_pairlist(esp_batch* b, void* stream, const float* pos4, double rlist, int cap);
int esp_batch_pairlist_check(esp_batch* b, int* needed_cap);

/* Velocity-Verlet halves on the concatenated arrays: vel4 = (vx, vy, vz,
 * mass). step1: v += dt/2 F/m; x += dt v (wrapped into the box).
 * step2: v += dt/2 F/m. With rigid molecules set (esp_batch_set_rigid_water)
 * step1 constrains their positions (SETTLE) and step2 their velocities
 * (RATTLE), which needs pos4 (the positions after step1); pos4 may be NULL
 * otherwise. */
int esp_batch_nve_step1(esp_batch* b, void* stream, float* pos4, float* vel4, const float* force4, double dt);
int esp_batch_nve_step2(esp_batch* b, void* stream, const float* pos4, float* vel4, const float* force4, double dt);

/* FP64 velocity-Verlet halves (double4 positions, velocities with mass in
 * w, forces), as esp_batch_nve_step1/2. */
int esp_batch_nve_step1_f64(esp_batch* b, void* stream, double* pos4, double* vel4, const double* force4, double dt);
int esp_batch_nve_step2_f64(esp_batch* b, void* stream, const double* pos4, double* vel4, const double* force4,
                            double dt);

/* Rigid three-site molecules (no reference counterpart: HOOMD supplies the
 * constraints the reference's users would run; the water workloads are rigid
 * O-H-H molecules). System s holds count[s] molecules as consecutive (O, H,
 * H) triples from its local particle first[s] on, with O-H distance d_oh and
 * H-H distance d_hh (the two H of a molecule of equal mass; masses from
 * vel4.w). The velocity-Verlet steps (esp_batch_nve_step1/2 and their FP64
 * forms, esp_batch_md_run) keep them rigid: SETTLE (Miyamoto & Kollman 1992)
 * for positions, RATTLE for velocities. The initial positions must satisfy
 * the constraints and velocities have no bond-stretching components.
 * first = count = NULL clears. Host arrays of nsys ints. */
int esp_batch_set_rigid_water(esp_batch* b, const int* first, const int* count, double d_oh, double d_hh);

/* Lennard-Jones core repulsion of the harness, 4 eps ((sigma/r)^12 -
 * (sigma/r)^6) for r < r_cut (no shift), over the full neighbour list:
 * ADDS the forces and half the pair energy per particle to force4 and each
 * system's LJ energy to energy[s] (device doubles, may be NULL). */
int esp_batch_lj(esp_batch* b, void* stream, const float* pos4, const unsigned* head, const unsigned* n_neigh,
                 const unsigned* nlist, double epsilon, double sigma, double r_cut, float* force4, double* energy);
int esp_batch_lj_f64(esp_batch* b, void* stream, const double* pos4, const unsigned* head, const unsigned* n_neigh,
                     const unsigned* nlist, double epsilon, double sigma, double r_cut, double* force4,
                     double* energy);

/* nsteps velocity-Verlet steps of every system of the batch: per step
 * step1, a full evaluation (ESP_ALL) at the new positions into force4 /
 * energy / virial, step2. force4 must hold the forces of the current
 * positions on entry. On return force4 (with per-particle energies in w),
 * energy and virial are those of the final positions; the steps before the
 * last, whose energies the next step overwrites, skip the pair energies.
 * With use_graph != 0 one step is captured in a CUDA graph on first use
 * (and whenever a pointer or dt changes; one graph per pointer set, a few
 * sets kept) and replayed. The neighbour list is used as given (no
 * rebuild). head = n_neigh = nlist = NULL: the library's pair list
 * (esp_batch_build_pairlist). */
int esp_batch_md_run(esp_batch* b, void* stream, float* pos4, float* vel4, const float* charge, const unsigned* head,
                     const unsigned* n_neigh, const unsigned* nlist, float* force4, double* energy, double* virial6,
                     int nsteps, double dt, int use_graph);

/* FP64 form of esp_batch_md_run for contexts created with precision
 * ESP_FP64 (the C1 harness: HOOMD double builds integrating ESP with a
 * Lennard-Jones core): nsteps velocity-Verlet steps (esp_batch_nve_step1_f64,
 * a full FP64 evaluation over the caller's HOOMD-layout neighbour list, and,
 * when lj_sigma > 0, the Lennard-Jones term of esp_batch_lj_f64 added to the
 * forces, the per-particle energies and energy[s]; esp_batch_nve_step2_f64).
 * force4 must hold the forces of the current positions on entry (ESP plus
 * Lennard-Jones when it is on); on return force4, energy (ESP plus
 * Lennard-Jones) and virial (ESP only) are those of the final positions. Rigid
 * water set by esp_batch_set_rigid_water is kept rigid. use_graph as in
 * esp_batch_md_run: one captured step per pointer set, dt and Lennard-Jones
 * parameters, replayed. The per-step sequence of the integration loop of
 * HOOMD's TwoStepNVE around ESPForceCompute::computeForces
 * (src/ESPForceCompute.cc:96-127) in one call. */
int esp_batch_md_run_f64(esp_batch* b, void* stream, double* pos4, double* vel4, const double* charge,
                         const unsigned* head, const unsigned* n_neigh, const unsigned* nlist, double* force4,
                         double* energy, double* virial6, int nsteps, double dt, double lj_epsilon, double lj_sigma,
                         double lj_r_cut, int use_graph);

/* ---------------------------------------------------------------- serving
 * Continuous-batching request server (no counterpart in the reference, whose
 * ForceCompute serves one HOOMD simulation). A request is one system: a
 * neighbour-list build, one evaluation (ESP_ALL) and `nsteps` velocity-Verlet
 * steps, each with a full evaluation. A worker thread admits arrived requests
 * in arrival order while their device footprint fits the budget (particle,
 * mesh, neighbour-list and tile ranges of arenas allocated once at create),
 * keeps each admitted system's particles, sorted records, meshes and
 * influence table resident across its steps, and advances every admitted
 * system by one evaluation per round: one launch per stage over all of them
 * (the batched kernels), so requests that arrive while others run join the
 * next round and share its launches. Influence tables are cached by (cutoff,
 * box, mesh) across requests. All systems of a server share one split
 * bandwidth c (chosen from the target error); the mesh of each request
 * follows its box and cutoff. Host input and output buffers stay owned by the
 * caller and must stay valid until the request is done (page-locked memory
 * lets the copies run asynchronously). */
typedef struct esp_server esp_server;

typedef struct esp_server_config {
    esp_params params;        /* order, target_error, window, tile; rcut is per request */
    long long hbm_budget;     /* device bytes for all request state (arenas), >= 256 MB */
    int max_systems;          /* systems admitted at once (slots), 1..4096 */
    int max_particles;        /* largest single request */
} esp_server_config;

typedef struct esp_request {
    int N;                    /* particles */
    double Lx, Ly, Lz;        /* orthorhombic box */
    double rcut;              /* real-space cutoff of this system */
    double skin;              /* neighbour-list buffer: list radius rcut + skin */
    int nlist_cap;            /* neighbour-list row capacity; 0 = from the mean density */
    int nsteps;               /* NVE steps after the first evaluation */
    double dt;
    double arrival;           /* seconds after esp_server_start at which the request arrives */
    const float* pos4;        /* host, 4N floats (x, y, z, unused) */
    const float* vel4;        /* host, 4N floats (vx, vy, vz, mass); NULL when nsteps == 0 */
    const float* charge;      /* host, N floats */
    float* out_pos4;          /* host outputs after the last step, each may be NULL */
    float* out_vel4;
    float* out_force4;        /* forces and per-particle energies of the last evaluation */
    double* out_energy;       /* total energy of the last evaluation */
    double rigid_doh, rigid_dhh; /* > 0: the system is rigid water -- (O, H, H) triples, O-H and H-H
                                    distances, kept rigid by SETTLE / RATTLE in the NVE steps */
} esp_request;

typedef struct esp_request_status {
    int state;                /* 0 waiting, 1 running, 2 done, < 0 failed (ESP_ERR_*) */
    double t_arrival, t_admit, t_done;  /* seconds after esp_server_start */
    int nx, ny, nz;           /* mesh chosen for the request */
    long long footprint;      /* device bytes held while admitted */
} esp_request_status;

typedef struct esp_server_stats {
    long long submitted, completed, failed;
    long long rounds;         /* evaluation rounds launched */
    long long particle_steps; /* particle evaluations completed (N per evaluation) */
    long long influence_builds, influence_hits;
    int max_active;           /* largest number of systems admitted at once */
    long long peak_bytes;     /* largest footprint admitted at once */
    long long arena_bytes;    /* device bytes of the arenas */
} esp_server_stats;

int esp_server_create(const esp_server_config* cfg, esp_server** out);
/* Queues a request (arrival times must not decrease from one submit to the
 * next); `id` receives its index (0, 1, 2, ...). */
int esp_server_submit(esp_server* s, const esp_request* r, long long* id);
/* Starts the clock that arrival times count from (requests submitted before
 * start wait for it). */
int esp_server_start(esp_server* s);
int esp_server_status(esp_server* s, long long id, esp_request_status* st);
/* Blocks until every submitted request is done or failed, or timeout_s
 * passes (ESP_ERR_INVALID then). */
int esp_server_wait_all(esp_server* s, double timeout_s);
int esp_server_get_stats(esp_server* s, esp_server_stats* st);
int esp_server_destroy(esp_server* s);

/* ---------------------------------------------------------------- timing
 * Per-stage CUDA-event timing on the launching stream (no counterpart in
 * the reference, whose Autotuner times kernels for block-size selection,
 * src/ESPForceComputeGPU.cc:52-61). Enabling resets the totals; events are
 * recorded without synchronising; esp_batch_stage_times synchronises once,
 * returns total milliseconds and launch counts per stage, and resets.
 * Graph replays are not timed per stage. */
#define ESP_STAGE_BIN 0
#define ESP_STAGE_SORT 1
#define ESP_STAGE_SPREAD 2
#define ESP_STAGE_FFT 3
#define ESP_STAGE_INTERP 4
#define ESP_STAGE_PAIR 5
#define ESP_STAGE_NLIST 6
#define ESP_STAGE_NVE 7
#define ESP_N_STAGES 8
int esp_batch_set_timing(esp_batch* b, int on);
int esp_batch_stage_times(esp_batch* b, double* ms, long long* counts);

#ifdef __cplusplus
}
#endif

#endif /* ESP_B200_H_ */
