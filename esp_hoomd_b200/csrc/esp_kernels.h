// Internal launch interface between the host orchestration (esp_host.cu)
// and the kernels (esp_kernels.cu, esp_md.cu). Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "esp_common.cuh"

namespace espb {

constexpr int SORT_CAP = 2048;  // particles per tile sorted in shared memory
constexpr int FFT_SMEM_MAX = 220 * 1024;  // shared memory of the plane / slab FFT passes

// shared memory (bytes) of the plane pass of an nx x ny plane and of the z
// pass of an nz x nxh slab; line strides are rounded up to odd numbers
// (two line buffers plus the twiddles of the transformed axes)
inline int fft_plane_smem(int nx, int ny) {
    const int np = (ny + 1) / 2, nxh = nx / 2 + 1;
    const int c = std::max(nx * (np | 1), ny * (nxh | 1));
    return (2 * c + nx + ny) * 8;
}
inline int fft_slab_smem(int nx, int nz) { return (2 * nz * ((nx / 2 + 1) | 1) + nz) * 8; }

// Split-polynomial coefficients of a batch, passed by value so the pair
// kernel's FMAs read them from the kernel-parameter constant bank.
struct PairCoef {
    float q[MAX_QC];  // Q(v)
    float d[MAX_QC];  // dQ/du in v
};

// The library's pair list: rows indexed by the cell-sorted slot of its
// build (head/nn/nl in the HOOMD layout, entries local slots), the slot <->
// particle maps of that build, and the slot-ordered copy of the wrapped
// positions and charges that the bin stage writes every evaluation (so that
// a row's neighbours are neighbours in memory too).
struct PairList {
    const uint32_t* slot2idx = nullptr;  // slot -> particle (concatenated index)
    const uint32_t* idx2slot = nullptr;  // particle -> slot
    float4* spos = nullptr;              // {x, y, z, q} by slot
    const uint32_t* head = nullptr;
    const uint32_t* nn = nullptr;
    const uint32_t* nl = nullptr;
    int cap = 0;
};

struct LaunchArgs {
    PairCoef pc{};
    const PairList* plist = nullptr;  // non-null: short-range term over the library's pair list
    const SysDev* sys = nullptr;
    const ParamSet* psets = nullptr;
    int nsys = 0, P = 8, T = 8, D = 10, PX = 0, PP = 0, tpp = 8, accumulate = 0, nq = 16;
    const int2* chunks = nullptr;   // {sys, first particle}, 256 particles each
    int n_chunks = 0;
    const int2* pchunks = nullptr;  // {sys, first particle}, 256/tpp particles each
    int n_pchunks = 0;
    const int* tile_sys = nullptr;
    int n_tiles = 0;
    uint32_t* tile_count = nullptr;
    uint32_t* tile_start = nullptr;
    const float4* pos_in = nullptr;
    const float* q_in = nullptr;
    float4* posq = nullptr;
    float4* trec = nullptr;
    uint32_t* rel = nullptr;
    uint32_t* key = nullptr;
    uint32_t* perm_u = nullptr;
    uint32_t* perm = nullptr;
    float4* srec = nullptr;
    uint32_t* srel = nullptr;
    double* rho = nullptr;
    float2* spec = nullptr;
    float* phi = nullptr;
    const float2* gtab = nullptr;
    const float2* tw = nullptr;
    const int4* xitems = nullptr;
    int n_xitems = 0;
    const int4* yitems = nullptr;
    int n_yitems = 0;
    const int4* zitems = nullptr;
    int n_zitems = 0;
    const int2* pitems = nullptr;  // {sys, z}: whole-plane x/y passes
    int n_pitems = 0;
    const int2* sitems = nullptr;  // {sys, y}: whole-slab z pass
    int n_sitems = 0;
    int smem_plane = 0, smem_slab = 0;
    float4* force = nullptr;
    double* acc = nullptr;
    double* energy = nullptr;
    double* virial = nullptr;
    int add_bg = 1;
    int want_virial = 1;
    int want_energy = 1;  // pair energies; 0 only inside MD steps whose energies are overwritten
    int spread_mode = 0;  // 0: tensor-core spreading when E == 16; 1: CUDA-core kernels  // accumulate the pair virial (skipped when no virial is requested)
    int configure_only = 0;
    int nmax_x = FFT_MAX_N, nmax_y = FFT_MAX_N, nmax_z = FFT_MAX_N;  // longest line per axis  // set kernel attributes (plan time) instead of launching
    const uint32_t* nl_head = nullptr;
    const uint32_t* nl_n = nullptr;
    const uint32_t* nl_list = nullptr;
    // HOOMD ForceCompute outputs: per-particle virial virial_pp[k * vpp_pitch + i]
    // (k = xx, xy, xz, yy, yz, zz; pair and exclusion terms, cleared by the
    // host first) and per system the terms no particle owns,
    // external[7 s] = {E_bg, W_k + E_bg I (6)}
    float* virial_pp = nullptr;
    int vpp_pitch = 0;
    double* external = nullptr;
    // TMA-staged interpolation: per-system tensor maps of the halo-padded
    // potential mesh (CUtensorMap[nsys], NULL: cp.async staging), the box's
    // x extent and rows (pitches of the staged region), and the kernels'
    // error word (bit 0: a TMA wait ran out)
    const void* tmaps = nullptr;
    int tma_bx = 0, tma_by = 0;
    int* kerr = nullptr;
    // tile-queue counter of the persistent interpolation kernel (device int;
    // NULL: one CTA per tile)
    int* queue = nullptr;
    const uint32_t* ex_n = nullptr;     // exclusions: row i holds ex_list[i * ex_pitch + k], k < ex_n[i]
    const uint32_t* ex_list = nullptr;
    int ex_pitch = 0;
};

cudaError_t launch_scan(const uint32_t* cnt, uint32_t* start, int n, cudaStream_t st);
cudaError_t launch_scatter(const int2* chunks, int n_chunks, const SysDev* sys, const uint32_t* key,
                           const uint32_t* start, uint32_t* cnt, uint32_t* perm_u, cudaStream_t st);
cudaError_t launch_bin(const LaunchArgs& a, cudaStream_t st);
cudaError_t launch_sort(const LaunchArgs& a, cudaStream_t st);
cudaError_t launch_spread(const LaunchArgs& a, cudaStream_t st);
cudaError_t launch_fft(const LaunchArgs& a, cudaStream_t st);
cudaError_t launch_interp(const LaunchArgs& a, cudaStream_t st);
cudaError_t launch_pair(const LaunchArgs& a, cudaStream_t st);
cudaError_t launch_exclusions(const LaunchArgs& a, cudaStream_t st);
cudaError_t launch_add_forces(const int2* chunks, int n_chunks, const SysDev* sys, const float4* add, float4* force,
                              cudaStream_t st);

// FP64 mode (esp_f64.cu): the shared fields of `a` (descriptors, chunks,
// tiles, keys, permutation, charge mesh, accumulators, neighbour list,
// exclusions) plus the FP64 arrays.
struct Launch64 {
    LaunchArgs a;
    bool long_range = true, short_range = true;
    const double4* pos_in = nullptr;
    const double* q_in = nullptr;
    double4 *posq = nullptr, *trec = nullptr, *srec = nullptr, *force = nullptr;
    const double* wcoef = nullptr;  // window [P][D+1]
    const double* qv = nullptr;     // split Q(v) coefficients
    int nq = 0;
    const double2* tw = nullptr;    // exp(-2 pi i t / n) per axis length
    double2* cbuf = nullptr;        // full complex spectrum
    double* phi = nullptr;          // potential mesh
    const double2* gtab = nullptr;  // {G, G B} half spectrum
    const int2* pchunks = nullptr;  // 32 particles per chunk (8 lanes per particle)
    int n_pchunks = 0;
    const int2 *xl = nullptr, *yl = nullptr, *zl = nullptr;  // {sys, first line}, 4 lines per item
    int n_xl = 0, n_yl = 0, n_zl = 0;
};
size_t spread64_smem(int P, int T);
cudaError_t launch64_configure(int P, int T);
cudaError_t launch64_eval(const Launch64& b, cudaStream_t st);
cudaError_t launch_influence64(const SysDev& S, const double* w1d, const double* tq, const double* wq, int nq,
                               double rcut, double psi_floor, double2* gtab, cudaStream_t st);
cudaError_t launch_finalize(const LaunchArgs& a, cudaStream_t st);
cudaError_t launch_influence(const SysDev& S, const double* w1d, const double* tq, const double* wq, int nq,
                             double rcut, double psi_floor, float2* gtab, cudaStream_t st);
cudaError_t launch_pswf_eval_pairs(int n, const double* rsq, const double* qiqj, double rcut, int n_segs,
                                   const double* screen, const double* dscreen, const double* r_lo,
                                   const double* dr_inv, double* force_divr, double* pair_eng, int* evaluated,
                                   cudaStream_t st);

}  // namespace espb
