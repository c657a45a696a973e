// Internal launch interface of the MD harness kernels (esp_md.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "esp_common.cuh"

namespace espb {

struct CellDev {
    int ncx, ncy, ncz, c_off;  // cell grid and first cell
    float inv_wx, inv_wy, inv_wz;
    long long nl_off;          // first neighbour-list entry of this system (HOOMD-layout rows)
};

struct NlistArgs {
    const int2* chunks = nullptr;
    int n_chunks = 0;
    const SysDev* sys = nullptr;
    const CellDev* cells = nullptr;
    const int* cell_sys = nullptr;
    int n_cells = 0;
    int total = 0;
    const float4* pos = nullptr;
    uint32_t* ckey = nullptr;
    uint32_t* ccount = nullptr;
    uint32_t* cstart = nullptr;
    uint32_t* perm_u = nullptr;
    float4* wpos = nullptr;
    float4* cpos = nullptr;
    float rlist2 = 0.f;
    int cap = 0;
    uint32_t* head = nullptr;
    uint32_t* nn = nullptr;
    uint32_t* nl = nullptr;
    int* overflow = nullptr;
    uint32_t* slot2idx = nullptr;  // cell-sorted slot -> particle (written by the cell sort)
    uint32_t* idx2slot = nullptr;  // particle -> cell-sorted slot (may be NULL)
    // true: the library's pair list -- rows, head and counts indexed by the
    // cell-sorted slot, entries local slots; false: HOOMD-layout rows
    // (indexed by particle, entries local particle indices)
    bool sorted = false;
    // exclusions (HOOMD's n_ex / ex_list layout, rows by particle, local
    // indices): when set, the built rows leave the excluded partners out
    const uint32_t* ex_n = nullptr;
    const uint32_t* ex_list = nullptr;
    int ex_pitch = 0;
};

cudaError_t launch_nlist(const NlistArgs& a, cudaStream_t st);
// skip: per-system local ranges of rigid molecules left to launch_settle1 (may be NULL)
cudaError_t launch_nve1(const int2* chunks, int n_chunks, const SysDev* sys, float4* pos, float4* vel,
                        const float4* force, float dt, cudaStream_t st, const int2* skip = nullptr);
cudaError_t launch_nve2(const int2* chunks, int n_chunks, const SysDev* sys, float4* vel, const float4* force,
                        float dt, cudaStream_t st);
cudaError_t launch_lj(const int2* chunks, int n_chunks, const SysDev* sys, const void* pos, const uint32_t* head,
                      const uint32_t* nn, const uint32_t* nl, double eps, double sigma, double rcut, void* force,
                      double* energy, bool f64, cudaStream_t st);
cudaError_t launch_nve64(int half, const int2* chunks, int n_chunks, const SysDev* sys, double4* pos, double4* vel,
                         const double4* force, double dt, cudaStream_t st, const int2* skip = nullptr);
// Rigid (O, H, H) molecules (esp_settle.cu): work items {system, first atom
// (concatenated index), molecules <= SETTLE_CHUNK, geometry index into geo
// = (d_OH, d_HH)}, one CTA each; f64 selects double4 arrays. settle1: first
// velocity-Verlet half with SETTLE; settle2: RATTLE velocity constraint after
// the second half kick.
constexpr int SETTLE_CHUNK = 128;
cudaError_t launch_settle1(const int4* items, int n_items, const SysDev* sys, void* pos, void* vel,
                           const void* force, double dt, const double2* geo, bool f64, cudaStream_t st);
cudaError_t launch_settle2(const int4* items, int n_items, const SysDev* sys, const void* pos, void* vel, bool f64,
                           cudaStream_t st);

}  // namespace espb
