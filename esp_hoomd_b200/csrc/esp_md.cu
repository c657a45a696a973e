// MD harness kernels: cell-list neighbour list and velocity-Verlet halves.
// These stand in for the HOOMD-blue pieces the reference relies on
// (NeighborList and the integrator; not vendored in the reference) so the
// ESP path can run standalone.
#include "esp_cells.cuh"
#include "esp_common.cuh"
#include "esp_kernels.h"
#include "esp_md.h"

namespace espb {

// Cell of each particle (cells of edge >= rlist, at least 3 per axis).
__global__ void k_cell_bin(const int2* __restrict__ chunks, const SysDev* __restrict__ sys,
                           const CellDev* __restrict__ cells, const float4* __restrict__ pos,
                           uint32_t* __restrict__ ckey, uint32_t* __restrict__ ccount, float4* __restrict__ wpos) {
    const int2 ch = chunks[blockIdx.x];
    const SysDev& S = sys[ch.x];
    const CellDev& C = cells[ch.x];
    const int i = ch.y + threadIdx.x;
    const bool valid = i < S.p_off + S.N;
    const float4 p = valid ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    float x = p.x - S.Lx * floorf(p.x * S.inv_Lx);
    float y = p.y - S.Ly * floorf(p.y * S.inv_Ly);
    float z = p.z - S.Lz * floorf(p.z * S.inv_Lz);
    if (x >= S.Lx) x -= S.Lx;
    if (y >= S.Ly) y -= S.Ly;
    if (z >= S.Lz) z -= S.Lz;
    int cx = min((int)(x * C.inv_wx), C.ncx - 1), cy = min((int)(y * C.inv_wy), C.ncy - 1),
        cz = min((int)(z * C.inv_wz), C.ncz - 1);
    cx = max(cx, 0);
    cy = max(cy, 0);
    cz = max(cz, 0);
    const uint32_t k = valid ? (uint32_t)(C.c_off + (cz * C.ncy + cy) * C.ncx + cx) : 0xffffffffu;
    // one atomic per distinct cell of the warp
    const unsigned grp = __match_any_sync(0xffffffffu, k);
    if (!valid) return;
    if ((threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&ccount[k], (uint32_t)__popc(grp));
    ckey[i] = k;
    wpos[i] = make_float4(x, y, z, __int_as_float(i));
}

// Deterministic order inside each cell (ascending particle index) and the
// cell-sorted positions.
__global__ void k_cell_sort(const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm_u,
                            const float4* __restrict__ wpos, float4* __restrict__ cpos,
                            uint32_t* __restrict__ slot2idx, uint32_t* __restrict__ idx2slot) {
    __shared__ __align__(16) uint32_t sm[1024];
    const uint32_t s0 = start[blockIdx.x];
    const uint32_t n = start[blockIdx.x + 1] - s0;
    if (n == 0) return;
    const bool cached = n <= 1024u;
    const uint32_t n4 = (n + 3u) >> 2;
    if (cached) {
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sm[i] = perm_u[s0 + i];
        // pad to whole 16-byte groups with a value no index is above
        if (threadIdx.x < 4u * n4 - n) sm[n + threadIdx.x] = 0xffffffffu;
    }
    __syncthreads();
    const uint32_t* src = cached ? sm : perm_u + s0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t v = src[i];
        uint32_t r = 0;
        if (cached) {
            // rank = number of smaller indices, four per shared load
            for (uint32_t j = 0; j < n4; ++j) {
                const uint4 u = reinterpret_cast<const uint4*>(sm)[j];
                r += (u.x < v ? 1u : 0u) + (u.y < v ? 1u : 0u) + (u.z < v ? 1u : 0u) + (u.w < v ? 1u : 0u);
            }
        } else {
            for (uint32_t j = 0; j < n; ++j) r += (src[j] < v) ? 1u : 0u;
        }
        cpos[s0 + r] = wpos[v];
        if (slot2idx) slot2idx[s0 + r] = v;
        if (idx2slot) idx2slot[v] = s0 + r;
    }
}

// One CTA per cell, one thread per particle of the cell (passes of
// NL_THREADS). The particles of the 27 surrounding cells are staged in
// shared memory, in the fixed (dz, dy, dx) order and ascending slot inside
// each cell (in windows of NL_STAGE when there are more), so every row is
// deterministic; each thread scans them with broadcast shared loads (one
// wavefront serves the whole warp). With at least 3 cells on every axis each
// surrounding cell is a distinct periodic image and its particles are staged
// already shifted by that image, so the test needs no wrap; smaller cell
// grids take the minimum-image test.
constexpr int NL_THREADS = 64;
constexpr int NL_STAGE = 1024;

// Appends the staged candidates within rlist of pi, other than `self`, to
// row (staged values are already local indices or slots); threads without a
// particle carry a NaN position, which tests false against everything. Hits
// past cap are counted, and stored over the row's last entry (so an
// overflowing row still holds only neighbours; the build reports it).
// One candidate's test and append, as straight-line predicated code (no
// branch per candidate): stores w at p when r2 < rlist2 and w != self, and
// returns 1 then (0 otherwise).
__device__ __forceinline__ uint32_t append_if(float r2, float rlist2, int w, int self, uint32_t* p) {
    uint32_t inc;
    asm volatile(
        "{\n\t.reg .pred q, r;\n\tsetp.lt.f32 q, %1, %2;\n\tsetp.ne.s32 r, %3, %4;\n\tand.pred q, q, r;\n\t"
        "@q st.global.u32 [%5], %3;\n\tselp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(inc)
        : "f"(r2), "f"(rlist2), "r"(w), "r"(self), "l"(p)
        : "memory");
    return inc;
}

template <bool MINIMG>
__device__ __forceinline__ uint32_t nl_scan(const float4* __restrict__ cand, int n, float4 pi, int self,
                                            const SysDev& S, float rlist2, uint32_t cap, uint32_t* __restrict__ row,
                                            uint32_t cnt) {
    const uint32_t cap1 = cap - 1u;
#pragma unroll 4
    for (int k = 0; k < n; ++k) {
        const float4 pj = cand[k];
        float ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
        if (MINIMG) {
            ddx -= S.Lx * rintf(ddx * S.inv_Lx);
            ddy -= S.Ly * rintf(ddy * S.inv_Ly);
            ddz -= S.Lz * rintf(ddz * S.inv_Lz);
        }
        cnt += append_if(ddx * ddx + ddy * ddy + ddz * ddz, rlist2, __float_as_int(pj.w), self, row + min(cnt, cap1));
    }
    return cnt;
}

// SORTED = false: HOOMD-layout rows -- the row of particle i at nl_off +
// local i * cap, entries local particle indices, head/nn indexed by
// particle. SORTED = true: the library's pair list -- the same layout indexed
// by the cell-sorted slot (row of slot s at nl_off + local s * cap, head and
// nn by slot), entries local slots. Rows longer than cap keep their first cap
// entries and set the overflow flag; overflow[1] receives the longest row.
template <bool SORTED>
__global__ void __launch_bounds__(NL_THREADS) k_nlist(const int* __restrict__ cell_sys, const SysDev* __restrict__ sys,
                                                      const CellDev* __restrict__ cells,
                                                      const uint32_t* __restrict__ cstart,
                                                      const float4* __restrict__ cpos, float rlist2, int cap,
                                                      uint32_t* __restrict__ head, uint32_t* __restrict__ nn,
                                                      uint32_t* __restrict__ nl, int* __restrict__ overflow) {
    __shared__ float4 cand[NL_STAGE];
    __shared__ CellNbhd nb;
    const uint32_t cidx = blockIdx.x;
    const uint32_t c0 = cstart[cidx], c1 = cstart[cidx + 1];
    if (c0 == c1) return;
    const int si = cell_sys[cidx];
    const SysDev& S = sys[si];
    const CellDev& C = cells[si];
    const int tid = threadIdx.x;
    if (tid < 32) cell_nbhd_warp((int)cidx - C.c_off, C, S, cstart, nb);
    __syncthreads();
    const bool minimg = nb.minimg != 0;
    const uint32_t total = nb.off[27];
    // staged value: the candidate's local particle index (HOOMD rows; the
    // cell-sorted positions carry the index) or its local slot (pair list)
    auto stage = [&](uint32_t base) {
        const uint32_t top = min(total, base + (uint32_t)NL_STAGE);
        for (int s = 0; s < 27; ++s) {
            const uint32_t lo = max(nb.off[s], base), hi = min(nb.off[s + 1], top);
            for (uint32_t g = lo + tid; g < hi; g += NL_THREADS) {
                const uint32_t slot = nb.src[s] + (g - nb.off[s]);
                float4 p = cpos[slot];
                p.x += nb.shift[s][0];
                p.y += nb.shift[s][1];
                p.z += nb.shift[s][2];
                // local values: the pair list's slot, or the particle index
                p.w = __int_as_float((SORTED ? (int)slot : __float_as_int(p.w)) - S.p_off);
                cand[g - base] = p;
            }
        }
    };
    const bool one_stage = total <= (uint32_t)NL_STAGE;
    if (one_stage) {
        stage(0);
        __syncthreads();
    }
    for (uint32_t p0 = c0; p0 < c1; p0 += NL_THREADS) {
        const uint32_t slot = p0 + tid;
        const bool active = slot < c1;
        const float4 pi = active ? cpos[slot] : make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, __int_as_float(-1));
        const int idx = __float_as_int(pi.w);
        const int self = (SORTED ? (int)slot : idx) - S.p_off;
        const uint32_t key = SORTED ? slot : (uint32_t)idx;  // owner of the row
        const long long hrow = C.nl_off + (long long)((int)key - S.p_off) * cap;
        uint32_t* row = nl + (active ? hrow : 0);
        uint32_t cnt = 0;
        for (uint32_t base = 0; base < total; base += NL_STAGE) {
            if (!one_stage) {
                __syncthreads();
                stage(base);
                __syncthreads();
            }
            const int n = (int)min((uint32_t)NL_STAGE, total - base);
            cnt = minimg ? nl_scan<true>(cand, n, pi, self, S, rlist2, (uint32_t)cap, row, cnt)
                         : nl_scan<false>(cand, n, pi, self, S, rlist2, (uint32_t)cap, row, cnt);
        }
        if (active) {
            head[key] = (uint32_t)hrow;
            nn[key] = cnt;
            if (cnt > (uint32_t)cap) {
                atomicOr(overflow, 1);
                atomicMax(overflow + 1, (int)cnt);
            }
        }
    }
}

// Leaves the excluded partners out of the rows just built (HOOMD's lists
// hold no excluded pairs): one thread per row with exclusions, in place, the
// kept entries in their order; the count drops by the entries removed from
// the stored part. Pair-list rows hold slots, so the excluded indices are
// mapped to slots first.
constexpr int NL_MAXEX = 8;  // exclusions per particle held in registers

template <bool SORTED>
__global__ void k_nlist_exclude(const int2* __restrict__ chunks, const SysDev* __restrict__ sys,
                                const uint32_t* __restrict__ head, uint32_t* __restrict__ nn,
                                uint32_t* __restrict__ nl, int cap, const uint32_t* __restrict__ ex_n,
                                const uint32_t* __restrict__ ex_list, int ex_pitch,
                                const uint32_t* __restrict__ slot2idx, const uint32_t* __restrict__ idx2slot) {
    const int2 ch = chunks[blockIdx.x];
    const SysDev& S = sys[ch.x];
    const int key = ch.y + threadIdx.x;  // the row: a slot (pair list) or a particle
    if (key >= S.p_off + S.N) return;
    const int i = SORTED ? (int)slot2idx[key] : key;
    const int ne = min((int)ex_n[i], ex_pitch);
    if (ne == 0) return;
    uint32_t ex[NL_MAXEX];
#pragma unroll
    for (int k = 0; k < NL_MAXEX; ++k) {
        uint32_t v = 0xffffffffu;
        if (k < ne) {
            const uint32_t jl = ex_list[(size_t)i * ex_pitch + k];
            v = SORTED ? idx2slot[S.p_off + jl] - (uint32_t)S.p_off : jl;
        }
        ex[k] = v;
    }
    uint32_t* row = nl + head[key];
    const uint32_t cnt = nn[key];
    const uint32_t n = min(cnt, (uint32_t)cap);
    uint32_t w = 0;
    for (uint32_t r = 0; r < n; ++r) {
        const uint32_t v = row[r];
        bool drop = false;
#pragma unroll
        for (int k = 0; k < NL_MAXEX; ++k) drop |= v == ex[k];
        for (int k = NL_MAXEX; k < ne; ++k) {  // rows with more exclusions than registers hold
            const uint32_t jl = ex_list[(size_t)i * ex_pitch + k];
            drop |= v == (SORTED ? idx2slot[S.p_off + jl] - (uint32_t)S.p_off : jl);
        }
        if (!drop) row[w++] = v;
    }
    nn[key] = cnt - (n - w);
}

// skip (may be NULL): per system, the local particle range [x, y) of rigid
// molecules, which the constraint kernels integrate instead
__global__ void k_nve1(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, float4* __restrict__ pos,
                       float4* __restrict__ vel, const float4* __restrict__ force, float dt,
                       const int2* __restrict__ skip) {
    const int2 ch = chunks[blockIdx.x];
    const SysDev& S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    if (i >= S.p_off + S.N) return;
    if (skip) {
        const int2 r = skip[ch.x];
        if (i - S.p_off >= r.x && i - S.p_off < r.y) return;
    }
    float4 v = vel[i];
    const float4 f = force[i];
    const float h = 0.5f * dt / v.w;
    v.x += h * f.x;
    v.y += h * f.y;
    v.z += h * f.z;
    float4 p = pos[i];
    p.x += dt * v.x;
    p.y += dt * v.y;
    p.z += dt * v.z;
    p.x -= S.Lx * floorf(p.x * S.inv_Lx);
    p.y -= S.Ly * floorf(p.y * S.inv_Ly);
    p.z -= S.Lz * floorf(p.z * S.inv_Lz);
    if (p.x >= S.Lx) p.x -= S.Lx;
    if (p.y >= S.Ly) p.y -= S.Ly;
    if (p.z >= S.Lz) p.z -= S.Lz;
    pos[i] = p;
    vel[i] = v;
}

__global__ void k_nve2(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, float4* __restrict__ vel,
                       const float4* __restrict__ force, float dt) {
    const int2 ch = chunks[blockIdx.x];
    const SysDev& S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    if (i >= S.p_off + S.N) return;
    float4 v = vel[i];
    const float4 f = force[i];
    const float h = 0.5f * dt / v.w;
    v.x += h * f.x;
    v.y += h * f.y;
    v.z += h * f.z;
    vel[i] = v;
}

// Lennard-Jones core repulsion of the MD harness (the C1 workload's
// LJ eps, sigma, r_cut), over the same full neighbour list: adds forces and
// half the pair energy per particle to force, the system total to energy[s].
template <typename T4, typename T>
__global__ void k_lj(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, const T4* __restrict__ pos,
                     const uint32_t* __restrict__ head, const uint32_t* __restrict__ nn,
                     const uint32_t* __restrict__ nl, T eps, T sig2, T rc2, T4* __restrict__ force,
                     double* __restrict__ energy) {
    __shared__ double red[32];
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    const T L[3] = {(T)S.Lxd, (T)S.Lyd, (T)S.Lzd};
    double e1[1] = {0.0};
    if (i < S.p_off + S.N) {
        const T4 pi = pos[i];
        T fx = 0, fy = 0, fz = 0, en = 0;
        const uint32_t h = head[i], n = nn[i];
        for (uint32_t k = 0; k < n; ++k) {
            const T4 pj = pos[S.p_off + (int)nl[h + k]];
            T d[3] = {pi.x - pj.x, pi.y - pj.y, pi.z - pj.z};
            for (int a = 0; a < 3; ++a) d[a] -= L[a] * rint(d[a] / L[a]);
            const T r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (r2 < rc2 && r2 > 0) {
                const T s2 = sig2 / r2, s6 = s2 * s2 * s2;
                const T fdr = (T)24 * eps * ((T)2 * s6 * s6 - s6) / r2;
                en += (T)4 * eps * (s6 * s6 - s6);
                fx += fdr * d[0];
                fy += fdr * d[1];
                fz += fdr * d[2];
            }
        }
        T4 f = force[i];
        f.x += fx;
        f.y += fy;
        f.z += fz;
        f.w += (T)0.5 * en;
        force[i] = f;
        e1[0] = 0.5 * (double)en;
    }
    block_sum_f64<1>(e1, red);
    if (threadIdx.x == 0 && energy) atomicAdd(&energy[ch.x], e1[0]);
}

__global__ void k64_nve1(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, double4* __restrict__ pos,
                         double4* __restrict__ vel, const double4* __restrict__ force, double dt,
                         const int2* __restrict__ skip) {
    const int2 ch = chunks[blockIdx.x];
    const SysDev& S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    if (i >= S.p_off + S.N) return;
    if (skip) {
        const int2 r = skip[ch.x];
        if (i - S.p_off >= r.x && i - S.p_off < r.y) return;
    }
    double4 v = vel[i];
    const double4 f = force[i];
    const double h = 0.5 * dt / v.w;
    v.x += h * f.x;
    v.y += h * f.y;
    v.z += h * f.z;
    double4 p = pos[i];
    const double L[3] = {S.Lxd, S.Lyd, S.Lzd};
    double x[3] = {p.x + dt * v.x, p.y + dt * v.y, p.z + dt * v.z};
    for (int a = 0; a < 3; ++a) {
        x[a] -= L[a] * floor(x[a] / L[a]);
        if (x[a] >= L[a]) x[a] -= L[a];
        if (x[a] < 0.0) x[a] += L[a];
    }
    pos[i] = make_double4(x[0], x[1], x[2], p.w);
    vel[i] = v;
}

__global__ void k64_nve2(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, double4* __restrict__ vel,
                         const double4* __restrict__ force, double dt) {
    const int2 ch = chunks[blockIdx.x];
    const SysDev& S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    if (i >= S.p_off + S.N) return;
    double4 v = vel[i];
    const double4 f = force[i];
    const double h = 0.5 * dt / v.w;
    v.x += h * f.x;
    v.y += h * f.y;
    v.z += h * f.z;
    vel[i] = v;
}

cudaError_t launch_lj(const int2* chunks, int n_chunks, const SysDev* sys, const void* pos, const uint32_t* head,
                      const uint32_t* nn, const uint32_t* nl, double eps, double sigma, double rcut, void* force,
                      double* energy, bool f64, cudaStream_t st) {
    if (n_chunks == 0) return cudaSuccess;
    if (f64)
        k_lj<double4, double><<<n_chunks, 256, 0, st>>>(chunks, sys, (const double4*)pos, head, nn, nl, eps,
                                                        sigma * sigma, rcut * rcut, (double4*)force, energy);
    else
        k_lj<float4, float><<<n_chunks, 256, 0, st>>>(chunks, sys, (const float4*)pos, head, nn, nl, (float)eps,
                                                      (float)(sigma * sigma), (float)(rcut * rcut), (float4*)force,
                                                      energy);
    return cudaGetLastError();
}

cudaError_t launch_nve64(int half, const int2* chunks, int n_chunks, const SysDev* sys, double4* pos, double4* vel,
                         const double4* force, double dt, cudaStream_t st, const int2* skip) {
    if (n_chunks == 0) return cudaSuccess;
    if (half == 1) k64_nve1<<<n_chunks, 256, 0, st>>>(chunks, sys, pos, vel, force, dt, skip);
    else k64_nve2<<<n_chunks, 256, 0, st>>>(chunks, sys, vel, force, dt);
    return cudaGetLastError();
}

cudaError_t launch_nlist(const NlistArgs& a, cudaStream_t st) {
    if (a.n_chunks == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(a.overflow, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) return e;
    k_cell_bin<<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.cells, a.pos, a.ckey, a.ccount, a.wpos);
    if ((e = launch_scan(a.ccount, a.cstart, a.n_cells, st)) != cudaSuccess) return e;
    if ((e = launch_scatter(a.chunks, a.n_chunks, a.sys, a.ckey, a.cstart, a.ccount, a.perm_u, st)) != cudaSuccess)
        return e;
    k_cell_sort<<<a.n_cells, 256, 0, st>>>(a.cstart, a.perm_u, a.wpos, a.cpos, a.slot2idx, a.idx2slot);
    if (a.sorted)
        k_nlist<true><<<a.n_cells, NL_THREADS, 0, st>>>(a.cell_sys, a.sys, a.cells, a.cstart, a.cpos, a.rlist2,
                                                        a.cap, a.head, a.nn, a.nl, a.overflow);
    else
        k_nlist<false><<<a.n_cells, NL_THREADS, 0, st>>>(a.cell_sys, a.sys, a.cells, a.cstart, a.cpos, a.rlist2,
                                                         a.cap, a.head, a.nn, a.nl, a.overflow);
    if (a.ex_n) {
        if (a.sorted)
            k_nlist_exclude<true><<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.head, a.nn, a.nl, a.cap, a.ex_n,
                                                               a.ex_list, a.ex_pitch, a.slot2idx, a.idx2slot);
        else
            k_nlist_exclude<false><<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.head, a.nn, a.nl, a.cap, a.ex_n,
                                                                a.ex_list, a.ex_pitch, a.slot2idx, a.idx2slot);
    }
    return cudaGetLastError();
}

cudaError_t launch_nve1(const int2* chunks, int n_chunks, const SysDev* sys, float4* pos, float4* vel,
                        const float4* force, float dt, cudaStream_t st, const int2* skip) {
    if (n_chunks == 0) return cudaSuccess;
    k_nve1<<<n_chunks, 256, 0, st>>>(chunks, sys, pos, vel, force, dt, skip);
    return cudaGetLastError();
}

cudaError_t launch_nve2(const int2* chunks, int n_chunks, const SysDev* sys, float4* vel, const float4* force,
                        float dt, cudaStream_t st) {
    if (n_chunks == 0) return cudaSuccess;
    k_nve2<<<n_chunks, 256, 0, st>>>(chunks, sys, vel, force, dt);
    return cudaGetLastError();
}

}  // namespace espb
