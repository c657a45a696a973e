// The library's cell-staged pair list and its pair kernel: the short-range
// term (EvaluatorPairPSWF, src/EvaluatorPairPSWF.h:274-295, over the
// neighbour loop HOOMD's PotentialPairGPU runs, src/module.cc:79) when the
// library builds the neighbour list itself. Lists the caller supplies in
// HOOMD's layout go through k_pair (esp_kernels.cu) unchanged.
//
// One CTA serves one cell of the list's cell grid. It stages the current
// positions of the particles of the 27 surrounding cells in shared memory,
// once, in the fixed enumeration order of esp_cells.cuh; a neighbour entry is
// the 16-bit index of the neighbour in that staging (its "staged index"), so
// a pair costs one 16-byte shared load instead of a gather from global memory
// in the caller's particle order, and the index stream is half the bytes of
// a 32-bit list. Each row is packed so that the 8 lanes serving a particle
// read 8 different 16-byte bank groups in every shared load.
//
// Positions are staged as the periodic image nearest to the centre of the
// CTA's cell: with at least 4 cells on every axis a neighbour cell's
// particles lie within 1.5 cell edges plus half the list's skin of that
// centre, less than half the box, so every staged image is the one the pair
// needs and no per-pair wrap is done. Grids with fewer cells on an axis keep
// the wrapped positions and take the minimum image per pair.
#include "esp_cells.cuh"
#include "esp_common.cuh"
#include "esp_kernels.h"
#include "esp_md.h"
#include "esp_pair.cuh"

namespace espb {

// ============================================================================
// Row packing. Entry class = staged index mod 8 = the 16-byte bank group of
// its staged position (the staging starts at offset 0 of shared memory). A
// row of n entries with per-class counts n_c and m = min_c n_c becomes
//   positions [0, 8m): groups r = 0..m-1 of 8 entries, group r holding the
//     r-th entry of every class, class c at position 8r + ((c - r) mod 8);
//   positions [8m, n): the remaining entries, class by class;
// the builder's padding (positions n .. up to a multiple of 8) stays. The
// pair kernel's lane l (of 8) takes groups l, l + 8, l + 16, ... and reads
// position e of its group in step e, which in a full group is class
// (e + l) mod 8: the 8 lanes of a particle read 8 distinct bank groups.
// One warp per row; entries keep their order within a class.
// ============================================================================
constexpr int PACK_WARPS = 8;

__global__ void __launch_bounds__(PACK_WARPS * 32)
    k_pairlist_pack(int rows, const uint32_t* __restrict__ nn, uint16_t* __restrict__ nl16, int cap) {
    extern __shared__ uint16_t pk[];  // per warp: the row in, the row out
    __shared__ int cnt_s[PACK_WARPS][8], run_s[PACK_WARPS][8], ex_s[PACK_WARPS][8];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = blockIdx.x * PACK_WARPS + w;
    if (r >= rows) return;  // warp-uniform
    const uint32_t n = min(nn[r], (uint32_t)cap);
    uint16_t* row = nl16 + (size_t)r * cap;
    uint16_t* in = pk + (size_t)w * 2 * cap;
    uint16_t* out = in + cap;
    if (lane < 8) {
        cnt_s[w][lane] = 0;
        run_s[w][lane] = 0;
    }
    for (uint32_t k = lane; k < n; k += 32) in[k] = row[k];
    __syncwarp();
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
        const uint32_t k = k0 + lane;
        const int c = k < n ? (int)(in[k] & 7u) : 8;
        const unsigned grp = __match_any_sync(0xffffffffu, c);
        if (c < 8 && lane == __ffs(grp) - 1) cnt_s[w][c] += __popc(grp);
        __syncwarp();
    }
    int m = 0;
    if (lane == 0) {
        m = cnt_s[w][0];
        for (int c = 1; c < 8; ++c) m = min(m, cnt_s[w][c]);
        int e = 0;
        for (int c = 0; c < 8; ++c) {
            ex_s[w][c] = e;
            e += cnt_s[w][c] - m;
        }
    }
    m = __shfl_sync(0xffffffffu, m, 0);
    __syncwarp();
    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
        const uint32_t k = k0 + lane;
        const int c = k < n ? (int)(in[k] & 7u) : 8;
        const unsigned grp = __match_any_sync(0xffffffffu, c);
        if (c < 8) {
            const int rank = run_s[w][c] + __popc(grp & lt);
            const int pos = rank < m ? 8 * rank + ((c - rank) & 7) : 8 * m + ex_s[w][c] + (rank - m);
            out[pos] = in[k];
        }
        __syncwarp();
        if (c < 8 && lane == __ffs(grp) - 1) run_s[w][c] += __popc(grp);
        __syncwarp();
    }
    for (uint32_t k = lane; k < n; k += 32) row[k] = out[k];
}

// ============================================================================
// The pair kernel.
// ============================================================================
constexpr int PC_THREADS = 128;  // 16 particles x 8 lanes per pass
constexpr int PC_LANES = 8;

size_t pair_cells_smem(int stage_cap) {
    return (size_t)(stage_cap + 1) * 16 + ((sizeof(CellNbhd) + 15) & ~(size_t)15) + 32 * 7 * sizeof(double);
}

// The groups of one row taken by this lane: stg holds staged indices
// [base, top) at [0, top - base); WIN: entries outside the window are
// skipped (neighbourhoods larger than the staging capacity).
template <int NQ, bool VIR, bool EN, bool MIN, bool WIN>
__device__ __forceinline__ void pc_row(PairEval<NQ, VIR, EN>& ev, const float4& pi, const uint4* __restrict__ row,
                                       uint32_t ng, uint32_t sub, const float4* __restrict__ stg, uint32_t base,
                                       uint32_t top) {
    uint4 en = sub < ng ? __ldg(&row[sub]) : make_uint4(0u, 0u, 0u, 0u);
    for (uint32_t gi = sub; gi < ng; gi += PC_LANES) {
        const uint4 e = en;  // this group; the next one is loaded ahead
        if (gi + PC_LANES < ng) en = __ldg(&row[gi + PC_LANES]);
        const uint32_t w4[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
        for (int h = 0; h < 4; ++h) {
#pragma unroll
            for (int hi = 0; hi < 2; ++hi) {
                const uint32_t g = hi ? (w4[h] >> 16) : (w4[h] & 0xffffu);
                if (WIN) {
                    if (g - base < top - base) ev.template pair<MIN, true>(pi, stg[g - base]);
                } else {
                    ev.template pair<MIN, true>(pi, stg[g]);
                }
            }
        }
    }
}

template <int NQ, bool VIR, bool EN>
__global__ void __launch_bounds__(PC_THREADS)
    k_pair_cells(const int* __restrict__ cell_sys, const SysDev* __restrict__ sys, const CellDev* __restrict__ cells,
                 const ParamSet* __restrict__ psets, const uint32_t* __restrict__ cstart,
                 const uint32_t* __restrict__ slot2idx, const float4* __restrict__ posq,
                 const uint32_t* __restrict__ nn, const uint16_t* __restrict__ nl16, int cap, int stage_cap,
                 float4* __restrict__ force, double* __restrict__ acc, int accumulate, const PairCoef pc,
                 float* __restrict__ vpp, int vpitch) {
    extern __shared__ __align__(128) unsigned char pc_smem[];
    float4* stg = reinterpret_cast<float4*>(pc_smem);
    CellNbhd& nb = *reinterpret_cast<CellNbhd*>(pc_smem + (size_t)(stage_cap + 1) * 16);
    double* red = reinterpret_cast<double*>(pc_smem + (size_t)(stage_cap + 1) * 16 +
                                            ((sizeof(CellNbhd) + 15) & ~(size_t)15));
    const uint32_t cidx = blockIdx.x;
    const uint32_t c0 = cstart[cidx], c1 = cstart[cidx + 1];
    if (c0 == c1) return;  // CTA-uniform
    const int si = cell_sys[cidx];
    const SysDev& S = sys[si];
    const CellDev& C = cells[si];
    const ParamSet& ps = psets[S.pset];
    const int tid = threadIdx.x;
    const int lc = (int)cidx - C.c_off;
    if (tid < 32) cell_nbhd_warp(lc, C, S, cstart, nb);
    __syncthreads();
    const uint32_t total = nb.off[27];
    const bool minimg = C.ncx < 4 || C.ncy < 4 || C.ncz < 4;
    const int cx = lc % C.ncx, cy = (lc / C.ncx) % C.ncy, cz = lc / (C.ncx * C.ncy);
    const float ox = (cx + 0.5f) * (S.Lx / C.ncx), oy = (cy + 0.5f) * (S.Ly / C.ncy),
                oz = (cz + 0.5f) * (S.Lz / C.ncz);
    auto fetch = [&](uint32_t slot) -> float4 {
        float4 p = posq[slot2idx[slot]];
        if (!minimg) {
            p.x -= S.Lx * rintf((p.x - ox) * S.inv_Lx);
            p.y -= S.Ly * rintf((p.y - oy) * S.inv_Ly);
            p.z -= S.Lz * rintf((p.z - oz) * S.inv_Lz);
        }
        return p;
    };
    const uint32_t scap = (uint32_t)stage_cap;
    auto stage = [&](uint32_t base) {
        const uint32_t top = min(total, base + scap);
        for (int s = 0; s < 27; ++s) {
            const uint32_t lo = max(nb.off[s], base), hi = min(nb.off[s + 1], top);
            for (uint32_t g = lo + tid; g < hi; g += PC_THREADS) stg[g - base] = fetch(nb.src[s] + (g - nb.off[s]));
        }
        // the rows' padding index (= total): a zero-charge particle far away
        if (tid == 0) stg[top - base] = make_float4(1e30f, 1e30f, 1e30f, 0.f);
    };
    const bool one = total <= scap;
    if (one) {
        stage(0);
        __syncthreads();
    }
    PairEval<NQ, VIR, EN> ev{pc};
    ev.rc2 = ps.rcut2;
    ev.irc = ps.inv_rcut;
    ev.irc2 = ps.inv_rcut * ps.inv_rcut;
    ev.tirc3 = ps.two_inv_rcut3;
    ev.Lx = S.Lx;
    ev.Ly = S.Ly;
    ev.Lz = S.Lz;
    ev.iLx = S.inv_Lx;
    ev.iLy = S.inv_Ly;
    ev.iLz = S.inv_Lz;
    const uint32_t sub = (uint32_t)tid & (PC_LANES - 1);
    double en_sys = 0.0;
    float vt[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // this lane's pair virial over all its particles
    for (uint32_t p0 = c0; p0 < c1; p0 += PC_THREADS / PC_LANES) {
        const uint32_t slot = p0 + (uint32_t)tid / PC_LANES;
        const bool valid = slot < c1;
        float4 pi = valid ? fetch(slot) : make_float4(0.f, 0.f, 0.f, 0.f);
        pi.w *= INV_4PI_F;
        const uint32_t n = valid ? min(nn[slot], (uint32_t)cap) : 0u;
        const uint32_t ng = (n + 7u) >> 3;
        const uint4* row = reinterpret_cast<const uint4*>(nl16 + (size_t)(valid ? slot : 0u) * cap);
        ev.fx = ev.fy = ev.fz = ev.en = 0.f;
        if (one) {
            if (minimg) pc_row<NQ, VIR, EN, true, false>(ev, pi, row, ng, sub, stg, 0u, total);
            else pc_row<NQ, VIR, EN, false, false>(ev, pi, row, ng, sub, stg, 0u, total);
        } else {
            for (uint32_t base = 0; base < total; base += scap) {
                __syncthreads();
                stage(base);
                __syncthreads();
                const uint32_t top = min(total, base + scap);
                if (minimg) pc_row<NQ, VIR, EN, true, true>(ev, pi, row, ng, sub, stg, base, top);
                else pc_row<NQ, VIR, EN, false, true>(ev, pi, row, ng, sub, stg, base, top);
            }
        }
        float fx = ev.fx, fy = ev.fy, fz = ev.fz, e = ev.en;
#pragma unroll
        for (int o = PC_LANES / 2; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
            if (EN) e += __shfl_xor_sync(0xffffffffu, e, o);
        }
        if (valid && sub == 0) {
            const uint32_t i = slot2idx[slot];
            float4 f = accumulate ? force[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            f.x += fx;
            f.y += fy;
            f.z += fz;
            if (EN) f.w += 0.5f * e;
            force[i] = f;
            if (EN) en_sys += 0.5 * (double)e;
        }
        if (VIR) {
            float v[6] = {ev.vxx, ev.vxy, ev.vxz, ev.vyy, ev.vyz, ev.vzz};
#pragma unroll
            for (int k = 0; k < 6; ++k) vt[k] += v[k];
            ev.vxx = ev.vxy = ev.vxz = ev.vyy = ev.vyz = ev.vzz = 0.f;
            if (vpp) {
                // this particle's half of its pairs' virial (HOOMD's per-particle virial)
#pragma unroll
                for (int o = PC_LANES / 2; o > 0; o >>= 1)
#pragma unroll
                    for (int k = 0; k < 6; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
                if (valid && sub == 0) {
                    const uint32_t i = slot2idx[slot];
#pragma unroll
                    for (int k = 0; k < 6; ++k) vpp[(size_t)k * vpitch + i] += 0.5f * v[k];
                }
            }
        }
    }
    if (VIR) {
        double v[7] = {en_sys, 0.5 * (double)vt[0], 0.5 * (double)vt[1], 0.5 * (double)vt[2],
                       0.5 * (double)vt[3], 0.5 * (double)vt[4], 0.5 * (double)vt[5]};
        block_sum_f64<7>(v, red);
        if (tid == 0) {
            atomicAdd(&acc[si * ACC_STRIDE + ACC_E], v[0]);
#pragma unroll
            for (int k = 0; k < 6; ++k) atomicAdd(&acc[si * ACC_STRIDE + ACC_WP + k], v[1 + k]);
        }
    } else if (EN) {
        double v[1] = {en_sys};
        block_sum_f64<1>(v, red);
        if (tid == 0) atomicAdd(&acc[si * ACC_STRIDE + ACC_E], v[0]);
    }
}

#define ESPB_PC_NQ(X) X(8) X(10) X(11) X(12) X(13) X(14) X(16) X(20) X(24) X(32)

template <bool VIR, bool EN>
static cudaError_t launch_pc_t(const LaunchArgs& a, cudaStream_t st) {
    const PairList& L = *a.plist;
    const size_t smem = pair_cells_smem(L.stage_cap);
#define ESPB_PC_LAUNCH(NQ)                                                                                         \
    if (a.nq <= NQ) {                                                                                              \
        k_pair_cells<NQ, VIR, EN><<<L.n_cells, PC_THREADS, smem, st>>>(                                            \
            L.cell_sys, a.sys, L.cells, a.psets, L.cstart, L.slot2idx, a.posq, L.nn, L.nl16, L.cap, L.stage_cap, \
            a.force, a.acc, a.accumulate, a.pc, a.virial_pp, a.vpp_pitch);                                         \
        return cudaGetLastError();                                                                                 \
    }
    ESPB_PC_NQ(ESPB_PC_LAUNCH)
#undef ESPB_PC_LAUNCH
    return cudaErrorInvalidValue;
}

cudaError_t launch_pair_cells(const LaunchArgs& a, cudaStream_t st) {
    if (!a.plist || a.plist->n_cells == 0) return cudaSuccess;
    if (a.want_virial) return launch_pc_t<true, true>(a, st);
    if (a.want_energy) return launch_pc_t<false, true>(a, st);
    return launch_pc_t<false, false>(a, st);
}

// The shared-memory limit is a property of each kernel function, shared by
// every batch in the process: it is only ever raised, so a batch planned
// later with a smaller staging capacity cannot lower it below the launch
// size of one planned earlier.
cudaError_t configure_pair_cells(int stage_cap) {
    static int configured = 0;
    const int smem = (int)pair_cells_smem(stage_cap);
    if (smem <= configured) return cudaSuccess;
    cudaError_t e = cudaSuccess;
#define ESPB_PC_CONF(NQ)                                                                                    \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_pair_cells<NQ, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_pair_cells<NQ, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); \
    if (e == cudaSuccess)                                                                                   \
        e = cudaFuncSetAttribute(k_pair_cells<NQ, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    ESPB_PC_NQ(ESPB_PC_CONF)
#undef ESPB_PC_CONF
    if (e == cudaSuccess) configured = smem;
    return e;
}

cudaError_t launch_pairlist_pack(int rows, const uint32_t* nn, uint16_t* nl16, int cap, cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    const size_t smem = (size_t)PACK_WARPS * 2 * cap * sizeof(uint16_t);
    k_pairlist_pack<<<(rows + PACK_WARPS - 1) / PACK_WARPS, PACK_WARPS * 32, smem, st>>>(rows, nn, nl16, cap);
    return cudaGetLastError();
}

}  // namespace espb
