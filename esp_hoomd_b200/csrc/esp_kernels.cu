// ESP hot-path kernels for sm_100a.
//
// Stage map to the reference (slweng0321/ESP_HOOMD):
//   k_bin / k_scan / k_scatter / k_tile_sort : new particle binning + stable
//       sort (nearest reference code: makeFraction+floorf in
//       src/ESPForceComputeGPU.cu:228-236)
//   k_spread_mma (tensor-core tiles; default), k_spread_dense, k_spread :
//       charge assignment, src/ESPForceComputeGPU.cu:206-272 (K2)
//   k_fft_plane_fwd, or k_fftx_fwd / k_ffty<false> : forward FFT,
//       src/ESPForceComputeGPU.cc:254-265 (K3)
//   k_fft_slab_z, or k_fftz_conv : influence multiply fused into the z pass,
//       src/ESPForceComputeGPU.cu:277-287 (K4), plus the k-space energy and
//       virial (stubs in src/ESPForceCompute.cc:236-248)
//   k_fft_plane_inv, or k_ffty<true> / k_fftx_inv : inverse FFT (missing in
//       the reference, src/ESPForceCompute.cc:225-232)
//   k_interp (one CTA per tile), k_interp_q (persistent, tile queue) : force
//       interpolation, src/ESPForceComputeGPU.cu:292-373 (K6)
//   k_pair     : EvaluatorPairPSWF over a neighbour list,
//       src/EvaluatorPairPSWF.h:274-295 with the HOOMD PotentialPair loop
//   k_exclusions : exclusion correction, src/ESPForceComputeGPU.cu:391-471 (K7)
//   k_influence: influence-function build (K1), src/ESPForceComputeGPU.cu:157-201
#include <cuda.h>

#include "esp_common.cuh"
#include "esp_kernels.h"
#include "esp_pair.cuh"

namespace espb {

// ============================================================================
// a1: bin + stable sort
// ============================================================================

__global__ void k_bin(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, int P, int T,
                      const float4* __restrict__ pos_in, const float* __restrict__ q_in,
                      float4* __restrict__ posq, float4* __restrict__ trec, uint32_t* __restrict__ rel,
                      uint32_t* __restrict__ key, uint32_t* __restrict__ tile_count, double* __restrict__ acc,
                      const uint32_t* __restrict__ idx2slot, float4* __restrict__ spos) {
    __shared__ double red[32 * 2];
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    double qs[2] = {0.0, 0.0};
    uint32_t kk = 0xffffffffu;  // tile of this lane (none for lanes past the system)
    if (i < S.p_off + S.N) {
        const float4 p = pos_in[i];
        const float q = q_in[i];
        float x = p.x - S.Lx * floorf(p.x * S.inv_Lx);
        float y = p.y - S.Ly * floorf(p.y * S.inv_Ly);
        float z = p.z - S.Lz * floorf(p.z * S.inv_Lz);
        if (x >= S.Lx) x -= S.Lx;
        if (y >= S.Ly) y -= S.Ly;
        if (z >= S.Lz) z -= S.Lz;
        if (x < 0.f) x += S.Lx;
        if (y < 0.f) y += S.Ly;
        if (z < 0.f) z += S.Lz;
        // grid coordinate and stencil origin in FP64 (exact product of the
        // FP32 position), so t carries no position-rounding amplification
        const double hp = 0.5 * P;
        double g[3] = {(double)x * S.gxd, (double)y * S.gyd, (double)z * S.gzd};
        const int n[3] = {S.nx, S.ny, S.nz};
        int i0m[3];
        float tt[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (g[d] >= n[d]) g[d] -= n[d];
            const int i0 = (int)floor(g[d] - hp) + 1;
            tt[d] = (float)((double)i0 + hp - g[d]);
            i0m[d] = i0 < 0 ? i0 + n[d] : (i0 >= n[d] ? i0 - n[d] : i0);
        }
        const int tx = i0m[0] / T, ty = i0m[1] / T, tz = i0m[2] / T;
        const uint32_t k = (uint32_t)(S.t_off + (tz * S.nty + ty) * S.ntx + tx);
        key[i] = k;
        kk = k;
        posq[i] = make_float4(x, y, z, q);
        // the pair list's slot-ordered copy (rows of that list index it)
        if (spos) spos[idx2slot[i]] = make_float4(x, y, z, q);
        trec[i] = make_float4(tt[0], tt[1], tt[2], q);
        rel[i] = (uint32_t)(i0m[0] - tx * T) | ((uint32_t)(i0m[1] - ty * T) << 8) |
                 ((uint32_t)(i0m[2] - tz * T) << 16);
        qs[0] = q;
        qs[1] = (double)q * q;
    }
    {
        // one atomic per distinct tile of the warp
        const unsigned grp = __match_any_sync(0xffffffffu, kk);
        if (kk != 0xffffffffu && (threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&tile_count[kk], (uint32_t)__popc(grp));
    }
    block_sum_f64<2>(qs, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_QSUM], qs[0]);
        atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_Q2SUM], qs[1]);
    }
}

// Exclusive scan of n counts (single CTA of 1024 threads); start[n] = total.
// Each round covers 1024 x SCAN_PER consecutive counts, SCAN_PER per thread
// (16-byte loads and stores when both arrays are 16-byte aligned).
constexpr int SCAN_PER = 16;

__global__ void __launch_bounds__(1024) k_scan(const uint32_t* __restrict__ cnt, uint32_t* __restrict__ start, int n) {
    __shared__ uint32_t wsum[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const bool vec = ((reinterpret_cast<uintptr_t>(cnt) | reinterpret_cast<uintptr_t>(start)) & 15u) == 0;
    uint32_t carry = 0;
    for (int base = 0; base < n; base += 1024 * SCAN_PER) {
        const int i0 = base + threadIdx.x * SCAN_PER;
        const bool full = vec && i0 + SCAN_PER <= n;
        uint32_t v[SCAN_PER];
        if (full) {
#pragma unroll
            for (int k = 0; k < SCAN_PER / 4; ++k) {
                const uint4 u = reinterpret_cast<const uint4*>(cnt + i0)[k];
                v[4 * k] = u.x;
                v[4 * k + 1] = u.y;
                v[4 * k + 2] = u.z;
                v[4 * k + 3] = u.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < SCAN_PER; ++k) v[k] = i0 + k < n ? cnt[i0 + k] : 0u;
        }
        uint32_t tsum = 0;
#pragma unroll
        for (int k = 0; k < SCAN_PER; ++k) tsum += v[k];
        uint32_t x = tsum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            uint32_t w = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        uint32_t run = carry + (wid > 0 ? wsum[wid - 1] : 0u) + x - tsum;
#pragma unroll
        for (int k = 0; k < SCAN_PER; ++k) {
            const uint32_t c = v[k];
            v[k] = run;
            run += c;
        }
        if (full) {
#pragma unroll
            for (int k = 0; k < SCAN_PER / 4; ++k)
                reinterpret_cast<uint4*>(start + i0)[k] = make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
        } else {
#pragma unroll
            for (int k = 0; k < SCAN_PER; ++k)
                if (i0 + k < n) start[i0 + k] = v[k];
        }
        const uint32_t total = wsum[31];
        __syncthreads();
        carry += total;
    }
    if (threadIdx.x == 0) start[n] = carry;
}

// Slot of each particle inside its tile; leaves tile_count at zero so the
// next step's histogram needs no memset.
__global__ void k_scatter(const int2* __restrict__ chunks, const SysDev* __restrict__ sys,
                          const uint32_t* __restrict__ key, const uint32_t* __restrict__ start,
                          uint32_t* __restrict__ cnt, uint32_t* __restrict__ perm_u) {
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    const bool valid = i < S.p_off + S.N;
    const uint32_t k = valid ? key[i] : 0xffffffffu;
    // lanes with the same tile take consecutive slots with one atomic
    const unsigned grp = __match_any_sync(0xffffffffu, k);
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    uint32_t top = 0;
    if (valid && lane == leader) top = atomicSub(&cnt[k], (uint32_t)__popc(grp));
    top = __shfl_sync(0xffffffffu, top, leader);
    if (valid) perm_u[start[k] + top - 1u - (uint32_t)__popc(grp & ((1u << lane) - 1u))] = (uint32_t)i;
}

// Deterministic per-tile order: the particles of one tile sorted by (y
// origin of the stencil inside the tile, index), so the permutation equals a
// stable sort on (key, y origin, index). Grouping equal y origins lets the
// spreading kernel's warps skip the k-steps whose stencil rows miss theirs.
// The composite rank key is (oy << 26) | (index - system's first particle).
// Also gathers the sorted particle records.
__device__ __forceinline__ uint32_t sort_key(uint32_t v, const uint32_t* __restrict__ rel, int p_off) {
    return (((rel[v] >> 8) & 255u) << 26) | (v - (uint32_t)p_off);
}

__global__ void k_tile_sort(const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm_u,
                            uint32_t* __restrict__ perm, const float4* __restrict__ trec,
                            const uint32_t* __restrict__ rel, float4* __restrict__ srec,
                            uint32_t* __restrict__ srel, const int* __restrict__ tile_sys,
                            const SysDev* __restrict__ sys) {
    __shared__ __align__(16) uint32_t sm[SORT_CAP];
    const uint32_t s0 = start[blockIdx.x];
    const uint32_t n = start[blockIdx.x + 1] - s0;
    if (n == 0) return;
    const int p_off = sys[tile_sys[blockIdx.x]].p_off;
    const bool cached = n <= (uint32_t)SORT_CAP;
    const uint32_t n4 = (n + 3u) >> 2;
    if (cached) {
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sm[i] = sort_key(perm_u[s0 + i], rel, p_off);
        // pad to whole 16-byte groups with a value no key is above
        if (threadIdx.x < 4u * n4 - n) sm[n + threadIdx.x] = 0xffffffffu;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t v = perm_u[s0 + i];
        const uint32_t kv = cached ? sm[i] : sort_key(v, rel, p_off);
        uint32_t r = 0;
        if (cached) {
            // rank = number of smaller keys, four per shared load
            for (uint32_t j = 0; j < n4; ++j) {
                const uint4 u = reinterpret_cast<const uint4*>(sm)[j];
                r += (u.x < kv ? 1u : 0u) + (u.y < kv ? 1u : 0u) + (u.z < kv ? 1u : 0u) + (u.w < kv ? 1u : 0u);
            }
        } else {
            for (uint32_t j = 0; j < n; ++j) r += (sort_key(perm_u[s0 + j], rel, p_off) < kv) ? 1u : 0u;
        }
        perm[s0 + r] = v;
        srec[s0 + r] = trec[v];
        srel[s0 + r] = rel[v];
    }
}

// ============================================================================
// a3: spreading. One CTA per tile; shared-memory accumulators with residue
// ownership: location X of the tile's extended region [0, T+P-1)^3 is owned
// by the threads whose residue is X mod P, so every (particle, stencil
// point) update has a single writer and is Kahan-compensated without atomics
// (sum and compensation interleaved: one 64-bit shared load and store per
// tap). Thread (rx, ry, zg) handles, for each particle, the CZ = P/ZS stencil
// points of its x/y residue in its block of z residues. Each tile is flushed
// once to the FP64 mesh (sum - comp, one atomic per footprint point).
// ============================================================================

template <int P>
struct SpreadCfg {
    static constexpr int P2 = P * P;
    static constexpr int P3 = P * P * P;
    // z-residue groups: the largest divisor of P with P^2 * ZS <= 160 threads
    static constexpr int zs(int d) { return d <= 1 ? 1 : ((P % d == 0 && P2 * d <= 160) ? d : zs(d - 1)); }
    static constexpr int ZS = zs(P);
    static constexpr int CZ = P / ZS;  // stencil points per particle per thread
    static constexpr int THREADS = P2 * ZS;
    static constexpr int CH = 32;  // particles staged per round
};

template <int P>
__global__ void __launch_bounds__(SpreadCfg<P>::THREADS)
    k_spread(const int* __restrict__ tile_sys, const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets,
             int T, int D, const uint32_t* __restrict__ start, const float4* __restrict__ srec,
             const uint32_t* __restrict__ srel, double* __restrict__ rho) {
    using C = SpreadCfg<P>;
    extern __shared__ float4 smem4[];
    const int t = blockIdx.x;
    const uint32_t s0 = start[t];
    const int np = (int)(start[t + 1] - s0);
    if (np == 0) return;
    const int si = tile_sys[t];
    const SysDev S = sys[si];
    const ParamSet& ps = psets[S.pset];
    const int E = T + P - 1;
    const int nb = (E + P - 1) / P;
    const int NL = nb * nb * nb * C::P3;
    float2* accc = reinterpret_cast<float2*>(smem4);       // [NL] (sum, comp)
    float* pwx = reinterpret_cast<float*>(accc + NL);       // [CH][P] x weights * q
    float* pwy = pwx + C::CH * P;                           // [CH][P]
    float* pwz = pwy + C::CH * P;                           // [CH][P] by z residue
    int* pzo = reinterpret_cast<int*>(pwz + C::CH * P);     // [CH][P] z slot offsets
    int* pxy = pzo + C::CH * P;                             // [CH] packed x/y origins
    float* wc = reinterpret_cast<float*>(pxy + C::CH);      // [P][D+1]
    const int tid = threadIdx.x;
    for (int i = tid; i < NL; i += C::THREADS) accc[i] = make_float2(0.f, 0.f);
    for (int i = tid; i < P * (D + 1); i += C::THREADS)
        wc[i] = ps.wcoef[(i / (D + 1)) * (MAX_D + 1) + (i % (D + 1))];
    __syncthreads();
    const int rx = tid % P, ry = (tid / P) % P, zg = tid / C::P2;
    const int nbP3 = nb * nb * C::P3;
    for (int base = 0; base < np; base += C::CH) {
        const int nc = min(C::CH, np - base);
        for (int k = tid; k < nc * 3 * P; k += C::THREADS) {
            const int p = k / (3 * P), r = k - p * 3 * P, ax = r / P, a = r - ax * P;
            const float4 rec = srec[s0 + base + p];
            const uint32_t rl = srel[s0 + base + p];
            const float tt = ax == 0 ? rec.x : (ax == 1 ? rec.y : rec.z);
            const float w = horner_w(&wc[a * (D + 1)], D, tt);
            if (ax == 0) {
                pwx[p * P + a] = w * rec.w;
            } else if (ax == 1) {
                pwy[p * P + a] = w;
            } else {
                const int Z = (int)((rl >> 16) & 255u) + a, rz = Z % P, bz = Z / P;
                pwz[p * P + rz] = w;
                pzo[p * P + rz] = bz * nbP3 + rz * C::P2;
            }
            if (r == 0) {
                const int ox = (int)(rl & 255u), oy = (int)((rl >> 8) & 255u);
                pxy[p] = ox | ((ox % P) << 8) | (oy << 16) | ((oy % P) << 24);
            }
        }
        __syncthreads();
        for (int p = 0; p < nc; ++p) {
            const int pk = pxy[p];
            const int ox = pk & 255, oy = (pk >> 16) & 255;
            int a = rx - ((pk >> 8) & 255);
            a += a < 0 ? P : 0;
            int b = ry - ((pk >> 24) & 255);
            b += b < 0 ? P : 0;
            const int bx = (ox + a) / P, by = (oy + b) / P;
            const float wxy = pwx[p * P + a] * pwy[p * P + b];
            const int bs = (by * nb + bx) * C::P3 + ry * P + rx;
            const float* wz = pwz + p * P + zg * C::CZ;
            const int* zo = pzo + p * P + zg * C::CZ;
#pragma unroll
            for (int k = 0; k < C::CZ; ++k) {
                const int sl = bs + zo[k];
                const float tap = wxy * wz[k];
                float2 v = accc[sl];
                const float y = __fsub_rn(tap, v.y);
                const float tsum = __fadd_rn(v.x, y);
                v.y = __fsub_rn(__fsub_rn(tsum, v.x), y);
                v.x = tsum;
                accc[sl] = v;
            }
        }
        __syncthreads();
    }
    // flush: one FP64 atomic per footprint point (region slots that wrap
    // onto the same mesh point are summed first)
    const int lt = t - S.t_off;
    const int X0 = (lt % S.ntx) * T, Y0 = ((lt / S.ntx) % S.nty) * T, Z0 = (lt / (S.ntx * S.nty)) * T;
    const int Ex = min(E, S.nx), Ey = min(E, S.ny), Ez = min(E, S.nz);
    for (int i = tid; i < Ex * Ey * Ez; i += C::THREADS) {
        const int X = i % Ex, Y = (i / Ex) % Ey, Z = i / (Ex * Ey);
        double v = 0.0;
        for (int Zs = Z; Zs < E; Zs += S.nz)
            for (int Ys = Y; Ys < E; Ys += S.ny)
                for (int Xs = X; Xs < E; Xs += S.nx) {
                    const int sl = ((Zs / P * nb + Ys / P) * nb + Xs / P) * C::P3 +
                                   ((Zs % P) * P + Ys % P) * P + Xs % P;
                    const float2 a2 = accc[sl];
                    v += (double)a2.x - (double)a2.y;
                }
        if (v != 0.0) {
            int gx = X0 + X, gy = Y0 + Y, gz = Z0 + Z;
            gx -= gx >= S.nx ? S.nx : 0;
            gy -= gy >= S.ny ? S.ny : 0;
            gz -= gz >= S.nz ? S.nz : 0;
            atomicAdd(&rho[S.m_off + ((long long)gz * S.ny + gy) * S.nx + gx], v);
        }
    }
}

// ----------------------------------------------------------------------------
// Dense spreading (tiles with E = T + P - 1 <= 16): thread (X, Y) owns the
// whole z-column (X, Y, 0..E-1) of the tile's extended region in
// registers. For each particle it adds wx[X-ox] wy[Y-oy] wz_shift[Z] into
// all E registers (wz_shift = the particle's z weights placed at oz, zero
// elsewhere; read as broadcast 128-bit loads) -- no per-tap shared-memory
// traffic and no per-tap index arithmetic. Sums are compensated blockwise:
// each block of SPREAD_KC particles is summed in FP32 and Kahan-merged into
// the column's (sum, comp) registers. Flush: one FP64 atomic per column
// point.
// ----------------------------------------------------------------------------
constexpr int SPREAD_EM = 16;   // z registers per column (E <= 16)
constexpr int SPREAD_KC = 16;   // particles per compensated block
constexpr int SPREAD_CHD = 64;  // particles staged per round

template <int P>
__global__ void __launch_bounds__(256)
    k_spread_dense(const int* __restrict__ tile_sys, const SysDev* __restrict__ sys,
                   const ParamSet* __restrict__ psets, int T, int D, const uint32_t* __restrict__ start,
                   const float4* __restrict__ srec, const uint32_t* __restrict__ srel, double* __restrict__ rho) {
    extern __shared__ float4 smd4[];
    const int t = blockIdx.x;
    const uint32_t s0 = start[t];
    const int np = (int)(start[t + 1] - s0);
    if (np == 0) return;
    const int si = tile_sys[t];
    const SysDev S = sys[si];
    const ParamSet& ps = psets[S.pset];
    const int E = T + P - 1;
    float4* wzs = smd4;                                          // [CH][4] shifted z weights
    float* pwx = reinterpret_cast<float*>(wzs + SPREAD_CHD * 4);  // [CH][P] x weights * q
    float* pwy = pwx + SPREAD_CHD * P;                           // [CH][P]
    int* pxy = reinterpret_cast<int*>(pwy + SPREAD_CHD * P);     // [CH] origins
    float* wc = reinterpret_cast<float*>(pxy + SPREAD_CHD);      // [P][D+1]
    const int tid = threadIdx.x;
    for (int i = tid; i < P * (D + 1); i += blockDim.x) wc[i] = ps.wcoef[(i / (D + 1)) * (MAX_D + 1) + (i % (D + 1))];
    const int X = tid % E, Y = tid / E;
    const bool owner = tid < E * E;
    float cs[SPREAD_EM], sum[SPREAD_EM], comp[SPREAD_EM];
#pragma unroll
    for (int z = 0; z < SPREAD_EM; ++z) {
        cs[z] = 0.f;
        sum[z] = 0.f;
        comp[z] = 0.f;
    }
    int inblk = 0;
    for (int base = 0; base < np; base += SPREAD_CHD) {
        const int nc = min(SPREAD_CHD, np - base);
        __syncthreads();  // coefficients loaded; previous chunk consumed
        for (int k = tid; k < nc * 16; k += blockDim.x) reinterpret_cast<float*>(wzs)[k] = 0.f;
        __syncthreads();
        for (int k = tid; k < nc * 3 * P; k += blockDim.x) {
            const int p = k / (3 * P), r = k - p * 3 * P, ax = r / P, a = r - ax * P;
            const float4 rec = srec[s0 + base + p];
            const uint32_t rl = srel[s0 + base + p];
            const float tt = ax == 0 ? rec.x : (ax == 1 ? rec.y : rec.z);
            const float w = horner_w(&wc[a * (D + 1)], D, tt);
            if (ax == 0) {
                pwx[p * P + a] = w * rec.w;
            } else if (ax == 1) {
                pwy[p * P + a] = w;
            } else {
                reinterpret_cast<float*>(wzs)[p * 16 + (int)((rl >> 16) & 255u) + a] = w;
            }
            if (r == 0) pxy[p] = (int)(rl & 0xffffu);
        }
        __syncthreads();
        for (int p = 0; p < nc; ++p) {
            const int pk = pxy[p];
            const int a = X - (pk & 255), b = Y - ((pk >> 8) & 255);
            if (owner && (unsigned)a < (unsigned)P && (unsigned)b < (unsigned)P) {
                const float wxy = pwx[p * P + a] * pwy[p * P + b];
                const float4 z0 = wzs[p * 4 + 0], z1 = wzs[p * 4 + 1], z2 = wzs[p * 4 + 2], z3 = wzs[p * 4 + 3];
                const float wz[16] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w,
                                      z2.x, z2.y, z2.z, z2.w, z3.x, z3.y, z3.z, z3.w};
#pragma unroll
                for (int z = 0; z < SPREAD_EM; ++z) cs[z] = fmaf(wxy, wz[z], cs[z]);
            }
            if (++inblk == SPREAD_KC) {
                inblk = 0;
#pragma unroll
                for (int z = 0; z < SPREAD_EM; ++z) {
                    const float y = __fsub_rn(cs[z], comp[z]);
                    const float ts = __fadd_rn(sum[z], y);
                    comp[z] = __fsub_rn(__fsub_rn(ts, sum[z]), y);
                    sum[z] = ts;
                    cs[z] = 0.f;
                }
            }
        }
    }
    if (!owner) return;
    const int lt = t - S.t_off;
    int gx = (lt % S.ntx) * T + X, gy = ((lt / S.ntx) % S.nty) * T + Y;
    const int Z0 = (lt / (S.ntx * S.nty)) * T;
    while (gx >= S.nx) gx -= S.nx;
    while (gy >= S.ny) gy -= S.ny;
    double* col = rho + S.m_off + (long long)gy * S.nx + gx;
    const long long zstride = (long long)S.ny * S.nx;
#pragma unroll
    for (int z = 0; z < SPREAD_EM; ++z) {
        if (z < E) {
            const double v = ((double)sum[z] - (double)comp[z]) + (double)cs[z];
            if (v != 0.0) {
                int gz = Z0 + z;
                while (gz >= S.nz) gz -= S.nz;
                atomicAdd(col + gz * zstride, v);
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Tensor-core spreading (tiles with E = T + P - 1 = 16). The tile's
// extended region is a dense contraction over the tile's particles,
//   rho[(X,Y), Z] = sum_p  (q wx_p[X-ox_p] wy_p[Y-oy_p]) * wz_p[Z-oz_p],
// i.e. a (256 x K) x (K x 16) product with K = particles (zero weights
// outside each stencil). Warp w owns rows Y = 2w, 2w+1 (two m16 tiles, X =
// 0..15) and both n8 tiles of Z; each k-step of 8 particles issues
// mma.sync m16n8k8 TF32 with 3xTF32 operand splitting (hi*hi + hi*lo +
// lo*hi: FP32-level products). Each staged particle has three 16-point
// rows, zero outside its stencil and already shifted to its origin (x
// weights times charge, y weights, z weights pre-split into TF32 parts), so
// a k-step's A fragments are one product and split per element and its B
// fragments are plain shared loads. The next chunk's particle records are
// prefetched into shared memory (cp.async) while the current chunk runs.
// Every eight k-steps (64 particles) the FP32 block accumulators are added
// to FP64 sums in shared memory, 16 per lane and private to it (no barrier,
// no atomic, no registers held); the tile is flushed with one FP64 atomic
// per point.
// ----------------------------------------------------------------------------
__device__ __forceinline__ uint32_t f2tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// x = hi + lo exactly in FP32; hi is x rounded to TF32, lo is passed as raw
// FP32 bits: the MMA reads its TF32 part (the dropped bits of lo are below
// 2^-21 |x|, the level of the omitted lo*lo term)
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    hi = f2tf32(x);
    lo = __float_as_uint(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

constexpr int SPREAD_CHM = 48;  // particles staged per round (multiple of 8; 4 CTAs of 256 threads per SM)
constexpr int SPREAD_MS = 24;   // staged row stride: rows of 4 consecutive particles hit disjoint banks

template <int P>
__global__ void __launch_bounds__(256, 4)
    k_spread_mma(const int* __restrict__ tile_sys, const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets,
                 int T, int D, const uint32_t* __restrict__ start, const float4* __restrict__ srec,
                 const uint32_t* __restrict__ srel, double* __restrict__ rho) {
    extern __shared__ float4 smm4[];
    // per k-step of the chunk: the tile rows Y that carry stencil weight
    // (particles are sorted by y origin inside a tile, so most k-steps touch
    // half of the 16 rows; a warp skips the k-steps that miss its two rows)
    __shared__ int ks_lo[SPREAD_CHM / 8], ks_hi[SPREAD_CHM / 8];
    const int t = blockIdx.x;
    const uint32_t s0 = start[t];
    const int np = (int)(start[t + 1] - s0);
    if (np == 0) return;
    const int si = tile_sys[t];
    const SysDev S = sys[si];
    const ParamSet& ps = psets[S.pset];
    // per staged particle, rows of 16 region points (stride SPREAD_MS), zero
    // outside the particle's stencil: x weights * q, y weights, and the z
    // weights already split into TF32 high and low parts
    float* wxs = reinterpret_cast<float*>(smm4);
    float* wys = wxs + SPREAD_CHM * SPREAD_MS;
    uint32_t* wzh = reinterpret_cast<uint32_t*>(wys + SPREAD_CHM * SPREAD_MS);
    uint32_t* wzl = wzh + SPREAD_CHM * SPREAD_MS;
    // FP64 block sums, private to each lane: [warp][mt][nt][i][lane]
    double* bsum = reinterpret_cast<double*>(wzl + SPREAD_CHM * SPREAD_MS);
    // particle records of the current and the next chunk (prefetched)
    float4* crec = reinterpret_cast<float4*>(bsum + 8 * 16 * 32);  // [2][CHM]
    uint32_t* crel = reinterpret_cast<uint32_t*>(crec + 2 * SPREAD_CHM);  // [2][CHM]
    float* wc = reinterpret_cast<float*>(crel + 2 * SPREAD_CHM);  // [P][D+1]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, tg = lane & 3;
    for (int i = tid; i < P * (D + 1); i += blockDim.x) wc[i] = ps.wcoef[(i / (D + 1)) * (MAX_D + 1) + (i % (D + 1))];
    float acc[2][2][4];
    double* mysum = bsum + warp * 16 * 32 + lane;  // element e at mysum[32 e]
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int n = 0; n < 2; ++n)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                acc[m][n][i] = 0.f;
                mysum[32 * ((m * 2 + n) * 4 + i)] = 0.0;
            }
    int ksteps = 0;
    auto prefetch = [&](int base, int buf) {
        const int n = min(SPREAD_CHM, np - base);
        if (tid < n) {
            const uint32_t d1 = (uint32_t)__cvta_generic_to_shared(&crec[buf * SPREAD_CHM + tid]);
            const uint32_t d2 = (uint32_t)__cvta_generic_to_shared(&crel[buf * SPREAD_CHM + tid]);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d1), "l"(srec + s0 + base + tid));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d2), "l"(srel + s0 + base + tid));
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    prefetch(0, 0);
    for (int base = 0, cb = 0; base < np; base += SPREAD_CHM, cb ^= 1) {
        const int nc = min(SPREAD_CHM, np - base);
        const int ncp = (nc + 7) & ~7;  // padded to whole k-steps (zero weights)
        __syncthreads();  // previous chunk consumed (weights and records)
        if (base + SPREAD_CHM < np) prefetch(base + SPREAD_CHM, cb ^ 1);
        else asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group 1;\n" ::);  // this chunk's records have landed
        __syncthreads();  // (every thread's copies)
        {
            // thread (a, p0) evaluates window segment a on all three axes of
            // particles p0, p0 + nla, ... and writes both the stencil point o + a
            // and the zero points (o + a + P), (o + a + 2P), ... mod 16 of each
            // 16-point row, so every row is written whole (padding particles
            // get zero rows)
            constexpr int DD = default_window_degree<P>();
            const int nla = blockDim.x / P, a = tid % P, p0 = tid / P;
            if (p0 < nla) {
                SegPoly<DD> sp;
                if (D == DD) sp.load(&wc[a * (D + 1)]);
                for (int p = p0; p < ncp; p += nla) {
                    float* rx = wxs + p * SPREAD_MS;
                    float* ry = wys + p * SPREAD_MS;
                    uint32_t* rzh = wzh + p * SPREAD_MS;
                    uint32_t* rzl = wzl + p * SPREAD_MS;
                    if (p < nc) {
                        const float4 rec = crec[cb * SPREAD_CHM + p];
                        const uint32_t rl = crel[cb * SPREAD_CHM + p];
                        const int ox = (int)(rl & 255u), oy = (int)((rl >> 8) & 255u), oz = (int)((rl >> 16) & 255u);
                        const float w0 = D == DD ? sp.w(rec.x) : horner_w(&wc[a * (D + 1)], D, rec.x);
                        const float w1 = D == DD ? sp.w(rec.y) : horner_w(&wc[a * (D + 1)], D, rec.y);
                        const float w2 = D == DD ? sp.w(rec.z) : horner_w(&wc[a * (D + 1)], D, rec.z);
                        uint32_t h, l;
                        split_tf32(w2, h, l);
                        rx[ox + a] = w0 * rec.w;
                        ry[oy + a] = w1;
                        rzh[oz + a] = h;
                        rzl[oz + a] = l;
#pragma unroll
                        for (int z = P + a; z < 16; z += P) {
                            rx[(ox + z) & 15] = 0.f;
                            ry[(oy + z) & 15] = 0.f;
                            rzh[(oz + z) & 15] = 0u;
                            rzl[(oz + z) & 15] = 0u;
                        }
                    } else {
#pragma unroll
                        for (int z = a; z < 16; z += P) {
                            rx[z] = 0.f;
                            ry[z] = 0.f;
                            rzh[z] = 0u;
                            rzl[z] = 0u;
                        }
                    }
                }
            }
            if (tid < ncp / 8) {
                int lo = 1 << 30, hi = -1;
                for (int j = 0; j < 8; ++j) {
                    const int p = tid * 8 + j;
                    if (p < nc) {
                        const int oy = (int)((crel[cb * SPREAD_CHM + p] >> 8) & 255u);
                        lo = min(lo, oy);
                        hi = max(hi, oy);
                    }
                }
                ks_lo[tid] = lo;
                ks_hi[tid] = hi + P - 1;
            }
        }
        __syncthreads();
        for (int k0 = 0; k0 < ncp; k0 += 8) {
            const int klo = ks_lo[k0 >> 3], khi = ks_hi[k0 >> 3];
            if (2 * warp + 1 < klo || 2 * warp > khi) continue;  // warp-uniform: only zero rows here
            const int r1 = (k0 + tg) * SPREAD_MS, r2 = r1 + 4 * SPREAD_MS;  // particles k0 + tg, k0 + tg + 4
            // B fragments: b0 = wz_{p1}[Z], b1 = wz_{p2}[Z], Z = 8 nt + g
            uint32_t bh[2][2], bl[2][2];
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                bh[nt][0] = wzh[r1 + 8 * nt + g];
                bl[nt][0] = wzl[r1 + 8 * nt + g];
                bh[nt][1] = wzh[r2 + 8 * nt + g];
                bl[nt][1] = wzl[r2 + 8 * nt + g];
            }
            const float wx1 = wxs[r1 + g], wx1b = wxs[r1 + g + 8], wx2 = wxs[r2 + g], wx2b = wxs[r2 + g + 8];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int Y = 2 * warp + mt;
                if (Y < klo || Y > khi) continue;
                const float wy1 = wys[r1 + Y], wy2 = wys[r2 + Y];
                uint32_t ah0, al0, ah1, al1, ah2, al2, ah3, al3;
                split_tf32(wx1 * wy1, ah0, al0);   // row X = g,     particle p1
                split_tf32(wx1b * wy1, ah1, al1);  // row X = g + 8, particle p1
                split_tf32(wx2 * wy2, ah2, al2);   // row X = g,     particle p2
                split_tf32(wx2b * wy2, ah3, al3);  // row X = g + 8, particle p2
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    mma_tf32(acc[mt][nt], al0, al1, al2, al3, bh[nt][0], bh[nt][1]);
                    mma_tf32(acc[mt][nt], ah0, ah1, ah2, ah3, bl[nt][0], bl[nt][1]);
                    mma_tf32(acc[mt][nt], ah0, ah1, ah2, ah3, bh[nt][0], bh[nt][1]);
                }
            }
            if (++ksteps == 8) {
                ksteps = 0;
#pragma unroll
                for (int m = 0; m < 2; ++m)
#pragma unroll
                    for (int n = 0; n < 2; ++n)
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            mysum[32 * ((m * 2 + n) * 4 + i)] += (double)acc[m][n][i];
                            acc[m][n][i] = 0.f;
                        }
            }
        }
    }
    // flush: C fragment element i of (mt, nt) is point X = g + 8 (i >> 1), Y = 2 warp + mt,
    // Z = 8 nt + 2 tg + (i & 1)
    const int lt = t - S.t_off;
    const int X0 = (lt % S.ntx) * T, Y0 = ((lt / S.ntx) % S.nty) * T, Z0 = (lt / (S.ntx * S.nty)) * T;
    const long long zstride = (long long)S.ny * S.nx;
    long long xo[2], zo[2][2];  // wrapped x offsets (X = g, g + 8), z offsets (Z = 8 nt + 2 tg + e)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        int gx = X0 + g + 8 * h;
        while (gx >= S.nx) gx -= S.nx;
        xo[h] = gx;
    }
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            int gz = Z0 + 8 * nt + 2 * tg + e;
            while (gz >= S.nz) gz -= S.nz;
            zo[nt][e] = gz * zstride;
        }
    double* rb = rho + S.m_off;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        int gy = Y0 + 2 * warp + mt;
        while (gy >= S.ny) gy -= S.ny;
        const long long yo = (long long)gy * S.nx;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double v = mysum[32 * ((mt * 2 + nt) * 4 + i)] + (double)acc[mt][nt][i];
                if (v != 0.0) atomicAdd(rb + zo[nt][i & 1] + yo + xo[i >> 1], v);
            }
    }
}

// ============================================================================
// a4-a6: FFT passes. Batched mixed-radix (2,3,4,5) Stockham transforms in
// shared memory; lines stored element-major s[i*B + b].
// ============================================================================

template <int R, bool INV>
__device__ __forceinline__ void dft_small(float2 (&v)[R]) {
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 3) {
        const float s1 = INV ? -0.86602540378443865f : 0.86602540378443865f;
        const float2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
        const float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
        v[0] = cadd(v[0], t1);
        // -i s1 t2 = (s1 t2.y, -s1 t2.x)
        v[1] = make_float2(m.x + s1 * t2.y, m.y - s1 * t2.x);
        v[2] = make_float2(m.x - s1 * t2.y, m.y + s1 * t2.x);
    } else if constexpr (R == 4) {
        const float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        const float2 c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        v[0] = cadd(a, c);
        v[2] = csub(a, c);
        if (INV) {
            v[1] = make_float2(b.x - d.y, b.y + d.x);
            v[3] = make_float2(b.x + d.y, b.y - d.x);
        } else {
            v[1] = make_float2(b.x + d.y, b.y - d.x);
            v[3] = make_float2(b.x - d.y, b.y + d.x);
        }
    } else if constexpr (R == 5) {
        const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
        const float s1 = INV ? -0.95105651629515357f : 0.95105651629515357f;
        const float s2 = INV ? -0.58778525229247313f : 0.58778525229247313f;
        const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        const float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
        const float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
        const float2 b1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
        const float2 b2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
        v[0] = cadd(v[0], cadd(t1, t2));
        // a -/+ i b
        v[1] = make_float2(a1.x + b1.y, a1.y - b1.x);
        v[4] = make_float2(a1.x - b1.y, a1.y + b1.x);
        v[2] = make_float2(a2.x + b2.y, a2.y - b2.x);
        v[3] = make_float2(a2.x - b2.y, a2.y + b2.x);
    }
}

// Quotient by a divisor fixed for a loop: n / d = umulhi(n, ceil(2^32 / d)),
// exact when n and d are below 2^16 (division by invariant integers,
// Granlund and Montgomery 1994). Every FFT index is below 2^16: lines are at
// most FFT_MAX_N = 256 points and a CTA holds at most 256 x 129 of them.
struct Div16 {
    uint32_t d, m;
    __device__ __forceinline__ explicit Div16(int dd) : d((uint32_t)dd), m(dd > 1 ? 0xffffffffu / (uint32_t)dd + 1u : 0u) {}
    __device__ __forceinline__ int div(int n) const { return d > 1 ? (int)__umulhi((uint32_t)n, m) : n; }
};

template <int R, bool INV>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ src, float2* __restrict__ dst, int n, int B,
                                          int SB, int Ns, const float2* __restrict__ tw) {
    const int m = n / R;
    const int stride = n / (Ns * R);
    const Div16 dB(B), dNs(Ns);
    for (int idx = threadIdx.x; idx < m * B; idx += blockDim.x) {
        const int j = dB.div(idx), b = idx - j * B, jq = dNs.div(j), k = j - jq * Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[(j + r * m) * SB + b];
        if (Ns > 1) {
            const int ts = k * stride;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = tw[ts * r];
                if (INV) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        dft_small<R, INV>(v);
        const int o = jq * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[(o + r * Ns) * SB + b] = v[r];
    }
}

// Runs all stages; returns the buffer that holds the result.
template <bool INV>
__device__ float2* fft_lines(float2* s0, float2* s1, int n, int B, int SB, const float2* __restrict__ tw,
                             uint32_t plan) {
    int Ns = 1;
    for (int s = 0; s < 8; ++s) {
        const int R = (int)((plan >> (4 * s)) & 15u);
        if (R == 0) break;
        switch (R) {
            case 2: fft_stage<2, INV>(s0, s1, n, B, SB, Ns, tw); break;
            case 3: fft_stage<3, INV>(s0, s1, n, B, SB, Ns, tw); break;
            case 4: fft_stage<4, INV>(s0, s1, n, B, SB, Ns, tw); break;
            case 5: fft_stage<5, INV>(s0, s1, n, B, SB, Ns, tw); break;
        }
        __syncthreads();
        float2* tmp = s0;
        s0 = s1;
        s1 = tmp;
        Ns *= R;
    }
    return s0;
}

// Forward x pass: real rows (FP64 mesh, read and cleared) -> half spectrum.
// Two real rows form one complex line; the half spectra are separated with
// A_k = (Z_k + conj Z_{n-k})/2, B_k = (Z_k - conj Z_{n-k})/(2i).
__global__ void k_fftx_fwd(const int4* __restrict__ items, const SysDev* __restrict__ sys,
                           const float2* __restrict__ tw, const double* __restrict__ rho, float2* __restrict__ spec) {
    extern __shared__ float2 sb[];
    const int4 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int z = it.y, y0 = it.z, n = S.nx;
    constexpr int B = FFT_B_X, SB = FFT_SB_X;  // padded line stride: conflict-free row access
    float2* s0 = sb;
    float2* s1 = sb + n * SB;
    const Div16 dn(n), dh(S.nxh);
    for (int idx = threadIdx.x; idx < B * n; idx += blockDim.x) {
        const int b = dn.div(idx), i = idx - b * n, y = y0 + 2 * b;
        float2 v = make_float2(0.f, 0.f);
        if (y < S.ny) {
            const long long g = S.m_off + ((long long)z * S.ny + y) * n + i;
            v.x = (float)rho[g];
            if (y + 1 < S.ny) v.y = (float)rho[g + n];
        }
        s0[i * SB + b] = v;
    }
    __syncthreads();
    const float2* r = fft_lines<false>(s0, s1, n, B, SB, tw + S.twx, S.radx);
    for (int idx = threadIdx.x; idx < B * S.nxh; idx += blockDim.x) {
        const int b = dh.div(idx), k = idx - b * S.nxh;
        const float2 zk = r[k * SB + b], zn = r[(k ? n - k : 0) * SB + b];
        const int y = y0 + 2 * b;
        if (y < S.ny)
            spec[S.s_off + ((long long)z * S.ny + y) * S.nxh + k] =
                make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
        if (y + 1 < S.ny)
            spec[S.s_off + ((long long)z * S.ny + y + 1) * S.nxh + k] =
                make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
    }
}

// y pass (C2C), forward or inverse, in place on the half spectrum.
template <bool INV>
__global__ void k_ffty(const int4* __restrict__ items, const SysDev* __restrict__ sys,
                       const float2* __restrict__ tw, float2* __restrict__ spec) {
    extern __shared__ float2 sb[];
    const int4 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int z = it.y, kx0 = it.z, n = S.ny;
    constexpr int B = FFT_B_YZ;
    float2* s0 = sb;
    float2* s1 = sb + n * B;
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        const int y = idx / B, b = idx - y * B, kx = kx0 + b;
        s0[idx] = kx < S.nxh ? spec[S.s_off + ((long long)z * S.ny + y) * S.nxh + kx] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const float2* r = fft_lines<INV>(s0, s1, n, B, B, tw + S.twy, S.rady);
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        const int y = idx / B, b = idx - y * B, kx = kx0 + b;
        if (kx < S.nxh) spec[S.s_off + ((long long)z * S.ny + y) * S.nxh + kx] = r[idx];
    }
}

// z pass: forward transform, k-space energy and virial (FP64), influence
// multiply, inverse transform -- the only pass that holds whole k-columns.
template <bool VIR>
__global__ void k_fftz_conv(const int4* __restrict__ items, const SysDev* __restrict__ sys,
                            const float2* __restrict__ tw, const float2* __restrict__ gtab,
                            float2* __restrict__ spec, double* __restrict__ acc) {
    extern __shared__ float2 sb[];
    __shared__ double red[32 * 7];
    const int4 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int y = it.y, kx0 = it.z, n = S.nz;
    constexpr int B = FFT_B_YZ;
    float2* s0 = sb;
    float2* s1 = sb + n * B;
    const long long rowstride = (long long)S.ny * S.nxh;
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        const int z = idx / B, b = idx - z * B, kx = kx0 + b;
        s0[idx] = kx < S.nxh ? spec[S.s_off + z * rowstride + (long long)y * S.nxh + kx] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* r = fft_lines<false>(s0, s1, n, B, B, tw + S.twz, S.radz);
    float2* other = (r == s0) ? s1 : s0;
    const double twopi = 6.283185307179586;
    const int fy = (y < (S.ny + 1) / 2) ? y : y - S.ny;
    const double kyv = twopi * fy / (double)S.Ly;
    const double ckx = twopi / (double)S.Lx, ckz = twopi / (double)S.Lz;  // 2 pi / L
    double e[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        const int z = idx / B, b = idx - z * B, kx = kx0 + b;
        if (kx >= S.nxh) {
            r[idx] = make_float2(0.f, 0.f);
            continue;
        }
        const float2 gb = gtab[S.g_off + z * rowstride + (long long)y * S.nxh + kx];
        const float2 d = r[idx];
        if (VIR) {
            const double p2 = (double)d.x * d.x + (double)d.y * d.y;
            const double mult = (kx == 0 || 2 * kx == S.nx) ? 0.5 : 1.0;
            const double ek = mult * (double)gb.x * p2, eb = mult * (double)gb.y * p2;
            const int fz = (z < (n + 1) / 2) ? z : z - n;
            const double kxv = ckx * kx, kzv = ckz * fz;
            e[0] += ek;
            e[1] += ek + eb * kxv * kxv;
            e[2] += eb * kxv * kyv;
            e[3] += eb * kxv * kzv;
            e[4] += ek + eb * kyv * kyv;
            e[5] += eb * kyv * kzv;
            e[6] += ek + eb * kzv * kzv;
        }
        r[idx] = make_float2(d.x * gb.x, d.y * gb.x);
    }
    __syncthreads();
    const float2* o = fft_lines<true>(r, other, n, B, B, tw + S.twz, S.radz);
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        const int z = idx / B, b = idx - z * B, kx = kx0 + b;
        if (kx < S.nxh) spec[S.s_off + z * rowstride + (long long)y * S.nxh + kx] = o[idx];
    }
    if (VIR) {
        block_sum_f64<7>(e, red);
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < 7; ++k) atomicAdd(&acc[it.x * ACC_STRIDE + ACC_EK + k], e[k]);
    }
}

// Inverse x pass (C2R): two Hermitian half-spectrum rows A, B are extended
// and combined as Z = A + iB; the inverse transform returns row A in the
// real part and row B in the imaginary part.
__global__ void k_fftx_inv(const int4* __restrict__ items, const SysDev* __restrict__ sys,
                           const float2* __restrict__ tw, const float2* __restrict__ spec, float* __restrict__ phi,
                           double* __restrict__ rho) {
    extern __shared__ float2 sb[];
    const int4 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int z = it.y, y0 = it.z, n = S.nx;
    constexpr int B = FFT_B_X, SB = FFT_SB_X;
    float2* s0 = sb;
    float2* s1 = sb + n * SB;
    const Div16 dn(n);
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        const int b = dn.div(idx), k = idx - b * n, ya = y0 + 2 * b, yb = ya + 1;
        const bool up = k >= S.nxh;
        const int kk = up ? n - k : k;
        float2 A = ya < S.ny ? spec[S.s_off + ((long long)z * S.ny + ya) * S.nxh + kk] : make_float2(0.f, 0.f);
        float2 Bv = yb < S.ny ? spec[S.s_off + ((long long)z * S.ny + yb) * S.nxh + kk] : make_float2(0.f, 0.f);
        if (up) {
            A.y = -A.y;
            Bv.y = -Bv.y;
        }
        if (k == 0 || 2 * k == n) {
            A.y = 0.f;
            Bv.y = 0.f;
        }
        s0[k * SB + b] = make_float2(A.x - Bv.y, A.y + Bv.x);
    }
    __syncthreads();
    const float2* r = fft_lines<true>(s0, s1, n, B, SB, tw + S.twx, S.radx);
    for (int idx = threadIdx.x; idx < n * B; idx += blockDim.x) {
        const int b = dn.div(idx), i = idx - b * n, y = y0 + 2 * b;
        if (y < S.ny) {
            const long long g = S.m_off + ((long long)z * S.ny + y) * n + i;
            rho[g] = 0.0;  // clear the charge mesh for the next spread
            if (y + 1 < S.ny) rho[g + n] = 0.0;
        }
    }
    // the rows and their periodic copies in the halo-padded potential mesh,
    // one warp per (row, copy)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int b = wid; b < 2 * B; b += nw) {
        const int y = y0 + b;  // source row b / 2 of the pair, real (even b) or imaginary part
        if (y >= S.ny) continue;
        for (int zz = z; zz < S.nzp; zz += S.nz)
            for (int yy = y; yy < S.nyp; yy += S.ny) {
                float* dst = phi + S.mp_off + ((long long)zz * S.nyp + yy) * S.nxp;
                for (int x = lane; x < S.nxp; x += 32) {
                    int xs = x;
                    while (xs >= n) xs -= n;
                    const float2 v = r[xs * SB + (b >> 1)];
                    dst[x] = (b & 1) ? v.y : v.x;
                }
            }
    }
}

// ----------------------------------------------------------------------------
// Plane and slab passes (meshes whose planes fit in shared memory): one CTA
// transforms a whole z-plane (x R2C + y C2C, and the inverse), or a whole
// xz-slab for the z pass, so every CTA carries enough independent work to
// hide memory latency. Line strides are odd so 64-bit shared accesses with
// a stride of one line are bank-conflict free.
// ----------------------------------------------------------------------------
__device__ __forceinline__ int odd_up(int v) { return v | 1; }

__global__ void __launch_bounds__(256)
    k_fft_plane_fwd(const int2* __restrict__ items, const SysDev* __restrict__ sys, const float2* __restrict__ tw,
                    const double* __restrict__ rho, float2* __restrict__ spec) {
    extern __shared__ float2 sb[];
    const int2 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int z = it.y, nx = S.nx, ny = S.ny, nxh = S.nxh;
    const int np = (ny + 1) / 2, SBx = odd_up(np), SBy = odd_up(nxh);
    const int cap = max(nx * SBx, ny * SBy);
    float2* s0 = sb;
    float2* s1 = sb + cap;
    float2* twx = sb + 2 * cap;  // twiddles of both axes, staged once
    float2* twy = twx + nx;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) twx[i] = tw[S.twx + i];
    for (int i = threadIdx.x; i < ny; i += blockDim.x) twy[i] = tw[S.twy + i];
    const double* src = rho + S.m_off + (long long)z * ny * nx;
    const Div16 dnx(nx), dnh(nxh);
    for (int idx = threadIdx.x; idx < np * nx; idx += blockDim.x) {
        const int b = dnx.div(idx), i = idx - b * nx, y = 2 * b;
        float2 v;
        v.x = (float)src[y * nx + i];
        v.y = (y + 1 < ny) ? (float)src[(y + 1) * nx + i] : 0.f;
        s0[i * SBx + b] = v;
    }
    __syncthreads();
    float2* r = fft_lines<false>(s0, s1, nx, np, SBx, twx, S.radx);
    float2* o = (r == s0) ? s1 : s0;
    for (int idx = threadIdx.x; idx < np * nxh; idx += blockDim.x) {
        const int b = dnh.div(idx), k = idx - b * nxh;
        const float2 zk = r[k * SBx + b], zn = r[(k ? nx - k : 0) * SBx + b];
        o[(2 * b) * SBy + k] = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
        if (2 * b + 1 < ny) o[(2 * b + 1) * SBy + k] = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
    }
    __syncthreads();
    const float2* r2 = fft_lines<false>(o, r, ny, nxh, SBy, twy, S.rady);
    float2* dst = spec + S.s_off + (long long)z * ny * nxh;
    for (int idx = threadIdx.x; idx < ny * nxh; idx += blockDim.x) {
        const int y = dnh.div(idx), k = idx - y * nxh;
        dst[idx] = r2[y * SBy + k];
    }
}

__global__ void __launch_bounds__(256)
    k_fft_plane_inv(const int2* __restrict__ items, const SysDev* __restrict__ sys, const float2* __restrict__ tw,
                    const float2* __restrict__ spec, float* __restrict__ phi, double* __restrict__ rho) {
    extern __shared__ float2 sb[];
    const int2 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int z = it.y, nx = S.nx, ny = S.ny, nxh = S.nxh;
    const int np = (ny + 1) / 2, SBx = odd_up(np), SBy = odd_up(nxh);
    const int cap = max(nx * SBx, ny * SBy);
    float2* s0 = sb;
    float2* s1 = sb + cap;
    float2* twx = sb + 2 * cap;  // twiddles of both axes, staged once
    float2* twy = twx + nx;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) twx[i] = tw[S.twx + i];
    for (int i = threadIdx.x; i < ny; i += blockDim.x) twy[i] = tw[S.twy + i];
    const float2* src = spec + S.s_off + (long long)z * ny * nxh;
    const Div16 dnx(nx), dnh(nxh);
    for (int idx = threadIdx.x; idx < ny * nxh; idx += blockDim.x) {
        const int y = dnh.div(idx), k = idx - y * nxh;
        s0[y * SBy + k] = src[idx];
    }
    __syncthreads();
    float2* r = fft_lines<true>(s0, s1, ny, nxh, SBy, twy, S.rady);
    float2* o = (r == s0) ? s1 : s0;
    for (int idx = threadIdx.x; idx < np * nx; idx += blockDim.x) {
        const int b = dnx.div(idx), k = idx - b * nx;
        const bool up = k >= nxh;
        const int kk = up ? nx - k : k;
        float2 A = r[(2 * b) * SBy + kk];
        float2 Bv = (2 * b + 1 < ny) ? r[(2 * b + 1) * SBy + kk] : make_float2(0.f, 0.f);
        if (up) {
            A.y = -A.y;
            Bv.y = -Bv.y;
        }
        if (k == 0 || 2 * k == nx) {
            A.y = 0.f;
            Bv.y = 0.f;
        }
        o[k * SBx + b] = make_float2(A.x - Bv.y, A.y + Bv.x);
    }
    __syncthreads();
    const float2* r2 = fft_lines<true>(o, r, nx, np, SBx, twx, S.radx);
    double* rz = rho + S.m_off + (long long)z * ny * nx;
    for (int idx = threadIdx.x; idx < ny * nx; idx += blockDim.x) rz[idx] = 0.0;  // cleared for the next spread
    // the plane and its periodic copies in the halo-padded potential mesh,
    // one warp per padded row
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int zz = z; zz < S.nzp; zz += S.nz) {
        float* dst = phi + S.mp_off + (long long)zz * S.nyp * S.nxp;
        for (int y = wid; y < S.nyp; y += nw) {
            int ys = y;
            while (ys >= ny) ys -= ny;
            const int b = ys >> 1;
            const bool hi = ys & 1;
            for (int x = lane; x < S.nxp; x += 32) {
                int xs = x;
                while (xs >= nx) xs -= nx;
                const float2 v = r2[xs * SBx + b];
                dst[(long long)y * S.nxp + x] = hi ? v.y : v.x;
            }
        }
    }
}

// z pass over a whole xz-slab (fixed y): forward, energy/virial (VIR: when
// the virial is requested), influence multiply, inverse.
template <bool VIR>
__global__ void __launch_bounds__(256)
    k_fft_slab_z(const int2* __restrict__ items, const SysDev* __restrict__ sys, const float2* __restrict__ tw,
                 const float2* __restrict__ gtab, float2* __restrict__ spec, double* __restrict__ acc) {
    extern __shared__ float2 sb[];
    __shared__ double red[32 * 7];
    const int2 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int y = it.y, nz = S.nz, nxh = S.nxh, SBz = odd_up(nxh);
    float2* s0 = sb;
    float2* s1 = sb + nz * SBz;
    float2* twz = sb + 2 * nz * SBz;  // twiddles, staged once
    for (int i = threadIdx.x; i < nz; i += blockDim.x) twz[i] = tw[S.twz + i];
    const long long rowstride = (long long)S.ny * nxh;
    float2* base = spec + S.s_off + (long long)y * nxh;
    const float2* gbase = gtab + S.g_off + (long long)y * nxh;
    const Div16 dnh(nxh);
    for (int idx = threadIdx.x; idx < nz * nxh; idx += blockDim.x) {
        const int z = dnh.div(idx), k = idx - z * nxh;
        s0[z * SBz + k] = base[z * rowstride + k];
    }
    __syncthreads();
    float2* r = fft_lines<false>(s0, s1, nz, nxh, SBz, twz, S.radz);
    float2* other = (r == s0) ? s1 : s0;
    const double twopi = 6.283185307179586;
    const int fy = (y < (S.ny + 1) / 2) ? y : y - S.ny;
    const double kyv = twopi * fy / (double)S.Ly;
    const double ckx = twopi / (double)S.Lx, ckz = twopi / (double)S.Lz;  // 2 pi / L
    double e[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int idx = threadIdx.x; idx < nz * nxh; idx += blockDim.x) {
        const int z = dnh.div(idx), kx = idx - z * nxh;
        const float2 gb = gbase[z * rowstride + kx];
        float2& d = r[z * SBz + kx];
        if (VIR) {
            const double p2 = (double)d.x * d.x + (double)d.y * d.y;
            const double mult = (kx == 0 || 2 * kx == S.nx) ? 0.5 : 1.0;
            const double ek = mult * (double)gb.x * p2, eb = mult * (double)gb.y * p2;
            const int fz = (z < (nz + 1) / 2) ? z : z - nz;
            const double kxv = ckx * kx, kzv = ckz * fz;
            e[0] += ek;
            e[1] += ek + eb * kxv * kxv;
            e[2] += eb * kxv * kyv;
            e[3] += eb * kxv * kzv;
            e[4] += ek + eb * kyv * kyv;
            e[5] += eb * kyv * kzv;
            e[6] += ek + eb * kzv * kzv;
        }
        d = make_float2(d.x * gb.x, d.y * gb.x);
    }
    __syncthreads();
    const float2* o = fft_lines<true>(r, other, nz, nxh, SBz, twz, S.radz);
    for (int idx = threadIdx.x; idx < nz * nxh; idx += blockDim.x) {
        const int z = dnh.div(idx), k = idx - z * nxh;
        base[z * rowstride + k] = o[z * SBz + k];
    }
    if (VIR) {
        block_sum_f64<7>(e, red);
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < 7; ++k) atomicAdd(&acc[it.x * ACC_STRIDE + ACC_EK + k], e[k]);
    }
}

// ============================================================================
// a5 (build): influence table {G, G*B} over the half spectrum, in FP64.
//   G  = Psi(|k| r_c) / (k^2 V w_x^2 w_y^2 w_z^2)
//   GB = (-2 Psi / k^2 + r_c Psi'(|k| r_c) / |k|) / (k^2 V w^2)
// Psi by Gauss-Legendre quadrature of the prolate (weights pre-scaled).
// ============================================================================
template <typename T2>
__global__ void k_influence(SysDev S, const double* __restrict__ w1d, const double* __restrict__ tq,
                            const double* __restrict__ wq, int nq, double rcut, double psi_floor,
                            T2* __restrict__ gtab) {
    const long long total = (long long)S.nz * S.ny * S.nxh;
    const double twopi = 6.283185307179586;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int kx = (int)(idx % S.nxh);
        const int y = (int)((idx / S.nxh) % S.ny);
        const int z = (int)(idx / ((long long)S.nxh * S.ny));
        const int fy = (y < (S.ny + 1) / 2) ? y : y - S.ny;
        const int fz = (z < (S.nz + 1) / 2) ? z : z - S.nz;
        const double kxv = twopi * kx / (double)S.Lx, kyv = twopi * fy / (double)S.Ly,
                     kzv = twopi * fz / (double)S.Lz;
        const double k2 = kxv * kxv + kyv * kyv + kzv * kzv;
        double gx = 0.0, gy = 0.0;
        // Nyquist planes of even meshes are dropped: there Psi(kappa_N) is
        // at the split's truncation level while 1/w^2 amplifies aliasing
        // and round-off the most
        const bool nyq = (2 * kx == S.nx) || (2 * y == S.ny) || (2 * z == S.nz);
        if (k2 > 0.0 && !nyq) {
            const double kk = sqrt(k2), kap = kk * rcut;
            double psi = 0.0, dpsi = 0.0;
            for (int j = 0; j < nq; ++j) {
                double s, c;
                sincos(kap * tq[j], &s, &c);
                psi += wq[j] * c;
                dpsi -= wq[j] * tq[j] * s;
            }
            if (psi > psi_floor) {
                const double w = w1d[kx] * w1d[S.nx + y] * w1d[S.nx + S.ny + z];
                const double den = k2 * S.V * w * w;
                gx = psi / den;
                gy = (-2.0 * psi / k2 + rcut * dpsi / kk) / den;
            }
        }
        T2 out;
        out.x = gx;
        out.y = gy;
        gtab[S.g_off + idx] = out;
    }
}

// ============================================================================
// a7: interpolation. One CTA per tile stages the potential of the tile's
// extended region in shared memory and, per chunk of particles, the 3P
// window weights and derivatives (computed once per particle by all
// threads). A group of G lanes serves one particle: lane c owns stencil
// plane z = oz + c and contracts it separably (x, then y) in registers;
// the group sums its four partials (potential, gradient) with shuffles.
// Each chunk's particle records and output slots are prefetched into shared
// memory (cp.async) while the previous chunk is interpolated.
// ============================================================================
// words of the interpolation staging area: the per-chunk weights, or (before
// the first chunk) the wrapped row offsets, shared row offsets and x
// indices of the region
__host__ __device__ inline int interp_stage_words(int P, int CH, int E) {
    return CH * (6 * P + 1) > 2 * E * E + E ? CH * (6 * P + 1) : 2 * E * E + E;
}

template <int P>
struct InterpCfg {
    static constexpr int G = P <= 4 ? 4 : (P <= 8 ? 8 : 16);  // lanes per particle
    static constexpr int THREADS = 128;
    static constexpr int NG = THREADS / G;  // particles in flight per CTA
    static constexpr int CH = 2 * NG;       // particles staged per round
};

// TMA: the extended region arrives as one cp.async.bulk.tensor box of the
// halo-padded potential mesh (tensor map per system, x rounded down to a
// 16-byte boundary, box PX x (PP / PX) x E floats); otherwise as 4-byte
// cp.async copies. A TMA wait that runs out (kTmaWaitLimit polls) sets
// kerr[0] and skips the tile.
constexpr int kTmaWaitLimit = 1 << 24;

__device__ __forceinline__ bool tma_wait(uint32_t mbar, uint32_t phase) {
    for (int it = 0; it < kTmaWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// One chunk of a tile's particles (records already in shared memory):
// window weights and derivatives, the processing order, and the contraction
// of each particle's stencil with the staged potential region; writes the
// particles' forces and energies and returns the chunk's energy (FP64).
// Called by every thread of the CTA (it synchronises).
template <int P, bool TMA>
__device__ __forceinline__ double interp_chunk(const float* __restrict__ sm, int PX, int PP, int xoff, int D,
                                               const float* __restrict__ wc, const float4* __restrict__ crec,
                                               const uint32_t* __restrict__ crel, const uint32_t* __restrict__ cprm,
                                               float* __restrict__ wts, float* __restrict__ qv, int* __restrict__ org,
                                               int* __restrict__ order, int nc, float gxs, float gys, float gzs,
                                               double self_coef, float4* __restrict__ force) {
    using C = InterpCfg<P>;
    constexpr int WS = 6 * P + 1;  // weight row stride (odd: conflict-free broadcasts)
    constexpr int K = 32 / C::G;   // particle groups per warp
    const int grp = threadIdx.x / C::G, gl = threadIdx.x % C::G;
    double esum = 0.0;
    {
        // thread (a, p0) evaluates window segment a (value and derivative)
        // on all three axes of particles p0, p0 + nla, ...
        constexpr int DD = default_window_degree<P>();
        const int nla = blockDim.x / P, a2 = threadIdx.x % P, p0 = threadIdx.x / P;
        if (p0 < nla) {
            SegPoly<DD> sp;
            if (D == DD) sp.load(&wc[a2 * (D + 1)]);
            for (int p = p0; p < nc; p += nla) {
                const float4 rec = crec[p];
                float* W = wts + p * WS + a2;
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) {
                    const float tt = ax == 0 ? rec.x : (ax == 1 ? rec.y : rec.z);
                    if (D == DD) {
                        W[ax * 2 * P] = sp.w(tt);
                        W[ax * 2 * P + P] = sp.dw(tt);
                    } else {
                        W[ax * 2 * P] = horner_w(&wc[a2 * (D + 1)], D, tt);
                        W[ax * 2 * P + P] = horner_dw(&wc[a2 * (D + 1)], D, tt);
                    }
                }
            }
        }
        for (int p = threadIdx.x; p < nc; p += blockDim.x) {
            qv[p] = crec[p].w;
            org[p] = (int)crel[p];
        }
    }
    __syncthreads();
    if (C::CH <= 32 && threadIdx.x < 32) {
        // processing order: queue position q prefers a particle whose
        // bank class (ox + oy) mod K is q mod K, so the K groups of a warp
        // read potential rows in disjoint bank classes (plane pitch = K
        // mod 32, row pitch = 1 mod K); particles left over fill the free
        // positions in order
        const int j = threadIdx.x;
        const unsigned full = 0xffffffffu, lt = (1u << j) - 1u;
        const bool valid = j < nc;
        // bank class of the particle's rows: (ox + oy) mod K for the padded
        // cp.async layout; ox + xoff mod K for the TMA box (pitches = 0 mod K)
        const int cls = valid ? ((TMA ? (org[j] & 255) + xoff : (org[j] & 255) + ((org[j] >> 8) & 255)) & (K - 1))
                              : -1;
        int rank = 0, cpos = 0;
        const int pk = j & (K - 1);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const unsigned m = __ballot_sync(full, cls == k);
            if (cls == k) rank = __popc(m & lt);
            if (pk == k) cpos = __popc(m);
        }
        const int slots = valid ? (nc - cls + K - 1) / K : 0;
        const bool placed = valid && rank < slots;
        const unsigned fm = __ballot_sync(full, j < nc && j / K >= cpos);
        const unsigned lm = __ballot_sync(full, valid && !placed);
        if (placed) order[cls + K * rank] = j;
        else if (valid) order[__fns(fm, 0, __popc(lm & lt) + 1)] = j;
    } else if (C::CH > 32) {
        for (int p = threadIdx.x; p < nc; p += blockDim.x) order[p] = p;
    }
    __syncthreads();
    for (int pp = 0; pp < nc; pp += C::NG) {
        const int qq = pp + grp;
        const int p = qq < nc ? order[qq] : qq;
        const bool act = qq < nc && gl < P;
        float pot = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
        if (act) {
            const float* W = wts + p * WS;
            float wx[P], dwx[P];
#pragma unroll
            for (int a2 = 0; a2 < P; ++a2) {
                wx[a2] = W[a2];
                dwx[a2] = W[P + a2];
            }
            const int rl = org[p];
            const int ox = rl & 255, oy = (rl >> 8) & 255, oz = (rl >> 16) & 255;
            const float* plane = sm + (oz + gl) * PP + oy * PX + ox + xoff;
            float Sv = 0.f, Dv = 0.f, Sy = 0.f;
#pragma unroll
            for (int b = 0; b < P; ++b) {
                const float* row = plane + b * PX;
                float sr = 0.f, dr = 0.f;
#pragma unroll
                for (int a2 = 0; a2 < P; ++a2) {
                    const float v = row[a2];
                    sr = fmaf(v, wx[a2], sr);
                    dr = fmaf(v, dwx[a2], dr);
                }
                const float wyb = W[2 * P + b], dwyb = W[3 * P + b];
                Sv = fmaf(sr, wyb, Sv);
                Dv = fmaf(dr, wyb, Dv);
                Sy = fmaf(sr, dwyb, Sy);
            }
            const float wzc = W[4 * P + gl], dwzc = W[5 * P + gl];
            pot = Sv * wzc;
            gx = Dv * wzc;
            gy = Sy * wzc;
            gz = Sv * dwzc;
        }
#pragma unroll
        for (int o = C::G / 2; o > 0; o >>= 1) {
            pot += __shfl_xor_sync(0xffffffffu, pot, o, C::G);
            gx += __shfl_xor_sync(0xffffffffu, gx, o, C::G);
            gy += __shfl_xor_sync(0xffffffffu, gy, o, C::G);
            gz += __shfl_xor_sync(0xffffffffu, gz, o, C::G);
        }
        if (qq < nc && gl == 0) {
            const float q = qv[p];
            const double e_i = 0.5 * (double)q * pot + self_coef * (double)q * q;
            force[cprm[p]] = make_float4(q * gxs * gx, q * gys * gy, q * gzs * gz, (float)e_i);
            esum += e_i;
        }
    }
    return esum;
}

template <int P, bool TMA>
__global__ void __launch_bounds__(128, 6)
    k_interp(const int* __restrict__ tile_sys, const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets,
             int T, int D, int PX, int PP, const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm,
             const float4* __restrict__ srec, const uint32_t* __restrict__ srel, const float* __restrict__ phi,
             float4* __restrict__ force, double* __restrict__ acc, const CUtensorMap* __restrict__ tmaps,
             int* __restrict__ kerr) {
    using C = InterpCfg<P>;
    extern __shared__ float4 sm4[];
    __shared__ double red[32];
    __shared__ __align__(8) uint64_t mbar;
    const int t = blockIdx.x;
    const uint32_t s0 = start[t];
    const int np = (int)(start[t + 1] - s0);
    if (np == 0) return;
    const int si = tile_sys[t];
    const SysDev S = sys[si];
    const ParamSet& ps = psets[S.pset];
    const int E = T + P - 1;
    // the potential region (128-byte aligned for the TMA box), then the
    // particle records (position/t, origin, output slot) of the current and
    // the next chunk: the next chunk's are prefetched while this one runs
    float* sm = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(sm4) + 127) & ~(uintptr_t)127);  // [E*PP]
    float4* crec = reinterpret_cast<float4*>(sm + ((E * PP + 3) & ~3));    // [2][CH]
    uint32_t* crel = reinterpret_cast<uint32_t*>(crec + 2 * C::CH);         // [2][CH]
    uint32_t* cprm = crel + 2 * C::CH;                                      // [2][CH]
    float* wts = reinterpret_cast<float*>(cprm + 2 * C::CH);  // [CH][6P] wx dwx wy dwy wz dwz (index tables first)
    float* qv = wts + interp_stage_words(P, C::CH, E);  // [CH] charges
    int* org = reinterpret_cast<int*>(qv + C::CH); // [CH] packed origins
    int* order = org + C::CH;                      // [CH] processing order of the chunk
    float* wc = reinterpret_cast<float*>(order + C::CH);  // [P][D+1]
    const int lt = t - S.t_off;
    const int X0 = (lt % S.ntx) * T, Y0 = ((lt / S.ntx) % S.nty) * T, Z0 = (lt / (S.ntx * S.nty)) * T;
    // TMA boxes start on a 16-byte boundary in x: the region sits xoff floats in
    const int xoff = TMA ? (X0 & 3) : 0;
    const uint32_t mbar_a = (uint32_t)__cvta_generic_to_shared(&mbar);
    if (TMA) {
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar_a) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
            const uint32_t bytes = (uint32_t)(E * PP) * 4u;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar_a), "r"(bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
                "[%5];\n" ::"r"((uint32_t)__cvta_generic_to_shared(sm)),
                "l"(reinterpret_cast<uint64_t>(tmaps + si)), "r"(X0 - xoff), "r"(Y0), "r"(Z0), "r"(mbar_a)
                : "memory");
        }
        __syncthreads();  // the barrier is initialised before anyone waits on it
    } else {
        // stage the extended region with asynchronous 4-byte copies (every
        // thread keeps all its loads in flight)
        // wrapped global row offsets and shared row offsets per (Y, Z) row,
        // wrapped x indices, then one 4-byte asynchronous copy per point
        // (all of a thread's copies in flight)
        int* rowo = reinterpret_cast<int*>(wts);  // the staging area holds the index tables first
        int* srow = rowo + E * E;
        int* xs = srow + E * E;
        for (int i = threadIdx.x; i < E * E; i += blockDim.x) {
            const int Y = i % E, Z = i / E;
            rowo[i] = ((Z0 + Z) * S.nyp + (Y0 + Y)) * S.nxp;  // the halo-padded mesh needs no wrap
            srow[i] = Z * PP + Y * PX;
        }
        for (int i = threadIdx.x; i < E; i += blockDim.x) xs[i] = X0 + i;
        __syncthreads();
        const float* base = phi + S.mp_off;
        const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
        // rows padded to a power of two wide, so the point index splits by shifts
        int sh = 4;
        while ((1 << sh) < E) ++sh;
        for (int idx = threadIdx.x; idx < (E * E) << sh; idx += blockDim.x) {
            const int r = idx >> sh, X = idx & ((1 << sh) - 1);
            if (X < E)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sbase + 4u * (uint32_t)(srow[r] + X)),
                             "l"(base + rowo[r] + xs[X]));
        }
        asm volatile("cp.async.commit_group;\n" ::);
    }
    auto prefetch = [&](int base, int buf) {
        const int n = min(C::CH, np - base);
        for (int p = threadIdx.x; p < n; p += blockDim.x) {
            const uint32_t d1 = (uint32_t)__cvta_generic_to_shared(&crec[buf * C::CH + p]);
            const uint32_t d2 = (uint32_t)__cvta_generic_to_shared(&crel[buf * C::CH + p]);
            const uint32_t d3 = (uint32_t)__cvta_generic_to_shared(&cprm[buf * C::CH + p]);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d1), "l"(srec + s0 + base + p));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d2), "l"(srel + s0 + base + p));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d3), "l"(perm + s0 + base + p));
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    prefetch(0, 0);
    asm volatile("cp.async.wait_group 0;\n" ::);  // region (cp.async form) and first chunk
    if (TMA) {
        const bool ok = tma_wait(mbar_a, 0u);
        if (__syncthreads_or(!ok)) {
            // the box did not arrive in time: report, let the copy drain
            // (bounded), skip the tile (the whole CTA)
            if (threadIdx.x == 0) atomicOr(kerr, 1);
            tma_wait(mbar_a, 0u);
            return;
        }
    }
    for (int i = threadIdx.x; i < P * (D + 1); i += blockDim.x)
        wc[i] = ps.wcoef[(i / (D + 1)) * (MAX_D + 1) + (i % (D + 1))];
    const float gxs = (float)S.gxd, gys = (float)S.gyd, gzs = (float)S.gzd;
    const double self_coef = ps.self_coef;
    double esum = 0.0;
    for (int base = 0, cb = 0; base < np; base += C::CH, cb ^= 1) {
        const int nc = min(C::CH, np - base);
        __syncthreads();  // region / coefficients / records staged; previous chunk consumed
        if (base + C::CH < np) prefetch(base + C::CH, cb ^ 1);
        esum += interp_chunk<P, TMA>(sm, PX, PP, xoff, D, wc, crec + cb * C::CH, crel + cb * C::CH,
                                     cprm + cb * C::CH, wts, qv, org, order, nc, gxs, gys, gzs, self_coef, force);
        asm volatile("cp.async.wait_group 0;\n" ::);  // next chunk's records (made visible by the top barrier)
    }
    double ev[1] = {esum};
    block_sum_f64<1>(ev, red);
    if (threadIdx.x == 0) atomicAdd(&acc[si * ACC_STRIDE + ACC_E], ev[0]);
}

// Persistent TMA form, fed from a tile queue: a grid of resident CTAs takes
// tiles from one counter (cleared by the host before the launch). Each CTA
// keeps two potential-region buffers: while it interpolates tile t, the box
// of the tile it takes next is already in flight into the other buffer, and
// that tile's first chunk of particle records is prefetched during t's last
// chunk. Thread 0 runs the queue three tiles ahead (counter, then the tile's
// system and record range, then the system's tile grid), one stage per tile,
// so none of those dependent loads is waited for. A box wait that runs out
// sets kerr[0]; the CTA then drains its copies (bounded) and leaves the rest
// of the queue to the other CTAs.
__host__ __device__ inline int interp_q_region_words(int E, int PP) {
    return (E * PP + 31) & ~31;  // 128-byte multiple
}

template <int P>
__host__ __device__ inline int interp_q_smem(int E, int PP) {
    using C = InterpCfg<P>;
    return 128 + 4 * (2 * interp_q_region_words(E, PP) + C::CH * (6 * P + 1) + 3 * C::CH + P * (MAX_D + 1)) +
           2 * C::CH * 24;
}

template <int P>
__global__ void __launch_bounds__(128, 5)
    k_interp_q(const int* __restrict__ tile_sys, const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets,
               int n_tiles, int T, int D, int PX, int PP, const uint32_t* __restrict__ start,
               const uint32_t* __restrict__ perm, const float4* __restrict__ srec, const uint32_t* __restrict__ srel,
               float4* __restrict__ force, double* __restrict__ acc, const CUtensorMap* __restrict__ tmaps,
               int* __restrict__ kerr, int* __restrict__ queue) {
    using C = InterpCfg<P>;
    extern __shared__ float4 sm4[];
    __shared__ double red[32];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ int s_tile[2], s_first[2], s_np[2];  // tile whose box goes to buffer b (n_tiles: none)
    const int E = T + P - 1;
    const int RW = interp_q_region_words(E, PP);
    float* reg0 = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(sm4) + 127) & ~(uintptr_t)127);
    float4* crec = reinterpret_cast<float4*>(reg0 + 2 * RW);       // [2][CH]
    uint32_t* crel = reinterpret_cast<uint32_t*>(crec + 2 * C::CH);  // [2][CH]
    uint32_t* cprm = crel + 2 * C::CH;                               // [2][CH]
    float* wts = reinterpret_cast<float*>(cprm + 2 * C::CH);         // [CH][6P + 1]
    float* qv = wts + C::CH * (6 * P + 1);                           // [CH]
    int* org = reinterpret_cast<int*>(qv + C::CH);                   // [CH]
    int* order = org + C::CH;                                        // [CH]
    float* wc = reinterpret_cast<float*>(order + C::CH);             // [P][D+1]
    const int tid = threadIdx.x;
    const uint32_t mb0 = (uint32_t)__cvta_generic_to_shared(&mbar[0]);
    const uint32_t box_bytes = (uint32_t)(E * PP) * 4u;
    // thread 0's queue pipeline: q0 = index from the counter; q1 = + system
    // and record range; q2 = + the system's tile grid (ready to issue)
    int q0 = n_tiles, q1 = n_tiles, q1_si = 0, q2 = n_tiles, q2_si = 0, q2_ntx = 1, q2_nty = 1, q2_toff = 0;
    uint32_t q1_f = 0, q1_e = 0, q2_f = 0, q2_np = 0;
    // shifts the pipeline by one tile; the tile leaving q2 gets its box
    // issued into buffer b (or buffer b is marked empty)
    auto advance = [&](int b) {
        const int t = q2;
        s_tile[b] = t;
        s_first[b] = (int)q2_f;
        s_np[b] = (int)q2_np;
        if (t < n_tiles) {
            const int lt = t - q2_toff;
            const int X0 = (lt % q2_ntx) * T, Y0 = ((lt / q2_ntx) % q2_nty) * T, Z0 = (lt / (q2_ntx * q2_nty)) * T;
            const uint32_t mb = mb0 + 8u * (uint32_t)b;
            // the buffer was last read by generic loads of this CTA
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mb), "r"(box_bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
                "[%5];\n" ::"r"((uint32_t)__cvta_generic_to_shared(reg0 + b * RW)),
                "l"(reinterpret_cast<uint64_t>(tmaps + q2_si)), "r"(X0 - (X0 & 3)), "r"(Y0), "r"(Z0), "r"(mb)
                : "memory");
        }
        q2 = q1;
        q2_si = q1_si;
        q2_f = q1_f;
        q2_np = q1_e - q1_f;
        if (q1 < n_tiles) {
            const SysDev& S = sys[q1_si];
            q2_ntx = S.ntx;
            q2_nty = S.nty;
            q2_toff = S.t_off;
        }
        q1 = q0;
        if (q0 < n_tiles) {
            q1_si = tile_sys[q0];
            q1_f = start[q0];
            q1_e = start[q0 + 1];
        }
        q0 = atomicAdd(queue, 1);
        if (q0 > n_tiles) q0 = n_tiles;
    };
    auto prefetch = [&](uint32_t first, int n, int buf) {
        for (int p = tid; p < n; p += blockDim.x) {
            const uint32_t d1 = (uint32_t)__cvta_generic_to_shared(&crec[buf * C::CH + p]);
            const uint32_t d2 = (uint32_t)__cvta_generic_to_shared(&crel[buf * C::CH + p]);
            const uint32_t d3 = (uint32_t)__cvta_generic_to_shared(&cprm[buf * C::CH + p]);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d1), "l"(srec + first + p));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d2), "l"(srel + first + p));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d3), "l"(perm + first + p));
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb0 + 8u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        q0 = min(atomicAdd(queue, 1), n_tiles);
        advance(1);  // fills the pipeline (buffer 1 marked empty on the way)
        advance(1);
        advance(0);  // the first tile's box
    }
    __syncthreads();
    int b = 0, cbuf = 0, cur_pset = -1;
    uint32_t ph[2] = {0u, 0u};
    int t = s_tile[0];
    if (t < n_tiles) prefetch((uint32_t)s_first[0], min(C::CH, s_np[0]), 0);
    while (t < n_tiles) {
        const uint32_t s0 = (uint32_t)s_first[b];
        const int np = s_np[b];
        const int si = tile_sys[t];
        const SysDev& S = sys[si];
        const ParamSet& ps = psets[S.pset];
        const int xoff = ((t - S.t_off) % S.ntx) * T & 3;
        if (S.pset != cur_pset) {  // read after the chunk loop's top barrier
            cur_pset = S.pset;
            for (int i = tid; i < P * (D + 1); i += blockDim.x)
                wc[i] = ps.wcoef[(i / (D + 1)) * (MAX_D + 1) + (i % (D + 1))];
        }
        const bool ok = tma_wait(mb0 + 8u * (uint32_t)b, ph[b]);
        ph[b] ^= 1u;
        if (__syncthreads_or(!ok)) {
            // the box did not arrive in time: report, drain this CTA's copies
            // (bounded) and stop taking tiles
            if (tid == 0) atomicOr(kerr, 1);
            tma_wait(mb0 + 8u * (uint32_t)b, ph[b] ^ 1u);
            asm volatile("cp.async.wait_group 0;\n" ::);
            return;
        }
        // this box has arrived and the previous tile is done: start the next one
        if (tid == 0) advance(b ^ 1);
        const float gxs = (float)S.gxd, gys = (float)S.gyd, gzs = (float)S.gzd;
        const double self_coef = ps.self_coef;
        double esum = 0.0;
        for (int base = 0; base < np; base += C::CH) {
            const int nc = min(C::CH, np - base);
            asm volatile("cp.async.wait_group 0;\n" ::);  // this chunk's records
            __syncthreads();  // records, coefficients and the next tile's range visible; previous chunk consumed
            if (base + C::CH < np) {
                prefetch(s0 + base + C::CH, min(C::CH, np - base - C::CH), cbuf ^ 1);
            } else if (s_tile[b ^ 1] < n_tiles) {
                prefetch((uint32_t)s_first[b ^ 1], min(C::CH, s_np[b ^ 1]), cbuf ^ 1);
            }
            esum += interp_chunk<P, true>(reg0 + b * RW, PX, PP, xoff, D, wc, crec + cbuf * C::CH,
                                          crel + cbuf * C::CH, cprm + cbuf * C::CH, wts, qv, org, order, nc, gxs, gys,
                                          gzs, self_coef, force);
            cbuf ^= 1;
        }
        if (np == 0) {
            // an empty tile: its box is not read; the next tile's range
            // becomes visible here, and its first records are prefetched
            __syncthreads();
            if (s_tile[b ^ 1] < n_tiles) prefetch((uint32_t)s_first[b ^ 1], min(C::CH, s_np[b ^ 1]), cbuf);
        }
        double ev[1] = {esum};
        block_sum_f64<1>(ev, red);
        if (tid == 0 && np > 0) atomicAdd(&acc[si * ACC_STRIDE + ACC_E], ev[0]);
        t = s_tile[b ^ 1];
        b ^= 1;
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// ============================================================================
// a8: short-range pair term over a HOOMD-layout neighbour list
// (neighbours of i: nlist[head[i] + k], k < n_neigh[i], local indices).
// TPP lanes cooperate on one particle; per pair
//   pair_eng = qiqj/(4 pi) (1/r - Q(u)/r_c),  u = r^2/r_c^2
//   force_divr = qiqj/(4 pi) (1/r^3 + 2 Q'(u)/r_c^3)
// (the split form of EvaluatorPairPSWF::evalForceAndEnergy).
// ============================================================================
// EN: pair energies (per particle and per system); without them the split
// polynomial Q itself is not needed, only Q', and the kernel (40 registers)
// keeps 6 CTAs per SM resident so that more position gathers are in flight.
// Each lane loads its next 16-byte row segment of neighbour indices one
// iteration ahead of the gathers that use it.
template <int TPP, int NQ, bool VIR, bool EN>
__global__ void __launch_bounds__(256, EN ? 5 : 6)
    k_pair(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets,
           const float4* __restrict__ posq, const uint32_t* __restrict__ head, const uint32_t* __restrict__ nn,
           const uint32_t* __restrict__ nlist, float4* __restrict__ force, double* __restrict__ acc, int accumulate,
           const PairCoef pc, float* __restrict__ vpp, int vpitch, const uint32_t* __restrict__ outidx) {
    __shared__ double red[32 * 7];
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const ParamSet& ps = psets[S.pset];
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
    const int i = ch.y + threadIdx.x / TPP;
    const int sub = threadIdx.x % TPP;
    const bool valid = i < S.p_off + S.N;
    // particles at least r_c from every face (positions are wrapped into
    // the box) see every in-cutoff neighbour in the same image; a warp whose
    // particles all are skips the minimum-image wrap (out-of-cutoff pairs
    // are masked whatever their displacement)
    bool inner = true;
    if (valid) {
        const float4 p = posq[i];
        const float rc = ps.rcut;
        inner = p.x >= rc && p.x <= S.Lx - rc && p.y >= rc && p.y <= S.Ly - rc && p.z >= rc && p.z <= S.Lz - rc;
    }
    const bool interior = __all_sync(0xffffffffu, inner);
    if (valid) {
        const float4 pi = posq[i];
        const uint32_t n = nn[i], h = head[i];
        const int po = S.p_off;
        uint32_t k0 = 0;
        if ((h & 3u) == 0u) {
            // 16-byte row segments: each lane streams 4 neighbour indices
            const uint4* row = reinterpret_cast<const uint4*>(nlist + h);
            const uint32_t n4 = n >> 2;
            if (interior) {
                uint4 jn = sub < n4 ? __ldg(&row[sub]) : make_uint4(0u, 0u, 0u, 0u);
                for (uint32_t k4 = sub; k4 < n4; k4 += TPP) {
                    const uint4 jj = jn;  // this row segment; the next one is loaded ahead
                    if (k4 + TPP < n4) jn = __ldg(&row[k4 + TPP]);
                    const float4 p0 = __ldg(&posq[po + (int)jj.x]);
                    const float4 p1 = __ldg(&posq[po + (int)jj.y]);
                    const float4 p2 = __ldg(&posq[po + (int)jj.z]);
                    const float4 p3 = __ldg(&posq[po + (int)jj.w]);
                    ev.template pair<false>(pi, p0);
                    ev.template pair<false>(pi, p1);
                    ev.template pair<false>(pi, p2);
                    ev.template pair<false>(pi, p3);
                }
            } else {
                uint4 jn = sub < n4 ? __ldg(&row[sub]) : make_uint4(0u, 0u, 0u, 0u);
                for (uint32_t k4 = sub; k4 < n4; k4 += TPP) {
                    const uint4 jj = jn;
                    if (k4 + TPP < n4) jn = __ldg(&row[k4 + TPP]);
                    const float4 p0 = __ldg(&posq[po + (int)jj.x]);
                    const float4 p1 = __ldg(&posq[po + (int)jj.y]);
                    const float4 p2 = __ldg(&posq[po + (int)jj.z]);
                    const float4 p3 = __ldg(&posq[po + (int)jj.w]);
                    ev.pair(pi, p0);
                    ev.pair(pi, p1);
                    ev.pair(pi, p2);
                    ev.pair(pi, p3);
                }
            }
            k0 = n4 << 2;
        }
        for (uint32_t k = k0 + sub; k < n; k += TPP) ev.pair(pi, __ldg(&posq[po + (int)__ldg(&nlist[h + k])]));
    }
    float fx = ev.fx, fy = ev.fy, fz = ev.fz, en = ev.en;
#pragma unroll
    for (int o = TPP / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
        en += __shfl_xor_sync(0xffffffffu, en, o);
    }
    // rows by slot (the library's pair list): results go to the particle of the slot
    const int oi = (outidx && valid) ? (int)outidx[i] : i;
    if (valid && sub == 0) {
        float4 f = accumulate ? force[oi] : make_float4(0.f, 0.f, 0.f, 0.f);
        f.x += fx;
        f.y += fy;
        f.z += fz;
        f.w += 0.5f * en;
        force[oi] = f;
    }
    if (VIR && vpp) {
        // this particle's half of its pairs' virial (HOOMD's per-particle virial)
        float v[6] = {ev.vxx, ev.vxy, ev.vxz, ev.vyy, ev.vyz, ev.vzz};
#pragma unroll
        for (int o = TPP / 2; o > 0; o >>= 1)
#pragma unroll
            for (int k = 0; k < 6; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        if (valid && sub == 0)
#pragma unroll
            for (int k = 0; k < 6; ++k) vpp[(size_t)k * vpitch + oi] += 0.5f * v[k];
    }
    if (VIR) {
        double e[7] = {sub == 0 ? 0.5 * (double)en : 0.0, 0.5 * (double)ev.vxx, 0.5 * (double)ev.vxy,
                       0.5 * (double)ev.vxz, 0.5 * (double)ev.vyy, 0.5 * (double)ev.vyz, 0.5 * (double)ev.vzz};
        block_sum_f64<7>(e, red);
        if (threadIdx.x == 0) {
            atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_E], e[0]);
#pragma unroll
            for (int k = 0; k < 6; ++k) atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_WP + k], e[1 + k]);
        }
    } else if (EN) {
        double e[1] = {sub == 0 ? 0.5 * (double)en : 0.0};
        block_sum_f64<1>(e, red);
        if (threadIdx.x == 0) atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_E], e[0]);
    }
}

// Energy and virial per system: E = sum_i e_i + E_bg; W = W_k + W_pair + E_bg I.
// external (may be NULL): the terms no particle owns, {E_bg, W_k + E_bg I}.
__global__ void k_finalize(const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets, int nsys,
                           const double* __restrict__ acc, double* __restrict__ energy, double* __restrict__ virial,
                           int add_bg, double* __restrict__ external) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const SysDev S = sys[s];
    const double* a = acc + s * ACC_STRIDE;
    const double Q = a[ACC_QSUM];
    const double ebg = add_bg ? psets[S.pset].bg_coef * Q * Q / S.V : 0.0;
    const int diag[6] = {1, 0, 0, 1, 0, 1};
    if (energy) energy[s] = a[ACC_E] + ebg;
    if (virial)
        for (int k = 0; k < 6; ++k)
            virial[s * 6 + k] = a[ACC_WK + k] + a[ACC_WP + k] + a[ACC_WX + k] + (diag[k] ? ebg : 0.0);
    if (external) {
        external[7 * s] = ebg;
        for (int k = 0; k < 6; ++k) external[7 * s + 1 + k] = a[ACC_WK + k] + (diag[k] ? ebg : 0.0);
    }
}

// ============================================================================
// Reference-format evaluator: detail::pswf_eval_L + evalForceAndEnergy of
// src/EvaluatorPairPSWF.h:113-143, 274-295, reading a PSWF_Coeffs.h-layout
// segment table. Rounding is pinned (_rn intrinsics, no FMA contraction)
// so the FP64 instance reproduces a host compile of the reference.
// ============================================================================
__device__ __forceinline__ double seg_horner5(const double* __restrict__ c, double t) {
    double v = c[4];
    v = __dadd_rn(c[3], __dmul_rn(t, v));
    v = __dadd_rn(c[2], __dmul_rn(t, v));
    v = __dadd_rn(c[1], __dmul_rn(t, v));
    v = __dadd_rn(c[0], __dmul_rn(t, v));
    return v;
}

__global__ void k_pswf_eval_pairs(int n, const double* __restrict__ rsq, const double* __restrict__ qiqj,
                                  double rcut, double rcutsq, int n_segs, const double* __restrict__ screen,
                                  const double* __restrict__ dscreen, const double* __restrict__ r_lo,
                                  const double* __restrict__ dr_inv, double* __restrict__ force_divr,
                                  double* __restrict__ pair_eng, int* __restrict__ evaluated) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double r2 = rsq[i], qq = qiqj[i];
    double fd = 0.0, pe = 0.0;
    int ok = 0;
    if (!(r2 >= rcutsq || qq == 0.0 || rcut < 1.0e-12)) {
        ok = 1;
        // the reference calls sqrtf() on a double (FP32 square root)
        const double r = (double)sqrtf((float)r2);
        const double rinv = 1.0 / r;
        double L = 0.0, negdLdr = 0.0;
        if (!(r < 1.0e-12 || r > rcut)) {
            double s = r / rcut;
            s = s < 0.0 ? 0.0 : (s > 1.0 - 1.0e-9 ? 1.0 - 1.0e-9 : s);
            unsigned int seg = (unsigned int)(s * (double)n_segs);
            seg = seg >= (unsigned int)n_segs ? (unsigned int)n_segs - 1u : seg;
            const double t = __dmul_rn(__dsub_rn(r, r_lo[seg]), dr_inv[seg]);
            const double S = seg_horner5(screen + (size_t)seg * 5, t);
            const double dS = seg_horner5(dscreen + (size_t)seg * 5, t);
            const double i4r = INV_4PI_D / r;
            const double i4r2 = i4r / r;
            L = __dmul_rn(S, i4r);
            negdLdr = __dsub_rn(__dmul_rn(S, i4r2), __dmul_rn(dS, i4r));
        }
        pe = __dmul_rn(qq, L);
        fd = __dmul_rn(__dmul_rn(qq, negdLdr), rinv);
    }
    force_divr[i] = fd;
    pair_eng[i] = pe;
    evaluated[i] = ok;
}

// ============================================================================
// host launch wrappers
// ============================================================================
template <int P>
static cudaError_t launch_spread_p(const LaunchArgs& a, cudaStream_t st) {
    using C = SpreadCfg<P>;
    const bool mma = a.T + P - 1 == SPREAD_EM && a.spread_mode == 0;
    const bool dense = a.T + P - 1 <= SPREAD_EM;
    const int nb = (a.T + 2 * P - 2) / P;
    const size_t NL = (size_t)nb * nb * nb * C::P3;
    const size_t smem = NL * sizeof(float2) + (size_t)C::CH * P * 4 * 4 + C::CH * 4 + P * (MAX_D + 1) * 4;
    const size_t smem_d = (size_t)SPREAD_CHD * 16 * 4 + (size_t)SPREAD_CHD * (2 * P + 1) * 4 + P * (MAX_D + 1) * 4;
    const size_t smem_m =
        (size_t)SPREAD_CHM * SPREAD_MS * 4 * 4 + 8 * 16 * 32 * 8 + 2 * SPREAD_CHM * 20 + P * (MAX_D + 1) * 4;
    if (a.configure_only) {
        cudaError_t e = cudaFuncSetAttribute(k_spread_mma<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_m);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k_spread_dense<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_d);
        if (e != cudaSuccess || dense) return e;
        return cudaFuncSetAttribute(k_spread<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    if (a.n_tiles == 0) return cudaSuccess;
    if (mma)
        k_spread_mma<P><<<a.n_tiles, 256, smem_m, st>>>(a.tile_sys, a.sys, a.psets, a.T, a.D, a.tile_start, a.srec,
                                                        a.srel, a.rho);
    else if (dense)
        k_spread_dense<P><<<a.n_tiles, 256, smem_d, st>>>(a.tile_sys, a.sys, a.psets, a.T, a.D, a.tile_start, a.srec,
                                                          a.srel, a.rho);
    else
        k_spread<P><<<a.n_tiles, C::THREADS, smem, st>>>(a.tile_sys, a.sys, a.psets, a.T, a.D, a.tile_start, a.srec,
                                                          a.srel, a.rho);
    return cudaGetLastError();
}

// shared memory of the interpolation kernel: the (128-byte aligned)
// potential region E x PP, the staging area, charges, origins, order and
// window coefficients, and two chunks of particle records
template <int P>
static size_t interp_smem(int E, int PP) {
    using C = InterpCfg<P>;
    return 128 + (size_t)((E * PP + 3) & ~3) * 4 +
           ((size_t)interp_stage_words(P, C::CH, E) + 3 * C::CH + P * (MAX_D + 1)) * 4 + 2 * C::CH * 24;
}

template <int P>
static cudaError_t launch_interp_p(const LaunchArgs& a, cudaStream_t st) {
    using C = InterpCfg<P>;
    const int E = a.T + P - 1;
    constexpr bool kTmaForm = P >= 5 && P <= 8;  // 8 lanes per particle: the box pitches give distinct banks
    const bool tma = kTmaForm && a.tmaps != nullptr;
    const int PX = tma ? a.tma_bx : a.PX, PP = tma ? a.tma_bx * a.tma_by : a.PP;
    if (a.configure_only) {
        // per-function limits shared by every batch of the process: raised
        // only, so a later plan with a smaller tile cannot lower them
        static int configured[3] = {0, 0, 0};
        cudaError_t e = cudaSuccess;
        const int s0 = (int)interp_smem<P>(E, a.PP);
        if (s0 > configured[0]) {
            e = cudaFuncSetAttribute(k_interp<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s0);
            if (e == cudaSuccess) configured[0] = s0;
        }
        const int s1 = (int)interp_smem<P>(E, a.tma_bx * a.tma_by);
        if (e == cudaSuccess && kTmaForm && a.tma_bx > 0 && s1 > configured[1]) {
            e = cudaFuncSetAttribute(k_interp<P, kTmaForm>, cudaFuncAttributeMaxDynamicSharedMemorySize, s1);
            if (e == cudaSuccess) configured[1] = s1;
        }
        const int s2 = interp_q_smem<P>(E, a.tma_bx * a.tma_by);
        if (e == cudaSuccess && kTmaForm && a.tma_bx > 0 && s2 > configured[2]) {
            e = cudaFuncSetAttribute(k_interp_q<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2);
            if (e == cudaSuccess) configured[2] = s2;
        }
        return e;
    }
    if (a.n_tiles == 0) return cudaSuccess;
    if (tma && a.queue) {
        // persistent CTAs, as many as are resident at once, fed from the queue
        const int smem = interp_q_smem<P>(E, PP);
        int per_sm = 0, dev = 0, n_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_interp_q<P>, C::THREADS, smem);
        if (e != cudaSuccess) return e;
        const int grid = std::max(1, std::min(a.n_tiles, std::max(per_sm, 1) * n_sm));
        if ((e = cudaMemsetAsync(a.queue, 0, sizeof(int), st)) != cudaSuccess) return e;
        k_interp_q<P><<<grid, C::THREADS, smem, st>>>(a.tile_sys, a.sys, a.psets, a.n_tiles, a.T, a.D, PX, PP,
                                                      a.tile_start, a.perm, a.srec, a.srel, a.force, a.acc,
                                                      reinterpret_cast<const CUtensorMap*>(a.tmaps), a.kerr, a.queue);
        return cudaGetLastError();
    }
    if (tma)
        k_interp<P, kTmaForm><<<a.n_tiles, C::THREADS, interp_smem<P>(E, PP), st>>>(
            a.tile_sys, a.sys, a.psets, a.T, a.D, PX, PP, a.tile_start, a.perm, a.srec, a.srel, a.phi, a.force, a.acc,
            reinterpret_cast<const CUtensorMap*>(a.tmaps), a.kerr);
    else
        k_interp<P, false><<<a.n_tiles, C::THREADS, interp_smem<P>(E, PP), st>>>(
            a.tile_sys, a.sys, a.psets, a.T, a.D, PX, PP, a.tile_start, a.perm, a.srec, a.srel, a.phi, a.force, a.acc,
            nullptr, a.kerr);
    return cudaGetLastError();
}

cudaError_t launch_scan(const uint32_t* cnt, uint32_t* start, int n, cudaStream_t st) {
    k_scan<<<1, 1024, 0, st>>>(cnt, start, n);
    return cudaGetLastError();
}

cudaError_t launch_scatter(const int2* chunks, int n_chunks, const SysDev* sys, const uint32_t* key,
                           const uint32_t* start, uint32_t* cnt, uint32_t* perm_u, cudaStream_t st) {
    if (n_chunks) k_scatter<<<n_chunks, 256, 0, st>>>(chunks, sys, key, start, cnt, perm_u);
    return cudaGetLastError();
}

cudaError_t launch_bin(const LaunchArgs& a, cudaStream_t st) {
    if (a.n_chunks == 0) return cudaSuccess;
    k_bin<<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.P, a.T, a.pos_in, a.q_in, a.posq, a.trec, a.rel, a.key,
                                      a.tile_count, a.acc, a.plist ? a.plist->idx2slot : nullptr,
                                      a.plist ? a.plist->spos : nullptr);
    return cudaGetLastError();
}

cudaError_t launch_sort(const LaunchArgs& a, cudaStream_t st) {
    k_scan<<<1, 1024, 0, st>>>(a.tile_count, a.tile_start, a.n_tiles);
    if (a.n_chunks) k_scatter<<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.key, a.tile_start, a.tile_count, a.perm_u);
    if (a.n_tiles)
        k_tile_sort<<<a.n_tiles, 128, 0, st>>>(a.tile_start, a.perm_u, a.perm, a.trec, a.rel, a.srec, a.srel,
                                               a.tile_sys, a.sys);
    return cudaGetLastError();
}

cudaError_t launch_spread(const LaunchArgs& a, cudaStream_t st) { ESPB_DISPATCH_P(launch_spread_p, a.P, a, st); }

cudaError_t launch_interp(const LaunchArgs& a, cudaStream_t st) { ESPB_DISPATCH_P(launch_interp_p, a.P, a, st); }

cudaError_t launch_fft(const LaunchArgs& a, cudaStream_t st) {
    // attributes allow the largest transform; launches request what the
    // batch's longest line on that axis needs (occupancy for small meshes)
    const size_t smx = 2 * (a.configure_only ? FFT_MAX_N : a.nmax_x) * FFT_SB_X * sizeof(float2);
    const size_t smy = 2 * (a.configure_only ? FFT_MAX_N : a.nmax_y) * FFT_B_YZ * sizeof(float2);
    const size_t smz = 2 * (a.configure_only ? FFT_MAX_N : a.nmax_z) * FFT_B_YZ * sizeof(float2);
    const size_t smyz = smy > smz ? smy : smz;
    if (a.configure_only) {
        cudaError_t e;
        if ((e = cudaFuncSetAttribute(k_fftx_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx))) return e;
        if ((e = cudaFuncSetAttribute(k_fftx_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx))) return e;
        if ((e = cudaFuncSetAttribute(k_ffty<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smyz))) return e;
        if ((e = cudaFuncSetAttribute(k_ffty<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smyz))) return e;
        if ((e = cudaFuncSetAttribute(k_fftz_conv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smyz))) return e;
        if ((e = cudaFuncSetAttribute(k_fftz_conv<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smyz)))
            return e;
        if ((e = cudaFuncSetAttribute(k_fft_plane_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, FFT_SMEM_MAX)))
            return e;
        if ((e = cudaFuncSetAttribute(k_fft_plane_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, FFT_SMEM_MAX)))
            return e;
        if ((e = cudaFuncSetAttribute(k_fft_slab_z<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, FFT_SMEM_MAX)))
            return e;
        return cudaFuncSetAttribute(k_fft_slab_z<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, FFT_SMEM_MAX);
    }
    if (a.n_pitems) k_fft_plane_fwd<<<a.n_pitems, 256, a.smem_plane, st>>>(a.pitems, a.sys, a.tw, a.rho, a.spec);
    if (a.n_xitems) k_fftx_fwd<<<a.n_xitems, 256, smx, st>>>(a.xitems, a.sys, a.tw, a.rho, a.spec);
    if (a.n_yitems) k_ffty<false><<<a.n_yitems, 256, smy, st>>>(a.yitems, a.sys, a.tw, a.spec);
    if (a.n_sitems) {
        if (a.want_virial)
            k_fft_slab_z<true><<<a.n_sitems, 256, a.smem_slab, st>>>(a.sitems, a.sys, a.tw, a.gtab, a.spec, a.acc);
        else
            k_fft_slab_z<false><<<a.n_sitems, 256, a.smem_slab, st>>>(a.sitems, a.sys, a.tw, a.gtab, a.spec, a.acc);
    }
    if (a.n_zitems) {
        if (a.want_virial)
            k_fftz_conv<true><<<a.n_zitems, 256, smz, st>>>(a.zitems, a.sys, a.tw, a.gtab, a.spec, a.acc);
        else
            k_fftz_conv<false><<<a.n_zitems, 256, smz, st>>>(a.zitems, a.sys, a.tw, a.gtab, a.spec, a.acc);
    }
    if (a.n_yitems) k_ffty<true><<<a.n_yitems, 256, smy, st>>>(a.yitems, a.sys, a.tw, a.spec);
    if (a.n_xitems) k_fftx_inv<<<a.n_xitems, 256, smx, st>>>(a.xitems, a.sys, a.tw, a.spec, a.phi, a.rho);
    if (a.n_pitems) k_fft_plane_inv<<<a.n_pitems, 256, a.smem_plane, st>>>(a.pitems, a.sys, a.tw, a.spec, a.phi, a.rho);
    return cudaGetLastError();
}

template <int TPP, bool VIR, bool EN>
static cudaError_t launch_pair_t(const LaunchArgs& a, cudaStream_t st) {
    // the library's pair list: rows by slot over the slot-ordered positions
    const PairList* pl = a.plist;
    const float4* posq = pl ? pl->spos : a.posq;
    const uint32_t* head = pl ? pl->head : a.nl_head;
    const uint32_t* nn = pl ? pl->nn : a.nl_n;
    const uint32_t* nl = pl ? pl->nl : a.nl_list;
    const uint32_t* outidx = pl ? pl->slot2idx : nullptr;
#define ESPB_PAIR(NQ)                                                                                          \
    k_pair<TPP, NQ, VIR, EN><<<a.n_pchunks, 256, 0, st>>>(a.pchunks, a.sys, a.psets, posq, head, nn, nl, a.force, \
                                                          a.acc, a.accumulate, a.pc, a.virial_pp, a.vpp_pitch,    \
                                                          outidx)
    if (a.nq <= 8) ESPB_PAIR(8);
    else if (a.nq <= 10) ESPB_PAIR(10);
    else if (a.nq <= 11) ESPB_PAIR(11);
    else if (a.nq <= 12) ESPB_PAIR(12);
    else if (a.nq <= 13) ESPB_PAIR(13);
    else if (a.nq <= 14) ESPB_PAIR(14);
    else if (a.nq <= 16) ESPB_PAIR(16);
    else if (a.nq <= 20) ESPB_PAIR(20);
    else if (a.nq <= 24) ESPB_PAIR(24);
    else ESPB_PAIR(32);
#undef ESPB_PAIR
    return cudaGetLastError();
}

cudaError_t launch_pair(const LaunchArgs& a, cudaStream_t st) {
    if (a.n_pchunks == 0) return cudaSuccess;
    if (a.want_virial) {
        switch (a.tpp) {
            case 4: return launch_pair_t<4, true, true>(a, st);
            case 8: return launch_pair_t<8, true, true>(a, st);
            case 16: return launch_pair_t<16, true, true>(a, st);
            case 32: return launch_pair_t<32, true, true>(a, st);
            default: return cudaErrorInvalidValue;
        }
    }
    if (a.want_energy) {
        switch (a.tpp) {
            case 4: return launch_pair_t<4, false, true>(a, st);
            case 8: return launch_pair_t<8, false, true>(a, st);
            case 16: return launch_pair_t<16, false, true>(a, st);
            case 32: return launch_pair_t<32, false, true>(a, st);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (a.tpp) {
        case 4: return launch_pair_t<4, false, false>(a, st);
        case 8: return launch_pair_t<8, false, false>(a, st);
        case 16: return launch_pair_t<16, false, false>(a, st);
        case 32: return launch_pair_t<32, false, false>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

// ============================================================================
// a9 (K7): exclusion correction, src/ESPForceComputeGPU.cu:391-471. The mesh
// sums q_i q_j Phi(r) over every pair, Phi = 1/(4 pi r) - L(r): that is
// Q(r^2/r_c^2) / (4 pi r_c) inside r_c and the bare 1/(4 pi r) beyond. For
// each excluded pair this kernel subtracts it: force, half the pair energy
// per side (exclusions are listed from both sides) and the virial. Unlike
// the reference, which skips excluded pairs beyond r_c, pairs at any
// distance are corrected. One thread per particle, after the interpolation
// has written the mesh forces.
// ============================================================================
__global__ void k_exclusions(const int2* __restrict__ chunks, const SysDev* __restrict__ sys,
                             const ParamSet* __restrict__ psets, const float4* __restrict__ posq,
                             const uint32_t* __restrict__ n_ex, const uint32_t* __restrict__ ex_list, int ex_pitch,
                             float4* __restrict__ force, double* __restrict__ acc, float* __restrict__ vpp,
                             int vpitch) {
    __shared__ double red[32 * 7];
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const ParamSet& ps = psets[S.pset];
    const int i = ch.y + threadIdx.x;
    const bool valid = i < S.p_off + S.N;
    const uint32_t n = valid ? n_ex[i] : 0u;
    float fx = 0.f, fy = 0.f, fz = 0.f, en = 0.f, v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (n > 0) {
        const float4 pi = posq[i];
        const float irc2 = ps.inv_rcut * ps.inv_rcut;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t jl = ex_list[(size_t)i * ex_pitch + k];
            if (jl >= (uint32_t)S.N) continue;
            const float4 pj = posq[S.p_off + (int)jl];
            float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            dx -= S.Lx * rintf(dx * S.inv_Lx);
            dy -= S.Ly * rintf(dy * S.inv_Ly);
            dz -= S.Lz * rintf(dz * S.inv_Lz);
            const float r2 = dx * dx + dy * dy + dz * dz;
            float phi, dphi_r;  // Phi and (dPhi/dr) / r
            if (r2 < ps.rcut2) {
                const float vv = fmaf(2.f * irc2, r2, -1.f);
                float qv = ps.qv[ps.nq - 1], dq = ps.nq >= 2 ? ps.dqv[ps.nq - 2] : 0.f;
                for (int c = ps.nq - 2; c >= 0; --c) qv = fmaf(qv, vv, ps.qv[c]);
                for (int c = ps.nq - 3; c >= 0; --c) dq = fmaf(dq, vv, ps.dqv[c]);
                phi = INV_4PI_F * qv * ps.inv_rcut;
                dphi_r = INV_4PI_F * ps.two_inv_rcut3 * dq;
            } else {
                float ri = rsqrtf(r2);
                ri = ri * fmaf(-0.5f * r2 * ri, ri, 1.5f);
                phi = INV_4PI_F * ri;
                dphi_r = -INV_4PI_F * ri * ri * ri;
            }
            const float qq = pi.w * pj.w;
            const float f = qq * dphi_r;
            fx = fmaf(f, dx, fx);
            fy = fmaf(f, dy, fy);
            fz = fmaf(f, dz, fz);
            en = fmaf(-0.5f * qq, phi, en);
            v[0] = fmaf(f * dx, dx, v[0]);
            v[1] = fmaf(f * dx, dy, v[1]);
            v[2] = fmaf(f * dx, dz, v[2]);
            v[3] = fmaf(f * dy, dy, v[3]);
            v[4] = fmaf(f * dy, dz, v[4]);
            v[5] = fmaf(f * dz, dz, v[5]);
        }
        float4 fo = force[i];
        fo.x += fx;
        fo.y += fy;
        fo.z += fz;
        fo.w += en;
        force[i] = fo;
        if (vpp)
#pragma unroll
            for (int k = 0; k < 6; ++k) vpp[(size_t)k * vpitch + i] += 0.5f * v[k];
    }
    double e[7] = {(double)en, 0.5 * v[0], 0.5 * v[1], 0.5 * v[2], 0.5 * v[3], 0.5 * v[4], 0.5 * v[5]};
    block_sum_f64<7>(e, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_E], e[0]);
#pragma unroll
        for (int k = 0; k < 6; ++k) atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_WX + k], e[1 + k]);
    }
}

// force += add (the concurrently computed pair forces and energies).
__global__ void k_add_forces(const int2* __restrict__ chunks, const SysDev* __restrict__ sys,
                             const float4* __restrict__ add, float4* __restrict__ force) {
    const int2 ch = chunks[blockIdx.x];
    const int i = ch.y + threadIdx.x;
    if (i >= sys[ch.x].p_off + sys[ch.x].N) return;
    const float4 b = add[i];
    float4 f = force[i];
    f.x += b.x;
    f.y += b.y;
    f.z += b.z;
    f.w += b.w;
    force[i] = f;
}

cudaError_t launch_add_forces(const int2* chunks, int n_chunks, const SysDev* sys, const float4* add, float4* force,
                              cudaStream_t st) {
    if (n_chunks) k_add_forces<<<n_chunks, 256, 0, st>>>(chunks, sys, add, force);
    return cudaGetLastError();
}

cudaError_t launch_exclusions(const LaunchArgs& a, cudaStream_t st) {
    if (a.n_chunks == 0 || !a.ex_n) return cudaSuccess;
    k_exclusions<<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.psets, a.posq, a.ex_n, a.ex_list, a.ex_pitch,
                                             a.force, a.acc, a.virial_pp, a.vpp_pitch);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const LaunchArgs& a, cudaStream_t st) {
    k_finalize<<<(a.nsys + 127) / 128, 128, 0, st>>>(a.sys, a.psets, a.nsys, a.acc, a.energy, a.virial, a.add_bg,
                                                     a.external);
    return cudaGetLastError();
}

cudaError_t launch_influence(const SysDev& S, const double* w1d, const double* tq, const double* wq, int nq,
                             double rcut, double psi_floor, float2* gtab, cudaStream_t st) {
    const long long total = (long long)S.nz * S.ny * S.nxh;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    k_influence<float2><<<blocks, 256, 0, st>>>(S, w1d, tq, wq, nq, rcut, psi_floor, gtab);
    return cudaGetLastError();
}

cudaError_t launch_influence64(const SysDev& S, const double* w1d, const double* tq, const double* wq, int nq,
                               double rcut, double psi_floor, double2* gtab, cudaStream_t st) {
    const long long total = (long long)S.nz * S.ny * S.nxh;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    k_influence<double2><<<blocks, 256, 0, st>>>(S, w1d, tq, wq, nq, rcut, psi_floor, gtab);
    return cudaGetLastError();
}

cudaError_t launch_pswf_eval_pairs(int n, const double* rsq, const double* qiqj, double rcut, int n_segs,
                                   const double* screen, const double* dscreen, const double* r_lo,
                                   const double* dr_inv, double* force_divr, double* pair_eng, int* evaluated,
                                   cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_pswf_eval_pairs<<<(n + 255) / 256, 256, 0, st>>>(n, rsq, qiqj, rcut, rcut * rcut, n_segs, screen, dscreen,
                                                        r_lo, dr_inv, force_divr, pair_eng, evaluated);
    return cudaGetLastError();
}

}  // namespace espb
