// FP64 mode of the ESP path: every stage in double precision, for HOOMD
// double builds (Scalar4 = double4 positions and forces) and for accuracy
// targets below the FP32 floor (~1e-7). Same algorithm, tiles and sorted
// order as the FP32 kernels:
//   k64_bin / k64_tile_sort : tile keys (shared sort kernels) with FP64
//                             stencil records;
//   k64_spread              : one CTA per tile, each thread summing one row
//                             of the tile's extended region in registers over
//                             the staged particles (no atomics inside the
//                             tile), one FP64 atomic per region point into the
//                             mesh;
//   k64_fft_pass            : one warp per mesh line, mixed-radix Stockham in
//                             shared memory on the half spectrum (two real x
//                             rows per complex line); the z pass multiplies by
//                             the influence table and accumulates the k-space
//                             energy and virial;
//   k64_interp              : one CTA per tile, the tile's potential region
//                             staged in shared memory, eight lanes per
//                             particle over the stencil rows;
//   k64_pair, k64_exclusions : as the FP32 kernels, in FP64.
// Reference stages: src/ESPForceComputeGPU.cu:157-471 (K1-K7).
#include <algorithm>

#include "esp_common.cuh"
#include "esp_kernels.h"

namespace espb {

// ----------------------------------------------------------------------------
// binning: FP64 stencil record (t_x, t_y, t_z, q) and wrapped position
// ----------------------------------------------------------------------------
__device__ __forceinline__ double wrap64(double x, double L) {
    x -= L * floor(x / L);
    if (x >= L) x -= L;
    if (x < 0.0) x += L;
    return x;
}

__global__ void k64_bin(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, int P, int T,
                        const double4* __restrict__ pos_in, const double* __restrict__ q_in,
                        double4* __restrict__ posq, double4* __restrict__ trec, uint32_t* __restrict__ rel,
                        uint32_t* __restrict__ key, uint32_t* __restrict__ tile_count, double* __restrict__ acc) {
    __shared__ double red[32 * 2];
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    double qs[2] = {0.0, 0.0};
    uint32_t kk = 0xffffffffu;  // this particle's tile (none: an idle lane)
    if (i < S.p_off + S.N) {
        const double4 p = pos_in[i];
        const double q = q_in[i];
        const double L[3] = {S.Lxd, S.Lyd, S.Lzd};
        const double gd[3] = {S.gxd, S.gyd, S.gzd};
        const int n[3] = {S.nx, S.ny, S.nz};
        const double x[3] = {wrap64(p.x, L[0]), wrap64(p.y, L[1]), wrap64(p.z, L[2])};
        const double hp = 0.5 * P;
        int i0m[3];
        double tt[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double g = x[d] * gd[d];
            if (g >= n[d]) g -= n[d];
            const int i0 = (int)floor(g - hp) + 1;
            tt[d] = (double)i0 + hp - g;
            i0m[d] = i0 < 0 ? i0 + n[d] : (i0 >= n[d] ? i0 - n[d] : i0);
        }
        const int tx = i0m[0] / T, ty = i0m[1] / T, tz = i0m[2] / T;
        const uint32_t k = (uint32_t)(S.t_off + (tz * S.nty + ty) * S.ntx + tx);
        key[i] = k;
        kk = k;
        posq[i] = make_double4(x[0], x[1], x[2], q);
        trec[i] = make_double4(tt[0], tt[1], tt[2], q);
        rel[i] = (uint32_t)(i0m[0] - tx * T) | ((uint32_t)(i0m[1] - ty * T) << 8) |
                 ((uint32_t)(i0m[2] - tz * T) << 16);
        qs[0] = q;
        qs[1] = q * q;
    }
    {
        // one atomic per distinct tile of the warp (neighbouring particles
        // mostly share a tile)
        const unsigned grp = __match_any_sync(0xffffffffu, kk);
        if (kk != 0xffffffffu && (threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&tile_count[kk], (uint32_t)__popc(grp));
    }
    block_sum_f64<2>(qs, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_QSUM], qs[0]);
        atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_Q2SUM], qs[1]);
    }
}

// Stable order inside each tile (ascending particle index), gathering the
// FP64 records.
__global__ void k64_tile_sort(const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm_u,
                              uint32_t* __restrict__ perm, const double4* __restrict__ trec,
                              const uint32_t* __restrict__ rel, double4* __restrict__ srec,
                              uint32_t* __restrict__ srel) {
    __shared__ uint32_t sm[SORT_CAP];
    const uint32_t s0 = start[blockIdx.x];
    const uint32_t n = start[blockIdx.x + 1] - s0;
    if (n == 0) return;
    const bool cached = n <= (uint32_t)SORT_CAP;
    if (cached)
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sm[i] = perm_u[s0 + i];
    __syncthreads();
    const uint32_t* src = cached ? sm : perm_u + s0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t v = src[i];
        uint32_t r = 0;
        for (uint32_t j = 0; j < n; ++j) r += (src[j] < v) ? 1u : 0u;
        perm[s0 + r] = v;
        srec[s0 + r] = trec[v];
        srel[s0 + r] = rel[v];
    }
}

__device__ __forceinline__ double horner64(const double* c, int D, double t) {
    double v = c[D];
    for (int j = D - 1; j >= 0; --j) v = fma(v, t, c[j]);
    return v;
}
__device__ __forceinline__ double dhorner64(const double* c, int D, double t) {
    double v = D * c[D];
    for (int j = D - 1; j >= 1; --j) v = fma(v, t, j * c[j]);
    return v;
}

// Mesh offsets of a tile's extended region [E]^3 with the periodic wrap:
// roff[r] = (gz ny + gy) nx for region row r = (z, y) = (r / E, r % E), xo[x] = gx.
__device__ __forceinline__ void region_tables(const SysDev& S, int X0, int Y0, int Z0, int E, int* roff, int* xo) {
    for (int r = threadIdx.x; r < E * E; r += blockDim.x) {
        int gy = Y0 + r % E, gz = Z0 + r / E;
        while (gy >= S.ny) gy -= S.ny;
        while (gz >= S.nz) gz -= S.nz;
        roff[r] = (gz * S.ny + gy) * S.nx;
    }
    for (int x = threadIdx.x; x < E; x += blockDim.x) {
        int gx = X0 + x;
        while (gx >= S.nx) gx -= S.nx;
        xo[x] = gx;
    }
}

// ----------------------------------------------------------------------------
// spreading: one CTA per tile (several when the tiles are few, each over a
// share of the tile's particle chunks); every thread owns one row (z, y) of
// the tile's extended region [E]^3 (E = T + P - 1) and sums it in registers,
// 16 points along x at a time. The tile's particles are staged K64S_CH at a time: per
// particle its x weights times q as a 16-point row segment pre-shifted to its
// stencil origin (zero elsewhere), its y and z weights and its origin. A
// thread adds, in particle order, every staged particle whose stencil covers
// its row: a broadcast read of the segment and 16 FMAs, no atomics, and a
// CTA's sums are deterministic. Row r = (r / E, r % E), so with E = 16 and 256
// threads a warp owns two z planes and the coverage test is nearly
// warp-uniform. The finished rows pass through shared memory (rows padded to
// an odd stride) so that the flush, one FP64 atomic per nonzero region point,
// is coalesced along x.
// ----------------------------------------------------------------------------
constexpr int K64S_THREADS = 256;
constexpr int K64S_CH = 48;   // particles staged per pass
constexpr int K64S_SEG = 16;  // register row segment along x

__host__ __device__ inline int spread64_stride(int E) { return E | 1; }
// region doubles, rounded up to an even count so that the x segments after it are 16-byte aligned
__host__ __device__ inline size_t spread64_region(int E) { return ((size_t)E * E * spread64_stride(E) + 1) & ~(size_t)1; }

__global__ void __launch_bounds__(K64S_THREADS)
    k64_spread(const int* __restrict__ tile_sys, const SysDev* __restrict__ sys, const double* __restrict__ wcoef,
               int P, int T, int D, const uint32_t* __restrict__ start, const double4* __restrict__ srec,
               const uint32_t* __restrict__ srel, double* __restrict__ rho) {
    // [E^2][ES] region | [K64S_CH][K64S_SEG] x segments | [K64S_CH][2P] y, z weights | [P][D+1] window
    // | [K64S_CH] origins | row and column offsets
    extern __shared__ double sreg[];
    const int t = blockIdx.x;
    const uint32_t s0 = start[t];
    const int np = (int)(start[t + 1] - s0);
    if (np == 0) return;
    const SysDev S = sys[tile_sys[t]];
    const int E = T + P - 1, ES = spread64_stride(E), E2 = E * E, D1 = D + 1;
    double* xs = sreg + spread64_region(E);
    double* yz = xs + K64S_CH * K64S_SEG;
    double* wc = yz + K64S_CH * 2 * P;
    uint32_t* org = reinterpret_cast<uint32_t*>(wc + P * D1);
    for (int k = threadIdx.x; k < P * D1; k += blockDim.x) wc[k] = wcoef[k];
    const int nseg = (E + K64S_SEG - 1) / K64S_SEG;
    for (int rb = 0; rb < E2; rb += blockDim.x) {
        const int r = rb + threadIdx.x;
        const bool own = r < E2;
        const int z = r / E, y = r - z * E;
        for (int seg = 0; seg < nseg; ++seg) {
            const int x0 = seg * K64S_SEG;
            double acc[K64S_SEG];
#pragma unroll
            for (int j = 0; j < K64S_SEG; ++j) acc[j] = 0.0;
            // CTA blockIdx.y of gridDim.y takes every gridDim.y-th chunk
            for (int p0 = blockIdx.y * K64S_CH; p0 < np; p0 += gridDim.y * K64S_CH) {
                const int m = min(K64S_CH, np - p0);
                __syncthreads();  // window staged / previous chunk consumed
                for (int k = threadIdx.x; k < m * K64S_SEG; k += blockDim.x) {
                    const int pp = k / K64S_SEG, a = x0 + (k - pp * K64S_SEG) - (int)(srel[s0 + p0 + pp] & 255u);
                    double v = 0.0;
                    if ((unsigned)a < (unsigned)P) {
                        const double4 rec = srec[s0 + p0 + pp];
                        v = horner64(wc + a * D1, D, rec.x) * rec.w;
                    }
                    xs[k] = v;
                }
                for (int k = threadIdx.x; k < m * 2 * P; k += blockDim.x) {
                    const int pp = k / (2 * P), l = k - pp * 2 * P, a = l < P ? l : l - P;
                    const double4 rec = srec[s0 + p0 + pp];
                    yz[k] = horner64(wc + a * D1, D, l < P ? rec.y : rec.z);
                }
                for (int k = threadIdx.x; k < m; k += blockDim.x) org[k] = srel[s0 + p0 + k];
                __syncthreads();
                if (own)
                    for (int pp = 0; pp < m; ++pp) {
                        const uint32_t rl = org[pp];
                        const int b = y - (int)((rl >> 8) & 255u), c = z - (int)((rl >> 16) & 255u);
                        if ((unsigned)b < (unsigned)P && (unsigned)c < (unsigned)P) {
                            const double cw = yz[pp * 2 * P + b] * yz[pp * 2 * P + P + c];
                            const double2* xr = reinterpret_cast<const double2*>(xs + pp * K64S_SEG);
#pragma unroll
                            for (int j = 0; j < K64S_SEG / 2; ++j) {
                                const double2 v = xr[j];
                                acc[2 * j] = fma(v.x, cw, acc[2 * j]);
                                acc[2 * j + 1] = fma(v.y, cw, acc[2 * j + 1]);
                            }
                        }
                    }
            }
            if (own) {
                double* row = sreg + (size_t)r * ES + x0;
#pragma unroll
                for (int j = 0; j < K64S_SEG; ++j)
                    if (x0 + j < E) row[j] = acc[j];
            }
        }
    }
    const int lt = t - S.t_off;
    const int X0 = (lt % S.ntx) * T, Y0 = ((lt / S.ntx) % S.nty) * T, Z0 = (lt / (S.ntx * S.nty)) * T;
    int* roff = reinterpret_cast<int*>(org + K64S_CH);
    int* xo = roff + E2;
    region_tables(S, X0, Y0, Z0, E, roff, xo);
    __syncthreads();
    double* mesh = rho + S.m_off;
    // element (r, x) stepped by the block size: consecutive threads along x
    const int dr = blockDim.x / E, dx = blockDim.x - dr * E;
    for (int x = threadIdx.x % E, r = threadIdx.x / E; r < E2;) {
        const double v = sreg[(size_t)r * ES + x];
        if (v != 0.0) atomicAdd(&mesh[roff[r] + xo[x]], v);
        x += dx;
        r += dr;
        if (x >= E) {
            x -= E;
            ++r;
        }
    }
}

// ----------------------------------------------------------------------------
// FFT: one warp per line, Stockham autosort in shared memory, radices
// 2/3/4/5 from the packed plan (one register-resident butterfly per radix);
// tw = exp(-2 pi i t / n) (the forward sign), staged in shared memory per CTA
// and conjugated for the inverse. A CTA transforms F64_WARPS neighbouring
// lines of one system; the strided (y, z) passes load and store them
// cooperatively, the F64_WARPS lines' elements adjacent in memory.
// ----------------------------------------------------------------------------
__device__ __forceinline__ double2 z_mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 z_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 z_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// s * i * a for s = +-1
__device__ __forceinline__ double2 z_rot(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }

// R-point DFT in registers, y_k = sum_r v_r exp(sign 2 pi i r k / R)
template <int R>
__device__ __forceinline__ void dft64(double2 (&v)[R], double s);
template <>
__device__ __forceinline__ void dft64<2>(double2 (&v)[2], double) {
    const double2 a = v[0], b = v[1];
    v[0] = z_add(a, b);
    v[1] = z_sub(a, b);
}
template <>
__device__ __forceinline__ void dft64<4>(double2 (&v)[4], double s) {
    const double2 ac = z_add(v[0], v[2]), am = z_sub(v[0], v[2]);
    const double2 bd = z_add(v[1], v[3]), jb = z_rot(z_sub(v[1], v[3]), s);
    v[0] = z_add(ac, bd);
    v[1] = z_add(am, jb);
    v[2] = z_sub(ac, bd);
    v[3] = z_sub(am, jb);
}
template <>
__device__ __forceinline__ void dft64<3>(double2 (&v)[3], double s) {
    constexpr double S3 = 0.86602540378443864676;  // sin(2 pi / 3)
    const double2 t1 = z_add(v[1], v[2]);
    const double2 m = make_double2(fma(-0.5, t1.x, v[0].x), fma(-0.5, t1.y, v[0].y));
    const double2 r = z_rot(z_sub(v[1], v[2]), s * S3);
    v[0] = z_add(v[0], t1);
    v[1] = z_add(m, r);
    v[2] = z_sub(m, r);
}
template <>
__device__ __forceinline__ void dft64<5>(double2 (&v)[5], double s) {
    constexpr double C1 = 0.30901699437494742410, S1 = 0.95105651629515357212;   // 2 pi / 5
    constexpr double C2 = -0.80901699437494742410, S2 = 0.58778525229247312917;  // 4 pi / 5
    const double2 a1 = z_add(v[1], v[4]), b1 = z_sub(v[1], v[4]);
    const double2 a2 = z_add(v[2], v[3]), b2 = z_sub(v[2], v[3]);
    const double2 p1 = make_double2(v[0].x + C1 * a1.x + C2 * a2.x, v[0].y + C1 * a1.y + C2 * a2.y);
    const double2 p2 = make_double2(v[0].x + C2 * a1.x + C1 * a2.x, v[0].y + C2 * a1.y + C1 * a2.y);
    const double2 q1 = z_rot(make_double2(S1 * b1.x + S2 * b2.x, S1 * b1.y + S2 * b2.y), s);
    const double2 q2 = z_rot(make_double2(S2 * b1.x - S1 * b2.x, S2 * b1.y - S1 * b2.y), s);
    v[0] = z_add(v[0], z_add(a1, a2));
    v[1] = z_add(p1, q1);
    v[4] = z_sub(p1, q1);
    v[2] = z_add(p2, q2);
    v[3] = z_sub(p2, q2);
}

// One Stockham stage of radix R: the R inputs of butterfly j are j + r n/R;
// twiddle index r k (n / (Ns R)) < n with k = j mod Ns.
template <int R>
__device__ __forceinline__ void stage64(const double2* src, double2* dst, int n, int Ns, const double2* tw,
                                        int sign, int lane) {
    const int nb = n / R, step = n / (Ns * R);
    const double s = (double)sign;
    for (int j = lane; j < nb; j += 32) {
        const int k = j % Ns;
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[j + r * nb];
        if (k > 0) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                double2 w = tw[r * k * step];
                w.y *= -s;  // tw holds the forward (sign -1) roots
                v[r] = z_mul(v[r], w);
            }
        }
        dft64<R>(v, s);
        const int o = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[o + r * Ns] = v[r];
    }
}

// Transforms the n points in a (scratch b); returns the buffer holding the result.
__device__ double2* fft64_line(double2* a, double2* b, int n, uint32_t plan, const double2* tw, int sign, int lane) {
    int Ns = 1;
    double2 *src = a, *dst = b;
    for (uint32_t pl = plan; pl; pl >>= 4) {
        const int R = pl & 15;
        if (R == 4) stage64<4>(src, dst, n, Ns, tw, sign, lane);
        else if (R == 2) stage64<2>(src, dst, n, Ns, tw, sign, lane);
        else if (R == 3) stage64<3>(src, dst, n, Ns, tw, sign, lane);
        else stage64<5>(src, dst, n, Ns, tw, sign, lane);
        __syncwarp();
        double2* x = src;
        src = dst;
        dst = x;
        Ns *= R;
    }
    return src;
}

constexpr int F64_WARPS = 4;

// Half spectrum, as the FP32 passes: the x passes transform two real rows
// (y, y + 1) as one complex line and store (or rebuild) their nx/2 + 1
// Hermitian halves, so the spectrum is [z][y][kx < nxh] and the y and z
// passes touch nxh of the nx columns.
// MODE 0: x forward (real mesh -> half spectrum, the mesh is cleared), 1: y
// forward, 2: z forward + influence multiply + energy/virial + z inverse,
// 3: y inverse, 4: x inverse (half spectrum -> real potential).
// Lines per system: x: ceil(ny/2) nz row pairs; y: nxh nz; z: nxh ny.
template <int MODE>
__global__ void __launch_bounds__(F64_WARPS * 32)
    k64_fft_pass(const int2* __restrict__ items, const SysDev* __restrict__ sys, const double2* __restrict__ tw,
                 double2* __restrict__ cbuf, double* __restrict__ rho, double* __restrict__ phi,
                 const double2* __restrict__ gtab, double* __restrict__ acc) {
    __shared__ double2 sb[F64_WARPS][2][FFT_MAX_N];
    __shared__ double2 stw[FFT_MAX_N];
    __shared__ long long lbase[F64_WARPS];
    __shared__ double red[32 * 7];
    const int2 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int AX = (MODE == 0 || MODE == 4) ? 0 : (MODE == 1 || MODE == 3) ? 1 : 2;
    const int nxh = S.nxh, nyp = (S.ny + 1) / 2;
    const int n = AX == 0 ? S.nx : (AX == 1 ? S.ny : S.nz);
    const long long nlines =
        AX == 0 ? (long long)nyp * S.nz : (AX == 1 ? (long long)nxh * S.nz : (long long)nxh * S.ny);
    const long long stride = AX == 1 ? (long long)nxh : (long long)nxh * S.ny;  // y and z lines
    const uint32_t plan = AX == 0 ? S.radx : (AX == 1 ? S.rady : S.radz);
    const double2* twa = tw + (AX == 0 ? S.twx : (AX == 1 ? S.twy : S.twz));
    for (int k = threadIdx.x; k < n; k += blockDim.x) stw[k] = twa[k];
    if (threadIdx.x < F64_WARPS) {
        const long long l = (long long)it.y + threadIdx.x;
        long long base = -1;
        if (l < nlines) {
            if (AX == 0) base = (l / nyp) * S.ny + 2 * (l % nyp);  // first row (z ny + y) of the pair
            else if (AX == 1) base = (l / nxh) * nxh * S.ny + l % nxh;
            else base = l;  // (y, kx) = (l / nxh, l % nxh): base y nxh + kx = l
        }
        lbase[threadIdx.x] = base;
    }
    __syncthreads();
    const long long l = (long long)it.y + warp;
    const bool active = l < nlines;
    // x row pairs: the pair's second row exists unless ny is odd and y = ny - 1
    const long long row0 = active && AX == 0 ? lbase[warp] : 0;
    const bool two = AX == 0 && active && (row0 % S.ny) + 1 < S.ny;
    double2* a = sb[warp][0];
    double2* b = sb[warp][1];
    // load: x row pairs one per warp (contiguous rows); y and z lines
    // cooperatively, the F64_WARPS lines' elements at one k adjacent in memory
    if (AX == 0) {
        if (active) {
            if (MODE == 0) {
                double* r0 = rho + S.m_off + row0 * S.nx;
                for (int k = lane; k < n; k += 32) a[k] = make_double2(r0[k], two ? r0[k + S.nx] : 0.0);
                // cleared in a loop of its own: the loads above are not ordered behind stores
                for (int k = lane; k < n; k += 32) {
                    r0[k] = 0.0;
                    if (two) r0[k + S.nx] = 0.0;
                }
            } else {
                // Z_k = A_k + i B_k, with A_{n-k} = conj(A_k) (and B) for k >= nxh
                const double2* c0 = cbuf + S.m_off + row0 * nxh;
                for (int k = lane; k < n; k += 32) {
                    const bool lo = k < nxh;
                    const int kk = lo ? k : n - k;
                    double2 A = c0[kk], B = two ? c0[kk + nxh] : make_double2(0.0, 0.0);
                    if (!lo) {
                        A.y = -A.y;
                        B.y = -B.y;
                    }
                    a[k] = make_double2(A.x - B.y, A.y + B.x);
                }
            }
        }
    } else {
        for (int idx = threadIdx.x; idx < F64_WARPS * n; idx += blockDim.x) {
            const int w = idx % F64_WARPS, k = idx / F64_WARPS;
            if (lbase[w] >= 0) sb[w][0][k] = cbuf[S.m_off + lbase[w] + k * stride];
        }
    }
    __syncthreads();
    double e[7] = {0, 0, 0, 0, 0, 0, 0};
    double2* res = a;
    if (active) {
        const int sign = MODE <= 2 ? -1 : 1;
        res = fft64_line(a, b, n, plan, stw, sign, lane);
        if (MODE == 2) {
            // (kx, ky) = (lx, ly) after the x and y passes; kz along the line;
            // the columns 0 < kx < nx/2 stand for their conjugates too
            const int ly = (int)(l / nxh), lx = (int)(l % nxh);
            const double tpx = 6.283185307179586 / S.Lxd, tpy = 6.283185307179586 / S.Lyd,
                         tpz = 6.283185307179586 / S.Lzd;
            const int fx = lx;
            const int fy = ly <= S.ny / 2 ? ly : ly - S.ny;
            const double wk = (lx == 0 || 2 * lx == S.nx) ? 1.0 : 2.0;
            for (int kz = lane; kz < n; kz += 32) {
                const int fz = kz <= S.nz / 2 ? kz : kz - S.nz;
                const double2 g = gtab[S.g_off + ((long long)kz * S.ny + ly) * nxh + lx];
                const double2 v = res[kz];
                const double a2 = wk * (v.x * v.x + v.y * v.y);
                const double ek = 0.5 * g.x * a2, eb = 0.5 * g.y * a2;
                const double kxv = tpx * fx, kyv = tpy * fy, kzv = tpz * fz;
                e[0] += ek;
                e[1] += ek + eb * kxv * kxv;
                e[2] += eb * kxv * kyv;
                e[3] += eb * kxv * kzv;
                e[4] += ek + eb * kyv * kyv;
                e[5] += eb * kyv * kzv;
                e[6] += ek + eb * kzv * kzv;
                res[kz] = make_double2(v.x * g.x, v.y * g.x);
            }
            __syncwarp();
            res = fft64_line(res, res == a ? b : a, n, plan, stw, +1, lane);
        }
    }
    if (AX == 0) {
        if (active) {
            if (MODE == 4) {
                // the potential rows: real part row y, imaginary part row y + 1
                double* p0 = phi + S.m_off + row0 * S.nx;
                for (int k = lane; k < n; k += 32) {
                    const double2 z = res[k];
                    p0[k] = z.x;
                    if (two) p0[k + S.nx] = z.y;
                }
            } else {
                // A_k = (Z_k + conj Z_{n-k}) / 2, B_k = (Z_k - conj Z_{n-k}) / (2i), k < nxh
                double2* c0 = cbuf + S.m_off + row0 * nxh;
                for (int k = lane; k < nxh; k += 32) {
                    const double2 z = res[k], zc = res[k == 0 ? 0 : n - k];
                    c0[k] = make_double2(0.5 * (z.x + zc.x), 0.5 * (z.y - zc.y));
                    if (two) c0[k + nxh] = make_double2(0.5 * (z.y + zc.y), -0.5 * (z.x - zc.x));
                }
            }
        }
    } else {
        // every line of the CTA has the same length and plan: its result sits
        // in buffer (stages mod 2) of its warp (buffer 0 after the two
        // transforms of the z pass)
        int stages = 0;
        for (uint32_t pl = plan; pl; pl >>= 4) ++stages;
        const int rb = MODE == 2 ? 0 : (stages & 1);
        __syncthreads();
        for (int idx = threadIdx.x; idx < F64_WARPS * n; idx += blockDim.x) {
            const int w = idx % F64_WARPS, k = idx / F64_WARPS;
            if (lbase[w] >= 0) cbuf[S.m_off + lbase[w] + k * stride] = sb[w][rb][k];
        }
    }
    if (MODE == 2) {
        block_sum_f64<7>(e, red);
        if (threadIdx.x == 0)
            for (int k = 0; k < 7; ++k) atomicAdd(&acc[it.x * ACC_STRIDE + ACC_EK + k], e[k]);
    }
}

// ----------------------------------------------------------------------------
// interpolation: one CTA (or a few) per tile. The tile's extended potential region
// [E]^3 (E = T + P - 1, periodic wrap) is staged in shared memory with
// coalesced loads along x (rows padded to an odd stride of doubles), then the
// tile's particles, in sorted order, are interpolated from it (by several
// CTAs per tile when the tiles are few): K64I_G lanes
// per particle (four particles per warp) share the P^2 stencil rows (y, z),
// each row a run of P values along x read with the x weights held in
// registers; potential, gradient and energy reduced over the particle's
// lanes. The stencil records (t, q) and origins come from the sort.
// ----------------------------------------------------------------------------
constexpr int K64I_WARPS = 4;
constexpr int K64I_G = 8;              // lanes per particle
constexpr int K64I_PPW = 32 / K64I_G;  // particles per warp pass

size_t interp64_smem(int P, int T) {
    const int E = T + P - 1;
    return ((size_t)E * E * spread64_stride(E) + (size_t)P * (MAX_D + 1)) * sizeof(double) +
           (size_t)(E * E + E) * sizeof(int);
}

template <int P>
__global__ void __launch_bounds__(K64I_WARPS * 32)
    k64_interp(const int* __restrict__ tile_sys, const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets,
               const double* __restrict__ wcoef, int T, int D, const uint32_t* __restrict__ start,
               const uint32_t* __restrict__ perm, const double4* __restrict__ srec,
               const uint32_t* __restrict__ srel, const double* __restrict__ phi, double4* __restrict__ force,
               double* __restrict__ acc) {
    extern __shared__ double sreg[];  // [E^2][ES] potential region, [P][D+1] window, row and column offsets
    __shared__ double red[32];
    __shared__ double wsh[K64I_WARPS * K64I_PPW][6 * P];  // W x | y | z, then dW x | y | z
    const int t = blockIdx.x;
    const uint32_t s0 = start[t];
    const int np = (int)(start[t + 1] - s0);
    if (np == 0) return;
    const int sid = tile_sys[t];
    const SysDev S = sys[sid];
    const int E = T + P - 1, ES = spread64_stride(E), E2 = E * E, D1 = D + 1;
    double* wc = sreg + (size_t)E2 * ES;
    for (int k = threadIdx.x; k < P * D1; k += blockDim.x) wc[k] = wcoef[k];
    const int lt = t - S.t_off;
    const int X0 = (lt % S.ntx) * T, Y0 = ((lt / S.ntx) % S.nty) * T, Z0 = (lt / (S.ntx * S.nty)) * T;
    const double* ph = phi + S.m_off;
    int* roff = reinterpret_cast<int*>(wc + P * (MAX_D + 1));
    int* xo = roff + E2;
    region_tables(S, X0, Y0, Z0, E, roff, xo);
    __syncthreads();
    // element (r, x) stepped by the block size: consecutive threads along x
    const int dr = blockDim.x / E, dx = blockDim.x - dr * E;
    for (int x = threadIdx.x % E, r = threadIdx.x / E; r < E2;) {
        sreg[(size_t)r * ES + x] = ph[roff[r] + xo[x]];
        x += dx;
        r += dr;
        if (x >= E) {
            x -= E;
            ++r;
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sub = lane % K64I_G, slot = lane / K64I_G;
    const double self = psets[S.pset].self_coef;
    double* W = wsh[warp * K64I_PPW + slot];
    double e_acc = 0.0;
    // CTA blockIdx.y of gridDim.y takes every gridDim.y-th group of K64I_WARPS * K64I_PPW particles
    for (int pb = (blockIdx.y * K64I_WARPS + warp) * K64I_PPW; pb < np; pb += gridDim.y * K64I_WARPS * K64I_PPW) {
        const int pp = pb + slot;
        const bool valid = pp < np;
        const double4 rec = valid ? srec[s0 + pp] : make_double4(0.0, 0.0, 0.0, 0.0);
        const uint32_t rl = valid ? srel[s0 + pp] : 0u;
        if (valid)
            for (int l = sub; l < 3 * P; l += K64I_G) {
                const int d = l / P, a = l - d * P;
                const double tt = d == 0 ? rec.x : (d == 1 ? rec.y : rec.z);
                W[l] = horner64(wc + a * D1, D, tt);
                W[3 * P + l] = dhorner64(wc + a * D1, D, tt);
            }
        __syncwarp();
        double pot = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        if (valid) {
            double wx[P], dwx[P];
#pragma unroll
            for (int a = 0; a < P; ++a) {
                wx[a] = W[a];
                dwx[a] = W[3 * P + a];
            }
            const double* base =
                sreg + ((size_t)((rl >> 16) & 255u) * E + ((rl >> 8) & 255u)) * ES + (rl & 255u);
            for (int r = sub; r < P * P; r += K64I_G) {
                const int c = r / P, b = r - c * P;
                const double* row = base + (size_t)(c * E + b) * ES;
                double sv = 0.0, sd = 0.0;
#pragma unroll
                for (int a = 0; a < P; ++a) {
                    const double v = row[a];
                    sv = fma(wx[a], v, sv);
                    sd = fma(dwx[a], v, sd);
                }
                const double wy = W[P + b], dwy = W[4 * P + b], wz = W[2 * P + c], dwz = W[5 * P + c];
                pot = fma(wz * wy, sv, pot);
                gx = fma(wz * wy, sd, gx);
                gy = fma(wz * dwy, sv, gy);
                gz = fma(dwz * wy, sv, gz);
            }
        }
#pragma unroll
        for (int o = K64I_G / 2; o > 0; o >>= 1) {
            pot += __shfl_xor_sync(0xffffffffu, pot, o);
            gx += __shfl_xor_sync(0xffffffffu, gx, o);
            gy += __shfl_xor_sync(0xffffffffu, gy, o);
            gz += __shfl_xor_sync(0xffffffffu, gz, o);
        }
        if (valid && sub == 0) {
            const double q = rec.w;
            const double e_i = 0.5 * q * pot + self * q * q;
            force[perm[s0 + pp]] = make_double4(q * S.gxd * gx, q * S.gyd * gy, q * S.gzd * gz, e_i);
            e_acc += e_i;
        }
        __syncwarp();  // the weights are rewritten for the next particles
    }
    double e1[1] = {e_acc};
    block_sum_f64<1>(e1, red);
    if (threadIdx.x == 0) atomicAdd(&acc[sid * ACC_STRIDE + ACC_E], e1[0]);
}

// CTAs per tile for the tile kernels when the tiles are fewer than two per SM
// (coarse meshes, large tiles): about four CTAs per SM, at most 8 per tile.
// Measured on 98,304 water charges (FP64 evaluation): 125 tiles in 5 CTAs
// each 0.65 ms against 0.99 unsplit and 0.71 in 3; 512 tiles in 2 CTAs each
// 4% slower than unsplit.
static int split64(int n_tiles) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    if (n_tiles >= 2 * sms) return 1;
    return std::min(8, std::max(1, (4 * sms + n_tiles - 1) / std::max(1, n_tiles)));
}

template <int P>
static cudaError_t configure64_interp_p(int T) {
    return cudaFuncSetAttribute(k64_interp<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)interp64_smem(P, T));
}

template <int P>
static cudaError_t launch64_interp_p(const Launch64& b, cudaStream_t st) {
    const LaunchArgs& a = b.a;
    // several CTAs per tile when the tiles are few, each staging the region
    // and taking a share of its particles
    k64_interp<P><<<dim3(a.n_tiles, split64(a.n_tiles)), K64I_WARPS * 32, interp64_smem(a.P, a.T), st>>>(
        a.tile_sys, a.sys, a.psets, b.wcoef, a.T, a.D, a.tile_start, a.perm, b.srec, a.srel, b.phi, b.force, a.acc);
    return cudaGetLastError();
}

// ----------------------------------------------------------------------------
// pair term (EvaluatorPairPSWF, src/EvaluatorPairPSWF.h:274-295) in FP64:
// 8 lanes per particle over its neighbour row
// ----------------------------------------------------------------------------
// without the virial: 64 registers, four CTAs per SM (measured 1-2% faster than 72 and three)
template <bool VIR>
__global__ void __launch_bounds__(256, VIR ? 3 : 4)
    k64_pair(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets,
             const double* __restrict__ qv, int nq, const double4* __restrict__ posq,
             const uint32_t* __restrict__ head, const uint32_t* __restrict__ nn, const uint32_t* __restrict__ nlist,
             double4* __restrict__ force, double* __restrict__ acc, int accumulate) {
    __shared__ double red[32 * 7];
    __shared__ double sq[MAX_QC];  // split coefficients (nq <= MAX_QC, checked by the planner)
    constexpr int TPP = 8;
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const ParamSet& ps = psets[S.pset];
    const double rc = ps.rcut_d, rc2 = rc * rc, irc = 1.0 / rc, irc2 = irc * irc, tirc3 = 2.0 * irc2 * irc;
    const double iLx = 1.0 / S.Lxd, iLy = 1.0 / S.Lyd, iLz = 1.0 / S.Lzd;
    for (int c = threadIdx.x; c < nq; c += blockDim.x) sq[c] = qv[c];
    __syncthreads();
    const int i = ch.y + threadIdx.x / TPP;
    const int sub = threadIdx.x % TPP;
    const bool valid = i < S.p_off + S.N;
    double fx = 0, fy = 0, fz = 0, en = 0, v[6] = {0, 0, 0, 0, 0, 0};
    const double4 pi = valid ? posq[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    auto pair = [&](const double4 pj, bool wrap) {
        double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        // minimum image by the reciprocal box length; a pair that it could image
        // differently from a division sits at |d| = L/2 > r_c
        if (wrap) {
            dx -= S.Lxd * rint(dx * iLx);
            dy -= S.Lyd * rint(dy * iLy);
            dz -= S.Lzd * rint(dz * iLz);
        }
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < rc2 && r2 > 0.0) {
            const double ri = rsqrt(r2);
            const double vv = fma(2.0 * irc2, r2, -1.0);
            // Q(v) and dQ/dv in one Horner pass over the staged coefficients
            double Q = sq[nq - 1], dQ = 0.0;
            for (int c = nq - 2; c >= 0; --c) {
                dQ = fma(dQ, vv, Q);
                Q = fma(Q, vv, sq[c]);
            }
            dQ *= 2.0;  // dQ/du = 2 dQ/dv
            const double qq = pi.w * pj.w * INV_4PI_D;
            const double fdr = qq * (tirc3 * dQ + ri * ri * ri);
            en += qq * (ri - Q * irc);
            fx += fdr * dx;
            fy += fdr * dy;
            fz += fdr * dz;
            if (VIR) {
                v[0] += fdr * dx * dx;
                v[1] += fdr * dx * dy;
                v[2] += fdr * dx * dz;
                v[3] += fdr * dy * dy;
                v[4] += fdr * dy * dz;
                v[5] += fdr * dz * dz;
            }
        }
    };
    // particles at least r_c from every face (posq holds wrapped positions)
    // see every in-cutoff neighbour in the same image: a warp whose particles
    // all are skips the minimum-image wrap (pairs beyond r_c stay masked)
    const bool inner = !valid || (pi.x >= rc && pi.x <= S.Lxd - rc && pi.y >= rc && pi.y <= S.Lyd - rc &&
                                  pi.z >= rc && pi.z <= S.Lzd - rc);
    const bool interior = __all_sync(0xffffffffu, inner);
    if (valid) {
        // one neighbour per lane and step: streaming 16-byte index segments
        // with four gathers in flight per lane measured 2-6% slower here
        const uint32_t n = nn[i], h = head[i];
        // the next neighbour index is loaded one step ahead of its gather
        uint32_t jn = sub < n ? nlist[h + sub] : 0u;
        if (interior)
            for (uint32_t k = sub; k < n; k += TPP) {
                const uint32_t j = jn;
                if (k + TPP < n) jn = nlist[h + k + TPP];
                pair(posq[S.p_off + (int)j], false);
            }
        else
            for (uint32_t k = sub; k < n; k += TPP) {
                const uint32_t j = jn;
                if (k + TPP < n) jn = nlist[h + k + TPP];
                pair(posq[S.p_off + (int)j], true);
            }
    }
#pragma unroll
    for (int o = TPP / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
        en += __shfl_xor_sync(0xffffffffu, en, o);
    }
    if (valid && sub == 0) {
        double4 f = accumulate ? force[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        f.x += fx;
        f.y += fy;
        f.z += fz;
        f.w += 0.5 * en;
        force[i] = f;
    }
    if (VIR) {
        double e[7] = {sub == 0 ? 0.5 * en : 0.0, 0.5 * v[0], 0.5 * v[1], 0.5 * v[2],
                       0.5 * v[3],                0.5 * v[4], 0.5 * v[5]};
        block_sum_f64<7>(e, red);
        if (threadIdx.x == 0) {
            atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_E], e[0]);
            for (int k = 0; k < 6; ++k) atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_WP + k], e[1 + k]);
        }
    } else {
        double e[1] = {sub == 0 ? 0.5 * en : 0.0};
        block_sum_f64<1>(e, red);
        if (threadIdx.x == 0) atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_E], e[0]);
    }
}

// exclusion correction (src/ESPForceComputeGPU.cu:391-471) in FP64: removes
// the mesh interaction Phi = 1/(4 pi r) - L(r) of every excluded pair
__global__ void k64_exclusions(const int2* __restrict__ chunks, const SysDev* __restrict__ sys,
                               const ParamSet* __restrict__ psets, const double* __restrict__ qv, int nq,
                               const double4* __restrict__ posq, const uint32_t* __restrict__ n_ex,
                               const uint32_t* __restrict__ ex_list, int ex_pitch, double4* __restrict__ force,
                               double* __restrict__ acc) {
    __shared__ double red[32 * 7];
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const ParamSet& ps = psets[S.pset];
    const double rc = ps.rcut_d, rc2 = rc * rc, irc = 1.0 / rc;
    const int i = ch.y + threadIdx.x;
    const bool valid = i < S.p_off + S.N;
    const uint32_t n = valid ? n_ex[i] : 0u;
    double fx = 0, fy = 0, fz = 0, en = 0, v[6] = {0, 0, 0, 0, 0, 0};
    if (n > 0) {
        const double4 pi = posq[i];
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t jl = ex_list[(size_t)i * ex_pitch + k];
            if (jl >= (uint32_t)S.N) continue;
            const double4 pj = posq[S.p_off + (int)jl];
            double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            dx -= S.Lxd * rint(dx / S.Lxd);
            dy -= S.Lyd * rint(dy / S.Lyd);
            dz -= S.Lzd * rint(dz / S.Lzd);
            const double r2 = dx * dx + dy * dy + dz * dz;
            double phiv, dphi_r;
            if (r2 < rc2) {
                const double vv = fma(2.0 * irc * irc, r2, -1.0);
                double Q = qv[nq - 1], dQ = (nq - 1) * qv[nq - 1];
                for (int c = nq - 2; c >= 0; --c) Q = fma(Q, vv, qv[c]);
                for (int c = nq - 2; c >= 1; --c) dQ = fma(dQ, vv, c * qv[c]);
                phiv = INV_4PI_D * Q * irc;
                dphi_r = INV_4PI_D * 2.0 * irc * irc * irc * (2.0 * dQ);
            } else {
                const double ri = 1.0 / sqrt(r2);
                phiv = INV_4PI_D * ri;
                dphi_r = -INV_4PI_D * ri * ri * ri;
            }
            const double qq = pi.w * pj.w;
            const double f = qq * dphi_r;
            fx += f * dx;
            fy += f * dy;
            fz += f * dz;
            en -= 0.5 * qq * phiv;
            v[0] += f * dx * dx;
            v[1] += f * dx * dy;
            v[2] += f * dx * dz;
            v[3] += f * dy * dy;
            v[4] += f * dy * dz;
            v[5] += f * dz * dz;
        }
        double4 fo = force[i];
        fo.x += fx;
        fo.y += fy;
        fo.z += fz;
        fo.w += en;
        force[i] = fo;
    }
    double e[7] = {en, 0.5 * v[0], 0.5 * v[1], 0.5 * v[2], 0.5 * v[3], 0.5 * v[4], 0.5 * v[5]};
    block_sum_f64<7>(e, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_E], e[0]);
        for (int k = 0; k < 6; ++k) atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_WX + k], e[1 + k]);
    }
}

// ----------------------------------------------------------------------------
// launchers
// ----------------------------------------------------------------------------
size_t spread64_smem(int P, int T) {
    const int E = T + P - 1;
    return (spread64_region(E) + (size_t)K64S_CH * (K64S_SEG + 2 * P) + (size_t)P * (MAX_D + 1)) *
               sizeof(double) +
           (size_t)(K64S_CH + E * E + E) * sizeof(uint32_t);
}

cudaError_t launch64_configure(int P, int T) {
    const cudaError_t e =
        cudaFuncSetAttribute(k64_spread, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)spread64_smem(P, T));
    if (e != cudaSuccess) return e;
    ESPB_DISPATCH_P(configure64_interp_p, P, T);
}

cudaError_t launch64_eval(const Launch64& b, cudaStream_t st) {
    const LaunchArgs& a = b.a;
    const bool lr = b.long_range, sr = b.short_range;
    if (a.n_chunks)
        k64_bin<<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.P, a.T, b.pos_in, b.q_in, b.posq, b.trec, a.rel,
                                            a.key, a.tile_count, a.acc);
    if (lr) {
        cudaError_t e = launch_scan(a.tile_count, a.tile_start, a.n_tiles, st);
        if (e != cudaSuccess) return e;
        e = launch_scatter(a.chunks, a.n_chunks, a.sys, a.key, a.tile_start, a.tile_count, a.perm_u, st);
        if (e != cudaSuccess) return e;
        if (a.n_tiles) {
            k64_tile_sort<<<a.n_tiles, 256, 0, st>>>(a.tile_start, a.perm_u, a.perm, b.trec, a.rel, b.srec, a.srel);
            k64_spread<<<dim3(a.n_tiles, split64(a.n_tiles)), K64S_THREADS, spread64_smem(a.P, a.T), st>>>(
                a.tile_sys, a.sys, b.wcoef, a.P, a.T, a.D, a.tile_start, b.srec, a.srel, a.rho);
        }
        if (b.n_xl) k64_fft_pass<0><<<b.n_xl, F64_WARPS * 32, 0, st>>>(b.xl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (b.n_yl) k64_fft_pass<1><<<b.n_yl, F64_WARPS * 32, 0, st>>>(b.yl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (b.n_zl) k64_fft_pass<2><<<b.n_zl, F64_WARPS * 32, 0, st>>>(b.zl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (b.n_yl) k64_fft_pass<3><<<b.n_yl, F64_WARPS * 32, 0, st>>>(b.yl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (b.n_xl) k64_fft_pass<4><<<b.n_xl, F64_WARPS * 32, 0, st>>>(b.xl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (a.n_tiles) {
            e = [&]() -> cudaError_t { ESPB_DISPATCH_P(launch64_interp_p, a.P, b, st); }();
            if (e != cudaSuccess) return e;
        }
        if (a.n_chunks && a.ex_n)
            k64_exclusions<<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.psets, b.qv, b.nq, b.posq, a.ex_n,
                                                       a.ex_list, a.ex_pitch, b.force, a.acc);
    }
    if (sr && b.n_pchunks)
    {
        if (a.want_virial)
            k64_pair<true><<<b.n_pchunks, 256, 0, st>>>(b.pchunks, a.sys, a.psets, b.qv, b.nq, b.posq, a.nl_head,
                                                        a.nl_n, a.nl_list, b.force, a.acc, lr ? 1 : 0);
        else
            k64_pair<false><<<b.n_pchunks, 256, 0, st>>>(b.pchunks, a.sys, a.psets, b.qv, b.nq, b.posq, a.nl_head,
                                                         a.nl_n, a.nl_list, b.force, a.acc, lr ? 1 : 0);
    }
    return cudaGetLastError();
}

}  // namespace espb
