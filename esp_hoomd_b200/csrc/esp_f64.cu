// FP64 mode of the ESP path: every stage in double precision, for HOOMD
// double builds (Scalar4 = double4 positions and forces) and for accuracy
// targets below the FP32 floor (~1e-7). Same algorithm and data layout as
// the FP32 kernels:
//   k64_bin / k64_tile_sort : tile keys (shared sort kernels) with FP64
//                             stencil records;
//   k64_spread              : one CTA per tile, FP64 accumulation of the
//                             tile's extended region in shared memory, one
//                             FP64 atomic per region point into the mesh;
//   k64_fft_pass            : one warp per mesh line, mixed-radix Stockham in
//                             shared memory on the full complex spectrum; the
//                             z pass multiplies by the influence table and
//                             accumulates the k-space energy and virial;
//   k64_interp, k64_pair, k64_exclusions : as the FP32 kernels, in FP64.
// Reference stages: src/ESPForceComputeGPU.cu:157-471 (K1-K7).
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
        atomicAdd(&tile_count[k], 1u);
        posq[i] = make_double4(x[0], x[1], x[2], q);
        trec[i] = make_double4(tt[0], tt[1], tt[2], q);
        rel[i] = (uint32_t)(i0m[0] - tx * T) | ((uint32_t)(i0m[1] - ty * T) << 8) |
                 ((uint32_t)(i0m[2] - tz * T) << 16);
        qs[0] = q;
        qs[1] = q * q;
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

// ----------------------------------------------------------------------------
// spreading: one CTA per tile, shared FP64 region [E]^3 (E = T + P - 1),
// one warp per particle (lanes over the P^3 stencil), FP64 shared atomics
// ----------------------------------------------------------------------------
constexpr int K64_WARPS = 8;

__global__ void __launch_bounds__(K64_WARPS * 32)
    k64_spread(const int* __restrict__ tile_sys, const SysDev* __restrict__ sys, const double* __restrict__ wcoef,
               int P, int T, int D, const uint32_t* __restrict__ start, const double4* __restrict__ srec,
               const uint32_t* __restrict__ srel, double* __restrict__ rho) {
    extern __shared__ double sreg[];  // [E^3] region, then [K64_WARPS][3 * MAX_P] weights
    const int t = blockIdx.x;
    const uint32_t s0 = start[t];
    const int np = (int)(start[t + 1] - s0);
    if (np == 0) return;
    const SysDev S = sys[tile_sys[t]];
    const int E = T + P - 1, E3 = E * E * E;
    double* wts = sreg + E3;
    for (int k = threadIdx.x; k < E3; k += blockDim.x) sreg[k] = 0.0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* W = wts + warp * 3 * MAX_P;
    for (int p = warp; p < np; p += K64_WARPS) {
        const double4 rec = srec[s0 + p];
        const uint32_t rl = srel[s0 + p];
        if (lane < 3 * P) {
            const int ax = lane / P, a = lane - ax * P;
            const double tt = ax == 0 ? rec.x : (ax == 1 ? rec.y : rec.z);
            W[lane] = horner64(wcoef + a * (D + 1), D, tt) * (ax == 0 ? rec.w : 1.0);
        }
        __syncwarp();
        const int ox = rl & 255, oy = (rl >> 8) & 255, oz = (rl >> 16) & 255;
        const int P3 = P * P * P;
        for (int k = lane; k < P3; k += 32) {
            const int a = k % P, b = (k / P) % P, c = k / (P * P);
            atomicAdd(&sreg[((oz + c) * E + (oy + b)) * E + ox + a], W[a] * W[P + b] * W[2 * P + c]);
        }
        __syncwarp();
    }
    __syncthreads();
    const int lt = t - S.t_off;
    const int X0 = (lt % S.ntx) * T, Y0 = ((lt / S.ntx) % S.nty) * T, Z0 = (lt / (S.ntx * S.nty)) * T;
    for (int k = threadIdx.x; k < E3; k += blockDim.x) {
        const double v = sreg[k];
        if (v == 0.0) continue;
        int gx = X0 + k % E, gy = Y0 + (k / E) % E, gz = Z0 + k / (E * E);
        while (gx >= S.nx) gx -= S.nx;
        while (gy >= S.ny) gy -= S.ny;
        while (gz >= S.nz) gz -= S.nz;
        atomicAdd(&rho[S.m_off + ((long long)gz * S.ny + gy) * S.nx + gx], v);
    }
}

// ----------------------------------------------------------------------------
// FFT: one warp per line, Stockham autosort, radices 2/3/4/5 from the packed
// plan; tw = exp(-2 pi i t / n) (the forward sign), conjugated for inverse
// ----------------------------------------------------------------------------
__device__ __forceinline__ double2 z_mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// R-point DFT in place, sign -1 forward / +1 inverse.
__device__ __forceinline__ void dft_small(double2* v, int R, int sign) {
    const double s = (double)sign;
    if (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = make_double2(a.x + b.x, a.y + b.y);
        v[1] = make_double2(a.x - b.x, a.y - b.y);
    } else if (R == 4) {
        const double2 a = v[0], b = v[1], c = v[2], d = v[3];
        const double2 ac = make_double2(a.x + c.x, a.y + c.y), am = make_double2(a.x - c.x, a.y - c.y);
        const double2 bd = make_double2(b.x + d.x, b.y + d.y), bm = make_double2(b.x - d.x, b.y - d.y);
        // multiply bm by (sign i): forward -i
        const double2 jb = make_double2(-s * bm.y, s * bm.x);
        v[0] = make_double2(ac.x + bd.x, ac.y + bd.y);
        v[1] = make_double2(am.x + jb.x, am.y + jb.y);
        v[2] = make_double2(ac.x - bd.x, ac.y - bd.y);
        v[3] = make_double2(am.x - jb.x, am.y - jb.y);
    } else {
        // generic O(R^2) for R = 3, 5 with the exact roots of unity
        const double c1 = R == 3 ? -0.5 : 0.30901699437494742410, s1 = R == 3 ? 0.86602540378443864676 : 0.95105651629515357212;
        const double c2 = -0.80901699437494742410, s2 = 0.58778525229247312917;
        double2 out[5];
        for (int k = 0; k < R; ++k) {
            double2 acc = make_double2(0.0, 0.0);
            for (int r = 0; r < R; ++r) {
                const int m = (r * k) % R;
                double cr, sr;
                if (m == 0) { cr = 1.0; sr = 0.0; }
                else if (R == 3) { cr = c1; sr = m == 1 ? s1 : -s1; }
                else if (m == 1 || m == 4) { cr = c1; sr = m == 1 ? s1 : -s1; }
                else { cr = c2; sr = m == 2 ? s2 : -s2; }
                // exp(sign * 2 pi i m / R) with the forward sign -1
                const double2 w = make_double2(cr, s * sr);
                acc.x += v[r].x * w.x - v[r].y * w.y;
                acc.y += v[r].x * w.y + v[r].y * w.x;
            }
            out[k] = acc;
        }
        for (int k = 0; k < R; ++k) v[k] = out[k];
    }
}

// Transforms the n points in a (scratch b); returns the buffer holding the result.
__device__ double2* fft64_line(double2* a, double2* b, int n, uint32_t plan, const double2* __restrict__ tw,
                               int sign, int lane) {
    int Ns = 1;
    double2 *src = a, *dst = b;
    for (uint32_t pl = plan; pl; pl >>= 4) {
        const int R = pl & 15;
        const int nb = n / R;
        const int step = n / (Ns * R);
        for (int j = lane; j < nb; j += 32) {
            const int k = j % Ns;
            double2 v[5];
            for (int r = 0; r < R; ++r) {
                v[r] = src[j + r * nb];
                if (r > 0 && k > 0) {
                    double2 w = tw[(r * k * step) % n];
                    if (sign > 0) w.y = -w.y;
                    v[r] = z_mul(v[r], w);
                }
            }
            dft_small(v, R, sign);
            const int idxD = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; ++r) dst[idxD + r * Ns] = v[r];
        }
        __syncwarp();
        double2* x = src;
        src = dst;
        dst = x;
        Ns *= R;
    }
    return src;
}

constexpr int F64_WARPS = 4;

// MODE 0: x forward (real mesh -> spectrum, the mesh is cleared), 1: y
// forward, 2: z forward + influence multiply + energy/virial + z inverse,
// 3: y inverse, 4: x inverse (spectrum -> real potential).
template <int MODE>
__global__ void __launch_bounds__(F64_WARPS * 32)
    k64_fft_pass(const int2* __restrict__ items, const SysDev* __restrict__ sys, const double2* __restrict__ tw,
                 double2* __restrict__ cbuf, double* __restrict__ rho, double* __restrict__ phi,
                 const double2* __restrict__ gtab, double* __restrict__ acc) {
    __shared__ double2 sb[F64_WARPS][2][FFT_MAX_N];
    __shared__ double red[32 * 7];
    const int2 it = items[blockIdx.x];
    const SysDev S = sys[it.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int AX = (MODE == 0 || MODE == 4) ? 0 : (MODE == 1 || MODE == 3) ? 1 : 2;
    const int n = AX == 0 ? S.nx : (AX == 1 ? S.ny : S.nz);
    const long long nlines = AX == 0 ? (long long)S.ny * S.nz : (AX == 1 ? (long long)S.nx * S.nz : (long long)S.nx * S.ny);
    const long long l = (long long)it.y + warp;
    double e[7] = {0, 0, 0, 0, 0, 0, 0};
    if (l < nlines) {
        long long base, stride;
        int lx = 0, ly = 0;
        if (AX == 0) {
            base = l * S.nx;
            stride = 1;
        } else if (AX == 1) {
            const long long z = l / S.nx, x = l % S.nx;
            base = z * S.nx * S.ny + x;
            stride = S.nx;
        } else {
            ly = (int)(l / S.nx);
            lx = (int)(l % S.nx);
            base = (long long)ly * S.nx + lx;
            stride = (long long)S.nx * S.ny;
        }
        const uint32_t plan = AX == 0 ? S.radx : (AX == 1 ? S.rady : S.radz);
        const double2* twa = tw + (AX == 0 ? S.twx : (AX == 1 ? S.twy : S.twz));
        double2* a = sb[warp][0];
        double2* b = sb[warp][1];
        for (int k = lane; k < n; k += 32) {
            const long long g = S.m_off + base + k * stride;
            if (MODE == 0) {
                a[k] = make_double2(rho[g], 0.0);
                rho[g] = 0.0;
            } else {
                a[k] = cbuf[g];
            }
        }
        __syncwarp();
        const int sign = (MODE <= 1) ? -1 : (MODE == 2 ? -1 : 1);
        double2* r = fft64_line(a, b, n, plan, twa, sign, lane);
        if (MODE == 2) {
            // (kx, ky) = (lx, ly) after the x and y passes; kz along the line
            const int nxh = S.nxh;
            const double tpx = 6.283185307179586 / S.Lxd, tpy = 6.283185307179586 / S.Lyd,
                         tpz = 6.283185307179586 / S.Lzd;
            const int fx = lx <= S.nx / 2 ? lx : lx - S.nx;
            const int fy = ly <= S.ny / 2 ? ly : ly - S.ny;
            for (int kz = lane; kz < n; kz += 32) {
                const int fz = kz <= S.nz / 2 ? kz : kz - S.nz;
                long long gi;
                if (lx < nxh) gi = ((long long)kz * S.ny + ly) * nxh + lx;
                else gi = ((long long)((S.nz - kz) % S.nz) * S.ny + (S.ny - ly) % S.ny) * nxh + (S.nx - lx);
                const double2 g = gtab[S.g_off + gi];
                const double2 v = r[kz];
                const double a2 = v.x * v.x + v.y * v.y;
                const double ek = 0.5 * g.x * a2, eb = 0.5 * g.y * a2;
                const double kxv = tpx * fx, kyv = tpy * fy, kzv = tpz * fz;
                e[0] += ek;
                e[1] += ek + eb * kxv * kxv;
                e[2] += eb * kxv * kyv;
                e[3] += eb * kxv * kzv;
                e[4] += ek + eb * kyv * kyv;
                e[5] += eb * kyv * kzv;
                e[6] += ek + eb * kzv * kzv;
                r[kz] = make_double2(v.x * g.x, v.y * g.x);
            }
            __syncwarp();
            double2* o = (r == a) ? b : a;
            r = fft64_line(r, o, n, plan, twa, +1, lane);
        }
        for (int k = lane; k < n; k += 32) {
            const long long g = S.m_off + base + k * stride;
            if (MODE == 4) phi[g] = r[k].x;
            else cbuf[g] = r[k];
        }
    }
    if (MODE == 2) {
        block_sum_f64<7>(e, red);
        if (threadIdx.x == 0)
            for (int k = 0; k < 7; ++k) atomicAdd(&acc[it.x * ACC_STRIDE + ACC_EK + k], e[k]);
    }
}

// ----------------------------------------------------------------------------
// interpolation: one thread per particle, potential, gradient and energy
// ----------------------------------------------------------------------------
__global__ void k64_interp(const int2* __restrict__ chunks, const SysDev* __restrict__ sys,
                           const ParamSet* __restrict__ psets, const double* __restrict__ wcoef, int P, int D,
                           const double4* __restrict__ posq, const double* __restrict__ phi,
                           double4* __restrict__ force, double* __restrict__ acc) {
    __shared__ double red[32];
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const int i = ch.y + threadIdx.x;
    double e1[1] = {0.0};
    if (i < S.p_off + S.N) {
        const double4 p = posq[i];
        const double x[3] = {p.x, p.y, p.z};
        const double gd[3] = {S.gxd, S.gyd, S.gzd};
        const int n[3] = {S.nx, S.ny, S.nz};
        double W[3][MAX_P], dW[3][MAX_P];
        int idx[3][MAX_P];
        for (int d = 0; d < 3; ++d) {
            double g = x[d] * gd[d];
            if (g >= n[d]) g -= n[d];
            const int i0 = (int)floor(g - 0.5 * P) + 1;
            const double tt = (double)i0 + 0.5 * P - g;
            int v = i0 < 0 ? i0 + n[d] : (i0 >= n[d] ? i0 - n[d] : i0);
            for (int a = 0; a < P; ++a) {
                W[d][a] = horner64(wcoef + a * (D + 1), D, tt);
                dW[d][a] = dhorner64(wcoef + a * (D + 1), D, tt);
                idx[d][a] = v;
                if (++v == n[d]) v = 0;
            }
        }
        const double* ph = phi + S.m_off;
        double pot = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        for (int c = 0; c < P; ++c)
            for (int b = 0; b < P; ++b) {
                const double* row = ph + ((long long)idx[2][c] * S.ny + idx[1][b]) * S.nx;
                double sv = 0.0, sd = 0.0;
                for (int a = 0; a < P; ++a) {
                    const double v = row[idx[0][a]];
                    sv = fma(W[0][a], v, sv);
                    sd = fma(dW[0][a], v, sd);
                }
                pot = fma(W[2][c] * W[1][b], sv, pot);
                gx = fma(W[2][c] * W[1][b], sd, gx);
                gy = fma(W[2][c] * dW[1][b], sv, gy);
                gz = fma(dW[2][c] * W[1][b], sv, gz);
            }
        const double q = p.w;
        const double e_i = 0.5 * q * pot + psets[S.pset].self_coef * q * q;
        force[i] = make_double4(q * S.gxd * gx, q * S.gyd * gy, q * S.gzd * gz, e_i);
        e1[0] = e_i;
    }
    block_sum_f64<1>(e1, red);
    if (threadIdx.x == 0) atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_E], e1[0]);
}

// ----------------------------------------------------------------------------
// pair term (EvaluatorPairPSWF, src/EvaluatorPairPSWF.h:274-295) in FP64:
// 8 lanes per particle over its neighbour row
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k64_pair(const int2* __restrict__ chunks, const SysDev* __restrict__ sys, const ParamSet* __restrict__ psets,
             const double* __restrict__ qv, int nq, const double4* __restrict__ posq,
             const uint32_t* __restrict__ head, const uint32_t* __restrict__ nn, const uint32_t* __restrict__ nlist,
             double4* __restrict__ force, double* __restrict__ acc, int accumulate, int want_virial) {
    __shared__ double red[32 * 7];
    constexpr int TPP = 8;
    const int2 ch = chunks[blockIdx.x];
    const SysDev S = sys[ch.x];
    const ParamSet& ps = psets[S.pset];
    const double rc = ps.rcut_d, rc2 = rc * rc, irc = 1.0 / rc, irc2 = irc * irc, tirc3 = 2.0 * irc2 * irc;
    const int i = ch.y + threadIdx.x / TPP;
    const int sub = threadIdx.x % TPP;
    const bool valid = i < S.p_off + S.N;
    double fx = 0, fy = 0, fz = 0, en = 0, v[6] = {0, 0, 0, 0, 0, 0};
    if (valid) {
        const double4 pi = posq[i];
        const uint32_t n = nn[i], h = head[i];
        for (uint32_t k = sub; k < n; k += TPP) {
            const double4 pj = posq[S.p_off + (int)nlist[h + k]];
            double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            dx -= S.Lxd * rint(dx / S.Lxd);
            dy -= S.Lyd * rint(dy / S.Lyd);
            dz -= S.Lzd * rint(dz / S.Lzd);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < rc2 && r2 > 0.0) {
                const double ri = 1.0 / sqrt(r2);
                const double vv = fma(2.0 * irc2, r2, -1.0);
                double Q = qv[nq - 1], dQ = (nq - 1) * qv[nq - 1];
                for (int c = nq - 2; c >= 0; --c) Q = fma(Q, vv, qv[c]);
                for (int c = nq - 2; c >= 1; --c) dQ = fma(dQ, vv, c * qv[c]);
                dQ *= 2.0;  // dQ/du = 2 dQ/dv
                const double qq = pi.w * pj.w * INV_4PI_D;
                const double fdr = qq * (tirc3 * dQ + ri * ri * ri);
                en += qq * (ri - Q * irc);
                fx += fdr * dx;
                fy += fdr * dy;
                fz += fdr * dz;
                if (want_virial) {
                    v[0] += fdr * dx * dx;
                    v[1] += fdr * dx * dy;
                    v[2] += fdr * dx * dz;
                    v[3] += fdr * dy * dy;
                    v[4] += fdr * dy * dz;
                    v[5] += fdr * dz * dz;
                }
            }
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
    double e[7] = {sub == 0 ? 0.5 * en : 0.0, 0.5 * v[0], 0.5 * v[1], 0.5 * v[2], 0.5 * v[3], 0.5 * v[4], 0.5 * v[5]};
    block_sum_f64<7>(e, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_E], e[0]);
        for (int k = 0; k < 6; ++k) atomicAdd(&acc[ch.x * ACC_STRIDE + ACC_WP + k], e[1 + k]);
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
    return ((size_t)E * E * E + (size_t)K64_WARPS * 3 * MAX_P) * sizeof(double);
}

cudaError_t launch64_configure(int P, int T) {
    return cudaFuncSetAttribute(k64_spread, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)spread64_smem(P, T));
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
            k64_spread<<<a.n_tiles, K64_WARPS * 32, spread64_smem(a.P, a.T), st>>>(
                a.tile_sys, a.sys, b.wcoef, a.P, a.T, a.D, a.tile_start, b.srec, a.srel, a.rho);
        }
        if (b.n_xl) k64_fft_pass<0><<<b.n_xl, F64_WARPS * 32, 0, st>>>(b.xl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (b.n_yl) k64_fft_pass<1><<<b.n_yl, F64_WARPS * 32, 0, st>>>(b.yl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (b.n_zl) k64_fft_pass<2><<<b.n_zl, F64_WARPS * 32, 0, st>>>(b.zl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (b.n_yl) k64_fft_pass<3><<<b.n_yl, F64_WARPS * 32, 0, st>>>(b.yl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (b.n_xl) k64_fft_pass<4><<<b.n_xl, F64_WARPS * 32, 0, st>>>(b.xl, a.sys, b.tw, b.cbuf, a.rho, b.phi, b.gtab, a.acc);
        if (a.n_chunks)
            k64_interp<<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.psets, b.wcoef, a.P, a.D, b.posq, b.phi, b.force,
                                                   a.acc);
        if (a.n_chunks && a.ex_n)
            k64_exclusions<<<a.n_chunks, 256, 0, st>>>(a.chunks, a.sys, a.psets, b.qv, b.nq, b.posq, a.ex_n,
                                                       a.ex_list, a.ex_pitch, b.force, a.acc);
    }
    if (sr && b.n_pchunks)
        k64_pair<<<b.n_pchunks, 256, 0, st>>>(b.pchunks, a.sys, a.psets, b.qv, b.nq, b.posq,
                                                               a.nl_head, a.nl_n, a.nl_list, b.force, a.acc,
                                                               lr ? 1 : 0, a.want_virial);
    return cudaGetLastError();
}

}  // namespace espb
