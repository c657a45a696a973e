// Shared device-side definitions for the ESP kernels (sm_100a).
//
// Every kernel is batched: it reads a per-system descriptor (SysDev) and a
// work-item list, so the plain one-system path is the same code launched on
// a batch of one. Mesh layout is x-fastest, cell = (z*ny + y)*nx + x, as in
// the reference (src/ESPForceComputeGPU.cu:267).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace espb {

constexpr int MAX_P = 12;      // ESP_MAX_ORDER (src/ESPForceCompute.h:63)
constexpr int MAX_D = 15;      // window polynomial degree limit
constexpr int MAX_QC = 32;     // split polynomial coefficients
constexpr int ACC_STRIDE = 24; // doubles of per-system accumulators
constexpr int FFT_MAX_N = 256; // longest 1D transform (2/3/5-smooth)
constexpr int FFT_B_YZ = 16;   // columns per CTA in the y/z passes
constexpr int FFT_B_X = 8;     // row pairs per CTA in the x passes
constexpr int FFT_SB_X = 9;    // padded line stride of the x passes (bank-conflict free)
constexpr float INV_4PI_F = 0.0795774715459476678f;
constexpr double INV_4PI_D = 0.079577471545947673;  // ESP_INV_4PI, src/ESPForceCompute.cc:36

// Accumulator slots (double[ACC_STRIDE] per system).
enum AccSlot {
    ACC_QSUM = 0,   // sum q
    ACC_Q2SUM = 1,  // sum q^2
    ACC_E = 2,      // sum of per-particle energies (mesh + self + pair)
    ACC_EK = 3,     // k-space energy (diagnostic, with the virial; equals the mesh energy)
    ACC_WK = 4,     // k-space virial xx,xy,xz,yy,yz,zz (4..9)
    ACC_WP = 10,    // pair virial (10..15)
    ACC_WX = 16,    // exclusion-correction virial (16..21)
};

struct SysDev {
    int N;             // particles
    int p_off;         // first particle in the concatenated arrays
    int nx, ny, nz, nxh;
    long long m_off;   // real-mesh element offset
    long long s_off;   // half-spectrum element offset (float2)
    long long g_off;   // influence-table element offset (float2)
    int ntx, nty, ntz, t_off;  // tile grid and first tile
    float Lx, Ly, Lz;
    float inv_Lx, inv_Ly, inv_Lz;
    double gxd, gyd, gzd;  // n / L in FP64
    double Lxd, Lyd, Lzd;  // box lengths in FP64 (FP64 mode)
    double V;
    int pset;          // parameter-set index
    int twx, twy, twz; // twiddle-table offsets per axis
    uint32_t radx, rady, radz;  // packed radix plans (4 bits per stage)
    // potential mesh with a periodic halo: nxp x nyp x nzp (x fastest) at
    // element offset mp_off, point (x, y, z) holding phi(x mod nx, y mod ny,
    // z mod nz), so every tile's extended region is one box without wrap
    long long mp_off;
    int nxp, nyp, nzp;
};

// Padded extent of the halo potential mesh along an axis of n points with
// tiles of edge T and support P: every tile's extended region [t T, t T +
// T + P - 1) lies inside; x rows are rounded up to whole 16-byte groups.
__host__ __device__ inline int halo_extent(int n, int T, int P, bool x_axis) {
    const int e = ((n + T - 1) / T) * T + P - 1;
    return x_axis ? (e + 3) & ~3 : e;
}

struct ParamSet {
    float wcoef[MAX_P * (MAX_D + 1)];  // window polynomial [a][j] in t
    float qv[MAX_QC];    // Q(v) = sum qv[j] v^j, v = 2u - 1, u = r^2/r_c^2
    float dqv[MAX_QC];   // dQ/du as a series in v
    int nq;              // number of Q coefficients (dQ has nq-1)
    float rcut, rcut2, inv_rcut, two_inv_rcut3;
    double self_coef;    // per-particle self energy = self_coef * q^2
    double bg_coef;      // E_bg = bg_coef * Q^2 / V
    double rcut_d;       // r_c in FP64 (FP64 mode)
};

// ----------------------------------------------------------------------------
// small helpers
// ----------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Kahan-compensated update of (sum, comp) in shared memory; rounding is
// pinned with the _rn intrinsics so the compiler cannot re-associate.
__device__ __forceinline__ void kahan_add(float* sum, float* comp, float v) {
    const float s = *sum;
    const float y = __fsub_rn(v, *comp);
    const float t = __fadd_rn(s, y);
    *comp = __fsub_rn(__fsub_rn(t, s), y);
    *sum = t;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide FP64 sum of K values; result valid in thread 0.
template <int K>
__device__ __forceinline__ void block_sum_f64(double (&v)[K], double* red /* smem [32*K] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) red[wid * K + k] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double x = lane < nw ? red[lane * K + k] : 0.0;
            v[k] = warp_sum(x);
        }
    }
}

// Window weights: every segment is evaluated at the same local t.
__device__ __forceinline__ float horner_w(const float* c, int D, float t) {
    float v = c[D];
    for (int j = D - 1; j >= 0; --j) v = fmaf(v, t, c[j]);
    return v;
}
__device__ __forceinline__ float horner_dw(const float* c, int D, float t) {
    float v = D * c[D];
    for (int j = D - 1; j >= 1; --j) v = fmaf(v, t, j * c[j]);
    return v;
}

// Default window degree of the FP32 path for support P (what the planner
// picks when the degree is not set; the staging kernels unroll this case
// fully): P for P >= 8 (fit error 4.7e-9 at P = 8, below the FP32
// evaluation's rounding), 9 below that. The FP64 mode uses max(P + 2, 9).
__host__ __device__ constexpr int default_window_degree(int P) { return P >= 8 ? P : 9; }
template <int P>
constexpr int default_window_degree() {
    return default_window_degree(P);
}

// One window segment held in registers by the thread that evaluates it
// (degree DD at compile time, or a runtime degree through shared memory).
template <int DD>
struct SegPoly {
    float c[DD + 1];  // w(t)  = sum_j c[j] t^j
    float d[DD];      // w'(t) = sum_j d[j] t^j, d[j] = (j+1) c[j+1]
    __device__ __forceinline__ void load(const float* wc_seg) {
#pragma unroll
        for (int j = 0; j <= DD; ++j) c[j] = wc_seg[j];
#pragma unroll
        for (int j = 0; j < DD; ++j) d[j] = (float)(j + 1) * c[j + 1];
    }
    __device__ __forceinline__ float w(float t) const {
        float v = c[DD];
#pragma unroll
        for (int j = DD - 1; j >= 0; --j) v = fmaf(v, t, c[j]);
        return v;
    }
    __device__ __forceinline__ float dw(float t) const {
        float v = d[DD - 1];
#pragma unroll
        for (int j = DD - 2; j >= 0; --j) v = fmaf(v, t, d[j]);
        return v;
    }
};

// Launch FN<P> for a stencil order known at run time (2..ESP_MAX_ORDER).
#define ESPB_DISPATCH_P(FN, P_, ...)                 \
    switch (P_) {                                    \
        case 2: return FN<2>(__VA_ARGS__);           \
        case 3: return FN<3>(__VA_ARGS__);           \
        case 4: return FN<4>(__VA_ARGS__);           \
        case 5: return FN<5>(__VA_ARGS__);           \
        case 6: return FN<6>(__VA_ARGS__);           \
        case 7: return FN<7>(__VA_ARGS__);           \
        case 8: return FN<8>(__VA_ARGS__);           \
        case 9: return FN<9>(__VA_ARGS__);           \
        case 10: return FN<10>(__VA_ARGS__);         \
        case 11: return FN<11>(__VA_ARGS__);         \
        case 12: return FN<12>(__VA_ARGS__);         \
        default: return cudaErrorInvalidValue;       \
    }

}  // namespace espb
