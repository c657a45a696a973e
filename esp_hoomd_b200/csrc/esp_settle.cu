// Rigid three-site molecules in the MD harness: SETTLE for positions and the
// RATTLE velocity constraint (Miyamoto & Kollman, J. Comput. Chem. 13, 952
// (1992)). The reference plugin has no constraint code -- HOOMD supplies the
// integrators -- but the water workloads are rigid (O, H, H) molecules.
//
// One thread per molecule over work items {system, first atom, molecules,
// geometry} of up to SETTLE_CHUNK consecutive (O, H, H) triples, the
// geometry an index into a table of (d_OH, d_HH); FP64 arithmetic
// relative to the molecule's oxygen (one periodic image per molecule),
// masses from the velocity arrays' w.
//
// Positions: the unconstrained velocity-Verlet update x0 -> x1 is corrected
// to x3 = x1 + Delta with m_i Delta_i a combination of the old bond vectors.
// Those lie in the old molecular plane, so in a frame whose z axis is normal
// to it the z coordinates keep their unconstrained values: the canonical
// triangle (O at (0, ra), H at (-/+rc, -rb) about the centre of mass)
// rotated by phi about x and psi about y reproduces them, and a rotation
// theta about z removes the constraint forces' net torque,
// A sin(theta) + B cos(theta) = C. The half-step velocity becomes
// (x3 - x0) / dt.
// Velocities: after the second half kick, v_i += sum_k mu_k dsigma_k/dx_i /
// m_i with the three multipliers solving r_k . v_k = 0 (bonds OH, OH, HH).
#include "esp_common.cuh"
#include "esp_md.h"

namespace espb {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 unit(D3 a) { return rsqrt(dot(a, a)) * a; }

template <typename T4>
__device__ __forceinline__ D3 xyz(const T4& p) {
    return d3((double)p.x, (double)p.y, (double)p.z);
}

// minimum image of d in an orthorhombic box
__device__ __forceinline__ D3 min_image(D3 d, const SysDev& S) {
    d.x -= S.Lxd * rint(d.x / S.Lxd);
    d.y -= S.Lyd * rint(d.y / S.Lyd);
    d.z -= S.Lzd * rint(d.z / S.Lzd);
    return d;
}

__device__ __forceinline__ double wrap1(double x, double L) {
    x -= L * floor(x / L);
    if (x >= L) x -= L;
    if (x < 0.0) x += L;
    return x;
}

// SETTLE of one molecule: old (constrained) positions a0 = 0, b0, c0 and
// unconstrained a1, b1, c1, all relative to the old oxygen; returns the
// constrained positions in a3, b3, c3.
__device__ void settle_one(D3 b0, D3 c0, D3 a1, D3 b1, D3 c1, double mo, double mh, double d_oh, double d_hh,
                           D3& a3, D3& b3, D3& c3) {
    const double mt = mo + 2.0 * mh;
    const double rc = 0.5 * d_hh;
    const double h = sqrt(d_oh * d_oh - rc * rc);
    const double ra = 2.0 * mh / mt * h, rb = h - ra;
    const D3 com = (1.0 / mt) * (mo * a1 + mh * (b1 + c1));
    const D3 A1 = a1 - com, B1 = b1 - com, C1 = c1 - com;
    const D3 ez = unit(cross(b0, c0));
    const D3 ex = unit(cross(A1, ez));
    const D3 ey = cross(ez, ex);
    const double xb0 = dot(b0, ex), yb0 = dot(b0, ey), xc0 = dot(c0, ex), yc0 = dot(c0, ey);
    const double za1 = dot(A1, ez);
    const double xb1 = dot(B1, ex), yb1 = dot(B1, ey), zb1 = dot(B1, ez);
    const double xc1 = dot(C1, ex), yc1 = dot(C1, ey), zc1 = dot(C1, ez);
    const double sphi = za1 / ra;
    const double cphi = sqrt(fmax(0.0, 1.0 - sphi * sphi));
    const double spsi = (zb1 - zc1) / (2.0 * rc * cphi);
    const double cpsi = sqrt(fmax(0.0, 1.0 - spsi * spsi));
    const double ya2 = ra * cphi, xb2 = -rc * cpsi;
    const double t1 = -rb * cphi, t2 = rc * spsi * sphi;
    const double yb2 = t1 - t2, yc2 = t1 + t2;
    const double A = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2;
    const double B = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2;
    const double C = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0;
    const double ab2 = A * A + B * B;
    const double sth = (A * C - B * sqrt(fmax(0.0, ab2 - C * C))) / ab2;
    const double cth = sqrt(fmax(0.0, 1.0 - sth * sth));
    a3 = com + (-ya2 * sth) * ex + (ya2 * cth) * ey + za1 * ez;
    b3 = com + (xb2 * cth - yb2 * sth) * ex + (xb2 * sth + yb2 * cth) * ey + zb1 * ez;
    c3 = com + (-xb2 * cth - yc2 * sth) * ex + (-xb2 * sth + yc2 * cth) * ey + zc1 * ez;
}

// Velocity-Verlet first half for the atoms of rigid molecules (k_nve1 skips
// them): v += dt/2 F/m, unconstrained x1 = x0 + dt v, SETTLE, v = (x3 - x0)/dt.
template <typename T4>
__global__ void __launch_bounds__(SETTLE_CHUNK)
    k_settle1(const int4* __restrict__ items, const SysDev* __restrict__ sys, T4* __restrict__ pos,
              T4* __restrict__ vel, const T4* __restrict__ force, double dt, const double2* __restrict__ geo) {
    const int4 it = items[blockIdx.x];
    if ((int)threadIdx.x >= it.z) return;
    const double d_oh = geo[it.w].x, d_hh = geo[it.w].y;
    const SysDev& S = sys[it.x];
    const int i = it.y + 3 * (int)threadIdx.x;
    T4 p[3], v[3];
    D3 x0[3], x1[3], vh[3];
    double m[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p[k] = pos[i + k];
        v[k] = vel[i + k];
        const T4 f = force[i + k];
        m[k] = (double)v[k].w;
        const double hk = 0.5 * dt / m[k];
        vh[k] = xyz(v[k]) + hk * xyz(f);
    }
    const D3 o = xyz(p[0]);
    x0[0] = d3(0.0, 0.0, 0.0);
    x0[1] = min_image(xyz(p[1]) - o, S);
    x0[2] = min_image(xyz(p[2]) - o, S);
#pragma unroll
    for (int k = 0; k < 3; ++k) x1[k] = x0[k] + dt * vh[k];
    D3 x3[3];
    settle_one(x0[1], x0[2], x1[0], x1[1], x1[2], m[0], 0.5 * (m[1] + m[2]), d_oh, d_hh, x3[0], x3[1], x3[2]);
    const double idt = 1.0 / dt;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const D3 vn = idt * (x3[k] - x0[k]);
        const D3 xa = o + x3[k];
        T4 po = p[k], ve = v[k];
        po.x = wrap1(xa.x, S.Lxd);
        po.y = wrap1(xa.y, S.Lyd);
        po.z = wrap1(xa.z, S.Lzd);
        ve.x = vn.x;
        ve.y = vn.y;
        ve.z = vn.z;
        pos[i + k] = po;
        vel[i + k] = ve;
    }
}

// RATTLE velocity constraint after the second half kick.
template <typename T4>
__global__ void __launch_bounds__(SETTLE_CHUNK)
    k_settle2(const int4* __restrict__ items, const SysDev* __restrict__ sys, const T4* __restrict__ pos,
              T4* __restrict__ vel) {
    const int4 it = items[blockIdx.x];
    if ((int)threadIdx.x >= it.z) return;
    const SysDev& S = sys[it.x];
    const int i = it.y + 3 * (int)threadIdx.x;
    T4 v[3];
    D3 x[3], u[3];
    double im[3];
    const D3 o = xyz(pos[i]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = vel[i + k];
        u[k] = xyz(v[k]);
        im[k] = 1.0 / (double)v[k].w;
        x[k] = k == 0 ? d3(0.0, 0.0, 0.0) : min_image(xyz(pos[i + k]) - o, S);
    }
    const D3 r0 = x[0] - x[1], r1 = x[0] - x[2], r2 = x[1] - x[2];
    const D3 w0 = u[0] - u[1], w1 = u[0] - u[2], w2 = u[1] - u[2];
    const double m00 = (im[0] + im[1]) * dot(r0, r0), m01 = im[0] * dot(r0, r1), m02 = -im[1] * dot(r0, r2);
    const double m10 = m01, m11 = (im[0] + im[2]) * dot(r1, r1), m12 = im[2] * dot(r1, r2);
    const double m20 = m02, m21 = m12, m22 = (im[1] + im[2]) * dot(r2, r2);
    const double b0 = -dot(r0, w0), b1 = -dot(r1, w1), b2 = -dot(r2, w2);
    // Cramer's rule
    const double det = m00 * (m11 * m22 - m12 * m21) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
    const double id = 1.0 / det;
    const double mu0 = id * (b0 * (m11 * m22 - m12 * m21) - m01 * (b1 * m22 - m12 * b2) + m02 * (b1 * m21 - m11 * b2));
    const double mu1 = id * (m00 * (b1 * m22 - m12 * b2) - b0 * (m10 * m22 - m12 * m20) + m02 * (m10 * b2 - b1 * m20));
    const double mu2 = id * (m00 * (m11 * b2 - b1 * m21) - m01 * (m10 * b2 - b1 * m20) + b0 * (m10 * m21 - m11 * m20));
    const D3 d[3] = {im[0] * (mu0 * r0 + mu1 * r1), im[1] * (mu2 * r2 - mu0 * r0), -im[2] * (mu1 * r1 + mu2 * r2)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        T4 ve = v[k];
        ve.x = u[k].x + d[k].x;
        ve.y = u[k].y + d[k].y;
        ve.z = u[k].z + d[k].z;
        vel[i + k] = ve;
    }
}

cudaError_t launch_settle1(const int4* items, int n_items, const SysDev* sys, void* pos, void* vel,
                           const void* force, double dt, const double2* geo, bool f64, cudaStream_t st) {
    if (n_items == 0) return cudaSuccess;
    if (f64)
        k_settle1<double4><<<n_items, SETTLE_CHUNK, 0, st>>>(items, sys, (double4*)pos, (double4*)vel,
                                                             (const double4*)force, dt, geo);
    else
        k_settle1<float4><<<n_items, SETTLE_CHUNK, 0, st>>>(items, sys, (float4*)pos, (float4*)vel,
                                                            (const float4*)force, dt, geo);
    return cudaGetLastError();
}

cudaError_t launch_settle2(const int4* items, int n_items, const SysDev* sys, const void* pos, void* vel, bool f64,
                           cudaStream_t st) {
    if (n_items == 0) return cudaSuccess;
    if (f64)
        k_settle2<double4><<<n_items, SETTLE_CHUNK, 0, st>>>(items, sys, (const double4*)pos, (double4*)vel);
    else
        k_settle2<float4><<<n_items, SETTLE_CHUNK, 0, st>>>(items, sys, (const float4*)pos, (float4*)vel);
    return cudaGetLastError();
}

}  // namespace espb
