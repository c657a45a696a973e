// Pair arithmetic of the short-range term (k_pair, esp_kernels.cu): per pair
//   pair_eng   = qiqj/(4 pi) (1/r - Q(u)/r_c),  u = r^2/r_c^2
//   force_divr = qiqj/(4 pi) (1/r^3 + 2 Q'(u)/r_c^3)
// (the split form of EvaluatorPairPSWF::evalForceAndEnergy,
// src/EvaluatorPairPSWF.h:274-295), Q and Q' as Horner series in v = 2u - 1
// with the coefficients in the kernel-parameter constant bank.
#pragma once

#include "esp_common.cuh"
#include "esp_kernels.h"

namespace espb {

template <int NQ, bool VIR, bool EN>
struct PairEval {
    const PairCoef& pc;  // the kernel parameter: constant-bank operands
    float rc2, irc2, irc, tirc3, Lx, Ly, Lz, iLx, iLy, iLz;
    float fx = 0.f, fy = 0.f, fz = 0.f, en = 0.f;
    float vxx = 0.f, vxy = 0.f, vxz = 0.f, vyy = 0.f, vyz = 0.f, vzz = 0.f;
    // QS: pi.w already holds q_i / (4 pi)
    template <bool WRAP = true, bool QS = false>
    __device__ __forceinline__ void pair(const float4& pi, const float4& pj) {
        float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        if (WRAP) {
            dx -= Lx * rintf(dx * iLx);
            dy -= Ly * rintf(dy * iLy);
            dz -= Lz * rintf(dz * iLz);
        }
        const float r2x = dx * dx + dy * dy + dz * dz;
        const bool in = r2x < rc2 && r2x > 0.f;
        const float r2 = in ? r2x : rc2;
        {
            const float ri = rsqrtf(r2);  // hardware estimate, a few ulp
            const float v = fmaf(2.f * irc2, r2, -1.f);
            float dq = pc.d[NQ - 2];
#pragma unroll
            for (int c = NQ - 3; c >= 0; --c) dq = fmaf(dq, v, pc.d[c]);
            const float qq = in ? (QS ? pi.w * pj.w : pi.w * pj.w * INV_4PI_F) : 0.f;
            const float fdr = qq * fmaf(tirc3, dq, ri * ri * ri);
            if (EN) {
                float qv = pc.q[NQ - 1];
#pragma unroll
                for (int c = NQ - 2; c >= 0; --c) qv = fmaf(qv, v, pc.q[c]);
                en = fmaf(qq, ri - qv * irc, en);
            }
            fx = fmaf(fdr, dx, fx);
            fy = fmaf(fdr, dy, fy);
            fz = fmaf(fdr, dz, fz);
            if (VIR) {
                vxx = fmaf(fdr * dx, dx, vxx);
                vxy = fmaf(fdr * dx, dy, vxy);
                vxz = fmaf(fdr * dx, dz, vxz);
                vyy = fmaf(fdr * dy, dy, vyy);
                vyz = fmaf(fdr * dy, dz, vyz);
                vzz = fmaf(fdr * dz, dz, vzz);
            }
        }
    }
};

}  // namespace espb
