// The 27-cell neighbourhood of a cell list, used by the neighbour-list
// builder (esp_md.cu: HOOMD-layout rows and the library's pair list), which
// enumerates the surrounding cells' particles in a fixed order: surrounding
// cell t = (iz * 3 + iy) * 3 + ix in that order, and inside each cell the
// cell-sorted slots in ascending order (so every row is deterministic).
#pragma once

#include "esp_common.cuh"
#include "esp_md.h"

namespace espb {

struct CellNbhd {
    uint32_t src[27];       // first cell-sorted slot of each surrounding cell
    uint32_t off[28];       // exclusive prefix of their counts (off[27] = total)
    float shift[27][3];     // periodic image of each surrounding cell (0 with minimg)
    int minimg;             // fewer than 3 cells on an axis: staged without shifts
};

// Fills `nb` for cell `cidx` (the global cell index, local index lc inside
// its system). Call from the whole first warp; the caller synchronises.
// With fewer than 3 cells on an axis the -1/+1 neighbours coincide, so only
// the distinct ones ({0, 1} for 2 cells, {0} for 1) are visited and no
// shifts are applied (the minimum-image test applies instead).
__device__ __forceinline__ void cell_nbhd_warp(int lc, const CellDev& C, const SysDev& S,
                                               const uint32_t* __restrict__ cstart, CellNbhd& nb) {
    const int lane = threadIdx.x & 31;
    const int cx = lc % C.ncx, cy = (lc / C.ncx) % C.ncy, cz = lc / (C.ncx * C.ncy);
    const bool minimg = C.ncx < 3 || C.ncy < 3 || C.ncz < 3;
    uint32_t n = 0;
    if (lane < 27) {
        const int ix = lane % 3, iy = (lane / 3) % 3, iz = lane / 9;
        const int dx = (C.ncx >= 3 ? -1 : 0) + ix, dy = (C.ncy >= 3 ? -1 : 0) + iy, dz = (C.ncz >= 3 ? -1 : 0) + iz;
        const bool ok = dx <= (C.ncx >= 3 ? 1 : C.ncx - 1) && dy <= (C.ncy >= 3 ? 1 : C.ncy - 1) &&
                        dz <= (C.ncz >= 3 ? 1 : C.ncz - 1);
        int xx = cx + dx, yy = cy + dy, zz = cz + dz;
        float sx = 0.f, sy = 0.f, sz = 0.f;
        if (xx < 0) { xx += C.ncx; sx = -S.Lx; } else if (xx >= C.ncx) { xx -= C.ncx; sx = S.Lx; }
        if (yy < 0) { yy += C.ncy; sy = -S.Ly; } else if (yy >= C.ncy) { yy -= C.ncy; sy = S.Ly; }
        if (zz < 0) { zz += C.ncz; sz = -S.Lz; } else if (zz >= C.ncz) { zz -= C.ncz; sz = S.Lz; }
        uint32_t b = 0;
        if (ok) {
            const uint32_t c = (uint32_t)(C.c_off + (zz * C.ncy + yy) * C.ncx + xx);
            b = cstart[c];
            n = cstart[c + 1] - b;
        }
        nb.src[lane] = b;
        nb.shift[lane][0] = minimg ? 0.f : sx;
        nb.shift[lane][1] = minimg ? 0.f : sy;
        nb.shift[lane][2] = minimg ? 0.f : sz;
    }
    uint32_t inc = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane < 27) nb.off[lane] = inc - n;
    if (lane == 26) nb.off[27] = inc;
    if (lane == 0) nb.minimg = minimg ? 1 : 0;
}

}  // namespace espb
