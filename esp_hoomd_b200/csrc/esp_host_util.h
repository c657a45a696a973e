// Host-side helpers shared by the batch planner (esp_host.cu) and the
// request server (esp_server.cu): error reporting into esp_last_error(),
// device allocation bookkeeping, the parameter rules of the planner, and the
// construction of parameter sets and influence tables.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "esp_b200.h"
#include "esp_kernels.h"
#include "esp_tables.h"

namespace espb {

// Records `msg` as this thread's last error and returns `code`.
int fail(int code, const std::string& msg);

#define ESPB_CK(x)                                                                                             \
    do {                                                                                                       \
        cudaError_t e_ = (x);                                                                                  \
        if (e_ != cudaSuccess) return ::espb::fail(ESP_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Required k-space resolution kappa_N = pi r_c / h for a relative RMS force
// target (measured against FP64 Ewald on rock-salt lattices, P = 8..12).
double kappa_required(double target);

// Split bandwidth c for a mesh spacing h: 0.93 kappa_N (kappa_N = pi r_c / h)
// rounded to 0.5 and clamped to [2, 60].
double split_c_for_spacing(double rcut, double h);

// Radix stages (4 bits each) of an n-point FFT; 0 if n is not 2/3/5-smooth
// or needs more than 8 stages.
uint32_t radix_plan(int n);

// (PX, PP) pitches of the interpolation tile (bank spread of the stencil planes).
void choose_pitch(int P, int E, int& PX, int& PP);

// cudaMalloc'd arrays released together.
struct DevAlloc {
    std::vector<void*> ptrs;
    long long bytes = 0;
    template <class T>
    int get(T*& p, size_t n) {
        p = nullptr;
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc((void**)&p, n * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(ESP_ERR_ALLOC, std::string("cudaMalloc of ") + std::to_string(n * sizeof(T)) +
                                           " bytes failed: " + cudaGetErrorString(e));
        }
        ptrs.push_back(p);
        bytes += (long long)(n * sizeof(T));
        return 0;
    }
    void release() {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
        bytes = 0;
    }
    ~DevAlloc() { release(); }
};

// Host tables of one parameter set (split + window).
struct PsetHost {
    Split split;
    Window win;
    double rcut = 0;
};

// Builds the split (bandwidth c) and window (P, c_w, degree D) tables and
// the device parameter block for cutoff rcut. Returns 0 or an ESP_ERR_* code.
int build_param_set(double c, double cw, int P, int D, double rcut, PsetHost& h, ParamSet& d, double tol = 1e-8);

// TMA box of the interpolation tile (extended region E): x extent BX >= E +
// 3 with BX = 4 (mod 8) and rows BY >= E odd, so that the staged region's
// plane pitch BX * BY is 4 x odd (mod 32) and the 8 stencil planes a particle
// group reads fall in 8 distinct banks.
void interp_box(int E, int& BX, int& BY);

// Tensor map (CUtensorMap, 128 bytes) of a system's halo-padded potential
// mesh for TMA boxes of BX x BY x BZ floats; false when the driver entry
// point is unavailable or the encoding fails.
bool encode_phi_map(void* map, float* base, int nxp, int nyp, int nzp, int BX, int BY, int BZ);

// Inputs of the influence kernel for system S: the window's Fourier
// transform per axis (w1d, nx + ny + nz values) and the quadrature nodes and
// pre-scaled weights (tq, wq) for Psi(|k| r_c).
void influence_inputs(const SysDev& S, const PsetHost& h, double Lx, double Ly, double Lz, double rcut,
                      std::vector<double>& w1d, std::vector<double>& tq, std::vector<double>& wq);

}  // namespace espb
