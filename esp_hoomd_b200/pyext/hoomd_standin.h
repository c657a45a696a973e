// A minimal stand-in for the HOOMD-blue classes the ESP plugin is written
// against -- SystemDefinition, ParticleData, ParticleGroup, ForceCompute and
// md::NeighborList -- with their member names and the ForceCompute output
// contract (m_force: Scalar4 per particle, force and per-particle energy;
// m_virial: 6 x pitch per-particle virial; m_external_energy,
// m_external_virial: terms no particle owns). HOOMD-blue itself is not
// installed here; these classes let the `_esp` module be compiled and tested
// against the interface HOOMD's headers declare. Scalar is float (HOOMD's
// single-precision build); device arrays are owned by the objects, or bound
// to memory a caller owns (the standalone Python harness binds its torch
// buffers).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "esp_b200.h"

namespace hoomd {

typedef float Scalar;
typedef float4 Scalar4;

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

inline void esp_check(int rc, const char* what) {
    if (rc != ESP_OK) throw std::runtime_error(std::string(what) + ": " + esp_last_error());
}

// Device array owned by the object, or bound to caller memory.
template <class T>
class DeviceArray {
  public:
    DeviceArray() = default;
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    ~DeviceArray() { release(); }
    void allocate(size_t n) {
        release();
        if (n == 0) n = 1;
        cuda_check(cudaMalloc((void**)&m_ptr, n * sizeof(T)), "cudaMalloc");
        cuda_check(cudaMemset(m_ptr, 0, n * sizeof(T)), "cudaMemset");
        m_n = n;
        m_own = true;
    }
    void bind(T* p, size_t n) {
        release();
        m_ptr = p;
        m_n = n;
        m_own = false;
    }
    void release() {
        if (m_own && m_ptr) cudaFree(m_ptr);
        m_ptr = nullptr;
        m_n = 0;
        m_own = false;
    }
    T* get() const { return m_ptr; }
    size_t size() const { return m_n; }

  private:
    T* m_ptr = nullptr;
    size_t m_n = 0;
    bool m_own = false;
};

// Orthorhombic box (HOOMD's BoxDim without tilt).
struct BoxDim {
    double L[3] = {1.0, 1.0, 1.0};
    BoxDim() = default;
    BoxDim(double Lx, double Ly, double Lz) : L{Lx, Ly, Lz} {}
};

class ParticleData {
  public:
    ParticleData(unsigned int N, const BoxDim& box) : m_N(N), m_box(box) {
        m_pos.allocate(N);
        m_charge.allocate(N);
    }
    unsigned int getN() const { return m_N; }
    const BoxDim& getBox() const { return m_box; }
    void setGlobalBox(const BoxDim& box) { m_box = box; }
    const Scalar4* getPositions() const { return m_pos.get(); }
    const Scalar* getCharges() const { return m_charge.get(); }
    // host upload: xyzw (4 floats per particle; w = type) and charges
    void setPositions(const float* xyzw) {
        cuda_check(cudaMemcpy(m_pos.get(), xyzw, (size_t)m_N * sizeof(Scalar4), cudaMemcpyHostToDevice),
                   "positions upload");
    }
    void setCharges(const float* q) {
        cuda_check(cudaMemcpy(m_charge.get(), q, (size_t)m_N * sizeof(Scalar), cudaMemcpyHostToDevice),
                   "charges upload");
    }
    // bind caller-owned device arrays (N float4, N floats)
    void bindPositions(uintptr_t p) { m_pos.bind(reinterpret_cast<Scalar4*>(p), m_N); }
    void bindCharges(uintptr_t p) { m_charge.bind(reinterpret_cast<Scalar*>(p), m_N); }

  private:
    unsigned int m_N;
    BoxDim m_box;
    DeviceArray<Scalar4> m_pos;
    DeviceArray<Scalar> m_charge;
};

class SystemDefinition {
  public:
    explicit SystemDefinition(std::shared_ptr<ParticleData> pdata) : m_pdata(std::move(pdata)) {}
    std::shared_ptr<ParticleData> getParticleData() const { return m_pdata; }

  private:
    std::shared_ptr<ParticleData> m_pdata;
};

// All particles (the ESP force applies to the whole system).
class ParticleGroup {
  public:
    explicit ParticleGroup(std::shared_ptr<SystemDefinition> sysdef) : m_sysdef(std::move(sysdef)) {}
    unsigned int getNumMembers() const { return m_sysdef->getParticleData()->getN(); }

  private:
    std::shared_ptr<SystemDefinition> m_sysdef;
};

class ForceCompute {
  public:
    explicit ForceCompute(std::shared_ptr<SystemDefinition> sysdef)
        : m_sysdef(std::move(sysdef)), m_pdata(m_sysdef->getParticleData()) {
        const unsigned int N = m_pdata->getN();
        m_virial_pitch = (N + 31u) & ~31u;  // rows padded as HOOMD's GPUArray pitch
        m_force.allocate(N);
        m_virial.allocate((size_t)6 * m_virial_pitch);
    }
    virtual ~ForceCompute() = default;
    virtual void compute(uint64_t timestep) = 0;

    unsigned int getN() const { return m_pdata->getN(); }
    unsigned int getVirialPitch() const { return m_virial_pitch; }
    const Scalar4* getForceArray() const { return m_force.get(); }
    const Scalar* getVirialArray() const { return m_virial.get(); }
    Scalar getExternalEnergy() const { return (Scalar)m_external_energy; }
    double getExternalEnergyD() const { return m_external_energy; }
    std::vector<double> getExternalVirial() const { return std::vector<double>(m_external_virial, m_external_virial + 6); }

    // host copies of the outputs
    std::vector<float> forcesHost() const {
        std::vector<float> h((size_t)4 * m_pdata->getN());
        cuda_check(cudaMemcpy(h.data(), m_force.get(), h.size() * sizeof(float), cudaMemcpyDeviceToHost), "forces");
        return h;
    }
    std::vector<float> virialsHost() const {
        std::vector<float> h((size_t)6 * m_virial_pitch);
        cuda_check(cudaMemcpy(h.data(), m_virial.get(), h.size() * sizeof(float), cudaMemcpyDeviceToHost), "virials");
        return h;
    }
    // total potential energy: per-particle energies + external (HOOMD's calcEnergySum)
    double calcEnergySum() const {
        const std::vector<float> f = forcesHost();
        double e = m_external_energy;
        for (size_t i = 0; i < f.size(); i += 4) e += f[i + 3];
        return e;
    }
    // redirect the outputs into caller-owned device arrays
    void bindOutputs(uintptr_t force, uintptr_t virial, unsigned int pitch) {
        if (pitch < m_pdata->getN()) throw std::invalid_argument("virial pitch below the particle count");
        m_force.bind(reinterpret_cast<Scalar4*>(force), m_pdata->getN());
        m_virial.bind(reinterpret_cast<Scalar*>(virial), (size_t)6 * pitch);
        m_virial_pitch = pitch;
    }

  protected:
    std::shared_ptr<SystemDefinition> m_sysdef;
    std::shared_ptr<ParticleData> m_pdata;
    DeviceArray<Scalar4> m_force;
    DeviceArray<Scalar> m_virial;
    unsigned int m_virial_pitch = 0;
    double m_external_energy = 0.0;
    double m_external_virial[6] = {0, 0, 0, 0, 0, 0};
};

namespace md {

// Full neighbour list in HOOMD's layout (neighbours of i:
// nlist[head[i] + k], k < n_neigh[i]) of all pairs within r_cut + r_buff.
// compute() builds it on the GPU (cell list of the ESP library's MD
// harness); bindLists() uses lists built elsewhere instead.
class NeighborList {
  public:
    NeighborList(std::shared_ptr<SystemDefinition> sysdef, Scalar r_buff)
        : m_sysdef(std::move(sysdef)), m_r_buff(r_buff) {}
    ~NeighborList() {
        if (m_batch) esp_batch_destroy(m_batch);
    }
    void setRCutPair(Scalar r_cut) { m_r_cut = std::max(m_r_cut, (double)r_cut); }
    Scalar getMaxRCut() const { return (Scalar)m_r_cut; }
    Scalar getRBuff() const { return (Scalar)m_r_buff; }
    void compute(uint64_t /*timestep*/) {
        if (m_bound) return;
        const auto pdata = m_sysdef->getParticleData();
        const int N = (int)pdata->getN();
        const BoxDim& box = pdata->getBox();
        if (!m_batch) {
            esp_params p;
            esp_check(esp_params_default(&p), "esp_params_default");
            p.rcut = std::max(m_r_cut, 1e-3);
            const double L[3] = {box.L[0], box.L[1], box.L[2]};
            esp_check(esp_batch_create(&p, 1, &N, L, nullptr, &m_batch), "neighbour-list harness");
            m_head.allocate(N);
            m_nn.allocate(N);
        }
        for (;;) {
            if (m_nl.size() < (size_t)N * m_cap) m_nl.allocate((size_t)N * m_cap);
            int rc = esp_batch_build_nlist(m_batch, nullptr, &pdata->getPositions()->x, m_r_cut + m_r_buff, m_cap,
                                           m_head.get(), m_nn.get(), m_nl.get());
            int need = 0;
            if (rc == ESP_OK) rc = esp_batch_nlist_check(m_batch, &need);  // waits for the build
            if (rc == ESP_ERR_OVERFLOW && m_cap < 65536) {
                while (m_cap < need && m_cap < 65536) m_cap *= 2;  // HOOMD grows its list the same way
                continue;
            }
            esp_check(rc, "neighbour-list build");
            break;
        }
    }
    const unsigned int* getHeadList() const { return m_head.get(); }
    const unsigned int* getNNeighArray() const { return m_nn.get(); }
    const unsigned int* getNListArray() const { return m_nl.get(); }
    void bindLists(uintptr_t head, uintptr_t n_neigh, uintptr_t nlist) {
        const unsigned int N = m_sysdef->getParticleData()->getN();
        m_head.bind(reinterpret_cast<unsigned int*>(head), N);
        m_nn.bind(reinterpret_cast<unsigned int*>(n_neigh), N);
        m_nl.bind(reinterpret_cast<unsigned int*>(nlist), 0);
        m_bound = true;
    }

  private:
    std::shared_ptr<SystemDefinition> m_sysdef;
    double m_r_cut = 0.0, m_r_buff = 0.0;
    int m_cap = 256;
    bool m_bound = false;
    esp_batch* m_batch = nullptr;
    DeviceArray<unsigned int> m_head, m_nn, m_nl;
};

}  // namespace md
}  // namespace hoomd
