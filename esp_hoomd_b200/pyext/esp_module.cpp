// The `_esp` extension module: the reference plugin's C++ classes with its
// Python-facing names and signatures (src/module.cc:57-85,
// src/ESPForceCompute.cc:411-509, src/ESPForceComputeGPU.cc:457-481), over
// the sm_100a library's C ABI (include/esp_b200.h):
//
//   ESPForceCompute(sysdef, nlist, group)   long-range part (mesh, self,
//       background): setParams(nx, ny, nz, order, kappa, rcut, alpha=0,
//       n_table), getResolution/getOrder/getKappa/getRCut/getAlpha/getQSum/
//       getQ2Sum/getTableSize/getTablePtr/getTableEntry, table, invalidate,
//       compute(timestep);
//   ESPForceComputeGPU                       the same class (every stage
//       runs on the GPU; the reference's CPU stages were stubs);
//   PotentialPairPSWF / PotentialPairPSWFGPU the short-range complement,
//       PotentialPair<EvaluatorPairPSWF>: setParams(type_i, type_j,
//       {"kappa", "alpha", "rcut", "V_cut"}) (src/EvaluatorPairPSWF.h:180-225);
//   ESPTableEntry                            one segment of the
//       introspection table (degree-4 Horner coefficients of L(r) and
//       -dL/dr with 1/(4 pi r) folded in, src/ESPForceCompute.h:69-83).
//
// Both forces fill the ForceCompute arrays as HOOMD's integrators read them
// (esp_compute_hoomd): m_force, the per-particle m_virial, and
// m_external_energy / m_external_virial for the terms no particle owns.
// HOOMD-blue is not installed here, so the module is compiled against
// hoomd_standin.h, whose classes it also exports for tests and for the
// standalone harness.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <map>
#include <sstream>

#include "esp_tables.h"
#include "hoomd_standin.h"

namespace py = pybind11;

namespace hoomd {
namespace md {

constexpr unsigned int ESP_TABLE_SEGMENTS = 512;  // the Python API's default (src/esp.py:94)

struct ESPTableEntry {
    double potential_coeffs[5];  // L(r) = sum_j c_j t^j, t = (r - r_lo) dr_inv
    double force_coeffs[5];      // -dL/dr
    double r_lo = 0.0, dr_inv = 0.0;
};

// Degree-4 interpolants of L and -dL/dr of the split at the Chebyshev points
// of each of n segments of [0, r_c].
static std::vector<ESPTableEntry> build_table(double c, double rcut, unsigned int n) {
    espb::Split sp;
    sp.build(c, 1e-12);
    std::vector<ESPTableEntry> tab(n);
    const double w = rcut / n;
    double tn[5], V[5][5], Vi[5][5];
    for (int j = 0; j < 5; ++j) tn[j] = 0.5 - 0.5 * std::cos(M_PI * (j + 0.5) / 5.0);
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) V[i][j] = std::pow(tn[i], j);
    // invert the 5x5 Vandermonde matrix (Gauss-Jordan)
    double A[5][10];
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 10; ++j) A[i][j] = j < 5 ? V[i][j] : (j - 5 == i ? 1.0 : 0.0);
    for (int k = 0; k < 5; ++k) {
        int p = k;
        for (int i = k + 1; i < 5; ++i)
            if (std::fabs(A[i][k]) > std::fabs(A[p][k])) p = i;
        for (int j = 0; j < 10; ++j) std::swap(A[k][j], A[p][j]);
        const double d = A[k][k];
        for (int j = 0; j < 10; ++j) A[k][j] /= d;
        for (int i = 0; i < 5; ++i)
            if (i != k) {
                const double f = A[i][k];
                for (int j = 0; j < 10; ++j) A[i][j] -= f * A[k][j];
            }
    }
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) Vi[i][j] = A[i][j + 5];
    const double inv4pi = 0.079577471545947673;
    for (unsigned int s = 0; s < n; ++s) {
        double L[5], D[5];
        for (int j = 0; j < 5; ++j) {
            const double r = (s + tn[j]) * w, u = r * r / (rcut * rcut);
            L[j] = inv4pi * (1.0 / r - sp.Q(u) / rcut);
            D[j] = inv4pi * r * (1.0 / (r * r * r) + 2.0 * sp.dQdu(u) / (rcut * rcut * rcut));
        }
        ESPTableEntry& e = tab[s];
        for (int i = 0; i < 5; ++i) {
            e.potential_coeffs[i] = 0.0;
            e.force_coeffs[i] = 0.0;
            for (int j = 0; j < 5; ++j) {
                e.potential_coeffs[i] += Vi[i][j] * L[j];
                e.force_coeffs[i] += Vi[i][j] * D[j];
            }
        }
        e.r_lo = s * w;
        e.dr_inv = 1.0 / w;
    }
    return tab;
}

// One esp_ctx in the FP32 ForceCompute contract; re-planned when the
// parameters or the box change.
class EspContext {
  public:
    ~EspContext() { reset(); }
    void reset() {
        if (m_ctx) esp_destroy(m_ctx);
        m_ctx = nullptr;
        if (m_ext) cudaFree(m_ext);
        m_ext = nullptr;
    }
    esp_ctx* get(const esp_params& p, const BoxDim& box, int N) {
        if (!m_ctx) {
            esp_check(esp_create(&p, box.L[0], box.L[1], box.L[2], N, &m_ctx), "esp_create");
            cuda_check(cudaMalloc((void**)&m_ext, 7 * sizeof(double)), "cudaMalloc");
        }
        return m_ctx;
    }
    // one evaluation of `flags` into the ForceCompute arrays; returns the
    // external terms {E, W xx..zz}
    std::vector<double> compute(const esp_params& p, const ParticleData& pd, Scalar4* force, Scalar* virial,
                                unsigned int pitch, const md::NeighborList* nl, int flags) {
        esp_ctx* c = get(p, pd.getBox(), (int)pd.getN());
        esp_check(esp_compute_hoomd(c, nullptr, &pd.getPositions()->x, pd.getCharges(), (int)pd.getN(),
                                    nl ? nl->getHeadList() : nullptr, nl ? nl->getNNeighArray() : nullptr,
                                    nl ? nl->getNListArray() : nullptr, &force->x, virial, (int)pitch, m_ext,
                                    flags),
                  "esp_compute_hoomd");
        std::vector<double> ext(7);
        cuda_check(cudaMemcpy(ext.data(), m_ext, 7 * sizeof(double), cudaMemcpyDeviceToHost), "external terms");
        return ext;
    }
    esp_info info() const {
        esp_info i{};
        if (m_ctx) esp_check(esp_get_info(m_ctx, &i), "esp_get_info");
        return i;
    }
    bool ready() const { return m_ctx != nullptr; }

  private:
    esp_ctx* m_ctx = nullptr;
    double* m_ext = nullptr;
};

class ESPForceCompute : public ForceCompute {
  public:
    ESPForceCompute(std::shared_ptr<SystemDefinition> sysdef, std::shared_ptr<NeighborList> nlist,
                    std::shared_ptr<ParticleGroup> group)
        : ForceCompute(std::move(sysdef)), m_nlist(std::move(nlist)), m_group(std::move(group)) {}

    // ESPForceCompute::setParams (src/ESPForceCompute.cc:71-89). kappa is
    // the split bandwidth in 1/length (prolate c = kappa * rcut; 0 = chosen
    // from the mesh spacing); alpha (Debye screening) must be 0.
    void setParams(unsigned int nx, unsigned int ny, unsigned int nz, unsigned int order, Scalar kappa, Scalar rcut,
                   Scalar alpha, unsigned int n_table) {
        if (nx == 0 || ny == 0 || nz == 0) throw std::invalid_argument("ESP: mesh dimensions must be positive");
        if (order < 2 || order > 12) throw std::invalid_argument("ESP: order must be in [2, 12]");
        if (!(rcut > 0)) throw std::invalid_argument("ESP: rcut must be positive");
        if (kappa < 0) throw std::invalid_argument("ESP: kappa must be >= 0");
        if (alpha != 0) throw std::invalid_argument("ESP: Debye screening (alpha != 0) is not supported");
        if (n_table < 16) throw std::invalid_argument("ESP: n_table must be >= 16");
        m_dim[0] = nx;
        m_dim[1] = ny;
        m_dim[2] = nz;
        m_order = order;
        m_kappa = kappa;
        m_rcut = rcut;
        m_alpha = alpha;
        m_n_table = n_table;
        m_params_set = true;
        invalidate();
        m_nlist->setRCutPair(rcut);
    }
    std::vector<unsigned int> getResolution() const { return {m_dim[0], m_dim[1], m_dim[2]}; }
    unsigned int getOrder() const { return m_order; }
    // the split bandwidth in use (c / rcut) once planned, else the requested one
    Scalar getKappa() const {
        if (m_ctx.ready()) {
            const esp_info i = m_ctx.info();
            return (Scalar)(i.c_split / i.rcut);
        }
        return m_kappa;
    }
    Scalar getRCut() const { return m_rcut; }
    Scalar getAlpha() const { return m_alpha; }
    Scalar getQSum() const { return (Scalar)m_q; }
    Scalar getQ2Sum() const { return (Scalar)m_q2; }
    unsigned int getTableSize() const { return m_n_table; }
    uintptr_t getTablePtr() const { return reinterpret_cast<uintptr_t>(m_table.data()); }
    const std::vector<ESPTableEntry>& getTable() const { return m_table; }
    ESPTableEntry getTableEntry(unsigned int i) const {
        if (i >= m_table.size()) throw std::out_of_range("ESP: table index out of range");
        return m_table[i];
    }
    void invalidate() { m_need_initialize = true; }

    void compute(uint64_t timestep) override {
        if (!m_params_set) throw std::runtime_error("ESP: setParams() must be called before compute()");
        if (m_need_initialize) initialize();
        (void)timestep;
        const std::vector<double> ext =
            m_ctx.compute(params(), *m_pdata, const_cast<Scalar4*>(getForceArray()),
                          const_cast<Scalar*>(getVirialArray()), m_virial_pitch, nullptr, ESP_LONG_RANGE);
        m_external_energy = ext[0];
        for (int k = 0; k < 6; ++k) m_external_virial[k] = ext[1 + k];
    }

  protected:
    esp_params params() const {
        esp_params p;
        esp_check(esp_params_default(&p), "esp_params_default");
        p.nx = (int)m_dim[0];
        p.ny = (int)m_dim[1];
        p.nz = (int)m_dim[2];
        p.order = (int)m_order;
        p.kappa = m_kappa;
        p.rcut = m_rcut;
        p.alpha = m_alpha;
        p.n_table = (int)m_n_table;
        return p;
    }
    void initialize() {
        m_ctx.reset();
        m_ctx.get(params(), m_pdata->getBox(), (int)m_pdata->getN());
        std::vector<float> q(m_pdata->getN());
        cuda_check(cudaMemcpy(q.data(), m_pdata->getCharges(), q.size() * sizeof(float), cudaMemcpyDeviceToHost),
                   "charges");
        m_q = m_q2 = 0.0;
        for (float v : q) {
            m_q += v;
            m_q2 += (double)v * v;
        }
        const esp_info i = m_ctx.info();
        m_table = build_table(i.c_split, m_rcut, m_n_table);
        m_need_initialize = false;
    }

    std::shared_ptr<NeighborList> m_nlist;
    std::shared_ptr<ParticleGroup> m_group;
    unsigned int m_dim[3] = {32, 32, 32};
    unsigned int m_order = 6, m_n_table = ESP_TABLE_SEGMENTS;
    Scalar m_kappa = 0, m_rcut = 0, m_alpha = 0;
    double m_q = 0, m_q2 = 0;
    bool m_params_set = false, m_need_initialize = true;
    std::vector<ESPTableEntry> m_table;
    EspContext m_ctx;
};

// The GPU class of the reference (every stage of this library runs on the GPU).
class ESPForceComputeGPU : public ESPForceCompute {
  public:
    using ESPForceCompute::ESPForceCompute;
};

// PotentialPair<EvaluatorPairPSWF>: the short-range term over the neighbour
// list with the split of (kappa, rcut); one parameter set (the evaluator
// does not depend on the particle types).
class PotentialPairPSWF : public ForceCompute {
  public:
    PotentialPairPSWF(std::shared_ptr<SystemDefinition> sysdef, std::shared_ptr<NeighborList> nlist)
        : ForceCompute(std::move(sysdef)), m_nlist(std::move(nlist)) {}
    void setParams(const std::string& a, const std::string& b, py::dict v) {
        Param p;
        p.rcut = v.contains("rcut") ? v["rcut"].cast<double>() : 0.0;
        p.kappa = v.contains("kappa") ? v["kappa"].cast<double>() : 0.0;
        p.alpha = v.contains("alpha") ? v["alpha"].cast<double>() : 0.0;
        p.V_cut = v.contains("V_cut") ? v["V_cut"].cast<double>() : 0.0;
        if (!(p.rcut > 0)) throw std::invalid_argument("ESP: pair parameter 'rcut' must be positive");
        if (p.alpha != 0) throw std::invalid_argument("ESP: Debye screening (alpha != 0) is not supported");
        if (p.V_cut != 0) throw std::invalid_argument("ESP: the split energy vanishes at r_c; V_cut must be 0");
        const std::string k = key(a, b);
        for (const auto& kv : m_params)
            if (kv.first != k && (kv.second.rcut != p.rcut || kv.second.kappa != p.kappa))
                throw std::invalid_argument("ESP: every type pair shares one split (kappa, rcut)");
        m_params[k] = p;
        m_nlist->setRCutPair((Scalar)p.rcut);
        m_ctx.reset();
    }
    py::dict getParams(const std::string& a, const std::string& b) const {
        auto it = m_params.find(key(a, b));
        if (it == m_params.end()) throw std::out_of_range("ESP: no parameters for this type pair");
        py::dict v;
        v["kappa"] = it->second.kappa;
        v["alpha"] = it->second.alpha;
        v["rcut"] = it->second.rcut;
        v["V_cut"] = it->second.V_cut;
        return v;
    }
    void compute(uint64_t timestep) override {
        if (m_params.empty()) throw std::runtime_error("ESP: pair parameters must be set before compute()");
        m_nlist->compute(timestep);
        const Param& p = m_params.begin()->second;
        esp_params e;
        esp_check(esp_params_default(&e), "esp_params_default");
        e.rcut = p.rcut;
        e.kappa = p.kappa;
        const std::vector<double> ext =
            m_ctx.compute(e, *m_pdata, const_cast<Scalar4*>(getForceArray()), const_cast<Scalar*>(getVirialArray()),
                          m_virial_pitch, m_nlist.get(), ESP_SHORT_RANGE);
        m_external_energy = ext[0];
        for (int k = 0; k < 6; ++k) m_external_virial[k] = ext[1 + k];
    }

  private:
    struct Param {
        double kappa = 0, alpha = 0, rcut = 0, V_cut = 0;
    };
    static std::string key(const std::string& a, const std::string& b) { return a < b ? a + "|" + b : b + "|" + a; }
    std::shared_ptr<NeighborList> m_nlist;
    std::map<std::string, Param> m_params;
    EspContext m_ctx;
};

class PotentialPairPSWFGPU : public PotentialPairPSWF {
  public:
    using PotentialPairPSWF::PotentialPairPSWF;
};

}  // namespace md
}  // namespace hoomd

using namespace hoomd;
using namespace hoomd::md;

// numpy views of the ForceCompute outputs: forces [N, 4], virials [6, N]
static py::array_t<float> forces_np(const ForceCompute& f) {
    const std::vector<float> h = f.forcesHost();
    py::array_t<float> a({(py::ssize_t)(h.size() / 4), (py::ssize_t)4});
    std::memcpy(a.mutable_data(), h.data(), h.size() * sizeof(float));
    return a;
}

static py::array_t<float> virials_np(const ForceCompute& f, unsigned int N) {
    const std::vector<float> h = f.virialsHost();
    const unsigned int pitch = f.getVirialPitch();
    py::array_t<float> a({(py::ssize_t)6, (py::ssize_t)N});
    for (int k = 0; k < 6; ++k) std::memcpy(a.mutable_data(k, 0), h.data() + (size_t)k * pitch, N * sizeof(float));
    return a;
}

PYBIND11_MODULE(_esp, m) {
    m.doc() = "ESP (Ewald summation with prolates) electrostatics on sm_100a: long-range mesh force and the "
              "matching short-range pair term, with the reference plugin's class names and signatures.";

    // ---- HOOMD stand-in classes (hoomd._hoomd in a HOOMD build)
    py::class_<BoxDim>(m, "BoxDim").def(py::init<double, double, double>()).def_property_readonly(
        "L", [](const BoxDim& b) { return py::make_tuple(b.L[0], b.L[1], b.L[2]); });
    py::class_<ParticleData, std::shared_ptr<ParticleData>>(m, "ParticleData")
        .def(py::init<unsigned int, const BoxDim&>(), py::arg("N"), py::arg("box"))
        .def("getN", &ParticleData::getN)
        .def("setPositions",
             [](ParticleData& pd, py::array_t<float, py::array::c_style | py::array::forcecast> xyzw) {
                 if (xyzw.ndim() != 2 || xyzw.shape(0) != pd.getN() || xyzw.shape(1) != 4)
                     throw std::invalid_argument("positions: float array [N, 4] expected");
                 pd.setPositions(xyzw.data());
             })
        .def("setCharges",
             [](ParticleData& pd, py::array_t<float, py::array::c_style | py::array::forcecast> q) {
                 if (q.ndim() != 1 || q.shape(0) != pd.getN())
                     throw std::invalid_argument("charges: float array [N] expected");
                 pd.setCharges(q.data());
             })
        .def("bindPositions", &ParticleData::bindPositions)
        .def("bindCharges", &ParticleData::bindCharges);
    py::class_<SystemDefinition, std::shared_ptr<SystemDefinition>>(m, "SystemDefinition")
        .def(py::init<std::shared_ptr<ParticleData>>())
        .def("getParticleData", &SystemDefinition::getParticleData);
    py::class_<ParticleGroup, std::shared_ptr<ParticleGroup>>(m, "ParticleGroup")
        .def(py::init<std::shared_ptr<SystemDefinition>>())
        .def("getNumMembers", &ParticleGroup::getNumMembers);
    py::class_<NeighborList, std::shared_ptr<NeighborList>>(m, "NeighborList")
        .def(py::init<std::shared_ptr<SystemDefinition>, Scalar>(), py::arg("sysdef"), py::arg("r_buff"))
        .def("setRCutPair", &NeighborList::setRCutPair)
        .def("getMaxRCut", &NeighborList::getMaxRCut)
        .def("compute", &NeighborList::compute)
        .def("bindLists", &NeighborList::bindLists);
    py::class_<ForceCompute, std::shared_ptr<ForceCompute>>(m, "ForceCompute")
        .def("compute", &ForceCompute::compute)
        .def("getForces", [](const ForceCompute& f) { return forces_np(f); })
        .def("getVirials", [](const ForceCompute& f) { return virials_np(f, f.getN()); })
        .def("getVirialPitch", &ForceCompute::getVirialPitch)
        .def("getExternalEnergy", &ForceCompute::getExternalEnergyD)
        .def("getExternalVirial", &ForceCompute::getExternalVirial)
        .def("calcEnergySum", &ForceCompute::calcEnergySum)
        .def("bindOutputs", &ForceCompute::bindOutputs);

    // ---- the plugin's classes (src/ESPForceCompute.cc:411-509)
    py::class_<ESPTableEntry>(m, "ESPTableEntry", "One segment of the ESP short-range introspection table.")
        .def_property_readonly("potential_coeffs",
                               [](const ESPTableEntry& e) {
                                   return py::make_tuple(e.potential_coeffs[0], e.potential_coeffs[1],
                                                         e.potential_coeffs[2], e.potential_coeffs[3]);
                               })
        .def_property_readonly("force_coeffs",
                               [](const ESPTableEntry& e) {
                                   return py::make_tuple(e.force_coeffs[0], e.force_coeffs[1], e.force_coeffs[2],
                                                         e.force_coeffs[3]);
                               })
        .def_property_readonly("potential_coeff4", [](const ESPTableEntry& e) { return e.potential_coeffs[4]; })
        .def_property_readonly("force_coeff4", [](const ESPTableEntry& e) { return e.force_coeffs[4]; })
        .def_property_readonly("r_lo", [](const ESPTableEntry& e) { return e.r_lo; })
        .def_property_readonly("dr_inv", [](const ESPTableEntry& e) { return e.dr_inv; })
        .def("__repr__", [](const ESPTableEntry& e) {
            std::ostringstream o;
            o << "<ESPTableEntry r_lo=" << e.r_lo << " dr_inv=" << e.dr_inv << ">";
            return o.str();
        });
    py::class_<ESPForceCompute, ForceCompute, std::shared_ptr<ESPForceCompute>>(
        m, "ESPForceCompute", "Long-range electrostatics by the ESP mesh method (mesh, self and background terms).")
        .def(py::init<std::shared_ptr<SystemDefinition>, std::shared_ptr<NeighborList>,
                      std::shared_ptr<ParticleGroup>>(),
             py::arg("sysdef"), py::arg("nlist"), py::arg("group"))
        .def("setParams", &ESPForceCompute::setParams, py::arg("nx"), py::arg("ny"), py::arg("nz"),
             py::arg("order"), py::arg("kappa"), py::arg("rcut"), py::arg("alpha") = 0.0f,
             py::arg("n_table") = ESP_TABLE_SEGMENTS)
        .def("getResolution", &ESPForceCompute::getResolution)
        .def("getOrder", &ESPForceCompute::getOrder)
        .def("getKappa", &ESPForceCompute::getKappa)
        .def("getRCut", &ESPForceCompute::getRCut)
        .def("getAlpha", &ESPForceCompute::getAlpha)
        .def("getQSum", &ESPForceCompute::getQSum)
        .def("getQ2Sum", &ESPForceCompute::getQ2Sum)
        .def("getTableSize", &ESPForceCompute::getTableSize)
        .def("getTablePtr", &ESPForceCompute::getTablePtr)
        .def("getTableEntry", &ESPForceCompute::getTableEntry, py::arg("index"))
        .def("invalidate", &ESPForceCompute::invalidate)
        .def("compute", &ESPForceCompute::compute)
        .def_property_readonly("table", &ESPForceCompute::getTable);
    py::class_<ESPForceComputeGPU, ESPForceCompute, std::shared_ptr<ESPForceComputeGPU>>(
        m, "ESPForceComputeGPU", "GPU long-range electrostatics (the same class: every stage runs on the GPU).")
        .def(py::init<std::shared_ptr<SystemDefinition>, std::shared_ptr<NeighborList>,
                      std::shared_ptr<ParticleGroup>>(),
             py::arg("sysdef"), py::arg("nlist"), py::arg("group"));
    py::class_<PotentialPairPSWF, ForceCompute, std::shared_ptr<PotentialPairPSWF>>(
        m, "PotentialPairPSWF", "Short-range ESP pair term, PotentialPair<EvaluatorPairPSWF>.")
        .def(py::init<std::shared_ptr<SystemDefinition>, std::shared_ptr<NeighborList>>(), py::arg("sysdef"),
             py::arg("nlist"))
        .def("setParams", &PotentialPairPSWF::setParams)
        .def("getParams", &PotentialPairPSWF::getParams)
        .def("compute", &PotentialPairPSWF::compute);
    py::class_<PotentialPairPSWFGPU, PotentialPairPSWF, std::shared_ptr<PotentialPairPSWFGPU>>(
        m, "PotentialPairPSWFGPU", "GPU short-range ESP pair term (the same class).")
        .def(py::init<std::shared_ptr<SystemDefinition>, std::shared_ptr<NeighborList>>(), py::arg("sysdef"),
             py::arg("nlist"));
    m.attr("gpu_enabled") = py::bool_(true);
}
