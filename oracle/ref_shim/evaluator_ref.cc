// Test-only build of the reference's own pair evaluator
// (src/EvaluatorPairPSWF.h with the shipped src/PSWF_Coeffs.h), compiled
// from the reference sources where they lie. The reference names its table
// arrays PSWF_SEG_R_LO / PSWF_SEG_DR_INV (src/EvaluatorPairPSWF.h:131-132)
// while the header defines PSWF_R_LO / PSWF_DR_INV (src/PSWF_Coeffs.h:8229,
// 8915); the two aliases below are the only addition.
#include "PSWF_Coeffs.h"

namespace hoomd {
namespace md {
namespace esp_pswf_coeffs {
inline constexpr const double* PSWF_SEG_R_LO = PSWF_R_LO;
inline constexpr const double* PSWF_SEG_DR_INV = PSWF_DR_INV;
}  // namespace esp_pswf_coeffs
}  // namespace md
}  // namespace hoomd

#include "EvaluatorPairPSWF.h"

extern "C" {

// EvaluatorPairPSWF(rsq, rcutsq, params).setCharge(qiqj, 1).evalForceAndEnergy
int ref_eval_pairs(int n, const double* rsq, const double* qiqj, double rcut, double* force_divr, double* pair_eng,
                   int* evaluated) {
    hoomd::md::EvaluatorPairPSWF::param_type p;
    p.rcut = rcut;
    for (int i = 0; i < n; ++i) {
        hoomd::md::EvaluatorPairPSWF ev(rsq[i], rcut * rcut, p);
        ev.setCharge(qiqj[i], 1.0);
        double f = 0.0, e = 0.0;
        evaluated[i] = ev.evalForceAndEnergy(f, e, false) ? 1 : 0;
        force_divr[i] = f;
        pair_eng[i] = e;
    }
    return 0;
}

// detail::pswf_eval_L: L(r) and -dL/dr
int ref_eval_L(int n, const double* r, double rcut, double* L, double* negdLdr) {
    for (int i = 0; i < n; ++i) hoomd::md::detail::pswf_eval_L(r[i], rcut, L[i], negdLdr[i]);
    return 0;
}
}
