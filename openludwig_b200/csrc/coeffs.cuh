// Aerodynamic coefficients from the nine surface-force sums, as the
// reference's integrate_surface_forces! finishes them (surface.jl:873-910):
// symmetry doubling of a half model, then C = F / (1/2 rho U^2 A) and
// Cm = M / (1/2 rho U^2 A c).
#pragma once
#include "../../include/openludwig_b200.h"

namespace ol {

// raw = {Fx_p, Fy_p, Fz_p, Fx_v, Fy_v, Fz_v, Mx, My, Mz}; out[12] as
// ol_ctx_case_coefficients documents it.
inline void coefficients_from_sums(const double raw[9], const ol_coeff_ref *ref, double out[12]) {
  double Fxp = raw[0], Fyp = raw[1], Fzp = raw[2], Fxv = raw[3], Fyv = raw[4], Fzv = raw[5];
  double Mx = raw[6], My = raw[7], Mz = raw[8];
  if (ref->symmetric) {
    Fxp *= 2.0; Fzp *= 2.0; Fxv *= 2.0; Fzv *= 2.0; My *= 2.0;
    Fyp = Fyv = 0.0;
    Mx = Mz = 0.0;
  }
  const double q_inf = 0.5 * ref->rho_ref * ref->u_ref * ref->u_ref;
  const double F_ref = q_inf * ref->area_ref, M_ref = F_ref * ref->chord_ref;
  const double Fx = Fxp + Fxv, Fy = Fyp + Fyv, Fz = Fzp + Fzv;
  for (int i = 0; i < 12; ++i) out[i] = 0.0;
  if (F_ref > 1e-10) { out[0] = Fx / F_ref; out[1] = Fz / F_ref; out[2] = Fy / F_ref; }
  if (M_ref > 1e-10) { out[3] = Mx / M_ref; out[4] = My / M_ref; out[5] = Mz / M_ref; }
  out[6] = Fx; out[7] = Fy; out[8] = Fz;
  out[9] = Mx; out[10] = My; out[11] = Mz;
}

}  // namespace ol
