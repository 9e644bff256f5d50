// Scalar fields of the pair kernels' arguments, derived from the pass
// parameters and the fitted polynomial (shared by the session and the server).
#pragma once

#include <cmath>

#include "photons_p2p.h"
#include "p2p_fit.h"
#include "p2p_internal.h"

namespace p2p {

// Everything in PairArgs except the buffers, counts and packing tables.
// per_particle_masses: the masses ride in the sources' .w, so out_scale
// leaves out the equal mass.
inline void fill_pass_scalars(PairArgs &a, const p2p_params &p, const PolyFit &fit,
                              bool per_particle_masses) {
    const double c = 0.5 / p.split_radius;
    a.cscale = c;
    a.eps2 = (float)((c * p.soften) * (c * p.soften));
    a.u0 = (float)fit.u0;
    a.ucut = (float)fit.umax;
    a.ucut_lo = (float)(fit.umax * (1.0 - kCutBand));
    a.ucut_hi = (float)(fit.umax * (1.0 + kCutBand));
    a.rcut2 = fit.umax / (c * c);
    a.eps2_box = p.soften * p.soften;
    for (int k = 0; k < kMaxCoef; ++k) {
        a.coef[k] = -fit.coef[k];
        a.coef2[k] = make_float2(a.coef[k], a.coef[k]);
    }
    a.uin = (float)(fit.umax * (1.0 - kInsideMargin));
    a.uout = (float)(fit.umax * (1.0 + kCutBand) * (1.0 + kOutsideMargin));
    a.out_scale = c * c * (per_particle_masses ? 1.0 : p.mass);
    a.soft = p.soften;
    a.r_soft = 1.0 / p.soften;
    a.rrs = 1.0 / p.split_radius;
    a.hrrs = 0.5 * a.rrs;
    a.coeff = 2.0 * (1.0 / std::sqrt(M_PI));
    a.xcut = p.x_cut;
    a.mass_eq = p.mass;
    a.leaf_warps = p.warps_per_leaf > 1 ? p.warps_per_leaf : 1;
}

}  // namespace p2p
