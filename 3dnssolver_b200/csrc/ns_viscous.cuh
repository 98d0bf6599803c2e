// ns_viscous.cuh -- centered viscous residual from its derivatives (device).
#pragma once

#include "ns_common.cuh"

namespace nsb {

// CenteredDiffusion::compute_residual (src/diffusion_schemes/centered_diffusion.cpp:70-182)
// with the stress helpers of diffusion_scheme.cpp:3-58 and dmu = 0 (the terms
// multiplied by dmu or dlamb are dropped, which is exact).  Reproduced as the
// reference computes them: Tauyy = tauxx (:143), the x work term uses
// Tauxy*dv_dy (:148), the y heat-flux term multiplies by 1 where the pressure
// belongs (:166), 2D terms only and rhoW untouched (:173-176).
// Derivatives of (rho, p, u, v) (index 0..3): Dx, Dy, Dxx, Dyy (the x-stencil
// scaled by 1/dy^2, cd-n.cpp:77); mixed Dxy = d/dy(dW/dx), Dyx = d/dx(dW/dy) of
// (u, v); Uc, Vc, P, RHO the cell's primitives.  Adds to r[1..3].
template <typename TV>
__device__ __forceinline__ void viscous_reference_terms(const TV Dx[4], const TV Dy[4], const TV Dxx[4],
                                                        const TV Dyy[4], const TV Dxy[2],
                                                        const TV Dyx[2], TV Uc, TV Vc, TV P, TV RHO,
                                                        const Consts& c, TV r[5]) {
    const TV mu = TV(c.mu), lamb = TV(c.lamb), two = TV(2);
    const TV du_dx = Dx[2], du_dy = Dy[2], du_dxdx = Dxx[2], du_dydy = Dyy[2];
    const TV du_dxdy = Dxy[0], du_dydx = Dyx[0];
    const TV dv_dy = Dy[3], dv_dx = Dx[3], dv_dxdx = Dxx[3], dv_dydy = Dyy[3];
    const TV dv_dydx = Dyx[1], dv_dxdy = Dxy[1];
    const TV drho_dx = Dx[0], dp_dx = Dx[1], drho_dxdx = Dxx[0], dp_dxdx = Dxx[1];
    const TV drho_dy = Dy[0], dp_dy = Dy[1], drho_dydy = Dyy[0], dp_dydy = Dyy[1];

    TV Dtauxx_dx = two * mu * du_dxdx + lamb * (du_dxdx + dv_dydx);
    TV Dtauyy_dy = two * mu * dv_dydy + lamb * (du_dxdy + dv_dydy);
    TV Dtauxy_dx = mu * (du_dydx + dv_dxdx);
    TV Dtauyx_dy = mu * (du_dydy + dv_dxdy);
    TV Tauxx = two * mu * du_dx + lamb * (du_dx + dv_dy);
    TV Tauyy = Tauxx;
    TV Tauxy = mu * (du_dy + dv_dx);
    TV Dtauvx_dx = Uc * Dtauxx_dx + Vc * Dtauxy_dx + Tauxx * du_dx + Tauxy * dv_dy;
    TV Dtauvy_dy = Uc * Dtauyx_dy + Vc * Dtauyy_dy + Tauyy * dv_dy + Tauxy * du_dy;
    TV ir = TV(1) / RHO, ir2 = ir * ir, ir3 = ir2 * ir;
    TV heat = TV(c.heat);
    TV Dqx_dx = -heat * (mu * (two * ir2 * drho_dx * dp_dx + ir * dp_dxdx + ir3 * P * drho_dx * drho_dx -
                               ir2 * P * drho_dxdx));
    TV Dqy_dy = -heat * (mu * (two * ir2 * drho_dy * dp_dy + ir * dp_dydy + ir3 * drho_dy * drho_dy -
                               ir2 * P * drho_dydy));
    r[1] += -Dtauvx_dx - Dtauvy_dy + Dqx_dx + Dqy_dy;
    r[2] += -Dtauxx_dx - Dtauyx_dy;
    r[3] += -Dtauyy_dy - Dtauxy_dx;
}

}  // namespace nsb
