// swpc_host.h -- host-side restatements shared by the C-ABI implementation
// and the setup entry points (swpc_setup.h).
#pragma once

#include "../../include/swpc_setup.h"

namespace swpc {

// momentrate (src/shared/m_fdtool.f90:472-497) in the reference's kinds:
// arguments real(SP), PI real(DP) so mixed expressions promote to double.
float momentrate(float t, int stftype, float ts, float tr);

// mean over the nm mechanisms of (i w ts)/(1 - i w ts) at w = 2 pi fq_ref
// (relaxed_medium, m_medium.f90:234-274): real and imaginary parts in SP,
// each term in DP
void relaxed_cc(int nm, const float *ts, float fq_ref, float *ccr, float *cci);

// layer table of vmodel_lhm after the velocity cut-off
// (m_vmodel_lhm.f90:93-101) and the velocity ceiling of lhm_rmed
// (m_vmodel_lhm_rmed.f90:95-98); r0 .. qb hold nlayer values each
void lhm_layers(const swpc_grid *g, int nlayer, const float *depth, const float *rho0, const float *vp0,
                const float *vs0, const float *qp0, const float *qs0, float vcut, float *r0, float *p0, float *s0,
                float *qa, float *qb, float *vmax_r);

}  // namespace swpc
