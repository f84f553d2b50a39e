// swpc_host.h -- host-side restatements shared by the C-ABI implementation
// and the setup entry points (swpc_setup.h).
#pragma once

namespace swpc {

// momentrate (src/shared/m_fdtool.f90:472-497) in the reference's kinds:
// arguments real(SP), PI real(DP) so mixed expressions promote to double.
float momentrate(float t, int stftype, float ts, float tr);

}  // namespace swpc
