// swpc2d_api.cu -- 2D P-SV / SH solvers (placeholder until the 2D kernels land).
#include "swpc_ctx.h"

namespace swpc {
int create_2d(swpc_ctx *c) { return set_err(c, SWPC_ERR_ARG, "2D solvers are not available in this build"); }
int upload_medium_2d(swpc_ctx *c, const swpc_medium_view *) { return set_err(c, SWPC_ERR_ARG, "2D not available"); }
int absorb_setup_2d(swpc_ctx *c, const float *, const float *, const float *, const float *) {
    return set_err(c, SWPC_ERR_ARG, "2D not available");
}
int update_stress_2d(swpc_ctx *c, int) { return set_err(c, SWPC_ERR_ARG, "2D not available"); }
int update_vel_2d(swpc_ctx *c, int) { return set_err(c, SWPC_ERR_ARG, "2D not available"); }
int wav_store_2d(swpc_ctx *c, int, const int *) { return set_err(c, SWPC_ERR_ARG, "2D not available"); }
int vmax_2d(swpc_ctx *c, float *) { return set_err(c, SWPC_ERR_ARG, "2D not available"); }
void destroy_2d(swpc_ctx *) {}
}  // namespace swpc
