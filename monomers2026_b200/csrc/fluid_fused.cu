// fluid_fused.cu - spectral-state fused form (placeholder until built).
#include "selm_engine.h"

int fused_allocate(selm_sim*) { return selm_fail(SELM_ERR_INVALID, "fused forms are not available in this build"); }
int fused_initial(selm_sim*) { return selm_fail(SELM_ERR_INVALID, "fused forms are not available"); }
int fused_step(selm_sim*) { return selm_fail(SELM_ERR_INVALID, "fused forms are not available"); }
int fused_get_field(selm_sim*, int, double*) { return selm_fail(SELM_ERR_INVALID, "fused forms are not available"); }
int fused_set_field(selm_sim*, int, const double*) { return selm_fail(SELM_ERR_INVALID, "fused forms are not available"); }
int fused_stream_changed(selm_sim*) { return SELM_OK; }
void fused_release(selm_sim*) {}
