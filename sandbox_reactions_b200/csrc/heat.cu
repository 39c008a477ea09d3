// heat.cu — P5 (placeholder until the FLD solver lands).
#include "heat.cuh"

struct HeatSolver {
    int dummy;
};

HeatSolver* heat_create(const sr_config&, cudaStream_t) {
    throw SrError{SR_E_UNSUPPORTED, "the heat pass is not built yet"};
}
void heat_destroy(HeatSolver* hs) { delete hs; }
void heat_step(HeatSolver*, float*, const float*, const double*, cudaStream_t, sr_heat_report*) {}
void heat_read_flux(HeatSolver*, float*, float*) {}
void heat_set_precond(HeatSolver*, uint32_t) {}
void heat_set_limits(HeatSolver*, uint32_t, uint32_t) {}
void heat_first_solve(HeatSolver*, const float*, const float*, double, uint32_t, cudaStream_t, double*, uint32_t*,
                      double*, double*) {}
