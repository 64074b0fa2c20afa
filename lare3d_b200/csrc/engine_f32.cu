// FP32 form: field arithmetic in FP32 (FMA contraction, approximate
// division); the CFL dt reduction, budgets and RKL2 coefficients stay FP64
// (engine.cuh).
#define LARE_VARIANT f32
#define LARE_FAST 1
#include "engine_impl.cuh"

namespace lare {
EngineBase* make_engine_f32(const lare_params* p, int nx, int ny, int nz, const double* const* metrics6,
                            std::string& err) {
  return make_engine<float>(p, nx, ny, nz, metrics6, err);
}
}  // namespace lare
