// FP64 product instantiation (precision 64).  FMA contraction is allowed and
// the Van Leer limiters and the other data-dependent quotients take their
// reciprocals once per point (fast_rcp / fdiv in common.cuh), so results
// differ from the reference's in the last bits; the bar is relative L2 of at
// most 1e-10 per field against the oracle after 100 steps.
#define LARE_VARIANT f64fast
#define LARE_FAST 1
#include "engine_impl.cuh"

namespace lare {
EngineBase* make_engine_f64(const lare_params* p, int nx, int ny, int nz, const double* const* metrics6,
                            std::string& err) {
  return make_engine<double>(p, nx, ny, nz, metrics6, err);
}
}  // namespace lare
