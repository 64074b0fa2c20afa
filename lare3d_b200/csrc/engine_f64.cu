// FP64 drop-in instantiation.  Built with --fmad=false so that every
// multiply and add rounds separately, as in a gfortran x86-64 build of the
// reference (no FMA contraction).
#include "engine_impl.cuh"

namespace lare {
EngineBase* make_engine_f64(const lare_params* p, int nx, int ny, int nz, const double* const* metrics6,
                            std::string& err) {
  return make_engine<double>(p, nx, ny, nz, metrics6, err);
}
}  // namespace lare
