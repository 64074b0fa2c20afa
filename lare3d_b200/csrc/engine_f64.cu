// FP64 parity instantiation (precision LARE_FP64_EXACT).  Built with
// --fmad=false so that every multiply and add rounds separately, as in a
// gfortran x86-64 build of the reference (no FMA contraction); divisions are
// IEEE quotients in the reference's expression order, so results equal the
// reference's arithmetic bit for bit.
#define LARE_VARIANT f64exact
#include "engine_impl.cuh"

namespace lare {
EngineBase* make_engine_f64_exact(const lare_params* p, int nx, int ny, int nz, const double* const* metrics6,
                                  std::string& err) {
  return make_engine<double>(p, nx, ny, nz, metrics6, err);
}
}  // namespace lare
