// Solver drivers (placeholder until the Krylov kernels land).
#include "solvers.hpp"

namespace gr {

std::unique_ptr<SolverTree> SolverTree::create(DeviceMatrix&, const std::string&) {
  fail(GR_EUNSUPPORTED, "solvers are not built yet");
}

}  // namespace gr
