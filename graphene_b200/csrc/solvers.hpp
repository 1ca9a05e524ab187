// Solver tree: configuration parsing and the solver drivers
// (matrix/solver/ of the reference).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "device.hpp"

namespace gr {

class SolverTree {
 public:
  virtual ~SolverTree() = default;
  // Configuration::fromJSON + Solver::createSolver.
  static std::unique_ptr<SolverTree> create(DeviceMatrix& A, const std::string& json);
  // Solver::solve(x, b) with device vectors in tile order.
  virtual gr_stats solve(void* x, DType xt, const void* b, DType bt) = 0;
  // Host vectors in natural order, copies included.
  virtual gr_stats solveHost(void* x, DType xt, const void* b, DType bt) = 0;
  // Runs the solve `reps` times back to back on the matrix's stream with no
  // host synchronisation in between and returns the mean device time per
  // run (ms) between two events. For timing single-application solvers
  // (ILU, a fixed number of Gauss-Seidel sweeps).
  virtual float timeRepeated(void* x, DType xt, const void* b, DType bt, int reps) = 0;
  virtual void copyPhi(void* out, DType t) = 0;
  // Per-system statistics of the last solve on a batch matrix.
  virtual std::vector<gr_stats> batchStats() const = 0;
  virtual std::string name() const = 0;
  // After the matrix's values were replaced (DeviceMatrix::updateValues):
  // recomputes every value-dependent part (ILU factors, packed level
  // blocks) in the buffers the tree already owns, so its captured iteration
  // graphs stay valid.
  virtual void refresh() = 0;
};

}  // namespace gr
