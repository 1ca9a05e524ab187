// Batched solves of many independent systems in one set of kernel launches
// (batch.cpp).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "device.hpp"
#include "host_matrix.hpp"
#include "solvers.hpp"

namespace gr {

// The block-diagonal union of `parts`: system s occupies tile-order rows
// [rowBegin[s], rowBegin[s] + rowReal[s]) and tiles [tileBegin[s],
// tileBegin[s + 1]), padded with decoupled unit rows to the next multiple of
// 32 rows. Only what the device side reads is filled (the layout, tile-local
// CRS, level sets and permutation).
std::shared_ptr<HostMatrix> concatForBatch(const std::vector<std::shared_ptr<HostMatrix>>& parts,
                                           std::vector<i64>& rowBegin, std::vector<i64>& rowReal,
                                           std::vector<i32>& tileBegin);

class BatchSolve {
 public:
  // json: a PBiCGStab configuration with the ILU preconditioner (run by the
  // ring substitution kernel, one tile per block).
  BatchSolve(std::vector<std::shared_ptr<HostMatrix>> parts, const std::string& json);
  ~BatchSolve();
  // Host vectors in each system's natural order; x in/out.
  std::vector<gr_stats> solveHost(const std::vector<void*>& x, const std::vector<const void*>& b, DType t);
  int systems() const { return static_cast<int>(parts_.size()); }

 private:
  std::vector<std::shared_ptr<HostMatrix>> parts_;
  std::shared_ptr<HostMatrix> union_;
  std::vector<i64> rowBegin_, rowReal_;
  std::vector<i32> tileBegin_;
  std::unique_ptr<DeviceMatrix> D_;
  std::unique_ptr<SolverTree> tree_;
};

}  // namespace gr
