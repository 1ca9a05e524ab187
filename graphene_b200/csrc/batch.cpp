// Batched solves: many independent systems, of uneven sizes, solved by one
// PBiCGStab whose every kernel launch covers all of them.
//
// The systems' host matrices are concatenated into one block-diagonal matrix
// (each keeps its own tile layout, tile-local CRS and level sets, shifted to
// its rows and tiles), each system padded by a tile of decoupled unit rows
// to a whole number of 32-row SELL chunks. The device matrix then carries
// a BatchSeg that splits the Krylov kernels per system: every system keeps
// its own state (rho, alpha, omega, norms, convergence, done) and its
// reductions run over the same block partition, in the same order, as a
// solve of that system alone, so a system's result in the batch is the
// result it gets alone. Converged systems drop out of the work (their blocks
// return at once) while the others continue.
#include "batch.hpp"

#include <algorithm>
#include <cstring>

#include "config.hpp"

namespace gr {

std::shared_ptr<HostMatrix> concatForBatch(const std::vector<std::shared_ptr<HostMatrix>>& parts,
                                           std::vector<i64>& rowBegin, std::vector<i64>& rowReal,
                                           std::vector<i32>& tileBegin) {
  if (parts.empty()) fail(GR_EINVAL, "a batch needs at least one system");
  const DType vt = parts[0]->valueType;
  auto U = std::make_shared<HostMatrix>();
  U->valueType = vt;
  U->spmvLayout = parts[0]->spmvLayout;
  bool anyRank = false;
  for (const auto& h : parts) {
    if (!h) fail(GR_EINVAL, "batch system is NULL");
    if (h->valueType != vt) fail(GR_EINVAL, "batch systems must share one coefficient type");
    anyRank = anyRank || !h->sumRank.empty();
  }
  rowBegin.clear();
  rowReal.clear();
  tileBegin.clear();
  i64 n = 0, m = 0;
  i32 P = 0;
  for (const auto& h : parts) {
    const i64 pad = (32 - h->n % 32) % 32;
    rowBegin.push_back(n);
    rowReal.push_back(h->n);
    tileBegin.push_back(P);
    n += h->n + pad;
    m += h->m;
    P += h->P + (pad > 0 ? 1 : 0);
  }
  tileBegin.push_back(P);
  if (n >= (i64(1) << 31) - 1) fail(GR_EUNSUPPORTED, "batch exceeds 2^31-2 rows");
  U->n = n;
  U->m = m;
  U->P = P;
  U->tileStart.reserve(P + 1);
  U->rowPtr.assign(1, 0);
  U->rowPtr.reserve(n + 1);
  U->colPerm.reserve(m);
  U->colLocal.reserve(m);
  U->offDiag.reserve(m);
  U->diag.reserve(n);
  U->iperm.reserve(n);
  U->lowerLevel.reserve(n);
  U->upperLevel.reserve(n);
  if (anyRank) U->sumRank.reserve(m);
  for (size_t s = 0; s < parts.size(); ++s) {
    const HostMatrix& H = *parts[s];
    const i64 r0 = rowBegin[s];
    const i64 pad = (32 - H.n % 32) % 32;
    for (i32 T = 0; T < H.P; ++T) {
      U->tileStart.push_back(r0 + H.tileStart[T]);
      U->nLowerLevels.push_back(H.nLowerLevels[T]);
      U->nUpperLevels.push_back(H.nUpperLevels[T]);
      U->tiles.push_back(H.tiles[T]);
    }
    for (i64 p = 0; p < H.n; ++p) {
      for (i64 k = H.rowPtr[p]; k < H.rowPtr[p + 1]; ++k) {
        U->colPerm.push_back(static_cast<i32>(r0 + H.colPerm[k]));
        U->colLocal.push_back(H.colLocal[k]);
        U->offDiag.push_back(H.offDiag[k]);
        if (anyRank) U->sumRank.push_back(H.sumRank.empty() ? static_cast<i32>(k - H.rowPtr[p]) : H.sumRank[k]);
      }
      U->rowPtr.push_back(static_cast<i64>(U->colPerm.size()));
      U->diag.push_back(H.diag[p]);
      U->iperm.push_back(static_cast<i32>(r0 + H.iperm[p]));
      U->lowerLevel.push_back(H.lowerLevel[p]);
      U->upperLevel.push_back(H.upperLevel[p]);
    }
    if (pad > 0) {
      // Padding tile: decoupled unit rows (diagonal 1, no off-diagonals).
      U->tileStart.push_back(r0 + H.n);
      U->nLowerLevels.push_back(1);
      U->nUpperLevels.push_back(1);
      HostMatrix::Tile t;
      t.nInterior = pad;
      U->tiles.push_back(t);
      for (i64 j = 0; j < pad; ++j) {
        U->rowPtr.push_back(static_cast<i64>(U->colPerm.size()));
        U->diag.push_back(1.0);
        U->iperm.push_back(static_cast<i32>(r0 + H.n + j));
        U->lowerLevel.push_back(0);
        U->upperLevel.push_back(0);
      }
    }
    U->maxTileRows = std::max(U->maxTileRows, std::max<i64>(H.maxTileRows, pad));
    U->numHaloTotal += H.numHaloTotal;
  }
  U->tileStart.push_back(n);
  U->perm.assign(n, 0);
  for (i64 p = 0; p < n; ++p) U->perm[U->iperm[p]] = static_cast<i32>(p);
  U->format = parts[0]->format;
  return U;
}

BatchSolve::BatchSolve(std::vector<std::shared_ptr<HostMatrix>> parts, const std::string& json)
    : parts_(std::move(parts)) {
  auto cfg = SolverConfig::fromText(json);
  if (cfg->type != "PBiCGStab" && !(cfg->type == "IterativeRefinement" && cfg->innerSolver &&
                                    cfg->innerSolver->type == "PBiCGStab"))
    fail(GR_EUNSUPPORTED, "batched solves run PBiCGStab, or IterativeRefinement over PBiCGStab");
  union_ = concatForBatch(parts_, rowBegin_, rowReal_, tileBegin_);
  D_ = std::make_unique<DeviceMatrix>(union_);
  D_->makeBatch(rowBegin_, rowReal_, tileBegin_);
  tree_ = SolverTree::create(*D_, json);
}

BatchSolve::~BatchSolve() {
  tree_.reset();  // synchronises the stream before its buffers go
  D_.reset();
}

std::vector<gr_stats> BatchSolve::solveHost(const std::vector<void*>& x, const std::vector<const void*>& b, DType t) {
  const size_t S = parts_.size();
  if (x.size() != S || b.size() != S) fail(GR_EINVAL, "one x and one b per system");
  if (t != DType::F32 && t != DType::F64) fail(GR_EINVAL, "x and b must be float32 or float64");
  const size_t vs = dtypeSize(t);
  const i64 n = union_->n;
  // Right-hand sides and initial guesses in the union's natural order
  // (system s at rows [rowBegin[s], rowBegin[s] + its rows), padding rows
  // 0, so that they solve 1 * x = 0), permuted into tile order on the
  // device.
  std::vector<unsigned char> bh(n * vs, 0), xh(n * vs, 0);
  for (size_t s = 0; s < S; ++s) {
    if (!x[s] || !b[s]) fail(GR_EINVAL, "x and b must not be NULL");
    std::memcpy(bh.data() + rowBegin_[s] * vs, b[s], rowReal_[s] * vs);
    std::memcpy(xh.data() + rowBegin_[s] * vs, x[s], rowReal_[s] * vs);
  }
  DBuf tmp(n * vs), xd(n * vs), bd(n * vs);
  cudaStream_t st = D_->stream;
  GR_CUDA(cudaMemcpyAsync(tmp.get(), bh.data(), n * vs, cudaMemcpyHostToDevice, st));
  launchPermute(*D_, tmp.get(), bd.get(), t, true, st);
  GR_CUDA(cudaMemcpyAsync(tmp.get(), xh.data(), n * vs, cudaMemcpyHostToDevice, st));
  launchPermute(*D_, tmp.get(), xd.get(), t, true, st);
  tree_->solve(xd.get(), t, bd.get(), t);
  launchPermute(*D_, xd.get(), tmp.get(), t, false, st);
  GR_CUDA(cudaMemcpyAsync(xh.data(), tmp.get(), n * vs, cudaMemcpyDeviceToHost, st));
  GR_CUDA(cudaStreamSynchronize(st));
  for (size_t s = 0; s < S; ++s) std::memcpy(x[s], xh.data() + rowBegin_[s] * vs, rowReal_[s] * vs);
  return tree_->batchStats();
}

}  // namespace gr
