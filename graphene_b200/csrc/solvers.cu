// Solver drivers (matrix/solver/ of the reference): the C++ host side that
// sequences the CUDA kernels. All vectors are device pointers in tile order.
//
// Each solver node mirrors one reference solver class:
//   IluNode          ilu::Solver              (ilu/Solver.cpp:44-574)
//   GsNode           gaussseidel::Solver      (gauss-seidel/Solver.cpp:39-160)
//   PbicgstabNode    pbicgstab::Solver        (pbicgstab/Solver.cpp:40-194)
//   MpirNode         iterativerefinement::Solver (iterative-refinement/Solver.cpp:48-128)
//   RestarterNode    restarter::Solver        (restarter/Solver.cpp:34-56)
// and Solver::createSolver's dispatch is makeNode (Solver.cpp:32-56).
#include <cstdio>
#include <cstring>
#include <mutex>

#include "config.hpp"
#include "krylov.hpp"
#include "solvers.hpp"

namespace gr {

namespace {

// The working type of a solve: the configured workingType, else x's type.
DType workingType(const SolverConfig& c, DType xt) {
  return c.workingType < 0 ? xt : static_cast<DType>(c.workingType);
}

class Node {
 public:
  Node(DeviceMatrix& A, const SolverConfig& c) : A_(A), cfg_(c) {}
  virtual ~Node() = default;
  // x: in/out, b: in; both of type W. gate (nullable): the enclosing
  // solver's state; kernels of this solve return early once it is done.
  virtual gr_stats solve(void* x, const void* b, DType W, const KState* gate) = 0;
  virtual bool usesInitialGuess() const = 0;
  virtual void copyPhi(void*, DType) { fail(GR_EUNSUPPORTED, "only IterativeRefinement keeps phi"); }
  // Allocates the scratch a solve of type W needs (before graph capture).
  virtual void prepare(DType) {}
  // Recomputes the parts that depend on the matrix's values, in place.
  virtual void refresh() {}
  // Per-system statistics of the last solve of a batch.
  virtual std::vector<gr_stats> batchStats() const {
    fail(GR_EUNSUPPORTED, "only PBiCGStab and IterativeRefinement solve batches");
  }
  // Batches: the systems the next solve leaves alone (nonzero entries; x of
  // those systems is not touched). Empty: none.
  virtual void setBatchSkip(const std::vector<int>&) {
    fail(GR_EUNSUPPORTED, "only PBiCGStab skips systems of a batch");
  }

 protected:
  DeviceMatrix& A_;
  const SolverConfig& cfg_;
  cudaStream_t s() const { return A_.stream; }
};

std::unique_ptr<Node> makeNode(DeviceMatrix& A, const SolverConfig& c);

void printStats(const SolverConfig& c, const DeviceMatrix& A, const gr_stats& st) {
  static const char* norms[] = {"L1", "L2", "LINF", "None"};
  std::fprintf(stderr,
               "%s: Solved on %d tiles, %s norm, Initial residual = %g, Final residual = %g, "
               "Iterations = %d, Converged = %s, Singular = %s\n",
               c.solverName().c_str(), A.P, norms[c.norm], st.initial_residual, st.final_residual,
               st.iterations, st.converged ? "true" : "false", st.singular ? "true" : "false");
}

// ---------------------------------------------------------------------------
class IluNode : public Node {
 public:
  IluNode(DeviceMatrix& A, const SolverConfig& c) : Node(A, c), dilu_(c.diagonalBased) {
    A.ensureLocalCrs();
    const size_t vs = dtypeSize(A.vt);
    // Streamed substitution when the ring and the tile slice fit in shared
    // memory for either vector type; the level-schedule kernel otherwise.
    // Substitution kernel: the bulk-copy ring kernel over the tile byte
    // stream (auto / "tma"), warp-per-tile over the same stream ("warp"), or
    // the level-schedule kernel ("levels", and auto when a tile does not fit
    // shared memory).
    kernel_ = 2;
    const size_t smemMax = static_cast<size_t>(maxDynamicSmem(A));
    if (c.iluKernel == 5) {
      // Warp per tile over the same host-scheduled level ring.
      ring_ = &A.levelRing(dilu_, c.ringBytes, 1, c.compactRing, RingKind::Ilu, c.ringRecords);
      if (iluWarpRingSmem(*ring_, DType::F64, c.warpsPerBlock) > smemMax)
        fail(GR_EUNSUPPORTED, "the warp ring ILU kernel does not fit this matrix's tiles in shared memory");
      kernel_ = 5;
    }
    if (c.iluKernel == 0 || c.iluKernel == 4) {
      LevelRing* R = nullptr;
      try {
        R = &A.levelRing(dilu_, c.ringBytes, c.tilesPerBlock > 0 ? c.tilesPerBlock : 1, c.compactRing,
                         RingKind::Ilu, c.ringRecords);
      } catch (const Error&) {
        if (c.iluKernel == 4) throw;  // the requested ring cannot hold the levels
      }
      if (R && iluRingSmem(A, *R, DType::F64) <= smemMax) {
        kernel_ = 4;
        ring_ = R;
        autoGroups(A, c, smemMax);
      } else if (c.iluKernel == 4) {
        fail(GR_EUNSUPPORTED, "the ring ILU kernel does not fit this matrix's tiles in shared memory");
      }
    }
    if (kernel_ == 2 && c.iluKernel != 2 && c.iluKernel != 4) {
      SweepStream& S = A.iluSweepStream(dilu_);
      const bool warpFits = iluWarpSmem(A, S, DType::F64) <= smemMax;
      const size_t tmaNeed = iluStreamSmem(A, S, DType::F64, c.ringLog2);
      const bool tmaFits = tmaNeed > 0 && tmaNeed <= smemMax;
      if (c.iluKernel == 0) kernel_ = tmaFits ? 1 : 2;
      else if (c.iluKernel == 3 && warpFits) kernel_ = 3;
      else if (c.iluKernel == 1 && tmaFits) kernel_ = 1;
      else fail(GR_EUNSUPPORTED, "the requested ILU kernel does not fit this matrix's tiles in shared memory");
    }
    inv_.alloc(A.n * vs);
    if (kernel_ == 4 || kernel_ == 5) {
      stream_.alloc(std::max<i64>(16, ring_->bytes));
    } else if (kernel_ != 2) {
      SweepStream& S = A.iluSweepStream(dilu_);
      sweep_ = &S;
      rowsPerLane_ = iluWarpRowsPerLane(A, S);
      stream_.alloc(std::max<i64>(16, S.bytes));
    } else {
      Lval_.alloc(std::max<i64>(1, A.schedule(SweepEntries::Lower).slots) * vs);
      Uval_.alloc(std::max<i64>(1, A.schedule(SweepEntries::UpperDesc).slots) * vs);
    }
    factorAndPack();
  }
  void refresh() override { factorAndPack(); }
  // ilu::Solver::factorize (ilu/Solver.cpp:44-51, :134-292) of the matrix's
  // current values, and the packing of the factors into this solver's own
  // level blocks (the buffers allocated at construction).
  void factorAndPack() {
    DeviceMatrix& A = A_;
    const size_t vs = dtypeSize(A.vt);
    DBuf F, D;
    if (!dilu_) {
      F.alloc(std::max<i64>(1, A.m) * vs);
      GR_CUDA(cudaMemcpyAsync(F.get(), A.offDiag.get(), A.m * vs, cudaMemcpyDeviceToDevice, s()));
    }
    D.alloc(A.n * vs);
    GR_CUDA(cudaMemcpyAsync(D.get(), A.diag.get(), A.n * vs, cudaMemcpyDeviceToDevice, s()));
    launchIluFactor(A, dilu_ ? nullptr : F.get(), D.get(), A.offDiag.get(), dilu_, s());
    launchInvert(A, D.get(), inv_.get(), s());
    const void* vals = dilu_ ? A.offDiag.get() : F.get();
    if (kernel_ == 4 || kernel_ == 5) {
      launchRingPack(A, *ring_, stream_.get(), vals, inv_.get(), s());
    } else if (kernel_ != 2) {
      launchStreamPack(A, *sweep_, stream_.get(), vals, inv_.get(), s());
    } else {
      launchPack(A, A.schedule(SweepEntries::Lower), vals, Lval_.get(), s());
      launchPack(A, A.schedule(SweepEntries::UpperDesc), vals, Uval_.get(), s());
    }
    GR_CUDA(cudaStreamSynchronize(s()));  // F and D are released on return
  }
  bool streamed() const { return sweep_ != nullptr; }
  bool ringKernel() const { return kernel_ == 4; }
  gr_stats solve(void* x, const void* b, DType W, const KState* gate) override {
    PrologueArgs pro;
    pro.kind = Prologue::Plain;
    pro.b = b;
    pro.st = gate;
    apply(pro, x, W);
    gr_stats st{};
    st.iterations = 1;  // ilu/Solver.cpp:571-573
    return st;
  }
  void apply(const PrologueArgs& pro, void* y, DType W) {
    if (kernel_ == 5)
      launchIluWarpRing(A_, *ring_, stream_.get(), dilu_, pro, y, W, cfg_.warpsPerBlock, cfg_.pairRows, s());
    else if (kernel_ == 4)
      launchIluRing(A_, *ring_, stream_.get(), dilu_, pro, y, W, cfg_.l2Ahead, cfg_.unrollRows != 0, s(),
                    cfg_.pairRows, cfg_.computeWarps != 0 ? cfg_.computeWarps : autoWarps_, cfg_.waitingWarp,
                    cfg_.producerWarp);
    else if (kernel_ == 3)
      launchIluWarp(A_, *sweep_, stream_.get(), dilu_, pro, y, W, rowsPerLane_, s());
    else if (kernel_ == 1)
      launchIluStream(A_, *sweep_, stream_.get(), dilu_, pro, y, W,
                      StreamTuning{cfg_.ringLog2, cfg_.prefetchChunks, cfg_.unrollRows == 1}, s());
    else
      launchIluApply(A_, Lval_.get(), Uval_.get(), inv_.get(), dilu_, pro, y, W, s());
  }
  bool usesInitialGuess() const override { return false; }

 private:
  bool dilu_;
  // Tile groups (automatic, ring kernel, FP32 coefficients, default warps):
  // two consecutive tiles a block with four compute warps when the tiles
  // fill at least two waves of one-tile blocks and the grouped blocks take
  // no more waves. The waiting and producer warps' per-level work is then
  // shared by two tiles; on B200 at 192^3 with 2368 tiles that ran the
  // substitution in 104.4 us against 111.8 (MPIR 121.7 against 125.0 ms),
  // while at 2048 tiles, where grouping adds a wave, it ran slower. FP64
  // coefficients keep one tile a block (their slices halve the blocks per
  // SM).
  void autoGroups(DeviceMatrix& A, const SolverConfig& c, size_t smemMax) {
    if (c.tilesPerBlock != 0 || c.computeWarps != 0 || !c.waitingWarp || !c.producerWarp || A.vt != DType::F32 ||
        A.batch)  // batched solves run one tile a block
      return;
    const long long b1 = iluRingBlocksPerSM(A, *ring_, DType::F32, 0);
    const long long slots1 = b1 * A.numSMs;
    if (b1 <= 0 || ring_->numGroups < 2 * slots1) return;
    const long long waves1 = (ring_->numGroups + slots1 - 1) / slots1;
    // A two-tile block holds twice the x slice and about twice the ring, so
    // at most (b1 + 1) / 2 fit an SM: skip building the grouped ring when
    // even that many would need more waves.
    const long long g2 = (ring_->numGroups + 1) / 2, slotsMax = (b1 + 1) / 2 * A.numSMs;
    if ((g2 + slotsMax - 1) / slotsMax > waves1) return;
    LevelRing* R2 = nullptr;
    try {
      R2 = &A.levelRing(dilu_, c.ringBytes, 2, c.compactRing, RingKind::Ilu, c.ringRecords);
    } catch (const Error&) {
      return;
    }
    if (iluRingSmem(A, *R2, DType::F64) > smemMax) return;
    const long long b2 = iluRingBlocksPerSM(A, *R2, DType::F32, 4);
    const long long slots2 = b2 * A.numSMs;
    if (b2 <= 0 || (R2->numGroups + slots2 - 1) / slots2 > waves1) return;
    ring_ = R2;
    autoWarps_ = 4;
  }
  int autoWarps_ = 0;  // compute warps chosen with automatic tile groups
  int kernel_ = 2;  // 1 tma ring, 2 level schedule, 3 warp per tile, 4 host-scheduled ring, 5 its warp-per-tile form
  int rowsPerLane_ = 2;
  DBuf inv_, Lval_, Uval_, stream_;
  const SweepStream* sweep_ = nullptr;
  const LevelRing* ring_ = nullptr;
};

// ---------------------------------------------------------------------------
class GsNode : public Node {
 public:
  GsNode(DeviceMatrix& A, const SolverConfig& c) : Node(A, c) {
    A.ensureLocalCrs();
    // The level-ring kernel when the tiles fit shared memory (for either
    // vector type): one ring with every entry, and one with the lower
    // entries only for sweeps that start from x = 0.
    if (c.gsKernel != 2) {
      try {
        ring_ = &A.levelRing(false, 0, 1, true, RingKind::GaussSeidel, c.ringRecords);
        ringLo_ = &A.levelRing(false, 0, 1, true, RingKind::GaussSeidelLower, c.ringRecords);
      } catch (const Error&) {
        if (c.gsKernel == 1 || c.gsKernel == 3) throw;
        ring_ = ringLo_ = nullptr;
      }
      const size_t smemMax = static_cast<size_t>(maxDynamicSmem(A));
      auto fits = [&](bool warp) {
        auto need = [&](const LevelRing& R) {
          return warp ? gsWarpRingSmem(R, DType::F64, c.warpsPerBlock) : iluRingSmem(A, R, DType::F64);
        };
        return need(*ring_) <= smemMax && need(*ringLo_) <= smemMax;
      };
      // Automatic: for float coefficients one warp per tile (on B200 a
      // 128^3 convection-diffusion sweep took 52.9 us against 70.7 us with a
      // block per tile); a block per tile for double coefficients (the
      // FP64 solve took 28.8 ms against 44.9 ms with a warp per tile, whose
      // slice holds twice the bytes) and in batches, whose tiles the block
      // kernel maps to their systems.
      warpRing_ = c.gsKernel == 3 || (c.gsKernel == 0 && !A.batch && A.vt == DType::F32);
      if (ring_ && warpRing_ && !fits(true)) {
        if (c.gsKernel == 3)
          fail(GR_EUNSUPPORTED, "the Gauss-Seidel ring kernel does not fit this matrix's tiles in shared memory");
        warpRing_ = false;
      }
      if (ring_ && !warpRing_ && !fits(false)) {
        if (c.gsKernel == 1)
          fail(GR_EUNSUPPORTED, "the Gauss-Seidel ring kernel does not fit this matrix's tiles in shared memory");
        ring_ = ringLo_ = nullptr;
      }
    }
    if (ring_) {
      stream_.alloc(std::max<i64>(16, ring_->bytes));
      streamLo_.alloc(std::max<i64>(16, ringLo_->bytes));
    } else {
      Gval_.alloc(std::max<i64>(1, A.schedule(SweepEntries::All).slots) * dtypeSize(A.vt));
    }
    refresh();
  }
  // Packs the matrix's current coefficients and diagonal into this
  // solver's level blocks.
  void refresh() override {
    if (ring_) {
      launchRingPack(A_, *ring_, stream_.get(), A_.offDiag.get(), A_.diag.get(), s());
      launchRingPack(A_, *ringLo_, streamLo_.get(), A_.offDiag.get(), A_.diag.get(), s());
    } else {
      launchPack(A_, A_.schedule(SweepEntries::All), A_.offDiag.get(), Gval_.get(), s());
    }
    GR_CUDA(cudaStreamSynchronize(s()));
  }

  // Whether the first sweep can take PBiCGStab's p / s update as its
  // right-hand side (the level-ring kernel), and that application:
  // numFixedIterations sweeps from x = 0.
  bool fusedPrologue() const { return ring_ != nullptr && cfg_.numFixedIterations > 0; }
  // The block ring kernel (one block per tile, which batches need).
  bool blockRing() const { return ring_ != nullptr && !warpRing_; }
  void applyFused(const PrologueArgs& pro, void* out, DType W) {
    ringSweeps(pro, out, W, cfg_.numFixedIterations, true);
  }

  // Sweeps ping-pong between x and a scratch vector; the result ends in x.
  void sweeps(void* x, const void* b, DType W, int count, bool xZero, const KState* gate) {
    if (count <= 0) return;
    if (ring_) {
      PrologueArgs pro;
      pro.kind = Prologue::Plain;
      pro.b = b;
      pro.st = gate;
      ringSweeps(pro, x, W, count, xZero);
      return;
    }
    ensureTmp(W);
    void* cur = x;
    void* other = tmp_.get();
    for (int k = 0; k < count; ++k) {
      launchGsSweep(A_, Gval_.get(), b, cfg_.gsSeedB, cur, xZero && k == 0, other, W, gate, s(), cfg_.gsDropHalo);
      std::swap(cur, other);
    }
    if (cur != x) GR_CUDA(cudaMemcpyAsync(x, cur, A_.n * dtypeSize(W), cudaMemcpyDeviceToDevice, s()));
  }

  gr_stats solve(void* x, const void* b, DType W, const KState* gate) override {
    return solveImpl(x, b, W, gate, false);
  }
  gr_stats solveFromZero(void* x, const void* b, DType W, const KState* gate) {
    return solveImpl(x, b, W, gate, true);
  }
  bool usesInitialGuess() const override { return true; }
  void prepare(DType W) override { ensureTmp(W); }

 private:
  gr_stats solveImpl(void* x, const void* b, DType W, const KState* gate, bool xZero) {
    gr_stats st{};
    // The working type (gauss-seidel/Solver.cpp:65, :114): the sweeps'
    // arithmetic and the convergence residual; x stays in its own type.
    const DType Wc = computeType(W);
    if (cfg_.numFixedIterations > 0) {
      // gauss-seidel/Solver.cpp:116-126
      sweeps(x, b, W, cfg_.numFixedIterations, xZero, gate);
      st.iterations = cfg_.numFixedIterations;
      return st;
    }
    if (gate) fail(GR_EUNSUPPORTED, "a GaussSeidel preconditioner needs numFixedIterations > 0");
    ensureTmp(W);
    DBuf r(A_.n * dtypeSize(Wc));
    double* d = A_.scalarOut.as<double>();
    double h = 0;
    if (cfg_.relTolerance > 0) {
      launchNorm(A_, b, W, cfg_.norm, d + 1, s());
      GR_CUDA(cudaMemcpyAsync(&h, d + 1, sizeof(double), cudaMemcpyDeviceToHost, s()));
      GR_CUDA(cudaStreamSynchronize(s()));
      st.b_norm = h;
    }
    auto residualNorm = [&]() {
      launchResidual(A_, x, W, b, W, r.get(), Wc, Wc, cfg_.norm, d, s());
      double v = 0;
      GR_CUDA(cudaMemcpyAsync(&v, d, sizeof(double), cudaMemcpyDeviceToHost, s()));
      GR_CUDA(cudaStreamSynchronize(s()));
      return v;
    };
    st.initial_residual = st.final_residual = residualNorm();
    bool conv = false;
    while (!((conv && st.iterations >= cfg_.minIterations) || st.iterations >= cfg_.maxIterations)) {
      // gauss-seidel/Solver.cpp:141-155: numSweeps sweeps per convergence check.
      sweeps(x, b, W, cfg_.numSweeps, xZero && st.iterations == 0, nullptr);
      st.iterations += cfg_.numSweeps;
      st.final_residual = residualNorm();
      conv = st.final_residual < cfg_.absTolerance || st.final_residual < st.initial_residual * cfg_.relResidual ||
             (cfg_.relTolerance > 0 && st.final_residual < st.b_norm * cfg_.relTolerance);
      if (!std::isfinite(st.final_residual)) {
        st.status = GR_ENONFINITE;
        break;
      }
      if (cfg_.printPerformanceEachIteration) {
        st.converged = conv;
        printStats(cfg_, A_, st);
      }
    }
    st.converged = conv;
    if (cfg_.printPerformanceAfterSolve) printStats(cfg_, A_, st);
    return st;
  }
  void ensureTmp(DType W) {
    const size_t bytes = A_.n * dtypeSize(W);
    if (tmp_.bytes() < bytes) tmp_.alloc(bytes);
  }
  // The sweeps' arithmetic type for vectors of type W: W, or float64 over
  // float32 vectors (level-ring kernel only).
  DType computeType(DType W) const {
    const DType Wc = workingType(cfg_, W);
    if (Wc == W) return W;
    if (!(W == DType::F32 && Wc == DType::F64))
      fail(GR_EUNSUPPORTED, "GaussSeidel workingType must be the vectors' type or float64 over float32 vectors");
    if (!ring_) fail(GR_EUNSUPPORTED, "a GaussSeidel workingType other than the vectors' needs the ring kernel");
    return Wc;
  }
  // Level-ring sweeps: the first takes its right-hand side from `first`
  // (b itself, or a fused p / s update, which it also writes); later ones
  // from b or the written p / s. A sweep from x = 0 uses the lower-only ring.
  void ringSweeps(const PrologueArgs& first, void* x, DType W, int count, bool xZero) {
    if (count <= 0) return;
    ensureTmp(W);
    PrologueArgs plain;
    plain.kind = Prologue::Plain;
    plain.b = first.kind == Prologue::Plain ? first.b : first.pOrS;
    plain.st = first.st;
    plain.stIndex = first.stIndex;
    void* cur = x;
    void* other = tmp_.get();
    for (int k = 0; k < count; ++k) {
      const bool zero = xZero && k == 0;
      launchGsRing(A_, zero ? *ringLo_ : *ring_, zero ? streamLo_.get() : stream_.get(), k == 0 ? first : plain,
                   cfg_.gsSeedB, cur, zero, other, W, computeType(W), s(), warpRing_ ? cfg_.warpsPerBlock : 0,
                   cfg_.gsDropHalo, cfg_.gsPairRows);
      std::swap(cur, other);
    }
    if (cur != x) GR_CUDA(cudaMemcpyAsync(x, cur, A_.n * dtypeSize(W), cudaMemcpyDeviceToDevice, s()));
  }
  const LevelRing* ring_ = nullptr;
  const LevelRing* ringLo_ = nullptr;
  bool warpRing_ = false;  // one warp per tile (else one block per tile)
  DBuf Gval_, tmp_, stream_, streamLo_;
};

// Pinned host mirrors of the Krylov state, handed out from slabs that are
// never returned: cudaFreeHost would wait for all work on the device (every
// other solve included) and pinning memory per solver is slow.
namespace {
constexpr size_t kPinnedSlot = 256;
constexpr size_t kPinnedSlab = 256;  // slots per cudaMallocHost
static_assert(sizeof(KState) + sizeof(int) <= kPinnedSlot, "KState and the error word must fit a pinned slot");
std::mutex g_pinnedMu;
std::vector<void*> g_pinnedFree;

void* acquirePinnedSlot() {
  std::lock_guard<std::mutex> lock(g_pinnedMu);
  if (g_pinnedFree.empty()) {
    void* slab = nullptr;
    GR_CUDA(cudaMallocHost(&slab, kPinnedSlot * kPinnedSlab));
    for (size_t i = 0; i < kPinnedSlab; ++i) g_pinnedFree.push_back(static_cast<char*>(slab) + i * kPinnedSlot);
  }
  void* p = g_pinnedFree.back();
  g_pinnedFree.pop_back();
  return p;
}

void releasePinnedSlot(void* p) {
  std::lock_guard<std::mutex> lock(g_pinnedMu);
  g_pinnedFree.push_back(p);
}
}  // namespace

// ---------------------------------------------------------------------------
// Right-preconditioned BiCGStab. One iteration is five kernels when the
// preconditioner is ILU (fused vector updates):
//   ilu_apply(p-update) -> spmv_dot(alpha) -> ilu_apply(s-update) ->
//   spmv_dot(omega) -> bicg_update(x, r, convergence, next rho/beta)
// Iterations are captured once into a CUDA graph of `kBatch` iterations
// that is replayed until the device-side state reports done.
class PbicgstabNode : public Node {
 public:
  static constexpr int kBatch = 8;

  PbicgstabNode(DeviceMatrix& A, const SolverConfig& c) : Node(A, c) {
    if (c.preconditioner) {
      pre_ = makeNode(A, *c.preconditioner);
      ilu_ = dynamic_cast<IluNode*>(pre_.get());
      gs_ = dynamic_cast<GsNode*>(pre_.get());
    }
    if (A.batch) {
      // A batch keeps one state per system; its preconditioner must look
      // up a block's system, which the block ring kernels (ILU substitution,
      // Gauss-Seidel sweeps) do.
      const bool iluOk = ilu_ && ilu_->ringKernel();
      const bool gsOk = gs_ && gs_->fusedPrologue() && gs_->blockRing();
      if (!iluOk && !gsOk)
        fail(GR_EUNSUPPORTED, "batched PBiCGStab needs the ILU preconditioner with the ring kernel, or Gauss-Seidel "
                              "with numFixedIterations > 0 on the block ring kernel");
      systems_ = A.batch->systems;
      GR_CUDA(cudaMallocHost(&host_, sizeof(KState) * systems_ + sizeof(int)));
      batchHost_ = true;
    } else {
      host_ = static_cast<KState*>(acquirePinnedSlot());
    }
    st_.alloc(sizeof(KState) * systems_);
  }
  ~PbicgstabNode() override {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (host_ && batchHost_) cudaFreeHost(host_);
    else if (host_) releasePinnedSlot(host_);
  }

  gr_stats solve(void* x, const void* b, DType Wx, const KState* gate) override {
    (void)gate;
    const DType W = workingType(cfg_, Wx);
    // workingType float64 over float32 x and b (pbicgstab/Solver.cpp:63-79):
    // every vector but x in double, x rounded to float at each update.
    mixed_ = W != Wx;
    if (mixed_ && !(Wx == DType::F32 && W == DType::F64))
      fail(GR_EUNSUPPORTED, "PBiCGStab workingType must be float64 over float32 vectors, or the vectors' type");
    if (mixed_ && A_.batch) fail(GR_EUNSUPPORTED, "batched PBiCGStab needs the working type of the vectors");
    const bool ref = cfg_.reduceRef;
    if (ref && (W != DType::F32 || A_.batch))
      fail(GR_EUNSUPPORTED, "reduce \"f32_ref_order\" needs float32 vectors and a single system");
    ensureBuffers(W);
    if (mixed_) {
      if (bw_.bytes() < A_.n * sizeof(double)) bw_.alloc(A_.n * sizeof(double));
      launchConvert(b, Wx, bw_.get(), W, static_cast<int>(A_.n), s());
    }
    const void* bW = mixed_ ? bw_.get() : b;
    if (ref && refTiles_.bytes() < 2 * static_cast<size_t>(A_.P) * sizeof(float))
      refTiles_.alloc(2 * static_cast<size_t>(A_.P) * sizeof(float));
    const size_t vb = A_.n * dtypeSize(W);
    KState init{};
    init.absTol = cfg_.absTolerance;
    init.relTol = cfg_.relTolerance;
    init.relRes = cfg_.relResidual;
    init.maxIter = cfg_.maxIterations;
    init.minIter = cfg_.minIterations;
    init.normKind = cfg_.norm;
    KState* st = st_.as<KState>();
    launchStateReset(st, init, s(), systems_);
    // The reference takes ||x|| here (pbicgstab/Solver.cpp:69-70); the norm
    // of b is what relTolerance is documented to use (SolverStats.hpp:52-60).
    if (cfg_.relTolerance > 0) {
      if (ref) {
        launchRefReduce(A_, RefRed{normRed(), b, nullptr}, RefRed{}, RefStage::BNorm, st, refTiles_.get(), s());
      } else if (!A_.batch) {
        launchNorm(A_, b, Wx, cfg_.norm, &st->bNorm, s());
      } else {
        for (int k = 0; k < systems_; ++k)
          launchNormN(A_, static_cast<const char*>(b) + A_.batch->rowBegin[k] * dtypeSize(W), A_.batch->rowReal[k], W,
                      cfg_.norm, &st[k].bNorm, s());
      }
    }
    if (mixed_) launchConvert(x, Wx, xw(), W, static_cast<int>(A_.n), s());
    else GR_CUDA(cudaMemcpyAsync(xw(), x, vb, cudaMemcpyDeviceToDevice, s()));
    launchBicgInit(A_, xw(), bW, buf(R), buf(R0), st, W, s(), ref);
    if (!skip_.empty()) launchSkipSystems(st, skipDev_.as<int>(), systems_, s());
    if (ref)
      launchRefReduce(A_, RefRed{RefKind::Dot, buf(R0), buf(R)}, RefRed{normRed(), buf(R), nullptr}, RefStage::Init,
                      st, refTiles_.get(), s());
    const bool graphable = ilu_ || !pre_ || (gs_ && cfg_.preconditioner->numFixedIterations > 0);
    const bool perIter = cfg_.printPerformanceEachIteration;
    int issued = 0;
    for (;;) {
      if (graphable && !perIter) {
        launchBatch(W);
        issued += kBatch;
      } else {
        iteration(W);
        issued += 1;
      }
      GR_CUDA(cudaMemcpyAsync(host_, st, sizeof(KState) * systems_, cudaMemcpyDeviceToHost, s()));
      // The matrix's error word rides along: a kernel whose bounded wait ran
      // out (or a status injected from the host) ends the solve here; the
      // tree reports it.
      GR_CUDA(cudaMemcpyAsync(errHost(), A_.errFlag.get(), sizeof(int), cudaMemcpyDeviceToHost, s()));
      GR_CUDA(cudaStreamSynchronize(s()));
      if (perIter) printStats(cfg_, A_, stats());
      if (*errHost() != 0) break;
      bool all = true;
      for (int k = 0; k < systems_; ++k) all = all && host_[k].done;
      if (all) break;
      if (issued > cfg_.maxIterations && issued > (1 << 30)) break;
    }
    if (mixed_) launchConvert(xw(), W, x, Wx, static_cast<int>(A_.n), s());  // exact: x holds float values
    else GR_CUDA(cudaMemcpyAsync(x, xw(), vb, cudaMemcpyDeviceToDevice, s()));
    GR_CUDA(cudaStreamSynchronize(s()));
    gr_stats out = stats();
    if (*errHost() != 0) {  // a device-side wait ran out (or an injected status)
      out.status = *errHost();
      out.converged = 0;
    }
    if (cfg_.printPerformanceAfterSolve) printStats(cfg_, A_, out);
    return out;
  }
  bool usesInitialGuess() const override { return true; }
  void refresh() override {
    if (pre_) pre_->refresh();
  }
  std::vector<gr_stats> batchStats() const override {
    std::vector<gr_stats> out(systems_);
    for (int k = 0; k < systems_; ++k) out[k] = statsOf(host_[k]);
    return out;
  }
  void setBatchSkip(const std::vector<int>& skip) override {
    if (!A_.batch) fail(GR_EINVAL, "skipping systems needs a batch");
    if (!skip.empty() && static_cast<int>(skip.size()) != systems_) fail(GR_EINVAL, "one skip flag per system");
    skip_ = skip;
    if (!skip_.empty()) {
      if (skipDev_.bytes() < sizeof(int) * systems_) skipDev_.alloc(sizeof(int) * systems_);
      GR_CUDA(cudaMemcpyAsync(skipDev_.get(), skip_.data(), sizeof(int) * systems_, cudaMemcpyHostToDevice, s()));
      GR_CUDA(cudaStreamSynchronize(s()));
    }
  }

 private:
  enum { X = 0, R, R0, P, V, Y, S, Z, T, NBUF };
  std::vector<int> skip_;
  DBuf skipDev_;
  int systems_ = 1;
  bool batchHost_ = false;
  std::unique_ptr<Node> pre_;
  IluNode* ilu_ = nullptr;
  GsNode* gs_ = nullptr;
  DBuf st_;
  KState* host_ = nullptr;
  DBuf vec_;
  DType bufType_ = DType::F32;
  bool haveBufs_ = false;
  cudaGraphExec_t exec_ = nullptr;
  DType graphType_ = DType::F32;
  int graphKernels_ = 0;

  void* buf(int i) { return static_cast<char*>(vec_.get()) + static_cast<size_t>(i) * A_.n * dtypeSize(bufType_); }
  DBuf refTiles_;  // per-tile values of the reference-order reductions
  DBuf bw_;        // b in the working type (workingType float64 over float32 vectors)
  bool mixed_ = false, graphMixed_ = false;
  RefKind normRed() const {
    return cfg_.norm == GR_NORM_L1 ? RefKind::Sum : (cfg_.norm == GR_NORM_LINF ? RefKind::Max : RefKind::SquareSum);
  }
  // Pinned host word for the matrix's error flag, after the states.
  int* errHost() { return reinterpret_cast<int*>(host_ + systems_); }
  void* xw() { return buf(X); }

  void ensureBuffers(DType W) {
    if (haveBufs_ && bufType_ == W) return;
    vec_.alloc(static_cast<size_t>(NBUF) * A_.n * dtypeSize(W));
    bufType_ = W;
    haveBufs_ = true;
    if (exec_) {
      cudaGraphExecDestroy(exec_);
      exec_ = nullptr;
    }
  }

  static gr_stats statsOf(const KState& h) {
    gr_stats o{};
    o.initial_residual = h.normInit;
    o.final_residual = h.normFinal;
    o.b_norm = h.bNorm;
    o.iterations = h.iter;
    o.converged = h.converged;
    o.singular = h.singular;
    o.status = h.status;
    return o;
  }
  // One system: its statistics. A batch: the slowest system's iterations,
  // converged / singular / status over all systems, system 0's norms.
  gr_stats stats() const {
    gr_stats o = statsOf(host_[0]);
    for (int k = 1; k < systems_; ++k) {
      o.iterations = std::max(o.iterations, host_[k].iter);
      o.converged = o.converged && host_[k].converged;
      o.singular = o.singular || host_[k].singular;
      if (o.status == GR_OK) o.status = host_[k].status;
    }
    return o;
  }

  // Applies the preconditioner to the prologue vector into out.
  void precondition(const PrologueArgs& pro, void* out, DType W) {
    KState* st = st_.as<KState>();
    if (ilu_) {
      ilu_->apply(pro, out, W);
      return;
    }
    if (!pre_) {
      launchPrologue(A_, pro, out, W, s());
      return;
    }
    if (gs_ && gs_->fusedPrologue()) {
      gs_->applyFused(pro, out, W);
      return;
    }
    launchPrologue(A_, pro, nullptr, W, s());
    const void* in = pro.pOrS;
    if (gs_) {
      gs_->solveFromZero(out, in, W, st);
      return;
    }
    if (pre_->usesInitialGuess()) GR_CUDA(cudaMemsetAsync(out, 0, A_.n * dtypeSize(W), s()));
    pre_->solve(out, in, W, st);
  }

  // One PBiCGStab iteration (pbicgstab/Solver.cpp:90-186).
  void iteration(DType W) {
    if (cfg_.reduceRef) {
      iterationRef(W);
      return;
    }
    KState* st = st_.as<KState>();
    PrologueArgs p;
    p.kind = Prologue::PUpdate;
    p.r = buf(R);
    p.pOrS = buf(P);
    p.v = buf(V);
    p.st = st;
    p.stIndex = A_.batch ? A_.batch->tileSys.as<int>() : nullptr;
    precondition(p, buf(Y), W);
    launchSpmvDot(A_, buf(Y), buf(V), buf(R0), 0, st, W, s());
    PrologueArgs q;
    q.kind = Prologue::SUpdate;
    q.r = buf(R);
    q.pOrS = buf(S);
    q.v = buf(V);
    q.st = st;
    q.stIndex = p.stIndex;
    precondition(q, buf(Z), W);
    launchSpmvDot(A_, buf(Z), buf(T), buf(S), 1, st, W, s());
    launchBicgUpdate(A_, xw(), buf(Y), buf(Z), buf(R), buf(S), buf(T), buf(R0), st, W, s(), false, mixed_);
  }

  // The same iteration with the reference's float reductions: the fused
  // kernels compute the vectors only, and each dot product / norm is a
  // reference-order reduction whose last step derives the scalars in float.
  void iterationRef(DType W) {
    KState* st = st_.as<KState>();
    void* tiles = refTiles_.get();
    PrologueArgs p;
    p.kind = Prologue::PUpdate;
    p.r = buf(R);
    p.pOrS = buf(P);
    p.v = buf(V);
    p.st = st;
    precondition(p, buf(Y), W);
    launchSpmvDot(A_, buf(Y), buf(V), buf(R0), 0, st, W, s(), true);
    launchRefReduce(A_, RefRed{RefKind::Dot, buf(R0), buf(V)}, RefRed{}, RefStage::Alpha, st, tiles, s());
    PrologueArgs q;
    q.kind = Prologue::SUpdate;
    q.r = buf(R);
    q.pOrS = buf(S);
    q.v = buf(V);
    q.st = st;
    precondition(q, buf(Z), W);
    launchSpmvDot(A_, buf(Z), buf(T), buf(S), 1, st, W, s(), true);
    launchRefReduce(A_, RefRed{RefKind::Dot, buf(T), buf(T)}, RefRed{RefKind::Dot, buf(T), buf(S)}, RefStage::Omega,
                    st, tiles, s());
    launchBicgUpdate(A_, xw(), buf(Y), buf(Z), buf(R), buf(S), buf(T), buf(R0), st, W, s(), true);
    launchRefReduce(A_, RefRed{RefKind::Dot, buf(R0), buf(R)}, RefRed{normRed(), buf(R), nullptr}, RefStage::Update,
                    st, tiles, s());
  }

  void launchBatch(DType W) {
    if (!exec_ || graphType_ != W || graphMixed_ != mixed_) {
      if (exec_) cudaGraphExecDestroy(exec_);
      exec_ = nullptr;
      cudaGraph_t g = nullptr;
      if (pre_) pre_->prepare(W);
      GR_CUDA(cudaStreamBeginCapture(s(), cudaStreamCaptureModeThreadLocal));
      setCapturing(true);
      int kernels = 0;
      try {
        const i64 c0 = capturedCount();
        for (int k = 0; k < kBatch; ++k) iteration(W);
        kernels = static_cast<int>(capturedCount() - c0);
      } catch (...) {
        setCapturing(false);
        cudaStreamEndCapture(s(), &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      setCapturing(false);
      GR_CUDA(cudaStreamEndCapture(s(), &g));
      GR_CUDA(cudaGraphInstantiate(&exec_, g, 0));
      cudaGraphDestroy(g);
      graphType_ = W;
      graphMixed_ = mixed_;
      graphKernels_ = kernels;
    }
    GR_CUDA(cudaGraphLaunch(exec_, s()));
    noteLaunch(graphKernels_);
  }
};

// ---------------------------------------------------------------------------
// Mixed-precision iterative refinement: the residual and the solution phi in
// the extended type E, the correction solve in the working type (float).
class MpirNode : public Node {
 public:
  MpirNode(DeviceMatrix& A, const SolverConfig& c) : Node(A, c), inner_(makeNode(A, *c.innerSolver)) {
    scal_.alloc(sizeof(double) * 4);
  }
  gr_stats solve(void* x, const void* b, DType W, const KState*) override {
    if (W != DType::F32)
      fail(GR_EUNSUPPORTED, "IterativeRefinement expects a float32 working precision (x and b)");
    E_ = cfg_.extendedPrecisionType < 0 ? W : static_cast<DType>(cfg_.extendedPrecisionType);
    if (A_.batch) return solveBatch(x, b);
    const int n = A_.n;
    gr_stats st{};
    double* d = scal_.as<double>();
    if (cfg_.relTolerance > 0) {
      launchNorm(A_, b, DType::F32, cfg_.norm, d + 1, s());
      GR_CUDA(cudaMemcpyAsync(&st.b_norm, d + 1, sizeof(double), cudaMemcpyDeviceToHost, s()));
    }
    if (r_.bytes() < n * sizeof(float)) r_.alloc(n * sizeof(float));
    if (phi_.bytes() < n * dtypeSize(E_)) phi_.alloc(n * dtypeSize(E_));
    float* r = r_.as<float>();
    // Initial residual of x in E, stored as float (iterative-refinement/Solver.cpp:79).
    launchResidual(A_, x, DType::F32, b, DType::F32, r, DType::F32, E_, cfg_.norm, d, s());
    st.initial_residual = st.final_residual = readScalar(d);
    launchCastUp(static_cast<const float*>(x), phi_.get(), E_, n, s());
    bool conv = false;
    int innerTotal = 0;
    while (!((conv && st.iterations >= cfg_.minIterations) || st.iterations >= cfg_.maxIterations)) {
      st.iterations += 1;
      if (inner_->usesInitialGuess()) GR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(float), s()));
      gr_stats is = inner_->solve(x, r, DType::F32, nullptr);
      innerTotal += is.inner_iterations > 0 ? is.inner_iterations : is.iterations;
      if (is.status != GR_OK) {  // the inner solve failed on the device: no correction to apply
        st.status = is.status;
        break;
      }
      launchPhiUpdate(phi_.get(), static_cast<const float*>(x), E_, n, s());
      launchResidual(A_, phi_.get(), E_, b, DType::F32, r, DType::F32, E_, cfg_.norm, d, s());
      st.final_residual = readScalar(d);
      conv = st.final_residual < cfg_.absTolerance || st.final_residual < st.initial_residual * cfg_.relResidual ||
             (cfg_.relTolerance > 0 && st.final_residual < st.b_norm * cfg_.relTolerance);
      if (!std::isfinite(st.final_residual)) {
        st.status = GR_ENONFINITE;
        break;
      }
      if (cfg_.printPerformanceEachIteration) {
        st.converged = conv;
        printStats(cfg_, A_, st);
      }
    }
    launchCastDown(phi_.get(), static_cast<float*>(x), E_, n, s());
    GR_CUDA(cudaStreamSynchronize(s()));
    st.converged = conv;
    st.inner_iterations = innerTotal;
    if (cfg_.printPerformanceAfterSolve) printStats(cfg_, A_, st);
    return st;
  }
  bool usesInitialGuess() const override { return true; }
  void refresh() override { inner_->refresh(); }
  void copyPhi(void* out, DType t) override {
    if (!phi_.get()) fail(GR_EINVAL, "no IterativeRefinement solve has run yet");
    launchConvert(phi_.get(), E_, out, t, A_.n, s());
    GR_CUDA(cudaStreamSynchronize(s()));
  }
  std::vector<gr_stats> batchStats() const override {
    if (batchStats_.empty()) fail(GR_EINVAL, "no batched IterativeRefinement solve has run yet");
    return batchStats_;
  }

 private:
  std::unique_ptr<Node> inner_;
  DType E_ = DType::F32;
  DBuf phi_, r_, scal_;
  std::vector<gr_stats> batchStats_;

  // The outer loop of every system of a batch at once
  // (iterative-refinement/Solver.cpp:48-123 per system): residuals and their
  // norms for all systems in one launch (each system reduced as it would
  // be alone), one batched inner solve for the systems still refining (the
  // others skipped: their correction stays zero and is not applied), phi
  // updated on the refining systems' rows only. A system's result equals
  // its solve alone.
  gr_stats solveBatch(void* x, const void* b) {
    const BatchSeg& B = *A_.batch;
    const int S = B.systems;
    const int n = A_.n;
    const size_t es = dtypeSize(E_);
    if (scal_.bytes() < sizeof(double) * (2 * static_cast<size_t>(S) + 4))
      scal_.alloc(sizeof(double) * (2 * static_cast<size_t>(S) + 4));
    double* d = scal_.as<double>();  // [0, S): residual norms, [S, 2S): norms of b
    if (r_.bytes() < n * sizeof(float)) r_.alloc(n * sizeof(float));
    if (phi_.bytes() < n * es) phi_.alloc(n * es);
    float* r = r_.as<float>();
    std::vector<double> res(S), bn(S, 0.0);
    auto readNorms = [&](const double* src, std::vector<double>& dst) {
      GR_CUDA(cudaMemcpyAsync(dst.data(), src, sizeof(double) * S, cudaMemcpyDeviceToHost, s()));
      GR_CUDA(cudaStreamSynchronize(s()));
    };
    if (cfg_.relTolerance > 0) {
      for (int k = 0; k < S; ++k)
        launchNormN(A_, static_cast<const float*>(b) + B.rowBegin[k], B.rowReal[k], DType::F32, cfg_.norm, d + S + k,
                    s());
      readNorms(d + S, bn);
    }
    launchResidual(A_, x, DType::F32, b, DType::F32, r, DType::F32, E_, cfg_.norm, d, s());
    readNorms(d, res);
    launchCastUp(static_cast<const float*>(x), phi_.get(), E_, n, s());
    batchStats_.assign(S, gr_stats{});
    std::vector<int> conv(S, 0), active(S, 1), skip(S, 0);
    auto finished = [&](int k) {
      return (conv[k] && batchStats_[k].iterations >= cfg_.minIterations) ||
             batchStats_[k].iterations >= cfg_.maxIterations;
    };
    for (int k = 0; k < S; ++k) {
      batchStats_[k].initial_residual = batchStats_[k].final_residual = res[k];
      batchStats_[k].b_norm = bn[k];
      if (finished(k)) active[k] = 0;
    }
    auto anyActive = [&]() { return std::find(active.begin(), active.end(), 1) != active.end(); };
    while (anyActive()) {
      for (int k = 0; k < S; ++k) {
        skip[k] = active[k] ? 0 : 1;
        if (active[k]) batchStats_[k].iterations += 1;
      }
      inner_->setBatchSkip(skip);
      if (inner_->usesInitialGuess()) GR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(float), s()));
      inner_->solve(x, r, DType::F32, nullptr);
      const std::vector<gr_stats> is = inner_->batchStats();
      for (int k = 0; k < S; ++k) {
        if (!active[k]) continue;
        batchStats_[k].inner_iterations += is[k].inner_iterations > 0 ? is[k].inner_iterations : is[k].iterations;
        if (is[k].status != GR_OK) {  // no correction to apply for this system
          batchStats_[k].status = is[k].status;
          active[k] = 0;
          continue;
        }
        launchPhiUpdate(static_cast<char*>(phi_.get()) + B.rowBegin[k] * es,
                        static_cast<const float*>(x) + B.rowBegin[k], E_, static_cast<int>(B.rowReal[k]), s());
      }
      launchResidual(A_, phi_.get(), E_, b, DType::F32, r, DType::F32, E_, cfg_.norm, d, s());
      readNorms(d, res);
      for (int k = 0; k < S; ++k) {
        if (!active[k]) continue;
        gr_stats& q = batchStats_[k];
        q.final_residual = res[k];
        conv[k] = q.final_residual < cfg_.absTolerance || q.final_residual < q.initial_residual * cfg_.relResidual ||
                  (cfg_.relTolerance > 0 && q.final_residual < q.b_norm * cfg_.relTolerance);
        if (!std::isfinite(q.final_residual)) {
          q.status = GR_ENONFINITE;
          active[k] = 0;
        } else if (finished(k)) {
          active[k] = 0;
        }
      }
    }
    inner_->setBatchSkip({});
    launchCastDown(phi_.get(), static_cast<float*>(x), E_, n, s());
    GR_CUDA(cudaStreamSynchronize(s()));
    gr_stats out = gr_stats{};
    out.converged = 1;
    for (int k = 0; k < S; ++k) {
      gr_stats& q = batchStats_[k];
      q.converged = conv[k];
      if (k == 0) {
        out.initial_residual = q.initial_residual;
        out.final_residual = q.final_residual;
        out.b_norm = q.b_norm;
      }
      out.iterations = std::max(out.iterations, q.iterations);
      out.inner_iterations = std::max(out.inner_iterations, q.inner_iterations);
      out.converged = out.converged && q.converged;
      if (out.status == GR_OK) out.status = q.status;
    }
    return out;
  }
  double readScalar(const double* d) {
    double v = 0;
    GR_CUDA(cudaMemcpyAsync(&v, d, sizeof(double), cudaMemcpyDeviceToHost, s()));
    GR_CUDA(cudaStreamSynchronize(s()));
    return v;
  }
};

// ---------------------------------------------------------------------------
class RestarterNode : public Node {
 public:
  RestarterNode(DeviceMatrix& A, const SolverConfig& c) : Node(A, c), inner_(makeNode(A, *c.innerSolver)) {}
  gr_stats solve(void* x, const void* b, DType W, const KState* gate) override {
    int restarts = 0;
    gr_stats st = inner_->solve(x, b, W, gate);
    int total = st.iterations;
    while (restarts < cfg_.maxRestarts && !st.converged && st.status == GR_OK) {
      restarts += 1;
      st = inner_->solve(x, b, W, gate);
      total += st.iterations;
    }
    st.inner_iterations = total;
    return st;
  }
  bool usesInitialGuess() const override { return inner_->usesInitialGuess(); }
  void copyPhi(void* out, DType t) override { inner_->copyPhi(out, t); }
  void refresh() override { inner_->refresh(); }

 private:
  std::unique_ptr<Node> inner_;
};

std::unique_ptr<Node> makeNode(DeviceMatrix& A, const SolverConfig& c) {
  if (c.type == "GaussSeidel") return std::make_unique<GsNode>(A, c);
  if (c.type == "IterativeRefinement") return std::make_unique<MpirNode>(A, c);
  if (c.type == "ILU") return std::make_unique<IluNode>(A, c);
  if (c.type == "PBiCGStab") return std::make_unique<PbicgstabNode>(A, c);
  if (c.type == "restarter") return std::make_unique<RestarterNode>(A, c);
  fail(GR_EPARSE, "Unknown solver: " + c.type);
}

class Tree : public SolverTree {
 public:
  Tree(DeviceMatrix& A, std::unique_ptr<SolverConfig> c) : A_(A), cfg_(std::move(c)) {
    root_ = makeNode(A, *cfg_);
    GR_CUDA(cudaEventCreate(&e0_));
    GR_CUDA(cudaEventCreate(&e1_));
  }
  ~Tree() override {
    // The nodes' buffers are released after this body: no work using them
    // may still be pending on the matrix's stream.
    cudaStreamSynchronize(A_.stream);
    cudaEventDestroy(e0_);
    cudaEventDestroy(e1_);
  }
  gr_stats solve(void* x, DType xt, const void* b, DType bt) override {
    if (xt != bt) fail(GR_EINVAL, "x and b must have the same type");
    if (xt == DType::DW) fail(GR_EUNSUPPORTED, "twofloat32 x / b");
    GR_CUDA(cudaEventRecord(e0_, A_.stream));
    gr_stats st = root_->solve(x, b, xt, nullptr);
    GR_CUDA(cudaEventRecord(e1_, A_.stream));
    GR_CUDA(cudaEventSynchronize(e1_));
    float ms = 0;
    GR_CUDA(cudaEventElapsedTime(&ms, e0_, e1_));
    st.solve_ms = ms;
    // A bounded device-side wait that ran out marks the solve as failed.
    int err = 0;
    GR_CUDA(cudaMemcpyAsync(&err, A_.errFlag.get(), sizeof(int), cudaMemcpyDeviceToHost, A_.stream));
    GR_CUDA(cudaStreamSynchronize(A_.stream));
    if (err != 0) {
      GR_CUDA(cudaMemsetAsync(A_.errFlag.get(), 0, sizeof(int), A_.stream));
      st.status = err;
      st.converged = 0;
    }
    return st;
  }
  float timeRepeated(void* x, DType xt, const void* b, DType bt, int reps) override {
    if (xt != bt) fail(GR_EINVAL, "x and b must have the same type");
    if (xt == DType::DW) fail(GR_EUNSUPPORTED, "twofloat32 x / b");
    if (reps < 1 || reps > 100000) fail(GR_EINVAL, "reps must be 1..100000");
    if (cfg_->type != "ILU" && !(cfg_->type == "GaussSeidel" && cfg_->numFixedIterations > 0))
      fail(GR_EUNSUPPORTED, "repeated timing is for ILU and fixed-sweep Gauss-Seidel solvers");
    GR_CUDA(cudaEventRecord(e0_, A_.stream));
    for (int i = 0; i < reps; ++i) root_->solve(x, b, xt, nullptr);
    GR_CUDA(cudaEventRecord(e1_, A_.stream));
    GR_CUDA(cudaEventSynchronize(e1_));
    float ms = 0;
    GR_CUDA(cudaEventElapsedTime(&ms, e0_, e1_));
    int err = 0;
    GR_CUDA(cudaMemcpyAsync(&err, A_.errFlag.get(), sizeof(int), cudaMemcpyDeviceToHost, A_.stream));
    GR_CUDA(cudaStreamSynchronize(A_.stream));
    if (err != 0) {
      GR_CUDA(cudaMemsetAsync(A_.errFlag.get(), 0, sizeof(int), A_.stream));
      fail(err, "a device-side wait ran out during the repeated runs");
    }
    return ms / static_cast<float>(reps);
  }
  gr_stats solveHost(void* x, DType xt, const void* b, DType bt) override {
    if (xt != bt) fail(GR_EINVAL, "x and b must have the same type");
    const size_t bytes = A_.n * dtypeSize(xt);
    void* tmp = A_.staging(0, bytes);
    void* xd = A_.staging(1, bytes);
    void* bd = A_.staging(2, bytes);
    cudaStream_t s = A_.stream;
    GR_CUDA(cudaMemcpyAsync(tmp, b, bytes, cudaMemcpyHostToDevice, s));
    launchPermute(A_, tmp, bd, xt, true, s);
    GR_CUDA(cudaMemcpyAsync(tmp, x, bytes, cudaMemcpyHostToDevice, s));
    launchPermute(A_, tmp, xd, xt, true, s);
    gr_stats st = solve(xd, xt, bd, bt);
    launchPermute(A_, xd, tmp, xt, false, s);
    GR_CUDA(cudaMemcpyAsync(x, tmp, bytes, cudaMemcpyDeviceToHost, s));
    GR_CUDA(cudaStreamSynchronize(s));
    return st;
  }
  void copyPhi(void* out, DType t) override { root_->copyPhi(out, t); }
  std::vector<gr_stats> batchStats() const override { return root_->batchStats(); }
  std::string name() const override { return cfg_->solverName(); }
  void refresh() override {
    root_->refresh();
    GR_CUDA(cudaStreamSynchronize(A_.stream));
  }

 private:
  DeviceMatrix& A_;
  std::unique_ptr<SolverConfig> cfg_;
  std::unique_ptr<Node> root_;
  cudaEvent_t e0_ = nullptr, e1_ = nullptr;
};

}  // namespace

std::unique_ptr<SolverTree> SolverTree::create(DeviceMatrix& A, const std::string& json) {
  auto cfg = SolverConfig::fromText(json);
  return std::make_unique<Tree>(A, std::move(cfg));
}

}  // namespace gr
