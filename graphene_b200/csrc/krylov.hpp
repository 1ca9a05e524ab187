// Device-resident solver state and the launchers of the preconditioner and
// Krylov kernels.
#pragma once

#include "device.hpp"

namespace gr {

// Scalars of one PBiCGStab / Gauss-Seidel solve, kept in device memory so
// that no iteration needs a host round trip. Written only by the last block
// of a grid reduction (or a single-thread kernel); read by the kernels that
// follow in stream order. Reductions accumulate in FP64.
struct KState {
  double rho, rhoOld, alpha, omega, beta;
  double normInit, normFinal, bNorm;
  double dot0, dot1;
  // configuration (SolverStats tolerances are floats in the reference)
  double absTol, relTol, relRes;
  int maxIter, minIter, normKind;
  // progress
  int iter, converged, singular, done, status;
  int pad[2];
};

// Prologue of a fused preconditioner application (the vector the
// preconditioner is applied to).
enum class Prologue : int {
  Plain = 0,   // b
  PUpdate = 1, // p = r (iteration 0) or p = r + beta (p - omega v); writes p
  SUpdate = 2  // s = r - alpha v; writes s
};

struct PrologueArgs {
  Prologue kind = Prologue::Plain;
  const void* b = nullptr;  // Plain: the right-hand side
  const void* r = nullptr;
  void* pOrS = nullptr;     // p (read and written) or s (written)
  const void* v = nullptr;
  const KState* st = nullptr;  // scalars; also the early-exit flag (may be null)
  const int* stIndex = nullptr;  // batches: state index per tile (ring kernel only)
};

// ---- ILU(0) / DILU ----------------------------------------------------
// F: tile-local CRS values (in / out), D: diagonal (in, factored in place).
void launchIluFactor(DeviceMatrix& A, void* F, void* D, const void* Aoff, bool dilu, cudaStream_t s);
// inv = 1 / D
void launchInvert(DeviceMatrix& A, const void* D, void* inv, cudaStream_t s);
// Packs the slot values of schedule S (out, S.slots entries) from the
// tile-local CRS values F.
void launchPack(DeviceMatrix& A, const LevelSchedule& S, const void* F, void* out, cudaStream_t s);
// y = M^-1 * prologue; vectors of type W. Lval / Uval: packed values of the
// Lower / UpperDesc schedules.
void launchIluApply(DeviceMatrix& A, const void* Lval, const void* Uval, const void* inv, bool dilu,
                    const PrologueArgs& pro, void* y, DType W, cudaStream_t s);

// Streamed substitution (kernels_stream.cu). iluStreamSmem returns the
// dynamic shared memory a launch with vector type W needs, 0 if the
// matrix's levels are too large for the ring.
// ringLog2: requested ring size (0 = the smallest that fits).
size_t iluStreamSmem(const DeviceMatrix& A, const SweepStream& S, DType W, int ringLog2 = 0);
int iluStreamRingLog2(const SweepStream& S, int requested);
// stream = template with the factor values F and inverse diagonal inv packed in.
void launchStreamPack(DeviceMatrix& A, const SweepStream& S, void* stream, const void* F, const void* inv,
                      cudaStream_t s);
// Tuning of the streamed kernel: ring size (log2 bytes, 0 = the smallest
// that fits), ring chunks kept prefetched into L2 beyond the ring (-1 = the
// default), and whether rows of up to four entries load all their terms at
// once.
struct StreamTuning {
  int ringLog2 = 0;
  int prefetchChunks = -1;
  bool unroll = false;
};
void launchIluStream(DeviceMatrix& A, const SweepStream& S, const void* stream, bool dilu,
                     const PrologueArgs& pro, void* y, DType W, const StreamTuning& tune, cudaStream_t s);
int maxDynamicSmem(const DeviceMatrix& A);
// Copies a stream template and packs factor values F and the inverse
// diagonal inv into it (element positions in units of the value type).
void launchPackBytes(DeviceMatrix& A, const void* templ, i64 bytes, const int* valPos, const int* valSrc, i64 nVal,
                     const int* invPos, const int* invSrc, i64 nInv, void* stream, const void* F, const void* inv,
                     cudaStream_t s);
// Host-scheduled ring substitution (kernels_ring.cu): dynamic shared memory
// per block, packing of a solver's copy of the level blocks, and the launch.
// Blocks of the ring kernel (value type vt) an SM holds when shared memory
// is not the limit (0 if unknown).
int ringBlocksPerSMWithoutSmem(DType vt, RingKind kind = RingKind::Ilu);
size_t iluRingSmem(const DeviceMatrix& A, const LevelRing& R, DType W);
// Blocks of the ring substitution kernel resident per SM for vectors of
// type W with the default compute warps (computeWarps 0) or four.
int iluRingBlocksPerSM(const DeviceMatrix& A, const LevelRing& R, DType W, int computeWarps);
void launchRingPack(DeviceMatrix& A, const LevelRing& R, void* stream, const void* F, const void* inv,
                    cudaStream_t s);
// l2Ahead: bytes kept prefetched into L2 beyond the issued copies (-1:
// default); unroll: rows of up to four entries load all their terms at once.
// The same substitution with one warp per tile (iluWarpRingKernel):
// dynamic shared memory of a block of warpsPerBlock tiles, and the launch.
size_t iluWarpRingSmem(const LevelRing& R, DType W, int warpsPerBlock);
void launchIluWarpRing(DeviceMatrix& A, const LevelRing& R, const void* stream, bool dilu, const PrologueArgs& pro,
                       void* y, DType W, int warpsPerBlock, bool pairRows, cudaStream_t s);
// pairRows: record levels process two rows a thread at once; producer
// false: the waiting warp issues the level copies (no producer warp).
void launchIluRing(DeviceMatrix& A, const LevelRing& R, const void* stream, bool dilu, const PrologueArgs& pro,
                   void* y, DType W, int l2Ahead, bool unroll, cudaStream_t s, bool pairRows = false, int computeWarps = 0,
                   bool waiter = true, bool producer = true);
// One Gauss-Seidel sweep through a Gauss-Seidel level ring (kernels_ring.cu):
// xout from xin (xinZero: xin is all zeros and is not read; the ring may
// then be a lower-only one). The right-hand side is the prologue's vector
// (seedB), or each row starts from its diagonal (seedB false, the
// reference's CodeDSL solver, gauss-seidel/Solver.cpp:74). stream: the ring
// template with the coefficients and the diagonal packed in. Vectors of
// type X, rows computed in W (X, or float64 over float32 vectors).
// warps > 0: the warp-per-tile form (gsWarpRingKernel) with `warps` tiles a
// block (pairRows: a lane takes two rows of a level at once);
// gsWarpRingSmem gives its dynamic shared memory.
void launchGsRing(DeviceMatrix& A, const LevelRing& R, const void* stream, const PrologueArgs& pro, bool seedB,
                  const void* xin, bool xinZero, void* xout, DType X, DType W, cudaStream_t s, int warps = 0,
                  bool dropHalo = false, bool pairRows = false);
size_t gsWarpRingSmem(const LevelRing& R, DType W, int warpsPerBlock);
// Warp-per-tile substitution (kernels_warp.cu): shared memory per block and
// the number of rows per lane to prefetch.
size_t iluWarpSmem(const DeviceMatrix& A, const SweepStream& S, DType W);
int iluWarpRowsPerLane(const DeviceMatrix& A, const SweepStream& S);
void launchIluWarp(DeviceMatrix& A, const SweepStream& S, const void* stream, bool dilu, const PrologueArgs& pro,
                   void* y, DType W, int J, cudaStream_t s);

// ---- Gauss-Seidel -------------------------------------------------------
// One sweep: xout from xin (xin may alias nothing; must differ from xout).
// seedB: start each row from b (true) or from the diagonal (false).
// Gval: packed values of the All schedule.
void launchGsSweep(DeviceMatrix& A, const void* Gval, const void* b, bool seedB, const void* xin,
                   bool xinZero, void* xout, DType W, const KState* st, cudaStream_t s,
                   bool dropHalo = false);

// ---- Krylov kernels ----------------------------------------------------
// r = b - A x, r0 = r; state initialised (norm, rho = r0.r, flags).
// stateless (this and the next two): the vectors only, no reduction and no
// state update (the reference-order reductions below do those).
void launchBicgInit(DeviceMatrix& A, const void* x, const void* b, void* r, void* r0, KState* st,
                    DType W, cudaStream_t s, bool stateless = false);
// y = A x and the dots of the step: mode 0: alpha = rho / (r0 . y);
// mode 1: omega = (y . s) / (y . y), singularity check.
void launchSpmvDot(DeviceMatrix& A, const void* x, void* y, const void* d1, int mode, KState* st,
                   DType W, cudaStream_t s, bool stateless = false);
// x = x + alpha y + omega z; r = s - omega t; convergence; next rho, beta.
void launchBicgUpdate(DeviceMatrix& A, void* x, const void* y, const void* z, void* r, const void* sv,
                      const void* t, const void* r0, KState* st, DType W, cudaStream_t s, bool stateless = false,
                      bool roundX = false);

// ---- the reference's reduction order ("reduce": "f32_ref_order") -------
// A reduction over the non-halo rows, per tile in the reference's order
// (six worker chunks, then the partials; dsl/tensor/Expression.cpp:472-481,
// :597-646) and across tiles in runs of 368, 736, 1472 and all tiles
// (:680-769), accumulating in float.
enum class RefKind : int { None = 0, Dot = 1, SquareSum = 2, Sum = 3, Max = 4 };
struct RefRed {
  RefKind kind = RefKind::None;
  const void* a = nullptr;
  const void* b = nullptr;  // Dot: a . b
};
// What the reduced values update in the state (one thread):
//  BNorm:  bNorm = norm(q0)
//  Init:   rho = q0 (r0 . r), normInit = normFinal = norm(q1), flags
//  Alpha:  alpha = rho / q0
//  Omega:  omega = q1 / q0 (q0 = t . t, q1 = t . s), singularity
//  Update: normFinal = norm(q1), convergence, iteration count, next rho
//          = q0 and beta, singularity
// Norms are rounded to float and compared in float, as the reference's
// SolverStats tensors are (SolverStats.hpp:33-36).
enum class RefStage : int { BNorm = 0, Init = 1, Alpha = 2, Omega = 3, Update = 4 };
// tiles: scratch of 2 P floats.
void launchRefReduce(DeviceMatrix& A, const RefRed& q0, const RefRed& q1, RefStage stage, KState* st, void* tiles,
                     cudaStream_t s);
// Elementwise prologue when no fused preconditioner is used; also copies
// the result into copyTo when non-null.
void launchPrologue(DeviceMatrix& A, const PrologueArgs& pro, void* copyTo, DType W, cudaStream_t s);
// Writes the initial state (single thread).
void launchStateReset(KState* st, const KState& init, cudaStream_t s, int count = 1);
// Batches: marks the systems whose skip[k] is nonzero done (their kernels
// then return at once and their x stays as it is).
void launchSkipSystems(KState* st, const int* skip, int count, cudaStream_t s);
// Norm of a vector into st->bNorm.
void launchNormInto(DeviceMatrix& A, const void* x, DType t, int normKind, double* out, cudaStream_t s);

// ---- mixed precision --------------------------------------------------
// phi (E) = x (float)
void launchCastUp(const float* x, void* phi, DType E, int n, cudaStream_t s);
// phi = phi + corr in E arithmetic
void launchPhiUpdate(void* phi, const float* corr, DType E, int n, cudaStream_t s);
// x = (float) phi
void launchCastDown(const void* phi, float* x, DType E, int n, cudaStream_t s);
// dst (t) = phi (E) converted
void launchConvert(const void* src, DType from, void* dst, DType to, int n, cudaStream_t s);

}  // namespace gr
