// Solver configuration tree, parsed from the reference's JSON schema
// (matrix/solver/Configuration.cpp:103-136 and the per-solver
// Configuration.cpp files). JSON comments are accepted, as
// nlohmann::json::parse(..., allow_comments=true) does in the reference's
// benchmark (applications/benchmark/benchmark.cpp:117-118). Unknown keys are
// ignored like the reference does; they are collected in `unknownKeys` so the
// caller can report them.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.hpp"

namespace gr {

// A parsed JSON value. Scalars keep their source text, like a property tree.
struct Json {
  enum Kind { Null, Bool, Number, String, Object, Array } kind = Null;
  std::string text;
  std::vector<std::pair<std::string, Json>> members;
  std::vector<Json> items;
  const Json* find(const std::string& key) const;
  static Json parse(const std::string& src);
};

enum class MultiColorMode { Off, On, Auto };  // solver/Configuration.hpp:27

struct SolverConfig {
  std::string type;  // PBiCGStab | ILU | GaussSeidel | IterativeRefinement | restarter
  // SolverStats tolerances (pbicgstab/Configuration.hpp:14-23 and siblings).
  float absTolerance = 0, relTolerance = 0, relResidual = 0;
  int maxIterations = 2147483647, minIterations = 0;
  bool printPerformanceAfterSolve = false, printPerformanceEachIteration = false;
  bool verbose = false;
  int norm = GR_NORM_L2;
  int workingType = -1;  // -1: the type of x
  // ILU (ilu/Configuration.hpp:13-15)
  MultiColorMode solveMulticolor = MultiColorMode::Auto;
  MultiColorMode factorizeMulticolor = MultiColorMode::Auto;
  bool diagonalBased = false;
  // Extension: substitution kernel, "auto" (the host-scheduled ring kernel
  // when a tile fits shared memory, else the level-schedule kernel), "ring",
  // "tma" (chunked byte ring with a producer warp), "warp" (warp per tile)
  // or "levels".
  int iluKernel = 0;  // 0 auto, 1 tma, 2 levels, 3 warp, 4 ring, 5 warp-per-tile ring
  int warpsPerBlock = 1;  // tiles (warps) per block of the warp-per-tile ring kernel
  // Extension: shared-memory ring bytes of the "ring" kernel (0: default).
  long long ringBytes = 0;
  // Extension: bytes the "ring" kernel keeps prefetched into L2 beyond its
  // issued copies (-1: default).
  int l2Ahead = -1;
  // Extension: tiles one thread block of the "ring" kernel runs in lockstep
  // (0: default).
  int tilesPerBlock = 0;
  // Extension: whether the "ring" kernel may use 16-bit row and column ids
  // (blocks of at most 65535 rows): a level stream about a quarter smaller
  // in HBM, at one more shared-memory load per entry. On by default: on
  // B200 at 192^3 with 2048 tiles it ran in 111.0 us against 116.8 for the
  // 32-bit layout.
  bool compactRing = true;
  // Level rings: 16-byte row records for the levels of 3 entries a row
  // (ILU and Gauss-Seidel "recordLevels"). On by default: on B200 at 192^3
  // with 2048 tiles the ILU(0) substitution ran in 108.6 us against 117.0
  // without, with identical results.
  bool ringRecords = true;
  // ILU "pairRows": in record levels each thread computes two rows at once.
  bool pairRows = false;
  // ILU "computeWarps" of the block ring kernel (0: 2 for float, 4 for
  // double working vectors; or 1, 2, 4, 8).
  int computeWarps = 0;
  // ILU "waitingWarp": false lets the compute warps wait for each level's
  // copy themselves (no waiting warp; default computeWarps only).
  bool waitingWarp = true;
  // ILU "producerWarp": false lets the waiting warp issue the level copies
  // after each level's barrier (no producer warp).
  bool producerWarp = true;
  // Extension: log2 of the streamed kernel's ring size in bytes (0: the
  // smallest ring that holds the largest level).
  int ringLog2 = 0;
  // Extensions: ring chunks the streamed kernel keeps prefetched into L2
  // beyond its ring (-1: default), and whether it loads all terms of short
  // rows at once.
  int prefetchChunks = -1;
  int unrollRows = -1;  // -1: the kernel's default, 0 off, 1 on
  // GaussSeidel (gauss-seidel/Configuration.hpp:19-21)
  int numSweeps = 1, numFixedIterations = 0;
  // Extension: "seed": "b" (default, the codelet specification
  // codelet/ipu/matrix/solvers/gauss-seidel.cpp:44) or "diag" (the CodeDSL
  // version, gauss-seidel/Solver.cpp:74).
  bool gsSeedB = true;
  // Extension: "halo": "stale" (default, the reference: the halo cells keep
  // the values of the sweep's start, gauss-seidel/Solver.cpp:61) or "drop"
  // (they read as 0: block Gauss-Seidel without couplings between tiles).
  bool gsDropHalo = false;
  // Extension: GaussSeidel "pairRows" of the warp-per-tile ring kernel (a
  // lane takes two rows of a level at once; false by default: one row at a
  // time measured faster on B200, 43.1 against 50.3 us a sweep at 128^3).
  bool gsPairRows = false;
  // PBiCGStab "reduce": false (default, "float64"): dot products and norms
  // accumulate in FP64; true ("f32_ref_order"): in float, in the reference's
  // own reduction order (dsl/tensor/Expression.cpp:472-481, :597-769), with
  // alpha, beta, omega and the convergence test in float, as the reference
  // computes them (float32 vectors only).
  bool reduceRef = false;
  // Gauss-Seidel sweep kernel: 0 auto (the level ring with one warp per
  // tile for float coefficients when a tile fits shared memory, a block per
  // tile for double coefficients and in batches), 1
  // the level ring with a block per tile, 2 level schedules in global
  // memory, 3 the level ring with one warp per tile.
  int gsKernel = 0;
  // IterativeRefinement (iterative-refinement/Configuration.hpp:23-25)
  int extendedPrecisionType = -1;  // -1: the type of x
  // restarter (restarter/Configuration.hpp:14)
  int maxRestarts = 1;
  std::unique_ptr<SolverConfig> preconditioner, innerSolver;
  std::vector<std::string> unknownKeys;

  std::string solverName() const;
  static std::unique_ptr<SolverConfig> fromJson(const Json& j);
  static std::unique_ptr<SolverConfig> fromText(const std::string& text);
};

}  // namespace gr
