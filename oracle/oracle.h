/*
 * CPU oracle for the graphene_b200 sparse-solver hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain C++ restatement of the
 * reference's algorithms (esa-tu-darmstadt/graphene, libgraphene/matrix),
 * used by tests/ as the parity checker and by bench.py as the timed CPU
 * baseline. The product library never links, loads or calls it.
 *
 * Parity pinning: the reference ships no golden vectors for this path
 * (its only result-pinning tests are the tensor reductions in
 * dsl/tensor/tests/TensorTests.cpp:136-261, 377-425); the reference cannot be
 * built here (Poplar SDK, METIS, Boost and the twofloat submodule are
 * absent). The oracle is therefore pinned by those reduction tests, by
 * hand-derived known answers and by scipy FP64 cross-checks (tests/golden).
 *
 * Vectors crossing this interface are in tile order without halo cells
 * (the decomposed vector layout of DistributedTileLayout.cpp:156-183);
 * internally the oracle keeps the reference's per-tile vectors with halo
 * cells and performs the halo exchange explicitly.
 */
#ifndef GRAPHENE_ORACLE_H
#define GRAPHENE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_matrix or_matrix;

/* Restates CRSHostMatrix(TripletMatrix, numTiles) after METIS: sorts the
 * triplets, converts to CRS with split diagonal, removes empty parts of
 * row_to_tile (raw part ids in [0, num_tiles)), builds tile layouts, local
 * addressings, colours. value_type: 0 float32, 1 float64. */
or_matrix* or_build(int64_t n, int64_t nnz, const int64_t* rows, const int64_t* cols,
                    const double* vals, int64_t num_tiles, const int32_t* row_to_tile,
                    int value_type);
/* An LDU matrix (LDUMatrix.hpp, LDUAddressing.hpp:42-91): faces with owner <
 * neighbour sorted by owner, lower / upper coefficients in face order (upper
 * NULL: upper = lower), diag. Built like or_build from the equivalent
 * triplets; SpMV and residual then run the reference's LDU row loops
 * (LDUMatrix.cpp:42-168) over per-tile LDU addressing. */
or_matrix* or_build_ldu(int64_t n, int64_t num_faces, const int64_t* owner, const int64_t* neighbour,
                        const double* diag, const double* lower, const double* upper, int64_t num_tiles,
                        const int32_t* row_to_tile, int value_type);
/* generate3DPoissonTripletMatrix (Poisson.cpp:26-69) then or_build. */
or_matrix* or_poisson(int64_t nx, int64_t ny, int64_t nz, int64_t num_tiles,
                      const int32_t* row_to_tile, int value_type);
void or_free(or_matrix* A);
const char* or_last_error(void);

/* Set the number of host threads used for per-tile loops (default 1). */
void or_set_threads(int threads);

int64_t or_num_rows(const or_matrix* A);
int64_t or_num_tiles(const or_matrix* A);
int64_t or_num_off_diag(const or_matrix* A);
int64_t or_num_halo(const or_matrix* A);
int or_row_to_tile(const or_matrix* A, int32_t* out);
int or_tile_sizes(const or_matrix* A, int64_t* out);            /* 3 per tile */
int or_local_to_global(const or_matrix* A, int64_t* out);       /* n + halo */
int or_local_crs(const or_matrix* A, int64_t* row_ptr, int32_t* col_ind, double* off_diag,
                 double* diag);
int or_colors(const or_matrix* A, int32_t* color);              /* tile order */
int or_multicolor_recommended(const or_matrix* A);

/* CRSMatrix::spmv with destType = intermediateType = t (0 f32, 1 f64). */
int or_spmv(const or_matrix* A, const void* x, void* y, int t);
/* CRSMatrix::residual: x of type xt (0 f32, 1 f64, 2 double-word pairs),
 * b of type bt, r of type rt, intermediate it. */
int or_residual(const or_matrix* A, const void* x, int xt, const void* b, int bt, void* r, int rt,
                int it);
/* Matrix::vectorNorm with FP64 accumulation. norm: 0 L1, 1 L2, 2 LINF. */
double or_norm(const or_matrix* A, const void* x, int t, int norm);
/* Reduction known-answer helper: sum of x[0..n) in FP64 (and FP32 when
 * f32 != 0, in the reference's per-worker chunk order of
 * Expression.cpp:472-481 for one tile). */
double or_reduce_sum(const float* x, int64_t n, int f32);
/* Dot product a . b and norm (0 L1, 1 L2, 2 LINF) of tile-ordered vectors
 * of type t (0 f32, 1 f64) in the reference's reduction order and operand
 * type (Expression.cpp:472-481, :597-769; see refReduce). */
double or_ref_dot(const or_matrix* A, const void* a, const void* b, int t);
double or_ref_norm(const or_matrix* A, const void* x, int t, int norm);

/* ILU(0) / DILU factorisation (ilu/Solver.cpp:134-292): writes the factored
 * off-diagonal values (tile-local CRS order, m entries) and the inverted
 * diagonal (tile order) in the stored coefficient type converted to double. */
int or_ilu_factorize(const or_matrix* A, int dilu, double* off_diag_out, double* inv_diag_out);
/* ilu solveCRS (ilu/Solver.cpp:367-550), sequential, x = M^-1 b, vector type t. */
int or_ilu_solve(const or_matrix* A, int dilu, const double* factor_off, const double* inv_diag,
                 const void* b, void* x, int t);
/* One Gauss-Seidel sweep (gauss-seidel/Solver.cpp:45-86) with halo exchange
 * at the start. seed_b: 1 seeds each row with b (the codelet spec,
 * codelet/ipu/matrix/solvers/gauss-seidel.cpp:44), 0 with the diagonal as the
 * reference's CodeDSL version does (gauss-seidel/Solver.cpp:74). */
int or_gs_sweep(const or_matrix* A, void* x, const void* b, int t, int seed_b, int drop_halo);

typedef struct {
  double initial_residual, final_residual, b_norm;
  int32_t iterations, converged, singular, inner_iterations;
} or_stats;

/* Runs a solver tree given as JSON (same schema as gr_solver_create) on
 * tile-ordered host vectors. x: in/out. For IterativeRefinement, phi_out
 * (nullable, double, n) receives the extended-precision solution. */
int or_solve(const or_matrix* A, const char* json, void* x, int xt, const void* b, int bt,
             or_stats* stats, double* phi_out, double* history, int history_len);

/* ---- seeded benchmark inputs (oracle/generators.cpp) ----------------------
 * The benchmark's synthetic inputs, restated for the oracle so that its
 * reference arm needs no part of the product library. */
/* Triplet count of a 7-point matrix on an nx x ny x nz grid. */
int64_t or_generate_nnz(int64_t nx, int64_t ny, int64_t nz);
/* Triplets sorted by (row, column) and grid coordinates (3 per row,
 * nullable) of kind 0 (constant Poisson, Poisson.cpp:26-69), 1
 * (variable-coefficient Poisson, params[0] = sigma) or 2 (upwind
 * convection-diffusion, params = velocity). */
int or_generate(int kind, int64_t nx, int64_t ny, int64_t nz, const double* params, uint64_t seed,
                int64_t* rows, int64_t* cols, double* vals, double* coords);
/* Seeded vector: dist 0 uniform [lo, hi), 1 standard normal. */
int or_random_vector(uint64_t seed, int64_t n, int dist, double lo, double hi, double* out);
/* Recursive coordinate bisection into `parts` parts (raw part ids). */
int or_partition_rcb(int64_t n, const double* coords, const int64_t* weights, int32_t parts, int32_t* out);

#ifdef __cplusplus
}
#endif

#endif
