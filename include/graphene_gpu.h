/*
 * graphene_gpu.h -- C ABI of the B200 sparse-solver hot path.
 *
 * This is the drop-in boundary for Graphene's matrix / solver surface
 * (libgraphene/matrix). Every entry point below names the reference
 * interface it replaces. The reference is a C++ graph-building API whose
 * calls record work that runs later on the IPU; here every call executes
 * immediately on the GPU (or on the host for matrix construction).
 *
 * Conventions
 *  - Every function returns an int status (GR_OK == 0). On failure
 *    gr_last_error() returns a thread-local message. No C++ exception
 *    crosses this boundary.
 *  - Handles are opaque and own their memory; release them with the
 *    matching *_destroy function. A device matrix keeps its host matrix
 *    alive (the reference's MatrixBase holds a reference to the host layout,
 *    matrix/details/MatrixBase.hpp:38).
 *  - Device vectors are in "tile order": the concatenation over tiles of
 *    each tile's interior rows followed by its separator rows, i.e. the
 *    reference's decomposed vector layout without halo cells
 *    (matrix/host/DistributedTileLayout.cpp:156-183). Halo cells are not
 *    stored: a kernel reads a neighbour tile's value directly from HBM,
 *    which is what the reference's halo exchange copies
 *    (matrix/details/MatrixBase.cpp:36-109).
 *  - Host vectors passed to gr_vector_decompose / gr_vector_compose are in
 *    natural (global row) order.
 *  - All device work of a matrix and of the solvers built on it runs on
 *    that matrix's CUDA stream (gr_matrix_set_stream, default: a stream
 *    owned by the matrix).
 */
#ifndef GRAPHENE_GPU_H
#define GRAPHENE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define GR_OK 0
#define GR_EINVAL 1       /* invalid argument (reference: std::invalid_argument) */
#define GR_ENOMEM 2       /* host or device allocation failed */
#define GR_EPARSE 3       /* malformed JSON or MatrixMarket input */
#define GR_ENOTCONV 4     /* solver stopped without converging */
#define GR_EBREAKDOWN 5   /* singular rho / omega (SolverStats::singular) */
#define GR_ETIMEOUT 6     /* a device-side wait ran out of its budget */
#define GR_ECUDA 7        /* CUDA runtime error */
#define GR_EUNSUPPORTED 8 /* combination not supported (reference: runtime_error) */
#define GR_EIO 9          /* file could not be opened */
#define GR_ENONFINITE 10  /* NaN or Inf detected in a residual norm */
#define GR_ECANCELED 11   /* a queued server request was cancelled before it ran */

/* ---- enumerations ---------------------------------------------------- */
/* Element types; names follow common/Type.hpp:125-214 (parseType accepts
 * "float32", "float64", "twofloat32"). TWOFLOAT32 is a pair {h, l} of
 * floats stored as two consecutive floats per element. */
typedef enum { GR_FLOAT32 = 0, GR_FLOAT64 = 1, GR_TWOFLOAT32 = 2 } gr_dtype;

/* matrix/MatrixFormat.hpp:22 */
typedef enum { GR_FORMAT_CRS = 0, GR_FORMAT_LDU = 1 } gr_format;

/* matrix/Norm.hpp (VectorNorm). L1 is the signed sum and LINF the signed
 * maximum, as in dsl/tensor/Tensor.cpp:425-439. */
typedef enum { GR_NORM_L1 = 0, GR_NORM_L2 = 1, GR_NORM_LINF = 2, GR_NORM_NONE = 3 } gr_norm;

/* Row partitioners that produce rowToTile. The reference uses METIS
 * (matrix/host/details/crs/CRSHostMatrix.cpp:139-271), which is not
 * available; these are this library's own deterministic partitioners. */
typedef enum {
  GR_PART_AUTO = 0,       /* RCB when grid coordinates exist, else multilevel bisection */
  GR_PART_CONTIGUOUS = 1, /* equal-weight blocks in natural row order */
  GR_PART_RCB = 2,        /* recursive coordinate bisection (generated grids) */
  GR_PART_BFS = 3,        /* recursive BFS-level-structure graph bisection */
  GR_PART_EXPLICIT = 4,   /* caller-supplied rowToTile */
  GR_PART_MULTILEVEL = 5  /* multilevel recursive bisection, minimum edge cut, weight = row entries + 1
                             (the role of METIS_PartGraphRecursive, CRSHostMatrix.cpp:139-271) */
} gr_partitioner;

typedef struct gr_host_matrix gr_host_matrix;
typedef struct gr_matrix gr_matrix;
typedef struct gr_solver gr_solver;

/* SolverStats (matrix/solver/SolverStats.hpp:29-69). Residual norms are
 * accumulated in FP64 on the device. */
typedef struct {
  double initial_residual;
  double final_residual;
  double b_norm;        /* 0 unless relTolerance > 0 */
  int32_t iterations;
  int32_t converged;
  int32_t singular;
  int32_t status;       /* GR_OK, GR_ETIMEOUT, GR_ENONFINITE, ... */
  int32_t inner_iterations; /* MPIR / restarter: total iterations of the inner solver */
  int32_t reserved;
  double solve_ms;      /* device time of the solve (CUDA events) */
} gr_stats;

typedef struct {
  int64_t num_rows;        /* n */
  int64_t num_off_diag;    /* m: stored off-diagonal entries */
  int64_t num_tiles;       /* tiles after empty-tile removal */
  int64_t num_halo_total;  /* sum over tiles of halo cells */
  int64_t max_tile_rows;   /* largest tile (interior + separator) */
  int64_t num_lower_levels_total;
  int64_t num_upper_levels_total;
  int32_t value_type;      /* gr_dtype of the stored coefficients */
  int32_t format;          /* gr_format */
  int32_t multicolor_recommended; /* CRSHostMatrix.cpp:648-669 */
  int32_t reserved;
} gr_matrix_info;

/* ---- library ---------------------------------------------------------- */
const char* gr_last_error(void);
int gr_version(void);
/* Number of kernel launches issued by this library since load (all
 * devices). Used to count launches inside a timed region. */
int64_t gr_launch_count(void);

/* ---- host matrices (matrix/host/HostMatrix.hpp:31-96) ---------------- */

/* Replaces HostMatrix(MatrixFormat::CRS, TripletMatrix, numTiles)
 * (matrix/host/HostMatrix.cpp:31-44): sorts the triplets by (row, col),
 * splits off the diagonal (CRSHostMatrix.cpp:88-137), partitions the rows,
 * builds the interior/separator/halo tile layout and the tile-local CRS
 * (CRSHostMatrix.cpp:273-525) and the per-tile level sets
 * (CRSHostMatrix.cpp:527-675). Values are rounded to value_type.
 * Duplicate (row, col) entries are rejected with GR_EINVAL.
 * coords (nullable) gives 3 doubles per row for GR_PART_RCB.
 * row_to_tile is read for GR_PART_EXPLICIT only. */
int gr_host_matrix_from_coo(int64_t num_rows, int64_t nnz, const int64_t* rows,
                            const int64_t* cols, const double* vals,
                            int64_t num_tiles, gr_partitioner partitioner,
                            const int32_t* row_to_tile, const double* coords,
                            gr_dtype value_type, gr_host_matrix** out);

/* Replaces generate3DPoissonMatrix(type, nx, ny, nz, numTiles)
 * (matrix/host/HostMatrix.hpp:94-96, details/Poisson.cpp:26-69). */
int gr_host_matrix_poisson(int64_t nx, int64_t ny, int64_t nz, int64_t num_tiles,
                           gr_partitioner partitioner, gr_dtype value_type,
                           gr_host_matrix** out);

/* Synthetic 3-D 7-point matrices (natural row order, neighbours outside the
 * grid dropped), an extension of generate3DPoissonMatrix:
 *   GR_GEN_POISSON      params unused: diagonal 6, off-diagonals -1
 *   GR_GEN_VAR_POISSON  params[0] = sigma: cell coefficient
 *                       exp(sigma * N(0,1)) from `seed`, harmonic-mean face
 *                       coefficients, Dirichlet faces add 2 k to the diagonal
 *   GR_GEN_CONVDIFF     params[0..2] = velocity (>= 0): upwind
 *                       convection-diffusion, unit diffusion and spacing */
typedef enum { GR_GEN_POISSON = 0, GR_GEN_VAR_POISSON = 1, GR_GEN_CONVDIFF = 2 } gr_generator;
int gr_host_matrix_generate(gr_generator kind, int64_t nx, int64_t ny, int64_t nz,
                            const double* params, uint64_t seed, int64_t num_tiles,
                            gr_partitioner partitioner, gr_dtype value_type,
                            gr_host_matrix** out);

/* The same generator with `like`'s structure: the new matrix's values come
 * from (kind, params, seed), its partition, tile layout, tile-local pattern
 * and level sets are copied from `like` (which must have been generated
 * with the same kind and grid; GR_EINVAL if the pattern differs). The cheap
 * way to produce many systems that share a sparsity pattern, e.g. a stream
 * of solves with fresh coefficients. No counterpart in the reference. */
int gr_host_matrix_generate_like(const gr_host_matrix* like, gr_generator kind, int64_t nx, int64_t ny,
                                 int64_t nz, const double* params, uint64_t seed, gr_host_matrix** out);
/* Structure identity of a host matrix (a hash of its value type, sparsity
 * pattern and tile map): equal keys mean equal partition, layout and level
 * sets. No counterpart in the reference. */
int gr_host_matrix_structure_key(const gr_host_matrix* h, uint64_t* key);
/* The values alone: generator (kind, params, seed) on `like`'s grid, written
 * in like's global CRS order - off-diagonals (like's num_off_diag, row by
 * row, columns ascending) to g_val, the diagonal (num_rows) to g_diag,
 * natural row order, FP64 before rounding. The input of
 * gr_server_submit_values. No counterpart in the reference. */
int gr_host_matrix_generate_values(const gr_host_matrix* like, gr_generator kind, int64_t nx, int64_t ny,
                                   int64_t nz, const double* params, uint64_t seed, double* g_val, double* g_diag);

/* Seeded vectors from the generators' counter-based stream: dist 0 =
 * uniform [lo, hi), dist 1 = standard normal. */
int gr_random_vector(uint64_t seed, int64_t n, int dist, double lo, double hi, double* out);

/* Global CRS with split diagonal in natural order (CRSHostMatrix.cpp:88-137):
 * row_ptr n + 1, col / off_diag m, diag n. Any pointer may be NULL. */
int gr_host_matrix_global_crs(const gr_host_matrix* h, int64_t* row_ptr, int64_t* col,
                              double* off_diag, double* diag);

/* Replaces loadMatrixFromFile(type, path, numTiles)
 * (matrix/host/HostMatrix.hpp:88-91, details/MatrixMarket.cpp:31-65). */
int gr_host_matrix_load_mm(const char* path, int64_t num_tiles, gr_partitioner partitioner,
                           gr_dtype value_type, gr_host_matrix** out);

/* LDU matrix (matrix/details/ldu/LDUMatrix.hpp:49, LDUAddressing.hpp:42-91):
 * num_cells cells and num_faces faces in natural numbering; owner[f]
 * (lowerAddr) < neighbour[f] (upperAddr), faces sorted by owner; lower[f]
 * and upper[f] are the face's coefficients in face order (upper NULL: upper
 * = lower, a symmetric matrix), diag[num_cells]. SpMV and residual sum each
 * row as the reference's LDUMatrix does: diag * x, then the owned faces in
 * face order, then the neighbouring faces in losort order. The reference has
 * no host-side LDU builder; its ILU and Gauss-Seidel solvers reject LDU
 * matrices (ilu/Solver.cpp:554-568, gauss-seidel/Solver.cpp:88-95), here they
 * run on the same coefficients in tile-local column order. Partitioning,
 * value_type and the other arguments as for gr_host_matrix_from_coo. */
int gr_host_matrix_from_ldu(int64_t num_cells, int64_t num_faces, const int64_t* owner,
                            const int64_t* neighbour, const double* diag, const double* lower,
                            const double* upper, int64_t num_tiles, gr_partitioner partitioner,
                            const int32_t* row_to_tile, const double* coords, gr_dtype value_type,
                            gr_host_matrix** out);

/* Synthetic unstructured-mesh stand-in in LDU form: an nx x ny x nz
 * hexahedral mesh, node positions jittered by U(-0.2, 0.2) spacings
 * (jitter_seed; cell centroids drive GR_PART_RCB / AUTO), cell ids permuted
 * (perm_seed), owner = smaller cell id, faces sorted by (owner, neighbour),
 * face coefficient c = 10^U(-2, 2) (coef_seed), off-diagonals -c, diagonal
 * = sum of the cell's face coefficients + 1e-3. */
int gr_host_matrix_ldu_mesh(int64_t nx, int64_t ny, int64_t nz, uint64_t jitter_seed,
                            uint64_t perm_seed, uint64_t coef_seed, int64_t num_tiles,
                            gr_partitioner partitioner, gr_dtype value_type, gr_host_matrix** out);

/* The LDU arrays of an LDU host matrix (values rounded to its value type):
 * writes *num_faces, and, where the pointer is not NULL, owner, neighbour,
 * lower, upper (num_faces each) and diag (num_cells). GR_EINVAL for a CRS
 * matrix. */
int gr_host_matrix_get_ldu(const gr_host_matrix* h, int64_t* num_faces, int64_t* owner,
                           int64_t* neighbour, double* lower, double* upper, double* diag);

void gr_host_matrix_destroy(gr_host_matrix* h);

/* A copy of h with the same partition and layout and its coefficients
 * stored as value_type (float64 keeps float32 values exactly; float32
 * rounds). Used to solve the identical system in another precision. */
int gr_host_matrix_astype(const gr_host_matrix* h, gr_dtype value_type, gr_host_matrix** out);

int gr_host_matrix_get_info(const gr_host_matrix* h, gr_matrix_info* out);

/* Partitioning::rowToTile after empty-tile removal (CRSHostMatrix.cpp:235-270). */
int gr_host_matrix_row_to_tile(const gr_host_matrix* h, int32_t* row_to_tile);

/* Off-diagonal entries whose column lies in another tile than their row
 * (each cut edge of a symmetric pattern counts twice). The reference logs
 * METIS's edge cut after partitioning (CRSHostMatrix.cpp:233). */
int gr_host_matrix_edge_cut(const gr_host_matrix* h, int64_t* cut);

/* Per tile: {numInteriorRows, numSeperatorRows, numHaloRows}
 * (DistributedTileLayout.hpp:309-328). out has 3*num_tiles entries. */
int gr_host_matrix_tile_sizes(const gr_host_matrix* h, int64_t* out);

/* TilePartition::localToGlobalRow of every tile, concatenated, halo cells
 * included (DistributedTileLayout.cpp:91-126). out has n + num_halo_total
 * entries. */
int gr_host_matrix_local_to_global(const gr_host_matrix* h, int64_t* out);

/* The tile-local CRS of every tile, concatenated in tile order
 * (CRSHostMatrix.cpp:379-432, 466-525): row_ptr has n + num_tiles entries
 * (each tile's local rowPtr, n_t + 1 entries, starting at 0), col_ind has m
 * entries of tile-local column ids (halo ids >= n_t), off_diag has m values,
 * diag has n values (tile order). Any output pointer may be NULL. */
int gr_host_matrix_local_crs(const gr_host_matrix* h, int64_t* row_ptr, int32_t* col_ind,
                             double* off_diag, double* diag);

/* Per-row level ("colour") of the lower-triangular dependency DAG in tile
 * order (CRSHostMatrix.cpp:527-614) and the upper-triangular levels used by
 * the backward sweep. Either pointer may be NULL. */
int gr_host_matrix_levels(const gr_host_matrix* h, int32_t* lower_level, int32_t* upper_level);

/* Builds the byte stream the streamed ILU(0) substitution kernel consumes
 * (dilu: DILU variant; value_type: stored coefficient type) and replays the
 * kernel's reads on the host, checking every index, the dependency order of
 * the levels and the shared-memory ring capacity. Host only. Writes the
 * ring size (log2 bytes) and stream length. No counterpart in the reference:
 * it validates this library's own device layout. */
int gr_host_matrix_check_ilu_stream(const gr_host_matrix* h, int dilu, gr_dtype value_type,
                                    int32_t* ring_log2, int64_t* stream_bytes);

/* Builds the level blocks and copy schedule of the host-scheduled ring
 * substitution kernel for a ring of ring_bytes (0: the default) with
 * tiles_per_block consecutive tiles per thread block (allow_compact: 1,
 * 16-bit row and column ids where the blocks are small enough; 2, the same
 * with 16-byte row records for levels of 3 entries a row), and replays
 * the kernel's copies and reads on the host, checking every index, the
 * dependency order of the levels, that no copy overwrites a level still to
 * be consumed and that every copy is issued before its level is needed.
 * Host only. Writes the ring size used, the stream length and the largest
 * number of levels of a tile. No counterpart in the reference. */
int gr_host_matrix_check_ilu_ring(const gr_host_matrix* h, int dilu, gr_dtype value_type, int64_t ring_bytes,
                                  int32_t tiles_per_block, int32_t allow_compact, int64_t* ring_bytes_used,
                                  int64_t* stream_bytes, int32_t* max_tile_levels);

/* The same for the Gauss-Seidel sweep's level ring (one tile per block):
 * every entry must read this sweep's value of an earlier row of its tile,
 * the sweep-start value of a later row or of a halo cell, or the zero slot
 * (lower_only: the ring of a sweep from x = 0, which keeps only the entries
 * of earlier rows). *in_place: the ring keeps no sweep-start copy because
 * every later row an entry reads lies in a later level (its slot still
 * holds the start value; checked). Host only. No counterpart in the
 * reference. */
int gr_host_matrix_check_gs_ring(const gr_host_matrix* h, int lower_only, gr_dtype value_type, int64_t ring_bytes,
                                 int32_t allow_compact, int64_t* ring_bytes_used, int64_t* stream_bytes,
                                 int32_t* max_tile_levels, int32_t* in_place);

/* DistributedTileLayout::loadVectorFromFile (DistributedTileLayout.cpp:185-206,
 * without halo): reads a MatrixMarket vector (a "vector" object, coordinate
 * or array, or the first column of a "matrix" object; unlisted entries are
 * 0), which must have as many rows as h, and writes it in tile order, type t
 * (float32 or float64). Host only. */
/* SpMV column encoding of this matrix's later device copies
 * (gr_matrix_create): -1 automatic (the default), 0 32-bit tile-order
 * columns, 1 16-bit column - row offsets with a side list for the columns
 * more than 32767 rows away (6 bytes a float slot instead of 8). Both
 * layouts give every row the same terms in the same order, so SpMV,
 * residual and solver results are identical. The 16-bit layout allows at
 * most 64 far columns per chunk of 32 rows (GR_EUNSUPPORTED at device copy
 * otherwise). Automatic is the 32-bit layout: on B200 it ran the 192^3
 * variable-coefficient SpMV faster (78.1 us against 104.6 us) although the
 * 16-bit one moves a quarter fewer bytes. No counterpart in the
 * reference (its CRS SpMV reads 32-bit local column indices,
 * matrix/details/crs/CRSMatrix.cpp:42-128). */
int gr_host_matrix_set_spmv_layout(gr_host_matrix* h, int32_t layout);
/* Builds the SpMV layout `layout` selects on the host and decodes every
 * slot of the 16-bit encoding, in the order the device's warps walk them,
 * against the 32-bit columns (GR_EINVAL on a mismatch). Reports whether
 * the 16-bit encoding was chosen, the slot count, the far entries and the
 * most far entries in one chunk. No device needed; no counterpart in the
 * reference. */
int gr_host_matrix_check_spmv_layout(const gr_host_matrix* h, int32_t layout, int32_t* compact, int64_t* slots,
                                     int64_t* far_entries, int64_t* max_chunk_far);
int gr_host_matrix_load_vector_mm(const gr_host_matrix* h, const char* path, gr_dtype t, void* tile_ordered);

/* Natural order <-> tile order (DistributedTileLayout::decomposeVector,
 * DistributedTileLayout.cpp:156-183, without halo). Host buffers. */
int gr_host_matrix_decompose_vector(const gr_host_matrix* h, const void* natural,
                                    void* tile_ordered, gr_dtype t);
int gr_host_matrix_compose_vector(const gr_host_matrix* h, const void* tile_ordered,
                                  void* natural, gr_dtype t);

/* ---- device matrices (matrix/Matrix.hpp:29-131) ---------------------- */

/* Replaces HostMatrix::copyToTile() (matrix/host/HostMatrix.hpp:53,
 * CRSHostMatrix.cpp:356-378): uploads the coefficients and addressing to the
 * current CUDA device. The device matrix holds a reference on the host
 * matrix. */
int gr_matrix_create(gr_host_matrix* h, gr_matrix** out);
void gr_matrix_destroy(gr_matrix* A);
/* Use an external cudaStream_t (NULL restores the matrix's own stream). */
int gr_matrix_set_stream(gr_matrix* A, void* cuda_stream);
int gr_matrix_get_info(const gr_matrix* A, gr_matrix_info* out);

/* Replaces Matrix::operator*(Tensor& x) (matrix/Matrix.hpp:95-97,
 * details/crs/CRSMatrix.cpp:42-83): y = A x. x and y are device pointers in
 * tile order; xt == yt (FLOAT32 or FLOAT64). */
/* The SpMV layout of a device matrix (see gr_host_matrix_set_spmv_layout):
 * 16-bit encoding or not, slots, far entries. No counterpart in the
 * reference. */
int gr_matrix_spmv_layout(const gr_matrix* A, int32_t* compact, int64_t* slots, int64_t* far_entries);
int gr_spmv(gr_matrix* A, const void* x, void* y, gr_dtype t);

/* SpMV autotuner (no counterpart in the reference): times the candidate
 * launch geometries of gr_spmv for vectors of type t (threads per block 128 /
 * 256 / 512, SELL chunks per warp, entry loads batched 4 / 8 / 16; every
 * candidate reps times on the matrix's stream, each launch timed alone with
 * L2 flushed first, as a solve meets a matrix larger than L2) and keeps the
 * fastest for later gr_spmv calls on this matrix. Every geometry computes each row in the
 * same order, so results do not change. Writes the choice and its mean time
 * (ms); chunks_per_warp 0 is the untuned grid. */
int gr_matrix_tune_spmv(gr_matrix* A, gr_dtype t, int32_t reps, int32_t* block, int32_t* chunks_per_warp,
                        int32_t* batch, float* ms);

/* Benchmarking (no counterpart in the reference): the mean device time (ms)
 * of y = A x (gr_spmv's kernel, current geometry) over reps launches, each
 * timed alone between two CUDA events on the matrix's stream, with L2
 * flushed before each launch when flush_l2 is nonzero (a 256 MB write). */
int gr_matrix_time_spmv(gr_matrix* A, const void* x, void* y, gr_dtype t, int32_t reps, int32_t flush_l2,
                        float* ms);

/* Replaces Matrix::residual(x, b, destType, intermediateType)
 * (matrix/Matrix.hpp:86-92, CRSMatrix.cpp:85-128): r = b - A x computed in
 * inter_t and rounded to r_t. x_t may be FLOAT32, FLOAT64 or TWOFLOAT32,
 * b is FLOAT32 or FLOAT64. */
int gr_residual(gr_matrix* A, const void* x, gr_dtype x_t, const void* b, gr_dtype b_t,
                void* r, gr_dtype r_t, gr_dtype inter_t);

/* Replaces Matrix::vectorNorm(norm, x) (matrix/Matrix.hpp:120-122,
 * details/MatrixBase.cpp:149-152). Accumulates in FP64. */
int gr_vector_norm(gr_matrix* A, gr_norm norm, const void* x, gr_dtype t, double* out);

/* Failure injection from the host (no counterpart in the reference):
 * stores `status` (GR_ETIMEOUT, ...) in the matrix's device error word, the
 * word a kernel whose bounded wait ran out writes. The next solve on A then
 * stops at its first convergence check and reports that status, and the
 * word is cleared, as after a real device-side timeout. No kernel runs and
 * nothing faults; tests use it to exercise the failure path. */
int gr_matrix_inject_status(gr_matrix* A, int32_t status);

/* Norms of `count` device vectors of n elements (vector j starts at element
 * j * ld of x), FP64 accumulation, written to out[0..count) (device
 * doubles) on `stream` (NULL: the default stream); returns without waiting.
 * No counterpart in the reference. Unlike gr_vector_norm it needs no
 * matrix and allocates no device memory: it reduces through a static
 * per-device scratch of 75,808 bytes. For callers that must not allocate
 * device memory at the call (a serving loop held to a fixed HBM footprint,
 * a caching allocator's own callbacks). Limits: count 1..8, n <= 2^31 - 1;
 * anything larger returns GR_EINVAL. Calls that overlap on one device
 * (several streams or threads) share the scratch and race: serialise them.
 * The first call on each device does the set-up (symbol lookup, scratch
 * counters cleared); make it before any stream capture. */
int gr_vector_norms_noalloc(const void* x, int64_t n, int64_t count, int64_t ld, gr_dtype t,
                            gr_norm norm, double* out, void* stream);

/* Natural order <-> tile order on the device. */
int gr_decompose_vector(gr_matrix* A, const void* natural, void* tile_ordered, gr_dtype t);
int gr_compose_vector(gr_matrix* A, const void* tile_ordered, void* natural, gr_dtype t);

/* ---- solvers (matrix/solver/) ---------------------------------------- */

/* Replaces Configuration::fromJSON + Solver::createSolver
 * (matrix/solver/Configuration.cpp:103-136, Solver.cpp:32-56). json is the
 * reference's solver tree ("type": PBiCGStab | ILU | GaussSeidel |
 * IterativeRefinement | restarter, nested "preconditioner" /
 * "innerSolver"); comments are allowed. Construction performs the ILU
 * factorisation as the reference's ilu::Solver constructor does
 * (ilu/Solver.cpp:44-51). */
int gr_solver_create(gr_matrix* A, const char* json, gr_solver** out);
void gr_solver_destroy(gr_solver* s);

/* Replaces Solver::solve(x, b) (matrix/solver/Solver.hpp:41) and
 * Matrix::solve (matrix/Matrix.cpp:26-30). x (in/out) and b are device
 * pointers in tile order of type x_t / b_t (FLOAT32 or FLOAT64; b_t must
 * equal x_t). Blocks until the solve has finished. */
int gr_solve(gr_solver* s, void* x, gr_dtype x_t, const void* b, gr_dtype b_t, gr_stats* stats);

/* Same as gr_solve with host buffers in natural order: copies b in, x in
 * and x out (the end-to-end path). */
int gr_solve_host(gr_solver* s, void* x, gr_dtype x_t, const void* b, gr_dtype b_t,
                  gr_stats* stats);

/* Benchmarking: runs an ILU or fixed-sweep Gauss-Seidel solver reps times
 * back to back on the matrix's stream (device pointers, tile order) without
 * host synchronisation in between and writes the mean device time per run
 * in ms. No counterpart in the reference. */
int gr_solver_time_repeated(gr_solver* s, void* x, gr_dtype x_t, const void* b, gr_dtype b_t, int32_t reps,
                            float* ms_per_run);

/* After an IterativeRefinement solve: the extended-precision solution phi
 * (iterative-refinement/Solver.cpp:84,103), copied to a device buffer of
 * type t in tile order. The reference returns only (float)phi. */
int gr_solver_phi(gr_solver* s, void* out, gr_dtype t);

/* Value updates on a resident structure (no counterpart in the reference,
 * whose graph is compiled for one matrix). gr_matrix_update_values replaces
 * A's coefficients by h's, where h has A's structure (equal
 * gr_host_matrix_structure_key, CRS; GR_EINVAL otherwise): the values are
 * uploaded and scattered into the device layout in place, and no host-side
 * layout work is redone. gr_solver_refresh then recomputes a solver's
 * value-dependent parts (ILU factors, packed level blocks) in the buffers
 * it owns. The pair costs one upload and one factorisation instead of a
 * new matrix and solver. */
int gr_matrix_update_values(gr_matrix* A, gr_host_matrix* h);
int gr_solver_refresh(gr_solver* s);
/* New coefficients for A from global CRS values in natural order (g_val:
 * off-diagonals in the order of gr_host_matrix_global_crs, g_diag: the
 * diagonal; FP64, host memory), gathered into the device layout by a kernel:
 * no host-side permutation or conversion. A must be a CRS matrix; results
 * equal those of gr_matrix_update_values with a host matrix holding these
 * values. Solvers on A then need gr_solver_refresh. No counterpart in the
 * reference. */
int gr_matrix_update_global_values(gr_matrix* A, const double* g_val, const double* g_diag);

/* Name of the solver tree, e.g. "IterativeRefinement(PBiCGStab(ILU(0)))". */
int gr_solver_name(const gr_solver* s, char* buf, size_t len);

/* Parses a solver configuration without a matrix or a GPU
 * (Configuration::fromJSON, matrix/solver/Configuration.cpp:103-136) and
 * writes the solver tree's name; unknown keys, which the reference ignores,
 * are listed in unknown_keys (comma separated, may be NULL). */
int gr_config_parse(const char* json, char* name, size_t name_len, char* unknown_keys,
                    size_t unknown_len);

/* ---- solve server ------------------------------------------------------
 * No counterpart in the reference (its Runtime runs one graph at a time).
 * Continuous batching of independent solves on one GPU: requests are
 * queued on arrival and admitted in arrival order as soon as a worker slot
 * is free and their estimated device footprint fits the budget; each slot
 * drives its own non-blocking CUDA stream, so admitted solves overlap on the
 * device. A (host matrix, configuration) pair stays resident after its
 * request (coefficients, layout, factors, solver buffers), so a later
 * request for the same pair skips upload and factorisation; idle pairs are
 * evicted oldest first when memory is needed. Results do not depend on what
 * else is running (the kernels are deterministic). */
typedef struct gr_server gr_server;

typedef struct {
  int32_t slots;            /* concurrent solves (worker threads / streams); 0: 4 */
  int32_t device;           /* CUDA device; -1: the current device */
  int64_t hbm_budget_bytes; /* admission limit on resident footprints; 0: 80% of free memory */
} gr_server_config;

typedef struct {
  double arrival_ms;   /* submit time, ms since the server was created */
  double admitted_ms;  /* a slot and memory were granted */
  double finished_ms;  /* result copied back */
  int64_t footprint_bytes; /* estimated device bytes of the request's resident pair */
  int32_t cache_hit;   /* 1: the pair was already resident; 2: a pair with the
                          same structure was, and took this matrix's values */
  int32_t slot;
  double solve_start_ms; /* values on the device and factorised: the solve (b in,
                            iterations, x out) starts */
} gr_request_times;

int gr_server_create(const gr_server_config* cfg, gr_server** out);
/* Queues the solve h x = b with the solver configuration json (the same
 * schema as gr_solver_create), x0 = 0. b is a host vector in natural order of
 * type t (FLOAT32 or FLOAT64), copied by the call; the server keeps h alive
 * while the request or its resident pair needs it. */
int gr_server_submit(gr_server* s, gr_host_matrix* h, const char* json, const void* b, gr_dtype t,
                     uint64_t* id);
/* Waits up to timeout_ms (< 0: no limit) for request id. On completion
 * copies x (natural order, the request's type) to x_out (may be NULL),
 * fills stats / times (may be NULL), forgets the request and returns the
 * request's own status (GR_OK, or the error of its solve, message in
 * gr_last_error). GR_ETIMEOUT if it has not finished in time (the request
 * stays queued); GR_EINVAL for an unknown id. */
int gr_server_wait(gr_server* s, uint64_t id, double timeout_ms, void* x_out, gr_stats* stats,
                   gr_request_times* times);
/* Current counts: queued, running, completed; device bytes held by resident
 * pairs; number of resident pairs. Any pointer may be NULL. */
int gr_server_counters(gr_server* s, int64_t* queued, int64_t* running, int64_t* completed,
                       int64_t* bytes_in_use, int64_t* resident);
/* Cancels request id if it is still queued (not yet admitted): *cancelled
 * = 1, and gr_server_wait then returns GR_ECANCELED for it. A request that
 * has been admitted runs to completion: *cancelled = 0. GR_EINVAL for an
 * unknown id. No counterpart in the reference (one compiled graph runs at a
 * time there). */
int gr_server_cancel(gr_server* s, uint64_t id, int32_t* cancelled);
/* Queues a solve of the matrix with `like`'s structure and the values g_val
 * (like's global CRS order, off-diagonals) and g_diag (natural order),
 * copied by the call, with the same meaning as gr_server_submit otherwise.
 * On a resident pair of that structure the values are uploaded and the
 * solver refactorised in place (cache_hit 2); otherwise a matrix is built
 * from like's layout and the values. The request never needs a host matrix
 * of its own - the form for streams of systems that share a pattern. */
int gr_server_submit_values(gr_server* s, gr_host_matrix* like, const double* g_val, const double* g_diag,
                            const char* json, const void* b, gr_dtype t, uint64_t* id);
/* Finishes the running solves, drops the queued ones, releases everything. */
void gr_server_destroy(gr_server* s);

/* ---- batched solves --------------------------------------------------
 * No counterpart in the reference. Solves count independent systems of any
 * sizes with one PBiCGStab whose every kernel launch covers all of them:
 * the systems are stored as one block-diagonal device matrix, each keeps its
 * own Krylov state and convergence test on the device, and a system that
 * has converged drops out of the work while the others continue. Each
 * system's result equals the result of solving it alone with the same
 * configuration. json: a PBiCGStab configuration with the ILU
 * preconditioner (the ring substitution kernel, one tile per block); the
 * systems share one coefficient type. */
typedef struct gr_batch gr_batch;
int gr_batch_create(gr_host_matrix* const* systems, int32_t count, const char* json, gr_batch** out);
/* x[i] (in: initial guess, out: solution) and b[i]: host vectors of system i
 * in natural order, type t; stats: count entries (may be NULL). */
int gr_batch_solve_host(gr_batch* b, void* const* x, const void* const* rhs, gr_dtype t, gr_stats* stats);
void gr_batch_destroy(gr_batch* b);

/* ---- self-test ----------------------------------------------------------
 * No counterpart in the reference. Every wait of this library's pipelined
 * kernels on an mbarrier (a copy landing, a level released) is bounded: after
 * 1 s it gives up, the kernel records GR_ETIMEOUT and exits. This runs that
 * wait on a barrier nothing arrives on and writes the status the kernel
 * reported (GR_ETIMEOUT when the bound works) and how long it waited (ns);
 * the device stays usable. Takes about a second. */
int gr_selftest_wait_timeout(int32_t* status, int64_t* elapsed_ns);

#ifdef __cplusplus
}
#endif

#endif /* GRAPHENE_GPU_H */
