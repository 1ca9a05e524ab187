// extern "C" boundary of graphene_b200 (include/graphene_gpu.h).
#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "device.hpp"
#include "host_matrix.hpp"
#include "config.hpp"
#include "solvers.hpp"
#include "server.hpp"
#include "batch.hpp"

struct gr_host_matrix {
  std::shared_ptr<gr::HostMatrix> m;
};

struct gr_matrix {
  std::unique_ptr<gr::DeviceMatrix> d;
};

struct gr_solver {
  std::unique_ptr<gr::SolverTree> s;
};

struct gr_server {
  std::unique_ptr<gr::Server> s;
};

struct gr_batch {
  std::unique_ptr<gr::BatchSolve> b;
};

namespace {

thread_local std::string g_lastError;

template <class F>
int guarded(F&& f) {
  try {
    f();
    g_lastError.clear();
    return GR_OK;
  } catch (const gr::Error& e) {
    g_lastError = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_lastError = "host allocation failed";
    return GR_ENOMEM;
  } catch (const std::exception& e) {
    g_lastError = e.what();
    return GR_EINVAL;
  } catch (...) {
    g_lastError = "unknown error";
    return GR_EINVAL;
  }
}

void need(const void* p, const char* what) {
  if (!p) gr::fail(GR_EINVAL, std::string(what) + " must not be NULL");
}

}  // namespace

extern "C" {

const char* gr_last_error(void) { return g_lastError.c_str(); }

int gr_version(void) { return 1; }

int64_t gr_launch_count(void) { return gr::launchCount(); }

int gr_host_matrix_from_coo(int64_t num_rows, int64_t nnz, const int64_t* rows, const int64_t* cols,
                            const double* vals, int64_t num_tiles, gr_partitioner partitioner,
                            const int32_t* row_to_tile, const double* coords, gr_dtype value_type,
                            gr_host_matrix** out) {
  return guarded([&] {
    need(out, "out");
    if (nnz < 0) gr::fail(GR_EINVAL, "nnz must be non-negative");
    if (nnz > 0) { need(rows, "rows"); need(cols, "cols"); need(vals, "vals"); }
    gr::Coo coo;
    coo.nrows = coo.ncols = num_rows;
    coo.row.assign(rows, rows + nnz);
    coo.col.assign(cols, cols + nnz);
    coo.val.assign(vals, vals + nnz);
    auto h = gr::HostMatrix::fromCoo(std::move(coo), num_tiles, partitioner, row_to_tile, coords,
                                     gr::toDType(value_type));
    *out = new gr_host_matrix{std::move(h)};
  });
}

int gr_host_matrix_poisson(int64_t nx, int64_t ny, int64_t nz, int64_t num_tiles,
                           gr_partitioner partitioner, gr_dtype value_type, gr_host_matrix** out) {
  return guarded([&] {
    need(out, "out");
    gr::GeneratedCsr g = gr::generatePoisson(nx, ny, nz);
    auto h = gr::HostMatrix::fromSortedCsr(g.n, std::move(g.rowPtr), std::move(g.col),
                                           std::move(g.val), num_tiles, partitioner, nullptr,
                                           std::move(g.coords), gr::toDType(value_type));
    *out = new gr_host_matrix{std::move(h)};
  });
}

int gr_host_matrix_generate(gr_generator kind, int64_t nx, int64_t ny, int64_t nz, const double* params,
                            uint64_t seed, int64_t num_tiles, gr_partitioner partitioner, gr_dtype value_type,
                            gr_host_matrix** out) {
  return guarded([&] {
    need(out, "out");
    GR_TRACE_SCOPE("gr_host_matrix_generate");
    gr::GeneratedCsr g;
    {
    GR_TRACE_SCOPE("generate CRS");
    switch (kind) {
      case GR_GEN_POISSON:
        g = gr::generatePoisson(nx, ny, nz);
        break;
      case GR_GEN_VAR_POISSON:
        need(params, "params");
        g = gr::generateVarPoisson(nx, ny, nz, params[0], seed);
        break;
      case GR_GEN_CONVDIFF:
        need(params, "params");
        if (params[0] < 0 || params[1] < 0 || params[2] < 0) gr::fail(GR_EINVAL, "velocity must be >= 0");
        g = gr::generateConvDiff(nx, ny, nz, params[0], params[1], params[2]);
        break;
      default:
        gr::fail(GR_EINVAL, "unknown generator");
    }
    }
    auto h = gr::HostMatrix::fromSortedCsr(g.n, std::move(g.rowPtr), std::move(g.col), std::move(g.val),
                                           num_tiles, partitioner, nullptr, std::move(g.coords),
                                           gr::toDType(value_type));
    *out = new gr_host_matrix{std::move(h)};
  });
}

int gr_host_matrix_generate_like(const gr_host_matrix* like, gr_generator kind, int64_t nx, int64_t ny,
                                 int64_t nz, const double* params, uint64_t seed, gr_host_matrix** out) {
  return guarded([&] {
    need(like, "like");
    need(out, "out");
    GR_TRACE_SCOPE("gr_host_matrix_generate_like");
    gr::GeneratedCsr g;
    switch (kind) {
      case GR_GEN_POISSON:
        g = gr::generatePoisson(nx, ny, nz);
        break;
      case GR_GEN_VAR_POISSON:
        need(params, "params");
        g = gr::generateVarPoisson(nx, ny, nz, params[0], seed);
        break;
      case GR_GEN_CONVDIFF:
        need(params, "params");
        if (params[0] < 0 || params[1] < 0 || params[2] < 0) gr::fail(GR_EINVAL, "velocity must be >= 0");
        g = gr::generateConvDiff(nx, ny, nz, params[0], params[1], params[2]);
        break;
      default:
        gr::fail(GR_EINVAL, "unknown generator");
    }
    if (g.n != like->m->n) gr::fail(GR_EINVAL, "the template matrix has another grid");
    *out = new gr_host_matrix{gr::HostMatrix::withValues(*like->m, g.rowPtr, g.col, g.val)};
  });
}

int gr_host_matrix_generate_values(const gr_host_matrix* like, gr_generator kind, int64_t nx, int64_t ny,
                                   int64_t nz, const double* params, uint64_t seed, double* g_val, double* g_diag) {
  return guarded([&] {
    need(like, "like");
    need(g_val, "g_val");
    need(g_diag, "g_diag");
    const double zero[3] = {0, 0, 0};
    if (kind != GR_GEN_POISSON) need(params, "params");
    if (nx * ny * nz != like->m->n || like->m->format != GR_FORMAT_CRS)
      gr::fail(GR_EINVAL, "the template matrix has another grid");
    if (!gr::generateValues(static_cast<int>(kind), nx, ny, nz, params ? params : zero, seed, like->m->gRowPtr,
                            g_val, g_diag))
      gr::fail(GR_EINVAL, "the template matrix does not have this generator's pattern");
  });
}

int gr_host_matrix_structure_key(const gr_host_matrix* h, uint64_t* key) {
  return guarded([&] {
    need(h, "matrix");
    need(key, "key");
    *key = h->m->structureKey;
  });
}

int gr_host_matrix_from_ldu(int64_t num_cells, int64_t num_faces, const int64_t* owner, const int64_t* neighbour,
                            const double* diag, const double* lower, const double* upper, int64_t num_tiles,
                            gr_partitioner partitioner, const int32_t* row_to_tile, const double* coords,
                            gr_dtype value_type, gr_host_matrix** out) {
  return guarded([&] {
    need(out, "out");
    auto h = gr::HostMatrix::fromLdu(num_cells, num_faces, owner, neighbour, diag, lower, upper, num_tiles,
                                     partitioner, row_to_tile, coords, gr::toDType(value_type));
    *out = new gr_host_matrix{std::move(h)};
  });
}

int gr_host_matrix_ldu_mesh(int64_t nx, int64_t ny, int64_t nz, uint64_t jitter_seed, uint64_t perm_seed,
                            uint64_t coef_seed, int64_t num_tiles, gr_partitioner partitioner, gr_dtype value_type,
                            gr_host_matrix** out) {
  return guarded([&] {
    need(out, "out");
    gr::LduMesh M = gr::generateLduMesh(nx, ny, nz, jitter_seed, perm_seed, coef_seed);
    auto h = gr::HostMatrix::fromLdu(M.n, static_cast<int64_t>(M.owner.size()), M.owner.data(),
                                     M.neighbour.data(), M.diag.data(), M.lower.data(), M.upper.data(), num_tiles,
                                     partitioner, nullptr, M.coords.data(), gr::toDType(value_type));
    *out = new gr_host_matrix{std::move(h)};
  });
}

int gr_host_matrix_get_ldu(const gr_host_matrix* h, int64_t* num_faces, int64_t* owner, int64_t* neighbour,
                           double* lower, double* upper, double* diag) {
  return guarded([&] {
    need(h, "host matrix");
    need(num_faces, "num_faces");
    const gr::HostMatrix& H = *h->m;
    if (H.format != GR_FORMAT_LDU) gr::fail(GR_EINVAL, "not an LDU matrix");
    const size_t F = H.lduOwner.size();
    *num_faces = static_cast<int64_t>(F);
    if (owner) std::copy(H.lduOwner.begin(), H.lduOwner.end(), owner);
    if (neighbour) std::copy(H.lduNeighbour.begin(), H.lduNeighbour.end(), neighbour);
    if (lower) std::copy(H.lduLower.begin(), H.lduLower.end(), lower);
    if (upper) std::copy(H.lduUpper.begin(), H.lduUpper.end(), upper);
    if (diag) std::copy(H.lduDiag.begin(), H.lduDiag.end(), diag);
  });
}

int gr_random_vector(uint64_t seed, int64_t n, int dist, double lo, double hi, double* out) {
  return guarded([&] {
    need(out, "out");
    if (n < 0) gr::fail(GR_EINVAL, "n must be non-negative");
    if (dist == 0) gr::generateUniform(seed, n, lo, hi, out);
    else if (dist == 1) gr::generateNormal(seed, n, out);
    else gr::fail(GR_EINVAL, "dist must be 0 (uniform) or 1 (normal)");
  });
}

int gr_host_matrix_global_crs(const gr_host_matrix* h, int64_t* row_ptr, int64_t* col, double* off_diag,
                              double* diag) {
  return guarded([&] {
    need(h, "matrix");
    const gr::HostMatrix& H = *h->m;
    if (row_ptr) std::memcpy(row_ptr, H.gRowPtr.data(), sizeof(int64_t) * (H.n + 1));
    if (col) std::memcpy(col, H.gCol.data(), sizeof(int64_t) * H.m);
    if (off_diag) std::memcpy(off_diag, H.gVal.data(), sizeof(double) * H.m);
    if (diag) std::memcpy(diag, H.gDiag.data(), sizeof(double) * H.n);
  });
}

int gr_host_matrix_load_mm(const char* path, int64_t num_tiles, gr_partitioner partitioner,
                           gr_dtype value_type, gr_host_matrix** out) {
  return guarded([&] {
    need(path, "path");
    need(out, "out");
    gr::Coo coo = gr::readMatrixMarket(path, gr::toDType(value_type));
    auto h = gr::HostMatrix::fromCoo(std::move(coo), num_tiles, partitioner, nullptr, nullptr,
                                     gr::toDType(value_type));
    *out = new gr_host_matrix{std::move(h)};
  });
}

void gr_host_matrix_destroy(gr_host_matrix* h) { delete h; }

int gr_host_matrix_astype(const gr_host_matrix* h, gr_dtype value_type, gr_host_matrix** out) {
  return guarded([&] {
    need(h, "matrix");
    need(out, "out");
    gr::DType t = gr::toDType(value_type);
    if (t == gr::DType::DW) gr::fail(GR_EUNSUPPORTED, "twofloat32 coefficients are not supported");
    auto c = std::make_shared<gr::HostMatrix>(*h->m);
    c->valueType = t;
    if (t == gr::DType::F32) {
      auto r = [](std::vector<double>& v) {
        for (double& x : v) x = static_cast<double>(static_cast<float>(x));
      };
      r(c->gVal); r(c->gDiag); r(c->offDiag); r(c->diag);
      r(c->lduLower); r(c->lduUpper); r(c->lduDiag);
    }
    *out = new gr_host_matrix{std::move(c)};
  });
}

int gr_host_matrix_get_info(const gr_host_matrix* h, gr_matrix_info* out) {
  return guarded([&] {
    need(h, "matrix");
    need(out, "out");
    *out = h->m->info();
  });
}

int gr_host_matrix_row_to_tile(const gr_host_matrix* h, int32_t* row_to_tile) {
  return guarded([&] {
    need(h, "matrix");
    need(row_to_tile, "row_to_tile");
    std::memcpy(row_to_tile, h->m->rowToTile.data(), sizeof(int32_t) * h->m->n);
  });
}

int gr_host_matrix_edge_cut(const gr_host_matrix* h, int64_t* cut) {
  return guarded([&] {
    need(h, "matrix");
    need(cut, "cut");
    *cut = gr::edgeCut(*h->m, h->m->rowToTile);
  });
}

int gr_host_matrix_tile_sizes(const gr_host_matrix* h, int64_t* out) {
  return guarded([&] {
    need(h, "matrix");
    need(out, "out");
    for (gr::i32 T = 0; T < h->m->P; ++T) {
      out[3 * T] = h->m->tiles[T].nInterior;
      out[3 * T + 1] = h->m->tiles[T].nSeparator;
      out[3 * T + 2] = h->m->tiles[T].nHalo;
    }
  });
}

int gr_host_matrix_local_to_global(const gr_host_matrix* h, int64_t* out) {
  return guarded([&] {
    need(h, "matrix");
    need(out, "out");
    const gr::HostMatrix& H = *h->m;
    int64_t o = 0;
    for (gr::i32 T = 0; T < H.P; ++T) {
      for (gr::i64 p = H.tileStart[T]; p < H.tileStart[T + 1]; ++p) out[o++] = H.iperm[p];
      for (gr::i32 R : H.tiles[T].haloRegions)
        for (gr::i64 g : H.regions[R].cells) out[o++] = g;
    }
  });
}

int gr_host_matrix_local_crs(const gr_host_matrix* h, int64_t* row_ptr, int32_t* col_ind,
                             double* off_diag, double* diag) {
  return guarded([&] {
    need(h, "matrix");
    const gr::HostMatrix& H = *h->m;
    if (row_ptr) {
      int64_t o = 0;
      for (gr::i32 T = 0; T < H.P; ++T) {
        gr::i64 b = H.tileStart[T];
        for (gr::i64 p = b; p <= H.tileStart[T + 1]; ++p) row_ptr[o++] = H.rowPtr[p] - H.rowPtr[b];
      }
    }
    if (col_ind) std::memcpy(col_ind, H.colLocal.data(), sizeof(int32_t) * H.m);
    if (off_diag) std::memcpy(off_diag, H.offDiag.data(), sizeof(double) * H.m);
    if (diag) std::memcpy(diag, H.diag.data(), sizeof(double) * H.n);
  });
}

int gr_host_matrix_levels(const gr_host_matrix* h, int32_t* lower_level, int32_t* upper_level) {
  return guarded([&] {
    need(h, "matrix");
    if (lower_level) std::memcpy(lower_level, h->m->lowerLevel.data(), sizeof(int32_t) * h->m->n);
    if (upper_level) std::memcpy(upper_level, h->m->upperLevel.data(), sizeof(int32_t) * h->m->n);
  });
}

int gr_host_matrix_check_ilu_stream(const gr_host_matrix* h, int dilu, gr_dtype value_type, int32_t* ring_log2,
                                    int64_t* stream_bytes) {
  return guarded([&] {
    need(h, "matrix");
    const gr::DType vt = gr::toDType(value_type);
    gr::HostStream S = gr::buildIluStream(*h->m, dilu != 0, vt);
    const int lg = gr::ringLog2ForLevel(S.maxSpanBytes);
    gr::checkIluStream(*h->m, S, dilu != 0, vt, lg);
    if (ring_log2) *ring_log2 = lg;
    if (stream_bytes) *stream_bytes = static_cast<int64_t>(S.bytes.size());
  });
}

int gr_host_matrix_check_ilu_ring(const gr_host_matrix* h, int dilu, gr_dtype value_type, int64_t ring_bytes,
                                  int32_t tiles_per_block, int32_t allow_compact, int64_t* ring_bytes_used,
                                  int64_t* stream_bytes, int32_t* max_tile_levels) {
  return guarded([&] {
    need(h, "matrix");
    const gr::DType vt = gr::toDType(value_type);
    gr::HostRing R = gr::buildLevelRing(*h->m, dilu != 0, vt, ring_bytes, tiles_per_block, gr::RingBudget{},
                                        allow_compact != 0, gr::RingKind::Ilu, allow_compact == 2);
    gr::checkLevelRing(*h->m, R, dilu != 0, vt);
    if (ring_bytes_used) *ring_bytes_used = R.ringBytes;
    if (stream_bytes) *stream_bytes = static_cast<int64_t>(R.bytes.size());
    if (max_tile_levels) *max_tile_levels = R.maxTileLevels;
  });
}

int gr_host_matrix_check_gs_ring(const gr_host_matrix* h, int lower_only, gr_dtype value_type, int64_t ring_bytes,
                                 int32_t allow_compact, int64_t* ring_bytes_used, int64_t* stream_bytes,
                                 int32_t* max_tile_levels, int32_t* in_place) {
  return guarded([&] {
    need(h, "matrix");
    const gr::DType vt = gr::toDType(value_type);
    gr::HostRing R = gr::buildLevelRing(*h->m, false, vt, ring_bytes, 1, gr::RingBudget{}, allow_compact != 0,
                                        lower_only ? gr::RingKind::GaussSeidelLower : gr::RingKind::GaussSeidel,
                                        allow_compact == 2);
    gr::checkLevelRing(*h->m, R, false, vt);
    if (ring_bytes_used) *ring_bytes_used = R.ringBytes;
    if (stream_bytes) *stream_bytes = static_cast<int64_t>(R.bytes.size());
    if (max_tile_levels) *max_tile_levels = R.maxTileLevels;
    if (in_place) *in_place = R.gsInPlace ? 1 : 0;
  });
}

int gr_host_matrix_set_spmv_layout(gr_host_matrix* h, int32_t layout) {
  return guarded([&] {
    need(h, "matrix");
    if (layout < -1 || layout > 1) gr::fail(GR_EINVAL, "spmv layout must be -1, 0 or 1");
    h->m->spmvLayout = layout;
  });
}

int gr_host_matrix_check_spmv_layout(const gr_host_matrix* h, int32_t layout, int32_t* compact, int64_t* slots,
                                     int64_t* far_entries, int64_t* max_chunk_far) {
  return guarded([&] {
    need(h, "matrix");
    gr::SellHost S = gr::buildSell(*h->m, layout);
    gr::checkSellDecode(S, h->m->n);
    if (compact) *compact = S.compact ? 1 : 0;
    if (slots) *slots = S.slots;
    if (far_entries) *far_entries = static_cast<int64_t>(S.farCol.size());
    if (max_chunk_far) *max_chunk_far = S.maxChunkFar;
  });
}

int gr_host_matrix_decompose_vector(const gr_host_matrix* h, const void* natural, void* tile_ordered,
                                    gr_dtype t) {
  return guarded([&] {
    need(h, "matrix");
    need(natural, "natural");
    need(tile_ordered, "tile_ordered");
    gr::DType dt = gr::toDType(t);
    if (dt == gr::DType::F32)
      h->m->decompose(static_cast<const float*>(natural), static_cast<float*>(tile_ordered));
    else
      h->m->decompose(static_cast<const double*>(natural), static_cast<double*>(tile_ordered));
  });
}

int gr_host_matrix_load_vector_mm(const gr_host_matrix* h, const char* path, gr_dtype t, void* tile_ordered) {
  return guarded([&] {
    need(h, "matrix");
    need(path, "path");
    need(tile_ordered, "tile_ordered");
    const gr::DType dt = gr::toDType(t);
    if (dt != gr::DType::F32 && dt != gr::DType::F64) gr::fail(GR_EUNSUPPORTED, "vectors are float32 or float64");
    const std::vector<double> v = gr::readMatrixMarketVector(path, dt);
    if (static_cast<gr::i64>(v.size()) != h->m->n)
      gr::fail(GR_EINVAL, "vector file has " + std::to_string(v.size()) + " rows, the matrix " +
                              std::to_string(h->m->n));
    if (dt == gr::DType::F32) {
      std::vector<float> f(v.begin(), v.end());
      h->m->decompose(f.data(), static_cast<float*>(tile_ordered));
    } else {
      h->m->decompose(v.data(), static_cast<double*>(tile_ordered));
    }
  });
}

int gr_host_matrix_compose_vector(const gr_host_matrix* h, const void* tile_ordered, void* natural,
                                  gr_dtype t) {
  return guarded([&] {
    need(h, "matrix");
    need(natural, "natural");
    need(tile_ordered, "tile_ordered");
    gr::DType dt = gr::toDType(t);
    if (dt == gr::DType::F32)
      h->m->compose(static_cast<const float*>(tile_ordered), static_cast<float*>(natural));
    else
      h->m->compose(static_cast<const double*>(tile_ordered), static_cast<double*>(natural));
  });
}

int gr_matrix_create(gr_host_matrix* h, gr_matrix** out) {
  return guarded([&] {
    need(h, "host matrix");
    need(out, "out");
    auto d = std::make_unique<gr::DeviceMatrix>(h->m);
    *out = new gr_matrix{std::move(d)};
  });
}

void gr_matrix_destroy(gr_matrix* A) { delete A; }

int gr_matrix_set_stream(gr_matrix* A, void* cuda_stream) {
  return guarded([&] {
    need(A, "matrix");
    A->d->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : A->d->ownStream;
  });
}

int gr_matrix_get_info(const gr_matrix* A, gr_matrix_info* out) {
  return guarded([&] {
    need(A, "matrix");
    need(out, "out");
    *out = A->d->host->info();
  });
}

int gr_matrix_spmv_layout(const gr_matrix* A, int32_t* compact, int64_t* slots, int64_t* far_entries) {
  return guarded([&] {
    need(A, "matrix");
    if (compact) *compact = A->d->sell.compact ? 1 : 0;
    if (slots) *slots = A->d->sell.slots;
    if (far_entries) *far_entries = A->d->sell.far;
  });
}

int gr_spmv(gr_matrix* A, const void* x, void* y, gr_dtype t) {
  return guarded([&] {
    need(A, "matrix");
    need(x, "x");
    need(y, "y");
    gr::launchSpmv(*A->d, x, y, gr::toDType(t), A->d->stream);
    GR_CUDA(cudaStreamSynchronize(A->d->stream));
  });
}

int gr_residual(gr_matrix* A, const void* x, gr_dtype x_t, const void* b, gr_dtype b_t, void* r,
                gr_dtype r_t, gr_dtype inter_t) {
  return guarded([&] {
    need(A, "matrix");
    need(x, "x");
    need(b, "b");
    need(r, "r");
    gr::launchResidual(*A->d, x, gr::toDType(x_t), b, gr::toDType(b_t), r, gr::toDType(r_t),
                       gr::toDType(inter_t), -1, nullptr, A->d->stream);
    GR_CUDA(cudaStreamSynchronize(A->d->stream));
  });
}

int gr_matrix_tune_spmv(gr_matrix* A, gr_dtype t, int32_t reps, int32_t* block, int32_t* chunks_per_warp,
                        int32_t* batch, float* ms) {
  return guarded([&] {
    need(A, "matrix");
    const gr::SpmvTuning g = gr::tuneSpmv(*A->d, gr::toDType(t), reps);
    if (block) *block = g.block;
    if (chunks_per_warp) *chunks_per_warp = g.chunksPerWarp;
    if (batch) *batch = g.batch;
    if (ms) *ms = g.ms;
  });
}

int gr_matrix_time_spmv(gr_matrix* A, const void* x, void* y, gr_dtype t, int32_t reps, int32_t flush_l2,
                        float* ms) {
  return guarded([&] {
    need(A, "matrix");
    need(x, "x");
    need(y, "y");
    need(ms, "ms");
    *ms = gr::timeSpmv(*A->d, x, y, gr::toDType(t), reps, flush_l2 != 0);
  });
}

int gr_vector_norm(gr_matrix* A, gr_norm norm, const void* x, gr_dtype t, double* out) {
  return guarded([&] {
    need(A, "matrix");
    need(x, "x");
    need(out, "out");
    if (norm == GR_NORM_NONE || norm < 0 || norm > GR_NORM_NONE) gr::fail(GR_EINVAL, "invalid norm");
    double* d = A->d->scalarOut.as<double>();
    gr::launchNorm(*A->d, x, gr::toDType(t), norm, d, A->d->stream);
    GR_CUDA(cudaMemcpyAsync(out, d, sizeof(double), cudaMemcpyDeviceToHost, A->d->stream));
    GR_CUDA(cudaStreamSynchronize(A->d->stream));
  });
}

int gr_matrix_inject_status(gr_matrix* A, int32_t status) {
  return guarded([&] {
    need(A, "matrix");
    if (status < 0) gr::fail(GR_EINVAL, "status must not be negative");
    GR_CUDA(cudaMemcpyAsync(A->d->errFlag.get(), &status, sizeof(int32_t), cudaMemcpyHostToDevice, A->d->stream));
    GR_CUDA(cudaStreamSynchronize(A->d->stream));
  });
}

int gr_vector_norms_noalloc(const void* x, int64_t n, int64_t count, int64_t ld, gr_dtype t,
                            gr_norm norm, double* out, void* stream) {
  return guarded([&] {
    need(x, "x");
    need(out, "out");
    if (norm == GR_NORM_NONE || norm < 0 || norm > GR_NORM_NONE) gr::fail(GR_EINVAL, "invalid norm");
    gr::launchNormsNoAlloc(x, n, count, ld, gr::toDType(t), norm, out, static_cast<cudaStream_t>(stream));
  });
}

int gr_decompose_vector(gr_matrix* A, const void* natural, void* tile_ordered, gr_dtype t) {
  return guarded([&] {
    need(A, "matrix");
    need(natural, "natural");
    need(tile_ordered, "tile_ordered");
    gr::launchPermute(*A->d, natural, tile_ordered, gr::toDType(t), true, A->d->stream);
    GR_CUDA(cudaStreamSynchronize(A->d->stream));
  });
}

int gr_compose_vector(gr_matrix* A, const void* tile_ordered, void* natural, gr_dtype t) {
  return guarded([&] {
    need(A, "matrix");
    need(natural, "natural");
    need(tile_ordered, "tile_ordered");
    gr::launchPermute(*A->d, tile_ordered, natural, gr::toDType(t), false, A->d->stream);
    GR_CUDA(cudaStreamSynchronize(A->d->stream));
  });
}

int gr_solver_create(gr_matrix* A, const char* json, gr_solver** out) {
  return guarded([&] {
    need(A, "matrix");
    need(json, "json");
    need(out, "out");
    auto s = gr::SolverTree::create(*A->d, json);
    *out = new gr_solver{std::move(s)};
  });
}

void gr_solver_destroy(gr_solver* s) { delete s; }

int gr_solve(gr_solver* s, void* x, gr_dtype x_t, const void* b, gr_dtype b_t, gr_stats* stats) {
  return guarded([&] {
    need(s, "solver");
    need(x, "x");
    need(b, "b");
    gr_stats st = s->s->solve(x, gr::toDType(x_t), b, gr::toDType(b_t));
    if (stats) *stats = st;
  });
}

int gr_solve_host(gr_solver* s, void* x, gr_dtype x_t, const void* b, gr_dtype b_t, gr_stats* stats) {
  return guarded([&] {
    need(s, "solver");
    need(x, "x");
    need(b, "b");
    gr_stats st = s->s->solveHost(x, gr::toDType(x_t), b, gr::toDType(b_t));
    if (stats) *stats = st;
  });
}

int gr_solver_time_repeated(gr_solver* s, void* x, gr_dtype x_t, const void* b, gr_dtype b_t, int32_t reps,
                            float* ms_per_run) {
  return guarded([&] {
    need(s, "solver");
    need(x, "x");
    need(b, "b");
    need(ms_per_run, "ms_per_run");
    *ms_per_run = s->s->timeRepeated(x, gr::toDType(x_t), b, gr::toDType(b_t), reps);
  });
}

int gr_matrix_update_values(gr_matrix* A, gr_host_matrix* h) {
  return guarded([&] {
    need(A, "matrix");
    need(h, "host matrix");
    A->d->updateValues(h->m);
  });
}

int gr_matrix_update_global_values(gr_matrix* A, const double* g_val, const double* g_diag) {
  return guarded([&] {
    need(A, "matrix");
    need(g_val, "g_val");
    need(g_diag, "g_diag");
    A->d->updateGlobalValues(g_val, g_diag, gr::DType::F64);
  });
}

int gr_solver_refresh(gr_solver* s) {
  return guarded([&] {
    need(s, "solver");
    s->s->refresh();
  });
}

int gr_solver_phi(gr_solver* s, void* out, gr_dtype t) {
  return guarded([&] {
    need(s, "solver");
    need(out, "out");
    s->s->copyPhi(out, gr::toDType(t));
  });
}

int gr_solver_name(const gr_solver* s, char* buf, size_t len) {
  return guarded([&] {
    need(s, "solver");
    need(buf, "buf");
    std::string nm = s->s->name();
    if (len == 0) gr::fail(GR_EINVAL, "buffer length is 0");
    std::strncpy(buf, nm.c_str(), len - 1);
    buf[len - 1] = '\0';
  });
}

int gr_config_parse(const char* json, char* name, size_t name_len, char* unknown_keys, size_t unknown_len) {
  return guarded([&] {
    need(json, "json");
    auto cfg = gr::SolverConfig::fromText(json);
    auto copy = [](const std::string& v, char* buf, size_t len) {
      if (!buf || len == 0) return;
      std::strncpy(buf, v.c_str(), len - 1);
      buf[len - 1] = '\0';
    };
    copy(cfg->solverName(), name, name_len);
    std::string unk;
    for (const gr::SolverConfig* c = cfg.get(); c;) {
      for (auto& k : c->unknownKeys) unk += (unk.empty() ? "" : ",") + k;
      if (c->preconditioner) {
        for (auto& k : c->preconditioner->unknownKeys) unk += (unk.empty() ? "" : ",") + k;
      }
      c = c->innerSolver.get();
    }
    copy(unk, unknown_keys, unknown_len);
  });
}


int gr_server_create(const gr_server_config* cfg, gr_server** out) {
  return guarded([&] {
    need(out, "out");
    gr_server_config c{0, -1, 0};
    if (cfg) c = *cfg;
    auto srv = std::make_unique<gr::Server>(c.slots, c.device, c.hbm_budget_bytes);
    *out = new gr_server{std::move(srv)};
  });
}

int gr_server_submit(gr_server* s, gr_host_matrix* h, const char* json, const void* b, gr_dtype t, uint64_t* id) {
  return guarded([&] {
    need(s, "server");
    need(h, "host matrix");
    need(json, "json");
    need(id, "id");
    *id = s->s->submit(h->m, json, b, gr::toDType(t));
  });
}

int gr_server_wait(gr_server* s, uint64_t id, double timeout_ms, void* x_out, gr_stats* stats,
                   gr_request_times* times) {
  int status = GR_OK, rc = GR_OK;
  std::string err;
  const int g = guarded([&] {
    need(s, "server");
    rc = s->s->wait(id, timeout_ms, x_out, stats, times, &status, &err);
  });
  if (g != GR_OK) return g;
  if (rc != GR_OK) {
    g_lastError = "request has not finished";
    return rc;
  }
  g_lastError = err;
  return status;
}

int gr_server_counters(gr_server* s, int64_t* queued, int64_t* running, int64_t* completed, int64_t* bytes_in_use,
                       int64_t* resident) {
  return guarded([&] {
    need(s, "server");
    s->s->counters(queued, running, completed, bytes_in_use, resident);
  });
}

int gr_server_submit_values(gr_server* s, gr_host_matrix* like, const double* g_val, const double* g_diag,
                            const char* json, const void* b, gr_dtype t, uint64_t* id) {
  return guarded([&] {
    need(s, "server");
    need(like, "like");
    need(g_val, "g_val");
    need(g_diag, "g_diag");
    need(json, "json");
    need(id, "id");
    *id = s->s->submitValues(like->m, g_val, g_diag, json, b, gr::toDType(t));
  });
}

int gr_server_cancel(gr_server* s, uint64_t id, int32_t* cancelled) {
  return guarded([&] {
    need(s, "server");
    const bool c = s->s->cancel(id);
    if (cancelled) *cancelled = c ? 1 : 0;
  });
}

void gr_server_destroy(gr_server* s) { delete s; }


int gr_batch_create(gr_host_matrix* const* systems, int32_t count, const char* json, gr_batch** out) {
  return guarded([&] {
    need(systems, "systems");
    need(json, "json");
    need(out, "out");
    if (count < 1 || count > 65536) gr::fail(GR_EINVAL, "count must be 1..65536");
    std::vector<std::shared_ptr<gr::HostMatrix>> parts;
    for (int32_t i = 0; i < count; ++i) {
      need(systems[i], "system");
      parts.push_back(systems[i]->m);
    }
    auto b = std::make_unique<gr::BatchSolve>(std::move(parts), json);
    *out = new gr_batch{std::move(b)};
  });
}

int gr_batch_solve_host(gr_batch* b, void* const* x, const void* const* rhs, gr_dtype t, gr_stats* stats) {
  return guarded([&] {
    need(b, "batch");
    need(x, "x");
    need(rhs, "b");
    const int S = b->b->systems();
    std::vector<void*> xs(x, x + S);
    std::vector<const void*> bs(rhs, rhs + S);
    std::vector<gr_stats> st = b->b->solveHost(xs, bs, gr::toDType(t));
    if (stats) std::copy(st.begin(), st.end(), stats);
  });
}

void gr_batch_destroy(gr_batch* b) { delete b; }

int gr_selftest_wait_timeout(int32_t* status, int64_t* elapsed_ns) {
  return guarded([&] {
    need(status, "status");
    need(elapsed_ns, "elapsed_ns");
    gr::selftestWaitTimeout(status, elapsed_ns);
  });
}

}  // extern "C"
