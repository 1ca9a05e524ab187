// Fused PBiCGStab kernels (pbicgstab/Solver.cpp:48-194) and the
// mixed-precision vector kernels of iterative refinement
// (iterative-refinement/Solver.cpp:48-123).
//
// Every reduction is a single-pass deterministic FP64 grid reduction whose
// last block also derives the scalars (alpha, omega, beta, convergence) and
// writes them into the device-resident KState, so an iteration runs without
// host round trips. Every kernel returns immediately once KState::done is
// set, which lets the host enqueue iterations ahead of the convergence test.
#include <algorithm>
#include <cmath>

#include "devmath.cuh"
#include "krylov.hpp"
#include "sell.cuh"

namespace gr {

namespace dev {

constexpr double kVsmall = 1e-37;  // Traits<float>::vsmall (common/Traits.hpp:43)

// SolverStats::checkConvergence (SolverStats.cpp:33-56).
__device__ __forceinline__ bool converged(const KState* st) {
  const double f = st->normFinal;
  bool c = f < st->absTol || f < st->normInit * st->relRes;
  if (st->relTol > 0) c = c || f < st->bNorm * st->relTol;
  return c;
}

// r = b - A x and r0 = r, with the norm of r and r0 . r.
template <class MV, class W, bool C16>
__global__ void __launch_bounds__(256) bicgInitKernel(SellView<MV> A, const W* __restrict__ x,
                                                       const W* __restrict__ b, W* __restrict__ r,
                                                       W* __restrict__ r0, KState* st, double* partials,
                                                       unsigned* counter, SegView seg, bool stateless) {
  __shared__ double smem[64];
  const SegPos sp = segPos(seg, A.n);
  st += sp.sys;
  const int lane = threadIdx.x & 31;
  const int nWarps = (sp.nb * blockDim.x) >> 5;
  const int cEnd = (sp.r1 + 31) >> 5;
  const int nk = st->normKind;
  double v[2] = {redIdentity(normOp(nk)), 0.0};
  const int ops[2] = {normOp(nk), RED_SUM};
  for (int c = (sp.r0 >> 5) + ((sp.rank * blockDim.x + threadIdx.x) >> 5); c < cEnd; c += nWarps) {
    const int row = c * 32 + lane;
    const W sum = sellRowSum<W, MV, W, C16>(A, x, c, lane, row < sp.r1);
    if (row < sp.r1) {
      W res = sub(__ldg(b + row), sum);
      r[row] = res;
      r0[row] = res;
      v[0] = normStep(v[0], toDouble(res), nk);
      v[1] = __dadd_rn(v[1], __dmul_rn(toDouble(res), toDouble(res)));
    }
  }
  if (stateless) return;  // the vectors only (reference-order reductions follow)
  double out[2];
  blockReduce<2>(v, ops, smem);
  if (gridReduceRank<2>(v, ops, partials + 2 * sp.b0, counter + sp.sys, smem, out, sp.rank, sp.nb) &&
      threadIdx.x == 0) {
    const double nrm = normFinish(out[0], nk);
    st->normInit = nrm;
    st->normFinal = nrm;
    st->rho = out[1];
    st->iter = 0;
    st->converged = 0;
    st->singular = fabs(out[1]) < kVsmall;
    st->status = isfinite(nrm) ? GR_OK : GR_ENONFINITE;
    st->done = st->maxIter <= 0 || st->singular || st->status != GR_OK;
  }
}

// y = A x with the step's dot products.
// mode 0: dot0 = r0 . y, alpha = rho / dot0 (pbicgstab/Solver.cpp:119-123)
// mode 1: dot0 = y . s, dot1 = y . y, omega = dot0 / dot1, singularity
//         check (pbicgstab/Solver.cpp:149-159)
template <class MV, class W, int MODE, bool C16>
__global__ void __launch_bounds__(256) spmvDotKernel(SellView<MV> A, const W* __restrict__ x,
                                                      W* __restrict__ y, const W* __restrict__ d1,
                                                      KState* st, double* partials, unsigned* counter,
                                                      SegView seg, bool stateless) {
  __shared__ double smem[64];
  const SegPos sp = segPos(seg, A.n);
  st += sp.sys;
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int nWarps = (sp.nb * blockDim.x) >> 5;
  const int cEnd = (sp.r1 + 31) >> 5;
  double v[2] = {0.0, 0.0};
  const int ops[2] = {RED_SUM, RED_SUM};
  for (int c = (sp.r0 >> 5) + ((sp.rank * blockDim.x + threadIdx.x) >> 5); c < cEnd; c += nWarps) {
    const int row = c * 32 + lane;
    const W yv = sellRowSum<W, MV, W, C16>(A, x, c, lane, row < sp.r1);
    if (row < sp.r1) {
      y[row] = yv;
      const double yd = toDouble(yv);
      v[0] = __dadd_rn(v[0], __dmul_rn(toDouble(__ldg(d1 + row)), yd));
      if (MODE == 1) v[1] = __dadd_rn(v[1], __dmul_rn(yd, yd));
    }
  }
  if (stateless) return;
  double out[2];
  blockReduce<2>(v, ops, smem);
  if (gridReduceRank<2>(v, ops, partials + 2 * sp.b0, counter + sp.sys, smem, out, sp.rank, sp.nb) &&
      threadIdx.x == 0) {
    if (MODE == 0) {
      st->dot0 = out[0];
      st->alpha = st->rho / out[0];
    } else {
      st->dot0 = out[0];
      st->dot1 = out[1];
      st->omega = out[0] / out[1];
      if (fabs(st->omega) < kVsmall) {
        st->singular = 1;
        st->done = 1;
      }
    }
  }
}

// x = x + alpha y + omega z, r = s - omega t (pbicgstab/Solver.cpp:164-168),
// then norm, convergence, iteration count and the next rho / beta.
// Four consecutive elements from index i (a multiple of 4 of a buffer
// aligned to 16 bytes): one 16-byte access for float, two for double.
__device__ __forceinline__ void load4(const float* p, int i, float (&o)[4]) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p + i));
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void load4(const double* p, int i, double (&o)[4]) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p + i));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p + i + 2));
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void store4(float* p, int i, const float (&o)[4]) {
  *reinterpret_cast<float4*>(p + i) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void store4(double* p, int i, const double (&o)[4]) {
  *reinterpret_cast<double2*>(p + i) = make_double2(o[0], o[1]);
  *reinterpret_cast<double2*>(p + i + 2) = make_double2(o[2], o[3]);
}

// x kept in float while the working type is double (workingType float64
// over float32 vectors, pbicgstab/Solver.cpp:63, :164): the update is
// evaluated in double and rounded to float.
__device__ __forceinline__ float roundTo(float v, bool) { return v; }
__device__ __forceinline__ double roundTo(double v, bool toFloat) {
  return toFloat ? static_cast<double>(__double2float_rn(v)) : v;
}

template <class W, bool VEC>
__global__ void __launch_bounds__(256) bicgUpdateKernel(W* __restrict__ x, const W* __restrict__ y,
                                                         const W* __restrict__ z, W* __restrict__ r,
                                                         const W* __restrict__ s, const W* __restrict__ t,
                                                         const W* __restrict__ r0, int n, KState* st,
                                                         double* partials, unsigned* counter, SegView seg,
                                                         bool stateless, bool roundX) {
  __shared__ double smem[64];
  const SegPos sp = segPos(seg, n);
  st += sp.sys;
  if (st->done) return;
  const W al = cvt<W>(st->alpha), om = cvt<W>(st->omega);
  const int nk = st->normKind;
  double v[2] = {redIdentity(normOp(nk)), 0.0};
  const int ops[2] = {normOp(nk), RED_SUM};
  // Four consecutive elements a thread, all loads issued before the
  // arithmetic, so that a warp keeps four times the bytes in flight; each
  // thread adds its elements to the reductions in index order.
  auto one = [&](int i) {
    x[i] = roundTo(add(add(x[i], mul(al, y[i])), mul(om, z[i])), roundX);
    const W rv = sub(s[i], mul(om, t[i]));
    r[i] = rv;
    v[0] = normStep(v[0], toDouble(rv), nk);
    v[1] = __dadd_rn(v[1], __dmul_rn(toDouble(__ldg(r0 + i)), toDouble(rv)));
  };
  const int stride = 4 * sp.nb * static_cast<int>(blockDim.x);
  for (int i0 = sp.r0 + 4 * (sp.rank * static_cast<int>(blockDim.x) + static_cast<int>(threadIdx.x)); i0 < sp.r1;
       i0 += stride) {
    if (VEC && i0 + 3 < sp.r1) {
      W xa[4], ya[4], za[4], sa[4], ta[4], ra[4];
      load4(x, i0, xa);
      load4(y, i0, ya);
      load4(z, i0, za);
      load4(s, i0, sa);
      load4(t, i0, ta);
      load4(r0, i0, ra);
      W xo[4], ro[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        xo[j] = roundTo(add(add(xa[j], mul(al, ya[j])), mul(om, za[j])), roundX);
        ro[j] = sub(sa[j], mul(om, ta[j]));
        v[0] = normStep(v[0], toDouble(ro[j]), nk);
        v[1] = __dadd_rn(v[1], __dmul_rn(toDouble(ra[j]), toDouble(ro[j])));
      }
      store4(x, i0, xo);
      store4(r, i0, ro);
    } else {
      for (int i = i0; i < min(i0 + 4, sp.r1); ++i) one(i);
    }
  }
  if (stateless) return;
  double out[2];
  blockReduce<2>(v, ops, smem);
  if (gridReduceRank<2>(v, ops, partials + 2 * sp.b0, counter + sp.sys, smem, out, sp.rank, sp.nb) &&
      threadIdx.x == 0) {
    st->normFinal = normFinish(out[0], nk);
    st->converged = converged(st);
    st->rhoOld = st->rho;
    st->iter += 1;
    if (!isfinite(st->normFinal)) st->status = GR_ENONFINITE;
    st->done = (st->converged && st->iter >= st->minIter) || st->iter >= st->maxIter ||
               st->status != GR_OK;
    if (!st->done) {
      // Next iteration's rho = r0 . r and beta (pbicgstab/Solver.cpp:91-99).
      st->rho = out[1];
      if (fabs(out[1]) < kVsmall) {
        st->singular = 1;
        st->done = 1;
      } else {
        st->beta = (st->rho / st->rhoOld) * (st->alpha / st->omega);
      }
    }
  }
}

// ---- the reference's reduction order --------------------------------------
// Float reductions in the order of Expression::reduce (Expression.cpp:
// 472-481, :597-769): per tile, six workers over chunks of floor(n_t/6/4)*4
// rows (worker 5 takes the rest), each chunk summed in row order from 0,
// then the six partials in worker order; with 6 rows or fewer in all, the
// tile's rows in order. Across tiles, runs of 368, 736, 1472 and then all
// tiles, each run summed in tile order (per worker first when some run has
// more than 6 values). Explicitly rounded operations only.
struct RefQ {
  int kind;  // RefKind
  const float* a;
  const float* b;
};

__device__ __forceinline__ float refVal(const RefQ& q, int i) {
  const float a = q.a[i];
  return q.kind == static_cast<int>(RefKind::Dot) ? __fmul_rn(a, q.b[i]) : a;
}
__device__ __forceinline__ float refStep(float acc, float v, int kind) {
  return kind == static_cast<int>(RefKind::SquareSum) ? __fadd_rn(acc, __fmul_rn(v, v)) : __fadd_rn(acc, v);
}

// One block (two warps) per tile: warp q computes reduction q, lanes 0..5
// being the reference's six workers.
__global__ void __launch_bounds__(64) refTileKernel(const int* __restrict__ tileStart, long long total, RefQ q0,
                                                    RefQ q1, float* __restrict__ out, int P, const KState* st) {
  __shared__ float part[2][6];
  if (st->done) return;
  const int T = blockIdx.x;
  const int base = tileStart[T];
  const int nt = tileStart[T + 1] - base;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const RefQ q = w == 0 ? q0 : q1;
  if (q.kind == static_cast<int>(RefKind::None)) return;  // warp-uniform
  if (q.kind == static_cast<int>(RefKind::Max)) {
    float m = -INFINITY;
    for (int i = lane; i < nt; i += 32) m = fmaxf(m, q.a[base + i]);
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) out[w * P + T] = m;
    return;
  }
  if (total > 6) {
    const int chunk = (nt / 6 / 4) * 4;
    if (lane < 6) {
      const int s0 = chunk * lane, e0 = lane == 5 ? nt : s0 + chunk;
      float acc = 0.0f;
      for (int i = s0; i < e0; ++i) acc = refStep(acc, refVal(q, base + i), q.kind);
      part[w][lane] = acc;
    }
    __syncwarp();
    if (lane == 0) {
      float acc = 0.0f;
      for (int k = 0; k < 6; ++k) acc = __fadd_rn(acc, part[w][k]);
      out[w * P + T] = acc;
    }
  } else if (lane == 0) {
    float acc = 0.0f;
    for (int i = 0; i < nt; ++i) acc = refStep(acc, refVal(q, base + i), q.kind);
    out[w * P + T] = acc;
  }
}

__device__ float refSeq(const float* v, int s0, int e0) {
  float acc = 0.0f;
  for (int i = s0; i < e0; ++i) acc = __fadd_rn(acc, v[i]);
  return acc;
}
__device__ float refWorkers(const float* v, int cnt) {
  const int chunk = (cnt / 6 / 4) * 4;
  float part[6];
  for (int w = 0; w < 6; ++w) part[w] = refSeq(v, chunk * w, w == 5 ? cnt : chunk * w + chunk);
  return refSeq(part, 0, 6);
}
constexpr int kRefMaxRuns = 256;  // values after the first stage: at most 368 * 256 tiles
// The cross-tile stages over the P per-tile values.
__device__ float refAcrossTiles(const float* v, int P, bool isMax) {
  if (isMax) {
    float m = -INFINITY;
    for (int t = 0; t < P; ++t) m = fmaxf(m, v[t]);
    return m;
  }
  if (P == 1) return v[0];
  float cur[kRefMaxRuns];
  int at[kRefMaxRuns];
  int n = 0;
  {
    const int G = 368;
    const bool pw = (P < G ? P : G) > 6;  // the first run is the largest
    for (int g = 0; g * G < P; ++g) {
      const int cnt = min(G, P - g * G);
      cur[n] = pw ? refWorkers(v + g * G, cnt) : refSeq(v + g * G, 0, cnt);
      at[n++] = g * G;
    }
  }
  const int runs[3] = {736, 1472, 0};  // 0: all
  for (int k = 0; k < 3 && n > 1; ++k) {
    const int G = runs[k];
    float nxt[kRefMaxRuns];
    int nat[kRefMaxRuns], start[kRefMaxRuns + 1];
    int m = 0;
    for (int i = 0; i < n; ++i) {
      const int key = G == 0 ? 0 : at[i] / G * G;
      if (m == 0 || nat[m - 1] != key) {
        nat[m] = key;
        start[m++] = i;
      }
    }
    start[m] = n;
    bool pw = false;
    for (int g = 0; g < m; ++g) pw = pw || start[g + 1] - start[g] > 6;
    for (int g = 0; g < m; ++g) {
      const int cnt = start[g + 1] - start[g];
      nxt[g] = pw ? refWorkers(cur + start[g], cnt) : refSeq(cur + start[g], 0, cnt);
    }
    for (int g = 0; g < m; ++g) {
      cur[g] = nxt[g];
      at[g] = nat[g];
    }
    n = m;
  }
  return cur[0];
}

__device__ __forceinline__ float refNormFinish(float v, int normKind) {
  return normKind == GR_NORM_L2 ? __fsqrt_rn(v) : v;
}

__global__ void refStateKernel(const float* __restrict__ tiles, int P, int kind0, int kind1, int stage,
                               KState* st) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const bool pre = stage == static_cast<int>(RefStage::BNorm) || stage == static_cast<int>(RefStage::Init);
  if (!pre && st->done) return;
  const float q0 = kind0 ? refAcrossTiles(tiles, P, kind0 == static_cast<int>(RefKind::Max)) : 0.0f;
  const float q1 = kind1 ? refAcrossTiles(tiles + P, P, kind1 == static_cast<int>(RefKind::Max)) : 0.0f;
  const float vsmall = 1e-37f;  // Traits<float>::vsmall (common/Traits.hpp:43)
  const int nk = st->normKind;
  switch (static_cast<RefStage>(stage)) {
    case RefStage::BNorm:
      st->bNorm = refNormFinish(q0, nk);
      break;
    case RefStage::Init: {
      const float nrm = refNormFinish(q1, nk);
      st->rho = q0;
      st->normInit = nrm;
      st->normFinal = nrm;
      st->iter = 0;
      st->converged = 0;
      st->singular = fabsf(q0) < vsmall;
      st->status = isfinite(nrm) ? GR_OK : GR_ENONFINITE;
      st->done = st->maxIter <= 0 || st->singular || st->status != GR_OK;
      break;
    }
    case RefStage::Alpha:
      st->alpha = __fdiv_rn(static_cast<float>(st->rho), q0);
      break;
    case RefStage::Omega: {
      const float om = __fdiv_rn(q1, q0);
      st->omega = om;
      st->singular = fabsf(om) < vsmall;
      st->done = st->singular;
      break;
    }
    case RefStage::Update: {
      const float fin = refNormFinish(q1, nk);
      const float init = static_cast<float>(st->normInit);
      bool c = fin < static_cast<float>(st->absTol) || fin < __fmul_rn(init, static_cast<float>(st->relRes));
      if (st->relTol > 0) c = c || fin < __fmul_rn(static_cast<float>(st->bNorm), static_cast<float>(st->relTol));
      st->normFinal = fin;
      st->converged = c;
      st->rhoOld = st->rho;
      st->iter += 1;
      st->status = isfinite(fin) ? GR_OK : GR_ENONFINITE;
      st->done = (c && st->iter >= st->minIter) || st->iter >= st->maxIter || st->status != GR_OK;
      if (!st->done) {
        st->rho = q0;
        if (fabsf(q0) < vsmall) {
          st->singular = 1;
          st->done = 1;
        } else {
          st->beta = __fmul_rn(__fdiv_rn(q0, static_cast<float>(st->rhoOld)),
                               __fdiv_rn(static_cast<float>(st->alpha), static_cast<float>(st->omega)));
        }
      }
      break;
    }
  }
}

__global__ void stateResetKernel(KState* st, KState init, int count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) st[i] = init;
}

__global__ void skipSystemsKernel(KState* st, const int* __restrict__ skip, int count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    if (skip[i]) st[i].done = 1;
}

// ---- mixed precision ---------------------------------------------------
__global__ void castUpKernel(const float* __restrict__ x, void* phi, int E, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (E == GR_FLOAT64) static_cast<double*>(phi)[i] = static_cast<double>(x[i]);
    else if (E == GR_TWOFLOAT32) static_cast<float2*>(phi)[i] = make_float2(x[i], 0.0f);
    else static_cast<float*>(phi)[i] = x[i];
  }
}

// phi = phi + corr.cast(E) (iterative-refinement/Solver.cpp:103).
__global__ void phiUpdateKernel(void* phi, const float* __restrict__ corr, int E, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (E == GR_FLOAT64) {
      double* p = static_cast<double*>(phi);
      p[i] = __dadd_rn(p[i], static_cast<double>(corr[i]));
    } else if (E == GR_TWOFLOAT32) {
      float2* p = static_cast<float2*>(phi);
      const float2 v = p[i];
      const dw s = dwPlusFp(dw{v.x, v.y}, corr[i]);
      p[i] = make_float2(s.h, s.l);
    } else {
      float* p = static_cast<float*>(phi);
      p[i] = __fadd_rn(p[i], corr[i]);
    }
  }
}

__global__ void convertKernel(const void* src, int from, void* dst, int to, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d;
    float f;
    if (from == GR_FLOAT64) {
      d = static_cast<const double*>(src)[i];
      f = __double2float_rn(d);
    } else if (from == GR_TWOFLOAT32) {
      const float2 v = static_cast<const float2*>(src)[i];
      d = static_cast<double>(v.x) + static_cast<double>(v.y);
      f = dwToFloat(dw{v.x, v.y});
    } else {
      f = static_cast<const float*>(src)[i];
      d = static_cast<double>(f);
    }
    if (to == GR_FLOAT64) static_cast<double*>(dst)[i] = d;
    else static_cast<float*>(dst)[i] = f;
  }
}

}  // namespace dev

// ---------------------------------------------------------------------------
namespace {

int elemBlocks(const DeviceMatrix& A, i64 n) {
  return static_cast<int>(std::max<i64>(1, std::min<i64>(A.redBlocks, (n + 255) / 256)));
}

int elemBlocksN(i64 n) { return static_cast<int>(std::max<i64>(1, std::min<i64>(148 * 8, (n + 255) / 256))); }

}  // namespace

namespace {
// Launch geometry and reduction scratch of a Krylov kernel: the whole matrix
// as one system, or the batch's per-system split (`chunk`: row-chunk kernels,
// else elementwise kernels).
struct Launch {
  int blocks;
  dev::SegView seg;
  double* partials;
  unsigned* counter;
};

Launch krylovLaunch(DeviceMatrix& A, bool chunk) {
  if (!A.batch) {
    return Launch{chunk ? A.spmvBlocks() : elemBlocks(A, A.n), dev::SegView{}, A.partials.as<double>(),
                  A.counter.as<unsigned>()};
  }
  const BatchSeg& B = *A.batch;
  dev::SegView g;
  if (chunk) {
    g.blockSys = B.chunkSys.as<int>();
    g.blockRank = B.chunkRank.as<int>();
    g.sysBlocks = B.chunkBlocks.as<int>();
    g.sysBlock0 = B.chunkBlock0.as<int>();
  } else {
    g.blockSys = B.elemSys.as<int>();
    g.blockRank = B.elemRank.as<int>();
    g.sysBlocks = B.elemBlocks.as<int>();
    g.sysBlock0 = B.elemBlock0.as<int>();
  }
  g.sysRow0 = B.row0.as<int>();
  g.sysRowEnd = B.rowEnd.as<int>();
  return Launch{chunk ? B.chunkGrid : B.elemGrid, g, B.partials.as<double>(), B.counters.as<unsigned>()};
}
}  // namespace

namespace {
template <class MV, class W>
void bicgInitT(DeviceMatrix& A, const void* x, const void* b, void* r, void* r0, KState* st, cudaStream_t s,
               bool stateless) {
  const Launch L = krylovLaunch(A, true);
  auto kernel = A.sell.compact ? dev::bicgInitKernel<MV, W, true> : dev::bicgInitKernel<MV, W, false>;
  kernel<<<L.blocks, 256, 0, s>>>(sellView<MV>(A), static_cast<const W*>(x), static_cast<const W*>(b),
                                  static_cast<W*>(r), static_cast<W*>(r0), st, L.partials, L.counter, L.seg,
                                  stateless);
}
}  // namespace

void launchBicgInit(DeviceMatrix& A, const void* x, const void* b, void* r, void* r0, KState* st, DType W,
                    cudaStream_t s, bool stateless) {
  if (A.vt == DType::F32 && W == DType::F32) bicgInitT<float, float>(A, x, b, r, r0, st, s, stateless);
  else if (A.vt == DType::F32 && W == DType::F64) bicgInitT<float, double>(A, x, b, r, r0, st, s, stateless);
  else if (A.vt == DType::F64 && W == DType::F64) bicgInitT<double, double>(A, x, b, r, r0, st, s, stateless);
  else fail(GR_EUNSUPPORTED, "PBiCGStab with float64 coefficients needs float64 vectors");
  checkLaunch("bicg_init");
}

namespace {
template <class MV, class W>
void spmvDotT(DeviceMatrix& A, const void* x, void* y, const void* d1, int mode, KState* st, cudaStream_t s,
              bool stateless) {
  const Launch L = krylovLaunch(A, true);
  const bool c16 = A.sell.compact;
  auto kernel = mode == 0 ? (c16 ? dev::spmvDotKernel<MV, W, 0, true> : dev::spmvDotKernel<MV, W, 0, false>)
                          : (c16 ? dev::spmvDotKernel<MV, W, 1, true> : dev::spmvDotKernel<MV, W, 1, false>);
  kernel<<<L.blocks, 256, 0, s>>>(sellView<MV>(A), static_cast<const W*>(x), static_cast<W*>(y),
                                  static_cast<const W*>(d1), st, L.partials, L.counter, L.seg, stateless);
}
}  // namespace

namespace {
template <class MV, class W, bool C16>
int occupancyOf() {
  const void* fns[3] = {reinterpret_cast<const void*>(dev::bicgInitKernel<MV, W, C16>),
                        reinterpret_cast<const void*>(dev::spmvDotKernel<MV, W, 0, C16>),
                        reinterpret_cast<const void*>(dev::spmvDotKernel<MV, W, 1, C16>)};
  int occ = 1 << 20;
  for (const void* f : fns) {
    int n = 0;
    GR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, 256, 0));
    occ = std::min(occ, n);
  }
  return occ;
}
}  // namespace

int sellKernelOccupancy(DType vt, bool c16) {
  if (vt == DType::F64) return c16 ? occupancyOf<double, double, true>() : occupancyOf<double, double, false>();
  const int a = c16 ? occupancyOf<float, float, true>() : occupancyOf<float, float, false>();
  const int b = c16 ? occupancyOf<float, double, true>() : occupancyOf<float, double, false>();
  return std::min(a, b);
}

void launchSpmvDot(DeviceMatrix& A, const void* x, void* y, const void* d1, int mode, KState* st, DType W,
                   cudaStream_t s, bool stateless) {
  if (A.vt == DType::F32 && W == DType::F32) spmvDotT<float, float>(A, x, y, d1, mode, st, s, stateless);
  else if (A.vt == DType::F32 && W == DType::F64) spmvDotT<float, double>(A, x, y, d1, mode, st, s, stateless);
  else if (A.vt == DType::F64 && W == DType::F64) spmvDotT<double, double>(A, x, y, d1, mode, st, s, stateless);
  else fail(GR_EUNSUPPORTED, "PBiCGStab with float64 coefficients needs float64 vectors");
  checkLaunch("spmv_dot");
}

void launchBicgUpdate(DeviceMatrix& A, void* x, const void* y, const void* z, void* r, const void* sv,
                      const void* t, const void* r0, KState* st, DType W, cudaStream_t s, bool stateless,
                      bool roundX) {
  const Launch L = krylovLaunch(A, false);
  // 16-byte accesses need every vector 16-byte aligned (segments start at
  // multiples of 32 rows); otherwise the same order element by element.
  const bool vec = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y) | reinterpret_cast<uintptr_t>(z) |
                     reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(sv) | reinterpret_cast<uintptr_t>(t) |
                     reinterpret_cast<uintptr_t>(r0)) &
                    15u) == 0;
  if (W == DType::F32)
    (vec ? dev::bicgUpdateKernel<float, true> : dev::bicgUpdateKernel<float, false>)<<<L.blocks, 256, 0, s>>>(
        static_cast<float*>(x), static_cast<const float*>(y), static_cast<const float*>(z), static_cast<float*>(r),
        static_cast<const float*>(sv), static_cast<const float*>(t), static_cast<const float*>(r0), A.n, st,
        L.partials, L.counter, L.seg, stateless, false);
  else
    (vec ? dev::bicgUpdateKernel<double, true> : dev::bicgUpdateKernel<double, false>)<<<L.blocks, 256, 0, s>>>(
        static_cast<double*>(x), static_cast<const double*>(y), static_cast<const double*>(z),
        static_cast<double*>(r), static_cast<const double*>(sv), static_cast<const double*>(t),
        static_cast<const double*>(r0), A.n, st, L.partials, L.counter, L.seg, stateless, roundX);
  checkLaunch("bicg_update");
}

void launchRefReduce(DeviceMatrix& A, const RefRed& q0, const RefRed& q1, RefStage stage, KState* st, void* tiles,
                     cudaStream_t s) {
  if (A.P > 368 * dev::kRefMaxRuns) fail(GR_EUNSUPPORTED, "reference-order reductions support up to 94208 tiles");
  auto q = [](const RefRed& r) {
    return dev::RefQ{static_cast<int>(r.kind), static_cast<const float*>(r.a), static_cast<const float*>(r.b)};
  };
  float* t = static_cast<float*>(tiles);
  dev::refTileKernel<<<A.P, 64, 0, s>>>(A.tileStart.as<int>(), static_cast<long long>(A.n), q(q0), q(q1), t, A.P, st);
  checkLaunch("ref_tile_reduce");
  dev::refStateKernel<<<1, 32, 0, s>>>(t, A.P, static_cast<int>(q0.kind), static_cast<int>(q1.kind),
                                       static_cast<int>(stage), st);
  checkLaunch("ref_state");
}

void launchStateReset(KState* st, const KState& init, cudaStream_t s, int count) {
  dev::stateResetKernel<<<(count + 255) / 256, 256, 0, s>>>(st, init, count);
  checkLaunch("state_reset");
}

void launchSkipSystems(KState* st, const int* skip, int count, cudaStream_t s) {
  dev::skipSystemsKernel<<<(count + 255) / 256, 256, 0, s>>>(st, skip, count);
  checkLaunch("skip_systems");
}

void launchNormInto(DeviceMatrix& A, const void* x, DType t, int normKind, double* out, cudaStream_t s) {
  launchNorm(A, x, t, normKind, out, s);
}

void launchCastUp(const float* x, void* phi, DType E, int n, cudaStream_t s) {
  dev::castUpKernel<<<elemBlocksN(n), 256, 0, s>>>(x, phi, static_cast<int>(E), n);
  checkLaunch("cast_up");
}

void launchPhiUpdate(void* phi, const float* corr, DType E, int n, cudaStream_t s) {
  dev::phiUpdateKernel<<<elemBlocksN(n), 256, 0, s>>>(phi, corr, static_cast<int>(E), n);
  checkLaunch("phi_update");
}

void launchCastDown(const void* phi, float* x, DType E, int n, cudaStream_t s) {
  dev::convertKernel<<<elemBlocksN(n), 256, 0, s>>>(phi, static_cast<int>(E), x, GR_FLOAT32, n);
  checkLaunch("cast_down");
}

void launchConvert(const void* src, DType from, void* dst, DType to, int n, cudaStream_t s) {
  dev::convertKernel<<<elemBlocksN(n), 256, 0, s>>>(src, static_cast<int>(from), dst, static_cast<int>(to), n);
  checkLaunch("convert");
}

}  // namespace gr
