// Fused PBiCGStab kernels (pbicgstab/Solver.cpp:48-194) and the
// mixed-precision vector kernels of iterative refinement
// (iterative-refinement/Solver.cpp:48-123).
//
// Every reduction is a single-pass deterministic FP64 grid reduction whose
// last block also derives the scalars (alpha, omega, beta, convergence) and
// writes them into the device-resident KState, so an iteration runs without
// host round trips. Every kernel returns immediately once KState::done is
// set, which lets the host enqueue iterations ahead of the convergence test.
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
template <class MV, class W>
__global__ void __launch_bounds__(256) bicgInitKernel(SellView<MV> A, const W* __restrict__ x,
                                                       const W* __restrict__ b, W* __restrict__ r,
                                                       W* __restrict__ r0, KState* st, double* partials,
                                                       unsigned* counter, SegView seg) {
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
    const int s0 = __ldg(A.base + c);
    const int K = (__ldg(A.base + c + 1) - s0) >> 5;
    if (row < sp.r1) {
      W res = sub(__ldg(b + row), sellRowSum<W>(A, x, row, s0, K, lane));
      r[row] = res;
      r0[row] = res;
      v[0] = normStep(v[0], toDouble(res), nk);
      v[1] = __dadd_rn(v[1], __dmul_rn(toDouble(res), toDouble(res)));
    }
  }
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
template <class MV, class W, int MODE>
__global__ void __launch_bounds__(256) spmvDotKernel(SellView<MV> A, const W* __restrict__ x,
                                                      W* __restrict__ y, const W* __restrict__ d1,
                                                      KState* st, double* partials, unsigned* counter,
                                                      SegView seg) {
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
    const int s0 = __ldg(A.base + c);
    const int K = (__ldg(A.base + c + 1) - s0) >> 5;
    if (row < sp.r1) {
      const W yv = sellRowSum<W>(A, x, row, s0, K, lane);
      y[row] = yv;
      const double yd = toDouble(yv);
      v[0] = __dadd_rn(v[0], __dmul_rn(toDouble(__ldg(d1 + row)), yd));
      if (MODE == 1) v[1] = __dadd_rn(v[1], __dmul_rn(yd, yd));
    }
  }
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

template <class W, bool VEC>
__global__ void __launch_bounds__(256) bicgUpdateKernel(W* __restrict__ x, const W* __restrict__ y,
                                                         const W* __restrict__ z, W* __restrict__ r,
                                                         const W* __restrict__ s, const W* __restrict__ t,
                                                         const W* __restrict__ r0, int n, KState* st,
                                                         double* partials, unsigned* counter, SegView seg) {
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
    x[i] = add(add(x[i], mul(al, y[i])), mul(om, z[i]));
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
        xo[j] = add(add(xa[j], mul(al, ya[j])), mul(om, za[j]));
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

__global__ void stateResetKernel(KState* st, KState init, int count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) st[i] = init;
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

void launchBicgInit(DeviceMatrix& A, const void* x, const void* b, void* r, void* r0, KState* st, DType W,
                    cudaStream_t s) {
  const Launch L = krylovLaunch(A, true);
  if (A.vt == DType::F32 && W == DType::F32)
    dev::bicgInitKernel<float, float><<<L.blocks, 256, 0, s>>>(
        sellView<float>(A), static_cast<const float*>(x), static_cast<const float*>(b), static_cast<float*>(r),
        static_cast<float*>(r0), st, L.partials, L.counter, L.seg);
  else if (A.vt == DType::F32 && W == DType::F64)
    dev::bicgInitKernel<float, double><<<L.blocks, 256, 0, s>>>(
        sellView<float>(A), static_cast<const double*>(x), static_cast<const double*>(b), static_cast<double*>(r),
        static_cast<double*>(r0), st, L.partials, L.counter, L.seg);
  else if (A.vt == DType::F64 && W == DType::F64)
    dev::bicgInitKernel<double, double><<<L.blocks, 256, 0, s>>>(
        sellView<double>(A), static_cast<const double*>(x), static_cast<const double*>(b), static_cast<double*>(r),
        static_cast<double*>(r0), st, L.partials, L.counter, L.seg);
  else
    fail(GR_EUNSUPPORTED, "PBiCGStab with float64 coefficients needs float64 vectors");
  checkLaunch("bicg_init");
}

namespace {
template <class MV, class W>
void spmvDotT(DeviceMatrix& A, const void* x, void* y, const void* d1, int mode, KState* st, cudaStream_t s) {
  const Launch L = krylovLaunch(A, true);
  if (mode == 0)
    dev::spmvDotKernel<MV, W, 0><<<L.blocks, 256, 0, s>>>(sellView<MV>(A), static_cast<const W*>(x),
                                                          static_cast<W*>(y), static_cast<const W*>(d1), st,
                                                          L.partials, L.counter, L.seg);
  else
    dev::spmvDotKernel<MV, W, 1><<<L.blocks, 256, 0, s>>>(sellView<MV>(A), static_cast<const W*>(x),
                                                          static_cast<W*>(y), static_cast<const W*>(d1), st,
                                                          L.partials, L.counter, L.seg);
}
}  // namespace

void launchSpmvDot(DeviceMatrix& A, const void* x, void* y, const void* d1, int mode, KState* st, DType W,
                   cudaStream_t s) {
  if (A.vt == DType::F32 && W == DType::F32) spmvDotT<float, float>(A, x, y, d1, mode, st, s);
  else if (A.vt == DType::F32 && W == DType::F64) spmvDotT<float, double>(A, x, y, d1, mode, st, s);
  else if (A.vt == DType::F64 && W == DType::F64) spmvDotT<double, double>(A, x, y, d1, mode, st, s);
  else fail(GR_EUNSUPPORTED, "PBiCGStab with float64 coefficients needs float64 vectors");
  checkLaunch("spmv_dot");
}

void launchBicgUpdate(DeviceMatrix& A, void* x, const void* y, const void* z, void* r, const void* sv,
                      const void* t, const void* r0, KState* st, DType W, cudaStream_t s) {
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
        L.partials, L.counter, L.seg);
  else
    (vec ? dev::bicgUpdateKernel<double, true> : dev::bicgUpdateKernel<double, false>)<<<L.blocks, 256, 0, s>>>(
        static_cast<double*>(x), static_cast<const double*>(y), static_cast<const double*>(z),
        static_cast<double*>(r), static_cast<const double*>(sv), static_cast<const double*>(t),
        static_cast<const double*>(r0), A.n, st, L.partials, L.counter, L.seg);
  checkLaunch("bicg_update");
}

void launchStateReset(KState* st, const KState& init, cudaStream_t s, int count) {
  dev::stateResetKernel<<<(count + 255) / 256, 256, 0, s>>>(st, init, count);
  checkLaunch("state_reset");
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
