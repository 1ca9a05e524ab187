// Tile-local preconditioners: block ILU(0) / DILU and Gauss-Seidel.
//
// One thread block per tile (the reference's IPU tile). A tile's rows are
// swept level by level (LevelSchedule); rows of a level run in parallel and
// a __syncthreads() separates levels, which reproduces the reference's
// sequential per-tile loops operation for operation
// (ilu/Solver.cpp:134-292 and :367-550, gauss-seidel/Solver.cpp:45-86).
// The tile's slice of the vector being solved for lives in shared memory
// when it fits (tile rows * sizeof(W) <= the opt-in shared memory limit),
// otherwise in the output vector in HBM.
#include <algorithm>

#include "devmath.cuh"
#include "krylov.hpp"
#include "sell.cuh"

namespace gr {

namespace dev {

struct SchedView {
  const int* __restrict__ tileLvlStart;
  const int* __restrict__ lvlRowStart;
  const long long* __restrict__ lvlSlotStart;
  const int* __restrict__ rows;
  const int* __restrict__ col;
};

inline SchedView schedView(const LevelSchedule& S) {
  return SchedView{S.tileLvlStart.as<int>(), S.lvlRowStart.as<int>(), S.lvlSlotStart.as<long long>(),
                   S.rows.as<int>(), S.col.as<int>()};
}

// Value of a[i, j] in the tile-local CRS (row given in tile order, column as
// tile-local id), 0 when the pattern has no such entry: getOffDiagValue
// (ilu/Solver.cpp:150-161).
template <class MV>
__device__ __forceinline__ MV lookup(const int* __restrict__ rowPtr, const int* __restrict__ colLocal,
                                     const MV* vals, int row, int j) {
  MV r = MV(0);
  for (int a = rowPtr[row]; a < rowPtr[row + 1]; ++a)
    if (colLocal[a] == j) r = vals[a];
  return r;
}

// ILU(0) / DILU factorisation of every tile (factorizeRow,
// ilu/Solver.cpp:167-218). F and D start as copies of the off-diagonal values
// (tile-local CRS order) and of the diagonal, and are factored in place.
template <class MV>
__global__ void __launch_bounds__(256) iluFactorKernel(const int* __restrict__ tileStart, SchedView L,
                                                        const int* __restrict__ rowPtr,
                                                        const int* __restrict__ colLocal, MV* F, MV* D,
                                                        const MV* __restrict__ Aoff, bool dilu) {
  const int T = blockIdx.x;
  const int base = tileStart[T];
  const int nRows = tileStart[T + 1] - base;
  for (int l = L.tileLvlStart[T]; l < L.tileLvlStart[T + 1]; ++l) {
    const int r0 = L.lvlRowStart[l], k = L.lvlRowStart[l + 1] - r0;
    for (int q = threadIdx.x; q < k; q += blockDim.x) {
      const int row = L.rows[r0 + q];
      const int il = row - base;
      const int iStart = rowPtr[row], iEnd = rowPtr[row + 1];
      for (int ik = iStart; ik < iEnd; ++ik) {
        const int kk = colLocal[ik];
        if (kk >= il) break;
        const int pk = base + kk;
        const MV a_kk = D[pk];
        if (!dilu) {
          F[ik] = dvd(F[ik], a_kk);
          const MV a_ik = F[ik];
          for (int ij = ik + 1; ij < iEnd; ++ij) {
            const int j = colLocal[ij];
            if (j >= nRows) break;
            const MV a_kj = lookup(rowPtr, colLocal, F, pk, j);
            F[ij] = sub(F[ij], mul(a_ik, a_kj));
          }
          const MV a_ki = lookup(rowPtr, colLocal, F, pk, il);
          D[row] = sub(D[row], mul(a_ik, a_ki));
        } else {
          const MV a_ik = Aoff[ik];
          const MV a_ki = lookup(rowPtr, colLocal, Aoff, pk, il);
          D[row] = sub(D[row], dvd(mul(a_ik, a_ki), a_kk));
        }
      }
    }
    __syncthreads();
  }
}

template <class MV>
__global__ void invertKernel(const MV* __restrict__ D, MV* __restrict__ inv, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    inv[i] = dvd(MV(1), D[i]);
}

template <class MV>
__global__ void packKernel(const int* __restrict__ src, const MV* __restrict__ F, MV* __restrict__ out,
                           long long slots) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < slots;
       s += (long long)gridDim.x * blockDim.x) {
    const int k = src[s];
    out[s] = k >= 0 ? F[k] : MV(0);
  }
}

// The vector a fused preconditioner application starts from.
template <class W>
struct Pro {
  int kind;
  const W* __restrict__ b;
  const W* __restrict__ r;
  W* pOrS;
  const W* __restrict__ v;
  const KState* st;

  __device__ __forceinline__ W operator()(int i, W beta, W omega, W alpha, bool first) const {
    if (kind == static_cast<int>(Prologue::Plain)) return b[i];
    if (kind == static_cast<int>(Prologue::PUpdate)) {
      // pA = rA + beta * (pA - omega * AyA) (pbicgstab/Solver.cpp:98-101)
      W p = first ? r[i] : add(r[i], mul(beta, sub(pOrS[i], mul(omega, v[i]))));
      pOrS[i] = p;
      return p;
    }
    // sA = rA - alpha * AyA (pbicgstab/Solver.cpp:129)
    W s = sub(r[i], mul(alpha, v[i]));
    pOrS[i] = s;
    return s;
  }
};

// y = M^-1 * prologue for every tile. L holds the strictly lower entries
// (ascending), U the upper non-halo entries (descending) of each row.
template <class MV, class W, bool SMEM>
__global__ void __launch_bounds__(256) iluApplyKernel(const int* __restrict__ tileStart, SchedView L,
                                                       const MV* __restrict__ Lval, SchedView U,
                                                       const MV* __restrict__ Uval, const MV* __restrict__ inv,
                                                       bool dilu, Pro<W> pro, W* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smemRaw[];
  if (pro.st && pro.st->done) return;
  const int T = blockIdx.x;
  const int base = tileStart[T];
  const int nRows = tileStart[T + 1] - base;
  W* xs = SMEM ? reinterpret_cast<W*>(smemRaw) : y + base;
  W beta = W(0), omega = W(0), alpha = W(0);
  bool first = true;
  if (pro.st) {
    beta = cvt<W>(pro.st->beta);
    omega = cvt<W>(pro.st->omega);
    alpha = cvt<W>(pro.st->alpha);
    first = pro.st->iter == 0;
  }
  for (int i = threadIdx.x; i < nRows; i += blockDim.x) xs[i] = pro(base + i, beta, omega, alpha, first);
  __syncthreads();
  // Forward substitution (ilu/Solver.cpp:380-411).
  for (int l = L.tileLvlStart[T]; l < L.tileLvlStart[T + 1]; ++l) {
    const int r0 = L.lvlRowStart[l], k = L.lvlRowStart[l + 1] - r0;
    const long long s0 = L.lvlSlotStart[l];
    const int E = static_cast<int>((L.lvlSlotStart[l + 1] - s0) / (k > 0 ? k : 1));
    for (int q = threadIdx.x; q < k; q += blockDim.x) {
      const int il = L.rows[r0 + q] - base;
      W temp = xs[il];
      for (int e = 0; e < E; ++e) {
        const long long s = s0 + (long long)e * k + q;
        const int c = __ldg(L.col + s);
        if (c < 0) break;
        temp = sub(temp, mul(cvt<W>(__ldg(Lval + s)), xs[c - base]));
      }
      xs[il] = dilu ? mul(temp, cvt<W>(__ldg(inv + base + il))) : temp;
    }
    __syncthreads();
  }
  // Backward substitution (ilu/Solver.cpp:413-442).
  for (int l = U.tileLvlStart[T]; l < U.tileLvlStart[T + 1]; ++l) {
    const int r0 = U.lvlRowStart[l], k = U.lvlRowStart[l + 1] - r0;
    const long long s0 = U.lvlSlotStart[l];
    const int E = static_cast<int>((U.lvlSlotStart[l + 1] - s0) / (k > 0 ? k : 1));
    for (int q = threadIdx.x; q < k; q += blockDim.x) {
      const int il = U.rows[r0 + q] - base;
      W temp = W(0);
      for (int e = 0; e < E; ++e) {
        const long long s = s0 + (long long)e * k + q;
        const int c = __ldg(U.col + s);
        if (c < 0) break;
        temp = sub(temp, mul(cvt<W>(__ldg(Uval + s)), xs[c - base]));
      }
      const W iv = cvt<W>(__ldg(inv + base + il));
      xs[il] = dilu ? add(xs[il], mul(temp, iv)) : mul(add(xs[il], temp), iv);
    }
    __syncthreads();
  }
  if (SMEM)
    for (int i = threadIdx.x; i < nRows; i += blockDim.x) y[base + i] = xs[i];
}

// One Gauss-Seidel sweep of every tile: rows in ascending tile-local order
// (as levels), each x_i = (seed - sum a_ij x_j) / d_i where x_j is this
// sweep's value for earlier rows of the tile and the sweep-start value for
// later rows and for other tiles' rows (the halo exchanged at the start of
// the sweep, gauss-seidel/Solver.cpp:61).
template <class MV, class W, bool SMEM>
__global__ void __launch_bounds__(256) gsSweepKernel(const int* __restrict__ tileStart, SchedView G,
                                                      const MV* __restrict__ Gval, const MV* __restrict__ diag,
                                                      const W* __restrict__ b, bool seedB,
                                                      const W* __restrict__ xin, bool xinZero,
                                                      W* __restrict__ xout, const KState* st, bool dropHalo) {
  extern __shared__ __align__(16) unsigned char smemRaw[];
  if (st && st->done) return;
  const int T = blockIdx.x;
  const int base = tileStart[T];
  const int nRows = tileStart[T + 1] - base;
  W* xold = SMEM ? reinterpret_cast<W*>(smemRaw) : nullptr;
  W* xnew = SMEM ? reinterpret_cast<W*>(smemRaw) + nRows : xout + base;
  if (SMEM) {
    for (int i = threadIdx.x; i < nRows; i += blockDim.x) xold[i] = xinZero ? W(0) : xin[base + i];
    __syncthreads();
  }
  for (int l = G.tileLvlStart[T]; l < G.tileLvlStart[T + 1]; ++l) {
    const int r0 = G.lvlRowStart[l], k = G.lvlRowStart[l + 1] - r0;
    const long long s0 = G.lvlSlotStart[l];
    const int E = static_cast<int>((G.lvlSlotStart[l + 1] - s0) / (k > 0 ? k : 1));
    for (int q = threadIdx.x; q < k; q += blockDim.x) {
      const int row = G.rows[r0 + q];
      const int il = row - base;
      const W d = cvt<W>(__ldg(diag + row));
      W sum = seedB ? b[row] : d;
      for (int e = 0; e < E; ++e) {
        const long long s = s0 + (long long)e * k + q;
        const int c = __ldg(G.col + s);
        if (c < 0) break;
        const int lc = c - base;
        W xv;
        if (lc >= 0 && lc < nRows) {
          if (lc < il) xv = xnew[lc];
          else xv = xinZero ? W(0) : (SMEM ? xold[lc] : xin[c]);
        } else {
          xv = xinZero || dropHalo ? W(0) : xin[c];
        }
        sum = sub(sum, mul(cvt<W>(__ldg(Gval + s)), xv));
      }
      xnew[il] = dvd(sum, d);
    }
    __syncthreads();
  }
  if (SMEM)
    for (int i = threadIdx.x; i < nRows; i += blockDim.x) xout[base + i] = xnew[i];
}

// Elementwise prologue (no fused preconditioner): writes p or s and
// optionally a copy (y = p or z = s without a preconditioner).
template <class W>
__global__ void prologueKernel(Pro<W> pro, W* copyTo, int n) {
  if (pro.st && pro.st->done) return;
  W beta = W(0), omega = W(0), alpha = W(0);
  bool first = true;
  if (pro.st) {
    beta = cvt<W>(pro.st->beta);
    omega = cvt<W>(pro.st->omega);
    alpha = cvt<W>(pro.st->alpha);
    first = pro.st->iter == 0;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    W v = pro(i, beta, omega, alpha, first);
    if (copyTo) copyTo[i] = v;
  }
}

}  // namespace dev

// ---------------------------------------------------------------------------
int maxDynamicSmem(const DeviceMatrix& A) {
  static std::atomic<int> cached[64] = {};
  const int d = A.device & 63;
  int v = cached[d].load();
  if (v == 0) {
    GR_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, A.device));
    cached[d].store(v);
  }
  return v;
}

namespace {

int maxSmem(const DeviceMatrix& A) { return maxDynamicSmem(A); }

template <class W>
dev::Pro<W> makePro(const PrologueArgs& p) {
  return dev::Pro<W>{static_cast<int>(p.kind), static_cast<const W*>(p.b), static_cast<const W*>(p.r),
                     static_cast<W*>(p.pOrS), static_cast<const W*>(p.v), p.st};
}

template <class K>
void setSmem(K kernel, size_t bytes) {
  ensureDynamicSmem(reinterpret_cast<const void*>(kernel), bytes);
}

int elemBlocks(const DeviceMatrix& A, i64 n) {
  return static_cast<int>(std::max<i64>(1, std::min<i64>(A.redBlocks, (n + 255) / 256)));
}

}  // namespace

void launchIluFactor(DeviceMatrix& A, void* F, void* D, const void* Aoff, bool dilu, cudaStream_t s) {
  A.ensureLocalCrs();
  LevelSchedule& L = A.schedule(SweepEntries::Lower);
  if (A.vt == DType::F32)
    dev::iluFactorKernel<float><<<A.P, 256, 0, s>>>(A.tileStart.as<int>(), dev::schedView(L), A.rowPtr.as<int>(),
                                                    A.colLocal.as<int>(), static_cast<float*>(F),
                                                    static_cast<float*>(D), static_cast<const float*>(Aoff), dilu);
  else
    dev::iluFactorKernel<double><<<A.P, 256, 0, s>>>(A.tileStart.as<int>(), dev::schedView(L), A.rowPtr.as<int>(),
                                                     A.colLocal.as<int>(), static_cast<double*>(F),
                                                     static_cast<double*>(D), static_cast<const double*>(Aoff), dilu);
  checkLaunch("ilu_factor");
}

void launchInvert(DeviceMatrix& A, const void* D, void* inv, cudaStream_t s) {
  const int blocks = elemBlocks(A, A.n);
  if (A.vt == DType::F32)
    dev::invertKernel<float><<<blocks, 256, 0, s>>>(static_cast<const float*>(D), static_cast<float*>(inv), A.n);
  else
    dev::invertKernel<double><<<blocks, 256, 0, s>>>(static_cast<const double*>(D), static_cast<double*>(inv), A.n);
  checkLaunch("invert");
}

void launchPack(DeviceMatrix& A, const LevelSchedule& S, const void* F, void* out, cudaStream_t s) {
  const int blocks = elemBlocks(A, S.slots);
  if (A.vt == DType::F32)
    dev::packKernel<float><<<blocks, 256, 0, s>>>(S.src.as<int>(), static_cast<const float*>(F),
                                                  static_cast<float*>(out), S.slots);
  else
    dev::packKernel<double><<<blocks, 256, 0, s>>>(S.src.as<int>(), static_cast<const double*>(F),
                                                   static_cast<double*>(out), S.slots);
  checkLaunch("pack");
}

namespace {

template <class MV, class W>
void iluApplyT(DeviceMatrix& A, const void* Lval, const void* Uval, const void* inv, bool dilu,
               const PrologueArgs& pro, void* y, cudaStream_t s) {
  LevelSchedule& L = A.schedule(SweepEntries::Lower);
  LevelSchedule& U = A.schedule(SweepEntries::UpperDesc);
  const size_t bytes = static_cast<size_t>(A.host->maxTileRows) * sizeof(W);
  auto args = [&](auto kernel, size_t smem) {
    kernel<<<A.P, 256, smem, s>>>(A.tileStart.as<int>(), dev::schedView(L), static_cast<const MV*>(Lval),
                                  dev::schedView(U), static_cast<const MV*>(Uval),
                                  static_cast<const MV*>(inv), dilu, makePro<W>(pro),
                                  static_cast<W*>(y));
  };
  if (bytes <= static_cast<size_t>(maxSmem(A))) {
    auto k = dev::iluApplyKernel<MV, W, true>;
    if (bytes > 48 * 1024) setSmem(k, bytes);
    args(k, bytes);
  } else {
    args(dev::iluApplyKernel<MV, W, false>, 0);
  }
  checkLaunch("ilu_apply");
}

template <class MV, class W>
void gsSweepT(DeviceMatrix& A, const void* Gval, const void* b, bool seedB, const void* xin, bool xinZero,
              void* xout, const KState* st, cudaStream_t s, bool dropHalo) {
  LevelSchedule& G = A.schedule(SweepEntries::All);
  const size_t bytes = 2 * static_cast<size_t>(A.host->maxTileRows) * sizeof(W);
  auto args = [&](auto kernel, size_t smem) {
    kernel<<<A.P, 256, smem, s>>>(A.tileStart.as<int>(), dev::schedView(G), static_cast<const MV*>(Gval),
                                  A.diag.as<MV>(),
                                  static_cast<const W*>(b), seedB, static_cast<const W*>(xin), xinZero,
                                  static_cast<W*>(xout), st, dropHalo);
  };
  if (bytes <= static_cast<size_t>(maxSmem(A))) {
    auto k = dev::gsSweepKernel<MV, W, true>;
    if (bytes > 48 * 1024) setSmem(k, bytes);
    args(k, bytes);
  } else {
    args(dev::gsSweepKernel<MV, W, false>, 0);
  }
  checkLaunch("gs_sweep");
}

}  // namespace

void launchIluApply(DeviceMatrix& A, const void* Lval, const void* Uval, const void* inv, bool dilu,
                    const PrologueArgs& pro, void* y, DType W, cudaStream_t s) {
  if (A.vt == DType::F32 && W == DType::F32) iluApplyT<float, float>(A, Lval, Uval, inv, dilu, pro, y, s);
  else if (A.vt == DType::F32 && W == DType::F64) iluApplyT<float, double>(A, Lval, Uval, inv, dilu, pro, y, s);
  else if (A.vt == DType::F64 && W == DType::F64) iluApplyT<double, double>(A, Lval, Uval, inv, dilu, pro, y, s);
  else fail(GR_EUNSUPPORTED, "ILU with float64 coefficients needs float64 vectors");
}

void launchGsSweep(DeviceMatrix& A, const void* Gval, const void* b, bool seedB, const void* xin, bool xinZero,
                   void* xout, DType W, const KState* st, cudaStream_t s, bool dropHalo) {
  if (A.vt == DType::F32 && W == DType::F32)
    gsSweepT<float, float>(A, Gval, b, seedB, xin, xinZero, xout, st, s, dropHalo);
  else if (A.vt == DType::F32 && W == DType::F64)
    gsSweepT<float, double>(A, Gval, b, seedB, xin, xinZero, xout, st, s, dropHalo);
  else if (A.vt == DType::F64 && W == DType::F64)
    gsSweepT<double, double>(A, Gval, b, seedB, xin, xinZero, xout, st, s, dropHalo);
  else fail(GR_EUNSUPPORTED, "Gauss-Seidel with float64 coefficients needs float64 vectors");
}

void launchPrologue(DeviceMatrix& A, const PrologueArgs& pro, void* copyTo, DType W, cudaStream_t s) {
  const int blocks = elemBlocks(A, A.n);
  if (W == DType::F32)
    dev::prologueKernel<float><<<blocks, 256, 0, s>>>(makePro<float>(pro), static_cast<float*>(copyTo), A.n);
  else
    dev::prologueKernel<double><<<blocks, 256, 0, s>>>(makePro<double>(pro), static_cast<double*>(copyTo), A.n);
  checkLaunch("prologue");
}

}  // namespace gr
