// Norms of device vectors without any device allocation.
//
// The matrix-bound norm (gr_vector_norm) reduces through per-block partials
// that a gr_matrix allocates when it is created. This variant takes a raw
// device vector and reduces through a file-scope __device__ scratch array
// instead, so a call makes no cudaMalloc / cudaFree and no call into an
// allocating library. It exists for callers that must not allocate device
// memory at the point of the call: a serving loop that has admitted its
// work against a fixed HBM footprint (an allocation there can fail or push
// the footprint past what admission granted), and code running inside a
// caching allocator's own callbacks (out-of-memory observers, statistics
// hooks), where a cudaMalloc would re-enter the allocator.
//
// Limits: at most kNaMaxVectors vectors per call, each of at most 2^31 - 1
// elements; larger requests are rejected with GR_EINVAL. The scratch holds
// kNaMaxVectors x kNaBlocks doubles of block partials and one arrival counter
// per vector (75,808 bytes per device).
//
// The counters must be zero when a launch starts: the set-up clears them,
// and the last block of each reduction resets its counter. Overlapping calls
// on one device (two streams, two host threads, or a call concurrent with
// another call still running on the GPU) share the scratch and race; the
// caller serialises them. The first call on each device performs the set-up
// (symbol lookup, which may load the module, and the counter clear); make it
// before any stream capture. Every call looks the symbol up again and
// repeats the set-up if its address changed (the device was reset and the
// module reloaded), so a reset needs no restart of the process.
//
// Every vector read (x .. x + ((count - 1) * ld + n) elements) and the count
// results written must lie inside one device allocation each, as the driver
// reports it; otherwise the call returns GR_EINVAL before anything runs.
#include <algorithm>
#include <climits>
#include <mutex>
#include <string>

#include "device.hpp"
#include "devmath.cuh"
#include "sell.cuh"

namespace gr {
namespace dev {

constexpr int kNaMaxVectors = 8;
constexpr int kNaBlocks = 148 * 8;  // 8 blocks of 256 threads per SM of a B200

struct NoAllocScratch {
  double partials[kNaMaxVectors * kNaBlocks];
  unsigned counter[kNaMaxVectors];
};

static __device__ __align__(256) NoAllocScratch g_naScratch;

// Block y reduces vector y (x + y * ld) exactly as normKernel reduces one
// vector: grid-stride partials, block reduction, and the last block's
// combination of the block partials in the same deterministic order as
// normKernel's gridReduce.
template <class T>
__global__ void __launch_bounds__(256) normsNoAllocKernel(const T* __restrict__ x, int n, long long ld,
                                                           int kind, double* __restrict__ out,
                                                           NoAllocScratch* scratch) {
  __shared__ double smem[32];
  const T* xv = x + static_cast<long long>(blockIdx.y) * ld;
  double part = redIdentity(normOp(kind));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    part = normStep(part, toDouble(__ldg(xv + i)), kind);
  double v[1] = {part};
  const int ops[1] = {normOp(kind)};
  double res[1];
  blockReduce<1>(v, ops, smem);
  if (gridReduce<1>(v, ops, scratch->partials + blockIdx.y * kNaBlocks, scratch->counter + blockIdx.y,
                    smem, res) &&
      threadIdx.x == 0)
    out[blockIdx.y] = normFinish(res[0], kind);
}

}  // namespace dev

namespace {

constexpr int kNaMaxDevices = 64;

struct NaDevice {
  dev::NoAllocScratch* scratch = nullptr;  // the address the set-up was done for
  int blocks = 0;  // reduction blocks: min(8 per SM, kNaBlocks)
};

NaDevice g_naDevices[kNaMaxDevices];
std::mutex g_naMutex;

// Per-device set-up on first use: the scratch's device address and the
// counters cleared. No allocation.
const NaDevice& naDevice() {
  int d = 0;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) fail(GR_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (d < 0 || d >= kNaMaxDevices) fail(GR_EUNSUPPORTED, "device index beyond the no-allocation table");
  std::lock_guard<std::mutex> lock(g_naMutex);
  NaDevice& nd = g_naDevices[d];
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, dev::g_naScratch);
  if (e != cudaSuccess) fail(GR_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  if (nd.scratch == p) return nd;
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
  if (e != cudaSuccess) fail(GR_ECUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
  auto* s = static_cast<dev::NoAllocScratch*>(p);
  e = cudaMemset(s->counter, 0, sizeof(s->counter));
  if (e != cudaSuccess) fail(GR_ECUDA, std::string("clearing the scratch counters: ") + cudaGetErrorString(e));
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) fail(GR_ECUDA, std::string("scratch set-up: ") + cudaGetErrorString(e));
  nd.blocks = std::max(1, std::min(dev::kNaBlocks, sms * 8));
  nd.scratch = s;
  return nd;
}

// Rejects pointers the GPU cannot dereference (plain host memory) and
// misaligned ones before anything is launched.
void needDevicePointer(const void* p, size_t align, const char* what) {
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(GR_EINVAL, std::string(what) + " is not a pointer the CUDA runtime knows");
  }
  if (a.type == cudaMemoryTypeUnregistered || a.devicePointer == nullptr)
    fail(GR_EINVAL, std::string(what) + " is not device-accessible memory");
  if (reinterpret_cast<uintptr_t>(p) % align != 0) fail(GR_EINVAL, std::string(what) + " is misaligned");
}

// The driver's allocation range query, found through the runtime (no link
// against the driver library): CUresult cuMemGetAddressRange(CUdeviceptr*
// base, size_t* size, CUdeviceptr ptr).
using MemRangeFn = int (*)(unsigned long long*, size_t*, unsigned long long);
MemRangeFn memRangeFn() {
  static MemRangeFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return static_cast<MemRangeFn>(nullptr);
    }
    return reinterpret_cast<MemRangeFn>(f);
  }();
  return fn;
}

// [p, p + bytes) must lie inside the device allocation that holds p.
void needRange(const void* p, size_t bytes, const char* what) {
  MemRangeFn fn = memRangeFn();
  if (!fn) fail(GR_EUNSUPPORTED, "the driver's allocation range query is unavailable");
  unsigned long long base = 0;
  size_t size = 0;
  const unsigned long long a = reinterpret_cast<unsigned long long>(p);
  if (fn(&base, &size, a) != 0)
    fail(GR_EINVAL, std::string(what) + " is not inside a device allocation the driver reports");
  if (a < base || bytes > size || a - base > size - bytes)
    fail(GR_EINVAL, std::string(what) + " extends past the end of its device allocation");
}

}  // namespace

void launchNormsNoAlloc(const void* x, i64 n, i64 count, i64 ld, DType t, int normKind, double* out,
                        cudaStream_t s) {
  if (count < 1 || count > dev::kNaMaxVectors)
    fail(GR_EINVAL, "count must be 1.." + std::to_string(dev::kNaMaxVectors) +
                        " (vectors per call that the static scratch holds)");
  if (n < 0 || n > INT_MAX) fail(GR_EINVAL, "n must be 0..2^31-1");
  if (count > 1 && ld < n) fail(GR_EINVAL, "ld must be at least n");
  if (t == DType::DW) fail(GR_EUNSUPPORTED, "norm of a twofloat32 vector");
  needDevicePointer(x, dtypeSize(t), "x");
  needDevicePointer(out, sizeof(double), "out");
  needRange(x, static_cast<size_t>((count - 1) * ld + n) * dtypeSize(t), "x (count vectors of n at stride ld)");
  needRange(out, static_cast<size_t>(count) * sizeof(double), "out (count results)");
  const NaDevice& nd = naDevice();
  const int blocks = std::max(1, std::min(nd.blocks, static_cast<int>((n + 255) / 256)));
  const dim3 grid(blocks, static_cast<unsigned>(count));
  if (t == DType::F32)
    dev::normsNoAllocKernel<float><<<grid, 256, 0, s>>>(static_cast<const float*>(x), static_cast<int>(n), ld,
                                                        normKind, out, nd.scratch);
  else
    dev::normsNoAllocKernel<double><<<grid, 256, 0, s>>>(static_cast<const double*>(x), static_cast<int>(n),
                                                         ld, normKind, out, nd.scratch);
  checkLaunch("normsNoAlloc");
}

}  // namespace gr
