// Self-test of the bounded mbarrier wait that every pipelined kernel uses
// (mbarWaitBounded, bulk.cuh). A single-thread kernel initialises an
// mbarrier that nothing ever arrives on and waits for its first phase: the
// wait must give up after its time limit and report GR_ETIMEOUT, leaving the
// context usable. This is how the kernels' waits are tested without making a
// GPU fault or hang.
#include "bulk.cuh"
#include "device.hpp"
#include "sell.cuh"

namespace gr {
namespace dev {

__global__ void waitTimeoutKernel(int* status, unsigned long long* elapsedNs) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = smemAddr(&bar);
  mbarInit(b, 1);
  fenceBarrierInit();
  const uint64_t t0 = globalTimerNs();
  const bool landed = mbarWaitBounded(b, 0);  // no arrival: runs out
  *elapsedNs = globalTimerNs() - t0;
  *status = landed ? GR_OK : GR_ETIMEOUT;
}

}  // namespace dev
}  // namespace gr

namespace gr {

void selftestWaitTimeout(int32_t* status, int64_t* elapsedNs) {
  DBuf out(16);
  int* st = out.as<int>();
  unsigned long long* ns = reinterpret_cast<unsigned long long*>(static_cast<char*>(out.get()) + 8);
  dev::waitTimeoutKernel<<<1, 1>>>(st, ns);
  checkLaunch("selftest_wait_timeout");
  int hs = 0;
  unsigned long long hns = 0;
  GR_CUDA(cudaMemcpy(&hs, st, sizeof(int), cudaMemcpyDeviceToHost));
  GR_CUDA(cudaMemcpy(&hns, ns, sizeof(hns), cudaMemcpyDeviceToHost));
  *status = hs;
  *elapsedNs = static_cast<int64_t>(hns);
}

}  // namespace gr
