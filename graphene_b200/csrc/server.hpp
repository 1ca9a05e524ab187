// Solve server: continuous batching of independent solves on one GPU.
//
// Requests (a host matrix, a solver configuration, a right-hand side) are
// queued on arrival and admitted, in arrival order, as soon as a worker slot
// is free and their estimated device footprint fits the HBM budget. Each slot
// is a host thread driving its own non-blocking CUDA stream, so the kernels
// of admitted requests overlap on the device while new requests keep being
// admitted as others finish. A (matrix, configuration) pair stays resident
// after its request - coefficients, tile layout, ILU factors, Krylov buffers
// and captured iteration graphs - so a later request for the same pair skips
// upload and factorisation; idle resident pairs are evicted oldest first
// when a new pair needs their memory. Kernels are deterministic, so a
// request's result does not depend on what else is running.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.hpp"
#include "host_matrix.hpp"

namespace gr {

struct DeviceMatrix;
class SolverTree;

// Upper estimate of the device memory a (matrix, configuration) pair holds
// while resident: coefficients in the SpMV layout, tile-local CRS, ILU
// factors and byte stream, solver vectors and the staging buffers of a
// host-buffer solve.
i64 estimateFootprint(const HostMatrix& H, const std::string& json, DType t);

class Server {
 public:
  Server(int slots, int device, i64 budgetBytes);
  ~Server();
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  u64 submit(std::shared_ptr<HostMatrix> H, const std::string& json, const void* b, DType t);
  // A request for the matrix with `like`'s structure and new values (global
  // CRS order: off-diagonals gVal, diagonal gDiag), copied.
  u64 submitValues(std::shared_ptr<HostMatrix> like, const double* gVal, const double* gDiag, const std::string& json,
                   const void* b, DType t);
  // GR_OK when the request finished (its own status in *status); GR_ETIMEOUT
  // when it did not finish within timeoutMs (< 0: wait forever).
  int wait(u64 id, double timeoutMs, void* x, gr_stats* stats, gr_request_times* times, int* status,
           std::string* err);
  void counters(i64* queued, i64* running, i64* completed, i64* bytesInUse, i64* resident);
  // Removes request id from the queue if it has not been admitted (true);
  // its wait then reports GR_ECANCELED. False when it is running or done.
  bool cancel(u64 id);

 private:
  struct Entry;
  struct Request;
  void worker(int slot);
  u64 enqueue(std::shared_ptr<HostMatrix> H, const std::string& json, const void* b, DType t, const double* gVal,
              const double* gDiag);
  double now() const;
  bool admissible(const Request& r, bool* needEvict);
  std::shared_ptr<Entry> findEntry(const Request& r);

  int device_ = 0;
  i64 budget_ = 0;
  std::chrono::steady_clock::time_point t0_;
  std::mutex mu_;
  std::condition_variable cvWork_, cvDone_;
  std::deque<std::shared_ptr<Request>> queue_;
  std::unordered_map<u64, std::shared_ptr<Request>> requests_;
  std::vector<std::shared_ptr<Entry>> resident_;
  i64 inUse_ = 0, running_ = 0, completed_ = 0;
  u64 nextId_ = 1, useClock_ = 0;
  bool stopping_ = false;
  std::vector<void*> streams_;
  std::vector<std::thread> threads_;
};

}  // namespace gr
