// Solve server (server.hpp): admission, worker slots, resident pairs.
#include "server.hpp"

#include <cstring>

#include "config.hpp"
#include "device.hpp"
#include "solvers.hpp"

namespace gr {

i64 estimateFootprint(const HostMatrix& H, const std::string& json, DType t) {
  (void)json;
  const i64 n = H.n, m = H.m;
  const i64 vs = static_cast<i64>(dtypeSize(H.valueType));
  // SpMV layout: chunks of 32 rows padded to their longest row.
  i64 slots = 0;
  for (i64 c = 0; c * 32 < n; ++c) {
    i64 mx = 0;
    for (i64 r = c * 32; r < std::min<i64>(n, c * 32 + 32); ++r) mx = std::max(mx, H.rowPtr[r + 1] - H.rowPtr[r]);
    slots += 32 * mx;
  }
  const i64 sell = slots * (4 + vs) + 4 * (n / 32 + 2);
  const i64 rows = n * (vs + 8) + 4 * (H.P + 1);                 // diagonal, tile starts, permutation
  const i64 localCrs = 4 * (n + 1) + m * (4 + vs);
  const i64 stream = 2 * (m * (4 + vs) + n * (8 + 2 * vs) + 64 * (i64(H.P) + 1));  // template + packed copy
  const i64 factors = m * vs + n * vs;
  const i64 vectors = 16 * n * std::max<i64>(8, static_cast<i64>(dtypeSize(t)));     // Krylov, MPIR, staging
  return sell + rows + localCrs + stream + factors + vectors + (i64(4) << 20);
}

struct Server::Entry {
  std::shared_ptr<HostMatrix> H;
  const HostMatrix* hid = nullptr;  // the matrix whose values are on the device (changed under mu_)
  u64 key = 0;                      // structure key (CRS matrices)
  bool crs = false;
  std::string json;
  i64 footprint = 0;
  bool busy = false, ready = false;
  u64 lastUse = 0;
  std::unique_ptr<DeviceMatrix> D;
  std::unique_ptr<SolverTree> tree;
};

struct Server::Request {
  u64 id = 0;
  std::shared_ptr<HostMatrix> H;
  std::string json;
  DType t = DType::F32;
  std::vector<unsigned char> b, x;
  i64 footprint = 0;
  double tArrive = 0, tAdmit = 0, tSolve = 0, tFinish = 0;
  gr_stats st{};
  int status = GR_OK, slot = -1;
  bool cacheHit = false, done = false, valuesUpdated = false;
  // Values-only requests: H is the structure's template, these its values.
  bool valuesOnly = false;
  // The values rounded to the coefficient type once, at submission (what a
  // resident pair uploads).
  std::vector<unsigned char> gValT, gDiagT;
  std::string err;
  std::shared_ptr<Entry> entry;
};

Server::Server(int slots, int device, i64 budgetBytes) : t0_(std::chrono::steady_clock::now()) {
  if (slots < 0 || slots > 64) fail(GR_EINVAL, "slots must be 0..64");
  if (slots == 0) slots = 4;
  if (budgetBytes < 0) fail(GR_EINVAL, "hbm_budget_bytes must not be negative");
  if (device < 0) {
    GR_CUDA(cudaGetDevice(&device_));
  } else {
    device_ = device;
  }
  GR_CUDA(cudaSetDevice(device_));
  if (budgetBytes == 0) {
    size_t freeB = 0, totalB = 0;
    GR_CUDA(cudaMemGetInfo(&freeB, &totalB));
    budgetBytes = static_cast<i64>(0.8 * static_cast<double>(freeB));
  }
  budget_ = budgetBytes;
  for (int i = 0; i < slots; ++i) {
    cudaStream_t s;
    GR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    streams_.push_back(s);
  }
  for (int i = 0; i < slots; ++i) threads_.emplace_back([this, i] { worker(i); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stopping_ = true;
    for (auto& r : queue_) {
      r->status = GR_EINVAL;
      r->err = "server destroyed before the request was admitted";
      r->done = true;
    }
    queue_.clear();
  }
  cvWork_.notify_all();
  for (auto& t : threads_) t.join();
  cudaSetDevice(device_);
  resident_.clear();  // solver trees synchronise their streams before releasing memory
  for (void* s : streams_) cudaStreamDestroy(static_cast<cudaStream_t>(s));
  cvDone_.notify_all();
}

double Server::now() const {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
}

u64 Server::submitValues(std::shared_ptr<HostMatrix> like, const double* gVal, const double* gDiag,
                         const std::string& json, const void* b, DType t) {
  if (!like) fail(GR_EINVAL, "host matrix must not be NULL");
  if (like->format != GR_FORMAT_CRS || !like->sumRank.empty())
    fail(GR_EUNSUPPORTED, "values-only requests are for CRS matrices");
  return enqueue(std::move(like), json, b, t, gVal, gDiag);
}

u64 Server::submit(std::shared_ptr<HostMatrix> H, const std::string& json, const void* b, DType t) {
  return enqueue(std::move(H), json, b, t, nullptr, nullptr);
}

u64 Server::enqueue(std::shared_ptr<HostMatrix> H, const std::string& json, const void* b, DType t,
                    const double* gVal, const double* gDiag) {
  if (!H) fail(GR_EINVAL, "host matrix must not be NULL");
  if (!b) fail(GR_EINVAL, "b must not be NULL");
  if (t != DType::F32 && t != DType::F64) fail(GR_EINVAL, "b must be float32 or float64");
  SolverConfig::fromText(json);  // reject a malformed configuration at submission
  auto r = std::make_shared<Request>();
  r->H = std::move(H);
  r->json = json;
  r->t = t;
  const size_t bytes = static_cast<size_t>(r->H->n) * dtypeSize(t);
  r->b.resize(bytes);
  std::memcpy(r->b.data(), b, bytes);
  r->x.assign(bytes, 0);
  if (gVal) {
    r->valuesOnly = true;
    const i64 m = r->H->m, n = r->H->n;
    if (r->H->valueType == DType::F32) {
      // Rounded to float here, in the submitting thread.
      r->gValT.resize(m * sizeof(float));
      r->gDiagT.resize(n * sizeof(float));
      float* fv = reinterpret_cast<float*>(r->gValT.data());
      float* fd = reinterpret_cast<float*>(r->gDiagT.data());
      for (i64 k = 0; k < m; ++k) fv[k] = static_cast<float>(gVal[k]);
      for (i64 k = 0; k < n; ++k) fd[k] = static_cast<float>(gDiag[k]);
    } else {
      r->gValT.resize(m * sizeof(double));
      r->gDiagT.resize(n * sizeof(double));
      std::memcpy(r->gValT.data(), gVal, m * sizeof(double));
      std::memcpy(r->gDiagT.data(), gDiag, n * sizeof(double));
    }
  }
  r->footprint = estimateFootprint(*r->H, json, t);
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (stopping_) fail(GR_EINVAL, "server is shutting down");
    r->id = nextId_++;
    r->tArrive = now();
    requests_[r->id] = r;
    queue_.push_back(r);
  }
  cvWork_.notify_one();
  return r->id;
}

// The resident pair of a request: the same matrix, or (CRS matrices) the
// same structure, whose values the worker then replaces.
std::shared_ptr<Server::Entry> Server::findEntry(const Request& r) {
  const bool crs = r.H->format == GR_FORMAT_CRS && r.H->sumRank.empty();
  for (auto& e : resident_) {
    if (e->json != r.json) continue;
    if ((e->hid == r.H.get() && !r.valuesOnly) || (crs && e->crs && e->key == r.H->structureKey)) return e;
  }
  return nullptr;
}

// Called with mu_ held. A request is admissible when its pair is resident
// and idle, or when its footprint fits next to the resident pairs (possibly
// after evicting idle ones, *needEvict).
bool Server::admissible(const Request& r, bool* needEvict) {
  *needEvict = false;
  if (auto e = findEntry(r)) return !e->busy;
  if (inUse_ + r.footprint <= budget_) return true;
  i64 idle = 0;
  for (auto& e : resident_)
    if (!e->busy) idle += e->footprint;
  if (inUse_ - idle + r.footprint <= budget_ || running_ == 0) {
    *needEvict = true;
    return true;
  }
  return false;
}

void Server::worker(int slot) {
  cudaSetDevice(device_);
  cudaStream_t stream = static_cast<cudaStream_t>(streams_[slot]);
  for (;;) {
    std::shared_ptr<Request> r;
    std::vector<std::shared_ptr<Entry>> evicted;
    {
      std::unique_lock<std::mutex> lk(mu_);
      for (;;) {
        if (stopping_) return;
        // Arrival order; a later request may pass the head only when its
        // pair is already resident and idle (it needs no new memory).
        bool found = false;
        for (auto it = queue_.begin(); it != queue_.end(); ++it) {
          bool evict = false;
          const bool head = it == queue_.begin();
          if (!head) {
            auto e = findEntry(**it);
            if (!e || e->busy) continue;
          }
          if (!admissible(**it, &evict)) continue;
          r = *it;
          queue_.erase(it);
          if (auto hit = findEntry(*r)) {
            r->entry = hit;
            r->cacheHit = true;
          } else {
            if (evict) {
              // Oldest idle pairs first until the request fits.
              std::vector<std::shared_ptr<Entry>> idle;
              for (auto& e2 : resident_)
                if (!e2->busy) idle.push_back(e2);
              std::sort(idle.begin(), idle.end(), [](auto& a, auto& b) { return a->lastUse < b->lastUse; });
              for (auto& e2 : idle) {
                if (inUse_ + r->footprint <= budget_) break;
                inUse_ -= e2->footprint;
                resident_.erase(std::find(resident_.begin(), resident_.end(), e2));
                evicted.push_back(e2);
              }
            }
            auto e = std::make_shared<Entry>();
            e->H = r->H;
            e->hid = r->H.get();
            e->key = r->H->structureKey;
            e->crs = r->H->format == GR_FORMAT_CRS && r->H->sumRank.empty();
            e->json = r->json;
            e->footprint = r->footprint;
            resident_.push_back(e);
            inUse_ += e->footprint;
            r->entry = e;
          }
          r->entry->busy = true;
          r->entry->lastUse = ++useClock_;
          r->tAdmit = now();
          r->slot = slot;
          ++running_;
          found = true;
          break;
        }
        if (found) break;
        cvWork_.wait(lk);
      }
    }
    evicted.clear();  // outside the lock: synchronises and frees their memory
    Entry& e = *r->entry;
    try {
      if (!e.ready && r->valuesOnly) {
        // A new pair for a values-only request: the template's layout with
        // the request's values.
        // The values as submitted were rounded to the coefficient type;
        // widened back they round to themselves.
        const i64 m = r->H->m, n = r->H->n;
        std::vector<double> gv(m), gd(n);
        if (r->H->valueType == DType::F32) {
          const float* fv = reinterpret_cast<const float*>(r->gValT.data());
          const float* fd = reinterpret_cast<const float*>(r->gDiagT.data());
          for (i64 k = 0; k < m; ++k) gv[k] = fv[k];
          for (i64 k = 0; k < n; ++k) gd[k] = fd[k];
        } else {
          std::memcpy(gv.data(), r->gValT.data(), m * sizeof(double));
          std::memcpy(gd.data(), r->gDiagT.data(), n * sizeof(double));
        }
        auto M = HostMatrix::withGlobalValues(*r->H, gv.data(), gd.data());
        e.H = M;
        std::lock_guard<std::mutex> lk(mu_);
        e.hid = M.get();
      }
      if (!e.ready) {
        e.D = std::make_unique<DeviceMatrix>(e.H);
        e.D->stream = stream;
        e.tree = SolverTree::create(*e.D, e.json);
        e.ready = true;
      }
      e.D->stream = stream;
      if (r->valuesOnly && r->cacheHit) {
        // Values-only request on a resident structure: the global values
        // are gathered into place on the device.
        e.D->updateGlobalValues(r->gValT.data(), r->gDiagT.data(), r->H->valueType);
        e.tree->refresh();
        std::lock_guard<std::mutex> lk(mu_);
        e.hid = nullptr;  // no host matrix holds these values
        r->valuesUpdated = true;
      } else if (!r->valuesOnly && e.hid != r->H.get()) {
        // Same structure, new values: upload them into the resident device
        // matrix and refactorise in place (no host layout work, no new
        // buffers, the captured iteration graphs stay valid).
        e.D->updateValues(r->H);
        e.tree->refresh();
        e.H = r->H;
        std::lock_guard<std::mutex> lk(mu_);
        e.hid = r->H.get();
        r->cacheHit = true;
        r->valuesUpdated = true;
      }
      r->tSolve = now();
      r->st = e.tree->solveHost(r->x.data(), r->t, r->b.data(), r->t);
    } catch (const Error& ex) {
      r->status = ex.code;
      r->err = ex.what();
    } catch (const std::bad_alloc&) {
      r->status = GR_ENOMEM;
      r->err = "host allocation failed";
    } catch (const std::exception& ex) {
      r->status = GR_EINVAL;
      r->err = ex.what();
    }
    cudaStreamSynchronize(stream);
    std::shared_ptr<Entry> drop;
    {
      std::lock_guard<std::mutex> lk(mu_);
      e.busy = false;
      if (!e.ready) {  // failed set-up: do not keep the pair
        inUse_ -= e.footprint;
        resident_.erase(std::find(resident_.begin(), resident_.end(), r->entry));
        drop = r->entry;
      }
      r->entry.reset();
      --running_;
      ++completed_;
      r->tFinish = now();
      r->done = true;
    }
    drop.reset();
    cvDone_.notify_all();
    cvWork_.notify_all();
  }
}

int Server::wait(u64 id, double timeoutMs, void* x, gr_stats* stats, gr_request_times* times, int* status,
                 std::string* err) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) fail(GR_EINVAL, "unknown request id " + std::to_string(id));
  std::shared_ptr<Request> r = it->second;
  auto pred = [&] { return r->done; };
  if (timeoutMs < 0) {
    cvDone_.wait(lk, pred);
  } else if (!cvDone_.wait_for(lk, std::chrono::duration<double, std::milli>(timeoutMs), pred)) {
    return GR_ETIMEOUT;
  }
  requests_.erase(id);
  if (x) std::memcpy(x, r->x.data(), r->x.size());
  if (stats) *stats = r->st;
  if (times) {
    times->arrival_ms = r->tArrive;
    times->admitted_ms = r->tAdmit;
    times->finished_ms = r->tFinish;
    times->footprint_bytes = r->footprint;
    times->cache_hit = r->valuesUpdated ? 2 : (r->cacheHit ? 1 : 0);
    times->slot = r->slot;
    times->solve_start_ms = r->tSolve;
  }
  *status = r->status;
  *err = r->err;
  return GR_OK;
}

bool Server::cancel(u64 id) {
  {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end()) fail(GR_EINVAL, "unknown request id " + std::to_string(id));
    std::shared_ptr<Request> r = it->second;
    auto q = std::find(queue_.begin(), queue_.end(), r);
    if (q == queue_.end()) return false;  // admitted (running or finished)
    queue_.erase(q);
    r->status = GR_ECANCELED;
    r->err = "request cancelled before it was admitted";
    r->tFinish = now();
    r->done = true;
  }
  cvDone_.notify_all();
  cvWork_.notify_all();  // the head may have changed
  return true;
}

void Server::counters(i64* queued, i64* running, i64* completed, i64* bytesInUse, i64* resident) {
  std::lock_guard<std::mutex> lk(mu_);
  if (queued) *queued = static_cast<i64>(queue_.size());
  if (running) *running = running_;
  if (completed) *completed = completed_;
  if (bytesInUse) *bytesInUse = inUse_;
  if (resident) *resident = static_cast<i64>(resident_.size());
}

}  // namespace gr
