// Serving loop: continuous batching of Walk-on-Spheres evaluation requests on
// one GPU.
//
// Requests (a mesh, a boundary problem, host points, a target standard error)
// are submitted from any host thread.  A worker thread owns the GPU side:
//
//  * Admission by device memory.  One device pool is allocated when the server
//    starts; a request is admitted when its points and per-point accumulators
//    fit in the pool (first fit) and the in-flight limit allows it, so the
//    request path never calls cudaMalloc.  Requests larger than the whole
//    pool are refused at submission.
//  * Ticks.  Each tick is ONE persistent walker launch over every in-flight
//    request (the batched walker of batch.cu): a walk budget is handed out
//    shortest-remaining-work first (every request still advances by at least
//    one point per tick), each request contributes its next range of points with
//    its current sweep's walks per point, and requests admitted during a tick
//    join the next one.  Small requests therefore overlap with large ones
//    instead of queueing behind them.
//  * Adaptive sweeps.  A sweep gives every point of a request the same number
//    of walks; after each sweep the maximum (or root mean square, per request)
//    of the per-point standard errors is reduced on the device and the next
//    sweep is sized from it
//    (N_needed = N_done * (stderr / target)^2, plus 10 %), until the target or
//    the walk cap is met.
//  * Determinism.  Walk w of point p in sweep s of a request is keyed by
//    (request seed, s; p * walks_per_point + w), whatever range or tick ran it,
//    and sweep sizes depend only on the request's own statistics, so a
//    request's estimates are the same alone and in any mix, up to the order of
//    FP64 additions.
//  * NC+2LMC requests.  A request in N2W_REQUEST_MODE_NC2LMC uses the cache
//    registered for its (mesh, problem) with n2w_server_set_nc.  Its sweeps
//    run as chunks of up to kNcChunk points (about one tick's walks) through n2w_nc2lmc_estimate_ex
//    on the request's own BVH (coarse walks truncated at depth m and closed by
//    the cache, plus residual walks) on a second stream: each worker
//    iteration enqueues the plain tick and the NC+2LMC chunks before waiting
//    for either, so their kernels share the device; the NC+2LMC walks per
//    iteration adapt so that the chunks end about when the tick does.  Each chunk is keyed by
//    (request seed, sweep, first point of the chunk), so these requests are also the same
//    alone and in a mix.  The chunk's statistics land in a scratch
//    area and are added to the request's totals; convergence uses the
//    estimator's standard error sqrt(var_c / N_c + var_r / N_r).
//
// The reference has no serving loop (it evaluates one point set per process);
// the walk itself is the reference's (src/cuda/cubql_bvh.cu:1323-1357).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.hpp"
#include "philox.cuh"
#include "problem.cuh"
#include "scene.hpp"
#include "walker.cuh"

namespace n2w {
namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Variance of the mean of c samples with sum s and sum of squares q (infinite
// below two samples).
__host__ __device__ inline double mean_variance(double s, double q, double c) {
  if (c < 2.0) return INFINITY;
  const double mean = s / c;
  return fmax(0.0, (q - c * mean * mean) / (c - 1.0)) / c;
}

// Per-point sample sums of one estimator level.
struct LevelSums {
  double* sum = nullptr;
  double* sum_sq = nullptr;
  uint32_t* count = nullptr;
};

// Max over points of the standard error (float bits; values >= 0 order like
// their bit patterns) and the sum of the estimator variances, one atomic each
// per warp.  The variance is var / n of level a, plus that of level b when
// b.sum is set (NC+2LMC: coarse + residual).
__global__ void stderr_kernel(LevelSums a, LevelSums b, int64_t n, unsigned* __restrict__ max_out,
                              double* __restrict__ sum_out) {
  float m = 0.0f;
  double v2 = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double ev = mean_variance(a.sum[i], a.sum_sq[i], a.count[i]);
    if (b.sum) ev += mean_variance(b.sum[i], b.sum_sq[i], b.count[i]);
    m = fmaxf(m, static_cast<float>(sqrt(ev)));
    v2 += ev;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    v2 += __shfl_xor_sync(0xffffffffu, v2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(max_out, __float_as_uint(m));
    atomicAdd(sum_out, v2);
  }
}

// First-fit allocator over offsets of one device pool (256-byte granules).
class PoolAllocator {
 public:
  explicit PoolAllocator(size_t bytes) : capacity_(bytes) { free_[0] = bytes; }
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) & ~size_t{255};
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes, start = it->first + bytes;
        free_.erase(it);
        if (rest) free_[start] = rest;
        used_ += bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 255) & ~size_t{255};
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t capacity() const { return capacity_; }
  size_t used() const { return used_; }

 private:
  size_t capacity_;
  size_t used_ = 0;
  std::map<size_t, size_t> free_;
};

// Device bytes a request of n points holds while in flight: points (12 B) and
// accumulators (sum, sum_sq, steps: 8 B; count, forced: 4 B); NC+2LMC adds
// the residual level's sum, sum_sq (8 B) and count (4 B).
size_t request_bytes(int64_t n, bool nc) {
  return static_cast<size_t>(n) * (nc ? 64 : 44) + (nc ? 8 : 5) * 256;
}

// Points per NC+2LMC chunk (the unit of work and of walk keying).  Small
// enough that one chunk (1,024 points x a few thousand walks) stays within
// a few tens of milliseconds, so NC work interleaves with the plain ticks.
constexpr int64_t kNcChunk = 1024;   // most points in one NC+2LMC chunk
constexpr int64_t kNcMinChunk = 32;  // fewest (a chunk may then exceed a tick's walks)

uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Adds one chunk's coarse and residual statistics (scratch, chunk-relative)
// into a request's totals at point offset `first`.
struct NcChunkAdd {
  const double *c_sum, *c_sum_sq, *r_sum, *r_sum_sq;
  const uint32_t *c_count, *c_forced, *r_count;
  const uint64_t* c_steps;
  double *t_c_sum, *t_c_sum_sq, *t_r_sum, *t_r_sum_sq;
  uint32_t *t_c_count, *t_c_forced, *t_r_count;
  uint64_t* t_c_steps;
};

__global__ void add_nc_chunk_kernel(NcChunkAdd a, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  a.t_c_sum[i] += a.c_sum[i];
  a.t_c_sum_sq[i] += a.c_sum_sq[i];
  a.t_c_count[i] += a.c_count[i];
  a.t_c_steps[i] += a.c_steps[i];
  a.t_c_forced[i] += a.c_forced[i];
  a.t_r_sum[i] += a.r_sum[i];
  a.t_r_sum_sq[i] += a.r_sum_sq[i];
  a.t_r_count[i] += a.r_count[i];
}

}  // namespace
}  // namespace n2w

using namespace n2w;

struct n2w_server {
  struct Request {
    int64_t id = 0;
    n2w_request req{};
    std::vector<float> h_points;
    int state = N2W_REQUEST_PENDING;
    std::string error;
    // device residency
    size_t pool_off = 0, pool_len = 0;
    n2w_vec3* d_points = nullptr;
    double *sum = nullptr, *sum_sq = nullptr;
    uint64_t* steps = nullptr;
    uint32_t *count = nullptr, *forced = nullptr;
    // NC+2LMC: the cache and the residual level (the fields above hold the coarse level)
    bool nc = false;
    n2w_server_nc ncfg{};
    double *r_sum = nullptr, *r_sum_sq = nullptr;
    uint32_t* r_count = nullptr;
    int residual_walks = 0;     // residual walks per point of the current sweep
    int64_t residual_done = 0;  // residual walks per point completed
    // progress
    int64_t cursor = 0;         // next point of the current sweep
    int sweep = 0;              // index of the current sweep
    int sweep_walks = 0;        // walks per point of the current sweep
    int64_t walks_done = 0;     // walks per point completed
    float max_stderr = INFINITY;
    float rms_stderr = INFINITY;
    int ticks = 0;
    // results
    std::vector<double> mean, stderr_;
    int64_t t_submit = 0, t_admit = 0, t_finish = 0;
  };

  std::unique_ptr<n2w_scene> scene;
  std::vector<const n2w_bvh*> bvhs;  // NC+2LMC requests walk the meshes' own BVHs
  std::map<std::pair<int, int>, n2w_server_nc> nc;  // (mesh, problem) -> cache; guarded by mu
  std::vector<n2w_problem> problems;
  n2w_problem* d_problems = nullptr;
  n2w_server_options opt{};
  int device = 0;
  cudaStream_t stream = nullptr;
  char* d_pool = nullptr;
  std::unique_ptr<PoolAllocator> pool;
  BatchInst* d_insts = nullptr;
  BatchInst* h_insts = nullptr;  // pinned staging of the tick's instance table
  float4* d_cpd = nullptr;
  int2* d_ids = nullptr;
  int64_t tick_point_cap = 0;
  char* d_hdr = nullptr;         // queue counter + run counters of a tick
  unsigned* d_conv = nullptr;    // per-slot max stderr (float bits)
  unsigned* h_conv = nullptr;    // pinned
  double* d_conv_sum = nullptr;  // per-slot sum over points of var / n
  double* h_conv_sum = nullptr;  // pinned
  n2w_walk_counters* h_counters = nullptr;  // pinned
  char* d_nc_scratch = nullptr;  // one chunk's coarse + residual statistics
  cudaEvent_t ev_tick0 = nullptr, ev_tick1 = nullptr;  // brackets a tick's walker launches
  cudaStream_t nc_stream = nullptr;  // NC+2LMC chunks, concurrent with the plain tick
  cudaEvent_t ev_admitted = nullptr;  // admission uploads done (nc_stream waits on it)
  // NC+2LMC walks a worker iteration enqueues while plain requests are in
  // flight; adapted so the chunks end about when the plain tick does
  int64_t nc_budget = 0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int64_t> pending;
  std::vector<int64_t> active;
  std::unordered_map<int64_t, std::unique_ptr<Request>> requests;
  int64_t next_id = 1;
  bool stop = false;
  std::string fatal;
  std::thread worker;
  n2w_server_stats stats{};
};

namespace {

// Residual walks per point of an NC+2LMC sweep with `coarse` coarse walks (at
// least two, so that the residual variance is defined after the first sweep).
int residual_walks_for(const n2w_server_nc& c, int coarse) {
  return std::max(2, static_cast<int>(std::ceil(static_cast<double>(c.residual_fraction) * coarse)));
}

void fail_all_locked(n2w_server& s, const std::string& msg) {
  s.fatal = msg;
  for (auto& kv : s.requests) {
    auto& r = *kv.second;
    if (r.state == N2W_REQUEST_PENDING || r.state == N2W_REQUEST_ACTIVE) {
      r.state = N2W_REQUEST_FAILED;
      r.error = msg;
      r.t_finish = now_ns();
    }
  }
  s.pending.clear();
  s.active.clear();
  s.cv_done.notify_all();
}

// Admits pending requests in arrival order while the pool and the in-flight
// limit allow; uploads points and zeroes accumulators.  Called without the lock.
void admit(n2w_server& s) {
  std::vector<n2w_server::Request*> admitted;
  {
    std::lock_guard<std::mutex> lk(s.mu);
    while (!s.pending.empty() && static_cast<int>(s.active.size()) < s.opt.max_inflight) {
      auto& r = *s.requests.at(s.pending.front());
      const int64_t n = r.req.point_count;
      size_t off = 0;
      if (!s.pool->alloc(request_bytes(n, r.nc), &off)) break;  // head-of-line waits for memory
      s.pending.pop_front();
      r.pool_off = off;
      r.pool_len = request_bytes(n, r.nc);
      char* base = s.d_pool + off;
      auto carve = [&](size_t bytes) {
        char* p = base;
        base += (bytes + 255) & ~size_t{255};
        return p;
      };
      r.sum = reinterpret_cast<double*>(carve(8 * n));
      r.sum_sq = reinterpret_cast<double*>(carve(8 * n));
      r.steps = reinterpret_cast<uint64_t*>(carve(8 * n));
      r.count = reinterpret_cast<uint32_t*>(carve(4 * n));
      r.forced = reinterpret_cast<uint32_t*>(carve(4 * n));
      r.d_points = reinterpret_cast<n2w_vec3*>(carve(12 * n));
      if (r.nc) {
        r.r_sum = reinterpret_cast<double*>(carve(8 * n));
        r.r_sum_sq = reinterpret_cast<double*>(carve(8 * n));
        r.r_count = reinterpret_cast<uint32_t*>(carve(4 * n));
      }
      r.state = N2W_REQUEST_ACTIVE;
      r.t_admit = now_ns();
      r.sweep_walks = std::min(r.req.max_walks_per_point, std::max(32, r.req.min_walks_per_point));
      if (r.nc) r.residual_walks = residual_walks_for(r.ncfg, r.sweep_walks);
      s.active.push_back(r.id);
      admitted.push_back(&r);
      s.stats.peak_inflight = std::max<int64_t>(s.stats.peak_inflight, static_cast<int64_t>(s.active.size()));
      s.stats.peak_pool_bytes = std::max<int64_t>(s.stats.peak_pool_bytes, static_cast<int64_t>(s.pool->used()));
    }
  }
  for (auto* r : admitted) {
    const int64_t n = r->req.point_count;
    N2W_CUDA(cudaMemsetAsync(r->sum, 0, 8 * n, s.stream));
    N2W_CUDA(cudaMemsetAsync(r->sum_sq, 0, 8 * n, s.stream));
    N2W_CUDA(cudaMemsetAsync(r->steps, 0, 8 * n, s.stream));
    N2W_CUDA(cudaMemsetAsync(r->count, 0, 4 * n, s.stream));
    N2W_CUDA(cudaMemsetAsync(r->forced, 0, 4 * n, s.stream));
    if (r->nc) {
      N2W_CUDA(cudaMemsetAsync(r->r_sum, 0, 8 * n, s.stream));
      N2W_CUDA(cudaMemsetAsync(r->r_sum_sq, 0, 8 * n, s.stream));
      N2W_CUDA(cudaMemsetAsync(r->r_count, 0, 4 * n, s.stream));
    }
    N2W_CUDA(cudaMemcpyAsync(r->d_points, r->h_points.data(), 12 * n, cudaMemcpyHostToDevice, s.stream));
  }
}

// Queues the standard-error reduction of every request in `swept` (slot i of
// d_conv / d_conv_sum) and its copy to the pinned host slots.
void launch_sweep_stderr(n2w_server& s, const std::vector<n2w_server::Request*>& swept) {
  const cudaStream_t st = s.stream;
  N2W_CUDA(cudaMemsetAsync(s.d_conv, 0, sizeof(unsigned) * swept.size(), st));
  N2W_CUDA(cudaMemsetAsync(s.d_conv_sum, 0, sizeof(double) * swept.size(), st));
  for (size_t i = 0; i < swept.size(); ++i) {
    const auto* r = swept[i];
    const int64_t n = r->req.point_count;
    const int grid = static_cast<int>(std::min<int64_t>((n + 255) / 256, 1024));
    LevelSums a{r->sum, r->sum_sq, r->count}, b{};
    if (r->nc) b = LevelSums{r->r_sum, r->r_sum_sq, r->r_count};
    stderr_kernel<<<grid, 256, 0, st>>>(a, b, n, s.d_conv + i, s.d_conv_sum + i);
    N2W_CUDA(cudaGetLastError());
  }
  N2W_CUDA(cudaMemcpyAsync(s.h_conv, s.d_conv, sizeof(unsigned) * swept.size(), cudaMemcpyDeviceToHost, st));
  N2W_CUDA(cudaMemcpyAsync(s.h_conv_sum, s.d_conv_sum, sizeof(double) * swept.size(), cudaMemcpyDeviceToHost, st));
}

// Sweep bookkeeping after the stream has synchronised: record the standard
// errors, then either finish the request (results to the host, pool space
// released) or size its next sweep.
void finish_sweeps(n2w_server& s, const std::vector<n2w_server::Request*>& swept) {
  const cudaStream_t st = s.stream;
  for (size_t i = 0; i < swept.size(); ++i) {
    auto* r = swept[i];
    float mx;
    std::memcpy(&mx, &s.h_conv[i], sizeof(float));
    r->max_stderr = mx;
    r->rms_stderr = static_cast<float>(std::sqrt(s.h_conv_sum[i] / static_cast<double>(r->req.point_count)));
    // the norm the request asked for drives both stopping and the next sweep's size
    const float se = r->req.stderr_norm == N2W_STDERR_RMS ? r->rms_stderr : r->max_stderr;
    r->walks_done += r->sweep_walks;
    r->residual_done += r->residual_walks;
    r->cursor = 0;
    r->sweep += 1;
    const bool reached = se <= r->req.target_stderr && r->walks_done >= r->req.min_walks_per_point;
    const bool capped = r->walks_done >= r->req.max_walks_per_point;
    if (reached || capped) {
      const int64_t n = r->req.point_count;
      std::vector<double> sum(n), sum_sq(n), rsum, rsum_sq;
      std::vector<uint32_t> cnt(n), rcnt;
      N2W_CUDA(cudaMemcpyAsync(sum.data(), r->sum, 8 * n, cudaMemcpyDeviceToHost, st));
      N2W_CUDA(cudaMemcpyAsync(sum_sq.data(), r->sum_sq, 8 * n, cudaMemcpyDeviceToHost, st));
      N2W_CUDA(cudaMemcpyAsync(cnt.data(), r->count, 4 * n, cudaMemcpyDeviceToHost, st));
      if (r->nc) {
        rsum.resize(n);
        rsum_sq.resize(n);
        rcnt.resize(n);
        N2W_CUDA(cudaMemcpyAsync(rsum.data(), r->r_sum, 8 * n, cudaMemcpyDeviceToHost, st));
        N2W_CUDA(cudaMemcpyAsync(rsum_sq.data(), r->r_sum_sq, 8 * n, cudaMemcpyDeviceToHost, st));
        N2W_CUDA(cudaMemcpyAsync(rcnt.data(), r->r_count, 4 * n, cudaMemcpyDeviceToHost, st));
      }
      N2W_CUDA(cudaStreamSynchronize(st));
      r->mean.resize(n);
      r->stderr_.resize(n);
      for (int64_t p = 0; p < n; ++p) {
        const double c = cnt[p];
        double m = c > 0 ? sum[p] / c : 0.0;
        double ev = mean_variance(sum[p], sum_sq[p], c);
        if (r->nc) {
          // NC+2LMC estimate: coarse mean + residual mean, variances add
          const double rc = rcnt[p];
          m += rc > 0 ? rsum[p] / rc : 0.0;
          ev += mean_variance(rsum[p], rsum_sq[p], rc);
        }
        r->mean[p] = m;
        r->stderr_[p] = std::sqrt(ev);
      }
      std::lock_guard<std::mutex> lk(s.mu);
      s.pool->release(r->pool_off, r->pool_len);
      r->state = reached ? N2W_REQUEST_DONE : N2W_REQUEST_CAPPED;
      r->t_finish = now_ns();
      r->h_points.clear();
      r->h_points.shrink_to_fit();
      s.active.erase(std::find(s.active.begin(), s.active.end(), r->id));
      s.stats.completed += 1;
      s.cv_done.notify_all();
    } else {
      // Next sweep: the walks the standard-error model predicts are still
      // needed (stderr ~ 1/sqrt(N)), plus 10 %, within [32, cap - done].
      const double need = static_cast<double>(r->walks_done) *
                              std::pow(static_cast<double>(se) / r->req.target_stderr, 2.0) * 1.1 -
                          static_cast<double>(r->walks_done);
      int64_t w = static_cast<int64_t>(std::ceil(std::isfinite(need) ? need : 1e9));
      w = std::max<int64_t>(w, std::max<int64_t>(32, r->req.min_walks_per_point - r->walks_done));
      w = std::min<int64_t>(w, r->req.max_walks_per_point - r->walks_done);
      w = std::min<int64_t>(w, 1 << 20);
      r->sweep_walks = static_cast<int>(std::max<int64_t>(w, 1));
      if (r->nc) r->residual_walks = residual_walks_for(r->ncfg, r->sweep_walks);
    }
  }
}

// In-flight plain requests a tick of tick_walks serves before it grows.
constexpr int64_t kRequestsPerBaseTick = 8;

struct Slice {
  n2w_server::Request* r;
  int64_t first, count;  // point range of this tick
};

// One tick, enqueued: share the walk budget and launch the batched walker over
// every active plain request's next point range on s.stream.  tick_finish
// synchronises, advances cursors and checks finished sweeps.
struct TickWork {
  std::vector<Slice> slices;
};

TickWork tick_launch(n2w_server& s) {
  TickWork tw;
  std::vector<n2w_server::Request*> act;
  {
    std::lock_guard<std::mutex> lk(s.mu);
    for (int64_t id : s.active) {
      auto* r = s.requests.at(id).get();
      if (!r->nc) act.push_back(r);
    }
  }
  if (act.empty()) return tw;
  // The tick's walk budget goes to the requests with the least remaining
  // sweep work first (shortest remaining work first keeps small requests
  // fast); below, every request still advances by at least one point per tick.
  std::vector<int64_t> want(act.size()), give(act.size(), 0);
  std::vector<size_t> order(act.size());
  bool small_in_flight = false;  // some request could finish its sweep within tick_walks
  for (size_t k = 0; k < act.size(); ++k) {
    want[k] = (act[k]->req.point_count - act[k]->cursor) * static_cast<int64_t>(act[k]->sweep_walks);
    order[k] = k;
    small_in_flight = small_in_flight || want[k] <= s.opt.tick_walks;
  }
  // Larger ticks when only large sweeps are in flight: a tick waits for its
  // slowest walk, so more walks per tick fill the GPU better, and no small
  // request is there to be delayed by the longer tick.  When many requests
  // are in flight the queue is building up, and the tick grows with their
  // number (every request still advances in every tick), trading a longer
  // tick for the throughput that drains the queue.
  int64_t budget = s.opt.tick_walks;
  if (s.opt.tick_walks_max > s.opt.tick_walks) {
    if (!small_in_flight) {
      budget = s.opt.tick_walks_max;
    } else {
      const int64_t scaled = s.opt.tick_walks * static_cast<int64_t>(act.size()) / kRequestsPerBaseTick;
      budget = std::min(std::max(scaled, s.opt.tick_walks), s.opt.tick_walks_max);
    }
  }
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return want[a] < want[b]; });
  int64_t left = budget;
  for (size_t k : order) {
    give[k] = std::min(want[k], left);
    left -= give[k];
  }
  std::vector<Slice>& slices = tw.slices;
  int64_t tick_points = 0;
  for (size_t k = 0; k < act.size(); ++k) {
    auto* r = act[k];
    int64_t pts = give[k] / r->sweep_walks;
    pts = std::max<int64_t>(pts, 1);  // every request advances every tick
    pts = std::min(pts, r->req.point_count - r->cursor);
    pts = std::min(pts, s.tick_point_cap - tick_points);
    if (pts <= 0) continue;
    slices.push_back({r, r->cursor, pts});
    tick_points += pts;
  }
  if (slices.empty()) return tw;
  const int chunk = s.opt.chunk > 0 ? s.opt.chunk : 1;
  int64_t cbase = 0, pbase = 0;
  for (size_t i = 0; i < slices.size(); ++i) {
    const Slice& sl = slices[i];
    auto* r = sl.r;
    BatchInst& I = s.h_insts[i];
    I = BatchInst{};
    I.points = r->d_points + sl.first;
    I.sum = r->sum + sl.first;
    I.sum_sq = r->sum_sq + sl.first;
    I.count = r->count + sl.first;
    I.steps = r->steps + sl.first;
    I.forced = r->forced + sl.first;
    I.point_base = pbase;
    I.point_count = sl.count;
    I.chunk_base = cbase;
    I.walks_per_point = r->sweep_walks;
    I.chunks_per_point = (r->sweep_walks + chunk - 1) / chunk;
    set_instance_geometry(I, *s.scene, r->req.mesh);
    set_instance_problem(I, s.problems[r->req.problem], s.d_problems + r->req.problem);
    // sweep key; walk ids p * W + w over the whole request (p = global point index)
    philox_key(r->req.seed + 0x9E3779B97F4A7C15ull * static_cast<uint64_t>(r->sweep + 1), 0u, I.k0, I.k1);
    I.wid_base = sl.first * static_cast<int64_t>(r->sweep_walks);
    pbase += sl.count;
    cbase += sl.count * I.chunks_per_point;
  }
  const cudaStream_t st = s.stream;
  N2W_CUDA(cudaMemcpyAsync(s.d_insts, s.h_insts, sizeof(BatchInst) * slices.size(), cudaMemcpyHostToDevice, st));
  N2W_CUDA(cudaMemsetAsync(s.d_hdr, 0, 512, st));
  WalkArgs a{};
  a.nodes = reinterpret_cast<const float4*>(s.scene->d_nodes);
  a.tris = reinterpret_cast<const float4*>(s.scene->d_tris);
  a.first_cpd = s.d_cpd;
  a.first_ids = s.d_ids;
  a.total_chunks = cbase;
  a.chunk = chunk;
  a.regen = s.opt.regen_threshold > 0 ? s.opt.regen_threshold : kDefaultRegen;
  a.max_steps = s.opt.max_steps;
  a.eps = s.opt.epsilon;
  a.step_scale = s.opt.step_scale;
  a.queue = reinterpret_cast<unsigned long long*>(s.d_hdr);
  a.counters = reinterpret_cast<n2w_walk_counters*>(s.d_hdr + 256);
  a.insts = s.d_insts;
  a.n_insts = static_cast<int>(slices.size());
  N2W_CUDA(cudaEventRecord(s.ev_tick0, st));
  launch_first_query_batch(a, pbase, s.d_cpd, s.d_ids, st);
  launch_walker_batch(a, s.opt.block_size > 0 ? s.opt.block_size : kDefaultWalkerThreads, 0, 0, st);
  N2W_CUDA(cudaEventRecord(s.ev_tick1, st));
  N2W_CUDA(cudaMemcpyAsync(s.h_counters, s.d_hdr + 256, sizeof(n2w_walk_counters), cudaMemcpyDeviceToHost, st));
  return tw;
}

void tick_finish(n2w_server& s, TickWork& tw) {
  const std::vector<Slice>& slices = tw.slices;
  if (slices.empty()) return;
  const cudaStream_t st = s.stream;
  // Requests whose sweep ends with this tick: reduce their standard errors.
  std::vector<n2w_server::Request*> swept;
  for (const Slice& sl : slices) {
    if (sl.first + sl.count == sl.r->req.point_count) swept.push_back(sl.r);
  }
  if (!swept.empty()) launch_sweep_stderr(s, swept);
  N2W_CUDA(cudaStreamSynchronize(st));
  float tick_ms = 0.0f;
  N2W_CUDA(cudaEventElapsedTime(&tick_ms, s.ev_tick0, s.ev_tick1));
  {
    std::lock_guard<std::mutex> lk(s.mu);
    s.stats.ticks += 1;
    s.stats.tick_gpu_us += static_cast<int64_t>(tick_ms * 1000.0f);
    s.stats.walks += static_cast<int64_t>(s.h_counters->walks);
    s.stats.walk_steps += static_cast<int64_t>(s.h_counters->steps);
    s.stats.overflow += static_cast<int64_t>(s.h_counters->overflow);
  }
  for (const Slice& sl : slices) {
    sl.r->cursor += sl.count;
    sl.r->ticks += 1;
  }
  finish_sweeps(s, swept);
}

// NC+2LMC work of one worker iteration, enqueued on s.nc_stream so that it
// runs on the device concurrently with the plain tick: chunks of up to kNcChunk
// points, shortest remaining sweep first, until s.nc_budget coarse + residual
// walks are enqueued (at least one chunk).  Each chunk is keyed by (request
// seed, sweep, first point of the chunk) alone, so the number of chunks per
// iteration changes no estimate.  nc_finish synchronises and checks sweeps.
struct NcWork {
  std::vector<n2w_server::Request*> swept;
  int64_t chunks = 0, walks = 0;
};

NcWork nc_launch(n2w_server& s) {
  NcWork nw;
  std::vector<n2w_server::Request*> act;
  {
    std::lock_guard<std::mutex> lk(s.mu);
    for (int64_t id : s.active) {
      auto* r = s.requests.at(id).get();
      if (r->nc) act.push_back(r);
    }
  }
  if (act.empty()) return nw;
  auto remaining = [](const n2w_server::Request* r) {
    return (r->req.point_count - r->cursor) * static_cast<int64_t>(r->sweep_walks + r->residual_walks);
  };
  std::stable_sort(act.begin(), act.end(),
                   [&](const n2w_server::Request* a, const n2w_server::Request* b) { return remaining(a) < remaining(b); });
  const cudaStream_t st = s.nc_stream;
  N2W_CUDA(cudaStreamWaitEvent(st, s.ev_admitted, 0));  // points and accumulators of new requests
  double* c_sum = reinterpret_cast<double*>(s.d_nc_scratch);
  double* c_sum_sq = c_sum + kNcChunk;
  double* r_sum = c_sum_sq + kNcChunk;
  double* r_sum_sq = r_sum + kNcChunk;
  uint64_t* c_steps = reinterpret_cast<uint64_t*>(r_sum_sq + kNcChunk);
  uint32_t* c_count = reinterpret_cast<uint32_t*>(c_steps + kNcChunk);
  uint32_t* c_forced = c_count + kNcChunk;
  uint32_t* r_count = c_forced + kNcChunk;
  int64_t left = s.nc_budget > 0 ? s.nc_budget : s.opt.tick_walks, chunks = 0, walks = 0;
  std::vector<n2w_server::Request*>& swept = nw.swept;
  for (auto* r : act) {
    if (left <= 0) break;
    while (left > 0 && r->cursor < r->req.point_count) {
      const int64_t first = r->cursor;
      // Chunk size from the request's own sweep: at most kNcChunk points and at
      // most about one tick's walks, so a chunk never holds the worker (and the
      // plain ticks behind it) for much longer than a tick.  It depends on
      // nothing else in flight, so the chunking -- and the walks -- are the same
      // alone and in any mix.
      const int64_t per_point = std::max<int64_t>(1, r->sweep_walks + r->residual_walks);
      const int64_t span = std::min(kNcChunk, std::max(kNcMinChunk, s.opt.tick_walks / per_point));
      const int64_t np = std::min(span, r->req.point_count - first);
      n2w_nc2lmc_options o{};
      o.coarse_walks = r->sweep_walks;
      o.residual_walks = r->residual_walks;
      o.depth_m = r->ncfg.depth_m;
      o.max_steps = s.opt.max_steps;
      o.epsilon = s.opt.epsilon;
      o.step_scale = s.opt.step_scale;
      o.seed = splitmix64(r->req.seed ^ splitmix64((static_cast<uint64_t>(r->sweep) << 40) +
                                                   static_cast<uint64_t>(first)));
      for (int k = 0; k < 3; ++k) {
        o.input_min[k] = r->ncfg.input_min[k];
        o.input_extent[k] = r->ncfg.input_extent[k];
      }
      n2w_point_stats co{c_sum, c_sum_sq, c_count, c_steps, c_forced};
      n2w_point_stats re{r_sum, r_sum_sq, r_count, nullptr, nullptr};
      const int rc = n2w_nc2lmc_estimate_ex(s.bvhs[r->req.mesh], &s.problems[r->req.problem], r->ncfg.cache,
                                            r->d_points + first, np, &o, co, re, nullptr, st);
      if (rc != N2W_OK) throw Error(rc, n2w_last_error());
      NcChunkAdd add;
      add.c_sum = c_sum;
      add.c_sum_sq = c_sum_sq;
      add.r_sum = r_sum;
      add.r_sum_sq = r_sum_sq;
      add.c_count = c_count;
      add.c_forced = c_forced;
      add.r_count = r_count;
      add.c_steps = c_steps;
      add.t_c_sum = r->sum + first;
      add.t_c_sum_sq = r->sum_sq + first;
      add.t_r_sum = r->r_sum + first;
      add.t_r_sum_sq = r->r_sum_sq + first;
      add.t_c_count = r->count + first;
      add.t_c_forced = r->forced + first;
      add.t_r_count = r->r_count + first;
      add.t_c_steps = r->steps + first;
      add_nc_chunk_kernel<<<static_cast<int>((np + 255) / 256), 256, 0, st>>>(add, np);
      N2W_CUDA(cudaGetLastError());
      const int64_t w = np * static_cast<int64_t>(r->sweep_walks + r->residual_walks);
      left -= w;
      walks += w;
      chunks += 1;
      r->cursor += np;
      r->ticks += 1;
    }
    if (r->cursor == r->req.point_count) swept.push_back(r);
  }
  nw.chunks = chunks;
  nw.walks = walks;
  return nw;
}

void nc_finish(n2w_server& s, NcWork& nw) {
  if (nw.chunks == 0) return;
  N2W_CUDA(cudaStreamSynchronize(s.nc_stream));
  if (!nw.swept.empty()) {
    // the standard-error reduction shares its buffers with the tick's: on s.stream, after it
    launch_sweep_stderr(s, nw.swept);
    N2W_CUDA(cudaStreamSynchronize(s.stream));
  }
  {
    std::lock_guard<std::mutex> lk(s.mu);
    s.stats.nc_chunks += nw.chunks;
    s.stats.nc_walks += nw.walks;
  }
  finish_sweeps(s, nw.swept);
}

// NC+2LMC walk budget of a worker iteration while plain requests are in
// flight.  A NC+2LMC walk costs several plain walks (residual walks carry the
// Poisson source samples, coarse walks the cache), so a budget equal to the
// plain tick's held the worker -- and every plain request -- for up to twice
// the tick.  Multiplicative steps keep the time the worker waits for the
// chunks after the tick has ended between 1/16 and 1/4 of the tick.
constexpr int64_t kNcBudgetMinDivisor = 8;  // floor: tick_walks / 8 (and always one chunk)

void adapt_nc_budget(n2w_server& s, int64_t tick_ns, int64_t wait_ns) {
  const int64_t hi = std::max(s.opt.tick_walks, s.opt.tick_walks_max);
  const int64_t lo = std::max<int64_t>(1, s.opt.tick_walks / kNcBudgetMinDivisor);
  int64_t b = s.nc_budget > 0 ? s.nc_budget : s.opt.tick_walks;
  if (4 * wait_ns > tick_ns) b = b * 3 / 4;
  else if (16 * wait_ns < tick_ns) b = b * 5 / 4 + 1;
  s.nc_budget = std::min(hi, std::max(lo, b));
}

void worker_loop(n2w_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty() || !s->active.empty(); });
      if (s->stop) return;
    }
    try {
      admit(*s);
      N2W_CUDA(cudaEventRecord(s->ev_admitted, s->stream));
      const int64_t t0 = now_ns();
      // plain tick and NC+2LMC chunks are both enqueued before either is
      // waited for, so their kernels overlap on the device
      TickWork tw = tick_launch(*s);
      NcWork nw = nc_launch(*s);
      const bool plain = !tw.slices.empty();
      tick_finish(*s, tw);
      const int64_t t1 = now_ns();
      nc_finish(*s, nw);
      const int64_t t2 = now_ns();
      if (plain && nw.chunks > 0) adapt_nc_budget(*s, t1 - t0, t2 - t1);
      std::lock_guard<std::mutex> lk(s->mu);
      s->stats.tick_us += (t1 - t0) / 1000;
      s->stats.nc_us += (t2 - t1) / 1000;
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lk(s->mu);
      fail_all_locked(*s, std::string("serving loop stopped: ") + e.what());
      return;
    }
  }
}

void destroy_server(n2w_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (auto& kv : s->requests) {
      auto& r = *kv.second;
      if (r.state == N2W_REQUEST_PENDING || r.state == N2W_REQUEST_ACTIVE) {
        r.state = N2W_REQUEST_FAILED;
        r.error = "server destroyed";
      }
    }
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->nc_stream) cudaStreamSynchronize(s->nc_stream);
  cudaFree(s->d_pool);
  cudaFree(s->d_insts);
  cudaFree(s->d_cpd);
  cudaFree(s->d_ids);
  cudaFree(s->d_hdr);
  cudaFree(s->d_conv);
  cudaFree(s->d_problems);
  cudaFreeHost(s->h_insts);
  cudaFreeHost(s->h_conv);
  cudaFree(s->d_conv_sum);
  cudaFree(s->d_nc_scratch);
  if (s->ev_tick0) cudaEventDestroy(s->ev_tick0);
  if (s->ev_tick1) cudaEventDestroy(s->ev_tick1);
  cudaFreeHost(s->h_conv_sum);
  cudaFreeHost(s->h_counters);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->nc_stream) cudaStreamDestroy(s->nc_stream);
  if (s->ev_admitted) cudaEventDestroy(s->ev_admitted);
  if (s->scene) {
    n2w_scene_destroy(s->scene.release());
  }
  delete s;
}

}  // namespace

extern "C" {

int n2w_server_options_default(n2w_server_options* out) {
  return guarded([&] {
    N2W_REQUIRE(out, "null output");
    *out = n2w_server_options{};
    out->pool_bytes = 0;
    out->pool_fraction = 0.25f;
    out->max_inflight = 256;
    out->tick_walks = 1 << 21;
    out->max_steps = 256;
    out->epsilon = 1.0e-3f;
    out->step_scale = 0.999f;
    out->block_size = 256;
    out->regen_threshold = 8;
    out->chunk = 1;
    out->tick_walks_max = int64_t{1} << 23;
  });
}

int n2w_server_create(const n2w_bvh* const* bvhs, int mesh_count, const n2w_problem* problems, int problem_count,
                      const n2w_server_options* options, n2w_server** out) {
  n2w_server* s = nullptr;
  const int st = guarded([&] {
    N2W_REQUIRE(bvhs && problems && out && mesh_count > 0 && problem_count > 0, "n2w_server_create: bad arguments");
    n2w_server_options o{};
    if (options) o = *options;
    else n2w_server_options_default(&o);
    N2W_REQUIRE(o.max_inflight >= 1 && o.max_inflight <= 65536, "max_inflight must be in [1, 65536]");
    N2W_REQUIRE(o.tick_walks >= 1024, "tick_walks must be >= 1024");
    N2W_REQUIRE(o.max_steps > 0 && o.epsilon > 0.0f && o.step_scale > 0.0f && o.step_scale <= 1.0f,
                "invalid walk options");
    N2W_REQUIRE(o.block_size == 0 || (o.block_size >= 32 && o.block_size <= kWalkerMaxThreads && o.block_size % 32 == 0),
                "block_size must be 0 or a multiple of 32 in [32, 256]");
    N2W_REQUIRE(o.chunk >= 0 && o.chunk <= 64, "chunk must be in [0, 64]");
    N2W_REQUIRE(o.tick_walks_max >= 0, "tick_walks_max must be >= 0 (values <= tick_walks disable larger ticks)");
    for (int p = 0; p < problem_count; ++p) validate_problem(problems[p]);
    s = new n2w_server();
    s->opt = o;
    N2W_CUDA(cudaGetDevice(&s->device));
    n2w_scene* sc = nullptr;
    const int rc = n2w_scene_create(bvhs, mesh_count, &sc);
    if (rc != N2W_OK) throw Error(rc, n2w_last_error());
    s->scene.reset(sc);
    s->bvhs.assign(bvhs, bvhs + mesh_count);
    s->problems.assign(problems, problems + problem_count);
    N2W_CUDA(cudaMalloc(&s->d_problems, sizeof(n2w_problem) * problem_count));
    N2W_CUDA(cudaMemcpy(s->d_problems, problems, sizeof(n2w_problem) * problem_count, cudaMemcpyHostToDevice));
    size_t pool = static_cast<size_t>(o.pool_bytes);
    if (pool == 0) {
      size_t fr = 0, tot = 0;
      N2W_CUDA(cudaMemGetInfo(&fr, &tot));
      const float f = o.pool_fraction > 0.0f && o.pool_fraction <= 0.9f ? o.pool_fraction : 0.25f;
      pool = static_cast<size_t>(static_cast<double>(fr) * f);
    }
    pool &= ~size_t{255};
    N2W_REQUIRE(pool >= (1u << 20), "device pool below 1 MiB");
    N2W_CUDA(cudaMalloc(&s->d_pool, pool));
    s->pool = std::make_unique<PoolAllocator>(pool);
    s->opt.pool_bytes = static_cast<int64_t>(pool);
    // A tick holds at most one instance per in-flight request and at most
    // (its budget) / 32 + max_inflight points (sweeps have >= 32 walks per point).
    s->tick_point_cap = std::max(o.tick_walks, o.tick_walks_max) / 32 + o.max_inflight;
    N2W_CUDA(cudaMalloc(&s->d_insts, sizeof(BatchInst) * o.max_inflight));
    N2W_CUDA(cudaMallocHost(&s->h_insts, sizeof(BatchInst) * o.max_inflight));
    N2W_CUDA(cudaMalloc(&s->d_cpd, sizeof(float4) * s->tick_point_cap));
    N2W_CUDA(cudaMalloc(&s->d_ids, sizeof(int2) * s->tick_point_cap));
    N2W_CUDA(cudaMalloc(&s->d_hdr, 512));
    N2W_CUDA(cudaMalloc(&s->d_conv, sizeof(unsigned) * o.max_inflight));
    N2W_CUDA(cudaMallocHost(&s->h_conv, sizeof(unsigned) * o.max_inflight));
    N2W_CUDA(cudaMalloc(&s->d_conv_sum, sizeof(double) * o.max_inflight));
    N2W_CUDA(cudaMallocHost(&s->h_conv_sum, sizeof(double) * o.max_inflight));
    N2W_CUDA(cudaMallocHost(&s->h_counters, sizeof(n2w_walk_counters)));
    // coarse sum, sum_sq, residual sum, sum_sq, coarse steps (8 B); coarse count, forced, residual count (4 B)
    N2W_CUDA(cudaMalloc(&s->d_nc_scratch, kNcChunk * (5 * 8 + 3 * 4)));
    N2W_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    N2W_CUDA(cudaStreamCreateWithFlags(&s->nc_stream, cudaStreamNonBlocking));
    N2W_CUDA(cudaEventCreateWithFlags(&s->ev_admitted, cudaEventDisableTiming));
    N2W_CUDA(cudaEventCreate(&s->ev_tick0));
    N2W_CUDA(cudaEventCreate(&s->ev_tick1));
    s->worker = std::thread(worker_loop, s);
    *out = s;
  });
  if (st != N2W_OK && s) destroy_server(s);
  return st;
}

int n2w_server_set_nc(n2w_server* s, int mesh, int problem, const n2w_server_nc* nc) {
  return guarded([&] {
    N2W_REQUIRE(s && nc, "n2w_server_set_nc: null argument");
    N2W_REQUIRE(mesh >= 0 && mesh < static_cast<int>(s->bvhs.size()), "mesh index out of range");
    N2W_REQUIRE(problem >= 0 && problem < static_cast<int>(s->problems.size()), "problem index out of range");
    N2W_REQUIRE(nc->depth_m >= 0, "depth_m must be >= 0");
    N2W_REQUIRE(nc->residual_fraction > 0.0f && nc->residual_fraction <= 1.0f, "residual_fraction must be in (0, 1]");
    for (int k = 0; k < 3; ++k) N2W_REQUIRE(nc->input_extent[k] > 0.0f, "input_extent must be positive");
    std::lock_guard<std::mutex> lk(s->mu);
    s->nc[{mesh, problem}] = *nc;
  });
}

int n2w_server_submit(n2w_server* s, const n2w_request* req, const float* h_points, int64_t* id_out) {
  return guarded([&] {
    N2W_REQUIRE(s && req && id_out, "n2w_server_submit: null argument");
    N2W_REQUIRE(req->mesh >= 0 && req->mesh < static_cast<int>(s->scene->meshes.size()), "mesh index out of range");
    N2W_REQUIRE(req->problem >= 0 && req->problem < static_cast<int>(s->problems.size()),
                "problem index out of range");
    N2W_REQUIRE(req->point_count > 0 && h_points, "a request needs at least one point");
    N2W_REQUIRE(req->target_stderr > 0.0f, "target_stderr must be positive");
    N2W_REQUIRE(req->stderr_norm == N2W_STDERR_MAX || req->stderr_norm == N2W_STDERR_RMS, "bad stderr_norm");
    N2W_REQUIRE(req->max_walks_per_point >= 1 && req->min_walks_per_point >= 0 &&
                    req->min_walks_per_point <= req->max_walks_per_point,
                "need 0 <= min_walks_per_point <= max_walks_per_point, max >= 1");
    N2W_REQUIRE(req->mode == N2W_REQUEST_MODE_PLAIN || req->mode == N2W_REQUEST_MODE_NC2LMC, "bad request mode");
    const bool nc = req->mode == N2W_REQUEST_MODE_NC2LMC;
    if (request_bytes(req->point_count, nc) > s->pool->capacity()) {
      throw Error(N2W_ENOMEM, "request of " + std::to_string(req->point_count) +
                                  " points needs more device memory than the whole serving pool (" +
                                  std::to_string(s->pool->capacity()) + " bytes)");
    }
    auto r = std::make_unique<n2w_server::Request>();
    r->req = *req;
    r->nc = nc;
    r->h_points.assign(h_points, h_points + 3 * req->point_count);
    r->t_submit = now_ns();
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->fatal.empty()) throw Error(N2W_ECUDA, s->fatal);
    if (nc) {
      auto it = s->nc.find({req->mesh, req->problem});
      N2W_REQUIRE(it != s->nc.end(), "NC+2LMC request: no cache registered for this (mesh, problem)");
      r->ncfg = it->second;
    }
    r->id = s->next_id++;
    *id_out = r->id;
    s->pending.push_back(r->id);
    s->requests.emplace(r->id, std::move(r));
    s->stats.submitted += 1;
    s->cv_work.notify_one();
  });
}

int n2w_server_poll(n2w_server* s, int64_t id, int* state_out) {
  return guarded([&] {
    N2W_REQUIRE(s && state_out, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    N2W_REQUIRE(it != s->requests.end(), "unknown request id");
    *state_out = it->second->state;
  });
}

int n2w_server_wait(n2w_server* s, int64_t id, double timeout_seconds, double* h_mean, double* h_stderr,
                    n2w_request_info* info) {
  return guarded([&] {
    N2W_REQUIRE(s, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    N2W_REQUIRE(it != s->requests.end(), "unknown request id (or already collected)");
    n2w_server::Request* r = it->second.get();
    auto finished = [&] {
      return r->state == N2W_REQUEST_DONE || r->state == N2W_REQUEST_CAPPED || r->state == N2W_REQUEST_FAILED;
    };
    if (timeout_seconds < 0) {
      s->cv_done.wait(lk, finished);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_seconds), finished)) {
      throw Error(N2W_ETIMEOUT, "request " + std::to_string(id) + " still running");
    }
    if (info) {
      *info = n2w_request_info{};
      info->state = r->state;
      info->walks_per_point = r->walks_done;
      info->sweeps = r->sweep;
      info->ticks = r->ticks;
      info->max_stderr = r->max_stderr;
      info->rms_stderr = r->rms_stderr;
      info->queue_seconds = (r->t_admit ? r->t_admit - r->t_submit : 0) * 1e-9;
      info->latency_seconds = (r->t_finish - r->t_submit) * 1e-9;
      info->residual_walks_per_point = r->residual_done;
    }
    if (r->state == N2W_REQUEST_FAILED) {
      const std::string msg = r->error;
      s->requests.erase(it);
      throw Error(N2W_ECUDA, msg);
    }
    const int64_t n = r->req.point_count;
    if (h_mean) std::memcpy(h_mean, r->mean.data(), 8 * n);
    if (h_stderr) std::memcpy(h_stderr, r->stderr_.data(), 8 * n);
    s->requests.erase(it);
  });
}

int n2w_server_get_stats(n2w_server* s, n2w_server_stats* out) {
  return guarded([&] {
    N2W_REQUIRE(s && out, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->inflight = static_cast<int64_t>(s->active.size());
    out->pending = static_cast<int64_t>(s->pending.size());
    out->pool_bytes = static_cast<int64_t>(s->pool->capacity());
    out->pool_used = static_cast<int64_t>(s->pool->used());
  });
}

void n2w_server_destroy(n2w_server* s) { destroy_server(s); }

}  // extern "C"
