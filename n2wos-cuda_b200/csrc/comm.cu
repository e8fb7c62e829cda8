// Multi-GPU exchange over NCCL, one process per GPU.
//
// Walk-on-Spheres work shards without communication (points or walks per
// rank); the only exchanges are the element-wise sums that combine per-point
// FP64 statistics of walk shards, the max / sum of per-rank timings, and, for
// data-parallel cache training, the sum of every rank's gradient before each
// Adam step.  All are all-reduces on caller-owned device buffers, issued on
// the caller's stream; the library owns only the communicator and an 8-byte
// device word for barriers.  Plain device loads and stores only: no peer
// memory, no multicast.
//
// The reference has no distributed code (one process, one GPU).
#include <cuda_runtime.h>
#include <nccl.h>

#include <cstring>

#include "internal.hpp"

struct n2w_comm {
  ncclComm_t comm = nullptr;
  int rank = 0;
  int world = 1;
  int device = 0;
  int* d_word = nullptr;
};

namespace n2w {
namespace {

#define N2W_NCCL(expr)                                                                          \
  do {                                                                                          \
    const ncclResult_t r__ = (expr);                                                            \
    if (r__ != ncclSuccess) throw Error(N2W_ECUDA, std::string("NCCL: ") + ncclGetErrorString(r__) + \
                                                       " in " #expr);                             \
  } while (false)

ncclDataType_t nccl_type(int dtype) {
  switch (dtype) {
    case N2W_DTYPE_F32: return ncclFloat32;
    case N2W_DTYPE_F64: return ncclFloat64;
    case N2W_DTYPE_U32: return ncclUint32;
    case N2W_DTYPE_U64: return ncclUint64;
    case N2W_DTYPE_I32: return ncclInt32;
    default: throw Error(N2W_EINVAL, "unknown dtype");
  }
}

ncclRedOp_t nccl_op(int op) {
  switch (op) {
    case N2W_OP_SUM: return ncclSum;
    case N2W_OP_MAX: return ncclMax;
    case N2W_OP_MIN: return ncclMin;
    default: throw Error(N2W_EINVAL, "unknown reduction op");
  }
}

}  // namespace
}  // namespace n2w

using namespace n2w;

extern "C" {

int n2w_comm_unique_id(uint8_t* id_out) {
  return guarded([&] {
    N2W_REQUIRE(id_out, "null output");
    static_assert(sizeof(ncclUniqueId) == N2W_COMM_ID_BYTES, "NCCL unique id size");
    ncclUniqueId id;
    N2W_NCCL(ncclGetUniqueId(&id));
    std::memcpy(id_out, &id, sizeof(id));
  });
}

int n2w_comm_create(const uint8_t* id, int world, int rank, n2w_comm** out) {
  return guarded([&] {
    N2W_REQUIRE(id && out, "null argument");
    N2W_REQUIRE(world >= 1 && rank >= 0 && rank < world, "need 0 <= rank < world");
    auto* c = new n2w_comm();
    c->rank = rank;
    c->world = world;
    try {
      N2W_CUDA(cudaGetDevice(&c->device));
      N2W_CUDA(cudaMalloc(&c->d_word, sizeof(int) * 2));
      ncclUniqueId uid;
      std::memcpy(&uid, id, sizeof(uid));
      N2W_NCCL(ncclCommInitRank(&c->comm, world, uid, rank));
    } catch (...) {
      if (c->d_word) cudaFree(c->d_word);
      delete c;
      throw;
    }
    *out = c;
  });
}

int n2w_comm_info(const n2w_comm* c, int* rank, int* world) {
  return guarded([&] {
    N2W_REQUIRE(c, "null communicator");
    if (rank) *rank = c->rank;
    if (world) *world = c->world;
  });
}

int n2w_comm_allreduce(n2w_comm* c, const void* d_send, void* d_recv, int64_t count, int dtype, int op,
                       n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(c && c->comm, "null communicator");
    N2W_REQUIRE(count >= 0, "count must be non-negative");
    if (count == 0) return;
    N2W_REQUIRE(d_send && d_recv, "null device buffer");
    N2W_NCCL(ncclAllReduce(d_send, d_recv, static_cast<size_t>(count), nccl_type(dtype), nccl_op(op), c->comm,
                           stream));
  });
}

int n2w_comm_allreduce_point_stats(n2w_comm* c, n2w_point_stats s, int64_t n, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(c && c->comm, "null communicator");
    N2W_REQUIRE(n >= 0, "n must be non-negative");
    if (n == 0) return;
    N2W_REQUIRE(s.d_sum && s.d_sum_sq && s.d_count, "sum, sum_sq and count are required");
    const size_t cnt = static_cast<size_t>(n);
    N2W_NCCL(ncclGroupStart());
    N2W_NCCL(ncclAllReduce(s.d_sum, s.d_sum, cnt, ncclFloat64, ncclSum, c->comm, stream));
    N2W_NCCL(ncclAllReduce(s.d_sum_sq, s.d_sum_sq, cnt, ncclFloat64, ncclSum, c->comm, stream));
    N2W_NCCL(ncclAllReduce(s.d_count, s.d_count, cnt, ncclUint32, ncclSum, c->comm, stream));
    if (s.d_steps) N2W_NCCL(ncclAllReduce(s.d_steps, s.d_steps, cnt, ncclUint64, ncclSum, c->comm, stream));
    if (s.d_forced) N2W_NCCL(ncclAllReduce(s.d_forced, s.d_forced, cnt, ncclUint32, ncclSum, c->comm, stream));
    N2W_NCCL(ncclGroupEnd());
  });
}

int n2w_comm_barrier(n2w_comm* c, n2w_stream_t stream) {
  return guarded([&] {
    N2W_REQUIRE(c && c->comm, "null communicator");
    N2W_CUDA(cudaMemsetAsync(c->d_word, 0, sizeof(int), stream));
    N2W_NCCL(ncclAllReduce(c->d_word, c->d_word + 1, 1, ncclInt32, ncclSum, c->comm, stream));
    N2W_CUDA(cudaStreamSynchronize(stream));
  });
}

void n2w_comm_destroy(n2w_comm* c) {
  if (!c) return;
  if (c->comm) ncclCommDestroy(c->comm);
  if (c->d_word) cudaFree(c->d_word);
  delete c;
}

}  // extern "C"
