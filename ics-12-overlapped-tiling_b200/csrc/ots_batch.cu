// ots_batch.cu -- many independent 2D grids in one persistent launch.
//
// The reference runs one grid per process and one kernel launch per time
// tile (opencl/jacobi-2d/jacobi-2d.cpp:905-931).  A batch of small, uneven
// grids run that way is launch-bound.  Here every grid's run is cut into work
// items (grid, time chunk of T_g steps, x/y tile) and all items go through
// one persistent kernel:
//
//   * the queue is ordered in rounds: round r holds chunk r of every grid
//     that has one, so items only ever depend on items earlier in the queue
//     and the launch always makes progress;
//   * a CTA takes the next item with one atomicAdd, waits until every tile
//     of the grid's previous chunk has completed (a per-(grid, chunk)
//     counter; a bounded spin that records an error and gives up after 2 s
//     or once another CTA has given up; the host can set the limit), runs
//     the overlapped tile
//     (tile_body, loads at L2 because other CTAs wrote them), and publishes
//     its completion (fence, then counter increment);
//   * per grid, the tile shape (T, block x, E) is its own -- chosen by the
//     cost model -- from the menu instantiated here;
//   * the counter reset and the launch are captured once in a CUDA graph.
//
// Stream mode (every grid's kernel = OTS_KERNEL_STREAM): the items are one
// warp's strip x y-segment of the y-streamed 2D kernel (stream2d_body) for
// one time chunk; each warp takes its own item and waits (bounded) for the
// grid's previous chunk, with the same queue order and counters.  T <= 4 keeps
// the strip halo (and so the strips) the same for a grid's last, shallower
// chunk.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/ots.h"
#include "ots_launch.cuh"
#include "ots_tile.cuh"

void ots_set_last_error(const char* msg);

namespace ots {

constexpr int kBatchThreads = 256;
constexpr int kBatchStreamThreads = 128;
constexpr int kBatchStreamMaxT = 4;

struct BatchGrid {
  int op;             // 0 jacobi-2d, 1 poisson-2d, 2 gradient-2d
  int n, steps, T, bx, eidx;
  int ntx, nty, rpbx, rpby;  // stream mode: nty = y segments
  int zseg;                  // stream mode: rows per segment
  int chunks;
  int cnt_off;        // this grid's first chunk counter
  int64_t sy;
  float* buf[2];
  const float* aux;
  OpArgs op_args;
  uint64_t wait_ns;   // limit of a dependency wait (2 s unless the host sets it)
  int hold;           // test hook: 1 = chunks >= 1 wait for a count never reached
};

constexpr uint64_t kBatchWaitNs = 2000000000ull;
constexpr unsigned kBatchMaxPolls = 1u << 26;  // a second bound, should the timer stall

__device__ __forceinline__ uint64_t batch_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <class Op>
__device__ __forceinline__ void batch_tile(const StepParams& p, int eidx, int txi, int tyi, int bx,
                                           float* smem) {
  const int by = kBatchThreads / bx;
  const int tx = threadIdx.x % bx, ty = threadIdx.x / bx;
  switch (eidx) {
    case 0: tile_body<Op, 1, 1, kLoadCg>(p, txi, tyi, 0, bx, by, 1, tx, ty, 0, smem); break;
    case 1: tile_body<Op, 2, 1, kLoadCg>(p, txi, tyi, 0, bx, by, 1, tx, ty, 0, smem); break;
    default: tile_body<Op, 4, 1, kLoadCg>(p, txi, tyi, 0, bx, by, 1, tx, ty, 0, smem); break;
  }
}

__global__ void __launch_bounds__(kBatchThreads) batch_kernel(const BatchGrid* __restrict__ grids,
                                                              const int4* __restrict__ items,
                                                              int nitems, int* next, int* counters,
                                                              int* err) {
  extern __shared__ float smem[];
  __shared__ int s_item, s_ok;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(next, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= nitems) break;
    const int4 w = items[it];
    const BatchGrid& g = grids[w.x];
    if (threadIdx.x == 0) {
      int ok = *(volatile int*)err == 0;
      if (ok && w.y > 0) {
        const int need = g.ntx * g.nty + g.hold;
        volatile int* c = counters + g.cnt_off + w.y - 1;
        const uint64_t t0 = batch_ns();
        unsigned i = 0;
        while (*c < need) {
          if (*(volatile int*)err != 0) {
            ok = 0;
            break;
          }
          if (((++i & 63) == 0 && batch_ns() - t0 > g.wait_ns) || i >= kBatchMaxPolls) {
            atomicOr(err, 2);
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
        __threadfence();  // acquire: the previous chunk's writes are visible
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) break;
    StepParams p{};
    p.in[0] = g.buf[w.y & 1];
    p.out[0] = g.buf[(w.y + 1) & 1];
    p.aux[0] = g.aux;
    p.L.n0 = g.n;
    p.L.n1 = g.n;
    p.L.n2 = 1;
    p.L.sy = g.sy;
    p.L.sz = g.sy * g.n;
    p.rpb[0] = g.rpbx;
    p.rpb[1] = g.rpby;
    p.rpb[2] = 1;
    p.T = g.T;
    p.steps = g.steps;
    p.base_step = w.y * g.T;
    p.phase_limit = 0;
    p.op = g.op_args;
    const int tyi = w.z / g.ntx, txi = w.z - tyi * g.ntx;
    switch (g.op) {
      case 0: batch_tile<OpJacobi2D>(p, g.eidx, txi, tyi, g.bx, smem); break;
      case 1: batch_tile<OpPoisson2D>(p, g.eidx, txi, tyi, g.bx, smem); break;
      default: batch_tile<OpGradient2D>(p, g.eidx, txi, tyi, g.bx, smem); break;
    }
    __threadfence();  // release: this thread's tile writes before the count
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(counters + g.cnt_off + w.y, 1);
  }
}

template <class Op>
__device__ __forceinline__ void batch_stream_unit(const Stream2dParams& p, int T, int strip,
                                                  int seg) {
  switch (T) {
    case 1: stream2d_body<Op, 1, kLoadCg>(p, strip, seg); break;
    case 2: stream2d_body<Op, 2, kLoadCg>(p, strip, seg); break;
    case 3: stream2d_body<Op, 3, kLoadCg>(p, strip, seg); break;
    default: stream2d_body<Op, 4, kLoadCg>(p, strip, seg); break;
  }
}

__global__ void __launch_bounds__(kBatchStreamThreads)
    batch_stream_kernel(const BatchGrid* __restrict__ grids, const int4* __restrict__ items,
                        int nitems, int* next, int* counters, int* err) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(next, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= nitems) break;
    const int4 w = items[it];
    const BatchGrid& g = grids[w.x];
    int ok = 1;
    if (lane == 0) {
      ok = *(volatile int*)err == 0;
      if (ok && w.y > 0) {
        const int need = g.ntx * g.nty + g.hold;
        volatile int* c = counters + g.cnt_off + w.y - 1;
        const uint64_t t0 = batch_ns();
        unsigned i = 0;
        while (*c < need) {
          if (*(volatile int*)err != 0) {
            ok = 0;
            break;
          }
          if (((++i & 63) == 0 && batch_ns() - t0 > g.wait_ns) || i >= kBatchMaxPolls) {
            atomicOr(err, 2);
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
      }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (!ok) break;
    __threadfence();  // acquire: the previous chunk's writes are visible to every lane
    Stream2dParams p{};
    p.in = g.buf[w.y & 1];
    p.out = g.buf[(w.y + 1) & 1];
    p.aux = g.aux;
    p.L.n0 = g.n;
    p.L.n1 = g.n;
    p.L.n2 = 1;
    p.L.sy = g.sy;
    p.L.sz = g.sy * g.n;
    p.ntx = g.ntx;
    p.nseg = g.nty;
    p.zseg = g.zseg;
    p.base_step = w.y * g.T;
    p.op = g.op_args;
    const int Tl = min(g.T, g.steps - w.y * g.T);  // the last chunk may be shallower
    const int seg = w.z / g.ntx, strip = w.z - seg * g.ntx;
    switch (g.op) {
      case 0: batch_stream_unit<OpJacobi2D>(p, Tl, strip, seg); break;
      case 1: batch_stream_unit<OpPoisson2D>(p, Tl, strip, seg); break;
      default: batch_stream_unit<OpGradient2D>(p, Tl, strip, seg); break;
    }
    __threadfence();  // release: this lane's writes before the count
    __syncwarp();
    if (lane == 0) atomicAdd(counters + g.cnt_off + w.y, 1);
  }
}

}  // namespace ots

struct ots_batch {
  int device = 0;
  int ngrids = 0;
  std::vector<ots_params> prm;
  std::vector<ots::BatchGrid> grids;  // host copy (device pointers inside)
  ots::BatchGrid* d_grids = nullptr;
  int4* d_items = nullptr;
  int nitems = 0;
  int* d_counters = nullptr;  // counters, then next, then err
  int ncounters = 0;
  float* pool = nullptr;
  size_t smem = 0;
  int ctas = 0;
  int64_t updates = 0;
  bool stream_mode = false;  // items are warps of the y-streamed 2D kernel
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<int> result_buf;  // per grid: buffer holding the last run's result
};

namespace {

ots_status bfail(ots_status s, const char* msg) {
  ots_set_last_error(msg);
  return s;
}

ots_status bcuda(cudaError_t e, const char* what) {
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  ots_set_last_error(buf);
  return e == cudaErrorMemoryAllocation ? OTS_ERR_OUT_OF_MEMORY : OTS_ERR_CUDA;
}

#define B_CUDA(call, what)                      \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) return bcuda(e_, what); \
  } while (0)

void free_batch(ots_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  cudaFree(b->d_grids);
  cudaFree(b->d_items);
  cudaFree(b->d_counters);
  cudaFree(b->pool);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

ots_status enqueue_batch(ots_batch* b) {
  const int nc = b->ncounters;
  B_CUDA(cudaMemsetAsync(b->d_counters, 0, (size_t)(nc + 2) * sizeof(int), b->stream),
         "reset counters");
  if (b->stream_mode)
    ots::batch_stream_kernel<<<b->ctas, ots::kBatchStreamThreads, 0, b->stream>>>(
        b->d_grids, b->d_items, b->nitems, b->d_counters + nc, b->d_counters,
        b->d_counters + nc + 1);
  else
    ots::batch_kernel<<<b->ctas, ots::kBatchThreads, b->smem, b->stream>>>(
        b->d_grids, b->d_items, b->nitems, b->d_counters + nc, b->d_counters,
        b->d_counters + nc + 1);
  B_CUDA(cudaGetLastError(), "batch kernel launch");
  return OTS_OK;
}

}  // namespace

extern "C" {

ots_status ots_batch_create(const ots_params* grids, int32_t n, int32_t device, ots_batch** out) {
  if (!grids || n < 1 || !out) return bfail(OTS_ERR_INVALID_ARGUMENT, "bad batch arguments");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return bfail(OTS_ERR_NO_DEVICE, "no CUDA device visible");
  }
  if (device < 0 || device >= ndev) return bfail(OTS_ERR_INVALID_ARGUMENT, "bad device");
  B_CUDA(cudaSetDevice(device), "cudaSetDevice");
  ots_batch* b = new ots_batch();
  b->device = device;
  b->ngrids = n;
  b->prm.assign(grids, grids + n);
  // validate and lay out
  size_t floats = 0;
  std::vector<size_t> off(n);
  int cnt = 0;
  b->stream_mode = grids[0].kernel == OTS_KERNEL_STREAM;
  for (int i = 0; i < n; ++i) {
    const ots_params& p = grids[i];
    ots::BatchGrid g{};
    if ((p.kernel == OTS_KERNEL_STREAM) != b->stream_mode) {
      free_batch(b);
      return bfail(OTS_ERR_UNSUPPORTED,
                   "batched grids must all use the stream kernel or all the tile kernel");
    }
    switch (p.stencil) {
      case OTS_JACOBI_2D: g.op = 0; break;
      case OTS_POISSON_2D: g.op = 1; break;
      case OTS_GRADIENT_2D: g.op = 2; break;
      default:
        free_batch(b);
        return bfail(OTS_ERR_UNSUPPORTED, "batched grids must be jacobi-2d, poisson-2d or gradient-2d");
    }
    if (p.problem_size < 1 || p.time_steps < 0 || p.time_tile < 1 || p.time_tile > 8) {
      free_batch(b);
      return bfail(OTS_ERR_INVALID_ARGUMENT, "batched grid: need n >= 1, steps >= 0, 1 <= T <= 8");
    }
    g.n = p.problem_size;
    g.steps = p.time_steps;
    g.T = p.time_tile;
    if (b->stream_mode) {
      if (g.T > ots::kBatchStreamMaxT) {
        free_batch(b);
        return bfail(OTS_ERR_UNSUPPORTED, "batched stream grid: T must be 1..4");
      }
      if (g.op == 1 && p.variant == OTS_VARIANT_REF) {
        free_batch(b);
        return bfail(OTS_ERR_UNSUPPORTED, "batched stream grid: poisson-2d baseline variant only");
      }
      // strips of 128 cells with a 4-cell halo (T <= 4); block_y > 1 = rows per segment
      g.rpbx = ots::kStream2dWidth - 2 * ots::stream2d_halo(ots::kBatchStreamMaxT);
      g.zseg = std::min(g.n, p.block_y > 1 ? p.block_y : 64);
      g.rpby = g.zseg;
      g.ntx = (g.n + g.rpbx - 1) / g.rpbx;
      g.nty = (g.n + g.zseg - 1) / g.zseg;
      g.bx = 32;
      g.eidx = 0;
    } else {
      if (!(p.block_x == 16 || p.block_x == 32 || p.block_x == 64)) {
        free_batch(b);
        return bfail(OTS_ERR_UNSUPPORTED,
                     "batched grid: block x must be 16, 32 or 64 (256 threads)");
      }
      const int E = p.elements_per_thread;
      g.eidx = E == 1 ? 0 : E == 2 ? 1 : E == 4 ? 2 : -1;
      if (g.eidx < 0) {
        free_batch(b);
        return bfail(OTS_ERR_UNSUPPORTED, "batched grid: E must be 1, 2 or 4");
      }
      g.bx = p.block_x;
      const int by = ots::kBatchThreads / g.bx;
      g.rpbx = g.bx - 2 * (g.T - 1);
      g.rpby = by * E - 2 * (g.T - 1);
      if (g.rpbx < 1 || g.rpby < 1) {
        free_batch(b);
        return bfail(OTS_ERR_INVALID_GEOMETRY, "batched grid: T too deep for its block");
      }
      g.ntx = (g.n + g.rpbx - 1) / g.rpbx;
      g.nty = (g.n + g.rpby - 1) / g.rpby;
    }
    g.chunks = g.steps > 0 ? (g.steps + g.T - 1) / g.T : 0;
    g.cnt_off = cnt;
    cnt += std::max(1, g.chunks);
    g.sy = (g.n + 31) / 32 * 32;
    g.op_args.variant = OTS_VARIANT_BASELINE;
    g.op_args.coef = g.op == 0 ? (p.coef != 0.0f ? p.coef : 1.0f / 5.0f) : p.coef;
    const double h = g.n > 1 ? 1.0 / (double)(g.n - 1) : 1.0;
    g.op_args.h2 = p.h2 != 0.0f ? p.h2 : (float)(h * h);
    g.wait_ns = ots::kBatchWaitNs;
    g.hold = 0;
    off[i] = floats;
    floats += (size_t)(g.op == 1 ? 3 : 2) * g.sy * g.n;
    b->updates += (int64_t)g.n * g.n * g.steps;
    b->grids.push_back(g);
  }
  b->ncounters = cnt;
  b->result_buf.assign(n, 0);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  if (e == cudaSuccess) e = cudaMalloc(&b->pool, std::max<size_t>(1, floats) * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(b->pool, 0, std::max<size_t>(1, floats) * sizeof(float));
  if (e != cudaSuccess) {
    ots_status s = bcuda(e, "batch allocation");
    free_batch(b);
    return s;
  }
  for (int i = 0; i < n; ++i) {
    ots::BatchGrid& g = b->grids[i];
    const size_t f = (size_t)g.sy * g.n;
    g.buf[0] = b->pool + off[i];
    g.buf[1] = b->pool + off[i] + f;
    g.aux = g.op == 1 ? b->pool + off[i] + 2 * f : nullptr;
  }
  // work queue in rounds of chunks; within a round the grids go stencil by
  // stencil, so the warps dequeued together mostly run the same unrolled
  // pipeline (the instruction cache holds one stencil's code, not three).
  // Every item waits only for its own grid's previous round, which lies
  // wholly earlier in the queue, whatever the order inside a round.
  std::vector<int4> items;
  int maxc = 0;
  for (auto& g : b->grids) maxc = std::max(maxc, g.chunks);
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int c) { return b->grids[a].op < b->grids[c].op; });
  for (int r = 0; r < maxc; ++r)
    for (int i : order)
      if (b->grids[i].chunks > r)
        for (int t = 0; t < b->grids[i].ntx * b->grids[i].nty; ++t) items.push_back(make_int4(i, r, t, 0));
  b->nitems = (int)items.size();
  // shared bytes: the largest tile of the menu (block 256 threads, E <= 4)
  size_t smem = 0;
  if (!b->stream_mode)
    for (auto& g : b->grids) {
      const int by = ots::kBatchThreads / g.bx;
      const int E = g.eidx == 0 ? 1 : g.eidx == 1 ? 2 : 4;
      smem = std::max(smem, (size_t)2 * (g.bx + 2) * (by * E + 2) * sizeof(float));
    }
  b->smem = smem;
  int per_sm = 1, sms = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (b->stream_mode) {
    // persistent warps: every resident slot, at most one warp per item
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ots::batch_stream_kernel,
                                                  ots::kBatchStreamThreads, 0);
    const int wpc = ots::kBatchStreamThreads / 32;
    b->ctas = std::max(1, std::min(sms * std::max(1, per_sm), (std::max(1, b->nitems) + wpc - 1) / wpc));
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ots::batch_kernel, ots::kBatchThreads,
                                                  smem);
    b->ctas = std::max(1, std::min(sms * std::max(1, per_sm), std::max(1, b->nitems)));
  }
  e = cudaMalloc(&b->d_grids, n * sizeof(ots::BatchGrid));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_grids, b->grids.data(), n * sizeof(ots::BatchGrid), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_items, std::max<size_t>(1, items.size()) * sizeof(int4));
  if (e == cudaSuccess && !items.empty())
    e = cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_counters, (size_t)(cnt + 2) * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->d_counters, 0, (size_t)(cnt + 2) * sizeof(int));
  if (e != cudaSuccess) {
    ots_status s = bcuda(e, "batch setup");
    free_batch(b);
    return s;
  }
  // capture reset + launch once
  e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    ots_status s = enqueue_batch(b);
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &b->graph);
    if (s != OTS_OK) {
      free_batch(b);
      return s;
    }
    e = e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) {
    ots_status s = bcuda(e, "batch graph");
    free_batch(b);
    return s;
  }
  *out = b;
  return OTS_OK;
}

void ots_batch_destroy(ots_batch* b) { free_batch(b); }

static ots_status upload_grids(ots_batch* b) {
  B_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
  B_CUDA(cudaStreamSynchronize(b->stream), "synchronize");
  B_CUDA(cudaMemcpy(b->d_grids, b->grids.data(), b->ngrids * sizeof(ots::BatchGrid),
                    cudaMemcpyHostToDevice),
         "grid table upload");
  return OTS_OK;
}

ots_status ots_batch_set_wait_limit(ots_batch* b, double seconds) {
  if (!b) return bfail(OTS_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (!(seconds > 0.0 && seconds <= 60.0))
    return bfail(OTS_ERR_INVALID_ARGUMENT, "wait limit must be in (0, 60] seconds");
  for (auto& g : b->grids) g.wait_ns = (uint64_t)(seconds * 1e9);
  return upload_grids(b);
}

ots_status ots_batch_debug_hold(ots_batch* b, int32_t grid) {
  if (!b) return bfail(OTS_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (grid >= b->ngrids) return bfail(OTS_ERR_INVALID_ARGUMENT, "bad grid index");
  for (int i = 0; i < b->ngrids; ++i) b->grids[i].hold = (i == grid) ? 1 : 0;
  return upload_grids(b);
}

ots_status ots_batch_info(const ots_batch* b, int64_t* updates, int32_t* items, int32_t* ctas) {
  if (!b) return bfail(OTS_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (updates) *updates = b->updates;
  if (items) *items = b->nitems;
  if (ctas) *ctas = b->ctas;
  return OTS_OK;
}

static ots_status batch_copy(ots_batch* b, int32_t gi, float* host, const float* chost, int which,
                             bool up) {
  if (!b || gi < 0 || gi >= b->ngrids) return bfail(OTS_ERR_INVALID_ARGUMENT, "bad grid index");
  B_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
  const ots::BatchGrid& g = b->grids[gi];
  float* dev = which == 2 ? const_cast<float*>(g.aux) : g.buf[which];
  if (!dev) return bfail(OTS_ERR_INVALID_ARGUMENT, "this grid has no aux field");
  if (up)
    B_CUDA(cudaMemcpy2DAsync(dev, g.sy * sizeof(float), chost, g.n * sizeof(float),
                             g.n * sizeof(float), g.n, cudaMemcpyHostToDevice, b->stream),
           "batch upload");
  else
    B_CUDA(cudaMemcpy2DAsync(host, g.n * sizeof(float), dev, g.sy * sizeof(float),
                             g.n * sizeof(float), g.n, cudaMemcpyDeviceToHost, b->stream),
           "batch download");
  B_CUDA(cudaStreamSynchronize(b->stream), "batch copy");
  return OTS_OK;
}

ots_status ots_batch_upload(ots_batch* b, int32_t grid, const float* state, const float* aux) {
  if (!state) return bfail(OTS_ERR_INVALID_ARGUMENT, "state is NULL");
  ots_status s = batch_copy(b, grid, nullptr, state, 0, true);
  if (s == OTS_OK && b->grids[grid].aux) {
    if (!aux) return bfail(OTS_ERR_INVALID_ARGUMENT, "this grid needs its aux field");
    s = batch_copy(b, grid, nullptr, aux, 2, true);
  }
  return s;
}

ots_status ots_batch_download(ots_batch* b, int32_t grid, float* state) {
  if (!state) return bfail(OTS_ERR_INVALID_ARGUMENT, "state is NULL");
  if (!b || grid < 0 || grid >= b->ngrids) return bfail(OTS_ERR_INVALID_ARGUMENT, "bad grid index");
  return batch_copy(b, grid, state, nullptr, b->result_buf[grid], false);
}

ots_status ots_batch_run(ots_batch* b, ots_timing* timing) {
  if (!b) return bfail(OTS_ERR_INVALID_ARGUMENT, "batch is NULL");
  B_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
  B_CUDA(cudaEventRecord(b->ev0, b->stream), "event");
  B_CUDA(cudaGraphLaunch(b->exec, b->stream), "graph launch");
  B_CUDA(cudaEventRecord(b->ev1, b->stream), "event");
  B_CUDA(cudaEventSynchronize(b->ev1), "batch execution");
  int err = 0;
  B_CUDA(cudaMemcpy(&err, b->d_counters + b->ncounters + 1, sizeof(int), cudaMemcpyDeviceToHost),
         "read error word");
  if (err) return bfail(OTS_ERR_TIMEOUT, "a bounded wait for a previous chunk gave up");
  for (int i = 0; i < b->ngrids; ++i) b->result_buf[i] = b->grids[i].chunks & 1;
  if (timing) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    timing->event_ms = ms;
    timing->wall_s = ms * 1e-3;
    timing->launches = 1;
    timing->steps = 0;
  }
  return OTS_OK;
}

ots_status ots_batch_stream(const ots_batch* b, void** stream) {
  if (!b || !stream) return bfail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  *stream = b->stream;
  return OTS_OK;
}

// Enqueue the captured graph without waiting (timed loops).
ots_status ots_batch_run_async(ots_batch* b) {
  if (!b) return bfail(OTS_ERR_INVALID_ARGUMENT, "batch is NULL");
  B_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
  B_CUDA(cudaGraphLaunch(b->exec, b->stream), "graph launch");
  for (int i = 0; i < b->ngrids; ++i) b->result_buf[i] = b->grids[i].chunks & 1;
  return OTS_OK;
}

// The comparator: the same grids one after another on one stream, the way
// separate runner processes would issue them -- OTS_KERNEL_PLAIN, one launch
// per time step, or OTS_KERNEL_TILE, one overlapped-tile launch per T steps
// with the grid's own (T, block, E).
ots_status ots_batch_run_sequential(ots_batch* b, int32_t kernel, ots_timing* timing) {
  if (!b) return bfail(OTS_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (kernel != OTS_KERNEL_PLAIN && kernel != OTS_KERNEL_TILE && kernel != OTS_KERNEL_STREAM)
    return bfail(OTS_ERR_INVALID_ARGUMENT, "sequential kernel must be PLAIN, TILE or STREAM");
  if ((kernel == OTS_KERNEL_STREAM) != b->stream_mode && kernel != OTS_KERNEL_PLAIN)
    return bfail(OTS_ERR_INVALID_ARGUMENT,
                 "sequential TILE / STREAM must match the batch's kernel family");
  B_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
  static const int kStencil[3] = {OTS_JACOBI_2D, OTS_POISSON_2D, OTS_GRADIENT_2D};
  int launches = 0;
  B_CUDA(cudaEventRecord(b->ev0, b->stream), "event");
  for (int i = 0; i < b->ngrids; ++i) {
    const ots::BatchGrid& g = b->grids[i];
    const ots::StencilKernels& K = ots::kernels_for(kStencil[g.op]);
    ots::StepParams sp{};
    sp.aux[0] = g.aux;
    sp.L.n0 = g.n;
    sp.L.n1 = g.n;
    sp.L.n2 = 1;
    sp.L.sy = g.sy;
    sp.L.sz = g.sy * g.n;
    sp.steps = g.steps;
    sp.op = g.op_args;
    int cur = 0;
    if (kernel == OTS_KERNEL_PLAIN) {
      const dim3 blk(32, 8, 1), grd((g.n + 31) / 32, (g.n + 7) / 8, 1);
      sp.T = 1;
      sp.rpb[0] = sp.rpb[1] = sp.rpb[2] = 1;
      for (int t = 0; t < g.steps; ++t) {
        sp.in[0] = g.buf[cur];
        sp.out[0] = g.buf[cur ^ 1];
        sp.base_step = t;
        B_CUDA(K.plain(sp, grd, blk, 0, b->stream), "plain launch");
        cur ^= 1;
        ++launches;
      }
    } else if (kernel == OTS_KERNEL_STREAM) {
      // the same strips, one y-streamed launch per chunk, with the segment
      // length a grid run on its own gets (more, shorter segments than in
      // the batch, where the other grids fill the GPU)
      int blocks = 1, sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
      if (!K.stream2d_occ[g.T] || K.stream2d_occ[g.T](&blocks) != cudaSuccess || blocks < 1)
        blocks = 1;
      ots::Stream2dParams s2{};
      s2.aux = g.aux;
      s2.L = sp.L;
      s2.ntx = g.ntx;
      s2.zseg = ots::stream2d_zseg(g.n, g.T, g.ntx, sms, blocks * (ots::kStream2dThreads / 32));
      s2.nseg = (g.n + s2.zseg - 1) / s2.zseg;
      s2.op = g.op_args;
      const int wpc = ots::kStream2dThreads / 32;
      const dim3 grd((g.ntx * s2.nseg + wpc - 1) / wpc);
      for (int c = 0; c < g.chunks; ++c) {
        const int Tl = std::min(g.T, g.steps - c * g.T);
        s2.in = g.buf[cur];
        s2.out = g.buf[cur ^ 1];
        s2.base_step = c * g.T;
        B_CUDA(K.stream2d[Tl](s2, grd, b->stream), "stream launch");
        cur ^= 1;
        ++launches;
      }
    } else {
      const int E = g.eidx == 0 ? 1 : g.eidx == 1 ? 2 : 4;
      const int by = ots::kBatchThreads / g.bx;
      const size_t smem = (size_t)2 * (g.bx + 2) * (by * E + 2) * sizeof(float);
      sp.T = g.T;
      sp.rpb[0] = g.rpbx;
      sp.rpb[1] = g.rpby;
      sp.rpb[2] = 1;
      for (int c = 0; c < g.chunks; ++c) {
        sp.in[0] = g.buf[cur];
        sp.out[0] = g.buf[cur ^ 1];
        sp.base_step = c * g.T;
        B_CUDA(K.tile[1][E](sp, dim3(g.ntx, g.nty, 1), dim3(g.bx, by, 1), smem, b->stream),
               "tile launch");
        cur ^= 1;
        ++launches;
      }
    }
    b->result_buf[i] = cur;
  }
  B_CUDA(cudaEventRecord(b->ev1, b->stream), "event");
  B_CUDA(cudaEventSynchronize(b->ev1), "sequential execution");
  if (timing) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    timing->event_ms = ms;
    timing->wall_s = ms * 1e-3;
    timing->launches = launches;
    timing->steps = 0;
  }
  return OTS_OK;
}

}  // extern "C"
