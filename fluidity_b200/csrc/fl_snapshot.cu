// Asynchronous device-to-host snapshots of a context's particle state.
//
// The role of the reference's CudaLiquidSnapshotQueue3D
// (native/include/fluidity/host/cuda_liquid_snapshot_3d.h:56-110,
// native/cuda/liquid_snapshot_3d_host.cc:148-380): two fixed reservations, each
// with a private non-blocking stream and two timing events; tickets holding a
// never-reused reservation number and the source epoch; Free -> Pending ->
// Ready -> Writer -> Free slots; nonblocking Poll, Finish with validation and a
// last valid host state; CUDA failures poison the queue.
//
// B200 layout of the same behaviour:
//  * The source is the context's current particle buffer, read in place (no
//    device staging copy). The copy's end is recorded as that buffer's fence,
//    and every write into the buffer waits on it, so the steps that follow
//    overlap the copy and only a write into the copied buffer is ordered
//    after it. A second copy of the same buffer waits for the first, so the
//    fence always covers both.
//  * Validation runs on the device, in a streaming kernel on the slot's
//    stream: every value finite and every position inside the block lattice
//    (the sort's rule). It writes a control record (count, epoch, failure
//    counts, first failing particle) that is copied behind the particles;
//    Finish checks those 64 bytes instead of scanning 15 x N floats.
//  * Three pinned host buffers, reference-counted between the two slots and
//    the last valid snapshot: Finish publishes the slot's buffer as the last
//    valid state without a host copy, and a Begin always finds a free buffer.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <cstring>
#include <new>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"
#include "fl_kernels.h"

namespace fl {
namespace {

struct SnapshotControl {
  unsigned long long count;
  unsigned long long generation;
  unsigned long long frame_ordinal;
  double time;
  unsigned long long nonfinite;      // particles with a non-finite value
  unsigned long long outside;        // finite particles outside the block lattice
  unsigned long long first_bad_not;  // ~(first failing particle), 0 if none
  unsigned long long buffer;         // the context buffer that was copied
};
static_assert(sizeof(SnapshotControl) == 64, "control record is one 64-byte line");

constexpr int kCheckThreads = 256;
constexpr int kCheckBlocksPerSm = 8;

// One pass over the state: 15 coalesced loads per particle, all issued before
// any test. Failure counts are summed per warp and added with one atomic each;
// the first failing index is kept as its bitwise complement under atomicMax
// (the record is zeroed beforehand, and ~i orders the smallest index highest).
__global__ void __launch_bounds__(kCheckThreads)
    k_snapshot_check(const float* __restrict__ base, size_t pcap, unsigned long long count, GridView g,
                     SnapshotControl* ctl, unsigned long long generation, unsigned long long frame, double time,
                     int buffer) {
  unsigned long long nonfinite = 0, outside = 0, first_not = 0;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    float v[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) v[k] = __ldg(base + (size_t)k * pcap + i);
    bool fin = true;
#pragma unroll
    for (int k = 0; k < 15; ++k) fin = fin && isfinite(v[k]);
    bool inside = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float X = lattice_coord(g, v[d], d);
      const bool ok = fin && fabsf(X) < 1.0e9f;
      const int b = ok ? floor_div8(__float2int_rd(X)) - g.blo[d] : -1;
      inside = inside && b >= 0 && b < g.bdim[d];
    }
    if (!fin)
      ++nonfinite;
    else if (!inside)
      ++outside;
    if (!(fin && inside)) first_not = max(first_not, ~i);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nonfinite += __shfl_xor_sync(0xffffffffu, nonfinite, o);
    outside += __shfl_xor_sync(0xffffffffu, outside, o);
    first_not = max(first_not, __shfl_xor_sync(0xffffffffu, first_not, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (nonfinite) atomicAdd(&ctl->nonfinite, nonfinite);
    if (outside) atomicAdd(&ctl->outside, outside);
    if (first_not) atomicMax(&ctl->first_bad_not, first_not);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->count = count;
    ctl->generation = generation;
    ctl->frame_ordinal = frame;
    ctl->time = time;
    ctl->buffer = (unsigned long long)buffer;
  }
}

enum SlotState { kFree, kPending, kReady, kWriter };

struct HostBuffer {
  float* data = nullptr;             // 15 x pcap floats, compacted to 15 x count by the copy
  SnapshotControl* ctl = nullptr;    // behind the floats, 64-byte aligned
  int refs = 0;                      // slot holding it + last valid snapshot
};

struct Slot {
  SlotState state = kFree;
  bool canceled = false;
  uint64_t reservation = 0;
  fl_epoch epoch{};
  uint64_t count = 0;
  int buffer = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t src = nullptr;                 // the producer's position in its stream
  cudaEvent_t ev[2] = {nullptr, nullptr};    // around the check and the copy
  float copy_ms = 0.0f;
};

bool same_epoch(const fl_epoch& a, const fl_epoch& b) {
  return a.generation == b.generation && a.frame_ordinal == b.frame_ordinal &&
         std::memcmp(&a.time, &b.time, sizeof(double)) == 0;
}

}  // namespace
}  // namespace fl

using namespace fl;

struct fl_snapshot_queue {
  fl_context* ctx = nullptr;
  int device = 0;
  int sms = 0;
  size_t pcap = 0;
  SnapshotControl* dctl = nullptr;  // device control records, one per slot
  HostBuffer buf[3];
  Slot slot[2];
  int last = -1;  // buffer of the last valid snapshot
  fl_epoch last_epoch{};
  uint64_t last_count = 0;
  float last_copy_ms = 0.0f;
  uint64_t next_reservation = 1;
  bool poisoned = false;
};

namespace {

// CUDA failure: the queue is poisoned (every later call but destroy and
// release returns FL_INTERNAL), as the reference's RuntimeResult does.
int runtime(fl_snapshot_queue* q, cudaError_t e) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    q->poisoned = true;
  }
  return q->poisoned ? FL_INTERNAL : FL_OK;
}

Slot* find(fl_snapshot_queue* q, const fl_snapshot_ticket* t) {
  if (!q || !t || t->slot >= 2) return nullptr;
  Slot& s = q->slot[t->slot];
  if (s.state == kFree || s.reservation != t->reservation || !same_epoch(s.epoch, t->epoch)) return nullptr;
  return &s;
}

void free_slot(fl_snapshot_queue* q, Slot& s) {
  if (s.buffer >= 0) --q->buf[s.buffer].refs;
  s.buffer = -1;
  s.state = kFree;
  s.canceled = false;
}

// The copy has completed (its end event observed): timing, then Ready, or the
// deferred cancellation.
int completed(fl_snapshot_queue* q, Slot& s, int* progress) {
  int st = runtime(q, cudaEventElapsedTime(&s.copy_ms, s.ev[0], s.ev[1]));
  if (st != FL_OK) return st;
  if (s.canceled) {
    free_slot(q, s);
    *progress = FL_SNAPSHOT_CANCELED;
    return FL_OK;
  }
  s.state = kReady;
  *progress = FL_SNAPSHOT_READY;
  return FL_OK;
}

void view_of(const fl_snapshot_queue* q, int buffer, uint64_t count, const fl_epoch& e, float ms,
             fl_snapshot_view* out) {
  out->soa = q->buf[buffer].data;
  out->count = count;
  out->epoch = e;
  out->copy_ms = ms;
}

void release_all(fl_snapshot_queue* q) {
  for (Slot& s : q->slot) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.src) cudaEventDestroy(s.src);
    for (cudaEvent_t& e : s.ev)
      if (e) cudaEventDestroy(e);
    if (s.stream) cudaStreamDestroy(s.stream);
  }
  for (HostBuffer& b : q->buf)
    if (b.data) cudaFreeHost(b.data);
  if (q->dctl) cudaFree(q->dctl);
  cudaGetLastError();
}

}  // namespace

extern "C" {

int fl_snapshot_queue_create(fl_context* ctx, fl_snapshot_queue** out) {
  if (!ctx || !out) return FL_INVALID_ARGUMENT;
  *out = nullptr;
  SnapshotSource src{};
  context_snapshot_source(ctx, &src);
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return FL_INTERNAL;
  }
  if (dev != src.device) return FL_FAILED_PRECONDITION;
  if (src.pcap > (SIZE_MAX - 128) / (15 * sizeof(float))) return FL_RESOURCE_EXHAUSTED;
  fl_snapshot_queue* q = new (std::nothrow) fl_snapshot_queue();
  if (!q) return FL_RESOURCE_EXHAUSTED;
  q->ctx = ctx;
  q->device = dev;
  q->pcap = src.pcap;
  int st = FL_OK;
  const size_t floats_bytes = (15 * sizeof(float) * src.pcap + 63) / 64 * 64;
  for (HostBuffer& b : q->buf) {
    void* p = nullptr;
    const cudaError_t e = cudaMallocHost(&p, floats_bytes + sizeof(SnapshotControl));
    if (e != cudaSuccess) {
      cudaGetLastError();
      st = e == cudaErrorMemoryAllocation ? FL_RESOURCE_EXHAUSTED : FL_INTERNAL;
      break;
    }
    b.data = static_cast<float*>(p);
    b.ctl = reinterpret_cast<SnapshotControl*>(static_cast<char*>(p) + floats_bytes);
  }
  if (st == FL_OK && cudaMalloc(&q->dctl, 2 * sizeof(SnapshotControl)) != cudaSuccess) st = FL_RESOURCE_EXHAUSTED;
  for (int i = 0; i < 2 && st == FL_OK; ++i) {
    Slot& s = q->slot[i];
    if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.src, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&s.ev[0]) != cudaSuccess || cudaEventCreate(&s.ev[1]) != cudaSuccess)
      st = FL_INTERNAL;
  }
  if (st == FL_OK && cudaDeviceGetAttribute(&q->sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    st = FL_INTERNAL;
  if (st != FL_OK) {
    release_all(q);
    delete q;
    return st;
  }
  context_attach_snapshot_queue(ctx, +1);
  *out = q;
  return FL_OK;
}

int fl_snapshot_queue_destroy(fl_snapshot_queue* q) {
  if (!q) return FL_OK;
  release_all(q);
  context_attach_snapshot_queue(q->ctx, -1);
  delete q;
  return FL_OK;
}

int fl_snapshot_begin(fl_snapshot_queue* q, const fl_epoch* epoch, void* stream, fl_snapshot_ticket* ticket) {
  if (!q || !epoch || !ticket) return FL_INVALID_ARGUMENT;
  if (q->poisoned) return FL_INTERNAL;
  if (epoch->generation == 0) return FL_INVALID_ARGUMENT;
  int dev = -1;
  if (runtime(q, cudaGetDevice(&dev)) != FL_OK) return FL_INTERNAL;
  if (dev != q->device) return FL_FAILED_PRECONDITION;
  if (epoch->generation <= q->last_epoch.generation) return FL_FAILED_PRECONDITION;
  for (const Slot& s : q->slot)
    if (s.state != kFree && same_epoch(s.epoch, *epoch)) return FL_ALREADY_EXISTS;
  if (q->next_reservation == UINT64_MAX) return FL_OUT_OF_RANGE;
  int si = -1;
  for (int i = 0; i < 2 && si < 0; ++i)
    if (q->slot[i].state == kFree) si = i;
  if (si < 0) return FL_UNAVAILABLE;
  int bi = -1;
  for (int i = 0; i < 3 && bi < 0; ++i)
    if (q->buf[i].refs == 0) bi = i;
  if (bi < 0) return runtime(q, cudaErrorUnknown);  // two slots and the last valid hold at most two
  SnapshotSource src{};
  context_snapshot_source(q->ctx, &src);
  if (src.count > q->pcap) return runtime(q, cudaErrorUnknown);

  Slot& s = q->slot[si];
  s.state = kPending;
  s.canceled = false;
  s.reservation = q->next_reservation++;
  s.epoch = *epoch;
  s.count = src.count;
  s.buffer = bi;
  s.copy_ms = 0.0f;
  q->buf[bi].refs = 1;
  // From here the slot owns the copy even on failure (drained at destroy).
  const cudaStream_t prod = (cudaStream_t)stream;
  const cudaEvent_t fence = context_buffer_fence(q->ctx, src.buffer);
  SnapshotControl* dctl = q->dctl + si;
  HostBuffer& hb = q->buf[bi];
  if (runtime(q, cudaEventRecord(s.src, prod)) != FL_OK) return FL_INTERNAL;
  if (runtime(q, cudaStreamWaitEvent(s.stream, s.src, 0)) != FL_OK) return FL_INTERNAL;
  if (runtime(q, cudaStreamWaitEvent(s.stream, fence, 0)) != FL_OK) return FL_INTERNAL;
  if (runtime(q, cudaEventRecord(s.ev[0], s.stream)) != FL_OK) return FL_INTERNAL;
  if (runtime(q, cudaMemsetAsync(dctl, 0, sizeof(SnapshotControl), s.stream)) != FL_OK) return FL_INTERNAL;
  const unsigned long long need = (src.count + kCheckThreads - 1) / kCheckThreads;
  const unsigned long long cap = (unsigned long long)q->sms * kCheckBlocksPerSm;
  const unsigned grid = (unsigned)(need == 0 ? 1 : (need < cap ? need : cap));
  ++g_kernel_launches;
  k_snapshot_check<<<grid, kCheckThreads, 0, s.stream>>>(src.base, src.pcap, src.count, src.g, dctl,
                                                          epoch->generation, epoch->frame_ordinal, epoch->time,
                                                          src.buffer);
  if (runtime(q, cudaGetLastError()) != FL_OK) return FL_INTERNAL;
  for (int k = 0; k < 15 && src.count; ++k)
    if (runtime(q, cudaMemcpyAsync(hb.data + (size_t)k * src.count, src.base + (size_t)k * src.pcap,
                                   sizeof(float) * src.count, cudaMemcpyDeviceToHost, s.stream)) != FL_OK)
      return FL_INTERNAL;
  if (runtime(q, cudaMemcpyAsync(hb.ctl, dctl, sizeof(SnapshotControl), cudaMemcpyDeviceToHost, s.stream)) != FL_OK)
    return FL_INTERNAL;
  if (runtime(q, cudaEventRecord(s.ev[1], s.stream)) != FL_OK) return FL_INTERNAL;
  if (runtime(q, cudaEventRecord(fence, s.stream)) != FL_OK) return FL_INTERNAL;
  ticket->slot = (uint32_t)si;
  ticket->reservation = s.reservation;
  ticket->epoch = s.epoch;
  return FL_OK;
}

int fl_snapshot_poll(fl_snapshot_queue* q, const fl_snapshot_ticket* t, int* progress) {
  if (!progress) return FL_INVALID_ARGUMENT;
  Slot* s = find(q, t);
  if (!s) return FL_FAILED_PRECONDITION;
  if (q->poisoned) return FL_INTERNAL;
  if (s->state == kWriter) return FL_FAILED_PRECONDITION;
  if (s->state == kReady) {
    *progress = FL_SNAPSHOT_READY;
    return FL_OK;
  }
  const cudaError_t e = cudaEventQuery(s->ev[1]);
  if (e == cudaErrorNotReady) {
    if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
    *progress = FL_SNAPSHOT_PENDING;
    return FL_OK;
  }
  if (runtime(q, e) != FL_OK) return FL_INTERNAL;
  return completed(q, *s, progress);
}

int fl_snapshot_wait(fl_snapshot_queue* q, const fl_snapshot_ticket* t, int* progress) {
  if (!progress) return FL_INVALID_ARGUMENT;
  Slot* s = find(q, t);
  if (!s) return FL_FAILED_PRECONDITION;
  if (q->poisoned) return FL_INTERNAL;
  if (s->state == kWriter) return FL_FAILED_PRECONDITION;
  if (s->state == kReady) {
    *progress = FL_SNAPSHOT_READY;
    return FL_OK;
  }
  if (runtime(q, cudaEventSynchronize(s->ev[1])) != FL_OK) return FL_INTERNAL;
  return completed(q, *s, progress);
}

int fl_snapshot_finish(fl_snapshot_queue* q, const fl_snapshot_ticket* t, fl_snapshot_view* out) {
  if (!out) return FL_INVALID_ARGUMENT;
  Slot* s = find(q, t);
  if (!s) return FL_FAILED_PRECONDITION;
  if (q->poisoned) return FL_INTERNAL;
  const fl_epoch& e = s->epoch;
  if (s->state != kReady || s->canceled || e.generation <= q->last_epoch.generation ||
      e.frame_ordinal < q->last_epoch.frame_ordinal || e.time < q->last_epoch.time)
    return FL_FAILED_PRECONDITION;
  const SnapshotControl& c = *q->buf[s->buffer].ctl;
  const bool intact = c.count == s->count && c.generation == e.generation && c.frame_ordinal == e.frame_ordinal &&
                      std::memcmp(&c.time, &e.time, sizeof(double)) == 0;
  if (!intact || c.nonfinite != 0 || c.outside != 0) {
    q->poisoned = true;
    return FL_DATA_LOSS;
  }
  if (q->last >= 0) --q->buf[q->last].refs;
  q->last = s->buffer;
  ++q->buf[q->last].refs;
  q->last_epoch = e;
  q->last_count = s->count;
  q->last_copy_ms = s->copy_ms;
  s->state = kWriter;
  view_of(q, s->buffer, s->count, e, s->copy_ms, out);
  return FL_OK;
}

int fl_snapshot_release(fl_snapshot_queue* q, const fl_snapshot_ticket* t) {
  Slot* s = find(q, t);
  if (!s || s->state != kWriter) return FL_FAILED_PRECONDITION;
  free_slot(q, *s);
  return FL_OK;
}

int fl_snapshot_cancel(fl_snapshot_queue* q, const fl_snapshot_ticket* t) {
  Slot* s = find(q, t);
  if (!s || s->state == kWriter) return FL_FAILED_PRECONDITION;
  if (q->poisoned) return FL_INTERNAL;
  s->canceled = true;
  if (s->state == kReady) free_slot(q, *s);
  return FL_OK;
}

int fl_snapshot_last_valid(fl_snapshot_queue* q, fl_snapshot_view* out) {
  if (!q || !out) return FL_INVALID_ARGUMENT;
  if (q->last < 0) return FL_FAILED_PRECONDITION;
  view_of(q, q->last, q->last_count, q->last_epoch, q->last_copy_ms, out);
  return FL_OK;
}

}  // extern "C"
