// Device task queue for sharing search subtrees between warps.
//
// Replaces the reference's worker list (include/queue.cuh:17-56: a ticket
// ring of idle block ids plus a per-block mailbox that a donor fills while
// the idle block spins, mce/mce_utils.cuh:241-263,1063-1113).  There, an idle
// block waits on its own mailbox without a limit, and the kernel only ends
// when every block of the grid sits in the ring, so the whole grid must be
// resident.  Here the queue holds self-contained tasks - a root and one node
// of its search tree (P, X and the chosen set as bitmaps over the root's
// later neighbours) - so any warp can take any task, nobody waits for a
// particular warp, and termination is a single counter:
//   work = warps still in their root phase + tasks queued or running.
// A warp that has run out of roots takes tasks until work == 0.  Push and
// pop never block (a full queue means "keep the subtree"); the only wait is
// an idle warp polling, bounded by a no-progress time limit.
#pragma once

#include "common.cuh"

namespace mce {

struct QueueHdr {
  uint32_t head, tail;  // ring positions (wrap modulo 2^32)
  uint32_t work;        // see above
  uint32_t idle;        // warps polling for a task
  uint32_t epoch;       // bumped on every push and task completion
  uint32_t pushed;      // tasks pushed (statistics)
  uint32_t pad[26];
};

struct QueueView {
  QueueHdr *hdr = nullptr;
  uint32_t *seq = nullptr;           // cap entries
  unsigned long long *pay = nullptr; // cap x words
  uint32_t cap = 0;                  // power of two
  uint32_t words = 0;                // u64 words per task
};

__global__ void queue_init_kernel(QueueView q);

// Claim a slot and publish `words` task words held by the warp (lane k holds
// words k, k+32, ...; supplied by `get(k)`).  Returns false if full.
template <typename Get>
__device__ __forceinline__ bool q_push(const QueueView &q, Get get) {
  const uint32_t lane = lane_id();
  uint32_t pos = 0;
  int ok = 0;
  if (lane == 0) {
    pos = ld_volatile(&q.hdr->tail);
    for (int tries = 0; tries < 64; ++tries) {
      const uint32_t s = ld_acquire(&q.seq[pos & (q.cap - 1)]);
      const int32_t diff = (int32_t)(s - pos);
      if (diff == 0) {
        const uint32_t seen = atomicCAS(&q.hdr->tail, pos, pos + 1);
        if (seen == pos) {
          ok = 1;
          break;
        }
        pos = seen;
      } else if (diff < 0) {
        break;  // full
      } else {
        pos = ld_volatile(&q.hdr->tail);
      }
    }
    if (ok) {
      atomicAdd(&q.hdr->work, 1u);  // counted before anyone can take it
      atomicAdd(&q.hdr->pushed, 1u);
    }
  }
  ok = __shfl_sync(MCE_FULL, ok, 0);
  if (!ok) return false;
  pos = __shfl_sync(MCE_FULL, pos, 0);
  unsigned long long *dst = q.pay + (size_t)(pos & (q.cap - 1)) * q.words;
  for (uint32_t k = lane; k < q.words; k += 32) dst[k] = get(k);
  __syncwarp();
  if (lane == 0) {
    __threadfence();
    st_release(&q.seq[pos & (q.cap - 1)], pos + 1);
    atomicAdd(&q.hdr->epoch, 1u);
  }
  __syncwarp();
  return true;
}

// Take a task: on success `put(k, word)` receives every word (lane-strided).
template <typename Put>
__device__ __forceinline__ bool q_pop(const QueueView &q, Put put) {
  const uint32_t lane = lane_id();
  uint32_t pos = 0;
  int ok = 0;
  if (lane == 0) {
    pos = ld_volatile(&q.hdr->head);
    for (int tries = 0; tries < 64; ++tries) {
      const uint32_t s = ld_acquire(&q.seq[pos & (q.cap - 1)]);
      const int32_t diff = (int32_t)(s - (pos + 1));
      if (diff == 0) {
        const uint32_t seen = atomicCAS(&q.hdr->head, pos, pos + 1);
        if (seen == pos) {
          ok = 1;
          break;
        }
        pos = seen;
      } else if (diff < 0) {
        break;  // empty
      } else {
        pos = ld_volatile(&q.hdr->head);
      }
    }
    if (ok) __threadfence();
  }
  ok = __shfl_sync(MCE_FULL, ok, 0);
  if (!ok) return false;
  pos = __shfl_sync(MCE_FULL, pos, 0);
  const volatile unsigned long long *src = q.pay + (size_t)(pos & (q.cap - 1)) * q.words;
  for (uint32_t k = lane; k < q.words; k += 32) put(k, src[k]);
  __syncwarp();
  if (lane == 0) st_release(&q.seq[pos & (q.cap - 1)], pos + q.cap);  // slot free again
  __syncwarp();
  return true;
}

// Donate a child only while more warps are waiting than tasks are queued.
__device__ __forceinline__ bool q_wants(const QueueView &q) {
  if (!q.hdr) return false;
  const uint32_t idle = ld_volatile(&q.hdr->idle);
  if (idle == 0) return false;
  const uint32_t queued = ld_volatile(&q.hdr->tail) - ld_volatile(&q.hdr->head);
  return idle > queued;
}

}  // namespace mce
