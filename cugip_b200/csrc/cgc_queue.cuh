// Work queue and tile locks of the asynchronous (work-queue) schedule.
//
// Instead of global rounds separated by grid barriers, every CTA takes the
// next tile from a device-wide FIFO, visits it and queues the tiles the visit
// made active.  `pending` counts queued tiles plus tiles being visited, so it
// reaches 0 exactly when the phase has nothing left to do; whoever brings it
// to 0 raises `done`.
//
// Ticket queue: a taker draws a ticket with one atomicAdd on `head` and waits
// on that ticket's slot until a producer fills it (or `done` is raised); a
// producer draws a ticket on `tail` and fills its slot.  Tickets map to slots
// 33 ints apart, so waiting takers poll different cache lines, and every
// counter sits on its own line: nothing is polled where atomics are made.
// A tile is queued at most once at a time (its stamp equals the phase id
// while it is queued; taking it clears the stamp) and at most one ticket per
// CTA waits, so live tickets span fewer than cap slots and a slot is reused
// only after its previous entry was taken.
//
// Push-relabel visits additionally lock the tile: a visit holds the writer
// bit of its tile and one reader count on each face neighbour, so two face
// neighbours are never visited at the same time (the halo heights a visit
// reads stay exact and labels stay valid, as under the parity schedule).  No
// CTA ever waits for a lock: a tile that cannot be locked goes back into the
// queue.
#pragma once
#include "cgc_device.cuh"

namespace cgc {

constexpr int32_t LOCK_W = 0x40000000;
constexpr int QCTL_LINE = 32;                  // ints per counter line
enum QueueCtl { Q_HEAD = 0, Q_TAIL = 1, Q_PENDING = 2, Q_VISITS = 3, Q_DONE = 4, Q_NCTL = 5 };
constexpr int QCTL_INTS = Q_NCTL * QCTL_LINE;  // one control block
constexpr int QSLOT_STRIDE = 33;               // coprime to the ring capacity

// ring capacity for T tiles: room for every tile plus one waiting ticket per
// CTA, and coprime to the slot stride
inline int32_t queue_capacity(int32_t T) {
  int32_t cap = T + 4096;
  while (cap % 3 == 0 || cap % 11 == 0) ++cap;
  return cap;
}

struct WorkQueue {
  int32_t* ring;      // cap slots, -1 = empty
  int32_t cap;
  int32_t* ctl;       // QueueCtl counters, QCTL_LINE ints apart
  uint64_t limit_ns;  // bound of every wait
  __device__ int32_t* c(QueueCtl k) const { return ctl + k * QCTL_LINE; }
  __device__ volatile int32_t* slot(int ticket) const {
    return ring + (int)(((int64_t)ticket * QSLOT_STRIDE) % cap);
  }
};

__device__ __forceinline__ int ld_volatile(const int32_t* p) { return *(volatile const int32_t*)p; }

__device__ __forceinline__ uint64_t q_globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Appends t (its stamp already set by the caller).  Data written before the
// call is visible to whoever takes the entry.  Returns false on a timeout.
__device__ inline bool wq_push(const WorkQueue& q, int t) {
  atomicAdd(q.c(Q_PENDING), 1);
  __threadfence();
  volatile int32_t* s = q.slot(atomicAdd(q.c(Q_TAIL), 1));
  if (*s != -1) {  // the previous entry of this slot was taken but not yet cleared
    const uint64_t t0 = q_globaltimer_ns();
    while (*s != -1) {
      __nanosleep(32);
      if (q_globaltimer_ns() - t0 > q.limit_ns) return false;
    }
  }
  *s = t;
  return true;
}

// One unit of work finished (a visit, or a take that went back to the queue).
__device__ inline void wq_release(const WorkQueue& q) {
  __threadfence();
  if (atomicSub(q.c(Q_PENDING), 1) == 1) atomicExch(q.c(Q_DONE), 1);
}

// Waits for the next entry: a tile index, -1 once the phase is over (`done`
// or an error), -2 on a timeout.  The caller then owns one `pending` count.
__device__ inline int wq_take(const WorkQueue& q, const int32_t* err) {
  if (ld_volatile(q.c(Q_DONE)) || ld_volatile(err)) return -1;
  volatile int32_t* s = q.slot(atomicAdd(q.c(Q_HEAD), 1));
  int t = *s;
  if (t < 0) {
    const uint64_t t0 = q_globaltimer_ns();
    unsigned ns = 32;
    while ((t = *s) < 0) {
      if (ld_volatile(q.c(Q_DONE)) || ld_volatile(err)) return -1;
      if (q_globaltimer_ns() - t0 > q.limit_ns) return -2;
      __nanosleep(ns);
      if (ns < 1024) ns <<= 1;
    }
  }
  *s = -1;
  __threadfence();
  return t;
}

// Writer bit on t and a reader count on each face neighbour, or nothing.
__device__ inline bool tile_try_lock(const DevPool& P, int t) {
  if (atomicCAS(P.tlock + t, 0, LOCK_W) != 0) return false;
  int got = 0;
  bool ok = true;
  for (int d = 0; d < 6; ++d) {
    const int nt = __ldcg(P.nbr + d * P.T + t);
    if (nt < 0) continue;
    const int old = atomicAdd(P.tlock + nt, 1);
    got |= 1 << d;
    if (old & LOCK_W) { ok = false; break; }
  }
  if (!ok) {
    for (int d = 0; d < 6; ++d)
      if ((got >> d) & 1) atomicSub(P.tlock + __ldcg(P.nbr + d * P.T + t), 1);
    atomicAnd(P.tlock + t, ~LOCK_W);
  }
  __threadfence();
  return ok;
}

__device__ inline void tile_unlock(const DevPool& P, int t) {
  __threadfence();
  for (int d = 0; d < 6; ++d) {
    const int nt = __ldcg(P.nbr + d * P.T + t);
    if (nt >= 0) atomicSub(P.tlock + nt, 1);
  }
  atomicAnd(P.tlock + t, ~LOCK_W);
}

}  // namespace cgc
