// Contacts between annihilation partners and their deterministic greedy
// matching, shared by the single-instance and batched paths.
#pragma once
#include <algorithm>
#include <cstdlib>

#include "amk_internal.cuh"

namespace amk {
namespace {

struct Contact {
  uint32_t a, b;   // owner, partner (indices)
  uint64_t prio;   // (owner id << 32) | partner id
};

// Greedy matching by locally-dominant selection. Each round selects every
// live contact whose priority is the minimum at both endpoints (these are
// exactly the contacts the sequential greedy pass takes), then retires
// contacts touching a matched particle. At least one contact (the global
// minimum) is selected per round, so the loop ends within `m` rounds.
//
// Large contact sets run kMatchRounds rounds over the whole grid first (two
// kernels per round: min + retire, then select), with two `best` arrays used
// alternately so that a round's reset of the next round's array never races
// with its own minimum; the one-CTA kernel below then finishes whatever is
// left (nothing, for the sparse contact graphs of a trap), so the result is
// the same set in every case.
constexpr int kMatchRounds = 12;

struct MatchState {
  unsigned long long live[kMatchRounds];  // live contacts entering each round
};

// The number of contacts may live on the device (graph replays).
__device__ __forceinline__ long match_count(long m_cap, const unsigned long long* m_count) {
  return m_count ? static_cast<long>(min(static_cast<unsigned long long>(m_cap), *m_count)) : m_cap;
}

__global__ void match_init_kernel(const Contact* __restrict__ e, long m_cap, const unsigned long long* __restrict__ m_count,
                                  unsigned long long* best0, unsigned long long* best1, uint8_t* matched,
                                  uint8_t* live_e, MatchState* st, unsigned long long* result) {
  const long m = match_count(m_cap, m_count);
  const long tid = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  const long nth = static_cast<long>(gridDim.x) * blockDim.x;
  for (long k = tid; k < m; k += nth) {
    const Contact c = e[k];
    live_e[k] = 1;
    matched[c.a] = matched[c.b] = 0;
    best0[c.a] = best0[c.b] = ~0ull;
    best1[c.a] = best1[c.b] = ~0ull;
  }
  if (tid < kMatchRounds) st->live[tid] = 0;
  if (tid == 0) result[0] = result[1] = 0;
}

// Retires contacts touching a particle matched in an earlier round, takes the
// minimum priority at both endpoints of the rest (into `cur`) and clears the
// endpoints' entries of `next`, the array of the following round.
__global__ void match_min_kernel(const Contact* __restrict__ e, long m_cap, const unsigned long long* __restrict__ m_count,
                                 int round, unsigned long long* cur, unsigned long long* next,
                                 const uint8_t* __restrict__ matched, uint8_t* live_e, MatchState* st) {
  if (round > 0 && st->live[round - 1] == 0) return;
  const long m = match_count(m_cap, m_count);
  const long nth = static_cast<long>(gridDim.x) * blockDim.x;
  unsigned long long mine = 0;
  for (long k = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; k < m; k += nth) {
    if (!live_e[k]) continue;
    const Contact c = e[k];
    if (matched[c.a] || matched[c.b]) {
      live_e[k] = 0;
      continue;
    }
    atomicMin(&cur[c.a], c.prio);
    atomicMin(&cur[c.b], c.prio);
    next[c.a] = next[c.b] = ~0ull;
    ++mine;
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&st->live[round], mine);
}

__global__ void match_select_kernel(const Contact* __restrict__ e, long m_cap, const unsigned long long* __restrict__ m_count,
                                    int round, const unsigned long long* __restrict__ cur, uint8_t* matched,
                                    const uint8_t* __restrict__ live_e, uint8_t* alive, const MatchState* st,
                                    unsigned long long* result) {
  if (st->live[round] == 0) return;
  const long m = match_count(m_cap, m_count);
  const long nth = static_cast<long>(gridDim.x) * blockDim.x;
  unsigned long long marked = 0;
  for (long k = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; k < m; k += nth) {
    if (!live_e[k]) continue;
    const Contact c = e[k];
    if (cur[c.a] == c.prio && cur[c.b] == c.prio) {
      matched[c.a] = matched[c.b] = 1;
      alive[c.a] = alive[c.b] = 0;
      marked += 2;
    }
  }
  for (int o = 16; o > 0; o >>= 1) marked += __shfl_xor_sync(0xffffffffu, marked, o);
  if ((threadIdx.x & 31) == 0 && marked) atomicAdd(&result[0], marked);
}

// One CTA: the whole matching (resume = 0), or the continuation of the
// grid-wide rounds from their live / matched flags and marked count
// (resume = 1; nothing left to do when the last grid round saw no live
// contact).
__global__ void __launch_bounds__(1024)
match_kernel(const Contact* __restrict__ e, long m_cap, const unsigned long long* __restrict__ m_count, unsigned long long* best, uint8_t* matched, uint8_t* live_e,
             uint8_t* alive, unsigned long long* result, int resume, const MatchState* st) {
  __shared__ int s_remaining;
  __shared__ unsigned long long s_marked;
  const long m = match_count(m_cap, m_count);
  if (resume && st->live[kMatchRounds - 1] == 0) return;  // converged in the grid rounds (result kept)
  if (!resume) {
    for (long k = threadIdx.x; k < m; k += blockDim.x) {
      live_e[k] = 1;
      matched[e[k].a] = 0;
      matched[e[k].b] = 0;
    }
  }
  if (threadIdx.x == 0) s_marked = resume ? result[0] : 0;
  __syncthreads();
  long rounds = 0;
  for (;;) {
    for (long k = threadIdx.x; k < m; k += blockDim.x)
      if (live_e[k]) {
        if (matched[e[k].a] || matched[e[k].b]) {
          live_e[k] = 0;
          continue;
        }
        best[e[k].a] = ~0ull;
        best[e[k].b] = ~0ull;
      }
    if (threadIdx.x == 0) s_remaining = 0;
    __syncthreads();
    for (long k = threadIdx.x; k < m; k += blockDim.x)
      if (live_e[k]) {
        atomicMin(&best[e[k].a], e[k].prio);
        atomicMin(&best[e[k].b], e[k].prio);
      }
    __syncthreads();
    for (long k = threadIdx.x; k < m; k += blockDim.x)
      if (live_e[k] && best[e[k].a] == e[k].prio && best[e[k].b] == e[k].prio) {
        matched[e[k].a] = 1;
        matched[e[k].b] = 1;
        alive[e[k].a] = 0;
        alive[e[k].b] = 0;
        atomicAdd(&s_marked, 2ull);
      }
    __syncthreads();
    int rem = 0;
    for (long k = threadIdx.x; k < m; k += blockDim.x)
      if (live_e[k]) {
        if (matched[e[k].a] || matched[e[k].b])
          live_e[k] = 0;
        else
          rem = 1;
      }
    if (rem) atomicOr(&s_remaining, 1);
    __syncthreads();
    ++rounds;
    if (s_remaining == 0 || rounds > m + 1) break;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    result[0] = s_marked;
    result[1] = s_remaining ? 1ull : 0ull;  // 1 = did not converge (cannot happen)
  }
}

// Contacts from which the grid-wide rounds are used (AMK_MATCH_GRID_MIN
// overrides it: tests of that path on small sets).
inline long match_grid_min() {
  const char* s = getenv("AMK_MATCH_GRID_MIN");
  if (s && *s) return atol(s);
  return 8192;
}

// Queues the matching of the contacts e[0, m) (m = min(m_cap, *m_count) when
// m_count is given) on `stream`: result[0] = particles marked, result[1] = 1
// if it did not converge. best0/best1 hold one word per particle, matched
// one byte per particle, live_e one byte per contact, st one MatchState.
inline int queue_matching(amk_ctx* c, cudaStream_t stream, const Contact* e, long m_cap,
                          const unsigned long long* m_count, unsigned long long* best0, unsigned long long* best1,
                          uint8_t* matched, uint8_t* live_e, uint8_t* alive, MatchState* st,
                          unsigned long long* result) {
  if (m_cap < match_grid_min()) {
    match_kernel<<<1, 1024, 0, stream>>>(e, m_cap, m_count, best0, matched, live_e, alive, result, 0, st);
    return check_launch(c, "match_kernel");
  }
  const unsigned grid = static_cast<unsigned>(std::min<long>((m_cap + 255) / 256, 148L * 8));
  match_init_kernel<<<grid, 256, 0, stream>>>(e, m_cap, m_count, best0, best1, matched, live_e, st, result);
  AMK_TRY(check_launch(c, "match_init_kernel"));
  for (int r = 0; r < kMatchRounds; ++r) {
    unsigned long long* cur = (r & 1) ? best1 : best0;
    unsigned long long* next = (r & 1) ? best0 : best1;
    match_min_kernel<<<grid, 256, 0, stream>>>(e, m_cap, m_count, r, cur, next, matched, live_e, st);
    AMK_TRY(check_launch(c, "match_min_kernel"));
    match_select_kernel<<<grid, 256, 0, stream>>>(e, m_cap, m_count, r, cur, matched, live_e, alive, st, result);
    AMK_TRY(check_launch(c, "match_select_kernel"));
  }
  match_kernel<<<1, 1024, 0, stream>>>(e, m_cap, m_count, best0, matched, live_e, alive, result, 1, st);
  return check_launch(c, "match_kernel");
}

}  // namespace
}  // namespace amk
