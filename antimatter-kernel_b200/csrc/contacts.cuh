// Contacts between annihilation partners and their deterministic greedy
// matching, shared by the single-instance and batched paths.
#pragma once
#include "amk_internal.cuh"

namespace amk {
namespace {

struct Contact {
  uint32_t a, b;   // owner, partner (indices)
  uint64_t prio;   // (owner id << 32) | partner id
};

// Greedy matching by locally-dominant selection, one CTA. Each round selects
// every live contact whose priority is the minimum at both endpoints (these
// are exactly the contacts the sequential greedy pass takes), then retires
// contacts touching a matched particle. At least one contact (the global
// minimum) is selected per round, so the loop ends within `m` rounds.
__global__ void __launch_bounds__(1024)
match_kernel(const Contact* __restrict__ e, long m_cap, const unsigned long long* __restrict__ m_count, unsigned long long* best, uint8_t* matched, uint8_t* live_e,
             uint8_t* alive, unsigned long long* result) {
  __shared__ int s_remaining;
  __shared__ unsigned long long s_marked;
  // the number of contacts may live on the device (graph replays)
  const long m = m_count ? static_cast<long>(min(static_cast<unsigned long long>(m_cap), *m_count)) : m_cap;
  for (long k = threadIdx.x; k < m; k += blockDim.x) {
    live_e[k] = 1;
    matched[e[k].a] = 0;
    matched[e[k].b] = 0;
  }
  if (threadIdx.x == 0) s_marked = 0;
  __syncthreads();
  long rounds = 0;
  for (;;) {
    for (long k = threadIdx.x; k < m; k += blockDim.x)
      if (live_e[k]) {
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


}  // namespace
}  // namespace amk
