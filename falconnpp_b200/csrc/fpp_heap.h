// fpp_heap.h — exact emulation of the binary heap behind std::priority_queue.
//
// The reference keeps every top-p list and every bucket in a
// std::priority_queue<IFPair> whose comparison looks at the float value only
// (src/Header.h:57-65).  When two values are equal, which element survives a
// pop and in which order equal elements leave the heap is decided by the heap
// algorithm of GCC's libstdc++, not by the ids.  The GPU kernels take a fast
// path (score desc, id asc) and detect ties; whenever a tie could change the
// reference's answer they replay the reference's exact heap operations with the
// functions below, so the results stay identical to the reference's.
//
// Algorithm restated (libstdc++ bits/stl_heap.h semantics, value-only compare):
//  * push = append at the end, then sift the new element up while the
//    comparison says the parent has strictly lower priority than it;
//  * pop  = move the last element out, move the top to the end, walk a hole
//    from the root down to a leaf always taking the higher-priority child
//    (the right child unless it is strictly lower-priority than the left),
//    fill the last odd left child, then sift the saved element up from the
//    hole.
// MinHeap=true mirrors priority_queue<IFPair, vector<IFPair>, greater<>>
// (top = smallest value, used for top-p lists, FalconnPP.cpp:96, :162, :383,
// :633); MinHeap=false mirrors priority_queue<IFPair> (top = largest, used for
// buckets FalconnPP.cpp:70 and the global probe merge FalconnPP.cpp:540).
// tests/test_heap_emulation.py checks this file against std::priority_queue.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define FPP_HD __host__ __device__ __forceinline__
#else
#define FPP_HD inline
#endif

namespace fpp {

// comp(a, b) of the container: "a has lower priority than b".
template <bool MinHeap>
FPP_HD bool heap_comp(float a, float b) {
  return MinHeap ? (a > b) : (a < b);
}

template <bool MinHeap, typename I>
FPP_HD void heap_sift_up(float* hv, I* hi, int hole, int top, float v, I id) {
  int parent = (hole - 1) / 2;
  while (hole > top && heap_comp<MinHeap>(hv[parent], v)) {
    hv[hole] = hv[parent];
    hi[hole] = hi[parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  hv[hole] = v;
  hi[hole] = id;
}

// priority_queue::emplace / push
template <bool MinHeap, typename I>
FPP_HD void heap_push(float* hv, I* hi, int& n, float v, I id) {
  heap_sift_up<MinHeap, I>(hv, hi, n, 0, v, id);
  ++n;
}

// priority_queue::pop (the removed top is hv[0]/hi[0] before the call)
template <bool MinHeap, typename I>
FPP_HD void heap_pop(float* hv, I* hi, int& n) {
  if (n > 1) {
    const int len = n - 1;
    const float v = hv[len];
    const I id = hi[len];
    hv[len] = hv[0];
    hi[len] = hi[0];
    int hole = 0;
    int child = 0;
    while (child < (len - 1) / 2) {
      child = 2 * (child + 1);
      if (heap_comp<MinHeap>(hv[child], hv[child - 1])) --child;
      hv[hole] = hv[child];
      hi[hole] = hi[child];
      hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
      child = 2 * (child + 1);
      hv[hole] = hv[child - 1];
      hi[hole] = hi[child - 1];
      hole = child - 1;
    }
    heap_sift_up<MinHeap, I>(hv, hi, hole, 0, v, id);
  }
  --n;
}

// The "keep the top-p, replace the current worst only on a strictly better
// value" step used for every bounded top list in the reference
// (e.g. FalconnPP.cpp:113-121, :650-657).
template <typename I>
FPP_HD void topp_offer(float* hv, I* hi, int& n, int cap, float v, I id) {
  if (n < cap) {
    heap_push<true, I>(hv, hi, n, v, id);
  } else if (v > hv[0]) {
    heap_pop<true, I>(hv, hi, n);
    heap_push<true, I>(hv, hi, n, v, id);
  }
}

// Order-preserving map float -> uint32 (ascending key == ascending value);
// -0.0f and +0.0f share one key because they compare equal.
FPP_HD uint32_t ord_key_bits(uint32_t u) {
  if ((u << 1) == 0u) return 0x80000000u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

}  // namespace fpp
