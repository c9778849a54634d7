// Compares the product's heap emulation (falconnpp_b200/csrc/fpp_heap.h) with
// libstdc++'s std::priority_queue on random, tie-heavy operation sequences.
// Built and run by tests/test_heap_emulation.py.  Prints "ok <ops>" or the
// first mismatch.
#include <cstdio>
#include <cstring>
#include <queue>
#include <random>
#include <vector>

#include "fpp_heap.h"

struct P {
  int id;
  float v;
  bool operator<(const P& o) const { return v < o.v; }
  bool operator>(const P& o) const { return v > o.v; }
};

template <bool Min>
int run(unsigned seed, int trials, long long* ops) {
  using Q = typename std::conditional<Min, std::priority_queue<P, std::vector<P>, std::greater<>>,
                                      std::priority_queue<P>>::type;
  std::mt19937 rng(seed);
  for (int t = 0; t < trials; ++t) {
    const int levels = 1 + rng() % 6;  // few distinct values: many ties
    const int cap = 1 + rng() % 40;
    Q q;
    std::vector<float> hv(4096);
    std::vector<int> hi(4096);
    int n = 0;
    const int steps = 1 + rng() % 300;
    for (int s = 0; s < steps; ++s) {
      const int op = rng() % 3;
      const float v = (float)(rng() % levels) * 0.5f - (float)(rng() % 2) * 0.0f;
      const int id = (int)(rng() % 100000);
      if (op == 2 && n > 0) {
        if (q.top().id != hi[0] || q.top().v != hv[0]) return t + 1;
        q.pop();
        fpp::heap_pop<Min, int>(hv.data(), hi.data(), n);
      } else if (op == 1 && Min) {  // bounded top-list step
        if ((int)q.size() < cap)
          q.push(P{id, v});
        else if (v > q.top().v) {
          q.pop();
          q.push(P{id, v});
        }
        fpp::topp_offer<int>(hv.data(), hi.data(), n, cap, v, id);
      } else if (n < 4000) {
        q.push(P{id, v});
        fpp::heap_push<Min, int>(hv.data(), hi.data(), n, v, id);
      }
      ++*ops;
      if ((int)q.size() != n) return t + 1;
    }
    while (n > 0) {  // drain order must match element by element
      if (q.top().id != hi[0] || q.top().v != hv[0]) return t + 1;
      q.pop();
      fpp::heap_pop<Min, int>(hv.data(), hi.data(), n);
      ++*ops;
    }
  }
  return 0;
}

int main() {
  long long ops = 0;
  for (unsigned seed = 1; seed <= 4; ++seed) {
    int r = run<true>(seed, 3000, &ops);
    if (r) {
      printf("mismatch min-heap seed %u trial %d\n", seed, r - 1);
      return 1;
    }
    r = run<false>(seed + 100, 3000, &ops);
    if (r) {
      printf("mismatch max-heap seed %u trial %d\n", seed, r - 1);
      return 1;
    }
  }
  // ord_key_bits orders floats like the float comparison, -0 == +0
  const float vals[] = {-1e30f, -2.5f, -1.0f, -1e-30f, -0.0f, 0.0f, 1e-30f, 1.0f, 2.5f, 1e30f};
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j) {
      unsigned a, b;
      memcpy(&a, &vals[i], 4);
      memcpy(&b, &vals[j], 4);
      const bool lt = vals[i] < vals[j], eq = vals[i] == vals[j];
      const unsigned ka = fpp::ord_key_bits(a), kb = fpp::ord_key_bits(b);
      if ((ka < kb) != lt || (ka == kb) != eq) {
        printf("ord_key mismatch %d %d\n", i, j);
        return 1;
      }
    }
  printf("ok %lld\n", ops);
  return 0;
}
