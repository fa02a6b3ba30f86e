// Checks the engine's host thread pool (dials_metal_spotfinder_b200/csrc/
// sf_pool.hh) on its own, for tests/test_pool.py: every index is run
// exactly once per call, calls follow one another on the same threads, an
// exception from any item reaches the caller after the others have run,
// and the pool keeps working after it. Exit 0 when all hold.

#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "../../dials_metal_spotfinder_b200/csrc/sf_pool.hh"

int main() {
  for (int threads : {1, 3, 7}) {
    sf::HostPool pool(threads);
    for (size_t n : {0ul, 1ul, 2ul, 16ul, 1000ul}) {
      for (int rep = 0; rep < 50; rep++) {
        std::vector<std::atomic<int>> hits(n);
        for (auto &h : hits)
          h.store(0);
        pool.run(n, [&](size_t i) { hits[i].fetch_add(1); });
        for (size_t i = 0; i < n; i++)
          if (hits[i].load() != 1) {
            std::fprintf(stderr, "threads %d n %zu: index %zu ran %d times\n", threads, n, i,
                         hits[i].load());
            return 1;
          }
      }
    }
    std::atomic<int> ran{0};
    bool thrown = false;
    try {
      pool.run(64, [&](size_t i) {
        ran.fetch_add(1);
        if (i == 17)
          throw std::invalid_argument("item 17");
      });
    } catch (const std::invalid_argument &) {
      thrown = true;
    }
    if (!thrown || ran.load() != 64) {
      std::fprintf(stderr, "threads %d: thrown %d, ran %d of 64\n", threads, thrown ? 1 : 0,
                   ran.load());
      return 1;
    }
    std::atomic<int> after{0};
    pool.run(10, [&](size_t) { after.fetch_add(1); });
    if (after.load() != 10) {
      std::fprintf(stderr, "threads %d: %d of 10 after an exception\n", threads, after.load());
      return 1;
    }
  }
  std::puts("ok");
  return 0;
}
