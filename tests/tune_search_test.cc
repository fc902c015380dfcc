// CPU check of the autotuner's search (flexrt_imaging_reion_b200/csrc/frt_tune.cc) against
// synthetic cost functions, built and run by tests/test_autotune.py. Prints one line per case:
// CASE <name> <rounds> <block> <grid> <chunk> <cost>
#include <cmath>
#include <cstdio>
#include <functional>

#include "frt_tune.h"

using frt::Shape;
using frt::ShapeSearch;

static void run(const char* name, ShapeSearch s, int rounds, std::function<double(const Shape&, int)> cost) {
  s.set_max_rounds(rounds);
  for (int r = 0; r < rounds; r++) {
    const auto cand = s.next_round();
    for (size_t k = 0; k < cand.size(); k++) s.record((int)k, cost(cand[k], r));
    s.end_round();
  }
  printf("CASE %s %d %d %d %d %.6f\n", name, s.rounds(), s.best().block, s.best().grid, s.best().chunk, s.best_cost());
}

int main() {
  // separable optimum at (128, 12, 128) away from the start (256, 8, 0)
  auto sep = [](const Shape& s, int) {
    return 1.0 + 0.3 * std::fabs(std::log2(s.grid / 12.0)) + (s.block == 128 ? 0.0 : 0.2) +
           0.25 * std::fabs(std::log2((s.chunk + 16.0) / 144.0));
  };
  {
    // the optimum's cost and the start's, for the test's bounds
    printf("REF separable %.6f %.6f\n", sep(Shape{128, 12, 128}, 0), sep(Shape{256, 8, 0}, 0));
  }
  run("separable", ShapeSearch("rp", Shape{256, 8, 0}, {128, 256}, {4, 8, 12, 16}, {0, 32, 128, 512}, 4), 3, sep);
  // the same costs, all scaled down each round (more work per unit later in a run): the winner of
  // a round is decided within the round, so the drift must not change the answer
  run("drift", ShapeSearch("rp", Shape{256, 8, 0}, {128, 256}, {4, 8, 12, 16}, {0, 32, 128, 512}, 4), 3,
      [&](const Shape& s, int r) { return sep(s, r) * std::pow(0.5, r); });
  // the start is already best: it stays
  run("start_best", ShapeSearch("walk", Shape{256, 8, 0}, {128, 256}, {4, 8, 16}, {0}, 4), 2,
      [](const Shape& s, int) { return (s.block == 256 && s.grid == 8) ? 1.0 : 2.0; });
  // one parameter only (blocks per SM), optimum at 2
  run("grid_only", ShapeSearch("split", Shape{256, 8, 0}, {256}, {2, 4, 8, 16}, {0}, 4), 2,
      [](const Shape& s, int) { return 1.0 + std::fabs(std::log2(s.grid / 2.0)); });
  return 0;
}
