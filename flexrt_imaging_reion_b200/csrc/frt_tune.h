// Launch-shape search of the autotuner (host only, no CUDA: the library's frt_autotune drives it
// with CUDA-event times, tests drive it with synthetic costs).
//
// The reference balances its OpenMP ray loops by moving rays between per-thread buffers
// (balance_cpus / free_cpu, mem_funcs.cc:186-299) and partitions them statically (size_cpu,
// global_variables.cc:44). Here the equivalent choices are launch shapes: block size and blocks
// per SM of each ray / cell kernel, and whether the ray pass hands out its moved rays as static
// per-warp slices or as chunks of a device-side queue (and how large). They are picked by
// measurement on the run's own state.
//
// Search: per kernel family, rounds of candidates; every candidate of a round is timed once on a
// comparable share of the same step's work (the ray pass: one of the step's C2Ray iterations;
// the walk, the cell pass and the compaction: one of k equal ray / cell ranges of the step), and
// its cost is the time per unit of work (crossing, ray, lit cell). The first round spreads over
// the parameter space, the next rounds vary one parameter at a time around the best so far
// (coordinate descent); the current best is always re-timed in a round, so a choice never rests
// on one early sample alone. The axes are visited in the order of the gain their round-0 probe
// showed, and along an axis the untried values nearest the current best come first.
#pragma once
#include <string>
#include <vector>

namespace frt {

struct Shape {
  int block = 256;   // threads per block
  int grid = 8;      // blocks per SM
  int chunk = 0;     // ray-pass queue chunk (0 = static slices); unused by the other families
  bool operator==(const Shape& o) const { return block == o.block && grid == o.grid && chunk == o.chunk; }
};

// One kernel family's search over the values allowed for each parameter.
class ShapeSearch {
 public:
  ShapeSearch() = default;
  ShapeSearch(std::string name, Shape start, std::vector<int> blocks, std::vector<int> grids, std::vector<int> chunks,
              int per_round);
  // candidates of the next round (per_round of them at most; the best so far first)
  std::vector<Shape> next_round();
  // the measured cost (time per unit of work) of candidate k of the round last handed out
  void record(int k, double cost);
  // closes the round: folds its costs into the per-shape record
  void end_round();
  const Shape& best() const { return best_; }
  double best_cost() const { return best_cost_; }
  bool done() const { return round_ >= max_rounds_; }
  int rounds() const { return round_; }
  const std::string& name() const { return name_; }
  void set_max_rounds(int r) { max_rounds_ = r; }

 private:
  struct Seen {
    Shape s;
    double cost_sum = 0.0;
    int n = 0;
    double mean() const { return n ? cost_sum / n : 1e300; }
  };
  Seen* find(const Shape& s);
  void add_unique(std::vector<Shape>* v, const Shape& s) const;
  std::string name_;
  Shape best_;
  double best_cost_ = 1e300;
  std::vector<int> blocks_, grids_, chunks_;
  int per_round_ = 4, round_ = 0, max_rounds_ = 2, axis_ = 0;
  int axis_order_[3] = {0, 1, 2};   // descent order of the axes (chunk, grid, block)
  int probe_axis_[8] = {-1, -1, -1, -1, -1, -1, -1, -1};   // round 0: the axis each candidate probes
  std::vector<Shape> cur_;
  std::vector<double> cur_cost_;
  std::vector<Seen> seen_;
};

}  // namespace frt
