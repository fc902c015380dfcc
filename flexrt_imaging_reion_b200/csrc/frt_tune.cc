// Launch-shape search of the autotuner (see frt_tune.h).
#include "frt_tune.h"

#include <algorithm>
#include <cstdlib>

namespace frt {

ShapeSearch::ShapeSearch(std::string name, Shape start, std::vector<int> blocks, std::vector<int> grids,
                         std::vector<int> chunks, int per_round)
    : name_(std::move(name)), best_(start), blocks_(std::move(blocks)), grids_(std::move(grids)),
      chunks_(std::move(chunks)), per_round_(std::max(2, per_round)) {}

ShapeSearch::Seen* ShapeSearch::find(const Shape& s) {
  for (Seen& x : seen_)
    if (x.s == s) return &x;
  return nullptr;
}

void ShapeSearch::add_unique(std::vector<Shape>* v, const Shape& s) const {
  if ((int)v->size() >= per_round_) return;
  for (const Shape& x : *v)
    if (x == s) return;
  v->push_back(s);
}

// Values of one axis of a shape: 0 chunk, 1 grid, 2 block.
static int& axis_value(Shape& s, int axis) { return axis == 0 ? s.chunk : (axis == 1 ? s.grid : s.block); }

std::vector<Shape> ShapeSearch::next_round() {
  cur_.clear();
  cur_.push_back(best_);   // the best so far is re-timed: the round compares like with like
  const std::vector<int>* lists[3] = {&chunks_, &grids_, &blocks_};
  for (int& a : probe_axis_) a = -1;
  if (round_ == 0) {
    // spread: one change per axis, to the value farthest from the start
    for (int a = 0; a < 3; a++) {
      const std::vector<int>& L = *lists[a];
      if (L.size() < 2) continue;
      Shape s = best_;
      int& v = axis_value(s, a);
      const int v0 = v;
      int far = L[0];
      for (int x : L)
        if (std::abs(x - v0) > std::abs(far - v0)) far = x;
      v = far;
      const size_t before = cur_.size();
      add_unique(&cur_, s);
      if (cur_.size() > before && cur_.size() <= 8) probe_axis_[cur_.size() - 1] = a;
    }
  }
  // coordinate descent around the best: the untried values of one axis (nearest the best's value
  // first), then the next axes
  for (int k = 0; k < 3 && (int)cur_.size() < per_round_; k++) {
    const int a = axis_order_[(axis_ + k) % 3];
    std::vector<int> vals = *lists[a];
    const int v0 = axis_value(best_, a);
    std::stable_sort(vals.begin(), vals.end(), [v0](int x, int y) { return std::abs(x - v0) < std::abs(y - v0); });
    for (int x : vals) {
      Shape s = best_;
      axis_value(s, a) = x;
      if (!find(s)) add_unique(&cur_, s);
    }
  }
  if (round_ > 0) axis_ = (axis_ + 1) % 3;
  cur_cost_.assign(cur_.size(), 1e300);
  return cur_;
}

void ShapeSearch::record(int k, double cost) {
  if (k >= 0 && k < (int)cur_cost_.size()) cur_cost_[k] = std::min(cur_cost_[k], cost);
}

void ShapeSearch::end_round() {
  // the round's winner (its candidates ran on comparable shares of one step's work)
  int w = -1;
  for (int k = 0; k < (int)cur_.size(); k++) {
    Seen* x = find(cur_[k]);
    if (!x) {
      seen_.push_back(Seen{cur_[k]});
      x = &seen_.back();
    }
    if (cur_cost_[k] < 1e299) {
      x->cost_sum += cur_cost_[k];
      x->n += 1;
      if (w < 0 || cur_cost_[k] < cur_cost_[w]) w = k;
    }
  }
  if (round_ == 0 && cur_cost_[0] < 1e299) {
    // the descent visits first the axes whose probe gained most against the start
    double gain[3] = {-1e300, -1e300, -1e300};
    for (int k = 1; k < (int)cur_.size() && k < 8; k++)
      if (probe_axis_[k] >= 0 && cur_cost_[k] < 1e299) gain[probe_axis_[k]] = cur_cost_[0] - cur_cost_[k];
    std::stable_sort(axis_order_, axis_order_ + 3, [&gain](int x, int y) { return gain[x] > gain[y]; });
  }
  if (w >= 0) {
    best_ = cur_[w];
    best_cost_ = cur_cost_[w];
  }
  round_ += 1;
}

}  // namespace frt
