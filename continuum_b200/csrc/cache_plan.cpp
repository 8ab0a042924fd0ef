// The lighting cache's page manager (see cache_plan.h for what it restates).
#include "cache_plan.h"

#include <algorithm>
#include <cmath>
#include <tuple>

namespace cc_bake {

// BakeModel::add (vcache.rs:1123-1146)
void BakeModel::add(float units, float bake_ms, float render_ms) {
  render = render == 0.0f ? render_ms : 0.7f * render + 0.3f * render_ms;
  if (units <= 0.0f) return;
  const double u = units, y = bake_ms;
  const double x[5] = {1.0, u, u * u, y, u * y};
  for (int i = 0; i < 5; ++i) sums[i] = 0.95 * sums[i] + x[i];
  const double w = sums[0], su = sums[1], suu = sums[2], sy = sums[3], suy = sums[4];
  const double mu = su / w, my = sy / w;
  const double var = suu / w - mu * mu;
  // Refit the cost only when the budget has varied enough to tell.
  if (w >= 4.0 && var > (0.1 * mu) * (0.1 * mu)) {
    const double c = (suy / w - mu * my) / var;
    cost = std::min(std::max((float)c, 1e-6f), 1.0f);
  }
  latency = std::min(std::max((float)(my - (double)cost * mu), 0.0f), 100.0f);
}

Planner::Planner(const Options& o) : opt_(o) {
  budget_ = opt_.frame_target_ms > 0.0f ? std::min(kStartBudget, (float)opt_.bake_budget) : (float)opt_.bake_budget;
  cap_ = (float)opt_.bake_budget;
  slot_key_.assign(opt_.pages, Key{{kEmpty, kEmpty, kEmpty}});
  last_used_.assign(opt_.pages, 0);
  // Slot 0 pops first (:1871).
  free_.reserve(opt_.pages);
  for (uint32_t s = opt_.pages; s-- > 0;) free_.push_back(s);
}

// The frame period's limit where frames at the floor already overrun it
// (:3015-3022).
float Planner::limit(float l) const {
  const float overrun = std::max(opt_.floor_overrun, 0.0f);
  const bool floor_known = floor_frame_ > 0 && floor_frame_ + kFloorFresh >= frame_;
  if (overrun > 0.0f && floor_known && floor_period_ > l) return (1.0f + overrun) * floor_period_;
  return l;
}

// begin_frame (:2976-3080): the budget, then eviction.
void Planner::begin_frame(const Timing& t, float bake_ms, float units) {
  // The previous frame's bake timing (collect, :3224-3243).
  if (bake_ms >= 0.0f && frame_ > 0) {
    const uint32_t timed = frame_ - 1;
    model_.add(units, bake_ms, t.render_ms);
    model_frame_ = timed;
    latest_ = std::max(latest_, timed);
  }
  bool has_period = false;
  float period = 0.0f;
  if (t.has_period) {
    periods_[0] = periods_[1];
    periods_[1] = periods_[2];
    periods_[2] = t.period_ms;
    float sorted[3] = {periods_[0], periods_[1], periods_[2]};
    std::sort(sorted, sorted + 3);
    // Until three frames have been timed, the latest.
    period = sorted[0] == 0.0f ? t.period_ms : sorted[1];
    has_period = true;
  }
  const float target = opt_.frame_target_ms;
  const float bake_budget = (float)opt_.bake_budget;
  const float floor = std::min(kMinBudget, bake_budget);
  if (target > 0.0f && has_period && budget_ <= 1.2f * floor) {
    floor_period_ = (floor_frame_ > 0 && floor_frame_ + 8 >= frame_) ? 0.8f * floor_period_ + 0.2f * period : period;
    floor_frame_ = frame_;
  }
  // The model steers while in-order timings keep coming (:3029-3048).
  const bool model = model_frame_ > 0 && model_frame_ + 32 >= frame_;
  if (target > 0.0f && model) {
    if (latest_ > 0) {
      // Alternate frames bake 20% less, so the fit can tell latency from cost.
      const float dither = (frame_ % 2 == 0) ? 1.0f : 0.8f;
      budget_ = std::min(std::max(model_.budget(target) * dither, floor), bake_budget);
    }
  } else if (target > 0.0f && has_period) {
    const float tl = limit(target);
    if (t.gpu_waited && period > tl) budget_ *= tl / period;
    else if (period < tl) budget_ *= 1.1f;
    budget_ = std::min(std::max(budget_, floor), bake_budget);
  }
  // The frame period's cap (:3065-3079), with a frame target only.
  if (opt_.frame_budget_ms > 0.0f && target > 0.0f && has_period) {
    const float bm = limit(opt_.frame_budget_ms);
    if (period > bm) cap_ = std::max(std::min(budget_, cap_) * bm / period, floor);
    else if (period < 0.85f * bm) cap_ = std::min(cap_ * 1.05f, bake_budget);
    budget_ = std::min(budget_, cap_);
  }
  // Pages unused for a while go once the pool is a quarter full (:3087-3092).
  if ((float)map_.size() > kEvictAbove * (float)opt_.pages) {
    queue_stale(kEvictAge);
    evicted_ += evict_queued(kEvictPerFrame, kEvictAge);
  }
}

// queue_stale (:3498-3512): every page unused for more than `age` frames,
// least recently used popped first.
void Planner::queue_stale(uint32_t age) {
  std::vector<std::pair<uint32_t, uint32_t>> stale;
  for (uint32_t s = 0; s < opt_.pages; ++s)
    if (slot_key_[s].k[0] != kEmpty && last_used_[s] + age < frame_) stale.emplace_back(last_used_[s], s);
  std::sort(stale.begin(), stale.end(), [](const auto& a, const auto& b) { return b < a; });
  evict_queue_.clear();
  for (const auto& p : stale) evict_queue_.push_back(p.second);
}

// evict_queued (:3515-3539)
uint32_t Planner::evict_queued(uint32_t count, uint32_t age) {
  uint32_t freed = 0;
  while (freed < count && !evict_queue_.empty()) {
    const uint32_t s = evict_queue_.back();
    evict_queue_.pop_back();
    if (slot_key_[s].k[0] == kEmpty || last_used_[s] + age >= frame_) continue;
    map_.erase(slot_key_[s]);
    slot_key_[s] = Key{{kEmpty, kEmpty, kEmpty}};
    free_.push_back(s);
    freed++;
  }
  return freed;
}

// plan (:3704-3790, the pixels' requests): new pages by priority within the
// budget. A request for a resident page counts as its use this frame.
void Planner::plan(const std::vector<Request>& requests) {
  planned_.clear();
  jobs_.clear();
  spent_ = 0;
  std::vector<std::tuple<uint32_t, Key, uint32_t>> order;
  order.reserve(requests.size());
  for (uint32_t i = 0; i < (uint32_t)requests.size(); ++i) {
    const Request& r = requests[i];
    auto it = map_.find(r.key);
    if (it != map_.end()) {
      last_used_[it->second] = frame_;
      continue;
    }
    order.emplace_back(r.priority, r.key, i);
  }
  // Each page costs at least one texel: no more than `budget` can fit.
  const uint32_t budget = std::max((uint32_t)budget_, kPageTexels);
  auto less = [](const auto& a, const auto& b) {
    if (std::get<0>(a) != std::get<0>(b)) return std::get<0>(a) < std::get<0>(b);
    if (!(std::get<1>(a) == std::get<1>(b))) return std::get<1>(a) < std::get<1>(b);
    return std::get<2>(a) < std::get<2>(b);
  };
  if (order.size() > budget) {
    std::nth_element(order.begin(), order.begin() + budget, order.end(), less);
    order.resize(budget);
  }
  std::sort(order.begin(), order.end(), less);
  bool evicted_now = false;
  for (const auto& o : order) {
    if (plan_page(requests[std::get<2>(o)], std::get<2>(o), budget, evicted_now) == Outcome::kFull) break;
  }
}

// plan_page (:3928-4060) for a page's direct light.
Planner::Outcome Planner::plan_page(const Request& r, uint32_t index, uint32_t budget, bool& evicted_now) {
  // A fingerprint collision can list a page twice.
  if (map_.count(r.key)) return Outcome::kSkipped;
  const uint32_t inside[2] = {std::min(r.inside[0], kStride), std::min(r.inside[1], kStride)};
  if (inside[0] == 0 || inside[1] == 0) return Outcome::kSkipped;
  // One texel past the grid on each side too (the shader skips texels
  // outside its own grid).
  const uint32_t listed[2] = {std::min(inside[0] + 1, kStride), std::min(inside[1] + 1, kStride)};
  const uint32_t cost = inside[0] * inside[1] * opt_.lights;
  // The first page always fits, so a page costlier than the whole budget
  // still gets baked.
  if (spent_ + cost > budget && !planned_.empty()) return Outcome::kFull;
  if (free_.empty() && !evicted_now) {
    // evict_now (:3541-3558): pages unused for more than 2 frames.
    evicted_now = true;
    queue_stale(2);
    evicted_ += evict_queued(kEvictPerFrame, 2);
  }
  if (free_.empty()) return Outcome::kFull;
  const uint32_t slot = free_.back();
  free_.pop_back();
  map_.emplace(r.key, slot);
  slot_key_[slot] = r.key;
  last_used_[slot] = frame_;
  const uint32_t b = (uint32_t)planned_.size();
  planned_.push_back(Planned{r.key, slot, index, {listed[0], listed[1]}});
  // Light by light, so neighbouring invocations trace one light.
  for (uint32_t l = 0; l < opt_.lights; ++l)
    for (uint32_t y = 0; y < listed[1]; ++y)
      for (uint32_t x = 0; x < listed[0]; ++x) {
        jobs_.push_back(b);
        jobs_.push_back((y * kStride + x) | (l << 8));
      }
  spent_ += cost;
  return Outcome::kPlanned;
}

}  // namespace cc_bake
