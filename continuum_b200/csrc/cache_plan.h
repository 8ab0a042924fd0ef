// The lighting cache's page manager on the host: which requested pages bake
// this frame within the cone budget, the budget's adaptation to the frame
// time, slot allocation and eviction, and the frame's bake job list.
//
// A restatement of crates/continuum-gpu/src/vcache.rs for the direct light of
// static lights: `plan` (:3704-3850) and `plan_page` (:3928-4060) without sky
// samples, bounce light, lighting levels or area texels; the budget update of
// `begin_frame` (:2976-3080) with `BakeModel` (:1105-1160); eviction by
// `queue_stale` / `evict_queued` / `evict_now` (:3492-3560). Pages are 8 x 8
// texels stored 9 x 9 (PAGE, STRIDE, PAGE_TEXELS, :32-35); a job is
// [bake-list index, texel | light << 8] (:4037-4043), listed light by light.
#pragma once
#include <cstdint>
#include <deque>
#include <map>
#include <unordered_map>
#include <vector>

namespace cc_bake {

constexpr uint32_t kPage = 8;
constexpr uint32_t kStride = kPage + 1;
constexpr uint32_t kPageTexels = kStride * kStride;
constexpr uint32_t kEmpty = 0xffffffffu;
constexpr float kMinBudget = 1000.0f;       // MIN_BUDGET (:52)
constexpr float kStartBudget = 8000.0f;     // START_BUDGET (:80)
constexpr uint32_t kEvictPerFrame = 2048;   // EVICT_PER_FRAME (:41)
constexpr uint32_t kEvictAge = 64;          // EVICT_AGE (:44)
constexpr float kEvictAbove = 0.25f;        // EVICT_ABOVE (:51)
constexpr uint32_t kFloorFresh = 120;       // FLOOR_FRESH (:55)

struct Options {
  uint32_t pages = 1u << 16;
  uint32_t lights = 1;
  uint32_t bake_budget = 1u << 20;
  float frame_target_ms = 0.0f;
  float frame_budget_ms = 0.0f;
  float floor_overrun = 0.25f;
};

struct Key {
  uint32_t k[3];
  bool operator==(const Key& o) const { return k[0] == o.k[0] && k[1] == o.k[1] && k[2] == o.k[2]; }
  bool operator<(const Key& o) const {
    if (k[0] != o.k[0]) return k[0] < o.k[0];
    if (k[1] != o.k[1]) return k[1] < o.k[1];
    return k[2] < o.k[2];
  }
};
struct KeyHash {
  size_t operator()(const Key& x) const {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    for (uint32_t v : x.k) h = (h ^ v) * 0x100000001b3ull;
    return (size_t)h;
  }
};

struct Request {
  Key key;
  uint32_t priority;   // lower first
  uint32_t inside[2];  // texels of the page inside its chart's grid, per axis
};

// A page planned this frame (the bake list's entry).
struct Planned {
  Key key;
  uint32_t slot;
  uint32_t request;    // its index in the frame's requests
  uint32_t listed[2];  // texels listed per axis: inside + 1, at most kStride
};

// Bake time against budget spent, fit as latency + cost x units over recent
// frames (least squares with exponential forgetting), :1105-1160.
struct BakeModel {
  double sums[5] = {0, 0, 0, 0, 0};  // weight, units, units^2, ms, units x ms
  float latency = 1.0f;
  float cost = 5e-4f;
  float render = 0.0f;
  void add(float units, float bake_ms, float render_ms);
  float budget(float target) const { return (target - render - latency) / cost; }
};

// What the caller measured for the previous frame.
struct Timing {
  bool has_period = false;
  float period_ms = 0;     // the caller's frame period
  bool gpu_waited = false; // the CPU waited more than 1 ms for the GPU in it
  float render_ms = 0;     // the camera passes' GPU time in it
};

class Planner {
 public:
  explicit Planner(const Options& o);

  // Before a frame: adapts the budget, evicts stale pages. `bake` is the
  // previous bake's measured GPU time (< 0: not measured) over `units` cones.
  void begin_frame(const Timing& t, float bake_ms, float units);
  // Plans the frame's bake from its requests; fills planned() and jobs().
  void plan(const std::vector<Request>& requests);
  // After the frame is submitted.
  void end_frame() { frame_++; }

  const std::vector<Planned>& planned() const { return planned_; }
  const std::vector<uint32_t>& jobs() const { return jobs_; }  // pairs
  float budget() const { return budget_; }
  uint32_t spent() const { return spent_; }
  uint32_t frame() const { return frame_; }
  uint32_t resident() const { return (uint32_t)map_.size(); }
  uint32_t evicted() const { return evicted_; }
  // The slot of a resident page, or kEmpty.
  uint32_t slot_of(const Key& k) const {
    auto it = map_.find(k);
    return it == map_.end() ? kEmpty : it->second;
  }
  const Options& options() const { return opt_; }

 private:
  enum class Outcome { kPlanned, kSkipped, kFull };
  Outcome plan_page(const Request& r, uint32_t index, uint32_t budget, bool& evicted_now);
  void queue_stale(uint32_t age);
  uint32_t evict_queued(uint32_t count, uint32_t age);
  float limit(float l) const;

  Options opt_;
  uint32_t frame_ = 0;
  float budget_;
  float cap_;
  float periods_[3] = {0, 0, 0};
  float floor_period_ = 0;
  uint32_t floor_frame_ = 0;
  uint32_t model_frame_ = 0;  // the frame of the latest bake timing (0: none yet)
  uint32_t latest_ = 0;       // the latest frame timed
  BakeModel model_;
  std::unordered_map<Key, uint32_t, KeyHash> map_;
  std::vector<Key> slot_key_;
  std::vector<uint32_t> last_used_;
  std::vector<uint32_t> free_;
  std::vector<uint32_t> evict_queue_;
  std::vector<Planned> planned_;
  std::vector<uint32_t> jobs_;
  uint32_t spent_ = 0;
  uint32_t evicted_ = 0;
};

}  // namespace cc_bake
