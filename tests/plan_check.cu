// Host-side checks of the windowed launch plans (no GPU): the work list of
// append_work and the deferred-list storage of deferred_words /
// attach_deferred, the arithmetic that keeps every kernel access of a launch
// inside its buffers.  Prints "ok" or the first failed check; exit status 1
// on a failure.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "radio_kernels.cuh"

using namespace c8r;

namespace {

int failures = 0;

void expect(bool ok, char const* what, unsigned long long a = 0, unsigned long long b = 0) {
  if (ok) return;
  std::printf("FAIL %s (%llu, %llu)\n", what, a, b);
  ++failures;
}

EventPlan event(uint32_t chunk, uint32_t chunks, uint32_t observers) {
  EventPlan e;
  std::memset(&e, 0, sizeof e);
  e.chunk_size = chunk;
  e.chunks = chunks;
  e.observer_count[0] = observers;
  e.observer_count[1] = observers;
  e.first_track = 0;
  e.last_track = ~0ull;
  return e;
}

WorkPlan plan_of(std::vector<EventPlan> const& events, int algorithm, uint64_t ctas) {
  WorkPlan plan;
  std::memset(&plan, 0, sizeof plan);
  plan.algorithm = algorithm;
  for (std::size_t i = 0; i < events.size(); ++i) append_work(plan, events[i], ctas, i + 1 == events.size());
  plan.deferred_stride = deferred_list_stride(plan);
  return plan;
}

// Every track of every event falls in exactly one item of the plan, and the
// items' chunks lie inside [first_track, first_track + chunks * chunk_size).
void check_work_list(std::vector<EventPlan> const& events, WorkPlan const& plan) {
  uint64_t items = 0;
  for (uint32_t e = 0; e < plan.event_count; ++e) {
    EventPlan const& p = plan.events[e];
    expect(p.first_item == items, "entries' items are consecutive", p.first_item, items);
    items += static_cast<uint64_t>(p.chunks) * p.observer_count[plan.algorithm];
    expect(p.chunk_size <= kMaxChunkTracks, "chunk within the deferred-entry offset bits", p.chunk_size);
    expect(p.chunk_size <= plan.deferred_stride, "list stride holds a chunk", p.chunk_size, plan.deferred_stride);
  }
  expect(items == plan.total_items, "total items", items, plan.total_items);
  uint64_t want_tracks = 0, got_tracks = 0;
  for (auto const& e : events) want_tracks += static_cast<uint64_t>(e.chunks) * e.chunk_size;
  for (uint32_t e = 0; e < plan.event_count; ++e) {
    EventPlan const& p = plan.events[e];
    uint64_t const stop = p.first_track + static_cast<uint64_t>(p.chunks) * p.chunk_size;
    uint64_t const end = stop < p.last_track ? stop : p.last_track;
    got_tracks += end - p.first_track;
  }
  expect(got_tracks == want_tracks, "every track in one item", got_tracks, want_tracks);
}

// The storage of a launch: the regions the kernels index are disjoint and
// inside deferred_words words.
void check_storage(WorkPlan plan, uint64_t ctas, bool fixed) {
  uint64_t const words = deferred_words(plan, ctas, fixed);
  // only addresses are compared: nothing is read or written through them
  unsigned* const base = reinterpret_cast<unsigned*>(uintptr_t{1} << 20);  // a 16-byte aligned stand-in
  attach_deferred(plan, base, ctas, fixed);
  uint64_t const lists = ctas * plan.deferred_stride;
  if (!two_pass(plan, ctas, fixed)) {
    expect(plan.item_state == nullptr && plan.drain_deferred == nullptr, "one pass: no second-pass storage");
    expect(words == lists, "one pass: the CTAs' lists", words, lists);
    return;
  }
  uint64_t const first = static_cast<uint64_t>(plan.deferred_capacity) * ctas;
  expect(plan.deferred_capacity >= plan.deferred_stride, "first-pass list holds an item",
         plan.deferred_capacity, plan.deferred_stride);
  expect(plan.drain_deferred == base + first, "second-pass lists follow the first pass's");
  unsigned* const states = reinterpret_cast<unsigned*>(plan.item_state);
  expect(states == base + first + lists, "item states follow the lists");
  expect(plan.drain_next_item == states + plan.total_items * (sizeof(ItemState) / sizeof(unsigned)),
         "counter follows the states");
  expect(static_cast<uint64_t>(plan.drain_next_item - base) + 1 == words, "storage ends at the counter",
         static_cast<uint64_t>(plan.drain_next_item - base) + 1, words);
  expect(words <= kTwoPassMaxWords, "two passes within the cap", words, kTwoPassMaxWords);
  // the kernels' last indices: first-pass list of the last CTA, its last
  // entry; second-pass list likewise; the last item's state
  expect((ctas - 1) * plan.deferred_capacity + plan.deferred_capacity - 1 < first, "first-pass index");
  expect(first + (ctas - 1) * plan.deferred_stride + plan.deferred_stride - 1 < first + lists, "second-pass index");
}

}  // namespace

int main() {
  // the 1e7 x 160 workload's ZHS launch, a served round, a batched launch of
  // several events, small launches, and one past the two-pass cap
  struct Case {
    std::vector<EventPlan> events;
    uint64_t ctas;
  };
  std::vector<Case> cases = {
      {{event(666688, 15, 160)}, 148},
      {{event(131072, 8, 64), event(131072, 3, 300), event(131072, 1, 16)}, 148},
      {{event(524288, 20, 300), event(524288, 4, 16), event(524288, 39, 120)}, 148},
      {{event(8192, 1, 16)}, 148},
      {{event(256, 79, 16)}, 148},
      {{event(1u << 30, 64, 300)}, 148},  // 2e13 pairs: one pass
  };
  for (auto const& c : cases) {
    for (int algorithm = 0; algorithm < 2; ++algorithm) {
      uint64_t ctas = c.ctas;
      WorkPlan plan = plan_of(c.events, algorithm, ctas);
      if (ctas > plan.total_items) ctas = plan.total_items;
      check_work_list(c.events, plan);
      for (bool fixed : {false, true}) {
        check_storage(plan, ctas, fixed);
        bool const expect_two = fixed && algorithm == 1 && two_pass_words(plan, ctas) <= kTwoPassMaxWords;
        expect(two_pass(plan, ctas, fixed) == expect_two, "two passes exactly for fixed ZHS within the cap");
      }
    }
  }
  {
    WorkPlan huge = plan_of({event(1u << 30, 64, 300)}, 1, 148);
    expect(!two_pass(huge, 148, true), "a launch past the cap runs one pass");
  }
  if (failures) return 1;
  std::printf("ok\n");
  return 0;
}
