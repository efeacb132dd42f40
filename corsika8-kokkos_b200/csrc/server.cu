// server.cu — serving many showers on one GPU (c8r_server_* in c8radio.h).
//
// Memory: one HBM arena reserved at creation is the admission budget.  An
// event holds a resident part (observer constants, refractivity table,
// traces, counters) from admission to fetch, plus kinematics blocks of
// block_tracks tracks that its producer fills through the ingest kernel; a
// block returns to the arena once the round that projected its last chunk
// has finished on the GPU.  Admission needs the resident part and one block.
//
// Scheduling: a scheduler thread builds rounds from the sealed blocks (full,
// or the last block of a closed event).  A round gives each ready event an
// equal share of about round_pairs track-antenna pairs as slices of chunk
// indices [chunk_begin, chunk_begin + chunks) of its blocks, and issues one
// persistent windowed launch per algorithm (and per precision / trace mode
// present) over all slices, on the server's compute stream.  At most two
// rounds are queued on the GPU, so an event that arrives while others run
// joins within about one round.  Fixed-point traces are exact sums, so an
// event's traces do not depend on the slices, rounds or neighbours it was
// projected with.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/c8radio.h"
#include "host_setup.hpp"
#include "radio_kernels.cuh"

namespace c8r {
void set_global_error(char const* message);  // accumulator.cu

namespace {

struct server_cuda_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct timeout_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check(cudaError_t err, char const* what) {
  if (err != cudaSuccess) throw server_cuda_error(std::string(what) + ": " + cudaGetErrorString(err));
}

constexpr std::size_t kGranule = 256;
std::size_t round_up(std::size_t bytes) { return (bytes + kGranule - 1) / kGranule * kGranule; }

// First-fit sub-allocator over one device reservation, coalescing on release.
class Arena {
 public:
  ~Arena() { free_all(); }
  void free_all() {
    if (base_) cudaFree(base_);
    base_ = nullptr;
  }
  void reserve(std::size_t bytes) {
    bytes = bytes / kGranule * kGranule;
    if (bytes == 0) throw std::invalid_argument("server budget must be at least 256 bytes");
    if (cudaMalloc(&base_, bytes) != cudaSuccess) {
      cudaGetLastError();
      throw std::bad_alloc();
    }
    size_ = bytes;
    free_[0] = bytes;
  }
  char* allocate(std::size_t bytes) {
    bytes = round_up(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      std::size_t const offset = it->first, rest = it->second - bytes;
      free_.erase(it);
      if (rest) free_[offset + bytes] = rest;
      used_ += bytes;
      peak_ = std::max(peak_, used_);
      return static_cast<char*>(base_) + offset;
    }
    return nullptr;
  }
  void release(char* p, std::size_t bytes) {
    if (!p) return;
    bytes = round_up(bytes);
    used_ -= bytes;
    std::size_t offset = static_cast<std::size_t>(p - static_cast<char*>(base_));
    auto next = free_.lower_bound(offset);
    if (next != free_.end() && offset + bytes == next->first) {
      bytes += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == offset) {
        prev->second += bytes;
        return;
      }
    }
    free_[offset] = bytes;
  }
  std::size_t size() const { return size_; }
  std::size_t used() const { return used_; }
  std::size_t peak() const { return peak_; }

 private:
  void* base_ = nullptr;
  std::size_t size_ = 0, used_ = 0, peak_ = 0;
  std::map<std::size_t, std::size_t> free_;  // offset -> bytes
};

struct Block {
  char* memory = nullptr;
  unsigned long long* slot = nullptr;  // valid tracks written by ingest
  double* tracks = nullptr;
  std::size_t records = 0;             // records ingested (bounds the valid tracks)
  cudaEvent_t ingested = nullptr;      // recorded after every ingest into the block
  bool sealed = false, waited = false;
  uint32_t chunks = 0, next_chunk = 0;
  uint64_t last_round = 0;
};

enum class EventState { kOpen, kClosed, kComplete };

struct ServedEvent {
  uint64_t id = 0;
  EventState state = EventState::kOpen;
  bool fixed = true, diagnostics = false;
  Precision precision = Precision::kFP64;
  double limit = 1.;
  std::vector<c8r_observer_snapshot> snapshots[2];
  uint32_t observers[2] = {0, 0};
  uint64_t bins[2] = {0, 0};
  uint32_t window = 1;
  char* memory = nullptr;
  std::size_t bytes = 0;
  ObserverCache* caches[2] = {nullptr, nullptr};
  unsigned long long* fixed_traces[2] = {nullptr, nullptr};
  double* float_traces[2] = {nullptr, nullptr};
  DeviceCounters* counters = nullptr;
  Propagation propagation{};
  IngestTerms terms{};       // source terms written at ingest (shared destination row)
  std::deque<Block> blocks;  // in fill order; the front ones retire first
  std::size_t records = 0;
  uint64_t last_round = 0, rounds = 0;
  double open_s = 0., admitted_s = 0., closed_s = 0., completed_s = 0.;
  bool fetching = false;
};

struct Slice {
  ServedEvent* event;
  Block* block;
  uint32_t chunk_begin, chunks;
};

struct Round {
  uint64_t id;
  cudaEvent_t done;
};

// The current device is per host thread: make the server's device current
// for the duration of a call and restore the caller's afterwards.
class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&previous_) != cudaSuccess) previous_ = -1;
    if (previous_ != device) check(cudaSetDevice(device), "cudaSetDevice");
    else previous_ = -1;
  }
  ~DeviceGuard() {
    if (previous_ >= 0) cudaSetDevice(previous_);
  }
  DeviceGuard(DeviceGuard const&) = delete;
  DeviceGuard& operator=(DeviceGuard const&) = delete;

 private:
  int previous_ = -1;
};

class Server {
 public:
  explicit Server(c8r_server_options const& options) {
    block_tracks_ = options.block_tracks ? options.block_tracks : (1u << 20);
    chunk_tracks_ = options.chunk_tracks ? options.chunk_tracks : 131072;
    round_pairs_ = options.round_pairs ? options.round_pairs : 1000000000ull;
    threads_ = options.team_size ? static_cast<int>(options.team_size) : kWindowThreads;
    if (chunk_tracks_ == 0 || chunk_tracks_ > kMaxChunkTracks || block_tracks_ % chunk_tracks_ != 0 ||
        block_tracks_ / chunk_tracks_ > 0xffffffffu)
      throw std::invalid_argument("server block_tracks must be a multiple of chunk_tracks");
    if (threads_ > kWindowThreads || threads_ % 32 != 0 || threads_ < 32)
      throw std::invalid_argument("server team_size must be a multiple of 32 up to 640");
    check(cudaGetDevice(&device_), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_), "SM count");
    max_window_ = windowed_max_bins(device_);
    if (max_window_ <= 0) throw server_cuda_error("windowed radio kernel does not fit on this device");
    block_bytes_ = kGranule + track_capacity(block_tracks_) * kTrackDoubles * sizeof(double);
    if (options.budget_bytes < block_bytes_)
      throw std::invalid_argument("server budget is smaller than one kinematics block");
    arena_.reserve(options.budget_bytes);
    check(cudaStreamCreateWithFlags(&compute_, cudaStreamNonBlocking), "stream");
    check(cudaStreamCreateWithFlags(&admit_, cudaStreamNonBlocking), "stream");
    check(cudaStreamCreateWithFlags(&fetch_, cudaStreamNonBlocking), "stream");
    check(cudaMalloc(&next_item_, 64 * sizeof(unsigned)), "work counters");
    epoch_ = std::chrono::steady_clock::now();
    scheduler_ = std::thread([this] { run(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    work_cv_.notify_all();
    memory_cv_.notify_all();
    done_cv_.notify_all();
    if (scheduler_.joinable()) scheduler_.join();
    int previous = -1;
    if (cudaGetDevice(&previous) != cudaSuccess || previous == device_) previous = -1;
    if (previous >= 0) cudaSetDevice(device_);
    cudaStreamSynchronize(compute_);
    for (auto& r : inflight_) cudaEventDestroy(r.done);
    for (auto e : spare_events_) cudaEventDestroy(e);
    for (auto& kv : events_)
      for (auto& b : kv.second->blocks)
        if (b.ingested) cudaEventDestroy(b.ingested);
    cudaStreamDestroy(compute_);
    cudaStreamDestroy(admit_);
    cudaStreamDestroy(fetch_);
    cudaFree(next_item_);
    if (deferred_) cudaFree(deferred_);
    arena_.free_all();
    if (previous >= 0) cudaSetDevice(previous);
  }

  uint64_t open(c8r_config const& config, int timeout_ms) {
    DeviceGuard guard(device_);
    double const opened = now();
    if (!config.enabled) throw std::invalid_argument("served radio event must be enabled");
    if (c8r_config_validate(&config) != C8R_OK) throw std::invalid_argument(c8r_last_global_error());
    if (config.precision > C8R_PRECISION_MIXED)
      throw std::invalid_argument("served radio events take FP64 or mixed precision");
    auto ev = std::make_unique<ServedEvent>();
    ev->open_s = opened;
    ev->fixed = config.deterministic != 0;
    ev->diagnostics = config.track_diagnostics != 0;
    ev->precision = config.precision == C8R_PRECISION_MIXED ? Precision::kMixed : Precision::kFP64;
    ev->limit = config.fixed_point_field_limit_v_per_m;
    if (config.coreas_enabled)
      ev->snapshots[0].assign(config.coreas_observers, config.coreas_observers + config.coreas_observer_count);
    if (config.zhs_enabled)
      ev->snapshots[1].assign(config.zhs_observers, config.zhs_observers + config.zhs_observer_count);
    auto const& p = config.propagation;
    bool const homogeneous = p.homogeneous_refractive_index > 0.;
    // host images of the resident part
    std::vector<ObserverCache> caches[2];
    uint64_t largest = 0;
    for (int a = 0; a < 2; ++a) {
      std::size_t offset = 0;
      for (auto const& s : ev->snapshots[a]) {
        caches[a].push_back(make_observer_cache(
            s, a, homogeneous, p.minimum_height_m, p.inverse_step_per_m,
            [&](uint64_t i) { return make_double2(p.refractivity[i], p.integrated_refractivity[i]); },
            ev->fixed, ev->limit, config.count_samples != 0, offset));
        offset += static_cast<std::size_t>(s.number_of_bins);
        largest = std::max<uint64_t>(largest, s.number_of_bins);
      }
      ev->bins[a] = offset;
      ev->observers[a] = static_cast<uint32_t>(caches[a].size());
    }
    ev->window = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(largest, max_window_)));
    std::vector<double2> table;
    if (!homogeneous) {
      table.resize(p.table_size);
      for (std::size_t i = 0; i < p.table_size; ++i)
        table[i] = make_double2(p.refractivity[i], p.integrated_refractivity[i]);
    }
    // resident layout: counters | caches CoREAS | caches ZHS | table | traces CoREAS | traces ZHS
    std::size_t const counters_off = 0;
    std::size_t const caches_off[2] = {round_up(sizeof(DeviceCounters)),
                                       round_up(sizeof(DeviceCounters)) +
                                           round_up(caches[0].size() * sizeof(ObserverCache))};
    std::size_t const table_off = caches_off[1] + round_up(caches[1].size() * sizeof(ObserverCache));
    std::size_t const traces_off[2] = {table_off + round_up(table.size() * sizeof(double2)),
                                       table_off + round_up(table.size() * sizeof(double2)) +
                                           round_up(3 * ev->bins[0] * sizeof(long long))};
    std::size_t const bytes = traces_off[1] + round_up(3 * ev->bins[1] * sizeof(long long));

    std::unique_lock<std::mutex> lock(mu_);
    rethrow_failure();
    auto const deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
    char* memory = nullptr;
    char* block = nullptr;
    for (;;) {
      memory = arena_.allocate(bytes);
      if (memory) {
        block = arena_.allocate(block_bytes_);
        if (block) break;
        arena_.release(memory, bytes);
        memory = nullptr;
      }
      if (stop_) throw std::logic_error("radio server is shutting down");
      if (timeout_ms < 0) {
        memory_cv_.wait(lock);
      } else if (memory_cv_.wait_until(lock, deadline) == std::cv_status::timeout) {
        memory = arena_.allocate(bytes);
        if (memory) {
          block = arena_.allocate(block_bytes_);
          if (block) break;
          arena_.release(memory, bytes);
        }
        throw timeout_error("radio event not admitted within the timeout (server budget full)");
      }
      rethrow_failure();
    }
    uint64_t const id = ++last_id_;
    ++stats_.events_admitted;
    ++stats_.blocks_allocated;
    lock.unlock();

    ev->id = id;
    ev->memory = memory;
    ev->bytes = bytes;
    ev->counters = reinterpret_cast<DeviceCounters*>(memory + counters_off);
    for (int a = 0; a < 2; ++a) {
      ev->caches[a] = reinterpret_cast<ObserverCache*>(memory + caches_off[a]);
      if (ev->fixed)
        ev->fixed_traces[a] = reinterpret_cast<unsigned long long*>(memory + traces_off[a]);
      else
        ev->float_traces[a] = reinterpret_cast<double*>(memory + traces_off[a]);
    }
    Propagation& prop = ev->propagation;
    prop.homogeneous = p.homogeneous_refractive_index;
    prop.min_height = p.minimum_height_m;
    prop.max_height = p.maximum_height_m;
    prop.step = p.step_m;
    prop.inv_step = p.inverse_step_per_m;
    prop.slope_n_lower = p.slope_refractivity_lower;
    prop.slope_i_lower = p.slope_integrated_refractivity_lower;
    prop.slope_n_upper = p.slope_refractivity_upper;
    prop.slope_i_upper = p.slope_integrated_refractivity_upper;
    prop.table_size = p.table_size;
    prop.refinement = config.zhs_subtrack_refinement;
    prop.table = homogeneous ? nullptr : reinterpret_cast<double2*>(memory + table_off);
    {
      std::vector<ObserverCache> all(caches[0]);
      all.insert(all.end(), caches[1].begin(), caches[1].end());
      Destination d{};
      ev->terms.enabled = shared_destination(all.data(), all.size(), d) ? 1 : 0;
      ev->terms.propagation = prop;
      ev->terms.destination = d;
    }
    Block b = make_block(block);
    try {
      check(cudaMemsetAsync(memory, 0, bytes, admit_), "server admission");
      for (int a = 0; a < 2; ++a)
        if (!caches[a].empty())
          check(cudaMemcpyAsync(ev->caches[a], caches[a].data(), caches[a].size() * sizeof(ObserverCache),
                                cudaMemcpyHostToDevice, admit_),
                "server admission");
      if (!table.empty())
        check(cudaMemcpyAsync(const_cast<double2*>(prop.table), table.data(), table.size() * sizeof(double2),
                              cudaMemcpyHostToDevice, admit_),
              "server admission");
      check(cudaMemsetAsync(b.slot, 0, sizeof(unsigned long long), admit_), "server admission");
      check(cudaStreamSynchronize(admit_), "server admission");
    } catch (...) {
      std::lock_guard<std::mutex> guard(mu_);
      if (b.ingested) cudaEventDestroy(b.ingested);
      arena_.release(block, block_bytes_);
      arena_.release(memory, bytes);
      memory_cv_.notify_all();
      throw;
    }
    ev->blocks.push_back(b);
    ev->admitted_s = now();
    lock.lock();
    events_[id] = std::move(ev);
    return id;
  }

  void add_device(uint64_t id, c8r_lepton_transport_record const* records, std::size_t count,
                  std::size_t extent, cudaStream_t stream) {
    DeviceGuard guard(device_);
    if (count > extent) throw std::out_of_range("radio track count exceeds input view");
    if (count != 0 && records == nullptr) throw std::invalid_argument("null device radio track input");
    std::unique_lock<std::mutex> lock(mu_);
    rethrow_failure();
    ServedEvent& ev = find(id);
    if (ev.state != EventState::kOpen) throw std::logic_error("radio event already closed");
    std::size_t done = 0;
    while (done < count) {
      Block* b = ev.blocks.empty() || ev.blocks.back().sealed ? nullptr : &ev.blocks.back();
      if (b == nullptr) {
        char* memory = nullptr;
        while ((memory = arena_.allocate(block_bytes_)) == nullptr) {
          if (stop_) throw std::logic_error("radio server is shutting down");
          memory_cv_.wait(lock);
          rethrow_failure();
        }
        ++stats_.blocks_allocated;
        ev.blocks.push_back(make_block(memory));
        b = &ev.blocks.back();
        check(cudaMemsetAsync(b->slot, 0, sizeof(unsigned long long), stream), "block slot clear");
      }
      std::size_t const n = std::min<std::size_t>(count - done, block_tracks_ - b->records);
      check(launch_ingest(records + done, n, b->tracks, block_tracks_, b->slot, ev.counters,
                          ev.diagnostics, ev.terms, stream),
            "server ingest launch");
      check(cudaEventRecord(b->ingested, stream), "server ingest event");
      b->records += n;
      ev.records += n;
      done += n;
      if (b->records == block_tracks_) {
        seal(*b);
        work_cv_.notify_all();
      }
    }
  }

  void close(uint64_t id) {
    DeviceGuard guard(device_);
    std::lock_guard<std::mutex> lock(mu_);
    rethrow_failure();
    ServedEvent& ev = find(id);
    if (ev.state != EventState::kOpen) throw std::logic_error("radio event already closed");
    if (!ev.blocks.empty() && !ev.blocks.back().sealed) {
      Block& b = ev.blocks.back();
      if (b.records == 0) {  // never written: nothing on the GPU reads it
        cudaEventDestroy(b.ingested);
        arena_.release(b.memory, block_bytes_);
        ev.blocks.pop_back();
        memory_cv_.notify_all();
      } else {
        seal(b);
      }
    }
    ev.state = EventState::kClosed;
    ev.closed_s = now();
    work_cv_.notify_all();
  }

  void wait(uint64_t id, int timeout_ms) {
    std::unique_lock<std::mutex> lock(mu_);
    auto done = [&] {
      if (!failure_.empty()) return true;
      return find(id).state == EventState::kComplete;
    };
    find(id);
    if (timeout_ms < 0) {
      done_cv_.wait(lock, done);
    } else if (!done_cv_.wait_for(lock, std::chrono::milliseconds(timeout_ms), done)) {
      throw timeout_error("radio event not complete within the timeout");
    }
    rethrow_failure();
  }

  // Copies traces (fixed: long long, else decoded doubles) and releases the event.
  void fetch(uint64_t id, void* coreas, void* zhs, bool fixed_out, c8r_counters* counters,
             c8r_server_event_info* info) {
    DeviceGuard guard(device_);
    std::unique_lock<std::mutex> lock(mu_);
    ServedEvent& ev = find(id);
    if (ev.fetching) throw std::logic_error("radio event already being fetched");
    done_cv_.wait(lock, [&] { return !failure_.empty() || ev.state == EventState::kComplete; });
    rethrow_failure();
    if (fixed_out && !ev.fixed) throw std::logic_error("fixed radio snapshot unavailable/already committed");
    ev.fetching = true;
    lock.unlock();
    DeviceCounters host{};
    std::vector<long long> staging;
    try {
      std::lock_guard<std::mutex> copy_lock(fetch_mu_);
      check(cudaMemcpyAsync(&host, ev.counters, sizeof host, cudaMemcpyDeviceToHost, fetch_), "server fetch");
      for (int a = 0; a < 2; ++a) {
        void* out = a == 0 ? coreas : zhs;
        std::size_t const values = 3 * ev.bins[a];
        if (values == 0 || out == nullptr) continue;
        void const* src = ev.fixed ? static_cast<void const*>(ev.fixed_traces[a])
                                   : static_cast<void const*>(ev.float_traces[a]);
        if (ev.fixed && !fixed_out) {
          staging.resize(values);
          check(cudaMemcpyAsync(staging.data(), src, values * sizeof(long long), cudaMemcpyDeviceToHost, fetch_),
                "server fetch");
          check(cudaStreamSynchronize(fetch_), "server fetch");
          decode(ev, a, staging.data(), static_cast<double*>(out));
        } else {
          check(cudaMemcpyAsync(out, src, values * sizeof(double), cudaMemcpyDeviceToHost, fetch_),
                "server fetch");
        }
      }
      check(cudaStreamSynchronize(fetch_), "server fetch");
    } catch (...) {
      lock.lock();
      ev.fetching = false;
      throw;
    }
    if (counters) std::memcpy(counters, &host, sizeof host);
    if (info) {
      info->records = ev.records;
      info->coreas_observers = ev.observers[0];
      info->zhs_observers = ev.observers[1];
      info->rounds = ev.rounds;
      info->open_s = ev.open_s;
      info->admitted_s = ev.admitted_s;
      info->closed_s = ev.closed_s;
      info->completed_s = ev.completed_s;
    }
    lock.lock();
    arena_.release(ev.memory, ev.bytes);
    events_.erase(id);
    memory_cv_.notify_all();
    if (!fixed_out && ev_overflowed(host))
      throw std::runtime_error("radio fixed-point accumulator overflowed; increase fixed_point_field_limit_V_per_m");
  }

  void stats(c8r_server_stats& out) {
    std::lock_guard<std::mutex> lock(mu_);
    out = stats_;
    out.arena_bytes = arena_.size();
    out.arena_used_bytes = arena_.used();
    out.arena_peak_bytes = arena_.peak();
  }

 private:
  static bool ev_overflowed(DeviceCounters const& c) { return c.fixed_point_overflows != 0; }

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - epoch_).count();
  }

  void rethrow_failure() const {
    if (!failure_.empty()) throw server_cuda_error(failure_);
  }

  ServedEvent& find(uint64_t id) {
    auto it = events_.find(id);
    if (it == events_.end()) throw std::invalid_argument("unknown radio event");
    return *it->second;
  }

  Block make_block(char* memory) {
    Block b;
    b.memory = memory;
    b.slot = reinterpret_cast<unsigned long long*>(memory);
    b.tracks = reinterpret_cast<double*>(memory + kGranule);
    check(cudaEventCreateWithFlags(&b.ingested, cudaEventDisableTiming), "server event");
    return b;
  }

  void seal(Block& b) {
    b.sealed = true;
    b.chunks = static_cast<uint32_t>((b.records + chunk_tracks_ - 1) / chunk_tracks_);
  }

  // downloadSet's decode (RadioAccumulator.inl:849-898), value x factor per observer.
  static void decode(ServedEvent const& ev, int a, long long const* in, double* out) {
    std::size_t const total = ev.bins[a];
    std::size_t offset = 0;
    for (auto const& s : ev.snapshots[a]) {
      double const f = decode_factor(s, a, ev.limit);
      std::size_t const n = static_cast<std::size_t>(s.number_of_bins);
      for (int row = 0; row < 3; ++row)
        for (std::size_t i = 0; i < n; ++i)
          out[row * total + offset + i] = static_cast<double>(in[row * total + offset + i]) * f;
      offset += n;
    }
  }

  // ------------------------------------------------------------ scheduler
  void run() {
    std::unique_lock<std::mutex> lock(mu_);
    try {
      check(cudaSetDevice(device_), "cudaSetDevice");
      for (;;) {
        retire_finished();
        complete_finished();
        if (stop_ && inflight_.empty()) break;
        if (inflight_.size() >= 2 || stop_) {
          if (inflight_.empty()) break;
          wait_front(lock);
          continue;
        }
        std::vector<Slice> slices = build_round();
        if (slices.empty()) {
          if (!inflight_.empty()) {
            wait_front(lock);
          } else {
            work_cv_.wait_for(lock, std::chrono::milliseconds(20));
          }
          continue;
        }
        launch(slices);
      }
    } catch (std::exception const& e) {
      failure_ = std::string("radio server: ") + e.what();
    }
    memory_cv_.notify_all();
    done_cv_.notify_all();
  }

  void wait_front(std::unique_lock<std::mutex>& lock) {
    cudaEvent_t const done = inflight_.front().done;
    lock.unlock();
    cudaError_t const err = cudaEventSynchronize(done);
    lock.lock();
    check(err, "server round");
  }

  void retire_finished() {
    bool progress = false;
    while (!inflight_.empty()) {
      cudaError_t const err = cudaEventQuery(inflight_.front().done);
      if (err == cudaErrorNotReady) break;
      check(err, "server round");
      retired_round_ = inflight_.front().id;
      spare_events_.push_back(inflight_.front().done);
      inflight_.pop_front();
      progress = true;
    }
    if (!progress) return;
    for (auto& kv : events_) {
      auto& blocks = kv.second->blocks;
      while (!blocks.empty()) {
        Block& b = blocks.front();
        if (!b.sealed || b.next_chunk != b.chunks || b.last_round > retired_round_) break;
        cudaEventDestroy(b.ingested);
        arena_.release(b.memory, block_bytes_);
        blocks.pop_front();
      }
    }
    memory_cv_.notify_all();
  }

  void complete_finished() {
    bool any = false;
    for (auto& kv : events_) {
      ServedEvent& ev = *kv.second;
      if (ev.state != EventState::kClosed || !ev.blocks.empty() || ev.last_round > retired_round_) continue;
      ev.state = EventState::kComplete;
      ev.completed_s = now();
      ++stats_.events_completed;
      any = true;
    }
    if (any) done_cv_.notify_all();
  }

  // Equal shares of round_pairs among the ready events (rotating start when
  // more slices than a launch holds), in chunk slices of their sealed blocks.
  std::vector<Slice> build_round() {
    std::vector<ServedEvent*> ready;
    for (auto& kv : events_) {
      ServedEvent& ev = *kv.second;
      if (ev.state == EventState::kComplete) continue;
      for (Block& b : ev.blocks) {
        if (b.sealed && b.next_chunk == b.chunks) continue;
        if (b.sealed) ready.push_back(&ev);
        break;
      }
    }
    std::vector<Slice> slices;
    if (ready.empty()) return slices;
    std::size_t const n = ready.size();
    std::size_t const start = rotate_++ % n;
    uint64_t const share = std::max<uint64_t>(1, round_pairs_ / n);
    for (std::size_t k = 0; k < n && slices.size() < static_cast<std::size_t>(kMaxEventsPerLaunch); ++k) {
      ServedEvent& ev = *ready[(start + k) % n];
      uint64_t const per_chunk =
          chunk_tracks_ * std::max<uint64_t>(1, static_cast<uint64_t>(ev.observers[0]) + ev.observers[1]);
      uint64_t give = share;
      for (Block& b : ev.blocks) {
        if (b.sealed && b.next_chunk == b.chunks) continue;
        if (!b.sealed) break;
        uint64_t const want = std::max<uint64_t>(1, (give + per_chunk - 1) / per_chunk);
        uint32_t const chunks = static_cast<uint32_t>(std::min<uint64_t>(b.chunks - b.next_chunk, want));
        slices.push_back({&ev, &b, b.next_chunk, chunks});
        b.next_chunk += chunks;
        uint64_t const used = chunks * per_chunk;
        give = used >= give ? 0 : give - used;
        if (give == 0 || slices.size() >= static_cast<std::size_t>(kMaxEventsPerLaunch)) break;
      }
    }
    return slices;
  }

  int ctas_per_sm(uint32_t window, bool fixed, Precision precision) {
    auto const key = std::make_tuple(window, fixed, static_cast<int>(precision));
    auto it = occupancy_.find(key);
    if (it != occupancy_.end()) return it->second;
    int const per_sm = windowed_ctas_per_sm(static_cast<int>(window), threads_, fixed, precision);
    if (per_sm <= 0) throw server_cuda_error("windowed radio kernel does not fit on this device");
    occupancy_[key] = per_sm;
    return per_sm;
  }

  // Grown after the rounds in flight on compute_ when a launch needs more.
  unsigned* deferred_lists(uint64_t entries) {
    if (deferred_entries_ < entries) {
      // twice what is asked: round sizes vary, and each growth synchronises
      // the device (the producers' ingest included)
      uint64_t const grown = std::max<uint64_t>(entries, 2 * deferred_entries_);
      check(cudaStreamSynchronize(compute_), "deferred list fence");
      if (deferred_) cudaFree(deferred_);
      deferred_ = nullptr;
      deferred_entries_ = 0;
      check(cudaMalloc(&deferred_, grown * sizeof(unsigned)), "deferred lists");
      deferred_entries_ = grown;
    }
    return deferred_;
  }

  void launch(std::vector<Slice> const& slices) {
    uint64_t const id = ++launched_rounds_;
    for (Slice const& s : slices) {
      if (s.block->waited) continue;
      check(cudaStreamWaitEvent(compute_, s.block->ingested, 0), "server ingest wait");
      s.block->waited = true;
    }
    for (int mode = 0; mode < 4; ++mode) {
      bool const fixed = mode < 2;
      Precision const precision = (mode & 1) ? Precision::kMixed : Precision::kFP64;
      for (int a = 0; a < 2; ++a) {
        WorkPlan plan;
        std::memset(&plan, 0, sizeof plan);
        plan.algorithm = a;
        uint32_t window = 1;
        std::vector<EventPlan> members;
        for (Slice const& s : slices) {
          ServedEvent const& ev = *s.event;
          if (ev.fixed != fixed || ev.precision != precision || ev.observers[a] == 0) continue;
          EventPlan e;
          std::memset(&e, 0, sizeof e);
          e.tracks = s.block->tracks;
          e.stride = block_tracks_;
          e.valid_tracks = s.block->slot;
          for (int k = 0; k < 2; ++k) {
            e.observers[k] = ev.caches[k];
            e.observer_count[k] = ev.observers[k];
            e.fixed[k] = ev.fixed_traces[k];
            e.floating[k] = ev.float_traces[k];
            e.total_bins[k] = ev.bins[k];
          }
          e.propagation = ev.propagation;
          e.counters = ev.counters;
          e.chunk_size = static_cast<uint32_t>(chunk_tracks_);
          e.chunks = s.chunks;
          e.first_track = static_cast<uint64_t>(s.chunk_begin) * chunk_tracks_;
          e.last_track = e.first_track + static_cast<uint64_t>(s.chunks) * chunk_tracks_;
          e.window = ev.window;
          e.precomputed = static_cast<uint32_t>(ev.terms.enabled);
          window = std::max(window, ev.window);
          members.push_back(e);
        }
        if (members.empty()) continue;
        unsigned* const counter = next_item_ + (stats_.launches % 64);
        plan.window = window;
        plan.next_item = counter;
        uint64_t ctas = static_cast<uint64_t>(ctas_per_sm(window, fixed, precision)) * sms_;
        // the last slice ends the round's work list on short items
        for (std::size_t m = 0; m < members.size(); ++m)
          append_work(plan, members[m], ctas, m + 1 == members.size());
        uint64_t const items = plan.total_items;
        if (ctas > items) ctas = items;
        plan.deferred_stride = deferred_list_stride(plan);
        attach_deferred(plan, deferred_lists(deferred_words(plan, ctas, fixed)), ctas, fixed);
        check(cudaMemsetAsync(counter, 0, sizeof(unsigned), compute_), "server work counter");
        check(launch_windowed(plan, fixed, precision, static_cast<int>(ctas), threads_, compute_),
              "server windowed launch");
        ++stats_.launches;
        stats_.work_items += items;
      }
    }
    cudaEvent_t done = nullptr;
    if (!spare_events_.empty()) {
      done = spare_events_.back();
      spare_events_.pop_back();
    } else {
      check(cudaEventCreateWithFlags(&done, cudaEventDisableTiming | cudaEventBlockingSync), "server event");
    }
    check(cudaEventRecord(done, compute_), "server round event");
    for (Slice const& s : slices) {
      s.block->last_round = id;
      if (s.event->last_round != id) {
        s.event->last_round = id;
        ++s.event->rounds;
      }
    }
    inflight_.push_back({id, done});
    ++stats_.rounds;
  }

  int device_ = 0, sms_ = 148, threads_ = kWindowThreads, max_window_ = 0;
  uint64_t block_tracks_ = 0, chunk_tracks_ = 0, round_pairs_ = 0;
  std::size_t block_bytes_ = 0;
  Arena arena_;
  cudaStream_t compute_ = nullptr, admit_ = nullptr, fetch_ = nullptr;
  unsigned* next_item_ = nullptr;
  unsigned* deferred_ = nullptr;  // the launches' per-CTA deferred-pair lists
  uint64_t deferred_entries_ = 0;
  std::chrono::steady_clock::time_point epoch_;
  std::mutex mu_, fetch_mu_;
  std::condition_variable work_cv_, memory_cv_, done_cv_;
  std::map<uint64_t, std::unique_ptr<ServedEvent>> events_;
  std::deque<Round> inflight_;
  std::vector<cudaEvent_t> spare_events_;
  std::map<std::tuple<uint32_t, bool, int>, int> occupancy_;
  uint64_t last_id_ = 0, launched_rounds_ = 0, retired_round_ = 0, rotate_ = 0;
  bool stop_ = false;
  std::string failure_;
  c8r_server_stats stats_{};
  std::thread scheduler_;
};

}  // namespace
}  // namespace c8r

// ============================================================== C boundary
struct c8r_server {
  c8r::Server* impl = nullptr;
};

namespace {

thread_local std::string g_server_error;

template <class F>
int server_guarded(F&& body) {
  try {
    body();
    return C8R_OK;
  } catch (c8r::timeout_error const& e) {
    g_server_error = e.what();
    return C8R_TIMEOUT;
  } catch (c8r::server_cuda_error const& e) {
    g_server_error = e.what();
    return C8R_CUDA_ERROR;
  } catch (std::invalid_argument const& e) {
    g_server_error = e.what();
    return C8R_INVALID_ARGUMENT;
  } catch (std::out_of_range const& e) {
    g_server_error = e.what();
    return C8R_OUT_OF_RANGE;
  } catch (std::length_error const& e) {
    g_server_error = e.what();
    return C8R_LENGTH_ERROR;
  } catch (std::logic_error const& e) {
    g_server_error = e.what();
    return C8R_LOGIC_ERROR;
  } catch (std::overflow_error const& e) {
    g_server_error = e.what();
    return C8R_OVERFLOW_ERROR;
  } catch (std::runtime_error const& e) {
    g_server_error = e.what();
    return C8R_RUNTIME_ERROR;
  } catch (std::bad_alloc const&) {
    g_server_error = "radio server allocation failed";
    return C8R_BAD_ALLOC;
  } catch (...) {
    g_server_error = "unknown radio server failure";
    return C8R_RUNTIME_ERROR;
  }
}

c8r::Server& server_of(c8r_server* s) {
  if (s == nullptr || s->impl == nullptr) throw std::invalid_argument("null radio server handle");
  return *s->impl;
}

}  // namespace

extern "C" {

int c8r_server_create(const c8r_server_options* options, c8r_server** server) {
  return server_guarded([&] {
    if (!options || !server) throw std::invalid_argument("null argument");
    *server = nullptr;
    auto handle = std::make_unique<c8r_server>();
    handle->impl = new c8r::Server(*options);
    *server = handle.release();
  });
}

void c8r_server_destroy(c8r_server* server) {
  if (!server) return;
  delete server->impl;
  delete server;
}

const char* c8r_server_last_error(const c8r_server* server) {
  (void)server;  // the message of this thread's last failed server call
  return g_server_error.c_str();
}

int c8r_server_open(c8r_server* server, const c8r_config* config, int timeout_ms, uint64_t* event) {
  return server_guarded([&] {
    if (!config || !event) throw std::invalid_argument("null argument");
    *event = server_of(server).open(*config, timeout_ms);
  });
}

int c8r_server_add_device(c8r_server* server, uint64_t event, const c8r_lepton_transport_record* records,
                          size_t count, size_t extent, void* stream) {
  return server_guarded([&] {
    server_of(server).add_device(event, records, count, extent, static_cast<cudaStream_t>(stream));
  });
}

int c8r_server_close(c8r_server* server, uint64_t event) {
  return server_guarded([&] { server_of(server).close(event); });
}

int c8r_server_wait(c8r_server* server, uint64_t event, int timeout_ms) {
  return server_guarded([&] { server_of(server).wait(event, timeout_ms); });
}

int c8r_server_fetch_fixed(c8r_server* server, uint64_t event, long long* coreas_xyz, long long* zhs_xyz,
                           c8r_counters* counters, c8r_server_event_info* info) {
  return server_guarded([&] { server_of(server).fetch(event, coreas_xyz, zhs_xyz, true, counters, info); });
}

int c8r_server_fetch(c8r_server* server, uint64_t event, double* coreas_xyz, double* zhs_xyz,
                     c8r_counters* counters, c8r_server_event_info* info) {
  return server_guarded([&] { server_of(server).fetch(event, coreas_xyz, zhs_xyz, false, counters, info); });
}

int c8r_server_get_stats(const c8r_server* server, c8r_server_stats* stats) {
  return server_guarded([&] {
    if (!stats) throw std::invalid_argument("null argument");
    server_of(const_cast<c8r_server*>(server)).stats(*stats);
  });
}

}  // extern "C"
