// shim_check.cpp — a reference-style C++ caller of include/c8radio.hpp, built
// by tests/test_shim.py with g++ against libc8radio.so.
//
//   shim_check host           checks that need no GPU: exception classes of
//                             validation, validate_fixed_radio,
//                             merge_radio_counters, CooperativeRadioMerge
//                             commit/take and decode_fixed_radio
//   shim_check gpu <dir>      reads a config and records from <dir> (written
//                             by the test), runs RadioAccumulator the way the
//                             reference's callers do, and writes the merged
//                             cooperative snapshot to <dir>/merged.bin for the
//                             test to compare with the oracle
//
// Prints "ok" and exits 0 when every check holds; otherwise prints the first
// failed check and exits 1.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <iterator>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "c8radio.hpp"

namespace {

using namespace c8radio;

int failures = 0;

void expect(bool ok, char const* what) {
  if (!ok && failures++ == 0) std::printf("FAILED: %s\n", what);
}

// Runs `f` and checks that it throws exactly class E (not a subclass it was
// not asked for: logic_error is the base of invalid_argument and friends).
template <class E>
void expect_throw(std::function<void()> const& f, char const* what) {
  try {
    f();
  } catch (E const& e) {
    if (typeid(e) == typeid(E)) return;
    expect(false, what);
    return;
  } catch (...) {
  }
  expect(false, what);
}

RadioObserverSnapshot observer(double x, double y, std::uint64_t bins) {
  RadioObserverSnapshot o{};
  o.position_m[0] = x;
  o.position_m[1] = y;
  o.position_m[2] = 0.;
  o.start_time_s = 0.;
  o.duration_s = static_cast<double>(bins - 1) * 1e-10;
  o.sample_rate_hz = 1e10;
  o.number_of_bins = bins;
  return o;
}

RadioConfig small_config() {
  RadioConfig c;
  c.enabled_ = true;
  c.propagation_.homogeneousRefractiveIndex_ = 1.0003;
  c.coreasObservers_ = {observer(10., 0., 8), observer(0., 20., 4)};
  c.zhsObservers_ = c.coreasObservers_;
  return c;
}

FixedRadioSnapshot snapshot(RadioConfig const& c, CooperativeEndpoint endpoint, std::int64_t base) {
  FixedRadioSnapshot s;
  s.showerIdentity_ = "shower-1";
  s.endpoint_ = endpoint;
  s.config_ = c;
  s.coreas_.resize(3 * 12);
  s.zhs_.resize(3 * 12);
  for (std::size_t i = 0; i < s.coreas_.size(); ++i) {
    s.coreas_[i] = base + static_cast<std::int64_t>(i);
    s.zhs_[i] = -base - static_cast<std::int64_t>(i);
  }
  s.counters_.coreas_contributions = 5;
  s.counters_.valid_tracks = 2;
  s.counters_.maximum_segment_length_m = static_cast<double>(base);
  return s;
}

void host_checks() {
  RadioConfig const c = small_config();

  // RadioAccumulator::validate through projectedDeviceBytes
  RadioConfig bad = c;
  bad.zhsSubtrackRefinement_ = 0;
  expect_throw<std::invalid_argument>([&] { RadioAccumulator::projectedDeviceBytes(bad); },
                                      "refinement 0 is std::invalid_argument");
  expect(RadioAccumulator::projectedDeviceBytes(c) > 0, "projected bytes of a valid config");

  // validate_fixed_radio
  auto good = snapshot(c, CooperativeEndpoint::Cuda, 100);
  validate_fixed_radio(good);
  auto s = good;
  s.showerIdentity_.clear();
  expect_throw<std::invalid_argument>([&] { validate_fixed_radio(s); }, "empty identity rejected");
  s = good;
  s.counters_.fixed_point_overflows = 1;
  expect_throw<std::invalid_argument>([&] { validate_fixed_radio(s); }, "overflowed snapshot rejected");
  s = good;
  s.zhs_.pop_back();
  expect_throw<std::invalid_argument>([&] { validate_fixed_radio(s); }, "extent mismatch rejected");
  s = good;
  s.endpoint_ = static_cast<CooperativeEndpoint>(2);
  expect_throw<std::invalid_argument>([&] { validate_fixed_radio(s); }, "unknown endpoint rejected");
  s = good;
  s.config_.deterministic_ = false;
  expect_throw<std::invalid_argument>([&] { validate_fixed_radio(s); }, "floating snapshot rejected");

  // merge_radio_counters
  RadioCounters a{}, b{};
  a.zhs_subtracks = std::numeric_limits<unsigned long long>::max();
  b.zhs_subtracks = 1;
  expect_throw<std::overflow_error>([&] { merge_radio_counters(a, b); }, "counter overflow");
  a = RadioCounters{};
  b = RadioCounters{};
  b.track_length_m = std::numeric_limits<double>::infinity();
  expect_throw<std::overflow_error>([&] { merge_radio_counters(a, b); }, "nonfinite diagnostics");
  b.track_length_m = 2.;
  a.track_length_m = 3.;
  a.maximum_segment_length_m = 7.;
  b.maximum_segment_length_m = 4.;
  auto const m = merge_radio_counters(a, b);
  expect(m.track_length_m == 5. && m.maximum_segment_length_m == 7., "counter merge values");

  // CooperativeRadioMerge
  expect_throw<std::invalid_argument>([&] { CooperativeRadioMerge("", c); }, "empty merge identity");
  {
    CooperativeRadioMerge merge("shower-1", c);
    expect_throw<std::logic_error>([&] { merge.take(); }, "take before both endpoints");
    merge.commit(good);
    expect_throw<std::invalid_argument>([&] { merge.commit(good); }, "duplicate endpoint");
    auto other = snapshot(c, CooperativeEndpoint::OpenMP, 7);
    auto wrong = other;
    wrong.showerIdentity_ = "shower-2";
    expect_throw<std::invalid_argument>([&] { merge.commit(wrong); }, "other identity");
    wrong = other;
    wrong.config_.fixedPointFieldLimitVPerM_ = 2.;
    expect_throw<std::invalid_argument>([&] { merge.commit(wrong); }, "other physics");
    wrong = other;
    wrong.config_.coreasObservers_[1].start_time_s = 1e-9;
    wrong.config_.zhsObservers_[1].start_time_s = 1e-9;
    expect_throw<std::invalid_argument>([&] { merge.commit(wrong); }, "other observers");
    wrong = other;
    wrong.coreas_[5] = std::numeric_limits<std::int64_t>::max();
    expect_throw<std::overflow_error>([&] { merge.commit(wrong); }, "bin overflow");
    wrong = other;
    wrong.counters_.valid_tracks = std::numeric_limits<unsigned long long>::max();
    expect_throw<std::overflow_error>([&] { merge.commit(wrong); }, "counter overflow in commit");
    merge.commit(other);  // the rejected commits changed nothing
    auto const merged = merge.take();
    bool sum_ok = merged.endpoint_ == CooperativeEndpoint::Cuda && merged.showerIdentity_ == "shower-1";
    for (std::size_t i = 0; i < merged.coreas_.size(); ++i)
      sum_ok = sum_ok && merged.coreas_[i] == good.coreas_[i] + other.coreas_[i] &&
               merged.zhs_[i] == good.zhs_[i] + other.zhs_[i];
    sum_ok = sum_ok && merged.counters_.coreas_contributions == 10 && merged.counters_.valid_tracks == 4 &&
             merged.counters_.maximum_segment_length_m == 100.;
    expect(sum_ok, "merged traces and counters are the checked sums");
    expect_throw<std::logic_error>([&] { merge.take(); }, "second take");
    expect_throw<std::logic_error>([&] { merge.commit(other); }, "commit after take");

    // decode_fixed_radio: int64 x limit / (2^62 factor), factor fs for ZHS
    auto const w = decode_fixed_radio(merged);
    double const unit = 1. / 4611686018427387904.0;
    expect(w.coreas_.size() == 2 && w.coreas_[0].x_.size() == 8 && w.coreas_[1].z_.size() == 4,
           "decoded shape");
    expect(w.coreas_[0].y_[3] == static_cast<double>(merged.coreas_[12 + 3]) * unit &&
               w.zhs_[1].x_[2] == static_cast<double>(merged.zhs_[8 + 2]) * (1. / (4611686018427387904.0 * 1e10)),
           "decoded values");
  }
}

// ---------------------------------------------------------------- GPU
std::vector<char> slurp(std::string const& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot read " + path);
  return std::vector<char>((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
}

template <class T>
std::vector<T> read_array(std::string const& path) {
  auto const bytes = slurp(path);
  std::vector<T> out(bytes.size() / sizeof(T));
  std::memcpy(out.data(), bytes.data(), out.size() * sizeof(T));
  return out;
}

void check_cuda(cudaError_t err, char const* what) {
  if (err != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(err));
}

void gpu_accumulators(std::string const& dir, RadioConfig const& config,
                      std::vector<LeptonTransportRecord> const& records, LeptonTransportRecord const* device,
                      cudaStream_t stream);

void gpu_checks(std::string const& dir) {
  // config.bin: 9 propagation doubles, limit; observers.bin; table.bin (n-1 | integral); records.bin
  auto const scalars = read_array<double>(dir + "/config.bin");
  auto const observers = read_array<RadioObserverSnapshot>(dir + "/observers.bin");
  auto const table = read_array<double>(dir + "/table.bin");
  auto const records = read_array<LeptonTransportRecord>(dir + "/records.bin");
  RadioConfig config;
  config.enabled_ = true;
  auto& p = config.propagation_;
  p.homogeneousRefractiveIndex_ = scalars[0];
  p.minimumHeightM_ = scalars[1];
  p.maximumHeightM_ = scalars[2];
  p.stepM_ = scalars[3];
  p.inverseStepPerM_ = scalars[4];
  p.slopeRefractivityLower_ = scalars[5];
  p.slopeIntegratedRefractivityLower_ = scalars[6];
  p.slopeRefractivityUpper_ = scalars[7];
  p.slopeIntegratedRefractivityUpper_ = scalars[8];
  config.fixedPointFieldLimitVPerM_ = scalars[9];
  p.refractivity_.assign(table.begin(), table.begin() + table.size() / 2);
  p.integratedRefractivity_.assign(table.begin() + table.size() / 2, table.end());
  config.coreasObservers_ = observers;
  config.zhsObservers_ = observers;
  config.kernel_ = C8R_KERNEL_WINDOWED;

  cudaStream_t stream = nullptr;
  check_cuda(cudaStreamCreate(&stream), "stream");
  LeptonTransportRecord* device = nullptr;
  std::size_t const n = records.size();
  check_cuda(cudaMalloc(reinterpret_cast<void**>(&device), n * sizeof(LeptonTransportRecord)), "malloc");
  check_cuda(cudaMemcpy(device, records.data(), n * sizeof(LeptonTransportRecord), cudaMemcpyHostToDevice),
             "upload");
  // the accumulators live in gpu_accumulators: destroyed (their queued work
  // completed) before their stream and records are
  gpu_accumulators(dir, config, records, device, stream);
  cudaFree(device);
  cudaStreamDestroy(stream);
}

void gpu_accumulators(std::string const& dir, RadioConfig const& config,
                      std::vector<LeptonTransportRecord> const& records, LeptonTransportRecord const* device,
                      cudaStream_t stream) {
  std::size_t const n = records.size(), half = n / 2;

  // endpoint "Cuda": the resident-record path (LeptonCascade.inl:81-83), first half
  RadioAccumulator gpu;
  gpu.initialize(config, {}, stream);
  expect_throw<std::logic_error>([&] { gpu.initialize(config, {}, stream); }, "second initialize");
  expect_throw<std::out_of_range>([&] { gpu.accumulateLeptonTracks(device, half + 1, half, stream); },
                                  "count beyond the view's extent");
  expect_throw<std::invalid_argument>([&] { gpu.accumulateLeptonTracks(device, half, n, reinterpret_cast<void*>(1)); },
                                      "another execution instance");
  gpu.accumulateLeptonTracks(device, half, n, stream);
  expect_throw<std::invalid_argument>([&] { gpu.downloadFixed("", CooperativeEndpoint::Cuda, stream); },
                                      "empty identity, nothing sealed");
  expect_throw<std::invalid_argument>(
      [&] { gpu.downloadFixed("shower-7", static_cast<CooperativeEndpoint>(3), stream); }, "unknown endpoint");
  auto const a = gpu.downloadFixed("shower-7", CooperativeEndpoint::Cuda, stream);
  validate_fixed_radio(a);
  expect_throw<std::logic_error>([&] { gpu.downloadFixed("shower-7", CooperativeEndpoint::Cuda); },
                                 "second downloadFixed");
  expect_throw<std::logic_error>([&] { gpu.download(); }, "download after downloadFixed");
  expect_throw<std::logic_error>([&] { gpu.accumulateLeptonTracks(device, half, n); },
                                 "tracks after the endpoint was committed");
  gpu.reset(stream);  // a reset endpoint can export again
  gpu.accumulateLeptonTracks(device, 1, n, stream);
  (void)gpu.downloadFixed("shower-8", CooperativeEndpoint::Cuda);

  // endpoint "OpenMP": host records (copied before return), second half
  RadioAccumulator host;
  host.initialize(config, {}, stream);
  host.enqueueHostLeptonTracks(records.data() + half, n - half, stream);
  auto const b = host.downloadFixed("shower-7", CooperativeEndpoint::OpenMP, stream);

  CooperativeRadioMerge merge("shower-7", config);
  merge.commit(b);
  merge.commit(a);
  auto const merged = merge.take();
  expect(merged.endpoint_ == CooperativeEndpoint::OpenMP, "merged endpoint is the first commit's");

  // all tracks in one accumulator: download() decodes exactly what the merge holds
  RadioAccumulator whole;
  whole.initialize(config, {}, stream);
  whole.accumulateLeptonTracks(device, n, n, stream);
  auto const w = whole.download(stream);
  auto const d = decode_fixed_radio(merged);
  bool same = w.coreas_.size() == d.coreas_.size() && w.zhs_.size() == d.zhs_.size();
  for (std::size_t k = 0; same && k < w.coreas_.size(); ++k)
    same = w.coreas_[k].x_ == d.coreas_[k].x_ && w.coreas_[k].y_ == d.coreas_[k].y_ &&
           w.coreas_[k].z_ == d.coreas_[k].z_ && w.zhs_[k].x_ == d.zhs_[k].x_ && w.zhs_[k].z_ == d.zhs_[k].z_;
  expect(same, "download() equals the decoded cooperative merge");
  expect_throw<std::logic_error>([&] { whole.download(); }, "download twice");

  // fixed-point overflow: download throws runtime_error, downloadFixed rejects and seals
  RadioConfig tiny = config;
  tiny.fixedPointFieldLimitVPerM_ = 1e-300;
  RadioAccumulator over;
  over.initialize(tiny, {}, stream);
  over.accumulateLeptonTracks(device, n, n, stream);
  expect_throw<std::runtime_error>([&] { over.download(); }, "overflow at download");
  RadioAccumulator sealed;
  sealed.initialize(tiny, {}, stream);
  sealed.accumulateLeptonTracks(device, n, n, stream);
  expect_throw<std::invalid_argument>([&] { sealed.downloadFixed("shower-9", CooperativeEndpoint::Cuda); },
                                      "overflowed export rejected");
  expect_throw<std::logic_error>([&] { sealed.downloadFixed("shower-9", CooperativeEndpoint::Cuda); },
                                 "a failed export stays sealed");

  // IRadioBackend over the same accumulator type
  B200RadioBackend backend(config, {}, stream);
  expect(backend.gpuRadioEnabled(), "backend enabled");
  backend.enqueueRadioTracks(records.data(), n);
  auto const bw = backend.downloadRadioWaveforms();
  bool backend_same = bw.coreas_.size() == w.coreas_.size();
  for (std::size_t k = 0; backend_same && k < bw.coreas_.size(); ++k)
    backend_same = bw.coreas_[k].x_ == w.coreas_[k].x_ && bw.zhs_[k].y_ == w.zhs_[k].y_;
  expect(backend_same, "IRadioBackend waveforms equal the device-record path's");

  std::ofstream out(dir + "/merged.bin", std::ios::binary);
  out.write(reinterpret_cast<char const*>(merged.coreas_.data()),
            static_cast<std::streamsize>(merged.coreas_.size() * sizeof(std::int64_t)));
  out.write(reinterpret_cast<char const*>(merged.zhs_.data()),
            static_cast<std::streamsize>(merged.zhs_.size() * sizeof(std::int64_t)));
  out.write(reinterpret_cast<char const*>(&merged.counters_), sizeof(merged.counters_));
}

}  // namespace

int main(int argc, char** argv) {
  try {
    std::string const mode = argc > 1 ? argv[1] : "host";
    if (mode == "host") {
      host_checks();
    } else if (mode == "gpu" && argc > 2) {
      gpu_checks(argv[2]);
    } else {
      std::printf("usage: shim_check host | gpu <dir>\n");
      return 2;
    }
  } catch (std::exception const& e) {
    std::printf("FAILED: unexpected %s\n", e.what());
    return 1;
  }
  if (failures) return 1;
  std::printf("ok\n");
  return 0;
}
