// tuning.cu — the persistent tuning cache: the autotuner's choice stored
// keyed by the device it was measured on, in the manner of the reference's
// c8-kokkos-tuning-v1 cache (corsika/kokkos/runtime/TuningCache.hpp:16-47,
// src/kokkos/runtime/TuningCache.cpp): a text file of key=value lines; a
// cache is used only when every key field equals the current device's, build's
// and workload's, and a malformed file is an error.
//
//   format=c8radio-b200-tuning-v1
//   device_name=, compute_capability=, multiprocessors=, driver_version=,
//   runtime_version=, library_version=, workload=
//   team_size=, track_tile_size=, observer_tile_size=   (0 = the default)
#include <cuda_runtime.h>

#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>

#include "../../include/c8radio.h"
#include "status.hpp"

namespace {

constexpr char kFormat[] = "c8radio-b200-tuning-v1";
thread_local std::string g_error;

std::map<std::string, std::string> current_key(std::string const& workload) {
  if (workload.empty() || workload.find('\n') != std::string::npos)
    throw std::invalid_argument("tuning workload label must be one non-empty line");
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) throw c8r::cuda_error("cudaGetDevice");
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) throw c8r::cuda_error("cudaGetDeviceProperties");
  int driver = 0, runtime = 0;
  cudaDriverGetVersion(&driver);
  cudaRuntimeGetVersion(&runtime);
  return {{"format", kFormat},
          {"device_name", prop.name},
          {"compute_capability", std::to_string(prop.major) + "." + std::to_string(prop.minor)},
          {"multiprocessors", std::to_string(prop.multiProcessorCount)},
          {"driver_version", std::to_string(driver)},
          {"runtime_version", std::to_string(runtime)},
          {"library_version", c8r_version()},
          {"workload", workload}};
}

std::string trim(std::string s) {
  std::size_t const b = s.find_first_not_of(" \t\r");
  if (b == std::string::npos) return {};
  std::size_t const e = s.find_last_not_of(" \t\r");
  return s.substr(b, e - b + 1);
}

// key=value lines; blank lines and '#' comments skipped; a line without '='
// or a repeated key is an error.
std::map<std::string, std::string> parse(std::string const& text) {
  std::map<std::string, std::string> fields;
  std::istringstream in(text);
  std::string line;
  while (std::getline(in, line)) {
    line = trim(line);
    if (line.empty() || line[0] == '#') continue;
    std::size_t const eq = line.find('=');
    if (eq == std::string::npos) throw std::runtime_error("invalid radio tuning-cache line without '='");
    std::string key = trim(line.substr(0, eq));
    if (key.empty() || !fields.emplace(key, trim(line.substr(eq + 1))).second)
      throw std::runtime_error("invalid or duplicate radio tuning-cache key");
  }
  return fields;
}

uint64_t parse_count(std::map<std::string, std::string> const& fields, std::string const& name) {
  auto const it = fields.find(name);
  if (it == fields.end()) throw std::runtime_error("radio tuning cache is missing field '" + name + "'");
  std::string const& text = it->second;
  if (text.empty() || text.size() > 19 || text.find_first_not_of("0123456789") != std::string::npos)
    throw std::runtime_error("radio tuning-cache field '" + name + "' is not a count");
  return std::stoull(text);
}

// A missing file is no match (an error when required); a malformed one is an
// error either way; both are decided before the device is queried.
void load(char const* path, char const* workload, bool require, c8r_tuning& out, int& matched) {
  matched = 0;
  if (path == nullptr || workload == nullptr) throw std::invalid_argument("null argument");
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    if (require) throw std::runtime_error(std::string("no radio tuning cache at ") + path);
    return;
  }
  std::ostringstream buffer;
  buffer << in.rdbuf();
  std::map<std::string, std::string> const fields = parse(buffer.str());
  std::map<std::string, std::string> const key = current_key(workload);
  for (auto const& [name, value] : key) {
    auto const it = fields.find(name);
    if (it == fields.end() || it->second != value) {
      if (require) throw std::runtime_error("radio tuning cache does not match this device, build or workload");
      return;
    }
  }
  c8r_tuning t{};
  t.team_size = parse_count(fields, "team_size");
  t.track_tile_size = parse_count(fields, "track_tile_size");
  t.observer_tile_size = parse_count(fields, "observer_tile_size");
  if (t.team_size > 640 || t.team_size % 32 != 0) throw std::runtime_error("radio tuning-cache team_size is invalid");
  out = t;
  matched = 1;
}

void store(char const* path, char const* workload, c8r_tuning const& t) {
  if (path == nullptr || workload == nullptr || path[0] == '\0') throw std::invalid_argument("null argument");
  if (t.team_size > 640 || t.team_size % 32 != 0) throw std::invalid_argument("radio tuning is invalid");
  std::map<std::string, std::string> const key = current_key(workload);
  std::string const temporary = std::string(path) + ".tmp";
  {
    std::ofstream out(temporary, std::ios::binary | std::ios::trunc);
    if (!out) throw std::runtime_error("cannot create radio tuning cache " + temporary);
    out << "format=" << key.at("format") << '\n';
    for (char const* name : {"device_name", "compute_capability", "multiprocessors", "driver_version",
                             "runtime_version", "library_version", "workload"})
      out << name << '=' << key.at(name) << '\n';
    out << "team_size=" << t.team_size << '\n'
        << "track_tile_size=" << t.track_tile_size << '\n'
        << "observer_tile_size=" << t.observer_tile_size << '\n';
    out.close();
    if (!out) throw std::runtime_error("failed while writing radio tuning cache " + temporary);
  }
  if (std::rename(temporary.c_str(), path) != 0) throw std::runtime_error(std::string("cannot replace ") + path);
}

}  // namespace

extern "C" {

int c8r_tuning_cache_load(const char* path, const char* workload, int require_match, c8r_tuning* tuning,
                          int* matched) {
  return c8r::guarded(&g_error, [&] {
    if (!tuning || !matched) throw std::invalid_argument("null argument");
    load(path, workload, require_match != 0, *tuning, *matched);
  });
}

int c8r_tuning_cache_store(const char* path, const char* workload, const c8r_tuning* tuning) {
  return c8r::guarded(&g_error, [&] {
    if (!tuning) throw std::invalid_argument("null argument");
    store(path, workload, *tuning);
  });
}

const char* c8r_tuning_cache_last_error(void) { return g_error.c_str(); }

}  // extern "C"
