// spool.cu — RadioTrackSpool version 1 (completed host tracks on disk) and
// its replay into an accumulator.
//
// Format (corsika/kokkos/radio/RadioTrackSpoolFormat.hpp:24-29,
// RadioTrackSpoolFormat.inl:11-92): a 32-byte header — the 16 bytes
// "C8_RADIO_TRACKS\0", version 1 and record size 140 as little-endian uint32,
// the record count as little-endian uint64 (all ones while the writer has not
// completed) — then one 140-byte record per track: pdg as uint32, start and
// end position, start and end direction (3 doubles each), start and end time,
// start and end kinetic energy and weight, every double as its little-endian
// IEEE-754 bit pattern.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "../../include/c8radio.h"

namespace c8r {
void set_global_error(char const* message);  // accumulator.cu
}

struct c8r_spool_writer {
  std::FILE* file = nullptr;
  uint64_t count = 0;
  bool completed = false;
};

struct c8r_spool_reader {
  std::FILE* file = nullptr;
  uint64_t count = 0;
  uint64_t consumed = 0;
};

namespace {

constexpr char kMagic[16] = {'C', '8', '_', 'R', 'A', 'D', 'I', 'O',
                             '_', 'T', 'R', 'A', 'C', 'K', 'S', '\0'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kRecordBytes = 17 * 8 + 4;
constexpr uint64_t kHeaderBytes = 32;
constexpr uint64_t kIncomplete = std::numeric_limits<uint64_t>::max();
constexpr double kElectronMassGeV = 5.109989e-4;  // corsika/kokkos/em/algorithms/TransportMass.hpp:20

// RadioTrackSpoolFormat.inl:11-13: every spool failure is a runtime_error.
void require(bool ok, char const* message) {
  if (!ok) throw std::runtime_error(message);
}

void put_u32(unsigned char* p, uint32_t v) {
  for (int i = 0; i < 4; ++i) p[i] = static_cast<unsigned char>((v >> (8 * i)) & 0xffu);
}
void put_u64(unsigned char* p, uint64_t v) {
  for (int i = 0; i < 8; ++i) p[i] = static_cast<unsigned char>((v >> (8 * i)) & 0xffu);
}
uint32_t get_u32(unsigned char const* p) {
  uint32_t v = 0;
  for (int i = 0; i < 4; ++i) v |= static_cast<uint32_t>(p[i]) << (8 * i);
  return v;
}
uint64_t get_u64(unsigned char const* p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; ++i) v |= static_cast<uint64_t>(p[i]) << (8 * i);
  return v;
}
void put_double(unsigned char* p, double v) {
  uint64_t bits;
  std::memcpy(&bits, &v, sizeof bits);
  put_u64(p, bits);
}
double get_double(unsigned char const* p) {
  uint64_t const bits = get_u64(p);
  double v;
  std::memcpy(&v, &bits, sizeof v);
  return v;
}

// radio_spool::validate, RadioTrackSpoolFormat.inl:52-66.
void validate(c8r_track_segment const& t) {
  require(t.pdg == 11 || t.pdg == -11, "Non-electron radio spool record");
  for (double const* c : {t.start_position_m, t.end_position_m, t.start_direction, t.end_direction})
    for (int axis = 0; axis < 3; ++axis) require(std::isfinite(c[axis]), "Non-finite radio spool coordinates");
  require(std::isfinite(t.start_time_s) && std::isfinite(t.end_time_s) &&
              std::isfinite(t.start_kinetic_energy_gev) && std::isfinite(t.end_kinetic_energy_gev) &&
              std::isfinite(t.weight),
          "Non-finite radio spool scalar");
  require(t.weight >= 0. && t.start_kinetic_energy_gev >= 0. && t.end_kinetic_energy_gev >= 0. &&
              t.end_time_s >= t.start_time_s,
          "Invalid radio spool energy, weight or time");
}

// radio_spool::write_track / read_track, RadioTrackSpoolFormat.inl:68-92.
void encode(c8r_track_segment const& t, unsigned char* p) {
  put_u32(p, static_cast<uint32_t>(t.pdg));
  p += 4;
  for (double const* c : {t.start_position_m, t.end_position_m, t.start_direction, t.end_direction})
    for (int axis = 0; axis < 3; ++axis, p += 8) put_double(p, c[axis]);
  for (double v : {t.start_time_s, t.end_time_s, t.start_kinetic_energy_gev, t.end_kinetic_energy_gev, t.weight}) {
    put_double(p, v);
    p += 8;
  }
}

c8r_track_segment decode(unsigned char const* p) {
  c8r_track_segment t;
  std::memset(&t, 0, sizeof t);
  uint32_t const pdg = get_u32(p);
  require(pdg == 11u || pdg == static_cast<uint32_t>(-11), "Non-electron radio spool record");
  t.pdg = pdg == 11u ? 11 : -11;
  p += 4;
  for (double* c : {t.start_position_m, t.end_position_m, t.start_direction, t.end_direction})
    for (int axis = 0; axis < 3; ++axis, p += 8) c[axis] = get_double(p);
  double* const scalars[5] = {&t.start_time_s, &t.end_time_s, &t.start_kinetic_energy_gev,
                              &t.end_kinetic_energy_gev, &t.weight};
  for (double* v : scalars) {
    *v = get_double(p);
    p += 8;
  }
  validate(t);
  return t;
}

// make_host_radio_record, HostRadioRecord.inl:11-31.
void to_record(c8r_track_segment const& s, c8r_lepton_transport_record& r) {
  if (s.pdg != 11 && s.pdg != -11)
    throw std::invalid_argument("only electron/positron tracks enter radio projection");
  std::memset(&r, 0, sizeof r);
  r.start.pid = r.end.pid = s.pdg;
  r.start.weight = r.end.weight = s.weight;
  r.start.time_s = s.start_time_s;
  r.end.time_s = s.end_time_s;
  r.start.energy_gev = s.start_kinetic_energy_gev + kElectronMassGeV;
  r.end.energy_gev = s.end_kinetic_energy_gev + kElectronMassGeV;
  for (int axis = 0; axis < 3; ++axis) {
    r.start.position_m[axis] = s.start_position_m[axis];
    r.end.position_m[axis] = s.end_position_m[axis];
    r.start.direction[axis] = s.start_direction[axis];
    r.end.direction[axis] = s.end_direction[axis];
  }
}

// RadioTrackSpoolReader::readBatch, RadioTrackSpoolReader.inl:31-41.
std::size_t read_batch(c8r_spool_reader& reader, c8r_track_segment* out, std::size_t maximum) {
  require(maximum > 0 && maximum <= 65536, "Invalid radio spool read batch");
  uint64_t const left = reader.count - reader.consumed;
  std::size_t const amount = static_cast<std::size_t>(left < maximum ? left : maximum);
  if (amount == 0) return 0;
  std::vector<unsigned char> bytes(amount * kRecordBytes);
  require(std::fread(bytes.data(), 1, bytes.size(), reader.file) == bytes.size(), "Truncated radio track spool");
  for (std::size_t i = 0; i < amount; ++i) out[i] = decode(bytes.data() + i * kRecordBytes);
  reader.consumed += amount;
  return amount;
}

template <class F>
int spool_guarded(F&& body) {
  try {
    body();
    return C8R_OK;
  } catch (std::invalid_argument const& e) {
    c8r::set_global_error(e.what());
    return C8R_INVALID_ARGUMENT;
  } catch (std::logic_error const& e) {
    c8r::set_global_error(e.what());
    return C8R_LOGIC_ERROR;
  } catch (std::runtime_error const& e) {
    c8r::set_global_error(e.what());
    return C8R_RUNTIME_ERROR;
  } catch (std::bad_alloc const&) {
    c8r::set_global_error("radio spool allocation failed");
    return C8R_BAD_ALLOC;
  } catch (...) {
    c8r::set_global_error("unknown radio spool failure");
    return C8R_RUNTIME_ERROR;
  }
}

}  // namespace

extern "C" {

// RadioTrackSpoolWriter::RadioTrackSpoolWriter, RadioTrackSpoolWriter.inl:11-21.
int c8r_spool_writer_create(const char* path, c8r_spool_writer** writer) {
  return spool_guarded([&] {
    if (!path || !writer) throw std::invalid_argument("null argument");
    *writer = nullptr;
    struct stat st;
    require(::stat(path, &st) != 0, "Radio track spool already exists");
    std::FILE* f = std::fopen(path, "wb");
    require(f != nullptr, "Cannot create radio track spool");
    unsigned char header[kHeaderBytes];
    std::memcpy(header, kMagic, sizeof kMagic);
    put_u32(header + 16, kVersion);
    put_u32(header + 20, kRecordBytes);
    put_u64(header + 24, kIncomplete);
    if (std::fwrite(header, 1, sizeof header, f) != sizeof header) {
      std::fclose(f);
      throw std::runtime_error("Cannot write radio track spool");
    }
    auto* w = new c8r_spool_writer;
    w->file = f;
    *writer = w;
  });
}

// RadioTrackSpoolWriter::append, RadioTrackSpoolWriter.inl:23-31 (each track validated first).
int c8r_spool_append(c8r_spool_writer* writer, const c8r_track_segment* tracks, size_t count) {
  return spool_guarded([&] {
    if (!writer) throw std::invalid_argument("null radio spool writer");
    if (count && !tracks) throw std::invalid_argument("null radio spool tracks");
    require(!writer->completed, "Cannot append to a completed radio track spool");
    unsigned char bytes[kRecordBytes];
    for (size_t i = 0; i < count; ++i) {
      require(writer->count < (kIncomplete - kHeaderBytes) / kRecordBytes, "Radio track spool size overflow");
      validate(tracks[i]);
      encode(tracks[i], bytes);
      require(std::fwrite(bytes, 1, sizeof bytes, writer->file) == sizeof bytes, "Cannot write radio track spool");
      ++writer->count;
    }
  });
}

// RadioTrackSpoolWriter::complete, RadioTrackSpoolWriter.inl:33-45: only a
// successful completion publishes the count.
int c8r_spool_complete(c8r_spool_writer* writer) {
  return spool_guarded([&] {
    if (!writer) throw std::invalid_argument("null radio spool writer");
    require(!writer->completed, "Radio track spool completed twice");
    require(std::fflush(writer->file) == 0, "Cannot flush radio track spool");
    require(std::fseek(writer->file, 24, SEEK_SET) == 0, "Cannot seek radio track spool");
    unsigned char count[8];
    put_u64(count, writer->count);
    require(std::fwrite(count, 1, sizeof count, writer->file) == sizeof count, "Cannot write radio track spool");
    int const closed = std::fclose(writer->file);
    writer->file = nullptr;
    require(closed == 0, "Cannot close radio track spool");
    writer->completed = true;
  });
}

int c8r_spool_writer_count(const c8r_spool_writer* writer, uint64_t* count) {
  return spool_guarded([&] {
    if (!writer || !count) throw std::invalid_argument("null argument");
    *count = writer->count;
  });
}

void c8r_spool_writer_destroy(c8r_spool_writer* writer) {
  if (!writer) return;
  if (writer->file) std::fclose(writer->file);  // incomplete: the header keeps its sentinel
  delete writer;
}

// RadioTrackSpoolReader::RadioTrackSpoolReader, RadioTrackSpoolReader.inl:11-29.
int c8r_spool_reader_open(const char* path, c8r_spool_reader** reader, uint64_t* count) {
  return spool_guarded([&] {
    if (!path || !reader) throw std::invalid_argument("null argument");
    *reader = nullptr;
    std::FILE* f = std::fopen(path, "rb");
    require(f != nullptr, "Cannot read radio track spool");
    try {
      unsigned char header[kHeaderBytes];
      require(std::fread(header, 1, 16, f) == 16 && std::memcmp(header, kMagic, 16) == 0,
              "Invalid radio track spool magic");
      require(std::fread(header + 16, 1, 16, f) == 16, "Truncated radio track spool");
      require(get_u32(header + 16) == kVersion, "Unsupported radio track spool version");
      require(get_u32(header + 20) == kRecordBytes, "Invalid radio track spool record size");
      uint64_t const n = get_u64(header + 24);
      require(n != kIncomplete && n <= (kIncomplete - kHeaderBytes) / kRecordBytes,
              "Incomplete or oversized radio track spool");
      struct stat st;
      require(::stat(path, &st) == 0 &&
                  static_cast<uint64_t>(st.st_size) == kHeaderBytes + n * kRecordBytes,
              "Radio track spool length does not match its record count");
      auto* r = new c8r_spool_reader;
      r->file = f;
      r->count = n;
      *reader = r;
      if (count) *count = n;
    } catch (...) {
      std::fclose(f);
      throw;
    }
  });
}

int c8r_spool_read(c8r_spool_reader* reader, c8r_track_segment* tracks, size_t maximum, size_t* read) {
  return spool_guarded([&] {
    if (!reader || !read) throw std::invalid_argument("null argument");
    *read = 0;
    if (maximum && !tracks) throw std::invalid_argument("null radio spool tracks");
    *read = read_batch(*reader, tracks, maximum);
  });
}

int c8r_spool_reader_state(const c8r_spool_reader* reader, uint64_t* consumed, int* finished) {
  return spool_guarded([&] {
    if (!reader) throw std::invalid_argument("null radio spool reader");
    if (consumed) *consumed = reader->consumed;
    if (finished) *finished = reader->consumed == reader->count ? 1 : 0;
  });
}

void c8r_spool_reader_destroy(c8r_spool_reader* reader) {
  if (!reader) return;
  if (reader->file) std::fclose(reader->file);
  delete reader;
}

int c8r_track_records(const c8r_track_segment* tracks, size_t count, c8r_lepton_transport_record* records) {
  return spool_guarded([&] {
    if (count && (!tracks || !records)) throw std::invalid_argument("null argument");
    for (size_t i = 0; i < count; ++i) to_record(tracks[i], records[i]);
  });
}

// The replay of testRadioSpoolReplay.cpp:85-111 and HostRadioCollector::append
// (HostRadioCollector.inl:20-24): every remaining track, read in batches of
// `batch` (1..65536), converted and enqueued as host tracks.
int c8r_spool_replay(c8r_spool_reader* reader, c8r_accumulator* accumulator, size_t batch) {
  int status = C8R_OK;
  int const guard = spool_guarded([&] {
    if (!reader || !accumulator) throw std::invalid_argument("null argument");
    require(batch > 0 && batch <= 65536, "Invalid radio spool read batch");
    std::vector<c8r_track_segment> tracks(batch);
    std::vector<c8r_lepton_transport_record> records(batch);
    for (;;) {
      std::size_t const n = read_batch(*reader, tracks.data(), batch);
      if (n == 0) break;
      for (std::size_t i = 0; i < n; ++i) to_record(tracks[i], records[i]);
      status = c8r_enqueue_host(accumulator, records.data(), n);
      if (status != C8R_OK) {
        c8r::set_global_error(c8r_last_error(accumulator));
        return;
      }
    }
  });
  return guard != C8R_OK ? guard : status;
}

}  // extern "C"
