// radio_device.cuh — device arithmetic of the radio projection (sm_100a).
//
// Every FP64 expression that decides a time bin, a branch or (in the FP64
// path) an amplitude is written with the reference's association order
// (corsika/detail/kokkos/radio/algorithms/RadioProjection.inl) and this file
// is compiled with -fmad=false, so no multiply-add is contracted: results are
// the IEEE-754 results the x86-64 host produces for the same source.
// Amplitudes take the type `Amp`: double for the FP64 drop-in, float for the
// mixed-precision path.
#pragma once

#include <cstdint>
#include <climits>

namespace c8r {

// corsika/kokkos/ScalarPhysicalConstants.hpp:18-20, RadioProjectionData.hpp:21-37
constexpr double kSpeedOfLight = 299792458.;
constexpr double kElementaryCharge = 1.6021766208e-19;
constexpr double kVacuumPermittivity = 8.8541878128e-12;
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kCoreasThreshold = 1.e-3;
constexpr double kHeadroom = 4611686018427387904.0;     // 2^62
constexpr double kSignedLimit = 9223372036854775808.0;  // 2^63
constexpr double kElectronMassGeV = 5.109989e-4;        // TransportMass.hpp:20

// Per-observer constants, derived on the host with the same IEEE operations
// the reference evaluates inline (destination bin of propagate, window end of
// add_sample, grid resolution and wavelength).
struct alignas(16) ObserverCache {
  double px, py, pz;
  double start_time;     // startTimeS_
  double end_time;       // startTimeS_ + durationS_   (RadioProjection.inl:273)
  double sample_rate;    // sampleRateHz_
  double resolution;     // 1. / sampleRateHz_         (:374, :396)
  double wavelength;     // c / sampleRateHz_          (:492)
  double fixed_scale;    // fixedPointScale_
  double bins_d;         // (double) numberOfBins_     (:280)
  uint64_t bins;
  uint64_t offset;       // waveformOffset_
  double dest_height;    // (z - minimumHeightM_) * inverseStepPerM_   (:184-185)
  double dest_n;         // refractivity_[dest] + 1.                   (:191)
  double dest_integral;  // integratedRefractivity_[dest]              (:192)
  uint64_t dest_index;   // static_cast<size_t>(dest_height + 0.5)      (:187)
  float fixed_scale_f;
  uint32_t count_samples;  // diagnostic: deposit 1 per component instead of the amplitude
};

// RadioPropagationView with the two tables interleaved as {n-1, integral}.
struct Propagation {
  double homogeneous;
  double min_height;
  double max_height;
  double step;
  double inv_step;
  double slope_n_lower;
  double slope_i_lower;
  double slope_n_upper;
  double slope_i_upper;
  const double2* table;  // .x = refractivity, .y = integrated refractivity
  uint64_t table_size;
  uint32_t refinement;
  uint32_t pad_;
};

// Track kinematics in registers (RadioTrackKinematics minus derived vectors).
struct Track {
  double sx, sy, sz, ex, ey, ez;
  double ts, te;
  double bx, by, bz;
  double length, beta_module, constant;
};

// Track workspace: a record of 24 doubles (192 bytes) per track.  The first
// 16: start xyz, end xyz, t_start, t_end, beta xyz, length, |beta|, charge
// constant, n_dst at the start point, one spare.  When every observer of the
// event shares one destination row (SourceTerms below), the last 8 hold the
// propagation terms of four source points, precomputed at ingest -- start,
// end, the ZHS segment midpoint (start + (start + (end - start))) / 2 and the
// CoREAS near-cone midpoint (start + end) / 2, each as (factor, n_src).
// Records are stored in tiles (track_column below).
enum TrackField : int {
  kSx = 0, kSy, kSz, kEx, kEy, kEz, kTs, kTe, kBx, kBy, kBz, kLen, kBmod, kConst, kNdstStart, kSpare,
  kFactorStart, kNsrcStart, kFactorEnd, kNsrcEnd, kFactorMidZhs, kNsrcMidZhs, kFactorMidCoreas,
  kNsrcMidCoreas, kTrackDoubles
};
static_assert(kTrackDoubles == 24, "192-byte track records");

// The workspace holds tiles of kTrackTile consecutive tracks (6144 bytes): in
// a tile, column k of the records (doubles 2k and 2k + 1, one 16-byte double2)
// is contiguous over the tile's 32 tracks.  The 32 lanes of a warp that read
// one column of 32 consecutive tracks then read 512 contiguous bytes (4 cache
// lines) where interleaved 192-byte records put every lane on its own line;
// the projection kernels' track loads were bound by the L1 data pipe's
// wavefronts with interleaved records.  A workspace is a whole number of tiles
// (track_capacity), so every column of a track below the capacity is inside it.
constexpr unsigned kTrackTile = 32;
constexpr unsigned kTrackColumns = kTrackDoubles / 2;

// Index (in double2 units) of column k of track i.
__host__ __device__ __forceinline__ uint64_t track_column(uint64_t i, unsigned k) {
  return (i / kTrackTile) * (kTrackTile * kTrackColumns) + k * kTrackTile + (i % kTrackTile);
}
// Column 0 of track i; column k is at [k * kTrackTile].
__host__ __device__ __forceinline__ double2 const* track_ref(double const* base, uint64_t i) {
  return reinterpret_cast<double2 const*>(base) + track_column(i, 0);
}
__host__ __device__ __forceinline__ double2* track_ref(double* base, uint64_t i) {
  return reinterpret_cast<double2*>(base) + track_column(i, 0);
}
// Field f of track i.
__host__ __device__ __forceinline__ double track_field(double const* base, uint64_t i, int f) {
  return base[2 * track_column(i, static_cast<unsigned>(f) / 2) + (f & 1)];
}
// Tracks a workspace for n tracks holds: n rounded up to whole tiles.
__host__ __device__ constexpr uint64_t track_capacity(uint64_t n) {
  return (n + kTrackTile - 1) / kTrackTile * kTrackTile;
}

struct Path {
  double time, n_src, n_dst, dist, kx, ky, kz;
};

// static_cast<int>(double) as x86-64 executes it (cvttsd2si): out of range and
// NaN give INT_MIN.  The reference's host build relies on it for ZHS bin spans
// and subtrack counts (RadioProjection.inl:457, :502).
__device__ __forceinline__ int x86_int(double v) {
  if (!(v > -2147483649.0 && v < 2147483648.0)) return INT_MIN;
  return static_cast<int>(v);
}

// static_cast<long long>(double) as x86-64 executes it (cvttsd2si, 64-bit).
__device__ __forceinline__ long long x86_ll(double v) {
  if (!(v >= -9223372036854775808.0 && v < 9223372036854775808.0)) return LLONG_MIN;
  return static_cast<long long>(v);
}

// observer_nearest_bin, RadioProjection.inl:75-82.
__device__ __forceinline__ double nearest_bin(double scaled) {
  double const integral = floor(scaled);
  return integral + (scaled - integral >= 0.5 ? 1. : 0.);
}

// co_reas_doppler, RadioProjection.inl:113-143 (device branch).
__device__ __forceinline__ double doppler(double index, double bx, double by, double bz,
                                          double kx, double ky, double kz) {
  double const ordinary = 1. - index * (bx * kx + by * ky + bz * kz);
  if (ordinary != 0.) return ordinary;
  double const px = bx * kx, py = by * ky, pz = bz * kz;
  double const ex = fma(bx, kx, -px), ey = fma(by, ky, -py), ez = fma(bz, kz, -pz);
  double const xy = px + py;
  double const xy_virtual = xy - px;
  double const xy_error = (px - (xy - xy_virtual)) + (py - xy_virtual);
  double const xyz = xy + pz;
  double const xyz_virtual = xyz - xy;
  double const xyz_error = (xy - (xyz - xyz_virtual)) + (pz - xyz_virtual);
  double const low = ex + ey + ez + xy_error + xyz_error;
  double const product = index * xyz;
  double const product_error = fma(index, xyz, -product) + index * low;
  return (1. - product) - product_error;
}

// The destination row of propagate (RadioProjection.inl:184-192) as the
// projection sees it: the observer's height in table steps, its table index,
// n and integrated refractivity there.  Observers with the same four values
// give the same source terms for a source point.
struct Destination {
  double height;
  uint64_t index;
  double n;
  double integral;
};

__device__ __forceinline__ Destination destination_of(ObserverCache const& o) {
  return Destination{o.dest_height, o.dest_index, o.dest_n, o.dest_integral};
}
inline Destination destination_of_host(ObserverCache const& o) {
  return Destination{o.dest_height, o.dest_index, o.dest_n, o.dest_integral};
}

// The part of propagate (RadioProjection.inl:170-238) that depends on the
// source's height and the destination row only: the travel time is
// factor * |d| / c, with factor = 1 + (I_src - I_dst) / height from the table
// (n for a homogeneous medium), and the refractive indices at both ends.
struct SourceTerms {
  double factor, n_src, n_dst;
};

__device__ __forceinline__ SourceTerms source_terms(Propagation const& p, Destination const& d, double sz) {
  if (p.homogeneous > 0.) return SourceTerms{p.homogeneous, p.homogeneous, p.homogeneous};
  double const sh = (sz - p.min_height) * p.inv_step;
  double const dh = d.height;
  uint64_t const last = p.table_size - 1;
  double n_src = 1., i_src = 1., n_dst = d.n, height = 1.;
  if (sh + 0.5 >= static_cast<double>(last)) {
    double2 const t = __ldg(p.table + last);
    n_src = t.x + p.slope_n_upper * fabs((sz - p.max_height) * p.inv_step) + 1.;
    i_src = t.y + p.slope_i_upper * fabs(p.max_height - sz);
    height = sh - dh;
  } else if (sh + 0.5 < static_cast<double>(last) && sh > 0.) {
    uint64_t const si = static_cast<uint64_t>(sh + 0.5);
    double2 const t = __ldg(p.table + si);
    n_src = t.x + 1.;
    i_src = t.y;
    height = static_cast<double>(static_cast<int64_t>(si) - static_cast<int64_t>(d.index)) * p.step;
    if (height == 0.) height = 1.;
  } else if (sh == 0.) {
    n_src = 1.;
    n_dst = 1.;
    i_src = __ldg(p.table).y;
    height = dh - sh;
  } else {
    double2 const t0 = __ldg(p.table);
    n_src = t0.x + p.slope_n_lower * fabs(sh) + 1.;
    i_src = t0.y + p.slope_i_lower * fabs(sh);
    n_dst = 1.;
    height = dh - fabs(sh);
  }
  return SourceTerms{1. + (i_src - d.integral) / height, n_src, n_dst};
}

// propagate, RadioProjection.inl:170-238, given the source terms of the
// point: the reference's (1 + (I_src - I_dst) / height) * dist / c with the
// parenthesised factor taken from `st` (the same IEEE value), or n dist / c.
// kTime = false skips the refractive index and travel time (the Fraunhofer
// midpoint uses only k and distance).  kApproxDirection = true returns
// k = d * RN(1/|d|): each component within 3.01 u |k| of the reference's
// RN(d/|d|) (u = 2^-53); distance, refractive indices and travel time are
// exact in both forms.
template <bool kTime, bool kApproxDirection = false>
__device__ __forceinline__ Path propagate_with(SourceTerms const& st, ObserverCache const& o,
                                               double sx, double sy, double sz) {
  Path r;
  double const dx = o.px - sx, dy = o.py - sy, dz = o.pz - sz;
  double const dist = sqrt(dx * dx + dy * dy + dz * dz);
  if (kApproxDirection) {
    double const inverse = 1. / dist;
    r.kx = dx * inverse;
    r.ky = dy * inverse;
    r.kz = dz * inverse;
  } else {
    r.kx = dx / dist;
    r.ky = dy / dist;
    r.kz = dz / dist;
  }
  r.dist = dist;
  if (!kTime) return r;
  r.time = st.factor * dist / kSpeedOfLight;
  r.n_src = st.n_src;
  r.n_dst = st.n_dst;
  return r;
}

// propagate, RadioProjection.inl:170-238: the source terms looked up in the
// table for this observer, then the path.
template <bool kTime, bool kApproxDirection = false>
__device__ __forceinline__ Path propagate(Propagation const& p, ObserverCache const& o,
                                          double sx, double sy, double sz) {
  SourceTerms const st = kTime ? source_terms(p, destination_of(o), sz) : SourceTerms{0., 0., 0.};
  return propagate_with<kTime, kApproxDirection>(st, o, sx, sy, sz);
}

// propagate (RadioProjection.inl:170-238) for the filtered decisions of the
// mixed-precision path.  The refractive indices and the integral ratio
// (i_src - i_dst) / height are the reference's (same table reads, same IEEE
// division); 1/|d| is an FP32 reciprocal square root refined by two Newton
// steps in FP64, |d| = RN(|d|^2 (1/|d|)), k = d (1/|d|), and the travel time
// multiplies by RN(1/c) instead of dividing by c.  With the final Newton
// residual r = 1 - |d|^2 y^2, y lies within |r|/2 + u of 1/|d| (u = 2^-53);
// `ok` requires |r| <= 2^-50, so y is within 5u, each direction component
// within 8u |k| of the reference's, and the time within 12u |time|
// (|d| within 7u, two products and RN(1/c) against one division):
// `time_err` = 2^-48 |time| (32u).  `ok` is false (the caller evaluates
// exactly) when |d|^2 lies outside [2^-100, 2^100], the residual is larger or
// the time is not finite.
struct FastPath {
  double time, n_src, n_dst, dist, kx, ky, kz, time_err;
  bool ok;
};

__device__ __forceinline__ FastPath propagate_fast_with(SourceTerms const& st, double ox, double oy, double oz,
                                                        double sx, double sy, double sz) {
  FastPath r;
  double const dx = ox - sx, dy = oy - sy, dz = oz - sz;
  double const s2 = dx * dx + dy * dy + dz * dz;
  r.ok = s2 >= 0x1p-100 && s2 <= 0x1p100;
  double y = static_cast<double>(rsqrtf(static_cast<float>(r.ok ? s2 : 1.)));
#pragma unroll
  for (int step = 0; step < 2; ++step) {
    double const h = s2 * y;
    y = fma(0.5 * y, fma(-h, y, 1.), y);
  }
  double const dist = s2 * y;
  r.ok = r.ok && fabs(fma(-dist, y, 1.)) <= 0x1p-50;
  r.kx = dx * y;
  r.ky = dy * y;
  r.kz = dz * y;
  r.dist = dist;
  constexpr double kInverseC = 1. / kSpeedOfLight;
  r.time = st.factor * dist * kInverseC;
  r.n_src = st.n_src;
  r.n_dst = st.n_dst;
  r.time_err = 0x1p-48 * fabs(r.time);
  r.ok = r.ok && r.time_err < 1.e300;  // false for infinite or NaN times
  return r;
}

__device__ __forceinline__ FastPath propagate_fast(Propagation const& p, ObserverCache const& o,
                                                   double sx, double sy, double sz) {
  return propagate_fast_with(source_terms(p, destination_of(o), sz), o.px, o.py, o.pz, sx, sy, sz);
}

// separate_same_bin_endpoints, RadioProjection.inl:303-336.
__device__ __forceinline__ void separate_same_bin(double& start, double& end, double res,
                                                  bool signed_order) {
  long long const sb = x86_ll(nearest_bin(start / res));
  long long const eb = x86_ll(nearest_bin(end / res));
  if (sb != eb) return;
  double const sf = start / res - floor(start / res);
  double const ef = end / res - floor(end / res);
  bool const forward = !signed_order || end >= start;
  if (forward) {
    if (sf >= 0.5 && ef >= 0.5) start -= res;
    else if (sf < 0.5 && ef < 0.5) end += res;
    else if (ef >= 1. - sf) end += res;
    else start -= res;
  } else {
    if (sf >= 0.5 && ef >= 0.5) end -= res;
    else if (sf < 0.5 && ef < 0.5) start += res;
    else if (sf >= 1. - ef) start += res;
    else end -= res;
  }
}

template <class T>
struct Vec3 {
  T x, y, z;
};

// k x (k x beta) (transverse_endpoint, :240-243) and k x (beta x k) (:438).
template <class T>
__device__ __forceinline__ Vec3<T> cross(Vec3<T> a, Vec3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Per-thread event counters (RadioCounters' projection fields).
struct Counts {
  unsigned long long coreas = 0, zhs = 0, subtracks = 0, overflows = 0;
  float mag = 0.f;  // sum of |fixed-point increments| added to a window without checks
};

}  // namespace c8r
