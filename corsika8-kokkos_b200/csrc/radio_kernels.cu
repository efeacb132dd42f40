// radio_kernels.cu — sm_100a kernels of the radio projection.
//
// Compiled with -fmad=false (see build.py): FP64 time/bin/branch arithmetic is
// the IEEE result of the reference's expressions, so fixed-point traces in the
// FP64 path are bit-identical to the reference's, and bin indices and branch
// decisions are identical in the mixed path too.
//
//   ingest_kernel    LeptonTransportRecord (752 B AoS) -> compacted SoA
//                    kinematics + counters (record_track, RadioProjection.inl:541-611)
//   direct_kernel    one thread per (track, antenna) pair, 64-bit global
//                    atomics per sample (RadioAccumulator.inl:663-697 shape)
//   windowed_kernel  persistent CTAs over a work list of (event, chunk,
//                    algorithm, antenna) items; the CTA owns that antenna's
//                    trace as an int64 window in shared memory, deposits with
//                    shared atomics and flushes non-zero bins with checked
//                    global atomics
//   decode_kernel    int64 fixed point -> V/m (V s/m) (RadioAccumulator.inl:849-898)
#include "radio_kernels.cuh"

#include <cuda_runtime.h>

#include <cstring>

#include "../../include/c8radio.h"

namespace c8r {
namespace {

constexpr double kEmConstant = 1. / (4. * kPi * kVacuumPermittivity * kSpeedOfLight);

// ---------------------------------------------------------------- fixed point
// add_radio_fixed_point, RadioProjection.inl:254-260.
// `mag` gains |v scale| (an upper bound of |out| up to half a unit) when the
// conversion succeeds.
__device__ __forceinline__ bool to_fixed(double v, ObserverCache const& o, long long& out,
                                         float& mag) {
  if (o.count_samples) {
    out = 1;
    mag += 1.f;
    return true;
  }
  double const s = v * o.fixed_scale;
  if (!(fabs(s) < kSignedLimit)) return false;  // also rejects NaN and infinities
  out = __double2ll_rn(s);
  mag += static_cast<float>(fabs(s));
  return true;
}
__device__ __forceinline__ bool to_fixed(float v, ObserverCache const& o, long long& out,
                                         float& mag) {
  if (o.count_samples) {
    out = 1;
    mag += 1.f;
    return true;
  }
  float const s = v * o.fixed_scale_f;
  if (!(fabsf(s) < 9223372036854775808.f)) return false;  // also rejects NaN and infinities
  out = __float2ll_rn(s);
  mag += fabsf(s);
  return true;
}

// checked_radio_atomic_add's overflow test on the returned previous value
// (RadioProjection.inl:246-251).
__device__ __forceinline__ bool checked(unsigned long long previous_bits, long long inc) {
  long long const previous = static_cast<long long>(previous_bits);
  return !((inc > 0 && previous > LLONG_MAX - inc) || (inc < 0 && previous < LLONG_MIN - inc));
}

__device__ __forceinline__ double amp_div(double a, double b) { return a / b; }
__device__ __forceinline__ float amp_div(float a, float b) { return __fdividef(a, b); }

template <class T>
__device__ __forceinline__ Vec3<T> scaled(Vec3<T> v, T s) {
  return {v.x * s, v.y * s, v.z * s};
}

// Signed overflow of the three adds previous + increment (two's complement),
// the condition checked_radio_atomic_add tests; increments whose conversion
// failed are passed as 0 and cannot overflow.
__device__ __forceinline__ bool no_overflow3(unsigned long long px, long long x,
                                             unsigned long long py, long long y,
                                             unsigned long long pz, long long z) {
  long long const sx = static_cast<long long>(px + static_cast<unsigned long long>(x));
  long long const sy = static_cast<long long>(py + static_cast<unsigned long long>(y));
  long long const sz = static_cast<long long>(pz + static_cast<unsigned long long>(z));
  long long const bad = ((static_cast<long long>(px) ^ sx) & (x ^ sx)) |
                        ((static_cast<long long>(py) ^ sy) & (y ^ sy)) |
                        ((static_cast<long long>(pz) ^ sz) & (z ^ sz));
  return bad >= 0;
}

// ---------------------------------------------------------------- sinks
// Trace rows of one observer: global X|Y|Z rows already offset to the
// observer's first bin.
struct GlobalSink {
  unsigned long long* row[3];
  double* frow[3];
  // All three components at one bin; false if a conversion failed or an add overflowed.
  __device__ __forceinline__ bool add3(uint64_t bin, long long x, long long y, long long z,
                                       bool ox, bool oy, bool oz, float mag, float& bound) {
    (void)mag;
    (void)bound;
    unsigned long long const px = ox ? atomicAdd(row[0] + bin, static_cast<unsigned long long>(x)) : 0ull;
    unsigned long long const py = oy ? atomicAdd(row[1] + bin, static_cast<unsigned long long>(y)) : 0ull;
    unsigned long long const pz = oz ? atomicAdd(row[2] + bin, static_cast<unsigned long long>(z)) : 0ull;
    return ox && oy && oz && no_overflow3(px, x, py, y, pz, z);
  }
  __device__ __forceinline__ void addf3(uint64_t bin, double x, double y, double z) {
    atomicAdd(frow[0] + bin, x);
    atomicAdd(frow[1] + bin, y);
    atomicAdd(frow[2] + bin, z);
  }
};

// Bins past a shared-memory window: checked global adds.  Inline: a call in
// the track loops costs the loop registers.
__device__ __forceinline__ bool spill3(unsigned long long* r0, unsigned long long* r1,
                                    unsigned long long* r2, long long x, long long y, long long z,
                                    bool ox, bool oy, bool oz) {
  unsigned long long const px = ox ? atomicAdd(r0, static_cast<unsigned long long>(x)) : 0ull;
  unsigned long long const py = oy ? atomicAdd(r1, static_cast<unsigned long long>(y)) : 0ull;
  unsigned long long const pz = oz ? atomicAdd(r2, static_cast<unsigned long long>(z)) : 0ull;
  return ox && oy && oz && no_overflow3(px, x, py, y, pz, z);
}

__device__ __forceinline__ void spillf3(double* r0, double* r1, double* r2, double x, double y,
                                     double z) {
  atomicAdd(r0, x);
  atomicAdd(r1, y);
  atomicAdd(r2, z);
}

// Shared-memory window of `width` bins starting at bin 0 (rows X|Y|Z), with
// bins past the window spilled to the global rows.
struct WindowSink {
  unsigned long long* win;
  double* fwin;
  uint32_t width;
  bool unchecked;
  unsigned long long* row[3];
  double* frow[3];
  // unchecked: window adds whose results are not read; `bound` then gains
  // |x| + |y| + |z| (as `mag`), and the kernel checks afterwards that no
  // partial sum of the window can have left the int64 range.
  __device__ __forceinline__ bool add3(uint64_t bin, long long x, long long y, long long z,
                                       bool ox, bool oy, bool oz, float mag, float& bound) {
    if (bin >= width)
      return spill3(row[0] + bin, row[1] + bin, row[2] + bin, x, y, z, ox, oy, oz);
    unsigned long long* const w = win + bin;
    if (unchecked) {
      if (ox) atomicAdd(w, static_cast<unsigned long long>(x));
      if (oy) atomicAdd(w + width, static_cast<unsigned long long>(y));
      if (oz) atomicAdd(w + 2 * width, static_cast<unsigned long long>(z));
      bound += mag;
      return ox && oy && oz;
    }
    unsigned long long const px = ox ? atomicAdd(w, static_cast<unsigned long long>(x)) : 0ull;
    unsigned long long const py = oy ? atomicAdd(w + width, static_cast<unsigned long long>(y)) : 0ull;
    unsigned long long const pz =
        oz ? atomicAdd(w + 2 * width, static_cast<unsigned long long>(z)) : 0ull;
    return ox && oy && oz && no_overflow3(px, x, py, y, pz, z);
  }
  __device__ __forceinline__ void addf3(uint64_t bin, double x, double y, double z) {
    if (bin >= width) {
      spillf3(frow[0] + bin, frow[1] + bin, frow[2] + bin, x, y, z);
      return;
    }
    double* const w = fwin + bin;
    atomicAdd(w, x);
    atomicAdd(w + width, y);
    atomicAdd(w + 2 * width, z);
  }
};

// ---------------------------------------------------------------- add_sample
// RadioProjection.inl:263-301.  kPotential selects the ZHS overload (no time
// gate).
template <bool kPotential>
__device__ __forceinline__ bool sample_bin(ObserverCache const& o, double t, uint64_t& bin) {
  if (!kPotential) {
    if (t < o.start_time || t > o.end_time) return false;
  }
  double const bv = nearest_bin((t - o.start_time) * o.sample_rate);
  if (!(bv >= 0. && bv < o.bins_d)) return false;
  bin = static_cast<uint64_t>(bv);
  return bin < o.bins;
}

template <class Amp>
struct Deposit {
  Vec3<Amp> value;
  long long ix, iy, iz;
  bool okx, oky, okz;
  float mag;  // |scaled components| that converted
};

template <bool kFixed, class Amp>
__device__ __forceinline__ Deposit<Amp> make_deposit(ObserverCache const& o, Vec3<Amp> v) {
  Deposit<Amp> d;
  d.value = v;
  d.mag = 0.f;
  if (kFixed) {
    d.okx = to_fixed(v.x, o, d.ix, d.mag);
    d.oky = to_fixed(v.y, o, d.iy, d.mag);
    d.okz = to_fixed(v.z, o, d.iz, d.mag);
  }
  return d;
}

template <bool kPotential, bool kFixed, class Amp, class Sink>
__device__ __forceinline__ void deposit(ObserverCache const& o, Sink& sink, double t,
                                        Deposit<Amp> const& d, unsigned long long& contributions,
                                        unsigned long long& overflows, float& bound) {
  uint64_t bin;
  if (!sample_bin<kPotential>(o, t, bin)) return;
  if (kFixed) {
    if (!sink.add3(bin, d.okx ? d.ix : 0, d.oky ? d.iy : 0, d.okz ? d.iz : 0, d.okx, d.oky, d.okz,
                   d.mag, bound)) {
      ++overflows;
      return;
    }
  } else {
    sink.addf3(bin, static_cast<double>(d.value.x), static_cast<double>(d.value.y),
               static_cast<double>(d.value.z));
  }
  ++contributions;
}

template <bool kPotential, bool kFixed, class Amp, class Sink>
__device__ __forceinline__ void add_sample(ObserverCache const& o, Sink& sink, double t,
                                           Vec3<Amp> v, unsigned long long& contributions,
                                           unsigned long long& overflows, float& bound) {
  uint64_t bin;
  if (!sample_bin<kPotential>(o, t, bin)) return;
  Deposit<Amp> const d = make_deposit<kFixed>(o, v);
  if (kFixed) {
    if (!sink.add3(bin, d.okx ? d.ix : 0, d.oky ? d.iy : 0, d.okz ? d.iz : 0, d.okx, d.oky, d.okz,
                   d.mag, bound)) {
      ++overflows;
      return;
    }
  } else {
    sink.addf3(bin, static_cast<double>(v.x), static_cast<double>(v.y), static_cast<double>(v.z));
  }
  ++contributions;
}

// A deposit at a bin already known to lie in [0, bins).
template <bool kFixed, class Amp, class Sink>
__device__ __forceinline__ void deposit_bin(Sink& sink, uint64_t bin, Deposit<Amp> const& d,
                                            unsigned long long& contributions,
                                            unsigned long long& overflows, float& bound) {
  if (kFixed) {
    if (!sink.add3(bin, d.okx ? d.ix : 0, d.oky ? d.iy : 0, d.okz ? d.iz : 0, d.okx, d.oky, d.okz,
                   d.mag, bound)) {
      ++overflows;
      return;
    }
  } else {
    sink.addf3(bin, static_cast<double>(d.value.x), static_cast<double>(d.value.y),
               static_cast<double>(d.value.z));
  }
  ++contributions;
}

// Near-Cherenkov branch of accumulate_co_reas (RadioProjection.inl:352-387):
// midpoint field over the Doppler-compressed duration.  Kept out of line: it
// is taken by a minority of pairs, and its third propagation would otherwise
// grow the hot loop's instruction footprint.  Returns the counts it adds.
template <bool kFixed, class Amp, bool kPre, class Sink>
__device__ __noinline__ Counts coreas_near_cone(Track const t, Propagation const& p,
                                                ObserverCache const& o, Sink sink,
                                                bool start_before_end, SourceTerms const pre_mid) {
  Counts c;
  Vec3<Amp> const beta{static_cast<Amp>(t.bx), static_cast<Amp>(t.by), static_cast<Amp>(t.bz)};
  double const cf = t.constant * o.sample_rate;
  double const mx = (t.sx + t.ex) * 0.5, my = (t.sy + t.ey) * 0.5, mz = (t.sz + t.ez) * 0.5;
  double const mt = (t.ts + t.te) * 0.5;
  Path const pm = kPre ? propagate_with<true>(pre_mid, o, mx, my, mz) : propagate<true>(p, o, mx, my, mz);
  double const mr = mt + pm.time;
  double const md = doppler(pm.n_src, t.bx, t.by, t.bz, pm.kx, pm.ky, pm.kz);
  Vec3<Amp> const k{static_cast<Amp>(pm.kx), static_cast<Amp>(pm.ky), static_cast<Amp>(pm.kz)};
  Vec3<Amp> fstart =
      scaled(cross(k, cross(k, beta)), amp_div(static_cast<Amp>(cf), static_cast<Amp>(md * pm.dist)));
  Vec3<Amp> fend = scaled(fstart, static_cast<Amp>(-1.));
  double dt = t.length / (kSpeedOfLight * t.beta_module) * fabs(md);
  double sr, er;
  if (start_before_end) {
    sr = mr - 0.5 * dt;
    er = mr + 0.5 * dt;
  } else {
    sr = mr + 0.5 * dt;
    er = mr - 0.5 * dt;
  }
  double const res = o.resolution;
  dt = er - sr;
  if (fabs(dt) < res) {
    Amp const s = static_cast<Amp>(fabs(dt / res));
    fstart = scaled(fstart, s);
    fend = scaled(fend, s);
    separate_same_bin(sr, er, res, true);
  }
  add_sample<false, kFixed>(o, sink, sr, fstart, c.coreas, c.overflows, c.mag);
  add_sample<false, kFixed>(o, sink, er, fend, c.coreas, c.overflows, c.mag);
  return c;
}

// ---------------------------------------------------------------- CoREAS
// accumulate_co_reas, RadioProjection.inl:339-409, every decision and (FP64
// path) every amplitude evaluated exactly as the reference.
// kPre: the start, end and midpoint source terms are `terms` (precomputed at
// ingest for the event's shared destination row), else looked up.
template <bool kFixed, class Amp, class Sink, bool kPre = false>
__device__ __forceinline__ void coreas_pair(Track const& t, Propagation const& p,
                                            ObserverCache const& o, Sink& sink, Counts& c,
                                            SourceTerms const* terms = nullptr) {
  Path const ps = kPre ? propagate_with<true>(terms[0], o, t.sx, t.sy, t.sz) : propagate<true>(p, o, t.sx, t.sy, t.sz);
  Path const pe = kPre ? propagate_with<true>(terms[1], o, t.ex, t.ey, t.ez) : propagate<true>(p, o, t.ex, t.ey, t.ez);
  double const pre = doppler(ps.n_src, t.bx, t.by, t.bz, ps.kx, ps.ky, ps.kz);
  double const post = doppler(pe.n_src, t.bx, t.by, t.bz, pe.kx, pe.ky, pe.kz);
  double sr = t.ts + ps.time;
  double er = t.te + pe.time;
  double const cf = t.constant * o.sample_rate;
  Vec3<Amp> const beta{static_cast<Amp>(t.bx), static_cast<Amp>(t.by), static_cast<Amp>(t.bz)};

  if (ps.n_dst > 1. && (fabs(pre) < kCoreasThreshold || fabs(post) < kCoreasThreshold)) {
    Counts const d = coreas_near_cone<kFixed, Amp, kPre>(t, p, o, sink, sr < er, kPre ? terms[2] : SourceTerms{});
    c.coreas += d.coreas;
    c.overflows += d.overflows;
    c.mag += d.mag;
    return;
  }

  Vec3<Amp> const ks{static_cast<Amp>(ps.kx), static_cast<Amp>(ps.ky), static_cast<Amp>(ps.kz)};
  Vec3<Amp> const ke{static_cast<Amp>(pe.kx), static_cast<Amp>(pe.ky), static_cast<Amp>(pe.kz)};
  Vec3<Amp> fstart =
      scaled(cross(ks, cross(ks, beta)), amp_div(static_cast<Amp>(cf), static_cast<Amp>(pre * ps.dist)));
  Vec3<Amp> fend =
      scaled(cross(ke, cross(ke, beta)), amp_div(static_cast<Amp>(-cf), static_cast<Amp>(post * pe.dist)));
  if (pre < 1.e-9 || post < 1.e-9) {
    double const res = o.resolution;
    double const dt = er - sr;
    if (fabs(dt) < res) {
      Amp const s = static_cast<Amp>(fabs(dt / res));
      fstart = scaled(fstart, s);
      fend = scaled(fend, s);
      separate_same_bin(sr, er, res, false);
    }
  }
  add_sample<false, kFixed>(o, sink, sr, fstart, c.coreas, c.overflows, c.mag);
  add_sample<false, kFixed>(o, sink, er, fend, c.coreas, c.overflows, c.mag);
}

// The propagation of the filtered paths: propagate_fast when kFast, else the
// exact propagate (time_err 0).  kPre: the point's source terms are `pre`
// (precomputed at ingest), else they are looked up in the table.
template <bool kFast, bool kPre = false>
__device__ __forceinline__ FastPath filtered_path(Propagation const& p, ObserverCache const& o,
                                                  double x, double y, double z,
                                                  SourceTerms const& pre = SourceTerms{}) {
  SourceTerms const st = kPre ? pre : source_terms(p, destination_of(o), z);
  if (kFast) return propagate_fast_with(st, o.px, o.py, o.pz, x, y, z);
  Path const e = propagate_with<true>(st, o, x, y, z);
  return FastPath{e.time, e.n_src, e.n_dst, e.dist, e.kx, e.ky, e.kz, 0., true};
}

// The common CoREAS pair of the windowed kernel (RadioProjection.inl:339-409
// without its near-Cherenkov branch).  Returns false, having deposited
// nothing, when the pair needs the near-Cherenkov branch or (kFilter) an exact
// evaluation; the kernel then defers it to coreas_drain_pair.
//
// kFilter (mixed precision): travel times, refractive indices and distances
// are exact; emission directions are d * RN(1/|d|) (propagate's
// kApproxDirection), so each Doppler factor 1 - n beta.k lies within
// 14 u n |beta|_1 + 2 u of the reference's (u = 2^-53; used below with a 4.5x
// margin).  The branches (near-Cherenkov |doppler| < 1e-3, the sign test
// doppler < 1e-9) are taken here only when that bound cannot move them, and
// pairs with |doppler| < 1e-6 are left to the exact evaluation.  Sample times
// are exact, so bins are the reference's.  Returns kCoreasDeposited, or the
// deferral: kCoreasExact, or kCoreasNearCone with bit 0 the branch's
// start-before-end order (sr < er, exact times), both decided exactly, so the
// drain evaluates only the near-Cherenkov branch itself.
constexpr int kCoreasDeposited = 0, kCoreasExact = 1, kCoreasNearCone = 2;
template <bool kFixed, bool kFilter, bool kPre, class Amp, class Sink>
__device__ __forceinline__ int coreas_common(Track const& t, Propagation const& p,
                                              ObserverCache const& o, Sink& sink, Counts& c,
                                              SourceTerms const& pre_start, SourceTerms const& pre_end) {
  Path const ps = kPre ? propagate_with<true, kFilter>(pre_start, o, t.sx, t.sy, t.sz)
                       : propagate<true, kFilter>(p, o, t.sx, t.sy, t.sz);
  Path const pe = kPre ? propagate_with<true, kFilter>(pre_end, o, t.ex, t.ey, t.ez)
                       : propagate<true, kFilter>(p, o, t.ex, t.ey, t.ez);
  double pre, post;
  if (kFilter) {
    pre = 1. - ps.n_src * (t.bx * ps.kx + t.by * ps.ky + t.bz * ps.kz);
    post = 1. - pe.n_src * (t.bx * pe.kx + t.by * pe.ky + t.bz * pe.kz);
    double const beta1 = fabs(t.bx) + fabs(t.by) + fabs(t.bz) + 1.;
    double const err_pre = ps.n_src * beta1 * 0x1p-47 + 0x1p-50;
    double const err_post = pe.n_src * beta1 * 0x1p-47 + 0x1p-50;
    bool const ambiguous =
        fabs(pre) < 1.e-6 || fabs(post) < 1.e-6 ||
        (ps.n_dst > 1. && (fabs(fabs(pre) - kCoreasThreshold) <= err_pre ||
                           fabs(fabs(post) - kCoreasThreshold) <= err_post));
    if (ambiguous) return kCoreasExact;
  } else {
    pre = doppler(ps.n_src, t.bx, t.by, t.bz, ps.kx, ps.ky, ps.kz);
    post = doppler(pe.n_src, t.bx, t.by, t.bz, pe.kx, pe.ky, pe.kz);
  }
  double sr = t.ts + ps.time;
  double er = t.te + pe.time;
  if (ps.n_dst > 1. && (fabs(pre) < kCoreasThreshold || fabs(post) < kCoreasThreshold))
    return kCoreasNearCone | (sr < er ? 1 : 0);
  Vec3<Amp> const beta{static_cast<Amp>(t.bx), static_cast<Amp>(t.by), static_cast<Amp>(t.bz)};
  Vec3<Amp> const ks{static_cast<Amp>(ps.kx), static_cast<Amp>(ps.ky), static_cast<Amp>(ps.kz)};
  Vec3<Amp> const ke{static_cast<Amp>(pe.kx), static_cast<Amp>(pe.ky), static_cast<Amp>(pe.kz)};
  double const cf = t.constant * o.sample_rate;
  Vec3<Amp> fstart =
      scaled(cross(ks, cross(ks, beta)), amp_div(static_cast<Amp>(cf), static_cast<Amp>(pre * ps.dist)));
  Vec3<Amp> fend =
      scaled(cross(ke, cross(ke, beta)), amp_div(static_cast<Amp>(-cf), static_cast<Amp>(post * pe.dist)));
  // with the filter |pre|, |post| >= 1e-6, so "< 1e-9" is the sign of the factor
  if (pre < 1.e-9 || post < 1.e-9) {
    double const res = o.resolution;
    double const dt = er - sr;
    if (fabs(dt) < res) {
      Amp const s = static_cast<Amp>(fabs(dt / res));
      fstart = scaled(fstart, s);
      fend = scaled(fend, s);
      separate_same_bin(sr, er, res, false);
    }
  }
  add_sample<false, kFixed>(o, sink, sr, fstart, c.coreas, c.overflows, c.mag);
  add_sample<false, kFixed>(o, sink, er, fend, c.coreas, c.overflows, c.mag);
  return kCoreasDeposited;
}

// Intermediate ZHS bins binned index by index with the reference's own
// expression (RadioProjection.inl:465-472).  Samples of index i land in bin
// nearest((d1 + i/fs - t0) fs), monotone in i and within a hundredth of a bin
// of x1 + i while all magnitudes stay below 2^40 bins; indices whose bin is
// surely outside [0, bins) are skipped, which changes no sum and no counter.
template <bool kFixed, class Amp, class Sink>
__device__ __noinline__ Counts zhs_indexed_bins(ObserverCache const& o, Sink sink, double d1,
                                                double x1, int nb, Deposit<Amp> const mid) {
  Counts c;
  double const fs = o.sample_rate;
  int lo = 1, hi = nb;
  double const span = 1099511627776.0;  // 2^40
  if (fabs(x1) < span && fabs(o.start_time * fs) < span && fabs(d1 * fs) < span &&
      static_cast<double>(nb) < span) {
    double const first = -x1 - 3.;
    double const last = o.bins_d - x1 + 3.;
    if (first > 1.) lo = first >= static_cast<double>(nb) ? nb : static_cast<int>(first);
    if (last < static_cast<double>(nb)) hi = last <= 1. ? 1 : static_cast<int>(last) + 1;
    if (hi > nb) hi = nb;
  }
  for (int index = lo; index < hi; ++index)
    deposit<true, kFixed>(o, sink, d1 + static_cast<double>(index) / fs, mid, c.zhs, c.overflows, c.mag);
  return c;
}

// ---------------------------------------------------------------- ZHS
// The multi-bin tail of a ZHS segment (first sample and intermediate bins,
// RadioProjection.inl:457-472), out of line: about half the segments take it,
// and keeping it out of the common path saves registers and instruction fetch.
template <bool kFixed, bool kRuns, class Amp, class Sink>
__device__ __noinline__ Counts zhs_multi_tail(ObserverCache const& o, Sink sink, double d1,
                                              double x1, double sb, int nb, Vec3<Amp> perp,
                                              double sc, double dd, double mc, bool run_ok) {
  Counts c;
  double const frac_first = fabs(sb + 0.5 - x1);
  add_sample<true, kFixed>(o, sink, d1,
                           scaled(perp, amp_div(static_cast<Amp>(sc * frac_first), static_cast<Amp>(dd))),
                           c.zhs, c.overflows, c.mag);
  if (nb > 1) {
    Deposit<Amp> const mid =
        make_deposit<kFixed>(o, scaled(perp, amp_div(static_cast<Amp>(mc), static_cast<Amp>(dd))));
    if (kRuns && run_ok) {
      long long const b1 = static_cast<long long>(floor(x1)) + (x1 - floor(x1) >= 0.5 ? 1 : 0);
      long long lo = 1, hi = nb;
      if (-b1 > lo) lo = -b1;
      long long const top = static_cast<long long>(o.bins) - b1;
      if (top < hi) hi = top;
      if (hi > lo) {
        uint64_t const first = static_cast<uint64_t>(b1 + lo);
        uint32_t const count = static_cast<uint32_t>(hi - lo);
        for (uint32_t j = 0; j < count; ++j)
          deposit_bin<kFixed>(sink, first + j, mid, c.zhs, c.overflows, c.mag);
      }
    } else {
      Counts const d = zhs_indexed_bins<kFixed, Amp>(o, sink, d1, x1, nb, mid);
      c.zhs += d.zhs;
      c.overflows += d.overflows;
      c.mag += d.mag;
    }
  }
  return c;
}

// accumulate_zhs_segment, RadioProjection.inl:412-480.
//
// kRuns = true (windowed kernel): the intermediate bins of a segment are the
// consecutive bins nearest(x1) + i whenever x1 lies farther than a rounding
// bound from a half bin (checked below); they are then deposited as one run,
// without the per-index division.  Otherwise, and always for kRuns = false
// (the reference-shaped direct kernel), each index is binned by the
// reference's own expression.
//
// kFilter = true (mixed precision): the emission direction is d * RN(1/|d|),
// so n beta.k lies within e_nbk of the reference's value and each detection
// time within e_d; every decision the segment takes (which detection time is
// first, the nearest bin and floor(x + 0.5) of both, |1 - n beta.k| > 1e-15,
// the consecutive-run test) is taken only when those bounds cannot change it,
// else the segment returns false having deposited nothing (the caller then
// evaluates it exactly).  Bins and counts are the reference's.
template <bool kFixed, bool kRuns, bool kFilter, class Amp, class Sink>
__device__ __forceinline__ bool zhs_segment(double p1x, double p1y, double p1z, double p2x,
                                            double p2y, double p2z, double t1, double t2,
                                            Track const& t, Propagation const& p,
                                            ObserverCache const& o, Sink& sink, Counts& c,
                                            bool subdivided) {
  double const mx = (p1x + p2x) * 0.5, my = (p1y + p2y) * 0.5, mz = (p1z + p2z) * 0.5;
  Path const path = propagate<true, kFilter>(p, o, mx, my, mz);
  double const bk = t.bx * path.kx + t.by * path.ky + t.bz * path.kz;
  double const nbk = path.n_src * bk;
  double const mt = (t1 + t2) * 0.5;
  double d1 = t1 + path.time - nbk * (t1 - mt);
  double d2 = t2 + path.time - nbk * (t2 - mt);
  double e_d = 0.;
  if (kFilter) {
    // |nbk - reference| <= 11.1 u n |beta|_1; each d within that times
    // |t - mt| plus two ulps of its terms (bounds used with margins >= 4x)
    double const beta1 = fabs(t.bx) + fabs(t.by) + fabs(t.bz) + 1.;
    double const e_nbk = path.n_src * beta1 * 0x1p-47 + 0x1p-50;
    double const h = fabs(t1 - mt) + fabs(t2 - mt);
    e_d = e_nbk * h + 0x1p-50 * (fabs(t1 + path.time) + fabs(t2 + path.time) + fabs(nbk) * h);
  }
  double sign = 1.;
  if (d1 > d2) {
    double const swap = d1;
    d1 = d2;
    d2 = swap;
    sign = -1.;
  }
  double const fs = o.sample_rate;
  double const x1 = (d1 - o.start_time) * fs;
  double const x2 = (d2 - o.start_time) * fs;
  double const sb = floor(x1 + 0.5);
  double const eb = floor(x2 + 0.5);
  double const den = 1. - nbk;
  int const nb = x86_int(eb - sb);
  // consecutive-run test for the intermediate bins.  Index i is binned at
  // y_i = RN(RN(RN(d1 + RN(i/fs)) - t0) fs); with u = 2^-53,
  // |y_i - (x1 + i)| <= 6 u M (1 + u)^4 < 2^-50 M for M = |x1| + i + |d1 fs|
  // + |t0 fs| + 2.  The nearest bin changes only at half-integers, which sit
  // at integer offsets from each other, so if x1 is farther than that bound
  // (plus, filtered, x1's own error) from a half-integer, nearest(y_i) =
  // nearest(x1) + i for every i < nb.
  double const f1 = fabs(x1 - floor(x1) - 0.5);
  double const mag = fabs(x1) + static_cast<double>(nb) + fabs(d1 * fs) + fabs(o.start_time * fs) + 2.;
  bool run_ok = mag < 0x1p50 && f1 > mag * 0x1p-48;
  if (kFilter) {
    double const e_x = (e_d + 0x1p-50 * (fabs(d1) + fabs(d2) + 2. * fabs(o.start_time))) * fs +
                       0x1p-50 * (fabs(x1) + fabs(x2));
    double const f2 = fabs(x2 - floor(x2) - 0.5);
    run_ok = run_ok && f1 > mag * 0x1p-48 + e_x;
    bool const ambiguous = fabs(d1 - d2) <= 2. * e_d || fabs(den) < 1.e-6 ||
                           f1 <= e_x + 0x1p-50 * (fabs(x1) + 1.) ||
                           f2 <= e_x + 0x1p-50 * (fabs(x2) + 1.) || (nb > 1 && !run_ok);
    if (ambiguous) return false;
  }
  Vec3<Amp> const k{static_cast<Amp>(path.kx), static_cast<Amp>(path.ky), static_cast<Amp>(path.kz)};
  Vec3<Amp> const beta{static_cast<Amp>(t.bx), static_cast<Amp>(t.by), static_cast<Amp>(t.bz)};
  Vec3<Amp> const perp = cross(k, cross(beta, k));
  double const sc = sign * t.constant;
  double const dd = den * path.dist;

  // The last sample (detection_time2) and, when both times share a bin, the
  // only one (:441-455); fraction and denominator selected, not branched.
  bool const single = sb == eb;
  bool const tiny = !(fabs(den) > 1.e-15);
  double const frac_last = single ? (tiny ? (t2 - t1) * fs : fabs(d2 * fs - d1 * fs))
                                  : fabs(x2 + 0.5 - eb);
  double const den_last = single && tiny ? path.dist : dd;
  add_sample<true, kFixed>(o, sink, d2,
                           scaled(perp, amp_div(static_cast<Amp>(sc * frac_last),
                                                static_cast<Amp>(den_last))),
                           c.zhs, c.overflows, c.mag);
  if (single) return true;
  Counts const d = zhs_multi_tail<kFixed, kRuns, Amp>(
      o, sink, d1, x1, sb, nb, perp, sc, dd, (subdivided ? 1. : sign) * t.constant, run_ok);
  c.zhs += d.zhs;
  c.overflows += d.overflows;
  c.mag += d.mag;
  return true;
}

// The samples of one ZHS segment, staged for the warp (windowed kernel): the
// in-range bins [start, start + count) of its first sample and intermediate
// bins (value perp * first at `start` when flag bit 0, perp * mid elsewhere)
// and its last sample at last_bin (flag bit 1).  Bins are consecutive there
// because the segment is staged only when its intermediate bins are
// nearest(x1) + i (the consecutive-run test of zhs_segment).
template <class Amp>
struct StagedSegment {
  Vec3<Amp> perp;
  Amp first, mid, last;
  uint32_t start, count, last_bin, flags;
};
// FP64 amplitudes: slots of 72 bytes (18 banks) rather than 64, which spreads
// the lanes' loads of different slots over the shared-memory banks (11% off
// the FP64 ZHS kernel; the same padding of the 40-byte FP32 slot cost 10%).
template <>
struct StagedSegment<double> {
  Vec3<double> perp;
  double first, mid, last;
  uint32_t start, count, last_bin, flags;
  uint32_t pad_[2];
};

// accumulate_zhs_segment (RadioProjection.inl:412-480) with every decision of
// zhs_segment<kRuns = true, kFilter>, its samples staged instead of
// deposited.  With kFilter the midpoint propagation is propagate_fast: its
// directions (8u) stay inside the n beta.k bound, and its time error adds to
// the detection-time bound e_d.  Returns false when the segment needs the
// per-index binning or (kFilter) an exact evaluation, or when the trace has
// 2^26 bins or more (staged counts then stay far inside 32 bits per warp);
// the caller then discards whatever `out` holds.  The filter's ambiguity
// test is applied at the end, after the samples are formed (the values it
// declines are discarded): with the decision off the critical path the
// kernel issues the staging arithmetic beside the bound arithmetic (7% off
// the ZHS kernel on the 1e7 x 160 workload).
template <bool kFilter, class Amp, bool kPre = false>
__device__ __forceinline__ bool zhs_stage(double p1x, double p1y, double p1z, double p2x,
                                          double p2y, double p2z, double t1, double t2,
                                          Track const& t, Propagation const& p,
                                          ObserverCache const& o, bool subdivided,
                                          StagedSegment<Amp>& out,
                                          SourceTerms const& pre = SourceTerms{}) {
  if (!(o.bins_d < 67108864.0)) return false;
  bool decided = true;
  double const mx = (p1x + p2x) * 0.5, my = (p1y + p2y) * 0.5, mz = (p1z + p2z) * 0.5;
  FastPath const path = filtered_path<kFilter, kPre>(p, o, mx, my, mz, pre);
  if (kFilter && !path.ok) return false;
  double const bk = t.bx * path.kx + t.by * path.ky + t.bz * path.kz;
  double const nbk = path.n_src * bk;
  double const mt = (t1 + t2) * 0.5;
  double d1 = t1 + path.time - nbk * (t1 - mt);
  double d2 = t2 + path.time - nbk * (t2 - mt);
  double e_d = 0.;
  if (kFilter) {
    double const beta1 = fabs(t.bx) + fabs(t.by) + fabs(t.bz) + 1.;
    double const e_nbk = path.n_src * beta1 * 0x1p-47 + 0x1p-50;
    double const h = fabs(t1 - mt) + fabs(t2 - mt);
    e_d = e_nbk * h + 0x1p-50 * (fabs(t1 + path.time) + fabs(t2 + path.time) + fabs(nbk) * h) +
          path.time_err;
  }
  double sign = 1.;
  if (d1 > d2) {
    double const swap = d1;
    d1 = d2;
    d2 = swap;
    sign = -1.;
  }
  double const fs = o.sample_rate;
  double const x1 = (d1 - o.start_time) * fs;
  double const x2 = (d2 - o.start_time) * fs;
  double const sb = floor(x1 + 0.5);
  double const eb = floor(x2 + 0.5);
  double const den = 1. - nbk;
  int const nb = x86_int(eb - sb);
  double const f1 = fabs(x1 - floor(x1) - 0.5);
  double const mag = fabs(x1) + static_cast<double>(nb) + fabs(d1 * fs) + fabs(o.start_time * fs) + 2.;
  bool run_ok = mag < 0x1p50 && f1 > mag * 0x1p-48;
  if (kFilter) {
    double const e_x = (e_d + 0x1p-50 * (fabs(d1) + fabs(d2) + 2. * fabs(o.start_time))) * fs +
                       0x1p-50 * (fabs(x1) + fabs(x2));
    double const f2 = fabs(x2 - floor(x2) - 0.5);
    run_ok = run_ok && f1 > mag * 0x1p-48 + e_x;
    bool const ambiguous = fabs(d1 - d2) <= 2. * e_d || fabs(den) < 1.e-6 ||
                           f1 <= e_x + 0x1p-50 * (fabs(x1) + 1.) ||
                           f2 <= e_x + 0x1p-50 * (fabs(x2) + 1.) || (nb > 1 && !run_ok);
    decided = !ambiguous;
  } else if (nb > 1 && !run_ok) {
    return false;
  }
  Vec3<Amp> const k{static_cast<Amp>(path.kx), static_cast<Amp>(path.ky), static_cast<Amp>(path.kz)};
  Vec3<Amp> const beta{static_cast<Amp>(t.bx), static_cast<Amp>(t.by), static_cast<Amp>(t.bz)};
  out.perp = cross(k, cross(beta, k));
  double const sc = sign * t.constant;
  double const dd = den * path.dist;
  bool const single = sb == eb;
  bool const tiny = !(fabs(den) > 1.e-15);
  double const frac_last = single ? (tiny ? (t2 - t1) * fs : fabs(d2 * fs - d1 * fs))
                                  : fabs(x2 + 0.5 - eb);
  double const den_last = single && tiny ? path.dist : dd;
  out.last = amp_div(static_cast<Amp>(sc * frac_last), static_cast<Amp>(den_last));
  out.flags = 0u;
  out.start = 0u;
  out.count = 0u;
  out.last_bin = 0u;
  // last sample, add_sample(detection_time2): bin nearest((d2 - t0) fs) = nearest(x2)
  double const bv2 = nearest_bin(x2);
  if (bv2 >= 0. && bv2 < o.bins_d) {
    out.last_bin = static_cast<uint32_t>(bv2);
    out.flags = 2u;
  }
  if (single) return decided;
  double const frac_first = fabs(sb + 0.5 - x1);
  out.first = amp_div(static_cast<Amp>(sc * frac_first), static_cast<Amp>(dd));
  double const mc = (subdivided ? 1. : sign) * t.constant;
  out.mid = amp_div(static_cast<Amp>(mc), static_cast<Amp>(dd));
  // first sample, add_sample(detection_time1): bin nearest(x1)
  double const bv1 = nearest_bin(x1);
  bool const first_in = bv1 >= 0. && bv1 < o.bins_d;
  if (first_in) {
    out.start = static_cast<uint32_t>(bv1);
    out.count = 1u;
    out.flags |= 1u;
  }
  if (nb > 1) {  // intermediate bins b1 + i, i in [1, nb), clipped to the trace
    long long const b1 = static_cast<long long>(floor(x1)) + (x1 - floor(x1) >= 0.5 ? 1 : 0);
    long long lo = 1, hi = nb;
    if (-b1 > lo) lo = -b1;
    long long const top = static_cast<long long>(o.bins) - b1;
    if (top < hi) hi = top;
    if (hi > lo) {
      if (first_in) {  // b1 = nearest(x1) >= 0, so lo = 1: one run from the first sample
        out.count = static_cast<uint32_t>(1 + (hi - lo));
      } else {
        out.start = static_cast<uint32_t>(b1 + lo);
        out.count = static_cast<uint32_t>(hi - lo);
      }
    }
  }
  return decided;
}

// Deposits the staged segments of a warp: every lane takes two bins of the
// flattened list (lane order, then bin order) per step, their owner searches
// interleaved.  Every lane of the
// warp calls it; `staging` is the warp's 32 slots in shared memory.
template <bool kFixed, class Amp, class Sink>
__device__ __forceinline__ void deposit_staged(StagedSegment<Amp>* staging,
                                               StagedSegment<Amp> const& seg,
                                               ObserverCache const& o, Sink& sink, Counts& c) {
  unsigned const lane = threadIdx.x & 31u;
  uint32_t const cnt = seg.count + ((seg.flags >> 1) & 1u);
  uint32_t incl = cnt;
#pragma unroll
  for (unsigned d = 1; d < 32u; d <<= 1) {
    uint32_t const v = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += v;
  }
  uint32_t const total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0u) return;
  staging[lane] = seg;
  __syncwarp();
  uint32_t const before_mine = incl - cnt;
  // the converting fields in registers: `o` lives in shared memory, which the
  // window atomics below might alias as far as the compiler can tell
  ObserverCache grid;
  grid.fixed_scale = o.fixed_scale;
  grid.fixed_scale_f = o.fixed_scale_f;
  grid.count_samples = o.count_samples;
  for (uint32_t base = 0; base < total; base += 64u) {
    uint32_t const j0 = base + lane, j1 = j0 + 32u;
    uint32_t owner0 = 0, owner1 = 0;
#pragma unroll
    for (uint32_t step = 16; step >= 1u; step >>= 1) {
      uint32_t const v0 = __shfl_sync(0xffffffffu, incl, owner0 + step - 1u);
      uint32_t const v1 = __shfl_sync(0xffffffffu, incl, owner1 + step - 1u);
      if (v0 <= j0) owner0 += step;
      if (v1 <= j1) owner1 += step;
    }
    uint32_t const before0 = __shfl_sync(0xffffffffu, before_mine, owner0 & 31u);
    uint32_t const before1 = __shfl_sync(0xffffffffu, before_mine, owner1 & 31u);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      uint32_t const j = u ? j1 : j0;
      uint32_t const owner = u ? owner1 : owner0;
      uint32_t const before = u ? before1 : before0;
      if (j < total) {
        StagedSegment<Amp> const& g = staging[owner];
        uint32_t const k = j - before;
        uint32_t bin;
        Amp scale;
        if (k < g.count) {
          bin = g.start + k;
          scale = (k == 0u && (g.flags & 1u)) ? g.first : g.mid;
        } else {
          bin = g.last_bin;
          scale = g.last;
        }
        deposit_bin<kFixed>(sink, bin, make_deposit<kFixed>(grid, scaled(g.perp, scale)), c.zhs,
                            c.overflows, c.mag);
      }
    }
  }
  __syncwarp();
}

// The fixed-point value of one component, as to_fixed computes it.
__device__ __forceinline__ long long fixed_value(float v, ObserverCache const& grid) {
  return __float2ll_rn(v * grid.fixed_scale_f);
}
__device__ __forceinline__ long long fixed_value(double v, ObserverCache const& grid) {
  return __double2ll_rn(v * grid.fixed_scale);
}

// The owner's half of the unchecked deposit of its staged segment (fixed
// point, the whole trace in the window, whose adds are not checked): shows
// once for the segment that every sample converts -- each component's
// |(p_c scale) fixed_scale| is at most max|p_c| max|scale| fixed_scale (1 +
// 2^-22), kept below 2^62 -- counts the samples as contributions and adds
// an upper bound of their |components| to the window bound (each factor's
// roundings, at most nine of 2^-24, inside the 2^-20 margin).  The deposit
// then converts and adds each sample with no check.  Returns false when a
// sample might not convert (huge or non-finite values) or in the diagnostic
// count-samples mode: the pair then goes to the checked drain.
template <class Amp>
__device__ __forceinline__ bool account_staged(StagedSegment<Amp> const& seg, ObserverCache const& o,
                                               Counts& c) {
  uint32_t const samples = seg.count + ((seg.flags >> 1) & 1u);
  if (samples == 0u) return true;
  if (o.count_samples) return false;
  bool const has_first = (seg.flags & 1u) != 0u;
  uint32_t const mids = seg.count - (has_first ? 1u : 0u);
  Amp const zero = static_cast<Amp>(0);
  Amp const af = has_first ? fabs(seg.first) : zero;
  Amp const am = mids ? fabs(seg.mid) : zero;
  Amp const al = (seg.flags & 2u) ? fabs(seg.last) : zero;
  Amp const px = fabs(seg.perp.x), py = fabs(seg.perp.y), pz = fabs(seg.perp.z);
  Amp const fs = sizeof(Amp) == sizeof(float) ? static_cast<Amp>(o.fixed_scale_f) : static_cast<Amp>(o.fixed_scale);
  Amp const largest = fmax(fmax(px, py), pz) * fmax(fmax(af, am), al) * fs;
  if (!(largest < static_cast<Amp>(0x1p62))) return false;  // also NaN and infinities
  Amp const sum = (af + am * static_cast<Amp>(mids) + al) * (px + py + pz) * fs *
                  static_cast<Amp>(1. + 0x1p-20);
  c.zhs += samples;
  c.mag += sizeof(Amp) == sizeof(float) ? static_cast<float>(sum)
                                        : __double2float_ru(static_cast<double>(sum));
  return true;
}

// The unchecked deposit of a warp's staged segments: deposit_staged's
// redistribution (every lane takes two bins of the flattened list per step),
// each sample converted and added to the window with no check, its counts
// and bound already taken by account_staged.  Every bin is below the trace's
// bins, which the window holds whole.
template <class Amp>
__device__ __forceinline__ void deposit_unchecked(StagedSegment<Amp>* staging, StagedSegment<Amp> const& seg,
                                                  ObserverCache const& o, WindowSink const& sink) {
  unsigned const lane = threadIdx.x & 31u;
  uint32_t const cnt = seg.count + ((seg.flags >> 1) & 1u);
  uint32_t incl = cnt;
#pragma unroll
  for (unsigned d = 1; d < 32u; d <<= 1) {
    uint32_t const v = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += v;
  }
  uint32_t const total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0u) return;
  staging[lane] = seg;
  __syncwarp();
  uint32_t const before_mine = incl - cnt;
  ObserverCache grid;  // the converting fields in registers
  grid.fixed_scale = o.fixed_scale;
  grid.fixed_scale_f = o.fixed_scale_f;
  // The adds go through a generic pointer: where the compiler can tell the
  // window is shared memory it emits shared-space 64-bit atomics, which this
  // GPU executes as about one instruction per active lane (the ZHS track
  // loop alone, one pass of two, ran at twice the atomic wavefronts of the
  // single-pass kernel's generic adds on the same samples).
  unsigned long long* win = sink.win;
  asm volatile("" : "+l"(win));
  uint32_t const width = sink.width;
  // kPer bins per lane per step, their owner searches interleaved
  constexpr int kPer = sizeof(Amp) == sizeof(float) ? 2 : 4;  // measured best of 2 and 4
  for (uint32_t base = 0; base < total; base += 32u * kPer) {
    uint32_t owner[kPer], before[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) owner[u] = 0u;
#pragma unroll
    for (uint32_t step = 16; step >= 1u; step >>= 1) {
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        uint32_t const v = __shfl_sync(0xffffffffu, incl, owner[u] + step - 1u);
        if (v <= base + lane + 32u * u) owner[u] += step;
      }
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) before[u] = __shfl_sync(0xffffffffu, before_mine, owner[u] & 31u);
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      uint32_t const j = base + lane + 32u * u;
      if (j < total) {
        StagedSegment<Amp> const& g = staging[owner[u]];
        uint32_t const k = j - before[u];
        bool const last = k >= g.count;
        uint32_t const bin = last ? g.last_bin : g.start + k;
        Amp const scale = last ? g.last : ((k == 0u && (g.flags & 1u)) ? g.first : g.mid);
        Vec3<Amp> const v = scaled(g.perp, scale);
        unsigned long long* const w = win + bin;
        atomicAdd(w, static_cast<unsigned long long>(fixed_value(v.x, grid)));
        atomicAdd(w + width, static_cast<unsigned long long>(fixed_value(v.y, grid)));
        atomicAdd(w + 2 * width, static_cast<unsigned long long>(fixed_value(v.z, grid)));
      }
    }
  }
  __syncwarp();
}

// accumulate_zhs, RadioProjection.inl:483-529, every decision exact.
template <bool kFixed, bool kRuns, class Amp, class Sink>
__device__ __forceinline__ void zhs_pair(Track const& t, Propagation const& p,
                                         ObserverCache const& o, Sink& sink, Counts& c) {
  double const mx = (t.sx + t.ex) * 0.5, my = (t.sy + t.ey) * 0.5, mz = (t.sz + t.ez) * 0.5;
  Path const pm = propagate<false>(p, o, mx, my, mz);
  double const uk = (t.bx * pm.kx + t.by * pm.ky + t.bz * pm.kz) / t.beta_module;
  double const s2 = 1. - uk * uk;
  double const fraunhofer = s2 * t.length * t.length / pm.dist / o.wavelength * 2. * kPi;
  double divisor = 1.;
  int subtracks = 1;
  if (fraunhofer > 1.) {
    divisor = sqrt(fraunhofer) + 1.;
    subtracks = x86_int(ceil(divisor));
  }
  c.subtracks += static_cast<unsigned long long>(static_cast<long long>(subtracks));
  int const refinement = static_cast<int>(p.refinement);
  // One segment when undivided: the loop below then evaluates
  // point2 = start + (end - start) / 1 / 1, exactly the reference's values.
  bool const subdivided = subtracks > 1 || refinement > 1;
  double rx = t.ex - t.sx, ry = t.ey - t.sy, rz = t.ez - t.sz, rt = t.te - t.ts;
  if (refinement > 1) {  // x / 1 == x exactly: undivided tracks skip the divisions
    double const rd = static_cast<double>(refinement);
    rx = rx / divisor / rd;
    ry = ry / divisor / rd;
    rz = rz / divisor / rd;
    rt = rt / divisor / rd;
  } else if (subdivided) {
    rx = rx / divisor;
    ry = ry / divisor;
    rz = rz / divisor;
    rt = rt / divisor;
  }
  double p1x = t.sx, p1y = t.sy, p1z = t.sz, t1 = t.ts;
  // subtrack-major, refinement-minor order of the reference's nested loops
  long long const segments = static_cast<long long>(subtracks) * refinement;
#pragma unroll 1
  for (long long index = 0; index < segments; ++index) {
    double const p2x = p1x + rx, p2y = p1y + ry, p2z = p1z + rz, t2 = t1 + rt;
    zhs_segment<kFixed, kRuns, false, Amp>(p1x, p1y, p1z, p2x, p2y, p2z, t1, t2, t, p, o, sink, c,
                                           subdivided);
    p1x = p2x;
    p1y = p2y;
    p1z = p2z;
    t1 = t2;
  }
  if (refinement > 1)
    c.subtracks += static_cast<unsigned long long>(
        static_cast<long long>(subtracks * (refinement - 1)));
}

// The common ZHS pair of the windowed kernel: one undivided segment, staged
// for the warp's cooperative deposit.  Returns false, staging nothing (`seg`
// cleared), when the track is subdivided (Fraunhofer number above 1, or
// refinement), when (kFilter) the Fraunhofer test is not surely below 1, or
// when zhs_stage declines the segment; the kernel then defers the pair to
// zhs_drain.  The FP32 Fraunhofer test and the staging of the one segment
// are independent and both evaluated; the test decides at the end.
//
// kFilter: F is estimated in FP32 as sin^2(theta) K with
// sin^2 = |beta x d|^2 / (|beta|^2 |d|^2) and K = 2 pi L^2 / (|d| lambda); its
// distance from the reference's FP64 F is at most 1.7e-6 sqrt(K F) + 4e-6 F +
// 1e-12 K (cross-product cancellation, the FP32 roundings and the approximate
// reciprocals; used with margins of 2.3x and more), so an estimate surely
// below 1 decides "one segment" exactly as the reference does.
template <bool kFilter, bool kPre, class Amp>
__device__ __forceinline__ bool zhs_common(Track const& t, Propagation const& p,
                                           ObserverCache const& o, Counts& c,
                                           StagedSegment<Amp>& seg, SourceTerms const& pre_mid) {
  if (p.refinement != 1u) return false;
  double const mx = (t.sx + t.ex) * 0.5, my = (t.sy + t.ey) * 0.5, mz = (t.sz + t.ez) * 0.5;
  bool surely_one = true;
  if (kFilter) {
    float const dx = static_cast<float>(o.px - mx), dy = static_cast<float>(o.py - my),
                dz = static_cast<float>(o.pz - mz);
    float const bx = static_cast<float>(t.bx), by = static_cast<float>(t.by),
                bz = static_cast<float>(t.bz);
    float const cx = by * dz - bz * dy, cy = bz * dx - bx * dz, cz = bx * dy - by * dx;
    float const d2 = dx * dx + dy * dy + dz * dz;
    float const b2 = bx * bx + by * by + bz * bz;
    float const length = static_cast<float>(t.length);
    // approximate reciprocals and square roots (relative errors near 2^-21,
    // inside the 4e-5 (f + 1) term below)
    float const s2 = __fdividef(cx * cx + cy * cy + cz * cz, b2 * d2);
    float const k = __fdividef(6.2831853f * length * length * rsqrtf(d2), static_cast<float>(o.wavelength));
    float const f = s2 * k;
    float const kf = k * (f + 1.f);
    float const root = kf > 0.f ? kf * rsqrtf(kf) : 0.f;
    float const margin = 4.e-6f * root + 4.e-5f * (f + 1.f) + 4.e-12f * k;
    surely_one = f + margin < 1.f;
  } else {
    Path const pm = propagate<false>(p, o, mx, my, mz);
    double const uk = (t.bx * pm.kx + t.by * pm.ky + t.bz * pm.kz) / t.beta_module;
    double const s2 = 1. - uk * uk;
    double const fraunhofer = s2 * t.length * t.length / pm.dist / o.wavelength * 2. * kPi;
    if (fraunhofer > 1.) return false;
  }
  bool const staged = zhs_stage<kFilter, Amp, kPre>(t.sx, t.sy, t.sz, t.sx + (t.ex - t.sx), t.sy + (t.ey - t.sy),
                                     t.sz + (t.ez - t.sz), t.ts, t.ts + (t.te - t.ts), t, p, o, false,
                                     seg, pre_mid);
  if (!(staged && surely_one)) {
    seg.count = 0u;
    seg.flags = 0u;
    return false;
  }
  c.subtracks += 1ull;
  return true;
}

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ Track load_track(const double* __restrict__ base, uint64_t stride,
                                            uint64_t i) {
  (void)stride;
  double2 const* r = track_ref(base, i);
  constexpr unsigned T = kTrackTile;
  double2 const a = __ldg(r + 0 * T), b = __ldg(r + 1 * T), c = __ldg(r + 2 * T), d = __ldg(r + 3 * T);
  double2 const e = __ldg(r + 4 * T), f = __ldg(r + 5 * T), g = __ldg(r + 6 * T);
  Track t;
  t.sx = a.x;
  t.sy = a.y;
  t.sz = b.x;
  t.ex = b.y;
  t.ey = c.x;
  t.ez = c.y;
  t.ts = d.x;
  t.te = d.y;
  t.bx = e.x;
  t.by = e.y;
  t.bz = f.x;
  t.length = f.y;
  t.beta_module = g.x;
  t.constant = g.y;
  return t;
}

// A track staged in shared memory as one interleaved 192-byte record (plain
// loads: __ldg reads the global space only).
__device__ __forceinline__ Track load_staged_track(double const* base, unsigned i) {
  double2 const* r = reinterpret_cast<double2 const*>(base + i * kTrackDoubles);
  double2 const a = r[0], b = r[1], c = r[2], d = r[3], e = r[4], f = r[5], g = r[6];
  Track t;
  t.sx = a.x;
  t.sy = a.y;
  t.sz = b.x;
  t.ex = b.y;
  t.ey = c.x;
  t.ez = c.y;
  t.ts = d.x;
  t.te = d.y;
  t.bx = e.x;
  t.by = e.y;
  t.bz = f.x;
  t.length = f.y;
  t.beta_module = g.x;
  t.constant = g.y;
  return t;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int d = 16; d > 0; d >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, d));
  return v;
}

// Adds per-thread counts into the event counters: one atomic per warp.
// Every lane of the warp must call it.
__device__ __forceinline__ void flush_counts(Counts& c, DeviceCounters* counters) {
  unsigned long long const a = warp_sum(c.coreas), b = warp_sum(c.zhs),
                           s = warp_sum(c.subtracks), f = warp_sum(c.overflows);
  if ((threadIdx.x & 31) == 0) {
    if (a) atomicAdd(&counters->coreas_contributions, a);
    if (b) atomicAdd(&counters->zhs_contributions, b);
    if (s) atomicAdd(&counters->zhs_subtracks, s);
    if (f) atomicAdd(&counters->fixed_point_overflows, f);
  }
  c = Counts{};
}

// RadioAtomicOperations::maximum (RadioAtomicOperations.inl:46-56): finite,
// non-negative maxima compare as their bit patterns.
__device__ __forceinline__ void atomic_max_nonnegative(double* address, double value) {
  atomicMax(reinterpret_cast<unsigned long long*>(address),
            static_cast<unsigned long long>(__double_as_longlong(value)));
}

// diagnostic_energy_bin, RadioProjection.inl:531-538.
__device__ __forceinline__ int energy_bin(double kinetic) {
  double const edges[14] = {1.e-3, 2.e-3, 5.e-3, 1.e-2, 2.e-2, 5.e-2, 1.e-1,
                            2.e-1, 5.e-1, 1.,    2.,    5.,    10.,   100.};
  int index = 0;
  while (index < 14 && kinetic > edges[index]) ++index;
  return index;
}

// ---------------------------------------------------------------- ingest
// The fields radio reads from a track step, from 752-byte records or from
// columns (one device array per field): the same arithmetic follows.
struct RecordSource {
  const c8r_lepton_transport_record* records;
  __device__ int pid(uint64_t i) const { return records[i].start.pid; }
  __device__ double weight(uint64_t i) const { return records[i].start.weight; }
  __device__ double start_energy(uint64_t i) const { return records[i].start.energy_gev; }
  __device__ double start_position(uint64_t i, int a) const { return records[i].start.position_m[a]; }
  __device__ double end_position(uint64_t i, int a) const { return records[i].end.position_m[a]; }
  __device__ double start_time(uint64_t i) const { return records[i].start.time_s; }
  __device__ double end_time(uint64_t i) const { return records[i].end.time_s; }
  __device__ double start_direction(uint64_t i, int a) const { return records[i].start.direction[a]; }
  __device__ double end_direction(uint64_t i, int a) const { return records[i].end.direction[a]; }
};

struct ColumnSource {
  c8r_track_columns columns;
  __device__ int pid(uint64_t i) const { return columns.pid[i]; }
  __device__ double weight(uint64_t i) const { return columns.weight[i]; }
  __device__ double start_energy(uint64_t i) const { return columns.start_energy_gev[i]; }
  __device__ double start_position(uint64_t i, int a) const { return columns.start_position_m[a][i]; }
  __device__ double end_position(uint64_t i, int a) const { return columns.end_position_m[a][i]; }
  __device__ double start_time(uint64_t i) const { return columns.start_time_s[i]; }
  __device__ double end_time(uint64_t i) const { return columns.end_time_s[i]; }
  __device__ double start_direction(uint64_t i, int a) const { return columns.start_direction[a][i]; }
  __device__ double end_direction(uint64_t i, int a) const { return columns.end_direction[a][i]; }
};

template <class Source>
__global__ void __launch_bounds__(256) ingest_kernel(
    const __grid_constant__ Source src, uint64_t count, double* __restrict__ tracks, uint64_t stride,
    unsigned long long* slot, DeviceCounters* counters, int diagnostics,
    const __grid_constant__ IngestTerms terms) {
  uint64_t const i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  bool valid = false;
  Track t;
  double duration = 0.;
  int pid = 0;
  if (i < count) {
    pid = src.pid(i);
    // make_radio_track_kinematics, RadioProjection.inl:145-168
    if (pid == 11 || pid == -11) {
      t.sx = src.start_position(i, 0);
      t.sy = src.start_position(i, 1);
      t.sz = src.start_position(i, 2);
      t.ex = src.end_position(i, 0);
      t.ey = src.end_position(i, 1);
      t.ez = src.end_position(i, 2);
      t.ts = src.start_time(i);
      t.te = src.end_time(i);
      duration = t.te - t.ts;
      double const dx = t.ex - t.sx, dy = t.ey - t.sy, dz = t.ez - t.sz;
      t.length = sqrt(dx * dx + dy * dy + dz * dz);
      if (duration > 0. && t.length > 0.) {
        double const denominator = kSpeedOfLight * duration;
        t.bx = dx / denominator;
        t.by = dy / denominator;
        t.bz = dz / denominator;
        t.beta_module = t.length / (kSpeedOfLight * duration);
        double const charge = pid == 11 ? -kElementaryCharge : kElementaryCharge;
        t.constant = charge * kEmConstant * src.weight(i);
        valid = true;
      }
    }
  }
  unsigned const ballot = __ballot_sync(0xffffffffu, valid);
  unsigned const lane = threadIdx.x & 31;
  unsigned long long base = 0;
  if (lane == 0 && ballot) base = atomicAdd(slot, static_cast<unsigned long long>(__popc(ballot)));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (valid) {
    uint64_t const j = base + __popc(ballot & ((1u << lane) - 1u));
    double2* r = track_ref(tracks, j);
    constexpr unsigned T = kTrackTile;
    r[0 * T] = make_double2(t.sx, t.sy);
    r[1 * T] = make_double2(t.sz, t.ex);
    r[2 * T] = make_double2(t.ey, t.ez);
    r[3 * T] = make_double2(t.ts, t.te);
    r[4 * T] = make_double2(t.bx, t.by);
    r[5 * T] = make_double2(t.bz, t.length);
    r[6 * T] = make_double2(t.beta_module, t.constant);
    if (terms.enabled) {
      // the source points of the windowed kernels, with the reference's own
      // arithmetic: the ZHS segment of an undivided track ends at
      // start + (end - start) (RadioProjection.inl:505-512), the CoREAS
      // near-cone midpoint is (start + end) / 2 (:357-359)
      Propagation const& p = terms.propagation;
      Destination const& d = terms.destination;
      SourceTerms const s = source_terms(p, d, t.sz);
      SourceTerms const e = source_terms(p, d, t.ez);
      SourceTerms const mz = source_terms(p, d, (t.sz + (t.sz + (t.ez - t.sz))) * 0.5);
      SourceTerms const mc = source_terms(p, d, (t.sz + t.ez) * 0.5);
      r[7 * T] = make_double2(s.n_dst, 0.);
      r[8 * T] = make_double2(s.factor, s.n_src);
      r[9 * T] = make_double2(e.factor, e.n_src);
      r[10 * T] = make_double2(mz.factor, mz.n_src);
      r[11 * T] = make_double2(mc.factor, mc.n_src);
    } else {
      r[7 * T] = make_double2(0., 0.);
    }
  }
  if (lane == 0 && ballot) atomicAdd(&counters->valid_tracks, static_cast<unsigned long long>(__popc(ballot)));
  if (!diagnostics) return;

  // record_track diagnostics, RadioProjection.inl:553-610 (warp-reduced).
  double w = 0., len = 0., wl = 0., ewl = 0., el = 0., pl = 0., sl = 0., dchg = 0., dchg2 = 0.,
         bdef = 0., tres = 0., maxlen = 0., maxchg = 0., sdx = 0., sdy = 0., sdz = 0.;
  int ebin = -1;
  double ebin_value = 0.;
  if (valid) {
    double const weight = src.weight(i);
    double const kinetic = src.start_energy(i) - kElectronMassGeV;
    if (isfinite(t.length) && t.length > 0. && isfinite(weight) && !(weight < 0.) &&
        isfinite(kinetic) && !(kinetic < 0.)) {
      double const weighted_length = weight * t.length;
      w = weight;
      len = t.length;
      wl = weighted_length;
      ewl = weighted_length * kinetic;
      maxlen = t.length;
      if (pid == 11) {
        el = weighted_length;
        sl = -weighted_length;
      } else {
        pl = weighted_length;
        sl = weighted_length;
      }
      ebin = energy_bin(kinetic);
      ebin_value = weighted_length;
      double direction_dot = 0.;
      double delta[3];
      for (int axis = 0; axis < 3; ++axis) {
        double const pre = src.start_direction(i, axis);
        double const post = src.end_direction(i, axis);
        direction_dot += pre * post;
        delta[axis] = post - pre;
      }
      double clamped = -1. > direction_dot ? -1. : direction_dot;
      clamped = 1. < clamped ? 1. : clamped;
      double const change = acos(clamped);
      double const residual = duration - t.length / kSpeedOfLight;
      dchg = weight * change;
      dchg2 = weight * change * change;
      bdef = weighted_length * (1. - t.beta_module);
      tres = weight * residual;
      maxchg = change;
      double const charge_sign = pid == 11 ? -1. : 1.;
      sdx = charge_sign * weight * delta[0];
      sdy = charge_sign * weight * delta[1];
      sdz = charge_sign * weight * delta[2];
    }
  }
  w = warp_sum(w);
  len = warp_sum(len);
  wl = warp_sum(wl);
  ewl = warp_sum(ewl);
  el = warp_sum(el);
  pl = warp_sum(pl);
  sl = warp_sum(sl);
  dchg = warp_sum(dchg);
  dchg2 = warp_sum(dchg2);
  bdef = warp_sum(bdef);
  tres = warp_sum(tres);
  sdx = warp_sum(sdx);
  sdy = warp_sum(sdy);
  sdz = warp_sum(sdz);
  maxlen = warp_max(maxlen);
  maxchg = warp_max(maxchg);
  if (lane == 0 && ballot) {
    atomicAdd(&counters->weighted_segment_count, w);
    atomicAdd(&counters->track_length_m, len);
    atomicAdd(&counters->weighted_track_length_m, wl);
    atomicAdd(&counters->energy_weighted_track_length_gev_m, ewl);
    atomicAdd(&counters->electron_weighted_track_length_m, el);
    atomicAdd(&counters->positron_weighted_track_length_m, pl);
    atomicAdd(&counters->signed_charge_weighted_track_length_m, sl);
    atomicAdd(&counters->weighted_direction_change_rad, dchg);
    atomicAdd(&counters->weighted_direction_change_squared_rad2, dchg2);
    atomicAdd(&counters->weighted_beta_deficit_track_length_m, bdef);
    atomicAdd(&counters->weighted_time_residual_s, tres);
    atomicAdd(&counters->signed_charge_weighted_direction_change[0], sdx);
    atomicAdd(&counters->signed_charge_weighted_direction_change[1], sdy);
    atomicAdd(&counters->signed_charge_weighted_direction_change[2], sdz);
    atomic_max_nonnegative(&counters->maximum_segment_length_m, maxlen);
    atomic_max_nonnegative(&counters->maximum_direction_change_rad, maxchg);
  }
  if (ebin >= 0) atomicAdd(&counters->weighted_track_length_by_kinetic_energy_m[ebin], ebin_value);
}

// ---------------------------------------------------------------- direct
template <bool kFixed, class Amp, bool kCoreas, bool kZhs>
__global__ void __launch_bounds__(256) direct_kernel(const __grid_constant__ EventPlan ev) {
  uint64_t const tracks = *ev.valid_tracks;
  uint32_t const observers =
      ev.observer_count[0] > ev.observer_count[1] ? ev.observer_count[0] : ev.observer_count[1];
  uint64_t const pairs = tracks * observers;
  Counts c;
  for (uint64_t pair = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; pair < pairs;
       pair += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint64_t const ti = pair / observers;
    uint32_t const oi = static_cast<uint32_t>(pair - ti * observers);
    Track const t = load_track(ev.tracks, ev.stride, ti);
    if (kCoreas && oi < ev.observer_count[0]) {
      ObserverCache const& o = ev.observers[0][oi];
      GlobalSink sink;
      for (int r = 0; r < 3; ++r) {
        sink.row[r] = kFixed ? ev.fixed[0] + r * ev.total_bins[0] + o.offset : nullptr;
        sink.frow[r] = kFixed ? nullptr : ev.floating[0] + r * ev.total_bins[0] + o.offset;
      }
      coreas_pair<kFixed, Amp>(t, ev.propagation, o, sink, c);
    }
    if (kZhs && oi < ev.observer_count[1]) {
      ObserverCache const& o = ev.observers[1][oi];
      GlobalSink sink;
      for (int r = 0; r < 3; ++r) {
        sink.row[r] = kFixed ? ev.fixed[1] + r * ev.total_bins[1] + o.offset : nullptr;
        sink.frow[r] = kFixed ? nullptr : ev.floating[1] + r * ev.total_bins[1] + o.offset;
      }
      zhs_pair<kFixed, false, Amp>(t, ev.propagation, o, sink, c);
    }
  }
  flush_counts(c, ev.counters);
}

// ---------------------------------------------------------------- tiled
// The reference's large-batch launch shape (RadioTileProjection,
// RadioAccumulator.inl:13-85, launched by project(), :699-847, for batches
// of 16384 tracks or more on a GPU): one 256-thread CTA per tile of
// kTileTracks tracks x kTileObservers observers, the tile's track kinematics
// and observer constants staged in shared memory, one thread per pair (lane
// l takes track l / 32 at observer l % 32, so a warp holds one track at 32
// observers), every sample a checked 64-bit global atomic.  Tiles are taken
// by a grid-stride loop over track tile x observer tile.
constexpr int kTileTracks = 8;      // RadioAccumulator.hpp:61 (TrackTileSize)
constexpr int kTileObservers = 32;  // RadioAccumulator.hpp:62 (ObserverTileSize)
constexpr int kTileThreads = kTileTracks * kTileObservers;
static_assert(sizeof(ObserverCache) % sizeof(double2) == 0, "observer constants in 16-byte words");

template <bool kFixed, class Amp, bool kCoreas, bool kZhs>
__global__ void __launch_bounds__(kTileThreads) tiled_kernel(const __grid_constant__ EventPlan ev,
                                                              uint64_t track_tiles) {
  __shared__ __align__(16) double tracks[kTileTracks * kTrackDoubles];
  __shared__ ObserverCache observers[2][kTileObservers];
  uint64_t const valid = *ev.valid_tracks;
  uint32_t const observer_count =
      ev.observer_count[0] > ev.observer_count[1] ? ev.observer_count[0] : ev.observer_count[1];
  uint64_t const observer_tiles = (observer_count + kTileObservers - 1) / kTileObservers;
  uint64_t const tiles = track_tiles * observer_tiles;
  unsigned const track_lane = threadIdx.x / kTileObservers;
  unsigned const observer_lane = threadIdx.x % kTileObservers;
  Counts c;
  for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    uint64_t const track_base = (tile / observer_tiles) * kTileTracks;
    uint64_t const observer_base = (tile % observer_tiles) * kTileObservers;
    __syncthreads();  // the previous tile's reads are done
    // column-major over the tile's tracks: consecutive threads read
    // consecutive tracks of one column (kTileTracks divides kTrackTile)
    for (unsigned i = threadIdx.x; i < kTileTracks * kTrackColumns; i += blockDim.x) {
      unsigned const k = i / kTileTracks, lane = i % kTileTracks;
      uint64_t const row = track_base + lane;
      reinterpret_cast<double2*>(tracks)[lane * kTrackColumns + k] =
          row < valid ? __ldg(track_ref(ev.tracks, row) + k * kTrackTile) : make_double2(0., 0.);
    }
    constexpr unsigned kWords = sizeof(ObserverCache) / sizeof(double2);
    for (int a = 0; a < 2; ++a) {
      if (!(a == 0 ? kCoreas : kZhs)) continue;
      for (unsigned i = threadIdx.x; i < kTileObservers * kWords; i += blockDim.x) {
        uint64_t const index = observer_base + i / kWords;
        if (index < ev.observer_count[a])
          reinterpret_cast<double2*>(observers[a])[i] =
              __ldg(reinterpret_cast<double2 const*>(ev.observers[a] + observer_base) + i);
      }
    }
    __syncthreads();
    uint64_t const ti = track_base + track_lane;
    uint64_t const oi = observer_base + observer_lane;
    if (ti < valid) {
      Track const t = load_staged_track(tracks, track_lane);
      if (kCoreas && oi < ev.observer_count[0]) {
        ObserverCache const& o = observers[0][observer_lane];
        GlobalSink sink;
        for (int r = 0; r < 3; ++r) {
          sink.row[r] = kFixed ? ev.fixed[0] + r * ev.total_bins[0] + o.offset : nullptr;
          sink.frow[r] = kFixed ? nullptr : ev.floating[0] + r * ev.total_bins[0] + o.offset;
        }
        coreas_pair<kFixed, Amp>(t, ev.propagation, o, sink, c);
      }
      if (kZhs && oi < ev.observer_count[1]) {
        ObserverCache const& o = observers[1][observer_lane];
        GlobalSink sink;
        for (int r = 0; r < 3; ++r) {
          sink.row[r] = kFixed ? ev.fixed[1] + r * ev.total_bins[1] + o.offset : nullptr;
          sink.frow[r] = kFixed ? nullptr : ev.floating[1] + r * ev.total_bins[1] + o.offset;
        }
        zhs_pair<kFixed, false, Amp>(t, ev.propagation, o, sink, c);
      }
    }
  }
  flush_counts(c, ev.counters);
}

// ---------------------------------------------------------------- windowed
constexpr int kWindowThreadsMax = kWindowThreads;
// Threads of a CTA of the one-pass ZHS kernel (floating traces, the
// no-allocation entry point, launches past the two-pass storage cap, and the
// third pass of two-pass launches).  Its drain's live state needs more
// registers than its track loop (168 against 112 in FP32, 135 in FP64), so a
// CTA sized for the drain runs 12 warps an SM.  Measured on the 1e7 x 160
// workload in one pass (ms per ZHS launch), FP32: 384 threads 96.8, 512
// 100.9, 576 97.3, 640 88.3, 768 79.9, 832 82.7, 864 80.6 -- the track loop
// gains more from the warps than the drain loses to its spills; FP64: 384
// 117.0, 480 128.5.
constexpr int kZhsThreadsFloat = 768;
constexpr int kZhsThreadsDouble = 384;
// Two passes (fixed point): the track loop alone runs larger CTAs (FP32 768
// threads, FP64 480: the most its 72-byte staging slots allow beside an
// 8192-bin window), the drain pass FP32 512 (ZHS 62.0 -> 60.7 ms on the 1e7 x
// 160 workload against 384; 768 ran slower), FP64 384.  FP64 track loops of
// 512 threads with unpadded 64-byte slots ran 110.3 ms against 96.2.
constexpr int kZhsLoopThreadsFloat = 768;
constexpr int kZhsLoopThreadsDouble = 480;
constexpr int kZhsDrainThreadsFloat = 512;
constexpr int kZhsDrainThreadsDouble = 384;
// kPass: 0 one pass; of a two-pass launch 1 the track loop, 2 the drain, 3
// the handed-back items in full (as one pass).
template <class Amp, int kPass = 0>
constexpr int zhs_threads_max() {
  return kPass == 2   ? (sizeof(Amp) == sizeof(float) ? kZhsDrainThreadsFloat : kZhsDrainThreadsDouble)
         : kPass == 1 ? (sizeof(Amp) == sizeof(float) ? kZhsLoopThreadsFloat : kZhsLoopThreadsDouble)
                      : (sizeof(Amp) == sizeof(float) ? kZhsThreadsFloat : kZhsThreadsDouble);
}
// The ZHS block for a team of `threads`: the team when it is smaller than the
// default team, else the largest block of the amplitude type and pass.
template <class Amp, int kPass = 0>
constexpr int zhs_block(int threads) {
  return threads < kWindowThreads
             ? (threads < zhs_threads_max<Amp, kPass>() ? threads : zhs_threads_max<Amp, kPass>())
             : zhs_threads_max<Amp, kPass>();
}
// staging slots of the ZHS kernel: 32 per warp of its largest CTA
template <class Amp>
constexpr size_t staging_bytes() {
  int const a = zhs_threads_max<Amp, 0>(), b = zhs_threads_max<Amp, 1>(), c = zhs_threads_max<Amp, 2>();
  int const most = a > b ? (a > c ? a : c) : (b > c ? b : c);
  return static_cast<size_t>(most) * sizeof(StagedSegment<Amp>);
}
constexpr size_t kStagingBytes =
    staging_bytes<float>() > staging_bytes<double>() ? staging_bytes<float>() : staging_bytes<double>();

__device__ __forceinline__ uint32_t find_event(EventPlan const* events, uint32_t n, uint64_t item) {
  uint32_t lo = 0, hi = n;  // last event with first_item <= item
  while (hi - lo > 1) {
    uint32_t const mid = (lo + hi) >> 1;
    if (events[mid].first_item <= item)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Deferred ZHS pairs of the windowed kernel, drained by the whole warp
// (accumulate_zhs, RadioProjection.inl:483-529).  Lanes below `count` take
// one deferred pair each and evaluate its Fraunhofer number and subdivision
// exactly; the warp then steps through segment index s = 0, 1, ...: every lane
// whose pair has a segment s forms its endpoints by the reference's
// sequential additions, stages it (kFilter: the filtered decisions first, the
// exact ones where those are ambiguous), and the warp deposits the staged
// samples together.  A segment that needs the per-index binning deposits on
// its own lane.  Every lane of the warp calls it.
template <bool kFixed, bool kFilter, class Amp, class Sink>
__device__ __noinline__ Counts zhs_drain(const double* __restrict__ tracks, uint64_t begin,
                                         unsigned const* list, unsigned count,
                                         Propagation const& p, ObserverCache const& o, Sink sink,
                                         StagedSegment<Amp>* staging) {
  Counts c;
  unsigned const lane = threadIdx.x & 31u;
  uint64_t row = 0;
  long long segments = 0;
  bool subdivided = false;
  double p1x = 0., p1y = 0., p1z = 0., t1 = 0., rx = 0., ry = 0., rz = 0., rt = 0.;
  if (lane < count) {
    row = begin + list[lane];
    Track const t = load_track(tracks, 0, row);
    double const mx = (t.sx + t.ex) * 0.5, my = (t.sy + t.ey) * 0.5, mz = (t.sz + t.ez) * 0.5;
    Path const pm = propagate<false>(p, o, mx, my, mz);
    double const uk = (t.bx * pm.kx + t.by * pm.ky + t.bz * pm.kz) / t.beta_module;
    double const s2 = 1. - uk * uk;
    double const fraunhofer = s2 * t.length * t.length / pm.dist / o.wavelength * 2. * kPi;
    double divisor = 1.;
    int subtracks = 1;
    if (fraunhofer > 1.) {
      divisor = sqrt(fraunhofer) + 1.;
      subtracks = x86_int(ceil(divisor));
    }
    int const refinement = static_cast<int>(p.refinement);
    c.subtracks += static_cast<unsigned long long>(static_cast<long long>(subtracks));
    if (refinement > 1)
      c.subtracks += static_cast<unsigned long long>(
          static_cast<long long>(subtracks * (refinement - 1)));
    subdivided = subtracks > 1 || refinement > 1;
    rx = t.ex - t.sx;
    ry = t.ey - t.sy;
    rz = t.ez - t.sz;
    rt = t.te - t.ts;
    if (refinement > 1) {  // x / 1 == x exactly: undivided tracks skip the divisions
      double const rd = static_cast<double>(refinement);
      rx = rx / divisor / rd;
      ry = ry / divisor / rd;
      rz = rz / divisor / rd;
      rt = rt / divisor / rd;
    } else if (subdivided) {
      rx = rx / divisor;
      ry = ry / divisor;
      rz = rz / divisor;
      rt = rt / divisor;
    }
    segments = static_cast<long long>(subtracks) * refinement;
    p1x = t.sx;
    p1y = t.sy;
    p1z = t.sz;
    t1 = t.ts;
  }
#pragma unroll 1
  for (long long s = 0; __any_sync(0xffffffffu, s < segments); ++s) {
    StagedSegment<Amp> seg;
    seg.count = 0u;
    seg.flags = 0u;
    if (s < segments) {
      // velocity and charge constant read again each step (L1): fewer
      // registers held across the warp's steps
      double2 const* r = track_ref(tracks, row);
      asm volatile("" : "+l"(r));
      double2 const e = __ldg(r + 4 * kTrackTile), f = __ldg(r + 5 * kTrackTile), g = __ldg(r + 6 * kTrackTile);
      Track t;
      t.bx = e.x;
      t.by = e.y;
      t.bz = f.x;
      t.length = f.y;
      t.beta_module = g.x;
      t.constant = g.y;
      double const p2x = p1x + rx, p2y = p1y + ry, p2z = p1z + rz, t2 = t1 + rt;
      bool staged =
          zhs_stage<kFilter, Amp>(p1x, p1y, p1z, p2x, p2y, p2z, t1, t2, t, p, o, subdivided, seg);
      if (kFilter && !staged)
        staged = zhs_stage<false, Amp>(p1x, p1y, p1z, p2x, p2y, p2z, t1, t2, t, p, o, subdivided,
                                       seg);
      if (!staged) {
        seg.count = 0u;
        seg.flags = 0u;
        zhs_segment<kFixed, true, false, Amp>(p1x, p1y, p1z, p2x, p2y, p2z, t1, t2, t, p, o, sink,
                                              c, subdivided);
      }
      p1x = p2x;
      p1y = p2y;
      p1z = p2z;
      t1 = t2;
    }
    deposit_staged<kFixed>(staging, seg, o, sink, c);
  }
  return c;
}

// A deferred CoREAS pair of the windowed kernel, loaded and evaluated exactly
// out of line (the caller passes the row, not the 112-byte track).  `hint`
// (kCoreasNearCone, as the track loop decided it, else 0): the pair takes the
// near-Cherenkov branch in the order of bit 0, evaluated here directly.
template <bool kFixed, class Amp, bool kPre, class Sink>
__device__ __noinline__ Counts coreas_drain_pair(const double* __restrict__ tracks, uint64_t row,
                                                 unsigned hint, Propagation const& p,
                                                 ObserverCache const& o, Sink sink) {
  Counts c;
  if (hint & static_cast<unsigned>(kCoreasNearCone)) {
    SourceTerms mid{};
    if (kPre) {
      double2 const m = __ldg(track_ref(tracks, row) + kFactorMidCoreas / 2 * kTrackTile);
      mid = SourceTerms{m.x, m.y, 0.};
    }
    return coreas_near_cone<kFixed, Amp, kPre>(load_track(tracks, 0, row), p, o, sink, (hint & 1u) != 0u, mid);
  }
  if (kPre) {
    double2 const* r = track_ref(tracks, row);
    constexpr unsigned T = kTrackTile;
    double2 const n = __ldg(r + kNdstStart / 2 * T), s = __ldg(r + kFactorStart / 2 * T),
                  e = __ldg(r + kFactorEnd / 2 * T), m = __ldg(r + kFactorMidCoreas / 2 * T);
    SourceTerms const pre[3] = {{s.x, s.y, n.x}, {e.x, e.y, 0.}, {m.x, m.y, 0.}};
    coreas_pair<kFixed, Amp, Sink, true>(load_track(tracks, 0, row), p, o, sink, c, pre);
  } else {
    coreas_pair<kFixed, Amp>(load_track(tracks, 0, row), p, o, sink, c);
  }
  return c;
}

// The precomputed source terms of a track's common path (kTrackDoubles):
// CoREAS start and end (n_dst at the start), ZHS segment midpoint.
template <int kAlgorithm>
__device__ __forceinline__ void load_source_terms(const double* __restrict__ base, uint64_t i,
                                                  SourceTerms& a, SourceTerms& b) {
  double2 const* r = track_ref(base, i);
  constexpr unsigned T = kTrackTile;
  if (kAlgorithm == 0) {
    double2 const n = __ldg(r + kNdstStart / 2 * T), s = __ldg(r + kFactorStart / 2 * T),
                  e = __ldg(r + kFactorEnd / 2 * T);
    a = SourceTerms{s.x, s.y, n.x};
    b = SourceTerms{e.x, e.y, 0.};
  } else {
    double2 const m = __ldg(r + kFactorMidZhs / 2 * T);
    a = SourceTerms{m.x, m.y, 0.};
  }
}

// kPass 0: one pass over every item.  Two passes (fixed-point ZHS):
// kPass 1 runs the track loop alone with unchecked window adds, appends the
// deferred pairs of all its items to its CTA's list, flushes each item whose
// window bound holds and records where its deferred pairs are; an item whose
// bound does not hold, whose trace is longer than the window or whose pairs
// do not fit in the list is handed back unflushed, and once its list has
// overflowed a CTA hands back its later items unprojected.  kPass 2 drains
// each recorded item's pairs into a fresh window; kPass 3 projects the
// handed-back items in full, as kPass 0 does.  The drain needs more
// registers than the track loop (168 against 80 FP32, 118 FP64), so apart
// the track loop runs without spills in larger CTAs.
template <bool kFixed, class Amp, int kAlgorithm, bool kPre, int kPass = 0>
__global__ void __launch_bounds__(kAlgorithm == 1 ? zhs_threads_max<Amp, kPass>() : kWindowThreadsMax, 1)
    windowed_kernel(const __grid_constant__ WorkPlan plan) {
  static_assert(kPass == 0 || (kFixed && kAlgorithm == 1), "two passes: fixed-point ZHS");
  extern __shared__ __align__(16) unsigned long long window[];
  __shared__ unsigned long long item_shared;
  __shared__ ObserverCache observer;
  __shared__ float window_bound;
  __shared__ unsigned deferred_total;
  // this CTA's list of the deferred pairs of its current item (kPass 1: of
  // all its items, from `used` on; kPass 2: of the items it projects in full)
  unsigned* const deferred_list =
      kPass >= 2 ? plan.drain_deferred + static_cast<size_t>(blockIdx.x) * plan.deferred_stride
      : kPass == 1 ? plan.deferred + static_cast<size_t>(blockIdx.x) * plan.deferred_capacity
                   : plan.deferred + static_cast<size_t>(blockIdx.x) * plan.deferred_stride;
  uint32_t used = 0;  // kPass 1: entries of the list taken by earlier items
  bool full = false;  // kPass 1: the list overflowed; later items are handed back
  Counts c;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item_shared = atomicAdd(plan.next_item, 1u);
    __syncthreads();
    uint64_t const item = item_shared;
    if (item >= plan.total_items) break;
    EventPlan const& ev = plan.events[find_event(plan.events, plan.event_count, item)];
    constexpr int algorithm = kAlgorithm;
    uint64_t const local = item - ev.first_item;
    uint32_t const per_chunk = ev.observer_count[algorithm];
    uint64_t const slice_chunk = local / per_chunk;
    uint32_t const oi = static_cast<uint32_t>(local - slice_chunk * per_chunk);
    uint64_t const valid = *ev.valid_tracks;
    uint64_t const track_count = valid < ev.last_track ? valid : ev.last_track;
    uint64_t const begin = ev.first_track + slice_chunk * ev.chunk_size;
    ItemState state{blockIdx.x, used, 0u, 0u};
    if constexpr (kPass >= 2) {
      state = plan.item_state[item];
      if (kPass == 2 && (state.redo || state.count == 0u)) continue;  // nothing to drain
      if (kPass == 3 && !state.redo) continue;                          // done by passes 1-2
    }
    bool const drain_only = kPass == 2;
    if (begin >= track_count) {
      if (kPass == 1 && threadIdx.x == 0) plan.item_state[item] = state;
      continue;
    }
    uint64_t const end = begin + ev.chunk_size < track_count ? begin + ev.chunk_size : track_count;
    uint64_t const bins = ev.observers[algorithm][oi].bins;
    uint32_t const width = static_cast<uint32_t>(bins < ev.window ? bins : ev.window);
    if (kPass == 1 && (full || bins > width)) {  // handed back unprojected
      if (threadIdx.x == 0) {
        plan.item_state[item] = ItemState{blockIdx.x, used, 0u, 1u};
        if (plan.handbacks) atomicAdd(plan.handbacks, 1ull);
      }
      continue;
    }
    if (threadIdx.x == 0) observer = ev.observers[algorithm][oi];
    ObserverCache const& o = observer;

    // zero the window (3 rows of width bins); the barrier also publishes `observer`
    for (uint32_t j = threadIdx.x; j < 3 * width; j += blockDim.x) window[j] = 0ull;
    if (threadIdx.x == 0) window_bound = 0.f;
    __syncthreads();

    WindowSink sink;
    sink.win = window;
    sink.fwin = reinterpret_cast<double*>(window);
    sink.width = width;
    uint64_t const total = ev.total_bins[algorithm];
    for (int row = 0; row < 3; ++row) {
      sink.row[row] = kFixed ? ev.fixed[algorithm] + row * total + o.offset : nullptr;
      sink.frow[row] = kFixed ? nullptr : ev.floating[algorithm] + row * total + o.offset;
    }
    constexpr bool kFilter = sizeof(Amp) == sizeof(float);  // mixed precision
    // Deferred pairs (track offsets in the chunk: CoREAS pairs for the
    // near-Cherenkov branch or an exact evaluation, ZHS pairs with subdivided
    // tracks or an exact evaluation) leave the common path, so rare paths do
    // not hold up the other lanes: they go to the CTA's list in global memory
    // and all warps drain it, 32 pairs at a time, after the item's tracks.
    // The track loop then holds no call, which keeps its registers free.
    // per-warp staging slots of the ZHS kernel's cooperative deposit
    StagedSegment<Amp>* const staging =
        reinterpret_cast<StagedSegment<Amp>*>(window + 3 * static_cast<size_t>(plan.window)) +
        (threadIdx.x >> 5) * 32u;
    unsigned const lane = threadIdx.x & 31u;
    Counts const saved = c;
    bool redo = false;  // kPass 1: the item goes back to the second pass
    unsigned n = 0;     // deferred pairs of the item
    // Fixed point, whole trace in the window: the window takes unchecked
    // adds, and `c.mag` bounds the sum of |increments| of this thread.  If the
    // block's bound stays below 2^61, no partial sum of any bin can have left
    // the int64 range in any order, so no add overflowed; else the item is
    // run again with checked adds.  An FP32 sum of n terms is off by a factor
    // below 1 + n 2^-24, so a thread's sum counts only while the thread made
    // fewer than 2^22 adds (factor below 1 + 2^-2); a thread with more (its
    // deposits since the attempt began: contributions plus failed
    // conversions, an upper bound of its window adds) sends the item to the
    // checked run.  Bins past the window and the flush below are always
    // checked.
    for (int attempt = 0;; ++attempt) {
      if (attempt > 0) {
        for (uint32_t j = threadIdx.x; j < 3 * width; j += blockDim.x) window[j] = 0ull;
        __syncthreads();
      }
      sink.unchecked = kFixed && attempt == 0 && bins <= width;
      c.mag = 0.f;
      if (threadIdx.x == 0) deferred_total = 0u;
      __syncthreads();
      for (uint64_t base = begin; !drain_only && base < end; base += blockDim.x) {
        uint64_t const i = base + threadIdx.x;
        bool deferred = false;
        unsigned hint = 0u;  // CoREAS: the near-Cherenkov decision, in the list entry's top bits
        StagedSegment<Amp> seg;
        seg.count = 0u;
        seg.flags = 0u;
        if (i < end) {
          Track const t = load_track(ev.tracks, ev.stride, i);
          SourceTerms pa{}, pb{};
          if (kPre) load_source_terms<kAlgorithm>(ev.tracks, i, pa, pb);
          if constexpr (kAlgorithm == 0) {
            int const code = coreas_common<kFixed, kFilter, kPre, Amp>(t, ev.propagation, o, sink, c, pa, pb);
            deferred = code != kCoreasDeposited;
            hint = code >= kCoreasNearCone ? static_cast<unsigned>(code) << kDeferredHintShift : 0u;
          } else {
            deferred = !zhs_common<kFilter, kPre, Amp>(t, ev.propagation, o, c, seg, pa);
          }
        }
        if (kAlgorithm == 1) {
          if (kFixed && sink.unchecked) {
            if (!deferred && !account_staged(seg, o, c)) {
              seg.count = 0u;
              seg.flags = 0u;
              deferred = true;
              c.subtracks -= 1ull;  // the drain counts the pair's subtracks
            }
            deposit_unchecked(staging, seg, o, sink);
          } else {
            if constexpr (kPass != 1) deposit_staged<kFixed>(staging, seg, o, sink, c);
          }
        }
        unsigned const ballot = __ballot_sync(0xffffffffu, deferred);
        unsigned const rank = __popc(ballot & ((1u << lane) - 1u));
        if (ballot) {
          unsigned slot = 0;
          if (lane == 0) slot = atomicAdd(&deferred_total, static_cast<unsigned>(__popc(ballot)));
          slot = __shfl_sync(0xffffffffu, slot, 0);
          uint64_t const at = static_cast<uint64_t>(used) + slot + rank;  // used: 0 but in kPass 1
          if (deferred && (kPass != 1 || at < plan.deferred_capacity))
            deferred_list[at] = static_cast<unsigned>(i - begin) | hint;
        }
      }
      __syncthreads();
      // at most end - begin <= deferred_stride (kPass 1: over the list's end
      // when used + n is)
      n = drain_only ? state.count : deferred_total;
      if (kPass == 1 && static_cast<uint64_t>(used) + n > plan.deferred_capacity) {
        redo = true;
        full = true;
        break;
      }
      unsigned const* const list =
          drain_only ? plan.deferred + static_cast<size_t>(state.cta) * plan.deferred_capacity + state.begin
                     : deferred_list;
      for (unsigned from = (threadIdx.x >> 5) * 32u; kPass != 1 && from < n; from += (blockDim.x >> 5) * 32u) {
        unsigned const count = n - from < 32u ? n - from : 32u;
        Counts d;
        if constexpr (kAlgorithm == 1 && kPass == 1) {
          (void)count;
        } else if (kAlgorithm == 1) {
          d = zhs_drain<kFixed, kFilter, Amp>(ev.tracks, begin, list + from, count,
                                              ev.propagation, o, sink, staging);
        } else if (lane < count) {
          unsigned const entry = list[from + lane];
          d = coreas_drain_pair<kFixed, Amp, kPre>(ev.tracks, begin + (entry & kDeferredOffsetMask),
                                                   entry >> kDeferredHintShift, ev.propagation, o, sink);
        }
        c.coreas += d.coreas;
        c.zhs += d.zhs;
        c.subtracks += d.subtracks;
        c.overflows += d.overflows;
        c.mag += d.mag;
        __syncwarp();
      }
      __syncthreads();
      if (!sink.unchecked) break;
      unsigned long long const adds = (c.coreas - saved.coreas) + (c.zhs - saved.zhs) +
                                      (c.overflows - saved.overflows);
      double const mine = adds < (1ull << 22) ? static_cast<double>(c.mag) : static_cast<double>(INFINITY);
      float const thread_bound = static_cast<float>(warp_sum(mine));
      if (lane == 0) atomicAdd(&window_bound, thread_bound);
      __syncthreads();
      float const block_bound = window_bound;
      __syncthreads();
      if (block_bound < 0x1p61f) break;
      if (kPass == 1) {
        redo = true;
        break;
      }
      if (threadIdx.x == 0 && plan.reruns) atomicAdd(plan.reruns, 1ull);
      c = saved;
    }
    if constexpr (kPass == 1) {
      if (redo) {  // unflushed: the second pass projects the item in full
        c = saved;
        if (threadIdx.x == 0) {
          plan.item_state[item] = ItemState{blockIdx.x, used, 0u, 1u};
          if (plan.handbacks) atomicAdd(plan.handbacks, 1ull);
        }
        continue;
      }
      if (threadIdx.x == 0) plan.item_state[item] = ItemState{blockIdx.x, used, n, 0u};
      used += n;
    }

    // flush: non-zero bins, checked global adds
    for (uint32_t j = threadIdx.x; j < 3 * width; j += blockDim.x) {
      unsigned long long const v = window[j];
      if (v == 0ull) continue;
      uint32_t const row = j / width;
      uint32_t const bin = j - row * width;
      if (kFixed) {
        long long const inc = static_cast<long long>(v);
        if (!checked(atomicAdd(sink.row[row] + bin, v), inc)) ++c.overflows;
      } else {
        atomicAdd(sink.frow[row] + bin, __longlong_as_double(static_cast<long long>(v)));
      }
    }
    flush_counts(c, ev.counters);
  }
}

// ---------------------------------------------------------------- decode
__global__ void decode_kernel(const long long* __restrict__ fixed, double* __restrict__ out,
                              uint64_t total_bins, const uint64_t* __restrict__ offsets,
                              const double* __restrict__ factors) {
  uint32_t const o = blockIdx.y;
  uint64_t const begin = offsets[o], end = offsets[o + 1];
  double const f = factors[o];
  for (uint64_t i = begin + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < end;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    out[i] = static_cast<double>(fixed[i]) * f;
    out[total_bins + i] = static_cast<double>(fixed[total_bins + i]) * f;
    out[2 * total_bins + i] = static_cast<double>(fixed[2 * total_bins + i]) * f;
  }
}

// The output step on the device: CoREAS fields added as they are, ZHS
// potentials differentiated into fields E_i = -(A_{i+1} - A_i) fs at the bin
// midpoints (RadioProcess.inl:213-223; one sample fewer per observer), both
// added into `out` (the observer add of CorsikaOutputSink.inl:255-278).
// Values are the decoded traces: fixed x factor of the observer, or the FP64
// traces.  `out` rows are [X | Y | Z] of total_bins - observers (ZHS) or
// total_bins (CoREAS) values.
__global__ void output_kernel(const long long* __restrict__ fixed, const double* __restrict__ floating,
                              double* __restrict__ out, uint64_t total_bins,
                              const ObserverCache* __restrict__ observers, const double* __restrict__ factors,
                              uint32_t observer_count, int differentiate) {
  uint32_t const o = blockIdx.y;
  ObserverCache const& oc = observers[o];
  double const f = fixed ? factors[o] : 1.;
  uint64_t const bins = oc.bins;
  uint64_t const samples = differentiate ? (bins > 0 ? bins - 1 : 0) : bins;
  uint64_t const out_total = differentiate ? total_bins - observer_count : total_bins;
  uint64_t const out_offset = differentiate ? oc.offset - o : oc.offset;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < samples;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    for (int r = 0; r < 3; ++r) {
      uint64_t const j = r * total_bins + oc.offset + i;
      double const a = fixed ? static_cast<double>(fixed[j]) * f : floating[j];
      double value = a;
      if (differentiate) {
        double const b = fixed ? static_cast<double>(fixed[j + 1]) * f : floating[j + 1];
        value = -(b - a) * oc.sample_rate;
      }
      out[r * out_total + out_offset + i] += value;
    }
  }
}

template <bool kFixed, class Amp>
cudaError_t direct_dispatch(EventPlan const& ev, uint64_t bound, bool coreas, bool zhs,
                            cudaStream_t stream) {
  uint32_t const observers =
      ev.observer_count[0] > ev.observer_count[1] ? ev.observer_count[0] : ev.observer_count[1];
  uint64_t const pairs = bound * observers;
  if (pairs == 0) return cudaSuccess;
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint64_t blocks = (pairs + 255) / 256;
  uint64_t const cap = static_cast<uint64_t>(sms) * 16;
  if (blocks > cap) blocks = cap;
  unsigned const grid = static_cast<unsigned>(blocks);
  if (coreas && zhs)
    direct_kernel<kFixed, Amp, true, true><<<grid, 256, 0, stream>>>(ev);
  else if (coreas)
    direct_kernel<kFixed, Amp, true, false><<<grid, 256, 0, stream>>>(ev);
  else if (zhs)
    direct_kernel<kFixed, Amp, false, true><<<grid, 256, 0, stream>>>(ev);
  return cudaGetLastError();
}

template <bool kFixed, class Amp>
cudaError_t tiled_dispatch(EventPlan const& ev, uint64_t bound, bool coreas, bool zhs, cudaStream_t stream) {
  uint32_t const observers =
      ev.observer_count[0] > ev.observer_count[1] ? ev.observer_count[0] : ev.observer_count[1];
  if (bound == 0 || observers == 0) return cudaSuccess;
  uint64_t const track_tiles = (bound + kTileTracks - 1) / kTileTracks;
  uint64_t const tiles = track_tiles * ((observers + kTileObservers - 1) / kTileObservers);
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint64_t const cap = static_cast<uint64_t>(sms) * 64;
  unsigned const grid = static_cast<unsigned>(tiles < cap ? tiles : cap);
  if (coreas && zhs)
    tiled_kernel<kFixed, Amp, true, true><<<grid, kTileThreads, 0, stream>>>(ev, track_tiles);
  else if (coreas)
    tiled_kernel<kFixed, Amp, true, false><<<grid, kTileThreads, 0, stream>>>(ev, track_tiles);
  else if (zhs)
    tiled_kernel<kFixed, Amp, false, true><<<grid, kTileThreads, 0, stream>>>(ev, track_tiles);
  return cudaGetLastError();
}

// window rows | (ZHS) per-warp staging slots
template <class Amp>
size_t windowed_smem_bytes(uint32_t window, int algorithm) {
  return static_cast<size_t>(window) * 3 * sizeof(unsigned long long) +
         (algorithm == 1 ? staging_bytes<Amp>() : 0);
}

// Every event of the plan carries precomputed source terms.
bool plan_precomputed(WorkPlan const& plan) {
  if (plan.event_count == 0) return false;
  for (uint32_t e = 0; e < plan.event_count; ++e)
    if (!plan.events[e].precomputed) return false;
  return true;
}

template <bool kFixed, class Amp, int kAlgorithm, bool kPre, int kPass = 0>
cudaError_t windowed_launch(WorkPlan const& plan, int ctas, int threads, cudaStream_t stream) {
  size_t const bytes = windowed_smem_bytes<Amp>(plan.window, kAlgorithm);
  cudaError_t err = cudaFuncSetAttribute(windowed_kernel<kFixed, Amp, kAlgorithm, kPre, kPass>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(bytes));
  if (err != cudaSuccess) return err;
  int const block = kAlgorithm == 1 ? zhs_block<Amp, kPass>(threads) : threads;
  windowed_kernel<kFixed, Amp, kAlgorithm, kPre, kPass><<<ctas, block, bytes, stream>>>(plan);
  return cudaGetLastError();
}

// The passes of a two-pass fixed-point ZHS launch, one after the other on
// the stream: the track loop, the drain, and the handed-back items in full;
// the last two draw items from their own counter.
template <class Amp, bool kPre>
cudaError_t windowed_two_pass(WorkPlan const& plan, int ctas, int threads, cudaStream_t stream) {
  cudaError_t err = windowed_launch<true, Amp, 1, kPre, 1>(plan, ctas, threads, stream);
  if (err != cudaSuccess) return err;
  WorkPlan later = plan;
  later.next_item = plan.drain_next_item;
  err = cudaMemsetAsync(plan.drain_next_item, 0, sizeof(unsigned), stream);
  if (err != cudaSuccess) return err;
  err = windowed_launch<true, Amp, 1, kPre, 2>(later, ctas, threads, stream);
  if (err != cudaSuccess) return err;
  err = cudaMemsetAsync(plan.drain_next_item, 0, sizeof(unsigned), stream);
  if (err != cudaSuccess) return err;
  return windowed_launch<true, Amp, 1, kPre, 3>(later, ctas, threads, stream);
}

template <bool kFixed, class Amp, int kAlgorithm>
cudaError_t windowed_dispatch_algorithm(WorkPlan const& plan, int ctas, int threads,
                                        cudaStream_t stream) {
  if (plan.deferred == nullptr || plan.deferred_stride < deferred_list_stride(plan))
    return cudaErrorInvalidValue;
  bool const pre = plan_precomputed(plan);
  if (plan.item_state != nullptr) {
    if constexpr (kFixed && kAlgorithm == 1) {
      if (plan.drain_deferred == nullptr || plan.drain_next_item == nullptr ||
          plan.deferred_capacity < plan.deferred_stride)
        return cudaErrorInvalidValue;
      return pre ? windowed_two_pass<Amp, true>(plan, ctas, threads, stream)
                 : windowed_two_pass<Amp, false>(plan, ctas, threads, stream);
    } else {
      return cudaErrorInvalidValue;
    }
  }
  return pre ? windowed_launch<kFixed, Amp, kAlgorithm, true>(plan, ctas, threads, stream)
             : windowed_launch<kFixed, Amp, kAlgorithm, false>(plan, ctas, threads, stream);
}

template <bool kFixed, class Amp>
cudaError_t windowed_dispatch(WorkPlan const& plan, int ctas, int threads, cudaStream_t stream) {
  return plan.algorithm == 0
             ? windowed_dispatch_algorithm<kFixed, Amp, 0>(plan, ctas, threads, stream)
             : windowed_dispatch_algorithm<kFixed, Amp, 1>(plan, ctas, threads, stream);
}

template <bool kFixed, class Amp>
int ctas_per_sm(int window, int threads) {
  int worst = 1 << 30;
  auto probe = [&](auto kernel, int block, int algorithm) {
    size_t const bytes = windowed_smem_bytes<Amp>(static_cast<uint32_t>(window), algorithm);
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, block, bytes) != cudaSuccess)
      blocks = 0;
    worst = blocks < worst ? blocks : worst;
  };
  probe(windowed_kernel<kFixed, Amp, 0, false>, threads, 0);
  probe(windowed_kernel<kFixed, Amp, 0, true>, threads, 0);
  probe(windowed_kernel<kFixed, Amp, 1, false>, zhs_block<Amp>(threads), 1);
  probe(windowed_kernel<kFixed, Amp, 1, true>, zhs_block<Amp>(threads), 1);
  if constexpr (kFixed) {  // the two passes
    probe(windowed_kernel<true, Amp, 1, false, 1>, zhs_block<Amp, 1>(threads), 1);
    probe(windowed_kernel<true, Amp, 1, true, 1>, zhs_block<Amp, 1>(threads), 1);
    probe(windowed_kernel<true, Amp, 1, false, 2>, zhs_block<Amp, 2>(threads), 1);
    probe(windowed_kernel<true, Amp, 1, true, 2>, zhs_block<Amp, 2>(threads), 1);
    probe(windowed_kernel<true, Amp, 1, false, 3>, zhs_block<Amp, 3>(threads), 1);
    probe(windowed_kernel<true, Amp, 1, true, 3>, zhs_block<Amp, 3>(threads), 1);
  }
  return worst;
}

}  // namespace

cudaError_t launch_ingest(const c8r_lepton_transport_record* records, uint64_t count,
                          double* tracks, uint64_t stride, unsigned long long* slot,
                          DeviceCounters* counters, bool diagnostics, IngestTerms const& terms,
                          cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  uint64_t const blocks = (count + 255) / 256;
  ingest_kernel<RecordSource><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
      RecordSource{records}, count, tracks, stride, slot, counters, diagnostics, terms);
  return cudaGetLastError();
}

cudaError_t launch_ingest_columns(c8r_track_columns const& columns, uint64_t count, double* tracks,
                                  uint64_t stride, unsigned long long* slot, DeviceCounters* counters,
                                  bool diagnostics, IngestTerms const& terms, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  uint64_t const blocks = (count + 255) / 256;
  ingest_kernel<ColumnSource><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
      ColumnSource{columns}, count, tracks, stride, slot, counters, diagnostics, terms);
  return cudaGetLastError();
}

bool shared_destination(ObserverCache const* observers, std::size_t count, Destination& out) {
  if (count == 0) return false;
  Destination const first = destination_of_host(observers[0]);
  for (std::size_t i = 1; i < count; ++i) {
    Destination const d = destination_of_host(observers[i]);
    if (std::memcmp(&d.height, &first.height, sizeof(double)) != 0 || d.index != first.index ||
        std::memcmp(&d.n, &first.n, sizeof(double)) != 0 ||
        std::memcmp(&d.integral, &first.integral, sizeof(double)) != 0)
      return false;
  }
  out = first;
  return true;
}

cudaError_t launch_direct(EventPlan const& event, uint64_t track_bound, bool coreas, bool zhs,
                          bool fixed, Precision precision, cudaStream_t stream) {
  if (fixed) {
    return precision == Precision::kFP64
               ? direct_dispatch<true, double>(event, track_bound, coreas, zhs, stream)
               : direct_dispatch<true, float>(event, track_bound, coreas, zhs, stream);
  }
  return precision == Precision::kFP64
             ? direct_dispatch<false, double>(event, track_bound, coreas, zhs, stream)
             : direct_dispatch<false, float>(event, track_bound, coreas, zhs, stream);
}

cudaError_t launch_tiled(EventPlan const& event, uint64_t track_bound, bool coreas, bool zhs,
                         bool fixed, Precision precision, cudaStream_t stream) {
  if (fixed) {
    return precision == Precision::kFP64
               ? tiled_dispatch<true, double>(event, track_bound, coreas, zhs, stream)
               : tiled_dispatch<true, float>(event, track_bound, coreas, zhs, stream);
  }
  return precision == Precision::kFP64
             ? tiled_dispatch<false, double>(event, track_bound, coreas, zhs, stream)
             : tiled_dispatch<false, float>(event, track_bound, coreas, zhs, stream);
}

cudaError_t launch_windowed(WorkPlan const& plan, bool fixed, Precision precision, int ctas,
                            int threads, cudaStream_t stream) {
  if (plan.total_items == 0) return cudaSuccess;
  if (fixed)
    return precision == Precision::kFP64 ? windowed_dispatch<true, double>(plan, ctas, threads, stream)
                                         : windowed_dispatch<true, float>(plan, ctas, threads, stream);
  return precision == Precision::kFP64 ? windowed_dispatch<false, double>(plan, ctas, threads, stream)
                                       : windowed_dispatch<false, float>(plan, ctas, threads, stream);
}

int windowed_max_bins(int device) {
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  // static shared memory of the kernel is a few hundred bytes; keep 1 KiB spare
  int const usable = optin - 1024 - static_cast<int>(kStagingBytes);
  return usable > 0 ? usable / static_cast<int>(3 * sizeof(unsigned long long)) : 0;
}

int windowed_ctas_per_sm(int window, int threads, bool fixed, Precision precision) {
  if (fixed)
    return precision == Precision::kFP64 ? ctas_per_sm<true, double>(window, threads)
                                         : ctas_per_sm<true, float>(window, threads);
  return precision == Precision::kFP64 ? ctas_per_sm<false, double>(window, threads)
                                       : ctas_per_sm<false, float>(window, threads);
}

cudaError_t launch_output(const long long* fixed, const double* floating, double* out, uint64_t total_bins,
                          const ObserverCache* observers, const double* factors, uint32_t observer_count,
                          uint64_t max_bins, bool differentiate, cudaStream_t stream) {
  if (observer_count == 0 || total_bins == 0) return cudaSuccess;
  uint64_t bx = (max_bins + 255) / 256;
  if (bx > 64) bx = 64;
  if (bx == 0) bx = 1;
  dim3 const grid(static_cast<unsigned>(bx), observer_count);
  output_kernel<<<grid, 256, 0, stream>>>(fixed, floating, out, total_bins, observers, factors,
                                          observer_count, differentiate ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_decode(const long long* fixed, double* out, uint64_t total_bins,
                          const uint64_t* observer_offsets, const double* factors,
                          uint32_t observer_count, uint64_t max_bins, cudaStream_t stream) {
  if (observer_count == 0 || total_bins == 0) return cudaSuccess;
  uint64_t bx = (max_bins + 255) / 256;
  if (bx > 64) bx = 64;
  if (bx == 0) bx = 1;
  dim3 const grid(static_cast<unsigned>(bx), observer_count);
  decode_kernel<<<grid, 256, 0, stream>>>(fixed, out, total_bins, observer_offsets, factors);
  return cudaGetLastError();
}

}  // namespace c8r
