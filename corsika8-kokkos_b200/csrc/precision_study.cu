// precision_study.cu — the radio projection with its arrival-time arithmetic
// in a chosen type, for the precision study of the three arithmetics:
//
//   T = double   FP64 (the reference's arithmetic; reproduces its bins)
//   T = DF       compensated double-FP32: a value hi + lo of two floats
//   T = float    plain FP32
//
// Every operation that decides an arrival time, a bin, a branch or the
// Cherenkov denominator 1 - n beta.k — source-to-antenna differences,
// distances, emission directions, refractive indices and travel times,
// detection times and the sample grid — is evaluated in T, in the
// reference's association order (accumulate_co_reas / accumulate_zhs,
// corsika/detail/kokkos/radio/algorithms/RadioProjection.inl:170-529).  Field
// and potential amplitudes are FP32.  One thread per (track, antenna) pair,
// checked 64-bit global adds: this kernel measures arithmetic, not speed.
#include <cuda_runtime.h>

#include "../../include/c8radio.h"
#include "radio_kernels.cuh"

namespace c8r {
namespace {

// ---------------------------------------------------------------- DF
// Double-FP32 values and their arithmetic: Knuth's TwoSum (TAOCP vol. 2,
// 4.2.2), Dekker's Fast2Sum, the error-free product through a fused
// multiply-add, and the double-double algorithms of Hida, Li and Bailey
// (quotient by two correction steps, square root by one Newton step) with
// float components.  About 44 significant bits.
struct DF {
  float hi, lo;
};

__device__ __forceinline__ DF fast_two_sum(float a, float b) {
  float const s = a + b;
  return {s, b - (s - a)};
}
__device__ __forceinline__ DF two_sum(float a, float b) {
  float const s = a + b;
  float const bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ DF two_prod(float a, float b) {
  float const p = a * b;
  return {p, fmaf(a, b, -p)};
}

__device__ __forceinline__ DF add(DF a, DF b) {
  DF s = two_sum(a.hi, b.hi);
  DF const t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ DF neg(DF a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ DF sub(DF a, DF b) { return add(a, neg(b)); }
__device__ __forceinline__ DF mul(DF a, DF b) {
  DF p = two_prod(a.hi, b.hi);
  p.lo = fmaf(a.hi, b.lo, p.lo);
  p.lo = fmaf(a.lo, b.hi, p.lo);
  return fast_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ DF div(DF a, DF b) {
  float const q1 = a.hi / b.hi;
  DF r = sub(a, mul(b, DF{q1, 0.f}));
  float const q2 = r.hi / b.hi;
  r = sub(r, mul(b, DF{q2, 0.f}));
  float const q3 = r.hi / b.hi;
  return add(fast_two_sum(q1, q2), DF{q3, 0.f});
}
__device__ __forceinline__ DF tsqrt(DF a) {
  if (!(a.hi > 0.f)) return DF{0.f, 0.f};
  float const s = sqrtf(a.hi);
  DF const r = sub(a, two_prod(s, s));
  return fast_two_sum(s, r.hi / (2.f * s));
}
__device__ __forceinline__ DF tabs(DF a) { return a.hi < 0.f ? neg(a) : a; }
__device__ __forceinline__ double to_d(DF a) {
  return static_cast<double>(a.hi) + static_cast<double>(a.lo);
}

// double and float: the native operations
__device__ __forceinline__ double add(double a, double b) { return a + b; }
__device__ __forceinline__ double sub(double a, double b) { return a - b; }
__device__ __forceinline__ double mul(double a, double b) { return a * b; }
__device__ __forceinline__ double div(double a, double b) { return a / b; }
__device__ __forceinline__ double tsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ double tabs(double a) { return fabs(a); }
__device__ __forceinline__ double to_d(double a) { return a; }
__device__ __forceinline__ float add(float a, float b) { return a + b; }
__device__ __forceinline__ float sub(float a, float b) { return a - b; }
__device__ __forceinline__ float mul(float a, float b) { return a * b; }
__device__ __forceinline__ float div(float a, float b) { return a / b; }
__device__ __forceinline__ float tsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ float tabs(float a) { return fabsf(a); }
__device__ __forceinline__ double to_d(float a) { return a; }

template <class T>
__device__ __forceinline__ T from_d(double v);
template <>
__device__ __forceinline__ double from_d<double>(double v) {
  return v;
}
template <>
__device__ __forceinline__ float from_d<float>(double v) {
  return static_cast<float>(v);
}
template <>
__device__ __forceinline__ DF from_d<DF>(double v) {
  float const hi = static_cast<float>(v);
  return {hi, static_cast<float>(v - static_cast<double>(hi))};
}

// ---------------------------------------------------------------- geometry
template <class T>
struct PathT {
  T time, n_src, n_dst, dist, kx, ky, kz;
};

// propagate (RadioProjection.inl:170-238) in T.
template <class T>
__device__ PathT<T> propagate_t(Propagation const& p, ObserverCache const& o, T sx, T sy, T sz) {
  PathT<T> r;
  T const one = from_d<T>(1.);
  T const dx = sub(from_d<T>(o.px), sx), dy = sub(from_d<T>(o.py), sy), dz = sub(from_d<T>(o.pz), sz);
  T const dist = tsqrt(add(add(mul(dx, dx), mul(dy, dy)), mul(dz, dz)));
  r.kx = div(dx, dist);
  r.ky = div(dy, dist);
  r.kz = div(dz, dist);
  r.dist = dist;
  T const c = from_d<T>(kSpeedOfLight);
  if (p.homogeneous > 0.) {
    T const n = from_d<T>(p.homogeneous);
    r.time = div(mul(n, dist), c);
    r.n_src = r.n_dst = n;
    return r;
  }
  T const sh = mul(sub(sz, from_d<T>(p.min_height)), from_d<T>(p.inv_step));
  T const dh = from_d<T>(o.dest_height);
  double const lastd = static_cast<double>(p.table_size - 1);
  double const sh_half = to_d(add(sh, from_d<T>(0.5)));
  T n_src = one, i_src = one, n_dst = from_d<T>(o.dest_n), height = one;
  if (sh_half >= lastd) {
    double2 const t = p.table[p.table_size - 1];
    n_src = add(add(from_d<T>(t.x), mul(from_d<T>(p.slope_n_upper),
                                         tabs(mul(sub(sz, from_d<T>(p.max_height)), from_d<T>(p.inv_step))))),
                one);
    i_src = add(from_d<T>(t.y), mul(from_d<T>(p.slope_i_upper), tabs(sub(from_d<T>(p.max_height), sz))));
    height = sub(sh, dh);
  } else if (sh_half < lastd && to_d(sh) > 0.) {
    uint64_t const si = static_cast<uint64_t>(sh_half);
    double2 const t = p.table[si];
    n_src = add(from_d<T>(t.x), one);
    i_src = from_d<T>(t.y);
    height = mul(from_d<T>(static_cast<double>(static_cast<int64_t>(si) - static_cast<int64_t>(o.dest_index))),
                 from_d<T>(p.step));
    if (to_d(height) == 0.) height = one;
  } else if (to_d(sh) == 0.) {
    n_src = one;
    n_dst = one;
    i_src = from_d<T>(p.table[0].y);
    height = sub(dh, sh);
  } else {
    double2 const t0 = p.table[0];
    n_src = add(add(from_d<T>(t0.x), mul(from_d<T>(p.slope_n_lower), tabs(sh))), one);
    i_src = add(from_d<T>(t0.y), mul(from_d<T>(p.slope_i_lower), tabs(sh)));
    n_dst = one;
    height = sub(dh, tabs(sh));
  }
  r.time = div(mul(add(one, div(sub(i_src, from_d<T>(o.dest_integral)), height)), dist), c);
  r.n_src = n_src;
  r.n_dst = n_dst;
  return r;
}

// co_reas_doppler (RadioProjection.inl:113-143): the compensated recovery of
// an exact zero is kept for FP64; the other arithmetics take 1 - n beta.k.
template <class T>
__device__ __forceinline__ T doppler_t(T n, T bx, T by, T bz, T kx, T ky, T kz) {
  return sub(from_d<T>(1.), mul(n, add(add(mul(bx, kx), mul(by, ky)), mul(bz, kz))));
}
template <>
__device__ __forceinline__ double doppler_t<double>(double n, double bx, double by, double bz,
                                                    double kx, double ky, double kz) {
  return doppler(n, bx, by, bz, kx, ky, kz);
}

// ---------------------------------------------------------------- samples
struct StudySink {
  unsigned long long* row[3];
  double* frow[3];
};

__device__ __forceinline__ bool fixed_of(float v, ObserverCache const& o, long long& out) {
  if (o.count_samples) {
    out = 1;
    return true;
  }
  float const s = v * o.fixed_scale_f;
  if (!(fabsf(s) < 9223372036854775808.f)) return false;
  out = __float2ll_rn(s);
  return true;
}

__device__ __forceinline__ bool checked_add(unsigned long long* address, long long v) {
  long long const previous =
      static_cast<long long>(atomicAdd(address, static_cast<unsigned long long>(v)));
  return !((v > 0 && previous > LLONG_MAX - v) || (v < 0 && previous < LLONG_MIN - v));
}

// add_sample (RadioProjection.inl:263-301), the time and its bin in T.
template <bool kFixed, bool kPotential, class T>
__device__ void sample_t(ObserverCache const& o, StudySink const& sink, T t, Vec3<float> v,
                         unsigned long long& contributions, unsigned long long& overflows) {
  if (!kPotential && (to_d(t) < o.start_time || to_d(t) > o.end_time)) return;
  double const bv = nearest_bin(to_d(mul(sub(t, from_d<T>(o.start_time)), from_d<T>(o.sample_rate))));
  if (!(bv >= 0. && bv < o.bins_d)) return;
  uint64_t const bin = static_cast<uint64_t>(bv);
  if (bin >= o.bins) return;
  if (kFixed) {
    long long ix = 0, iy = 0, iz = 0;
    bool const ox = fixed_of(v.x, o, ix), oy = fixed_of(v.y, o, iy), oz = fixed_of(v.z, o, iz);
    bool ok = ox && oy && oz;
    if (ox) ok = checked_add(sink.row[0] + bin, ix) && ok;
    if (oy) ok = checked_add(sink.row[1] + bin, iy) && ok;
    if (oz) ok = checked_add(sink.row[2] + bin, iz) && ok;
    if (!ok) {
      ++overflows;
      return;
    }
  } else {
    atomicAdd(sink.frow[0] + bin, static_cast<double>(v.x));
    atomicAdd(sink.frow[1] + bin, static_cast<double>(v.y));
    atomicAdd(sink.frow[2] + bin, static_cast<double>(v.z));
  }
  ++contributions;
}

// separate_same_bin_endpoints (RadioProjection.inl:303-336) in T.
template <class T>
__device__ void separate_t(T& start, T& end, T res, bool signed_order) {
  double const qs = to_d(div(start, res)), qe = to_d(div(end, res));
  long long const sb = x86_ll(nearest_bin(qs));
  long long const eb = x86_ll(nearest_bin(qe));
  if (sb != eb) return;
  double const sf = qs - floor(qs);
  double const ef = qe - floor(qe);
  bool const forward = !signed_order || to_d(end) >= to_d(start);
  if (forward) {
    if (sf >= 0.5 && ef >= 0.5) start = sub(start, res);
    else if (sf < 0.5 && ef < 0.5) end = add(end, res);
    else if (ef >= 1. - sf) end = add(end, res);
    else start = sub(start, res);
  } else {
    if (sf >= 0.5 && ef >= 0.5) end = sub(end, res);
    else if (sf < 0.5 && ef < 0.5) start = add(start, res);
    else if (sf >= 1. - ef) start = add(start, res);
    else end = sub(end, res);
  }
}

__device__ __forceinline__ Vec3<float> scaled3(Vec3<float> v, float s) { return {v.x * s, v.y * s, v.z * s}; }

template <class T>
__device__ __forceinline__ Vec3<float> to_f(T x, T y, T z) {
  return {static_cast<float>(to_d(x)), static_cast<float>(to_d(y)), static_cast<float>(to_d(z))};
}

// ---------------------------------------------------------------- CoREAS
// accumulate_co_reas (RadioProjection.inl:339-409).
template <bool kFixed, class T>
__device__ void coreas_t(Track const& t, Propagation const& p, ObserverCache const& o,
                         StudySink const& sink, Counts& c) {
  T const sx = from_d<T>(t.sx), sy = from_d<T>(t.sy), sz = from_d<T>(t.sz);
  T const ex = from_d<T>(t.ex), ey = from_d<T>(t.ey), ez = from_d<T>(t.ez);
  T const bx = from_d<T>(t.bx), by = from_d<T>(t.by), bz = from_d<T>(t.bz);
  T const ts = from_d<T>(t.ts), te = from_d<T>(t.te);
  T const half = from_d<T>(0.5);
  PathT<T> const ps = propagate_t<T>(p, o, sx, sy, sz);
  PathT<T> const pe = propagate_t<T>(p, o, ex, ey, ez);
  T const pre = doppler_t<T>(ps.n_src, bx, by, bz, ps.kx, ps.ky, ps.kz);
  T const post = doppler_t<T>(pe.n_src, bx, by, bz, pe.kx, pe.ky, pe.kz);
  T sr = add(ts, ps.time);
  T er = add(te, pe.time);
  Vec3<float> const beta{static_cast<float>(t.bx), static_cast<float>(t.by), static_cast<float>(t.bz)};
  double const cf = t.constant * o.sample_rate;
  T const res = from_d<T>(o.resolution);
  if (to_d(ps.n_dst) > 1. && (fabs(to_d(pre)) < kCoreasThreshold || fabs(to_d(post)) < kCoreasThreshold)) {
    T const mx = mul(add(sx, ex), half), my = mul(add(sy, ey), half), mz = mul(add(sz, ez), half);
    T const mt = mul(add(ts, te), half);
    PathT<T> const pm = propagate_t<T>(p, o, mx, my, mz);
    T const mr = add(mt, pm.time);
    T const md = doppler_t<T>(pm.n_src, bx, by, bz, pm.kx, pm.ky, pm.kz);
    Vec3<float> const k = to_f(pm.kx, pm.ky, pm.kz);
    Vec3<float> fstart =
        scaled3(cross(k, cross(k, beta)), static_cast<float>(cf / to_d(mul(md, pm.dist))));
    Vec3<float> fend = scaled3(fstart, -1.f);
    T dt = mul(div(from_d<T>(t.length), mul(from_d<T>(kSpeedOfLight), from_d<T>(t.beta_module))),
               tabs(md));
    bool const forward = to_d(sr) < to_d(er);
    sr = forward ? sub(mr, mul(half, dt)) : add(mr, mul(half, dt));
    er = forward ? add(mr, mul(half, dt)) : sub(mr, mul(half, dt));
    dt = sub(er, sr);
    if (to_d(tabs(dt)) < to_d(res)) {
      float const s = static_cast<float>(fabs(to_d(div(dt, res))));
      fstart = scaled3(fstart, s);
      fend = scaled3(fend, s);
      separate_t<T>(sr, er, res, true);
    }
    sample_t<kFixed, false>(o, sink, sr, fstart, c.coreas, c.overflows);
    sample_t<kFixed, false>(o, sink, er, fend, c.coreas, c.overflows);
    return;
  }
  Vec3<float> const ks = to_f(ps.kx, ps.ky, ps.kz), ke = to_f(pe.kx, pe.ky, pe.kz);
  Vec3<float> fstart =
      scaled3(cross(ks, cross(ks, beta)), static_cast<float>(cf / to_d(mul(pre, ps.dist))));
  Vec3<float> fend =
      scaled3(cross(ke, cross(ke, beta)), static_cast<float>(-cf / to_d(mul(post, pe.dist))));
  if (to_d(pre) < 1.e-9 || to_d(post) < 1.e-9) {
    T const dt = sub(er, sr);
    if (to_d(tabs(dt)) < to_d(res)) {
      float const s = static_cast<float>(fabs(to_d(div(dt, res))));
      fstart = scaled3(fstart, s);
      fend = scaled3(fend, s);
      separate_t<T>(sr, er, res, false);
    }
  }
  sample_t<kFixed, false>(o, sink, sr, fstart, c.coreas, c.overflows);
  sample_t<kFixed, false>(o, sink, er, fend, c.coreas, c.overflows);
}

// ---------------------------------------------------------------- ZHS
// accumulate_zhs_segment (RadioProjection.inl:412-480), every index binned.
template <bool kFixed, class T>
__device__ void zhs_segment_t(T p1x, T p1y, T p1z, T p2x, T p2y, T p2z, T t1, T t2, Track const& t,
                              Propagation const& p, ObserverCache const& o, StudySink const& sink,
                              Counts& c, bool subdivided) {
  T const half = from_d<T>(0.5);
  T const mx = mul(add(p1x, p2x), half), my = mul(add(p1y, p2y), half), mz = mul(add(p1z, p2z), half);
  PathT<T> const path = propagate_t<T>(p, o, mx, my, mz);
  T const bx = from_d<T>(t.bx), by = from_d<T>(t.by), bz = from_d<T>(t.bz);
  T const bk = add(add(mul(bx, path.kx), mul(by, path.ky)), mul(bz, path.kz));
  T const nbk = mul(path.n_src, bk);
  T const mt = mul(add(t1, t2), half);
  T d1 = sub(add(t1, path.time), mul(nbk, sub(t1, mt)));
  T d2 = sub(add(t2, path.time), mul(nbk, sub(t2, mt)));
  double sign = 1.;
  if (to_d(d1) > to_d(d2)) {
    T const swap = d1;
    d1 = d2;
    d2 = swap;
    sign = -1.;
  }
  T const t0 = from_d<T>(o.start_time), fs = from_d<T>(o.sample_rate);
  T const x1 = mul(sub(d1, t0), fs), x2 = mul(sub(d2, t0), fs);
  double const sb = floor(to_d(add(x1, half)));
  double const eb = floor(to_d(add(x2, half)));
  Vec3<float> const k = to_f(path.kx, path.ky, path.kz);
  Vec3<float> const beta{static_cast<float>(t.bx), static_cast<float>(t.by), static_cast<float>(t.bz)};
  Vec3<float> const perp = cross(k, cross(beta, k));
  T const den = sub(from_d<T>(1.), nbk);
  double const dd = to_d(mul(den, path.dist));
  double const sc = sign * t.constant;
  if (sb == eb) {
    double amplitude;
    if (fabs(to_d(den)) > 1.e-15) {
      double const fraction = fabs(to_d(sub(mul(d2, fs), mul(d1, fs))));
      amplitude = sc * fraction / dd;
    } else {
      double const fraction = to_d(mul(sub(t2, t1), fs));
      amplitude = sc * fraction / to_d(path.dist);
    }
    sample_t<kFixed, true>(o, sink, d2, scaled3(perp, static_cast<float>(amplitude)), c.zhs, c.overflows);
    return;
  }
  int const nb = x86_int(eb - sb);
  double const frac_first = fabs(to_d(sub(from_d<T>(sb + 0.5), x1)));
  sample_t<kFixed, true>(o, sink, d1, scaled3(perp, static_cast<float>(sc * frac_first / dd)), c.zhs,
                         c.overflows);
  Vec3<float> const mid = scaled3(perp, static_cast<float>((subdivided ? 1. : sign) * t.constant / dd));
  for (int index = 1; index < nb; ++index)
    sample_t<kFixed, true>(o, sink, add(d1, div(from_d<T>(static_cast<double>(index)), fs)), mid, c.zhs,
                           c.overflows);
  double const frac_last = fabs(to_d(sub(add(x2, half), from_d<T>(eb))));
  sample_t<kFixed, true>(o, sink, d2, scaled3(perp, static_cast<float>(sc * frac_last / dd)), c.zhs,
                         c.overflows);
}

// accumulate_zhs (RadioProjection.inl:483-529): Fraunhofer subdivision in T.
template <bool kFixed, class T>
__device__ void zhs_t(Track const& t, Propagation const& p, ObserverCache const& o,
                      StudySink const& sink, Counts& c) {
  T const half = from_d<T>(0.5);
  T const sx = from_d<T>(t.sx), sy = from_d<T>(t.sy), sz = from_d<T>(t.sz);
  T const ex = from_d<T>(t.ex), ey = from_d<T>(t.ey), ez = from_d<T>(t.ez);
  T const mx = mul(add(sx, ex), half), my = mul(add(sy, ey), half), mz = mul(add(sz, ez), half);
  PathT<T> const pm = propagate_t<T>(p, o, mx, my, mz);
  T const bx = from_d<T>(t.bx), by = from_d<T>(t.by), bz = from_d<T>(t.bz);
  T const uk = div(add(add(mul(bx, pm.kx), mul(by, pm.ky)), mul(bz, pm.kz)), from_d<T>(t.beta_module));
  T const s2 = sub(from_d<T>(1.), mul(uk, uk));
  T const length = from_d<T>(t.length);
  T const fraunhofer = mul(mul(div(div(mul(mul(s2, length), length), pm.dist),
                                   from_d<T>(o.wavelength)), from_d<T>(2.)), from_d<T>(kPi));
  double divisor = 1.;
  int subtracks = 1;
  if (to_d(fraunhofer) > 1.) {
    divisor = to_d(add(tsqrt(fraunhofer), from_d<T>(1.)));
    subtracks = x86_int(ceil(divisor));
  }
  c.subtracks += static_cast<unsigned long long>(static_cast<long long>(subtracks));
  int const refinement = static_cast<int>(p.refinement);
  bool const subdivided = subtracks > 1 || refinement > 1;
  T rx = sub(ex, sx), ry = sub(ey, sy), rz = sub(ez, sz);
  T const ts = from_d<T>(t.ts);
  T rt = sub(from_d<T>(t.te), ts);
  if (subdivided) {
    T const dv = from_d<T>(divisor), rd = from_d<T>(static_cast<double>(refinement));
    rx = div(div(rx, dv), rd);
    ry = div(div(ry, dv), rd);
    rz = div(div(rz, dv), rd);
    rt = div(div(rt, dv), rd);
  }
  T p1x = sx, p1y = sy, p1z = sz, t1 = ts;
  long long const segments = static_cast<long long>(subtracks) * refinement;
  for (long long index = 0; index < segments; ++index) {
    T const p2x = add(p1x, rx), p2y = add(p1y, ry), p2z = add(p1z, rz), t2 = add(t1, rt);
    zhs_segment_t<kFixed, T>(p1x, p1y, p1z, p2x, p2y, p2z, t1, t2, t, p, o, sink, c, subdivided);
    p1x = p2x;
    p1y = p2y;
    p1z = p2z;
    t1 = t2;
  }
  if (refinement > 1)
    c.subtracks += static_cast<unsigned long long>(static_cast<long long>(subtracks * (refinement - 1)));
}

// ---------------------------------------------------------------- kernel
__device__ __forceinline__ unsigned long long lane_sum(unsigned long long v) {
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
  return v;
}

__device__ __forceinline__ Track study_track(const double* base, uint64_t i) {
  Track t;
  t.sx = track_field(base, i, kSx);
  t.sy = track_field(base, i, kSy);
  t.sz = track_field(base, i, kSz);
  t.ex = track_field(base, i, kEx);
  t.ey = track_field(base, i, kEy);
  t.ez = track_field(base, i, kEz);
  t.ts = track_field(base, i, kTs);
  t.te = track_field(base, i, kTe);
  t.bx = track_field(base, i, kBx);
  t.by = track_field(base, i, kBy);
  t.bz = track_field(base, i, kBz);
  t.length = track_field(base, i, kLen);
  t.beta_module = track_field(base, i, kBmod);
  t.constant = track_field(base, i, kConst);
  return t;
}

template <bool kFixed, class T, bool kCoreas, bool kZhs>
__global__ void __launch_bounds__(256) study_kernel(const __grid_constant__ EventPlan ev) {
  uint64_t const tracks = *ev.valid_tracks;
  uint32_t const observers =
      ev.observer_count[0] > ev.observer_count[1] ? ev.observer_count[0] : ev.observer_count[1];
  uint64_t const pairs = tracks * observers;
  Counts c;
  for (uint64_t pair = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; pair < pairs;
       pair += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint64_t const ti = pair / observers;
    uint32_t const oi = static_cast<uint32_t>(pair - ti * observers);
    Track const t = study_track(ev.tracks, ti);
    for (int a = 0; a < 2; ++a) {
      if ((a == 0 && !kCoreas) || (a == 1 && !kZhs) || oi >= ev.observer_count[a]) continue;
      ObserverCache const& o = ev.observers[a][oi];
      StudySink sink;
      for (int r = 0; r < 3; ++r) {
        sink.row[r] = kFixed ? ev.fixed[a] + r * ev.total_bins[a] + o.offset : nullptr;
        sink.frow[r] = kFixed ? nullptr : ev.floating[a] + r * ev.total_bins[a] + o.offset;
      }
      if (a == 0)
        coreas_t<kFixed, T>(t, ev.propagation, o, sink, c);
      else
        zhs_t<kFixed, T>(t, ev.propagation, o, sink, c);
    }
  }
  unsigned long long const a = lane_sum(c.coreas), b = lane_sum(c.zhs), s = lane_sum(c.subtracks),
                           f = lane_sum(c.overflows);
  if ((threadIdx.x & 31) == 0) {
    if (a) atomicAdd(&ev.counters->coreas_contributions, a);
    if (b) atomicAdd(&ev.counters->zhs_contributions, b);
    if (s) atomicAdd(&ev.counters->zhs_subtracks, s);
    if (f) atomicAdd(&ev.counters->fixed_point_overflows, f);
  }
}

template <bool kFixed, class T>
cudaError_t study_dispatch(EventPlan const& ev, uint64_t bound, bool coreas, bool zhs,
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
  dim3 const grid(static_cast<unsigned>(blocks));
  if (coreas && zhs)
    study_kernel<kFixed, T, true, true><<<grid, 256, 0, stream>>>(ev);
  else if (coreas)
    study_kernel<kFixed, T, true, false><<<grid, 256, 0, stream>>>(ev);
  else
    study_kernel<kFixed, T, false, true><<<grid, 256, 0, stream>>>(ev);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_study(EventPlan const& event, uint64_t track_bound, bool coreas, bool zhs,
                         bool fixed, TimeArithmetic arithmetic, cudaStream_t stream) {
  switch (arithmetic) {
    case TimeArithmetic::kDoubleFloat:
      return fixed ? study_dispatch<true, DF>(event, track_bound, coreas, zhs, stream)
                   : study_dispatch<false, DF>(event, track_bound, coreas, zhs, stream);
    case TimeArithmetic::kFloat:
      return fixed ? study_dispatch<true, float>(event, track_bound, coreas, zhs, stream)
                   : study_dispatch<false, float>(event, track_bound, coreas, zhs, stream);
    default:
      return fixed ? study_dispatch<true, double>(event, track_bound, coreas, zhs, stream)
                   : study_dispatch<false, double>(event, track_bound, coreas, zhs, stream);
  }
}

}  // namespace c8r
