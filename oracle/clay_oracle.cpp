// clay_oracle.cpp - CPU restatement of clay-engine's fluid hot path (test infrastructure).
//
// Compiled with -O2 -ffp-contract=off (see oracle/Makefile): no fused multiply-add, no
// reassociation, so every f32 expression below is evaluated exactly as written, in the
// order the reference's WGSL writes it. Template parameter T selects binary32 (the port)
// or binary64 (the error reference). Constants that the reference computes in JavaScript
// (binary64) are computed in double and converted once with `K<T>(...)`.
#include "clay_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <class T>
inline T K(double x) { return static_cast<T>(x); }

template <class T>
struct V3 {
  T x, y, z;
};
template <class T>
inline V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T>
inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T>
inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
// WGSL dot/length: ((x*x + y*y) + z*z), left to right.
template <class T>
inline T dot(V3<T> a, V3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T>
inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T>
inline T vmin(T a, T b) { return b < a ? b : a; }
template <class T>
inline T vmax(T a, T b) { return a < b ? b : a; }
template <class T>
inline T clampT(T x, T lo, T hi) { return vmin(vmax(x, lo), hi); }
template <class T>
inline V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// WGSL mix(a, b, t) = a * (1 - t) + b * t.
template <class T>
inline T mixT(T a, T b, T t) { return a * (T(1) - t) + b * t; }

// Saturating float -> i32 with NaN -> 0 (WGSL value conversion; CUDA cvt.rzi.s32.f32).
template <class T>
inline int32_t to_i32(T f) {
  if (!(f == f)) return 0;
  if (f >= T(2147483647.0)) return 2147483647;
  if (f <= T(-2147483648.0)) return (-2147483647 - 1);
  return static_cast<int32_t>(f);
}

uint16_t f32_to_f16(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  uint32_t sign = (x >> 16) & 0x8000u;
  uint32_t exp = (x >> 23) & 0xffu;
  uint32_t mant = x & 0x7fffffu;
  if (exp == 0xffu) return static_cast<uint16_t>(sign | (mant ? 0x7fffu : 0x7c00u));
  int e = static_cast<int>(exp) - 127 + 15;
  if (e >= 31) return static_cast<uint16_t>(sign | 0x7c00u);
  if (e <= 0) {
    if (e < -10) return static_cast<uint16_t>(sign);
    mant |= 0x800000u;
    int shift = 14 - e;
    uint32_t half = mant >> shift;
    uint32_t rem = mant & ((1u << shift) - 1u);
    uint32_t mid = 1u << (shift - 1);
    if (rem > mid || (rem == mid && (half & 1u))) half++;
    return static_cast<uint16_t>(sign | half);
  }
  uint32_t half = (static_cast<uint32_t>(e) << 10) | (mant >> 13);
  uint32_t rem = mant & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (half & 1u))) half++;
  return static_cast<uint16_t>(sign | half);
}

float f16_to_f32(uint16_t h) {
  uint32_t sign = (static_cast<uint32_t>(h) & 0x8000u) << 16;
  uint32_t exp = (h >> 10) & 0x1fu;
  uint32_t mant = h & 0x3ffu;
  uint32_t x;
  if (exp == 0) {
    if (mant == 0) {
      x = sign;
    } else {
      int e = -1;
      do {
        e++;
        mant <<= 1;
      } while ((mant & 0x400u) == 0);
      mant &= 0x3ffu;
      x = sign | (static_cast<uint32_t>(127 - 15 - e) << 23) | (mant << 13);
    }
  } else if (exp == 31) {
    x = sign | 0x7f800000u | (mant << 13);
  } else {
    x = sign | ((exp + 127 - 15) << 23) | (mant << 13);
  }
  float f;
  std::memcpy(&f, &x, 4);
  return f;
}

// ----------------------------------------------------------------------------------------
// math/gpu.ts:103-117
uint32_t hash_mix(uint32_t x) {
  x = x ^ (x >> 16);
  x = x * 0x7feb352du;
  x = x ^ (x >> 15);
  x = x * 0x846ca68bu;
  x = x ^ (x >> 16);
  return x;
}
float hash1f(uint32_t seed) {
  return static_cast<float>(hash_mix(seed) & 0xffffffu) * (1.0f / 16777216.0f);
}

// ----------------------------------------------------------------------------------------
// SdfVolume sampling (volume.ts:220-313) and volumeField (trace/field.ts:102-180).
// The VolumeParams uniform is f32; it is derived from the f64 options as volume.ts:220-230.
template <class T>
struct VolU {
  int res, mips;
  T origin[3], voxel, extent, band, center[3], half;
  T grad_h;
  const uint16_t* dist;
  const uint16_t* mat;
  T offset[3];
  bool has_offset;
  T dyn[3];  // offset applied outermost, set by the extractor from its motion centre
  bool has_dyn;
};

// offsetField (trace/field.ts:396-429): the outermost offset is subtracted first.
template <class T>
V3<T> leaf_point(const VolU<T>& u, V3<T> p) {
  V3<T> q = p;
  if (u.has_dyn) q = q - v3(u.dyn[0], u.dyn[1], u.dyn[2]);
  if (u.has_offset) q = q - v3(u.offset[0], u.offset[1], u.offset[2]);
  return q;
}

template <class T>
VolU<T> make_volu(const orc_volume& v, const double* off) {
  VolU<T> u;
  u.res = v.res;
  u.mips = v.mips;
  double half = v.world_size / 2;
  for (int k = 0; k < 3; k++) {
    u.origin[k] = K<T>(v.origin[k]);
    u.center[k] = K<T>(v.origin[k] + half);
  }
  u.voxel = K<T>(v.world_size / v.res);
  u.extent = K<T>(v.world_size);
  u.band = K<T>(v.band);
  u.half = K<T>(half);
  // gradient: h = voxelSize * gradScale, both f32 (volume.ts:299-302).
  u.grad_h = u.voxel * K<T>(v.gradient_voxels);
  u.dist = v.dist;
  u.mat = v.mat;
  u.has_offset = false;
  u.has_dyn = false;
  for (int k = 0; k < 3; k++) {
    u.dyn[k] = T(0);
    u.offset[k] = off ? K<T>(off[k]) : T(0);
    if (off && off[k] != 0.0) u.has_offset = true;
  }
  return u;
}

// @typegpu/sdf sdBox3d (Quilez's box): q = abs(p) - b;
// length(max(q, 0)) + min(max(q.x, max(q.y, q.z)), 0).
template <class T>
T sd_box(V3<T> p, V3<T> b) {
  V3<T> q = v3(std::fabs(p.x) - b.x, std::fabs(p.y) - b.y, std::fabs(p.z) - b.z);
  V3<T> m = v3(vmax(q.x, T(0)), vmax(q.y, T(0)), vmax(q.z, T(0)));
  return length(m) + vmin(vmax(q.x, vmax(q.y, q.z)), T(0));
}

// textureSampleLevel(.., uv, 0).x with linear filtering and clamp-to-edge, written with
// exact weights: t = uv*R - 0.5, i0 = floor(t), f = t - i0, lerp(a,b,f) = a + (b-a)*f along
// x, then y, then z. The reference's hardware filter uses reduced-precision weights; this
// choice is shared with the CUDA path so the two agree exactly.
template <class T>
T trilinear(const VolU<T>& u, V3<T> p) {
  V3<T> rel = p - v3(u.origin[0], u.origin[1], u.origin[2]);
  V3<T> uv = v3(rel.x / u.extent, rel.y / u.extent, rel.z / u.extent);
  const int R = u.res;
  const T Rf = static_cast<T>(R);
  T t[3] = {uv.x * Rf - T(0.5), uv.y * Rf - T(0.5), uv.z * Rf - T(0.5)};
  int i0[3], i1[3];
  T fr[3];
  for (int k = 0; k < 3; k++) {
    T fl = std::floor(t[k]);
    fr[k] = t[k] - fl;
    int ii = to_i32(fl);
    i0[k] = std::min(std::max(ii, 0), R - 1);
    int jj = ii == 2147483647 ? ii : ii + 1;
    i1[k] = std::min(std::max(jj, 0), R - 1);
  }
  auto at = [&](int x, int y, int z) -> T {
    size_t idx = static_cast<size_t>(x) + static_cast<size_t>(R) * (static_cast<size_t>(y) + static_cast<size_t>(R) * z);
    return static_cast<T>(f16_to_f32(u.dist[idx]));
  };
  auto lerp = [](T a, T b, T f) { return a + (b - a) * f; };
  T c00 = lerp(at(i0[0], i0[1], i0[2]), at(i1[0], i0[1], i0[2]), fr[0]);
  T c10 = lerp(at(i0[0], i1[1], i0[2]), at(i1[0], i1[1], i0[2]), fr[0]);
  T c01 = lerp(at(i0[0], i0[1], i1[2]), at(i1[0], i0[1], i1[2]), fr[0]);
  T c11 = lerp(at(i0[0], i1[1], i1[2]), at(i1[0], i1[1], i1[2]), fr[0]);
  T c0 = lerp(c00, c10, fr[1]);
  T c1 = lerp(c01, c11, fr[1]);
  return lerp(c0, c1, fr[2]);
}

// volumeField.sample(p, 0) (trace/field.ts:135-146): (dBox, 1) outside the box, else
// (raw * bandWorld(0), raw) with bandWorld(m) = band * voxelSize * exp2(m) (volume.ts:269-272).
template <class T>
void vol_sample(const VolU<T>& u, V3<T> p, T out[2]) {
  V3<T> c = v3(u.center[0], u.center[1], u.center[2]);
  T dbox = sd_box(p - c, v3(u.half, u.half, u.half));
  if (dbox > T(0)) {
    out[0] = dbox;
    out[1] = T(1);
    return;
  }
  T raw = trilinear(u, p);
  T bw = u.band * u.voxel * T(1);
  out[0] = raw * bw;
  out[1] = raw;
}

// sampleDist(p, 0) (volume.ts:277-286).
template <class T>
T vol_dist(const VolU<T>& u, V3<T> p) {
  V3<T> c = v3(u.center[0], u.center[1], u.center[2]);
  T dbox = sd_box(p - c, v3(u.half, u.half, u.half));
  if (dbox > T(0)) return dbox;
  return trilinear(u, p) * (u.band * u.voxel * T(1));
}

// gradient (volume.ts:300-313): central differences, normalised as g * (1/len), (0,1,0)
// when len <= 1e-8.
template <class T>
V3<T> vol_normal(const VolU<T>& u, V3<T> p) {
  T h = u.grad_h;
  V3<T> dx = v3(h, T(0), T(0)), dy = v3(T(0), h, T(0)), dz = v3(T(0), T(0), h);
  V3<T> g = v3(vol_dist(u, p + dx) - vol_dist(u, p - dx), vol_dist(u, p + dy) - vol_dist(u, p - dy),
               vol_dist(u, p + dz) - vol_dist(u, p - dz));
  T len = length(g);
  if (len > K<T>(1e-8)) {
    T inv = T(1) / len;
    return g * inv;
  }
  return v3(T(0), T(1), T(0));
}

template <class T>
struct FieldU {
  int n;
  VolU<T> v[8];
};

template <class T>
FieldU<T> make_field(const orc_field* f) {
  FieldU<T> fu;
  fu.n = f ? f->n : 0;
  for (int i = 0; i < fu.n; i++) fu.v[i] = make_volu<T>(f->vol[i], f->offset[i]);
  return fu;
}

// unionField (trace/field.ts:264-313): the whole pair of the nearer child; on a tie the
// later child wins (`select(sb, sa, sa.x < sb.x)`), so a left-to-right fold that replaces
// the best when `!(best.x < cur.x)` reproduces any tree of unions.
template <class T>
int field_pick(const FieldU<T>& f, V3<T> p, T out[2]) {
  int best = -1;
  T bs[2] = {T(0), T(0)};
  for (int i = 0; i < f.n; i++) {
    const VolU<T>& u = f.v[i];
    V3<T> q = leaf_point(u, p);
    T s[2];
    vol_sample(u, q, s);
    if (best < 0 || !(bs[0] < s[0])) {
      best = i;
      bs[0] = s[0];
      bs[1] = s[1];
    }
  }
  out[0] = bs[0];
  out[1] = bs[1];
  return best;
}

template <class T>
V3<T> field_normal(const FieldU<T>& f, V3<T> p, int child) {
  const VolU<T>& u = f.v[child];
  return vol_normal(u, leaf_point(u, p));
}

// field(p, 0).y of the child field_pick chose (trace/field.ts:147-150,288-293,412-415,
// volume.ts:288-296): the material plane, trilinear like the distance, 0 outside the box.
template <class T>
T field_material(const FieldU<T>& f, V3<T> p, int child) {
  if (child < 0) return T(0);
  VolU<T> u = f.v[child];
  V3<T> q = leaf_point(u, p);
  V3<T> c = v3(u.center[0], u.center[1], u.center[2]);
  if (sd_box(q - c, v3(u.half, u.half, u.half)) > T(0)) return T(0);
  u.dist = u.mat;
  return trilinear(u, q);
}

// ----------------------------------------------------------------------------------------
// FluidSim constants (fluid.ts:143-266).
struct Derived {
  double h, poly6, spiky, mass, rest;
  int G;
  double gorig[3], wlo[3], whi[3];
};

double rest_density_f64(double spacing, double h) {
  double poly6 = 315 / (64 * M_PI * std::pow(h, 9));
  double mass = std::pow(spacing, 3);
  double rest = 0;
  int reach = static_cast<int>(std::ceil(h / spacing));
  for (int z = -reach; z <= reach; z++)
    for (int y = -reach; y <= reach; y++)
      for (int x = -reach; x <= reach; x++) {
        double r2 = static_cast<double>(x * x + y * y + z * z) * spacing * spacing;
        if (r2 < h * h) rest += mass * poly6 * std::pow(h * h - r2, 3);
      }
  return rest;
}

Derived derive(const orc_fluid_cfg& c) {
  Derived d;
  d.h = c.h;
  d.poly6 = 315 / (64 * M_PI * std::pow(c.h, 9));
  d.spiky = -45 / (M_PI * std::pow(c.h, 6));
  d.mass = std::pow(c.spacing, 3);
  d.rest = rest_density_f64(c.spacing, c.h);
  d.G = static_cast<int>(std::ceil(c.world_size / c.h)) + 2;
  for (int k = 0; k < 3; k++) {
    d.gorig[k] = c.origin[k] - c.h;
    d.wlo[k] = c.origin[k] + c.radius;
    d.whi[k] = c.origin[k] + c.world_size - c.radius;
  }
  return d;
}

// The f32 (or f64) literals the shaders see.
template <class T>
struct FluidK {
  T h, h2, inv_h, h6, mass, mass_poly6, spiky, rest, rest_floor, radius;
  T gorig[3], wlo[3], whi[3];
  int G;
  uint32_t bucket;
};

template <class T>
FluidK<T> make_k(const orc_fluid_cfg& c, const Derived& d) {
  FluidK<T> k;
  k.h = K<T>(d.h);
  k.h2 = K<T>(d.h * d.h);
  k.inv_h = K<T>(1 / d.h);
  k.h6 = K<T>(std::pow(d.h, 6));
  k.mass = K<T>(d.mass);
  k.mass_poly6 = K<T>(d.mass * d.poly6);
  k.spiky = K<T>(d.spiky);
  k.rest = K<T>(d.rest);
  k.rest_floor = K<T>(d.rest * 0.1);
  k.radius = K<T>(c.radius);
  for (int i = 0; i < 3; i++) {
    k.gorig[i] = K<T>(d.gorig[i]);
    k.wlo[i] = K<T>(d.wlo[i]);
    k.whi[i] = K<T>(d.whi[i]);
  }
  k.G = d.G;
  k.bucket = c.bucket;
  return k;
}

// cellOf (fluid.ts:253-257): vec3i(floor((p - gridOrigin) * (1/h))).
template <class T>
void cell_of(const FluidK<T>& k, V3<T> p, int c[3]) {
  c[0] = to_i32(std::floor((p.x - k.gorig[0]) * k.inv_h));
  c[1] = to_i32(std::floor((p.y - k.gorig[1]) * k.inv_h));
  c[2] = to_i32(std::floor((p.z - k.gorig[2]) * k.inv_h));
}
inline bool in_grid(const int c[3], int G) {
  return c[0] >= 0 && c[1] >= 0 && c[2] >= 0 && c[0] < G && c[1] < G && c[2] < G;
}
// cellIndex (fluid.ts:258-262) for an in-grid cell.
inline uint32_t cell_index(const int c[3], int G) {
  uint32_t g = static_cast<uint32_t>(G);
  return static_cast<uint32_t>(c[0]) + g * (static_cast<uint32_t>(c[1]) + g * static_cast<uint32_t>(c[2]));
}

// The bucket grid after clearGrid + insert (fluid.ts:293-331), with the first `bucket`
// particles of each cell kept in ascending index order.
struct Buckets {
  std::vector<uint32_t> start;  // G^3 + 1
  std::vector<uint32_t> items;
  uint32_t G, bucket;
  void range(uint32_t cell, uint32_t& b, uint32_t& n) const {
    b = start[cell];
    uint32_t m = start[cell + 1] - b;
    n = m < bucket ? m : bucket;
  }
};

template <class T, class P>
Buckets build_buckets(const FluidK<T>& k, const P* parts, uint32_t count) {
  Buckets B;
  B.G = static_cast<uint32_t>(k.G);
  B.bucket = k.bucket;
  size_t cells = static_cast<size_t>(B.G) * B.G * B.G;
  B.start.assign(cells + 1, 0);
  std::vector<uint32_t> key(count);
  for (uint32_t i = 0; i < count; i++) {
    int c[3];
    cell_of(k, v3<T>(parts[i].pos[0], parts[i].pos[1], parts[i].pos[2]), c);
    if (in_grid(c, k.G)) {
      key[i] = cell_index(c, k.G);
      B.start[key[i] + 1]++;
    } else {
      key[i] = 0xffffffffu;
    }
  }
  for (size_t c = 0; c < cells; c++) B.start[c + 1] += B.start[c];
  B.items.resize(B.start[cells]);
  std::vector<uint32_t> fill(B.start.begin(), B.start.end() - 1);
  for (uint32_t i = 0; i < count; i++)
    if (key[i] != 0xffffffffu) B.items[fill[key[i]]++] = i;
  return B;
}

template <class T>
void set_threads(int threads) {
#ifdef _OPENMP
  omp_set_num_threads(threads > 0 ? threads : 1);
#else
  (void)threads;
#endif
}

// density (fluid.ts:333-368). pow(x, 3) is evaluated as (x*x)*x.
template <class T, class P>
void density_pass(const FluidK<T>& k, const Buckets& B, const P* parts, uint32_t count,
                  T stiffness, T* dens, T* pres, int threads) {
  set_threads<T>(threads);
#pragma omp parallel for schedule(dynamic, 256) if (threads > 1)
  for (int64_t ii = 0; ii < static_cast<int64_t>(count); ii++) {
    uint32_t i = static_cast<uint32_t>(ii);
    V3<T> pi = v3<T>(parts[i].pos[0], parts[i].pos[1], parts[i].pos[2]);
    int base[3];
    cell_of(k, pi, base);
    T rho = T(0);
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int c[3] = {base[0] + dx, base[1] + dy, base[2] + dz};
          if (!in_grid(c, k.G)) continue;
          uint32_t b, n;
          B.range(cell_index(c, k.G), b, n);
          for (uint32_t q = 0; q < n; q++) {
            uint32_t j = B.items[b + q];
            V3<T> pj = v3<T>(parts[j].pos[0], parts[j].pos[1], parts[j].pos[2]);
            V3<T> d = pi - pj;
            T r2 = dot(d, d);
            if (r2 < k.h2) {
              T w = k.h2 - r2;
              rho = rho + k.mass_poly6 * ((w * w) * w);
            }
          }
        }
    dens[i] = vmax(rho, k.rest_floor);
    pres[i] = vmax(stiffness * (rho - k.rest), T(0));
  }
}

template <class T>
struct PrmT {
  V3<T> gravity;
  T dt, max_speed, stiffness, viscosity, damping, contact_depth;
  uint32_t count;
};
template <class T>
PrmT<T> make_prm(const orc_params& p) {
  PrmT<T> q;
  q.gravity = v3<T>(p.gravity[0], p.gravity[1], p.gravity[2]);
  q.dt = p.dt;
  q.max_speed = p.max_speed;
  q.stiffness = p.stiffness;
  q.viscosity = p.viscosity;
  q.damping = p.damping;
  q.contact_depth = p.contact_depth;
  q.count = p.count;
  return q;
}

// forces (fluid.ts:370-439): returns nvel.
template <class T, class P>
V3<T> forces_one(const FluidK<T>& k, const Buckets& B, const P* parts, const T* dens,
                 const T* pres, const PrmT<T>& prm, uint32_t i) {
  V3<T> mpos = v3<T>(parts[i].pos[0], parts[i].pos[1], parts[i].pos[2]);
  V3<T> mvel = v3<T>(parts[i].vel[0], parts[i].vel[1], parts[i].vel[2]);
  T md = dens[i], mp = pres[i];
  int base[3];
  cell_of(k, mpos, base);
  V3<T> fp = v3(T(0), T(0), T(0));
  V3<T> vsum = mvel * k.h6;
  T wsum = k.h6;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        int c[3] = {base[0] + dx, base[1] + dy, base[2] + dz};
        if (!in_grid(c, k.G)) continue;
        uint32_t b, n;
        B.range(cell_index(c, k.G), b, n);
        for (uint32_t q = 0; q < n; q++) {
          uint32_t j = B.items[b + q];
          if (j == i) continue;
          V3<T> opos = v3<T>(parts[j].pos[0], parts[j].pos[1], parts[j].pos[2]);
          V3<T> dv = mpos - opos;
          T r2 = dot(dv, dv);
          if (r2 >= k.h2) continue;
          T inv = T(1) / dens[j];
          T w0 = k.h2 - r2;
          T w = (w0 * w0) * w0;
          V3<T> ovel = v3<T>(parts[j].vel[0], parts[j].vel[1], parts[j].vel[2]);
          vsum = vsum + ovel * w;
          wsum = wsum + w;
          T r = std::sqrt(r2);
          if (r > K<T>(1e-6)) {
            T hr = k.h - r;
            T s = k.mass * (mp + pres[j]) * T(0.5) * inv * k.spiky * (hr * hr);
            fp = fp - (dv * (T(1) / r)) * s;
          }
        }
      }
  V3<T> acc = fp * (T(1) / md) + prm.gravity;
  T t = clampT(prm.viscosity, T(0), T(1));
  V3<T> mean = vsum * (T(1) / wsum);
  V3<T> v = v3(mixT(mvel.x, mean.x, t), mixT(mvel.y, mean.y, t), mixT(mvel.z, mean.z, t));
  v = (v + acc * prm.dt) * prm.damping;
  T speed = length(v);
  if (speed > prm.max_speed) v = v * (prm.max_speed / speed);
  return v;
}

// integrate (fluid.ts:449-491). Returns whether a contact was appended.
template <class T>
bool integrate_one(const FluidK<T>& k, const FieldU<T>& world, const PrmT<T>& prm, V3<T> pos,
                   V3<T> nvel, V3<T>& out_pos, V3<T>& out_vel, T contact[4]) {
  V3<T> v = nvel;
  V3<T> p = pos + v * prm.dt;
  bool hit = false;
  if (world.n > 0) {
    T s[2];
    int child = field_pick(world, p, s);
    T dw = s[0];
    if (dw < k.radius) {
      V3<T> nrm = field_normal(world, p, child);
      p = p + nrm * (k.radius - dw);
      v = v - nrm * vmin(dot(v, nrm), T(0));
      if (dw < prm.contact_depth) {
        hit = true;
        contact[0] = p.x;
        contact[1] = p.y;
        contact[2] = p.z;
        contact[3] = length(v);
      }
    }
  }
  V3<T> cl = v3(clampT(p.x, k.wlo[0], k.whi[0]), clampT(p.y, k.wlo[1], k.whi[1]),
                clampT(p.z, k.wlo[2], k.whi[2]));
  out_vel = v3(cl.x == p.x ? v.x : T(0), cl.y == p.y ? v.y : T(0), cl.z == p.z ? v.z : T(0));
  out_pos = cl;
  return hit;
}

template <class T, class P>
void substep(const orc_fluid_cfg* cfg, const orc_params* prm_in, const orc_field* world_in,
             P* parts, uint32_t* contact_count, float* contact_points, uint32_t* contact_ids,
             uint32_t max_ids, int threads) {
  Derived d = derive(*cfg);
  FluidK<T> k = make_k<T>(*cfg, d);
  FieldU<T> world = make_field<T>(world_in);
  PrmT<T> prm = make_prm<T>(*prm_in);
  uint32_t count = prm.count;
  if (count > cfg->capacity) count = cfg->capacity;
  Buckets B = build_buckets(k, parts, count);
  std::vector<T> dens(count), pres(count);
  density_pass(k, B, parts, count, prm.stiffness, dens.data(), pres.data(), threads);
  std::vector<V3<T>> nv(count);
  set_threads<T>(threads);
#pragma omp parallel for schedule(dynamic, 256) if (threads > 1)
  for (int64_t ii = 0; ii < static_cast<int64_t>(count); ii++)
    nv[ii] = forces_one(k, B, parts, dens.data(), pres.data(), prm, static_cast<uint32_t>(ii));
  std::vector<unsigned char> hit(count, 0);
  std::vector<T> cpts(static_cast<size_t>(count) * 4);
#pragma omp parallel for schedule(static) if (threads > 1)
  for (int64_t ii = 0; ii < static_cast<int64_t>(count); ii++) {
    uint32_t i = static_cast<uint32_t>(ii);
    V3<T> op, ov;
    T c4[4];
    bool h = integrate_one(k, world, prm, v3<T>(parts[i].pos[0], parts[i].pos[1], parts[i].pos[2]),
                           nv[i], op, ov, c4);
    parts[i].pos[0] = op.x;
    parts[i].pos[1] = op.y;
    parts[i].pos[2] = op.z;
    parts[i].vel[0] = ov.x;
    parts[i].vel[1] = ov.y;
    parts[i].vel[2] = ov.z;
    parts[i].nvel[0] = nv[i].x;
    parts[i].nvel[1] = nv[i].y;
    parts[i].nvel[2] = nv[i].z;
    parts[i].density = dens[i];
    parts[i].pressure = pres[i];
    if (h) {
      hit[i] = 1;
      for (int q = 0; q < 4; q++) cpts[static_cast<size_t>(i) * 4 + q] = c4[q];
    }
  }
  uint32_t n = 0;
  for (uint32_t i = 0; i < count; i++) {
    if (!hit[i]) continue;
    if (contact_points && n < 32)
      for (int q = 0; q < 4; q++) contact_points[n * 4 + q] = static_cast<float>(cpts[static_cast<size_t>(i) * 4 + q]);
    if (contact_ids && n < max_ids) contact_ids[n] = i;
    n++;
  }
  if (contact_count) *contact_count = n;
}

// ----------------------------------------------------------------------------------------
// SplatField (splat.ts:147-276).
struct SplatLevel {
  int r;
  int64_t off;
  double voxel, bw;
};

std::vector<SplatLevel> splat_levels(const orc_splat_cfg& c) {
  std::vector<SplatLevel> L;
  int64_t total = 0;
  for (int m = 0; m < c.mips; m++) {
    SplatLevel l;
    l.r = c.res >> m;
    l.off = total;
    // voxelSizeAt(m) = voxelSize * 2**m with voxelSize = worldSize / resolution (volume.ts:165,336).
    l.voxel = (c.world_size / c.res) * std::pow(2.0, m);
    l.bw = c.band * l.voxel;
    total += static_cast<int64_t>(l.r) * l.r * l.r;
    L.push_back(l);
  }
  return L;
}

inline bool cloud_live(const orc_cloud& c, uint32_t i) {
  if (c.live_mode == 1) return i < c.live_a;
  if (c.live_mode == 2) return i >= c.live_a && i < c.live_a + c.live_b;
  return true;
}

// quatRotate (math/gpu.ts:21-25): t = cross(q.xyz, v) * 2; v + t * q.w + cross(q.xyz, t).
template <class T>
V3<T> quat_rotate(const float* q, V3<T> v) {
  V3<T> qv = v3<T>(q[0], q[1], q[2]);
  V3<T> t = cross(qv, v) * T(2);
  return (v + t * static_cast<T>(q[3])) + cross(qv, t);
}

template <class T>
struct SplatParticle {
  V3<T> p;
  V3<T> n;
};

// contribution (splat.ts:170-184): sphere length(delta) - radius, or with normals
// max(dot(delta, n), length(delta) - radius).
template <class T>
inline T contribution(bool has_n, V3<T> delta, V3<T> n, T radius) {
  if (has_n) return vmax(dot(delta, n), length(delta) - radius);
  return length(delta) - radius;
}

template <class T, class Sink>
void splat_particles(const orc_splat_cfg& c, const orc_cloud& cloud, int threads, Sink sink) {
  std::vector<SplatLevel> L = splat_levels(c);
  T origin[3] = {K<T>(c.origin[0]), K<T>(c.origin[1]), K<T>(c.origin[2])};
  bool has_n = cloud.nrm != nullptr;
  T radius = K<T>(c.radius);
  for (int m = 0; m < c.mips; m++) {
    const SplatLevel& l = L[m];
    T voxel = K<T>(l.voxel);
    T bw = K<T>(l.bw);
    T reach = K<T>(c.radius + l.bw);
    T inv_voxel = K<T>(1 / l.voxel);
    int last = l.r - 1;
    set_threads<T>(threads);
#pragma omp parallel for schedule(dynamic, 64) if (threads > 1)
    for (int64_t ii = 0; ii < static_cast<int64_t>(cloud.capacity); ii++) {
      uint32_t i = static_cast<uint32_t>(ii);
      if (!cloud_live(cloud, i)) continue;
      const float* pp = cloud.pos + static_cast<size_t>(i) * cloud.pos_stride;
      V3<T> p = v3<T>(static_cast<T>(pp[0]) - origin[0], static_cast<T>(pp[1]) - origin[1],
                      static_cast<T>(pp[2]) - origin[2]);
      V3<T> nrm = v3(T(0), T(0), T(0));
      if (has_n) {
        const float* nn = cloud.nrm + static_cast<size_t>(i) * cloud.nrm_stride;
        nrm = v3<T>(nn[0], nn[1], nn[2]);
        if (cloud.quat) nrm = quat_rotate<T>(cloud.quat, nrm);
      }
      int lo[3] = {to_i32(std::floor((p.x - reach) * inv_voxel)), to_i32(std::floor((p.y - reach) * inv_voxel)),
                   to_i32(std::floor((p.z - reach) * inv_voxel))};
      int hi[3] = {to_i32(std::floor((p.x + reach) * inv_voxel)), to_i32(std::floor((p.y + reach) * inv_voxel)),
                   to_i32(std::floor((p.z + reach) * inv_voxel))};
      for (int z = std::max(lo[2], 0); z <= std::min(hi[2], last); z++)
        for (int y = std::max(lo[1], 0); y <= std::min(hi[1], last); y++)
          for (int x = std::max(lo[0], 0); x <= std::min(hi[0], last); x++) {
            V3<T> cc = v3((static_cast<T>(x) + T(0.5)) * voxel, (static_cast<T>(y) + T(0.5)) * voxel,
                          (static_cast<T>(z) + T(0.5)) * voxel);
            T sd = contribution(has_n, cc - p, nrm, radius);
            if (sd < bw) {
              int64_t idx = l.off + x + static_cast<int64_t>(l.r) * (y + static_cast<int64_t>(l.r) * z);
              sink(idx, sd, bw);
            }
          }
    }
  }
}

template <class T>
inline void atomic_min_u32(uint32_t* a, uint32_t v) {
  uint32_t cur = __atomic_load_n(a, __ATOMIC_RELAXED);
  while (v < cur && !__atomic_compare_exchange_n(a, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
}

template <class T>
inline void atomic_min_f64(double* a, double v) {
  uint64_t* ai = reinterpret_cast<uint64_t*>(a);
  uint64_t cur = __atomic_load_n(ai, __ATOMIC_RELAXED);
  for (;;) {
    double c;
    std::memcpy(&c, &cur, 8);
    if (!(v < c)) return;
    uint64_t nv;
    std::memcpy(&nv, &v, 8);
    if (__atomic_compare_exchange_n(ai, &cur, nv, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
  }
}

// ----------------------------------------------------------------------------------------
// Brush fold (brush.ts:239-372, builder.ts:76-142), f32.
struct BrushF {
  V3<float> pos;
  float scale;
  float rot[4];
  V3<float> size;
  float radius, material, blend, bound, mask;
  uint32_t kind, op;
};

// Primitive distances in local space. sphere/box/roundBox/capsule/boxFrame are the
// published Quilez formulas that @typegpu/sdf@0.12.0 implements; the rest restate
// brush.ts:253-348 directly.
float eval_local(uint32_t kind, V3<float> p, V3<float> s, float radius) {
  const double PHI = (1 + std::sqrt(5.0)) / 2;
  switch (kind) {
    case 0:  // sphere
      return length(p) - s.x;
    case 1:  // box
      return sd_box(p, s);
    case 2: {  // roundBox: q = abs(p) - (size - r); length(max(q,0)) + min(max(q),0) - r
      V3<float> q = v3(std::fabs(p.x) - (s.x - radius), std::fabs(p.y) - (s.y - radius),
                       std::fabs(p.z) - (s.z - radius));
      V3<float> m = v3(vmax(q.x, 0.0f), vmax(q.y, 0.0f), vmax(q.z, 0.0f));
      return length(m) + vmin(vmax(q.x, vmax(q.y, q.z)), 0.0f) - radius;
    }
    case 3: {  // capsule from (0,-size.y,0) to (0,size.y,0)
      V3<float> a = v3(0.0f, -s.y, 0.0f), b = v3(0.0f, s.y, 0.0f);
      V3<float> pa = p - a, ba = b - a;
      float h = clampT(dot(pa, ba) / dot(ba, ba), 0.0f, 1.0f);
      return length(pa - ba * h) - radius;
    }
    case 4: {  // torus
      float qx = std::sqrt(p.x * p.x + p.z * p.z) - s.x;
      float qy = p.y;
      return std::sqrt(qx * qx + qy * qy) - radius;
    }
    case 5: {  // cylinder
      float dx = std::sqrt(p.x * p.x + p.z * p.z) - s.x;
      float dy = std::fabs(p.y) - s.y;
      float mx = vmax(dx, 0.0f), my = vmax(dy, 0.0f);
      return vmin(vmax(dx, dy), 0.0f) + std::sqrt(mx * mx + my * my);
    }
    case 6:  // plane
      return p.y - radius;
    case 7: {  // boxFrame (Quilez): p = abs(p) - b; q = abs(p + e) - e; three min terms
      V3<float> pp = v3(std::fabs(p.x) - s.x, std::fabs(p.y) - s.y, std::fabs(p.z) - s.z);
      V3<float> q = v3(std::fabs(pp.x + radius) - radius, std::fabs(pp.y + radius) - radius,
                       std::fabs(pp.z + radius) - radius);
      auto term = [](float a, float b, float c) {
        V3<float> m = v3(vmax(a, 0.0f), vmax(b, 0.0f), vmax(c, 0.0f));
        return length(m) + vmin(vmax(a, vmax(b, c)), 0.0f);
      };
      float t1 = term(pp.x, q.y, q.z), t2 = term(q.x, pp.y, q.z), t3 = term(q.x, q.y, pp.z);
      return vmin(vmin(t1, t2), t3);
    }
    case 9: {  // capped cone (brush.ts:267-282)
      float qx = std::sqrt(p.x * p.x + p.z * p.z), qy = p.y;
      float k1x = s.z, k1y = s.y;
      float k2x = s.z - s.x, k2y = 2 * s.y;
      float cax = qx - vmin(qx, qy < 0 ? s.x : s.z);
      float cay = std::fabs(qy) - s.y;
      float num = (k1x - qx) * k2x + (k1y - qy) * k2y;
      float den = vmax(k2x * k2x + k2y * k2y, 1e-20f);
      float t = clampT(num / den, 0.0f, 1.0f);
      float cbx = qx - k1x + k2x * t, cby = qy - k1y + k2y * t;
      float sgn = (cbx < 0 && cay < 0) ? -1.0f : 1.0f;
      return sgn * std::sqrt(vmin(cax * cax + cay * cay, cbx * cbx + cby * cby));
    }
    case 10: {  // octahedron (brush.ts:283-302)
      V3<float> a = v3(std::fabs(p.x), std::fabs(p.y), std::fabs(p.z));
      float m = a.x + a.y + a.z - s.x;
      V3<float> q;
      if (3 * a.x < m) q = a;
      else if (3 * a.y < m) q = v3(a.y, a.z, a.x);
      else if (3 * a.z < m) q = v3(a.z, a.x, a.y);
      else return m * static_cast<float>(1 / std::sqrt(3.0));
      float k = clampT(0.5f * (q.z - q.y + s.x), 0.0f, s.x);
      return length(v3(q.x, q.y - s.x + k, q.z - k));
    }
    case 11: {  // tetrahedron (brush.ts:312-319)
      float m = vmax(vmax(-p.x - p.y - p.z, -p.x + p.y + p.z), vmax(p.x - p.y + p.z, p.x + p.y - p.z)) *
                static_cast<float>(1 / std::sqrt(3.0));
      return m - s.x / 3;
    }
    case 12: {  // dodecahedron (brush.ts:320-334)
      V3<float> q = v3(std::fabs(p.x), std::fabs(p.y), std::fabs(p.z));
      float phi = static_cast<float>(PHI);
      float m = vmax(vmax(phi * q.y + q.z, q.x + phi * q.z), phi * q.x + q.y) *
                static_cast<float>(1 / std::sqrt(1 + PHI * PHI));
      return m - s.x * static_cast<float>(std::sqrt((5 + 2 * std::sqrt(5.0)) / 15));
    }
    case 13: {  // icosahedron (brush.ts:335-344)
      V3<float> q = v3(std::fabs(p.x), std::fabs(p.y), std::fabs(p.z));
      float phi = static_cast<float>(PHI), iphi = static_cast<float>(PHI - 1);
      float m = vmax(vmax(q.x + q.y + q.z, q.y * phi + q.z * iphi), vmax(q.x * iphi + q.z * phi, q.x * phi + q.y * iphi)) *
                static_cast<float>(1 / std::sqrt(3.0));
      return m - s.x * static_cast<float>(std::sqrt((5 + 2 * std::sqrt(5.0)) / 15));
    }
    default:
      return 1e9f;
  }
}

float eval_brush(const BrushF& b, V3<float> p) {
  float inv_scale = 1.0f / vmax(b.scale, 1e-5f);
  float conj[4] = {-b.rot[0], -b.rot[1], -b.rot[2], b.rot[3]};
  V3<float> local = quat_rotate<float>(conj, p - b.pos) * inv_scale;
  return eval_local(b.kind, local, b.size, b.radius) * b.scale;
}

inline float smoothstep(float e0, float e1, float x) {
  float t = clampT((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

// applyBrush (brush.ts:484-511) with sminPolyWeighted / smaxPolyWeighted (gpu.ts:87-137).
void apply_brush(float acc[2], const BrushF& b, V3<float> p) {
  float dist = eval_brush(b, p);
  float keep = b.mask >= 0 ? 1.0f - smoothstep(0.25f, 0.75f, std::fabs(acc[1] - b.mask)) : 1.0f;
  if (b.op == 0) {
    float kk = vmax(b.blend, 1e-6f);
    float h = clampT(0.5f + 0.5f * (acc[0] - dist) / kk, 0.0f, 1.0f);
    float rx = mixT(acc[0], dist, h) - kk * h * (1.0f - h);
    float ry = h;
    float nx = rx, ny = mixT(acc[1], b.material, ry);
    acc[0] = mixT(acc[0], nx, keep);
    acc[1] = mixT(acc[1], ny, keep);
    return;
  }
  if (b.op == 1) {
    float a = -dist;
    float kk = vmax(b.blend, 1e-6f);
    float h = clampT(0.5f - 0.5f * (acc[0] - a) / kk, 0.0f, 1.0f);
    float rx = mixT(acc[0], a, h) + kk * h * (1.0f - h);
    float ry = h;
    float nx = rx, ny = mixT(acc[1], b.material, ry * 0.85f);
    acc[0] = mixT(acc[0], nx, keep);
    acc[1] = mixT(acc[1], ny, keep);
    return;
  }
  float w = 1.0f - smoothstep(-vmax(b.blend, 1e-4f), 0.0f, dist);
  acc[1] = mixT(acc[1], b.material, w * keep);
}

BrushF to_brushf(const orc_brush& o) {
  BrushF b;
  b.pos = v3(o.pos[0], o.pos[1], o.pos[2]);
  b.scale = o.scale;
  for (int i = 0; i < 4; i++) b.rot[i] = o.rot[i];
  b.size = v3(o.size[0], o.size[1], o.size[2]);
  b.radius = o.radius;
  b.material = o.material;
  b.blend = o.blend;
  b.bound = o.bound;
  b.mask = o.mask;
  b.kind = o.kind;
  b.op = o.op;
  return b;
}

}  // namespace

// ========================================================================================
extern "C" {

float orc_hash1(uint32_t seed) { return hash1f(seed); }
void orc_hash3(uint32_t seed, float out[3]) {
  out[0] = hash1f(seed * 3u + 0u);
  out[1] = hash1f(seed * 3u + 1u);
  out[2] = hash1f(seed * 3u + 2u);
}
uint16_t orc_f32_to_f16(float f) { return f32_to_f16(f); }
float orc_f16_to_f32(uint16_t h) { return f16_to_f32(h); }

int32_t orc_volume_mip_levels(int32_t resolution, int32_t requested, char* err, int32_t errlen) {
  const int TILE = 8;
  int mips = requested;
  if (requested <= 0) {
    int halvings = 0;
    double n = static_cast<double>(resolution) / TILE;
    while (n == std::floor(n) && std::fmod(n, 2.0) == 0.0) {
      halvings++;
      n /= 2;
    }
    int lg = static_cast<int>(std::log2(static_cast<double>(resolution) / TILE));
    mips = std::max(1, std::min(lg, halvings + 1));
  }
  long long need = static_cast<long long>(TILE) << (mips - 1);
  if (resolution % need != 0) {
    if (err && errlen > 0)
      std::snprintf(err, errlen, "SdfVolume: resolution %d must be a multiple of %lld for %d mip levels",
                    resolution, need, mips);
    return -1;
  }
  return mips;
}

int64_t orc_volume_total_voxels(int32_t res, int32_t mips) {
  int64_t t = 0;
  for (int m = 0; m < mips; m++) {
    int64_t r = res >> m;
    t += r * r * r;
  }
  return t;
}

void orc_field_query_f32(const orc_field* f, const float p[3], float sample_xy[2], float nrm[3]) {
  FieldU<float> fu = make_field<float>(f);
  V3<float> q = v3(p[0], p[1], p[2]);
  float s[2];
  int child = field_pick(fu, q, s);
  sample_xy[0] = s[0];
  sample_xy[1] = s[1];
  V3<float> n = child >= 0 ? field_normal(fu, q, child) : v3(0.0f, 1.0f, 0.0f);
  nrm[0] = n.x;
  nrm[1] = n.y;
  nrm[2] = n.z;
}

void orc_field_query_f64(const orc_field* f, const double p[3], double sample_xy[2], double nrm[3]) {
  FieldU<double> fu = make_field<double>(f);
  V3<double> q = v3(p[0], p[1], p[2]);
  double s[2];
  int child = field_pick(fu, q, s);
  sample_xy[0] = s[0];
  sample_xy[1] = s[1];
  V3<double> n = child >= 0 ? field_normal(fu, q, child) : v3(0.0, 1.0, 0.0);
  nrm[0] = n.x;
  nrm[1] = n.y;
  nrm[2] = n.z;
}

double orc_rest_density(double spacing, double h) { return rest_density_f64(spacing, h); }

void orc_fluid_derive(const orc_fluid_cfg* cfg, orc_fluid_derived* out) {
  Derived d = derive(*cfg);
  out->h = d.h;
  out->poly6 = d.poly6;
  out->spiky_grad = d.spiky;
  out->mass = d.mass;
  out->rest_density = d.rest;
  out->grid_res = d.G;
  for (int k = 0; k < 3; k++) {
    out->grid_origin[k] = d.gorig[k];
    out->wall_lo[k] = d.wlo[k];
    out->wall_hi[k] = d.whi[k];
  }
}

void orc_fluid_cells(const orc_fluid_cfg* cfg, const orc_particle* parts, uint32_t count, uint32_t* keys) {
  Derived d = derive(*cfg);
  FluidK<float> k = make_k<float>(*cfg, d);
  for (uint32_t i = 0; i < count; i++) {
    int c[3];
    cell_of(k, v3(parts[i].pos[0], parts[i].pos[1], parts[i].pos[2]), c);
    keys[i] = in_grid(c, k.G) ? cell_index(c, k.G) : 0xffffffffu;
  }
}

// emit (fluid.ts:268-291). pow(r.x, 1/3) is evaluated in binary64 and rounded to f32;
// normalize(v) = v / length(v).
void orc_fluid_emit(const orc_fluid_cfg* cfg, const orc_params* prm, orc_particle* parts) {
  const float third = static_cast<float>(1.0 / 3.0);
  for (uint32_t i = 0; i < prm->emit_count; i++) {
    uint32_t slot = (prm->emit_base + i) % cfg->capacity;
    float r[3];
    orc_hash3(prm->emit_seed * 9781u + i, r);
    V3<float> d = v3((r[0] * 2.0f - 1.0f) + static_cast<float>(1e-4), (r[1] * 2.0f - 1.0f) + static_cast<float>(1e-4),
                     (r[2] * 2.0f - 1.0f) + static_cast<float>(1e-4));
    float len = length(d);
    V3<float> dir = v3(d.x / len, d.y / len, d.z / len);
    float pw = static_cast<float>(std::pow(static_cast<double>(r[0]), static_cast<double>(third)));
    float s = prm->emit_radius * pw;
    orc_particle& q = parts[slot];
    q.pos[0] = prm->emit_pos[0] + dir.x * s;
    q.pos[1] = prm->emit_pos[1] + dir.y * s;
    q.pos[2] = prm->emit_pos[2] + dir.z * s;
    q.density = 0;
    for (int k = 0; k < 3; k++) {
      q.vel[k] = prm->emit_vel[k];
      q.nvel[k] = prm->emit_vel[k];
    }
    q.pressure = 0;
  }
}

void orc_fluid_substep_f32(const orc_fluid_cfg* cfg, const orc_params* prm, const orc_field* world,
                           orc_particle* parts, uint32_t* contact_count, float* contact_points,
                           uint32_t* contact_ids, uint32_t max_ids, int32_t threads) {
  substep<float, orc_particle>(cfg, prm, world, parts, contact_count, contact_points, contact_ids, max_ids, threads);
}

void orc_fluid_substep_f64(const orc_fluid_cfg* cfg, const orc_params* prm, const orc_field* world,
                           orc_particle_d* parts, int32_t threads) {
  substep<double, orc_particle_d>(cfg, prm, world, parts, nullptr, nullptr, nullptr, 0, threads);
}

void orc_fluid_density_f64(const orc_fluid_cfg* cfg, const orc_params* prm, const orc_particle* parts,
                           double* out, int32_t threads) {
  Derived d = derive(*cfg);
  FluidK<double> k = make_k<double>(*cfg, d);
  uint32_t count = std::min(prm->count, cfg->capacity);
  Buckets B = build_buckets(k, parts, count);
  std::vector<double> dens(count), pres(count);
  density_pass(k, B, parts, count, static_cast<double>(prm->stiffness), dens.data(), pres.data(), threads);
  for (uint32_t i = 0; i < count; i++) {
    out[2 * i] = dens[i];
    out[2 * i + 1] = pres[i];
  }
}

// clear (splat.ts:200-210) then splat[m] (:223-256): atomicMin of
// u32((clamp(sd / bandWorld, -1, 1) + 1) * 32767.5).
void orc_splat_keys(const orc_splat_cfg* cfg, const orc_cloud* cloud, uint32_t* keys, int32_t threads) {
  int64_t total = orc_volume_total_voxels(cfg->res, cfg->mips);
  for (int64_t i = 0; i < total; i++) keys[i] = 65535u;
  splat_particles<float>(*cfg, *cloud, threads, [&](int64_t idx, float sd, float bw) {
    atomic_min_u32<float>(&keys[idx], orc_splat_encode(sd, bw));
  });
}

uint32_t orc_splat_encode(float sd, float bw) {
  float v = clampT(sd / bw, -1.0f, 1.0f);
  return static_cast<uint32_t>((v + 1.0f) * 32767.5f);
}

float orc_splat_decode(uint32_t key) { return static_cast<float>(key) * static_cast<float>(1 / 32767.5) - 1.0f; }

void orc_splat_resolve(const orc_splat_cfg* cfg, const uint32_t* keys, uint16_t* dist_f16, uint16_t* mat_f16) {
  int64_t total = orc_volume_total_voxels(cfg->res, cfg->mips);
  const float inv = static_cast<float>(1 / 32767.5);
  uint16_t mat = f32_to_f16(static_cast<float>(cfg->material));
  for (int64_t i = 0; i < total; i++) {
    float v = static_cast<float>(keys[i]) * inv - 1.0f;
    dist_f16[i] = f32_to_f16(v);
    if (mat_f16) mat_f16[i] = mat;
  }
}

void orc_splat_values_f64(const orc_splat_cfg* cfg, const orc_cloud* cloud, double* vals, int32_t threads) {
  int64_t total = orc_volume_total_voxels(cfg->res, cfg->mips);
  std::vector<double> best(total, std::numeric_limits<double>::infinity());
  std::vector<double> bwv(total, 1.0);
  splat_particles<double>(*cfg, *cloud, threads, [&](int64_t idx, double sd, double bw) {
    atomic_min_f64<double>(&best[idx], sd);
    bwv[idx] = bw;
  });
  for (int64_t i = 0; i < total; i++) {
    if (std::isinf(best[i])) vals[i] = 1.0;
    else vals[i] = clampT(best[i] / bwv[i], -1.0, 1.0);
  }
}

void orc_eval_brush(const orc_brush* b, const float* pts, int32_t n, float* out) {
  BrushF bf = to_brushf(*b);
  for (int i = 0; i < n; i++) out[i] = eval_brush(bf, v3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]));
}

void orc_build_brushes(const orc_volume* vol, const orc_brush* brushes, int32_t n, uint16_t* dist_f16,
                       uint16_t* mat_f16, int32_t threads) {
  const int TILE = 8;
  const int MAX_TILE_BRUSHES = 64;
  n = std::min(n, 256);
  std::vector<BrushF> bs(n);
  for (int i = 0; i < n; i++) bs[i] = to_brushf(brushes[i]);
  int64_t off = 0;
  float ox = static_cast<float>(vol->origin[0]), oy = static_cast<float>(vol->origin[1]),
        oz = static_cast<float>(vol->origin[2]);
  for (int m = 0; m < vol->mips; m++) {
    int R = vol->res >> m;
    int tiles = R / TILE;
    double voxel_d = (vol->world_size / vol->res) * std::pow(2.0, m);
    double tile_size_d = voxel_d * TILE;
    double bw_d = vol->band * voxel_d;
    float voxel = static_cast<float>(voxel_d), tile_size = static_cast<float>(tile_size_d);
    float tile_half = static_cast<float>(tile_size_d / 2), bw = static_cast<float>(bw_d);
    float empty = static_cast<float>(bw_d * 4);
    set_threads<float>(threads);
#pragma omp parallel for schedule(dynamic, 1) if (threads > 1)
    for (int64_t t = 0; t < static_cast<int64_t>(tiles) * tiles * tiles; t++) {
      int wx = static_cast<int>(t % tiles), wy = static_cast<int>((t / tiles) % tiles),
          wz = static_cast<int>(t / (static_cast<int64_t>(tiles) * tiles));
      V3<float> tmin = v3(ox + static_cast<float>(wx) * tile_size, oy + static_cast<float>(wy) * tile_size,
                          oz + static_cast<float>(wz) * tile_size);
      V3<float> tc = tmin + v3(tile_half, tile_half, tile_half);
      int ids[64];
      int cnt = 0;
      for (int b = 0; b < n; b++) {
        V3<float> d = bs[b].pos - tc;
        V3<float> near = v3(vmax(std::fabs(d.x) - tile_half, 0.0f), vmax(std::fabs(d.y) - tile_half, 0.0f),
                            vmax(std::fabs(d.z) - tile_half, 0.0f));
        if (length(near) < bs[b].bound + bw && cnt < MAX_TILE_BRUSHES) ids[cnt++] = b;
      }
      for (int lz = 0; lz < TILE; lz++)
        for (int ly = 0; ly < TILE; ly++)
          for (int lx = 0; lx < TILE; lx++) {
            V3<float> p = tmin + v3((static_cast<float>(lx) + 0.5f) * voxel, (static_cast<float>(ly) + 0.5f) * voxel,
                                    (static_cast<float>(lz) + 0.5f) * voxel);
            float acc[2] = {empty, 0.0f};
            for (int q = 0; q < cnt; q++) apply_brush(acc, bs[ids[q]], p);
            int x = wx * TILE + lx, y = wy * TILE + ly, z = wz * TILE + lz;
            int64_t idx = off + x + static_cast<int64_t>(R) * (y + static_cast<int64_t>(R) * z);
            dist_f16[idx] = f32_to_f16(clampT(acc[0] / bw, -1.0f, 1.0f));
            if (mat_f16) mat_f16[idx] = f32_to_f16(acc[1]);
          }
    }
    off += static_cast<int64_t>(R) * R * R;
  }
}

}  // extern "C"


// ----------------------------------------------------------------------------------------
// volumeField.sample(p, mip) / field(p, mip) (trace/field.ts:117-150, volume.ts:262-296) with
// the level capped at the volume's top level, and their union / offset composition
// (:264-293, :396-415). Level m: side res >> m, planes after the finer levels, bandWorld(m) =
// band * voxelSize * 2^m.
namespace {
template <class T>
void leaf_sample_mip(const VolU<T>& u0, V3<T> p, int mip, T out[3]) {
  VolU<T> u = u0;
  V3<T> q = leaf_point(u, p);
  V3<T> c = v3(u.center[0], u.center[1], u.center[2]);
  T dbox = sd_box(q - c, v3(u.half, u.half, u.half));
  if (dbox > T(0)) {
    out[0] = dbox;
    out[1] = T(1);
    out[2] = T(0);
    return;
  }
  const int m = std::min(std::max(mip, 0), u.mips - 1);
  size_t off = 0;
  for (int l = 0; l < m; l++) {
    const size_t r = static_cast<size_t>(u.res >> l);
    off += r * r * r;
  }
  const uint16_t* dist = u.dist;
  const uint16_t* mat = u.mat;
  u.res = u0.res >> m;
  u.dist = dist + off;
  const T raw = trilinear(u, q);
  u.dist = mat + off;
  const T material = trilinear(u, q);
  const T bw = (u.band * u.voxel) * std::ldexp(T(1), m);
  out[0] = raw * bw;
  out[1] = raw;
  out[2] = material;
}
}  // namespace

void orc_field_query_mip_f32(const orc_field* f, const float p[3], int mip, float sample_xy[2], float field_xy[2]) {
  FieldU<float> fu = make_field<float>(f);
  float best[3] = {0.0f, 0.0f, 0.0f};
  for (int i = 0; i < fu.n; i++) {
    float o[3];
    leaf_sample_mip(fu.v[i], v3(p[0], p[1], p[2]), mip, o);
    if (i == 0 || !(best[0] < o[0])) {
      best[0] = o[0];
      best[1] = o[1];
      best[2] = o[2];
    }
  }
  sample_xy[0] = best[0];
  sample_xy[1] = best[1];
  field_xy[0] = best[0];
  field_xy[1] = best[2];
}

void orc_field_query_mip_batch(const orc_field* f, const float* pts, int64_t n, int mip, float* sample_xy,
                               float* field_xy, int threads) {
#ifdef _OPENMP
  omp_set_num_threads(threads > 0 ? threads : 1);
#endif
#pragma omp parallel for schedule(static) if (threads > 1)
  for (int64_t i = 0; i < n; i++) orc_field_query_mip_f32(f, pts + 3 * i, mip, sample_xy + 2 * i, field_xy + 2 * i);
}

// ----------------------------------------------------------------------------------------
// SurfaceExtractor.extract (sim/extract.ts:194-436) in f32, with the slot order of the CUDA
// path: dual vertices in lattice order, quads by lattice point then +x, +y, +z edge (the
// reference's atomics leave the order unspecified). Reductions follow the 256-thread
// strided sums and tree of the reference's single-workgroup passes.
namespace {
constexpr int kThreads = 256;

float ext_dist(const FieldU<float>& f, float x, float y, float z) {
  float s[2] = {0.0f, 0.0f};
  if (f.n > 0) field_pick(f, v3(x, y, z), s);
  return s[0];
}

void ext_cross(float ax, float ay, float az, float da, float bx, float by, float bz, float db, float acc[4]) {
  float cx = 0.0f, cy = 0.0f, cz = 0.0f, cw = 0.0f;
  if (!(da * db >= 0.0f)) {
    float t = da / (da - db);
    t = std::min(std::max(t, 0.0f), 1.0f);
    const float u = 1.0f - t;
    cx = ax * u + bx * t;
    cy = ay * u + by * t;
    cz = az * u + bz * t;
    cw = 1.0f;
  }
  acc[0] = acc[0] + cx;
  acc[1] = acc[1] + cy;
  acc[2] = acc[2] + cz;
  acc[3] = acc[3] + cw;
}
}  // namespace

void orc_extract(const orc_extract_cfg* cfg, const orc_field* field, float* motion, unsigned char* particles,
                 unsigned char* bodies, uint32_t* indices, uint32_t* draw_args, uint32_t* counters, uint32_t* id_grid) {
  FieldU<float> f = make_field<float>(field);
  const int R = cfg->res;
  const int64_t cells = static_cast<int64_t>(R) * R * R;
  counters[0] = counters[1] = 0;
  // reset
  if (cfg->has_motion && motion) {
    const unsigned char* bd = bodies + static_cast<size_t>(cfg->body) * 64;
    uint32_t first, count;
    std::memcpy(&first, bd + 12, 4);
    std::memcpy(&count, bd + 44, 4);
    const bool keep = cfg->preserve != 0;
    std::vector<float> sum(static_cast<size_t>(kThreads) * 6, 0.0f);
    if (keep)
      for (int li = 0; li < kThreads; li++)
        for (uint32_t t = li; t < count; t += kThreads) {
          const float* p = reinterpret_cast<const float*>(particles + static_cast<size_t>(first + t) * 96);
          for (int k = 0; k < 3; k++) {
            sum[li * 6 + k] = sum[li * 6 + k] + p[k];
            sum[li * 6 + 3 + k] = sum[li * 6 + 3 + k] + p[8 + k];
          }
        }
    for (int h = kThreads / 2; h > 0; h >>= 1)
      for (int li = 0; li < h; li++)
        for (int k = 0; k < 6; k++) sum[li * 6 + k] = sum[li * 6 + k] + sum[(li + h) * 6 + k];
    if (keep && count > 0) {
      const float inv = 1.0f / static_cast<float>(count);
      for (int k = 0; k < 3; k++) {
        motion[k] = sum[k] * inv;
        motion[4 + k] = sum[3 + k] * inv;
      }
    }
  }
  if (cfg->has_motion && motion && cfg->offset_by_motion)
    for (int i = 0; i < f.n; i++) {
      f.v[i].has_dyn = true;
      for (int k = 0; k < 3; k++) f.v[i].dyn[k] = motion[k];
    }
  float ox = cfg->origin[0], oy = cfg->origin[1], oz = cfg->origin[2];
  if (cfg->has_motion && motion) {
    ox = ox + motion[0];
    oy = oy + motion[1];
    oz = oz + motion[2];
  }
  float vx = cfg->vel[0], vy = cfg->vel[1], vz = cfg->vel[2];
  if (cfg->has_motion && motion) {
    vx = motion[4];
    vy = motion[5];
    vz = motion[6];
  }
  const float c = cfg->cell;
  // cells
  uint32_t slot = 0;
  for (int64_t idx = 0; idx < cells; idx++) {
    const int gx = static_cast<int>(idx % R), gy = static_cast<int>((idx / R) % R), gz = static_cast<int>(idx / (static_cast<int64_t>(R) * R));
    const float x0 = ox + static_cast<float>(gx) * c, y0 = oy + static_cast<float>(gy) * c, z0 = oz + static_cast<float>(gz) * c;
    const float x1 = x0 + c, y1 = y0 + c, z1 = z0 + c;
    const float d0 = ext_dist(f, x0, y0, z0), dx = ext_dist(f, x1, y0, z0), dy = ext_dist(f, x0, y1, z0),
                dz = ext_dist(f, x0, y0, z1), dxy = ext_dist(f, x1, y1, z0), dxz = ext_dist(f, x1, y0, z1),
                dyz = ext_dist(f, x0, y1, z1), dxyz = ext_dist(f, x1, y1, z1);
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    ext_cross(x0, y0, z0, d0, x1, y0, z0, dx, acc);
    ext_cross(x0, y1, z0, dy, x1, y1, z0, dxy, acc);
    ext_cross(x0, y0, z1, dz, x1, y0, z1, dxz, acc);
    ext_cross(x0, y1, z1, dyz, x1, y1, z1, dxyz, acc);
    ext_cross(x0, y0, z0, d0, x0, y1, z0, dy, acc);
    ext_cross(x1, y0, z0, dx, x1, y1, z0, dxy, acc);
    ext_cross(x0, y0, z1, dz, x0, y1, z1, dyz, acc);
    ext_cross(x1, y0, z1, dxz, x1, y1, z1, dxyz, acc);
    ext_cross(x0, y0, z0, d0, x0, y0, z1, dz, acc);
    ext_cross(x1, y0, z0, dx, x1, y0, z1, dxz, acc);
    ext_cross(x0, y1, z0, dy, x0, y1, z1, dyz, acc);
    ext_cross(x1, y1, z0, dxy, x1, y1, z1, dxyz, acc);
    if (acc[3] < 0.5f) {
      id_grid[idx] = 0;
      continue;
    }
    counters[0]++;
    const float inv = 1.0f / acc[3];
    const V3<float> v = v3(acc[0] * inv, acc[1] * inv, acc[2] * inv);
    float s[2] = {0.0f, 0.0f};
    V3<float> n = v3(0.0f, 1.0f, 0.0f);
    if (f.n > 0) {
      const int child = field_pick(f, v, s);
      n = field_normal(f, v, child);
    }
    const V3<float> p = v3(v.x - n.x * s[0], v.y - n.y * s[0], v.z - n.z * s[0]);
    float mat = 0.0f;
    if (f.n > 0) {
      float s2[2];
      const int ch = field_pick(f, p, s2);
      mat = field_material(f, p, ch);
    }
    const uint32_t sl = slot++;
    if (sl >= static_cast<uint32_t>(cfg->capacity)) {
      id_grid[idx] = 0;
      continue;
    }
    const uint32_t id = static_cast<uint32_t>(cfg->base) + sl;
    float* out = reinterpret_cast<float*>(particles + static_cast<size_t>(id) * 96);
    const uint32_t body = static_cast<uint32_t>(cfg->body);
    float rec[24] = {p.x, p.y, p.z, 0.0f, p.x, p.y, p.z, mat, vx, vy, vz, 0.0f, vx, vy, vz, 0.0f,
                     p.x, p.y, p.z, 0.0f, n.x, n.y, n.z, 0.0f};
    std::memcpy(&rec[3], &body, 4);
    std::memcpy(out, rec, sizeof(rec));
    id_grid[idx] = id + 1;
  }
  // quads
  const uint32_t hi = static_cast<uint32_t>(R) - 1u;
  auto cid = [&](uint32_t x, uint32_t y, uint32_t z) {
    return id_grid[x + static_cast<uint32_t>(R) * (y + static_cast<uint32_t>(R) * z)];
  };
  uint32_t qslot = 0;
  for (int64_t idx = 0; idx < cells; idx++) {
    const uint32_t i = static_cast<uint32_t>(idx % R), j = static_cast<uint32_t>((idx / R) % R),
                   k = static_cast<uint32_t>(idx / (static_cast<int64_t>(R) * R));
    const float lx = ox + static_cast<float>(i) * c, ly = oy + static_cast<float>(j) * c, lz = oz + static_cast<float>(k) * c;
    const float dL = ext_dist(f, lx, ly, lz);
    const bool flip = !(dL < 0.0f);
    for (int a = 0; a < 3; a++) {
      uint32_t q[4];
      if (a == 0) {
        if (!(j >= 1 && k >= 1 && j <= hi && k <= hi)) continue;
        if (!(ext_dist(f, lx + c, ly + 0.0f, lz + 0.0f) * dL < 0.0f)) continue;
        q[0] = cid(i, j - 1, k - 1), q[1] = cid(i, j, k - 1), q[2] = cid(i, j, k), q[3] = cid(i, j - 1, k);
      } else if (a == 1) {
        if (!(i >= 1 && k >= 1 && i <= hi && k <= hi)) continue;
        if (!(ext_dist(f, lx + 0.0f, ly + c, lz + 0.0f) * dL < 0.0f)) continue;
        q[0] = cid(i - 1, j, k - 1), q[1] = cid(i - 1, j, k), q[2] = cid(i, j, k), q[3] = cid(i, j, k - 1);
      } else {
        if (!(i >= 1 && j >= 1 && i <= hi && j <= hi)) continue;
        if (!(ext_dist(f, lx + 0.0f, ly + 0.0f, lz + c) * dL < 0.0f)) continue;
        q[0] = cid(i - 1, j - 1, k), q[1] = cid(i, j - 1, k), q[2] = cid(i, j, k), q[3] = cid(i - 1, j, k);
      }
      if (q[0] == 0 || q[1] == 0 || q[2] == 0 || q[3] == 0) continue;
      counters[1]++;
      const uint32_t qs = qslot++;
      if (qs >= static_cast<uint32_t>(cfg->quad_cap)) continue;
      uint32_t* o = indices + static_cast<size_t>(qs) * 6;
      const uint32_t i0 = q[0] - 1, i1 = (flip ? q[3] : q[1]) - 1, i2 = q[2] - 1, i3 = (flip ? q[1] : q[3]) - 1;
      o[0] = i0, o[1] = i1, o[2] = i2, o[3] = i0, o[4] = i2, o[5] = i3;
    }
  }
  // finish
  const uint32_t n = std::min(counters[0], static_cast<uint32_t>(cfg->capacity));
  std::vector<float> g(static_cast<size_t>(kThreads) * 3, 0.0f);
  for (int li = 0; li < kThreads; li++)
    for (uint32_t t = li; t < n; t += kThreads) {
      const float* p = reinterpret_cast<const float*>(particles + static_cast<size_t>(cfg->base + t) * 96 + 64);
      for (int k = 0; k < 3; k++) g[li * 3 + k] = g[li * 3 + k] + p[k];
    }
  for (int h = kThreads / 2; h > 0; h >>= 1)
    for (int li = 0; li < h; li++)
      for (int k = 0; k < 3; k++) g[li * 3 + k] = g[li * 3 + k] + g[(li + h) * 3 + k];
  const float inv = 1.0f / std::max(static_cast<float>(n), 1.0f);
  const float com[3] = {g[0] * inv, g[1] * inv, g[2] * inv};
  unsigned char* bd = bodies + static_cast<size_t>(cfg->body) * 64;
  const uint32_t first = static_cast<uint32_t>(cfg->base);
  const float rot[4] = {0.0f, 0.0f, 0.0f, 1.0f};
  std::memcpy(bd + 0, com, 12);
  std::memcpy(bd + 12, &first, 4);
  std::memcpy(bd + 16, rot, 16);
  std::memcpy(bd + 32, com, 12);
  std::memcpy(bd + 44, &n, 4);
  const uint32_t q = std::min(counters[1], static_cast<uint32_t>(cfg->quad_cap));
  draw_args[0] = q * 6;
  draw_args[1] = 1;
  draw_args[2] = 0;
  draw_args[3] = 0;
}


// ----------------------------------------------------------------------------------------
// ClaySolver.step (sim/pbd.ts:144-416) in f32, particle passes in index order (each touches
// only its own record), the match pass as the reference's 256-thread workgroup per body:
// per-thread strided sums, then a tree.
namespace {
// sin and cos by Cody-Waite reduction by pi/2 and Taylor polynomials on [-pi/4, pi/4]: the
// same steps as the CUDA path, so both sides round alike (WGSL leaves sin/cos precision open).
void orc_sincos(float x, float& s, float& c) {
  const float k = std::nearbyint(x * 0.636619746685028076171875f);
  const float r = ((x - k * 1.57080078125f) - k * -4.453584551811218e-06f) - k * -8.705515752716053e-10f;
  const float r2 = r * r;
  const float ps = r + r * (r2 * (-0.16666667163372039794921875f +
                                 r2 * (0.008333333767950534820556640625f +
                                       r2 * (-0.000198412701138295233249664306640625f + r2 * 2.7557318844628753140568733215332031e-06f))));
  const float pc = 1.0f + r2 * (-0.5f + r2 * (0.041666667908430099487304687500f +
                                            r2 * (-0.0013888889225199818611145019531f +
                                                  r2 * (2.4801587642286904156208038330078e-05f + r2 * -2.7557319981497130356729030609131e-07f))));
  const int q = static_cast<int>(k) & 3;
  s = q == 0 ? ps : q == 1 ? pc : q == 2 ? -ps : -pc;
  c = q == 0 ? pc : q == 1 ? -ps : q == 2 ? -pc : ps;
}

struct Qf {
  float x, y, z, w;
};
Qf qmul(Qf a, Qf b) {
  return {((a.w * b.x + a.x * b.w) + a.y * b.z) - a.z * b.y, ((a.w * b.y - a.x * b.z) + a.y * b.w) + a.z * b.x,
          ((a.w * b.z + a.x * b.y) - a.y * b.x) + a.z * b.w, ((a.w * b.w - a.x * b.x) - a.y * b.y) - a.z * b.z};
}
void cross3f(float ax, float ay, float az, float bx, float by, float bz, float& cx, float& cy, float& cz) {
  cx = ay * bz - az * by;
  cy = az * bx - ax * bz;
  cz = ax * by - ay * bx;
}
void qrot(Qf q, float vx, float vy, float vz, float& ox, float& oy, float& oz) {
  float tx, ty, tz, ux, uy, uz;
  cross3f(q.x, q.y, q.z, vx, vy, vz, tx, ty, tz);
  tx = tx * 2.0f;
  ty = ty * 2.0f;
  tz = tz * 2.0f;
  cross3f(q.x, q.y, q.z, tx, ty, tz, ux, uy, uz);
  ox = (vx + tx * q.w) + ux;
  oy = (vy + ty * q.w) + uy;
  oz = (vz + tz * q.w) + uz;
}
float dot3f(float ax, float ay, float az, float bx, float by, float bz) { return (ax * bx + ay * by) + az * bz; }
float len3f(float x, float y, float z) { return std::sqrt(dot3f(x, y, z, x, y, z)); }
float clampf_(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }

// extractRotation (math/gpu.ts:55-77)
Qf extract_rot(const float a[9], Qf q, int iters) {
  for (int it = 0; it < iters; it++) {
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    const float c0[3] = {1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w)};
    const float c1[3] = {2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w)};
    const float c2[3] = {2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y)};
    const float d = (dot3f(c0[0], c0[1], c0[2], a[0], a[1], a[2]) + dot3f(c1[0], c1[1], c1[2], a[3], a[4], a[5])) +
                    dot3f(c2[0], c2[1], c2[2], a[6], a[7], a[8]);
    const float denom = std::fabs(d) + 1e-9f;
    float e0x, e0y, e0z, e1x, e1y, e1z, e2x, e2y, e2z;
    cross3f(c0[0], c0[1], c0[2], a[0], a[1], a[2], e0x, e0y, e0z);
    cross3f(c1[0], c1[1], c1[2], a[3], a[4], a[5], e1x, e1y, e1z);
    cross3f(c2[0], c2[1], c2[2], a[6], a[7], a[8], e2x, e2y, e2z);
    const float inv = 1.0f / denom;
    const float ox = ((e0x + e1x) + e2x) * inv, oy = ((e0y + e1y) + e2y) * inv, oz = ((e0z + e1z) + e2z) * inv;
    const float wl = len3f(ox, oy, oz);
    if (wl < 1e-9f) break;
    const float iw = 1.0f / wl;
    float sh, ch;
    orc_sincos(wl * 0.5f, sh, ch);
    const Qf r = {(ox * iw) * sh, (oy * iw) * sh, (oz * iw) * sh, ch};
    const Qf m = qmul(r, q);
    const float l = std::sqrt(((m.x * m.x + m.y * m.y) + m.z * m.z) + m.w * m.w);
    q = {m.x / l, m.y / l, m.z / l, m.w / l};
  }
  return q;
}
}  // namespace

void orc_sincos_f32(float x, float sc[2]) { orc_sincos(x, sc[0], sc[1]); }

void orc_solver_step(const orc_solve_cfg* cfg, const orc_field* world, unsigned char* particles, unsigned char* bodies,
                     int body_count) {
  if (body_count == 0) return;
  const FieldU<float> f = make_field<float>(world);
  const uint32_t maxb = static_cast<uint32_t>(cfg->max_bodies);
  auto P = [&](uint32_t i) { return reinterpret_cast<float*>(particles + static_cast<size_t>(i) * 96); };
  auto B = [&](uint32_t b) { return reinterpret_cast<float*>(bodies + static_cast<size_t>(b) * 64); };
  auto U = [](const float* p, int k) {
    uint32_t u;
    std::memcpy(&u, p + k, 4);
    return u;
  };
  auto owner = [&](uint32_t i) -> uint32_t {
    const uint32_t b = U(P(i), 3);
    if (b >= maxb) return maxb;
    const float* bd = B(b);
    const uint32_t first = U(bd, 3), count = U(bd, 11);
    if (i < first || i >= first + count) return maxb;
    return b;
  };
  auto sample = [&](const float q[3], float& dw, float n[3]) {
    float s[2];
    const int child = field_pick(f, v3(q[0], q[1], q[2]), s);
    dw = s[0];
    const V3<float> nn = field_normal(f, v3(q[0], q[1], q[2]), child);
    n[0] = nn.x;
    n[1] = nn.y;
    n[2] = nn.z;
  };
  const uint32_t cap = static_cast<uint32_t>(cfg->capacity);
  if (cfg->kicking)
    for (uint32_t i = 0; i < cap; i++) {
      const uint32_t b = owner(i);
      if (b != cfg->push_body || b >= maxb || (U(B(b), 15) & 1u)) continue;
      float* p = P(i);
      for (int k = 0; k < 3; k++) {
        const float dv = cfg->kick[k];
        const float vel = p[8 + k], vp = p[12 + k], prev = p[4 + k];
        p[8 + k] = vel + dv;
        p[12 + k] = vp + dv;
        p[4 + k] = prev - dv * cfg->h;
      }
    }
  for (int sub = 0; sub < cfg->substeps; sub++) {
    // predict
    for (uint32_t i = 0; i < cap; i++) {
      const uint32_t b = owner(i);
      if (b >= maxb) continue;
      const uint32_t flags = U(B(b), 15);
      if (flags & 1u) continue;
      float* p = P(i);
      float acc[3];
      for (int k = 0; k < 3; k++) {
        acc[k] = (flags & 2u) ? 0.0f : cfg->gravity[k];
        if (b == cfg->push_body) acc[k] = acc[k] + cfg->push[k];
      }
      const float third = 0.3333333432674407958984375f;
      const float h23 = (2.0f * cfg->h) / 3.0f;
      float q[3];
      for (int k = 0; k < 3; k++) {
        const float vpred = (p[8 + k] * 4.0f - p[12 + k]) * third + acc[k] * h23;
        q[k] = (p[k] * 4.0f - p[4 + k]) * third + vpred * h23;
      }
      float prev[3] = {p[0], p[1], p[2]};
      float dw, n[3];
      sample(q, dw, n);
      if (dw < cfg->radius) {
        const float push = cfg->radius - dw;
        for (int k = 0; k < 3; k++) q[k] = q[k] + n[k] * push;
        for (int k = 0; k < 3; k++) prev[k] = p[k] + n[k] * push;
        const float dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
        const float dn = dot3f(dx, dy, dz, n[0], n[1], n[2]);
        q[0] = q[0] - (dx - n[0] * dn) * cfg->friction;
        q[1] = q[1] - (dy - n[1] * dn) * cfg->friction;
        q[2] = q[2] - (dz - n[2] * dn) * cfg->friction;
      }
      for (int k = 0; k < 3; k++) {
        p[4 + k] = prev[k];
        p[k] = q[k];
      }
    }
    // match
    constexpr int T = 256;
    for (int b = 0; b < body_count; b++) {
      float* bd = B(static_cast<uint32_t>(b));
      const uint32_t first = U(bd, 3), count = U(bd, 11);
      // the slice clipped to the set: a record reaching past the capacity reads no further
      const uint32_t live = first >= cap ? 0u : std::min(count, cap - first);
      std::vector<float> g(static_cast<size_t>(T) * 9, 0.0f);
      for (int li = 0; li < T; li++)
        for (uint32_t t = li; t < live; t += T) {
          const float* p = P(first + t);
          for (int k = 0; k < 3; k++) {
            g[li * 9 + k] = g[li * 9 + k] + p[k];
            g[li * 9 + 3 + k] = g[li * 9 + 3 + k] + p[16 + k];
          }
        }
      auto reduce = [&]() {
        for (int h = T / 2; h > 0; h >>= 1)
          for (int li = 0; li < h; li++)
            for (int k = 0; k < 9; k++) g[li * 9 + k] = g[li * 9 + k] + g[(li + h) * 9 + k];
      };
      reduce();
      const float inv = 1.0f / std::max(static_cast<float>(count), 1.0f);
      const float com[3] = {g[0] * inv, g[1] * inv, g[2] * inv};
      const float rcom[3] = {g[3] * inv, g[4] * inv, g[5] * inv};
      std::fill(g.begin(), g.end(), 0.0f);
      for (int li = 0; li < T; li++)
        for (uint32_t t = li; t < live; t += T) {
          const float* p = P(first + t);
          const float pr[3] = {p[0] - com[0], p[1] - com[1], p[2] - com[2]};
          const float rr[3] = {p[16] - rcom[0], p[17] - rcom[1], p[18] - rcom[2]};
          for (int c = 0; c < 3; c++)
            for (int k = 0; k < 3; k++) g[li * 9 + 3 * c + k] = g[li * 9 + 3 * c + k] + pr[k] * rr[c];
        }
      reduce();
      if (count > 0) {
        const Qf q0 = {bd[4], bd[5], bd[6], bd[7]};
        const Qf r = extract_rot(&g[0], q0, cfg->rot_iters);
        bd[0] = com[0], bd[1] = com[1], bd[2] = com[2];
        bd[8] = rcom[0], bd[9] = rcom[1], bd[10] = rcom[2];
        bd[4] = r.x, bd[5] = r.y, bd[6] = r.z, bd[7] = r.w;
      }
    }
    // apply
    for (uint32_t i = 0; i < cap; i++) {
      const uint32_t b = owner(i);
      if (b >= maxb) continue;
      const float* bf = B(b);
      if (U(bf, 15) & 1u) continue;
      float* p = P(i);
      const Qf rot = {bf[4], bf[5], bf[6], bf[7]};
      float tx, ty, tz;
      qrot(rot, p[16] - bf[8], p[17] - bf[9], p[18] - bf[10], tx, ty, tz);
      const float target[3] = {bf[0] + tx, bf[1] + ty, bf[2] + tz};
      const float st = clampf_(bf[12], 0.0f, 1.0f), om = 1.0f - st;
      float q[3];
      for (int k = 0; k < 3; k++) q[k] = p[k] * om + target[k] * st;
      float dw, n[3];
      sample(q, dw, n);
      if (dw < cfg->radius) {
        const float push = cfg->radius - dw;
        for (int k = 0; k < 3; k++) q[k] = q[k] + n[k] * push;
        for (int k = 0; k < 3; k++) p[4 + k] = p[4 + k] + n[k] * push;
      }
      const float r0[3] = {p[16], p[17], p[18]};
      for (int k = 0; k < 3; k++) p[k] = q[k];
      if (bf[13] > 0.0f) {
        const Qf cj = {-rot.x, -rot.y, -rot.z, rot.w};
        float rx, ry, rz;
        qrot(cj, q[0] - bf[0], q[1] - bf[1], q[2] - bf[2], rx, ry, rz);
        const float rest[3] = {rx + bf[8], ry + bf[9], rz + bf[10]};
        const float pl = clampf_(bf[13], 0.0f, 1.0f), om2 = 1.0f - pl;
        for (int k = 0; k < 3; k++) p[16 + k] = r0[k] * om2 + rest[k] * pl;
      }
    }
    // finalize
    for (uint32_t i = 0; i < cap; i++) {
      const uint32_t b = owner(i);
      if (b >= maxb || (U(B(b), 15) & 1u)) continue;
      float* p = P(i);
      const float ih = 1.0f / std::max(cfg->h, 1e-6f);
      float v[3];
      for (int k = 0; k < 3; k++) v[k] = ((p[k] - p[4 + k]) * ih) * cfg->damping;
      const float speed = len3f(v[0], v[1], v[2]);
      if (speed > cfg->max_speed) {
        const float sc = cfg->max_speed / speed;
        for (int k = 0; k < 3; k++) v[k] = v[k] * sc;
      }
      for (int k = 0; k < 3; k++) {
        p[12 + k] = p[8 + k];
        p[8 + k] = v[k];
      }
    }
  }
}
