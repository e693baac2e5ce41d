// Grid-to-particle update and the whitewater advance.
//
// k_g2p walks the particles in cell order (B) and writes the new state back to A at the same slot:
// FLIP/PIC blend over valid faces, explicit Euler advection, obstacle collision with friction, the glass
// walls and floor, drains, the free-flight mark of sub-grid drops, their merging with the pool (ripple
// impulse + crown splash at K = We·Oh^-0.4) and whitewater spawning.
// Reference: blender_addon/suiri_lab/solver.py:527-673 and src/js/31-wgsl-sim2.js:9-251. Positions and
// velocities are float64 inside the kernel, stored as float32; the grid-to-particle sums are float32.
//
// Spawning randomness is the reference WGSL's integer hash (src/js/30-wgsl-sim.js:36-37) seeded by the
// particle's carried id and the sub-step number, so it does not depend on particle order.
#include <algorithm>

#include "launch.cuh"
#include "sdf.cuh"

namespace suiri {

__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}
__device__ __forceinline__ double rnd(uint32_t& s) {
  s = hash_u32(s);
  return (double)(s >> 8) / 16777216.0;
}

struct Fp { double lx, lz, hx, hz; };
__device__ __forceinline__ Fp footprint(const TankDev& T) {
  Fp f;
  f.lx = T.ox; f.lz = T.oz;
  f.hx = T.ox + T.nx * T.h; f.hz = T.oz + T.nz * T.h;
  return f;
}
__device__ __forceinline__ bool in_fp(const Fp& f, double x, double z) { return x > f.lx && x < f.hx && z > f.lz && z < f.hz; }

// glass walls below the rim, floor, re-entry from outside (solver.py:290-301, 31-wgsl-sim2.js:66-80)
__device__ inline void tank_clamp(const TankDev& T, const double x0[3], double x[3], double v[3], double r) {
  const Fp f = footprint(T);
  const bool was = in_fp(f, x0[0], x0[2]);
  if (was && x[1] < T.rim) {
    if (x[0] < f.lx + r) { x[0] = f.lx + r; v[0] = fmax(v[0], 0.0); }
    if (x[0] > f.hx - r) { x[0] = f.hx - r; v[0] = fmin(v[0], 0.0); }
    if (x[2] < f.lz + r) { x[2] = f.lz + r; v[2] = fmax(v[2], 0.0); }
    if (x[2] > f.hz - r) { x[2] = f.hz - r; v[2] = fmin(v[2], 0.0); }
  }
  if (was && x[1] < T.oy + r) { x[1] = T.oy + r; v[1] = fmax(v[1], 0.0); }
  if (!was && x[1] < T.rim && in_fp(f, x[0], x[2])) {
    x[0] = x0[0]; x[2] = x0[2];
    v[0] *= -0.2; v[2] *= -0.2;
  }
}

__device__ __forceinline__ int count_at(const TankDev& T, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= T.nx || j >= T.ny || k >= T.nz) return 0;
  const int c = cell_idx(T, i, j, k);
  return T.off[c + 1] - T.off[c];
}
__device__ __forceinline__ bool air_at(const TankDev& T, int i, int j, int k) {
  if (j >= T.ny) return true;
  if (i < 0 || j < 0 || k < 0 || i >= T.nx || k >= T.nz) return false;
  return count_at(T, i, j, k) == 0;
}

// Corner loads of the transfer. GlobalFaces reads the node arrays (the staggered lower corner of the other two
// axes is missing at the first half cell); BrickFaces reads a brick's shared copy of the nodes
// [i0−1, i0+9) × [j0−1, j0+9) × [k0−1, k0+9) of each component, where nodes outside the grid hold (0, NaN).
struct GlobalFaces {
  __device__ __forceinline__ void load(const TankDev& T, int comp, int bx, int by, int bz, float2 c[8]) const {
    const float2* __restrict__ vv = T.vv + (size_t)comp * T.nnodes + node_idx(T, bx, by, bz);
    const bool lx = bx >= 0, ly = by >= 0, lz = bz >= 0;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int dx = e >> 2, dy = (e >> 1) & 1, dz = e & 1;
      const bool ok = (dx || lx) && (dy || ly) && (dz || lz);
      c[e] = ok ? __ldg(vv + dx + dy * T.sx + dz * T.sxy) : make_float2(0.f, __int_as_float(0x7fc00000));
    }
  }
};

constexpr int kGBN = kBrick + 2;              // staged nodes per brick edge (one below, one above the cells)
constexpr int kGBNodes = kGBN * kGBN * kGBN;

struct BrickFaces {
  const float2* s;
  int i0, j0, k0;
  __device__ __forceinline__ void load(const TankDev&, int comp, int bx, int by, int bz, float2 c[8]) const {
    const float2* b = s + comp * kGBNodes + (bx - i0 + 1) + kGBN * ((by - j0 + 1) + kGBN * (bz - k0 + 1));
#pragma unroll
    for (int e = 0; e < 8; ++e) c[e] = b[(e >> 2) + kGBN * ((e >> 1) & 1) + kGBN * kGBN * (e & 1)];
  }
};

// PIC and FLIP velocity of one component from faces that took weight this step (solver.py:236-249), at a
// grid position inside the grid (0 ≤ g < n on every axis; both callers check). Along the component's own
// axis both corner nodes then exist; on the other two axes the staggered lower corner is node −1 at the
// first half cell, the only corners that can be missing. The 8 corner loads (one float2 each: projected
// v, P2G v or NaN where the face took no weight) are issued together, then summed in the reference's
// corner order, in float32 as the reference's GPU path sums them (31-wgsl-sim2.js:9-36); the weights come
// from the float64 position.
template <class F>
__device__ __forceinline__ void transfer_from(const TankDev& T, const F& faces, double gx, double gy, double gz, int comp,
                                              double vp, double& pic, double& flip) {
  const double qx = gx - (comp == 0 ? 0.0 : 0.5), qy = gy - (comp == 1 ? 0.0 : 0.5), qz = gz - (comp == 2 ? 0.0 : 0.5);
  const int bx = (int)floor(qx), by = (int)floor(qy), bz = (int)floor(qz);
  const double fx = qx - bx, fy = qy - by, fz = qz - bz;
  const double wx[2] = {1 - fx, fx}, wy[2] = {1 - fy, fy}, wz[2] = {1 - fz, fz};
  float2 c[8];
  faces.load(T, comp, bx, by, bz, c);
  const float wxf[2] = {(float)wx[0], (float)wx[1]}, wyf[2] = {(float)wy[0], (float)wy[1]}, wzf[2] = {(float)wz[0], (float)wz[1]};
  float sn = 0.f, so = 0.f, sw = 0.f;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    if (isnan(c[e].y)) continue;
    const float w = (wxf[e >> 2] * wyf[(e >> 1) & 1]) * wzf[e & 1];
    sn += w * c[e].x;
    so += w * c[e].y;
    sw += w;
  }
  if (sw >= 1e-6f) {
    const float rw = __frcp_rn(sw);         // one reciprocal for both quotients (float32, held to tolerance)
    pic = (double)(sn * rw);
    flip = vp + (double)((sn - so) * rw);
  } else {
    pic = vp;
    flip = vp;
  }
}

__device__ __forceinline__ void transfer(const TankDev& T, double gx, double gy, double gz, int comp, double vp,
                                         double& pic, double& flip) {
  transfer_from(T, GlobalFaces{}, gx, gy, gz, comp, vp, pic, flip);
}

__device__ inline void ripple_deposit(const TankDev& T, double x, double z, double impulse, double cap) {
  if (T.rx <= 0) return;
  const Fp f = footprint(T);
  const double u = (x - f.lx) / (f.hx - f.lx), w = (z - f.lz) / (f.hz - f.lz);
  const int i = (int)fmin(fmax(rint(u * T.rx), 0.0), (double)T.rx);
  const int j = (int)fmin(fmax(rint(w * T.rz), 0.0), (double)T.rz);
  const double imp = fmin(fmax(impulse, 0.0), cap);
  atomicAdd((unsigned long long*)&T.rsrc[(size_t)j * (T.rx + 1) + i], (unsigned long long)__double2ll_rn(imp * kRippleFix));
}

__device__ inline void ww_write(const TankDev& T, int k, double px, double py, double pz, double life, double vx, double vy, double vz) {
  const int cur = T.ctr->ww_cur & 1;
  float4* wp = cur ? T.wpos + T.ww_cap : T.wpos;
  float4* wv = cur ? T.wvel + T.ww_cap : T.wvel;
  wp[k] = make_float4((float)px, (float)py, (float)pz, (float)life);
  wv[k] = make_float4((float)vx, (float)vy, (float)vz, 0.f);
}

// Diameter of a sub-grid drop when the tank gives drops their own sizes (no reference counterpart: there
// every merging drop has the particle mass). Lognormal with median drop_d_median and log-standard-deviation
// drop_d_sigma, drawn from the drop's carried id so that a drop keeps its size from emission to impact:
// z = sqrt(−2 ln u1)·cos(2π u2) (Box–Muller) from two draws of the id's hash stream, |z| clamped to 4.
__device__ inline double drop_diameter(const TankDev& T, uint32_t id) {
  uint32_t s = hash_u32(id * 0x9E3779B1u + 0x632BE5ABu);
  const double u1 = rnd(s) + 0.5 / 16777216.0;
  const double u2 = rnd(s);
  const double z = fmin(fmax(sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2), -4.0), 4.0);
  return T.drop_d_median * exp(T.drop_d_sigma * z);
}

// crown splash of a drop of mass m at speed U (solver.py:632-657, 31-wgsl-sim2.js:119-148)
__device__ inline void crown(const TankDev& T, double cx, double cy, double cz, double U, double m, uint32_t id, int frame) {
  if (!T.whitewater) return;
  const double D = pow(6 * m / (M_PI * 998.0), 1.0 / 3.0);
  const double We = 998.0 * U * U * D / 0.0728;
  const double Oh = 0.001 / sqrt(998.0 * 0.0728 * D);
  const double K = We * pow(Oh, -0.4);
  const int n = (int)fmin(fmax(rint(4 * (K / 2100 - 1)), 0.0), 24.0);
  const int nj = K > 700 ? (K > 2100 ? 2 : 1) : 0;
  if (n + nj == 0) return;
  uint32_t s = hash_u32(id * 2654435761u + (uint32_t)frame * 97u + 3u);
  const int base = atomicAdd(&T.ctr->ww_count, n + nj);
  const double r0 = 0.6 * D;
  const double ph0 = rnd(s) * 2 * M_PI;
  for (int i = 0; i < n; ++i) {
    const double ph = ph0 + 2 * M_PI * (i + 0.3 * rnd(s)) / n;
    const double el = 0.9 + 0.45 * rnd(s);
    const double sp = U * (0.15 + 0.2 * rnd(s));
    const double life = 0.5 + 0.4 * rnd(s);
    const double dx = cos(ph), dz = sin(ph);
    if (base + i < T.ww_cap)
      ww_write(T, base + i, cx + dx * r0, cy, cz + dz * r0, life, dx * cos(el) * sp, sin(el) * sp, dz * cos(el) * sp);
  }
  for (int j = 0; j < nj; ++j) {
    const double sp = U * (0.22 + 0.04 * j) * (0.9 + 0.2 * rnd(s));
    const double vx = (rnd(s) - 0.5) * 0.05;
    const double vz = (rnd(s) - 0.5) * 0.05;
    if (base + n + j < T.ww_cap) ww_write(T, base + n + j, cx, cy + 0.001 * j, cz, 0.7, vx, sp, vz);
  }
}

// One particle of the sorted array B (slot `local`, state P, V): the transfer at its position with corners from
// `faces`, advection, collision, walls, drains, the free-flight mark and merging of sub-grid drops and
// whitewater spawning; writes the new state to A at the same slot. Returns 1 + the float64 bits of its
// capped speed when it is inside the grid (0 otherwise), for the speed maximum.
// kFast: the common path only. Where the particle needs a rare branch (RK2, an obstacle within reach, the
// free-flight test of a sparse cell, a falling drop, a whitewater spawn) it sets *defer and returns without
// writing; the full body then runs for it in a second pass (k_g2p_deferred), from the same inputs, so every
// particle gets exactly the arithmetic of the full body. Without those branches the fast body needs far
// fewer registers, and more warps fit per SM.
template <class F, bool kFast = false>
__device__ __forceinline__ unsigned long long g2p_particle(const TankDev& T, int local, const float4 P, const float4 V,
                                                           const F& faces, bool* defer = nullptr) {
  unsigned long long vbits = 0ull;
  const int flags = flags_of(P.w);
  const uint32_t id = __float_as_uint(V.w);
  const double dt = T.dt, h = T.h;
  const double x0[3] = {(double)P.x, (double)P.y, (double)P.z};
  const double vold[3] = {(double)V.x, (double)V.y, (double)V.z};
  double g[3];
  grid_pos(T, x0[0], x0[1], x0[2], g[0], g[1], g[2]);
  const bool ing = in_grid(T, g[0], g[1], g[2]);
  double v[3] = {vold[0], vold[1], vold[2]};
  const int c0[3] = {(int)floor(g[0]), (int)floor(g[1]), (int)floor(g[2])};
  int n0 = 0;
  double u0[3];      // interpolated grid velocity at x0 (RK2)
  if (ing) {
    n0 = count_at(T, c0[0], c0[1], c0[2]);
    for (int a = 0; a < 3; ++a) {
      double pic, flip;
      transfer_from(T, faces, g[0], g[1], g[2], a, vold[a], pic, flip);
      v[a] = pic + T.flip * (flip - pic);
      u0[a] = pic;
    }
  } else {
    v[1] -= T.g * dt;
  }
  double x[3] = {x0[0] + v[0] * dt, x0[1] + v[1] * dt, x0[2] + v[2] * dt};
  if (kFast && T.advect && ing) { *defer = true; return 0ull; }
  if (!kFast && T.advect && ing) {
    // midpoint rule through the grid velocity (no reference counterpart): xm = x0 + u0·dt/2, x = x0 +
    // u(xm)·dt; u falls back to u0 where no face took weight, Euler if the midpoint leaves the grid
    const double hd = 0.5 * dt;
    const double xm[3] = {x0[0] + u0[0] * hd, x0[1] + u0[1] * hd, x0[2] + u0[2] * hd};
    double gm[3];
    grid_pos(T, xm[0], xm[1], xm[2], gm[0], gm[1], gm[2]);
    if (in_grid(T, gm[0], gm[1], gm[2])) {
      for (int a = 0; a < 3; ++a) {
        double pic, flip;
        transfer(T, gm[0], gm[1], gm[2], a, u0[a], pic, flip);
        x[a] = x0[a] + pic * dt;
      }
    }
  }
  const double rc = 0.32 * h;
  // a particle of a cell that no obstacle (drain) can reach, moving less than kNearMove·h, skips the obstacle
  // (drain) tests: they would all fail (see cell_near)
  uint8_t reach = kNearObst | kNearDrain;
  if (T.nobj && ing) {
    const double dx = x[0] - x0[0], dy = x[1] - x0[1], dz = x[2] - x0[2];
    const double lim = kNearMove * h;
    if (dx * dx + dy * dy + dz * dz <= lim * lim) reach = T.near[cell_idx(T, c0[0], c0[1], c0[2])];
  }
  const bool may = T.has_obst && (reach & kNearObst) && maybe_within(T, x[0], x[1], x[2], rc);
  if (kFast && may) { *defer = true; return 0ull; }
  if (!kFast && may) {
    int near = -1;
    double other = -kBig;
    const double d = T.sdf_mode == kSdfAnalytic ? scene_sdf_nearest(T.objs, T.nobj, x[0], x[1], x[2], near, other)
                                                : tank_sdf(T, x[0], x[1], x[2]);
    if (d < rc) {
      double nx, ny, nz;
      tank_normal_near(T, x[0], x[1], x[2], d, near, other, nx, ny, nz);
      x[0] += nx * (rc - d); x[1] += ny * (rc - d); x[2] += nz * (rc - d);
      double vs[3];
      tank_solid_vel(T, x[0], x[1], x[2], vs[0], vs[1], vs[2]);
      const double rel[3] = {v[0] - vs[0], v[1] - vs[1], v[2] - vs[2]};
      const double vn = rel[0] * nx + rel[1] * ny + rel[2] * nz;
      if (vn < 0) {
        const double kf = 1 - T.friction;
        v[0] = vs[0] + (rel[0] - nx * vn) * kf;
        v[1] = vs[1] + (rel[1] - ny * vn) * kf;
        v[2] = vs[2] + (rel[2] - nz * vn) * kf;
      }
    }
  }
  tank_clamp(T, x0, x, v, rc);
  const Fp fp = footprint(T);
  bool alive = true;
  if (T.nobj && (reach & kNearDrain) && in_drain(T.objs, T.nobj, x[0], x[1], x[2])) alive = false;
  if (!in_fp(fp, x[0], x[2]) && x[1] < 0.002) alive = false;
  if (fabs(x[0]) > 20 || fabs(x[2]) > 20 || x[1] < -1 || x[1] > 30) alive = false;
  // free-flight mark of sub-grid drops (solver.py:565-583)
  bool air = flags & kFlagAir;
  if (ing) {
    if (n0 >= 4) {
      air = false;
    } else if (n0 <= 2 && c0[1] + 2 < T.ny) {
      if (kFast) { *defer = true; return 0ull; }
      int around = 0, above = 0;
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
#pragma unroll
          for (int dy = -1; dy <= 1; ++dy) around += count_at(T, c0[0] + dx, c0[1] + dy, c0[2] + dz);
          above += count_at(T, c0[0] + dx, c0[1] + 1, c0[2] + dz) + count_at(T, c0[0] + dx, c0[1] + 2, c0[2] + dz);
        }
      if (around <= 4 && above == 0) air = true;
    }
  }
  // merging with the pool (solver.py:584-606)
  const int frame = T.ctr->frame;
  double g1[3] = {-1.0, -1.0, -1.0};
  const bool falling = air && vold[1] < -0.3;
  if (kFast && falling) { *defer = true; return 0ull; }
  if (falling) grid_pos(T, x[0], x[1], x[2], g1[0], g1[1], g1[2]);     // only a falling drop may merge
  if (falling && in_grid(T, g1[0], g1[1], g1[2])) {
    const int c1[3] = {(int)floor(g1[0]), (int)floor(g1[1]), (int)floor(g1[2])};
    const int same = (c1[0] == c0[0] && c1[1] == c0[1] && c1[2] == c0[2]) ? 1 : 0;
    const int cnt1 = count_at(T, c1[0], c1[1], c1[2]);
    if (cnt1 - same >= 3) {
      double vl[3];
      for (int a = 0; a < 3; ++a) {
        double pic, flip;
        transfer(T, g1[0], g1[1], g1[2], a, v[a], pic, flip);
        vl[a] = pic;
      }
      const double dv = vl[1] - vold[1];
      if (dv > 0.3) {
        v[0] = vl[0]; v[1] = vl[1]; v[2] = vl[2];
        air = false;
        atomicAdd(&T.ctr->impacts, 1);
        double m = T.drop_mass;
        if (T.drop_d_median > 0) {
          const double D = drop_diameter(T, id);
          m = 998.0 * (M_PI / 6.0) * D * D * D;
        }
        ripple_deposit(T, x[0], x[2], 2.0 * m * fmin(dv, 8.0), 2e-3);
        const double level = T.oy + (c1[1] + fmin(cnt1 / T.ppc, 1.0)) * h;
        crown(T, x[0], level + 0.25 * h, x[2], -vold[1], m, id, frame);
      }
    }
  }
  if (ing) {
    const double sp = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    // stored +1 so that 0 means "no in-grid particle this sub-step" (the reference keeps vmax then)
    vbits = (unsigned long long)__double_as_longlong(fmin(sp, 60.0)) + 1ull;
    if (T.whitewater && sp > 0.75) {
      // the six face neighbours, loaded together
      bool near = false;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int sg = -1; sg <= 1; sg += 2)
          near |= air_at(T, c0[0] + (a == 0 ? sg : 0), c0[1] + (a == 1 ? sg : 0), c0[2] + (a == 2 ? sg : 0));
      if (near) {
        uint32_t s = hash_u32(id * 9781u + (uint32_t)frame * 6271u + 17u);
        const double e = fmin(fmax((sp - 0.75) / 1.6, 0.0), 1.0);
        if (kFast && rnd(s) < T.ww_rate * e * e * dt) { *defer = true; return 0ull; }
        if (!kFast && rnd(s) < T.ww_rate * e * e * dt) {
          const double j0 = rnd(s) - 0.5, j1 = rnd(s) - 0.5, j2 = rnd(s) - 0.5;
          const double life = 1.0 + 2.5 * rnd(s);
          const double f = 0.8 + 0.35 * rnd(s);
          atomicAdd(&T.ctr->ww_spawned, 1);
          const int k = atomicAdd(&T.ctr->ww_count, 1);
          if (k < T.ww_cap)
            ww_write(T, k, x[0] + j0 * h * 0.6, x[1] + j1 * h * 0.6, x[2] + j2 * h * 0.6, life,
                     v[0] * f + j0 * 0.35, v[1] * f + j1 * 0.35, v[2] * f + j2 * 0.35);
        }
      }
    }
  }
  const float fl = (float)((air ? kFlagAir : 0) | (alive ? 0 : kFlagDead));
  T.pA[local] = make_float4((float)x[0], (float)x[1], (float)x[2], fl);
  T.vA[local] = make_float4((float)v[0], (float)v[1], (float)v[2], __uint_as_float(id));
  return vbits;
}

template <bool kSplit>
__global__ void __launch_bounds__(kThreads, kSplit ? 3 : 2) k_g2p(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ pfx,
                                                  int* __restrict__ defer_list, int* __restrict__ defer_n) {
  const int total = pfx[ntanks];
  const int stride = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  // Warp-uniform grid-stride walk over the sorted particles of all tanks: the speed maximum is reduced over
  // the warp before its one atomic (one global address per tank would otherwise take an atomic from every
  // particle). The particle of the next iteration is loaded at the top of this one (its tank lookup,
  // descriptor and the two float4 streamed from HBM), so that its load latency overlaps this particle's work.
  int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31);
  int nt = -1, nlocal = 0;
  float4 nP = make_float4(0.f, 0.f, 0.f, 0.f), nV = nP;
  auto fetch = [&](int q) {
    nt = -1;
    if (q < total) {
      nt = find_slot(pfx, ntanks, q);
      nlocal = q - pfx[nt];
      nP = __ldcs(tanks[nt].pB + nlocal);
      nV = __ldcs(tanks[nt].vB + nlocal);
    }
  };
  fetch(base + lane);
  for (; base < total; base += stride) {
    const int t = nt, local = nlocal;
    const float4 P = nP, V = nV;
    fetch(base + stride + lane);
    unsigned long long vbits = 0ull;
    const int tt = t;
    if (kSplit) {
      bool defer = false;
      if (t >= 0) vbits = g2p_particle<GlobalFaces, true>(tanks[t], local, P, V, GlobalFaces{}, &defer);
      // the deferred particles of the warp: one atomic, then consecutive entries
      const unsigned m = __ballot_sync(0xffffffffu, defer);
      if (m) {
        int at = 0;
        if (lane == __ffs(m) - 1) at = atomicAdd(defer_n, __popc(m));
        at = __shfl_sync(0xffffffffu, at, __ffs(m) - 1);
        if (defer) defer_list[at + __popc(m & ((1u << lane) - 1))] = base + lane;
      }
    } else if (t >= 0) {
      vbits = g2p_particle(tanks[t], local, P, V, GlobalFaces{});
    }
    // non-negative doubles order like their bit patterns: a warp max, then one atomic per warp and tank
    const int t0 = __shfl_sync(0xffffffffu, tt, 0);
    if (__all_sync(0xffffffffu, tt == t0 || tt < 0)) {
      unsigned long long m = vbits;
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, m, o);
        m = x > m ? x : m;
      }
      if (lane == 0 && m && t0 >= 0) atomicMax((unsigned long long*)&tanks[t0].ctr->vmax_bits64, m);
    } else if (vbits) {
      atomicMax((unsigned long long*)&tanks[tt].ctr->vmax_bits64, vbits);
    }
  }
}

// the deferred particles of k_g2p<true> with the full body (sorted index q over all tanks); the list was
// filled by the kernel before in the stream, so its count is read here
__global__ void __launch_bounds__(kThreads) k_g2p_deferred(const TankDev* __restrict__ tanks, int ntanks,
                                                           const int* __restrict__ pfx, const int* __restrict__ defer_list,
                                                           const int* __restrict__ defer_n) {
  const int n = *defer_n;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int q = defer_list[e];
    const int t = find_slot(pfx, ntanks, q);
    const int local = q - pfx[t];
    const TankDev& T = tanks[t];
    const unsigned long long vb = g2p_particle(T, local, __ldcs(T.pB + local), __ldcs(T.vB + local), GlobalFaces{});
    if (vb) atomicMax((unsigned long long*)&T.ctr->vmax_bits64, vb);
  }
}

// The per-brick form: one block per 8×8×8-cell brick of each tank, plus one block per tank for its particles
// outside the grid. A brick's block first copies the face nodes its particles' transfers reach (the box of
// nodes [i0−1, i0+9)³ of each component, 24 KB) into shared memory, then walks the brick's particles (a
// (j,k) row of cells is contiguous in the sorted array) with their 24 corner loads served from there; the
// transfers at other positions (RK2 midpoint, a drop's landing point) read the node arrays. One speed
// maximum per block. Same particles as the grid-stride walk, bit for bit.
__global__ void __launch_bounds__(kThreads) k_g2p_brick(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx) {
  __shared__ float2 s_vv[3 * kGBNodes];
  __shared__ int s_row0[kBrick * kBrick];
  __shared__ int s_rowp[kBrick * kBrick + 1];
  __shared__ unsigned long long s_vmax;
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int lb = blockIdx.x - bpfx[t];
  const int bnx = (T.nx + kBrick - 1) / kBrick, bny = (T.ny + kBrick - 1) / kBrick, bnz = (T.nz + kBrick - 1) / kBrick;
  const bool tail = lb == bnx * bny * bnz;        // the tank's particles outside the grid
  const int bi = lb % bnx, bj = (lb / bnx) % bny, bk = lb / (bnx * bny);
  const int i0 = bi * kBrick, j0 = bj * kBrick, k0 = bk * kBrick;
  if (threadIdx.x == 0) s_vmax = 0ull;
  if (tail) {
    if (threadIdx.x == 0) {
      s_row0[0] = T.off[T.ncells];
      s_rowp[1] = T.off[T.ncells + 1] - T.off[T.ncells];
    }
  } else if (threadIdx.x < kBrick * kBrick) {
    const int j = j0 + (threadIdx.x % kBrick), k = k0 + (threadIdx.x / kBrick);
    int a = 0, b = 0;
    if (j < T.ny && k < T.nz) {
      const int c = cell_idx(T, i0, j, k);
      a = T.off[c];
      b = T.off[c + min(kBrick, T.nx - i0)];
    }
    s_row0[threadIdx.x] = a;
    s_rowp[threadIdx.x + 1] = b - a;
  }
  __syncthreads();
  const int nrows = tail ? 1 : kBrick * kBrick;
  if (threadIdx.x == 0) {
    s_rowp[0] = 0;
    for (int r = 1; r <= nrows; ++r) s_rowp[r] += s_rowp[r - 1];
  }
  __syncthreads();
  const int total = s_rowp[nrows];
  if (total == 0) return;                        // nothing in this brick
  if (!tail) {
    const float2 none = make_float2(0.f, __int_as_float(0x7fc00000));
    const size_t nn = T.nnodes;
    for (int e = threadIdx.x; e < 3 * kGBNodes; e += blockDim.x) {
      const int a = e / kGBNodes, ln = e - a * kGBNodes;
      const int ix = i0 - 1 + ln % kGBN, iy = j0 - 1 + (ln / kGBN) % kGBN, iz = k0 - 1 + ln / (kGBN * kGBN);
      const bool in = ix >= 0 && iy >= 0 && iz >= 0 && ix <= T.nx && iy <= T.ny && iz <= T.nz;
      s_vv[e] = in ? __ldg(T.vv + a * nn + node_idx(T, ix, iy, iz)) : none;
    }
    __syncthreads();
  }
  const BrickFaces faces{s_vv, i0, j0, k0};
  auto slot = [&](int q) {
    int lo = 0, hi = nrows - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_rowp[mid] <= q) lo = mid; else hi = mid - 1;
    }
    return s_row0[lo] + (q - s_rowp[lo]);
  };
  unsigned long long vmax = 0ull;
  int q = threadIdx.x;
  int pi = q < total ? slot(q) : 0;
  float4 P = q < total ? __ldcs(T.pB + pi) : make_float4(0.f, 0.f, 0.f, 0.f);
  float4 V = q < total ? __ldcs(T.vB + pi) : P;
  for (; q < total; q += blockDim.x) {
    // the next particle's state is loaded before this one is processed
    const int qn = q + blockDim.x;
    const int pn = qn < total ? slot(qn) : 0;
    const float4 Pn = qn < total ? __ldcs(T.pB + pn) : P, Vn = qn < total ? __ldcs(T.vB + pn) : V;
    const unsigned long long vb = tail ? g2p_particle(T, pi, P, V, GlobalFaces{}) : g2p_particle(T, pi, P, V, faces);
    vmax = vb > vmax ? vb : vmax;
    pi = pn; P = Pn; V = Vn;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, vmax, o);
    vmax = x > vmax ? x : vmax;
  }
  if ((threadIdx.x & 31) == 0 && vmax) atomicMax(&s_vmax, vmax);
  __syncthreads();
  if (threadIdx.x == 0 && s_vmax) atomicMax((unsigned long long*)&T.ctr->vmax_bits64, s_vmax);
}

// ---------------------------------------------------------------------------------------- whitewater
// spray falls with drag, foam rides the surface, bubbles rise (solver.py:675-713, 31-wgsl-sim2.js:361-409)
__device__ inline double sample_vel(const TankDev& T, const double g[3], int comp) {
  const double qx = g[0] - (comp == 0 ? 0.0 : 0.5), qy = g[1] - (comp == 1 ? 0.0 : 0.5), qz = g[2] - (comp == 2 ? 0.0 : 0.5);
  const double fbx = floor(qx), fby = floor(qy), fbz = floor(qz);
  const int bx = (int)fbx, by = (int)fby, bz = (int)fbz;
  const double fx = qx - fbx, fy = qy - fby, fz = qz - fbz;
  double s = 0.0;
  for (int dx = 0; dx < 2; ++dx) {
    const double wx = dx ? fx : 1 - fx;
    const int ix = min(max(bx + dx, 0), T.nx);
    for (int dy = 0; dy < 2; ++dy) {
      const double wy = dy ? fy : 1 - fy;
      const int iy = min(max(by + dy, 0), T.ny);
      for (int dz = 0; dz < 2; ++dz) {
        const double wz = dz ? fz : 1 - fz;
        const int iz = min(max(bz + dz, 0), T.nz);
        const float4 vn = __ldg(T.vel + node_idx(T, ix, iy, iz));
        s += wx * wy * wz * (double)(comp == 0 ? vn.x : (comp == 1 ? vn.y : vn.z));
      }
    }
  }
  return s;
}

__global__ void __launch_bounds__(kThreads) k_whitewater(const TankDev* __restrict__ tanks, int ntanks, double frame_dt) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = 0; t < ntanks; ++t) {
    const TankDev& T = tanks[t];
    const int cur = T.ctr->ww_cur & 1;
    const int n = min(T.ctr->ww_count, T.ww_cap);
    const float4* wp = cur ? T.wpos + T.ww_cap : T.wpos;
    const float4* wv = cur ? T.wvel + T.ww_cap : T.wvel;
    float4* op = cur ? T.wpos : T.wpos + T.ww_cap;
    float4* ov = cur ? T.wvel : T.wvel + T.ww_cap;
    const double dt = frame_dt;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
      const float4 P = wp[q], V = wv[q];
      double x[3] = {(double)P.x, (double)P.y, (double)P.z};
      double v[3] = {(double)V.x, (double)V.y, (double)V.z};
      double life = (double)P.w;
      const double kind0 = (double)V.w;
      double g[3];
      grid_pos(T, x[0], x[1], x[2], g[0], g[1], g[2]);
      double kind = 0.0;
      if (in_grid(T, g[0], g[1], g[2])) {
        const int c[3] = {(int)g[0], (int)g[1], (int)g[2]};
        const int nc = count_at(T, c[0], c[1], c[2]);
        const int up = count_at(T, c[0], c[1] + 1, c[2]);
        if (nc > 0) kind = up > 0 ? 2.0 : ((g[1] - c[1] < fmin(nc / T.ppc, 1.0)) ? 1.0 : 0.0);
      }
      if (kind0 < 0.5 && kind > 0.5 && (double)V.y < -0.3) ripple_deposit(T, x[0], x[2], 4.2e-6 * -(double)V.y, 1e-4);
      if (kind == 0.0) {
        v[1] -= T.g * dt;
        const double damp = 1.0 / (1.0 + 0.6 * dt);
        v[0] *= damp; v[1] *= damp; v[2] *= damp;
        life -= dt * 0.7;
      } else {
        const double vf[3] = {sample_vel(T, g, 0), sample_vel(T, g, 1), sample_vel(T, g, 2)};
        if (kind == 1.0) { v[0] = vf[0] * 1; v[1] = vf[1] * 0.2; v[2] = vf[2] * 1; life -= dt * 0.5; }
        else { v[0] = vf[0] + 0; v[1] = vf[1] + 0.16; v[2] = vf[2] + 0; life -= dt * 0.3; }
      }
      const double x0[3] = {x[0], x[1], x[2]};
      x[0] = x0[0] + v[0] * dt; x[1] = x0[1] + v[1] * dt; x[2] = x0[2] + v[2] * dt;
      if (maybe_within(T, x[0], x[1], x[2], 0.0)) {
        const double d = tank_sdf(T, x[0], x[1], x[2]);
        if (d < 0) {
          double nx, ny, nz;
          tank_normal(T, x[0], x[1], x[2], nx, ny, nz);
          x[0] -= nx * d; x[1] -= ny * d; x[2] -= nz * d;
        }
      }
      tank_clamp(T, x0, x, v, 0.001);
      const Fp fp = footprint(T);
      const bool outside = !in_fp(fp, x[0], x[2]) && x[1] < 0.001;
      const bool drained = T.nobj && in_drain(T.objs, T.nobj, x[0], x[1], x[2]);
      if (life > 0 && !outside && x[1] > -0.5 && !drained) {
        const int k = atomicAdd(&T.ctr->ww_next, 1);
        if (k < T.ww_cap) {
          op[k] = make_float4((float)x[0], (float)x[1], (float)x[2], (float)life);
          ov[k] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)kind);
        }
      }
    }
  }
}

__global__ void k_whitewater_end(const TankDev* __restrict__ tanks, int ntanks) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntanks) return;
  Counters* c = tanks[t].ctr;
  c->ww_count = min(c->ww_next, tanks[t].ww_cap);
  c->ww_next = 0;
  c->ww_cur ^= 1;
}

// k_g2p's grid: at most the blocks that fit on the GPU at once (its register count allows fewer per SM
// than the other particle kernels), so that the grid-stride loop runs in one wave
int g2p_blocks(const LaunchCtx& L) {
  static int resident[128] = {};
  return std::min(L.particle_blocks, resident_grid((const void*)k_g2p<false>, resident));
}

// form 0: the grid-stride walk; 1: per brick with the faces in shared memory; 2: the walk's common path with
// the rare branches deferred to a second pass over a list
void launch_g2p(const LaunchCtx& L, int form) {
  if (form == 1) {
    k_g2p_brick<<<L.nblocks[kFamG2P], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamG2P]);
  } else if (form == 2) {
    static int resident[128] = {}, resident_d[128] = {};
    cudaMemsetAsync(L.defer_n, 0, sizeof(int), L.stream);
    const int nb = std::min(2 * L.particle_blocks, resident_grid((const void*)k_g2p<true>, resident));
    k_g2p<true><<<nb, kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.ppfx_sorted, L.defer_list, L.defer_n);
    k_g2p_deferred<<<resident_grid((const void*)k_g2p_deferred, resident_d), kThreads, 0, L.stream>>>(
        L.tanks, L.ntanks, L.ppfx_sorted, L.defer_list, L.defer_n);
  } else {
    k_g2p<false><<<g2p_blocks(L), kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.ppfx_sorted, nullptr, nullptr);
  }
}
void launch_whitewater(const LaunchCtx& L, double frame_dt) {
  k_whitewater<<<L.particle_blocks, kThreads, 0, L.stream>>>(L.tanks, L.ntanks, frame_dt);
  k_whitewater_end<<<(L.ntanks + 127) / 128, 128, 0, L.stream>>>(L.tanks, L.ntanks);
}

}  // namespace suiri
