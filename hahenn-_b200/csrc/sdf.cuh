// Obstacle signed distances on the device, float64.
//
// Shapes follow the reference's WGSL library (src/js/30-wgsl-sim.js:40-114; JS mirror and parameter
// packing src/js/10-scene.js:125-171). Each operation is a plain IEEE-754 double +,-,*,/,sqrt,min,max
// (the library is built with -fmad=false), so lattice values agree bit for bit with a float64 CPU
// evaluation written in the same order.
#pragma once
#include "common.cuh"

namespace suiri {

__device__ __forceinline__ double len3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }
__device__ __forceinline__ double len2(double x, double y) { return sqrt(x * x + y * y); }

__device__ __forceinline__ void to_local(const Obj& o, double px, double py, double pz, double& qx, double& qy, double& qz) {
  const double dx = px - o.pos[0], dy = py - o.pos[1], dz = pz - o.pos[2];
  const double* R = o.rot;
  qx = R[0] * dx + R[3] * dy + R[6] * dz;
  qy = R[1] * dx + R[4] * dy + R[7] * dz;
  qz = R[2] * dx + R[5] * dy + R[8] * dz;
}

__device__ __forceinline__ double sd_round_box(double px, double py, double pz, double bx, double by, double bz, double r) {
  const double qx = fabs(px) - bx + r, qy = fabs(py) - by + r, qz = fabs(pz) - bz + r;
  const double out = len3(fmax(qx, 0.0), fmax(qy, 0.0), fmax(qz, 0.0));
  return out + fmin(fmax(qx, fmax(qy, qz)), 0.0) - r;
}

__device__ __forceinline__ double sd_cyl(double px, double py, double pz, double r, double hh) {
  const double dx = len2(px, pz) - r;
  const double dy = fabs(py) - hh;
  return fmin(fmax(dx, dy), 0.0) + len2(fmax(dx, 0.0), fmax(dy, 0.0));
}

__device__ __forceinline__ double sd_cone(double px, double py, double pz, double r, double hh) {
  const double qx = len2(px, pz), qy = py;
  const double k2x = -r, k2y = 2.0 * hh;
  const double cax = qx - fmin(qx, qy < 0.0 ? r : 0.0);
  const double cay = fabs(qy) - hh;
  double t = ((0.0 - qx) * k2x + (hh - qy) * k2y) / (k2x * k2x + k2y * k2y);
  t = fmin(fmax(t, 0.0), 1.0);
  const double cbx = qx - 0.0 + k2x * t;
  const double cby = qy - hh + k2y * t;
  const double s = (cbx < 0.0 && cay < 0.0) ? -1.0 : 1.0;
  return s * sqrt(fmin(cax * cax + cay * cay, cbx * cbx + cby * cby));
}

__device__ inline double shape_sdf(const Obj& o, double px, double py, double pz) {
  double qx, qy, qz;
  to_local(o, px, py, pz, qx, qy, qz);
  const double* d = o.dims;
  switch (o.type) {
    case 0: return sd_round_box(qx, qy, qz, d[0], d[1], d[2], d[3]);
    case 1: return len3(qx, qy, qz) - d[0];
    case 2: return sd_cyl(qx, qy, qz, d[0], d[1]);
    case 3: return sd_cone(qx, qy, qz, d[0], d[1]);
    case 4: return len2(len2(qx, qz) - d[0], qy) - d[1];
    case 5: return fmax(sd_cyl(qx, qy, qz, d[0], d[1]), -sd_cyl(qx, qy - d[2], qz, d[0] - d[2], d[1]));
    case 6: return fmax(sd_round_box(qx, qy, qz, d[0], d[1], d[2], 0.002),
                        -sd_round_box(qx, qy - d[3], qz, d[0] - d[3], d[1], d[2] - d[3], 0.001));
    case 7: {
      const double a = fabs(len2(qy, qz) - d[1]) - 0.5 * d[2];
      return fmax(fmax(a, qy), fabs(qx) - d[0]);
    }
    default: return kBig;
  }
}

// minimum over obstacles; `cull` skips objects whose bounding sphere is farther than the current best,
// as the WGSL loop does (src/js/30-wgsl-sim.js:83). For shapes whose distance is bounded by their
// bounding sphere that changes nothing; the gutter's is not, so the culled value is the web version's.
__device__ inline double scene_sdf(const Obj* __restrict__ objs, int n, double px, double py, double pz, bool cull) {
  double best = kBig;
  for (int i = 0; i < n; ++i) {
    const Obj& o = objs[i];
    if (o.flag != 1) continue;
    if (cull) {
      const double c = len3(px - o.pos[0], py - o.pos[1], pz - o.pos[2]) - o.bound;
      if (c > best) continue;
    }
    best = fmin(best, shape_sdf(o, px, py, pz));
  }
  return best;
}

// scene_sdf(…, cull = true), also giving the obstacle that holds the minimum (`near`, -1: none) and a lower
// bound on every other obstacle's distance (`other`: its distance where the loop computed it, its
// bounding-sphere distance where the cull skipped it; -kBig with a gutter, whose distance that sphere does not
// bound). The same loop and fmin order, so the same value.
__device__ inline double scene_sdf_nearest(const Obj* __restrict__ objs, int n, double px, double py, double pz, int& near,
                                           double& other) {
  double best = kBig;
  near = -1;
  other = kBig;
  for (int i = 0; i < n; ++i) {
    const Obj& o = objs[i];
    if (o.flag != 1) continue;
    if (o.type == 7) other = -kBig;
    const double c = len3(px - o.pos[0], py - o.pos[1], pz - o.pos[2]) - o.bound;
    if (c > best) {
      other = fmin(other, c);
      continue;
    }
    const double d = shape_sdf(o, px, py, pz);
    if (d < best) {
      if (near >= 0) other = fmin(other, best);
      best = d;
      near = i;
    } else {
      other = fmin(other, d);
    }
  }
  return best;
}

// velocity of the nearest obstacle (src/js/30-wgsl-sim.js:96-106)
__device__ inline void solid_vel_analytic(const Obj* __restrict__ objs, int n, double px, double py, double pz,
                                          double& vx, double& vy, double& vz) {
  double best = kBig;
  vx = vy = vz = 0.0;
  for (int i = 0; i < n; ++i) {
    const Obj& o = objs[i];
    if (o.flag != 1) continue;
    if (len3(px - o.pos[0], py - o.pos[1], pz - o.pos[2]) - o.bound > best) continue;
    const double d = shape_sdf(o, px, py, pz);
    if (d < best) {
      best = d;
      const double rx = px - o.pos[0], ry = py - o.pos[1], rz = pz - o.pos[2];
      vx = o.lin[0] + (o.ang[1] * rz - o.ang[2] * ry);
      vy = o.lin[1] + (o.ang[2] * rx - o.ang[0] * rz);
      vz = o.lin[2] + (o.ang[0] * ry - o.ang[1] * rx);
    }
  }
}

__device__ inline bool in_drain(const Obj* __restrict__ objs, int n, double px, double py, double pz) {
  for (int i = 0; i < n; ++i) {
    const Obj& o = objs[i];
    if (o.flag != 2) continue;
    // a drain's cylinder (radius r, half height 0.012) lies within r + 0.0121 of its centre and its bound is
    // r + 0.02: a point outside the bound sphere is not in it
    const double ex = px - o.pos[0], ey = py - o.pos[1], ez = pz - o.pos[2];
    if (ex * ex + ey * ey + ez * ez > o.bound * o.bound) continue;
    double qx, qy, qz;
    to_local(o, px, py, pz, qx, qy, qz);
    if (len2(qx, qz) < o.dims[0] && fabs(qy) < o.dims[1]) return true;
  }
  return false;
}

// trilinear distance in the half-cell lattice (blender_addon/suiri_lab/solver.py:116-140)
__device__ inline double lattice_sdf(const TankDev& T, double px, double py, double pz) {
  const double hh = T.h / 2;
  const double gx = (px - T.ox) / hh, gy = (py - T.oy) / hh, gz = (pz - T.oz) / hh;
  const int sx = 2 * T.nx + 1, sy = 2 * T.nyl + 1, sz = 2 * T.nz + 1;
  if (!(gx >= 0.0 && gy >= 0.0 && gz >= 0.0 && gx <= (double)(sx - 1) && gy <= (double)(sy - 1) && gz <= (double)(sz - 1)))
    return kBig;
  const int bx = min((int)floor(gx), sx - 2), by = min((int)floor(gy), sy - 2), bz = min((int)floor(gz), sz - 2);
  const double fx = gx - bx, fy = gy - by, fz = gz - bz;
  const double* L = T.lattice;
  double acc = 0.0;
  for (int dx = 0; dx < 2; ++dx) {
    const double wx = dx ? fx : 1 - fx;
    for (int dy = 0; dy < 2; ++dy) {
      const double wy = dy ? fy : 1 - fy;
      for (int dz = 0; dz < 2; ++dz) {
        const double wz = dz ? fz : 1 - fz;
        acc += wx * wy * wz * L[(bx + dx) + sx * ((by + dy) + (size_t)sy * (bz + dz))];
      }
    }
  }
  return acc;
}

__device__ __forceinline__ double tank_sdf(const TankDev& T, double px, double py, double pz) {
  if (!T.has_obst) return kBig;
  if (T.sdf_mode == kSdfLattice) return lattice_sdf(T, px, py, pz);
  return scene_sdf(T.objs, T.nobj, px, py, pz, true);
}

// Half extents, in the obstacle's own frame, of a box holding the shape (the outer part of the cup and the
// trough: their distance is the max of the outer shape's and a carved one's).
__device__ __forceinline__ void local_box(const Obj& o, double& bx, double& by, double& bz) {
  const double* d = o.dims;
  switch (o.type) {
    case 0: case 6: bx = d[0]; by = d[1]; bz = d[2]; return;          // (round) box, trough
    case 2: case 3: case 5: bx = d[0]; by = d[1]; bz = d[0]; return;  // cylinder, cone, cup
    case 4: bx = d[0] + d[1]; by = d[1]; bz = d[0] + d[1]; return;    // torus
    default: bx = by = bz = d[0]; return;                             // sphere
  }
}

// False only where the scene distance is certainly at least `r`: in analytic mode, when the point lies
// beyond r (+1e-6, far above rounding) of every obstacle's bounding sphere, or of the box in the obstacle's
// frame that holds it. Every shape but the gutter (type 7) lies inside both and its distance function is at
// least the distance to the shape (exact, or the max of exact ones), so then every term of the scene
// minimum, culled or not, is ≥ r. Lattice mode, or any gutter, always answers true. (A sphere's box adds
// nothing to its sphere; a rotated box's or a cylinder's takes a quarter of the points its sphere does.)
__device__ __forceinline__ bool maybe_within(const TankDev& T, double px, double py, double pz, double r) {
  if (!T.has_obst) return false;
  if (T.sdf_mode != kSdfAnalytic) return true;
  for (int i = 0; i < T.nobj; ++i) {
    const Obj& o = T.objs[i];
    if (o.flag != 1) continue;
    if (o.type == 7) return true;
    const double ex = px - o.pos[0], ey = py - o.pos[1], ez = pz - o.pos[2];
    const double lim = r + o.bound + 1e-6;
    if (ex * ex + ey * ey + ez * ez >= lim * lim) continue;
    if (o.type == 1) return true;
    double qx, qy, qz, bx, by, bz;
    to_local(o, px, py, pz, qx, qy, qz);
    local_box(o, bx, by, bz);
    const double ox = fmax(fabs(qx) - bx, 0.0), oy = fmax(fabs(qy) - by, 0.0), oz = fmax(fabs(qz) - bz, 0.0);
    const double rb = r + 1e-6;
    if (ox * ox + oy * oy + oz * oz < rb * rb) return true;
  }
  return false;
}

// A point within kNearReach·h of a cell's centre: a particle that starts in the cell (at most √3/2·h from its
// centre) and moves at most kNearMove·h in the sub-step.
constexpr double kNearMove = 0.98;
constexpr double kNearReach = 0.8660254037844387 + kNearMove + 1e-3;

// The cell's entry of T.near (k_geom), two bits. Bit kNearObst is clear only when maybe_within(p, r) is false
// for every p within kNearReach·h of the centre c, i.e. when c is beyond r + 1e-6 + kNearReach·h (+1e-6) of
// every obstacle's bounding sphere or of its box in its own frame. Both distances change by at most |p − c|
// between c and p (the distance to a ball or to a box is 1-Lipschitz, and the rotation keeps lengths), so
// maybe_within's tests fail at every such p. Bit kNearDrain is clear only when c is beyond every drain's
// bound + kNearReach·h (+1e-6), so in_drain(p) is false at every such p.
constexpr uint8_t kNearObst = 1, kNearDrain = 2;
__device__ __forceinline__ uint8_t cell_near(const TankDev& T, double cx, double cy, double cz, double r) {
  const double reach = kNearReach * T.h + 1e-6;
  uint8_t bits = 0;
  if (T.has_obst && T.sdf_mode != kSdfAnalytic) bits |= kNearObst;
  for (int i = 0; i < T.nobj; ++i) {
    const Obj& o = T.objs[i];
    const double ex = cx - o.pos[0], ey = cy - o.pos[1], ez = cz - o.pos[2];
    const double e2 = ex * ex + ey * ey + ez * ez;
    if (o.flag == 2) {
      const double lim = o.bound + reach;
      if (e2 <= lim * lim) bits |= kNearDrain;
      continue;
    }
    if (o.flag != 1 || (bits & kNearObst)) continue;
    if (o.type == 7) { bits |= kNearObst; continue; }
    const double lim = r + o.bound + 1e-6 + reach;
    if (e2 >= lim * lim) continue;
    if (o.type == 1) { bits |= kNearObst; continue; }
    double qx, qy, qz, bx, by, bz;
    to_local(o, cx, cy, cz, qx, qy, qz);
    local_box(o, bx, by, bz);
    const double ox = fmax(fabs(qx) - bx, 0.0), oy = fmax(fabs(qy) - by, 0.0), oz = fmax(fabs(qz) - bz, 0.0);
    const double rb = r + 1e-6 + reach;
    if (ox * ox + oy * oy + oz * oz < rb * rb) bits |= kNearObst;
  }
  return bits;
}

// central differences, e = 6e-4 (solver.py:142-151, 30-wgsl-sim.js:88-95)
constexpr double kNormalStep = 0.0006;
__device__ __forceinline__ void normal_from(double nx, double ny, double nz, double& ox, double& oy, double& oz) {
  const double l = sqrt(nx * nx + ny * ny + nz * nz);
  if (l > 1e-9) { ox = nx / l; oy = ny / l; oz = nz / l; } else { ox = 0.0; oy = 1.0; oz = 0.0; }
}
__device__ inline void tank_normal(const TankDev& T, double px, double py, double pz, double& nx, double& ny, double& nz) {
  const double e = kNormalStep;
  normal_from(tank_sdf(T, px + e, py, pz) - tank_sdf(T, px - e, py, pz),
              tank_sdf(T, px, py + e, pz) - tank_sdf(T, px, py - e, pz),
              tank_sdf(T, px, py, pz + e) - tank_sdf(T, px, py, pz - e), nx, ny, nz);
}

// tank_normal at p, where the scene distance d came from scene_sdf_nearest: when every other obstacle is more
// than d + 2e (+1e-6) away, each of the six samples (within e of p, the distances 1-Lipschitz) has its minimum
// at obstacle `near` and no cull skips it, so the scene distance there is that obstacle's own: six shape
// evaluations instead of six scene loops, the same values
__device__ inline void tank_normal_near(const TankDev& T, double px, double py, double pz, double d, int near, double other,
                                        double& nx, double& ny, double& nz) {
  const double e = kNormalStep;
  if (T.sdf_mode == kSdfAnalytic && near >= 0 && other > d + 2 * e + 1e-6) {
    const Obj& o = T.objs[near];
    normal_from(shape_sdf(o, px + e, py, pz) - shape_sdf(o, px - e, py, pz),
                shape_sdf(o, px, py + e, pz) - shape_sdf(o, px, py - e, pz),
                shape_sdf(o, px, py, pz + e) - shape_sdf(o, px, py, pz - e), nx, ny, nz);
  } else {
    tank_normal(T, px, py, pz, nx, ny, nz);
  }
}

__device__ inline void tank_solid_vel(const TankDev& T, double px, double py, double pz, double& vx, double& vy, double& vz) {
  vx = vy = vz = 0.0;
  if (!T.has_obst || !T.moving) return;
  if (T.sdf_mode == kSdfLattice) {
    if (!T.oid) return;
    const double hh = T.h / 2;
    const int sx = 2 * T.nx + 1, sy = 2 * T.nyl + 1, sz = 2 * T.nz + 1;
    int ix = (int)rint((px - T.ox) / hh), iy = (int)rint((py - T.oy) / hh), iz = (int)rint((pz - T.oz) / hh);
    ix = min(max(ix, 0), sx - 1); iy = min(max(iy, 0), sy - 1); iz = min(max(iz, 0), sz - 1);
    const int id = T.oid[ix + sx * (iy + (size_t)sy * iz)];
    int k = 0;
    for (int i = 0; i < T.nobj; ++i) {
      const Obj& o = T.objs[i];
      if (o.flag != 1) continue;
      if (k == id) {
        const double rx = px - o.pos[0], ry = py - o.pos[1], rz = pz - o.pos[2];
        vx = o.lin[0] + (o.ang[1] * rz - o.ang[2] * ry);
        vy = o.lin[1] + (o.ang[2] * rx - o.ang[0] * rz);
        vz = o.lin[2] + (o.ang[0] * ry - o.ang[1] * rx);
        return;
      }
      ++k;
    }
    return;
  }
  solid_vel_analytic(T.objs, T.nobj, px, py, pz, vx, vy, vz);
}

}  // namespace suiri
