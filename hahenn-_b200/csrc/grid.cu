// Grid kernels of the sub-step: face open fractions, particle-to-grid, node and cell preparation for
// the pressure solve, and the projection.
#include "launch.cuh"
#include "sdf.cuh"

namespace suiri {

__device__ __forceinline__ void node_coord(const TankDev& T, int n, int& i, int& j, int& k) {
  k = divu(n, T.dsxy);
  const int r = n - k * T.sxy;
  j = divu(r, T.dsx);
  i = r - j * T.sx;
}

// ------------------------------------------------------------------------------------------------ GEOM
// Open fraction of each staggered face from the obstacle distances at its 4 corners and (twice) its
// centre (src/js/30-wgsl-sim.js:118-157; blender_addon/suiri_lab/solver.py:176-207). The sample points
// are the half-cell lattice points origin + (h/2)·L; in lattice mode they are read from the lattice,
// in analytic mode the web version's sceneSdf is evaluated there (float64, culled like the WGSL loop).
__device__ __forceinline__ double lattice_at(const TankDev& T, int lx, int ly, int lz) {
  if (T.sdf_mode == kSdfLattice) {
    const int sx = 2 * T.nx + 1, sy = 2 * T.nyl + 1;
    return T.lattice[lx + sx * (ly + (size_t)sy * lz)];
  }
  const double hh = T.h / 2;
  return scene_sdf(T.objs, T.nobj, T.ox + hh * lx, T.oy + hh * ly, T.oz + hh * lz, true);
}

__device__ __forceinline__ double open_frac(double s0, double s1, double s2, double s3, double sc) {
  const double pos = fmax(s0, 0.0) + fmax(s1, 0.0) + fmax(s2, 0.0) + fmax(s3, 0.0) + 2 * fmax(sc, 0.0);
  const double tot = fabs(s0) + fabs(s1) + fabs(s2) + fabs(s3) + 2 * fabs(sc);
  if (tot < 1e-12) return 1.0;
  return fmin(fmax(pos / fmax(tot, 1e-30), 0.0), 1.0);
}

__global__ void __launch_bounds__(kThreads) k_geom(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx) {
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int n = (blockIdx.x - bpfx[t]) * blockDim.x + threadIdx.x;
  if (n >= T.nnodes) return;
  int i, j, k;
  node_coord(T, n, i, j, k);
  const int nx = T.nx, ny = T.ny, nz = T.nz;
  double f[3] = {0.0, 0.0, 0.0};
  double sv[3] = {0.0, 0.0, 0.0};
  const bool obst = T.has_obst;
  const double h = T.h;
  // x face (i, j+1/2, k+1/2), 0 < i < nx
  if (j < ny && k < nz && i > 0 && i < nx) {
    if (obst) {
      const int L = 2 * i;
      f[0] = open_frac(lattice_at(T, L, 2 * j, 2 * k), lattice_at(T, L, 2 * j + 2, 2 * k), lattice_at(T, L, 2 * j + 2, 2 * k + 2),
                       lattice_at(T, L, 2 * j, 2 * k + 2), lattice_at(T, L, 2 * j + 1, 2 * k + 1));
    } else {
      f[0] = 1.0;
    }
    if (obst && T.moving) {
      double vx, vy, vz;
      tank_solid_vel(T, T.ox + h * (i + 0.0), T.oy + h * (j + 0.5), T.oz + h * (k + 0.5), vx, vy, vz);
      sv[0] = vx;
    }
  }
  // y face (i+1/2, j, k+1/2), 0 < j; the top (j = ny) is open air
  if (i < nx && k < nz && j > 0) {
    if (j >= ny) {
      f[1] = 1.0;
    } else {
      if (obst) {
        const int L = 2 * j;
        f[1] = open_frac(lattice_at(T, 2 * i, L, 2 * k), lattice_at(T, 2 * i + 2, L, 2 * k), lattice_at(T, 2 * i + 2, L, 2 * k + 2),
                         lattice_at(T, 2 * i, L, 2 * k + 2), lattice_at(T, 2 * i + 1, L, 2 * k + 1));
      } else {
        f[1] = 1.0;
      }
      if (obst && T.moving) {
        double vx, vy, vz;
        tank_solid_vel(T, T.ox + h * (i + 0.5), T.oy + h * (j + 0.0), T.oz + h * (k + 0.5), vx, vy, vz);
        sv[1] = vy;
      }
    }
  }
  // z face (i+1/2, j+1/2, k), 0 < k < nz
  if (i < nx && j < ny && k > 0 && k < nz) {
    if (obst) {
      const int L = 2 * k;
      f[2] = open_frac(lattice_at(T, 2 * i, 2 * j, L), lattice_at(T, 2 * i + 2, 2 * j, L), lattice_at(T, 2 * i + 2, 2 * j + 2, L),
                       lattice_at(T, 2 * i, 2 * j + 2, L), lattice_at(T, 2 * i + 1, 2 * j + 1, L));
    } else {
      f[2] = 1.0;
    }
    if (obst && T.moving) {
      double vx, vy, vz;
      tank_solid_vel(T, T.ox + h * (i + 0.5), T.oy + h * (j + 0.5), T.oz + h * (k + 0.0), vx, vy, vz);
      sv[2] = vz;
    }
  }
  T.fracd[n] = f[0];
  T.fracd[T.nnodes + n] = f[1];
  T.fracd[2 * T.nnodes + n] = f[2];
  // whether a particle of this cell may come within a collision radius (0.32h, the grid-to-particle pass's)
  // of an obstacle this sub-step
  if (i < nx && j < ny && k < nz)
    T.near[cell_idx(T, i, j, k)] = cell_near(T, T.ox + h * (i + 0.5), T.oy + h * (j + 0.5), T.oz + h * (k + 0.5), 0.32 * h);
  T.frac[n] = make_float4((float)f[0], (float)f[1], (float)f[2], 0.f);
  T.svel[n] = make_float4((float)sv[0], (float)sv[1], (float)sv[2], 0.f);
}

// ------------------------------------------------------------------------------------------------ P2G
// One block per 8×8×8-cell brick. The brick's particles are contiguous per (j,k) row in the sorted
// array, so the block walks them coalesced and splats into a shared-memory copy of the 10×10×10 nodes
// they can reach, as fixed-point integers (exact, order independent; 32-bit halves while the brick's
// cell counts allow, 64-bit otherwise), then adds the non-zero
// node sums into the global accumulator. Weights follow blender_addon/suiri_lab/solver.py:443-460
// (float64; per corner w = (wx·wy)·wz, zero weights skipped, velocity clamped to ±30) and
// src/js/30-wgsl-sim.js:159-200 (fixed point). The global accumulator is zeroed by the node pass that
// consumes it.
constexpr int kBN = kBrick + 2;              // nodes per brick edge, halo included
constexpr int kBNodes = kBN * kBN * kBN;

__global__ void __launch_bounds__(kThreads) k_p2g(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx) {
  __shared__ long long s_acc[6][kBNodes];
  __shared__ int s_row0[kBrick * kBrick];
  __shared__ int s_rowp[kBrick * kBrick + 1];
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int lb = blockIdx.x - bpfx[t];
  const int bnx = (T.nx + kBrick - 1) / kBrick, bny = (T.ny + kBrick - 1) / kBrick;
  const int bi = lb % bnx, bj = (lb / bnx) % bny, bk = lb / (bnx * bny);
  const int i0 = bi * kBrick, j0 = bj * kBrick, k0 = bk * kBrick;
  const int i1 = min(i0 + kBrick, T.nx);
  __shared__ int s_maxc;
  for (int e = threadIdx.x; e < 6 * kBNodes; e += blockDim.x) (&s_acc[0][0])[e] = 0;
  if (threadIdx.x == 0) s_maxc = 0;
  __syncthreads();
  if (threadIdx.x < kBrick * kBrick) {
    const int j = j0 + (threadIdx.x % kBrick), k = k0 + (threadIdx.x / kBrick);
    int a = 0, b = 0, mc = 0;
    if (j < T.ny && k < T.nz) {
      const int* o = T.off + cell_idx(T, i0, j, k);
      a = o[0];
      int prev = a;
      for (int i = 1; i <= i1 - i0; ++i) {
        const int x = o[i];
        mc = max(mc, x - prev);
        prev = x;
      }
      b = prev;
    }
    s_row0[threadIdx.x] = a;
    s_rowp[threadIdx.x + 1] = b - a;
    if (mc > 0) atomicMax(&s_maxc, mc);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s_rowp[0] = 0;
    for (int r = 1; r <= kBrick * kBrick; ++r) s_rowp[r] += s_rowp[r - 1];
  }
  __syncthreads();
  const int total = s_rowp[kBrick * kBrick];
  if (total == 0) return;                      // an empty brick adds nothing
  const int nsx = T.nx + 1, nsy = T.ny + 1, nsz = T.nz + 1;
  // Walk the brick's particles in a strided permutation q = j·P mod total (P coprime to total, about a
  // warp's share apart): consecutive lanes of a warp then take particles of cells far apart, so their
  // shared-memory atomics hit different nodes instead of the same 8 (sorted neighbours share a cell).
  __shared__ int s_P;
  if (threadIdx.x == 0) {
    int P = (total / 32) | 1;
    if (P < 1) P = 1;
    auto gcd = [](int a, int b) { while (b) { const int t = a % b; a = b; b = t; } return a; };
    while (total > 1 && gcd(P, total) != 1) ++P;
    s_P = P;
  }
  __syncthreads();
  const long long P = s_P;
  // A node takes terms from the particles of at most 2·3·3 cells of the brick (its own axis: the two cells
  // either side; the other axes: three cells, half of the outer two), so at most 18·(largest cell count)
  // terms. Within kSplitMaxTerms the split 32-bit sums are exact; above it the 64-bit shared atomics are used.
  const bool split = 18 * s_maxc <= kSplitMaxTerms;
  unsigned* s_lo = reinterpret_cast<unsigned*>(&s_acc[0][0]);
  int* s_hi = reinterpret_cast<int*>(&s_acc[0][0]) + 6 * kBNodes;
  for (int j = threadIdx.x; j < total; j += blockDim.x) {
    const int q = (int)((j * P) % total);
    int lo = 0, hi = kBrick * kBrick - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_rowp[mid] <= q) lo = mid; else hi = mid - 1;
    }
    const int pi = s_row0[lo] + (q - s_rowp[lo]);
    const float4 Pp = T.pB[pi];
    const float4 V = T.vB[pi];
    double g[3];
    grid_pos(T, (double)Pp.x, (double)Pp.y, (double)Pp.z, g[0], g[1], g[2]);
    const double vv[3] = {fmin(fmax((double)V.x, -30.0), 30.0), fmin(fmax((double)V.y, -30.0), 30.0),
                          fmin(fmax((double)V.z, -30.0), 30.0)};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double qx = g[0] - (a == 0 ? 0.0 : 0.5), qy = g[1] - (a == 1 ? 0.0 : 0.5), qz = g[2] - (a == 2 ? 0.0 : 0.5);
      const int bx = (int)floor(qx), by = (int)floor(qy), bz = (int)floor(qz);
      const double fx = qx - bx, fy = qy - by, fz = qz - bz;
      const double wx[2] = {1 - fx, fx}, wy[2] = {1 - fy, fy}, wz[2] = {1 - fz, fz};
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int dx = e >> 2, dy = (e >> 1) & 1, dz = e & 1;
        const int ix = bx + dx, iy = by + dy, iz = bz + dz;
        if (ix < 0 || ix >= nsx || iy < 0 || iy >= nsy || iz < 0 || iz >= nsz) continue;
        const double w = (wx[dx] * wy[dy]) * wz[dz];
        if (!(w > 0.0)) continue;
        const int ln = (ix - i0 + 1) + kBN * ((iy - j0 + 1) + kBN * (iz - k0 + 1));
        const long long tm = __double2ll_rn(w * vv[a] * kFix), tw = __double2ll_rn(w * kFix);
        if (split) {
          // term = quotient·2^19 + remainder: two native 32-bit shared atomics, exact (see common.cuh)
          atomicAdd(s_lo + a * kBNodes + ln, (unsigned)(tm & ((1LL << kSplit) - 1)));
          atomicAdd(s_hi + a * kBNodes + ln, (int)(tm >> kSplit));
          atomicAdd(s_lo + (3 + a) * kBNodes + ln, (unsigned)(tw & ((1LL << kSplit) - 1)));
          atomicAdd(s_hi + (3 + a) * kBNodes + ln, (int)(tw >> kSplit));
        } else {
          atomicAdd((unsigned long long*)&s_acc[a][ln], (unsigned long long)tm);
          atomicAdd((unsigned long long*)&s_acc[3 + a][ln], (unsigned long long)tw);
        }
      }
    }
  }
  __syncthreads();
  for (int ln = threadIdx.x; ln < kBNodes; ln += blockDim.x) {
    const int li = ln % kBN, lj = (ln / kBN) % kBN, lk = ln / (kBN * kBN);
    const int ix = i0 - 1 + li, iy = j0 - 1 + lj, iz = k0 - 1 + lk;
    if (ix < 0 || iy < 0 || iz < 0 || ix >= nsx || iy >= nsy || iz >= nsz) continue;
    const int n = node_idx(T, ix, iy, iz);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const long long w = split ? (long long)s_hi[(3 + a) * kBNodes + ln] * (1LL << kSplit) + (long long)s_lo[(3 + a) * kBNodes + ln]
                                : s_acc[3 + a][ln];
      if (w == 0) continue;
      atomicAdd((unsigned long long*)&T.acc[(size_t)(3 + a) * T.nnodes + n], (unsigned long long)w);
      const long long m = split ? (long long)s_hi[a * kBNodes + ln] * (1LL << kSplit) + (long long)s_lo[a * kBNodes + ln]
                                : s_acc[a][ln];
      if (m != 0) atomicAdd((unsigned long long*)&T.acc[(size_t)a * T.nnodes + n], (unsigned long long)m);
    }
  }
}

// ---------------------------------------------------------------------------------------- node pass
// momentum / weight → velocity where the weight exceeds 4e-6 (solver.py:456-460); keep that as the
// FLIP reference with the valid-face mask; gravity on y faces; closed faces take the solid velocity;
// cut-cell fluxes f·v + (1-f)·s for the divergence (solver.py:461-468; 30-wgsl-sim.js:203-238).
__global__ void __launch_bounds__(kThreads) k_grid_nodes(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx) {
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int n = (blockIdx.x - bpfx[t]) * blockDim.x + threadIdx.x;
  if (n >= T.nnodes) return;
  const size_t nn = T.nnodes;
  // every load first (one round of memory latency), then the arithmetic, then the stores
  long long* __restrict__ acc = T.acc;
  const double* __restrict__ fracd = T.fracd;
  long long W[3], M[3];
  double f[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    W[a] = acc[(3 + a) * nn + n];
    M[a] = acc[a * nn + n];
    f[a] = fracd[a * nn + n];
  }
  const float4 s4 = T.svel[n];
  double v[3];
  int mask = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const bool m = (double)W[a] * kFixInv > 4e-6;
    v[a] = m ? (double)M[a] / (double)W[a] : 0.0;
    mask |= m ? (1 << a) : 0;
  }
  const float4 vo = make_float4((float)v[0], (float)v[1], (float)v[2], (float)mask);
  v[1] -= T.g * T.dt;
  const double s[3] = {(double)s4.x, (double)s4.y, (double)s4.z};
  double fl[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (f[a] <= 0.0) v[a] = s[a];
    fl[a] = f[a] * v[a] + (1 - f[a]) * s[a];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {            // a node no particle reached is zero already
    if (W[a]) acc[(3 + a) * nn + n] = 0;
    if (M[a]) acc[a * nn + n] = 0;
  }
  double* __restrict__ flux = T.flux;
#pragma unroll
  for (int a = 0; a < 3; ++a) flux[a * nn + n] = fl[a];
  T.velold[n] = vo;
  T.vel[n] = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
}

// ---------------------------------------------------------------------------------------- cell pass
// divergence with the drift correction (solver.py:467-472), the float32 SOR right-hand side h²·div
// (solver.py:487), the per-cell SOR code (open / partial faces, active = liquid with an open face:
// solver.py:478-486) and the warm start: liquid cells keep last sub-step's pressure, others 0 (:474).
__global__ void __launch_bounds__(kThreads) k_grid_cells(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx,
                                                         int* __restrict__ apfx, unsigned* __restrict__ ticket) {
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int c0 = (blockIdx.x - bpfx[t]) * blockDim.x + threadIdx.x;
  const bool valid = c0 < T.ncells;
  const int c = valid ? c0 : T.ncells - 1;
  const int row = divu(c, T.dnx);
  const int k = divu(row, T.dny);
  const int i = c - row * T.nx, j = row - k * T.ny;
  const int count = T.off[c + 1] - T.off[c];
  const bool fluid = count > 0;
  const int n = node_idx(T, i, j, k);
  const size_t nn = T.nnodes;
  double div = 0.0;
  if (fluid) {
    const double* F = T.flux;
    div = F[n + 1] - F[n];
    div = div + F[nn + n + T.sx];
    div = div - F[nn + n];
    div = div + F[2 * nn + n + T.sxy];
    div = div - F[2 * nn + n];
    div = div / T.h;
    div = div - T.drift * fmax((double)count / T.ppc - 1, 0.0);
  }
  const float rhs = (float)(T.h * T.h * div);
  const float4 f0 = T.frac[n];
  const float C[6] = {f0.x, T.frac[n + 1].x, f0.y, T.frac[n + T.sx].y, f0.z, T.frac[n + T.sxy].z};
  float den = C[0];
#pragma unroll
  for (int d = 1; d < 6; ++d) den = den + C[d];
  uint32_t code = 0;
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    if (C[d] == 1.0f) code |= 1u << d;
    else if (C[d] > 0.0f) code |= kCodePartial;
  }
  if (fluid && den > 0.0f) code |= kCodeActive;
  const int col = (i + j + k) & 1;
  const int hs = half_idx(T, i, j, k);
  const size_t s = (size_t)col * T.nhalf + hs;
  if (valid) {
    T.rhs[s] = rhs;
    T.code[s] = code;
    if (!fluid) T.pres[s] = 0.f;
  }
  // the active cells' slots, per colour, for the sweeps (one atomic per warp and colour; the order in the
  // lists does not matter, a sweep updates each cell from the other colour only)
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int cc = 0; cc < 2; ++cc) {
    const bool mine = valid && (code & kCodeActive) && col == cc;
    const unsigned m = __ballot_sync(0xffffffffu, mine);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    int at = 0;
    if (lane == leader) at = atomicAdd(&T.ctr->n_act[cc], __popc(m));
    at = __shfl_sync(0xffffffffu, at, leader);
    if (mine)
      T.act[(size_t)cc * T.nhalf + at + __popc(m & ((1u << lane) - 1))] =
          make_int4(hs, (int)code, __float_as_int(rhs), __float_as_int(__frcp_rn(den)));
  }
  // the last block: per colour, the prefix over tanks of the active counts (the sweeps' item → tank map)
  if (last_block(ticket)) {
    for (int cc = 0; cc < 2; ++cc)
      tank_prefix(ntanks, apfx + cc * (ntanks + 1), [&](int u) { return __ldcg(&tanks[u].ctr->n_act[cc]); });
  }
}

// ---------------------------------------------------------------------------------------- projection
// v -= (p⁺ - p⁻)/h on faces with a liquid cell on either side; closed faces take the solid velocity
// (solver.py:510-523, src/js/30-wgsl-sim.js:299-341). Outside the side walls and floor counts as solid,
// above the grid as air; non-liquid cells hold p = 0.
__device__ __forceinline__ bool cell_fluid(const TankDev& T, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= T.nx || j >= T.ny || k >= T.nz) return false;
  const int c = cell_idx(T, i, j, k);
  return T.off[c + 1] > T.off[c];
}
__device__ __forceinline__ double cell_pres(const TankDev& T, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= T.nx || j >= T.ny || k >= T.nz) return 0.0;
  return (double)T.pres[(size_t)((i + j + k) & 1) * T.nhalf + half_idx(T, i, j, k)];
}

__global__ void __launch_bounds__(kThreads) k_project(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx) {
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int n = (blockIdx.x - bpfx[t]) * blockDim.x + threadIdx.x;
  if (n >= T.nnodes) return;
  int i, j, k;
  node_coord(T, n, i, j, k);
  float4 v = T.vel[n];
  const float4 f = T.frac[n];
  const float4 s = T.svel[n];
  const double h = T.h;
  if (j < T.ny && k < T.nz) {
    if (f.x <= 0.f) v.x = s.x;
    else if (cell_fluid(T, i - 1, j, k) || cell_fluid(T, i, j, k))
      v.x = (float)((double)v.x - (cell_pres(T, i, j, k) - cell_pres(T, i - 1, j, k)) / h);
  }
  if (i < T.nx && k < T.nz) {
    if (f.y <= 0.f) v.y = s.y;
    else if (cell_fluid(T, i, j - 1, k) || cell_fluid(T, i, j, k))
      v.y = (float)((double)v.y - (cell_pres(T, i, j, k) - cell_pres(T, i, j - 1, k)) / h);
  }
  if (i < T.nx && j < T.ny) {
    if (f.z <= 0.f) v.z = s.z;
    else if (cell_fluid(T, i, j, k - 1) || cell_fluid(T, i, j, k))
      v.z = (float)((double)v.z - (cell_pres(T, i, j, k) - cell_pres(T, i, j, k - 1)) / h);
  }
  T.vel[n] = v;
  // compact per-component pairs for the G2P gathers: one 8-byte load per corner; NaN marks a face that
  // took no particle weight (it is skipped, solver.py:240-245)
  const float4 vo = T.velold[n];
  const int m = (int)vo.w;
  const float qnan = __int_as_float(0x7fc00000);
  const size_t nn = T.nnodes;
  T.vv[n] = make_float2(v.x, (m & 1) ? vo.x : qnan);
  T.vv[nn + n] = make_float2(v.y, (m & 2) ? vo.y : qnan);
  T.vv[2 * nn + n] = make_float2(v.z, (m & 4) ? vo.z : qnan);
}

void launch_geom(const LaunchCtx& L) {
  k_geom<<<L.nblocks[kFamNodes], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamNodes]);
}
void launch_p2g(const LaunchCtx& L) {
  k_p2g<<<L.nblocks[kFamBricks], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamBricks]);
}
void launch_grid_nodes(const LaunchCtx& L) {
  k_grid_nodes<<<L.nblocks[kFamNodes], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamNodes]);
}
void launch_grid_cells(const LaunchCtx& L) {
  k_grid_cells<<<L.nblocks[kFamCells], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamCells], L.apfx, L.ticket + 0);
}
void launch_project(const LaunchCtx& L) {
  k_project<<<L.nblocks[kFamNodes], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamNodes]);
}

}  // namespace suiri
