// Liquid surface mesh of a frame, for the per-frame export (blender_addon/suiri_lab/meshing.py:52-199,
// bake.py:228-235).
//
//   classify   a particle with at most 6 particles in the 3×3×3 cells around its own (counted at the frame
//              end; none outside the grid) is drawn as its own icosphere; the others form the body, whose
//              bounding box (float32 positions, ordered-key atomics) sizes the lattice
//   splat      the body's distance field on a lattice of spacing h/2 around that box: every particle
//              lowers the 4×4×4 nodes around it to |node - x| - r (float64, kept float32 by an ordered-key
//              minimum, so the field does not depend on the order of the atomics); far value 2·spacing. The
//              particles are put in cell order first, and one block per tile of 8×4×4 cells takes its minima
//              in shared memory and then one global minimum per node it lowered
//   smooth     clipped to [-r, far], blurred along x, y, z with normalised Gaussian taps, each tap added in
//              float64 and rounded to float32 as the reference's float32 array accumulates it
//   nets       surface nets: a vertex per cell whose corners change sign (the mean of its edge crossings),
//              a quad per sign-changing lattice edge, turned outwards. Vertices are numbered in cell order
//              (x slowest) and quads by edge axis, then edge order, by one ordered compaction over all of
//              them (per-block counts, one scan, per-block ranks from warp ballots), so the numbering is the
//              reference's and does not depend on scheduling
//   finish     lattice → world, the body held inside the glass and above the floor, 42 icosphere vertices
//              per lone particle (particle order), every vertex within 0.6h of the wet top-view height map
//              settled onto it, and the liquid's face velocity sampled trilinearly at each vertex
//
// float64 geometry built without FMA contraction, so that vertices and velocities round as the reference's
// NumPy code does.
#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.h"

namespace suiri {

namespace {

constexpr int kMeshThreads = 1024;   // threads of a compaction block
constexpr int kMeshItems = 8;        // consecutive items per thread: a block's tile is 8192 items
constexpr int kMeshPhases = 5;       // classify, distance field, blur, surface nets, finish (device time each)
constexpr int kMaxTaps = 33;

struct MeshCounters {
  unsigned lo_key[3], hi_key[3];     // ordered keys of the body's float32 position extremes
  int n_body, n_lone;
};

struct MeshTaps { double w[kMaxTaps]; int n; };

struct MeshGeom {
  int X, Y, Z;                       // lattice nodes per axis
  double lo[3], sp, r, far_;         // lattice origin, spacing, sphere radius, far value
  float r32, far32;
};

// segments of the one ordered compaction: mixed cells, edges along x, y, z, lone particles
struct MeshSegs {
  long long n[5];
  int first_block[6];
};

__device__ __forceinline__ unsigned okey(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float okey_inv(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__device__ __forceinline__ int cell_count(const TankDev& T, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= T.nx || j >= T.ny || k >= T.nz) return 0;
  const int c = cell_idx(T, i, j, k);
  return T.off[c + 1] - T.off[c];
}

// per particle of A∪E: 0 body, 1 lone, 2 dead (meshing.py:60-73)
__global__ void __launch_bounds__(256) k_mesh_classify(const TankDev* __restrict__ Tp, uint8_t* __restrict__ kind,
                                                       MeshCounters* __restrict__ mc) {
  const TankDev& T = *Tp;
  const int n_live = T.ctr->n_live, n = n_live + T.ctr->n_emit;
  const int lane = threadIdx.x & 31;
  unsigned lo[3] = {~0u, ~0u, ~0u}, hi[3] = {0u, 0u, 0u};
  int nb = 0, nl = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float4 p = q < n_live ? T.pA[q] : T.pE[q - n_live];
    if (flags_of(p.w) & kFlagDead) { kind[q] = 2; continue; }
    double gx, gy, gz;
    grid_pos(T, (double)p.x, (double)p.y, (double)p.z, gx, gy, gz);
    int near = 0;
    if (in_grid(T, gx, gy, gz)) {
      const int ci = (int)floor(gx), cj = (int)floor(gy), ck = (int)floor(gz);
      for (int dk = -1; dk <= 1; ++dk)
        for (int dj = -1; dj <= 1; ++dj)
          for (int di = -1; di <= 1; ++di) near += cell_count(T, ci + di, cj + dj, ck + dk);
    }
    const bool lone = near <= 6;
    kind[q] = lone ? 1 : 0;
    if (lone) { ++nl; continue; }
    ++nb;
    const float c[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) { lo[a] = min(lo[a], okey(c[a])); hi[a] = max(hi[a], okey(c[a])); }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nb += __shfl_xor_sync(~0u, nb, o);
    nl += __shfl_xor_sync(~0u, nl, o);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = min(lo[a], __shfl_xor_sync(~0u, lo[a], o));
      hi[a] = max(hi[a], __shfl_xor_sync(~0u, hi[a], o));
    }
  }
  if (lane == 0) {
    if (nb) {
      atomicAdd(&mc->n_body, nb);
      for (int a = 0; a < 3; ++a) { atomicMin(&mc->lo_key[a], lo[a]); atomicMax(&mc->hi_key[a], hi[a]); }
    }
    if (nl) atomicAdd(&mc->n_lone, nl);
  }
}

__global__ void k_mesh_fill(unsigned* __restrict__ key, long long n, unsigned v) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) key[e] = v;
}

// Cell order of the in-grid particles of A∪E (the counts and offsets of the frame-end count pass): their
// indices, grouped by cell, so that a tile of cells finds its particles as a few contiguous runs
__global__ void __launch_bounds__(256) k_mesh_order(const TankDev* __restrict__ Tp, int* __restrict__ fill,
                                                    int* __restrict__ order) {
  const TankDev& T = *Tp;
  const int n_live = T.ctr->n_live, n = n_live + T.ctr->n_emit;
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += gridDim.x * blockDim.x) {
    const int q = base + lane;
    int cell = -1;
    if (q < n) {
      const float4 p = q < n_live ? T.pA[q] : T.pE[q - n_live];
      if (!(flags_of(p.w) & kFlagDead)) {
        double gx, gy, gz;
        grid_pos(T, (double)p.x, (double)p.y, (double)p.z, gx, gy, gz);
        if (in_grid(T, gx, gy, gz)) cell = cell_idx(T, (int)gx, (int)gy, (int)gz);
      }
    }
    const unsigned act = __ballot_sync(0xffffffffu, cell >= 0);
    if (cell >= 0) {
      const unsigned peers = __match_any_sync(act, (unsigned)cell);
      const int leader = __ffs(peers) - 1;
      int first = 0;
      if (lane == leader) first = atomicAdd(fill + cell, __popc(peers));
      first = __shfl_sync(act, first, leader);
      order[T.off[cell] + first + __popc(peers & ((1u << lane) - 1u))] = q;
    }
  }
}

// The body's distance field per tile of kTX×kTY×kTZ cells: the particles of the tile's cells that are not lone
// (the same 27-cell count test as k_mesh_classify, per cell) lower the lattice nodes around them in a
// shared-memory copy of the nodes the tile can reach, then each node the tile lowered takes one global
// minimum. Same values as one global minimum per particle and node: a minimum does not depend on order.
constexpr int kTX = 8, kTY = 4, kTZ = 4;
constexpr int kBX = 2 * kTX + 6, kBY = 2 * kTY + 6, kBZ = 2 * kTZ + 6;   // node box: 2 nodes a cell + margins
__global__ void __launch_bounds__(256) k_mesh_splat_tiles(const TankDev* __restrict__ Tp, const int* __restrict__ order,
                                                          MeshGeom G, unsigned far_key, unsigned* __restrict__ key) {
  __shared__ unsigned s_key[kBX * kBY * kBZ];
  __shared__ int s_row0[kTY * kTZ], s_rowp[kTY * kTZ + 1];
  __shared__ unsigned char s_lone[kTX * kTY * kTZ];
  const TankDev& T = *Tp;
  const int tnx = (T.nx + kTX - 1) / kTX, tny = (T.ny + kTY - 1) / kTY;
  const int ci0 = (blockIdx.x % tnx) * kTX, cj0 = ((blockIdx.x / tnx) % tny) * kTY, ck0 = (blockIdx.x / (tnx * tny)) * kTZ;
  const int ci1 = min(ci0 + kTX, T.nx);
  if (threadIdx.x < kTY * kTZ) {
    const int j = cj0 + threadIdx.x % kTY, k = ck0 + threadIdx.x / kTY;
    int a = 0, b = 0;
    if (j < T.ny && k < T.nz) {
      a = T.off[cell_idx(T, ci0, j, k)];
      b = T.off[cell_idx(T, ci1 - 1, j, k) + 1];
    }
    s_row0[threadIdx.x] = a;
    s_rowp[threadIdx.x + 1] = b - a;
  }
  for (int c = threadIdx.x; c < kTX * kTY * kTZ; c += blockDim.x) {
    const int i = ci0 + c % kTX, j = cj0 + (c / kTX) % kTY, k = ck0 + c / (kTX * kTY);
    int near = 0;
    if (i < T.nx && j < T.ny && k < T.nz)
      for (int dk = -1; dk <= 1; ++dk)
        for (int dj = -1; dj <= 1; ++dj)
          for (int di = -1; di <= 1; ++di) near += cell_count(T, i + di, j + dj, k + dk);
    s_lone[c] = near <= 6;
  }
  for (int e = threadIdx.x; e < kBX * kBY * kBZ; e += blockDim.x) s_key[e] = far_key;
  __syncthreads();
  if (threadIdx.x == 0) {
    s_rowp[0] = 0;
    for (int r = 1; r <= kTY * kTZ; ++r) s_rowp[r] += s_rowp[r - 1];
  }
  __syncthreads();
  const int total = s_rowp[kTY * kTZ];
  if (total == 0) return;
  // the node box's first node per axis: two below the lattice node of the tile's low cell corner
  const long long b0[3] = {(long long)floor(((T.ox + ci0 * T.h) - G.lo[0]) / G.sp) - 2,
                           (long long)floor(((T.oy + cj0 * T.h) - G.lo[1]) / G.sp) - 2,
                           (long long)floor(((T.oz + ck0 * T.h) - G.lo[2]) / G.sp) - 2};
  const int n_live = T.ctr->n_live, n_all = n_live + T.ctr->n_emit;
  // the tile's particles in a strided permutation j·P mod total (P about a warp's share, coprime to total):
  // the lanes of a warp take particles of cells far apart, so their minima seldom hit the same node
  __shared__ int s_P;
  if (threadIdx.x == 0) {
    int P = (total / 32) | 1;
    auto gcd = [](int a, int b) { while (b) { const int t = a % b; a = b; b = t; } return a; };
    while (total > 1 && gcd(P, total) != 1) ++P;
    s_P = P;
  }
  __syncthreads();
  const long long Pst = s_P;
  for (int jj = threadIdx.x; jj < total; jj += blockDim.x) {
    const int qq = (int)((jj * Pst) % total);
    int lo = 0, hi = kTY * kTZ - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_rowp[mid] <= qq) lo = mid; else hi = mid - 1;
    }
    const int slot = s_row0[lo] + (qq - s_rowp[lo]);
    const int q = order[slot];
    if (q < 0 || q >= n_all) continue;
    const float4 p = q < n_live ? T.pA[q] : T.pE[q - n_live];
    double gx, gy, gz;
    grid_pos(T, (double)p.x, (double)p.y, (double)p.z, gx, gy, gz);
    const int ci = (int)gx - ci0, cj = (int)gy - cj0, ck = (int)gz - ck0;
    if (ci < 0 || ci >= kTX || cj < 0 || cj >= kTY || ck < 0 || ck >= kTZ) continue;
    if (s_lone[ci + kTX * (cj + kTY * ck)]) continue;
    const double u[3] = {((double)p.x - G.lo[0]) / G.sp, ((double)p.y - G.lo[1]) / G.sp, ((double)p.z - G.lo[2]) / G.sp};
    const long long b[3] = {(long long)floor(u[0]), (long long)floor(u[1]), (long long)floor(u[2])};
    for (int ox = -1; ox <= 2; ++ox) {
      const long long x = b[0] + ox;
      if (x < 0 || x >= G.X) continue;
      const double ex = ((double)x - u[0]) * G.sp;
      for (int oy = -1; oy <= 2; ++oy) {
        const long long y = b[1] + oy;
        if (y < 0 || y >= G.Y) continue;
        const double ey = ((double)y - u[1]) * G.sp;
        for (int oz = -1; oz <= 2; ++oz) {
          const long long z = b[2] + oz;
          if (z < 0 || z >= G.Z) continue;
          const double ez = ((double)z - u[2]) * G.sp;
          const double d = sqrt(ex * ex + ey * ey + ez * ez) - G.r;
          if (!(d < G.far_)) continue;
          const unsigned kv = okey(__double2float_rn(d));
          const long long lx = x - b0[0], ly = y - b0[1], lz = z - b0[2];
          if (lx >= 0 && lx < kBX && ly >= 0 && ly < kBY && lz >= 0 && lz < kBZ)
            atomicMin(s_key + lx + kBX * (ly + kBY * lz), kv);
          else
            atomicMin(key + (x * G.Y + y) * G.Z + z, kv);    // outside the box (not expected): directly
        }
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kBX * kBY * kBZ; e += blockDim.x) {
    const unsigned v = s_key[e];
    if (v == far_key) continue;
    const long long x = b0[0] + e % kBX, y = b0[1] + (e / kBX) % kBY, z = b0[2] + e / (kBX * kBY);
    if (x < 0 || x >= G.X || y < 0 || y >= G.Y || z < 0 || z >= G.Z) continue;
    atomicMin(key + (x * G.Y + y) * G.Z + z, v);
  }
}

// one axis of the separable blur with held edges (meshing.py:8-23); axis 0 reads the keys and clips
template <int kAxis>
__global__ void __launch_bounds__(256) k_mesh_blur(const void* __restrict__ in, float* __restrict__ out, MeshGeom G, MeshTaps W) {
  const long long n = (long long)G.X * G.Y * G.Z;
  const int r = W.n / 2;
  const long long stride = kAxis == 0 ? (long long)G.Y * G.Z : (kAxis == 1 ? G.Z : 1);
  const int len = kAxis == 0 ? G.X : (kAxis == 1 ? G.Y : G.Z);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)((e / stride) % len);
    const long long base = e - (long long)c * stride;
    float acc = 0.f;
    for (int t = 0; t < W.n; ++t) {
      const int s = min(max(c + t - r, 0), len - 1);
      float v;
      if (kAxis == 0) v = fminf(fmaxf(okey_inv(((const unsigned*)in)[base + s * stride]), -G.r32), G.far32);
      else v = ((const float*)in)[base + s * stride];
      acc = __double2float_rn(__dadd_rn((double)acc, __dmul_rn(W.w[t], (double)v)));
    }
    out[e] = acc;
  }
}

// --- the ordered compaction
__device__ __forceinline__ int seg_of(const MeshSegs& S, int block) {
  int s = 0;
  while (s < 4 && block >= S.first_block[s + 1]) ++s;
  return s;
}

__device__ __forceinline__ bool cell_mixed(const float* __restrict__ phi, const MeshGeom& G, long long c) {
  const int Zc = G.Z - 1, Yc = G.Y - 1;
  const int k = (int)(c % Zc);
  const long long t = c / Zc;
  const int j = (int)(t % Yc), i = (int)(t / Yc);
  int nin = 0;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int d = 0; d < 2; ++d) nin += phi[((long long)(i + a) * G.Y + (j + b)) * G.Z + (k + d)] < 0.f;
  return nin > 0 && nin < 8;
}

// lattice edge e along axis ax (edge array: that axis one shorter), as node (i, j, k)
__device__ __forceinline__ void edge_node(const MeshGeom& G, int ax, long long e, int& i, int& j, int& k) {
  const int ex = G.X - (ax == 0), ey = G.Y - (ax == 1), ez = G.Z - (ax == 2);
  k = (int)(e % ez);
  const long long t = e / ez;
  j = (int)(t % ey);
  i = (int)(t / ey);
  (void)ex;
}

__device__ __forceinline__ bool edge_crossing(const float* __restrict__ phi, const MeshGeom& G, int ax, long long e,
                                              bool* lo_in) {
  int i, j, k;
  edge_node(G, ax, e, i, j, k);
  const int dim[3] = {G.X, G.Y, G.Z};
  const int c[3] = {i, j, k};
  // the four cells around the edge need 1 <= index <= dim - 2 on both other axes
#pragma unroll
  for (int a = 0; a < 3; ++a)
    if (a != ax && (c[a] == 0 || c[a] == dim[a] - 1)) return false;
  const long long n0 = ((long long)i * G.Y + j) * G.Z + k;
  const long long step = ax == 0 ? (long long)G.Y * G.Z : (ax == 1 ? G.Z : 1);
  const bool a = phi[n0] < 0.f, b = phi[n0 + step] < 0.f;
  *lo_in = a;
  return a != b;
}

__device__ __forceinline__ bool seg_flag(int seg, long long item, const float* __restrict__ phi, const MeshGeom& G,
                                         const uint8_t* __restrict__ kind) {
  if (seg == 0) return cell_mixed(phi, G, item);
  if (seg <= 3) { bool lo; return edge_crossing(phi, G, seg - 1, item, &lo); }
  return kind[item] == 1;
}

// exclusive prefix of the threads' counts in thread order; the block's total in *total
__device__ __forceinline__ int block_excl(int v, int* total) {
  __shared__ int s_w[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(~0u, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_w[w] = inc;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    const int x = lane < nw ? s_w[lane] : 0;
    int iw = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(~0u, iw, o);
      if (lane >= o) iw += y;
    }
    if (lane < nw) s_w[lane] = iw - x;
    if (lane == 31) *total = iw;
  }
  __syncthreads();
  const int r = s_w[w] + inc - v;
  __syncthreads();
  return r;
}

// the first item of this thread's run of kMeshItems consecutive items in block `blk` of a segment
__device__ __forceinline__ long long run_first(int blk_in_seg) {
  return ((long long)blk_in_seg * kMeshThreads + threadIdx.x) * kMeshItems;
}

__global__ void __launch_bounds__(kMeshThreads) k_mesh_count(const float* __restrict__ phi, MeshGeom G, MeshSegs S,
                                                             const uint8_t* __restrict__ kind, int* __restrict__ bcount) {
  __shared__ int s_tot;
  const int seg = seg_of(S, blockIdx.x);
  const long long first = run_first(blockIdx.x - S.first_block[seg]);
  int cnt = 0;
  for (int m = 0; m < kMeshItems; ++m) {
    const long long item = first + m;
    if (item < S.n[seg] && seg_flag(seg, item, phi, G, kind)) ++cnt;
  }
  block_excl(cnt, &s_tot);
  if (threadIdx.x == 0) bcount[blockIdx.x] = s_tot;
}

// exclusive prefix of the block counts, one block
__global__ void __launch_bounds__(1024) k_mesh_scan(int* __restrict__ bcount, int nb) {
  __shared__ int s[1024];
  const int per = (nb + 1023) / 1024;
  const int lo = threadIdx.x * per, hi = min(lo + per, nb);
  int sum = 0;
  for (int b = lo; b < hi; ++b) sum += bcount[b];
  s[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int a = (int)threadIdx.x >= o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += a;
    __syncthreads();
  }
  int run = s[threadIdx.x] - sum;
  for (int b = lo; b < hi; ++b) { const int c = bcount[b]; bcount[b] = run; run += c; }
  if (threadIdx.x == 1023) bcount[nb] = s[1023];
}

// surface-nets vertex of a mixed cell in lattice units: the mean of the crossings on its 12 edges, edges in the
// order of the corner pairs (a < b, corners x slowest) (meshing.py:130-144)
__device__ void nets_vertex(const float* __restrict__ phi, const MeshGeom& G, long long c, double v[3]) {
  const int Zc = G.Z - 1, Yc = G.Y - 1;
  const int k = (int)(c % Zc);
  const long long t = c / Zc;
  const int j = (int)(t % Yc), i = (int)(t / Yc);
  float f[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) f[q] = phi[((long long)(i + (q >> 2)) * G.Y + (j + ((q >> 1) & 1))) * G.Z + (k + (q & 1))];
  double acc[3] = {0.0, 0.0, 0.0};
  int cnt = 0;
#pragma unroll
  for (int pa = 0; pa < 8; ++pa)
#pragma unroll
    for (int pb = 0; pb < 8; ++pb) {
      const int dif = pa ^ pb;
      if (pb <= pa || __popc(dif) != 1) continue;
      const float fa = f[pa], fb = f[pb];
      if ((fa < 0.f) == (fb < 0.f)) continue;
      const double tpar = (double)__fdiv_rn(fa, __fsub_rn(fa, fb));
      const double pt[3] = {(double)(pa >> 2) + (dif == 4 ? tpar : 0.0), (double)((pa >> 1) & 1) + (dif == 2 ? tpar : 0.0),
                            (double)(pa & 1) + (dif == 1 ? tpar : 0.0)};
#pragma unroll
      for (int a = 0; a < 3; ++a) acc[a] = __dadd_rn(acc[a], pt[a]);
      ++cnt;
    }
  const double den = (double)max(cnt, 1);
  v[0] = __dadd_rn((double)i, __ddiv_rn(acc[0], den));
  v[1] = __dadd_rn((double)j, __ddiv_rn(acc[1], den));
  v[2] = __dadd_rn((double)k, __ddiv_rn(acc[2], den));
}

__global__ void __launch_bounds__(kMeshThreads) k_mesh_cells(const float* __restrict__ phi, MeshGeom G, MeshSegs S,
                                                             const int* __restrict__ bbase, int* __restrict__ vid,
                                                             double* __restrict__ vtx) {
  __shared__ int s_tot;
  const long long first = run_first(blockIdx.x);
  unsigned mixed = 0;
  for (int m = 0; m < kMeshItems; ++m) {
    const long long c = first + m;
    if (c < S.n[0] && cell_mixed(phi, G, c)) mixed |= 1u << m;
  }
  int id = bbase[blockIdx.x] + block_excl(__popc(mixed), &s_tot);
  for (int m = 0; m < kMeshItems; ++m) {
    const long long c = first + m;
    if (c >= S.n[0]) break;
    if (!((mixed >> m) & 1u)) { vid[c] = -1; continue; }
    vid[c] = id;
    double v[3];
    nets_vertex(phi, G, c, v);
    vtx[3 * (size_t)id] = v[0]; vtx[3 * (size_t)id + 1] = v[1]; vtx[3 * (size_t)id + 2] = v[2];
    ++id;
  }
}

// quads around crossing edges (meshing.py:146-174): cells (o1, o2) back on the two other axes in the order
// (1,1), (0,1), (0,0), (1,0), reversed where the edge's low node is outside (for y: inside)
__global__ void __launch_bounds__(kMeshThreads) k_mesh_quads(const float* __restrict__ phi, MeshGeom G, MeshSegs S,
                                                             const int* __restrict__ bbase, const int* __restrict__ vid,
                                                             int4* __restrict__ quads) {
  __shared__ int s_tot;
  const int blk = blockIdx.x + S.first_block[1];
  const int seg = seg_of(S, blk);
  const int ax = seg - 1;
  const long long first = run_first(blk - S.first_block[seg]);
  unsigned cross = 0, low_in = 0;
  for (int m = 0; m < kMeshItems; ++m) {
    const long long e = first + m;
    bool lo_in = false;
    if (e < S.n[seg] && edge_crossing(phi, G, ax, e, &lo_in)) {
      cross |= 1u << m;
      if (lo_in) low_in |= 1u << m;
    }
  }
  int id = bbase[blk] + block_excl(__popc(cross), &s_tot) - bbase[S.first_block[1]];
  const int a1 = ax == 0 ? 1 : 0, a2 = ax == 2 ? 1 : 2;
  for (int m = 0; m < kMeshItems; ++m) {
    if (!((cross >> m) & 1u)) continue;
    int i, j, k;
    edge_node(G, ax, first + m, i, j, k);
    auto cell = [&](int o1, int o2) {
      int c[3] = {i, j, k};
      c[a1] -= o1; c[a2] -= o2;
      return vid[((long long)c[0] * (G.Y - 1) + c[1]) * (G.Z - 1) + c[2]];
    };
    int4 q = make_int4(cell(1, 1), cell(0, 1), cell(0, 0), cell(1, 0));
    const bool lo_in = (low_in >> m) & 1u;
    const bool rev = ax == 1 ? lo_in : !lo_in;
    if (rev) q = make_int4(q.w, q.z, q.y, q.x);
    quads[id++] = q;
  }
}

__global__ void __launch_bounds__(kMeshThreads) k_mesh_lone(MeshSegs S, const uint8_t* __restrict__ kind,
                                                            const int* __restrict__ bbase, int* __restrict__ lone_idx) {
  __shared__ int s_tot;
  const int blk = blockIdx.x + S.first_block[4];
  const long long first = run_first(blockIdx.x);
  unsigned lone = 0;
  for (int m = 0; m < kMeshItems; ++m) {
    const long long q = first + m;
    if (q < S.n[4] && kind[q] == 1) lone |= 1u << m;
  }
  int id = bbase[blk] + block_excl(__popc(lone), &s_tot) - bbase[S.first_block[4]];
  for (int m = 0; m < kMeshItems; ++m)
    if ((lone >> m) & 1u) lone_idx[id++] = (int)(first + m);
}

struct FinishParams {
  int nbody, nverts, W;              // body vertices, all vertices, top map texels (0: no settling)
  double ox, oy, oz, h, rim, x1, z1, size_x, size_z;
  const double* top;
  const double* ico;                 // 42 unit icosphere vertices
};

// liquid face velocity at world point p: trilinear per component with clamped taps, zero outside the grid
// (bake.py:231-235, solver.py:251-266)
__device__ void sample_vel(const TankDev& T, const double p[3], double out[3]) {
  const double g[3] = {(p[0] - T.ox) / T.h, (p[1] - T.oy) / T.h, (p[2] - T.oz) / T.h};
  if (!in_grid(T, g[0], g[1], g[2])) { out[0] = out[1] = out[2] = 0.0; return; }
  const int hi[3] = {T.nx, T.ny, T.nz};
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    double qv[3], f[3];
    int b[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      qv[a] = g[a] - (a == comp ? 0.0 : 0.5);
      const double fl = floor(qv[a]);
      b[a] = (int)fl;
      f[a] = qv[a] - fl;
    }
    double s = 0.0;
#pragma unroll
    for (int dx = 0; dx < 2; ++dx) {
      const double wx = dx ? f[0] : 1.0 - f[0];
      const int ci = min(max(b[0] + dx, 0), hi[0]);
#pragma unroll
      for (int dy = 0; dy < 2; ++dy) {
        const double wy = dy ? f[1] : 1.0 - f[1];
        const int cj = min(max(b[1] + dy, 0), hi[1]);
#pragma unroll
        for (int dz = 0; dz < 2; ++dz) {
          const double wz = dz ? f[2] : 1.0 - f[2];
          const int ck = min(max(b[2] + dz, 0), hi[2]);
          const float4 v = T.vel[node_idx(T, ci, cj, ck)];
          const float vc = comp == 0 ? v.x : (comp == 1 ? v.y : v.z);
          s = __dadd_rn(s, __dmul_rn(__dmul_rn(__dmul_rn(wx, wy), wz), (double)vc));
        }
      }
    }
    out[comp] = s;
  }
}

__global__ void __launch_bounds__(256) k_mesh_finish(const TankDev* __restrict__ Tp, MeshGeom G, FinishParams F,
                                                     const double* __restrict__ vtx, const int* __restrict__ lone_idx,
                                                     float* __restrict__ pos, float* __restrict__ vel) {
  const TankDev& T = *Tp;
  const int n_live = T.ctr->n_live;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < F.nverts; v += gridDim.x * blockDim.x) {
    double p[3];
    if (v < F.nbody) {
#pragma unroll
      for (int a = 0; a < 3; ++a) p[a] = __dadd_rn(G.lo[a], __dmul_rn(vtx[3 * (size_t)v + a], G.sp));
      // held inside the glass and above the floor where the vertex lies in the tank (meshing.py:96-102)
      const double m = 0.0005;
      if (p[0] > T.ox - G.sp && p[0] < F.x1 + G.sp && p[2] > T.oz - G.sp && p[2] < F.z1 + G.sp && p[1] < F.rim) {
        p[0] = fmin(fmax(p[0], T.ox + m), F.x1 - m);
        p[2] = fmin(fmax(p[2], T.oz + m), F.z1 - m);
        p[1] = fmax(p[1], m);
      }
    } else {
      const int d = (v - F.nbody) / 42, j = (v - F.nbody) - 42 * d;
      const int q = lone_idx[d];
      const float4 c = q < n_live ? T.pA[q] : T.pE[q - n_live];
      const double cc[3] = {(double)c.x, (double)c.y, (double)c.z};
#pragma unroll
      for (int a = 0; a < 3; ++a) p[a] = __dadd_rn(cc[a], __dmul_rn(F.ico[3 * j + a], G.r));
    }
    if (F.W > 0) {   // settle onto the top-view height map (meshing.py:177-199)
      const int W = F.W;
      const double u = __dsub_rn(__dmul_rn(__ddiv_rn(__dsub_rn(p[0], T.ox), F.size_x), (double)W), 0.5);
      const double w = __dsub_rn(__dmul_rn(__ddiv_rn(__dsub_rn(p[2], T.oz), F.size_z), (double)W), 0.5);
      if (u >= 0.0 && u <= W - 1 && w >= 0.0 && w <= W - 1) {
        const int bx = min((int)floor(u), W - 2), bz = min((int)floor(w), W - 2);
        const double fx = u - bx, fz = w - bz;
        const double h00 = F.top[(size_t)bz * W + bx], h10 = F.top[(size_t)bz * W + bx + 1];
        const double h01 = F.top[(size_t)(bz + 1) * W + bx], h11 = F.top[(size_t)(bz + 1) * W + bx + 1];
        if (h00 >= 0 && h10 >= 0 && h01 >= 0 && h11 >= 0) {
          const double lvl = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(h00, 1.0 - fx), __dmul_rn(h10, fx)), 1.0 - fz),
                                       __dmul_rn(__dadd_rn(__dmul_rn(h01, 1.0 - fx), __dmul_rn(h11, fx)), fz));
          const double band = 0.6 * T.h;
          if (p[1] > lvl - band && p[1] < lvl + band) p[1] = lvl;
        }
      }
    }
    double u[3];
    sample_vel(T, p, u);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      pos[3 * (size_t)v + a] = __double2float_rn(p[a]);
      vel[3 * (size_t)v + a] = __double2float_rn(u[a]);
    }
  }
}

}  // namespace

// unit icosphere, one subdivision: the 12 corners of the icosahedron, then each edge midpoint (normalised)
// the first time a face asks for it, faces in order, each split into its corner triangles and the middle one
// (meshing.py:26-49; the 20-face table is the icosahedron's standard connectivity)
static void icosphere(std::vector<double>& V, std::vector<int>& F) {
  const double p = (1 + sqrt(5.0)) / 2;
  const double base[12][3] = {{-1, p, 0}, {1, p, 0}, {-1, -p, 0}, {1, -p, 0}, {0, -1, p}, {0, 1, p},
                              {0, -1, -p}, {0, 1, -p}, {p, 0, -1}, {p, 0, 1}, {-p, 0, -1}, {-p, 0, 1}};
  static const int faces[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                                   {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                                   {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
  V.clear(); F.clear();
  auto push_unit = [&](const double* a) {
    const double n = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int c = 0; c < 3; ++c) V.push_back(a[c] / n);
  };
  for (auto& b : base) push_unit(b);
  std::vector<std::pair<std::pair<int, int>, int>> cache;
  auto mid = [&](int a, int b) {
    const std::pair<int, int> key(std::min(a, b), std::max(a, b));
    for (auto& e : cache) if (e.first == key) return e.second;
    const double m[3] = {V[3 * a] + V[3 * b], V[3 * a + 1] + V[3 * b + 1], V[3 * a + 2] + V[3 * b + 2]};
    push_unit(m);
    const int id = (int)V.size() / 3 - 1;
    cache.push_back({key, id});
    return id;
  };
  for (auto& f : faces) {
    const int a = f[0], b = f[1], c = f[2];
    const int ab = mid(a, b), bc = mid(b, c), ca = mid(c, a);
    const int tri[4][3] = {{a, ab, ca}, {b, bc, ab}, {c, ca, bc}, {ab, bc, ca}};
    for (auto& t : tri) F.insert(F.end(), t, t + 3);
  }
}

struct MeshState {
  MeshCounters* d_mc = nullptr;
  MeshCounters* h_mc = nullptr;      // pinned
  int* h_base = nullptr;             // pinned: segment bases after the scan
  double* d_ico = nullptr;
  std::vector<int> ico_f;
  uint8_t* kind = nullptr; size_t kind_cap = 0;
  unsigned* key = nullptr; size_t key_cap = 0;
  float* phiA = nullptr; size_t phiA_cap = 0;
  float* phiB = nullptr; size_t phiB_cap = 0;
  int* vid = nullptr; size_t vid_cap = 0;
  int* bcount = nullptr; size_t bcount_cap = 0;
  double* vtx = nullptr; size_t vtx_cap = 0;
  int4* quads = nullptr; size_t quad_cap = 0;
  int* lone_idx = nullptr; size_t lone_cap = 0;
  int* fill = nullptr; size_t fill_cap = 0;          // per cell, the particles placed in cell order so far
  int* order = nullptr; size_t order_cap = 0;        // in-grid particles in cell order
  float* pos = nullptr; size_t pos_cap = 0;
  float* vel = nullptr; size_t vel_cap = 0;
  MeshInfo info{};
  bool built = false;
  cudaEvent_t ev[2 * kMeshPhases] = {};   // start and end of each phase
};

template <class T>
static void grow(T*& p, size_t& cap, size_t need) {
  if (need <= cap && p) return;
  if (p) CK(cudaFree(p));
  p = nullptr;
  const size_t n = std::max<size_t>(need + need / 4, 1024);
  CK(cudaMalloc((void**)&p, n * sizeof(T)));
  cap = n;
}

void free_mesh(Tank& t) {
  MeshState* m = (MeshState*)t.mesh;
  if (!m) return;
  void* dev[] = {m->d_mc, m->d_ico, m->kind, m->key, m->phiA, m->phiB, m->vid, m->bcount, m->vtx, m->quads,
                 m->lone_idx, m->pos, m->vel, m->fill, m->order};
  for (void* p : dev) if (p) cudaFree(p);
  if (m->h_mc) cudaFreeHost(m->h_mc);
  if (m->h_base) cudaFreeHost(m->h_base);
  for (cudaEvent_t e : m->ev) if (e) cudaEventDestroy(e);
  delete m;
  t.mesh = nullptr;
}

static int nb_of(long long n) {
  const long long tile = (long long)kMeshThreads * kMeshItems;
  return (int)((n + tile - 1) / tile);
}

MeshInfo build_surface_mesh(Tank& t, double smooth) {
  if (!(smooth > 0) || smooth > 6.0) throw Error(-1, "surface mesh: smooth (blur sigma in lattice nodes) in (0, 6]");
  t.count_pass();                    // cell counts of the particles as they are (at a frame end: the frame's)
  t.read_counters();
  const long long n = (long long)t.h_ctr->n_live + t.h_ctr->n_emit;
  if (!t.mesh) {
    MeshState* m = new MeshState();
    t.mesh = m;
    CK(cudaMalloc(&m->d_mc, sizeof(MeshCounters)));
    CK(cudaMallocHost(&m->h_mc, sizeof(MeshCounters)));
    CK(cudaMallocHost(&m->h_base, 4 * sizeof(int)));
    std::vector<double> V;
    icosphere(V, m->ico_f);
    CK(cudaMalloc(&m->d_ico, V.size() * 8));
    CK(cudaMemcpyAsync(m->d_ico, V.data(), V.size() * 8, cudaMemcpyHostToDevice, t.stream));
    CK(cudaStreamSynchronize(t.stream));
    for (cudaEvent_t& e : m->ev) CK(cudaEventCreate(&e));
  }
  MeshState& M = *(MeshState*)t.mesh;
  M.built = false;
  const TankDev& D = t.d;
  const TankDev* dT = t.solo->d_tanks;   // the tank's descriptor on the device (uploaded by count_pass)
  const int grid = t.solo->sm_count * 8;
  grow(M.kind, M.kind_cap, (size_t)std::max<long long>(n, 1));
  MeshCounters init{};
  for (int a = 0; a < 3; ++a) { init.lo_key[a] = ~0u; init.hi_key[a] = 0u; }
  *M.h_mc = init;
  CK(cudaMemcpyAsync(M.d_mc, M.h_mc, sizeof(MeshCounters), cudaMemcpyHostToDevice, t.stream));
  CK(cudaEventRecord(M.ev[0], t.stream));
  if (n > 0) k_mesh_classify<<<grid, 256, 0, t.stream>>>(dT, M.kind, M.d_mc);
  CK(cudaGetLastError());
  CK(cudaEventRecord(M.ev[1], t.stream));
  CK(cudaMemcpyAsync(M.h_mc, M.d_mc, sizeof(MeshCounters), cudaMemcpyDeviceToHost, t.stream));
  CK(cudaStreamSynchronize(t.stream));
  const MeshCounters mc = *M.h_mc;

  MeshInfo info{};
  info.smooth = smooth;
  // blur taps (meshing.py:9-11): radius max(1, ceil(2.5σ)), normalised by their sum taken in order
  MeshTaps taps{};
  const int rad = std::max(1, (int)ceil(2.5 * smooth));
  taps.n = 2 * rad + 1;
  double ksum = 0;
  for (int i = -rad; i <= rad; ++i) { const double x = i / smooth; taps.w[i + rad] = exp(-0.5 * (x * x)); }
  for (int i = 0; i < taps.n; ++i) ksum += taps.w[i];
  for (int i = 0; i < taps.n; ++i) { taps.w[i] = taps.w[i] / ksum; info.weights[i] = taps.w[i]; }
  info.taps = taps.n;

  MeshGeom G{};
  G.sp = D.h / 2;
  G.r = 0.5 * D.h * 1.05;
  G.far_ = 2 * G.sp;
  G.r32 = (float)G.r;
  G.far32 = (float)G.far_;
  if (mc.n_body > 0) {
    // lattice around the body (meshing.py:77-80)
    const double pad = G.r + 4 * G.sp;
    long long dims[3];
    for (int a = 0; a < 3; ++a) {
      auto val = [](unsigned k) {
        const unsigned b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
        float f;
        memcpy(&f, &b, 4);
        return (double)f;
      };
      const double lo = val(mc.lo_key[a]) - pad, hi = val(mc.hi_key[a]) + pad;
      G.lo[a] = lo;
      dims[a] = (long long)ceil((hi - lo) / G.sp) + 1;
    }
    const long long nodes = dims[0] * dims[1] * dims[2];
    if (nodes > (1LL << 31) - 1) throw Error(-1, "surface mesh: lattice too large");
    G.X = (int)dims[0]; G.Y = (int)dims[1]; G.Z = (int)dims[2];
    grow(M.key, M.key_cap, (size_t)nodes);
    grow(M.phiA, M.phiA_cap, (size_t)nodes);
    grow(M.phiB, M.phiB_cap, (size_t)nodes);
    const unsigned far_key = [&] { unsigned b; memcpy(&b, &G.far32, 4); return (b & 0x80000000u) ? ~b : (b | 0x80000000u); }();
    CK(cudaEventRecord(M.ev[2], t.stream));
    k_mesh_fill<<<grid, 256, 0, t.stream>>>(M.key, nodes, far_key);
    // the in-grid particles in cell order, then one block per tile of cells
    grow(M.fill, M.fill_cap, (size_t)D.ncells);
    grow(M.order, M.order_cap, (size_t)std::max<long long>(n, 1));
    CK(cudaMemsetAsync(M.fill, 0, (size_t)D.ncells * sizeof(int), t.stream));
    k_mesh_order<<<grid, 256, 0, t.stream>>>(dT, M.fill, M.order);
    const int tiles = ((D.nx + kTX - 1) / kTX) * ((D.ny + kTY - 1) / kTY) * ((D.nz + kTZ - 1) / kTZ);
    k_mesh_splat_tiles<<<tiles, 256, 0, t.stream>>>(dT, M.order, G, far_key, M.key);
    CK(cudaEventRecord(M.ev[3], t.stream));
    CK(cudaEventRecord(M.ev[4], t.stream));
    k_mesh_blur<0><<<grid, 256, 0, t.stream>>>(M.key, M.phiA, G, taps);
    k_mesh_blur<1><<<grid, 256, 0, t.stream>>>(M.phiA, M.phiB, G, taps);
    k_mesh_blur<2><<<grid, 256, 0, t.stream>>>(M.phiB, M.phiA, G, taps);
    CK(cudaGetLastError());
    CK(cudaEventRecord(M.ev[5], t.stream));
  } else {
    for (int k = 2; k < 6; ++k) CK(cudaEventRecord(M.ev[k], t.stream));
  }
  CK(cudaEventRecord(M.ev[6], t.stream));
  MeshSegs S{};
  if (mc.n_body > 0) {
    const long long X = G.X, Y = G.Y, Z = G.Z;
    S.n[0] = (X - 1) * (Y - 1) * (Z - 1);
    S.n[1] = (X - 1) * Y * Z;
    S.n[2] = X * (Y - 1) * Z;
    S.n[3] = X * Y * (Z - 1);
  }
  S.n[4] = n;
  S.first_block[0] = 0;
  for (int s = 0; s < 5; ++s) S.first_block[s + 1] = S.first_block[s] + nb_of(S.n[s]);
  const int B = S.first_block[5];
  if (B > 0) {
    grow(M.bcount, M.bcount_cap, (size_t)B + 1);
    CK(cudaEventRecord(M.ev[6], t.stream));
    const float* phi = M.phiA;
    k_mesh_count<<<B, kMeshThreads, 0, t.stream>>>(phi, G, S, M.kind, M.bcount);
    k_mesh_scan<<<1, 1024, 0, t.stream>>>(M.bcount, B);
    CK(cudaMemcpyAsync(M.h_base + 0, M.bcount + S.first_block[1], 4, cudaMemcpyDeviceToHost, t.stream));
    CK(cudaMemcpyAsync(M.h_base + 1, M.bcount + S.first_block[4], 4, cudaMemcpyDeviceToHost, t.stream));
    CK(cudaMemcpyAsync(M.h_base + 2, M.bcount + B, 4, cudaMemcpyDeviceToHost, t.stream));
    CK(cudaStreamSynchronize(t.stream));
  } else {
    M.h_base[0] = M.h_base[1] = M.h_base[2] = 0;
  }
  const long long nbv = M.h_base[0], nq = (long long)M.h_base[1] - M.h_base[0], nl = (long long)M.h_base[2] - M.h_base[1];
  const long long nv = nbv + 42 * nl;
  if (nv > (1LL << 31) - 1) throw Error(-1, "surface mesh: too many vertices");
  if (S.n[0] > 0) {
    grow(M.vid, M.vid_cap, (size_t)S.n[0]);
    grow(M.vtx, M.vtx_cap, 3 * (size_t)std::max<long long>(nbv, 1));
    k_mesh_cells<<<nb_of(S.n[0]), kMeshThreads, 0, t.stream>>>(M.phiA, G, S, M.bcount, M.vid, M.vtx);
    grow(M.quads, M.quad_cap, (size_t)std::max<long long>(nq, 1));
    const int qb = S.first_block[4] - S.first_block[1];
    if (qb > 0) k_mesh_quads<<<qb, kMeshThreads, 0, t.stream>>>(M.phiA, G, S, M.bcount, M.vid, M.quads);
  }
  grow(M.lone_idx, M.lone_cap, (size_t)std::max<long long>(nl, 1));
  if (S.n[4] > 0) k_mesh_lone<<<nb_of(S.n[4]), kMeshThreads, 0, t.stream>>>(S, M.kind, M.bcount, M.lone_idx);
  CK(cudaEventRecord(M.ev[7], t.stream));
  grow(M.pos, M.pos_cap, 3 * (size_t)std::max<long long>(nv, 1));
  grow(M.vel, M.vel_cap, 3 * (size_t)std::max<long long>(nv, 1));
  FinishParams F{};
  F.nbody = (int)nbv; F.nverts = (int)nv;
  int W = 0;
  F.top = ripple_top(t, &W);
  F.W = F.top ? W : 0;
  F.x1 = D.ox + D.nx * D.h; F.z1 = D.oz + D.nz * D.h;
  F.rim = D.rim;
  F.size_x = D.nx * D.h; F.size_z = D.nz * D.h;
  F.ico = M.d_ico;
  CK(cudaEventRecord(M.ev[8], t.stream));
  if (nv > 0) k_mesh_finish<<<grid, 256, 0, t.stream>>>(dT, G, F, M.vtx, M.lone_idx, M.pos, M.vel);
  CK(cudaGetLastError());
  CK(cudaEventRecord(M.ev[9], t.stream));
  CK(cudaStreamSynchronize(t.stream));
  for (int k = 0; k < kMeshPhases; ++k) {     // the surface nets phase includes the read of the three counts
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, M.ev[2 * k], M.ev[2 * k + 1]));
    info.phase_ms[k] = ms;
  }
  info.verts = nv; info.quads = nq; info.tris = 80 * nl; info.body_verts = nbv; info.lone = nl;
  info.lattice[0] = G.X; info.lattice[1] = G.Y; info.lattice[2] = G.Z;
  for (int a = 0; a < 3; ++a) info.lo[a] = G.lo[a];
  info.spacing = G.sp;
  M.info = info;
  M.built = true;
  return info;
}

void read_surface_mesh(Tank& t, float* pos, float* vel, int32_t* quads, int32_t* tris, long long max_verts,
                       long long max_quads, long long max_tris) {
  MeshState* m = (MeshState*)t.mesh;
  if (!m || !m->built) throw Error(-1, "surface mesh: build it first");
  const MeshInfo& I = m->info;
  if ((pos && max_verts < I.verts) || (vel && max_verts < I.verts) || (quads && max_quads < I.quads) ||
      (tris && max_tris < I.tris))
    throw Error(-1, "surface mesh: output arrays smaller than the mesh");
  if (pos && I.verts) CK(cudaMemcpyAsync(pos, m->pos, 12 * (size_t)I.verts, cudaMemcpyDeviceToHost, t.stream));
  if (vel && I.verts) CK(cudaMemcpyAsync(vel, m->vel, 12 * (size_t)I.verts, cudaMemcpyDeviceToHost, t.stream));
  if (quads && I.quads) CK(cudaMemcpyAsync(quads, m->quads, 16 * (size_t)I.quads, cudaMemcpyDeviceToHost, t.stream));
  if (tris) {                        // 80 triangles of the icosphere per lone particle, after the body's vertices
    const std::vector<int>& f = m->ico_f;
    for (long long d = 0; d < I.lone; ++d) {
      const long long b = I.body_verts + 42 * d;
      for (int k = 0; k < 240; ++k) tris[240 * d + k] = (int32_t)(b + f[k]);
    }
  }
  CK(cudaStreamSynchronize(t.stream));
}

}  // namespace suiri
