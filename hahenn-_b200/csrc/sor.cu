// Red-black SOR pressure sweep.
//
// Cells are stored split by colour (slot = (i>>1) + hx·row), so a thread's own pressure, right-hand side
// and code load coalesced, and its six neighbours come from the other colour's array (two of them in the
// same slot column, coalesced as well).
//
// Arithmetic is float32 in exactly the order of the reference's NumPy solve
// (blender_addon/suiri_lab/solver.py:494-505):
//   num = C0·p(x-) + C1·p(x+) + C2·p(y-) + C3·p(y+) + C4·p(z-) + C5·p(z+)    (each product rounded, summed left to right)
//   p  += ω·(((num − rhs)·inv) − p),   inv = 1/(C0+…+C5) correctly rounded
// with explicit round-to-nearest intrinsics, so the pressures equal the reference's bit for bit given the
// same operands. Faces on the tank walls and floor have C = 0 (Neumann); the open top has C = 1 with p = 0
// above (Dirichlet); non-liquid cells hold 0 and are not updated (src/js/30-wgsl-sim.js:267-297 is the
// same update as a WGSL `mix`).
//
// Most cells have every face either closed or fully open; their coefficients come from the 6 "open"
// bits of the code and the float fractions are only read for cut cells next to obstacles.
//
// Four launch forms, all giving the same pressures bit for bit (the tuner picks one):
//   k_sor          one colour of every tank per launch (2·iters launches per solve, in the sub-step graph),
//                  with programmatic dependent launch between sweeps; over the listed active cells, the
//                  grid capped at the blocks resident at once (threads loop past it)
//   k_sor_persist  the whole solve in one cooperative launch: all blocks resident, each holding its share of
//                  the active-cell lists and their own pressures in shared memory for the whole solve, a
//                  grid barrier after every colour sweep. The barrier's wait is bounded: after the
//                  watchdog's polls it records an error in the tank counters and every block returns.
//   k_sor_tbl      two sweeps per launch over per-tile lists of active cells (temporal blocking)
//   k_sor_tb<4>    four sweeps per launch on shared-memory tiles with halos
#include <type_traits>

#include "launch.cuh"

namespace suiri {

// p + ω·(((num − rhs)·inv) − p) with the reference's rounding steps (see the file comment)
__device__ __forceinline__ float sor_update(const float C[6], const float nb[6], float rhs, float p, float omega) {
  float num = __fmul_rn(C[0], nb[0]);
  float den = C[0];
#pragma unroll
  for (int d = 1; d < 6; ++d) {
    num = __fadd_rn(num, __fmul_rn(C[d], nb[d]));
    den = __fadd_rn(den, C[d]);
  }
  const float inv = __frcp_rn(den);
  float r = __fsub_rn(num, rhs);
  r = __fmul_rn(r, inv);
  r = __fsub_rn(r, p);
  r = __fmul_rn(r, omega);
  return __fadd_rn(p, r);
}

// the same update with inv = 1/(C0+…+C5) given (computed in that order and correctly rounded by the caller)
__device__ __forceinline__ float sor_update_inv(const float C[6], const float nb[6], float rhs, float p, float omega,
                                                float inv) {
  float num = __fmul_rn(C[0], nb[0]);
#pragma unroll
  for (int d = 1; d < 6; ++d) num = __fadd_rn(num, __fmul_rn(C[d], nb[d]));
  float r = __fsub_rn(num, rhs);
  r = __fmul_rn(r, inv);
  r = __fsub_rn(r, p);
  r = __fmul_rn(r, omega);
  return __fadd_rn(p, r);
}

// 1/(C0+…+C5) as sor_update forms it: for a cell without cut faces the coefficients are 0 or 1, their float
// sum is the number of open faces exactly, and its correctly rounded reciprocal comes from a table
__device__ __forceinline__ float coeff_inv(bool cut, unsigned open6, const float C[6]) {
  if (cut) {
    float den = C[0];
#pragma unroll
    for (int d = 1; d < 6; ++d) den = __fadd_rn(den, C[d]);
    return __frcp_rn(den);
  }
  const int n = __popc(open6 & 0x3Fu);
  return n == 1 ? 1.f : n == 2 ? 0.5f : n == 3 ? 0x1.555556p-2f : n == 4 ? 0.25f : n == 5 ? 0x1.99999ap-3f
       : n == 6 ? 0x1.555556p-3f : __frcp_rn(0.f);
}

// The update of a cell without cut faces, whose coefficients are 0 or 1 (the open bits): each product C·p_nb
// is p_nb or a zero, so num is the sum of the open neighbours taken in the same order, with zeros where a face
// is closed. It equals sor_update's bit for bit: the products are exact, and a zero product of the reference
// can differ only in its sign, which no sum of these values carries to the result (no pressure is -0: the
// solve starts from +0 or a previous result, and a round-to-nearest sum is -0 only if both terms are).
__device__ __forceinline__ float sor_update_open(uint32_t open6, const float nb[6], float rhs, float p, float omega,
                                                 float inv) {
  float num = (open6 & 1u) ? nb[0] : 0.f;
#pragma unroll
  for (int d = 1; d < 6; ++d) num = __fadd_rn(num, (open6 >> d) & 1u ? nb[d] : 0.f);
  float r = __fsub_rn(num, rhs);
  r = __fmul_rn(r, inv);
  r = __fsub_rn(r, p);
  r = __fmul_rn(r, omega);
  return __fadd_rn(p, r);
}

// the six face coefficients of a cut cell: its own x, y, z face fractions and those of the +x, +y, +z
// neighbours' faces
__device__ __forceinline__ void cut_coeffs(const TankDev& T, int i, int j, int k, float C[6]) {
  const int n = node_idx(T, i, j, k);
  const float4 f0 = T.frac[n];
  C[0] = f0.x; C[1] = T.frac[n + 1].x; C[2] = f0.y; C[3] = T.frac[n + T.sx].y; C[4] = f0.z; C[5] = T.frac[n + T.sxy].z;
}

__device__ __forceinline__ void sor_cell(const TankDev& T, int color, int s) {
  const int hx = T.hx, nx = T.nx, ny = T.ny, nz = T.nz;
  const int row = divu(s, T.dhx), ti = s - row * hx;
  const int k = divu(row, T.dny), j = row - k * ny;
  const int i = 2 * ti + ((j + k + color) & 1);
  if (i >= nx) return;
  const size_t own = (size_t)color * T.nhalf + s;
  const uint32_t code = T.code[own];
  if (!(code & kCodeActive)) return;
  const float* __restrict__ po = T.pres + (size_t)(1 - color) * T.nhalf;
  const float rhs = T.rhs[own];
  const float p = T.pres[own];
  const int rowb = hx * row;
  float nb[6];
  nb[0] = i > 0 ? po[((i - 1) >> 1) + rowb] : 0.f;
  nb[1] = i + 1 < nx ? po[((i + 1) >> 1) + rowb] : 0.f;
  nb[2] = j > 0 ? po[ti + rowb - hx] : 0.f;
  nb[3] = j + 1 < ny ? po[ti + rowb + hx] : 0.f;
  nb[4] = k > 0 ? po[ti + rowb - hx * ny] : 0.f;
  nb[5] = k + 1 < nz ? po[ti + rowb + hx * ny] : 0.f;
  float C[6];
  if (code & kCodePartial) {
    cut_coeffs(T, i, j, k, C);
  } else {
#pragma unroll
    for (int d = 0; d < 6; ++d) C[d] = (code >> d) & 1u ? 1.0f : 0.0f;
  }
  T.pres[own] = sor_update(C, nb, rhs, p, T.omega);
}

// relax the listed cell of entry e (slot, code, rhs, 1/ΣC): its pressure and six neighbours in one round of
// loads (cut cells also read their face fractions)
__device__ __forceinline__ void sor_entry(const TankDev& T, int color, int4 e) {
  const int hx = T.hx, nx = T.nx, ny = T.ny, nz = T.nz;
  const int s = e.x;
  const uint32_t code = (uint32_t)e.y;
  const int row = divu(s, T.dhx), ti = s - row * hx;
  const int k = divu(row, T.dny), j = row - k * ny;
  const int i = 2 * ti + ((j + k + color) & 1);
  const float* __restrict__ po = T.pres + (size_t)(1 - color) * T.nhalf;
  const int rowb = hx * row;
  float nb[6];
  nb[0] = i > 0 ? po[((i - 1) >> 1) + rowb] : 0.f;
  nb[1] = i + 1 < nx ? po[((i + 1) >> 1) + rowb] : 0.f;
  nb[2] = j > 0 ? po[ti + rowb - hx] : 0.f;
  nb[3] = j + 1 < ny ? po[ti + rowb + hx] : 0.f;
  nb[4] = k > 0 ? po[ti + rowb - hx * ny] : 0.f;
  nb[5] = k + 1 < nz ? po[ti + rowb + hx * ny] : 0.f;
  const size_t own = (size_t)color * T.nhalf + s;
  const float p = T.pres[own];
  const float rhs = __int_as_float(e.z), inv = __int_as_float(e.w);
  if (code & kCodePartial) {
    float C[6];
    cut_coeffs(T, i, j, k, C);
    T.pres[own] = sor_update_inv(C, nb, rhs, p, T.omega, inv);
  } else {
    T.pres[own] = sor_update_open(code, nb, rhs, p, T.omega, inv);
  }
}

// Launched with programmatic stream serialisation (all but the first sweep of a solve): the next sweep's
// blocks may start as soon as every block of this one has started. Before griddepcontrol.wait a block
// reads only what no sweep writes (its tank descriptor, the cell's code, rhs and cut-cell fractions, all
// written by kernels that completed before the first sweep, which is launched without the attribute), so
// that part overlaps the previous sweep; after the wait, which returns once the previous sweep has
// completed and its writes are visible, it reads the pressures, one round of loads, and writes its own.
template <bool kLoop>
__global__ void __launch_bounds__(kSorThreads) k_sor(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ apfx,
                                                     int color, int sweep) {
  // thread q relaxes the q-th active cell of this colour over all tanks (the cell pass listed them);
  // blocks past the active cells leave at once, so the blocks of consecutive sweeps fit on the GPU together.
  // kLoop: the grid is capped at what is resident at once and thread q also takes cells q + G, q + 2G, …
  // (G = the grid's threads), after the wait.
  const int* __restrict__ pfx = apfx + color * (ntanks + 1);
  const int q = blockIdx.x * kSorThreads + threadIdx.x;
  if ((int)(blockIdx.x * kSorThreads) >= pfx[ntanks]) return;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const bool live = q < pfx[ntanks];
  const int t = find_slot(pfx, ntanks, live ? q : 0);
  const TankDev& T = tanks[t];
  const int hx = T.hx, nx = T.nx, ny = T.ny, nz = T.nz, nhalf = T.nhalf;
  const bool on = live && sweep < T.iters;
  float* const pres = T.pres;
  const float omega = T.omega;
  // the cell's list entry carries its slot, code, rhs and 1/ΣC (written by the cell pass)
  int4 e = make_int4(0, 0, 0, 0);
  if (on) e = T.act[(size_t)color * nhalf + (q - pfx[t])];
  const int s = e.x;
  const uint32_t code = (uint32_t)e.y;
  const float rhs = __int_as_float(e.z), inv = __int_as_float(e.w);
  const int row = divu(s, T.dhx), ti = s - row * hx;
  const int k = divu(row, T.dny), j = row - k * ny;
  const int i = 2 * ti + ((j + k + color) & 1);
  float C[6];
  if (code & kCodePartial) cut_coeffs(T, i, j, k, C);
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (on) {
    const float* __restrict__ po = pres + (size_t)(1 - color) * nhalf;
    const int rowb = hx * row;
    float nb[6];
    nb[0] = i > 0 ? po[((i - 1) >> 1) + rowb] : 0.f;
    nb[1] = i + 1 < nx ? po[((i + 1) >> 1) + rowb] : 0.f;
    nb[2] = j > 0 ? po[ti + rowb - hx] : 0.f;
    nb[3] = j + 1 < ny ? po[ti + rowb + hx] : 0.f;
    nb[4] = k > 0 ? po[ti + rowb - hx * ny] : 0.f;
    nb[5] = k + 1 < nz ? po[ti + rowb + hx * ny] : 0.f;
    const float p = pres[(size_t)color * nhalf + s];
    pres[(size_t)color * nhalf + s] = (code & kCodePartial) ? sor_update_inv(C, nb, rhs, p, omega, inv)
                                                            : sor_update_open(code, nb, rhs, p, omega, inv);
  }
  if (kLoop) {
    for (int r = q + (int)gridDim.x * kSorThreads; r < pfx[ntanks]; r += (int)gridDim.x * kSorThreads) {
      const int t2 = find_slot(pfx, ntanks, r);
      const TankDev& T2 = tanks[t2];
      if (sweep < T2.iters) sor_entry(T2, color, T2.act[(size_t)color * T2.nhalf + (r - pfx[t2])]);
    }
  }
}

// Barrier over all blocks of a cooperative launch on a count that only grows: block arrivals add 1, and the
// n-th barrier of the solve (from 1) is passed once the count reaches n·blocks (the count is cleared before
// the launch). The wait is bounded: after `limit` polls, or once another block has given up, it records the
// failure and returns false.
__device__ __forceinline__ bool grid_barrier(GridBarrier* b, unsigned target, unsigned limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    atomicAdd(&b->count, 1u);
    unsigned spins = 0;
    for (;;) {
      unsigned c;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(c) : "l"(&b->count) : "memory");
      if (c >= target) break;
      if (++spins > limit || *(volatile int*)&b->err) { ok = 0; break; }
    }
    __threadfence();
    if (!ok) atomicExch(&b->err, 1);
    s_ok = ok;
  }
  __syncthreads();
  return s_ok;
}

// The whole solve in one cooperative launch. Block b owns a fixed share of each colour's active-cell list
// (entries [b·N/G, (b+1)·N/G) of the lists over all tanks) and keeps as many of its entries as fit in shared
// memory for the whole solve, with the tank in the code's upper bits and the cell's own pressure beside it:
// its own pressures are written only by this block, so they are read from shared memory, and written to
// global memory for the neighbours. A sweep then reads from global memory only the six neighbour pressures
// of each cell (through L2: other SMs wrote them), and a grid barrier separates the sweeps. Entries beyond
// the shared-memory share are read from the lists each sweep. Same updates as the per-sweep launches, in the
// same colour order, so the same pressures bit for bit.
constexpr int kResThreads = 1024;
constexpr int kResEntryBytes = 20;      // int4 entry + the cell's own pressure
__global__ void __launch_bounds__(kResThreads, 1) k_sor_persist(const TankDev* __restrict__ tanks, int ntanks,
                                                                const int* __restrict__ apfx, int max_iters,
                                                                GridBarrier* bar, unsigned limit, int cap) {
  extern __shared__ int4 s_ent[];
  float* s_p = reinterpret_cast<float*>(s_ent + cap);
  const int G = gridDim.x, b = blockIdx.x;
  int r0[2], n[2], cached[2], base[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const long long N = apfx[c * (ntanks + 1) + ntanks];
    r0[c] = (int)(N * b / G);
    n[c] = (int)(N * (b + 1) / G) - r0[c];
  }
  // the shared share of each colour, in proportion to its entries
  const int tot = n[0] + n[1];
  cached[0] = tot <= cap ? n[0] : (int)((long long)cap * n[0] / max(tot, 1));
  cached[1] = min(n[1], cap - cached[0]);
  base[0] = 0; base[1] = cached[0];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const int* __restrict__ pfx = apfx + c * (ntanks + 1);
    for (int e = threadIdx.x; e < cached[c]; e += kResThreads) {
      const int q = r0[c] + e;
      const int t = find_slot(pfx, ntanks, q);
      const TankDev& T = tanks[t];
      int4 ent = T.act[(size_t)c * T.nhalf + (q - pfx[t])];
      s_p[base[c] + e] = T.pres[(size_t)c * T.nhalf + ent.x];
      ent.y = (ent.y & 0xFFFF) | (t << 16);
      s_ent[base[c] + e] = ent;
    }
  }
  __syncthreads();
  for (int sweep = 0; sweep < 2 * max_iters; ++sweep) {
    const int c = sweep & 1, it = sweep >> 1;
    const int* __restrict__ pfx = apfx + c * (ntanks + 1);
    for (int e = threadIdx.x; e < n[c]; e += kResThreads) {
      int4 ent;
      int t;
      const bool in_smem = e < cached[c];
      if (in_smem) {
        ent = s_ent[base[c] + e];
        t = ent.y >> 16;
      } else {
        const int q = r0[c] + e;
        t = find_slot(pfx, ntanks, q);
        ent = tanks[t].act[(size_t)c * tanks[t].nhalf + (q - pfx[t])];
      }
      const TankDev& T = tanks[t];
      if (it >= T.iters) continue;
      const int hx = T.hx, nx = T.nx, ny = T.ny, nz = T.nz;
      const int s = ent.x;
      const uint32_t code = (uint32_t)ent.y & 0xFFFFu;
      const int row = divu(s, T.dhx), ti = s - row * hx;
      const int k = divu(row, T.dny), j = row - k * ny;
      const int i = 2 * ti + ((j + k + c) & 1);
      const float* __restrict__ po = T.pres + (size_t)(1 - c) * T.nhalf;
      const int rowb = hx * row;
      float nb[6];
      nb[0] = i > 0 ? __ldcg(po + ((i - 1) >> 1) + rowb) : 0.f;
      nb[1] = i + 1 < nx ? __ldcg(po + ((i + 1) >> 1) + rowb) : 0.f;
      nb[2] = j > 0 ? __ldcg(po + ti + rowb - hx) : 0.f;
      nb[3] = j + 1 < ny ? __ldcg(po + ti + rowb + hx) : 0.f;
      nb[4] = k > 0 ? __ldcg(po + ti + rowb - hx * ny) : 0.f;
      nb[5] = k + 1 < nz ? __ldcg(po + ti + rowb + hx * ny) : 0.f;
      const size_t own = (size_t)c * T.nhalf + s;
      const float p = in_smem ? s_p[base[c] + e] : __ldcg(T.pres + own);
      const float rhs = __int_as_float(ent.z), inv = __int_as_float(ent.w);
      float np;
      if (code & kCodePartial) {
        float C[6];
        cut_coeffs(T, i, j, k, C);
        np = sor_update_inv(C, nb, rhs, p, T.omega, inv);
      } else {
        np = sor_update_open(code, nb, rhs, p, T.omega, inv);
      }
      __stcg(T.pres + own, np);
      if (in_smem) s_p[base[c] + e] = np;
    }
    if (sweep + 1 < 2 * max_iters && !grid_barrier(bar, (unsigned)G * (unsigned)(sweep + 1), limit)) {
      if (threadIdx.x == 0)
        for (int t = 0; t < ntanks; ++t) atomicOr(&tanks[t].ctr->err, kErrBarrier);
      return;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Temporal blocking: S colour sweeps per launch (S = 2 or 4). A block owns a kTbX×kTbY×kTbZ tile of cells and
// stages the tile plus a halo of S cells (clipped at the tank walls) in shared memory: pressure, rhs and a
// 16-bit code per cell, split by colour like the global arrays. Sweep s (0-based, n sweeps in the launch)
// updates the cells of its colour within n−1−s cells of the tile: a red-black sweep reads only the other
// colour, so a cell updated there sees exactly the neighbour values the per-sweep launches would give it,
// and after the n sweeps the tile itself holds exactly the per-sweep result. The tile is written to the
// other pressure buffer (halos are read from the input buffer by neighbouring blocks while this one
// writes), so launches alternate between pres and pres2.
//
// Like k_sor, a block reads what the solve never writes (code, rhs, cut-cell fractions) before
// griddepcontrol.wait, overlapping the previous launch, and the pressures after it, one batch of loads.
// Cut cells keep their six coefficients in a shared table (kTbCut entries; beyond that they are read from
// the face fractions in global memory). The smem code: 0 inactive; 0x4000|open bits for a cell whose faces
// are all closed or fully open; 0x8000|table index for a cut cell (0x7FFF: not in the table).
constexpr int kTbCut = 512;
template <int S>
struct TbShape {
  static constexpr int RX = kTbX + 2 * S, RY = kTbY + 2 * S, RZ = kTbZ + 2 * S;
  static constexpr int HX = RX / 2;
  static constexpr int SLOTS = HX * RY * RZ;                              // per colour
  static constexpr int PER = (2 * SLOTS + kTbThreads - 1) / kTbThreads;    // region slots per thread
  static constexpr int SMEM = 2 * SLOTS * 4 * 2 + 2 * SLOTS * 2 + kTbCut * 6 * 4;
  static_assert(kTbX % 2 == 0 && S % 2 == 0, "tile and halo keep the region's x origin even");
  static_assert(SLOTS < 0x7FFF, "table index fits the code");
};

template <int S>
__global__ void __launch_bounds__(kTbThreads, 2) k_sor_tb(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx,
                                                          int sweep0, int nsweeps, int dir) {
  using G = TbShape<S>;
  extern __shared__ __align__(16) unsigned char tb_smem[];
  float* sp = reinterpret_cast<float*>(tb_smem);               // [2][SLOTS] pressure
  float* srhs = sp + 2 * G::SLOTS;                             // [2][SLOTS]
  uint16_t* scode = reinterpret_cast<uint16_t*>(srhs + 2 * G::SLOTS);
  float* stab = reinterpret_cast<float*>(scode + 2 * G::SLOTS);  // [kTbCut][6]
  __shared__ int s_ncut;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int nx = T.nx, ny = T.ny, nz = T.nz, hx = T.hx;
  const size_t nh = T.nhalf;
  const int lb = blockIdx.x - bpfx[t];
  const int tnx = (nx + kTbX - 1) / kTbX, tny = (ny + kTbY - 1) / kTbY;
  const int x0 = (lb % tnx) * kTbX, y0 = ((lb / tnx) % tny) * kTbY, z0 = (lb / (tnx * tny)) * kTbZ;
  const int rx0 = max(x0 - S, 0), ry0 = max(y0 - S, 0), rz0 = max(z0 - S, 0);
  const int rx1 = min(x0 + kTbX + S, nx), ry1 = min(y0 + kTbY + S, ny), rz1 = min(z0 + kTbZ + S, nz);
  const float* __restrict__ pin = dir ? T.pres2 : T.pres;
  float* __restrict__ pout = dir ? T.pres : T.pres2;
  const int iters = T.iters;
  const float omega = T.omega;
  // region slot q (colour q >= SLOTS) → global index within its colour, or −1 outside the tank
  auto region = [&](int q, int& i, int& j, int& k) -> int {
    const int c = q >= G::SLOTS;
    const int ls = q - c * G::SLOTS;
    const int lti = ls % G::HX, lrow = ls / G::HX;
    j = ry0 + lrow % G::RY;
    k = rz0 + lrow / G::RY;
    i = rx0 + 2 * lti + ((j + k + c) & 1);
    return (i < rx1 && j < ry1 && k < rz1) ? (i >> 1) + hx * (j + ny * k) : -1;
  };
  if (threadIdx.x == 0) s_ncut = 0;
  __syncthreads();
  // constant operands, in chunks of loads issued together
  constexpr int CH = 6;
#pragma unroll
  for (int u0 = 0; u0 < G::PER; u0 += CH) {
    uint32_t cd[CH];
    float rh[CH];
#pragma unroll
    for (int v = 0; v < CH; ++v) {
      const int q = threadIdx.x + (u0 + v) * kTbThreads;
      cd[v] = 0; rh[v] = 0.f;
      if (u0 + v < G::PER && q < 2 * G::SLOTS) {
        int i, j, k;
        const int g = region(q, i, j, k);
        if (g >= 0) {
          const size_t gg = (q >= G::SLOTS ? nh : 0) + g;
          cd[v] = T.code[gg];
          rh[v] = T.rhs[gg];
        }
      }
    }
#pragma unroll
    for (int v = 0; v < CH; ++v) {
      const int q = threadIdx.x + (u0 + v) * kTbThreads;
      if (u0 + v >= G::PER || q >= 2 * G::SLOTS) continue;
      uint16_t code16 = 0;
      float r = 0.f;
      if (cd[v] & kCodeActive) {
        r = rh[v];
        if (cd[v] & kCodePartial) {
          const int e = atomicAdd(&s_ncut, 1);
          if (e < kTbCut) {
            int i, j, k;
            region(q, i, j, k);
            float C[6];
            cut_coeffs(T, i, j, k, C);
#pragma unroll
            for (int d = 0; d < 6; ++d) stab[6 * e + d] = C[d];
            code16 = (uint16_t)(0x8000 | e);
          } else {
            code16 = 0xFFFF;
          }
        } else {
          code16 = (uint16_t)(0x4000 | (cd[v] & 0x3F));
        }
      }
      srhs[q] = r;
      scode[q] = code16;
    }
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // pressures: every load of the thread in flight at once
  {
    float pv[G::PER];
#pragma unroll
    for (int u = 0; u < G::PER; ++u) {
      const int q = threadIdx.x + u * kTbThreads;
      pv[u] = 0.f;
      if (q < 2 * G::SLOTS) {
        int i, j, k;
        const int g = region(q, i, j, k);
        if (g >= 0) pv[u] = pin[(q >= G::SLOTS ? nh : 0) + g];
      }
    }
#pragma unroll
    for (int u = 0; u < G::PER; ++u) {
      const int q = threadIdx.x + u * kTbThreads;
      if (q < 2 * G::SLOTS) sp[q] = pv[u];
    }
  }
  __syncthreads();
  for (int s = 0; s < nsweeps; ++s) {
    const int sw = sweep0 + s;
    if (sw < 2 * iters) {
      const int c = sw & 1, e = nsweeps - 1 - s;
      const int bx0 = max(x0 - e, rx0), bx1 = min(x0 + kTbX + e, rx1);
      const int by0 = max(y0 - e, ry0), by1 = min(y0 + kTbY + e, ry1);
      const int bz0 = max(z0 - e, rz0), bz1 = min(z0 + kTbZ + e, rz1);
      const float* so = sp + (1 - c) * G::SLOTS;
      for (int ls = threadIdx.x; ls < G::SLOTS; ls += kTbThreads) {
        const int lti = ls % G::HX, lrow = ls / G::HX;
        const int lj = lrow % G::RY, lk = lrow / G::RY;
        const int j = ry0 + lj, k = rz0 + lk;
        const int i = rx0 + 2 * lti + ((j + k + c) & 1);
        if (i < bx0 || i >= bx1 || j < by0 || j >= by1 || k < bz0 || k >= bz1) continue;
        const int own = c * G::SLOTS + ls;
        const unsigned cd = scode[own];
        if (!cd) continue;
        const int rowb = ls - lti;       // G::HX · (lj + G::RY · lk)
        const int li = i - rx0;
        float nb[6];
        nb[0] = i > 0 ? so[((li - 1) >> 1) + rowb] : 0.f;
        nb[1] = i + 1 < nx ? so[((li + 1) >> 1) + rowb] : 0.f;
        nb[2] = j > 0 ? so[lti + rowb - G::HX] : 0.f;
        nb[3] = j + 1 < ny ? so[lti + rowb + G::HX] : 0.f;
        nb[4] = k > 0 ? so[lti + rowb - G::HX * G::RY] : 0.f;
        nb[5] = k + 1 < nz ? so[lti + rowb + G::HX * G::RY] : 0.f;
        float C[6];
        if (cd & 0x8000) {
          const unsigned x = cd & 0x7FFF;
          if (x < kTbCut) {
#pragma unroll
            for (int d = 0; d < 6; ++d) C[d] = stab[6 * x + d];
          } else {
            cut_coeffs(T, i, j, k, C);
          }
        } else {
#pragma unroll
          for (int d = 0; d < 6; ++d) C[d] = (cd >> d) & 1u ? 1.0f : 0.0f;
        }
        sp[own] = sor_update(C, nb, srhs[own], sp[own], omega);
      }
    }
    __syncthreads();
  }
  constexpr int kTileSlots = (kTbX / 2) * kTbY * kTbZ;
  for (int q = threadIdx.x; q < 2 * kTileSlots; q += kTbThreads) {
    const int c = q >= kTileSlots;
    const int r = q - c * kTileSlots;
    const int mi = r % (kTbX / 2), rr = r / (kTbX / 2);
    const int j = y0 + rr % kTbY, k = z0 + rr / kTbY;
    const int i = x0 + 2 * mi + ((j + k + c) & 1);
    if (i >= nx || j >= ny || k >= nz) continue;
    const int ls = c * G::SLOTS + ((i - rx0) >> 1) + G::HX * ((j - ry0) + G::RY * (k - rz0));
    pout[c * nh + (size_t)(i >> 1) + (size_t)hx * (j + (size_t)ny * k)] = sp[ls];
  }
}

// ---------------------------------------------------------------------------- two sweeps per launch, listed
// A launch relaxes colour 0 then colour 1 (one iteration) on 16×16×8 tiles. The first sweep relaxes the
// active colour-0 cells of the tile and of its face ring (the cells one step outside a face: the colour-0
// neighbours of the tile's cells); ring cells are relaxed by each tile that needs them, from the same
// operands as by their own tile, so the values agree. The second sweep relaxes the tile's active colour-1
// cells with those neighbours from shared memory. Before griddepcontrol.wait a block only reads constant
// data: the tile's lists, built once per sub-step by k_tbl_lists. After it, each thread issues the
// global loads of its (at most 3) colour-0 cells together, as a per-sweep launch does for its one cell,
// so a launch costs about one per-sweep launch for two sweeps. Pressures ping-pong between pres and pres2
// (a neighbouring tile may still read the values this block replaces); inactive cells are constant over
// the solve and k_tbl_lists makes the two buffers agree on them.
//
// List entry (uint2): x = box coordinates (bits 0-4, 5-9, 10-13: i − x0 + 1, j − y0 + 1, k − z0 + 1), open
// bits (14-19), cut cell (20), inside the tile (21); y = rhs bits. In shared memory bits 22-30 carry the
// cut-table index (kTblCut: not held, read from the face fractions).
constexpr int kTblBX = kTbX + 2, kTblBY = kTbY + 2, kTblBZ = kTbZ + 2;
constexpr int kTblBox = kTblBX * kTblBY * kTblBZ;
constexpr int kTblCapA = kTbX * kTbY * kTbZ / 2 + kTbY * kTbZ + kTbX * kTbZ + kTbX * kTbY;   // colour 0: tile + face ring
constexpr int kTblCapB = kTbX * kTbY * kTbZ / 2;                                           // colour 1: tile
constexpr int kTblThreads = 512;
constexpr int kTblCut = 256;
constexpr int kTblPerA = (kTblCapA + kTblThreads - 1) / kTblThreads;
constexpr int kTblPerB = (kTblCapB + kTblThreads - 1) / kTblThreads;
static_assert(kTblBX <= 32 && kTblBY <= 32 && kTblBZ <= 16, "box coordinates fit their bits");

struct TblSmem {
  float box[kTblBox];          // colour-0 values of the box: sweep-1 results, constants of inactive cells
  int sa[kTblCapA];            // global slots (colour 1: + nhalf)
  int sb[kTblCapB];
  uint2 ea[kTblCapA];          // entries as listed, cut-table index added
  uint2 eb[kTblCapB];
  float cut[kTblCut * 6];
  int ncut;
};

__device__ __forceinline__ void tbl_cell(uint32_t m, int x0, int y0, int z0, int& bidx, int& i, int& j, int& k) {
  const int bi = m & 31, bj = (m >> 5) & 31, bk = (m >> 10) & 15;
  bidx = bi + kTblBX * (bj + kTblBY * bk);
  i = x0 - 1 + bi;
  j = y0 - 1 + bj;
  k = z0 - 1 + bk;
}

__device__ __forceinline__ void tbl_coeffs(const TankDev& T, uint32_t m, const float* cut, int i, int j, int k, float C[6]) {
  if (m & (1u << 20)) {
    const unsigned x = (m >> 22) & 0x1FF;
    if (x < kTblCut) {
#pragma unroll
      for (int d = 0; d < 6; ++d) C[d] = cut[6 * x + d];
    } else {
      cut_coeffs(T, i, j, k, C);
    }
  } else {
#pragma unroll
    for (int d = 0; d < 6; ++d) C[d] = (m >> (14 + d)) & 1u ? 1.0f : 0.0f;
  }
}

__device__ __forceinline__ void tbl_tile(const TankDev& T, int lt, int& x0, int& y0, int& z0) {
  const int tnx = (T.nx + kTbX - 1) / kTbX, tny = (T.ny + kTbY - 1) / kTbY;
  x0 = (lt % tnx) * kTbX;
  y0 = ((lt / tnx) % tny) * kTbY;
  z0 = (lt / (tnx * tny)) * kTbZ;
}

// Once per sub-step, before the solve: per tile, the lists of active cells (A: colour 0 in the tile and its
// face ring; B: colour 1 in the tile), the colour-0 cells of the box whose constant pressure is not +0 (C),
// and pres2 = pres on the tile's inactive cells.
__global__ void __launch_bounds__(kThreads) k_tbl_lists(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx,
                                                        uint2* __restrict__ list, int* __restrict__ cnt, int2* __restrict__ clist) {
  __shared__ int s_na, s_nb, s_nc;
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int nx = T.nx, ny = T.ny, nz = T.nz, hx = T.hx;
  const size_t nh = T.nhalf;
  int x0, y0, z0;
  tbl_tile(T, blockIdx.x - bpfx[t], x0, y0, z0);
  if (threadIdx.x == 0) { s_na = 0; s_nb = 0; s_nc = 0; }
  __syncthreads();
  uint2* la = list + (size_t)blockIdx.x * (kTblCapA + kTblCapB);
  uint2* lb = la + kTblCapA;
  int2* lc = clist + (size_t)blockIdx.x * kTblCapA;
  for (int b = threadIdx.x; b < kTblBox; b += blockDim.x) {
    const int bi = b % kTblBX, bj = (b / kTblBX) % kTblBY, bk = b / (kTblBX * kTblBY);
    const int i = x0 - 1 + bi, j = y0 - 1 + bj, k = z0 - 1 + bk;
    if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) continue;
    const int nout = (bi == 0 || bi == kTblBX - 1) + (bj == 0 || bj == kTblBY - 1) + (bk == 0 || bk == kTblBZ - 1);
    const int col = (i + j + k) & 1;
    if (nout > 1 || (col == 1 && nout == 1)) continue;        // no neighbour of a tile cell in the other colour
    const size_t s = (size_t)col * nh + (i >> 1) + (size_t)hx * (j + (size_t)ny * k);
    const uint32_t code = T.code[s];
    if (code & kCodeActive) {
      const uint32_t m = (uint32_t)(bi | (bj << 5) | (bk << 10)) | ((code & 0x3Fu) << 14) |
                         ((code & kCodePartial) ? 1u << 20 : 0u) | (nout == 0 ? 1u << 21 : 0u);
      const uint2 e = make_uint2(m, __float_as_uint(T.rhs[s]));
      if (col == 0) la[atomicAdd(&s_na, 1)] = e;
      else lb[atomicAdd(&s_nb, 1)] = e;
    } else {
      const float p = T.pres[s];
      if (col == 0 && __float_as_uint(p) != 0u) lc[atomicAdd(&s_nc, 1)] = make_int2(b, __float_as_int(p));
      if (nout == 0) T.pres2[s] = p;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cnt[3 * blockIdx.x] = s_na;
    cnt[3 * blockIdx.x + 1] = s_nb;
    cnt[3 * blockIdx.x + 2] = s_nc;
  }
}

__global__ void __launch_bounds__(kTblThreads, 2) k_sor_tbl(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx,
                                                           const uint2* __restrict__ list, const int* __restrict__ cnt,
                                                           const int2* __restrict__ clist, int sweep0, int dir) {
  extern __shared__ __align__(16) unsigned char tbl_smem[];
  TblSmem& S = *reinterpret_cast<TblSmem*>(tbl_smem);
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int na = cnt[3 * blockIdx.x], nb = cnt[3 * blockIdx.x + 1], nc = cnt[3 * blockIdx.x + 2];
  if (na + nb == 0) return;                  // no active cell: nothing to relax or carry
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int nx = T.nx, ny = T.ny, nz = T.nz, hx = T.hx;
  const int nh = T.nhalf;
  int x0, y0, z0;
  tbl_tile(T, blockIdx.x - bpfx[t], x0, y0, z0);
  const bool on = sweep0 < 2 * T.iters;    // a batch runs to its largest count; the others are carried
  const float omega = T.omega;
  const uint2* __restrict__ la = list + (size_t)blockIdx.x * (kTblCapA + kTblCapB);
  const uint2* __restrict__ lb = la + kTblCapA;
  const int2* __restrict__ lc = clist + (size_t)blockIdx.x * kTblCapA;
  for (int b = threadIdx.x; b < kTblBox; b += kTblThreads) S.box[b] = 0.f;
  if (threadIdx.x == 0) S.ncut = 0;
  __syncthreads();
  for (int e = threadIdx.x; e < nc; e += kTblThreads) {
    const int2 v = lc[e];
    S.box[v.x] = __int_as_float(v.y);
  }
  // the lists into shared memory: all of a thread's loads first
  {
    uint2 ea[kTblPerA], eb[kTblPerB];
#pragma unroll
    for (int u = 0; u < kTblPerA; ++u) {
      const int e = threadIdx.x + u * kTblThreads;
      ea[u] = e < na ? la[e] : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int u = 0; u < kTblPerB; ++u) {
      const int e = threadIdx.x + u * kTblThreads;
      eb[u] = e < nb ? lb[e] : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int u = 0; u < kTblPerA + kTblPerB; ++u) {
      const bool isa = u < kTblPerA;
      const int e = threadIdx.x + (isa ? u : u - kTblPerA) * kTblThreads;
      if (e >= (isa ? na : nb)) continue;
      uint2 en = isa ? ea[u] : eb[u - kTblPerA];
      int bidx, i, j, k;
      tbl_cell(en.x, x0, y0, z0, bidx, i, j, k);
      if (en.x & (1u << 20)) {
        const int x = atomicAdd(&S.ncut, 1);
        if (x < kTblCut) {
          float C[6];
          cut_coeffs(T, i, j, k, C);
#pragma unroll
          for (int d = 0; d < 6; ++d) S.cut[6 * x + d] = C[d];
        }
        en.x |= (uint32_t)min(x, kTblCut) << 22;
      }
      const int s = (isa ? 0 : nh) + (i >> 1) + hx * (j + ny * k);
      if (isa) { S.sa[e] = s; S.ea[e] = en; }
      else { S.sb[e] = s; S.eb[e] = en; }
    }
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  __syncthreads();
  const float* __restrict__ pin = dir ? T.pres2 : T.pres;
  float* __restrict__ pout = dir ? T.pres : T.pres2;
  // every global load of the thread: own values of its colour-1 cells, neighbours and own values of its
  // colour-0 cells
  float pb[kTblPerB], pa[kTblPerA], nba[kTblPerA][6];
#pragma unroll
  for (int u = 0; u < kTblPerB; ++u) {
    const int e = threadIdx.x + u * kTblThreads;
    pb[u] = e < nb ? pin[S.sb[e]] : 0.f;
  }
  const float* __restrict__ po = pin + nh;
#pragma unroll
  for (int u = 0; u < kTblPerA; ++u) {
    const int e = threadIdx.x + u * kTblThreads;
    pa[u] = 0.f;
#pragma unroll
    for (int d = 0; d < 6; ++d) nba[u][d] = 0.f;
    if (e < na) {
      const int s = S.sa[e];
      int bidx, i, j, k;
      tbl_cell(S.ea[e].x, x0, y0, z0, bidx, i, j, k);
      const int rowb = s - (i >> 1);
      pa[u] = pin[s];
      if (on) {
        nba[u][0] = i > 0 ? po[((i - 1) >> 1) + rowb] : 0.f;
        nba[u][1] = i + 1 < nx ? po[((i + 1) >> 1) + rowb] : 0.f;
        nba[u][2] = j > 0 ? po[(i >> 1) + rowb - hx] : 0.f;
        nba[u][3] = j + 1 < ny ? po[(i >> 1) + rowb + hx] : 0.f;
        nba[u][4] = k > 0 ? po[(i >> 1) + rowb - hx * ny] : 0.f;
        nba[u][5] = k + 1 < nz ? po[(i >> 1) + rowb + hx * ny] : 0.f;
      }
    }
  }
#pragma unroll
  for (int u = 0; u < kTblPerA; ++u) {
    const int e = threadIdx.x + u * kTblThreads;
    if (e >= na) continue;
    const uint2 en = S.ea[e];
    int bidx, i, j, k;
    tbl_cell(en.x, x0, y0, z0, bidx, i, j, k);
    float v = pa[u];
    if (on) {
      float C[6];
      tbl_coeffs(T, en.x, S.cut, i, j, k, C);
      v = sor_update(C, nba[u], __uint_as_float(en.y), pa[u], omega);
    }
    S.box[bidx] = v;
    if (en.x & (1u << 21)) pout[S.sa[e]] = v;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < kTblPerB; ++u) {
    const int e = threadIdx.x + u * kTblThreads;
    if (e >= nb) continue;
    const uint2 en = S.eb[e];
    int bidx, i, j, k;
    tbl_cell(en.x, x0, y0, z0, bidx, i, j, k);
    float v = pb[u];
    if (on) {
      float nbv[6];
      nbv[0] = i > 0 ? S.box[bidx - 1] : 0.f;
      nbv[1] = i + 1 < nx ? S.box[bidx + 1] : 0.f;
      nbv[2] = j > 0 ? S.box[bidx - kTblBX] : 0.f;
      nbv[3] = j + 1 < ny ? S.box[bidx + kTblBX] : 0.f;
      nbv[4] = k > 0 ? S.box[bidx - kTblBX * kTblBY] : 0.f;
      nbv[5] = k + 1 < nz ? S.box[bidx + kTblBX * kTblBY] : 0.f;
      float C[6];
      tbl_coeffs(T, en.x, S.cut, i, j, k, C);
      v = sor_update(C, nbv, __uint_as_float(en.y), pb[u], omega);
    }
    pout[S.sb[e]] = v;
  }
}

void launch_tbl_lists(const LaunchCtx& L) {
  k_tbl_lists<<<L.nblocks[kFamTiles], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamTiles], L.tbl_list, L.tbl_cnt, L.tbl_c);
}

size_t tbl_list_bytes(int tiles) {
  return (size_t)tiles * ((kTblCapA + kTblCapB) * sizeof(uint2) + 3 * sizeof(int) + kTblCapA * sizeof(int2));
}

void tbl_assign(LaunchCtx& L, void* base, int tiles) {
  char* p = static_cast<char*>(base);
  L.tbl_list = reinterpret_cast<uint2*>(p);
  p += (size_t)tiles * (kTblCapA + kTblCapB) * sizeof(uint2);
  L.tbl_c = reinterpret_cast<int2*>(p);
  p += (size_t)tiles * kTblCapA * sizeof(int2);
  L.tbl_cnt = reinterpret_cast<int*>(p);
}

// pres ← pres2 (after an odd number of temporal-blocked launches)
__global__ void __launch_bounds__(kThreads) k_sor_copy(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx) {
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int s = (blockIdx.x - bpfx[t]) * blockDim.x + threadIdx.x;
  if (s >= T.nhalf) return;
  T.pres[s] = T.pres2[s];
  T.pres[T.nhalf + s] = T.pres2[T.nhalf + s];
}

cudaError_t sor_tb_prepare() {
  const cudaError_t e = cudaFuncSetAttribute(k_sor_tbl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TblSmem));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_sor_tb<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, TbShape<4>::SMEM);
}

void launch_sor_tb(const LaunchCtx& L, int sweeps_per_launch, int sweep0, int nsweeps, int dir) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(L.nblocks[kFamTiles]);
  cfg.blockDim = dim3(sweeps_per_launch == 2 ? kTblThreads : kTbThreads);
  cfg.dynamicSmemBytes = sweeps_per_launch == 2 ? sizeof(TblSmem) : TbShape<4>::SMEM;
  cfg.stream = L.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = sweep0 > 0 ? 1 : 0;     // the first launch waits for the grid pass (and the lists) in full
  if (sweeps_per_launch == 2)
    cudaLaunchKernelEx(&cfg, k_sor_tbl, L.tanks, L.ntanks, (const int*)L.bpfx[kFamTiles], (const uint2*)L.tbl_list,
                       (const int*)L.tbl_cnt, (const int2*)L.tbl_c, sweep0, dir);
  else
    cudaLaunchKernelEx(&cfg, k_sor_tb<4>, L.tanks, L.ntanks, (const int*)L.bpfx[kFamTiles], sweep0, nsweeps, dir);
}

void launch_sor_copy(const LaunchCtx& L) {
  k_sor_copy<<<L.nblocks[kFamHalf], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamHalf]);
}

// ---------------------------------------------------------------------------- cluster-resident solve
// The whole solve in one launch, each tank held on chip by one thread-block cluster: the tank is cut into
// pieces of whole z planes, one piece per CTA, and each CTA keeps its planes' pressure (both colours),
// right-hand side and a one-byte cell code in shared memory for all 2·iters colour sweeps. No global memory
// and no launch between sweeps; the hardware cluster barrier (barrier.cluster arrive.release / wait.acquire)
// separates them. Small tanks share a cluster (a piece only talks to the pieces of its own tank), and every
// CTA takes part in every barrier of its cluster.
//
// The pressure of a piece is stored padded: each row of a colour has a zero slot before and after it, each
// plane a zero row below and above, and the piece a ghost plane below and above. Outside the tank the
// padding holds 0, which is what the reference's zero-padded pressure reads there (solver.py:489-506), so a
// cell's six neighbours are six loads at fixed offsets with no tests. A ghost plane next to another piece
// holds that piece's boundary plane: loaded from global memory at the start, then written by the neighbour
// (st.shared::cluster into this CTA's shared memory) each time it relaxes that plane. Sweep order per CTA:
// wait (the neighbours' boundary planes of the previous sweep, with their pushes, are complete), relax the
// boundary planes and push them, arrive, relax the interior planes (their neighbours are all in this
// piece), CTA barrier. A piece's ghost plane is rewritten only after the neighbour has passed the wait that
// follows every read of it. The update is sor_update's in the same colour order: the pressures equal one
// launch per sweep bit for bit.
//
// Shared layout per CTA (W = hx + 2, RY = ny + 2, NP = np + 2, np = the tank's planes per piece, the same
// for all its pieces): pressure [2][NP·RY·W] f32 padded; rhs [2][np·ny·hx] f32 and code [2][np·ny·hx] u8
// (bits 0-5 open faces, 6 cut cell, 7 active) unpadded; the sweeps' work counters.
constexpr int kClusterThreads = 1024;

__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

__device__ __forceinline__ unsigned cluster_ctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// store v at the same shared-memory offset as `local` in the CTA of cluster rank `rank`
__device__ __forceinline__ void st_cluster(float* local, unsigned rank, float v) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(local);
  unsigned ra;
  asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(ra), "f"(v) : "memory");
}

struct ClusterLayout {
  int W, RY, PS, US;          // padded row width, padded rows per plane, padded and unpadded slots per colour
};
__host__ __device__ __forceinline__ ClusterLayout cluster_layout(int hx, int ny, int np) {
  ClusterLayout c;
  c.W = hx + 2;
  c.RY = ny + 2;
  c.PS = (np + 2) * c.RY * c.W;
  c.US = np * ny * hx;
  return c;
}

__global__ void __launch_bounds__(kClusterThreads, 1) k_sor_cluster(const TankDev* __restrict__ tanks,
                                                                    const ClusterPiece* __restrict__ pieces, int max_iters) {
  extern __shared__ __align__(16) unsigned char cl_smem[];
  const ClusterPiece pc = pieces[blockIdx.x];
  const bool on = pc.tank >= 0;
  const TankDev& T = tanks[on ? pc.tank : 0];
  const int hx = T.hx, nx = T.nx, ny = T.ny, nz = T.nz;
  const int k0 = pc.k0, nk = on ? pc.nk : 0, np_ = on ? pc.np : 0;
  const ClusterLayout G = cluster_layout(hx, ny, np_);
  const int W = G.W, RY = G.RY, PS = on ? G.PS : 0, US = on ? G.US : 0;
  const int U = nk * ny * hx;                         // this piece's own slots per colour
  const size_t nh = T.nhalf;
  float* sp = reinterpret_cast<float*>(cl_smem);     // [2][PS]
  float* sr = sp + 2 * PS;                           // [2][US]
  int* s_cnt = reinterpret_cast<int*>(sr + 2 * US);  // [8] (spare)
  uint8_t* sc = reinterpret_cast<uint8_t*>(s_cnt + 8);   // [2][US]
  uint16_t* sl = reinterpret_cast<uint16_t*>(sc + 2 * US);   // [2][US]: the active slots, by colour and region
  __shared__ int s_n[2][3], s_o[2][3], s_f[2][3];    // per colour and region (first plane, last plane, interior)
  const unsigned rank = cluster_ctarank();
  if (threadIdx.x < 6) { (&s_n[0][0])[threadIdx.x] = 0; (&s_f[0][0])[threadIdx.x] = 0; }
  __syncthreads();
  // pressure of the own planes and the ghost planes, zero in the padding and outside the tank
  for (int q = threadIdx.x; q < 2 * PS; q += kClusterThreads) {
    const int c = q >= PS, L = q - c * PS;
    const int tp = L % W, rest = L / W, jp = rest % RY, kl = rest / RY - 1;
    const int ti = tp - 1, j = jp - 1, k = k0 + kl;
    float v = 0.f;
    if (ti >= 0 && ti < hx && j >= 0 && j < ny && kl <= nk && k >= 0 && k < nz)
      v = T.pres[c * nh + ti + (size_t)hx * (j + (size_t)ny * k)];
    sp[q] = v;
  }
  const size_t g0 = (size_t)hx * ny * k0;            // first slot of the piece in each colour's global array
  const int iters = on ? T.iters : 0;
  const float omega = T.omega;
  const DivU dny = T.dny, dhx = T.dhx;
  const bool below = on && k0 > 0, above = on && k0 + nk < nz;   // neighbour pieces (remote planes)
  // rows [0, lo_r): first plane (it reads and feeds the piece below); [hi_r, nk·ny): last plane (the piece
  // above); [lo_r, hi_r): interior. A single plane with neighbours on both sides is the first range.
  const int lo_r = below ? ny : 0;
  const int hi_r = (above && !(below && nk == 1)) ? (nk - 1) * ny : nk * ny;
  auto region = [&](int l) { const int row = divu(l, dhx); return row < lo_r ? 0 : (row >= hi_r ? 1 : 2); };
  for (int q = threadIdx.x; q < 2 * U; q += kClusterThreads) {
    const int c = q >= U, l = q - c * U;
    const size_t g = c * nh + g0 + l;
    const uint32_t cd = T.code[g];
    sr[c * US + l] = T.rhs[g];
    sc[c * US + l] = (uint8_t)((cd & 0x3Fu) | ((cd & kCodePartial) ? 0x40u : 0u) | ((cd & kCodeActive) ? 0x80u : 0u));
    if (cd & kCodeActive) atomicAdd(&s_n[c][region(l)], 1);
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    const int c = threadIdx.x;
    s_o[c][0] = c * US; s_o[c][1] = s_o[c][0] + s_n[c][0]; s_o[c][2] = s_o[c][1] + s_n[c][1];
  }
  __syncthreads();
  // the lists of active slots: the sweeps visit only liquid cells with an open face
  for (int q = threadIdx.x; q < 2 * U; q += kClusterThreads) {
    const int c = q >= U, l = q - c * U;
    if (!(sc[c * US + l] & 0x80u)) continue;
    const int r = region(l);
    sl[s_o[c][r] + atomicAdd(&s_f[c][r], 1)] = (uint16_t)l;
  }
  __syncthreads();
  const int ghost_above_plane = np_ + 1;             // the piece below stores this piece's first plane here
  // 1/n for the cells without cut faces, n their open faces (the correctly rounded reciprocals)
  __shared__ float s_inv[8];
  if (threadIdx.x < 8) s_inv[threadIdx.x] = threadIdx.x ? __frcp_rn((float)threadIdx.x) : 0.f;
  __syncthreads();
  auto relax = [&](auto push, int c, int reg) {
    const float* po = sp + (1 - c) * PS;
    float* pw = sp + c * PS;
    const float* rw = sr + c * US;
    const uint8_t* cw = sc + c * US;
    const uint16_t* lst = sl + s_o[c][reg];
    const int cnt = s_n[c][reg];
#pragma unroll 1
    for (int e = threadIdx.x; e < cnt; e += kClusterThreads) {
      const int l = lst[e];
      const int row = divu(l, dhx), ti = l - row * hx;
      const uint32_t cd = cw[l];
      const int kl = divu(row, dny), j = row - kl * ny, k = k0 + kl;
      const int s = (j + k + c) & 1;
      const int L = (ti + 1) + W * ((j + 1) + RY * (kl + 1));
      float nb[6];
      nb[0] = po[L - 1 + s];
      nb[1] = po[L + s];
      nb[2] = po[L - W];
      nb[3] = po[L + W];
      nb[4] = po[L - W * RY];
      nb[5] = po[L + W * RY];
      const float rhs = rw[l], p = pw[L];
      float v;
      if (cd & 0x40u) {
        float C[6];
        cut_coeffs(T, 2 * ti + s, j, k, C);
        v = sor_update_inv(C, nb, rhs, p, omega, coeff_inv(true, cd, C));
      } else {
        v = sor_update_open(cd, nb, rhs, p, omega, s_inv[__popc(cd & 0x3Fu)]);
      }
      pw[L] = v;
      if (push) {
        if (kl == 0 && below) st_cluster(pw + (ti + 1) + W * ((j + 1) + RY * ghost_above_plane), rank - 1, v);
        if (kl == nk - 1 && above) st_cluster(pw + (ti + 1) + W * (j + 1), rank + 1, v);
      }
    }
  };
  const std::true_type with_push;
  const std::false_type no_push;
  cluster_arrive();                       // this piece is loaded
  for (int it = 0; it < max_iters; ++it) {
#pragma unroll 1
    for (int c = 0; c < 2; ++c) {
      const bool go = it < iters;
      cluster_wait();
      if (go) {
        relax(with_push, c, 0);
        relax(with_push, c, 1);
      }
      cluster_arrive();
      if (go) relax(no_push, c, 2);
      __syncthreads();
    }
  }
  cluster_wait();                         // no neighbour writes this piece's ghost planes any more
  for (int q = threadIdx.x; q < 2 * U; q += kClusterThreads) {
    const int c = q >= U, l = q - c * U;
    const int row = divu(l, T.dhx), ti = l - row * hx;
    const int kl = divu(row, dny), j = row - kl * ny;
    T.pres[c * nh + g0 + l] = sp[c * PS + (ti + 1) + W * ((j + 1) + RY * (kl + 1))];
  }
}

// shared bytes of a piece of np planes: padded pressure, rhs, the work counters and the codes
int cluster_smem_bytes(const TankDev& D, int np) {
  const ClusterLayout G = cluster_layout(D.hx, D.ny, np);
  return ((8 * G.PS + 8 * G.US + 32 + 2 * G.US + 4 * G.US) + 15) & ~15;
}

cudaError_t sor_cluster_prepare(int smem_bytes, int cluster) {
  cudaError_t e = cudaFuncSetAttribute(k_sor_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
  if (e != cudaSuccess) return e;
  if (cluster > 8) e = cudaFuncSetAttribute(k_sor_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

static void cluster_config(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* attr, int nblocks, int smem_bytes, int cluster,
                           cudaStream_t stream) {
  cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = smem_bytes;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
}

int sor_cluster_max_active(int smem_bytes, int cluster) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr[1];
  cluster_config(cfg, attr, cluster, smem_bytes, cluster, nullptr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_sor_cluster, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

void launch_sor_cluster(const LaunchCtx& L, const ClusterPiece* pieces, int nblocks, int smem_bytes, int cluster,
                        int max_iters) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr[1];
  cluster_config(cfg, attr, nblocks, smem_bytes, cluster, L.stream);
  cudaLaunchKernelEx(&cfg, k_sor_cluster, L.tanks, pieces, max_iters);
}

void launch_sor_sweep(const LaunchCtx& L, int color, int sweep) {
  cudaLaunchConfig_t cfg = {};
  // A grid larger than what is resident at once is capped there and loops: the next sweep's blocks then
  // find room while this sweep runs (on 256×128×128 this took a solve from 1.60 to 0.98 ms).
  static int resident[128] = {};
  const int cap = resident_grid((const void*)k_sor<true>, resident);
  const bool loop = L.nblocks[kFamSor] > cap;
  cfg.gridDim = dim3(loop ? cap : L.nblocks[kFamSor]);
  cfg.blockDim = dim3(kSorThreads);
  cfg.stream = L.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = (color | sweep) ? 1 : 0;     // the first sweep waits for the grid pass in full
  if (loop) cudaLaunchKernelEx(&cfg, k_sor<true>, L.tanks, L.ntanks, (const int*)L.apfx, color, sweep);
  else cudaLaunchKernelEx(&cfg, k_sor<false>, L.tanks, L.ntanks, (const int*)L.apfx, color, sweep);
}

// FP64 residual of the solve just finished, per active cell of `color`: r = Σ C_d·p_nb − rhs − (Σ C_d)·p,
// evaluated in float64 from the float32 coefficients, right-hand side and pressures (outside the grid p = 0).
// It is the residual of the linear system the float32 sweeps approximate; max |r|, max |rhs| and Σ r² go to
// the tank counters, one atomic per warp where the warp's cells belong to one tank.
__global__ void __launch_bounds__(kThreads) k_sor_residual(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ apfx,
                                                           int color) {
  const int* __restrict__ pfx = apfx + color * (ntanks + 1);
  const int total = pfx[ntanks];
  if ((int)(blockIdx.x * blockDim.x) >= total) return;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = q < total;
  const int t = find_slot(pfx, ntanks, live ? q : total - 1);
  double ra = 0.0, rh = 0.0, r2 = 0.0;
  if (live) {
    const TankDev& T = tanks[t];
    const int hx = T.hx, nx = T.nx, ny = T.ny, nz = T.nz;
    const int s = T.act[(size_t)color * T.nhalf + (q - pfx[t])].x;
    const int row = divu(s, T.dhx), ti = s - row * hx;
    const int k = divu(row, T.dny), j = row - k * ny;
    const int i = 2 * ti + ((j + k + color) & 1);
    const size_t own = (size_t)color * T.nhalf + s;
    const uint32_t code = T.code[own];
    const float* __restrict__ po = T.pres + (size_t)(1 - color) * T.nhalf;
    const int rowb = hx * row;
    float nb[6];
    nb[0] = i > 0 ? po[((i - 1) >> 1) + rowb] : 0.f;
    nb[1] = i + 1 < nx ? po[((i + 1) >> 1) + rowb] : 0.f;
    nb[2] = j > 0 ? po[ti + rowb - hx] : 0.f;
    nb[3] = j + 1 < ny ? po[ti + rowb + hx] : 0.f;
    nb[4] = k > 0 ? po[ti + rowb - hx * ny] : 0.f;
    nb[5] = k + 1 < nz ? po[ti + rowb + hx * ny] : 0.f;
    float C[6];
    if (code & kCodePartial) {
      cut_coeffs(T, i, j, k, C);
    } else {
#pragma unroll
      for (int d = 0; d < 6; ++d) C[d] = (code >> d) & 1u ? 1.0f : 0.0f;
    }
    double num = 0.0, den = 0.0;
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      num = __dadd_rn(num, __dmul_rn((double)C[d], (double)nb[d]));
      den = __dadd_rn(den, (double)C[d]);
    }
    const double rhs = (double)T.rhs[own];
    const double r = __dsub_rn(__dsub_rn(num, rhs), __dmul_rn(den, (double)T.pres[own]));
    ra = fabs(r);
    rh = fabs(rhs);
    r2 = __dmul_rn(r, r);
  }
  const unsigned lanes = __ballot_sync(0xffffffffu, true);
  const int t0 = __shfl_sync(lanes, t, 0);
  if (__all_sync(lanes, t == t0)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ra = fmax(ra, __shfl_xor_sync(lanes, ra, o));
      rh = fmax(rh, __shfl_xor_sync(lanes, rh, o));
      r2 = __dadd_rn(r2, __shfl_xor_sync(lanes, r2, o));
    }
    if ((threadIdx.x & 31) != 0) return;
  } else if (!live) {
    return;
  }
  Counters* c = tanks[t].ctr;
  atomicMax(&c->res_max_bits, (unsigned long long)__double_as_longlong(ra));
  atomicMax(&c->rhs_max_bits, (unsigned long long)__double_as_longlong(rh));
  atomicAdd(&c->res_sum2, r2);
}

void launch_sor_residual(const LaunchCtx& L) {
  for (int c = 0; c < 2; ++c)
    k_sor_residual<<<L.nblocks[kFamSor], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, (const int*)L.apfx, c);
}

// shared memory a block of the persistent solve may take (the device's opt-in maximum less its static part)
static int sor_persist_smem(int device) {
  static int cache[128] = {};
  if (device < 0 || device >= 128) return 0;
  if (!cache[device]) {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    const int bytes = optin - 1024;
    cudaFuncSetAttribute(k_sor_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cache[device] = bytes;
  }
  return cache[device];
}

int sor_persist_max_blocks(int device) {
  int per_sm = 0, sms = 0;
  const int smem = sor_persist_smem(device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sor_persist, kResThreads, smem);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm * sms;
}

void launch_sor_persist(const LaunchCtx& L, int max_iters, int blocks, unsigned limit, int smem_cap) {
  int dev = 0;
  cudaGetDevice(&dev);
  const int smem = smem_cap > 0 ? std::min(smem_cap, sor_persist_smem(dev)) : sor_persist_smem(dev);
  const int cap = smem / kResEntryBytes;
  // the barrier starts every solve cleared: a solve whose wait gave up leaves its counts behind
  cudaMemsetAsync(L.barrier, 0, sizeof(GridBarrier), L.stream);
  // cooperative launch: the runtime refuses it unless every block can be resident at once
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kResThreads);
  cfg.dynamicSmemBytes = (size_t)cap * kResEntryBytes;
  cfg.stream = L.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_sor_persist, L.tanks, L.ntanks, (const int*)L.apfx, max_iters, L.barrier, limit, cap);
}

}  // namespace suiri
