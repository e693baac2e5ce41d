// Shared device-side definitions of the FLIP step: the per-tank descriptor that every kernel reads,
// fixed-point scales, and small helpers. All kernels are batched: a launch covers any number of tanks,
// each described by one TankDev record in device memory.
//
// Grid layout in HBM (x fastest, like the reference's WGSL indexing, src/js/30-wgsl-sim.js:25-33):
//   node n = i + (nx+1)*(j + (ny+1)*k),  i∈[0,nx], j∈[0,ny], k∈[0,nz]   (staggered face "nodes")
//   cell c = i + nx*(j + ny*k)
//   SOR arrays are split by colour (i+j+k)&1: slot s = (i>>1) + hx*(j + ny*k), hx = (nx+1)/2.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace suiri {

// P2G sums are integer fixed point: order independent, so every run and every batch mix gives the same
// bits. 2^38 keeps 3.6e-12 resolution per contribution (|w·v| ≤ 30 → |term| < 2^43), so a node's 64-bit
// sum has headroom for 2^20 terms. Inside a P2G brick a term also splits exactly into a 22-bit remainder
// and a signed quotient, which 32-bit shared atomics can sum without overflow while a node takes at most
// kSplitMaxTerms terms (1023·(2^22 − 1) < 2^32 and 1023·2^21 < 2^31).
constexpr double kFix = 274877906944.0;           // 2^38
constexpr double kFixInv = 1.0 / 274877906944.0;
constexpr int kSplit = 22;                        // remainder bits of the split shared-memory sums
constexpr int kSplitMaxTerms = 1023;              // terms per node for which both halves stay exact
constexpr double kRippleFix = 281474976710656.0;  // 2^48, ripple impulses [N·s]
constexpr double kBig = 1e9;

constexpr int kMaxObj = 64;                       // like the reference's MAX_OBJ (src/js/50-sim.js:9)

// SOR cell code bits (one uint32 per cell, colour-split)
constexpr uint32_t kCodeActive = 1u << 12;         // liquid cell with at least one open face
constexpr uint32_t kCodePartial = 1u << 13;        // some face fraction strictly between 0 and 1
// bits 0..5: face d (x-, x+, y-, y+, z-, z+) fully open (fraction exactly 1)

enum SdfMode { kSdfAnalytic = 0, kSdfLattice = 1 };

// Division by a divisor fixed per tank as a multiply-high and a shift (Granlund & Montgomery, "Division by
// invariant integers using multiplication", 1994, round-up variant): with l = ceil(log2 d) and
// mul = floor(2^32 (2^l − d) / d) + 1, n / d = (umulhi(n, mul) + n) >> l exactly for 0 ≤ n < 2^31.
struct DivU {
  uint32_t mul, shr;
};
inline DivU make_divu(uint32_t d) {
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  return DivU{(uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1), l};
}

// An obstacle (flag 1) or drain (flag 2). Doubles: obstacle geometry feeds the bit-exact face fractions.
struct Obj {
  double pos[3];
  double rot[9];      // world-from-local R, row major (q = Rᵀ (p - pos))
  double dims[4];
  double lin[3], ang[3];
  double bound;
  int type, flag;
  int pad[2];
};

// A fixed-rate emitter running on the device every sub-step: shape 0 disc outlet (faucet), 3 rain area.
struct EmitterDev {
  double pos[3], dir[3], u[3], w[3];
  double radius, speed, per_substep;   // particles per sub-step (fractional parts accumulate)
  double radius_z;                     // rain: half extent along z
  int shape, airborne;
};

struct Counters {
  unsigned long long vmax_bits64;  // 1 + float64 bits of max min(|v|, 60) over in-grid particles; 0: none
  int n_live;         // particles in A (previous sub-step's output, dead ones flagged)
  int n_emit;         // particles in E (emitted for this sub-step)
  int n_sorted;       // alive particles in B after binning
  int n_ingrid;       // of those, inside the grid (B[0, n_ingrid))
  int impacts;        // merged sub-grid drops (cumulative)
  int ww_count;       // whitewater particles in the current buffer
  int ww_next;        // whitewater survivors written by the advance
  int ww_cur;         // which half of the whitewater buffers is current
  int full;           // capacity was reached
  int frame;          // sub-step counter (seeds the hash RNG)
  int ww_spawned;     // whitewater spawned in the last sub-step
  int err;            // device-side error flags
  unsigned next_id;   // id of the next particle emitted on the device
  int pad;
  int n_act[2];       // active cells of each colour this sub-step (entries of TankDev::act)
  double emit_acc[8]; // fractional particles carried by the fixed emitters
  // FP64 residual of the last solve (when enabled): max |r| and max |rhs| as float64 bits (non-negative
  // doubles order like their bits), and Σ r², over the active cells
  unsigned long long res_max_bits, rhs_max_bits;
  double res_sum2;
};

struct TankDev {
  // geometry
  int nx, ny, nz, hx;
  int sx, sxy;              // node strides (nx+1), (nx+1)(ny+1)
  int nnodes, ncells, nhalf;
  int nyl;                  // lattice covers 2*nyl+1 points vertically
  DivU dnx, dny, dhx, dsx, dsxy;   // exact division by nx, ny, hx, sx, sxy
  double h, ox, oy, oz, rim;
  // physics
  double g, flip, friction, ppc, drift, ww_rate, dt;
  double vp, drop_mass;     // particle volume (h/2)³ and mass 998·(h/2)³ (host libm pow, as the reference)
  float omega;
  int iters, whitewater, nobj, sdf_mode, has_obst, moving;
  int advect;               // 0 explicit Euler, 1 RK2 midpoint through the grid velocity
  double drop_d_median, drop_d_sigma;   // > 0: sub-grid drops have lognormal diameters from their ids
  int cap, emit_cap, ww_cap;
  int rx, rz;               // ripple vertices (rx+1)×(rz+1); 0 = no ripple layer
  // particles: A live, E emitted, B sorted; pos.w = flags (bit0 airborne, bit1 dead), vel.w = id bits
  float4 *pA, *vA, *pE, *vE, *pB, *vB;
  uint32_t* rank;           // rank of a particle of A∪E inside its cell
  int* cnt;                 // ncells+1 (last: outside the grid)
  int* off;                 // ncells+2 exclusive prefix
  long long* acc;           // 6*nnodes: mom x,y,z then weight x,y,z
  float4* vel;              // after forces/solids, later projected
  float4* velold;           // P2G velocity, .w = valid-face mask bits
  float4* frac;             // face open fractions, float32
  double* fracd;            // 3*nnodes, float64 (divergence)
  uint8_t* near;            // ncells: whether an obstacle's cull (bit 1) or a drain (bit 2) can hold for a
                            // point within kNearReach·h of the cell's centre (built with the face fractions)
  float4* svel;             // solid velocity at faces
  float2* vv;               // 3*nnodes: per component (projected v, P2G v or NaN where the face took no weight)
  double* flux;             // 3*nnodes cut-cell face fluxes (divergence operand)
  float* pres;              // 2*nhalf colour-split pressure
  float* pres2;             // 2*nhalf, the other buffer of the temporal-blocked solve
  int4* act;                // 2*nhalf: per colour, the active cells of this sub-step: (colour slot, SOR code,
                            //   rhs bits, 1/ΣC bits), so a sweep reads a cell's constants in one load
  float* rhs;               // 2*nhalf h²·div
  uint32_t* code;           // 2*nhalf
  const Obj* objs;
  const double* lattice;    // (2nx+1)(2nyl+1)(2nz+1), i fastest; null unless lattice mode
  const int* oid;           // lattice nearest-obstacle index or null
  Counters* ctr;
  float4 *wpos, *wvel;      // whitewater, 2*ww_cap (two halves, ww_cur current): pos.w life, vel.w kind
  long long* rsrc;          // (rz+1)(rx+1) ripple impulses, fixed point 2^48
  const EmitterDev* emitters;
  int nemit;
  uint32_t seed;
};

constexpr int kMaxEmitters = 8;

// grid barrier of a persistent (cooperative) launch; err is set when a bounded wait gave up
struct GridBarrier {
  unsigned count, gen;
  int err, pad;
};
constexpr int kErrBarrier = 1;    // Counters::err bit: a grid barrier wait ran out

constexpr int kFlagAir = 1;
constexpr int kFlagDead = 2;

#ifdef __CUDACC__
__device__ __forceinline__ int find_slot(const int* __restrict__ pfx, int n, int x) {
  // largest t with pfx[t] <= x, t in [0, n)
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(pfx + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int node_idx(const TankDev& T, int i, int j, int k) { return i + T.sx * j + T.sxy * k; }
__device__ __forceinline__ int cell_idx(const TankDev& T, int i, int j, int k) { return i + T.nx * (j + T.ny * k); }
__device__ __forceinline__ int half_idx(const TankDev& T, int i, int j, int k) { return (i >> 1) + T.hx * (j + T.ny * k); }

// grid coordinate in float64, exactly (x - origin) / h as the reference computes it (solver.py:210-211)
__device__ __forceinline__ void grid_pos(const TankDev& T, double x, double y, double z, double& gx, double& gy, double& gz) {
  gx = (x - T.ox) / T.h;
  gy = (y - T.oy) / T.h;
  gz = (z - T.oz) / T.h;
}
__device__ __forceinline__ bool in_grid(const TankDev& T, double gx, double gy, double gz) {
  return gx >= 0.0 && gy >= 0.0 && gz >= 0.0 && gx < (double)T.nx && gy < (double)T.ny && gz < (double)T.nz;
}

__device__ __forceinline__ int flags_of(float w) { return (int)w; }

__device__ __forceinline__ int divu(int n, DivU v) {
  return (int)((__umulhi((unsigned)n, v.mul) + (unsigned)n) >> v.shr);
}
// Every block calls this once, with all its threads, after its last global write. It returns true in exactly
// one block, the last to arrive, which then sees the writes of all the others (each block fences before it
// takes its ticket; read them with __ldcg). The ticket is left at 0 for the next launch.
__device__ __forceinline__ bool last_block(unsigned* ticket) {
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned k = atomicAdd(ticket, 1u);
    s_last = k == gridDim.x - 1;
    if (s_last) *ticket = 0u;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last != 0;
}

// exclusive prefix over tanks of v(t) into pfx[0 … ntanks], by one block of up to 1024 threads; v is
// called once per tank
template <class V>
__device__ void tank_prefix(int ntanks, int* pfx, V v) {
  __shared__ int s[1024];
  int carry = 0;
  for (int base = 0; base < ntanks; base += blockDim.x) {
    const int t = base + threadIdx.x;
    const int x = t < ntanks ? v(t) : 0;
    s[threadIdx.x] = x;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
      const int a = (int)threadIdx.x >= o ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += a;
      __syncthreads();
    }
    if (t < ntanks) pfx[t] = carry + s[threadIdx.x] - x;
    carry += s[blockDim.x - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) pfx[ntanks] = carry;
  __syncthreads();
}
#endif  // __CUDACC__

}  // namespace suiri
