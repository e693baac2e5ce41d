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
// Two launch forms:
//   k_sor          one colour of every tank per launch (2·iters launches per solve, in the sub-step graph)
//   k_sor_persist  the whole solve in one cooperative launch: all blocks resident, a grid barrier after
//                  every colour sweep. The barrier's wait is bounded: after kSpinLimit polls it records
//                  an error in the tank counters and every block returns.
#include "launch.cuh"

namespace suiri {

__device__ __forceinline__ void sor_cell(const TankDev& T, int color, int s) {
  const int hx = T.hx, nx = T.nx, ny = T.ny, nz = T.nz;
  const int ti = s % hx, row = s / hx;
  const int j = row % ny, k = row / ny;
  const int i = 2 * ti + ((j + k + color) & 1);
  if (i >= nx) return;
  const size_t own = (size_t)color * T.nhalf + s;
  const uint32_t code = T.code[own];
  if (!(code & kCodeActive)) return;
  const float* __restrict__ po = T.pres + (size_t)(1 - color) * T.nhalf;
  const float rhs = T.rhs[own];
  float p = T.pres[own];
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
    const int n = node_idx(T, i, j, k);
    const float4 f0 = T.frac[n];
    C[0] = f0.x; C[1] = T.frac[n + 1].x; C[2] = f0.y; C[3] = T.frac[n + T.sx].y; C[4] = f0.z; C[5] = T.frac[n + T.sxy].z;
  } else {
#pragma unroll
    for (int d = 0; d < 6; ++d) C[d] = (code >> d) & 1u ? 1.0f : 0.0f;
  }
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
  r = __fmul_rn(r, T.omega);
  p = __fadd_rn(p, r);
  T.pres[own] = p;
}

__global__ void __launch_bounds__(kThreads) k_sor(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx,
                                                  int color, int sweep) {
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  if (sweep >= T.iters) return;
  const int s = (blockIdx.x - bpfx[t]) * blockDim.x + threadIdx.x;
  if (s >= T.nhalf) return;
  sor_cell(T, color, s);
}

constexpr unsigned kSpinLimit = 1u << 22;

// sense-free generation barrier over all blocks of a cooperative launch; false if the wait gave up
__device__ __forceinline__ bool grid_barrier(GridBarrier* b, unsigned nblocks) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g = *(volatile unsigned*)&b->gen;
    __threadfence();
    if (atomicAdd(&b->count, 1u) == nblocks - 1) {
      b->count = 0;
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      unsigned spins = 0;
      while (*(volatile unsigned*)&b->gen == g) {
        if (++spins > kSpinLimit || *(volatile int*)&b->err) { ok = 0; break; }
        __nanosleep(32);
      }
    }
    __threadfence();
    if (!ok) atomicExch(&b->err, 1);
    s_ok = ok;
  }
  __syncthreads();
  return s_ok;
}

__global__ void __launch_bounds__(kThreads) k_sor_persist(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ hpfx,
                                                          int max_iters, GridBarrier* bar) {
  const int total = hpfx[ntanks];
  const int stride = gridDim.x * blockDim.x;
  for (int sweep = 0; sweep < 2 * max_iters; ++sweep) {
    const int color = sweep & 1, it = sweep >> 1;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += stride) {
      const int t = find_slot(hpfx, ntanks, q);
      const TankDev& T = tanks[t];
      if (it < T.iters) sor_cell(T, color, q - hpfx[t]);
    }
    if (sweep + 1 < 2 * max_iters && !grid_barrier(bar, gridDim.x)) {
      if (threadIdx.x == 0 && blockIdx.x == 0)
        for (int t = 0; t < ntanks; ++t) atomicOr(&tanks[t].ctr->err, kErrBarrier);
      return;
    }
  }
}

void launch_sor_sweep(const LaunchCtx& L, int color, int sweep) {
  k_sor<<<L.nblocks[kFamHalf], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamHalf], color, sweep);
}

int sor_persist_max_blocks(int device) {
  int per_sm = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sor_persist, kThreads, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm * sms;
}

void launch_sor_persist(const LaunchCtx& L, int max_iters, int blocks) {
  // cooperative launch: the runtime refuses it unless every block can be resident at once
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kThreads);
  cfg.stream = L.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_sor_persist, L.tanks, L.ntanks, (const int*)L.hpfx, max_iters, L.barrier);
}

}  // namespace suiri
