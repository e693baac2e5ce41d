// Red-black SOR pressure sweep.
//
// One launch relaxes one colour of every tank. Cells are stored split by colour (slot = (i>>1) + hx·row),
// so a thread's own pressure, right-hand side and code load coalesced, and its six neighbours come from
// the other colour's array (two of them in the same slot column, coalesced as well).
//
// Arithmetic is float32 in exactly the order of the reference's NumPy solve
// (blender_addon/suiri_lab/solver.py:494-505):
//   num = C0·p(x-) + C1·p(x+) + C2·p(y-) + C3·p(y+) + C4·p(z-) + C5·p(z+)    (each product rounded, summed left to right)
//   p  += ω·(((num − rhs)·inv) − p),   inv = 1/(C0+…+C5) correctly rounded
// with the library built without FMA contraction, so the pressures equal the reference's bit for bit
// given the same operands. Faces on the tank walls and floor have C = 0 (Neumann); the open top has
// C = 1 with p = 0 above (Dirichlet); non-liquid cells hold 0 and are not updated
// (src/js/30-wgsl-sim.js:267-297 is the same update as a WGSL `mix`).
//
// Most cells have every face either closed or fully open; their coefficients come from the 6 "open"
// bits of the code and the float fractions are only read for cut cells next to obstacles.
#include "launch.cuh"

namespace suiri {

__global__ void __launch_bounds__(kThreads) k_sor(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx,
                                                  int color, int sweep) {
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  if (sweep >= T.iters) return;
  const int s = (blockIdx.x - bpfx[t]) * blockDim.x + threadIdx.x;
  if (s >= T.nhalf) return;
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

void launch_sor_sweep(const LaunchCtx& L, int color, int sweep) {
  k_sor<<<L.nblocks[kFamHalf], kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamHalf], color, sweep);
}

}  // namespace suiri
