// Cell binning of particles: a counting sort by cell that also drops particles killed in the previous
// sub-step and appends the ones emitted for this one.
//
//   bin      per particle of A∪E: its cell (float64 grid coordinate, exactly the reference's
//            floor((x - origin)/h), blender_addon/suiri_lab/solver.py:430-436), a warp-aggregated
//            atomicAdd on the cell counter (__match_any_sync groups lanes of the same cell: particles
//            arrive sorted, so most lanes share one), and the particle's rank inside its cell.
//   scan     exclusive prefix of the counts per tank → off[c]; count(c) = off[c+1] - off[c].
//            The per-cell counts equal np.bincount bit for bit (integers).
//   scatter  B[off[cell] + rank] = particle: B holds every tank's particles grouped by cell, the
//            particles outside the grid (above the tank) after the last cell.
//
// The reference counts cells with global u32 atomics inside P2G (src/js/30-wgsl-sim.js:192-195) and
// removes dead particles with a separate unordered compaction pass (src/js/31-wgsl-sim2.js:317-328);
// here one sort serves binning, compaction and the memory locality of P2G/G2P.
#include "launch.cuh"

namespace suiri {

// one block: prefix over tanks of |A∪E| for a count pass between sub-steps (the sub-step itself writes it in
// k_emit_begin, which also advances the sub-step counters)
__global__ void k_count_prefix(const TankDev* __restrict__ tanks, int ntanks, int* __restrict__ pfx) {
  tank_prefix(ntanks, pfx, [&](int t) { return tanks[t].ctr->n_live + tanks[t].ctr->n_emit; });
}

__device__ __forceinline__ int particle_cell(const TankDev& T, float4 p) {
  if (flags_of(p.w) & kFlagDead) return -1;
  double gx, gy, gz;
  grid_pos(T, (double)p.x, (double)p.y, (double)p.z, gx, gy, gz);
  if (!in_grid(T, gx, gy, gz)) return T.ncells;           // outside: the extra last slot
  return cell_idx(T, (int)gx, (int)gy, (int)gz);
}

__device__ __forceinline__ float4 load_in(const TankDev& T, int local, int n_live, const float4* a, const float4* e) {
  return local < n_live ? a[local] : e[local - n_live];
}

__global__ void __launch_bounds__(kThreads) k_bin(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ pfx) {
  const int total = pfx[ntanks];
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < total; base += stride) {
    const int idx = base + lane;
    int cell = -1, t = 0, local = 0;
    const TankDev* T = nullptr;
    if (idx < total) {
      t = find_slot(pfx, ntanks, idx);
      T = tanks + t;
      local = idx - pfx[t];
      const int n_live = T->ctr->n_live;
      cell = particle_cell(*T, load_in(*T, local, n_live, T->pA, T->pE));
    }
    const unsigned act = __ballot_sync(0xffffffffu, cell >= 0);
    if (cell >= 0) {
      const unsigned long long key = ((unsigned long long)(unsigned)t << 32) | (unsigned)cell;
      const unsigned peers = __match_any_sync(act, key);
      const int leader = __ffs(peers) - 1;
      const unsigned below = peers & ((1u << lane) - 1u);
      int first = 0;
      if (lane == leader) first = atomicAdd(T->cnt + cell, __popc(peers));
      first = __shfl_sync(act, first, leader);   // every lane of `act` reads its own group's leader
      T->rank[local] = (uint32_t)(first + __popc(below));
    }
  }
}

// the cell counts alone, for a count pass between sub-steps (no ranks: the next sub-step bins again)
__global__ void __launch_bounds__(kThreads) k_bin_count(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ pfx) {
  const int total = pfx[ntanks];
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < total; base += stride) {
    const int idx = base + lane;
    int cell = -1, t = 0;
    const TankDev* T = nullptr;
    if (idx < total) {
      t = find_slot(pfx, ntanks, idx);
      T = tanks + t;
      const int local = idx - pfx[t];
      const int n_live = T->ctr->n_live;
      cell = particle_cell(*T, load_in(*T, local, n_live, T->pA, T->pE));
    }
    const unsigned act = __ballot_sync(0xffffffffu, cell >= 0);
    if (cell >= 0) {
      const unsigned peers = __match_any_sync(act, ((unsigned long long)(unsigned)t << 32) | (unsigned)cell);
      if (lane == __ffs(peers) - 1) atomicAdd(T->cnt + cell, __popc(peers));   // result unused: a reduction
    }
  }
}

// --- scan: tiles of kScanTile cells; bsum[block] = tile sum; then per tile: prefix of earlier tiles of the
// same tank + in-tile exclusive scan
__device__ __forceinline__ int block_sum(int v, int* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) red[w] = v;
  __syncthreads();
  int r = 0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0;
    for (int o = 16; o; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;   // valid in thread 0
}

__global__ void __launch_bounds__(kThreads) k_scan_a(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx,
                                                     long long* __restrict__ bsum) {
  __shared__ int red[32];
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int tile = blockIdx.x - bpfx[t];
  const int n = T.ncells + 1;
  const int b0 = tile * kScanTile;
  int v = 0;
  for (int e = threadIdx.x; e < kScanTile; e += blockDim.x) {
    const int c = b0 + e;
    if (c < n) v += T.cnt[c];
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) bsum[blockIdx.x] = v;
}

__global__ void __launch_bounds__(kThreads) k_scan_b(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ bpfx,
                                                     const long long* __restrict__ bsum) {
  __shared__ int red[32];
  __shared__ int s_pre;
  __shared__ int s_warp[kThreads / 32];
  const int t = find_slot(bpfx, ntanks, blockIdx.x);
  const TankDev& T = tanks[t];
  const int first_block = bpfx[t];
  const int tile = blockIdx.x - first_block;
  const int n = T.ncells + 1;
  // prefix of the earlier tiles of this tank
  long long pre = 0;
  for (int b = first_block + threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) pre += bsum[b];
  const int pre_i = block_sum((int)pre, red);
  if (threadIdx.x == 0) s_pre = pre_i;
  __syncthreads();
  // each thread owns 8 consecutive cells of the tile
  constexpr int kPer = kScanTile / kThreads;
  const int c0 = tile * kScanTile + threadIdx.x * kPer;
  int vals[kPer];
  int mine = 0;
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int c = c0 + e;
    vals[e] = c < n ? T.cnt[c] : 0;
    mine += vals[e];
  }
  // block exclusive scan of `mine`
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = mine;
  for (int o = 1; o < 32; o <<= 1) {
    const int a = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += a;
  }
  if (lane == 31) s_warp[w] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { const int x = s_warp[i]; s_warp[i] = acc; acc += x; }
  }
  __syncthreads();
  int run = s_pre + s_warp[w] + inc - mine;
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int c = c0 + e;
    if (c < n) {
      T.off[c] = run;
      T.cnt[c] = 0;                 // counts live on in off[]; clear for the next sub-step
      run += vals[e];
      if (c == n - 1) {             // the outside slot closes the tank
        T.off[n] = run;
        T.ctr->n_sorted = run;
        T.ctr->n_ingrid = run - vals[e];
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_scatter(const TankDev* __restrict__ tanks, int ntanks, const int* __restrict__ pfx,
                                                      int* __restrict__ spfx, unsigned* __restrict__ ticket) {
  const int total = pfx[ntanks];
  const int stride = gridDim.x * blockDim.x;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += stride) {
    const int t = find_slot(pfx, ntanks, idx);
    const TankDev& T = tanks[t];
    const int local = idx - pfx[t];
    const int n_live = T.ctr->n_live;
    const float4 p = load_in(T, local, n_live, T.pA, T.pE);
    const int cell = particle_cell(T, p);
    if (cell < 0) continue;
    const float4 v = load_in(T, local, n_live, T.vA, T.vE);
    const int dst = T.off[cell] + (int)T.rank[local];
    T.pB[dst] = p;
    T.vB[dst] = v;
  }
  // the last block, once every block has read n_live: prefix of the sorted particles over tanks; A will
  // hold exactly B's particles after G2P
  if (last_block(ticket)) {
    tank_prefix(ntanks, spfx, [&](int u) {
      Counters* c = tanks[u].ctr;
      const int v = __ldcg(&c->n_sorted);
      c->n_live = v;
      c->n_emit = 0;
      return v;
    });
  }
}

void launch_begin_count(const LaunchCtx& L) {
  k_count_prefix<<<1, 1024, 0, L.stream>>>(L.tanks, L.ntanks, L.ppfx_in);
}
// binning and scatter are chains of dependent loads per particle: as many resident threads as fit
void launch_bin(const LaunchCtx& L) {
  static int resident[128] = {};
  k_bin<<<resident_grid((const void*)k_bin, resident), kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.ppfx_in);
}
void launch_bin_count(const LaunchCtx& L) {
  static int resident[128] = {};
  k_bin_count<<<resident_grid((const void*)k_bin_count, resident), kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.ppfx_in);
}
void launch_scan(const LaunchCtx& L) {
  const int nb = L.nblocks[kFamScan];
  k_scan_a<<<nb, kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamScan], L.scan_bsum);
  k_scan_b<<<nb, kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.bpfx[kFamScan], L.scan_bsum);
}
void launch_scatter(const LaunchCtx& L) {
  static int resident[128] = {};
  k_scatter<<<resident_grid((const void*)k_scatter, resident), kThreads, 0, L.stream>>>(L.tanks, L.ntanks, L.ppfx_in,
                                                                                      L.ppfx_sorted, L.ticket + 1);
}

}  // namespace suiri
