// Host engine: tank state on the device, batched groups, the sub-step and frame sequence, emission,
// read-back and snapshots.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/suiri.h"
#include "sdf.cuh"

namespace suiri {

uint32_t hash_host(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation) throw Error(-3, std::string("CUDA out of memory in ") + what);
    throw Error(-2, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

// ------------------------------------------------------------------------------------ small kernels
__global__ void k_set_dt(TankDev* tanks, int n, double dt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) tanks[t].dt = dt;
}
__global__ void k_set_emit(Counters* c, int n) { c->n_emit = n; }

// Read-back compaction: the live particles of A then E, in that order, into the sorted buffers B (scratch
// between sub-steps: the binning of the next one rewrites them) in the layout of the C ABI, pos4 (x, y, z,
// airborne 0/1) and vel4 (vx, vy, vz, id bits). Tiles of kReadTile particles: a count per tile, one scan of
// the counts, then each tile writes its live particles at its prefix, ranked by warp ballots.
constexpr int kReadThreads = 256, kReadPer = 4, kReadTile = kReadThreads * kReadPer;

__device__ __forceinline__ float4 read_src(const float4* __restrict__ a, const float4* __restrict__ e, int nl, int i) {
  return i < nl ? a[i] : e[i - nl];
}

__global__ void __launch_bounds__(kReadThreads) k_read_count(const float4* __restrict__ pA, const float4* __restrict__ pE,
                                                             int nl, int tot, int* __restrict__ cnt) {
  __shared__ int s_w[kReadThreads / 32];
  int c = 0;
#pragma unroll
  for (int r = 0; r < kReadPer; ++r) {
    const int i = blockIdx.x * kReadTile + r * kReadThreads + threadIdx.x;
    if (i < tot) c += ((int)read_src(pA, pE, nl, i).w & kFlagDead) ? 0 : 1;
  }
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
#pragma unroll
    for (int w = 0; w < kReadThreads / 32; ++w) t += s_w[w];
    cnt[blockIdx.x] = t;
  }
}

// exclusive prefix of cnt[0, n) in place, the total in cnt[n]; one block of 1024 threads
__global__ void __launch_bounds__(1024) k_read_scan(int* __restrict__ cnt, int n) {
  __shared__ int s_w[32];
  __shared__ int s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < n ? cnt[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = s_w[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_w[lane] = w;
    }
    __syncthreads();
    const int before = s_carry + (warp ? s_w[warp - 1] : 0);
    if (i < n) cnt[i] = before + x - v;
    __syncthreads();
    if (threadIdx.x == 1023) s_carry = before + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) cnt[n] = s_carry;
}

__global__ void __launch_bounds__(kReadThreads) k_read_write(const float4* __restrict__ pA, const float4* __restrict__ vA,
                                                             const float4* __restrict__ pE, const float4* __restrict__ vE,
                                                             int nl, int tot, const int* __restrict__ pfx,
                                                             float4* __restrict__ outp, float4* __restrict__ outv) {
  __shared__ int s_w[kReadThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int off = pfx[blockIdx.x];
  for (int r = 0; r < kReadPer; ++r) {
    const int i = blockIdx.x * kReadTile + r * kReadThreads + threadIdx.x;
    float4 P = make_float4(0.f, 0.f, 0.f, 0.f);
    bool live = false;
    if (i < tot) {
      P = read_src(pA, pE, nl, i);
      live = !((int)P.w & kFlagDead);
    }
    const unsigned m = __ballot_sync(0xffffffffu, live);
    if (lane == 0) s_w[warp] = __popc(m);
    __syncthreads();
    int before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kReadThreads / 32; ++w) {
      const int c = s_w[w];
      before += w < warp ? c : 0;
      all += c;
    }
    if (live) {
      const int k = off + before + __popc(m & ((1u << lane) - 1));
      outp[k] = make_float4(P.x, P.y, P.z, ((int)P.w & kFlagAir) ? 1.f : 0.f);
      if (outv) outv[k] = read_src(vA, vE, nl, i);
    }
    off += all;
    __syncthreads();
  }
}

// particles added from the host, copied packed as the caller gave them (positions, then velocities and
// airborne marks where given, float32), into E's pos+flags / vel+id layout; ids count on from `first`
__global__ void k_unpack_added(float4* __restrict__ pE, float4* __restrict__ vE, const float* __restrict__ pos,
                               const float* __restrict__ vel, const float* __restrict__ air, int n, uint32_t first) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float a = air ? air[i] : 0.f;
  pE[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], a > 0.5f ? (float)kFlagAir : 0.f);
  const float vx = vel ? vel[3 * i] : 0.f, vy = vel ? vel[3 * i + 1] : 0.f, vz = vel ? vel[3 * i + 2] : 0.f;
  vE[i] = make_float4(vx, vy, vz, __uint_as_float(first + (uint32_t)i));
}

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}
__device__ __forceinline__ double rnd01(uint32_t& s) {
  s = hash32(s);
  return (double)(s >> 8) / 16777216.0;
}

// Emission record: shape 0 disc outlet (stream/shower), 1 sphere (drop/burst), 2 jittered lattice (water
// block), 3 rain area — the records of src/js/55-emit.js:13-106, emitted as src/js/31-wgsl-sim2.js:262-315 does.
struct EmitRec {
  double a[4], b[4], c[4], d[4];
  int shape, count, base;     // particles, first slot in E
  uint32_t seed, first_id;
  int pad;
};

__global__ void k_emit(TankDev T, const EmitRec* __restrict__ recs, int nrec, int total) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= total) return;
  int r = 0, acc = 0;
  for (int i = 0; i < nrec; ++i) {
    if (q < acc + recs[i].count) { r = i; break; }
    acc += recs[i].count;
  }
  const EmitRec& e = recs[r];
  const int local = q - acc;
  uint32_t s = hash32((uint32_t)local * 747796405u + e.seed * 2891336453u + 1u);
  double p[3] = {0, 0, 0}, v[3] = {0, 0, 0};
  double mark = 0.0;
  bool alive = true;
  if (e.shape == 0) {
    const double rr = e.a[3] * sqrt(rnd01(s));
    const double th = 6.283185307179586 * rnd01(s);
    const double ct = cos(th), st = sin(th);
    const double along = rnd01(s) * e.d[3];
    for (int k = 0; k < 3; ++k) p[k] = e.a[k] + (e.c[k] * ct + e.d[k] * st) * rr + e.b[k] * along;
    double dv[3] = {e.b[0], e.b[1], e.b[2]};
    if (e.c[3] > 0.0) {
      const double ca = 1.0 - rnd01(s) * (1.0 - cos(e.c[3]));
      const double sa = sqrt(fmax(1.0 - ca * ca, 0.0));
      const double ph = 6.283185307179586 * rnd01(s);
      for (int k = 0; k < 3; ++k) dv[k] = e.b[k] * ca + (e.c[k] * cos(ph) + e.d[k] * sin(ph)) * sa;
    }
    const double j0 = rnd01(s) - 0.5, j1 = rnd01(s) - 0.5, j2 = rnd01(s) - 0.5;
    v[0] = dv[0] * e.b[3] + j0 * (0.02 * e.b[3]);
    v[1] = dv[1] * e.b[3] + j1 * (0.02 * e.b[3]);
    v[2] = dv[2] * e.b[3] + j2 * (0.02 * e.b[3]);
  } else if (e.shape == 1) {
    double dd[3] = {rnd01(s) * 2 - 1 + 1e-4, rnd01(s) * 2 - 1 + 1e-4, rnd01(s) * 2 - 1 + 1e-4};
    const double l = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
    const double rad = e.a[3] * pow(rnd01(s), 1.0 / 3.0);
    for (int k = 0; k < 3; ++k) { p[k] = e.a[k] + dd[k] / l * rad; v[k] = e.b[k]; }
    mark = e.b[3];
  } else if (e.shape == 2) {
    const int nx = (int)e.b[0], ny = (int)e.b[1];
    const int i = local % nx, j = (local / nx) % ny, k = local / (nx * ny);
    const double ji[3] = {(rnd01(s) - 0.5) * 0.3, (rnd01(s) - 0.5) * 0.3, (rnd01(s) - 0.5) * 0.3};
    p[0] = e.a[0] + (i + 0.5 + ji[0]) * e.a[3];
    p[1] = e.a[1] + (j + 0.5 + ji[1]) * e.a[3];
    p[2] = e.a[2] + (k + 0.5 + ji[2]) * e.a[3];
    for (int c = 0; c < 3; ++c) v[c] = e.c[c];
    if (e.b[3] > 0.5) {            // pouring into running water: skip cells at least half full
      double g[3];
      grid_pos(T, p[0], p[1], p[2], g[0], g[1], g[2]);
      if (in_grid(T, g[0], g[1], g[2])) {
        const int c = cell_idx(T, (int)g[0], (int)g[1], (int)g[2]);
        if ((double)(T.off[c + 1] - T.off[c]) >= 0.5 * T.ppc) alive = false;
      }
    }
  } else {
    p[0] = e.a[0] + (rnd01(s) * 2 - 1) * e.a[3];
    p[1] = e.a[1] - rnd01(s) * e.d[3];
    p[2] = e.a[2] + (rnd01(s) * 2 - 1) * e.a[3];
    for (int c = 0; c < 3; ++c) v[c] = e.b[c];
    mark = 1.0;
  }
  if (alive && T.has_obst && tank_sdf(T, p[0], p[1], p[2]) < 0.0) alive = false;
  const int flags = (mark > 0.5 ? kFlagAir : 0) | (alive ? 0 : kFlagDead);
  const int slot = e.base + local;
  T.pE[slot] = make_float4((float)p[0], (float)p[1], (float)p[2], (float)flags);
  T.vE[slot] = make_float4((float)v[0], (float)v[1], (float)v[2], __uint_as_float(e.first_id + (uint32_t)local));
}

// Start of a sub-step, one block per tank, inside the captured sub-step. The tank's fixed-rate emitters
// append their particles to E: a disc outlet emits as the stream source of src/js/31-wgsl-sim2.js:276-288,
// the rain area as :307-310. Ids of device-emitted particles carry the top bit so they never meet
// host-assigned ids. Then the last block to finish advances every tank's sub-step counters and writes the
// prefix over tanks of |A∪E|.
__global__ void k_emit_begin(const TankDev* __restrict__ tanks, int ntanks, int* __restrict__ pfx, unsigned* __restrict__ ticket) {
  const TankDev& T = tanks[blockIdx.x];
  if (T.nemit > 0) {
    __shared__ int s_base, s_total, s_first[kMaxEmitters + 1];
    __shared__ unsigned s_id;
    Counters* c = T.ctr;
    if (threadIdx.x == 0) {
      const int base = c->n_emit;
      long long room = (long long)T.cap - (c->n_live + c->n_emit) - 64;
      room = min(room, (long long)T.emit_cap - c->n_emit);
      int total = 0;
      for (int e = 0; e < T.nemit; ++e) {
        const double acc = c->emit_acc[e] + T.emitters[e].per_substep;
        const double fl = floor(acc);
        c->emit_acc[e] = acc - fl;
        int n = (int)fl;
        if (n > room - total) { n = (int)max(0LL, room - total); c->full = 1; }
        s_first[e] = total;
        total += n;
      }
      s_first[T.nemit] = total;
      s_base = base;
      s_total = total;
      s_id = c->next_id;
    }
    __syncthreads();
    const int frame = c->frame + 1;
    for (int q = threadIdx.x; q < s_total; q += blockDim.x) {
      int e = 0;
      while (q >= s_first[e + 1]) ++e;
      const EmitterDev& E = T.emitters[e];
      const int local = q - s_first[e];
      uint32_t s = hash32((uint32_t)local * 747796405u + hash32(T.seed * 2891336453u + (uint32_t)frame * 97u + (uint32_t)e) + 1u);
      double p[3], v[3];
      if (E.shape == 0) {
        const double rr = E.radius * sqrt(rnd01(s));
        const double th = 6.283185307179586 * rnd01(s);
        const double ct = cos(th), st = sin(th);
        const double along = rnd01(s) * (E.speed * T.dt);
        const double j0 = rnd01(s) - 0.5, j1 = rnd01(s) - 0.5, j2 = rnd01(s) - 0.5;
        for (int k = 0; k < 3; ++k) p[k] = E.pos[k] + (E.u[k] * ct + E.w[k] * st) * rr + E.dir[k] * along;
        v[0] = E.dir[0] * E.speed + j0 * (0.02 * E.speed);
        v[1] = E.dir[1] * E.speed + j1 * (0.02 * E.speed);
        v[2] = E.dir[2] * E.speed + j2 * (0.02 * E.speed);
      } else {
        p[0] = E.pos[0] + (rnd01(s) * 2 - 1) * E.radius;
        p[1] = E.pos[1] - rnd01(s) * (E.speed * T.dt);
        p[2] = E.pos[2] + (rnd01(s) * 2 - 1) * E.radius_z;
        v[0] = 0.0; v[1] = -E.speed; v[2] = 0.0;
      }
      // the bounding-sphere test first (the outlet is usually far from every obstacle): same result
      const bool alive = !(T.has_obst && maybe_within(T, p[0], p[1], p[2], 0.0) && tank_sdf(T, p[0], p[1], p[2]) < 0.0);
      const int flags = (E.airborne ? kFlagAir : 0) | (alive ? 0 : kFlagDead);
      const int slot = s_base + q;
      T.pE[slot] = make_float4((float)p[0], (float)p[1], (float)p[2], (float)flags);
      T.vE[slot] = make_float4((float)v[0], (float)v[1], (float)v[2], __uint_as_float(0x80000000u | (s_id + (unsigned)q)));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      c->n_emit = s_base + s_total;
      c->next_id = s_id + (unsigned)s_total;
    }
  }
  if (last_block(ticket)) {
    tank_prefix(ntanks, pfx, [&](int u) {
      Counters* c = tanks[u].ctr;
      const int v = __ldcg(&c->n_live) + __ldcg(&c->n_emit);
      c->frame += 1;
      c->vmax_bits64 = 0ull;
      c->ww_spawned = 0;
      c->n_act[0] = c->n_act[1] = 0;
      c->res_max_bits = c->rhs_max_bits = 0ull;
      c->res_sum2 = 0.0;
      return v;
    });
  }
}

__global__ void k_eval_sdf(TankDev T, const double* __restrict__ pts, double* __restrict__ out, long long n) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= n) return;
  out[q] = tank_sdf(T, pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
}

// Staging for suiri_eval_sdf_static: the points (3 doubles each) followed by the distances, for at most
// kSdfStaticMax points. 2 MiB that every GPU which loads the library holds until the process exits.
constexpr long long kSdfStaticMax = 65536;
static __device__ __align__(256) double g_sdf_static[4 * kSdfStaticMax];

namespace {
std::mutex g_static_mu;
double* g_static_ptr[128] = {};

// Device address of g_sdf_static on `dev` (host code cannot use the symbol itself: its host-side name is a
// stand-in, not a device address). Looked up once per device, with that device current; the calling
// thread's current device is put back afterwards.
double* sdf_static_scratch(int dev) {
  if (dev < 0 || dev >= 128) throw Error(SUIRI_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> g(g_static_mu);
  if (!g_static_ptr[dev]) {
    int prev = 0;
    CK(cudaGetDevice(&prev));
    CK(cudaSetDevice(dev));
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sdf_static);
    CK(cudaSetDevice(prev));
    CK(e);
    g_static_ptr[dev] = (double*)p;
  }
  return g_static_ptr[dev];
}
}  // namespace

void Tank::eval_sdf_static(const double* pts, long long n, double* out) {
  if (n > kSdfStaticMax)
    throw Error(SUIRI_ERR_INVALID, "suiri_eval_sdf_static: " + std::to_string(n) + " points, at most " + std::to_string(kSdfStaticMax) +
                        " per call (the static staging array is fixed)");
  join();
  if (n <= 0) return;
  double* s = sdf_static_scratch(cfg.device);
  CK(cudaSetDevice(cfg.device));
  CK(cudaMemcpyAsync(s, pts, n * 24, cudaMemcpyHostToDevice, stream));
  k_eval_sdf<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(d, s, s + 3 * kSdfStaticMax, n);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, s + 3 * kSdfStaticMax, n * 8, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
}

void Tank::eval_sdf(const double* pts, long long n, double* out) {
  join();
  if (n <= 0) return;
  double *dp = nullptr, *dout = nullptr;
  CK(cudaMallocAsync((void**)&dp, n * 24, stream));
  CK(cudaMallocAsync((void**)&dout, n * 8, stream));
  CK(cudaMemcpyAsync(dp, pts, n * 24, cudaMemcpyHostToDevice, stream));
  k_eval_sdf<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(d, dp, dout, n);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, dout, n * 8, cudaMemcpyDeviceToHost, stream));
  CK(cudaFreeAsync(dp, stream));
  CK(cudaFreeAsync(dout, stream));
  CK(cudaStreamSynchronize(stream));
}

// ------------------------------------------------------------------------------------ Tank
Tank::Tank(const TankConfig& c) : cfg(c) {
  if (cfg.nx < 2 || cfg.ny < 2 || cfg.nz < 2 || !(cfg.h > 0)) throw Error(-1, "grid must be at least 2×2×2 with h > 0");
  if ((long long)cfg.nx * cfg.ny * cfg.nz > (1LL << 30)) throw Error(-1, "grid too large");
  if (cfg.cap < 1) throw Error(-1, "capacity must be positive");
  CK(cudaSetDevice(cfg.device));
  if (cfg.stream) { stream = cfg.stream; own_stream = false; }
  else CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&ev_own, cudaEventDisableTiming));
  TankDev& D = d;
  D.nx = cfg.nx; D.ny = cfg.ny; D.nz = cfg.nz; D.hx = (cfg.nx + 1) / 2;
  D.sx = cfg.nx + 1; D.sxy = (cfg.nx + 1) * (cfg.ny + 1);
  D.dnx = make_divu(D.nx); D.dny = make_divu(D.ny); D.dhx = make_divu(D.hx);
  D.dsx = make_divu(D.sx); D.dsxy = make_divu(D.sxy);
  D.nnodes = (cfg.nx + 1) * (cfg.ny + 1) * (cfg.nz + 1);
  D.ncells = cfg.nx * cfg.ny * cfg.nz;
  D.nhalf = D.hx * cfg.ny * cfg.nz;
  D.nyl = std::max(cfg.nyl, cfg.ny);
  D.h = cfg.h; D.ox = cfg.origin[0]; D.oy = cfg.origin[1]; D.oz = cfg.origin[2];
  D.rim = cfg.ny * cfg.h;
  D.g = cfg.g; D.flip = cfg.flip; D.friction = cfg.friction; D.ppc = cfg.ppc; D.drift = cfg.drift; D.ww_rate = cfg.ww_rate;
  D.dt = 1.0 / 60;
  D.vp = pow(cfg.h / 2, 3);
  D.drop_mass = 998.0 * pow(0.5 * cfg.h, 3.0);
  D.omega = (float)cfg.omega;
  D.iters = cfg.iters; D.whitewater = cfg.whitewater;
  D.sdf_mode = cfg.sdf_mode;
  D.seed = cfg.seed;
  D.advect = cfg.advect;
  D.drop_d_median = cfg.drop_d_median; D.drop_d_sigma = cfg.drop_d_sigma;
  D.cap = (int)cfg.cap;
  emit_cap = cfg.cap;
  D.emit_cap = (int)emit_cap;
  D.ww_cap = (int)std::max(1LL, cfg.ww_cap);
  D.rx = std::max(0, cfg.rx); D.rz = std::max(0, cfg.rz);
  const size_t nn = D.nnodes, nc = D.ncells, nh = D.nhalf, cap = cfg.cap;
  D.pA = (float4*)alloc(cap * 16); D.vA = (float4*)alloc(cap * 16);
  D.pE = (float4*)alloc(emit_cap * 16); D.vE = (float4*)alloc(emit_cap * 16);
  D.pB = (float4*)alloc(cap * 16); D.vB = (float4*)alloc(cap * 16);
  D.rank = (uint32_t*)alloc((cap + emit_cap) * 4);
  D.cnt = (int*)alloc((nc + 1) * 4);
  D.off = (int*)alloc((nc + 2) * 4);
  D.acc = (long long*)alloc(6 * nn * 8);
  D.vel = (float4*)alloc(nn * 16); D.velold = (float4*)alloc(nn * 16);
  D.frac = (float4*)alloc(nn * 16); D.svel = (float4*)alloc(nn * 16);
  D.fracd = (double*)alloc(3 * nn * 8); D.flux = (double*)alloc(3 * nn * 8);
  D.near = (uint8_t*)alloc(nc);
  CK(cudaMemsetAsync(D.near, 3, nc, stream));      // test obstacles and drains until the geometry pass builds it
  D.vv = (float2*)alloc(3 * nn * 8);
  D.pres = (float*)alloc(2 * nh * 4); D.rhs = (float*)alloc(2 * nh * 4); D.code = (uint32_t*)alloc(2 * nh * 4);
  D.pres2 = (float*)alloc(2 * nh * 4);
  D.act = (int4*)alloc(2 * nh * 16);
  d_objs = (Obj*)alloc(kMaxObj * sizeof(Obj));
  D.objs = d_objs;
  D.ctr = (Counters*)alloc(sizeof(Counters));
  D.wpos = (float4*)alloc(2 * (size_t)D.ww_cap * 16); D.wvel = (float4*)alloc(2 * (size_t)D.ww_cap * 16);
  if (D.rx > 0) D.rsrc = (long long*)alloc((size_t)(D.rx + 1) * (D.rz + 1) * 8);
  h_ctr = new Counters();          // read back with a synchronised copy: host memory needs no pinning
  CK(cudaStreamSynchronize(stream));
  solo = new Group({this}, stream);
}

Tank::~Tank() {
  delete solo;
  cudaSetDevice(cfg.device);
  if (stream) cudaStreamSynchronize(stream);
  for (void* p : dmem) cudaFreeAsync(p, stream);
  if (d_stage) cudaFreeAsync(d_stage, stream);
  if (d_rcnt) cudaFreeAsync(d_rcnt, stream);
  if (stream) cudaStreamSynchronize(stream);
  if (snap.p) { cudaFree(snap.p); cudaFree(snap.v); cudaFree(snap.wp); cudaFree(snap.wv); cudaFree(snap.pres); cudaFree(snap.ripple); }
  free_ripple(*this);
  free_mesh(*this);
  delete h_ctr;
  for (int k = 0; k < 2; ++k) {
    pinned_put(h_stage[k], stage_cap[k]);
    if (stage_ev[k]) cudaEventDestroy(stage_ev[k]);
  }
  if (copy_ev) cudaEventDestroy(copy_ev);
  pinned_put(h_poll, sizeof(Counters));
  pinned_put(h_read_p, read_cap * 16);
  pinned_put(h_read_v, read_cap * 16);
  pinned_put(h_rcount, sizeof(int));
  for (cudaEvent_t e : read_ev) cudaEventDestroy(e);
  if (poll_ev) cudaEventDestroy(poll_ev);
  if (ev_own) cudaEventDestroy(ev_own);
  if (stream && own_stream) cudaStreamDestroy(stream);
}

void Tank::join() {
  if (dep) {
    CK(cudaStreamWaitEvent(stream, dep, 0));
    dep = nullptr;
  }
  dirty = true;
}

namespace {
std::mutex g_pin_m;
std::map<size_t, std::vector<void*>> g_pin_free;
size_t g_pin_cached = 0;
constexpr size_t kPinCacheMax = 2ull << 30;
size_t pin_class(size_t b) {
  size_t c = 4096;
  while (c < b) c <<= 1;
  return c;
}
}  // namespace

void* pinned_get(size_t bytes, size_t* got) {
  const size_t c = pin_class(bytes);
  if (got) *got = c;
  {
    std::lock_guard<std::mutex> g(g_pin_m);
    auto it = g_pin_free.find(c);
    if (it != g_pin_free.end() && !it->second.empty()) {
      void* p = it->second.back();
      it->second.pop_back();
      g_pin_cached -= c;
      return p;
    }
  }
  void* p = nullptr;
  CK(cudaHostAlloc(&p, c, cudaHostAllocPortable));
  return p;
}

bool host_pinned(const void* p, size_t bytes) {
  if (!p || !bytes) return false;
  for (const char* q : {(const char*)p, (const char*)p + bytes - 1}) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (a.type != cudaMemoryTypeHost) return false;
  }
  return true;
}

void pinned_put(void* p, size_t bytes) {
  if (!p) return;
  const size_t c = pin_class(bytes);
  {
    std::lock_guard<std::mutex> g(g_pin_m);
    if (g_pin_cached + c <= kPinCacheMax) {
      g_pin_free[c].push_back(p);
      g_pin_cached += c;
      return;
    }
  }
  cudaFreeHost(p);
}

size_t tank_bytes(const TankConfig& c) {
  const size_t nn = (size_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1), nc = (size_t)c.nx * c.ny * c.nz;
  const size_t nh = (size_t)((c.nx + 1) / 2) * c.ny * c.nz, cap = (size_t)c.cap;
  size_t b = cap * 16 * 6 + cap * 2 * 4;                      // A, E, B (pos, vel), ranks
  b += (nc + 1) * 4 + (nc + 2) * 4;                           // counts, offsets
  b += nn * (6 * 8 + 4 * 16 + 2 * 3 * 8 + 3 * 8);            // accumulator, vel/velold/frac/svel, fracd/flux, vv
  b += nc;                                                    // obstacle reach per cell
  b += 2 * nh * 32;                                           // pressure (two buffers), rhs, code, active lists
  b += kMaxObj * sizeof(Obj) + sizeof(Counters) + kMaxEmitters * sizeof(EmitterDev);
  b += 2 * (size_t)std::max(1LL, c.ww_cap) * 32;
  if (c.rx > 0) {
    const size_t nv = (size_t)(c.rx + 1) * (c.rz + 1), W = (size_t)c.wmap;
    b += nv * 8 + nv * 20 + (size_t)(2 * c.rx) * (2 * c.rz) * 16 + W * W * 28 + (size_t)(2 * c.rx + 2 * c.rz) * 8;
    if (c.ripple_depth > 0) b += (size_t)(2 * c.rx) * (2 * c.rz) * 40;   // the fixed-depth update per mode
  }
  return b + (64 << 10) * 24;                                 // allocation granularity
}

// Tank memory comes from the device's stream-ordered pool, which keeps freed blocks for reuse (release
// threshold raised once per device): scenes that come and go (serving) then cost no driver allocation.
void* Tank::alloc(size_t bytes) {
  static std::once_flag once[128];
  const int dev = cfg.device;
  if (dev >= 0 && dev < 128)
    std::call_once(once[dev], [dev] {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        unsigned long long keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
    });
  void* p = nullptr;
  CK(cudaMallocAsync(&p, std::max<size_t>(bytes, 16), stream));
  dmem.push_back(p);
  CK(cudaMemsetAsync(p, 0, std::max<size_t>(bytes, 16), stream));
  return p;
}

void Tank::set_objects(const std::vector<Obj>& o) {
  join();
  if (o.size() > (size_t)kMaxObj) throw Error(-1, "at most 64 obstacles and drains");
  objs = o;
  d.nobj = (int)objs.size();
  d.has_obst = 0;
  d.moving = 0;
  for (const Obj& x : objs)
    if (x.flag == 1) {
      d.has_obst = 1;
      for (int a = 0; a < 3; ++a)
        if (x.lin[a] != 0.0 || x.ang[a] != 0.0) d.moving = 1;
    }
  if (d.sdf_mode == kSdfLattice && d_lattice) d.has_obst = 1;
  if (!objs.empty()) CK(cudaMemcpyAsync(d_objs, objs.data(), objs.size() * sizeof(Obj), cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  geom_dirty = true;
  ++version;
}

void Tank::set_lattice(const double* sdf, const int* oid, int lx, int ly, int lz) {
  join();
  if (lx != 2 * d.nx + 1 || lz != 2 * d.nz + 1 || ly < 2 * d.ny + 1 || (ly - 1) % 2)
    throw Error(-1, "lattice must be (2nx+1) × (2nyl+1) × (2nz+1) with nyl >= ny");
  d.nyl = (ly - 1) / 2;
  const size_t n = (size_t)lx * ly * lz;
  if (!d_lattice) { d_lattice = (double*)alloc(n * 8); d_oid = (int*)alloc(n * 4); }
  CK(cudaMemcpyAsync(d_lattice, sdf, n * 8, cudaMemcpyHostToDevice, stream));
  if (oid) CK(cudaMemcpyAsync(d_oid, oid, n * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  d.lattice = d_lattice;
  d.oid = oid ? d_oid : nullptr;
  d.sdf_mode = kSdfLattice;
  bool any = false;
  for (const Obj& x : objs) any |= x.flag == 1;
  d.has_obst = 1;
  (void)any;
  geom_dirty = true;
  ++version;
}

void Tank::read_counters() {
  join();
  CK(cudaMemcpyAsync(h_ctr, d.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  n_upper = h_ctr->n_live + h_ctr->n_emit;
}

bool Tank::poll_counters(Counters& out) {
  join();
  bool fresh = false;
  if (poll_pending) {
    const cudaError_t q = cudaEventQuery(poll_ev);
    if (q == cudaSuccess) {
      out = *h_poll;
      fresh = true;
      poll_pending = false;
    } else if (q != cudaErrorNotReady) {
      CK(q);
    }
  }
  if (!poll_pending) {
    if (!h_poll) {
      h_poll = (Counters*)pinned_get(sizeof(Counters));
      CK(cudaEventCreateWithFlags(&poll_ev, cudaEventDisableTiming));
    }
    CK(cudaMemcpyAsync(h_poll, d.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, stream));
    CK(cudaEventRecord(poll_ev, stream));
    poll_pending = true;
  }
  return fresh;
}

// n packed particles (positions, then velocities and marks where given) copied to d_stage are unpacked into E
// after the particles staged before them
void Tank::unpack_staged(long long n, bool has_vel, bool has_air) {
  const float* pos = reinterpret_cast<const float*>(d_stage);
  const float* vel = has_vel ? pos + 3 * n : nullptr;
  const float* air = has_air ? pos + (has_vel ? 6 : 3) * n : nullptr;
  k_unpack_added<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(d.pE + n_emit_host, d.vE + n_emit_host, pos, vel,
                                                                   air, (int)n, next_id);
  n_emit_host += n;
  k_set_emit<<<1, 1, 0, stream>>>(d.ctr, (int)n_emit_host);
  CK(cudaGetLastError());
  n_upper += n;
}

void Tank::ensure_d_stage(size_t bytes) {
  if (bytes <= d_stage_cap) return;
  if (d_stage) CK(cudaFreeAsync(d_stage, stream));
  d_stage_cap = bytes;
  CK(cudaMallocAsync((void**)&d_stage, d_stage_cap, stream));
}

void Tank::add_particles(const float* pos, const float* vel, const float* air, long long n, uint32_t* first) {
  join();
  if (n < 0 || (n > 0 && !pos)) throw Error(-1, "add_particles: bad arrays");
  if (first) *first = next_id;
  if (n == 0) return;
  long long room = std::min<long long>(cfg.cap - n_upper, emit_cap - n_emit_host);
  if (n > room) {
    read_counters();
    room = std::min<long long>(cfg.cap - n_upper, emit_cap - n_emit_host);
  }
  long long take = std::max(0LL, std::min(n, room));
  const size_t bp = (size_t)take * 12, bv = vel ? bp : 0, ba = air ? (size_t)take * 4 : 0;
  if (take > 0 && host_pinned(pos, bp) && (!vel || host_pinned(vel, bv)) && (!air || host_pinned(air, ba)) &&
      cudaStreamQuery(stream) == cudaSuccess) {
    // page-locked arrays and nothing queued on the tank's stream: the copy engine reads them directly, and
    // the call returns once it has (the caller may then reuse them)
    ensure_d_stage(bp + bv + ba);
    CK(cudaMemcpyAsync(d_stage, pos, bp, cudaMemcpyHostToDevice, stream));
    if (vel) CK(cudaMemcpyAsync(d_stage + bp, vel, bv, cudaMemcpyHostToDevice, stream));
    if (air) CK(cudaMemcpyAsync(d_stage + bp + bv, air, ba, cudaMemcpyHostToDevice, stream));
    if (!copy_ev) CK(cudaEventCreateWithFlags(&copy_ev, cudaEventDisableTiming));
    CK(cudaEventRecord(copy_ev, stream));
    unpack_staged(take, vel != nullptr, air != nullptr);
    CK(cudaEventSynchronize(copy_ev));
  } else if (take > 0) {
    // two pinned staging buffers in turn: a buffer is refilled once the copy out of it two calls ago has
    // finished (an event, not a wait for the whole stream, so the host stays ahead of the device)
    const int k = stage_k;
    stage_k ^= 1;
    if (stage_ev[k]) CK(cudaEventSynchronize(stage_ev[k]));
    else CK(cudaEventCreateWithFlags(&stage_ev[k], cudaEventDisableTiming));
    if (bp + bv + ba > stage_cap[k]) {
      pinned_put(h_stage[k], stage_cap[k]);
      h_stage[k] = nullptr;
      stage_cap[k] = 0;
      h_stage[k] = (unsigned char*)pinned_get(bp + bv + ba, &stage_cap[k]);
    }
    memcpy(h_stage[k], pos, bp);
    if (vel) memcpy(h_stage[k] + bp, vel, bv);
    if (air) memcpy(h_stage[k] + bp + bv, air, ba);
    ensure_d_stage(bp + bv + ba);
    CK(cudaMemcpyAsync(d_stage, h_stage[k], bp + bv + ba, cudaMemcpyHostToDevice, stream));
    CK(cudaEventRecord(stage_ev[k], stream));
    unpack_staged(take, vel != nullptr, air != nullptr);
  }
  next_id += (uint32_t)take;
  if (take < n) {
    h_ctr->full = 1;
    throw Error(-4, "particle capacity reached: " + std::to_string(take) + " of " + std::to_string(n) + " added");
  }
}

namespace {
void launch_emit(Tank& t, std::vector<EmitRec>& recs) {
  if (recs.empty()) return;
  int total = 0;
  for (auto& r : recs) { r.base = (int)t.n_emit_host + total; total += r.count; }
  EmitRec* d_recs = nullptr;
  CK(cudaMallocAsync((void**)&d_recs, recs.size() * sizeof(EmitRec), t.stream));
  CK(cudaMemcpyAsync(d_recs, recs.data(), recs.size() * sizeof(EmitRec), cudaMemcpyHostToDevice, t.stream));
  k_emit<<<(total + 255) / 256, 256, 0, t.stream>>>(t.d, d_recs, (int)recs.size(), total);
  CK(cudaGetLastError());
  CK(cudaFreeAsync(d_recs, t.stream));
  CK(cudaStreamSynchronize(t.stream));     // recs lives on the host stack
  t.n_emit_host += total;
  k_set_emit<<<1, 1, 0, t.stream>>>(t.d.ctr, (int)t.n_emit_host);
  CK(cudaGetLastError());
  t.n_upper += total;
}

// budget like writeEmits (src/js/50-sim.js:222-246): room = cap - count - 64
int clip_to_room(Tank& t, std::vector<EmitRec>& recs) {
  long long room = std::min<long long>(t.cfg.cap - t.n_upper - 64, t.emit_cap - t.n_emit_host);
  bool full = false;
  for (auto& r : recs) {
    if (r.count > room) { r.count = (int)std::max(0LL, room); full = true; }
    room -= r.count;
  }
  recs.erase(std::remove_if(recs.begin(), recs.end(), [](const EmitRec& r) { return r.count <= 0; }), recs.end());
  if (full) t.h_ctr->full = 1;
  return full;
}
}  // namespace

void Tank::count_pass() {
  join();
  solo->ensure_uploaded();
  launch_begin_count(solo->ctx);
  launch_bin_count(solo->ctx);
  launch_scan(solo->ctx);
  CK(cudaGetLastError());
}

void Tank::emit_block(const double lo_in[3], const double hi_in[3], bool fill) {
  join();
  // blockEmits (src/js/55-emit.js:83-106) / emit_block (solver.py:317-343)
  const double sp = d.h / 2;
  double lo[3] = {lo_in[0], lo_in[1], lo_in[2]}, hi[3] = {hi_in[0], hi_in[1], hi_in[2]};
  const double tlo[3] = {d.ox + sp * 0.5, 0.0005, d.oz + sp * 0.5};
  const double thi[3] = {-d.ox - sp * 0.5, INFINITY, -d.oz - sp * 0.5};
  if (lo[0] < thi[0] && hi[0] > tlo[0] && lo[2] < thi[2] && hi[2] > tlo[2]) {
    for (int k : {0, 2}) { lo[k] = std::max(lo[k], tlo[k]); hi[k] = std::min(hi[k], thi[k]); }
    lo[1] = std::max(lo[1], tlo[1]);
  }
  long long n[3];
  for (int k = 0; k < 3; ++k) n[k] = (long long)std::max(0.0, floor((hi[k] - lo[k]) / sp));
  const long long total = n[0] * n[1] * n[2];
  if (total <= 0) return;
  if (fill) count_pass();
  EmitRec r{};
  r.shape = 2;
  for (int k = 0; k < 3; ++k) r.a[k] = lo[k] + ((hi[k] - lo[k]) - n[k] * sp) / 2;
  r.a[3] = sp;
  r.b[0] = (double)n[0]; r.b[1] = (double)n[1]; r.b[2] = (double)n[2]; r.b[3] = fill ? 1.0 : 0.0;
  r.count = (int)std::min<long long>(total, 1LL << 30);
  r.seed = hash_host(cfg.seed * 2654435761u + next_id * 40503u + 7u);
  r.first_id = next_id;
  std::vector<EmitRec> recs{r};
  const bool full = clip_to_room(*this, recs);
  if (!recs.empty()) {
    next_id += (uint32_t)recs[0].count;
    launch_emit(*this, recs);
  }
  if (full) throw Error(-4, "particle capacity reached while filling a water block");
}

void Tank::source_emits(double dt) {
  join();
  // sourceEmits (src/js/55-emit.js:13-69): per source an accumulator of volume, drop timers, bursts, rain
  if (scene.sources.empty()) return;
  const double Vp = d.vp, DEG = M_PI / 180.0, RAIN_SPEED = 6.5;
  std::vector<EmitRec> recs;
  auto clampd = [](double x, double a, double b) { return std::min(std::max(x, a), b); };
  auto jround = [](double x) { return floor(x + 0.5); };     // JavaScript Math.round
  for (const SourceItem& src : scene.sources) {
    if (!src.enabled) continue;
    std::vector<double>& st = emit_state[src.id];
    if (st.empty()) st.assign(4, 0.0);       // acc, liters, timer, fired
    if (src.total > 0 && st[1] >= src.total) continue;
    const double p = src.pitch * DEG, y = src.yaw * DEG;
    const double dir[3] = {cos(p) * sin(y), sin(p), cos(p) * cos(y)};
    const double ref[3] = {fabs(dir[1]) < 0.95 ? 0.0 : 1.0, fabs(dir[1]) < 0.95 ? 1.0 : 0.0, 0.0};
    double u[3] = {dir[1] * ref[2] - dir[2] * ref[1], dir[2] * ref[0] - dir[0] * ref[2], dir[0] * ref[1] - dir[1] * ref[0]};
    const double ul = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    for (double& c : u) c /= ul;
    const double w[3] = {dir[1] * u[2] - dir[2] * u[1], dir[2] * u[0] - dir[0] * u[2], dir[0] * u[1] - dir[1] * u[0]};
    EmitRec r{};
    r.seed = hash_host(cfg.seed * 2654435761u + (uint32_t)src.id * 97u + (uint32_t)(h_ctr->frame + 1) * 7919u + (uint32_t)recs.size());
    r.first_id = 0;
    if (src.mode == "stream" || src.mode == "shower") {
      const double Q = src.flow / 60000;
      st[0] += (Q * dt) / Vp;
      const double n = floor(st[0]);
      st[0] -= n;
      if (n <= 0) continue;
      const bool shower = src.mode == "shower";
      const double noz = sqrt(4 * Q / (M_PI * std::max(src.speed, 0.05)));
      const double rr = shower ? std::max(noz / 2, 0.022) : std::max(noz / 2, 0.0005);
      const double spread = shower ? clampd(src.spread, 0, 80) * DEG : 0;
      r.shape = 0;
      for (int k = 0; k < 3; ++k) { r.a[k] = src.pos[k] + dir[k] * 0.002; r.b[k] = dir[k]; r.c[k] = u[k]; r.d[k] = w[k]; }
      r.a[3] = rr; r.b[3] = src.speed; r.c[3] = spread; r.d[3] = src.speed * dt;
      r.count = (int)n;
      st[1] += n * Vp * 1000;
    } else if (src.mode == "drops") {
      st[2] -= dt;
      if (st[2] > 0) continue;
      st[2] += 1 / clampd(src.drop_rate, 0.05, 60);
      if (st[2] < 0) st[2] = 0;
      const double dd = clampd(src.drop_d, 1, 40) / 1000;
      const double V = M_PI / 6 * dd * dd * dd;
      const double n = std::max(1.0, jround(V / Vp));
      const double R = std::max(dd / 2, cbrt((3 * n * Vp) / (4 * M_PI)) * 0.9);
      r.shape = 1;
      for (int k = 0; k < 3; ++k) { r.a[k] = src.pos[k] + dir[k] * (R + 0.002); r.b[k] = dir[k] * src.speed; }
      r.a[3] = n == 1 ? 0 : R; r.b[3] = n <= 8 ? 1 : 0;
      r.count = (int)n;
      st[1] += n * Vp * 1000;
    } else if (src.mode == "burst") {
      if (st[3] != 0) {
        if (!(src.burst_every > 0)) continue;
        st[2] -= dt;
        if (st[2] > 0) continue;
      }
      st[3] = 1;
      st[2] = src.burst_every > 0 ? src.burst_every : 0;
      const double V = clampd(src.burst, 0.01, 50) / 1000;
      const double n = std::max(1.0, jround(V / Vp));
      const double R = cbrt((3 * V) / (4 * M_PI));
      r.shape = 1;
      for (int k = 0; k < 3; ++k) { r.a[k] = src.pos[k] + dir[k] * (R + 0.004); r.b[k] = dir[k] * src.speed; }
      r.a[3] = R; r.b[3] = 0;
      r.count = (int)n;
      st[1] += n * Vp * 1000;
    } else if (src.mode == "rain") {
      const double side = clampd(src.rain_size, 0.05, 2);
      const double flux = (clampd(src.rain_rate, 1, 500) / 3.6e6) * side * side;
      st[0] += (flux * dt) / Vp;
      const double n = floor(st[0]);
      st[0] -= n;
      if (n <= 0) continue;
      r.shape = 3;
      for (int k = 0; k < 3; ++k) r.a[k] = src.pos[k];
      r.a[3] = side / 2;
      r.b[0] = 0; r.b[1] = -RAIN_SPEED; r.b[2] = 0;
      r.d[3] = RAIN_SPEED * dt;
      r.count = (int)n;
      st[1] += n * Vp * 1000;
    } else {
      continue;
    }
    recs.push_back(r);
  }
  if (recs.empty()) return;
  clip_to_room(*this, recs);
  for (EmitRec& r : recs) { r.first_id = next_id; next_id += (uint32_t)r.count; }
  launch_emit(*this, recs);
}

void Tank::clear() {
  join();
  // clearWater (src/js/50-sim.js:365-373)
  CK(cudaStreamSynchronize(stream));
  CK(cudaMemsetAsync(d.ctr, 0, sizeof(Counters), stream));
  CK(cudaMemsetAsync(d.pres, 0, 2 * (size_t)d.nhalf * 4, stream));
  if (d.rsrc) CK(cudaMemsetAsync(d.rsrc, 0, (size_t)(d.rx + 1) * (d.rz + 1) * 8, stream));
  clear_ripple(*this);
  CK(cudaStreamSynchronize(stream));
  memset(h_ctr, 0, sizeof(Counters));
  n_emit_host = 0; n_upper = 0; time = 0; vmax = 1.0;
  emit_state.clear();
}

void Tank::reset() {
  // restartWater (src/js/90-main.js:15-19): clear, objects again, refill the water blocks
  clear();
  for (const WaterBlock& b : scene.blocks) emit_block(b.lo, b.hi, false);
}

void Tank::substep(double dt) {
  join();
  solo->use_graphs = use_graphs;
  solo->substep(dt);
}

int Tank::step(double frame_dt) {
  join();
  if (!(frame_dt > 0)) return 0;
  read_counters();
  if (h_ctr->vmax_bits64 != 0ull) {
    const unsigned long long b = h_ctr->vmax_bits64 - 1ull;
    double v;
    memcpy(&v, &b, 8);
    vmax = v;
  }
  const double vm = std::max(vmax, 0.4);
  const int n = (int)std::min(std::max(ceil(frame_dt / (1.4 * d.h / vm)), 1.0), 6.0);
  const double dt = frame_dt / n;
  for (int s = 0; s < n; ++s) {
    source_emits(dt);
    substep(dt);
  }
  frame_end(frame_dt);
  return n;
}

// the end of a frame after its sub-steps: cell counts, whitewater advance, top height and ripples
// (solver.py:720-728)
void Tank::frame_end(double frame_dt) {
  join();
  count_pass();
  if (d.whitewater) launch_whitewater(solo->ctx, frame_dt);
  ripple_frame(*this, frame_dt);
  CK(cudaGetLastError());
}

// Particles of A then E (the previous sub-step's output and the pending emissions), dead ones skipped, in that
// order: compacted on the device into the ABI layout (k_read_*), then the live count and as many particles as
// the caller takes are copied into pinned buffers kept by the tank, in chunks whose copy into the caller's
// arrays overlaps the transfer of the next.
long long Tank::read_particles(float* pos4, float* vel4, long long cap) {
  read_counters();
  const long long nl = h_ctr->n_live, ne = h_ctr->n_emit, tot = nl + ne;
  if (tot <= 0) return 0;
  if (tot > cfg.cap) throw Error(-2, "particle counters above the capacity");   // B holds the compacted copy
  const int nb = (int)((tot + kReadTile - 1) / kReadTile);
  if ((size_t)nb + 1 > rcnt_cap) {
    if (d_rcnt) CK(cudaFreeAsync(d_rcnt, stream));
    rcnt_cap = (size_t)nb + 1;
    CK(cudaMallocAsync((void**)&d_rcnt, rcnt_cap * sizeof(int), stream));
  }
  if (!h_rcount) h_rcount = (int*)pinned_get(sizeof(int));
  const bool want_p = pos4 != nullptr && cap > 0, want_v = vel4 != nullptr && cap > 0;
  k_read_count<<<nb, kReadThreads, 0, stream>>>(d.pA, d.pE, (int)nl, (int)tot, d_rcnt);
  k_read_scan<<<1, 1024, 0, stream>>>(d_rcnt, nb);
  if (want_p || want_v)
    k_read_write<<<nb, kReadThreads, 0, stream>>>(d.pA, d.vA, d.pE, d.vE, (int)nl, (int)tot, d_rcnt, d.pB,
                                                  want_v ? d.vB : nullptr);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h_rcount, d_rcnt + nb, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  const long long k = *h_rcount, m = std::min(k, want_p || want_v ? cap : 0LL);
  if (m <= 0) return k;
  // caller arrays in page-locked memory: the copy engine writes them directly
  if ((!want_p || host_pinned(pos4, (size_t)m * 16)) && (!want_v || host_pinned(vel4, (size_t)m * 16))) {
    if (want_p) CK(cudaMemcpyAsync(pos4, d.pB, (size_t)m * 16, cudaMemcpyDeviceToHost, stream));
    if (want_v) CK(cudaMemcpyAsync(vel4, d.vB, (size_t)m * 16, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return k;
  }
  if ((size_t)m > read_cap) {
    pinned_put(h_read_p, read_cap * 16);
    pinned_put(h_read_v, read_cap * 16);
    h_read_p = h_read_v = nullptr;
    read_cap = 0;
    size_t got = 0;
    h_read_p = (float4*)pinned_get((size_t)m * 16, &got);
    h_read_v = (float4*)pinned_get((size_t)m * 16);
    read_cap = got / 16;
  }
  constexpr long long kChunk = 1 << 20;
  const int nch = (int)((m + kChunk - 1) / kChunk);
  while ((int)read_ev.size() < nch) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    read_ev.push_back(e);
  }
  for (int c = 0; c < nch; ++c) {
    const long long a = c * kChunk, n = std::min(kChunk, m - a);
    if (want_p) CK(cudaMemcpyAsync(h_read_p + a, d.pB + a, n * 16, cudaMemcpyDeviceToHost, stream));
    if (want_v) CK(cudaMemcpyAsync(h_read_v + a, d.vB + a, n * 16, cudaMemcpyDeviceToHost, stream));
    CK(cudaEventRecord(read_ev[c], stream));
  }
  for (int c = 0; c < nch; ++c) {
    const long long a = c * kChunk, n = std::min(kChunk, m - a);
    CK(cudaEventSynchronize(read_ev[c]));
    if (want_p) memcpy(pos4 + 4 * a, h_read_p + a, n * 16);
    if (want_v) memcpy(vel4 + 4 * a, h_read_v + a, n * 16);
  }
  return k;
}

long long Tank::read_whitewater(float* pos4, float* vel4, long long cap) {
  read_counters();
  const long long n = std::min<long long>(h_ctr->ww_count, d.ww_cap);
  const size_t half = (h_ctr->ww_cur & 1) ? (size_t)d.ww_cap : 0;
  const long long k = std::min(n, cap);
  if (k > 0) {
    if (pos4) CK(cudaMemcpyAsync(pos4, d.wpos + half, k * 16, cudaMemcpyDeviceToHost, stream));
    if (vel4) CK(cudaMemcpyAsync(vel4, d.wvel + half, k * 16, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }
  return n;
}

void Tank::add_whitewater(const float* pos4, const float* vel4, long long n) {
  if (n < 0 || (n > 0 && (!pos4 || !vel4))) throw Error(-1, "add_whitewater: bad arrays");
  read_counters();
  const long long cur = std::min<long long>(h_ctr->ww_count, d.ww_cap);
  const long long take = std::min<long long>(n, d.ww_cap - cur);
  const size_t half = (h_ctr->ww_cur & 1) ? (size_t)d.ww_cap : 0;
  if (take > 0) {
    CK(cudaMemcpyAsync(d.wpos + half + cur, pos4, take * 16, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(d.wvel + half + cur, vel4, take * 16, cudaMemcpyHostToDevice, stream));
    const int count = (int)(cur + take);
    CK(cudaMemcpyAsync(&d.ctr->ww_count, &count, sizeof(int), cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    h_ctr->ww_count = count;
  }
  if (take < n) throw Error(-4, "whitewater capacity reached: " + std::to_string(take) + " of " + std::to_string(n) + " added");
}

void Tank::read_grid(int field, void* out, size_t bytes) {
  join();
  const size_t nn = d.nnodes, nc = d.ncells;
  auto need = [&](size_t b) { if (bytes < b) throw Error(-1, "read_grid: output buffer too small (" + std::to_string(b) + " bytes needed)"); };
  CK(cudaStreamSynchronize(stream));
  if (field == 0) {
    need(nc * 4);
    std::vector<int> off(nc + 2);
    CK(cudaMemcpy(off.data(), d.off, (nc + 2) * 4, cudaMemcpyDeviceToHost));
    int* o = (int*)out;
    for (size_t c = 0; c < nc; ++c) o[c] = off[c + 1] - off[c];
  } else if (field >= 1 && field <= 4) {
    const float4* src = field == 1 ? d.frac : (field == 2 ? d.vel : d.velold);
    std::vector<float4> v(nn);
    CK(cudaMemcpy(v.data(), src, nn * 16, cudaMemcpyDeviceToHost));
    if (field == 4) {
      need(3 * nn);
      uint8_t* o = (uint8_t*)out;
      for (size_t n = 0; n < nn; ++n) {
        const int m = (int)v[n].w;
        for (int a = 0; a < 3; ++a) o[a * nn + n] = (m >> a) & 1;
      }
    } else {
      need(3 * nn * 4);
      float* o = (float*)out;
      for (size_t n = 0; n < nn; ++n) { o[n] = v[n].x; o[nn + n] = v[n].y; o[2 * nn + n] = v[n].z; }
    }
  } else if (field == 5 || field == 6) {
    need(nc * 4);
    std::vector<float> h(2 * (size_t)d.nhalf);
    CK(cudaMemcpy(h.data(), field == 5 ? d.pres : d.rhs, h.size() * 4, cudaMemcpyDeviceToHost));
    float* o = (float*)out;
    for (int k = 0; k < d.nz; ++k)
      for (int j = 0; j < d.ny; ++j)
        for (int i = 0; i < d.nx; ++i) {
          const size_t c = i + (size_t)d.nx * (j + (size_t)d.ny * k);
          const size_t s = (size_t)((i + j + k) & 1) * d.nhalf + (i >> 1) + (size_t)d.hx * (j + (size_t)d.ny * k);
          o[c] = h[s];
        }
  } else {
    read_ripple_field(*this, field, out, bytes);
  }
}

int Tank::snapshot() {
  // saveWater (src/js/50-sim.js:111-125)
  read_counters();
  const size_t cap = cfg.cap;
  if (!snap.p) {
    CK(cudaMalloc(&snap.p, cap * 16)); CK(cudaMalloc(&snap.v, cap * 16));
    CK(cudaMalloc(&snap.wp, 2 * (size_t)d.ww_cap * 16)); CK(cudaMalloc(&snap.wv, 2 * (size_t)d.ww_cap * 16));
    CK(cudaMalloc(&snap.pres, 2 * (size_t)d.nhalf * 4));
    snap.ripple_bytes = ripple_state_bytes(*this);
    if (snap.ripple_bytes) CK(cudaMalloc(&snap.ripple, snap.ripple_bytes));
  }
  // pending emissions are kept by folding them into the copy: copy A then E behind it
  const long long nl = h_ctr->n_live, ne = h_ctr->n_emit;
  if (nl + ne > (long long)cap) throw Error(-4, "snapshot: more particles than capacity");
  CK(cudaMemcpyAsync(snap.p, d.pA, nl * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(snap.v, d.vA, nl * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(snap.p + nl, d.pE, ne * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(snap.v + nl, d.vE, ne * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(snap.wp, d.wpos, 2 * (size_t)d.ww_cap * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(snap.wv, d.wvel, 2 * (size_t)d.ww_cap * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(snap.pres, d.pres, 2 * (size_t)d.nhalf * 4, cudaMemcpyDeviceToDevice, stream));
  if (snap.ripple_bytes) copy_ripple_state(*this, snap.ripple, true);
  CK(cudaStreamSynchronize(stream));
  snap.ctr = *h_ctr;
  snap.ctr.n_live = (int)(nl + ne);
  snap.ctr.n_emit = 0;
  snap.n = nl + ne;
  snap.time = time; snap.vmax = vmax; snap.next_id = next_id;
  snap.emit_state = emit_state;
  static int serial = 0;
  snap.id = ++serial;
  snap.valid = true;
  return snap.id;
}

void Tank::restore(int id) {
  join();
  // restoreWater (src/js/50-sim.js:127-141): only the latest copy, once
  if (!snap.valid || snap.id != id) throw Error(-6, "no water copy with that id");
  CK(cudaStreamSynchronize(stream));
  CK(cudaMemcpyAsync(d.pA, snap.p, snap.n * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(d.vA, snap.v, snap.n * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(d.wpos, snap.wp, 2 * (size_t)d.ww_cap * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(d.wvel, snap.wv, 2 * (size_t)d.ww_cap * 16, cudaMemcpyDeviceToDevice, stream));
  CK(cudaMemcpyAsync(d.pres, snap.pres, 2 * (size_t)d.nhalf * 4, cudaMemcpyDeviceToDevice, stream));
  if (snap.ripple_bytes) copy_ripple_state(*this, snap.ripple, false);
  *h_ctr = snap.ctr;
  CK(cudaMemcpyAsync(d.ctr, h_ctr, sizeof(Counters), cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  n_emit_host = 0; n_upper = snap.n;
  time = snap.time; vmax = snap.vmax; next_id = snap.next_id;
  emit_state = snap.emit_state;
  snap.valid = false;
}

// ------------------------------------------------------------------------------------ Group
namespace {
int blocks_for(int fam, const TankDev& D) {
  switch (fam) {
    case kFamNodes: return (D.nnodes + kThreads - 1) / kThreads;
    case kFamCells: return (D.ncells + kThreads - 1) / kThreads;
    case kFamHalf: return (D.nhalf + kThreads - 1) / kThreads;
    case kFamBricks: return ((D.nx + kBrick - 1) / kBrick) * ((D.ny + kBrick - 1) / kBrick) * ((D.nz + kBrick - 1) / kBrick);
    case kFamScan: return (D.ncells + 1 + kScanTile - 1) / kScanTile;
    case kFamSor: return (D.nhalf + kSorThreads - 1) / kSorThreads;     // one active cell per thread at most
    case kFamTiles: return ((D.nx + kTbX - 1) / kTbX) * ((D.ny + kTbY - 1) / kTbY) * ((D.nz + kTbZ - 1) / kTbZ);
    case kFamG2P: return blocks_for(kFamBricks, D) + 1;       // the bricks and the particles outside the grid
  }
  return 0;
}
}  // namespace

Group::Group(const std::vector<Tank*>& t, cudaStream_t s, bool async_setup) : tanks(t) {
  if (tanks.empty()) throw Error(-1, "a batch needs at least one tank");
  device = tanks[0]->cfg.device;
  for (Tank* x : tanks)
    if (x->cfg.device != device) throw Error(-1, "all tanks of a batch must be on one device");
  CK(cudaSetDevice(device));
  if (s) { stream = s; } else { CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); own_stream = true; }
  CK(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
  if (async_setup) {
    CK(cudaStreamCreateWithFlags(&setup, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&setup_done, cudaEventDisableTiming));
  }
  const cudaStream_t q = async_setup ? setup : stream;   // where the tables are allocated and filled
  CK(sor_tb_prepare());
  const int n = (int)tanks.size();
  CK(cudaMallocAsync(&d_tanks, n * sizeof(TankDev), q));
  h_tanks = new TankDev[n];
  CK(cudaMallocAsync(&d_bpfx, kFamCount * (n + 1) * sizeof(int), q));
  CK(cudaMallocAsync(&d_ppfx, 2 * (n + 1) * sizeof(int), q));
  CK(cudaMemsetAsync(d_ppfx, 0, 2 * (n + 1) * sizeof(int), q));
  std::vector<int> pf(kFamCount * (n + 1));
  for (int f = 0; f < kFamCount; ++f) {
    int acc = 0;
    for (int i = 0; i < n; ++i) { pf[f * (n + 1) + i] = acc; acc += blocks_for(f, tanks[i]->d); }
    pf[f * (n + 1) + n] = acc;
    ctx.nblocks[f] = acc;
    ctx.bpfx[f] = d_bpfx + f * (n + 1);
  }
  CK(cudaMallocAsync(&d_bsum, std::max(1, ctx.nblocks[kFamScan]) * sizeof(long long), q));
  CK(cudaMemcpyAsync(d_bpfx, pf.data(), pf.size() * sizeof(int), cudaMemcpyHostToDevice, q));
  std::vector<int> hp(n + 1, 0);
  for (int i = 0; i < n; ++i) hp[i + 1] = hp[i] + tanks[i]->d.nhalf;
  CK(cudaMallocAsync(&d_hpfx, (n + 1) * sizeof(int), q));
  CK(cudaMallocAsync(&d_apfx, 2 * (n + 1) * sizeof(int), q));
  CK(cudaMemsetAsync(d_apfx, 0, 2 * (n + 1) * sizeof(int), q));
  CK(cudaMemcpyAsync(d_hpfx, hp.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, q));
  CK(cudaMallocAsync(&d_barrier, sizeof(GridBarrier), q));
  CK(cudaMemsetAsync(d_barrier, 0, sizeof(GridBarrier), q));
  CK(cudaMallocAsync(&d_ticket, 4 * sizeof(unsigned), q));
  CK(cudaMemsetAsync(d_ticket, 0, 4 * sizeof(unsigned), q));
  size_t defer_cap = 1;                 // G2P form 2: every particle of the group may be deferred
  for (Tank* x : tanks) defer_cap += (size_t)x->d.cap + (size_t)std::max(x->d.emit_cap, 0);
  CK(cudaMallocAsync(&d_defer, defer_cap * sizeof(int) + 16, q));
  // the persistent solve: one block of 1024 threads per SM at most, and no more blocks than ~4 cells a thread
  // (the grid barrier's cost grows with the number of arriving blocks); a batch shares the SMs among its lanes
  sor_blocks = std::min(std::min(sor_persist_max_blocks(device), sm_count), std::max(1, (2 * hp[n] + 4095) / 4096));
  if (async_setup) {
    CK(cudaEventRecord(setup_done, setup));
    CK(cudaStreamWaitEvent(stream, setup_done, 0));
  } else {
    CK(cudaStreamSynchronize(stream));
  }
  ctx.hpfx = d_hpfx;
  ctx.apfx = d_apfx;
  ctx.barrier = d_barrier;
  ctx.ticket = d_ticket;
  ctx.defer_n = d_defer;
  ctx.defer_list = d_defer + 4;
  ctx.stream = stream;
  ctx.tanks = d_tanks;
  ctx.ntanks = n;
  ctx.ppfx_in = d_ppfx;
  ctx.ppfx_sorted = d_ppfx + (n + 1);
  ctx.scan_bsum = d_bsum;
  ctx.particle_blocks = blocks_per_sm * sm_count;
  uploaded.assign(n, 0);
  for (Tank* x : tanks) watchdog_polls = std::min<unsigned>(watchdog_polls, (unsigned)x->cfg.watchdog_polls);
  // the solve form the first tank asks for; -1: cluster-resident where every tank fits, else per sweep
  const int want = tanks[0]->cfg.sor_mode;
  if (want == 4 || want == -1) {
    try {
      plan_cluster();
      sor_mode = 4;
    } catch (const Error&) {
      if (want == 4) throw;
      sor_mode = 0;
    }
  } else {
    if (want == 2) ensure_tbl();
    sor_mode = (want == 1 && n > 65535) ? 0 : want;     // the persistent solve keys its entries by a 16-bit tank
  }
}

Group::~Group() {
  cudaSetDevice(device);
  if (!settled) cudaStreamSynchronize(stream);
  drop_graph();
  for (cudaEvent_t e : ev_ph)
    if (e) cudaEventDestroy(e);
  if (ev_done) {
    for (Tank* t : tanks)
      if (t->dep == ev_done) { cudaStreamWaitEvent(t->stream, ev_done, 0); t->dep = nullptr; }
    cudaEventDestroy(ev_done);
  }
  // stream-ordered frees: no device-wide synchronisation (other batches keep running)
  drop_cluster_classes();
  if (cl_fork) cudaEventDestroy(cl_fork);
  for (void* p : {(void*)d_hpfx, (void*)d_apfx, (void*)d_barrier, (void*)d_ticket, d_tbl, (void*)d_tanks, (void*)d_bpfx,
                  (void*)d_ppfx, (void*)d_bsum, (void*)d_pieces, (void*)d_defer})
    if (p) cudaFreeAsync(p, stream);
  delete[] h_tanks;
  if (setup) cudaStreamDestroy(setup);
  if (setup_done) cudaEventDestroy(setup_done);
  if (own_stream) cudaStreamDestroy(stream);
}

void Group::ensure_tbl() {
  if (d_tbl) return;
  CK(cudaSetDevice(device));
  const int tiles = std::max(1, ctx.nblocks[kFamTiles]);
  CK(cudaMallocAsync(&d_tbl, tbl_list_bytes(tiles), stream));
  CK(cudaStreamSynchronize(stream));
  tbl_assign(ctx, d_tbl, tiles);
}

// The CTA plan of the cluster-resident solve. Each tank is cut into m pieces of np whole z planes, as few as fit
// the shared memory a CTA may take (cl_piece_kb, or the device's opt-in maximum less the kernel's static
// share). The tanks with the same m form a class: one launch of clusters of m CTAs, a cluster per tank, so
// that the cluster barrier couples only the pieces of one tank. The classes' launches run on streams of their
// own, forked from and joined back to the group's stream. Throws if a tank needs more than kClusterMax pieces
// or the device cannot hold one cluster of a class.
void Group::drop_cluster_classes() {
  for (ClusterClass& c : cl_classes) {
    if (c.done) cudaEventDestroy(c.done);
    if (c.stream) cudaStreamDestroy(c.stream);
  }
  cl_classes.clear();
}

void Group::plan_cluster() {
  CK(cudaSetDevice(device));
  int optin = 0;
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  optin -= 256;                                // the kernel's static shared memory
  const int budget = cl_piece_kb > 0 ? std::min(optin, cl_piece_kb * 1024) : optin;
  const int n = (int)tanks.size();
  std::vector<int> m(n), np(n);
  for (int i = 0; i < n; ++i) {
    const TankDev& D = tanks[i]->d;
    int npm = 0;                              // the most planes whose piece fits the budget
    while (npm < D.nz && cluster_smem_bytes(D, npm + 1) <= budget) ++npm;
    if (npm < 1) throw Error(-1, "cluster solve: one z plane of a tank does not fit a CTA's shared memory");
    int mi = (D.nz + npm - 1) / npm;
    np[i] = (D.nz + mi - 1) / mi;
    m[i] = (D.nz + np[i] - 1) / np[i];
    if (m[i] > kClusterMax) throw Error(-1, "cluster solve: a tank needs more than 16 CTAs");
  }
  CK(sor_cluster_prepare(optin, kClusterMax));
  std::vector<ClusterPiece> pcs;
  std::vector<ClusterClass> classes;
  for (int size = 1; size <= kClusterMax; ++size) {
    ClusterClass c;
    c.size = size;
    c.first = (int)pcs.size();
    c.smem = 16;
    for (int i = 0; i < n; ++i) {
      if (m[i] != size) continue;
      for (int p = 0; p < size; ++p) {
        const int k0 = p * np[i];
        pcs.push_back(ClusterPiece{i, k0, std::min(np[i], tanks[i]->d.nz - k0), np[i]});
      }
      c.smem = std::max(c.smem, cluster_smem_bytes(tanks[i]->d, np[i]));
    }
    c.blocks = (int)pcs.size() - c.first;
    if (!c.blocks) continue;
    if (sor_cluster_max_active(c.smem, size) < 1)
      throw Error(-1, "cluster solve: the device cannot hold one cluster of " + std::to_string(size) + " CTAs");
    classes.push_back(c);
  }
  drop_cluster_classes();
  if (d_pieces) CK(cudaFreeAsync(d_pieces, stream));
  CK(cudaMallocAsync((void**)&d_pieces, pcs.size() * sizeof(ClusterPiece), stream));
  CK(cudaMemcpyAsync(d_pieces, pcs.data(), pcs.size() * sizeof(ClusterPiece), cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  if (classes.size() > 1) {
    if (!cl_fork) CK(cudaEventCreateWithFlags(&cl_fork, cudaEventDisableTiming));
    for (ClusterClass& c : classes) {
      CK(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
    }
  }
  cl_classes = classes;
}

Batch::Batch(const std::vector<Tank*>& t, const int* lane_of) {
  if (t.empty()) throw Error(-1, "a batch needs at least one tank");
  for (Tank* x : t)
    if (x->cfg.device != t[0]->cfg.device) throw Error(-1, "all tanks of a batch must be on one device");
  std::vector<Tank*> by_lane[kMaxLanes];
  for (size_t i = 0; i < t.size(); ++i) {
    const int l = lane_of ? lane_of[i] : size_lane((long long)t[i]->d.nx * t[i]->d.ny * t[i]->d.nz);
    if (l < 0 || l >= kMaxLanes) throw Error(-1, "lane index out of range");
    by_lane[l].push_back(t[i]);
  }
  for (auto& v : by_lane)
    if (!v.empty()) lanes.emplace_back(new Group(v, nullptr));
  if (lanes.size() == 1) {
    stream = lanes[0]->stream;
    return;
  }
  // the lanes' persistent solves run at the same time: their blocks together fit on the SMs at once, each
  // lane's share in proportion to its cells
  long long all = 0;
  std::vector<long long> cells(lanes.size(), 0);
  for (size_t l = 0; l < lanes.size(); ++l) {
    for (Tank* x : lanes[l]->tanks) cells[l] += (long long)x->d.nx * x->d.ny * x->d.nz;
    all += cells[l];
  }
  for (size_t l = 0; l < lanes.size(); ++l) {
    const int share = (int)(lanes[l]->sm_count * cells[l] / std::max(all, 1LL));
    lanes[l]->sor_blocks = std::max(1, std::min(lanes[l]->sor_blocks, share));
  }
  CK(cudaSetDevice(t[0]->cfg.device));
  CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  own_stream = true;
  CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  join.resize(lanes.size());
  for (auto& e : join) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

Batch::~Batch() {
  if (own_stream) cudaStreamSynchronize(stream);
  lanes.clear();
  if (fork) cudaEventDestroy(fork);
  for (cudaEvent_t e : join) cudaEventDestroy(e);
  if (own_stream) cudaStreamDestroy(stream);
}

void Batch::substep(double dt) {
  if (lanes.size() == 1) {
    lanes[0]->substep(dt);
    return;
  }
  CK(cudaEventRecord(fork, stream));
  for (size_t i = 0; i < lanes.size(); ++i) {
    CK(cudaStreamWaitEvent(lanes[i]->stream, fork, 0));
    lanes[i]->substep(dt);
    CK(cudaEventRecord(join[i], lanes[i]->stream));
    CK(cudaStreamWaitEvent(stream, join[i], 0));
  }
}

void Group::set_profile(bool on) {
  if (on == profile) return;
  if (on && !ev_ph[0])
    for (cudaEvent_t& e : ev_ph) CK(cudaEventCreate(&e));
  profile = on;
  CK(cudaStreamSynchronize(stream));
  drop_graph();
}

double Group::phase_ms(int k) {
  if (!profile) throw Error(-6, "profiling is off");
  if (k < 0 || k >= kPhases) throw Error(-1, "phase index out of range");
  CK(cudaEventSynchronize(ev_ph[kPhases]));
  float f = 0;
  CK(cudaEventElapsedTime(&f, ev_ph[k], ev_ph[k + 1]));
  return f;
}

double Group::sor_phase_ms() { return phase_ms(3); }

void Group::drop_graph() {
  if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
  if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
}

void Group::ensure_uploaded() {
  bool stale = false;
  for (size_t i = 0; i < tanks.size(); ++i) stale |= uploaded[i] != tanks[i]->version;
  if (!stale) return;
  // the first upload of a group set up on its own stream goes the same way (nothing has used the table yet);
  // later ones wait until the sub-steps queued with the old table have run
  const bool first_async = setup && !uploaded_once;
  if (!first_async) CK(cudaStreamSynchronize(stream));
  int mi = 0;
  for (size_t i = 0; i < tanks.size(); ++i) {
    h_tanks[i] = tanks[i]->d;
    uploaded[i] = tanks[i]->version;
    mi = std::max(mi, tanks[i]->d.iters);
  }
  if (first_async) {
    CK(cudaMemcpyAsync(d_tanks, h_tanks, tanks.size() * sizeof(TankDev), cudaMemcpyHostToDevice, setup));
    CK(cudaEventRecord(setup_done, setup));
    CK(cudaStreamWaitEvent(stream, setup_done, 0));
  } else {
    CK(cudaMemcpyAsync(d_tanks, h_tanks, tanks.size() * sizeof(TankDev), cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  }
  uploaded_once = true;
  dt_on_device = false;                          // the host images carry no sub-step dt
  // the graph's shape depends only on the iteration count (the emitter kernel reads nemit on the device)
  if (mi != max_iters) { max_iters = mi; drop_graph(); }
}

void Tank::set_emitters(const std::vector<EmitterDev>& e) {
  join();
  if (e.size() > (size_t)kMaxEmitters) throw Error(-1, "at most 8 fixed emitters");
  if (!d_emitters) d_emitters = (EmitterDev*)alloc(kMaxEmitters * sizeof(EmitterDev));
  CK(cudaStreamSynchronize(stream));
  if (!e.empty()) CK(cudaMemcpyAsync(d_emitters, e.data(), e.size() * sizeof(EmitterDev), cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  d.emitters = d_emitters;
  d.nemit = (int)e.size();
  emit_per_substep = 0;
  for (const auto& x : e) emit_per_substep += x.per_substep;
  ++version;
}

void Group::set_dt(double dt) {
  if (dt_on_device && dt == dev_dt) return;      // the device descriptors carry it already
  const int n = (int)tanks.size();
  k_set_dt<<<(n + 127) / 128, 128, 0, stream>>>(d_tanks, n, dt);
  CK(cudaGetLastError());
  dev_dt = dt;
  dt_on_device = true;
}

void Group::enqueue_body() {
  // inside a capture an event record must be an external event node to be replayed with the graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (profile) CK(cudaStreamIsCapturing(stream, &cap));
  const unsigned evflags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
  auto mark = [&](int k) {
    if (profile) CK(cudaEventRecordWithFlags(ev_ph[k], stream, evflags));
  };
  mark(0);
  k_emit_begin<<<(int)tanks.size(), 128, 0, stream>>>(d_tanks, (int)tanks.size(), ctx.ppfx_in, ctx.ticket + 2);
  launch_bin(ctx);
  launch_scan(ctx);
  launch_scatter(ctx);
  mark(1);
  launch_p2g(ctx);
  mark(2);
  launch_grid_nodes(ctx);
  launch_grid_cells(ctx);
  mark(3);
  if (sor_mode == 1 && max_iters > 0) {
    launch_sor_persist(ctx, max_iters, sor_blocks, watchdog_polls, cl_piece_kb * 1024);
    CK(cudaGetLastError());
  } else if (sor_mode == 2 || sor_mode == 3) {
    // S sweeps per launch; launch l reads pres (l even) or pres2 and writes the other; an odd count ends in pres2
    const int S = sor_mode == 2 ? 2 : 4;
    if (S == 2) launch_tbl_lists(ctx);
    const int sweeps = 2 * max_iters, nl = (sweeps + S - 1) / S;
    for (int l = 0; l < nl; ++l) launch_sor_tb(ctx, S, l * S, std::min(S, sweeps - l * S), l & 1);
    if (nl & 1) launch_sor_copy(ctx);
    CK(cudaGetLastError());
  } else if (sor_mode == 4) {
    if (max_iters > 0) {
      if (cl_classes.size() == 1) {
        const ClusterClass& c = cl_classes[0];
        launch_sor_cluster(ctx, d_pieces, c.blocks, c.smem, c.size, max_iters);
      } else {
        CK(cudaEventRecord(cl_fork, stream));
        for (const ClusterClass& c : cl_classes) {
          CK(cudaStreamWaitEvent(c.stream, cl_fork, 0));
          LaunchCtx L = ctx;
          L.stream = c.stream;
          launch_sor_cluster(L, d_pieces + c.first, c.blocks, c.smem, c.size, max_iters);
          CK(cudaEventRecord(c.done, c.stream));
          CK(cudaStreamWaitEvent(stream, c.done, 0));
        }
      }
    }
    CK(cudaGetLastError());
  } else {
    for (int it = 0; it < max_iters; ++it) {
      launch_sor_sweep(ctx, 0, it);
      launch_sor_sweep(ctx, 1, it);
    }
    CK(cudaGetLastError());
  }
  mark(4);
  if (residual) {
    launch_sor_residual(ctx);
    CK(cudaGetLastError());
  }
  launch_project(ctx);
  mark(5);
  launch_g2p(ctx, g2p_form);
  mark(6);
}

void Group::substep(double dt) {
  CK(cudaSetDevice(device));
  // work a tank enqueued on its own stream (staging, emission) must come first
  for (Tank* t : tanks)
    if (t->stream != stream && t->dirty) {
      CK(cudaEventRecord(t->ev_own, t->stream));
      CK(cudaStreamWaitEvent(stream, t->ev_own, 0));
      t->dirty = false;
    }
  ensure_uploaded();
  bool geom = false;
  for (Tank* t : tanks) geom |= t->geom_dirty;
  if (geom) {
    launch_geom(ctx);
    CK(cudaGetLastError());
    for (Tank* t : tanks) t->geom_dirty = false;
  }
  set_dt(dt);
  if (use_graphs) {
    if (!exec) {
      CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      enqueue_body();
      cudaError_t e = cudaStreamEndCapture(stream, &graph);
      CK(e);
      CK(cudaGetLastError());
      CK(cudaGraphInstantiate(&exec, graph, 0));
    }
    CK(cudaGraphLaunch(exec, stream));
  } else {
    enqueue_body();
    CK(cudaGetLastError());
  }
  for (Tank* t : tanks) {
    t->time += dt;
    t->n_emit_host = 0;
    t->n_upper += (long long)ceil(t->emit_per_substep);
  }
  // later work on a tank's own stream (reads, emission) must follow this sub-step: it waits on ev_done
  bool others = false;
  for (Tank* t : tanks) others |= t->stream != stream;
  if (others) {
    if (!ev_done) CK(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
    CK(cudaEventRecord(ev_done, stream));
    for (Tank* t : tanks)
      if (t->stream != stream) t->dep = ev_done;
  }
}

}  // namespace suiri
