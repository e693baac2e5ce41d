// Top-view water height map and the capillary-gravity ripple layer, once per frame.
//
// Height map (blender_addon/suiri_lab/solver.py:738-779): per texel the highest particle, every particle
// widened to a sphere cap of radius 1.3125h (a dilation with the precomputed disc of cap heights), then a
// separable Gaussian over wet texels only. Float64, with the same maxima and sums in the same order as
// the reference, so the map agrees bit for bit.
//
// Ripple layer (solver.py:855-907, src/js/64-ripple.js): the impulses deposited by merging drops are
// mirrored into a (2Rz)×(2Rx) cosine domain (reflecting walls), transformed, every mode advanced by the
// exact damped oscillator of ω² = (gk + σ/ρ k³) tanh(kd) and kicked by the impulse, transformed back to
// heights and slopes, multiplied by the absorption mask (obstacle walls at the water line, dry floor)
// and transformed forward again. The reference's square layer is Rx = Rz; here the layer may be
// rectangular. The 2D FFTs are written here: rows, then columns, each line in shared memory, radix-4
// Stockham stages (natural order, no bit-reversed load) and one radix-2 stage for odd log2 lengths,
// twiddles from a table computed in float64 (as the reference's WGSL does, 64-ripple.js:32-33, :175-178),
// complex64 data.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.h"
#include "sdf.cuh"

namespace suiri {

struct RippleState {
  int W = 0, Mx = 0, Mz = 0, lx = 0, lz = 0;
  double Lx = 0, Lz = 0;
  double sigma_rho = 0.0728 / 998.0, rho = 998.0, g = 9.81;
  double depth = 0.0;           // fixed dispersion depth; 0: mean depth of the liquid each frame
  unsigned* topkey = nullptr;   // W² ordered float keys of the highest particle
  double* hA = nullptr;         // W² float64 work maps
  double* hB = nullptr;
  double* top = nullptr;        // W² final height map, -1 dry
  float* mask = nullptr;        // (rz+1)(rx+1)
  float4* field = nullptr;      // (rz+1)(rx+1): h, slope x, slope z
  float2* S = nullptr;          // Mz×Mx spectral state
  float2* A = nullptr;          // Mz×Mx work
  float2* twx = nullptr;        // Mx twiddles (cos, sin)(2πt/Mx)
  float2* twz = nullptr;
  double* mx_coord = nullptr;   // rx+1 x coordinates of the ripple vertices
  double* mz_coord = nullptr;
  int4* disc = nullptr;         // dilation offsets (ox, oy) with cap height index
  double* disc_h = nullptr;
  int ndisc = 0;
  double* blur_w = nullptr;
  int blur_rad = 0;
  double texel[2] = {0, 0};
  double4* coef = nullptr;      // fixed depth: per mode the exact update over coef_dt as a 2×2 matrix
  double* kick = nullptr;       //   and the impulse kick factor
  double coef_dt = -1.0;
  unsigned long long* light = nullptr;   // W² floor light in 2^-44 fixed point (frame maps)
  float4* maps = nullptr;       // W²: top height, ripple slope x, slope z, floor light
  std::vector<void*> mem;
};

namespace {

RippleState* rs(Tank& t) { return (RippleState*)t.ripple; }

__device__ __forceinline__ unsigned fkey(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float funkey(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void k_top_scatter(TankDev T, unsigned* __restrict__ key, int W, double tx, double tz) {
  const int n = T.ctr->n_live;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float4 p = T.pA[q];
    if (flags_of(p.w) & kFlagDead) continue;
    if (!((double)p.y <= T.rim + 0.01)) continue;
    const double fx = floor(((double)p.x - T.ox) / tx), fz = floor(((double)p.z - T.oz) / tz);
    if (fx < 0 || fz < 0 || fx >= W || fz >= W) continue;
    atomicMax(key + (size_t)fz * W + (int)fx, fkey(p.y));
  }
}

// H = max(-1, max over the disc of (top[y+oy][x+ox] + cap)) ; dry where nothing reaches
__global__ void k_top_dilate(const unsigned* __restrict__ key, double* __restrict__ H, int W, const int4* __restrict__ disc,
                             const double* __restrict__ cap, int ndisc, int any) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= W * W) return;
  const int x = e % W, y = e / W;
  double h = -1.0;
  if (any) {
    for (int d = 0; d < ndisc; ++d) {
      const int xs = x + disc[d].x, ys = y + disc[d].y;
      if (xs < 0 || ys < 0 || xs >= W || ys >= W) continue;
      const unsigned k = key[(size_t)ys * W + xs];
      if (k == 0u) continue;
      h = fmax(h, (double)funkey(k) + cap[d]);
    }
  }
  H[e] = h;
}

// wet-only Gaussian along x (axis 0) or z (axis 1); wet = the unblurred map >= 0 (wet0)
__global__ void k_top_blur(const double* __restrict__ in, const double* __restrict__ wet0, double* __restrict__ out, int W,
                           const double* __restrict__ w, int rad, int along_z) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= W * W) return;
  const int x = e % W, y = e / W;
  if (!(wet0[e] >= 0.0)) { out[e] = -1.0; return; }
  double s = 0.0, ws = 0.0;
  for (int i = -rad; i <= rad; ++i) {
    int xi = x, yi = y;
    if (along_z) yi = min(max(y + i, 0), W - 1); else xi = min(max(x + i, 0), W - 1);
    const size_t o = (size_t)yi * W + xi;
    const double k = w[i + rad];
    if (wet0[o] >= 0.0) { s += in[o] * k; ws += k; } else { s += 0.0; ws += 0.0; }
  }
  out[e] = s / fmax(ws, 1e-12);
}

__global__ void k_ripple_mask(TankDev T, const double* __restrict__ top, int W, const double* __restrict__ X,
                              const double* __restrict__ Z, float* __restrict__ mask) {
  const int rx = T.rx, rz = T.rz;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (rx + 1) * (rz + 1)) return;
  const int i = e % (rx + 1), j = e / (rx + 1);
  const double lx = T.ox, lz = T.oz, hx = T.ox + T.nx * T.h, hz = T.oz + T.nz * T.h;
  const double x = X[i], z = Z[j];
  const int ti = (int)fmin(fmax((x - lx) / (hx - lx) * W, 0.0), (double)(W - 1));
  const int tj = (int)fmin(fmax((z - lz) / (hz - lz) * W, 0.0), (double)(W - 1));
  const double h = top[(size_t)tj * W + ti];
  double m = 0.75;
  if (h >= 0) {
    const double d = tank_sdf(T, x, h - 0.002, z);
    double t = (d - -0.003) / (0.006 - -0.003);
    t = fmin(fmax(t, 0.0), 1.0);
    m = t * t * (3.0 - 2.0 * t);
  }
  mask[e] = (float)m;
}

// mirrored source (impulse density) → complex input of the forward transform (64-ripple.js:18-31)
__global__ void k_ripple_src(TankDev T, const long long* __restrict__ src, float2* __restrict__ out, int Mx, int Mz, double inv_area) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Mx * Mz) return;
  const int i = e % Mx, j = e / Mx;
  const int pi = i <= T.rx ? i : Mx - i, pj = j <= T.rz ? j : Mz - j;
  const double v = (double)src[(size_t)pj * (T.rx + 1) + pi] * (1.0 / kRippleFix) * inv_area;
  out[e] = make_float2((float)v, 0.f);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// Stockham autosort FFT of a power-of-two length M in shared memory (natural order in and out): radix-4
// stages, then one radix-2 stage when log2 M is odd, ping-ponging between two buffers. A stage takes the
// R inputs of butterfly j at stride M/R, multiplies input r by w^(r·(j mod Ns)) with w = e^(±2πi/(Ns·R))
// (from the table tw[k] = e^(2πik/M)), transforms them, and writes them at stride Ns from
// (j − j mod Ns)·R + j mod Ns. Unnormalised; sign −1 forward, +1 inverse.
template <int R>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ in, float2* __restrict__ out, int M, int Ns, int j,
                                          const float2* __restrict__ tw, float sign) {
  float2 v[R];
  const int k = j & (Ns - 1);
  const int step = M / (Ns * R);
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = in[j + r * (M / R)];
  // one table read per butterfly: w, then w^2 and w^3 by multiplication
  float2 w = __ldg(tw + k * step);
  w.y *= sign;
  float2 wr = w;
#pragma unroll
  for (int r = 1; r < R; ++r) {
    v[r] = cmul(v[r], wr);
    if (r + 1 < R) wr = cmul(wr, w);
  }
  if (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = make_float2(a.x + b.x, a.y + b.y);
    v[1] = make_float2(a.x - b.x, a.y - b.y);
  } else {
    // y1 = b + (i·sign)·d, y3 = b − (i·sign)·d with a = x0 + x2, b = x0 − x2, c = x1 + x3, d = x1 − x3
    const float2 a = make_float2(v[0].x + v[2].x, v[0].y + v[2].y), b = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
    const float2 c = make_float2(v[1].x + v[3].x, v[1].y + v[3].y), d = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
    const float2 id = make_float2(-sign * d.y, sign * d.x);
    v[0] = make_float2(a.x + c.x, a.y + c.y);
    v[2] = make_float2(a.x - c.x, a.y - c.y);
    v[1] = make_float2(b.x + id.x, b.y + id.y);
    v[3] = make_float2(b.x - id.x, b.y - id.y);
  }
  const int d0 = (j - k) * R + k;
#pragma unroll
  for (int r = 0; r < R; ++r) out[d0 + r * Ns] = v[r];
}

// the transform of C lines of length M stored line after line in buf (two buffers of C·M); returns the
// buffer holding the result
__device__ __forceinline__ float2* fft_lines(float2* a, float2* b, int M, int C, const float2* __restrict__ tw, float sign) {
  int logM = 0;
  while ((1 << logM) < M) ++logM;
  for (int Ns = 1; Ns < M;) {
    const int R = M / Ns >= 4 ? 4 : 2;
    const int lper = logM - (R == 4 ? 2 : 1), per = 1 << lper;
    for (int e = threadIdx.x; e < per * C; e += blockDim.x) {
      const int cl = e >> lper, j = e & (per - 1);
      if (R == 4) fft_stage<4>(a + cl * M, b + cl * M, M, Ns, j, tw, sign);
      else fft_stage<2>(a + cl * M, b + cl * M, M, Ns, j, tw, sign);
    }
    __syncthreads();
    float2* t = a; a = b; b = t;
    Ns *= R;
  }
  return a;
}

// one line per block: rows of length M (stride 1) starting at data + line*M
__global__ void k_fft_rows(float2* __restrict__ data, int M, int logM, const float2* __restrict__ tw, float sign) {
  extern __shared__ float2 s[];
  float2* row = data + (size_t)blockIdx.x * M;
  for (int i = threadIdx.x; i < M; i += blockDim.x) s[i] = row[i];
  __syncthreads();
  const float2* res = fft_lines(s, s + M, M, 1, tw, sign);
  for (int i = threadIdx.x; i < M; i += blockDim.x) row[i] = res[i];
}

// C columns per block: columns of length M with row stride `ld`
__global__ void k_fft_cols(float2* __restrict__ data, int M, int logM, int ld, int C, const float2* __restrict__ tw, float sign) {
  extern __shared__ float2 s[];
  const int c0 = blockIdx.x * C;
  for (int e = threadIdx.x; e < M * C; e += blockDim.x) {
    const int r = e / C, cl = e % C;
    s[cl * M + r] = data[(size_t)r * ld + c0 + cl];
  }
  __syncthreads();
  const float2* res = fft_lines(s, s + M * C, M, C, tw, sign);
  for (int e = threadIdx.x; e < M * C; e += blockDim.x) {
    const int r = e / C, cl = e % C;
    data[(size_t)r * ld + c0 + cl] = res[cl * M + r];
  }
}

// exact damped oscillator per mode plus the impulse kick (solver.py:882-899, 64-ripple.js:58-90)
__global__ void k_ripple_evolve(TankDev T, float2* __restrict__ S, const float2* __restrict__ hat, int Mx, int Mz, double Lx,
                                double Lz, double dt, double g, double sigma_rho, double rho, double fixed_depth) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Mx * Mz) return;
  const int i = e % Mx, j = e / Mx;
  const int Rx = T.rx, Rz = T.rz;
  const int mx = i < Rx ? i : i - Mx, mz = j < Rz ? j : j - Mz;
  if ((mx == 0 && mz == 0) || mx == -Rx || mz == -Rz) { S[e] = make_float2(0.f, 0.f); return; }
  const double n = (double)T.ctr->n_sorted;
  const double depth = fixed_depth > 0 ? fixed_depth : fmin(fmax(n * T.vp / (T.nx * T.nz * T.h * T.h), 0.003), T.rim);
  const double kx = mx * M_PI / Lx, kz = mz * M_PI / Lz;
  const double kk = sqrt(kx * kx + kz * kz);
  const double D = fmax(depth, 0.002);
  const double kd = fmin(kk * D, 15.0);
  const double th = tanh(kd);
  const double nu = 1.0e-6, film = 0.3;
  const double w2 = (g * kk + sigma_rho * kk * kk * kk) * th;
  const double w = sqrt(w2);
  const double gam = 2 * nu * kk * kk + film * kk * sqrt(nu * w * 0.125) + kk * sqrt(nu * w * 0.5) / fmax(sinh(fmin(2 * kd, 30.0)), 1e-4);
  const double wd = sqrt(fmax(w2 - gam * gam, 1e-6));
  double Hs = S[e].x, Vs = S[e].y;
  if (dt > 0) {
    const double c = cos(wd * dt), sn = sin(wd * dt), ex = exp(-gam * dt);
    const double H2 = ex * (Hs * c + (Vs + gam * Hs) / wd * sn);
    const double V2 = ex * (Vs * c - (w2 * Hs + gam * Vs) / wd * sn);
    Hs = H2; Vs = V2;
  }
  const double kh = 2 * M_PI / 0.12;
  const double hp = 1 - exp(-(kk * kk) / (kh * kh));
  const double sw = fmax(1.2 * Lx / Rx, 0.003);
  const double spread = exp(-0.5 * kk * kk * sw * sw);
  Vs = Vs - (kk * th / rho) * (double)hat[e].x * hp * spread;
  S[e] = make_float2((float)Hs, (float)Vs);
}

// With a fixed depth the update of a mode over dt is the same every frame: the damped rotation above as
// (H, V) ← [[a11, a12], [a21, a22]]·(H, V), then V −= kick·Re(hat). Computed once per dt by
// k_ripple_coef (same formulas, rearranged: a11 = e^(−γdt)(cos + γ sin/ω_d), a12 = e^(−γdt) sin/ω_d,
// a21 = −e^(−γdt) ω² sin/ω_d, a22 = e^(−γdt)(cos − γ sin/ω_d)) and applied by k_ripple_evolve_fixed.
__global__ void k_ripple_coef(TankDev T, double4* __restrict__ coef, double* __restrict__ kick, int Mx, int Mz, double Lx,
                              double Lz, double dt, double g, double sigma_rho, double rho, double depth) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Mx * Mz) return;
  const int i = e % Mx, j = e / Mx;
  const int Rx = T.rx, Rz = T.rz;
  const int mx = i < Rx ? i : i - Mx, mz = j < Rz ? j : j - Mz;
  if ((mx == 0 && mz == 0) || mx == -Rx || mz == -Rz) {
    coef[e] = make_double4(0.0, 0.0, 0.0, 0.0);
    kick[e] = 0.0;
    return;
  }
  const double kx = mx * M_PI / Lx, kz = mz * M_PI / Lz;
  const double kk = sqrt(kx * kx + kz * kz);
  const double D = fmax(depth, 0.002);
  const double kd = fmin(kk * D, 15.0);
  const double th = tanh(kd);
  const double nu = 1.0e-6, film = 0.3;
  const double w2 = (g * kk + sigma_rho * kk * kk * kk) * th;
  const double w = sqrt(w2);
  const double gam = 2 * nu * kk * kk + film * kk * sqrt(nu * w * 0.125) + kk * sqrt(nu * w * 0.5) / fmax(sinh(fmin(2 * kd, 30.0)), 1e-4);
  const double wd = sqrt(fmax(w2 - gam * gam, 1e-6));
  const double c = cos(wd * dt), sn = sin(wd * dt), ex = exp(-gam * dt);
  coef[e] = make_double4(ex * (c + gam * sn / wd), ex * sn / wd, -ex * w2 * sn / wd, ex * (c - gam * sn / wd));
  const double kh = 2 * M_PI / 0.12;
  const double hp = 1 - exp(-(kk * kk) / (kh * kh));
  const double sw = fmax(1.2 * Lx / Rx, 0.003);
  const double spread = exp(-0.5 * kk * kk * sw * sw);
  kick[e] = (kk * th / rho) * hp * spread;
}

__global__ void k_ripple_evolve_fixed(float2* __restrict__ S, const float2* __restrict__ hat, const double4* __restrict__ coef,
                                      const double* __restrict__ kick, int n) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double4 a = coef[e];
  const float2 v = S[e];
  const double Hs = v.x, Vs = v.y;
  const double H2 = a.x * Hs + a.y * Vs;
  const double V2 = a.z * Hs + a.w * Vs - kick[e] * (double)hat[e].x;
  S[e] = make_float2((float)H2, (float)V2);
}

// field = ifft (already in S, unnormalised) → heights and slopes; masked = field · mirrored mask → A
__global__ void k_ripple_field(TankDev T, const float2* __restrict__ S, float2* __restrict__ A, const float* __restrict__ mask,
                               float4* __restrict__ field, int Mx, int Mz, double dx, double dz) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Mx * Mz) return;
  const int i = e % Mx, j = e / Mx;
  const double inv = 1.0 / ((double)Mx * Mz);
  const int pi = i <= T.rx ? i : Mx - i, pj = j <= T.rz ? j : Mz - j;
  const float m = mask[(size_t)pj * (T.rx + 1) + pi];
  const float2 v = S[e];
  A[e] = make_float2((float)(v.x * inv) * m, (float)(v.y * inv) * m);
  if (i <= T.rx && j <= T.rz) {
    const double h = v.x * inv;
    const double hl = S[(size_t)j * Mx + (i + Mx - 1) % Mx].x * inv, hr = S[(size_t)j * Mx + (i + 1) % Mx].x * inv;
    const double hd = S[(size_t)((j + Mz - 1) % Mz) * Mx + i].x * inv, hu = S[(size_t)((j + 1) % Mz) * Mx + i].x * inv;
    field[(size_t)j * (T.rx + 1) + i] = make_float4((float)h, (float)((hr - hl) / (2 * dx)), (float)((hu - hd) / (2 * dz)), 0.f);
  }
}

// ---------------------------------------------------------------------------------------------- frame maps
// Per frame the bake exports two maps over the footprint (bake.py:241-249): the surface (top height and the
// ripple slopes at texel centres) and the floor light (solver.py:796-846). The light is gathered by
// splatting: the footprint is sampled 2×2 per texel, each wet sample refracts the sun (index 1.333) through
// the normal of the height map's slope plus the ripple slope, keeps 1 - Fresnel of it and lands displaced by
// its depth times the refracted ray's tilt less flat water's; a dry sample lands where it is with all of
// its light. Its quarter of a texel's light is spread bilinearly over the four texels around the landing
// point, in 2^-32 fixed point so that the sums do not depend on the order of the atomics (the whole map's
// light is at most W², below 2^26 for W <= 8192, so no texel can overflow). A 5-point cross with wrap-around
// then blurs it. Float64 throughout, on the float32 ripple field.
constexpr double kLightFix = 4294967296.0;   // 2^32

struct LightParams {
  double sun[3];               // unit vector towards the sun
  double flat[3];              // the refracted ray under flat water
  double tex[2];               // texel size (footprint / W)
  double Lx, Lz;               // footprint size (ripple vertex spacing Lx / rx)
  double mtex[2];              // texel size of the surface map (nx·h / W)
};

// slope of the wet height map at texel (i, k): central differences with wrap-around neighbours, a dry
// neighbour standing in as the centre, none on a dry texel (solver.py:813-819)
__device__ __forceinline__ void height_slope(const double* __restrict__ H, int W, int i, int k, const LightParams& P,
                                             double& gx, double& gz) {
  const double c = H[(size_t)k * W + i];
  gx = 0.0; gz = 0.0;
  if (!(c >= 0.0)) return;
  auto at = [&](int ii, int kk) { const double v = H[(size_t)kk * W + ii]; return v >= 0.0 ? v : c; };
  const int ip = i + 1 < W ? i + 1 : 0, im = i > 0 ? i - 1 : W - 1;
  const int kp = k + 1 < W ? k + 1 : 0, km = k > 0 ? k - 1 : W - 1;
  gx = (at(ip, k) - at(im, k)) / (2 * P.tex[0]);
  gz = (at(i, kp) - at(i, km)) / (2 * P.tex[1]);
}

// ripple slopes at (x, z) from the footprint corner, bilinear in the vertex field (solver.py:909-919)
__device__ __forceinline__ void ripple_slope(const float4* __restrict__ F, int rx, int rz, double Lx, double Lz, double x,
                                             double z, double& sx, double& sz) {
  const double qx = fmin(fmax(x / Lx * rx, 0.0), (double)rx), qz = fmin(fmax(z / Lz * rz, 0.0), (double)rz);
  const int bx = min((int)floor(qx), rx - 1), bz = min((int)floor(qz), rz - 1);
  const double fx = qx - bx, fz = qz - bz;
  const size_t o = (size_t)bz * (rx + 1) + bx;
  const float4 a = F[o], b = F[o + 1], c = F[o + rx + 1], d = F[o + rx + 2];
  sx = ((double)a.y * (1 - fx) + (double)b.y * fx) * (1 - fz) + ((double)c.y * (1 - fx) + (double)d.y * fx) * fz;
  sz = ((double)a.z * (1 - fx) + (double)b.z * fx) * (1 - fz) + ((double)c.z * (1 - fx) + (double)d.z * fx) * fz;
}

__device__ __forceinline__ double fresnel_water(double c) {
  const double x = fmin(fmax(1.0 - c, 0.0), 1.0);
  const double x2 = x * x;
  return 0.0204 + 0.9796 * (x2 * x2 * x);
}

// one thread per sample (2W × 2W)
__global__ void __launch_bounds__(256) k_light_splat(const double* __restrict__ H, const float4* __restrict__ F, int W,
                                                     int rx, int rz, LightParams P, unsigned long long* __restrict__ light) {
  const int S = 2 * W;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= S * S) return;
  const int si = e % S, sj = e / S;
  const double u = (si + 0.5) / 2 - 0.5, w = (sj + 0.5) / 2 - 0.5;   // texel coordinates, centres at integers
  // bilinear taps with held edges (solver.py:808-812)
  const int i0 = min(max((int)floor(u), 0), W - 1), k0 = min(max((int)floor(w), 0), W - 1);
  const int i1 = min(i0 + 1, W - 1), k1 = min(k0 + 1, W - 1);
  const double ax = fmin(fmax(u - i0, 0.0), 1.0), az = fmin(fmax(w - k0, 0.0), 1.0);
  auto lerp2 = [&](double a00, double a10, double a01, double a11) {
    return (a00 * (1 - ax) + a10 * ax) * (1 - az) + (a01 * (1 - ax) + a11 * ax) * az;
  };
  const double h00 = H[(size_t)k0 * W + i0], h10 = H[(size_t)k0 * W + i1];
  const double h01 = H[(size_t)k1 * W + i0], h11 = H[(size_t)k1 * W + i1];
  auto dry = [](double v) { return v >= 0.0 ? v : -1.0; };
  auto wetf = [](double v) { return v >= 0.0 ? 1.0 : 0.0; };
  const double h = lerp2(dry(h00), dry(h10), dry(h01), dry(h11));
  const bool wet = h >= 0.0 && lerp2(wetf(h00), wetf(h10), wetf(h01), wetf(h11)) > 0.999;
  const double x = (u + 0.5) * P.tex[0], z = (w + 0.5) * P.tex[1];
  double px = x, pz = z, energy = 1.0 / 4;
  if (wet) {
    double g[4][2];
    height_slope(H, W, i0, k0, P, g[0][0], g[0][1]);
    height_slope(H, W, i1, k0, P, g[1][0], g[1][1]);
    height_slope(H, W, i0, k1, P, g[2][0], g[2][1]);
    height_slope(H, W, i1, k1, P, g[3][0], g[3][1]);
    double rsx, rsz;
    ripple_slope(F, rx, rz, P.Lx, P.Lz, x, z, rsx, rsz);
    double nx = -lerp2(g[0][0], g[1][0], g[2][0], g[3][0]) - rsx, ny = 1.0;
    double nz = -lerp2(g[0][1], g[1][1], g[2][1], g[3][1]) - rsz;
    const double len = sqrt(nx * nx + ny * ny + nz * nz);
    nx /= len; ny /= len; nz /= len;
    const double c = nx * P.sun[0] + ny * P.sun[1] + nz * P.sun[2];
    const double eta = 1 / 1.333;
    const double k = 1 - eta * eta * (1 - c * c);
    const double q = eta * c - sqrt(fmax(k, 0.0));
    const double r0 = -P.sun[0] * eta + nx * q, r1 = -P.sun[1] * eta + ny * q, r2 = -P.sun[2] * eta + nz * q;
    const double fall = h / fmax(-r1, 0.05);
    px = x + (r0 * fall - P.flat[0] * h / -P.flat[1]);
    pz = z + (r2 * fall - P.flat[2] * h / -P.flat[1]);
    energy = (1 - fresnel_water(c)) / 4;
  }
  const double lx = px / P.tex[0] - 0.5, lz = pz / P.tex[1] - 0.5;
  const double fx0 = floor(lx), fz0 = floor(lz);
  if (!(fx0 > -2.0 && fx0 < W && fz0 > -2.0 && fz0 < W)) return;     // no tap inside the map (NaN too)
  const int x0 = (int)fx0, z0 = (int)fz0;
  const double bx = lx - fx0, bz = lz - fz0;
  const double wt[4] = {(1 - bx) * (1 - bz), bx * (1 - bz), (1 - bx) * bz, bx * bz};
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int xi = x0 + (t & 1), zi = z0 + (t >> 1);
    if (xi < 0 || xi >= W || zi < 0 || zi >= W) continue;
    const unsigned long long q = __double2ull_rn(energy * wt[t] * kLightFix);
    if (q) atomicAdd(light + (size_t)zi * W + xi, q);
  }
}

// one thread per texel: the blurred light and the surface map (top height, ripple slopes at the texel centre)
__global__ void __launch_bounds__(256) k_light_maps(const unsigned long long* __restrict__ light, const double* __restrict__ H,
                                                    const float4* __restrict__ F, int W, int rx, int rz, LightParams P,
                                                    float4* __restrict__ maps) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= W * W) return;
  const int i = e % W, k = e / W;
  const int ip = i + 1 < W ? i + 1 : 0, im = i > 0 ? i - 1 : W - 1;
  const int kp = k + 1 < W ? k + 1 : 0, km = k > 0 ? k - 1 : W - 1;
  auto L = [&](int ii, int kk) { return (double)light[(size_t)kk * W + ii] / kLightFix; };
  const double c = L(i, k) + L(i, km) + L(i, kp) + L(im, k) + L(ip, k);
  double sx = 0.0, sz = 0.0;
  if (rx > 0) ripple_slope(F, rx, rz, P.Lx, P.Lz, (i + 0.5) * P.mtex[0], (k + 0.5) * P.mtex[1], sx, sz);
  maps[e] = make_float4((float)H[e], (float)sx, (float)sz, (float)(c / 5));
}

int ilog2(int x) { int l = 0; while ((1 << l) < x) ++l; return l; }

void fft2(Tank& t, float2* data, float sign) {
  RippleState& r = *rs(t);
  const int lx = ilog2(r.Mx), lz = ilog2(r.Mz);
  k_fft_rows<<<r.Mz, 256, 2 * r.Mx * sizeof(float2), t.stream>>>(data, r.Mx, lx, r.twx, sign);
  int C = 4;                        // columns per block: 32 B of each row per load, two buffers in shared memory
  while (C > 1 && 2 * (size_t)r.Mz * C * sizeof(float2) > 96 * 1024) C >>= 1;
  while (r.Mx % C) C >>= 1;
  k_fft_cols<<<r.Mx / C, 256, 2 * r.Mz * C * sizeof(float2), t.stream>>>(data, r.Mz, lz, r.Mx, C, r.twz, sign);
  CK(cudaGetLastError());
}

// host table → device, ordered on the tank's stream after the zero-fill of the same buffer (the tank's
// stream does not synchronise with the legacy default stream), complete before the host buffer is reused
void upload(Tank& t, void* dst, const void* src, size_t bytes) {
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, t.stream));
  CK(cudaStreamSynchronize(t.stream));
}

void* ralloc(Tank& t, RippleState& r, size_t bytes) {
  void* p = nullptr;
  CK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
  CK(cudaMemsetAsync(p, 0, std::max<size_t>(bytes, 16), t.stream));
  r.mem.push_back(p);
  return p;
}

RippleState& ensure(Tank& t) {
  if (t.ripple) return *rs(t);
  const TankDev& D = t.d;
  auto pow2 = [](int x) { return x > 0 && (x & (x - 1)) == 0; };
  if (!pow2(D.rx) || !pow2(D.rz)) throw Error(-1, "ripple layer sizes must be powers of two");
  RippleState* r = new RippleState();
  t.ripple = r;
  r->W = t.cfg.wmap;
  r->Mx = 2 * D.rx; r->Mz = 2 * D.rz;
  r->sigma_rho = t.cfg.ripple_sigma / t.cfg.ripple_rho;
  r->rho = t.cfg.ripple_rho;
  r->g = t.cfg.g;
  r->depth = t.cfg.ripple_depth;
  r->Lx = D.nx * D.h; r->Lz = D.nz * D.h;
  const int W = r->W;
  static_assert(sizeof(float2) == 8, "");
  CK(cudaFuncSetAttribute(k_fft_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  CK(cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  if (2 * (size_t)r->Mx * 8 > 200 * 1024 || 2 * (size_t)r->Mz * 8 > 200 * 1024) throw Error(-1, "ripple layer too large");
  r->topkey = (unsigned*)ralloc(t, *r, (size_t)W * W * 4);
  r->hA = (double*)ralloc(t, *r, (size_t)W * W * 8);
  r->hB = (double*)ralloc(t, *r, (size_t)W * W * 8);
  r->top = (double*)ralloc(t, *r, (size_t)W * W * 8);
  r->mask = (float*)ralloc(t, *r, (size_t)(D.rx + 1) * (D.rz + 1) * 4);
  r->field = (float4*)ralloc(t, *r, (size_t)(D.rx + 1) * (D.rz + 1) * 16);
  r->S = (float2*)ralloc(t, *r, (size_t)r->Mx * r->Mz * 8);
  r->A = (float2*)ralloc(t, *r, (size_t)r->Mx * r->Mz * 8);
  r->twx = (float2*)ralloc(t, *r, (size_t)r->Mx * 8);
  r->twz = (float2*)ralloc(t, *r, (size_t)r->Mz * 8);
  r->mx_coord = (double*)ralloc(t, *r, (size_t)(D.rx + 1) * 8);
  r->mz_coord = (double*)ralloc(t, *r, (size_t)(D.rz + 1) * 8);
  // host tables
  std::vector<float2> tw(std::max(r->Mx, r->Mz));
  for (int pass = 0; pass < 2; ++pass) {
    const int M = pass ? r->Mz : r->Mx;
    for (int k = 0; k < M; ++k) tw[k] = make_float2((float)cos(2 * M_PI * k / M), (float)sin(2 * M_PI * k / M));
    upload(t, pass ? r->twz : r->twx, tw.data(), M * 8);
  }
  // ripple vertex coordinates: lo + linspace(0, 1, R+1)·(hi - lo) as NumPy forms them (solver.py:784-785)
  const double lo[2] = {D.ox, D.oz}, hi[2] = {D.ox + D.nx * D.h, D.oz + D.nz * D.h};
  for (int a = 0; a < 2; ++a) {
    const int R = a ? D.rz : D.rx;
    std::vector<double> c(R + 1);
    const double step = 1.0 / R;
    for (int i = 0; i <= R; ++i) {
      const double u = i == R ? 1.0 : i * step + 0.0;
      c[i] = lo[a] + u * (hi[a] - lo[a]);
    }
    upload(t, a ? r->mz_coord : r->mx_coord, c.data(), (R + 1) * 8);
  }
  // dilation disc and blur weights (solver.py:752-768)
  r->texel[0] = (hi[0] - lo[0]) / W;
  r->texel[1] = (hi[1] - lo[1]) / W;
  const double rad = (0.5 * D.h * 1.05) * 1.25;
  const int ri = (int)ceil(rad / std::min(r->texel[0], r->texel[1]));
  std::vector<int4> disc;
  std::vector<double> cap;
  for (int oy = -ri; oy <= ri; ++oy)
    for (int ox = -ri; ox <= ri; ++ox) {
      const double q = rad * rad - (ox * r->texel[0]) * (ox * r->texel[0]) - (oy * r->texel[1]) * (oy * r->texel[1]);
      if (q <= 0) continue;
      disc.push_back(make_int4(ox, oy, 0, 0));     // H[y][x] takes top[y + oy][x + ox] (solver.py:759-763)
      cap.push_back(sqrt(q));
    }
  r->ndisc = (int)disc.size();
  r->disc = (int4*)ralloc(t, *r, disc.size() * 16);
  r->disc_h = (double*)ralloc(t, *r, cap.size() * 8);
  upload(t, r->disc, disc.data(), disc.size() * 16);
  upload(t, r->disc_h, cap.data(), cap.size() * 8);
  const double sigma = 1.5 * D.h / std::min(r->texel[0], r->texel[1]);
  r->blur_rad = (int)ceil(2.5 * sigma);
  std::vector<double> bw(2 * r->blur_rad + 1);
  for (int i = -r->blur_rad; i <= r->blur_rad; ++i) {
    const double x = i / sigma;
    bw[i + r->blur_rad] = exp(-0.5 * (x * x));
  }
  r->blur_w = (double*)ralloc(t, *r, bw.size() * 8);
  upload(t, r->blur_w, bw.data(), bw.size() * 8);
  CK(cudaStreamSynchronize(t.stream));
  return *r;
}

}  // namespace

size_t ripple_state_bytes(Tank& t) {
  if (t.d.rx <= 0) return 0;
  return (size_t)(2 * t.d.rx) * (2 * t.d.rz) * 8;
}

void clear_ripple(Tank& t) {
  if (t.d.rx <= 0 || !t.ripple) return;
  RippleState& r = *rs(t);
  CK(cudaMemsetAsync(r.S, 0, (size_t)r.Mx * r.Mz * 8, t.stream));
  CK(cudaMemsetAsync(r.field, 0, (size_t)(t.d.rx + 1) * (t.d.rz + 1) * 16, t.stream));
}

void free_ripple(Tank& t) {
  if (!t.ripple) return;
  RippleState* r = rs(t);
  for (void* p : r->mem) cudaFree(p);
  delete r;
  t.ripple = nullptr;
}

void copy_ripple_state(Tank& t, void* buf, bool save) {
  if (t.d.rx <= 0) return;
  RippleState& r = ensure(t);
  const size_t b = (size_t)r.Mx * r.Mz * 8;
  if (save) CK(cudaMemcpyAsync(buf, r.S, b, cudaMemcpyDeviceToDevice, t.stream));
  else CK(cudaMemcpyAsync(r.S, buf, b, cudaMemcpyDeviceToDevice, t.stream));
}

void compute_top_height(Tank& t) {
  RippleState& r = ensure(t);
  const int W = r.W;
  const int nb = (W * W + 255) / 256;
  CK(cudaMemsetAsync(r.topkey, 0, (size_t)W * W * 4, t.stream));
  k_top_scatter<<<t.solo->sm_count * 4, 256, 0, t.stream>>>(t.d, r.topkey, W, r.texel[0], r.texel[1]);
  k_top_dilate<<<nb, 256, 0, t.stream>>>(r.topkey, r.hA, W, r.disc, r.disc_h, r.ndisc, 1);
  k_top_blur<<<nb, 256, 0, t.stream>>>(r.hA, r.hA, r.hB, W, r.blur_w, r.blur_rad, 0);
  k_top_blur<<<nb, 256, 0, t.stream>>>(r.hB, r.hA, r.top, W, r.blur_w, r.blur_rad, 1);
  CK(cudaGetLastError());
}

void ripple_frame(Tank& t, double frame_dt) {
  if (t.d.rx <= 0) return;
  RippleState& r = ensure(t);
  compute_top_height(t);
  const int nv = (t.d.rx + 1) * (t.d.rz + 1);
  k_ripple_mask<<<(nv + 255) / 256, 256, 0, t.stream>>>(t.d, r.top, r.W, r.mx_coord, r.mz_coord, r.mask);
  const int nm = r.Mx * r.Mz, nb = (nm + 255) / 256;
  const double dx = r.Lx / t.d.rx, dz = r.Lz / t.d.rz;
  k_ripple_src<<<nb, 256, 0, t.stream>>>(t.d, t.d.rsrc, r.A, r.Mx, r.Mz, 1.0 / (dx * dz));
  CK(cudaMemsetAsync(t.d.rsrc, 0, (size_t)nv * 8, t.stream));
  fft2(t, r.A, -1.f);
  if (r.depth > 0 && frame_dt > 0) {
    if (!r.coef) {
      r.coef = (double4*)ralloc(t, r, (size_t)nm * sizeof(double4));
      r.kick = (double*)ralloc(t, r, (size_t)nm * sizeof(double));
    }
    if (frame_dt != r.coef_dt) {
      k_ripple_coef<<<nb, 256, 0, t.stream>>>(t.d, r.coef, r.kick, r.Mx, r.Mz, r.Lx, r.Lz, frame_dt, r.g, r.sigma_rho, r.rho, r.depth);
      r.coef_dt = frame_dt;
    }
    k_ripple_evolve_fixed<<<nb, 256, 0, t.stream>>>(r.S, r.A, r.coef, r.kick, nm);
  } else {
    k_ripple_evolve<<<nb, 256, 0, t.stream>>>(t.d, r.S, r.A, r.Mx, r.Mz, r.Lx, r.Lz, frame_dt, r.g, r.sigma_rho, r.rho, r.depth);
  }
  fft2(t, r.S, 1.f);
  k_ripple_field<<<nb, 256, 0, t.stream>>>(t.d, r.S, r.A, r.mask, r.field, r.Mx, r.Mz, dx, dz);
  fft2(t, r.A, -1.f);
  std::swap(r.S, r.A);
  CK(cudaGetLastError());
}

const double* ripple_top(Tank& t, int* W) {
  if (t.d.rx <= 0 || !t.ripple) return nullptr;
  *W = rs(t)->W;
  return rs(t)->top;
}

void frame_maps(Tank& t, const double sun_dir[3], float* out, size_t bytes) {
  const TankDev& D = t.d;
  if (D.rx <= 0) throw Error(-6, "this tank has no ripple layer");
  t.join();
  RippleState& r = ensure(t);
  const int W = r.W;
  const size_t nt = (size_t)W * W;
  if (out && bytes < nt * 16) throw Error(-1, "frame_maps: output buffer too small (" + std::to_string(nt * 16) + " bytes needed)");
  const double sn = sqrt(sun_dir[0] * sun_dir[0] + sun_dir[1] * sun_dir[1] + sun_dir[2] * sun_dir[2]);
  if (!(sn > 0) || !std::isfinite(sn)) throw Error(-1, "frame_maps: the sun direction must be a finite non-zero vector");
  LightParams P{};
  for (int a = 0; a < 3; ++a) P.sun[a] = sun_dir[a] / sn;
  const double st = sqrt(std::max(1 - P.sun[1] * P.sun[1], 0.0)) / 1.333;
  P.flat[0] = -P.sun[0] / 1.333; P.flat[1] = -sqrt(1 - st * st); P.flat[2] = -P.sun[2] / 1.333;
  P.tex[0] = r.texel[0]; P.tex[1] = r.texel[1];
  P.Lx = r.Lx; P.Lz = r.Lz;
  P.mtex[0] = D.nx * D.h / W; P.mtex[1] = D.nz * D.h / W;
  if (!r.light) {
    r.light = (unsigned long long*)ralloc(t, r, nt * 8);
    r.maps = (float4*)ralloc(t, r, nt * 16);
  }
  CK(cudaMemsetAsync(r.light, 0, nt * 8, t.stream));
  const int ns = 4 * W * W;
  k_light_splat<<<(ns + 255) / 256, 256, 0, t.stream>>>(r.top, r.field, W, D.rx, D.rz, P, r.light);
  k_light_maps<<<(int)((nt + 255) / 256), 256, 0, t.stream>>>(r.light, r.top, r.field, W, D.rx, D.rz, P, r.maps);
  CK(cudaGetLastError());
  if (out) {
    CK(cudaMemcpyAsync(out, r.maps, nt * 16, cudaMemcpyDeviceToHost, t.stream));
    CK(cudaStreamSynchronize(t.stream));
  }
}

void read_ripple_field(Tank& t, int field, void* out, size_t bytes) {
  const TankDev& D = t.d;
  if (D.rx <= 0) throw Error(-6, "this tank has no ripple layer");
  RippleState& r = ensure(t);
  CK(cudaStreamSynchronize(t.stream));
  const size_t nv = (size_t)(D.rx + 1) * (D.rz + 1);
  auto need = [&](size_t b) { if (bytes < b) throw Error(-1, "read_grid: output buffer too small (" + std::to_string(b) + " bytes needed)"); };
  if (field == 7) {
    need(nv * 8);
    std::vector<long long> v(nv);
    CK(cudaMemcpy(v.data(), D.rsrc, nv * 8, cudaMemcpyDeviceToHost));
    double* o = (double*)out;
    for (size_t i = 0; i < nv; ++i) o[i] = (double)v[i] / kRippleFix;
  } else if (field == 8) {
    need(nv * 12);
    std::vector<float4> v(nv);
    CK(cudaMemcpy(v.data(), r.field, nv * 16, cudaMemcpyDeviceToHost));
    float* o = (float*)out;
    for (size_t i = 0; i < nv; ++i) { o[3 * i] = v[i].x; o[3 * i + 1] = v[i].y; o[3 * i + 2] = v[i].z; }
  } else if (field == 9) {
    need((size_t)r.W * r.W * 4);
    std::vector<double> v((size_t)r.W * r.W);
    CK(cudaMemcpy(v.data(), r.top, v.size() * 8, cudaMemcpyDeviceToHost));
    float* o = (float*)out;
    for (size_t i = 0; i < v.size(); ++i) o[i] = (float)v[i];
  } else if (field == 10) {
    need((size_t)r.Mx * r.Mz * 8);
    CK(cudaMemcpy(out, r.S, (size_t)r.Mx * r.Mz * 8, cudaMemcpyDeviceToHost));
  } else if (field == 11) {
    need(nv * 4);
    CK(cudaMemcpy(out, r.mask, nv * 4, cudaMemcpyDeviceToHost));
  } else if (field == 12) {
    need((size_t)r.W * r.W * 8);
    CK(cudaMemcpy(out, r.top, (size_t)r.W * r.W * 8, cudaMemcpyDeviceToHost));
  } else {
    throw Error(-1, "unknown grid field");
  }
}

}  // namespace suiri
