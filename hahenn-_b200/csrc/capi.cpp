// extern "C" surface of libsuiri_cuda.so (include/suiri.h): argument checks, error codes and messages,
// no exception crosses the ABI.
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

#include "../../include/suiri.h"
#include "engine.h"
#include "server.h"

using namespace suiri;

struct suiri_tank {
  std::unique_ptr<Tank> t;
  std::string err;
};
struct suiri_batch {
  std::unique_ptr<Batch> b;
  std::string err;
};
struct suiri_server {
  std::unique_ptr<Server> s;
  std::string err;
};

// tank configuration from parameters and an optional scene (FluidSim sizing, quality presets)
TankConfig make_config(const suiri_params& p, const char* scene_json, Scene& sc);
// device records of fixed-rate emitters (direction normalised, outlet basis as basisOf, src/js/55-emit.js:4-9)
std::vector<EmitterDev> emitters_from(const suiri_emitter* e, int n);

namespace {

thread_local std::string g_err;

template <class F>
int guard(std::string* err, F&& f) {
  try {
    f();
    return SUIRI_OK;
  } catch (const Error& e) {
    if (err) *err = e.what();
    g_err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    const char* m = "host out of memory";
    if (err) *err = m;
    g_err = m;
    return SUIRI_ERR_NOMEM;
  } catch (const std::exception& e) {
    if (err) *err = e.what();
    g_err = e.what();
    return SUIRI_ERR_INVALID;
  }
}

struct Quality { const char* name; double h; long long cap, ww; int iters, ripple, wmap; };
// quality presets (src/js/50-sim.js:4-8, solver.py:23-27)
const Quality kQ[] = {{"low", 0.012, 140000, 60000, 28, 128, 256},
                      {"standard", 0.0085, 320000, 140000, 40, 256, 256},
                      {"high", 0.0065, 700000, 260000, 56, 512, 384}};

const Quality& quality(const char* q) {
  if (q)
    for (const auto& x : kQ)
      if (strcmp(x.name, q) == 0) return x;
  if (q && *q) throw Error(SUIRI_ERR_INVALID, std::string("unknown quality '") + q + "'");
  return kQ[1];
}

double js_round(double x) { return floor(x + 0.5); }

void rotvec(const double R[9], double out[3]) {
  // m3.log (src/js/00-util.js:53-60)
  const double c = std::min(std::max((R[0] + R[4] + R[8] - 1) / 2, -1.0), 1.0);
  const double ang = acos(c);
  out[0] = out[1] = out[2] = 0;
  if (ang < 1e-6) return;
  const double s = 2 * sin(ang);
  if (fabs(s) < 1e-6) return;
  out[0] = (R[7] - R[5]) / s * ang;
  out[1] = (R[2] - R[6]) / s * ang;
  out[2] = (R[3] - R[1]) / s * ang;
}

// obstacles of a scene → device records with velocities from the previous transforms (src/js/50-sim.js:165-211)
bool apply_solids(Tank& t, const std::vector<SceneItem>& items, double dt_move) {
  std::vector<Obj> objs;
  std::map<int, PrevXf> next;
  bool moving = false;
  for (const SceneItem& it : items) {
    if (objs.size() >= (size_t)kMaxObj) break;
    Obj o = it.obj;
    double lin[3] = {0, 0, 0}, ang[3] = {0, 0, 0};
    auto p = t.prev_xf.find(it.id);
    if (p != t.prev_xf.end() && dt_move > 0) {
      for (int a = 0; a < 3; ++a) lin[a] = (o.pos[a] - p->second.pos[a]) / dt_move;
      double M[9];   // R · prevᵀ
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
          M[r * 3 + c] = it.R[r * 3] * p->second.R[c * 3] + it.R[r * 3 + 1] * p->second.R[c * 3 + 1] + it.R[r * 3 + 2] * p->second.R[c * 3 + 2];
      rotvec(M, ang);
      for (int a = 0; a < 3; ++a) ang[a] /= dt_move;
      const double ll = sqrt(lin[0] * lin[0] + lin[1] * lin[1] + lin[2] * lin[2]);
      const double la = sqrt(ang[0] * ang[0] + ang[1] * ang[1] + ang[2] * ang[2]);
      if (ll > 1e-5 || la > 1e-4) moving = true;
      if (ll > 4) for (double& v : lin) v *= 4 / ll;
      if (la > 40) for (double& v : ang) v *= 40 / la;
    }
    PrevXf x;
    memcpy(x.pos, o.pos, sizeof(x.pos));
    memcpy(x.R, it.R, sizeof(x.R));
    next[it.id] = x;
    if (o.flag == 1) { memcpy(o.lin, lin, sizeof(lin)); memcpy(o.ang, ang, sizeof(ang)); }
    objs.push_back(o);
  }
  t.prev_xf = next;
  // a changed object list re-runs GEOM (the reference compares a signature of the packed records)
  bool same = objs.size() == t.objs.size();
  for (size_t i = 0; same && i < objs.size(); ++i) same = memcmp(&objs[i], &t.objs[i], sizeof(Obj)) == 0;
  if (!same) t.set_objects(objs);
  return moving;
}

Tank* T(suiri_tank* h) {
  if (!h || !h->t) throw Error(SUIRI_ERR_INVALID, "null tank handle");
  return h->t.get();
}

}  // namespace

namespace {
// the public stats from a copy of the device counters (alive = A without the dead flags + pending
// emissions: A's dead are only known after binning; n_sorted counts them out once the next sub-step, or a
// count pass, has run)
void fill_stats(Tank& t, const Counters& c, suiri_stats* s) {
  if (c.vmax_bits64 != 0ull) {
    const unsigned long long b = c.vmax_bits64 - 1ull;
    memcpy(&t.vmax, &b, 8);
  }
  const long long alive = (long long)c.n_live + c.n_emit;
  memset(s, 0, sizeof(*s));
  s->count = alive;
  s->ww_count = std::min<long long>(c.ww_count, t.d.ww_cap);
  s->impacts = c.impacts;
  s->vmax = t.vmax;
  s->time = t.time;
  s->liters = alive * t.d.vp * 1000;
  s->full = c.full;
  s->frame = c.frame;
  s->errors = c.err;
  s->nx = t.d.nx; s->ny = t.d.ny; s->nz = t.d.nz; s->h = t.d.h;
  s->origin[0] = t.d.ox; s->origin[1] = t.d.oy; s->origin[2] = t.d.oz;
  s->active_cells = (long long)c.n_act[0] + c.n_act[1];
  double rmax, hmax;
  memcpy(&rmax, &c.res_max_bits, 8);
  memcpy(&hmax, &c.rhs_max_bits, 8);
  s->residual_max = rmax;
  s->rhs_max = hmax;
  s->residual_rms = s->active_cells > 0 ? sqrt(c.res_sum2 / (double)s->active_cells) : 0.0;
  s->ripple_rx = std::max(t.d.rx, 0); s->ripple_rz = std::max(t.d.rz, 0);
  s->wmap = t.cfg.wmap;
}
}  // namespace

extern "C" {

int suiri_params_default(suiri_params* p) {
  if (!p) { g_err = "null params"; return SUIRI_ERR_INVALID; }
  memset(p, 0, sizeof(*p));
  p->size = sizeof(suiri_params);
  p->quality = "standard";
  p->clamp_tank = 1;
  p->flip = 0.96; p->omega = 1.6; p->iters = 0; p->gravity = 9.81; p->friction = 0.03;
  p->ppc = 8.0; p->drift = 6.0; p->ww_rate = 7.0; p->whitewater = 1;
  p->capacity = 0; p->ww_capacity = 0; p->ripple_rx = 0; p->ripple_rz = 0; p->wmap = 0;
  p->sdf_mode = 0; p->device = 0; p->seed = 1;
  p->ripple_sigma = 0.0728; p->ripple_rho = 998.0; p->ripple_depth = 0.0;
  p->sor_mode = 0; p->watchdog_polls = kWatchdogPolls;
  return SUIRI_OK;
}

int suiri_create(const char* scene_json, const suiri_params* params, suiri_tank** out) {
  if (!out) { g_err = "null output handle"; return SUIRI_ERR_INVALID; }
  *out = nullptr;
  suiri_params p;
  suiri_params_default(&p);
  if (params) {
    if (params->size != sizeof(suiri_params)) { g_err = "suiri_params.size mismatch (use suiri_params_default)"; return SUIRI_ERR_INVALID; }
    p = *params;
  }
  std::unique_ptr<suiri_tank> h(new suiri_tank());
  const int rc = guard(nullptr, [&] {
    Scene sc;
    const TankConfig c = make_config(p, scene_json, sc);
    h->t.reset(new Tank(c));
    h->t->scene = sc;
    apply_solids(*h->t, sc.solids, 0.0);
    for (const WaterBlock& b : sc.blocks) h->t->emit_block(b.lo, b.hi, false);
  });
  if (rc != SUIRI_OK) return rc;
  *out = h.release();
  return SUIRI_OK;
}

}  // extern "C"

TankConfig make_config(const suiri_params& p, const char* scene_json, Scene& sc) {
    const Quality& q = quality(p.quality);
    std::string err;
    if (scene_json) {
      const bool ok = parse_scene(scene_json, p.clamp_tank != 0, sc, err);
      if (!ok) throw Error(SUIRI_ERR_PARSE, err);
    }
    TankConfig c;
    if (p.nx > 0 && p.ny > 0 && p.nz > 0 && p.h > 0) {
      c.nx = p.nx; c.ny = p.ny; c.nz = p.nz; c.h = p.h;
    } else if (p.nx != 0 || p.ny != 0 || p.nz != 0 || p.h != 0) {
      throw Error(SUIRI_ERR_INVALID, "explicit grid needs nx, ny, nz and h all positive");
    } else {
      // FluidSim sizing (src/js/50-sim.js:33-38)
      c.nx = (int)std::max(8.0, js_round(sc.tank[0] / q.h));
      c.ny = (int)std::max(8.0, js_round(sc.tank[1] / q.h));
      c.nz = (int)std::max(8.0, js_round(sc.tank[2] / q.h));
      c.h = std::min(std::min(sc.tank[0] / c.nx, sc.tank[1] / c.ny), sc.tank[2] / c.nz);
    }
    c.origin[0] = -c.nx * c.h / 2; c.origin[1] = 0.0; c.origin[2] = -c.nz * c.h / 2;
    c.nyl = c.ny + std::max(0, (int)ceil(p.extra_height / c.h));
    c.flip = p.flip; c.omega = p.omega; c.g = p.gravity; c.friction = p.friction; c.ppc = p.ppc; c.drift = p.drift;
    c.ww_rate = p.ww_rate; c.whitewater = p.whitewater ? 1 : 0;
    c.iters = p.iters > 0 ? p.iters : q.iters;
    c.cap = p.capacity > 0 ? p.capacity : q.cap;
    c.ww_cap = p.ww_capacity > 0 ? p.ww_capacity : q.ww;
    if (p.ripple_rx < 0 || p.ripple_rz < 0) { c.rx = c.rz = 0; }
    else if (p.ripple_rx == 0 && p.ripple_rz == 0) { c.rx = c.rz = q.ripple; }
    else { c.rx = p.ripple_rx; c.rz = p.ripple_rz; }
    c.wmap = p.wmap > 0 ? p.wmap : q.wmap;
    if (c.wmap > 8192) throw Error(SUIRI_ERR_INVALID, "wmap at most 8192 texels a side");
    c.sdf_mode = p.sdf_mode;
    c.device = p.device;
    c.seed = p.seed;
    if (!(p.ripple_sigma >= 0) || !(p.ripple_rho > 0) || !(p.ripple_depth >= 0))
      throw Error(SUIRI_ERR_INVALID, "ripple sigma >= 0, rho > 0, depth >= 0");
    c.ripple_sigma = p.ripple_sigma; c.ripple_rho = p.ripple_rho; c.ripple_depth = p.ripple_depth;
    if (p.advect != 0 && p.advect != 1) throw Error(SUIRI_ERR_INVALID, "advect is 0 (Euler) or 1 (RK2)");
    c.advect = p.advect;
    if (!(p.drop_d_median >= 0) || !(p.drop_d_sigma_log >= 0) || p.drop_d_median > 0.02)
      throw Error(SUIRI_ERR_INVALID, "drop_d_median in [0, 0.02] m, drop_d_sigma_log >= 0");
    c.drop_d_median = p.drop_d_median; c.drop_d_sigma = p.drop_d_sigma_log;
    if (p.sor_mode < -1 || p.sor_mode > 4) throw Error(SUIRI_ERR_INVALID, "sor_mode is -1 (auto) or 0..4");
    if (p.watchdog_polls < 0 || p.watchdog_polls > 0xFFFFFFFFLL) throw Error(SUIRI_ERR_INVALID, "watchdog_polls in [0, 2^32)");
    c.sor_mode = p.sor_mode;
    c.watchdog_polls = p.watchdog_polls;
    if (!(c.omega > 0 && c.omega < 2)) throw Error(SUIRI_ERR_INVALID, "omega must be in (0, 2)");
    if (c.cap > (1LL << 30)) throw Error(SUIRI_ERR_INVALID, "capacity above 2^30 particles");
    return c;
}

extern "C" {

int suiri_destroy(suiri_tank* t) {
  if (!t) return SUIRI_ERR_INVALID;
  const int rc = guard(nullptr, [&] { t->t.reset(); });
  delete t;
  return rc;
}

const char* suiri_last_error(const suiri_tank* t) {
  if (t) return t->err.c_str();
  return g_err.c_str();
}

int suiri_reset(suiri_tank* h) {
  return guard(h ? &h->err : nullptr, [&] { T(h)->reset(); });
}
int suiri_clear(suiri_tank* h) {
  return guard(h ? &h->err : nullptr, [&] { T(h)->clear(); });
}

int suiri_set_objects(suiri_tank* h, const char* items_json, double dt_move, int32_t* moving) {
  return guard(h ? &h->err : nullptr, [&] {
    Tank* t = T(h);
    if (!items_json) throw Error(SUIRI_ERR_INVALID, "null items JSON");
    JVal root;
    std::string err;
    if (!json_parse(items_json, root, err)) throw Error(SUIRI_ERR_PARSE, err);
    const JVal* items = &root;
    if (root.kind == JVal::Obj) {
      const JVal* s = root.get("scene");
      items = (s ? s : &root)->get("items");
      if (!items) throw Error(SUIRI_ERR_PARSE, "scene JSON: no items");
    }
    Scene sc;
    if (!parse_items(*items, sc, err)) throw Error(SUIRI_ERR_PARSE, err);
    const bool mv = apply_solids(*t, sc.solids, dt_move);
    t->scene.sources = sc.sources;
    t->scene.blocks = sc.blocks;
    if (moving) *moving = mv ? 1 : 0;
  });
}

int suiri_set_obstacles(suiri_tank* h, const suiri_object* objs, int32_t n) {
  return guard(h ? &h->err : nullptr, [&] {
    Tank* t = T(h);
    if (n < 0 || n > kMaxObj || (n > 0 && !objs)) throw Error(SUIRI_ERR_INVALID, "0..64 objects expected");
    std::vector<Obj> v(n);
    for (int i = 0; i < n; ++i) {
      Obj& o = v[i];
      memset(&o, 0, sizeof(o));
      const suiri_object& s = objs[i];
      if (s.flag != 1 && s.flag != 2) throw Error(SUIRI_ERR_INVALID, "object flag must be 1 (obstacle) or 2 (drain)");
      o.type = s.type; o.flag = s.flag;
      memcpy(o.pos, s.pos, sizeof(o.pos)); memcpy(o.rot, s.rot, sizeof(o.rot)); memcpy(o.dims, s.dims, sizeof(o.dims));
      memcpy(o.lin, s.lin, sizeof(o.lin)); memcpy(o.ang, s.ang, sizeof(o.ang));
      o.bound = s.flag == 1 ? bound_radius(o.type, o.dims) + 0.002 : o.dims[0] + 0.02;
    }
    t->set_objects(v);
  });
}

int suiri_set_lattice(suiri_tank* h, const double* sdf, const int32_t* oid, int32_t lx, int32_t ly, int32_t lz) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!sdf) throw Error(SUIRI_ERR_INVALID, "null lattice");
    T(h)->set_lattice(sdf, oid, lx, ly, lz);
  });
}

int suiri_eval_sdf(suiri_tank* h, const double* pts, int64_t n, double* out) {
  return guard(h ? &h->err : nullptr, [&] {
    if (n < 0 || (n > 0 && (!pts || !out))) throw Error(SUIRI_ERR_INVALID, "bad point arrays");
    T(h)->eval_sdf(pts, n, out);
  });
}

namespace {
std::mutex g_host_m;
std::map<void*, size_t> g_host_blocks;   // blocks handed out by suiri_host_alloc and their request sizes
}  // namespace

int suiri_host_alloc(size_t bytes, void** out) {
  return guard(nullptr, [&] {
    if (!out || bytes == 0) throw Error(SUIRI_ERR_INVALID, "bad host allocation arguments");
    *out = nullptr;
    void* p = pinned_get(bytes);
    std::lock_guard<std::mutex> g(g_host_m);
    g_host_blocks[p] = bytes;
    *out = p;
  });
}

int suiri_host_free(void* p) {
  return guard(nullptr, [&] {
    if (!p) return;
    size_t bytes = 0;
    {
      std::lock_guard<std::mutex> g(g_host_m);
      auto it = g_host_blocks.find(p);
      if (it == g_host_blocks.end()) throw Error(SUIRI_ERR_INVALID, "not a block of suiri_host_alloc");
      bytes = it->second;
      g_host_blocks.erase(it);
    }
    pinned_put(p, bytes);
  });
}

int suiri_eval_sdf_static(suiri_tank* h, const double* pts, int64_t n, double* out) {
  return guard(h ? &h->err : nullptr, [&] {
    if (n < 0 || (n > 0 && (!pts || !out))) throw Error(SUIRI_ERR_INVALID, "bad point arrays");
    T(h)->eval_sdf_static(pts, n, out);
  });
}

int suiri_scene_validate(const char* scene_json, int32_t clamp_tank, char* out, size_t cap, size_t* len) {
  return guard(nullptr, [&] {
    if (!scene_json || !len) throw Error(SUIRI_ERR_INVALID, "null scene or length");
    Scene sc;
    std::string err;
    if (!parse_scene(scene_json, clamp_tank != 0, sc, err)) throw Error(SUIRI_ERR_PARSE, err);
    const std::string txt = scene_json_text(sc);
    *len = txt.size();
    if (!out) return;
    if (cap <= txt.size()) throw Error(SUIRI_ERR_INVALID, "output buffer too small (" + std::to_string(txt.size() + 1) + " bytes needed)");
    memcpy(out, txt.c_str(), txt.size() + 1);
  });
}

int suiri_estimate_bytes(const char* scene_json, const suiri_params* params, double* bytes) {
  return guard(nullptr, [&] {
    if (!bytes) throw Error(SUIRI_ERR_INVALID, "null output");
    suiri_params p;
    suiri_params_default(&p);
    if (params) {
      if (params->size != sizeof(suiri_params)) throw Error(SUIRI_ERR_INVALID, "suiri_params.size mismatch");
      p = *params;
    }
    Scene sc;
    *bytes = (double)tank_bytes(make_config(p, scene_json, sc));
  });
}

int suiri_add_particles(suiri_tank* h, const float* pos, const float* vel, const float* airborne, int64_t n, uint32_t* first_id) {
  return guard(h ? &h->err : nullptr, [&] { T(h)->add_particles(pos, vel, airborne, n, first_id); });
}

int suiri_set_emitters(suiri_tank* h, const suiri_emitter* e, int32_t n) {
  return guard(h ? &h->err : nullptr, [&] { T(h)->set_emitters(emitters_from(e, n)); });
}

}  // extern "C"

std::vector<EmitterDev> emitters_from(const suiri_emitter* e, int n) {
    if (n < 0 || n > kMaxEmitters || (n > 0 && !e)) throw Error(SUIRI_ERR_INVALID, "0..8 emitters expected");
    std::vector<EmitterDev> v(n);
    for (int i = 0; i < n; ++i) {
      EmitterDev& d = v[i];
      memset(&d, 0, sizeof(d));
      if (e[i].shape != 0 && e[i].shape != 3) throw Error(SUIRI_ERR_INVALID, "emitter shape must be 0 (disc) or 3 (rain)");
      if (!(e[i].per_substep >= 0) || !(e[i].radius >= 0)) throw Error(SUIRI_ERR_INVALID, "emitter rate and radius must be >= 0");
      d.shape = e[i].shape; d.airborne = e[i].airborne ? 1 : 0;
      d.radius = e[i].radius; d.speed = e[i].speed; d.per_substep = e[i].per_substep;
      d.radius_z = e[i].radius_z > 0 ? e[i].radius_z : e[i].radius;
      memcpy(d.pos, e[i].pos, sizeof(d.pos));
      double l = sqrt(e[i].dir[0] * e[i].dir[0] + e[i].dir[1] * e[i].dir[1] + e[i].dir[2] * e[i].dir[2]);
      if (!(l > 0)) { d.dir[1] = -1; l = 1; } else { for (int a = 0; a < 3; ++a) d.dir[a] = e[i].dir[a] / l; }
      // basisOf (src/js/55-emit.js:4-9)
      const double ref[3] = {fabs(d.dir[1]) < 0.95 ? 0.0 : 1.0, fabs(d.dir[1]) < 0.95 ? 1.0 : 0.0, 0.0};
      double u[3] = {d.dir[1] * ref[2] - d.dir[2] * ref[1], d.dir[2] * ref[0] - d.dir[0] * ref[2], d.dir[0] * ref[1] - d.dir[1] * ref[0]};
      const double ul = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      for (int a = 0; a < 3; ++a) d.u[a] = u[a] / ul;
      d.w[0] = d.dir[1] * d.u[2] - d.dir[2] * d.u[1];
      d.w[1] = d.dir[2] * d.u[0] - d.dir[0] * d.u[2];
      d.w[2] = d.dir[0] * d.u[1] - d.dir[1] * d.u[0];
    }
    return v;
}

extern "C" {

int suiri_emit_block(suiri_tank* h, const double lo[3], const double hi[3], int32_t fill) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!lo || !hi) throw Error(SUIRI_ERR_INVALID, "null block corners");
    T(h)->emit_block(lo, hi, fill != 0);
  });
}

int suiri_substep(suiri_tank* h, double dt) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!(dt > 0) || !std::isfinite(dt)) throw Error(SUIRI_ERR_INVALID, "dt must be positive");
    T(h)->substep(dt);
  });
}

int suiri_step(suiri_tank* h, double frame_dt, int32_t* substeps) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!std::isfinite(frame_dt)) throw Error(SUIRI_ERR_INVALID, "frame_dt must be finite");
    const int n = T(h)->step(frame_dt);
    if (substeps) *substeps = n;
  });
}

int suiri_frame_end(suiri_tank* h, double frame_dt) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!(frame_dt > 0) || !std::isfinite(frame_dt)) throw Error(SUIRI_ERR_INVALID, "frame_dt must be positive");
    T(h)->frame_end(frame_dt);
  });
}

int suiri_sync(suiri_tank* h) {
  return guard(h ? &h->err : nullptr, [&] { CK(cudaStreamSynchronize(T(h)->stream)); });
}

int suiri_read_particles(suiri_tank* h, float* pos4, float* vel4, int64_t cap, int64_t* n) {
  return guard(h ? &h->err : nullptr, [&] {
    const long long k = T(h)->read_particles(pos4, vel4, cap);
    if (n) *n = k;
  });
}

int suiri_read_whitewater(suiri_tank* h, float* pos4, float* vel4, int64_t cap, int64_t* n) {
  return guard(h ? &h->err : nullptr, [&] {
    const long long k = T(h)->read_whitewater(pos4, vel4, cap);
    if (n) *n = k;
  });
}

int suiri_add_whitewater(suiri_tank* h, const float* pos4, const float* vel4, int64_t n) {
  return guard(h ? &h->err : nullptr, [&] { T(h)->add_whitewater(pos4, vel4, n); });
}

int suiri_read_grid(suiri_tank* h, int32_t field, void* out, size_t bytes) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!out) throw Error(SUIRI_ERR_INVALID, "null output");
    T(h)->read_grid(field, out, bytes);
  });
}

int suiri_frame_maps(suiri_tank* h, const double sun_dir[3], float* out, size_t bytes) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!sun_dir) throw Error(SUIRI_ERR_INVALID, "null sun direction");
    frame_maps(*T(h), sun_dir, out, bytes);
  });
}

int suiri_surface_mesh(suiri_tank* h, double smooth, suiri_mesh_info* info) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!info) throw Error(SUIRI_ERR_INVALID, "null mesh info");
    if (!(smooth > 0) || smooth > 6.0) throw Error(SUIRI_ERR_INVALID, "smooth (blur sigma in lattice nodes) in (0, 6]");
    const MeshInfo m = build_surface_mesh(*T(h), smooth);
    memset(info, 0, sizeof(*info));
    info->verts = m.verts; info->quads = m.quads; info->tris = m.tris;
    info->body_verts = m.body_verts; info->lone = m.lone;
    for (int a = 0; a < 3; ++a) { info->lattice[a] = m.lattice[a]; info->lo[a] = m.lo[a]; }
    info->taps = m.taps;
    info->spacing = m.spacing; info->smooth = m.smooth;
    for (int k = 0; k < m.taps && k < 33; ++k) info->weights[k] = m.weights[k];
    for (int k = 0; k < 5; ++k) info->phase_ms[k] = m.phase_ms[k];
  });
}

int suiri_surface_mesh_read(suiri_tank* h, float* verts, float* vel, int32_t* quads, int32_t* tris, int64_t max_verts,
                            int64_t max_quads, int64_t max_tris) {
  return guard(h ? &h->err : nullptr, [&] {
    read_surface_mesh(*T(h), verts, vel, quads, tris, max_verts, max_quads, max_tris);
  });
}

int suiri_get_stats(suiri_tank* h, suiri_stats* s) {
  return guard(h ? &h->err : nullptr, [&] {
    Tank* t = T(h);
    if (!s) throw Error(SUIRI_ERR_INVALID, "null stats");
    t->read_counters();
    fill_stats(*t, *t->h_ctr, s);
  });
}

int suiri_poll_stats(suiri_tank* h, suiri_stats* s, int32_t* fresh) {
  return guard(h ? &h->err : nullptr, [&] {
    Tank* t = T(h);
    if (!s) throw Error(SUIRI_ERR_INVALID, "null stats");
    Counters c;
    const bool f = t->poll_counters(c);
    if (fresh) *fresh = f ? 1 : 0;
    if (f) fill_stats(*t, c, s);
  });
}

size_t suiri_stats_readback_bytes(void) { return sizeof(Counters); }

int suiri_snapshot(suiri_tank* h, int32_t* id) {
  return guard(h ? &h->err : nullptr, [&] {
    const int k = T(h)->snapshot();
    if (id) *id = k;
  });
}

int suiri_restore(suiri_tank* h, int32_t id) {
  return guard(h ? &h->err : nullptr, [&] { T(h)->restore(id); });
}

int suiri_stream(suiri_tank* h, void** stream) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!stream) throw Error(SUIRI_ERR_INVALID, "null output");
    *stream = (void*)T(h)->stream;
  });
}

int suiri_use_graphs(suiri_tank* h, int32_t on) {
  return guard(h ? &h->err : nullptr, [&] { T(h)->use_graphs = on != 0; });
}

int suiri_batch_create(suiri_tank* const* tanks, int32_t n, suiri_batch** out) {
  if (!out || !tanks || n <= 0) { g_err = "batch needs tanks"; return SUIRI_ERR_INVALID; }
  *out = nullptr;
  std::unique_ptr<suiri_batch> b(new suiri_batch());
  const int rc = guard(nullptr, [&] {
    std::vector<Tank*> v;
    for (int i = 0; i < n; ++i) v.push_back(T(tanks[i]));
    b->b.reset(new Batch(v));
  });
  if (rc != SUIRI_OK) return rc;
  *out = b.release();
  return SUIRI_OK;
}

int suiri_batch_create_lanes(suiri_tank* const* tanks, int32_t n, const int32_t* lane_of, suiri_batch** out) {
  if (!out || !tanks || n <= 0) { g_err = "batch needs tanks"; return SUIRI_ERR_INVALID; }
  *out = nullptr;
  std::unique_ptr<suiri_batch> b(new suiri_batch());
  const int rc = guard(nullptr, [&] {
    std::vector<Tank*> v;
    std::vector<int> l;
    for (int i = 0; i < n; ++i) {
      v.push_back(T(tanks[i]));
      if (lane_of) {
        if (lane_of[i] < 0 || lane_of[i] >= kMaxLanes) throw Error(SUIRI_ERR_INVALID, "lane index in 0..7");
        l.push_back(lane_of[i]);
      }
    }
    b->b.reset(new Batch(v, lane_of ? l.data() : nullptr));
  });
  if (rc != SUIRI_OK) return rc;
  *out = b.release();
  return SUIRI_OK;
}

int suiri_batch_destroy(suiri_batch* b) {
  if (!b) return SUIRI_ERR_INVALID;
  const int rc = guard(nullptr, [&] { b->b.reset(); });
  delete b;
  return rc;
}

int suiri_batch_substep(suiri_batch* b, double dt) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b) throw Error(SUIRI_ERR_INVALID, "null batch");
    if (!(dt > 0) || !std::isfinite(dt)) throw Error(SUIRI_ERR_INVALID, "dt must be positive");
    b->b->substep(dt);
  });
}

int suiri_batch_sync(suiri_batch* b) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b) throw Error(SUIRI_ERR_INVALID, "null batch");
    CK(cudaStreamSynchronize(b->b->stream));
  });
}

static void tune_group(Group& g, int32_t particle_blocks_per_sm, int32_t sor_mode) {
  if (particle_blocks_per_sm < 1 || particle_blocks_per_sm > 32) throw Error(SUIRI_ERR_INVALID, "blocks per SM in 1..32");
  if (sor_mode < 0 || sor_mode > 4) throw Error(SUIRI_ERR_INVALID, "sor_mode is 0, 1, 2, 3 or 4");
  if (sor_mode == 1 && g.tanks.size() > 65535) throw Error(SUIRI_ERR_INVALID, "sor_mode 1 takes at most 65535 tanks");
  CK(cudaStreamSynchronize(g.stream));
  if (sor_mode == 4) g.plan_cluster();     // throws (and changes nothing else) when a tank does not fit
  g.blocks_per_sm = particle_blocks_per_sm;
  g.ctx.particle_blocks = particle_blocks_per_sm * g.sm_count;
  if (sor_mode == 2) g.ensure_tbl();
  g.sor_mode = sor_mode;
  g.drop_graph();
}

static void tune_piece(Group& g, int32_t piece_kb) {
  if (piece_kb < 0) throw Error(SUIRI_ERR_INVALID, "piece_kb must be >= 0");
  CK(cudaStreamSynchronize(g.stream));
  const int old = g.cl_piece_kb;
  g.cl_piece_kb = piece_kb;
  if (g.sor_mode == 4) {
    try {
      g.plan_cluster();
    } catch (...) {
      g.cl_piece_kb = old;
      throw;
    }
    g.drop_graph();
  } else if (g.sor_mode == 1) {
    g.drop_graph();                         // the persistent solve's shared memory per block
  }
}

static void tune_g2p(Group& g, int32_t form) {
  if (form < 0 || form > 2) throw Error(SUIRI_ERR_INVALID, "g2p form is 0, 1 or 2");
  if (form == g.g2p_form) return;
  CK(cudaStreamSynchronize(g.stream));
  g.g2p_form = form;
  g.drop_graph();
}

int suiri_tune_g2p(suiri_tank* h, int32_t form) {
  return guard(h ? &h->err : nullptr, [&] { tune_g2p(*T(h)->solo, form); });
}

int suiri_batch_tune_g2p(suiri_batch* b, int32_t form) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b) throw Error(SUIRI_ERR_INVALID, "null batch");
    for (auto& g : b->b->lanes) tune_g2p(*g, form);
  });
}

int suiri_batch_tune_lane(suiri_batch* b, int32_t lane, int32_t particle_blocks_per_sm, int32_t sor_mode,
                          int32_t piece_kb, int32_t g2p_form) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b) throw Error(SUIRI_ERR_INVALID, "null batch");
    if (lane < 0 || lane >= (int32_t)b->b->lanes.size()) throw Error(SUIRI_ERR_INVALID, "lane out of range");
    Group& g = *b->b->lanes[lane];
    tune_piece(g, piece_kb);
    tune_group(g, particle_blocks_per_sm, sor_mode);
    tune_g2p(g, g2p_form);
  });
}

static void set_residual(Group& g, bool on) {
  if (on == g.residual) return;
  CK(cudaStreamSynchronize(g.stream));
  g.residual = on;
  g.drop_graph();
}

int suiri_tune_piece(suiri_tank* h, int32_t piece_kb) {
  return guard(h ? &h->err : nullptr, [&] { tune_piece(*T(h)->solo, piece_kb); });
}

int suiri_batch_tune_piece(suiri_batch* b, int32_t piece_kb) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b) throw Error(SUIRI_ERR_INVALID, "null batch");
    for (auto& g : b->b->lanes) tune_piece(*g, piece_kb);
  });
}

int suiri_residual(suiri_tank* h, int32_t on) {
  return guard(h ? &h->err : nullptr, [&] { set_residual(*T(h)->solo, on != 0); });
}

int suiri_batch_residual(suiri_batch* b, int32_t on) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b) throw Error(SUIRI_ERR_INVALID, "null batch");
    for (auto& g : b->b->lanes) set_residual(*g, on != 0);
  });
}

int suiri_batch_tune(suiri_batch* b, int32_t particle_blocks_per_sm, int32_t sor_mode) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b) throw Error(SUIRI_ERR_INVALID, "null batch");
    for (auto& g : b->b->lanes) tune_group(*g, particle_blocks_per_sm, sor_mode);
  });
}

int suiri_tune(suiri_tank* h, int32_t particle_blocks_per_sm, int32_t sor_mode) {
  return guard(h ? &h->err : nullptr, [&] { tune_group(*T(h)->solo, particle_blocks_per_sm, sor_mode); });
}

int suiri_batch_stream(suiri_batch* b, void** stream) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b || !stream) throw Error(SUIRI_ERR_INVALID, "null batch or output");
    *stream = (void*)b->b->stream;
  });
}

int suiri_time_substeps(suiri_tank* h, double dt, int32_t steps, double* ms) {
  return guard(h ? &h->err : nullptr, [&] {
    Tank* t = T(h);
    if (!ms || steps <= 0) throw Error(SUIRI_ERR_INVALID, "bad timing arguments");
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    t->substep(dt);                        // make sure GEOM and graph capture are outside the timed region
    CK(cudaEventRecord(a, t->stream));
    for (int i = 0; i < steps; ++i) t->substep(dt);
    CK(cudaEventRecord(b, t->stream));
    CK(cudaEventSynchronize(b));
    float f = 0;
    CK(cudaEventElapsedTime(&f, a, b));
    *ms = f;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

int suiri_batch_time_substeps(suiri_batch* bt, double dt, int32_t steps, double* ms) {
  return guard(bt ? &bt->err : nullptr, [&] {
    if (!bt || !bt->b || !ms || steps <= 0) throw Error(SUIRI_ERR_INVALID, "bad timing arguments");
    Batch& g = *bt->b;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    g.substep(dt);
    CK(cudaEventRecord(a, g.stream));
    for (int i = 0; i < steps; ++i) g.substep(dt);
    CK(cudaEventRecord(b, g.stream));
    CK(cudaEventSynchronize(b));
    float f = 0;
    CK(cudaEventElapsedTime(&f, a, b));
    *ms = f;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

int suiri_profile(suiri_tank* h, int32_t on) {
  return guard(h ? &h->err : nullptr, [&] { T(h)->solo->set_profile(on != 0); });
}

int suiri_sor_phase_ms(suiri_tank* h, double* ms) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!ms) throw Error(SUIRI_ERR_INVALID, "null output");
    *ms = T(h)->solo->sor_phase_ms();
  });
}

int suiri_batch_profile(suiri_batch* b, int32_t on) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b) throw Error(SUIRI_ERR_INVALID, "null batch");
    for (auto& g : b->b->lanes) g->set_profile(on != 0);
  });
}

int suiri_batch_sor_phase_ms(suiri_batch* b, double* ms) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b || !ms) throw Error(SUIRI_ERR_INVALID, "null batch or output");
    double m = 0;
    for (auto& g : b->b->lanes) m = std::max(m, g->sor_phase_ms());   // lanes overlap: the longest
    *ms = m;
  });
}

int suiri_phase_ms(suiri_tank* h, double* ms) {
  return guard(h ? &h->err : nullptr, [&] {
    if (!ms) throw Error(SUIRI_ERR_INVALID, "null output");
    for (int k = 0; k < Group::kPhases; ++k) ms[k] = T(h)->solo->phase_ms(k);
  });
}

int suiri_batch_lanes(suiri_batch* b, int32_t* n) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b || !n) throw Error(SUIRI_ERR_INVALID, "null batch or output");
    *n = (int32_t)b->b->lanes.size();
  });
}

int suiri_batch_phase_ms(suiri_batch* b, int32_t lane, double* ms) {
  return guard(b ? &b->err : nullptr, [&] {
    if (!b || !b->b || !ms) throw Error(SUIRI_ERR_INVALID, "null batch or output");
    if (lane < 0 || lane >= (int32_t)b->b->lanes.size()) throw Error(SUIRI_ERR_INVALID, "lane out of range");
    for (int k = 0; k < Group::kPhases; ++k) ms[k] = b->b->lanes[lane]->phase_ms(k);
  });
}

int suiri_server_create(int32_t device, double budget_bytes, double dt, suiri_server** out) {
  if (!out) { g_err = "null output handle"; return SUIRI_ERR_INVALID; }
  *out = nullptr;
  std::unique_ptr<suiri_server> s(new suiri_server());
  const int rc = guard(nullptr, [&] {
    if (!(budget_bytes > 0) || !(dt > 0)) throw Error(SUIRI_ERR_INVALID, "budget and dt must be positive");
    s->s.reset(new Server(device, budget_bytes, dt));
  });
  if (rc != SUIRI_OK) return rc;
  *out = s.release();
  return SUIRI_OK;
}

int suiri_server_destroy(suiri_server* s) {
  if (!s) return SUIRI_ERR_INVALID;
  const int rc = guard(nullptr, [&] { s->s.reset(); });
  delete s;
  return rc;
}

int suiri_server_submit(suiri_server* s, const suiri_request* r, int64_t* id) {
  return guard(s ? &s->err : nullptr, [&] {
    if (!s || !s->s || !r || !id) throw Error(SUIRI_ERR_INVALID, "null server, request or output");
    if (r->size != sizeof(suiri_request)) throw Error(SUIRI_ERR_INVALID, "suiri_request.size mismatch");
    if (r->steps <= 0) throw Error(SUIRI_ERR_INVALID, "steps must be positive");
    suiri_params p;
    suiri_params_default(&p);
    if (r->params) {
      if (r->params->size != sizeof(suiri_params)) throw Error(SUIRI_ERR_INVALID, "suiri_params.size mismatch");
      p = *r->params;
    }
    std::unique_ptr<Request> q(new Request());
    q->cfg = make_config(p, r->scene_json, q->scene);
    q->emitters = emitters_from(r->emitters, r->n_emitters);
    q->steps = r->steps;
    q->keep_result = r->keep_result != 0;
    *id = s->s->submit(std::move(q));
  });
}

int suiri_server_poll(suiri_server* s, int64_t id, int32_t* state, double* latency_ms, int64_t* count) {
  return guard(s ? &s->err : nullptr, [&] {
    if (!s || !s->s) throw Error(SUIRI_ERR_INVALID, "null server");
    Server& S = *s->s;
    std::lock_guard<std::mutex> g(S.m);
    auto it = S.reqs.find(id);
    if (it == S.reqs.end()) throw Error(SUIRI_ERR_INVALID, "unknown request id");
    const Request& q = *it->second;
    if (state) *state = q.state;
    if (latency_ms) {
      const double now = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
      *latency_ms = 1000.0 * ((q.state >= kDone ? q.t_done : now) - q.t_submit);
    }
    if (count) *count = q.final_count;
    if (q.state == kFailed) s->err = q.err;
  });
}

int suiri_server_wait(suiri_server* s, int64_t id, double timeout_s) {
  return guard(s ? &s->err : nullptr, [&] {
    if (!s || !s->s) throw Error(SUIRI_ERR_INVALID, "null server");
    Server& S = *s->s;
    std::unique_lock<std::mutex> g(S.m);
    auto it = S.reqs.find(id);
    if (it == S.reqs.end()) throw Error(SUIRI_ERR_INVALID, "unknown request id");
    Request* q = it->second.get();
    const bool ok = S.cv.wait_for(g, std::chrono::duration<double>(timeout_s), [&] { return q->state >= kDone; });
    if (!ok) throw Error(SUIRI_ERR_STATE, "request not finished within the timeout");
    if (q->state == kFailed) throw Error(SUIRI_ERR_STATE, "request failed: " + q->err);
  });
}

int suiri_server_result(suiri_server* s, int64_t id, float* pos4, float* vel4, int64_t cap, int64_t* n) {
  return guard(s ? &s->err : nullptr, [&] {
    if (!s || !s->s) throw Error(SUIRI_ERR_INVALID, "null server");
    Server& S = *s->s;
    std::lock_guard<std::mutex> g(S.m);
    auto it = S.reqs.find(id);
    if (it == S.reqs.end()) throw Error(SUIRI_ERR_INVALID, "unknown request id");
    const Request& q = *it->second;
    if (q.state != kDone || !q.keep_result) throw Error(SUIRI_ERR_STATE, "no result (not done, or submitted without keep_result)");
    const long long k = (long long)q.res_pos.size() / 4;
    const long long m = std::min<long long>(k, cap);
    if (pos4 && m) memcpy(pos4, q.res_pos.data(), m * 16);
    if (vel4 && m) memcpy(vel4, q.res_vel.data(), m * 16);
    if (n) *n = k;
  });
}

int suiri_server_get_stats(suiri_server* s, suiri_server_stats* st) {
  return guard(s ? &s->err : nullptr, [&] {
    if (!s || !s->s || !st) throw Error(SUIRI_ERR_INVALID, "null server or output");
    const ServerStats x = s->s->stats();
    st->completed = x.completed; st->queued = x.queued; st->running = x.running; st->failed = x.failed;
    st->rebuilds = x.rebuilds; st->substeps = x.substeps; st->particle_steps = x.particle_steps;
    st->elapsed_s = x.elapsed_s; st->used_bytes = x.used_bytes; st->budget_bytes = x.budget_bytes;
    st->p50_ms = x.p50_ms; st->p99_ms = x.p99_ms; st->mean_active = x.mean_active;
  });
}

int suiri_time_sor(suiri_tank* h, int32_t iters, double* ms) {
  return guard(h ? &h->err : nullptr, [&] {
    Tank* t = T(h);
    if (!ms || iters <= 0) throw Error(SUIRI_ERR_INVALID, "bad timing arguments");
    Group& g = *t->solo;
    g.ensure_uploaded();
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, g.stream));
    for (int it = 0; it < iters; ++it) {
      launch_sor_sweep(g.ctx, 0, 0);
      launch_sor_sweep(g.ctx, 1, 0);
    }
    CK(cudaEventRecord(b, g.stream));
    CK(cudaEventSynchronize(b));
    CK(cudaGetLastError());
    float f = 0;
    CK(cudaEventElapsedTime(&f, a, b));
    *ms = f / (2.0 * iters);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

}  // extern "C"
