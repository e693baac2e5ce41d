// Serving: a request loop that admits scene solves by HBM budget and advances every resident scene with
// shared batched launches (continuous batching). Requests arriving while others run are admitted at the
// next sub-step boundary as memory frees up; finished ones leave at a boundary and their memory returns
// to the budget. Resident scenes are grouped in lanes by size, one stream and one batch per lane; each lane
// queues up to kLaneRunAhead sub-steps ahead of the device and is refilled as its sub-steps complete. All
// device work is issued by one worker thread; the state of a request stays on the device from admission
// to completion.
#include "server.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

namespace suiri {

namespace {
double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

Server::Server(int device, double budget_bytes, double dt_) : budget(budget_bytes), dt(dt_), dev(device) {
  CK(cudaSetDevice(device));
  for (Lane& L : lanes) CK(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
  t_start = now_s();
  worker = std::thread([this] { loop(); });
}

int Server::lane_of(const TankConfig& c) { return size_lane((long long)c.nx * c.ny * c.nz); }

Server::~Server() {
  {
    std::lock_guard<std::mutex> g(m);
    stop = true;
  }
  cv.notify_all();
  if (worker.joinable()) worker.join();
  cudaSetDevice(dev);
  for (Lane& L : lanes) {
    try {
      settle(L, true);
    } catch (const Error&) {
      for (auto& r : L.retired) if (r.ev) cudaEventDestroy(r.ev);
      L.retired.clear();
    }
    L.group.reset();
  }
  for (auto& kv : reqs) kv.second->tank.reset();
  for (Lane& L : lanes) {
    cudaStreamSynchronize(L.stream);
    for (cudaEvent_t e : L.inflight) cudaEventDestroy(e);
    for (cudaEvent_t e : L.spare) cudaEventDestroy(e);
    cudaStreamDestroy(L.stream);
  }
}

long long Server::submit(std::unique_ptr<Request> r) {
  r->t_submit = now_s();
  r->bytes = tank_bytes(r->cfg);
  std::lock_guard<std::mutex> g(m);
  const long long id = ++next_id;
  r->id = id;
  if ((double)r->bytes > budget) {
    r->state = kFailed;
    r->err = "request needs " + std::to_string(r->bytes) + " bytes, more than the whole budget";
    r->t_done = r->t_submit;
  } else {
    queue.push_back(r.get());
  }
  reqs[id] = std::move(r);
  cv.notify_all();
  return id;
}

void Server::admit_locked(std::vector<Request*>& admitted) {
  // FIFO admission: the head waits until it fits, so large scenes are not starved by small ones
  while (!queue.empty()) {
    Request* r = queue.front();
    if (used + (double)r->bytes > budget) break;
    queue.pop_front();
    used += (double)r->bytes;
    r->state = kRunning;
    admitted.push_back(r);
  }
}

void Server::start_request(Request* r) {
  try {
    r->cfg.stream = lanes[lane_of(r->cfg)].stream;
    r->cfg.device = dev;
    r->tank.reset(new Tank(r->cfg));
    Tank& t = *r->tank;
    t.scene = r->scene;
    apply(t, r->scene);
    for (const WaterBlock& b : r->scene.blocks) t.emit_block(b.lo, b.hi, false);
    if (!r->emitters.empty()) t.set_emitters(r->emitters);
    t.read_counters();
    r->start_count = t.h_ctr->n_live + t.h_ctr->n_emit;
    r->t_admit = now_s();
  } catch (const Error& e) {
    r->tank.reset();
    r->state = kFailed;
    r->err = e.what();
    r->t_done = now_s();
    std::lock_guard<std::mutex> g(m);
    used -= (double)r->bytes;
  }
}

void Server::finish_request(Request* r) {
  Tank& t = *r->tank;
  t.read_counters();
  r->final_count = t.h_ctr->n_live;
  if (const int bits = t.h_ctr->err) {
    // a bounded device wait of this scene's solves gave up: its results are not those of the full solve
    r->tank.reset();
    const double tdone = now_s();
    std::lock_guard<std::mutex> g(m);
    used -= (double)r->bytes;
    r->err = "device error bits " + std::to_string(bits) + " (1: a grid-barrier wait of the pressure solve gave up)";
    r->t_done = tdone;
    r->state = kFailed;
    cv.notify_all();
    return;
  }
  if (r->keep_result) {
    const long long n = t.read_particles(nullptr, nullptr, 0);
    r->res_pos.resize(4 * n);
    r->res_vel.resize(4 * n);
    t.read_particles(r->res_pos.data(), r->res_vel.data(), n);
  }
  r->tank.reset();
  const double tdone = now_s();
  std::lock_guard<std::mutex> g(m);
  used -= (double)r->bytes;
  r->t_done = tdone;
  r->state = kDone;
  lat_ms.push_back(1000.0 * (r->t_done - r->t_submit));
  ++completed;
  cv.notify_all();
}

// a lane's group is replaced without waiting for its queued sub-steps: it is kept, with the requests that
// ended with it, until an event after its last sub-step has completed
void Server::retire(Lane& L, std::vector<Request*> done) {
  Lane::Retired r;
  r.group = std::move(L.group);
  r.done = std::move(done);
  CK(cudaEventCreateWithFlags(&r.ev, cudaEventDisableTiming));
  CK(cudaEventRecord(r.ev, L.stream));
  L.retired.push_back(std::move(r));
}

void Server::settle(Lane& L, bool wait) {
  while (!L.retired.empty()) {
    Lane::Retired& r = L.retired.front();
    if (wait) {
      CK(cudaEventSynchronize(r.ev));
    } else {
      const cudaError_t q = cudaEventQuery(r.ev);
      if (q == cudaErrorNotReady) break;
      CK(q);
    }
    if (r.group) r.group->settled = true;
    r.group.reset();
    cudaEventDestroy(r.ev);
    std::vector<Request*> done = std::move(r.done);
    L.retired.pop_front();
    for (Request* q : done) finish_request(q);
  }
}

bool Server::advance(Lane& L) {
  settle(L, false);
  // sub-steps of this lane that have finished on the device free their places
  while (!L.inflight.empty()) {
    const cudaError_t q = cudaEventQuery(L.inflight.front());
    if (q == cudaErrorNotReady) break;
    CK(q);
    L.spare.push_back(L.inflight.front());
    L.inflight.pop_front();
  }
  if ((int)L.inflight.size() >= kLaneRunAhead) return false;
  if (L.changed || !L.group) {
    if (L.group) retire(L, {});
    std::vector<Tank*> ts;
    for (Request* r : L.active) ts.push_back(r->tank.get());
    L.group.reset(new Group(ts, L.stream, true));
    // the lanes run at the same time: a lane's persistent solve (sor_mode 1) takes at most its share of the SMs,
    // so that the cooperative launches of all lanes are resident together
    L.group->sor_blocks = std::max(1, std::min(L.group->sor_blocks, L.group->sm_count / kSizeLanes));
    ++rebuilds;
    L.changed = false;
  }
  try {
    L.group->substep(dt);
  } catch (const Error& e) {
    // a failed launch ends every request of this batch with the message; the server keeps serving
    for (Request* r : L.active) {
      r->state = kFailed;
      r->err = e.what();
      r->t_done = now_s();
      r->tank.reset();
      std::lock_guard<std::mutex> g(m);
      used -= (double)r->bytes;
    }
    L.active.clear();
    L.group.reset();
    return true;
  }
  cudaEvent_t ev;
  if (L.spare.empty()) {
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  } else {
    ev = L.spare.back();
    L.spare.pop_back();
  }
  CK(cudaEventRecord(ev, L.stream));
  L.inflight.push_back(ev);
  ++substeps;
  {
    // work done: every resident scene of the lane advanced one sub-step (particles counted at admission)
    double w = 0;
    for (Request* r : L.active) w += (double)r->start_count;
    std::lock_guard<std::mutex> g(m);
    total_particle_steps += w;
  }
  std::vector<Request*> still, done;
  for (Request* r : L.active) (++r->steps_done >= r->steps ? done : still).push_back(r);
  if (!done.empty()) {
    retire(L, std::move(done));      // the group refers to the tanks, which are freed once it has run
    L.changed = true;
  }
  L.active.swap(still);
  return true;
}

void Server::loop() {
  cudaSetDevice(dev);
  while (true) {
    std::vector<Request*> admitted;
    bool idle = true;
    for (Lane& L : lanes) idle &= L.active.empty() && L.retired.empty();
    {
      std::unique_lock<std::mutex> g(m);
      if (idle && queue.empty()) cv.wait_for(g, std::chrono::milliseconds(20));
      if (stop) break;
      admit_locked(admitted);
    }
    for (Request* r : admitted) {
      start_request(r);
      if (r->state == kRunning) {
        Lane& L = lanes[lane_of(r->cfg)];
        L.active.push_back(r);
        L.changed = true;
      }
    }
    bool any = false, moved = false;
    long long resident = 0;
    for (Lane& L : lanes) resident += (long long)L.active.size();
    for (Lane& L : lanes) {
      if (L.active.empty()) {
        settle(L, false);
        continue;
      }
      any = true;
      moved |= advance(L);
    }
    if (!any) {
      std::this_thread::sleep_for(std::chrono::microseconds(20));   // only retired groups left to finish
      continue;
    }
    if (moved) {
      ++rounds;
      sum_active += (double)resident;
    } else {
      std::this_thread::sleep_for(std::chrono::microseconds(20));   // every lane is its run-ahead in front
    }
  }
}

void Server::apply(Tank& t, const Scene& sc) {
  std::vector<Obj> objs;
  for (const SceneItem& it : sc.solids) objs.push_back(it.obj);
  if (!objs.empty()) t.set_objects(objs);
}

ServerStats Server::stats() {
  std::lock_guard<std::mutex> g(m);
  ServerStats s;
  s.completed = completed;
  s.queued = (long long)queue.size();
  long long running = 0, failed = 0;
  for (auto& kv : reqs) {
    running += kv.second->state == kRunning;
    failed += kv.second->state == kFailed;
  }
  s.running = running;
  s.failed = failed;
  s.particle_steps = total_particle_steps;
  s.elapsed_s = now_s() - t_start;
  s.used_bytes = used;
  s.budget_bytes = budget;
  s.rebuilds = rebuilds;
  s.substeps = substeps;
  s.mean_active = rounds ? sum_active / rounds : 0.0;
  std::vector<double> l = lat_ms;
  std::sort(l.begin(), l.end());
  auto pct = [&](double q) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)floor(q * (l.size() - 1) + 0.5))]; };
  s.p50_ms = pct(0.50);
  s.p99_ms = pct(0.99);
  return s;
}

}  // namespace suiri
