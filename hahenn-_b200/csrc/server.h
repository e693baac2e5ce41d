// Serving loop (server.cpp): continuous batching of scene solves under an HBM budget.
#pragma once
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.h"

namespace suiri {

enum ReqState { kQueued = 0, kRunning = 1, kDone = 2, kFailed = 3 };

struct Request {
  long long id = 0;
  TankConfig cfg;
  Scene scene;
  std::vector<EmitterDev> emitters;
  int steps = 0, steps_done = 0;
  bool keep_result = false;
  size_t bytes = 0;
  std::unique_ptr<Tank> tank;
  int state = kQueued;
  std::string err;
  double t_submit = 0, t_admit = 0, t_done = 0;
  double acc_particle_steps = 0, particle_steps = 0;
  long long start_count = 0;      // liquid particles at admission (after the scene's water blocks)
  long long final_count = 0;
  std::vector<float> res_pos, res_vel;
};

struct ServerStats {
  long long completed = 0, queued = 0, running = 0, failed = 0, rebuilds = 0, substeps = 0;
  double particle_steps = 0, elapsed_s = 0, used_bytes = 0, budget_bytes = 0, p50_ms = 0, p99_ms = 0, mean_active = 0;
};

// Resident scenes are batched by size lane (size_lane, engine.h): each lane has its own stream and batched
// graph and advances at its own pace, so a small scene's sub-steps do not wait for the largest scene's, and
// the lanes' kernels overlap on the GPU.
constexpr int kLanes = kSizeLanes;
constexpr int kLaneRunAhead = 4;                                      // sub-steps queued per lane at most

struct Lane {
  cudaStream_t stream = nullptr;
  std::vector<Request*> active;
  std::unique_ptr<Group> group;
  bool changed = false;
  std::deque<cudaEvent_t> inflight;   // one per queued sub-step, oldest first
  std::vector<cudaEvent_t> spare;
  // groups replaced while their sub-steps were still queued: each is destroyed, and the requests that ended
  // with it are finished, once the event recorded after its last sub-step has completed
  struct Retired {
    std::unique_ptr<Group> group;
    cudaEvent_t ev = nullptr;
    std::vector<Request*> done;
  };
  std::deque<Retired> retired;
};

struct Server {
  double budget, used = 0, dt;
  int dev;
  Lane lanes[kLanes];
  std::mutex m;
  std::condition_variable cv;
  std::deque<Request*> queue;
  std::map<long long, std::unique_ptr<Request>> reqs;
  std::thread worker;
  bool stop = false;
  long long next_id = 0, completed = 0, rebuilds = 0, substeps = 0, rounds = 0;
  double total_particle_steps = 0, sum_active = 0, t_start = 0;
  std::vector<double> lat_ms;

  Server(int device, double budget_bytes, double dt);
  ~Server();
  void retire(Lane& L, std::vector<Request*> done);
  void settle(Lane& L, bool wait);    // destroy the retired groups whose work has run (wait: all of them)
  long long submit(std::unique_ptr<Request> r);
  ServerStats stats();

 private:
  void loop();
  void admit_locked(std::vector<Request*>& admitted);
  void start_request(Request* r);
  void finish_request(Request* r);
  static int lane_of(const TankConfig& c);
  bool advance(Lane& L);                 // queue one sub-step of the lane if it may run ahead; true if it did
  void apply(Tank& t, const Scene& sc);
};

}  // namespace suiri
