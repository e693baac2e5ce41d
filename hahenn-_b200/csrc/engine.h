// Host-side engine: tanks (device state of one scene), groups (tanks stepped by shared batched launches)
// and the sub-step / frame sequence. The C ABI (capi.cpp) is a thin layer over this.
#pragma once
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "launch.cuh"
#include "scene.h"

namespace suiri {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);
#define CK(x) ::suiri::cuda_check((x), #x)

struct Group;
struct Tank;

// ripple layer and top-view height map (ripple.cu)
size_t ripple_state_bytes(Tank& t);
void clear_ripple(Tank& t);
void ripple_frame(Tank& t, double frame_dt);
void read_ripple_field(Tank& t, int field, void* out, size_t bytes);
void frame_maps(Tank& t, const double sun_dir[3], float* out, size_t bytes);   // W² float4 (top, slope x, slope z, light)
void copy_ripple_state(Tank& t, void* dst_or_src, bool save);
void free_ripple(Tank& t);

const double* ripple_top(Tank& t, int* W);   // the last frame's top-view height map (W², -1 dry) or null

// surface mesh of the liquid (mesh.cu)
struct MeshInfo {
  long long verts = 0, quads = 0, tris = 0, body_verts = 0, lone = 0;
  int lattice[3] = {0, 0, 0};
  int taps = 0;
  double lo[3] = {0, 0, 0}, spacing = 0, smooth = 0;
  double weights[33] = {};
  double phase_ms[5] = {};        // device time: classify, distance field, blur, surface nets, finish
};
MeshInfo build_surface_mesh(Tank& t, double smooth);
void read_surface_mesh(Tank& t, float* pos, float* vel, int32_t* quads, int32_t* tris, long long max_verts,
                       long long max_quads, long long max_tris);
void free_mesh(Tank& t);

uint32_t hash_host(uint32_t x);

struct TankConfig {
  int nx = 0, ny = 0, nz = 0, nyl = 0;
  double h = 0, origin[3] = {0, 0, 0};
  double flip = 0.96, omega = 1.6, g = 9.81, friction = 0.03, ppc = 8.0, drift = 6.0, ww_rate = 7.0;
  int iters = 40, whitewater = 1;
  long long cap = 320000, ww_cap = 140000;
  int rx = 256, rz = 256, wmap = 256;
  int sdf_mode = kSdfAnalytic, device = 0;
  uint32_t seed = 1;
  double ripple_sigma = 0.0728, ripple_rho = 998.0, ripple_depth = 0.0;
  int advect = 0;                 // 0 explicit Euler (the reference), 1 RK2 midpoint through the grid velocity
  double drop_d_median = 0, drop_d_sigma = 0;   // lognormal sub-grid drop diameters (0: the particle mass)
  int sor_mode = 0;               // form of the pressure solve of the tank's own group (-1: cluster-resident where it fits)
  long long watchdog_polls = kWatchdogPolls;    // polls of a bounded device wait before it gives up
  cudaStream_t stream = nullptr;  // use this stream instead of creating one (not owned)
};

// device bytes a tank of this configuration allocates (admission by HBM budget)
size_t tank_bytes(const TankConfig& c);

// Pinned host memory through a process-wide cache of blocks (powers of two from 4 KB, up to 2 GB cached):
// handing pinned memory back to the driver synchronises the device, which would stall every batch running
// on it whenever a scene is released (serving). pinned_get returns a block of at least `bytes` (its size in
// *got when given); pinned_put takes it back with the same request size.
void* pinned_get(size_t bytes, size_t* got = nullptr);
void pinned_put(void* p, size_t bytes);
// true when both ends of [p, p + bytes) are page-locked host memory (registered or allocated by CUDA)
bool host_pinned(const void* p, size_t bytes);

struct PrevXf { double pos[3]; double R[9]; };

struct Snapshot {
  int id = 0;
  bool valid = false;
  float4 *p = nullptr, *v = nullptr, *wp = nullptr, *wv = nullptr;
  float* pres = nullptr;
  void* ripple = nullptr;
  size_t ripple_bytes = 0;
  Counters ctr{};
  long long n = 0;
  double time = 0, vmax = 1;
  uint32_t next_id = 0;
  std::map<int, std::vector<double>> emit_state;
};

struct Tank {
  TankConfig cfg;
  TankDev d{};                    // host image of the device descriptor
  Counters* h_ctr = nullptr;      // host mirror for reads
  cudaStream_t stream = nullptr;
  std::vector<void*> dmem;        // device allocations owned by the tank
  Obj* d_objs = nullptr;
  double* d_lattice = nullptr;
  int* d_oid = nullptr;
  Scene scene;                    // water blocks and sources of the scene (reset, step)
  std::vector<Obj> objs;
  std::map<int, PrevXf> prev_xf;
  std::map<int, std::vector<double>> emit_state;   // per source: acc, liters, timer, fired
  bool geom_dirty = true;
  int version = 1;                // bumps when the descriptor changes
  double time = 0, vmax = 1.0;
  uint32_t next_id = 0;
  long long n_emit_host = 0;      // particles staged in E for the next sub-step
  long long n_upper = 0;          // upper bound of live particles (exact after a stats read)
  unsigned char* h_stage[2] = {};  // pinned staging of added particles (packed as given), used in turn
  size_t stage_cap[2] = {};        // bytes
  unsigned char* d_stage = nullptr;  // their device copy, unpacked into E by a kernel
  size_t d_stage_cap = 0;
  cudaEvent_t copy_ev = nullptr;  // a direct copy from page-locked caller arrays has finished
  cudaEvent_t stage_ev[2] = {};   // the copies out of each staging buffer have finished
  int stage_k = 0;
  Counters* h_poll = nullptr;     // pinned target of the asynchronous counter read
  float4 *h_read_p = nullptr, *h_read_v = nullptr;   // pinned landing buffers of particle read-back
  size_t read_cap = 0;
  int* d_rcnt = nullptr;          // per-block live counts of the read-back compaction, then their prefix
  size_t rcnt_cap = 0;
  int* h_rcount = nullptr;        // pinned: the live count
  std::vector<cudaEvent_t> read_ev;   // one per copied chunk of the read-back
  cudaEvent_t poll_ev = nullptr;
  bool poll_pending = false;
  std::string err;
  Group* solo = nullptr;
  bool use_graphs = true;
  void* ripple = nullptr;          // ripple.cu state
  void* mesh = nullptr;            // mesh.cu state (allocated by the first surface mesh)
  Snapshot snap;
  long long emit_cap = 0;
  EmitterDev* d_emitters = nullptr;
  double emit_per_substep = 0;    // fixed emitters, particles per sub-step (host bound tracking)
  bool own_stream = true;
  cudaEvent_t ev_own = nullptr;   // marks this tank's own-stream work for a batch to wait on
  cudaEvent_t dep = nullptr;      // a batch's event this tank's own stream must wait for
  bool dirty = false;             // own-stream work enqueued since the last batch sub-step
  void join();                    // order own-stream work after the last batch sub-step

  void set_emitters(const std::vector<EmitterDev>& e);
  void eval_sdf(const double* pts, long long n, double* out);
  void eval_sdf_static(const double* pts, long long n, double* out);   // no device allocation

  explicit Tank(const TankConfig& c);
  ~Tank();
  void* alloc(size_t bytes);
  void upload_objects();
  void set_objects(const std::vector<Obj>& o);
  void set_lattice(const double* sdf, const int* oid, int lx, int ly, int lz);
  void read_counters();           // synchronous
  bool poll_counters(Counters& out);   // non-blocking: the last finished read into out (true); starts the next
  void add_particles(const float* pos, const float* vel, const float* air, long long n, uint32_t* first);
  void ensure_d_stage(size_t bytes);
  void unpack_staged(long long n, bool has_vel, bool has_air);
  void emit_block(const double lo[3], const double hi[3], bool fill);
  void clear();
  void reset();
  void substep(double dt);
  int step(double frame_dt);
  void frame_end(double frame_dt);
  void count_pass();
  void source_emits(double dt);
  long long read_particles(float* pos4, float* vel4, long long cap);
  long long read_whitewater(float* pos4, float* vel4, long long cap);
  void add_whitewater(const float* pos4, const float* vel4, long long n);
  void read_grid(int field, void* out, size_t bytes);
  int snapshot();
  void restore(int id);
};

struct Group {
  std::vector<Tank*> tanks;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  TankDev* d_tanks = nullptr;
  TankDev* h_tanks = nullptr;     // host images, uploaded by ensure_uploaded
  int* d_bpfx = nullptr;
  int* d_ppfx = nullptr;          // [0, n+1) in, [n+1, 2n+2) sorted
  long long* d_bsum = nullptr;
  LaunchCtx ctx{};
  std::vector<int> uploaded;      // tank versions last uploaded
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int max_iters = 0;
  cudaEvent_t ev_done = nullptr;  // recorded after every sub-step (tanks on other streams wait for it)
  int* d_hpfx = nullptr;          // colour-slot prefix for the persistent SOR
  int* d_apfx = nullptr;          // per colour, prefix of the active cells over the tanks
  void* d_tbl = nullptr;          // per-tile lists of the two-sweeps-per-launch solve (allocated when tuned to it)
  unsigned* d_ticket = nullptr;   // last-block tickets of the kernels that end in a prefix over tanks
  int* d_defer = nullptr;         // G2P form 2: the count, then the deferred particles' sorted indices
  void ensure_tbl();
  GridBarrier* d_barrier = nullptr;
  int sor_mode = 0;               // 0: one launch per colour sweep, 1: one cooperative launch per solve,
                                  // 2, 3: 2 or 4 sweeps per launch (temporal blocking), 4: cluster-resident
  int sor_blocks = 0;
  unsigned watchdog_polls = kWatchdogPolls;   // polls of a bounded device wait before it gives up (tanks' min)
  // cluster-resident solve (sor_mode 4): the CTA plan, planned by plan_cluster when tuned to it
  ClusterPiece* d_pieces = nullptr;
  struct ClusterClass {           // the tanks cut into `size` pieces: one launch of clusters of that size
    int size = 1, blocks = 0, smem = 0, first = 0;   // first = offset of its pieces in d_pieces
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
  };
  std::vector<ClusterClass> cl_classes;
  cudaEvent_t cl_fork = nullptr;
  void drop_cluster_classes();
  int cl_piece_kb = 0;            // shared memory per CTA at most, modes 4 and 1 (tile knob; 0: the device maximum)
  void plan_cluster();            // throws if a tank cannot be held by one cluster
  bool residual = false;          // FP64 residual of every solve into the tank counters
  int g2p_form = 0;               // 0 grid-stride walk, 1 per-brick with the faces in shared memory, 2 the walk's
                                  // common path with the rare branches deferred to a second pass (tuner knob)
  bool profile = false;           // record events between the phases of the sub-step (inside the graph too)
  static constexpr int kPhases = 6;   // binning+sort, P2G, node+cell passes, pressure solve, projection, G2P
  cudaEvent_t ev_ph[kPhases + 1] = {};
  double phase_ms(int k);         // phase k of the last sub-step (waits for it)
  int blocks_per_sm = 4;
  void set_profile(bool on);
  double sor_phase_ms();          // SOR phase of the last sub-step (waits for it)
  bool use_graphs = true;
  int sm_count = 148;

  // async_setup: the group's tables are set up on a stream of its own that the group's stream then waits for,
  // so building a group does not wait for work already queued on that stream (a serving lane replaces its
  // group while the previous one's sub-steps run)
  Group(const std::vector<Tank*>& t, cudaStream_t s, bool async_setup = false);
  ~Group();
  cudaStream_t setup = nullptr;   // async_setup: the stream of the first uploads
  cudaEvent_t setup_done = nullptr;
  bool uploaded_once = false;
  bool settled = false;           // the owner saw every launch of this group finish: no wait when destroyed
  void ensure_uploaded();
  void set_dt(double dt);
  double dev_dt = 0;              // the sub-step dt the device descriptors hold, when dt_on_device
  bool dt_on_device = false;
  void enqueue_body();            // the sub-step without GEOM
  void substep(double dt);
  void drop_graph();
};

// Size lanes: tanks under 2^16 cells, under 2^19, and larger. A batch (and the server) advances each lane
// as its own group on its own stream, so a lane of small tanks does not wait for the largest tank's
// kernels and the lanes' kernels overlap on the GPU.
constexpr int kSizeLanes = 3;
constexpr int kMaxLanes = 8;    // lanes a batch may be given explicitly
inline int size_lane(long long cells) { return cells < (1LL << 16) ? 0 : (cells < (1LL << 19) ? 1 : 2); }

// A batch of tanks: one group per occupied size lane. Every sub-step forks from the batch's stream to the
// lanes and joins back to it, so work ordered on that stream sees all of the batch's tanks.
struct Batch {
  std::vector<std::unique_ptr<Group>> lanes;
  cudaStream_t stream = nullptr;  // the single lane's stream, or an own stream the lanes fork from and join
  bool own_stream = false;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;

  explicit Batch(const std::vector<Tank*>& t, const int* lane_of = nullptr);   // lane_of: a lane per tank
  ~Batch();
  void substep(double dt);
};

}  // namespace suiri
