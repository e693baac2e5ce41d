/* libsuiri_cuda.so — B200-native FLIP liquid step of 水理ラボ (suiri-lab), C ABI.
 *
 * Plain pointers and sizes only; no CUDA or PyTorch types in the signatures. Every function returns
 * SUIRI_OK (0) or a negative SUIRI_ERR_* code; the message of the last failure of a handle is
 * suiri_last_error(handle) (suiri_last_error(NULL): the last failure of this thread without a handle).
 * No exception crosses the ABI.
 *
 * Coordinates are the reference's solver coordinates: metres, y up, floor at y = 0, the tank centred on
 * x = z = 0 (blender_addon/suiri_lab/solver.py:5-7, src/js/50-sim.js:38).
 *
 * Threading: a handle belongs to one host thread at a time. Each tank (and each batch) has its own CUDA
 * stream; stepping functions enqueue work and return; reads, stats and suiri_sync block.
 */
#ifndef SUIRI_H
#define SUIRI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SUIRI_OK 0
#define SUIRI_ERR_INVALID (-1)   /* bad argument or handle */
#define SUIRI_ERR_CUDA (-2)      /* a CUDA call failed (message names it) */
#define SUIRI_ERR_NOMEM (-3)     /* device memory or HBM budget exhausted */
#define SUIRI_ERR_CAPACITY (-4)  /* particle capacity reached (the particles that fit were kept) */
#define SUIRI_ERR_PARSE (-5)     /* malformed scene JSON */
#define SUIRI_ERR_STATE (-6)     /* call not valid now (e.g. restoring a consumed snapshot) */

typedef struct suiri_tank suiri_tank;
typedef struct suiri_batch suiri_batch;
typedef struct suiri_server suiri_server;

/* Construction parameters. Fill with suiri_params_default, then change what differs. */
typedef struct suiri_params {
  uint32_t size;           /* sizeof(suiri_params) */
  /* grid: nx,ny,nz,h > 0 give it explicitly; otherwise it is derived from the scene's tank size and
     the quality's cell size like FluidSim (src/js/50-sim.js:31-38): n = max(8, round(size/h)),
     h = min(w/nx, h/ny, d/nz), origin (-nx h/2, 0, -nz h/2) */
  int32_t nx, ny, nz;
  double h;
  const char* quality;     /* "low" | "standard" | "high" (src/js/50-sim.js:4-8) */
  int32_t clamp_tank;      /* 1: the editor's tank limits apply to scene JSON (src/js/80-ui.js:459) */
  double extra_height;     /* obstacle lattice above the rim [m] (solver.py:69-70) */
  /* physics (src/js/50-sim.js:151-162, solver.py:11-21) */
  double flip;             /* FLIP/PIC blend (0.96) */
  double omega;            /* SOR over-relaxation (1.6) */
  int32_t iters;           /* SOR iterations (quality) */
  double gravity;          /* 9.81 */
  double friction;         /* 0.03 */
  double ppc;              /* particles per cell at rest (8) */
  double drift;            /* drift correction strength (6) */
  double ww_rate;          /* whitewater spawn rate (7) */
  int32_t whitewater;      /* 1: spawn and advance whitewater */
  /* capacities */
  int64_t capacity;        /* particles (quality cap) */
  int64_t ww_capacity;     /* whitewater particles (quality ww) */
  /* ripple layer: (rx+1)×(rz+1) vertices over the footprint; 0,0 → quality R×R; -1 → none */
  int32_t ripple_rx, ripple_rz;
  int32_t wmap;            /* top-view height map texels per side (256/384) */
  int32_t sdf_mode;        /* 0 analytic obstacle shapes (web version), 1 distance lattice (Blender) */
  int32_t device;          /* CUDA device ordinal */
  uint32_t seed;           /* emission jitter seed */
  /* ripple dispersion ω² = (g k + σ/ρ k³) tanh(k d) (solver.py:887; 64-ripple.js:74) */
  double ripple_sigma;     /* surface tension σ [N/m] (0.0728) */
  double ripple_rho;       /* density ρ [kg/m³] (998) */
  double ripple_depth;     /* d [m]; 0: mean depth from the liquid volume each frame (solver.py:726) */
  /* particle advection: 0 explicit Euler x0 + v·dt with the blended velocity, as the reference
     (solver.py:545-550, 31-wgsl-sim2.js:168); 1 second-order midpoint (RK2) through the interpolated grid
     velocity u for in-grid particles, x0 + u(x0 + u(x0)·dt/2)·dt (not in the reference) */
  int32_t advect;
  /* sub-grid drop diameters (not in the reference, whose merging drops all carry the particle mass
     998·(h/2)³, src/js/31-wgsl-sim2.js:224, solver.py:596): drop_d_median > 0 gives every drop its own
     diameter, lognormal with this median [m] and log-standard-deviation drop_d_sigma_log, drawn from the
     drop's carried id; its impulse and crown then use the drop's mass 998·π/6·D³ */
  double drop_d_median;
  double drop_d_sigma_log;
  /* form of the pressure solve of the tank's own sub-steps, and of a batch or serving lane whose first tank
     it is (sor_mode of suiri_tune, 0..4; -1: cluster-resident where the lane's tanks fit, else one launch per
     sweep) */
  int32_t sor_mode;
  /* polls of a bounded device wait (the cooperative solve's grid barrier) before it gives up, records error
     bit 1 in the tank's stats and returns (default 2^22; a batch or lane takes its tanks' smallest) */
  int64_t watchdog_polls;
} suiri_params;

typedef struct suiri_stats {
  int64_t count;           /* liquid particles */
  int64_t ww_count;        /* whitewater particles */
  int64_t impacts;         /* sub-grid drops merged so far */
  double vmax;             /* max speed of in-grid particles in the last sub-step */
  double time;             /* simulated time [s] */
  double liters;           /* count · (h/2)³ · 1000 (src/js/50-sim.js:375) */
  int32_t full;            /* capacity was reached */
  int32_t frame;           /* sub-steps taken */
  int32_t errors;          /* device error bits: 1 = a grid-barrier wait of the persistent solve gave up */
  int32_t pad;
  int32_t nx, ny, nz;
  double h;
  double origin[3];
  int64_t active_cells;    /* liquid cells with an open face, relaxed by the last solve (both colours) */
  /* FP64 residual of the last pressure solve, r = Σ C·p_nb − h²·div − (Σ C)·p over the active cells, in
     float64 from the float32 operands (the check solver.py:473-509's operands allow); 0 unless switched on
     with suiri_residual / suiri_batch_residual */
  double residual_max;     /* max |r| */
  double residual_rms;     /* sqrt(Σ r² / active_cells) */
  double rhs_max;          /* max |h²·div| over the same cells (the scale of r) */
  int32_t ripple_rx, ripple_rz;   /* ripple layer vertices - 1 per side (0: none) */
  int32_t wmap;            /* top-view height map texels per side */
  int32_t pad2;
} suiri_stats;

/* An obstacle or drain in binary form (instead of scene JSON items). */
typedef struct suiri_object {
  int32_t type;            /* 0 round box, 1 sphere, 2 cylinder, 3 cone, 4 torus, 5 cup, 6 container,
                              7 gutter; 9 drain cylinder */
  int32_t flag;            /* 1 obstacle, 2 drain */
  double pos[3];
  double rot[9];           /* world-from-local rotation, row major */
  double dims[4];          /* shape parameters as src/js/10-scene.js:143-157 packs them */
  double lin[3], ang[3];   /* solid velocity: linear and angular */
} suiri_object;

/* grid fields for suiri_read_grid (parity dumps; arrays x fastest) */
enum suiri_field {
  SUIRI_FIELD_CELL_COUNT = 0,  /* int32 [nz][ny][nx]: particles per cell */
  SUIRI_FIELD_FRAC = 1,        /* float32 [3][nz+1][ny+1][nx+1]: face open fractions */
  SUIRI_FIELD_VEL = 2,         /* float32 [3][nz+1][ny+1][nx+1]: face velocity (after projection) */
  SUIRI_FIELD_VELOLD = 3,      /* float32 [3][nz+1][ny+1][nx+1]: P2G face velocity */
  SUIRI_FIELD_MASK = 4,        /* uint8  [3][nz+1][ny+1][nx+1]: face took particle weight */
  SUIRI_FIELD_PRES = 5,        /* float32 [nz][ny][nx]: pressure */
  SUIRI_FIELD_RHS = 6,         /* float32 [nz][ny][nx]: h²·divergence (SOR right-hand side) */
  SUIRI_FIELD_RIPPLE_SRC = 7,  /* float64 [rz+1][rx+1]: pending ripple impulses [N·s] */
  SUIRI_FIELD_RIPPLE = 8,      /* float32 [rz+1][rx+1][3]: ripple height, slope x, slope z */
  SUIRI_FIELD_TOP = 9,         /* float32 [wmap][wmap]: top-view water height, -1 dry */
  SUIRI_FIELD_RIPPLE_STATE = 10, /* float32 [2rz][2rx][2]: spectral state (height + i·velocity) */
  SUIRI_FIELD_RIPPLE_MASK = 11, /* float32 [rz+1][rx+1]: absorption mask of the last frame */
  SUIRI_FIELD_TOP64 = 12       /* float64 [wmap][wmap]: top-view water height as computed, -1 dry */
};

/* ---------------------------------------------------------------- one tank (the plain drop-in path) */

int suiri_params_default(suiri_params* p);

/* FluidSim constructor + setObjects + emitNow(blockEmits) (src/js/50-sim.js:29-89, src/js/90-main.js:5-13).
   scene_json may be NULL: an empty tank with the explicit grid of `params`. */
int suiri_create(const char* scene_json, const suiri_params* params, suiri_tank** out);
int suiri_destroy(suiri_tank* t);
const char* suiri_last_error(const suiri_tank* t);

/* restartWater (src/js/90-main.js:15-19): clear, then refill the scene's water blocks */
int suiri_reset(suiri_tank* t);
/* clearWater (src/js/50-sim.js:365-373) */
int suiri_clear(suiri_tank* t);

/* setObjects (src/js/50-sim.js:165-211): obstacles and drains from scene items JSON ([…] or {items:[…]});
   velocities from the previous transforms over dt_move; *moving = 1 if any moves (may be NULL) */
int suiri_set_objects(suiri_tank* t, const char* items_json, double dt_move, int32_t* moving);
/* the same from binary records */
int suiri_set_obstacles(suiri_tank* t, const suiri_object* objs, int32_t n);
/* Solids lattice of the Blender host (solver.py:47-56, bake.py:83-181): distances at the half-cell points
   origin + h/2·(i,j,k), (2nx+1)(2nyl+1)(2nz+1), i fastest; oid (may be NULL) = obstacle index per point.
   Switches the tank to lattice mode for face fractions and collisions. */
int suiri_set_lattice(suiri_tank* t, const double* sdf, const int32_t* oid, int32_t lx, int32_t ly, int32_t lz);

/* distance to the nearest obstacle at n points (host arrays, n×3 → n), as the step sees it: analytic
   shapes or the lattice (sceneSdf, src/js/30-wgsl-sim.js:78-87; sdf_at, solver.py:116-140; the editor's
   mirror for picking and placement, src/js/10-scene.js:124-176). 1e9 where there is no obstacle. */
int suiri_eval_sdf(suiri_tank* t, const double* pts, int64_t n, double* out);
/* The same distances without allocating anything on the device. No counterpart in the reference: it is
   for callers that cannot allocate device memory when they ask — a host whose device memory is fully
   committed (a server that has admitted scenes up to its whole HBM budget, where a per-call allocation
   could fail or take memory promised to resident scenes), or an interactive loop that queries distances
   every frame (picking, placement) and must keep the allocator off that path. suiri_eval_sdf stages the
   points and distances in memory it allocates per call; this one stages them in one fixed array inside
   the library, at most 65536 points per call (more: SUIRI_ERR_INVALID). The array (2 MiB) exists on every
   GPU that loads the library, until the process exits. The first call on a device looks up the array's
   address there; make that first call before any stream capture. Like every call on a tank, it leaves the
   tank's device current for the calling thread. All calls share the one array: calls that overlap on the
   GPU (two threads, two tanks on different streams) race on it, so serialise them. Every call writes all
   the staging it reads, so nothing is left over from the previous call. */
int suiri_eval_sdf_static(suiri_tank* t, const double* pts, int64_t n, double* out);
/* validScene (src/js/80-ui.js:430-459) without creating a tank (needs no GPU): the scene as the library reads
   it, as JSON {"tank":{w,h,d},"items":[…]}, the tank clamped to the editor's limits when clamp_tank is 1,
   items of an unknown kind dropped, every field missing or unusable taken from a fresh item of the same kind
   (src/js/10-scene.js:56-86; an unknown shape is a box, an unknown material or source mode the fresh item's),
   ids kept when positive, integral and not seen before, the others numbered on from the largest.
   *len = the text's length without its terminating NUL; it is written to out (NUL-terminated) when cap is
   larger than that, else nothing is written and SUIRI_ERR_INVALID returned (out may be NULL to query the
   length). SUIRI_ERR_PARSE for malformed JSON or a tank without positive w, h, d. */
int suiri_scene_validate(const char* scene_json, int32_t clamp_tank, char* out, size_t cap, size_t* len);
/* device bytes a tank of these parameters and scene would take (admission planning) */
int suiri_estimate_bytes(const char* scene_json, const suiri_params* params, double* bytes);

/* particles from host arrays, appended before the next sub-step (emit_block/_add, solver.py:304-343).
   pos, vel: n×3 float32 (vel NULL: at rest); airborne: n floats (0/1) or NULL. The arrays cross to the
   device packed as given (12 B a particle for positions alone), and a kernel lays them out: arrays in
   page-locked memory are read by the copy engine directly when nothing is queued on the tank's stream (the
   call returns once they have been read), others are copied into pinned staging first. Either way the
   caller may reuse the arrays on return. *first_id (may be NULL) = id of the first. */
int suiri_add_particles(suiri_tank* t, const float* pos, const float* vel, const float* airborne, int64_t n,
                        uint32_t* first_id);
/* Fixed-rate emitters run on the device inside every sub-step (also inside a captured CUDA graph): shape 0
   a disc outlet of `radius` at pos pointing along dir at `speed` (the stream source, src/js/31-wgsl-sim2.js:
   276-288), shape 3 a square rain area of half side `radius` falling at `speed` (:307-310). per_substep
   particles each sub-step, fractions carried over. At most 8; n = 0 removes them. */
typedef struct suiri_emitter {
  int32_t shape;
  int32_t airborne;        /* 1: emitted particles carry the free-flight mark (sub-grid drops) */
  double pos[3];
  double dir[3];
  double radius;           /* disc radius; rain: half extent along x */
  double speed;
  double per_substep;
  double radius_z;         /* rain: half extent along z (0: same as radius) */
} suiri_emitter;
int suiri_set_emitters(suiri_tank* t, const suiri_emitter* e, int32_t n);

/* a water block as a jittered half-cell lattice clipped to the tank (src/js/55-emit.js:83-106, solver.py:317-343);
   fill = 1 skips cells already at least half full */
int suiri_emit_block(suiri_tank* t, const double lo[3], const double hi[3], int32_t fill);

/* one sub-step of fixed length dt (FluidSim.encodeSubstep, src/js/50-sim.js:276-297; solver.py:438-525) */
int suiri_substep(suiri_tank* t, double dt);
/* one frame: CFL sub-steps, scene sources, whitewater, top height and ripples
   (FluidSim.step src/js/50-sim.js:300-336; Solver.step solver.py:716-728). *substeps may be NULL. */
int suiri_step(suiri_tank* t, double frame_dt, int32_t* substeps);
/* the end of a frame after sub-steps the caller took with suiri_substep: cell counts, whitewater advance over
   frame_dt, top height and ripples (Solver.step solver.py:720-728, the part after the sub-step loop) */
int suiri_frame_end(suiri_tank* t, double frame_dt);
int suiri_sync(suiri_tank* t);

/* page-locked host memory for the arrays of suiri_add_particles and suiri_read_particles, so that a host
   without CUDA headers (a Node addon) gets the direct copies: at least `bytes`, from the library's cache of
   pinned blocks (handing pinned memory back to the driver synchronises the device, so freed blocks are kept
   for reuse, up to 2 GB); suiri_host_free takes back a block suiri_host_alloc gave */
int suiri_host_alloc(size_t bytes, void** out);
int suiri_host_free(void* p);

/* liquid particles (alive) to host memory: pos4 = (x, y, z, airborne), vel4 = (vx, vy, vz, id as uint32 bits);
   either pointer may be NULL; *n = number available (written even when cap is too small). Arrays in
   page-locked memory (suiri_host_alloc, cudaHostRegister, cudaMallocHost) are written by the copy engine
   directly; others through the tank's pinned buffers. */
int suiri_read_particles(suiri_tank* t, float* pos4, float* vel4, int64_t cap, int64_t* n);
/* whitewater: pos4 = (x, y, z, life), vel4 = (vx, vy, vz, kind) */
int suiri_read_whitewater(suiri_tank* t, float* pos4, float* vel4, int64_t cap, int64_t* n);
/* whitewater particles appended from host memory, in the layout suiri_read_whitewater gives (life in pos4.w,
   kind in vel4.w: 0 spray, 1 foam, 2 bubble), e.g. a state saved by a host (the Blender add-on keeps its
   wpos/wvel/wlife/wkind arrays, solver.py:86-89). SUIRI_ERR_CAPACITY if they do not all fit (those that fit
   are kept). */
int suiri_add_whitewater(suiri_tank* t, const float* pos4, const float* vel4, int64_t n);
/* a grid field (enum suiri_field) into out (bytes long) */
int suiri_read_grid(suiri_tank* t, int32_t field, void* out, size_t bytes);

/* The per-frame maps over the footprint that the bake exports (blender_addon/suiri_lab/bake.py:241-249), from
   the last frame's top-view height map and ripple field: float32 [wmap][wmap][4] = top height (-1 dry), ripple
   slope d/dx and d/dz at the texel centre (solver.py:909-919), and the floor light relative to plain sunlight,
   the sun (towards it, any length) refracted through the surface (Solver.caustics, solver.py:796-846).
   bytes >= wmap²·16; out NULL builds the maps on the device only (they are kept until the next call).
   SUIRI_ERR_INVALID for a zero or non-finite sun direction; -6 without a ripple layer. */
int suiri_frame_maps(suiri_tank* t, const double sun_dir[3], float* out, size_t bytes);

/* The liquid's surface mesh for the frame export (meshing.surface + settle_on_top + the vertex velocity,
   blender_addon/suiri_lab/meshing.py:52-199, bake.py:228-235), built on the device from the particles as they
   are: the body's distance field on a lattice of spacing h/2, blurred (Gaussian of sigma `smooth` lattice
   nodes, the reference's default 0.8), meshed with surface nets (quads, outward); lone particles (at most 6
   particles in the 3×3×3 cells around theirs) as 42-vertex icospheres (80 triangles each, after the body's
   vertices, in particle order as suiri_read_particles returns them); vertices within 0.6h of the wet top-view
   height map of the last frame settled onto it (none before the first frame or without a ripple layer); the
   liquid's face velocity at every vertex. suiri_surface_mesh builds it and fills `info`; suiri_surface_mesh_read
   copies it out: verts and vel float32 [verts][3], quads int32 [quads][4], tris int32 [tris][3]; any output may
   be NULL; each array must hold the counts `info` gave (max_* are their capacities). */
typedef struct suiri_mesh_info {
  int64_t verts, quads, tris;
  int64_t body_verts, lone;        /* surface-nets vertices; lone particles (42 vertices each) */
  int32_t lattice[3];              /* distance-field lattice nodes per axis (0 without a body) */
  int32_t taps;                    /* blur taps used, weights[0 .. taps) (normalised) */
  double lo[3], spacing, smooth;   /* lattice origin [m], spacing h/2 [m], blur sigma [nodes] */
  double weights[33];
  double phase_ms[5];              /* device time of the build: classify, distance field, blur, surface nets, finish */
} suiri_mesh_info;

int suiri_surface_mesh(suiri_tank* t, double smooth, suiri_mesh_info* info);
int suiri_surface_mesh_read(suiri_tank* t, float* verts, float* vel, int32_t* quads, int32_t* tris, int64_t max_verts,
                            int64_t max_quads, int64_t max_tris);
int suiri_get_stats(suiri_tank* t, suiri_stats* s);
/* Non-blocking stats, as the reference's FluidSim.pollStats (src/js/50-sim.js:346-363) maps its staging
   buffers asynchronously. One read of the device counters is in flight at a time. If it has finished, *s
   gets those stats and *fresh = 1 (else *s is left as it is and *fresh = 0); when no read is in flight any
   more, a new one is enqueued on the tank's stream behind the work enqueued so far. The stats returned
   therefore date from the call that started their read. fresh may be NULL. */
int suiri_poll_stats(suiri_tank* t, suiri_stats* s, int32_t* fresh);
/* bytes one stats read (suiri_get_stats, suiri_poll_stats) copies from the device */
size_t suiri_stats_readback_bytes(void);

/* saveWater / restoreWater (src/js/50-sim.js:111-141): one copy slot per tank, on the device */
int suiri_snapshot(suiri_tank* t, int32_t* id);
int suiri_restore(suiri_tank* t, int32_t id);

/* interop: the tank's cudaStream_t (as void*) and device ordinal */
int suiri_stream(suiri_tank* t, void** stream);
/* 1: capture the sub-step as a CUDA graph and replay it (default 1) */
int suiri_use_graphs(suiri_tank* t, int32_t on);

/* ---------------------------------------------------------------- batching: many tanks, one set of launches */

/* a batch steps existing tanks (same device) together: every kernel of the sub-step covers all the tanks of
   a size lane (under 2^16 cells, under 2^19, larger) in one launch, through per-tank descriptor and
   block-offset tables, and each lane's sub-step is one CUDA graph on the lane's own stream. A sub-step forks
   from the batch's stream (suiri_batch_stream) to the lanes and joins back to it, so the lanes' kernels
   overlap and small tanks do not wait for the largest one's kernels. */
int suiri_batch_create(suiri_tank* const* tanks, int32_t n, suiri_batch** out);
/* as suiri_batch_create with the lanes given: lane_of[i] in 0..7 is tank i's lane (each occupied lane is a
   group with its own stream and graph; NULL: the size lanes, under 2^16 cells, under 2^19, larger) */
int suiri_batch_create_lanes(suiri_tank* const* tanks, int32_t n, const int32_t* lane_of, suiri_batch** out);
int suiri_batch_destroy(suiri_batch* b);
int suiri_batch_substep(suiri_batch* b, double dt);
int suiri_batch_sync(suiri_batch* b);
/* tuning knobs picked by the autotuner: blocks per SM of the persistent particle kernels, and the form of
   the pressure solve, sor_mode: 0 one launch per colour sweep; 1 the whole solve in one cooperative launch
   with a grid barrier between sweeps; 2 two colour sweeps per launch over per-tile lists of active cells
   (allocates those lists for the tank or batch, once); 3 four sweeps per launch on shared-memory tiles with
   halos; 4 the whole solve in one launch with each tank held in the shared memory of one thread-block
   cluster (distributed shared memory between its CTAs, the hardware cluster barrier between sweeps); it
   fails with SUIRI_ERR_INVALID when a tank needs more than 16 CTAs of shared memory (then keep another
   form). The tile of mode 4 is the shared memory a CTA takes, set by suiri_tune_piece. All five forms give
   the same pressures bit for bit. */
int suiri_batch_tune(suiri_batch* b, int32_t particle_blocks_per_sm, int32_t sor_mode);
int suiri_tune(suiri_tank* t, int32_t particle_blocks_per_sm, int32_t sor_mode);
/* tile knob of the cluster-resident solve: at most piece_kb KiB of shared memory per CTA (0: the device's
   maximum), i.e. fewer z planes per CTA and more CTAs per tank; applies now if tuned to sor_mode 4, else at
   the next suiri_tune with it */
int suiri_tune_piece(suiri_tank* t, int32_t piece_kb);
int suiri_batch_tune_piece(suiri_batch* b, int32_t piece_kb);
/* form of the grid-to-particle pass: 0 a grid-stride walk over the sorted particles (corner loads from the
   node arrays), 1 one block per 8×8×8-cell brick with the brick's face nodes copied to shared memory first.
   Both give the same particles bit for bit. */
/* form of the grid-to-particle pass: 0 a grid-stride walk over the sorted particles; 1 one block per 8³ brick with
   its faces staged in shared memory; 2 the walk's common path (fewer registers, more warps) with the particles
   that need a rare branch (RK2, an obstacle within reach, a sparse cell's free-flight test, a falling drop, a
   whitewater spawn) deferred to a second pass that runs the full update for them. All give the same particles. */
int suiri_tune_g2p(suiri_tank* t, int32_t form);
int suiri_batch_tune_g2p(suiri_batch* b, int32_t form);
/* all knobs of one size lane of a batch (lane in [0, suiri_batch_lanes)): the lanes run concurrently and may
   each prefer another form (small tanks the cluster-resident solve, large ones one launch per sweep) */
int suiri_batch_tune_lane(suiri_batch* b, int32_t lane, int32_t particle_blocks_per_sm, int32_t sor_mode,
                          int32_t piece_kb, int32_t g2p_form);
/* 1: after every pressure solve, evaluate its FP64 residual on the device (two extra launches); read it
   with suiri_get_stats (residual_max, residual_rms, rhs_max) */
int suiri_residual(suiri_tank* t, int32_t on);
int suiri_batch_residual(suiri_batch* b, int32_t on);
int suiri_batch_stream(suiri_batch* b, void** stream);

/* ---------------------------------------------------------------- serving: continuous batching under an HBM budget */

/* A scene solve: grid and physics as in suiri_create, the scene JSON (tank, obstacles, drains, water
   blocks), fixed-rate emitters, and the number of sub-steps. No reference counterpart: the reference runs
   one scene per page (src/js/90-main.js) or per Blender bake (bake.py). */
typedef struct suiri_request {
  uint32_t size;                    /* sizeof(suiri_request) */
  const suiri_params* params;       /* may be NULL: defaults */
  const char* scene_json;
  const suiri_emitter* emitters;
  int32_t n_emitters;
  int32_t steps;
  int32_t keep_result;              /* 1: keep the final particles for suiri_server_result */
} suiri_request;

typedef struct suiri_server_stats {
  int64_t completed, queued, running, failed, rebuilds;
  int64_t substeps;                 /* batched sub-steps issued, summed over the size lanes */
  double particle_steps;            /* work done so far: per batched sub-step, the liquid particles (counted at
                                       admission) of every scene it advanced */
  double elapsed_s, used_bytes, budget_bytes;
  double p50_ms, p99_ms;            /* request latency: submit → results ready */
  double mean_active;               /* resident scenes (all lanes) per round in which some lane advanced */
} suiri_server_stats;

/* a worker thread admits requests FIFO while their device memory fits the budget, and retires finished ones at
   sub-step boundaries. Resident scenes are batched in three lanes by size (under 2^16 cells, under 2^19,
   larger), each with its own stream: a lane advances its scenes one batched sub-step of length dt at a time,
   keeping up to 4 sub-steps queued on the device, so small scenes do not wait for large ones */
int suiri_server_create(int32_t device, double budget_bytes, double dt, suiri_server** out);
int suiri_server_destroy(suiri_server* s);
int suiri_server_submit(suiri_server* s, const suiri_request* r, int64_t* id);
/* state: 0 queued, 1 running, 2 done, 3 failed; latency_ms: submit → done/failed, or the time waited so far
   for a request still queued or running; count = final liquid particles */
int suiri_server_poll(suiri_server* s, int64_t id, int32_t* state, double* latency_ms, int64_t* count);
/* block until the request is done or failed, at most timeout_s seconds (SUIRI_ERR_STATE on timeout) */
int suiri_server_wait(suiri_server* s, int64_t id, double timeout_s);
/* final particles of a finished request submitted with keep_result (as suiri_read_particles) */
int suiri_server_result(suiri_server* s, int64_t id, float* pos4, float* vel4, int64_t cap, int64_t* n);
int suiri_server_get_stats(suiri_server* s, suiri_server_stats* st);

/* ---------------------------------------------------------------- timing helpers (device events) */

/* milliseconds of device time of `steps` sub-steps of dt, events on the tank's / batch's own stream */
int suiri_time_substeps(suiri_tank* t, double dt, int32_t steps, double* ms);
int suiri_batch_time_substeps(suiri_batch* b, double dt, int32_t steps, double* ms);
/* milliseconds per launch of the SOR sweeps alone, timed over `iters` iterations on the current state
   (this relaxes the current pressure further) */
int suiri_time_sor(suiri_tank* t, int32_t iters, double* ms);
/* 1: record device events around the pressure solve of every sub-step (inside the captured graph);
   suiri_sor_phase_ms then gives the last sub-step's pressure-solve time (waits for it) */
int suiri_profile(suiri_tank* t, int32_t on);
int suiri_sor_phase_ms(suiri_tank* t, double* ms);
int suiri_batch_profile(suiri_batch* b, int32_t on);
/* the longest of the lanes' pressure-solve times (the lanes run concurrently) */
int suiri_batch_sor_phase_ms(suiri_batch* b, double* ms);
/* with profiling on, the device time of each phase of the last sub-step, ms[6]: binning and sort, P2G, node and
   cell passes, pressure solve, projection (with the residual when on), G2P */
#define SUIRI_PHASES 6
int suiri_phase_ms(suiri_tank* t, double* ms);
/* the same for one size lane of a batch (lane in [0, suiri_batch_lanes)); occupied lanes in order of size
   (under 2^16 cells, under 2^19, larger) */
int suiri_batch_lanes(suiri_batch* b, int32_t* n);
int suiri_batch_phase_ms(suiri_batch* b, int32_t lane, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* SUIRI_H */
