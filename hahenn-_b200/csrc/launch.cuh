// Host-side launch context shared by the kernel files: which tanks a launch covers and how its blocks
// map onto them.
#pragma once
#include "common.cuh"

namespace suiri {

constexpr int kThreads = 256;
constexpr int kScanTile = 2048;          // cells per scan block (256 threads × 8)
constexpr int kBrick = 8;                // P2G brick edge in cells
constexpr int kTbX = 16, kTbY = 16, kTbZ = 8;   // temporal-blocked SOR tile (cells)
constexpr int kTbThreads = 512;

// block families: blocks of one launch are laid out tank after tank; pfx[t] = first block of tank t
constexpr int kSorThreads = 256;        // block size of a per-sweep SOR launch (128, 512, 1024 measured slower)
enum Family { kFamNodes = 0, kFamCells, kFamHalf, kFamBricks, kFamScan, kFamTiles, kFamSor, kFamG2P, kFamCount };

struct LaunchCtx {
  cudaStream_t stream;
  const TankDev* tanks;     // device array of ntanks descriptors
  int ntanks;
  const int* bpfx[kFamCount];   // device: ntanks+1 block prefixes per family
  int nblocks[kFamCount];       // host copy of the totals
  int* ppfx_in;             // device: ntanks+1 prefix of particles in A∪E
  int* ppfx_sorted;         // device: ntanks+1 prefix of particles in B
  long long* scan_bsum;     // device: one partial sum per scan block
  int particle_blocks;      // persistent grid for particle kernels
  int* hpfx;                // device: ntanks+1 prefix of colour slots (nhalf) for the persistent SOR
  int* apfx;                // device: 2·(ntanks+1), per colour the prefix of the active cells (this sub-step)
  GridBarrier* barrier;     // device: grid barrier of the persistent SOR
  unsigned* ticket;         // device: last-block tickets (0 cell pass, 1 scatter, 2 sub-step start)
  uint2* tbl_list;          // device, two sweeps per launch: per tile the active-cell lists (k_tbl_lists)
  int* tbl_cnt;             //   per tile: entries of list A, B, C
  int2* tbl_c;              //   per tile: colour-0 cells with a constant pressure other than +0
  int* defer_list;          // device, G2P form 2: sorted indices of the particles deferred to the full body
  int* defer_n;             //   and their count
};

// One CTA of the cluster-resident solve: planes [k0, k0+nk) of tank `tank` (index into the launch's
// descriptors; -1: an idle CTA that only takes part in its cluster's barriers). np = planes per piece of
// that tank, the same for all its pieces (the last may hold fewer); a tank's pieces sit on consecutive
// cluster ranks, first plane first.
struct ClusterPiece {
  int tank, k0, nk, np;
};

// Blocks of kThreads threads of kernel k that fit on the current GPU at once (cached per device in cache[]).
// The grid-stride particle kernels are launched with this many blocks: all resident, one wave.
inline int resident_grid(const void* k, int* cache) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 128) return 1;
  if (!cache[dev]) {
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = per_sm * sms > 0 ? per_sm * sms : 1;
  }
  return cache[dev];
}

// per-kernel launchers (bin.cu, grid.cu, sor.cu, g2p.cu)
void launch_begin_count(const LaunchCtx& L);   // prefix only, for a count pass between sub-steps
void launch_bin(const LaunchCtx& L);
void launch_bin_count(const LaunchCtx& L);     // cell counts only, for a count pass
void launch_scan(const LaunchCtx& L);
void launch_scatter(const LaunchCtx& L);
void launch_geom(const LaunchCtx& L);
void launch_p2g(const LaunchCtx& L);
void launch_grid_nodes(const LaunchCtx& L);
void launch_grid_cells(const LaunchCtx& L);
void launch_sor_sweep(const LaunchCtx& L, int color, int sweep);
// whole solve, one cooperative launch; a barrier wait gives up after `limit` polls (error bit in the counters)
// smem_cap > 0: at most that much shared memory per block for its resident entries (tile knob)
void launch_sor_persist(const LaunchCtx& L, int max_iters, int blocks, unsigned limit, int smem_cap = 0);
constexpr unsigned kWatchdogPolls = 1u << 22;                            // default poll limit of a bounded wait
int sor_persist_max_blocks(int device);                                  // co-resident blocks of k_sor_persist
cudaError_t sor_tb_prepare();                                            // once per device, outside capture
void launch_sor_tb(const LaunchCtx& L, int sweeps_per_launch, int sweep0, int nsweeps, int dir);  // 2 or 4; dir 0: pres→pres2
void launch_sor_copy(const LaunchCtx& L);                                // pres ← pres2
void launch_tbl_lists(const LaunchCtx& L);                               // per sub-step, before a 2-sweep solve
size_t tbl_list_bytes(int tiles);                                        // device bytes of those lists
void tbl_assign(LaunchCtx& L, void* base, int tiles);                    // point the context into them
// cluster-resident solve (one launch per solve; each tank's field held in one cluster's shared memory)
constexpr int kClusterMax = 16;                                          // CTAs per cluster (non-portable above 8)
int cluster_smem_bytes(const TankDev& D, int np);                        // shared bytes of a piece of np planes
cudaError_t sor_cluster_prepare(int smem_bytes, int cluster);            // once per device, outside capture
int sor_cluster_max_active(int smem_bytes, int cluster);                 // co-resident clusters (0: cannot launch)
void launch_sor_cluster(const LaunchCtx& L, const ClusterPiece* pieces, int nblocks, int smem_bytes, int cluster,
                        int max_iters);
// FP64 residual of the solve just finished, max |r| and Σ r² over the active cells into the tank counters
void launch_sor_residual(const LaunchCtx& L);
void launch_project(const LaunchCtx& L);
// form 0: grid-stride walk over the sorted particles; 1: one block per brick with its faces in shared memory
void launch_g2p(const LaunchCtx& L, int form);
void launch_whitewater(const LaunchCtx& L, double frame_dt);

}  // namespace suiri
