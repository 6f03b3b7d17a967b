// Data structures and kernel declarations of the batched cell-centred MGPCG.
#pragma once

#include "gd_internal.cuh"

namespace gd {

// Hierarchy rules.  A level is coarsened (ceil(ny/2) x ceil(nx/2)) while it has
// more than kCoarsestCells cells; the first level with at most kBottomCells
// cells (a plan may choose another limit) whose levels down to the coarsest
// fit in kBottomSmem bytes of shared memory (padded b, u and classes) is
// handled, with everything below it, by one CTA per instance; the coarsest
// level is solved with a dense FP64 inverse.
constexpr int kCoarsestCells = 64;
constexpr int kBottomCells = 4096;
constexpr int kBottomSmem = 220 * 1024;
constexpr int kBottomLevels = 24;  // most levels one bottom holds
// Coarse levels (below level 0, above the bottom) with at most kTileCells
// cells run on the shared-memory tile kernels; larger ones on the strips.
constexpr int kTileCells = 1 << 18;

// Fine-level (level 0) kernels: 64 rows x 128 columns per CTA of 128 threads
// (four warps, each 16 rows x 128 columns).  Down / up kernels use the same
// CTA shape with a per-level strip height.
constexpr int kFTY = 64, kFTX = 128, kFThreads = 128;
constexpr int kVThreads = 128;     // down / up kernels
constexpr int kBThreads = 1024;    // bottom kernel
constexpr int kLastWarps = kFThreads / 32;

enum : int { BC_DIR = 0, BC_NEU = 1, BC_MASK = 2 };
// FLAG_RU: an FP64 refresh is due (set by cgupdate, cleared by the residual).
// FLAG_DZERO: the correction d restarts from zero (set when a solve starts and
// at every refresh, cleared by the next cgupdate, which then writes d = alpha p
// without reading the stale d, so nobody has to write zeros into it).
enum : int { FLAG_RU = 1, FLAG_DZERO = 2 };
// Slot of the plan's counter array that holds the device error word: bits set
// by a kernel whose bounded wait gave up, cleared when a solve starts.
constexpr int kErrWord = 15;

// Programmatic dependent launch.  The kernels of a solve may be launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, which lets their CTAs be
// scheduled before the kernel ahead of them in the stream has finished.  Such a
// kernel reads only the plan's tables that no kernel writes (the tile lists and
// the level descriptors) before dep_wait(), which returns once the kernel
// ahead has completed and its writes are visible; then dep_release() lets the
// next kernel's CTAs be scheduled in turn.  Without the attribute both are
// no-ops.
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void dep_release() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void dep_enter() {
  dep_wait();
  dep_release();
}

struct LevelInfo {
  int ny, nx, pitch, inst;
  int bc, level, coarse, is_bottom;
  float wall, pad0;
  int rows_per_warp;  // strip height of the down / up kernels on this level (even)
  // bottom levels: byte offsets of the padded b, u, residual and class arrays
  // in the bottom kernel's shared memory, their row pitch (nx + 3), the FP64
  // right-hand side of the dense solve (coarsest level; the dense inverse
  // follows it at sm_d + kCoarsestCells doubles) and the end of the layout
  int sm_r;
  int sm_b, sm_u, sm_c, sm_px, sm_d, sm_end;
  long long b_off, u_off;  // element offsets into the T arena
  long long w_off;         // pre-smoothed iterate written by down, read by up
  long long code_off;      // byte offset into the code arena, -1 if rectangle
  long long inv_off;       // coarsest level: element offset of its dense inverse, else -1
};

struct InstInfo {
  int ny, nx, pitch, bc;
  int level0, bottom, coarsest, nlevels;
  long long r_off, p_off, d_off, z_off, q_off;  // p is double-buffered: p_off / q_off
  long long xs_off;  // the plan's own FP64 copy of the solution (element offset, row pitch `pitch`)
  int fine_begin, fine_end;  // tile range in the fine map
  int up0_begin, up0_end;    // range of its r.z group partials (empty if bottom is level 0)
  int zero_mean;
  int rz_rows;  // rows per r.z group partial: level 0's strip height for the instance alone
  // set per solve
  const double *f;
  double *x;
  long long upitch;
  double scale;
  double cells_active;
};

struct InstState {
  double rz, beta, pAp, alpha, rr, rr_ref, ff, rr_true, mean, fmean, rr_prev;
  int status, iters, flags, first;
  int pcur;  // which of the two p buffers holds the current direction
  int xcur;  // where the current solution is: 0 the caller's x, 1 the plan's copy
  int refreshes;  // FP64 refreshes after the initial residual
  int xzero;      // the solution is known to be zero (zero-start solve, nothing folded yet)
  int mean_known; // mean holds the solution's mean (set by a refresh that folds)
  int pad;
};

struct Tile {
  int level;  // LevelInfo index (fine level for down/up, level 0 for fine maps)
  int inst;
  int ty, tx;
};

template <typename T>
struct Args {
  const LevelInfo *lv;
  const InstInfo *inst;
  InstState *st;
  T *arena;
  double *xs;  // the plan's FP64 solution copies
  const unsigned char *codes;
  const double *dense;
  double *part0;
  double *part1;
  unsigned *counter;
  int *n_active;
  const Tile *tiles;
  int ninst;
  double tol2, delta2;
  int max_iter;
  int zero_start;  // solves start from x = 0 without reading the caller's x
};

// Cell class: 0 = no unknown, else 1 + number of walls (missing neighbours).
__host__ __device__ __forceinline__ int rect_class(int y, int x, int ny, int nx) {
  return 1 + (y == 0) + (y == ny - 1) + (x == 0) + (x == nx - 1);
}

__device__ __forceinline__ int cell_class(const LevelInfo &L, const unsigned char *codes, int y,
                                          int x) {
  if (y < 0 || y >= L.ny || x < 0 || x >= L.nx) return 0;
  if (L.code_off >= 0) return codes[L.code_off + (long long)y * L.pitch + x];
  return rect_class(y, x, L.ny, L.nx);
}

// Diagonal of the positive operator for a cell of class c on a level with wall
// coefficient w: interior neighbours count 1, walls count w (Neumann w = 0,
// Dirichlet w = 1 on the finest level and 2 on coarse levels).
__host__ __device__ __forceinline__ double class_diag(int c, float w) {
  return 4.0 - (double)(c - 1) * (1.0 - (double)w);
}

}  // namespace gd
