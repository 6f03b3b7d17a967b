// Kernels of the batched cell-centred MGPCG.  Included by gd_mg.cu only.
//
// Operator: A u = d_p u_p - sum of neighbour values, neighbours outside the
// grid or without an unknown contribute zero; d_p = 4 - walls * (1 - w) with
// w the level's wall coefficient.  On the finest level this is exactly
// -h^2 laplacian (Dirichlet, operators.py:86-107), -divergence(gradient(.))
// (Neumann, test_operators.py:51-57) or the masked Perez matrix negated
// (poisson.py:190-204).
//
// V-cycle (the B200 replacement of multigrid.py:184-215): cell-centred
// coarsening to ceil(n/2), bilinear prolongation P (weights 3/4, 1/4 per axis,
// Neumann ghosts mirror, Dirichlet ghosts zero), restriction R = P^T,
// red-black Gauss-Seidel with colour 0 then 1 before restriction and colour 1
// then 0 after prolongation, so the cycle is a symmetric operator.  Each level
// costs two passes over HBM (the register-streaming kernels of gd_stream.cuh):
// `down` smooths from zero, forms the residual and restricts it; `up`
// recomputes that pre-smoothed iterate from b instead of storing it, adds P e
// and post-smooths.  Small levels run in `k_bottom` (this file), one CTA per
// instance, down to a dense FP64 solve.
#pragma once

#include <cuda_pipeline.h>

#include "gd_mg.cuh"

namespace gd {

__device__ __forceinline__ bool in_grid(const LevelInfo &L, int y, int x) {
  return y >= 0 && y < L.ny && x >= 0 && x < L.nx;
}

// Last-CTA handshake: every CTA calls it once; returns true in the last one.
__device__ __forceinline__ bool last_block(unsigned *counter) {
  __shared__ bool am_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(counter, 1u);
    am_last = (prev == gridDim.x - 1);
    if (am_last) *counter = 0u;
  }
  __syncthreads();
  if (am_last) __threadfence();
  return am_last;
}

// Deterministic per-instance sum of partials [b, e) by one warp (L2 reads).
__device__ __forceinline__ double warp_range_sum(const double *p, int b, int e) {
  double s = 0.0;
#pragma unroll 8
  for (int k = b + (threadIdx.x & 31); k < e; k += 32) s += __ldcg(p + k);
  return warp_sum(s);
}

// The search direction lives in two buffers: k_pupdate reads the current one
// (including halo cells owned by other CTAs) and writes the other, so no CTA
// overwrites a value another CTA still has to read.
__device__ __forceinline__ long long p_offset(const InstInfo &I, int which) {
  return which ? I.q_off : I.p_off;
}

__device__ __forceinline__ void finish_rz(InstState &S, double rz) {
  if (!(rz > 0.0) || !isfinite(rz)) {
    S.status = GD_BREAKDOWN;
    S.flags |= FLAG_RU;
    return;
  }
  S.beta = S.first ? 0.0 : rz / S.rz;
  S.first = 0;
  S.rz = rz;
}

template <typename T>
__device__ __forceinline__ void make_tables(T *diag, T *dinv, float wall) {
  if (threadIdx.x < 8) {
    const int c = threadIdx.x;
    const double d = c >= 1 && c <= 5 ? class_diag(c, wall) : 1.0;
    diag[c] = (T)d;
    dinv[c] = (c >= 1 && c <= 5 && d > 0.0) ? (T)(1.0 / d) : (T)0;
  }
}

// Bilinear-adjoint weights of one axis for fine offsets 2I-1 .. 2I+2.
__device__ __forceinline__ float rweight(int a) { return (a == 0 || a == 3) ? 0.25f : 0.75f; }

// Neumann restriction reads the mirrored residual at fine index -1 and, for an
// even fine size n, at index n (the clamped ghost of P^T).
__device__ __forceinline__ int mirror_fine(int f, int n, bool neumann) {
  if (!neumann) return f;
  if (f == -1) return 0;
  if (f == n && !(n & 1)) return n - 1;
  return f;
}

// ---------------------------------------------------------------------------
// Bottom: the remaining V-cycle of one instance, every level in shared memory,
// one CTA of kBThreads threads per instance.
//
// Each level keeps b, u and the cell classes in arrays padded with a ring of
// zero ghosts (one row / column before the grid, two after; the restriction of
// an odd-sized level reaches two cells past its edge).  A missing neighbour
// then reads 0, as the operator defines, and Dirichlet / masked transfers read
// zero ghosts, so no stencil needs a bounds check.  A warp works on whole rows
// and its lanes on columns, so no index is divided.  The residual goes to its
// own array, so b stays in shared memory for the up pass; only the top level's
// b comes from (and its u goes back to) global memory.  The dense inverse of
// the coarsest level is copied in by cp.async while the down pass runs.

template <typename T>
__device__ __forceinline__ void bot_sweep(T *u, const T *b, const unsigned char *c, int ny,
                                          int nx, int px, const T *dinv, int colour) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int y = warp; y < ny; y += kBThreads / 32) {
    const int row = (y + 1) * px + 1;
    for (int x = 2 * lane + ((colour + y) & 1); x < nx; x += 64) {
      const int i = row + x;
      const int cl = c[i];
      if (cl) u[i] = (b[i] + u[i - px] + u[i + px] + u[i - 1] + u[i + 1]) * dinv[cl];
    }
  }
  __syncthreads();
}

// Padded index of fine row / column f for the restriction: Neumann mirrors the
// ghost at -1 and, for an even size n, the ghost at n (the adjoint of the
// clamped prolongation); every other ghost reads zero.
__device__ __forceinline__ int bot_mirror(int f, int n, bool neu) {
  if (neu) {
    if (f == -1) return 0;
    if (f == n && !(n & 1)) return n - 1;
  }
  return f;
}

// The few fields of a bottom level its phases read, staged in shared memory
// once per launch: every phase after a barrier then finds them at shared-memory
// latency instead of reloading the level descriptors from global memory.
struct BotLevel {
  int ny, nx, px, neu;
  int sm_b, sm_u, sm_r, sm_c;
};

// The bottom of one active instance, by the whole CTA (kBThreads threads); the
// CTA's shared memory is free on entry and may be reused on return.  Every
// phase runs on all warps: a phase's time is the chain of rows its busiest warp
// walks, so fewer warps on the small levels were measured slower.
template <typename T, int S1, int S2>
__device__ __forceinline__ void bottom_instance(const Args<T> &a, const int inst,
                                                unsigned char *smem) {
  InstState &S = a.st[inst];
  __shared__ T tdiag[kBottomLevels][8], tdinv[kBottomLevels][8];
  __shared__ BotLevel bl[kBottomLevels];
  const int bottom = a.inst[inst].bottom, coarsest = a.inst[inst].coarsest;
  const bool top_is_fine = bottom == a.inst[inst].level0;
  const int nb = coarsest - bottom + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NW = kBThreads / 32;
  const int nq = a.lv[coarsest].ny * a.lv[coarsest].nx;
  const int sm_d = a.lv[coarsest].sm_d;
  double *const inv_s = reinterpret_cast<double *>(smem + sm_d) + kCoarsestCells;
  {  // the coarsest inverse travels while the levels above are worked on
    const double *inv_g = a.dense + a.lv[coarsest].inv_off;
    for (int k = threadIdx.x; k < nq * nq; k += kBThreads)
      __pipeline_memcpy_async(inv_s + k, inv_g + k, sizeof(double));
    __pipeline_commit();
  }
  {  // zero every padded array up to the inverse (ghost rings stay zero for the whole launch)
    const int bytes = sm_d + kCoarsestCells * (int)sizeof(double);
    uint4 *z = reinterpret_cast<uint4 *>(smem);
    for (int k = threadIdx.x; k < bytes / 16; k += kBThreads) z[k] = make_uint4(0, 0, 0, 0);
  }
  for (int q = threadIdx.x; q < nb * 8; q += kBThreads) {
    const int l = q >> 3, c = q & 7;
    const float w = a.lv[bottom + l].wall;
    const double d = c >= 1 && c <= 5 ? class_diag(c, w) : 1.0;
    tdiag[l][c] = (T)d;
    tdinv[l][c] = (c >= 1 && c <= 5 && d > 0.0) ? (T)(1.0 / d) : T(0);
    if (c == 0) {
      const LevelInfo &L = a.lv[bottom + l];
      bl[l] = BotLevel{L.ny, L.nx, L.sm_px, L.bc == BC_NEU ? 1 : 0, L.sm_b, L.sm_u, L.sm_r,
                       L.sm_c};
    }
  }
  __syncthreads();
  // classes of every level, and b of the top level
  for (int q = 0; q < nb; ++q) {
    const LevelInfo L = a.lv[bottom + q];
    unsigned char *c = smem + L.sm_c;
    const int px = L.sm_px;
    for (int y = warp; y < L.ny; y += NW)
      for (int x = lane; x < L.nx; x += 32)
        c[(y + 1) * px + 1 + x] = (unsigned char)cell_class(L, a.codes, y, x);
  }
  {
    const LevelInfo &L = a.lv[bottom];
    const T *B = a.arena + L.b_off;
    const long long pitch = L.pitch;
    const BotLevel Q = bl[0];
    T *b = reinterpret_cast<T *>(smem + Q.sm_b);
    for (int y = warp; y < Q.ny; y += NW)
      for (int x = lane; x < Q.nx; x += 32)
        b[(y + 1) * Q.px + 1 + x] = B[(long long)y * pitch + x];
  }
  __syncthreads();
  // down: smooth from zero, residual (into b), restriction
  for (int q = 0; q + 1 < nb; ++q) {
    const BotLevel L = bl[q];
    const BotLevel C = bl[q + 1];
    T *u = reinterpret_cast<T *>(smem + L.sm_u);
    const T *b = reinterpret_cast<const T *>(smem + L.sm_b);
    T *res = reinterpret_cast<T *>(smem + L.sm_r);
    const unsigned char *c = smem + L.sm_c;
    const int px = L.px;
    for (int s = 0; s < S1; ++s) {
      bot_sweep(u, b, c, L.ny, L.nx, px, tdinv[q], 0);
      bot_sweep(u, b, c, L.ny, L.nx, px, tdinv[q], 1);
    }
    for (int y = warp; y < L.ny; y += NW) {
      const int row = (y + 1) * px + 1;
      for (int x = lane; x < L.nx; x += 32) {
        const int i = row + x;
        const int cl = c[i];
        const T nbs = u[i - px] + u[i + px] + u[i - 1] + u[i + 1];
        res[i] = cl ? b[i] - (tdiag[q][cl] * u[i] - nbs) : T(0);
      }
    }
    __syncthreads();
    T *bc = reinterpret_cast<T *>(smem + C.sm_b);
    const unsigned char *cc = smem + C.sm_c;
    const bool neu = L.neu != 0;
    const int cpx = C.px;
    for (int Iy = warp; Iy < C.ny; Iy += NW) {
      int fy[4];
#pragma unroll
      for (int pp = 0; pp < 4; ++pp) fy[pp] = (bot_mirror(2 * Iy - 1 + pp, L.ny, neu) + 1) * px + 1;
      for (int Jx = lane; Jx < C.nx; Jx += 32) {
        const int ci = (Iy + 1) * cpx + 1 + Jx;
        T acc = T(0);
        if (cc[ci]) {
          int fx[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) fx[r] = bot_mirror(2 * Jx - 1 + r, L.nx, neu);
#pragma unroll
          for (int pp = 0; pp < 4; ++pp) {
            T rowv = T(0);
#pragma unroll
            for (int r = 0; r < 4; ++r) rowv += (T)rweight(r) * res[fy[pp] + fx[r]];
            acc += (T)rweight(pp) * rowv;
          }
        }
        bc[ci] = acc;
      }
    }
    __syncthreads();
  }
  const BotLevel Lc = bl[nb - 1];
  {  // coarsest: dense FP64 inverse, one warp per row
    const int n = Lc.ny * Lc.nx;
    const int px = Lc.px;
    double *bd = reinterpret_cast<double *>(smem + sm_d);
    const T *b = reinterpret_cast<const T *>(smem + Lc.sm_b);
    T *u = reinterpret_cast<T *>(smem + Lc.sm_u);
    for (int k = threadIdx.x; k < n; k += kBThreads) {
      const int y = k / Lc.nx, x = k - y * Lc.nx;
      bd[k] = (double)b[(y + 1) * px + 1 + x];
    }
    __pipeline_wait_prior(0);
    __syncthreads();
    // a warp's rows (at most kRowsPerWarp) are summed side by side, so their
    // shuffle reductions overlap
    constexpr int kRowsPerWarp = (kCoarsestCells + NW - 1) / NW;
    const double *inv = inv_s;
    double acc[kRowsPerWarp];
#pragma unroll
    for (int r = 0; r < kRowsPerWarp; ++r) {
      const int t = warp + r * NW;
      double v = 0.0;
      if (t < n)
        for (int j = lane; j < n; j += 32) v += inv[(long long)t * n + j] * bd[j];
      acc[r] = v;
    }
#pragma unroll
    for (int r = 0; r < kRowsPerWarp; ++r) acc[r] = warp_sum(acc[r]);
    if (lane == 0) {
#pragma unroll
      for (int r = 0; r < kRowsPerWarp; ++r) {
        const int t = warp + r * NW;
        if (t < n) {
          const int y = t / Lc.nx, x = t - y * Lc.nx;
          u[(y + 1) * px + 1 + x] = (T)acc[r];
        }
      }
    }
    __syncthreads();
  }
  // up: reload b, add the prolonged correction, post-smooth
  for (int q = nb - 2; q >= 0; --q) {
    const BotLevel L = bl[q];
    const BotLevel C = bl[q + 1];
    T *u = reinterpret_cast<T *>(smem + L.sm_u);
    T *b = reinterpret_cast<T *>(smem + L.sm_b);
    const T *e = reinterpret_cast<const T *>(smem + C.sm_u);
    const unsigned char *c = smem + L.sm_c;
    const bool neu = L.neu != 0;
    const int px = L.px, cpx = C.px;
    for (int y = warp; y < L.ny; y += NW) {
      const int row = (y + 1) * px + 1;
      const int cy = y >> 1;
      int cy2 = (y & 1) ? cy + 1 : cy - 1;
      if (neu) cy2 = min(max(cy2, 0), C.ny - 1);
      const int r1 = (cy + 1) * cpx + 1, r2 = (cy2 + 1) * cpx + 1;
      for (int x = lane; x < L.nx; x += 32) {
        const int i = row + x;
        if (!c[i]) continue;
        const int cx = x >> 1;
        int cx2 = (x & 1) ? cx + 1 : cx - 1;
        if (neu) cx2 = min(max(cx2, 0), C.nx - 1);
        u[i] += (T)0.5625 * e[r1 + cx] + (T)0.1875 * (e[r2 + cx] + e[r1 + cx2]) +
                (T)0.0625 * e[r2 + cx2];
      }
    }
    __syncthreads();
    for (int s = 0; s < S2; ++s) {
      bot_sweep(u, b, c, L.ny, L.nx, px, tdinv[q], 1);
      bot_sweep(u, b, c, L.ny, L.nx, px, tdinv[q], 0);
    }
  }
  const BotLevel L0 = bl[0];
  const LevelInfo &G0 = a.lv[bottom];
  T *U = a.arena + G0.u_off;
  const long long pitch0 = G0.pitch;
  const T *u0 = reinterpret_cast<const T *>(smem + L0.sm_u);
  const T *b0 = reinterpret_cast<const T *>(smem + L0.sm_b);
  double part = 0.0;
  for (int y = warp; y < L0.ny; y += NW) {
    const int row = (y + 1) * L0.px + 1;
    for (int x = lane; x < L0.nx; x += 32) {
      const T v = u0[row + x];
      U[(long long)y * pitch0 + x] = v;
      part += (double)b0[row + x] * (double)v;
    }
  }
  if (top_is_fine) {
    part = block_sum<kBThreads>(part);
    if (threadIdx.x == 0) finish_rz(S, part);
  }
}

// One CTA per instance.
template <typename T, int S1, int S2>
__global__ void __launch_bounds__(kBThreads, 1) k_bottom(Args<T> a) {
  dep_enter();
  if (a.st[blockIdx.x].status != GD_ACTIVE) return;
  extern __shared__ __align__(16) unsigned char smem[];
  bottom_instance<T, S1, S2>(a, blockIdx.x, smem);
}

// ---------------------------------------------------------------------------
// Elementwise level-0 kernels over 64 x 128 tiles (the Krylov kernels with
// halos are in gd_stream.cuh).

// x += d for instances with a pending FP64 refresh (d then restarts from zero
// through FLAG_DZERO instead of being cleared here).  A thread owns one
// column of the 64 x 128 tile, so every warp access is 32 consecutive
// elements; the independent rows are unrolled for several loads in flight.
// Sum of column x over rows y0 .. y1 - 1 of an FP64 array, eight independent
// loads in flight per thread and a fixed summation tree.
__device__ __forceinline__ double column_sum(const double *A, long long pitch, int y0, int y1,
                                             int x) {
  double s[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) s[k] = 0.0;
  for (int yb = y0; yb < y1; yb += 8) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = yb + k < y1 ? A[(long long)(yb + k) * pitch + x] : 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] += v[k];
  }
  return ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
}

// Mean of the right-hand side of zero-mean (Neumann) instances: the constant
// component of f is outside the range of A and is dropped, as the DCT solver
// drops it by zeroing the DC coefficient (solvers.py:258-261).
template <typename T>
__global__ void __launch_bounds__(kFThreads) k_fmean(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  dep_enter();
  if (blockIdx.x == 0 && threadIdx.x == 0) a.counter[kErrWord] = 0u;  // a solve starts
  const InstInfo &I = a.inst[tl.inst];
  double part = 0.0;
  if (I.zero_mean) {
    const int Y0 = tl.ty * kFTY, gx = tl.tx * kFTX + threadIdx.x;
    if (gx < I.nx) part = column_sum(I.f, I.upitch, Y0, min(Y0 + kFTY, I.ny), gx);
  }
  part = block_sum<kFThreads>(part);
  if (threadIdx.x == 0) a.part0[blockIdx.x] = part;
  if (!last_block(a.counter + 5)) return;
  const int warp = threadIdx.x >> 5;
  for (int i = warp; i < a.ninst; i += kLastWarps) {
    const InstInfo &J = a.inst[i];
    const double s = J.zero_mean ? warp_range_sum(a.part0, J.fine_begin, J.fine_end) : 0.0;
    if ((threadIdx.x & 31) == 0) a.st[i].fmean = s / ((double)J.ny * (double)J.nx);
  }
}

// Mean removal for zero-mean (Neumann) instances: partial sums, then subtract.
template <typename T>
__global__ void __launch_bounds__(kFThreads) k_mean(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  dep_enter();
  const InstInfo &I = a.inst[tl.inst];
  double part = 0.0;
  // only solutions no refresh has summed: a caller's x that met the tolerance at once
  if (I.zero_mean && !a.st[tl.inst].mean_known) {
    const bool own = a.st[tl.inst].xcur != 0;
    const double *X = own ? a.xs + I.xs_off : I.x;
    const long long pitch = own ? (long long)I.pitch : I.upitch;
    const int Y0 = tl.ty * kFTY, gx = tl.tx * kFTX + threadIdx.x;
    if (gx < I.nx) part = column_sum(X, pitch, Y0, min(Y0 + kFTY, I.ny), gx);
  }
  part = block_sum<kFThreads>(part);
  if (threadIdx.x == 0) a.part0[blockIdx.x] = part;
  if (!last_block(a.counter + 4)) return;
  const int warp = threadIdx.x >> 5;
  for (int i = warp; i < a.ninst; i += kLastWarps) {
    const InstInfo &J = a.inst[i];
    if (!J.zero_mean || a.st[i].mean_known) continue;
    const double s = warp_range_sum(a.part0, J.fine_begin, J.fine_end);
    if ((threadIdx.x & 31) == 0) a.st[i].mean = s / ((double)J.ny * (double)J.nx);
  }
}

// The solution into the caller's buffer: x - mean for zero-mean instances, a
// copy when the last refresh left the solution in the plan's own copy, zeros
// when a zero-start solve ended without folding a correction (the caller's x
// was never read and may hold anything).
template <typename T>
__global__ void __launch_bounds__(kFThreads) k_submean(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  dep_enter();
  const InstInfo &Ig = a.inst[tl.inst];
  const bool own = a.st[tl.inst].xcur != 0;
  const bool xz = a.st[tl.inst].xzero != 0;
  if (!Ig.zero_mean && !own && !xz) return;
  const int ny = Ig.ny, nx = Ig.nx;
  const long long upitch = Ig.upitch;
  double *const X = Ig.x;
  const double *const src = own ? a.xs + Ig.xs_off : X;
  const long long spitch = own ? (long long)Ig.pitch : upitch;
  const double m = Ig.zero_mean ? a.st[tl.inst].mean : 0.0;
  const int Y0 = tl.ty * kFTY, gx = tl.tx * kFTX + threadIdx.x;
  if (gx >= nx) return;
  const int y1 = min(Y0 + kFTY, ny);
  for (int yb = Y0; yb < y1; yb += 8) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
      v[k] = (yb + k < y1 && !xz) ? src[(long long)(yb + k) * spitch + gx] : 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (yb + k < y1) X[(long long)(yb + k) * upitch + gx] = v[k] - m;
  }
}

// ---------------------------------------------------------------------------
// Setup kernels.

// Level-0 classes of a masked instance from the caller's unknown mask.
__global__ void k_codes_fine(unsigned char *code, int pitch, const unsigned char *mask,
                             int mpitch, int ny, int nx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ny * nx) return;
  const int y = k / nx, x = k - y * nx;
  auto on = [&](int yy, int xx) {
    return yy >= 0 && yy < ny && xx >= 0 && xx < nx && mask[(long long)yy * mpitch + xx] != 0;
  };
  unsigned char c = 0;
  if (on(y, x)) c = (unsigned char)(1 + !on(y - 1, x) + !on(y + 1, x) + !on(y, x - 1) + !on(y, x + 1));
  code[(long long)y * pitch + x] = c;
}

// Coarse activity: a coarse cell has an unknown when any of its children has.
__global__ void k_codes_coarse_act(unsigned char *cc, int cpitch, int cny, int cnx,
                                   const unsigned char *fc, int fpitch, int fny, int fnx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= cny * cnx) return;
  const int y = k / cnx, x = k - y * cnx;
  int any = 0;
  for (int dy = 0; dy < 2; ++dy)
    for (int dx = 0; dx < 2; ++dx) {
      const int fy = 2 * y + dy, fx = 2 * x + dx;
      if (fy < fny && fx < fnx && fc[(long long)fy * fpitch + fx]) any = 1;
    }
  cc[(long long)y * cpitch + x] = (unsigned char)any;
}

// Turn activity flags into classes (1 + walls); in place is safe because a
// value is non-zero exactly when the cell is active, before and after.
__global__ void k_codes_classes(unsigned char *cc, int pitch, int ny, int nx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ny * nx) return;
  const int y = k / nx, x = k - y * nx;
  auto on = [&](int yy, int xx) {
    return yy >= 0 && yy < ny && xx >= 0 && xx < nx && cc[(long long)yy * pitch + xx] != 0;
  };
  if (!on(y, x)) return;
  const int w = !on(y - 1, x) + !on(y + 1, x) + !on(y, x - 1) + !on(y, x + 1);
  cc[(long long)y * pitch + x] = (unsigned char)(1 + w);
}

// Dense FP64 inverse of the coarsest operator of each instance by in-place
// Gauss-Jordan (the matrix is SPD, or SPD after adding J/n for Neumann).
__global__ void __launch_bounds__(256) k_coarse_inverse(const LevelInfo *lv, const InstInfo *inst,
                                                        const unsigned char *codes,
                                                        double *dense) {
  const InstInfo &I = inst[blockIdx.x];
  const LevelInfo L = lv[I.coarsest];
  const int n = L.ny * L.nx;
  __shared__ double A[kCoarsestCells * kCoarsestCells];
  __shared__ unsigned char cls[kCoarsestCells];
  for (int k = threadIdx.x; k < n; k += blockDim.x)
    cls[k] = (unsigned char)cell_class(L, codes, k / L.nx, k % L.nx);
  __syncthreads();
  const double reg = (L.bc == BC_NEU) ? 1.0 / n : 0.0;
  for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
    const int i = k / n, j = k - i * n;
    const int yi = i / L.nx, xi = i - yi * L.nx, yj = j / L.nx, xj = j - yj * L.nx;
    double v = reg;
    if (!cls[i] || !cls[j]) {
      v = (i == j && !cls[i]) ? 1.0 : 0.0;
    } else if (i == j) {
      v += class_diag(cls[i], L.wall);
    } else if (abs(yi - yj) + abs(xi - xj) == 1) {
      v -= 1.0;
    }
    A[k] = v;
  }
  __syncthreads();
  __shared__ double piv_inv;
  __shared__ double colk[kCoarsestCells];
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x == 0) piv_inv = 1.0 / A[k * n + k];
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      A[k * n + j] = (j == k ? 1.0 : A[k * n + j]) * piv_inv;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) colk[i] = A[i * n + k];
    __syncthreads();
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
      const int i = q / n, j = q - i * n;
      if (i == k) continue;
      const double f = colk[i];
      A[q] = (j == k ? 0.0 : A[q]) - f * A[k * n + j];
    }
    __syncthreads();
  }
  double *out = dense + L.inv_off;
  for (int k = threadIdx.x; k < n * n; k += blockDim.x) out[k] = A[k];
}

}  // namespace gd
