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
// Bottom: the remaining V-cycle of one instance in shared memory.
struct BottomLevel {
  int ny, nx, bc;
  float wall;
  int off_b, off_u, off_c;  // shared-memory offsets (T elements / bytes)
};

template <typename T>
__device__ __forceinline__ T sm_at(const T *u, int y, int x, int ny, int nx) {
  return (y >= 0 && y < ny && x >= 0 && x < nx) ? u[y * nx + x] : T(0);
}

template <typename T>
__device__ void bottom_smooth(T *u, const T *b, const unsigned char *c, const BottomLevel &L,
                              const T *dinv, int colour) {
  const int hw = (L.nx + 1) >> 1;
  for (int k = threadIdx.x; k < L.ny * hw; k += blockDim.x) {
    const int y = k / hw;
    const int x = 2 * (k - y * hw) + ((colour + y) & 1);
    if (x >= L.nx) continue;
    const int i = y * L.nx + x;
    const int cl = c[i];
    if (cl)
      u[i] = (b[i] + sm_at(u, y - 1, x, L.ny, L.nx) + sm_at(u, y + 1, x, L.ny, L.nx) +
              sm_at(u, y, x - 1, L.ny, L.nx) + sm_at(u, y, x + 1, L.ny, L.nx)) * dinv[cl];
  }
  __syncthreads();
}

template <typename T, int S1, int S2>
__global__ void __launch_bounds__(kBThreads) k_bottom(Args<T> a) {
  const int inst = blockIdx.x;
  InstState &S = a.st[inst];
  if (S.status != GD_ACTIVE) return;
  const InstInfo &I = a.inst[inst];
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BottomLevel bl[24];
  __shared__ T tdiag[24][8], tdinv[24][8];
  __shared__ int nb_s, res_off_s, dense_off_s, cbytes_off_s;
  if (threadIdx.x == 0) {
    int nb = 0, off = 0;
    for (int l = I.bottom;; ++l) {
      const LevelInfo &L = a.lv[l];
      BottomLevel &B = bl[nb++];
      B.ny = L.ny; B.nx = L.nx; B.bc = L.bc; B.wall = L.wall;
      B.off_b = off; off += L.ny * L.nx;
      B.off_u = off; off += L.ny * L.nx;
      if (l == I.coarsest || nb == 24) break;
    }
    nb_s = nb;
    res_off_s = off;
    off += bl[0].ny * bl[0].nx;
    // double buffer for the dense solve, 8-byte aligned in T units
    off = (off * (int)sizeof(T) + 7) / 8 * 8 / (int)sizeof(T);
    dense_off_s = off;
    off += 2 * kCoarsestCells * (int)(sizeof(double) / sizeof(T));
    int cb = off * (int)sizeof(T);
    for (int q = 0; q < nb; ++q) { bl[q].off_c = cb; cb += bl[q].ny * bl[q].nx; }
    cbytes_off_s = cb;
  }
  __syncthreads();
  const int nb = nb_s;
  T *sm = reinterpret_cast<T *>(smem);
  for (int q = threadIdx.x; q < nb * 8; q += blockDim.x) {
    const int l = q >> 3, c = q & 7;
    const double d = c >= 1 && c <= 5 ? class_diag(c, bl[l].wall) : 1.0;
    tdiag[l][c] = (T)d;
    tdinv[l][c] = (c >= 1 && c <= 5) ? (T)(1.0 / d) : T(0);
  }
  // classes of every level, and b of the bottom level
  for (int q = 0; q < nb; ++q) {
    const LevelInfo &L = a.lv[I.bottom + q];
    unsigned char *c = smem + bl[q].off_c;
    for (int k = threadIdx.x; k < L.ny * L.nx; k += blockDim.x) {
      const int y = k / L.nx, x = k - y * L.nx;
      c[k] = (unsigned char)cell_class(L, a.codes, y, x);
    }
  }
  {
    const LevelInfo &L = a.lv[I.bottom];
    const T *B = a.arena + L.b_off;
    T *b0 = sm + bl[0].off_b;
    for (int k = threadIdx.x; k < L.ny * L.nx; k += blockDim.x) {
      const int y = k / L.nx, x = k - y * L.nx;
      b0[k] = B[(long long)y * L.pitch + x];
    }
  }
  __syncthreads();
  T *res = sm + res_off_s;
  for (int q = 0; q + 1 < nb; ++q) {
    const BottomLevel &L = bl[q];
    T *u = sm + L.off_u;
    const T *b = sm + L.off_b;
    const unsigned char *c = smem + L.off_c;
    const int n = L.ny * L.nx;
    for (int k = threadIdx.x; k < n; k += blockDim.x) u[k] = T(0);
    __syncthreads();
    for (int s = 0; s < S1; ++s) {
      bottom_smooth(u, b, c, L, tdinv[q], 0);
      bottom_smooth(u, b, c, L, tdinv[q], 1);
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int y = k / L.nx, x = k - y * L.nx;
      const int cl = c[k];
      const T nbs = sm_at(u, y - 1, x, L.ny, L.nx) + sm_at(u, y + 1, x, L.ny, L.nx) +
                    sm_at(u, y, x - 1, L.ny, L.nx) + sm_at(u, y, x + 1, L.ny, L.nx);
      res[k] = cl ? b[k] - (tdiag[q][cl] * u[k] - nbs) : T(0);
    }
    __syncthreads();
    const BottomLevel &Cl = bl[q + 1];
    T *bc = sm + Cl.off_b;
    const unsigned char *cc = smem + Cl.off_c;
    const bool neu = L.bc == BC_NEU;
    for (int k = threadIdx.x; k < Cl.ny * Cl.nx; k += blockDim.x) {
      const int Iy = k / Cl.nx, Jx = k - Iy * Cl.nx;
      T acc = T(0);
      if (cc[k]) {
        for (int p = 0; p < 4; ++p) {
          const int fy = mirror_fine(2 * Iy - 1 + p, L.ny, neu);
          T row = T(0);
          for (int r = 0; r < 4; ++r) {
            const int fx = mirror_fine(2 * Jx - 1 + r, L.nx, neu);
            row += (T)rweight(r) * sm_at(res, fy, fx, L.ny, L.nx);
          }
          acc += (T)rweight(p) * row;
        }
      }
      bc[k] = acc;
    }
    __syncthreads();
  }
  {  // coarsest: dense FP64 inverse
    const BottomLevel &L = bl[nb - 1];
    const int n = L.ny * L.nx;
    double *bd = reinterpret_cast<double *>(sm + dense_off_s);
    const T *b = sm + L.off_b;
    T *u = sm + L.off_u;
    for (int k = threadIdx.x; k < n; k += blockDim.x) bd[k] = (double)b[k];
    __syncthreads();
    const double *inv = a.dense + a.lv[I.coarsest].inv_off;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      double acc = 0.0;
      for (int j = 0; j < n; ++j) acc += inv[(long long)t * n + j] * bd[j];
      u[t] = (T)acc;
    }
    __syncthreads();
  }
  for (int q = nb - 2; q >= 0; --q) {
    const BottomLevel &L = bl[q];
    const BottomLevel &Cl = bl[q + 1];
    T *u = sm + L.off_u;
    const T *b = sm + L.off_b;
    const T *e = sm + Cl.off_u;
    const unsigned char *c = smem + L.off_c;
    const bool neu = L.bc == BC_NEU;
    for (int k = threadIdx.x; k < L.ny * L.nx; k += blockDim.x) {
      if (!c[k]) continue;
      const int y = k / L.nx, x = k - y * L.nx;
      const int cy = y >> 1, cx = x >> 1;
      const int cy2 = (y & 1) ? cy + 1 : cy - 1, cx2 = (x & 1) ? cx + 1 : cx - 1;
      auto E = [&](int yy, int xx) -> T {
        if (neu) {
          yy = min(max(yy, 0), Cl.ny - 1);
          xx = min(max(xx, 0), Cl.nx - 1);
          return e[yy * Cl.nx + xx];
        }
        return sm_at(e, yy, xx, Cl.ny, Cl.nx);
      };
      u[k] += (T)0.5625 * E(cy, cx) + (T)0.1875 * (E(cy2, cx) + E(cy, cx2)) +
              (T)0.0625 * E(cy2, cx2);
    }
    __syncthreads();
    for (int s = 0; s < S2; ++s) {
      bottom_smooth(u, b, c, L, tdinv[q], 1);
      bottom_smooth(u, b, c, L, tdinv[q], 0);
    }
  }
  const LevelInfo &L0 = a.lv[I.bottom];
  T *U = a.arena + L0.u_off;
  const T *u0 = sm + bl[0].off_u;
  const T *b0 = sm + bl[0].off_b;
  double part = 0.0;
  for (int k = threadIdx.x; k < L0.ny * L0.nx; k += blockDim.x) {
    const int y = k / L0.nx, x = k - y * L0.nx;
    U[(long long)y * L0.pitch + x] = u0[k];
    part += (double)b0[k] * (double)u0[k];
  }
  if (I.bottom == I.level0) {
    part = block_sum<kBThreads>(part);
    if (threadIdx.x == 0) finish_rz(S, part);
  }
}

// ---------------------------------------------------------------------------
// Elementwise level-0 kernels over 64 x 128 tiles (the Krylov kernels with
// halos are in gd_stream.cuh).

// x += d, d = 0 for instances with a pending FP64 refresh.  A thread owns one
// column of the 64 x 128 tile, so every warp access is 32 consecutive
// elements; the independent rows are unrolled for several loads in flight.
template <typename T>
__global__ void __launch_bounds__(kFThreads) k_fold(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  if (!(a.st[tl.inst].flags & FLAG_RU)) return;
  // descriptor fields in registers: the stores below could alias the descriptor
  const InstInfo &Ig = a.inst[tl.inst];
  const int ny = Ig.ny, nx = Ig.nx, pitch = Ig.pitch;
  const long long upitch = Ig.upitch;
  double *const X = Ig.x;
  T *const d = a.arena + Ig.d_off;
  const int x = tl.tx * kFTX + threadIdx.x;
  const int y0 = tl.ty * kFTY;
  if (x >= nx) return;
  const int y1 = min(y0 + kFTY, ny);
#pragma unroll 8
  for (int y = y0; y < y1; ++y) {
    const long long g = (long long)y * pitch + x;
    X[(long long)y * upitch + x] += (double)d[g];
    d[g] = T(0);
  }
}

// Mean of the right-hand side of zero-mean (Neumann) instances: the constant
// component of f is outside the range of A and is dropped, as the DCT solver
// drops it by zeroing the DC coefficient (solvers.py:258-261).
template <typename T>
__global__ void __launch_bounds__(kFThreads) k_fmean(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  const InstInfo &I = a.inst[tl.inst];
  double part = 0.0;
  if (I.zero_mean) {
    const int Y0 = tl.ty * kFTY, X0 = tl.tx * kFTX;
    for (int k = threadIdx.x; k < kFTY * kFTX; k += blockDim.x) {
      const int gy = Y0 + k / kFTX, gx = X0 + k % kFTX;
      if (gy < I.ny && gx < I.nx) part += I.f[(long long)gy * I.upitch + gx];
    }
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
  const InstInfo &I = a.inst[tl.inst];
  double part = 0.0;
  if (I.zero_mean) {
    const int Y0 = tl.ty * kFTY, X0 = tl.tx * kFTX;
    for (int k = threadIdx.x; k < kFTY * kFTX; k += blockDim.x) {
      const int gy = Y0 + k / kFTX, gx = X0 + k % kFTX;
      if (gy < I.ny && gx < I.nx) part += I.x[(long long)gy * I.upitch + gx];
    }
  }
  part = block_sum<kFThreads>(part);
  if (threadIdx.x == 0) a.part0[blockIdx.x] = part;
  if (!last_block(a.counter + 4)) return;
  const int warp = threadIdx.x >> 5;
  for (int i = warp; i < a.ninst; i += kLastWarps) {
    const InstInfo &J = a.inst[i];
    if (!J.zero_mean) continue;
    const double s = warp_range_sum(a.part0, J.fine_begin, J.fine_end);
    if ((threadIdx.x & 31) == 0) a.st[i].mean = s / ((double)J.ny * (double)J.nx);
  }
}

template <typename T>
__global__ void __launch_bounds__(kFThreads) k_submean(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  const InstInfo &Ig = a.inst[tl.inst];
  if (!Ig.zero_mean) return;
  const int ny = Ig.ny, nx = Ig.nx;
  const long long upitch = Ig.upitch;
  double *const X = Ig.x;
  const double m = a.st[tl.inst].mean;
  const int Y0 = tl.ty * kFTY, X0 = tl.tx * kFTX;
  for (int k = threadIdx.x; k < kFTY * kFTX; k += blockDim.x) {
    const int gy = Y0 + k / kFTX, gx = X0 + k % kFTX;
    if (gy < ny && gx < nx) X[(long long)gy * upitch + gx] -= m;
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
