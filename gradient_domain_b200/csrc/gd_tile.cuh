// Shared-memory tile kernels for the small coarse levels of the V-cycle.
//
// The register-streaming kernels of gd_stream.cuh walk every strip row by row;
// on a small level a launch has too few strips to fill the GPU and each warp
// waits on the latency of its own row chain, so a level costs a fixed 15-30 us
// whatever its size.  Here a CTA instead loads one tile of the level plus a
// halo into shared memory and runs every phase (a red-black half sweep, the
// residual, the restriction or the prolongation) over the whole tile at once,
// with a barrier between phases: all cells of a phase are independent, so the
// CTA's threads work in parallel and a small level costs a few microseconds.
//
// Tiles are kTY x kTX cells of the level.  A half sweep that reads neighbours
// leaves the outermost exact ring of the loaded region one cell further in, so
// the down kernel (whose first half sweep, from zero, reads only b) loads a
// halo of 2 S1 + 1 cells (2 S1 - 1 for the sweeps, one for the residual's
// neighbours, one for the restriction's reach) and the up kernel 2 S2.  Cells
// outside the grid have class 0: they hold zeros and are never updated, which
// is the operator's definition of a missing neighbour.
#pragma once

#include "gd_mg_kernels.cuh"

namespace gd {
namespace tile {

constexpr int kTY = 32, kTX = 64;  // cells of a tile (even: whole coarse cells)
constexpr int kThreads = 256;

template <typename T, int S1>
struct DownT {
  static constexpr int H = 2 * S1 + 1;
  static constexpr int RY = kTY + 2 * H, RX = kTX + 2 * H, N = RY * RX;
  static constexpr size_t smem = (size_t)N * (2 * sizeof(T) + 1) + 16;
};

template <typename T, int S2>
struct UpT {
  static constexpr int H = 2 * S2;
  static constexpr int RY = kTY + 2 * H, RX = kTX + 2 * H, N = RY * RX;
  static constexpr int CY = RY / 2 + 3, CX = RX / 2 + 3, CN = CY * CX;
  static constexpr size_t smem = (size_t)(2 * N + CN) * sizeof(T) + N + 16;
};

template <typename T>
__device__ __forceinline__ void diag_tables(T *tdiag, T *tdinv, float wall) {
  if (threadIdx.x < 8) {
    const int c = threadIdx.x;
    const double d = c >= 1 && c <= 5 ? class_diag(c, wall) : 1.0;
    tdiag[c] = (T)d;
    tdinv[c] = (c >= 1 && c <= 5 && d > 0.0) ? (T)(1.0 / d) : T(0);
  }
}

// One red-black half sweep over the interior of an RY x RX region whose
// corner is grid cell (gy0, gx0); colour is the parity of (row + column).
// The cells of one colour only read cells of the other, so each thread first
// gathers the operands of all its cells and then writes them: the shared-memory
// loads of different cells overlap instead of waiting behind earlier stores.
template <typename T, int RY, int RX>
__device__ __forceinline__ void tsweep(T *u, const T *b, const unsigned char *c, const T *dinv,
                                       int colour, int gy0, int gx0) {
  constexpr int HX = (RX - 1) / 2;  // cells of one colour in a row interior, at most
  constexpr int M = (RY - 2) * HX;
  constexpr int IT = (M + kThreads - 1) / kThreads;
  int idx[IT];
  T val[IT];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int k = threadIdx.x + it * kThreads;
    const int ry = 1 + k / HX;
    const int j = k - (ry - 1) * HX;
    const int rx = 1 + 2 * j + ((colour + gy0 + gx0 + ry + 1) & 1);
    const int i = ry * RX + rx;
    const int cl = (k < M && rx < RX - 1) ? c[i] : 0;
    idx[it] = cl ? i : -1;
    val[it] = cl ? (b[i] + u[i - RX] + u[i + RX] + u[i - 1] + u[i + 1]) * dinv[cl] : T(0);
  }
#pragma unroll
  for (int it = 0; it < IT; ++it)
    if (idx[it] >= 0) u[idx[it]] = val[it];
  __syncthreads();
}

// Restriction index of fine row / column f (Neumann mirrors the ghost at -1
// and, for an even size n, the ghost at n).
__device__ __forceinline__ int tmirror(int f, int n, bool neu) {
  if (neu) {
    if (f == -1) return 0;
    if (f == n && !(n & 1)) return n - 1;
  }
  return f;
}

// Down on one tile: S1 pre-sweeps from zero, the pre-smoothed iterate to w,
// residual, restriction (P^T) into the coarse right-hand side.
template <typename T, int S1>
__global__ void __launch_bounds__(kThreads) k_down_t(Args<T> a) {
  using G = DownT<T, S1>;
  constexpr int RY = G::RY, RX = G::RX, H = G::H, N = G::N;
  const Tile tl = a.tiles[blockIdx.x];
  if (a.st[tl.inst].status != GD_ACTIVE) return;
  const LevelInfo L = a.lv[tl.level];
  const LevelInfo Lc = a.lv[L.coarse];
  extern __shared__ __align__(16) unsigned char smem[];
  T *sb = reinterpret_cast<T *>(smem);
  T *su = sb + N;
  unsigned char *sc = reinterpret_cast<unsigned char *>(su + N);
  __shared__ T tdiag[8], tdinv[8];
  diag_tables(tdiag, tdinv, L.wall);
  __syncthreads();
  const int y0 = tl.ty * kTY, x0 = tl.tx * kTX;
  const int gy0 = y0 - H, gx0 = x0 - H;
  const T *B = a.arena + L.b_off;
  // load, with the first half sweep (colour 0 from zero reads only b) applied
  // on the whole region, its outermost ring included; every load of a thread
  // is issued before the first is used
  {
    constexpr int IT = (N + kThreads - 1) / kThreads;
    T bv[IT];
    int cl[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int k = threadIdx.x + it * kThreads;
      const int ry = k / RX, rx = k - ry * RX;
      const int y = gy0 + ry, x = gx0 + rx;
      const bool in = k < N && y >= 0 && y < L.ny && x >= 0 && x < L.nx;
      bv[it] = in ? B[(long long)y * L.pitch + x] : T(0);
      cl[it] = in ? cell_class(L, a.codes, y, x) : 0;
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int k = threadIdx.x + it * kThreads;
      if (k >= N) break;
      const int ry = k / RX, rx = k - ry * RX;
      sb[k] = bv[it];
      su[k] = ((gy0 + ry + gx0 + rx) & 1) == 0 ? bv[it] * tdinv[cl[it]] : T(0);
      sc[k] = (unsigned char)cl[it];
    }
  }
  __syncthreads();
  tsweep<T, RY, RX>(su, sb, sc, tdinv, 1, gy0, gx0);
  for (int s = 1; s < S1; ++s) {
    tsweep<T, RY, RX>(su, sb, sc, tdinv, 0, gy0, gx0);
    tsweep<T, RY, RX>(su, sb, sc, tdinv, 1, gy0, gx0);
  }
  T *W = a.arena + L.w_off;
  for (int k = threadIdx.x; k < kTY * kTX; k += kThreads) {
    const int ty = k / kTX, tx = k - ty * kTX;
    const int y = y0 + ty, x = x0 + tx;
    if (y < L.ny && x < L.nx) W[(long long)y * L.pitch + x] = su[(ty + H) * RX + tx + H];
  }
  // residual on the tile plus one ring, in place into b (each cell reads only
  // its own b and the unchanged u)
  {
    constexpr int QY = kTY + 2, QX = kTX + 2, M = QY * QX;
    constexpr int IT = (M + kThreads - 1) / kThreads;
    T val[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int k = threadIdx.x + it * kThreads;
      const int qy = k / QX, qx = k - qy * QX;
      const int i = (qy + H - 1) * RX + (qx + H - 1);
      const int cl = k < M ? sc[i] : 0;
      const T nbs = cl ? su[i - RX] + su[i + RX] + su[i - 1] + su[i + 1] : T(0);
      val[it] = cl ? sb[i] - (tdiag[cl] * su[i] - nbs) : T(0);
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int k = threadIdx.x + it * kThreads;
      const int qy = k / QX, qx = k - qy * QX;
      if (k < M) sb[(qy + H - 1) * RX + (qx + H - 1)] = val[it];
    }
  }
  __syncthreads();
  const bool neu = L.bc == BC_NEU;
  T *Bc = a.arena + Lc.b_off;
  constexpr int CTY = kTY / 2, CTX = kTX / 2;
  for (int k = threadIdx.x; k < CTY * CTX; k += kThreads) {
    const int qy = k / CTX, qx = k - qy * CTX;
    const int I = (y0 >> 1) + qy, J = (x0 >> 1) + qx;
    if (I >= Lc.ny || J >= Lc.nx) continue;
    T acc = T(0);
    if (cell_class(Lc, a.codes, I, J)) {
      int fx[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) fx[r] = tmirror(2 * J - 1 + r, L.nx, neu) - gx0;
#pragma unroll
      for (int pp = 0; pp < 4; ++pp) {
        const T *row = sb + (tmirror(2 * I - 1 + pp, L.ny, neu) - gy0) * RX;
        T rowv = T(0);
#pragma unroll
        for (int r = 0; r < 4; ++r) rowv += (T)rweight(r) * row[fx[r]];
        acc += (T)rweight(pp) * rowv;
      }
    }
    Bc[(long long)I * Lc.pitch + J] = acc;
  }
}

// Up on one tile: u = w + P e (bilinear; Neumann clamps at the edge, other
// boundaries read zero outside), then S2 post-sweeps, colour 1 first.
template <typename T, int S2>
__global__ void __launch_bounds__(kThreads) k_up_t(Args<T> a) {
  using G = UpT<T, S2>;
  constexpr int RY = G::RY, RX = G::RX, H = G::H, N = G::N, CX = G::CX;
  const Tile tl = a.tiles[blockIdx.x];
  if (a.st[tl.inst].status != GD_ACTIVE) return;
  const LevelInfo L = a.lv[tl.level];
  const LevelInfo Lc = a.lv[L.coarse];
  extern __shared__ __align__(16) unsigned char smem[];
  T *sb = reinterpret_cast<T *>(smem);
  T *su = sb + N;
  T *se = su + N;
  unsigned char *sc = reinterpret_cast<unsigned char *>(se + G::CN);
  __shared__ T tdiag[8], tdinv[8];
  diag_tables(tdiag, tdinv, L.wall);
  const int y0 = tl.ty * kTY, x0 = tl.tx * kTX;
  const int gy0 = y0 - H, gx0 = x0 - H;
  const bool neu = L.bc == BC_NEU;
  // coarse correction around the region: coarse rows (gy0 >> 1) - 1 ..
  const int cy0 = (gy0 >> 1) - 1, cx0 = (gx0 >> 1) - 1;
  const T *E = a.arena + Lc.u_off;
  const T *B = a.arena + L.b_off;
  const T *W = a.arena + L.w_off;
  {  // every load of a thread is issued before the first is used
    constexpr int ITC = (G::CN + kThreads - 1) / kThreads;
    constexpr int IT = (N + kThreads - 1) / kThreads;
    T ev[ITC], bv[IT], wv[IT];
    int cl[IT];
#pragma unroll
    for (int it = 0; it < ITC; ++it) {
      const int k = threadIdx.x + it * kThreads;
      const int ry = k / CX, rx = k - ry * CX;
      int cy = cy0 + ry, cx = cx0 + rx;
      bool ok = k < G::CN;
      if (neu) {
        cy = min(max(cy, 0), Lc.ny - 1);
        cx = min(max(cx, 0), Lc.nx - 1);
      } else {
        ok = ok && cy >= 0 && cy < Lc.ny && cx >= 0 && cx < Lc.nx;
      }
      ev[it] = ok ? E[(long long)cy * Lc.pitch + cx] : T(0);
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int k = threadIdx.x + it * kThreads;
      const int ry = k / RX, rx = k - ry * RX;
      const int y = gy0 + ry, x = gx0 + rx;
      const bool in = k < N && y >= 0 && y < L.ny && x >= 0 && x < L.nx;
      cl[it] = in ? cell_class(L, a.codes, y, x) : 0;
      bv[it] = in ? B[(long long)y * L.pitch + x] : T(0);
      wv[it] = cl[it] ? W[(long long)y * L.pitch + x] : T(0);
    }
#pragma unroll
    for (int it = 0; it < ITC; ++it) {
      const int k = threadIdx.x + it * kThreads;
      if (k < G::CN) se[k] = ev[it];
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int k = threadIdx.x + it * kThreads;
      if (k >= N) break;
      sb[k] = bv[it];
      su[k] = wv[it];
      sc[k] = (unsigned char)cl[it];
    }
  }
  __syncthreads();
  {  // u += P e (each cell reads the coarse values and only its own u)
    constexpr int IT = (N + kThreads - 1) / kThreads;
    T val[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int k = threadIdx.x + it * kThreads;
      val[it] = T(0);
      if (k < N && sc[k]) {
        const int ry = k / RX, rx = k - ry * RX;
        const int y = gy0 + ry, x = gx0 + rx;
        const int cy = y >> 1, cx = x >> 1;
        const int cy2 = (y & 1) ? cy + 1 : cy - 1, cx2 = (x & 1) ? cx + 1 : cx - 1;
        const T *r1 = se + (cy - cy0) * CX - cx0, *r2 = se + (cy2 - cy0) * CX - cx0;
        val[it] = (T)0.5625 * r1[cx] + (T)0.1875 * (r2[cx] + r1[cx2]) + (T)0.0625 * r2[cx2];
      }
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int k = threadIdx.x + it * kThreads;
      if (k < N) su[k] += val[it];
    }
  }
  __syncthreads();
  for (int s = 0; s < S2; ++s) {
    tsweep<T, RY, RX>(su, sb, sc, tdinv, 1, gy0, gx0);
    tsweep<T, RY, RX>(su, sb, sc, tdinv, 0, gy0, gx0);
  }
  T *U = a.arena + L.u_off;
  for (int k = threadIdx.x; k < kTY * kTX; k += kThreads) {
    const int ty = k / kTX, tx = k - ty * kTX;
    const int y = y0 + ty, x = x0 + tx;
    if (y < L.ny && x < L.nx) U[(long long)y * L.pitch + x] = su[(ty + H) * RX + tx + H];
  }
}

}  // namespace tile
}  // namespace gd
