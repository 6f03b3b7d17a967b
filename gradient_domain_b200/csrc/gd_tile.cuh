// Shared-memory tile kernels for the coarse levels of the V-cycle.
//
// The register-streaming kernels of gd_stream.cuh walk every strip row by row;
// on a small level a launch has too few strips to fill the GPU and each warp
// waits on the latency of its own row chain, so a level costs a fixed 15-30 us
// whatever its size.  Here a CTA instead loads one tile of the level plus a
// halo into shared memory and runs every phase (a red-black half sweep, the
// residual, the restriction or the prolongation) over the whole tile at once,
// with a barrier between phases: all cells of a phase are independent, so the
// CTA's threads work in parallel.
//
// A thread works on groups of four consecutive cells of a row (one 16-byte
// shared-memory access per array, the four cell classes in one word); region
// rows start on 16-byte boundaries because the horizontal halo is kHX = 8
// cells and tiles start on multiples of kTX.  A half sweep that reads
// neighbours leaves the outermost exact ring of the loaded region one cell
// further in, so the down kernel (whose first half sweep, from zero, reads
// only b and is applied while loading) needs 2 S1 + 1 halo rows (2 S1 - 1 for
// the sweeps, one for the residual's neighbours, one for the restriction's
// reach) and the up kernel 2 S2; kHX covers both in x for up to 3 sweeps.
// Cells outside the grid have class 0: they hold zeros and are never updated,
// which is the operator's definition of a missing neighbour.
#pragma once

#include "gd_stream.cuh"

namespace gd {
namespace tile {

// Two tile shapes.  Levels with at least one 32 x 64 tile per SM run those
// tiles on CTAs of 256 threads (throughput).  Smaller levels, where one CTA's
// chain of phases is the launch's duration, run 16 x 32 tiles on CTAs of 384
// threads: every phase is one pass per thread, and the level spreads over four
// times as many SMs, so each SM issues a quarter of the instructions.
constexpr int kTY = 32, kTX = 64;    // cells of a large tile (even: whole coarse cells)
constexpr int kTYs = 16, kTXs = 32;  // cells of a small tile
constexpr int kHX = 8;               // halo columns on each side
constexpr int kThreads = 256, kThreadsSmall = 384;

template <typename T, int S1, int TY = kTY, int TX = kTX>
struct DownT {
  static constexpr int H = 2 * S1 + 1;
  static constexpr int RY = TY + 2 * H, RX = TX + 2 * kHX, N = RY * RX, GX = RX / 4;
  static constexpr size_t smem = (size_t)N * (2 * sizeof(T) + 1) + 16;
};

template <typename T, int S2, int TY = kTY, int TX = kTX>
struct UpT {
  static constexpr int H = 2 * S2;
  static constexpr int RY = TY + 2 * H, RX = TX + 2 * kHX, N = RY * RX, GX = RX / 4;
  static constexpr int CY = RY / 2 + 3, CX = RX / 2 + 3, CN = CY * CX;
  static constexpr size_t smem = (size_t)(2 * N + CN) * sizeof(T) + N + 16;
};

static_assert(kHX % 4 == 0 && kTX % 4 == 0 && kTXs % 4 == 0 && kHX >= 7, "tile geometry");
static_assert(kTY % 2 == 0 && kTYs % 2 == 0, "tiles hold whole coarse cells");
// one group of four cells per thread and phase on small tiles (up to three sweeps)
static_assert((kTYs + 2 * 7) * ((kTXs + 2 * kHX) / 4) <= kThreadsSmall, "small tile threads");

template <typename T>
__device__ __forceinline__ void diag_tables(T *tdiag, T *tdinv, float wall) {
  if (threadIdx.x < 8) {
    const int c = threadIdx.x;
    const double d = c >= 1 && c <= 5 ? class_diag(c, wall) : 1.0;
    tdiag[c] = (T)d;
    tdinv[c] = (c >= 1 && c <= 5 && d > 0.0) ? (T)(1.0 / d) : T(0);
  }
}

// Cells x .. x + 3 of row y (x a multiple of 4), zero outside the grid.
template <typename T>
__device__ __forceinline__ st::V4<T> load_group(const T *A, const LevelInfo &L, int y, int x) {
  if (y < 0 || y >= L.ny || x < 0 || x >= L.nx) return st::zero4<T>();
  const T *p = A + (long long)y * L.pitch + x;
  if (x + 3 < L.nx) return st::ld4(p);
  st::V4<T> r;
#pragma unroll
  for (int j = 0; j < 4; ++j) r.v[j] = (x + j < L.nx) ? p[j] : T(0);
  return r;
}

template <typename T>
__device__ __forceinline__ void store_group(T *A, const LevelInfo &L, int y, int x,
                                            const st::V4<T> &v) {
  if (y >= L.ny || x >= L.nx) return;
  T *p = A + (long long)y * L.pitch + x;
  if (x + 3 < L.nx) {
    st::st4(p, v);
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (x + j < L.nx) p[j] = v.v[j];
  }
}

// One red-black half sweep over the interior rows of an RY x RX region;
// `par0` is the parity of the region corner's grid coordinates.  A cell of one
// colour only reads cells of the other, so every thread gathers the operands
// of all its groups before it writes: the loads of different groups overlap.
template <typename T, int RY, int RX, int NT>
__device__ __forceinline__ void tsweep(T *u, const T *b, const unsigned *c, const T *dinv,
                                       int colour, int par0) {
  constexpr int GX = RX / 4, M = (RY - 2) * GX, IT = (M + NT - 1) / NT;
  int at[IT];
  T v0[IT], v1[IT];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int g = threadIdx.x + it * NT;
    at[it] = -1;
    if (g < M) {
      const int ry = 1 + g / GX, gx = g - (ry - 1) * GX;
      const int i = ry * RX + 4 * gx;
      const st::V4<T> uc = st::ld4(u + i), up = st::ld4(u + i - RX), dn = st::ld4(u + i + RX);
      const st::V4<T> bb = st::ld4(b + i);
      const unsigned cl = c[g + GX];
      if (((colour + par0 + ry) & 1) == 0) {
        const T left = gx > 0 ? u[i - 1] : T(0);
        v0[it] = (bb.v[0] + up.v[0] + dn.v[0] + left + uc.v[1]) * dinv[st::cls(cl, 0)];
        v1[it] = (bb.v[2] + up.v[2] + dn.v[2] + uc.v[1] + uc.v[3]) * dinv[st::cls(cl, 2)];
        at[it] = i;
      } else {
        const T right = gx < GX - 1 ? u[i + 4] : T(0);
        v0[it] = (bb.v[1] + up.v[1] + dn.v[1] + uc.v[0] + uc.v[2]) * dinv[st::cls(cl, 1)];
        v1[it] = (bb.v[3] + up.v[3] + dn.v[3] + uc.v[2] + right) * dinv[st::cls(cl, 3)];
        at[it] = i + 1;
      }
    }
  }
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    if (at[it] >= 0) {
      u[at[it]] = v0[it];
      u[at[it] + 2] = v1[it];
    }
  }
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
// residual, restriction (P^T) into the coarse right-hand side.  Called by the
// whole CTA (NT threads) for an active instance's tile; the CTA's shared
// memory is free on entry and may be reused on return.
template <typename T, int S1, int NT, int TY = kTY, int TX = kTX>
__device__ __forceinline__ void down_tile(const Args<T> &a, const Tile tl, const LevelInfo &L,
                                          const LevelInfo &Lc, unsigned char *smem) {
  using G = DownT<T, S1, TY, TX>;
  constexpr int RY = G::RY, RX = G::RX, H = G::H, N = G::N, GX = G::GX;
  T *sb = reinterpret_cast<T *>(smem);
  T *su = sb + N;
  unsigned *sc = reinterpret_cast<unsigned *>(su + N);
  __shared__ T tdiag[8], tdinv[8];
  diag_tables(tdiag, tdinv, L.wall);
  __syncthreads();
  const int y0 = tl.ty * TY, x0 = tl.tx * TX;
  const int gy0 = y0 - H, gx0 = x0 - kHX;
  const int par0 = (gy0 + gx0) & 1;
  {  // load, applying the first half sweep (colour 0 from zero: u = b / d)
    const T *B = a.arena + L.b_off;
    constexpr int NG = RY * GX, IT = (NG + NT - 1) / NT;
    st::V4<T> bv[IT];
    unsigned cv[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int g = threadIdx.x + it * NT;
      const int ry = g / GX, gx = g - ry * GX;
      const int y = gy0 + ry, x = gx0 + 4 * gx;
      bv[it] = g < NG ? load_group(B, L, y, x) : st::zero4<T>();
      cv[it] = g < NG ? st::row_classes(L, a.codes, y, x) : 0u;
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int g = threadIdx.x + it * NT;
      if (g >= NG) break;
      const int ry = g / GX;
      const int p = (par0 + ry) & 1;  // cells j with (j & 1) == p have colour 0
      st::V4<T> u0;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        u0.v[j] = ((j & 1) == p) ? bv[it].v[j] * tdinv[st::cls(cv[it], j)] : T(0);
      st::st4(sb + 4 * g, bv[it]);  // RX = 4 GX: group g starts at cell 4 g
      st::st4(su + 4 * g, u0);
      sc[g] = cv[it];
    }
  }
  __syncthreads();
  tsweep<T, RY, RX, NT>(su, sb, sc, tdinv, 1, par0);
  for (int s = 1; s < S1; ++s) {
    tsweep<T, RY, RX, NT>(su, sb, sc, tdinv, 0, par0);
    tsweep<T, RY, RX, NT>(su, sb, sc, tdinv, 1, par0);
  }
  {  // the pre-smoothed iterate of the tile, for the up kernel
    T *W = a.arena + L.w_off;
    constexpr int TG = TX / 4, M = TY * TG;
    for (int g = threadIdx.x; g < M; g += NT) {
      const int ty = g / TG, q = g - ty * TG;
      store_group(W, L, y0 + ty, x0 + 4 * q, st::ld4(su + (ty + H) * RX + kHX + 4 * q));
    }
  }
  {  // residual on the tile plus one ring, in place into b (groups 1 .. TX/4 + 2)
    constexpr int QG = TX / 4 + 2, M = (TY + 2) * QG, IT = (M + NT - 1) / NT;
    st::V4<T> res[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int g = threadIdx.x + it * NT;
      res[it] = st::zero4<T>();
      if (g < M) {
        const int qy = g / QG, q = g - qy * QG;
        const int ry = qy + H - 1, gx = q + 1;
        const int i = ry * RX + 4 * gx;
        const st::V4<T> uc = st::ld4(su + i), up = st::ld4(su + i - RX),
                        dn = st::ld4(su + i + RX), bb = st::ld4(sb + i);
        const T left = su[i - 1], right = su[i + 4];
        const unsigned cl = sc[ry * GX + gx];
        const T lf[4] = {left, uc.v[0], uc.v[1], uc.v[2]};
        const T rt[4] = {uc.v[1], uc.v[2], uc.v[3], right};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int k = st::cls(cl, j);
          res[it].v[j] = k ? bb.v[j] - (tdiag[k] * uc.v[j] - (up.v[j] + dn.v[j] + lf[j] + rt[j]))
                           : T(0);
        }
      }
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int g = threadIdx.x + it * NT;
      if (g < M) {
        const int qy = g / QG, q = g - qy * QG;
        st::st4(sb + (qy + H - 1) * RX + 4 * (q + 1), res[it]);
      }
    }
  }
  __syncthreads();
  const bool neu = L.bc == BC_NEU;
  T *Bc = a.arena + Lc.b_off;
  constexpr int CTY = TY / 2, CTX = TX / 2;
  for (int k = threadIdx.x; k < CTY * CTX; k += NT) {
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
// boundaries read zero outside), then S2 post-sweeps, colour 1 first.  Same
// calling convention as down_tile.
template <typename T, int S2, int NT, int TY = kTY, int TX = kTX>
__device__ __forceinline__ void up_tile(const Args<T> &a, const Tile tl, const LevelInfo &L,
                                        const LevelInfo &Lc, unsigned char *smem) {
  using G = UpT<T, S2, TY, TX>;
  constexpr int RY = G::RY, RX = G::RX, H = G::H, N = G::N, GX = G::GX, CX = G::CX;
  T *sb = reinterpret_cast<T *>(smem);
  T *su = sb + N;
  T *se = su + N;
  unsigned *sc = reinterpret_cast<unsigned *>(se + G::CN);
  __shared__ T tdiag[8], tdinv[8];
  diag_tables(tdiag, tdinv, L.wall);
  const int y0 = tl.ty * TY, x0 = tl.tx * TX;
  const int gy0 = y0 - H, gx0 = x0 - kHX;
  const int par0 = (gy0 + gx0) & 1;
  const bool neu = L.bc == BC_NEU;
  // coarse correction around the region, from coarse row / column cy0 / cx0
  const int cy0 = (gy0 >> 1) - 1, cx0 = (gx0 >> 1) - 1;
  {  // every load of a thread is issued before the first is used
    const T *E = a.arena + Lc.u_off;
    const T *B = a.arena + L.b_off;
    const T *W = a.arena + L.w_off;
    constexpr int ITC = (G::CN + NT - 1) / NT;
    constexpr int NG = RY * GX, IT = (NG + NT - 1) / NT;
    T ev[ITC];
    st::V4<T> bv[IT], wv[IT];
    unsigned cv[IT];
#pragma unroll
    for (int it = 0; it < ITC; ++it) {
      const int k = threadIdx.x + it * NT;
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
      const int g = threadIdx.x + it * NT;
      const int ry = g / GX, gx = g - ry * GX;
      const int y = gy0 + ry, x = gx0 + 4 * gx;
      cv[it] = g < NG ? st::row_classes(L, a.codes, y, x) : 0u;
      bv[it] = g < NG ? load_group(B, L, y, x) : st::zero4<T>();
      wv[it] = g < NG ? load_group(W, L, y, x) : st::zero4<T>();
    }
#pragma unroll
    for (int it = 0; it < ITC; ++it) {
      const int k = threadIdx.x + it * NT;
      if (k < G::CN) se[k] = ev[it];
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int g = threadIdx.x + it * NT;
      if (g >= NG) break;
      st::V4<T> w = wv[it];
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (!st::cls(cv[it], j)) w.v[j] = T(0);
      st::st4(sb + 4 * g, bv[it]);  // RX = 4 GX: group g starts at cell 4 g
      st::st4(su + 4 * g, w);
      sc[g] = cv[it];
    }
  }
  __syncthreads();
  {  // u += P e on cells with an unknown (each group reads the coarse values
     // and only its own u)
    constexpr int NG = RY * GX, IT = (NG + NT - 1) / NT;
    st::V4<T> pe[IT];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int g = threadIdx.x + it * NT;
      pe[it] = st::zero4<T>();
      const unsigned cl = g < NG ? sc[g] : 0u;
      if (cl) {
        const int ry = g / GX, gx = g - ry * GX;
        const int y = gy0 + ry;
        const int cy = y >> 1, cy2 = (y & 1) ? cy + 1 : cy - 1;
        // coarse columns x/2 - 1 .. x/2 + 2 of rows cy and cy2 (x = gx0 + 4 gx)
        const T *r1 = se + (cy - cy0) * CX + 2 * gx;
        const T *r2 = se + (cy2 - cy0) * CX + 2 * gx;
        T e1[4], e2[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          e1[k] = r1[k];
          e2[k] = r2[k];
        }
        const T v[4] = {
            (T)0.5625 * e1[1] + (T)0.1875 * (e2[1] + e1[0]) + (T)0.0625 * e2[0],
            (T)0.5625 * e1[1] + (T)0.1875 * (e2[1] + e1[2]) + (T)0.0625 * e2[2],
            (T)0.5625 * e1[2] + (T)0.1875 * (e2[2] + e1[1]) + (T)0.0625 * e2[1],
            (T)0.5625 * e1[2] + (T)0.1875 * (e2[2] + e1[3]) + (T)0.0625 * e2[3]};
#pragma unroll
        for (int j = 0; j < 4; ++j) pe[it].v[j] = st::cls(cl, j) ? v[j] : T(0);
      }
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int g = threadIdx.x + it * NT;
      if (g < NG && sc[g]) {
        st::V4<T> u = st::ld4(su + 4 * g);
#pragma unroll
        for (int j = 0; j < 4; ++j) u.v[j] += pe[it].v[j];
        st::st4(su + 4 * g, u);
      }
    }
  }
  __syncthreads();
  for (int s = 0; s < S2; ++s) {
    tsweep<T, RY, RX, NT>(su, sb, sc, tdinv, 1, par0);
    tsweep<T, RY, RX, NT>(su, sb, sc, tdinv, 0, par0);
  }
  T *U = a.arena + L.u_off;
  constexpr int TG = TX / 4, M = TY * TG;
  for (int g = threadIdx.x; g < M; g += NT) {
    const int ty = g / TG, q = g - ty * TG;
    store_group(U, L, y0 + ty, x0 + 4 * q, st::ld4(su + (ty + H) * RX + kHX + 4 * q));
  }
}

// One launch per level: a CTA per tile.  A level's coarse level is the next
// entry of the level table (levels of an instance are stored finest first), so
// the status word and both descriptors are requested together.
template <typename T, int S1, int NT = kThreads, int TY = kTY, int TX = kTX>
__global__ void __launch_bounds__(NT) k_down_t(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  const LevelInfo L = a.lv[tl.level];
  const LevelInfo Lc = a.lv[tl.level + 1];
  dep_enter();
  if (a.st[tl.inst].status != GD_ACTIVE) return;
  extern __shared__ __align__(16) unsigned char smem[];
  down_tile<T, S1, NT, TY, TX>(a, tl, L, Lc, smem);
}

template <typename T, int S2, int NT = kThreads, int TY = kTY, int TX = kTX>
__global__ void __launch_bounds__(NT) k_up_t(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  const LevelInfo L = a.lv[tl.level];
  const LevelInfo Lc = a.lv[tl.level + 1];
  dep_enter();
  if (a.st[tl.inst].status != GD_ACTIVE) return;
  extern __shared__ __align__(16) unsigned char smem[];
  up_tile<T, S2, NT, TY, TX>(a, tl, L, Lc, smem);
}

}  // namespace tile
}  // namespace gd
