// Register-streaming kernels of the batched cell-centred MGPCG.
//
// Every kernel here works on vertical strips.  A warp owns 128 consecutive
// columns (4 per lane, one 128-bit vector for FP32) and walks down its strip
// one row at a time; the rows it still needs live in small register windows,
// vertical neighbours are window entries and horizontal neighbours at lane
// boundaries come from warp shuffles.  Nothing is staged in shared memory.
//
// The smoothing kernels pipeline the red-black half sweeps: when row y is
// loaded, half sweep 1 runs on row y, half sweep 2 on row y-1, ..., so after
// the last stage a row has seen every sweep and the residual / restriction /
// prolongation / output stages follow further up the window.  Each half sweep
// widens the set of cells whose value depends on data outside the strip by
// one column, so the outermost lanes of a warp ("halo lanes") compute values
// that are never written; rows at the top of a strip are likewise warm-up
// rows.  Halo lanes and warm-up rows are the only redundant work.
#pragma once

#include <cuda_pipeline.h>

#include "gd_bulk.cuh"
#include "gd_mg_kernels.cuh"

namespace gd {
namespace st {

constexpr int kLanes = 32;
constexpr int kWarps = 4;          // warps per CTA of the Krylov and refresh kernels
constexpr int kThreads = kWarps * kLanes;
// The down / up kernels run one warp (one strip) per CTA: the block scheduler
// then spreads a launch's strips evenly over the SMs (a launch of four-warp
// CTAs that fits one wave left some SMs one CTA short of others).
constexpr int kSWarps = 1;
constexpr int kSThreads = kSWarps * kLanes;
// ... except the level-0 up kernel, whose CTAs each add an r.z partial and
// take a ticket for the last-CTA reduction: four warps per CTA keep those
// fences and atomics four times fewer (one warp per CTA was measured slower).
template <bool LEVEL0>
struct UpCta {
  static constexpr int W = LEVEL0 ? 4 : 1;
  static constexpr int NT = W * kLanes;
};
constexpr int kKrylovRows = 16;    // rows per warp in the Krylov kernels
constexpr int kKrylovCols = 128;   // columns per warp (and per CTA)

template <typename T>
struct V4 {
  T v[4];
};

template <typename T>
__device__ __forceinline__ V4<T> ld4(const T *p) {
  V4<T> r;
  if constexpr (sizeof(T) == 4) {
    const float4 q = *reinterpret_cast<const float4 *>(p);
    r.v[0] = q.x; r.v[1] = q.y; r.v[2] = q.z; r.v[3] = q.w;
  } else {
    const double2 a = *reinterpret_cast<const double2 *>(p);
    const double2 b = *reinterpret_cast<const double2 *>(p + 2);
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = b.x; r.v[3] = b.y;
  }
  return r;
}

template <typename T>
__device__ __forceinline__ void st4(T *p, const V4<T> &r) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
  } else {
    *reinterpret_cast<double2 *>(p) = make_double2(r.v[0], r.v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(r.v[2], r.v[3]);
  }
}

template <typename T>
__device__ __forceinline__ V4<T> zero4() {
  V4<T> r;
#pragma unroll
  for (int j = 0; j < 4; ++j) r.v[j] = T(0);
  return r;
}

// Classes of the 4 cells x0..x0+3 of row y, packed one byte each.
__device__ __forceinline__ unsigned row_classes(const LevelInfo &L, const unsigned char *codes,
                                                int y, int x0) {
  if (y < 0 || y >= L.ny || x0 >= L.nx || x0 + 3 < 0) return 0u;
  if (L.code_off >= 0) {
    if (x0 < 0) return 0u;  // x0 is a multiple of 4: a lane is wholly left of the grid or in it
    return *reinterpret_cast<const unsigned *>(codes + L.code_off + (long long)y * L.pitch + x0);
  }
  const int wy = (y == 0) + (y == L.ny - 1);
  unsigned packed = 0u;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int x = x0 + j;
    if (x >= 0 && x < L.nx) {
      const unsigned c = 1u + wy + (x == 0) + (x == L.nx - 1);
      packed |= c << (8 * j);
    }
  }
  return packed;
}

__device__ __forceinline__ int cls(unsigned packed, int j) { return (packed >> (8 * j)) & 0xff; }

template <typename T>
__device__ __forceinline__ T shfl_up1(T v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <typename T>
__device__ __forceinline__ T shfl_dn1(T v) { return __shfl_down_sync(0xffffffffu, v, 1); }

// Per-lane ring of RS row slices (4 elements each) in shared memory, filled
// with cp.async so that RS - 1 rows per lane are in flight while the current
// row is processed.  A lane only ever reads back the bytes it copied itself,
// so a per-thread wait_group is the only synchronisation.  Slot s of a lane
// sits at ((s * kThreads) + threadIdx.x) * 4 elements: a warp touches 512
// (FP32) contiguous bytes per slot, free of bank conflicts.
constexpr int kRing = 8;

template <typename T, int NT = kThreads>
struct Ring {
  T *base;
  __device__ __forceinline__ explicit Ring(T *smem) : base(smem + threadIdx.x * 4) {}
  __device__ __forceinline__ T *slot(int s) const { return base + (s & (kRing - 1)) * NT * 4; }
  // Copy A[y, x0 .. x0 + 3] into slot s, or zeros when the row or lane is outside the grid.
  __device__ __forceinline__ void issue(int s, const T *A, const LevelInfo &L, int y, int x0) const {
    const bool ok = y >= 0 && y < L.ny && x0 >= 0 && x0 < L.nx;
    const T *src = ok ? A + (long long)y * L.pitch + x0 : A;
    T *dst = slot(s);
    constexpr int chunks = (int)(4 * sizeof(T) / 16);
#pragma unroll
    for (int k = 0; k < chunks; ++k)
      __pipeline_memcpy_async(dst + k * (16 / sizeof(T)), src + (ok ? k * (16 / sizeof(T)) : 0),
                              16, ok ? 0 : 16);
  }
  __device__ __forceinline__ V4<T> read(int s) const { return ld4(slot(s)); }
};

// Per-lane ring of packed cell classes of masked levels (4 bytes per row).
template <int NT = kThreads>
struct CodeRing {
  unsigned *base;
  __device__ __forceinline__ explicit CodeRing(unsigned *smem) : base(smem + threadIdx.x) {}
  __device__ __forceinline__ unsigned *slot(int s) const {
    return base + (s & (kRing - 1)) * NT;
  }
  __device__ __forceinline__ void issue(int s, const LevelInfo &L, const unsigned char *codes,
                                        int y, int x0) const {
    const bool ok = y >= 0 && y < L.ny && x0 >= 0 && x0 < L.nx;
    const unsigned char *src = ok ? codes + L.code_off + (long long)y * L.pitch + x0 : codes;
    __pipeline_memcpy_async(slot(s), src, 4, ok ? 0 : 4);
  }
  __device__ __forceinline__ unsigned read(int s) const { return *slot(s); }
};

// Per-lane ring of one element per row: the column just outside the warp
// (left of lane 0, right of lane 31), so edge values arrive with their row.
template <typename T>
struct EdgeRing {
  T *base;
  __device__ __forceinline__ explicit EdgeRing(T *smem) : base(smem + threadIdx.x) {}
  __device__ __forceinline__ T *slot(int s) const { return base + (s & (kRing - 1)) * kThreads; }
  __device__ __forceinline__ void issue(int s, const T *A, const LevelInfo &L, int y, int x) const {
    const bool ok = y >= 0 && y < L.ny && x >= 0 && x < L.nx;
    __pipeline_memcpy_async(slot(s), ok ? A + (long long)y * L.pitch + x : A, sizeof(T),
                            ok ? 0 : sizeof(T));
  }
  __device__ __forceinline__ T read(int s) const { return *slot(s); }
};

// Dynamic shared memory of the streaming kernels (rings).
template <typename T, int NT = kThreads>
constexpr size_t ring_bytes() { return (size_t)kRing * NT * 4 * sizeof(T); }
template <typename T, int NT = kSThreads>
constexpr size_t level_smem() {
  return 2 * ring_bytes<T, NT>() + (size_t)kRing * NT * 4;
}
template <typename T>
constexpr size_t edge_bytes() { return (size_t)kRing * kThreads * sizeof(T); }

template <typename T>
constexpr size_t pupdate_smem() { return 2 * ring_bytes<T>() + 2 * edge_bytes<T>(); }
template <typename T>
constexpr size_t cgupdate_smem() { return 3 * ring_bytes<T>() + edge_bytes<T>(); }

// Lanes whose output is exact for a dependency radius of R columns.
template <int R>
struct Halo {
  static constexpr int HL = (R + 3) / 4;
  static constexpr int OUT_LANES = kLanes - 2 * HL;
  static constexpr int OW = 4 * OUT_LANES;  // output columns per strip
};

// ---------------------------------------------------------------------------
// Shared by the smoothing kernels.
//
// Diagonal entries by cell class, in shared memory: one LDS replaces a chain
// of compares in the general path.  Strips that touch no grid boundary and no
// mask ("interior" strips, almost all of them on large rectangles) skip the
// classes altogether and use the interior diagonal as a constant.
template <typename T>
struct ClassTable {
  T d[8], inv[8];
};

template <typename T>
__device__ __forceinline__ void fill_table(ClassTable<T> &t, float wall) {
  if (threadIdx.x < 8) {
    const int c = threadIdx.x;
    const double dd = (c >= 1 && c <= 5) ? 4.0 - (double)(c - 1) * (1.0 - (double)wall) : 0.0;
    t.d[c] = (T)dd;
    t.inv[c] = dd > 0.0 ? (T)(1.0 / dd) : T(0);
  }
  __syncthreads();
}

template <typename T, bool INT>
struct Coef {
  const ClassTable<T> &tab;
  T d_int, inv_int;
  __device__ __forceinline__ T inv(unsigned c, int j) const {
    if constexpr (INT) return inv_int;
    else return tab.inv[cls(c, j)];
  }
  __device__ __forceinline__ T d(unsigned c, int j) const {
    if constexpr (INT) return d_int;
    else return tab.d[cls(c, j)];
  }
  __device__ __forceinline__ bool on(unsigned c, int j) const {
    if constexpr (INT) return true;
    else return cls(c, j) != 0;
  }
};

// ---------------------------------------------------------------------------
// Arithmetic of the smoothing kernels.  Every cell value is one fixed sequence
// of round-to-nearest operations (nothing left to the compiler's contraction),
// written once per cell for the general strips (FP32 and FP64) and once per
// pair of cells for the FP32 interior strips, which evaluate it with the paired
// FP32 instructions of sm_100 (two cells per instruction).  Both give the same
// bits, so which strip computes a cell never changes its value.
//
// A lane's four columns x0 .. x0+3 (x0 a multiple of 4) are held by the
// interior strips as two pairs, E = (v0, v2) and O = (v1, v3): the cells of a
// pair have the same colour on every row, so a red-black half sweep updates
// exactly one pair of each lane.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// Sum of a cell's four neighbours and its right-hand side: nbA is the
// horizontal neighbour inside the lane's four columns on the side of the
// cell's pair partner (the right one for even columns, the left one for odd
// columns), nbB the other one; dn, the row a pipelined sweep updated last, is
// added last so that it ends the dependency chain.
template <typename T>
__device__ __forceinline__ T nsum1(T up, T nbA, T nbB, T b, T dn) {
  return add_rn(add_rn(add_rn(add_rn(up, nbA), nbB), b), dn);
}
// Prolongation of a coarse correction onto a fine cell: w + 3/4 near + 1/4 far.
template <typename T>
__device__ __forceinline__ T prolong1(T w, T near, T far) {
  return fma_rn(T(0.25), far, fma_rn(T(0.75), near, w));
}
// Full weighting along one axis: 1/4 a + 3/4 b + 3/4 c + 1/4 d.
template <typename T>
__device__ __forceinline__ T weigh1(T a, T b, T c, T d) {
  return fma_rn(T(0.25), d, fma_rn(T(0.75), c, fma_rn(T(0.75), b, mul_rn(T(0.25), a))));
}
// Linear interpolation 3/4 near + 1/4 far.
template <typename T>
__device__ __forceinline__ T interp1(T near, T far) {
  return fma_rn(T(0.25), far, mul_rn(T(0.75), near));
}
// Dot product of a lane's four cells.
template <typename T>
__device__ __forceinline__ T dot1(const V4<T> &b, const V4<T> &v) {
  return add_rn(fma_rn(b.v[1], v.v[1], mul_rn(b.v[0], v.v[0])),
                fma_rn(b.v[3], v.v[3], mul_rn(b.v[2], v.v[2])));
}

// Paired forms (element-wise the scalar ones above).
struct P4 {
  float2 e, o;  // (v0, v2), (v1, v3)
};
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 nsum2(float2 up, float2 nbA, float2 nbB, float2 b, float2 dn) {
  return add2(add2(add2(add2(up, nbA), nbB), b), dn);
}
__device__ __forceinline__ P4 split4(const float4 &q) {
  return P4{make_float2(q.x, q.z), make_float2(q.y, q.w)};
}
__device__ __forceinline__ float4 join4(const P4 &p) {
  return make_float4(p.e.x, p.o.x, p.e.y, p.o.y);
}
__device__ __forceinline__ P4 zero_p4() { return P4{make_float2(0.f, 0.f), make_float2(0.f, 0.f)}; }

// Half sweep of the even pair (J0 = 0) or the odd pair (J0 = 1) of a row of an
// interior strip, diagonal inverse `inv` for every cell.
template <int J0>
__device__ __forceinline__ void psweep(P4 &u, const P4 &up, const P4 &dn, const P4 &b, float2 inv) {
  if constexpr (J0 == 0) {
    const float left = shfl_up1(u.o.y);
    u.e = mul2(nsum2(up.e, u.o, make_float2(left, u.o.x), b.e, dn.e), inv);
  } else {
    const float right = shfl_dn1(u.e.x);
    u.o = mul2(nsum2(up.o, u.e, make_float2(u.e.y, right), b.o, dn.o), inv);
  }
}

// Half sweep on one row; J0 (first updated cell of the lane) is compile-time.
template <int J0, typename T, bool INT>
__device__ __forceinline__ void hsweep(V4<T> &u, const V4<T> &up, const V4<T> &dn,
                                       const V4<T> &b, unsigned c, const Coef<T, INT> &K) {
  if constexpr (J0 == 0) {
    const T left = shfl_up1(u.v[3]);
    u.v[0] = mul_rn(nsum1(up.v[0], u.v[1], left, b.v[0], dn.v[0]), K.inv(c, 0));
    u.v[2] = mul_rn(nsum1(up.v[2], u.v[3], u.v[1], b.v[2], dn.v[2]), K.inv(c, 2));
  } else {
    const T right = shfl_dn1(u.v[0]);
    u.v[1] = mul_rn(nsum1(up.v[1], u.v[0], u.v[2], b.v[1], dn.v[1]), K.inv(c, 1));
    u.v[3] = mul_rn(nsum1(up.v[3], u.v[2], right, b.v[3], dn.v[3]), K.inv(c, 3));
  }
}

template <int J0, typename T, bool INT>
__device__ __forceinline__ void hsweep_zero(V4<T> &u, const V4<T> &b, unsigned c,
                                            const Coef<T, INT> &K) {
#pragma unroll
  for (int j = 0; j < 4; ++j) u.v[j] = ((j & 1) == J0) ? mul_rn(b.v[j], K.inv(c, j)) : T(0);
}

// A u on a row (zero where there is no unknown).
template <typename T, bool INT>
__device__ __forceinline__ V4<T> arow(const V4<T> &u, const V4<T> &up, const V4<T> &dn, T left,
                                      T right, unsigned c, const Coef<T, INT> &K) {
  V4<T> r;
  const T lf[4] = {left, u.v[0], u.v[1], u.v[2]};
  const T rt[4] = {u.v[1], u.v[2], u.v[3], right};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const T v = K.d(c, j) * u.v[j] - (up.v[j] + dn.v[j] + lf[j] + rt[j]);
    r.v[j] = K.on(c, j) ? v : T(0);
  }
  return r;
}

// Window slot of "row y - k" at unrolled phase PH of a circular window of U rows.
template <int U>
__host__ __device__ constexpr int wslot(int ph, int k) {
  return ((ph - k) % U + U) % U;
}

// ---------------------------------------------------------------------------
// Down: S1 pre-sweeps from zero, residual, restriction (P^T) of one strip.
// Radius: 2 S1 - 1 (sweeps) + 1 (residual) + 1 (restriction) columns.
template <typename T, int S1>
struct DownGeom {
  using H = Halo<2 * S1 + 1>;
  static constexpr int U = 2 * S1 + 2;  // rows in every circular window (even)
};

template <typename T, int S1, bool INT>
__device__ __forceinline__ void down_strip(const Args<T> &a, const LevelInfo &L,
                                           const LevelInfo &Lc, const ClassTable<T> &tab,
                                           int x0, bool out_lane, int y_start, int y_last,
                                           int y_out0, int y_out1, int I_begin, int I_end,
                                           unsigned char *smem) {
  constexpr int U = DownGeom<T, S1>::U;
  constexpr int K = 2 * S1;  // window index of the residual row
  const Coef<T, INT> C{tab, tab.d[1], tab.inv[1]};
  const bool neu = L.bc == BC_NEU;
  const bool masked = L.code_off >= 0;
  const T *B = a.arena + L.b_off;
  T *Bc = a.arena + Lc.b_off;
  T *Wp = a.arena + L.w_off;
  const bool store_lane = out_lane && x0 >= 0 && x0 < L.nx;
  const Ring<T, kSThreads> ring(reinterpret_cast<T *>(smem));
  const CodeRing<kSThreads> cring(reinterpret_cast<unsigned *>(smem + 2 * ring_bytes<T, kSThreads>()));
  V4<T> Bw[U], Uw[U], F[U];
  unsigned Cw[U];
#pragma unroll
  for (int k = 0; k < U; ++k) { Bw[k] = zero4<T>(); Uw[k] = zero4<T>(); F[k] = zero4<T>(); Cw[k] = 0u; }
  const int m_left = -1 - x0;
  const int m_right = L.nx - x0;
  for (int q = 0; q < kRing - 1; ++q) {
    ring.issue(q, B, L, y_start + q, x0);
    if (!INT && masked) cring.issue(q, L, a.codes, y_start + q, x0);
    __pipeline_commit();
  }
  for (int base = y_start; base <= y_last; base += U) {
#pragma unroll
    for (int ph = 0; ph < U; ++ph) {
      const int y = base + ph;
      if (y > y_last) break;
      const int step = y - y_start;
      __pipeline_wait_prior(kRing - 2);
      Bw[wslot<U>(ph, 0)] = ring.read(step);
      if (!INT) Cw[wslot<U>(ph, 0)] = masked ? cring.read(step) : row_classes(L, nullptr, y, x0);
      if (y + kRing - 1 <= y_last) {  // no copy of rows past the strip
        ring.issue(step + kRing - 1, B, L, y + kRing - 1, x0);
        if (!INT && masked) cring.issue(step + kRing - 1, L, a.codes, y + kRing - 1, x0);
      }
      __pipeline_commit();
      // y_start is even, so the parity of y is the parity of ph
      if ((ph & 1) == 0)
        hsweep_zero<0, T, INT>(Uw[wslot<U>(ph, 0)], Bw[wslot<U>(ph, 0)], Cw[wslot<U>(ph, 0)], C);
      else
        hsweep_zero<1, T, INT>(Uw[wslot<U>(ph, 0)], Bw[wslot<U>(ph, 0)], Cw[wslot<U>(ph, 0)], C);
#pragma unroll
      for (int h = 2; h <= 2 * S1; ++h) {
        const int k = h - 1;
        if (((h - 1 + ph - k) & 1) == 0)
          hsweep<0, T, INT>(Uw[wslot<U>(ph, k)], Uw[wslot<U>(ph, k + 1)], Uw[wslot<U>(ph, k - 1)],
                            Bw[wslot<U>(ph, k)], Cw[wslot<U>(ph, k)], C);
        else
          hsweep<1, T, INT>(Uw[wslot<U>(ph, k)], Uw[wslot<U>(ph, k + 1)], Uw[wslot<U>(ph, k - 1)],
                            Bw[wslot<U>(ph, k)], Cw[wslot<U>(ph, k)], C);
      }
      {  // row y - (2 S1 - 1) has seen every pre-sweep: keep it for the up kernel
        constexpr int KP = 2 * S1 - 1;
        const int yw = y - KP;
        if (yw >= y_out0 && yw < y_out1 && store_lane) {
          const V4<T> &v = Uw[wslot<U>(ph, KP)];
          T *dst = Wp + (long long)yw * L.pitch + x0;
          if (x0 + 3 < L.nx) {
            st4(dst, v);
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (x0 + j < L.nx) dst[j] = v.v[j];
          }
        }
      }
      // residual of row yr = y - 2 S1
      const int yr = y - K;
      const V4<T> &uK = Uw[wslot<U>(ph, K)];
      const T left = shfl_up1(uK.v[3]);
      const T right = shfl_dn1(uK.v[0]);
      const unsigned cK = Cw[wslot<U>(ph, K)];
      const V4<T> &bK = Bw[wslot<U>(ph, K)];
      const V4<T> &upK = Uw[wslot<U>(ph, K + 1)], &dnK = Uw[wslot<U>(ph, K - 1)];
      const T lf[4] = {left, uK.v[0], uK.v[1], uK.v[2]};
      const T rt[4] = {uK.v[1], uK.v[2], uK.v[3], right};
      V4<T> res;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        // b - A u = (b + neighbours) - d u, neighbours summed as in the sweeps
        const T s = (j & 1) ? nsum1(upK.v[j], lf[j], rt[j], bK.v[j], dnK.v[j])
                            : nsum1(upK.v[j], rt[j], lf[j], bK.v[j], dnK.v[j]);
        res.v[j] = C.on(cK, j) ? fma_rn(-C.d(cK, j), uK.v[j], s) : T(0);
      }
      T e[6];
      e[0] = shfl_up1(res.v[3]);
      e[1] = res.v[0]; e[2] = res.v[1]; e[3] = res.v[2]; e[4] = res.v[3];
      e[5] = shfl_dn1(res.v[0]);
      if (!INT && neu) {
        if (m_left == -1) e[0] = e[1];
        if (!(L.nx & 1)) {
#pragma unroll
          for (int m = 0; m <= 4; ++m)
            if (m == m_right) e[m + 1] = e[m];
        }
      }
      V4<T> &Fr = F[wslot<U>(ph, K)];
      Fr.v[0] = weigh1(e[0], e[1], e[2], e[3]);
      Fr.v[1] = weigh1(e[2], e[3], e[4], e[5]);
      // coarse row I = yr / 2 - 1 from residual rows 2I-1 .. 2I+2 (yr even <=> ph even)
      if ((ph & 1) == 0) {
        const int I = (yr >> 1) - 1;
        if (I >= I_begin && I < I_end) {
          T rows[4][2];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            rows[q][0] = F[wslot<U>(ph, K + 3 - q)].v[0];
            rows[q][1] = F[wslot<U>(ph, K + 3 - q)].v[1];
          }
          if (!INT && neu) {
            if (I == 0) { rows[0][0] = rows[1][0]; rows[0][1] = rows[1][1]; }
            if (!(L.ny & 1)) {
#pragma unroll
              for (int q = 1; q < 4; ++q)
                if (2 * I - 1 + q == L.ny) { rows[q][0] = rows[q - 1][0]; rows[q][1] = rows[q - 1][1]; }
            }
          }
          if (out_lane) {
            const int J0 = x0 >> 1;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const int J = J0 + q;
              if (J >= 0 && J < Lc.nx) {
                T v = weigh1(rows[0][q], rows[1][q], rows[2][q], rows[3][q]);
                if (!INT && Lc.code_off >= 0 && !a.codes[Lc.code_off + (long long)I * Lc.pitch + J])
                  v = T(0);
                Bc[(long long)I * Lc.pitch + J] = v;
              }
            }
          }
        }
      }
    }
  }
  __pipeline_wait_prior(0);  // no copy may land after this warp's shared memory is released
}

// Phases of one unrolled pass of the interior strips: a multiple of the window
// length U and at least 6, so that the ring slot (P slots, P - 1 rows in
// flight per lane) and every window and coarse slot is a compile-time index.
template <int U>
struct FastGeom {
  static constexpr int P = U >= 6 ? U : 2 * U;
  // Ring slots per array (P - 1 rows in flight per lane; 2P slots, the passes
  // alternating between the two halves, was measured no faster).
  static constexpr int R = P;
  static_assert(P % U == 0 && P % 2 == 0 && (R == P || R == 2 * P), "interior strip pass");
};

// Dynamic shared memory of the down / up kernels: the general strips' rings or
// the fast FP32 strips' rings, whichever is larger (ANY), or the fast strips'
// alone.
// Coarse-row ring of the fast up strips: per slot 8 bytes per lane (the lane's
// two coarse columns) and 8 bytes per warp (the columns just outside it).
template <int R, int NT>
constexpr size_t coarse_ring_bytes() { return (size_t)R * (NT * 8 + (NT / kLanes) * 8); }

// The up kernels stream two arrays and the coarse rows, the down kernels one
// array; NT threads per CTA.
template <typename T, int S, bool UP, bool ANY = true, int NT = kSThreads>
constexpr size_t strip_smem() {
  constexpr int R = FastGeom<2 * S + 2>::R;
  const size_t fast = sizeof(T) != 4 ? 0
                      : UP       ? (size_t)2 * R * NT * 16 + coarse_ring_bytes<R, NT>()
                                 : (size_t)R * NT * 16;
  if (!ANY) return fast;
  // the masked form adds a ring of packed row classes (4 bytes per lane and row)
  const size_t mask = sizeof(T) == 4 ? fast + (size_t)R * NT * 4 : 0;
  return level_smem<T, NT>() > mask ? level_smem<T, NT>() : mask;
}

// Per-lane constants of the fast strips on rectangle levels in any position
// (RECT): which of the lane's four columns are in the grid and how many walls
// each has, and the diagonal inverse and negated diagonal of its cells in rows
// without a wall, as same-colour pairs.  Rows with walls (1, or 2 on a level
// one row high) look their cells' values up in the class table; rows outside
// the grid (kind 3) have no unknowns.  Values come from the class table, as in
// the general strips.
struct LaneRect {
  P4 inv0, negd0;
  unsigned on;  // bit j: column x0 + j is in the grid
  unsigned wx;  // bits 2j, 2j + 1: walls of column x0 + j
};

__device__ __forceinline__ LaneRect lane_rect(const LevelInfo &L, const ClassTable<float> &tab,
                                              int x0) {
  LaneRect r;
  r.on = 0u;
  r.wx = 0u;
  float iv[4], nd[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int x = x0 + j;
    const bool in = x >= 0 && x < L.nx;
    const int wx = (x == 0) + (x == L.nx - 1);
    if (in) r.on |= 1u << j;
    r.wx |= (unsigned)wx << (2 * j);
    const int c = in ? 1 + wx : 0;
    iv[j] = tab.inv[c];
    nd[j] = -tab.d[c];
  }
  r.inv0 = P4{make_float2(iv[0], iv[2]), make_float2(iv[1], iv[3])};
  r.negd0 = P4{make_float2(nd[0], nd[2]), make_float2(nd[1], nd[3])};
  return r;
}

// Diagonal inverse (NEG = false) or negated diagonal (NEG = true) of the lane's
// cells in a row of kind `kind`.
template <bool NEG>
__device__ __forceinline__ P4 rect_diag(const LaneRect &lr, const ClassTable<float> &tab,
                                        int kind) {
  if (kind == 0) return NEG ? lr.negd0 : lr.inv0;
  float v[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = (kind < 3 && ((lr.on >> j) & 1u)) ? 1 + kind + (int)((lr.wx >> (2 * j)) & 3u) : 0;
    v[j] = NEG ? -tab.d[c] : tab.inv[c];
  }
  return P4{make_float2(v[0], v[2]), make_float2(v[1], v[3])};
}

// Kind of row y: walls (0, 1, 2), or 3 outside the grid.
__device__ __forceinline__ int row_kind(const LevelInfo &L, int y) {
  return (y < 0 || y >= L.ny) ? 3 : (y == 0) + (y == L.ny - 1);
}

// Zero the cells of a row that have no unknown (rows outside the grid, columns
// outside it).
__device__ __forceinline__ P4 mask_on(const P4 &v, unsigned on, int kind) {
  if (kind == 3) return zero_p4();
  return P4{make_float2((on & 1u) ? v.e.x : 0.f, (on & 4u) ? v.e.y : 0.f),
            make_float2((on & 2u) ? v.o.x : 0.f, (on & 8u) ? v.o.y : 0.f)};
}

// Masked levels (MASK): the classes of a lane's four cells come packed from the
// level's class bytes, one 32-bit word per row; diagonal inverse (NEG = false)
// or negated diagonal (NEG = true) of the four cells as same-colour pairs, and
// the row with its cells of class 0 (no unknown) zeroed.
template <bool NEG>
__device__ __forceinline__ P4 mask_diag(const ClassTable<float> &tab, unsigned c) {
  float v[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) v[j] = NEG ? -tab.d[cls(c, j)] : tab.inv[cls(c, j)];
  return P4{make_float2(v[0], v[2]), make_float2(v[1], v[3])};
}
__device__ __forceinline__ P4 mask_cls(const P4 &v, unsigned c) {
  return P4{make_float2(cls(c, 0) ? v.e.x : 0.f, cls(c, 2) ? v.e.y : 0.f),
            make_float2(cls(c, 1) ? v.o.x : 0.f, cls(c, 3) ? v.o.y : 0.f)};
}

// Down on an FP32 strip of an unmasked level whose next level is unmasked: the
// same cells as down_strip<float, S1, INT>, bit for bit, with ring slots and
// window slots fixed per unrolled phase, running row offsets and the
// arithmetic on same-colour cell pairs.  RECT = false: every row and column
// the strip loads is an interior cell (no walls, no bounds tests); RECT = true:
// any strip of a rectangle level (copies outside the grid are zero-filled,
// walls take their cells' diagonals, Neumann restriction mirrors its ghosts);
// MASK = true (with RECT): a masked level, every row's classes copied from its
// class bytes through a ring of their own (the same cells as the general
// masked strips, bit for bit).
template <int S1, bool RECT, bool MASK = false>
__device__ __forceinline__ void down_strip_fast(const Args<float> &a, const LevelInfo &L,
                                                const LevelInfo &Lc, const ClassTable<float> &tab,
                                                int x0, bool out_lane, int y_start, int y_last,
                                                int y_out0, int y_out1, int I_begin, int I_end,
                                                unsigned char *smem) {
  constexpr int U = DownGeom<float, S1>::U;
  constexpr int P = FastGeom<U>::P, R = FastGeom<U>::R;
  constexpr int K = 2 * S1;       // window index of the residual row
  constexpr int KP = 2 * S1 - 1;  // window index of the row written as w
  const float2 q25 = splat2(0.25f), q75 = splat2(0.75f);
  const float *B = a.arena + L.b_off;
  float *Bc = a.arena + Lc.b_off;
  float *Wp = a.arena + L.w_off + x0;
  const int pitch = L.pitch;
  float *ring = reinterpret_cast<float *>(smem) + threadIdx.x * 4;
  constexpr int kSlot = kSThreads * 4;  // floats between two slots of a lane
  // interior: one diagonal for every cell
  const P4 inv_i{splat2(tab.inv[1]), splat2(tab.inv[1])};
  const float2 negd_i = splat2(-tab.d[1]);
  LaneRect lr;
  bool lane_in = true, full = true, neu = false;
  int J0 = x0 >> 1;  // x0 is a multiple of 4, so this is exact for negative x0 too
  bool st0 = true, st1 = true;  // coarse columns J0, J0 + 1 are in the coarse grid
  // the warp's 128 columns are all interior columns (no wall, none outside)
  const int xl = x0 - 4 * (int)(threadIdx.x & 31);
  const bool cols_plain = xl >= 1 && xl + 127 <= L.nx - 2;
  if constexpr (RECT) {
    if constexpr (!MASK) lr = lane_rect(L, tab, x0);
    lane_in = x0 >= 0 && x0 < L.nx;
    full = x0 + 3 < L.nx;
    neu = L.bc == BC_NEU;
    st0 = J0 >= 0 && J0 < Lc.nx;
    st1 = J0 + 1 >= 0 && J0 + 1 < Lc.nx;
  }
  // MASK: the class bytes (row pitch `pitch`) and their ring, after the b ring
  const unsigned char *codes = a.codes + (MASK ? L.code_off : 0);
  unsigned *cring = reinterpret_cast<unsigned *>(smem + (size_t)R * kSlot * 4) + threadIdx.x;
  P4 Bw[U], Uw[U];
  float2 F[U];
  int Kw[U];       // row kinds of the window rows (RECT)
  unsigned Cw[U];  // packed classes of the window rows (MASK)
#pragma unroll
  for (int k = 0; k < U; ++k) {
    Bw[k] = zero_p4(); Uw[k] = zero_p4(); F[k] = make_float2(0.f, 0.f); Kw[k] = 3; Cw[k] = 0u;
  }
  auto issue = [&](float *dst, int y, int gofs) {
    if constexpr (RECT) {
      const bool ok = lane_in && y >= 0 && y < L.ny;
      __pipeline_memcpy_async(dst, ok ? B + gofs : B, 16, ok ? 0 : 16);
      if constexpr (MASK) {
        unsigned *cdst = cring + (dst - ring) / 4;  // the same slot of the class ring
        __pipeline_memcpy_async(cdst, ok ? codes + gofs : codes, 4, ok ? 0 : 4);
      }
    } else {
      __pipeline_memcpy_async(dst, B + gofs, 16);
    }
  };
  int gofs = y_start * pitch + x0;  // row offset of the next row to copy
#pragma unroll
  for (int q = 0; q < R - 1; ++q) {
    issue(ring + q * kSlot, y_start + q, gofs);
    __pipeline_commit();
    gofs += pitch;
  }
  int wofs = (y_start - KP) * pitch;  // row offset of the w row written this step
  int half = 0;  // ring slot of this pass's first row (0 or P when R == 2P)
  for (int base = y_start; base <= y_last; base += P) {
    float *cur = ring + half * kSlot;
    float *prev = ring + (R == P ? 0 : (half ^ P)) * kSlot;  // half the slot before ph = 0 is in
#pragma unroll
    for (int ph = 0; ph < P; ++ph) {
      const int y = base + ph;
      if (y > y_last) break;
      __pipeline_wait_prior(R - 2);
      const float4 qb = *reinterpret_cast<const float4 *>(cur + ph * kSlot);
      if (y + R - 1 <= y_last)  // no copy of rows past the strip; the slot read one step ago
        issue(ph > 0 ? cur + (ph - 1) * kSlot : prev + (P - 1) * kSlot, y + R - 1, gofs);
      __pipeline_commit();
      gofs += pitch;
      P4 &b0 = Bw[wslot<U>(ph, 0)];
      b0 = split4(qb);
      if constexpr (MASK) Cw[wslot<U>(ph, 0)] = cring[(cur - ring) / 4 + ph * kSThreads];
      else if constexpr (RECT) Kw[wslot<U>(ph, 0)] = row_kind(L, y);
      // rectangle strips: every row the step touches (y - U + 1 .. y) has no wall
      // and is in the grid (kv = 0, per-lane constants), or some row is special
      // (kv = 1, per-row kinds); one copy runs, chosen by a warp-uniform branch
      // (masked levels: always the per-row classes)
      const bool rows_plain = MASK ? false : !RECT || (y - (U - 1) >= 1 && y <= L.ny - 2);
#pragma unroll
      for (int kv = MASK ? 1 : 0; kv < (RECT ? 2 : 1); ++kv) {
        if ((kv == 1) == rows_plain) continue;
        const bool kinds = kv == 1;
        auto inv_of = [&](int k) -> P4 {
          if constexpr (MASK) return mask_diag<false>(tab, Cw[wslot<U>(ph, k)]);
          else if constexpr (RECT)
            return kinds ? rect_diag<false>(lr, tab, Kw[wslot<U>(ph, k)]) : lr.inv0;
          else return inv_i;
        };
        // first half sweep (colour 0) from a zero iterate on row y
        if ((ph & 1) == 0) {
          Uw[wslot<U>(ph, 0)].e = mul2(b0.e, inv_of(0).e);
          Uw[wslot<U>(ph, 0)].o = make_float2(0.f, 0.f);
        } else {
          Uw[wslot<U>(ph, 0)].o = mul2(b0.o, inv_of(0).o);
          Uw[wslot<U>(ph, 0)].e = make_float2(0.f, 0.f);
        }
        // half sweep h on row y - (h - 1); its updated pair is the parity of y
#pragma unroll
        for (int h = 2; h <= 2 * S1; ++h) {
          const int k = h - 1;
          if ((ph & 1) == 0)
            psweep<0>(Uw[wslot<U>(ph, k)], Uw[wslot<U>(ph, k + 1)], Uw[wslot<U>(ph, k - 1)],
                      Bw[wslot<U>(ph, k)], inv_of(k).e);
          else
            psweep<1>(Uw[wslot<U>(ph, k)], Uw[wslot<U>(ph, k + 1)], Uw[wslot<U>(ph, k - 1)],
                      Bw[wslot<U>(ph, k)], inv_of(k).o);
        }
        // residual of row y - K and its horizontal restriction
        const P4 &uK = Uw[wslot<U>(ph, K)], &upK = Uw[wslot<U>(ph, K + 1)];
        const P4 &dnK = Uw[wslot<U>(ph, K - 1)], &bK = Bw[wslot<U>(ph, K)];
        const float left = shfl_up1(uK.o.y), right = shfl_dn1(uK.e.x);
        P4 nd{negd_i, negd_i};
        if constexpr (MASK) nd = mask_diag<true>(tab, Cw[wslot<U>(ph, K)]);
        else if constexpr (RECT) nd = kinds ? rect_diag<true>(lr, tab, Kw[wslot<U>(ph, K)]) : lr.negd0;
        P4 r;
        r.e = fma2(nd.e, uK.e, nsum2(upK.e, uK.o, make_float2(left, uK.o.x), bK.e, dnK.e));
        r.o = fma2(nd.o, uK.o, nsum2(upK.o, uK.e, make_float2(uK.e.y, right), bK.o, dnK.o));
        if constexpr (MASK) {
          r = mask_cls(r, Cw[wslot<U>(ph, K)]);
        } else if constexpr (RECT) {
          if (kinds) r = mask_on(r, lr.on, Kw[wslot<U>(ph, K)]);
          else if (!cols_plain) r = mask_on(r, lr.on, 0);
        }
        const float e0 = shfl_up1(r.o.y), e5 = shfl_dn1(r.e.x);
        float2 fA = make_float2(e0, r.o.x), fB = r.e, fC = r.o, fD = make_float2(r.e.y, e5);
        if constexpr (RECT) {
          if (neu && !cols_plain) {  // Neumann ghosts of the restriction mirror the edge cells
            float e[6] = {e0, r.e.x, r.o.x, r.e.y, r.o.y, e5};
            if (x0 == 0) e[0] = e[1];
            if (!(L.nx & 1)) {
              const int mr = L.nx - x0;
#pragma unroll
              for (int m = 0; m <= 4; ++m)
                if (m == mr) e[m + 1] = e[m];
            }
            fA = make_float2(e[0], e[2]); fB = make_float2(e[1], e[3]);
            fC = make_float2(e[2], e[4]); fD = make_float2(e[3], e[5]);
          }
        }
        // (weigh1(e0, e1, e2, e3), weigh1(e2, e3, e4, e5))
        F[wslot<U>(ph, K)] = fma2(q25, fD, fma2(q75, fC, fma2(q75, fB, mul2(q25, fA))));
      }
      {  // row y - KP has seen every pre-sweep: keep it for the up kernel
        const int yw = y - KP;
        if (out_lane && lane_in && yw >= y_out0 && yw < y_out1) {
          const float4 v = join4(Uw[wslot<U>(ph, KP)]);
          if (full) {
            *reinterpret_cast<float4 *>(Wp + wofs) = v;
          } else {
            const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (x0 + j < L.nx) Wp[wofs + j] = vv[j];
          }
        }
        wofs += pitch;
      }
      // coarse row I = (y - K) / 2 - 1 from the restricted rows 2I-1 .. 2I+2
      if ((ph & 1) == 0) {
        const int I = ((y - K) >> 1) - 1;
        if (out_lane && I >= I_begin && I < I_end) {
          float2 rows[4] = {F[wslot<U>(ph, K + 3)], F[wslot<U>(ph, K + 2)],
                            F[wslot<U>(ph, K + 1)], F[wslot<U>(ph, K)]};
          if constexpr (RECT) {
            if (neu) {
              if (I == 0) rows[0] = rows[1];
              if (!(L.ny & 1)) {
#pragma unroll
                for (int q = 1; q < 4; ++q)
                  if (2 * I - 1 + q == L.ny) rows[q] = rows[q - 1];
              }
            }
          }
          float2 v =
              fma2(q25, rows[3], fma2(q75, rows[2], fma2(q75, rows[1], mul2(q25, rows[0]))));
          if constexpr (MASK) {  // coarse cells without an unknown stay zero
            if (Lc.code_off >= 0) {
              const unsigned char *cc = a.codes + Lc.code_off + I * Lc.pitch + J0;
              if (st0 && !cc[0]) v.x = 0.f;
              if (st1 && !cc[1]) v.y = 0.f;
            }
          }
          float *dst = Bc + I * Lc.pitch + J0;
          if (st0 && st1) {
            *reinterpret_cast<float2 *>(dst) = v;
          } else {
            if (st0) dst[0] = v.x;
            if (st1) dst[1] = v.y;
          }
        }
      }
    }
    if constexpr (R != P) half ^= P;
  }
  __pipeline_wait_prior(0);  // no copy may land after this warp's shared memory is released
}

// Is every cell a strip loads an interior cell of an unmasked level?
__device__ __forceinline__ bool strip_interior(const LevelInfo &L, int y_lo, int y_hi, int x_lo,
                                               int x_hi) {
  return L.code_off < 0 && y_lo >= 1 && y_hi <= L.ny - 2 && x_lo >= 1 && x_hi <= L.nx - 2;
}

// The fast FP32 strips take unmasked levels whose next level is unmasked and
// whose row offsets fit 32 bits ...
__device__ __forceinline__ bool fast_levels(const LevelInfo &L, const LevelInfo &Lc) {
  return L.code_off < 0 && Lc.code_off < 0 && (long long)(L.ny + 16) * L.pitch < (1LL << 31);
}
// ... and, in their masked form, masked levels.
__device__ __forceinline__ bool mask_levels(const LevelInfo &L) {
  return L.code_off >= 0 && (long long)(L.ny + 16) * L.pitch < (1LL << 31);
}

// Error word bit: a rectangle-only strip kernel met a level it does not handle
// (the host launches those kernels only for levels without masked instances).
constexpr unsigned kErrStrip = 8u;

// CTAs per SM the strip kernels are compiled for: FP32 kernels with the
// general (masked) strips need up to 128 (down) / 168 (up) registers; the
// rectangle-only forms (ANY = false) fit more CTAs.
template <typename T, bool UP, int NT, int S>
constexpr int strip_min_ctas() {
  // FP32: 12 up warps per SM (16 at 128 registers spilled: slower), 16 down
  // warps (12 with three sweeps, whose longer window needs more registers)
  return sizeof(T) != 4 ? 1 : (UP || S > 2 ? 12 : 16) * kLanes / NT;
}

template <typename T, int S1, bool ANY = true>
__global__ void __launch_bounds__(kSThreads, strip_min_ctas<T, false, kSThreads, S1>())
    k_down_s(Args<T> a) {
  using G = DownGeom<T, S1>;
  using H = typename G::H;
  __shared__ ClassTable<T> tab;
  const Tile tl = a.tiles[blockIdx.x];
  const LevelInfo L = a.lv[tl.level];
  const LevelInfo Lc = a.lv[tl.level + 1];  // the next entry: levels are stored finest first
  dep_enter();
  if (a.st[tl.inst].status != GD_ACTIVE) return;
  fill_table(tab, L.wall);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int RB = L.rows_per_warp;  // even
  const int y_out0 = (tl.ty * kSWarps + warp) * RB;
  if (y_out0 >= L.ny) return;
  const int xl = tl.tx * H::OW - 4 * H::HL;
  const int x0 = xl + 4 * lane;
  const bool out_lane = lane >= H::HL && lane < kLanes - H::HL;
  const int I_begin = y_out0 >> 1;
  const int I_end = min((y_out0 + RB) >> 1, Lc.ny);
  const int y_out1 = min(y_out0 + RB, L.ny);
  const int y_start = (y_out0 - 1 - 2 * S1) & ~1;  // even, at least the rows the sweeps need
  const int y_last = max(2 * I_end + 2 * S1, y_out1 - 1 + 2 * S1 - 1);
  extern __shared__ __align__(16) unsigned char smem[];
  const bool interior = strip_interior(L, y_start, y_last, xl, xl + 127);
  if constexpr (sizeof(T) == 4) {
    if (fast_levels(L, Lc)) {
      if (interior)
        down_strip_fast<S1, false>(a, L, Lc, tab, x0, out_lane, y_start, y_last, y_out0,
                                   y_out1, I_begin, I_end, smem);
      else
        down_strip_fast<S1, true>(a, L, Lc, tab, x0, out_lane, y_start, y_last, y_out0,
                                  y_out1, I_begin, I_end, smem);
      return;
    }
    if constexpr (ANY) {
      if (mask_levels(L)) {
        down_strip_fast<S1, true, true>(a, L, Lc, tab, x0, out_lane, y_start, y_last, y_out0,
                                        y_out1, I_begin, I_end, smem);
        return;
      }
    }
  }
  if constexpr (ANY) {
    if (interior)
      down_strip<T, S1, true>(a, L, Lc, tab, x0, out_lane, y_start, y_last, y_out0, y_out1,
                              I_begin, I_end, smem);
    else
      down_strip<T, S1, false>(a, L, Lc, tab, x0, out_lane, y_start, y_last, y_out0, y_out1,
                               I_begin, I_end, smem);
  } else if (lane == 0) {
    atomicOr(a.counter + kErrWord, kErrStrip);
  }
}

// ---------------------------------------------------------------------------
// Up: u = (pre-smoothed iterate from down) + P e, then S2 post-sweeps (colour
// 1 first).  Radius: 2 S2 columns.  On level 0 also r.z.  (S1 only selects the
// matching down kernel's plan; the up kernel does not depend on it.)
template <typename T, int S1, int S2>
struct UpGeom {
  using H = Halo<2 * S2>;
  static constexpr int O = 2 * S2;   // window index of the output row
  static constexpr int U = O + 2;    // rows in every circular window (even)
};

// r.z partials of the level-0 up kernel: one per group of rows and column
// strip, at a fixed place (the instance's base + group x column strips +
// column strip).  An instance's group height (InstInfo::rz_rows, a power of
// two) is the level-0 strip height it would get alone, and a batch's strip
// height is a power-of-two multiple of it, so a group never spans two warps and
// the grouping does not depend on the batch: a warp adds its lanes' products
// over the group's rows and writes the group's warp sum when the group ends.
// The last CTA of the launch sums an instance's partials in a fixed pattern, so
// an instance gives the same r.z whatever strip heights its batch chose.
constexpr int kRzRows = 8;  // the smallest group (and strip) height
struct RzGroups {
  double *base;  // partial of group 0 of this column strip
  int stride;    // column strips of the instance
  int rows;      // rows per group
  double acc;    // this lane's share of the open group
  __device__ __forceinline__ void add(double v) { acc += v; }
  __device__ __forceinline__ void row_done(int yo, int y_out1) {
    if ((yo & (rows - 1)) == rows - 1 || yo == y_out1 - 1) {
      flush(acc, base + (yo / rows) * stride);
      acc = 0.0;
    }
  }
  // one copy of the flush for all unrolled phases (instruction-cache footprint)
  static __device__ __noinline__ void flush(double acc, double *dst) {
    const double sum = warp_sum(acc);  // xor tree: the same sum in every lane
    if ((threadIdx.x & 31) == 0) *dst = sum;
  }
};

// The lane's two coarse values (columns x0/2, x0/2 + 1) of coarse row cy, with
// Neumann ghosts mirrored and Dirichlet ghosts zero.
// Lanes 0 and 31 also load the coarse column just outside the warp (c0 - 1,
// resp. c0 + 2), so the interpolated row is exact in every lane of the warp.
template <typename T>
struct Pair {
  T v0, v1, outer;
};

template <typename T>
__device__ __forceinline__ T coarse_at(const T *row, const LevelInfo &Lc, int c, bool neu) {
  if (neu) return row[min(max(c, 0), Lc.nx - 1)];
  return (c >= 0 && c < Lc.nx) ? row[c] : T(0);
}

template <typename T>
__device__ __forceinline__ Pair<T> coarse_pair(const T *E, const LevelInfo &Lc, int cy, int x0,
                                               bool neu) {
  const int c0 = x0 >> 1;  // x0 may be negative; x0 is a multiple of 4 so this is exact
  const int lane = threadIdx.x & 31;
  Pair<T> r{T(0), T(0), T(0)};
  int yy = cy;
  bool row_ok = true;
  if (neu) yy = min(max(cy, 0), Lc.ny - 1);
  else row_ok = cy >= 0 && cy < Lc.ny;
  if (row_ok) {
    const T *row = E + (long long)yy * Lc.pitch;
    r.v0 = coarse_at(row, Lc, c0, neu);
    r.v1 = coarse_at(row, Lc, c0 + 1, neu);
    if (lane == 0) r.outer = coarse_at(row, Lc, c0 - 1, neu);
    if (lane == 31) r.outer = coarse_at(row, Lc, c0 + 2, neu);
  }
  return r;
}

// Horizontal interpolation of a coarse pair to the lane's four fine columns.
template <typename T>
__device__ __forceinline__ V4<T> coarse_interp(const Pair<T> &c) {
  const T v0 = c.v0, v1 = c.v1;
  const int lane = threadIdx.x & 31;
  T lft = shfl_up1(v1);   // coarse column c0 - 1
  T rgt = shfl_dn1(v0);   // coarse column c0 + 2
  if (lane == 0) lft = c.outer;
  if (lane == 31) rgt = c.outer;
  V4<T> h;
  h.v[0] = interp1(v0, lft);
  h.v[1] = interp1(v0, v1);
  h.v[2] = interp1(v1, v0);
  h.v[3] = interp1(v1, rgt);
  return h;
}

template <typename T, int S1, int S2, bool LEVEL0, bool INT>
__device__ __forceinline__ void up_strip(const Args<T> &a, const LevelInfo &L,
                                         const LevelInfo &Lc, const ClassTable<T> &tab, int x0,
                                         bool out_lane, int y_start, int y_out0, int y_out1,
                                         RzGroups &rz, unsigned char *smem) {
  using G = UpGeom<T, S1, S2>;
  constexpr int U = G::U, O = G::O;
  const Coef<T, INT> C{tab, tab.d[1], tab.inv[1]};
  const bool neu = L.bc == BC_NEU;
  const bool masked = L.code_off >= 0;
  const T *B = a.arena + L.b_off;
  const T *Wp = a.arena + L.w_off;
  const T *E = a.arena + Lc.u_off;
  T *Uo = a.arena + L.u_off;
  const int y_last = y_out1 - 1 + O;
  V4<T> Bw[U], Uw[U], Ce[3];
  unsigned Cw[U];
#pragma unroll
  for (int k = 0; k < U; ++k) { Bw[k] = zero4<T>(); Uw[k] = zero4<T>(); Cw[k] = 0u; }
  int ce_top = (y_start >> 1) - 1;  // coarse row held in Ce[0]
#pragma unroll
  for (int q = 0; q < 3; ++q) Ce[q] = coarse_interp(coarse_pair(E, Lc, ce_top + q, x0, neu));
  Pair<T> next0 = coarse_pair(E, Lc, ce_top + 3, x0, neu);
  Pair<T> next1 = coarse_pair(E, Lc, ce_top + 4, x0, neu);
  constexpr int NT = UpCta<LEVEL0>::NT;
  const Ring<T, NT> rb(reinterpret_cast<T *>(smem));
  const Ring<T, NT> rw(reinterpret_cast<T *>(smem) + kRing * NT * 4);
  const CodeRing<NT> cring(reinterpret_cast<unsigned *>(smem + 2 * ring_bytes<T, NT>()));
  for (int q = 0; q < kRing - 1; ++q) {
    rb.issue(q, B, L, y_start + q, x0);
    rw.issue(q, Wp, L, y_start + q, x0);
    if (!INT && masked) cring.issue(q, L, a.codes, y_start + q, x0);
    __pipeline_commit();
  }
  for (int base = y_start; base <= y_last; base += U) {
#pragma unroll
    for (int ph = 0; ph < U; ++ph) {
      const int y = base + ph;
      if (y > y_last) break;
      const int step = y - y_start;
      __pipeline_wait_prior(kRing - 2);
      Bw[wslot<U>(ph, 0)] = rb.read(step);
      V4<T> u = rw.read(step);
      if (!INT) Cw[wslot<U>(ph, 0)] = masked ? cring.read(step) : row_classes(L, nullptr, y, x0);
      if (y + kRing - 1 <= y_last) {  // no copy of rows past the strip
        rb.issue(step + kRing - 1, B, L, y + kRing - 1, x0);
        rw.issue(step + kRing - 1, Wp, L, y + kRing - 1, x0);
        if (!INT && masked) cring.issue(step + kRing - 1, L, a.codes, y + kRing - 1, x0);
      }
      __pipeline_commit();
      {  // prolongation of row y; the coarse window holds rows cy - 1, cy, cy + 1
        const int cy = y >> 1;
        if (ce_top + 1 < cy) {
          Ce[0] = Ce[1];
          Ce[1] = Ce[2];
          Ce[2] = coarse_interp(next0);
          next0 = next1;
          ++ce_top;
          next1 = coarse_pair(E, Lc, ce_top + 4, x0, neu);
        }
        const unsigned c = Cw[wslot<U>(ph, 0)];
        const V4<T> &oth = (ph & 1) ? Ce[2] : Ce[0];  // y odd <=> ph odd (y_start even)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          u.v[j] = C.on(c, j) ? prolong1(u.v[j], Ce[1].v[j], oth.v[j]) : T(0);
        Uw[wslot<U>(ph, 0)] = u;
      }
      // post half sweep g runs on row y - g with colour g & 1, so its first
      // updated cell is (g + y - g) & 1 = ph & 1 for every g
#pragma unroll
      for (int g = 1; g <= 2 * S2; ++g) {
        if ((ph & 1) == 0)
          hsweep<0, T, INT>(Uw[wslot<U>(ph, g)], Uw[wslot<U>(ph, g + 1)], Uw[wslot<U>(ph, g - 1)],
                            Bw[wslot<U>(ph, g)], Cw[wslot<U>(ph, g)], C);
        else
          hsweep<1, T, INT>(Uw[wslot<U>(ph, g)], Uw[wslot<U>(ph, g + 1)], Uw[wslot<U>(ph, g - 1)],
                            Bw[wslot<U>(ph, g)], Cw[wslot<U>(ph, g)], C);
      }
      const int yo = y - O;
      if (yo >= y_out0 && yo < y_out1) {
        if (out_lane) {
          V4<T> v = Uw[wslot<U>(ph, O)];
          const unsigned c = Cw[wslot<U>(ph, O)];
#pragma unroll
          for (int j = 0; j < 4; ++j) v.v[j] = C.on(c, j) ? v.v[j] : T(0);
          T *dst = Uo + (long long)yo * L.pitch + x0;
          if (x0 + 3 < L.nx) {
            st4(dst, v);
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (x0 + j < L.nx) dst[j] = v.v[j];
          }
          if (LEVEL0) rz.add((double)dot1(Bw[wslot<U>(ph, O)], v));
        }
        if (LEVEL0) rz.row_done(yo, y_out1);
      }
    }
  }
  __pipeline_wait_prior(0);
}

// Up on an FP32 strip of an unmasked level whose next level is unmasked: the
// same cells and the same r.z partial as up_strip<float, S1, S2, LEVEL0, INT>,
// bit for bit, laid out like down_strip_fast (RECT as there).  The coarse
// correction's rows travel through the copy ring too: coarse row Y/2 + 1 is
// copied in the commit group of fine row Y (Y even), so it has landed when
// row Y is processed and is interpolated then.  The interpolated rows live in
// a circular window of NC slots indexed by the coarse row's distance from the
// strip's first one, so they rotate without moves.
template <int S1, int S2, bool LEVEL0, bool RECT, bool MASK = false>
__device__ __forceinline__ void up_strip_fast(const Args<float> &a, const LevelInfo &L,
                                              const LevelInfo &Lc, const ClassTable<float> &tab,
                                              int x0, bool out_lane, int y_start, int y_out0,
                                              int y_out1, RzGroups &rz, unsigned char *smem) {
  using G = UpGeom<float, S1, S2>;
  constexpr int U = G::U, O = G::O;
  constexpr int P = FastGeom<U>::P, R = FastGeom<U>::R;
  constexpr int NC = P / 2;  // coarse rows per pass; at least 3
  static_assert(NC >= 3, "coarse window");
  const float2 q25 = splat2(0.25f), q75 = splat2(0.75f);
  const P4 inv_i{splat2(tab.inv[1]), splat2(tab.inv[1])};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float *B = a.arena + L.b_off;
  const float *Wp = a.arena + L.w_off;
  const int c0 = x0 >> 1;  // x0 is a multiple of 4, so this is exact for negative x0 too
  const float *E = a.arena + Lc.u_off;
  float *Uo = a.arena + L.u_off + x0;
  const int pitch = L.pitch;
  const int y_last = y_out1 - 1 + O;
  const bool edge_lane = lane == 0 || lane == 31;
  const int outer_c = c0 + (lane == 0 ? -1 : 2);
  LaneRect lr;
  bool lane_in = true, full = true, neu = false, pair_in = true;
  // the warp's 128 columns are all interior columns (no wall, none outside)
  const int xl = x0 - 4 * lane;
  const bool cols_plain = xl >= 1 && xl + 127 <= L.nx - 2;
  if constexpr (RECT) {
    if constexpr (!MASK) lr = lane_rect(L, tab, x0);
    lane_in = x0 >= 0 && x0 < L.nx;
    full = x0 + 3 < L.nx;
    neu = L.bc == BC_NEU;
    pair_in = c0 >= 0 && c0 + 1 < Lc.nx;
  }
  constexpr int NT = UpCta<LEVEL0>::NT;
  constexpr int kSlot = NT * 4;
  float *rb = reinterpret_cast<float *>(smem) + threadIdx.x * 4;
  float *rw = rb + R * kSlot;
  // coarse ring: slot q holds the lane's two coarse columns and the warp's two
  // outer columns of the coarse row copied with fine slot q
  float2 *rc = reinterpret_cast<float2 *>(smem + (size_t)2 * R * kSlot * 4) + threadIdx.x;
  float *ro = reinterpret_cast<float *>(smem + (size_t)2 * R * kSlot * 4 + (size_t)R * NT * 8) +
              warp * 2 + (lane == 31);
  constexpr int kCSlot = NT;  // float2 between two coarse slots of a lane
  constexpr int kOSlot = (NT / kLanes) * 2;
  // copy of one coarse column into the ring: Neumann ghosts mirror the edge,
  // Dirichlet ghosts and rows outside are zero
  auto ccopy1 = [&](float *dst, const float *row, bool row_ok, int c) {
    if (neu) c = min(max(c, 0), Lc.nx - 1);
    const bool ok = row_ok && c >= 0 && c < Lc.nx;
    __pipeline_memcpy_async(dst, ok ? row + c : E, 4, ok ? 0 : 4);
  };
  auto cissue = [&](int q, int cy) {
    float2 *dv = rc + q * kCSlot;
    float *dout = ro + q * kOSlot;
    if constexpr (RECT) {
      const int yy = neu ? min(max(cy, 0), Lc.ny - 1) : cy;
      const bool row_ok = yy >= 0 && yy < Lc.ny;
      const float *row = E + (row_ok ? yy : 0) * Lc.pitch;
      if (pair_in) {
        __pipeline_memcpy_async(dv, row_ok ? row + c0 : E, 8, row_ok ? 0 : 8);
      } else {
        ccopy1(reinterpret_cast<float *>(dv), row, row_ok, c0);
        ccopy1(reinterpret_cast<float *>(dv) + 1, row, row_ok, c0 + 1);
      }
      if (edge_lane) ccopy1(dout, row, row_ok, outer_c);
    } else {
      // interior strips: every coarse row they use is in the grid; rows past the
      // last are clamped and never used
      const float *row = E + min(cy, Lc.ny - 1) * Lc.pitch;
      __pipeline_memcpy_async(dv, row + c0, 8);
      if (edge_lane) __pipeline_memcpy_async(dout, row + outer_c, 4);
    }
  };
  auto cread = [&](int q) {
    const float2 v = rc[q * kCSlot];
    const float outer = edge_lane ? ro[q * kOSlot] : 0.f;
    float lft = shfl_up1(v.y), rgt = shfl_dn1(v.x);
    if (lane == 0) lft = outer;
    if (lane == 31) rgt = outer;
    const float2 m = mul2(q75, v);  // interp1(near, far) on both pairs
    return P4{fma2(q25, make_float2(lft, v.x), m), fma2(q25, make_float2(v.y, rgt), m)};
  };
  // MASK: the level's class bytes and their ring, after the coarse ring
  const unsigned char *codes = a.codes + (MASK ? L.code_off : 0);
  unsigned *crow = reinterpret_cast<unsigned *>(smem + (size_t)2 * R * kSlot * 4 +
                                                coarse_ring_bytes<R, NT>()) +
                   threadIdx.x;
  auto issue = [&](int q, int y, int gofs) {
    float *db = rb + q * kSlot, *dw = rw + q * kSlot;
    if constexpr (RECT) {
      const bool ok = lane_in && y >= 0 && y < L.ny;
      __pipeline_memcpy_async(db, ok ? B + gofs + x0 : B, 16, ok ? 0 : 16);
      __pipeline_memcpy_async(dw, ok ? Wp + gofs + x0 : Wp, 16, ok ? 0 : 16);
      if constexpr (MASK)
        __pipeline_memcpy_async(crow + q * NT, ok ? codes + gofs + x0 : codes, 4, ok ? 0 : 4);
    } else {
      __pipeline_memcpy_async(db, B + gofs + x0, 16);
      __pipeline_memcpy_async(dw, Wp + gofs + x0, 16);
    }
    if (!(y & 1)) cissue(q, (y >> 1) + 1);  // the coarse row interpolated at row y
  };
  P4 Bw[U], Uw[U], H[NC];
  int Kw[U];       // row kinds of the window rows (RECT)
  unsigned Cw[U];  // packed classes of the window rows (MASK)
#pragma unroll
  for (int k = 0; k < U; ++k) { Bw[k] = zero_p4(); Uw[k] = zero_p4(); Kw[k] = 3; Cw[k] = 0u; }
  // coarse rows relative to cy0 = y_start / 2: window slot of row cy0 + k is
  // k mod NC.  Rows cy0 - 1 and cy0 come through coarse slots 1 and 3, which
  // the loop never uses (a coarse row travels with an even fine row, and even
  // rows take even slots).
  const int cy0 = y_start >> 1;
  cissue(1, cy0 - 1);
  cissue(3, cy0);
  __pipeline_commit();
  int gofs = y_start * pitch;
#pragma unroll
  for (int q = 0; q < R - 1; ++q) {
    issue(q, y_start + q, gofs);
    __pipeline_commit();
    gofs += pitch;
  }
  __pipeline_wait_prior(R - 1);
  H[NC - 1] = cread(1);
  H[0] = cread(3);
  int oofs = (y_start - O) * pitch;  // row offset of the output row of this step
  int half = 0;  // ring slot of this pass's first row (0 or P when R == 2P)
  for (int base = y_start; base <= y_last; base += P) {
    const int prev = R == P ? 0 : (half ^ P);  // half the slot before ph = 0 is in
#pragma unroll
    for (int ph = 0; ph < P; ++ph) {
      const int y = base + ph;
      if (y > y_last) break;
      __pipeline_wait_prior(R - 2);
      const float4 qb = *reinterpret_cast<const float4 *>(rb + (half + ph) * kSlot);
      const float4 qw = *reinterpret_cast<const float4 *>(rw + (half + ph) * kSlot);
      const int c = ph >> 1;  // coarse row of y relative to the pass's first
      if ((ph & 1) == 0) H[(c + 1) % NC] = cread(half + ph);  // row c + 1 for rows 2c, 2c + 1
      if (y + R - 1 <= y_last)  // no copy of rows past the strip; the slot read one step ago
        issue(ph > 0 ? half + ph - 1 : prev + P - 1, y + R - 1, gofs);
      __pipeline_commit();
      gofs += pitch;
      Bw[wslot<U>(ph, 0)] = split4(qb);
      if constexpr (MASK) Cw[wslot<U>(ph, 0)] = crow[(half + ph) * NT];
      else if constexpr (RECT) Kw[wslot<U>(ph, 0)] = row_kind(L, y);
      const P4 &hn = H[c % NC];
      const P4 &hf = (ph & 1) ? H[(c + 1) % NC] : H[(c + NC - 1) % NC];
      const P4 w = split4(qw);
      // rectangle strips: per-lane constants when every row the step touches
      // (y - U + 1 .. y) has no wall and is in the grid (kv = 0), per-row kinds
      // otherwise (kv = 1); one copy runs, chosen by a warp-uniform branch
      // (masked levels: always the per-row classes)
      const bool rows_plain = MASK ? false : !RECT || (y - (U - 1) >= 1 && y <= L.ny - 2);
      P4 v;  // the output row y - O
#pragma unroll
      for (int kv = MASK ? 1 : 0; kv < (RECT ? 2 : 1); ++kv) {
        if ((kv == 1) == rows_plain) continue;
        const bool kinds = kv == 1;
        auto inv_of = [&](int k) -> P4 {
          if constexpr (MASK) return mask_diag<false>(tab, Cw[wslot<U>(ph, k)]);
          else if constexpr (RECT)
            return kinds ? rect_diag<false>(lr, tab, Kw[wslot<U>(ph, k)]) : lr.inv0;
          else return inv_i;
        };
        P4 &u = Uw[wslot<U>(ph, 0)];
        u.e = fma2(q25, hf.e, fma2(q75, hn.e, w.e));  // prolong1 on both pairs
        u.o = fma2(q25, hf.o, fma2(q75, hn.o, w.o));
        if constexpr (MASK) {
          u = mask_cls(u, Cw[wslot<U>(ph, 0)]);
        } else if constexpr (RECT) {
          if (kinds) u = mask_on(u, lr.on, Kw[wslot<U>(ph, 0)]);
          else if (!cols_plain) u = mask_on(u, lr.on, 0);
        }
        // post half sweep g on row y - g; its updated pair is the parity of y
#pragma unroll
        for (int g = 1; g <= 2 * S2; ++g) {
          if ((ph & 1) == 0)
            psweep<0>(Uw[wslot<U>(ph, g)], Uw[wslot<U>(ph, g + 1)], Uw[wslot<U>(ph, g - 1)],
                      Bw[wslot<U>(ph, g)], inv_of(g).e);
          else
            psweep<1>(Uw[wslot<U>(ph, g)], Uw[wslot<U>(ph, g + 1)], Uw[wslot<U>(ph, g - 1)],
                      Bw[wslot<U>(ph, g)], inv_of(g).o);
        }
        v = Uw[wslot<U>(ph, O)];
        if constexpr (MASK) {
          v = mask_cls(v, Cw[wslot<U>(ph, O)]);
        } else if constexpr (RECT) {
          if (kinds) v = mask_on(v, lr.on, Kw[wslot<U>(ph, O)]);
          else if (!cols_plain) v = mask_on(v, lr.on, 0);
        }
      }
      if (y - O >= y_out0) {
        if (out_lane) {
          const float4 q = join4(v);
          if (full) {
            *reinterpret_cast<float4 *>(Uo + oofs) = q;
          } else {
            const float vv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if (x0 + j < L.nx) Uo[oofs + j] = vv[j];
          }
          if (LEVEL0) {
            const P4 &bo = Bw[wslot<U>(ph, O)];
            const float2 t = fma2(bo.o, v.o, mul2(bo.e, v.e));  // dot1
            rz.add((double)__fadd_rn(t.x, t.y));
          }
        }
        if (LEVEL0) rz.row_done(y - O, y_out1);
      }
      oofs += pitch;
    }
    if constexpr (R != P) half ^= P;
  }
  __pipeline_wait_prior(0);
}

// FP32: three CTAs per SM (above 170 registers only two fit, which was measured
// slower); the FP64 form needs more registers than that and is left unbounded.
template <typename T, int S1, int S2, bool LEVEL0, bool ANY = true>
__global__ void __launch_bounds__(UpCta<LEVEL0>::NT,
                                  strip_min_ctas<T, true, UpCta<LEVEL0>::NT, S2>())
    k_up_s(Args<T> a) {
  using G = UpGeom<T, S1, S2>;
  using H = typename G::H;
  __shared__ ClassTable<T> tab;
  const Tile tl = a.tiles[blockIdx.x];
  const LevelInfo L = a.lv[tl.level];
  const LevelInfo Lc = a.lv[tl.level + 1];  // the next entry: levels are stored finest first
  dep_enter();
  const bool active = a.st[tl.inst].status == GD_ACTIVE;
  if (active) {
    fill_table(tab, L.wall);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int RB = L.rows_per_warp;  // level 0: a multiple of the instance's rz_rows
    const int y_out0 = (tl.ty * UpCta<LEVEL0>::W + warp) * RB;
    const InstInfo &II = a.inst[tl.inst];
    RzGroups rz{a.part0 + II.up0_begin + tl.tx, (L.nx + H::OW - 1) / H::OW, II.rz_rows, 0.0};
    if (y_out0 < L.ny) {
      const int y_out1 = min(y_out0 + RB, L.ny);
      const int xl = tl.tx * H::OW - 4 * H::HL;
      const int x0 = xl + 4 * lane;
      const bool out_lane = lane >= H::HL && lane < kLanes - H::HL && x0 >= 0 && x0 < L.nx;
      const int y_start = (y_out0 - 2 * S2) & ~1;
      const int y_last = y_out1 - 1 + G::O;
      extern __shared__ __align__(16) unsigned char smem[];
      const bool interior = strip_interior(L, y_start, y_last, xl, xl + 127);
      bool fast = false;
      if constexpr (sizeof(T) == 4) {
        fast = fast_levels(L, Lc);
        if (fast && interior)
          up_strip_fast<S1, S2, LEVEL0, false>(a, L, Lc, tab, x0, out_lane, y_start, y_out0,
                                               y_out1, rz, smem);
        else if (fast)
          up_strip_fast<S1, S2, LEVEL0, true>(a, L, Lc, tab, x0, out_lane, y_start, y_out0,
                                              y_out1, rz, smem);
        if constexpr (ANY) {
          if (!fast && mask_levels(L)) {
            up_strip_fast<S1, S2, LEVEL0, true, true>(a, L, Lc, tab, x0, out_lane, y_start,
                                                      y_out0, y_out1, rz, smem);
            fast = true;
          }
        }
      }
      if constexpr (ANY) {
        if (fast) {
          // done above
        } else if (interior)
          up_strip<T, S1, S2, LEVEL0, true>(a, L, Lc, tab, x0, out_lane, y_start, y_out0, y_out1,
                                            rz, smem);
        else
          up_strip<T, S1, S2, LEVEL0, false>(a, L, Lc, tab, x0, out_lane, y_start, y_out0,
                                             y_out1, rz, smem);
      } else if (!fast && lane == 0) {
        atomicOr(a.counter + kErrWord, kErrStrip);
      }
    }
  }
  if (!LEVEL0) return;
  // the lane that wrote a warp's group partials makes them visible before the
  // CTA takes its ticket (one fence per warp)
  if ((threadIdx.x & 31) == 0) __threadfence();
  if (!last_block(a.counter + 3)) return;
  // one warp per instance (instances in parallel): each lane sums every 32nd of
  // the instance's groups, then a fixed shuffle tree, so an instance gets the
  // same r.z in any batch
  const int warp = threadIdx.x >> 5, nw = UpCta<LEVEL0>::NT >> 5;
  for (int i = warp; i < a.ninst; i += nw) {
    const InstInfo &I = a.inst[i];
    if (I.up0_end <= I.up0_begin) continue;
    InstState &S = a.st[i];
    if (S.status != GD_ACTIVE) continue;
    const double rz = warp_range_sum(a.part0, I.up0_begin, I.up0_end);
    if ((threadIdx.x & 31) == 0) finish_rz(S, rz);
  }
}

// ---------------------------------------------------------------------------
// Krylov kernels on level 0: a warp covers 128 columns x kKrylovRows rows and
// the CTA four such row bands.  The one column outside the warp on each side
// comes from a scalar load by lanes 0 and 31.

template <typename T>
__device__ __forceinline__ T edge_value(const T *A, const LevelInfo &L, int y, int x) {
  return (y >= 0 && y < L.ny && x >= 0 && x < L.nx) ? A[(long long)y * L.pitch + x] : T(0);
}

template <typename T, bool INT>
__device__ __forceinline__ double pupdate_rows(const Args<T> &a, const InstInfo &I,
                                               const LevelInfo &L, const ClassTable<T> &tab,
                                               int lane, int x0, int y0, int y1, T beta,
                                               const T *z, const T *p, T *pn,
                                               unsigned char *smem) {
  const Coef<T, INT> C{tab, tab.d[1], tab.inv[1]};
  const Ring<T> rz(reinterpret_cast<T *>(smem));
  const Ring<T> rp(reinterpret_cast<T *>(smem) + kRing * kThreads * 4);
  const EdgeRing<T> ez(reinterpret_cast<T *>(smem) + 2 * kRing * kThreads * 4);
  const EdgeRing<T> ep(reinterpret_cast<T *>(smem) + 2 * kRing * kThreads * 4 + kRing * kThreads);
  const int xe = lane == 0 ? x0 - 1 : x0 + 4;  // edge column of lanes 0 and 31
  const bool edge_lane = lane == 0 || lane == 31;
  const bool read_p = beta != T(0);
  const int nsteps = y1 - y0 + 2;  // rows y0 - 1 .. y1; nothing past them is copied
  auto issue = [&](int q) {
    if (q < nsteps) {
      const int y = y0 - 1 + q;
      rz.issue(q, z, L, y, x0);
      if (read_p) rp.issue(q, p, L, y, x0);
      if (edge_lane) {
        ez.issue(q, z, L, y, xe);
        if (read_p) ep.issue(q, p, L, y, xe);
      }
    }
    __pipeline_commit();
  };
  for (int q = 0; q < kRing - 1; ++q) issue(q);
  int step = 0;
  T edge_next = T(0);
  // The first direction is p = z: with beta == 0 the old buffer is not read
  // (it need not be initialised), so the rings for p are left idle.
  const bool use_p = beta != T(0);
  auto newp = [&]() {
    __pipeline_wait_prior(kRing - 2);
    V4<T> zz = rz.read(step);
    T e = edge_lane ? ez.read(step) : T(0);
    if (use_p) {
      const V4<T> pp = rp.read(step);
      if (edge_lane) e += beta * ep.read(step);
#pragma unroll
      for (int j = 0; j < 4; ++j) zz.v[j] += beta * pp.v[j];
    }
    edge_next = e;
    issue(step + kRing - 1);
    ++step;
    return zz;
  };
  double part = 0.0;
  V4<T> up = newp(), cu = newp(), dn;
  T edge_cu = edge_next;
  const bool full = x0 + 3 < L.nx;
  for (int y = y0; y < y1; ++y) {
    dn = newp();
    T left = shfl_up1(cu.v[3]), right = shfl_dn1(cu.v[0]);
    if (lane == 0) left = edge_cu;
    if (lane == 31) right = edge_cu;
    edge_cu = edge_next;
    const unsigned c = INT ? 0u : row_classes(L, a.codes, y, x0);
    const V4<T> ap = arow(cu, up, dn, left, right, c, C);
    T acc = T(0);
#pragma unroll
    for (int j = 0; j < 4; ++j) acc += cu.v[j] * ap.v[j];
    part += (double)acc;
    if (x0 < L.nx) {
      T *dst = pn + (long long)y * L.pitch + x0;
      if (full) st4(dst, cu);
      else
        for (int j = 0; j < 4 && x0 + j < L.nx; ++j) dst[j] = cu.v[j];
    }
    up = cu;
    cu = dn;
  }
  __pipeline_wait_prior(0);
  return part;
}

// p_new = z + beta p_old (read from one buffer, written to the other) and p.Ap.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pupdate_s(Args<T> a) {
  __shared__ ClassTable<T> tab;
  const Tile tl = a.tiles[blockIdx.x];
  dep_enter();
  const bool active = a.st[tl.inst].status == GD_ACTIVE;
  double part = 0.0;
  if (active) {
    const InstInfo &I = a.inst[tl.inst];
    const LevelInfo L = a.lv[I.level0];
    fill_table(tab, L.wall);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y0 = (tl.ty * kWarps + warp) * kKrylovRows;
    const int xl = tl.tx * kKrylovCols;
    const int x0 = xl + 4 * lane;
    if (y0 < L.ny) {
      const int y1 = min(y0 + kKrylovRows, L.ny);
      const T beta = (T)a.st[tl.inst].beta;
      const int cur = a.st[tl.inst].pcur;
      const T *z = a.arena + I.z_off;
      const T *p = a.arena + p_offset(I, cur);
      T *pn = a.arena + p_offset(I, cur ^ 1);
      extern __shared__ __align__(16) unsigned char smem[];
      if (strip_interior(L, y0, y1 - 1, xl, xl + 127))
        part = pupdate_rows<T, true>(a, I, L, tab, lane, x0, y0, y1, beta, z, p, pn, smem);
      else
        part = pupdate_rows<T, false>(a, I, L, tab, lane, x0, y0, y1, beta, z, p, pn, smem);
    }
  }
  part = block_sum<kThreads>(part);
  if (threadIdx.x == 0) a.part0[blockIdx.x] = part;
  if (!last_block(a.counter + 0)) return;
  const int warp = threadIdx.x >> 5;
  for (int i = warp; i < a.ninst; i += kWarps) {
    InstState &S = a.st[i];
    if (S.status != GD_ACTIVE) continue;
    const InstInfo &I = a.inst[i];
    const double pAp = warp_range_sum(a.part0, I.fine_begin, I.fine_end);
    if ((threadIdx.x & 31) == 0) {
      const double alpha = S.rz / pAp;
      S.pAp = pAp;
      S.pcur ^= 1;
      if (!(pAp > 0.0) || !isfinite(alpha)) {
        S.status = GD_BREAKDOWN;
        S.flags |= FLAG_RU;
      } else {
        S.alpha = alpha;
      }
    }
  }
}

template <typename T, bool INT>
__device__ __forceinline__ double cgupdate_rows(const Args<T> &a, const LevelInfo &L,
                                                const ClassTable<T> &tab, int lane, int x0,
                                                int y0, int y1, T alpha, const T *p, T *d, T *r,
                                                bool dzero, unsigned char *smem) {
  const Coef<T, INT> C{tab, tab.d[1], tab.inv[1]};
  const Ring<T> rp(reinterpret_cast<T *>(smem));
  const Ring<T> rd(reinterpret_cast<T *>(smem) + kRing * kThreads * 4);
  const Ring<T> rr(reinterpret_cast<T *>(smem) + 2 * kRing * kThreads * 4);
  const EdgeRing<T> ep(reinterpret_cast<T *>(smem) + 3 * kRing * kThreads * 4);
  const int xe = lane == 0 ? x0 - 1 : x0 + 4;  // edge column of lanes 0 and 31
  const bool edge_lane = lane == 0 || lane == 31;
  // p streams rows y0 - 1 .. y1; d and r the band's own rows y0 .. y1 - 1, used
  // one step later (the slots of the two halo rows are never read); nothing past
  // row y1 is copied
  const int nsteps = y1 - y0 + 2;
  auto issue = [&](int q) {
    if (q < nsteps) {
      const int y = y0 - 1 + q;
      const bool own = y >= y0 && y < y1;
      rp.issue(q, p, L, y, x0);
      if (own && !dzero) rd.issue(q, d, L, y, x0);
      if (own) rr.issue(q, r, L, y, x0);
      if (edge_lane) ep.issue(q, p, L, y, xe);
    }
    __pipeline_commit();
  };
  for (int q = 0; q < kRing - 1; ++q) issue(q);
  int step = 0;
  V4<T> dcur, rcur, dnext = zero4<T>(), rnext = zero4<T>();
  T edge_next = T(0);
  auto next = [&]() {
    __pipeline_wait_prior(kRing - 2);
    const V4<T> pp = rp.read(step);
    dcur = dnext;
    rcur = rnext;
    dnext = dzero ? zero4<T>() : rd.read(step);
    rnext = rr.read(step);
    edge_next = edge_lane ? ep.read(step) : T(0);
    issue(step + kRing - 1);
    ++step;
    return pp;
  };
  double part = 0.0;
  V4<T> up = next(), cu = next(), dn;
  T edge_cu = edge_next;
  const bool full = x0 + 3 < L.nx;
  for (int y = y0; y < y1; ++y) {
    dn = next();
    T left = shfl_up1(cu.v[3]), right = shfl_dn1(cu.v[0]);
    if (lane == 0) left = edge_cu;
    if (lane == 31) right = edge_cu;
    edge_cu = edge_next;
    const unsigned c = INT ? 0u : row_classes(L, a.codes, y, x0);
    const V4<T> ap = arow(cu, up, dn, left, right, c, C);
    if (x0 < L.nx) {
      const long long g = (long long)y * L.pitch + x0;
      if (full) {
        V4<T> dd = dcur, rv = rcur;
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dd.v[j] += alpha * cu.v[j];
          rv.v[j] -= alpha * ap.v[j];
          acc += rv.v[j] * rv.v[j];
        }
        part += (double)acc;
        st4(d + g, dd);
        st4(r + g, rv);
      } else {
        for (int j = 0; j < 4 && x0 + j < L.nx; ++j) {
          d[g + j] = (dzero ? T(0) : d[g + j]) + alpha * cu.v[j];
          const T rn = r[g + j] - alpha * ap.v[j];
          r[g + j] = rn;
          part += (double)rn * (double)rn;
        }
      }
    }
    up = cu;
    cu = dn;
  }
  __pipeline_wait_prior(0);
  return part;
}

// d += alpha p, r -= alpha A p and r.r; schedules FP64 refreshes.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_cgupdate_s(Args<T> a) {
  __shared__ ClassTable<T> tab;
  const Tile tl = a.tiles[blockIdx.x];
  dep_enter();
  const bool active = a.st[tl.inst].status == GD_ACTIVE;
  double part = 0.0;
  if (active) {
    const InstInfo &I = a.inst[tl.inst];
    const LevelInfo L = a.lv[I.level0];
    fill_table(tab, L.wall);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y0 = (tl.ty * kWarps + warp) * kKrylovRows;
    const int xl = tl.tx * kKrylovCols;
    const int x0 = xl + 4 * lane;
    if (y0 < L.ny) {
      const int y1 = min(y0 + kKrylovRows, L.ny);
      const T alpha = (T)a.st[tl.inst].alpha;
      const T *p = a.arena + p_offset(I, a.st[tl.inst].pcur);
      T *d = a.arena + I.d_off;
      T *r = a.arena + I.r_off;
      const bool dzero = a.st[tl.inst].flags & FLAG_DZERO;
      extern __shared__ __align__(16) unsigned char smem[];
      if (strip_interior(L, y0, y1 - 1, xl, xl + 127))
        part = cgupdate_rows<T, true>(a, L, tab, lane, x0, y0, y1, alpha, p, d, r, dzero, smem);
      else
        part = cgupdate_rows<T, false>(a, L, tab, lane, x0, y0, y1, alpha, p, d, r, dzero, smem);
    }
  }
  part = block_sum<kThreads>(part);
  if (threadIdx.x == 0) a.part0[blockIdx.x] = part;
  if (!last_block(a.counter + 1)) return;
  const int warp = threadIdx.x >> 5;
  for (int i = warp; i < a.ninst; i += kWarps) {
    InstState &S = a.st[i];
    if (S.status != GD_ACTIVE) continue;
    const InstInfo &I = a.inst[i];
    const double rr = warp_range_sum(a.part0, I.fine_begin, I.fine_end);
    if ((threadIdx.x & 31) == 0) {
      S.rr = rr;
      S.iters += 1;
      S.flags &= ~FLAG_DZERO;  // every CTA of this launch has read it
      if (rr <= a.delta2 * S.rr_ref || rr <= a.tol2 * S.ff || S.iters >= a.max_iter ||
          !isfinite(rr))
        S.flags |= FLAG_RU;
    }
  }
}

// FP64 refresh: x' = x + d (the FP32 correction folded into the FP64
// solution), r = scale (f - fmean) - A x', the residual norm and the
// convergence decision per instance, in one pass.  With INIT: the residual of
// the caller's initial x, nothing to fold.
//
// The solution alternates between the caller's buffer and the plan's own FP64
// copy (InstState::xcur names the current one): the pass reads the current
// copy and d and writes x' into the other one, so the halo rows and edge
// columns that neighbouring warps read are never rewritten while it runs.
// When d restarted since the last refresh (FLAG_DZERO) there is nothing to
// fold and the current copy stays where it is.
//
// A warp covers 128 columns (four per lane) and kKrylovRows rows of the
// 64 x 128 fine tile, plus one halo row above and below; horizontal
// neighbours come from shuffles and lanes 0 and 31 take the column just
// outside the warp.  Rows arrive through a ring of kRefRing slots in shared
// memory: slot q holds x, d and the classes of row y0 - 1 + q, and f and the
// edge column of the row before it, the row completed at step q.  On
// rectangle strips whose 128 columns are inside the grid and whose caller
// rows are 16-byte aligned (almost all strips), lane 0 fills a slot with
// three bulk copies (x, f, d row segments) completed on the slot's mbarrier;
// elsewhere every lane copies its own four columns with cp.async, element by
// element at the ragged right end and on unaligned caller rows.  The edge
// columns always travel by cp.async (lanes 0 and 31).
constexpr int kRefRing = 4;

template <typename T>
struct RefSmem {
  // per-thread cp.async ring
  static constexpr int DCH = (int)(4 * sizeof(T) / 16);  // 16-byte chunks of d per lane and row
  static constexpr int CH = 4 + DCH;                       // chunks: x 0-1, f 2-3, d 4..
  static constexpr size_t main = (size_t)kRefRing * CH * kThreads * 16;
  static constexpr size_t edge = (size_t)kRefRing * kWarps * 2 * 16;  // x and d, per side
  static constexpr size_t code = (size_t)kRefRing * kThreads * 4;
  static constexpr size_t ecode = (size_t)kRefRing * kWarps * 2 * 4;
  static constexpr size_t general = main + edge + code + ecode;
  // bulk ring: per warp and slot the x, f and d row segments, then the
  // barriers, then the edge ring laid out as above
  static constexpr size_t SB = 2048 + 128 * sizeof(T);
  static constexpr size_t rows = (size_t)kWarps * kRefRing * SB;
  static constexpr size_t bars = (size_t)kWarps * kRefRing * 8;
  static constexpr size_t bulk = rows + bars + edge;
  static constexpr size_t bytes = general > bulk ? general : bulk;
};

template <typename T>
constexpr size_t refresh_smem() { return RefSmem<T>::bytes; }

static_assert(kFTX == 4 * kLanes && kFTY == kWarps * kKrylovRows,
              "the refresh maps one warp to 128 columns and kKrylovRows rows of a fine tile");

// x[x0 .. x0 + 3] of one FP64 row into two 16-byte chunks; `nv` (0..4) of the
// four columns are inside the grid, the others are zero-filled.  `row` is any
// valid address when nv is 0.
__device__ __forceinline__ void copy_row4(unsigned char *c0, unsigned char *c1, const double *row,
                                          int nv) {
  if (nv == 4 && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
    __pipeline_memcpy_async(c0, row, 16);
    __pipeline_memcpy_async(c1, row + 2, 16);
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      __pipeline_memcpy_async((j < 2 ? c0 : c1) + 8 * (j & 1), j < nv ? row + j : row, 8,
                              j < nv ? 0 : 8);
  }
}

__device__ __forceinline__ void read_row4(double (&v)[4], const unsigned char *c0,
                                          const unsigned char *c1) {
  const double2 a = *reinterpret_cast<const double2 *>(c0);
  const double2 b = *reinterpret_cast<const double2 *>(c1);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// What one warp of the refresh works on, resolved once per launch.
template <typename T>
struct RefWarp {
  const double *src;  // the current solution copy
  long long spitch;
  double *dst;        // the other copy (written when folding)
  long long dpitch;
  double *X;          // the caller's buffer (INIT zeroes it where there is no unknown)
  long long upitch;
  const double *F;
  const T *D;
  T *R;
  const unsigned char *codes;
  int ny, nx, pitch, x0, nv, y0, y1, ecol;
  bool masked, ecol_in;
  bool xz;  // x is zero: nothing of it is read
  double scale, fmean, omw;
};

// One warp's rows.  FAST: a rectangle strip whose 128 columns are all inside
// the grid, on 16-byte aligned caller rows; lane 0 moves whole row segments
// with bulk copies, rows outside the grid are not copied and read as zeros,
// and no cell needs a class test.  Both paths do the same arithmetic in the
// same order.
template <typename T, bool INIT, bool FOLD, bool FAST>
__device__ __forceinline__ void refresh_strip(const RefWarp<T> &w, unsigned char *smem,
                                              unsigned *err, double &part, double &part_f) {
  using SM = RefSmem<T>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool edge_lane = lane == 0 || lane == 31;
  const int side = lane == 31;
  const bool masked = !FAST && w.masked;
  const int x0 = w.x0, nv = FAST ? 4 : w.nv, y0 = w.y0, y1 = w.y1, ny = w.ny;
  const int col0 = x0 - 4 * lane;
  double dgc[4];  // diagonal of the lane's columns away from the top and bottom rows
#pragma unroll
  for (int j = 0; j < 4; ++j)
    dgc[j] = 4.0 - (double)((x0 + j == 0) + (x0 + j == w.nx - 1)) * w.omw;
  // per-thread ring (general strips)
  auto chunk = [&](int s, int k) {
    return smem + ((size_t)(s * SM::CH + k) * kThreads + threadIdx.x) * 16;
  };
  auto cslot = [&](int s) {
    return reinterpret_cast<unsigned *>(smem + SM::main + SM::edge) + s * kThreads + threadIdx.x;
  };
  auto ecslot = [&](int s) {
    return reinterpret_cast<unsigned *>(smem + SM::main + SM::edge + SM::code) +
           (s * kWarps + warp) * 2 + side;
  };
  // bulk ring (FAST strips)
  unsigned char *const brow = smem + (size_t)warp * kRefRing * SM::SB;
  uint64_t *const bar = reinterpret_cast<uint64_t *>(smem + SM::rows) + warp * kRefRing;
  auto eslot = [&](int s) {
    return smem + (FAST ? SM::rows + SM::bars : SM::main) +
           ((size_t)(s * kWarps + warp) * 2 + side) * 16;
  };
  if constexpr (FAST) {
    if (lane == 0)
      for (int s = 0; s < kRefRing; ++s) bulk::init(bar + s, 1);
    bulk::init_fence();
    __syncwarp();
  }
  // step q: x, d, classes of row y0 - 1 + q; f and the edge column of the row before
  auto issue = [&](int q) {
    const int s = q & (kRefRing - 1);
    const int yy = y0 - 1 + q;
    const bool rok = yy >= 0 && yy < ny && nv > 0;
    const int p = yy - 1;
    const bool pin = p >= y0 && p < y1;
    const bool pok = pin && nv > 0;
    if constexpr (FAST) {
      if (lane == 0) {
        unsigned char *slot = brow + s * SM::SB;
        const unsigned xb = 128 * sizeof(double), db = FOLD ? 128 * sizeof(T) : 0;
        const bool xok = rok && !w.xz;
        bulk::arrive_expect(bar + s, (xok ? xb : 0u) + (rok ? db : 0u) + (pok ? xb : 0u));
        if (xok) bulk::copy(slot, w.src + yy * w.spitch + col0, xb, bar + s);
        if (FOLD && rok) bulk::copy(slot + 2 * xb, w.D + (long long)yy * w.pitch + col0, db, bar + s);
        if (pok) bulk::copy(slot + xb, w.F + p * w.upitch + col0, xb, bar + s);
      }
    } else {
      copy_row4(chunk(s, 0), chunk(s, 1), rok ? w.src + yy * w.spitch + x0 : w.src,
                rok && !w.xz ? nv : 0);
      if constexpr (FOLD) {
        const T *dr = rok ? w.D + (long long)yy * w.pitch + x0 : w.D;
#pragma unroll
        for (int k = 0; k < SM::DCH; ++k)
          __pipeline_memcpy_async(chunk(s, 4 + k), dr + (rok ? k * (16 / sizeof(T)) : 0), 16,
                                  rok ? 0 : 16);
      }
      if (masked)
        __pipeline_memcpy_async(cslot(s), w.codes + (rok ? (long long)yy * w.pitch + x0 : 0), 4,
                                rok ? 0 : 4);
      copy_row4(chunk(s, 2), chunk(s, 3), pok ? w.F + p * w.upitch + x0 : w.F, pok ? nv : 0);
    }
    if (edge_lane) {
      const bool eok = pin && w.ecol_in;
      const bool exok = eok && !w.xz;
      __pipeline_memcpy_async(eslot(s), exok ? w.src + p * w.spitch + w.ecol : w.src, 8,
                              exok ? 0 : 8);
      if constexpr (FOLD)
        __pipeline_memcpy_async(eslot(s) + 8, eok ? w.D + (long long)p * w.pitch + w.ecol : w.D,
                                sizeof(T), eok ? 0 : sizeof(T));
      if (masked) {
        // the aligned word holding the edge column: byte 3 left of lane 0, byte 0 right of lane 31
        const int wc = lane == 0 ? x0 - 4 : x0 + 4;
        __pipeline_memcpy_async(ecslot(s), w.codes + (eok ? (long long)p * w.pitch + wc : 0), 4,
                                eok ? 0 : 4);
      }
    }
  };
  const int nsteps = y1 - y0 + 2;
#pragma unroll
  for (int q = 0; q < kRefRing - 1; ++q) {
    if (q < nsteps) issue(q);
    __pipeline_commit();
  }
  double xu[4] = {0.0, 0.0, 0.0, 0.0}, xc[4] = {0.0, 0.0, 0.0, 0.0};
  unsigned cc = 0u;  // classes of the row in xc (masked)
  for (int q = 0; q < nsteps; ++q) {
    const int s = q & (kRefRing - 1);
    const int yy = y0 - 1 + q;
    const bool rok = yy >= 0 && yy < ny;
    double xd[4], fv[4];
    T dv[4] = {T(0), T(0), T(0), T(0)};
    if constexpr (FAST) {
      bulk::wait(bar + s, (unsigned)(q / kRefRing) & 1u, err);
      __pipeline_wait_prior(kRefRing - 2);
      const unsigned char *slot = brow + s * SM::SB;
      const bool pok = yy - 1 >= y0;
      if (rok && !w.xz) {
        read_row4(xd, slot + lane * 32, slot + lane * 32 + 16);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) xd[j] = 0.0;
      }
      if (pok) {
        read_row4(fv, slot + 1024 + lane * 32, slot + 1024 + lane * 32 + 16);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) fv[j] = 0.0;
      }
      if (FOLD && rok) {
        const V4<T> t = ld4(reinterpret_cast<const T *>(slot + 2048) + 4 * lane);
#pragma unroll
        for (int j = 0; j < 4; ++j) dv[j] = t.v[j];
      }
    } else {
      __pipeline_wait_prior(kRefRing - 2);
      read_row4(xd, chunk(s, 0), chunk(s, 1));
      read_row4(fv, chunk(s, 2), chunk(s, 3));
      if constexpr (FOLD) {
        if constexpr (sizeof(T) == 4) {
          const float4 t = *reinterpret_cast<const float4 *>(chunk(s, 4));
          dv[0] = t.x; dv[1] = t.y; dv[2] = t.z; dv[3] = t.w;
        } else {
          const double2 t0 = *reinterpret_cast<const double2 *>(chunk(s, 4));
          const double2 t1 = *reinterpret_cast<const double2 *>(chunk(s, 5));
          dv[0] = t0.x; dv[1] = t0.y; dv[2] = t1.x; dv[3] = t1.y;
        }
      }
    }
    const unsigned cw = masked ? *cslot(s) : 0u;
    double ex = 0.0, ed = 0.0;
    unsigned ecw = 0u;
    if (edge_lane) {
      ex = *reinterpret_cast<const double *>(eslot(s));
      if constexpr (FOLD) ed = (double)*reinterpret_cast<const T *>(eslot(s) + 8);
      if (masked) ecw = *ecslot(s);
    }
    if (q + kRefRing - 1 < nsteps) {
      if constexpr (FAST) {
        __syncwarp();  // every lane has read the slot refilled now (step q - 1's)
        if (lane == 0) bulk::proxy_fence();
      }
      issue(q + kRefRing - 1);
    }
    __pipeline_commit();
    // x' of row yy, zero where there is no unknown
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const bool on = FAST || (rok && j < nv && (!masked || ((cw >> (8 * j)) & 0xffu) != 0u));
      xd[j] = on ? xd[j] + (double)dv[j] : 0.0;
    }
    if (q >= 2) {  // row p = yy - 1 has x' above, at and below it
      const int p = yy - 1;
      bool eon = true;
      if (!FAST && edge_lane) {
        eon = w.ecol_in;
        if (masked) eon = eon && ((lane == 0 ? (ecw >> 24) : ecw) & 0xffu) != 0u;
      }
      const double ev = eon ? ex + ed : 0.0;
      double left = shfl_up1(xc[3]), right = shfl_dn1(xc[0]);
      if (lane == 0) left = ev;
      if (lane == 31) right = ev;
      const double rowd = (double)((p == 0) + (p == ny - 1)) * w.omw;
      double res[4], fq[4];
      bool on[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        double dg = dgc[j] - rowd;
        on[j] = FAST || j < nv;
        if (masked) {
          const int c = (int)((cc >> (8 * j)) & 0xffu);
          on[j] = on[j] && c != 0;
          dg = 4.0 - (double)(c - 1) * w.omw;
        }
        const double lf = j == 0 ? left : xc[j - 1];
        const double rt = j == 3 ? right : xc[j + 1];
        fq[j] = on[j] ? w.scale * (fv[j] - w.fmean) : 0.0;
        res[j] = on[j] ? fq[j] - (dg * xc[j] - ((xu[j] + xd[j]) + (lf + rt))) : 0.0;
      }
      part += (res[0] * res[0] + res[1] * res[1]) + (res[2] * res[2] + res[3] * res[3]);
      if (INIT) part_f += (fq[0] * fq[0] + fq[1] * fq[1]) + (fq[2] * fq[2] + fq[3] * fq[3]);
      V4<T> rv;
#pragma unroll
      for (int j = 0; j < 4; ++j) rv.v[j] = (T)res[j];
      if (FAST || nv > 0) st4(w.R + (long long)p * w.pitch + x0, rv);
      if constexpr (FOLD) {
        part_f += (xc[0] + xc[1]) + (xc[2] + xc[3]);  // the solution's sum, for its mean
        double *drow = w.dst + p * w.dpitch + x0;
        if (FAST || (nv == 4 && (reinterpret_cast<uintptr_t>(drow) & 15) == 0)) {
          *reinterpret_cast<double2 *>(drow) = make_double2(xc[0], xc[1]);
          *reinterpret_cast<double2 *>(drow + 2) = make_double2(xc[2], xc[3]);
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (j < nv) drow[j] = xc[j];
        }
      }
      if (INIT && masked && !w.xz) {  // the caller's x is zero where there is no unknown
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nv && !on[j]) w.X[p * w.upitch + x0 + j] = 0.0;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      xu[j] = xc[j];
      xc[j] = xd[j];
    }
    cc = cw;
  }
  __pipeline_wait_prior(0);  // no copy may land after the shared memory is released
}

// Initial residual of a zero-start solve: with x = 0, r = scale (f - fmean)
// where there is an unknown, no stencil, and ||r||^2 = ||f'||^2.  Element-wise
// over the warp's rows with eight rows' loads in flight per thread.
template <typename T>
__device__ __forceinline__ void init_zero_rows(const RefWarp<T> &w, double &part,
                                               double &part_f) {
  const int x0 = w.x0, nv = w.nv;
  if (nv <= 0) return;
  constexpr int K = 8;
  for (int yb = w.y0; yb < w.y1; yb += K) {
    double fv[K][4];
    unsigned cw[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int y = yb + k;
      cw[k] = 0u;
#pragma unroll
      for (int j = 0; j < 4; ++j) fv[k][j] = 0.0;
      if (y < w.y1) {
        const double *row = w.F + y * w.upitch + x0;
        if (nv == 4 && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
          const double2 a0 = *reinterpret_cast<const double2 *>(row);
          const double2 a1 = *reinterpret_cast<const double2 *>(row + 2);
          fv[k][0] = a0.x; fv[k][1] = a0.y; fv[k][2] = a1.x; fv[k][3] = a1.y;
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (j < nv) fv[k][j] = row[j];
        }
        if (w.masked)
          cw[k] = *reinterpret_cast<const unsigned *>(w.codes + (long long)y * w.pitch + x0);
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int y = yb + k;
      if (y >= w.y1) break;
      V4<T> rv;
      double fq[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const bool on = j < nv && (!w.masked || ((cw[k] >> (8 * j)) & 0xffu) != 0u);
        fq[j] = on ? w.scale * (fv[k][j] - w.fmean) : 0.0;
        rv.v[j] = (T)fq[j];
      }
      // grouped as the stencil path groups its squares, so both give the same bits
      const double sq = (fq[0] * fq[0] + fq[1] * fq[1]) + (fq[2] * fq[2] + fq[3] * fq[3]);
      part += sq;
      part_f += sq;
      st4(w.R + (long long)y * w.pitch + x0, rv);
    }
  }
}

template <typename T, bool INIT>
__global__ void __launch_bounds__(kThreads, 4) k_refresh_s(Args<T> a) {
  const Tile tl = a.tiles[blockIdx.x];
  dep_enter();
  const int flags = a.st[tl.inst].flags;
  const bool work = INIT || (flags & FLAG_RU);
  double part = 0.0, part_f = 0.0;
  extern __shared__ __align__(16) unsigned char smem[];
  if (work) {
    // descriptor fields in registers: the stores below could alias the descriptor
    const InstInfo &Ig = a.inst[tl.inst];
    const LevelInfo L = a.lv[Ig.level0];
    const bool own = !INIT && a.st[tl.inst].xcur != 0;
    double *const XS = a.xs + Ig.xs_off;
    RefWarp<T> w;
    w.X = Ig.x;
    w.upitch = Ig.upitch;
    w.src = own ? XS : w.X;
    w.spitch = own ? (long long)L.pitch : w.upitch;
    w.dst = own ? w.X : XS;
    w.dpitch = own ? w.upitch : (long long)L.pitch;
    w.F = Ig.f;
    w.D = a.arena + Ig.d_off;
    w.R = a.arena + Ig.r_off;
    w.masked = L.code_off >= 0;
    w.codes = a.codes + (w.masked ? L.code_off : 0);
    w.ny = L.ny;
    w.nx = L.nx;
    w.pitch = L.pitch;
    w.scale = Ig.scale;
    w.fmean = a.st[tl.inst].fmean;
    w.omw = 1.0 - (double)L.wall;
    w.xz = INIT ? a.zero_start != 0 : a.st[tl.inst].xzero != 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col0 = tl.tx * kFTX;
    w.x0 = col0 + 4 * lane;
    w.nv = max(0, min(4, w.nx - w.x0));
    w.y0 = tl.ty * kFTY + warp * kKrylovRows;
    w.y1 = min(w.y0 + kKrylovRows, w.ny);
    w.ecol = lane == 0 ? w.x0 - 1 : w.x0 + 4;
    w.ecol_in = w.ecol >= 0 && w.ecol < w.nx;
    unsigned *const err = a.counter + kErrWord;
    if (w.y0 < w.ny) {
      const bool fast = !w.masked && col0 + kFTX <= w.nx &&
                        ((reinterpret_cast<uintptr_t>(w.X) | reinterpret_cast<uintptr_t>(w.F)) &
                         15) == 0 &&
                        (w.upitch & 1) == 0;
      if constexpr (INIT) {
        if (w.xz) init_zero_rows<T>(w, part, part_f);
        else if (fast) refresh_strip<T, true, false, true>(w, smem, err, part, part_f);
        else refresh_strip<T, true, false, false>(w, smem, err, part, part_f);
      } else if (!(flags & FLAG_DZERO)) {
        if (fast) refresh_strip<T, false, true, true>(w, smem, err, part, part_f);
        else refresh_strip<T, false, true, false>(w, smem, err, part, part_f);
      } else {
        if (fast) refresh_strip<T, false, false, true>(w, smem, err, part, part_f);
        else refresh_strip<T, false, false, false>(w, smem, err, part, part_f);
      }
    }
    part = block_sum<kThreads>(part);
    __syncthreads();
    part_f = block_sum<kThreads>(part_f);
  }
  if (threadIdx.x == 0) {
    a.part0[blockIdx.x] = part;
    a.part1[blockIdx.x] = part_f;  // INIT: ||f||^2; a refresh that folds: the sum of x + d
  }
  if (!last_block(a.counter + 2)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int active = 0;
  for (int i = warp; i < a.ninst; i += kWarps) {
    InstState &S = a.st[i];
    const InstInfo &I = a.inst[i];
    const bool part_of = INIT || (S.flags & FLAG_RU);
    if (part_of) {
      const double rr = warp_range_sum(a.part0, I.fine_begin, I.fine_end);
      const double p1 = warp_range_sum(a.part1, I.fine_begin, I.fine_end);
      if (lane == 0) {
        if (INIT) {
          S.ff = p1;
          S.mean = 0.0;
          S.mean_known = a.zero_start;  // a zero start has mean zero
          S.iters = 0;
          S.first = 1;
          S.rz = 0.0;
          S.beta = 0.0;
          S.pcur = 0;
          S.xcur = 0;
          S.xzero = a.zero_start;
          S.refreshes = 0;
          S.status = GD_ACTIVE;
        } else {
          S.refreshes += 1;
          if (!(S.flags & FLAG_DZERO)) {
            S.xcur ^= 1;  // x + d went to the other copy
            S.xzero = 0;
            S.mean = p1 / ((double)I.ny * (double)I.nx);  // of the new solution
            S.mean_known = 1;
          }
        }
        // A refresh that barely lowers the true residual (less than 3x), once
        // it is already below 1e-6 of ||f||, means the FP64 rounding floor is
        // reached: stop with the current iterate instead of iterating on noise.
        const bool stalled = !INIT && rr > 0.1 * S.rr_prev && rr <= 1e-12 * S.ff;
        if (INIT || rr < S.rr_prev) S.rr_prev = rr;
        S.rr_true = rr;
        S.rr_ref = rr;
        S.rr = rr;
        if (rr <= a.tol2 * S.ff) {
          S.status = GD_CONVERGED;
        } else if (!isfinite(rr)) {
          S.status = GD_BREAKDOWN;
        } else if (S.status == GD_ACTIVE && stalled) {
          S.status = GD_STAGNATED;
        } else if (S.status == GD_ACTIVE && S.iters >= a.max_iter) {
          S.status = GD_MAX_ITERATIONS;
        }
        S.flags = FLAG_DZERO;  // the correction restarts after every refresh
      }
    }
    if (lane == 0 && S.status == GD_ACTIVE) ++active;
  }
  __shared__ int cnt[kWarps];
  if (lane == 0) cnt[warp] = active;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kWarps; ++w) t += cnt[w];
    *a.n_active = t;
  }
}

}  // namespace st
}  // namespace gd
