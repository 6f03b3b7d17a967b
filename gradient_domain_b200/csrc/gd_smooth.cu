// Temporally blocked red-black Gauss-Seidel: `sweeps` (1-4) sweeps of
// multigrid._smooth (gradient-domain/src/gradient_domain/multigrid.py:147-165)
// in one pass over memory: u and b are read once, the result written once.
//
// The reference updates the cells with (i + j) % 2 == 0, then those with
// (i + j) % 2 == 1, each as u = 0.25 * (((up + down) + left) + right - h^2 b)
// with zeros outside the array.  The kernel evaluates exactly that expression
// with round-to-nearest intrinsics (no FMA contraction), so its FP64 result is
// bitwise the reference's and its FP32 result bitwise the same expression
// evaluated in float32.
//
// Layout of the work: a warp owns 128 columns (4 per lane) of a band of rows
// and walks the band one row at a time with the rows it still needs in a
// register window; the 2 * sweeps half sweeps are pipelined down the window
// (half sweep g runs on the row g steps behind the newest one).  Each half
// sweep widens the set of cells that depend on data outside the warp by one
// column and one row, so the outer lanes ("halo lanes") and the first rows of
// a band are recomputed, never written.  Even bands walk down and odd bands
// walk up: two neighbouring bands then load the rows they share at the same
// time (both at their start, or both at their end), and the second load is
// served by L2 instead of HBM; neighbouring strips of a band share their halo
// columns the same way.  Rows are prefetched into registers (U rows ahead for
// FP32, 2 for FP64); the b values of the window sit in shared memory.

#include <algorithm>
#include <atomic>

#include "gd_internal.cuh"

namespace gd {
namespace {

constexpr int kSmThreads = 128;  // four warps per CTA

template <typename T>
struct Q4 {
  T v[4];
};

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

template <int S>
struct SmGeom {
  static constexpr int R = 2 * S;               // half sweeps = rows and columns of dependency
  static constexpr int HL = (R + 3) / 4;        // halo lanes on each side of a warp
  static constexpr int OW = 4 * (32 - 2 * HL);  // columns a warp writes
  static constexpr int U = R + 2;               // rows in the window (even)
};

template <typename T>
struct SmoothArgs {
  const T *u;
  T *out;
  const T *b;
  int ny, nx, pitch;
  T h2;
  int rows;    // output rows per band (even)
  int strips;  // strips across the width
  int items;   // strips * bands
};

// Row y, columns x0 .. x0 + 3 of A; zero outside the array.  VEC: rows are
// 16-byte aligned, so an in-range group is one (FP32) or two (FP64) vector loads.
template <typename T, bool VEC, bool INT>
__device__ __forceinline__ Q4<T> load4(const T *A, const SmoothArgs<T> &a, int y, int x0) {
  Q4<T> q;
  if (INT || (y >= 0 && y < a.ny && x0 >= 0 && x0 + 3 < a.nx)) {
    const T *p = A + (long long)y * a.pitch + x0;
    if (VEC) {
      if (sizeof(T) == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
        q.v[0] = (T)t.x; q.v[1] = (T)t.y; q.v[2] = (T)t.z; q.v[3] = (T)t.w;
      } else {
        const double2 t0 = __ldg(reinterpret_cast<const double2 *>(p));
        const double2 t1 = __ldg(reinterpret_cast<const double2 *>(p) + 1);
        q.v[0] = (T)t0.x; q.v[1] = (T)t0.y; q.v[2] = (T)t1.x; q.v[3] = (T)t1.y;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) q.v[j] = __ldg(p + j);
    }
    return q;
  }
  const bool row_ok = y >= 0 && y < a.ny;
  const T *p = A + (long long)(row_ok ? y : 0) * a.pitch;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int x = x0 + j;
    q.v[j] = (row_ok && x >= 0 && x < a.nx) ? __ldg(p + x) : T(0);
  }
  return q;
}

// One half sweep on row window entry u (row r); J0 = first updated cell of the
// lane, (r + J0) % 2 == colour; bq = the lane's four b values of row r.
// `inside` has bit j set where (r, x0 + j) is a cell of the array; the other
// cells keep their zero.
template <int J0, typename T>
__device__ __forceinline__ void half_row(Q4<T> &u, const Q4<T> &nb1, const Q4<T> &nb2,
                                         const T *bq, T h2, unsigned inside) {
  // one 16-byte read per lane (FP32; two for FP64): a warp reads 512 contiguous
  // bytes without bank conflicts, where scalar reads at a 16-byte stride conflict 4-way
  T bv[4];
  if (sizeof(T) == 4) {
    const float4 t = *reinterpret_cast<const float4 *>(bq);
    bv[0] = (T)t.x; bv[1] = (T)t.y; bv[2] = (T)t.z; bv[3] = (T)t.w;
  } else {
    const double2 t0 = reinterpret_cast<const double2 *>(bq)[0];
    const double2 t1 = reinterpret_cast<const double2 *>(bq)[1];
    bv[0] = (T)t0.x; bv[1] = (T)t0.y; bv[2] = (T)t1.x; bv[3] = (T)t1.y;
  }
  T side;
  if (J0 == 0) side = __shfl_up_sync(0xffffffffu, u.v[3], 1);  // column x0 - 1
  else side = __shfl_down_sync(0xffffffffu, u.v[0], 1);        // column x0 + 4
#pragma unroll
  for (int j = J0; j < 4; j += 2) {
    const T left = j == 0 ? side : u.v[j - 1];
    const T right = j == 3 ? side : u.v[j + 1];
    // ((up + down) + left) + right; up + down commutes exactly, whichever walk direction
    const T s = add_rn(add_rn(add_rn(nb1.v[j], nb2.v[j]), left), right);
    const T v = mul_rn(T(0.25), sub_rn(s, mul_rn(h2, bv[j])));
    if (inside & (1u << j)) u.v[j] = v;
  }
}

// The lane's four values to q (16-byte aligned): its slot of the warp's b window,
// or an output row of a vector-aligned array.
template <typename T>
__device__ __forceinline__ void put4(T *q, const Q4<T> &v) {
  if (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(q) =
        make_float4((float)v.v[0], (float)v.v[1], (float)v.v[2], (float)v.v[3]);
  } else {
    reinterpret_cast<double2 *>(q)[0] = make_double2((double)v.v[0], (double)v.v[1]);
    reinterpret_cast<double2 *>(q)[1] = make_double2((double)v.v[2], (double)v.v[3]);
  }
}

template <int U>
__device__ __forceinline__ constexpr int sl(int ph, int k) {
  return ((ph - k) % U + U) % U;
}

// Rows of prefetch in registers: U for FP32, 2 for FP64 (both divide the even U).
// (Measured alternatives for one FP32 sweep on 4096^2: eight rows need 157
// registers, or spill at 128; a per-lane cp.async ring in shared memory with five
// rows in flight at 59 registers was 3-7 % slower.)
template <typename T, int S>
struct SmPrefetch {
  static constexpr int P = sizeof(T) == 4 ? SmGeom<S>::U : 2;
};

// bw: this warp's b window in shared memory, U rows of 128 values; a lane only
// reads back the values it stored itself, so no barrier is needed.
template <typename T, int S, bool VEC, bool INT, bool DOWN>
__device__ __forceinline__ void smooth_band(const SmoothArgs<T> &a, T *bw, int x0, bool out_lane,
                                            unsigned colmask, int y_out0, int y_out1) {
  using G = SmGeom<S>;
  constexpr int U = G::U, R = G::R, P = SmPrefetch<T, S>::P;
  static_assert(U % P == 0, "prefetch depth must divide the window");
  const int lane = threadIdx.x & 31;
  T *bl = bw + 4 * lane;
  // first row loaded (even, so the window phase has the row's parity) and the step count
  const int y_first = DOWN ? ((y_out0 - R) & ~1) : ((y_out1 - 1 + R + 1) & ~1);
  const int y_end = DOWN ? y_out1 - 1 + R : y_out0 - R;
  const int nsteps = DOWN ? y_end - y_first + 1 : y_first - y_end + 1;
  Q4<T> Uw[U], Pu[P], Pb[P];
#pragma unroll
  for (int k = 0; k < U; ++k) {
#pragma unroll
    for (int j = 0; j < 4; ++j) Uw[k].v[j] = T(0);
    put4(bl + k * 128, Uw[k]);
  }
#pragma unroll
  for (int k = 0; k < P; ++k) {
    const int y = DOWN ? y_first + k : y_first - k;
    Pu[k] = load4<T, VEC, INT>(a.u, a, y, x0);
    Pb[k] = load4<T, VEC, INT>(a.b, a, y, x0);
  }
  for (int base = 0; base < nsteps; base += U) {
#pragma unroll
    for (int ph = 0; ph < U; ++ph) {
      const int step = base + ph;
      if (step >= nsteps) break;
      const int y = DOWN ? y_first + step : y_first - step;
      Uw[ph] = Pu[ph % P];
      put4(bl + ph * 128, Pb[ph % P]);
      if (step + P < nsteps) {
        const int yp = DOWN ? y + P : y - P;
        Pu[ph % P] = load4<T, VEC, INT>(a.u, a, yp, x0);
        Pb[ph % P] = load4<T, VEC, INT>(a.b, a, yp, x0);
      }
      // half sweep g (colour (g - 1) & 1) on the row g steps back: its first updated
      // cell is ((g - 1) + (y -+ g)) & 1 = (y + 1) & 1 = (ph + 1) & 1 for every g
#pragma unroll
      for (int g = 1; g <= R; ++g) {
        const int yg = DOWN ? y - g : y + g;
        const unsigned inside = INT ? 0xfu : ((yg >= 0 && yg < a.ny) ? colmask : 0u);
        const T *bq = bl + sl<U>(ph, g) * 128;
        if ((ph & 1) == 0)
          half_row<1, T>(Uw[sl<U>(ph, g)], Uw[sl<U>(ph, g - 1)], Uw[sl<U>(ph, g + 1)], bq, a.h2,
                         inside);
        else
          half_row<0, T>(Uw[sl<U>(ph, g)], Uw[sl<U>(ph, g - 1)], Uw[sl<U>(ph, g + 1)], bq, a.h2,
                         inside);
      }
      const int yo = DOWN ? y - R : y + R;
      if (out_lane && yo >= y_out0 && yo < y_out1) {
        const Q4<T> &v = Uw[sl<U>(ph, R)];
        T *dst = a.out + (long long)yo * a.pitch + x0;
        if (VEC && x0 + 3 < a.nx) {
          put4(dst, v);
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (x0 + j < a.nx) dst[j] = v.v[j];
        }
      }
    }
  }
}

template <typename T, int S, bool VEC>
__global__ void __launch_bounds__(kSmThreads) k_rbgs(SmoothArgs<T> a) {
  using G = SmGeom<S>;
  __shared__ __align__(16) T b_window[kSmThreads / 32][G::U * 128];
  const int lane = threadIdx.x & 31;
  T *bw = b_window[threadIdx.x >> 5];
  const int nwarps = gridDim.x * (kSmThreads / 32);
  for (int item = (blockIdx.x * kSmThreads + threadIdx.x) >> 5; item < a.items; item += nwarps) {
    const int sx = item % a.strips, band = item / a.strips;
    const int y_out0 = band * a.rows;
    const int y_out1 = min(y_out0 + a.rows, a.ny);
    const int xw = sx * G::OW - 4 * G::HL;  // first column of the warp (multiple of 4)
    const int x0 = xw + 4 * lane;
    const bool out_lane = lane >= G::HL && lane < 32 - G::HL && x0 < a.nx;
    unsigned colmask = 0u;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (x0 + j >= 0 && x0 + j < a.nx) colmask |= 1u << j;
    const bool down = (band & 1) == 0;
    // every loaded row and column inside the array: no masks, no per-element checks
    const bool interior = y_out0 - G::R - 1 >= 0 && y_out1 + G::R + 1 <= a.ny && xw >= 0 &&
                          xw + 127 < a.nx;
    if (interior) {
      if (down) smooth_band<T, S, VEC, true, true>(a, bw, x0, out_lane, colmask, y_out0, y_out1);
      else smooth_band<T, S, VEC, true, false>(a, bw, x0, out_lane, colmask, y_out0, y_out1);
    } else {
      if (down) smooth_band<T, S, VEC, false, true>(a, bw, x0, out_lane, colmask, y_out0, y_out1);
      else smooth_band<T, S, VEC, false, false>(a, bw, x0, out_lane, colmask, y_out0, y_out1);
    }
  }
}

// Kernel kinds: 0 scalar global accesses, 1 vector accesses (16-byte aligned rows).
template <typename T, int S, int KIND>
constexpr auto kernel_of() {
  return &k_rbgs<T, S, KIND == 1>;
}

// Resident CTAs per SM of one kernel, looked up once.
template <typename T, int S, int KIND>
int resident_ctas() {
  static std::atomic<int> cached{0};
  int v = cached.load(std::memory_order_relaxed);
  if (v > 0) return v;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_of<T, S, KIND>(), kSmThreads, 0) !=
          cudaSuccess ||
      n <= 0)
    n = 1;
  cached.store(n, std::memory_order_relaxed);
  return n;
}

template <typename T, int S, int KIND>
int launch_rbgs(const T *u, T *out, const T *b, int ny, int nx, int pitch, double spacing,
                cudaStream_t st) {
  using G = SmGeom<S>;
  int dev = 0, sms = 0;
  GD_CHECK_CUDA(cudaGetDevice(&dev));
  GD_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int ctas = resident_ctas<T, S, KIND>() * sms;
  SmoothArgs<T> a;
  a.u = u;
  a.out = out;
  a.b = b;
  a.ny = ny;
  a.nx = nx;
  a.pitch = pitch;
  a.h2 = (T)(spacing * spacing);
  a.strips = ceil_div(nx, G::OW);
  // one band per resident warp where the grid allows it, at least 4 R rows tall
  const int warps = ctas * (kSmThreads / 32);
  const int bands_target = std::max(1, warps / a.strips);
  int rows = ceil_div(ny, bands_target);
  rows = std::max(rows, 4 * G::R);
  rows = (rows + 1) & ~1;
  a.rows = rows;
  const long long items = (long long)a.strips * ceil_div(ny, rows);
  GD_REQUIRE(items < (1ll << 30), GD_ERR_ARG, "gd_rbgs_smooth: grid too large");
  a.items = (int)items;
  const int grid = (int)std::min<long long>(ceil_div(a.items, kSmThreads / 32), ctas);
  kernel_of<T, S, KIND>()<<<grid, kSmThreads, 0, st>>>(a);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

template <typename T>
int dispatch(const T *u, T *out, const T *b, int ny, int nx, int pitch, double spacing,
             int sweeps, cudaStream_t st) {
  const bool vec = (reinterpret_cast<uintptr_t>(u) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(b) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(out) & 15) == 0 &&
                   ((size_t)pitch * sizeof(T)) % 16 == 0;
#define GD_RBGS_CASE(S)                                                           \
  case S:                                                                         \
    return vec ? launch_rbgs<T, S, 1>(u, out, b, ny, nx, pitch, spacing, st)      \
               : launch_rbgs<T, S, 0>(u, out, b, ny, nx, pitch, spacing, st);
  switch (sweeps) {
    GD_RBGS_CASE(1)
    GD_RBGS_CASE(2)
    GD_RBGS_CASE(3)
    GD_RBGS_CASE(4)
  }
#undef GD_RBGS_CASE
  set_error("gd_rbgs_smooth: sweeps must be 1 to 4 per call (got %d)", sweeps);
  return GD_ERR_ARG;
}

}  // namespace
}  // namespace gd

extern "C" int gd_rbgs_smooth(const void *u, void *out, const void *b, int32_t ny, int32_t nx,
                              int32_t pitch, int32_t fp64, double spacing, int32_t sweeps,
                              cudaStream_t stream) {
  GD_REQUIRE(u && out && b && ny > 0 && nx > 0 && pitch >= nx && (fp64 == 0 || fp64 == 1),
             GD_ERR_ARG, "gd_rbgs_smooth: bad arguments");
  GD_REQUIRE(out != u && out != b, GD_ERR_ARG,
             "gd_rbgs_smooth: out must not be u or b (the sweeps read neighbouring columns "
             "and rows that other warps write)");
  if (fp64)
    return gd::dispatch<double>(static_cast<const double *>(u), static_cast<double *>(out),
                                static_cast<const double *>(b), ny, nx, pitch, spacing, sweeps,
                                stream);
  return gd::dispatch<float>(static_cast<const float *>(u), static_cast<float *>(out),
                             static_cast<const float *>(b), ny, nx, pitch, spacing, sweeps,
                             stream);
}
