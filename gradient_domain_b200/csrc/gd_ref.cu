// Reference-exact vertex-centred FP64 multigrid (the "port-equivalent" path).
//
// These kernels reproduce gradient-domain/src/gradient_domain/multigrid.py
// operation by operation: red-black Gauss-Seidel with colour (i + j) % 2 == 0
// first (multigrid.py:147-165), full-weighting restriction (:169-174) and
// bilinear prolongation (:177-181) on the m -> (m - 1) // 2 hierarchy, and the
// coarsest-grid sweeps (:205-207).  Arithmetic uses explicit round-to-nearest
// intrinsics in the same order as the NumPy/SciPy expressions, so no FMA
// contraction changes the result; products by 0.5, 0.25 and 1.0 are exact.
// They are plain one-pass-per-operation kernels on purpose: this path is the
// all-FP64 GPU translation of the reference that the fused solver is measured
// against, and the parity hook for v_cycle / multigrid.solve.

#include <mutex>

#include "gd_internal.cuh"

namespace gd {
namespace {

__device__ __forceinline__ double at(const double *a, int i, int j, int m, int n) {
  return (i >= 0 && i < m && j >= 0 && j < n) ? a[(size_t)i * n + j] : 0.0;
}

// neighbours = up + down + left + right, evaluated left to right (operators.py:104-106).
__device__ __forceinline__ double nbr_sum(const double *u, int i, int j, int m, int n) {
  double s = __dadd_rn(at(u, i - 1, j, m, n), at(u, i + 1, j, m, n));
  s = __dadd_rn(s, at(u, i, j - 1, m, n));
  return __dadd_rn(s, at(u, i, j + 1, m, n));
}

// One colour of one RB-GS sweep: u = 0.25 * (neighbours - h^2 b) on parity cells.
__global__ void ref_rb_colour(double *__restrict__ u, const double *__restrict__ b, int m, int n,
                              double h2, int parity) {
  const int half = (n + 1) / 2;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)m * half) return;
  const int i = (int)(k / half);
  const int j = 2 * (int)(k % half) + ((parity + i) & 1);
  if (j >= n) return;
  const double s = nbr_sum(u, i, j, m, n);
  u[(size_t)i * n + j] = __dmul_rn(0.25, __dsub_rn(s, __dmul_rn(h2, b[(size_t)i * n + j])));
}

// r = b - (neighbours - 4 u) / h^2  (multigrid.py:210 with operators.py:107).
__global__ void ref_residual_kernel(double *__restrict__ r, const double *__restrict__ u,
                                    const double *__restrict__ b, int m, int n, double h2) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)m * n) return;
  const int i = (int)(k / n), j = (int)(k % n);
  const double lap = __ddiv_rn(__dsub_rn(nbr_sum(u, i, j, m, n), __dmul_rn(4.0, u[k])), h2);
  r[k] = __dsub_rn(b[k], lap);
}

// rc = 0.25 * Rows^T r Cols: rows first (fine rows 2I, 2I+1, 2I+2 in order),
// then columns, as scipy's csc products accumulate them.
__global__ void ref_restrict_kernel(double *__restrict__ rc, const double *__restrict__ r, int m,
                                    int n, int mc, int nc) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)mc * nc) return;
  const int I = (int)(k / nc), J = (int)(k % nc);
  double t[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int j = 2 * J + q;
    const double *c = r + j;
    double s = __dmul_rn(0.5, c[(size_t)(2 * I) * n]);
    s = __dadd_rn(s, c[(size_t)(2 * I + 1) * n]);
    t[q] = __dadd_rn(s, __dmul_rn(0.5, c[(size_t)(2 * I + 2) * n]));
  }
  double s = __dadd_rn(__dmul_rn(0.5, t[0]), t[1]);
  s = __dadd_rn(s, __dmul_rn(0.5, t[2]));
  rc[k] = __dmul_rn(s, 0.25);
}

// Interpolate one fine index from the coarse axis: returns the count of
// contributing coarse indices (c0, c1) and their weight.
__device__ __forceinline__ int prolong_sources(int i, int nc, int *c0, int *c1, double *w) {
  if (i & 1) {
    const int s = (i - 1) >> 1;
    *c0 = s;
    *w = 1.0;
    return (s >= 0 && s < nc) ? 1 : 0;
  }
  int cnt = 0;
  const int a = (i >> 1) - 1, b = i >> 1;
  *w = 0.5;
  if (a >= 0 && a < nc) { *c0 = a; cnt = 1; }
  if (b >= 0 && b < nc) {
    if (cnt == 0) *c0 = b; else *c1 = b;
    ++cnt;
  }
  return cnt;
}

// u += Rows e Cols^T: inner sum over coarse rows, then coarse columns.
__global__ void ref_prolong_add_kernel(double *__restrict__ u, const double *__restrict__ e, int m,
                                       int n, int mc, int nc) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)m * n) return;
  const int i = (int)(k / n), j = (int)(k % n);
  int ri0 = 0, ri1 = 0, cj0 = 0, cj1 = 0;
  double wi, wj;
  const int ni = prolong_sources(i, mc, &ri0, &ri1, &wi);
  const int nj = prolong_sources(j, nc, &cj0, &cj1, &wj);
  double total = 0.0;
  if (ni > 0 && nj > 0) {
    double col[2];
    const int cj[2] = {cj0, cj1};
    for (int q = 0; q < nj; ++q) {
      double s = __dmul_rn(wi, e[(size_t)ri0 * nc + cj[q]]);
      if (ni == 2) s = __dadd_rn(s, __dmul_rn(wi, e[(size_t)ri1 * nc + cj[q]]));
      col[q] = s;
    }
    total = __dmul_rn(wj, col[0]);
    if (nj == 2) total = __dadd_rn(total, __dmul_rn(wj, col[1]));
  }
  u[k] = __dadd_rn(u[k], total);
}

// Coarsest grid: `sweeps` RB-GS sweeps by one CTA (multigrid.py:205-207).
// Uses shared memory when the grid fits, global memory otherwise.
constexpr int kCoarseThreads = 1024;
constexpr int kCoarseSmemCells = 2560;  // 2 arrays x 8 B x 2560 = 40 KB

__global__ void __launch_bounds__(kCoarseThreads)
ref_coarse_kernel(double *__restrict__ u_g, const double *__restrict__ b_g, int m, int n,
                  double h2, int sweeps) {
  __shared__ double su[kCoarseSmemCells], sb[kCoarseSmemCells];
  const int cells = m * n;
  const bool in_smem = cells <= kCoarseSmemCells;
  double *u = in_smem ? su : u_g;
  const double *b = in_smem ? sb : b_g;
  if (in_smem) {
    for (int k = threadIdx.x; k < cells; k += blockDim.x) {
      su[k] = u_g[k];
      sb[k] = b_g[k];
    }
  }
  __syncthreads();
  const int half = (n + 1) / 2;
  for (int s = 0; s < sweeps; ++s) {
    for (int parity = 0; parity < 2; ++parity) {
      for (int k = threadIdx.x; k < m * half; k += blockDim.x) {
        const int i = k / half;
        const int j = 2 * (k % half) + ((parity + i) & 1);
        if (j < n) {
          const double nb = nbr_sum(u, i, j, m, n);
          u[i * n + j] = __dmul_rn(0.25, __dsub_rn(nb, __dmul_rn(h2, b[i * n + j])));
        }
      }
      __syncthreads();
      if (!in_smem) __threadfence_block();
    }
  }
  if (in_smem)
    for (int k = threadIdx.x; k < cells; k += blockDim.x) u_g[k] = su[k];
}

constexpr int kReduceThreads = 256;
constexpr int kReduceBlocks = 592;  // 4 x 148 SMs

__global__ void __launch_bounds__(kReduceThreads)
ref_dot_partial(double *__restrict__ part, const double *__restrict__ a,
                const double *__restrict__ b, long long count) {
  double s = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x)
    s += a[k] * b[k];
  s = block_sum<kReduceThreads>(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kReduceThreads)
ref_dot_final(double *__restrict__ out, const double *__restrict__ part, int nparts) {
  double s = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) s += part[k];
  s = block_sum<kReduceThreads>(s);
  if (threadIdx.x == 0) out[0] = s;
}

__global__ void ref_axpby_kernel(double *__restrict__ y, const double *__restrict__ x, double alpha,
                                 double beta, long long count) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count) y[k] = __dadd_rn(__dmul_rn(alpha, x[k]), __dmul_rn(beta, y[k]));
}

inline unsigned blocks_for(long long work, int threads) {
  return (unsigned)((work + threads - 1) / threads);
}

struct RefLevel {
  int m, n;
  size_t u_off, b_off, r_off;  // byte offsets in the workspace (levels >= 1 use u, b)
};

// Level list of the reference recursion: stops at the first grid that is
// coarsest (min side <= coarsest_size or coarse side < 2).
int ref_levels(int m, int n, int coarsest_size, RefLevel *lv, int max_levels, size_t *bytes) {
  size_t off = 0;
  int count = 0;
  while (true) {
    if (count >= max_levels) return -1;
    RefLevel &L = lv[count++];
    L.m = m;
    L.n = n;
    const size_t cells = (size_t)m * n * sizeof(double);
    L.r_off = off;
    off = align_up(off + cells, 256);
    if (count > 1) {
      L.u_off = off;
      off = align_up(off + cells, 256);
      L.b_off = off;
      off = align_up(off + cells, 256);
    } else {
      L.u_off = L.b_off = 0;
    }
    const int mc = (m - 1) / 2, nc = (n - 1) / 2;
    if (m <= coarsest_size || n <= coarsest_size || mc < 2 || nc < 2) break;
    m = mc;
    n = nc;
  }
  *bytes = off + 1024 * sizeof(double);  // + dot partials
  return count;
}

int ref_vcycle_rec(RefLevel *lv, int nlev, int l, double *u, const double *b, double h,
                   int pre, int post, int sweeps, char *ws, cudaStream_t st) {
  const RefLevel &L = lv[l];
  const int m = L.m, n = L.n, T = 256;
  const double h2 = h * h;
  if (l == nlev - 1) {
    ref_coarse_kernel<<<1, kCoarseThreads, 0, st>>>(u, b, m, n, h2, sweeps);
    GD_CHECK_LAUNCH();
    return GD_OK;
  }
  const unsigned g_col = blocks_for((long long)m * ((n + 1) / 2), T);
  for (int s = 0; s < pre; ++s)
    for (int p = 0; p < 2; ++p) ref_rb_colour<<<g_col, T, 0, st>>>(u, b, m, n, h2, p);
  double *r = (double *)(ws + L.r_off);
  ref_residual_kernel<<<blocks_for((long long)m * n, T), T, 0, st>>>(r, u, b, m, n, h2);
  const RefLevel &C = lv[l + 1];
  double *uc = (double *)(ws + C.u_off);
  double *bc = (double *)(ws + C.b_off);
  ref_restrict_kernel<<<blocks_for((long long)C.m * C.n, T), T, 0, st>>>(bc, r, m, n, C.m, C.n);
  GD_CHECK_LAUNCH();
  GD_CHECK_CUDA(cudaMemsetAsync(uc, 0, (size_t)C.m * C.n * sizeof(double), st));
  int rc = ref_vcycle_rec(lv, nlev, l + 1, uc, bc, 2.0 * h, pre, post, sweeps, ws, st);
  if (rc != GD_OK) return rc;
  ref_prolong_add_kernel<<<blocks_for((long long)m * n, T), T, 0, st>>>(u, uc, m, n, C.m, C.n);
  for (int s = 0; s < post; ++s)
    for (int p = 0; p < 2; ++p) ref_rb_colour<<<g_col, T, 0, st>>>(u, b, m, n, h2, p);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

}  // namespace
}  // namespace gd

using namespace gd;

extern "C" size_t gd_ref_workspace_bytes(int32_t m, int32_t n, int32_t coarsest_size) {
  RefLevel lv[64];
  size_t bytes = 0;
  if (m <= 0 || n <= 0) return 0;
  if (ref_levels(m, n, coarsest_size, lv, 64, &bytes) < 0) return 0;
  return bytes;
}

extern "C" int gd_ref_vcycle(double *u, const double *b, int32_t m, int32_t n, double spacing,
                             int32_t pre, int32_t post, int32_t coarsest_size,
                             int32_t coarsest_sweeps, void *ws, size_t bytes, cudaStream_t st) {
  GD_REQUIRE(u && b && m > 0 && n > 0 && pre >= 0 && post >= 0 && coarsest_sweeps >= 0,
             GD_ERR_ARG, "gd_ref_vcycle: bad arguments");
  RefLevel lv[64];
  size_t need = 0;
  const int nlev = ref_levels(m, n, coarsest_size, lv, 64, &need);
  GD_REQUIRE(nlev > 0, GD_ERR_ARG, "gd_ref_vcycle: hierarchy too deep");
  GD_REQUIRE(ws != nullptr && bytes >= need, GD_ERR_ARG,
             "gd_ref_vcycle: workspace of %zu bytes, need %zu", bytes, need);
  return ref_vcycle_rec(lv, nlev, 0, u, b, spacing, pre, post, coarsest_sweeps, (char *)ws, st);
}

extern "C" int gd_ref_residual(double *r, const double *u, const double *b, int32_t m, int32_t n,
                               double spacing, cudaStream_t st) {
  GD_REQUIRE(r && u && b && m > 0 && n > 0, GD_ERR_ARG, "gd_ref_residual: bad arguments");
  ref_residual_kernel<<<blocks_for((long long)m * n, 256), 256, 0, st>>>(r, u, b, m, n,
                                                                         spacing * spacing);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_ref_dot(double *out, const double *a, const double *b, int64_t count, void *ws,
                          size_t bytes, cudaStream_t st) {
  GD_REQUIRE(out && a && b && count >= 0, GD_ERR_ARG, "gd_ref_dot: bad arguments");
  GD_REQUIRE(ws && bytes >= kReduceBlocks * sizeof(double), GD_ERR_ARG,
             "gd_ref_dot: workspace needs %zu bytes", (size_t)kReduceBlocks * sizeof(double));
  double *part = (double *)ws;
  ref_dot_partial<<<kReduceBlocks, kReduceThreads, 0, st>>>(part, a, b, count);
  ref_dot_final<<<1, kReduceThreads, 0, st>>>(out, part, kReduceBlocks);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_ref_axpby(double *y, const double *x, double alpha, double beta, int64_t count,
                            cudaStream_t st) {
  GD_REQUIRE(y && x && count >= 0, GD_ERR_ARG, "gd_ref_axpby: bad arguments");
  if (count == 0) return GD_OK;
  ref_axpby_kernel<<<blocks_for(count, 256), 256, 0, st>>>(y, x, alpha, beta, count);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_ref_restrict(double *rc, const double *r, int32_t m, int32_t n,
                               cudaStream_t st) {
  GD_REQUIRE(rc && r && m >= 3 && n >= 3, GD_ERR_ARG,
             "gd_ref_restrict: needs a fine grid of at least 3 x 3");
  const int mc = (m - 1) / 2, nc = (n - 1) / 2;
  ref_restrict_kernel<<<blocks_for((long long)mc * nc, 256), 256, 0, st>>>(rc, r, m, n, mc, nc);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_ref_prolong_add(double *u, const double *e, int32_t m, int32_t n, int32_t mc,
                                  int32_t nc, cudaStream_t st) {
  GD_REQUIRE(u && e && m > 0 && n > 0 && mc > 0 && nc > 0, GD_ERR_ARG,
             "gd_ref_prolong_add: bad arguments");
  ref_prolong_add_kernel<<<blocks_for((long long)m * n, 256), 256, 0, st>>>(u, e, m, n, mc, nc);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of gd_ref_vcycle.
//
// Some callers cannot allocate device memory when they need a V-cycle: code
// running while a CUDA stream is being captured into a graph (cudaMalloc is
// not permitted there), real-time loops that forbid allocation after start-up,
// and host applications that own the whole device memory budget and give
// plug-ins no allocator.  gd_ref_vcycle_static takes its coarse-level scratch
// from the file-scope array below instead of a caller workspace.  The array
// is GD_STATIC_SCRATCH_BYTES (4 MiB) on every GPU that loads this library and
// stays allocated until the process exits.  In host code `g_static_scratch`
// names a host-side stand-in, not device memory, so its device address is
// looked up with cudaGetSymbolAddress once per device and cached.
namespace gd {
namespace {

__device__ __align__(256) unsigned char g_static_scratch[GD_STATIC_SCRATCH_BYTES];

constexpr int kMaxStaticDevices = 64;
void *g_static_ptr[kMaxStaticDevices] = {};
std::mutex g_static_mu;

// Device address of g_static_scratch on the current device (looked up once).
int static_scratch(void **out) {
  int dev = 0;
  GD_CHECK_CUDA(cudaGetDevice(&dev));
  GD_REQUIRE(dev >= 0 && dev < kMaxStaticDevices, GD_ERR_UNSUPPORTED,
             "gd_ref_vcycle_static: device %d beyond the %d supported", dev, kMaxStaticDevices);
  std::lock_guard<std::mutex> hold(g_static_mu);
  if (g_static_ptr[dev] == nullptr) {
    void *p = nullptr;
    GD_CHECK_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
    g_static_ptr[dev] = p;
  }
  *out = g_static_ptr[dev];
  return GD_OK;
}

}  // namespace
}  // namespace gd

extern "C" int gd_ref_vcycle_static(double *u, const double *b, int32_t m, int32_t n,
                                    double spacing, int32_t pre, int32_t post,
                                    int32_t coarsest_size, int32_t coarsest_sweeps,
                                    cudaStream_t st) {
  GD_REQUIRE(u && b && m > 0 && n > 0 && pre >= 0 && post >= 0 && coarsest_sweeps >= 0,
             GD_ERR_ARG, "gd_ref_vcycle_static: bad arguments");
  RefLevel lv[64];
  size_t need = 0;
  const int nlev = ref_levels(m, n, coarsest_size, lv, 64, &need);
  GD_REQUIRE(nlev > 0, GD_ERR_ARG, "gd_ref_vcycle_static: hierarchy too deep");
  // a single-level hierarchy is the coarsest solve in place on u: no scratch at all
  void *ws = nullptr;
  if (nlev > 1) {
    GD_REQUIRE(need <= (size_t)GD_STATIC_SCRATCH_BYTES, GD_ERR_ARG,
               "gd_ref_vcycle_static: a %d x %d grid needs %zu bytes of scratch, more than "
               "the %zu-byte static array; use gd_ref_vcycle with a workspace",
               m, n, need, (size_t)GD_STATIC_SCRATCH_BYTES);
    const int rc = static_scratch(&ws);
    if (rc != GD_OK) return rc;
  }
  // ref_vcycle_rec zeroes every coarse iterate before use, so the contents left
  // by the previous call do not leak into this one.
  return ref_vcycle_rec(lv, nlev, 0, u, b, spacing, pre, post, coarsest_sweeps, (char *)ws, st);
}
