// Exact Neumann Poisson solve by the discrete cosine transform: the algorithm
// of solvers.py:224-262 (dctn type 2 "ortho", division by the eigenvalues
// 2 cos(pi i / m) + 2 cos(pi j / n) - 4 with the constant mode dropped, idctn),
// on the device.  An alternative to the MGPCG for rectangles with Neumann
// boundaries and a cross-check of it.
//
// Each 1-D orthonormal DCT-II of length N is one real FFT of length N
// (Makhoul's reordering): v = (x0, x2, x4, ..., x5, x3, x1), V = FFT(v),
// X_k = Re(exp(-i pi k / 2N) V_k) scaled by sqrt(1/N) (k = 0) or sqrt(2/N).
// Its inverse forms W_k = exp(i pi k / 2N) (X_k - i X_{N-k}) from the
// unscaled coefficients, takes the real inverse FFT and undoes the reordering.
// The 2-D transform runs along rows, is transposed (fused into the twiddle
// kernel), runs along the former columns, and the inverse retraces the steps;
// the eigenvalue division is fused into the second twiddle.  FFTs are cuFFT
// (created without automatic work-area allocation); every buffer, the cuFFT
// work area included, is the caller's workspace.

#include <cufft.h>

#include <algorithm>
#include <cstdint>

#include "gd_internal.cuh"

struct gd_dct_plan_s {
  int h = 0, w = 0;
  cufftHandle fr = 0, fc = 0, ir = 0, ic = 0;  // forward / inverse, along rows (w) / columns (h)
  bool made[4] = {false, false, false, false};
  size_t work = 0;                             // largest cuFFT work area
  size_t o_r1 = 0, o_r2 = 0, o_cx = 0, o_wk = 0, o_tab = 0, total = 0;
  char *ws = nullptr;
};

namespace gd {
namespace {

constexpr int kT = 32;  // transpose tile

inline unsigned nblocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// v[r][n] = x[r][src(n)], src(n) = 2n (n < ceil(N/2)) or 2(N - 1 - n) + 1
__global__ void k_dct_permute(double *__restrict__ v, const double *__restrict__ x, int rows,
                              int n, long long xpitch) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)rows * n) return;
  const int r = (int)(k / n), c = (int)(k % n);
  const int half = (n + 1) / 2;
  const int src = c < half ? 2 * c : 2 * (n - 1 - c) + 1;
  v[k] = x[(long long)r * xpitch + src];
}

__device__ __forceinline__ double dct_scale(int k, int n) {
  return k == 0 ? sqrt(1.0 / (double)n) : sqrt(2.0 / (double)n);
}

// Per-plan tables, computed once at bind: twiddles (cos, sin)(pi k / 2n) for
// both lengths and the eigenvalue terms 2 cos(pi i / n).
struct DctTables {
  double2 *tw_w, *tw_h;  // w and h entries
  double *eig_w, *eig_h;
};

__global__ void k_dct_tables(DctTables t, int h, int w) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double s, c;
  if (k < w) {
    sincospi((double)k / (2.0 * (double)w), &s, &c);
    t.tw_w[k] = make_double2(c, s);
    t.eig_w[k] = 2.0 * cos(M_PI * (double)k / (double)w);
  }
  if (k < h) {
    sincospi((double)k / (2.0 * (double)h), &s, &c);
    t.tw_h[k] = make_double2(c, s);
    t.eig_h[k] = 2.0 * cos(M_PI * (double)k / (double)h);
  }
}

// Orthonormal DCT coefficient k of row r from the half spectrum V (n/2 + 1 per row).
__device__ __forceinline__ double dct_coef(const cufftDoubleComplex *V, const double2 *tw, int r,
                                           int k, int n) {
  const int nh = n / 2 + 1;
  cufftDoubleComplex z;
  if (k < nh) {
    z = V[(long long)r * nh + k];
  } else {  // V_k = conj(V_{n-k}) for a real input
    z = V[(long long)r * nh + (n - k)];
    z.y = -z.y;
  }
  const double2 t = tw[k];
  return (z.x * t.x + z.y * t.y) * dct_scale(k, n);
}

// Position of element r in the even/odd reordering of a length-n sequence.
__device__ __forceinline__ int dct_pos(int r, int n) {
  return (r & 1) ? n - 1 - (r >> 1) : (r >> 1);
}

// out (n x rows) = transpose of the row coefficients (rows x n), via a shared
// tile, each output row already in the even/odd order of the next transform.
__global__ void k_dct_twiddle_t(double *__restrict__ out, const cufftDoubleComplex *__restrict__ V,
                                const double2 *__restrict__ tw, int rows, int n) {
  __shared__ double tile[kT][kT + 1];
  const int r0 = blockIdx.y * kT, k0 = blockIdx.x * kT;
  for (int dy = threadIdx.y; dy < kT; dy += blockDim.y) {
    const int r = r0 + dy, k = k0 + threadIdx.x;
    if (r < rows && k < n) tile[dy][threadIdx.x] = dct_coef(V, tw, r, k, n);
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < kT; dy += blockDim.y) {
    const int k = k0 + dy, r = r0 + threadIdx.x;
    if (k < n && r < rows) out[(long long)k * rows + dct_pos(r, rows)] = tile[threadIdx.x][dy];
  }
}

// Second axis: row j of the transposed layout holds column j of the image;
// coefficient (i, j) divided by the eigenvalue, the constant mode set to zero.
__global__ void k_dct_twiddle_div(double *__restrict__ out,
                                  const cufftDoubleComplex *__restrict__ V, DctTables t, int w,
                                  int h) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)w * h) return;
  const int j = (int)(q / h), i = (int)(q % h);
  if (i == 0 && j == 0) {
    out[q] = 0.0;
    return;
  }
  const double lam = t.eig_h[i] + t.eig_w[j] - 4.0;
  out[q] = dct_coef(V, t.tw_h, j, i, h) / lam;
}

// Inverse, first step: W_k = exp(i pi k / 2n) (X_k - i X_{n-k}) for k <= n/2,
// X the unscaled coefficients of row r.
__global__ void k_idct_pretwiddle(cufftDoubleComplex *__restrict__ W, const double *__restrict__ Xo,
                                  const double2 *__restrict__ tw, int rows, int n) {
  const int nh = n / 2 + 1;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)rows * nh) return;
  const int r = (int)(q / nh), k = (int)(q % nh);
  const double *row = Xo + (long long)r * n;
  const double a = row[k] / dct_scale(k, n);
  const double b = k == 0 ? 0.0 : row[n - k] / dct_scale(n - k, n);
  const double c = tw[k].x, s = tw[k].y;
  // (c + i s)(a - i b) = (c a + s b) + i (s a - c b)
  W[q].x = c * a + s * b;
  W[q].y = s * a - c * b;
}

// Undo the reordering of the inverse FFT output (scaled by 1/n), transposing
// (rows x n -> n x rows) through a shared tile.
__global__ void k_idct_unpermute_t(double *__restrict__ out, const double *__restrict__ v,
                                   int rows, int n) {
  __shared__ double tile[kT][kT + 1];
  const int r0 = blockIdx.y * kT, c0 = blockIdx.x * kT;
  const double inv_n = 1.0 / (double)n;
  for (int dy = threadIdx.y; dy < kT; dy += blockDim.y) {
    const int r = r0 + dy, c = c0 + threadIdx.x;  // c: position in the original order
    if (r < rows && c < n) {
      const int src = (c & 1) ? n - 1 - (c >> 1) : (c >> 1);
      tile[dy][threadIdx.x] = v[(long long)r * n + src] * inv_n;
    }
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < kT; dy += blockDim.y) {
    const int c = c0 + dy, r = r0 + threadIdx.x;
    if (c < n && r < rows) out[(long long)c * rows + r] = tile[threadIdx.x][dy];
  }
}

// Last step: undo the reordering in place order (no transpose), into the
// caller's array with its row pitch.
__global__ void k_idct_unpermute(double *__restrict__ out, long long pitch,
                                 const double *__restrict__ v, int rows, int n) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)rows * n) return;
  const int r = (int)(q / n), c = (int)(q % n);
  const int src = (c & 1) ? n - 1 - (c >> 1) : (c >> 1);
  out[(long long)r * pitch + c] = v[(long long)r * n + src] * (1.0 / (double)n);
}

int plan_fft(cufftHandle *hdl, bool *made, int n, int batch, cufftType type, size_t *work) {
  if (cufftCreate(hdl) != CUFFT_SUCCESS) {
    set_error("gd_dct_plan_create: cufftCreate failed");
    return GD_ERR_CUDA;
  }
  *made = true;
  cufftSetAutoAllocation(*hdl, 0);
  int dims[1] = {n};
  size_t ws = 0;
  const cufftResult r = cufftMakePlanMany(*hdl, 1, dims, nullptr, 1, 0, nullptr, 1, 0, type,
                                          batch, &ws);
  if (r != CUFFT_SUCCESS) {
    set_error("gd_dct_plan_create: cufftMakePlanMany(n=%d, batch=%d) failed (%d)", n, batch,
              (int)r);
    return GD_ERR_CUDA;
  }
  *work = std::max(*work, ws);
  return GD_OK;
}

}  // namespace
}  // namespace gd

using namespace gd;

extern "C" void gd_dct_plan_destroy(gd_dct_plan p) {
  if (!p) return;
  if (p->made[0]) cufftDestroy(p->fr);
  if (p->made[1]) cufftDestroy(p->fc);
  if (p->made[2]) cufftDestroy(p->ir);
  if (p->made[3]) cufftDestroy(p->ic);
  delete p;
}

extern "C" int gd_dct_plan_create(int32_t h, int32_t w, gd_dct_plan *out) {
  GD_REQUIRE(out && h > 1 && w > 1, GD_ERR_ARG,
             "gd_dct_plan_create: the grid needs at least 2 x 2 cells");
  *out = nullptr;
  gd_dct_plan p = new gd_dct_plan_s();
  p->h = h;
  p->w = w;
  int rc = plan_fft(&p->fr, &p->made[0], w, h, CUFFT_D2Z, &p->work);
  if (rc == GD_OK) rc = plan_fft(&p->fc, &p->made[1], h, w, CUFFT_D2Z, &p->work);
  if (rc == GD_OK) rc = plan_fft(&p->ir, &p->made[2], h, w, CUFFT_Z2D, &p->work);
  if (rc == GD_OK) rc = plan_fft(&p->ic, &p->made[3], w, h, CUFFT_Z2D, &p->work);
  if (rc != GD_OK) {
    gd_dct_plan_destroy(p);
    return rc;
  }
  auto a256 = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t n = (size_t)h * w;
  const size_t nc = std::max((size_t)h * (w / 2 + 1), (size_t)w * (h / 2 + 1));
  size_t o = 0;
  p->o_r1 = o;
  o = a256(o + n * sizeof(double));
  p->o_r2 = o;
  o = a256(o + n * sizeof(double));
  p->o_cx = o;
  o = a256(o + nc * sizeof(cufftDoubleComplex));
  p->o_wk = o;
  o = a256(o + std::max<size_t>(p->work, 256));
  p->o_tab = o;
  o = a256(o + (size_t)(h + w) * (sizeof(double2) + sizeof(double)));
  p->total = o;
  *out = p;
  return GD_OK;
}

extern "C" size_t gd_dct_workspace_bytes(gd_dct_plan p) { return p ? p->total : 0; }

namespace {
DctTables dct_tables(gd_dct_plan p) {
  DctTables t;
  char *b = p->ws + p->o_tab;
  t.tw_w = reinterpret_cast<double2 *>(b);
  t.tw_h = t.tw_w + p->w;
  t.eig_w = reinterpret_cast<double *>(t.tw_h + p->h);
  t.eig_h = t.eig_w + p->w;
  return t;
}
}  // namespace

extern "C" int gd_dct_plan_bind(gd_dct_plan p, void *ws, size_t bytes) {
  GD_REQUIRE(p && ws, GD_ERR_ARG, "gd_dct_plan_bind: bad arguments");
  GD_REQUIRE(bytes >= p->total, GD_ERR_ARG, "gd_dct_plan_bind: workspace %zu < %zu bytes", bytes,
             p->total);
  GD_REQUIRE(((uintptr_t)ws & 255) == 0, GD_ERR_ARG, "gd_dct_plan_bind: workspace must be "
                                                     "256-byte aligned");
  p->ws = static_cast<char *>(ws);
  void *wk = p->ws + p->o_wk;
  const cufftHandle hs[4] = {p->fr, p->fc, p->ir, p->ic};
  for (cufftHandle hd : hs)
    GD_REQUIRE(cufftSetWorkArea(hd, wk) == CUFFT_SUCCESS, GD_ERR_CUDA,
               "gd_dct_plan_bind: cufftSetWorkArea failed");
  const int n = std::max(p->h, p->w);
  k_dct_tables<<<nblocks(n, 256), 256>>>(dct_tables(p), p->h, p->w);
  GD_CHECK_LAUNCH();
  // the tables must be complete before a solve on any stream (set-up, once per plan)
  GD_CHECK_CUDA(cudaStreamSynchronize(nullptr));
  return GD_OK;
}

extern "C" int gd_dct_solve_neumann(gd_dct_plan p, const double *b, double *u, int32_t pitch,
                                    cudaStream_t st) {
  GD_REQUIRE(p && p->ws && b && u && pitch >= p->w, GD_ERR_ARG,
             "gd_dct_solve_neumann: bad arguments or unbound plan");
  const int h = p->h, w = p->w;
  const long long n = (long long)h * w;
  double *r1 = reinterpret_cast<double *>(p->ws + p->o_r1);
  double *r2 = reinterpret_cast<double *>(p->ws + p->o_r2);
  cufftDoubleComplex *cx = reinterpret_cast<cufftDoubleComplex *>(p->ws + p->o_cx);
  const cufftHandle hs[4] = {p->fr, p->fc, p->ir, p->ic};
  for (cufftHandle hd : hs)
    GD_REQUIRE(cufftSetStream(hd, st) == CUFFT_SUCCESS, GD_ERR_CUDA,
               "gd_dct_solve_neumann: cufftSetStream failed");
  const dim3 tb(kT, 8);
  const DctTables t = dct_tables(p);
  // forward along rows (length w), then the transposed columns (length h); the
  // transposing twiddle writes the columns already reordered for their FFT
  k_dct_permute<<<nblocks(n, 256), 256, 0, st>>>(r1, b, h, w, pitch);
  GD_REQUIRE(cufftExecD2Z(p->fr, r1, cx) == CUFFT_SUCCESS, GD_ERR_CUDA,
             "gd_dct_solve_neumann: forward row FFT failed");
  k_dct_twiddle_t<<<dim3(nblocks(w, kT), nblocks(h, kT)), tb, 0, st>>>(r2, cx, t.tw_w, h, w);
  GD_REQUIRE(cufftExecD2Z(p->fc, r2, cx) == CUFFT_SUCCESS, GD_ERR_CUDA,
             "gd_dct_solve_neumann: forward column FFT failed");
  k_dct_twiddle_div<<<nblocks(n, 256), 256, 0, st>>>(r2, cx, t, w, h);
  // inverse along the transposed columns (length h), transpose back, rows (length w)
  k_idct_pretwiddle<<<nblocks((long long)w * (h / 2 + 1), 256), 256, 0, st>>>(cx, r2, t.tw_h, w,
                                                                              h);
  GD_REQUIRE(cufftExecZ2D(p->ir, cx, r1) == CUFFT_SUCCESS, GD_ERR_CUDA,
             "gd_dct_solve_neumann: inverse column FFT failed");
  k_idct_unpermute_t<<<dim3(nblocks(h, kT), nblocks(w, kT)), tb, 0, st>>>(r2, r1, w, h);
  k_idct_pretwiddle<<<nblocks((long long)h * (w / 2 + 1), 256), 256, 0, st>>>(cx, r2, t.tw_w, h,
                                                                              w);
  GD_REQUIRE(cufftExecZ2D(p->ic, cx, r1) == CUFFT_SUCCESS, GD_ERR_CUDA,
             "gd_dct_solve_neumann: inverse row FFT failed");
  k_idct_unpermute<<<nblocks(n, 256), 256, 0, st>>>(u, pitch, r1, h, w);
  GD_CHECK_LAUNCH();
  return GD_OK;
}
