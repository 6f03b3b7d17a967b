// Right-hand-side assembly on the device, error reporting and version.
//
// gd_gradient follows operators.py:30-50 (forward differences, last column of
// gx and last row of gy zero), gd_divergence follows operators.py:53-83
// (backward differences with the
// edge rows/columns taken from the adjacent gradient), gd_fold_dirichlet
// follows operators.py:139-169 as solve_dirichlet calls it (poisson.py:131-143,
// spacing 1), and gd_masked_rhs follows the masked assembly of
// poisson.py:216-224.  All three keep the reference's order of additions.

#include <cstdarg>
#include <cstdio>

#include "gd_internal.cuh"

namespace gd {

static thread_local char g_error[512] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}

namespace {

__global__ void k_divergence(double *__restrict__ out, const double *__restrict__ gx,
                             const double *__restrict__ gy, int h, int w) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)h * w) return;
  const int i = (int)(k / w), j = (int)(k % w);
  double dx = 0.0, dy = 0.0;
  if (w > 1) {
    if (j == 0) dx = gx[k];
    else if (j == w - 1) dx = -gx[k - 1];
    else dx = __dsub_rn(gx[k], gx[k - 1]);
  }
  if (h > 1) {
    if (i == 0) dy = gy[k];
    else if (i == h - 1) dy = -gy[k - w];
    else dy = __dsub_rn(gy[k], gy[k - w]);
  }
  out[k] = __dadd_rn(dx, dy);
}

__global__ void k_gradient(double *__restrict__ gx, double *__restrict__ gy,
                           const double *__restrict__ u, int h, int w) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)h * w) return;
  const int i = (int)(k / w), j = (int)(k % w);
  gx[k] = j < w - 1 ? __dsub_rn(u[k + 1], u[k]) : 0.0;
  gy[k] = i < h - 1 ? __dsub_rn(u[k + w], u[k]) : 0.0;
}

__global__ void k_fold(double *__restrict__ f, const double *__restrict__ div,
                       const double *__restrict__ bnd, int h, int w, double scale) {
  const int m = h - 2, n = w - 2;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)m * n) return;
  const int i = (int)(k / n), j = (int)(k % n);
  double v = div[(long long)(i + 1) * w + (j + 1)];
  if (i == 0) v = __dsub_rn(v, bnd[j + 1]);
  if (i == m - 1) v = __dsub_rn(v, bnd[(long long)(h - 1) * w + j + 1]);
  if (j == 0) v = __dsub_rn(v, bnd[(long long)(i + 1) * w]);
  if (j == n - 1) v = __dsub_rn(v, bnd[(long long)(i + 1) * w + w - 1]);
  f[k] = __dmul_rn(scale, v);
}

__global__ void k_masked_rhs(double *__restrict__ f, const double *__restrict__ div,
                             const double *__restrict__ img, const unsigned char *__restrict__ unk,
                             int h, int w, double scale) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)h * w) return;
  const int i = (int)(k / w), j = (int)(k % w);
  if (!unk[k]) {
    f[k] = 0.0;
    return;
  }
  double v = div[k];
  const int di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int y = i + di[q], x = j + dj[q];
    if (y < 0 || y >= h || x < 0 || x >= w) continue;  // unknowns never touch the border
    const long long g = (long long)y * w + x;
    if (!unk[g]) v = __dsub_rn(v, img[g]);
  }
  f[k] = __dmul_rn(scale, v);
}

inline unsigned blocks(long long work) { return (unsigned)((work + 255) / 256); }

}  // namespace
}  // namespace gd

using namespace gd;

extern "C" const char *gd_last_error(void) { return g_error; }

extern "C" const char *gd_version(void) { return "gd_poisson 0.1 sm_100a"; }

extern "C" int gd_divergence(double *out, const double *gx, const double *gy, int32_t h, int32_t w,
                             cudaStream_t st) {
  GD_REQUIRE(out && gx && gy && h > 0 && w > 0, GD_ERR_ARG, "gd_divergence: bad arguments");
  k_divergence<<<blocks((long long)h * w), 256, 0, st>>>(out, gx, gy, h, w);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_gradient(double *gx, double *gy, const double *u, int32_t h, int32_t w,
                           cudaStream_t st) {
  GD_REQUIRE(gx && gy && u && h > 0 && w > 0, GD_ERR_ARG, "gd_gradient: bad arguments");
  k_gradient<<<blocks((long long)h * w), 256, 0, st>>>(gx, gy, u, h, w);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_fold_dirichlet(double *f, const double *div, const double *bnd, int32_t h,
                                 int32_t w, double scale, cudaStream_t st) {
  GD_REQUIRE(f && div && bnd && h > 2 && w > 2, GD_ERR_ARG, "gd_fold_dirichlet: bad arguments");
  k_fold<<<blocks((long long)(h - 2) * (w - 2)), 256, 0, st>>>(f, div, bnd, h, w, scale);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_masked_rhs(double *f, const double *div, const double *img, const uint8_t *unk,
                             int32_t h, int32_t w, double scale, cudaStream_t st) {
  GD_REQUIRE(f && div && img && unk && h > 0 && w > 0, GD_ERR_ARG, "gd_masked_rhs: bad arguments");
  k_masked_rhs<<<blocks((long long)h * w), 256, 0, st>>>(f, div, img, unk, h, w, scale);
  GD_CHECK_LAUNCH();
  return GD_OK;
}
