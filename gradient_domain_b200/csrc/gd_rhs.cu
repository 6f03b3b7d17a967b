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

// fold_boundary for any spacing and channel count (operators.py:139-169):
// rhs and out are (h-2, w-2, c), bnd is (h, w, c), channels interleaved.  The
// four ring subtractions run in the reference's order (first row, last row,
// first column, last column), each subtracting the rounded product
// weight * boundary, so a corner cell sees two of them in that order.
__global__ void k_fold_ring(double *out, const double *rhs, const double *__restrict__ bnd,
                            int h, int w, int c, double weight) {
  const int m = h - 2, n = w - 2;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)m * n * c) return;
  const int ch = (int)(k % c);
  const long long cell = k / c;
  const int i = (int)(cell / n), j = (int)(cell % n);
  auto ring = [&](int r, int col) { return bnd[((long long)r * w + col) * c + ch]; };
  double v = rhs[k];
  if (i == 0) v = __dsub_rn(v, __dmul_rn(weight, ring(0, j + 1)));
  if (i == m - 1) v = __dsub_rn(v, __dmul_rn(weight, ring(h - 1, j + 1)));
  if (j == 0) v = __dsub_rn(v, __dmul_rn(weight, ring(i + 1, 0)));
  if (j == n - 1) v = __dsub_rn(v, __dmul_rn(weight, ring(i + 1, w - 1)));
  out[k] = v;
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

// Guidance fields built on the fly (poisson.py:52-92 and the field set-up of
// seamless_clone, texture_flatten and illumination_change, poisson.py:306-431):
// the forward-difference gradient of an interleaved (H, W, C) image channel,
// combined per cell as the field kind says.
struct FieldView {
  gd_field_desc d;
  __device__ __forceinline__ double at(const double *img, int y, int x) const {
    return img[((long long)y * d.width + x) * d.channels + d.channel];
  }
  // forward differences of one image (operators.py:30-50)
  __device__ __forceinline__ void grad(const double *img, int y, int x, double &gx,
                                       double &gy) const {
    const double c = at(img, y, x);
    gx = x < d.width - 1 ? __dsub_rn(at(img, y, x + 1), c) : 0.0;
    gy = y < d.height - 1 ? __dsub_rn(at(img, y + 1, x), c) : 0.0;
  }
  __device__ __forceinline__ void field(int y, int x, double &gx, double &gy) const {
    double tx, ty;
    grad(d.target, y, x, tx, ty);
    switch (d.kind) {
      case GD_FIELD_IMPORT:
      case GD_FIELD_MIXED:
      case GD_FIELD_AVERAGE: {
        if (!d.select[(long long)y * d.width + x]) {  // GuidanceField.select: target outside
          gx = tx;
          gy = ty;
          return;
        }
        double sx, sy;
        grad(d.source, y, x, sx, sy);
        if (d.kind == GD_FIELD_IMPORT) {
          gx = sx;
          gy = sy;
        } else if (d.kind == GD_FIELD_MIXED) {  // mix_by_magnitude: the larger, source on ties
          gx = fabs(sx) >= fabs(tx) ? sx : tx;
          gy = fabs(sy) >= fabs(ty) ? sy : ty;
        } else {
          gx = __dmul_rn(0.5, __dadd_rn(sx, tx));
          gy = __dmul_rn(0.5, __dadd_rn(sy, ty));
        }
        return;
      }
      case GD_FIELD_WEIGHTED: {  // texture_flatten: gradient times the edge weights
        const double w = d.weights[(long long)y * d.width + x];
        gx = __dmul_rn(tx, w);
        gy = __dmul_rn(ty, w);
        return;
      }
      default: {  // illumination_change: alpha^beta * max(|g|, eps)^(-beta)
        const double m = sqrt(__dadd_rn(__dmul_rn(tx, tx), __dmul_rn(ty, ty)));
        const double f = __dmul_rn(d.alpha_pow_beta, pow(fmax(m, d.epsilon), -d.beta));
        gx = __dmul_rn(tx, f);
        gy = __dmul_rn(ty, f);
        return;
      }
    }
  }
};

// Divergence (operators.py:53-83) of the field over a window whose corner is
// image cell (row0, col0).  Interior cells take the backward differences; the
// window's outer ring is written 0 (no consumer of a window reads it) or, with
// `edges`, follows operators.py's edge rules for the window as a whole image.
__global__ void k_guidance_div(double *__restrict__ out, FieldView fv, int row0, int col0, int h,
                               int w) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)h * w) return;
  const int i = (int)(k / w), j = (int)(k % w);
  const int y = row0 + i, x = col0 + j;
  const bool ring = i == 0 || j == 0 || i == h - 1 || j == w - 1;
  if (ring && !fv.d.edges) {
    out[k] = 0.0;
    return;
  }
  double gx, gy, gxl = 0.0, gyl = 0.0, unused;
  fv.field(y, x, gx, gy);
  if (j > 0) fv.field(y, x - 1, gxl, unused);
  if (i > 0) fv.field(y - 1, x, unused, gyl);
  double dx = 0.0, dy = 0.0;
  if (w > 1) dx = j == 0 ? gx : j == w - 1 ? -gxl : __dsub_rn(gx, gxl);
  if (h > 1) dy = i == 0 ? gy : i == h - 1 ? -gyl : __dsub_rn(gy, gyl);
  out[k] = __dadd_rn(dx, dy);
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

extern "C" int gd_fold_boundary(double *out, const double *rhs, const double *bnd, int32_t h,
                                int32_t w, int32_t channels, double spacing, cudaStream_t st) {
  GD_REQUIRE(out && rhs && bnd && h > 2 && w > 2 && channels > 0, GD_ERR_ARG,
             "gd_fold_boundary: bad arguments");
  GD_REQUIRE(spacing != 0.0 && std::isfinite(spacing), GD_ERR_ARG,
             "gd_fold_boundary: spacing must be finite and nonzero");
  const double weight = 1.0 / (spacing * spacing);
  k_fold_ring<<<blocks((long long)(h - 2) * (w - 2) * channels), 256, 0, st>>>(
      out, rhs, bnd, h, w, channels, weight);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_guidance_divergence(double *div, const gd_field_desc *field, int32_t row0,
                                      int32_t col0, int32_t h, int32_t w, cudaStream_t st) {
  GD_REQUIRE(div && field && field->target && h > 0 && w > 0 && (field->edges || (h > 2 && w > 2)),
             GD_ERR_ARG, "gd_guidance_divergence: bad arguments");
  const gd_field_desc &d = *field;
  GD_REQUIRE(d.kind >= GD_FIELD_IMPORT && d.kind <= GD_FIELD_ILLUMINATION, GD_ERR_ARG,
             "gd_guidance_divergence: unknown field kind %d", d.kind);
  GD_REQUIRE(d.height > 0 && d.width > 0 && d.channels > 0 && d.channel >= 0 &&
                 d.channel < d.channels,
             GD_ERR_ARG, "gd_guidance_divergence: bad image geometry");
  GD_REQUIRE(row0 >= 0 && col0 >= 0 && row0 + h <= d.height && col0 + w <= d.width, GD_ERR_ARG,
             "gd_guidance_divergence: window outside the image");
  GD_REQUIRE(d.kind > GD_FIELD_AVERAGE || (d.source && d.select), GD_ERR_ARG,
             "gd_guidance_divergence: cloning fields need a source and a selection");
  GD_REQUIRE(d.kind != GD_FIELD_WEIGHTED || d.weights, GD_ERR_ARG,
             "gd_guidance_divergence: weighted fields need weights");
  k_guidance_div<<<blocks((long long)h * w), 256, 0, st>>>(div, FieldView{d}, row0, col0, h, w);
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
