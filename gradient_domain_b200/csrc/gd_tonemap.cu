// Gradient-domain tone mapping on the device: the steps of hdr.py:73-185
// around the Neumann solve.
//
//   gd_tm_log_luminance   luminance = max(radiance . (0.2126, 0.7152, 0.0722), tiny)
//                         and its logarithm (hdr.py:168-170)
//   gd_tm_downsample      5-tap binomial blur with edge replication, every other
//                         sample (hdr.py:73-80, `_downsample`)
//   gd_tm_level_factor    one level of the attenuation field: central-difference
//                         gradient magnitude, its mean, the local factor, times the
//                         bilinear upsampling of the coarser level's factor
//                         (hdr.py:83-134, `_upsample`, `_central_gradient`,
//                         `attenuation_field`)
//   gd_tm_compose         exp(c - max c), chromatic ratios to the saturation power,
//                         99.5th percentile (NumPy's linear method), normalise and
//                         clip (hdr.py:178-185)
//
// Element-wise arithmetic uses explicitly rounded FP64 operations in the
// reference's order, so the results differ from NumPy's only where a library
// function (log, exp, pow, sqrt) or a reduction order differs.  Reductions are
// fixed trees (deterministic).  The percentile is exact: a radix selection on
// the order-preserving bit patterns of the non-negative image values.
// Scratch memory is the caller's (gd_tm_scratch_bytes).

#include <cstdint>

#include "gd_internal.cuh"

namespace gd {
namespace {

constexpr int kTmThreads = 256;
constexpr int kTmBlocks = 296;  // fixed grid of the reductions: 2 x 148 SMs

inline unsigned blocks_for(long long n) { return (unsigned)((n + kTmThreads - 1) / kTmThreads); }

__device__ __forceinline__ double block_reduce_sum(double v) {
  __shared__ double part[kTmThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) part[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < kTmThreads / 32; ++k) s = __dadd_rn(s, part[k]);
  return s;
}

__device__ __forceinline__ double block_reduce_max(double v) {
  __shared__ double part[kTmThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) part[warp] = v;
  __syncthreads();
  double s = -INFINITY;
  if (threadIdx.x == 0)
    for (int k = 0; k < kTmThreads / 32; ++k) s = fmax(s, part[k]);
  return s;
}

// The kTmBlocks partials reduced once, in a fixed order, into p[kTmBlocks].
__global__ void k_tm_finish_sum(double *p) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int k = 0; k < kTmBlocks; ++k) s = __dadd_rn(s, p[k]);
  p[kTmBlocks] = s;
}

__global__ void k_tm_finish_max(double *p) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = -INFINITY;
  for (int k = 0; k < kTmBlocks; ++k) s = fmax(s, p[k]);
  p[kTmBlocks] = s;
}

__global__ void k_tm_luminance(double *__restrict__ logl, double *__restrict__ lum,
                               const double *__restrict__ rad, long long n) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double *p = rad + 3 * k;
  double l = __dadd_rn(__dadd_rn(__dmul_rn(p[0], 0.2126), __dmul_rn(p[1], 0.7152)),
                       __dmul_rn(p[2], 0.0722));
  l = fmax(l, 2.2250738585072014e-308);  // np.finfo(float).tiny
  lum[k] = l;
  logl[k] = log(l);
}

// Output (i, j) = vertical blur of the horizontally blurred rows 2i-2 .. 2i+2
// at column 2j, both with edge replication and the weights 1 4 6 4 1 / 16
// summed left to right from zero, as the reference's `sum(...)` does.
__global__ void k_tm_downsample(double *__restrict__ out, const double *__restrict__ in, int h,
                                int w) {
  const int oh = (h + 1) / 2, ow = (w + 1) / 2;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)oh * ow) return;
  const int i = (int)(k / ow), j = (int)(k % ow);
  const double wgt[5] = {1.0 / 16.0, 4.0 / 16.0, 6.0 / 16.0, 4.0 / 16.0, 1.0 / 16.0};
  double acc = 0.0;
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const int r = min(max(2 * i + a - 2, 0), h - 1);
    const double *row = in + (long long)r * w;
    double hb = 0.0;
#pragma unroll
    for (int b = 0; b < 5; ++b) {
      const int c = min(max(2 * j + b - 2, 0), w - 1);
      hb = __dadd_rn(hb, __dmul_rn(wgt[b], row[c]));
    }
    acc = __dadd_rn(acc, __dmul_rn(wgt[a], hb));
  }
  out[k] = acc;
}

// Central-difference gradient magnitude of one level at (i, j), edges replicated.
__device__ __forceinline__ double tm_magnitude(const double *a, int h, int w, int i, int j,
                                               double two_spacing) {
  const double *row = a + (long long)i * w;
  const double gx = __dsub_rn(row[min(j + 1, w - 1)], row[max(j - 1, 0)]) / two_spacing;
  const double gy = __dsub_rn(a[(long long)min(i + 1, h - 1) * w + j],
                              a[(long long)max(i - 1, 0) * w + j]) / two_spacing;
  return sqrt(__dadd_rn(__dmul_rn(gx, gx), __dmul_rn(gy, gy)));
}

__global__ void __launch_bounds__(kTmThreads) k_tm_mag_partials(double *__restrict__ part,
                                                                const double *__restrict__ a,
                                                                int h, int w, double two_spacing) {
  const long long n = (long long)h * w;
  double s = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    s = __dadd_rn(s, tm_magnitude(a, h, w, (int)(k / w), (int)(k % w), two_spacing));
  s = block_reduce_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// np.linspace(0, n_coarse - 1, n_fine)[i] (hdr.py:85-86)
__device__ __forceinline__ double tm_linspace(int i, int n_coarse, int n_fine) {
  if (n_fine <= 1) return 0.0;
  if (i == n_fine - 1) return (double)(n_coarse - 1);
  const double step = (double)(n_coarse - 1) / (double)(n_fine - 1);
  return __dmul_rn((double)i, step);
}

__global__ void k_tm_factor(double *__restrict__ factor, const double *__restrict__ a,
                            const double *__restrict__ coarse, const double *__restrict__ part,
                            int h, int w, int ch, int cw, double two_spacing, double alpha,
                            double beta, double eps) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)h * w) return;
  const int i = (int)(k / w), j = (int)(k % w);
  const double mean = part[kTmBlocks] / (double)((long long)h * w);
  const double scale = __dmul_rn(alpha, fmax(mean, eps));
  const double m = fmax(tm_magnitude(a, h, w, i, j, two_spacing), eps);
  const double local = __dmul_rn(scale / m, pow(m / scale, beta));
  if (!coarse) {
    factor[k] = local;
    return;
  }
  const double ry = tm_linspace(i, ch, h), rx = tm_linspace(j, cw, w);
  const int r0 = (int)floor(ry), c0 = (int)floor(rx);
  const int r1 = min(r0 + 1, ch - 1), c1 = min(c0 + 1, cw - 1);
  const double wy = __dsub_rn(ry, (double)r0), wx = __dsub_rn(rx, (double)c0);
  const double *p0 = coarse + (long long)r0 * cw, *p1 = coarse + (long long)r1 * cw;
  const double top = __dadd_rn(__dmul_rn(p0[c0], __dsub_rn(1.0, wx)), __dmul_rn(p0[c1], wx));
  const double bot = __dadd_rn(__dmul_rn(p1[c0], __dsub_rn(1.0, wx)), __dmul_rn(p1[c1], wx));
  const double up = __dadd_rn(__dmul_rn(top, __dsub_rn(1.0, wy)), __dmul_rn(bot, wy));
  factor[k] = __dmul_rn(up, local);
}

__global__ void __launch_bounds__(kTmThreads) k_tm_max_partials(double *__restrict__ part,
                                                                const double *__restrict__ c,
                                                                long long n) {
  double s = -INFINITY;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    s = fmax(s, c[k]);
  s = block_reduce_max(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// image = (radiance / luminance) ** saturation * exp(c - max c)   (hdr.py:178-182)
__global__ void k_tm_image(double *__restrict__ image, const double *__restrict__ rad,
                           const double *__restrict__ lum, const double *__restrict__ comp,
                           const double *__restrict__ part, long long n, double saturation) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double result = exp(__dsub_rn(comp[k], part[kTmBlocks]));
  const double l = lum[k];
#pragma unroll
  for (int c = 0; c < 3; ++c)
    image[3 * k + c] = __dmul_rn(pow(rad[3 * k + c] / l, saturation), result);
}

// Radix selection of the element of rank `rank` among n non-negative doubles:
// their IEEE bit patterns order like the values, so eight passes of an 8-bit
// digit histogram over the keys that match the digits chosen so far find it.
struct SelectState {
  unsigned long long prefix, mask, rank;
  unsigned long long count_le, min_above;  // for the neighbour of rank + 1
};

__global__ void __launch_bounds__(kTmThreads) k_select_hist(unsigned *__restrict__ hist,
                                                            const double *__restrict__ v,
                                                            long long n,
                                                            const SelectState *__restrict__ s,
                                                            int shift) {
  __shared__ unsigned h[256];
  for (int b = threadIdx.x; b < 256; b += blockDim.x) h[b] = 0u;
  __syncthreads();
  const unsigned long long prefix = s->prefix, mask = s->mask;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const unsigned long long key = (unsigned long long)__double_as_longlong(v[k]);
    if ((key & mask) == prefix) atomicAdd(&h[(key >> shift) & 0xffull], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < 256; b += blockDim.x)
    if (h[b]) atomicAdd(&hist[b], h[b]);
}

__global__ void k_select_digit(unsigned *__restrict__ hist, SelectState *__restrict__ s,
                               int shift) {
  if (threadIdx.x != 0) return;
  unsigned long long rank = s->rank, below = 0;
  int d = 0;
  for (; d < 255; ++d) {
    if (below + hist[d] > rank) break;
    below += hist[d];
  }
  s->rank = rank - below;
  s->prefix |= (unsigned long long)d << shift;
  s->mask |= 0xffull << shift;
  for (int b = 0; b < 256; ++b) hist[b] = 0u;  // ready for the next pass
}

// After the selection: how many values are <= the selected one, and the
// smallest value above it (the element of rank + 1 when the count allows).
__global__ void __launch_bounds__(kTmThreads) k_select_next(const double *__restrict__ v,
                                                            long long n,
                                                            SelectState *__restrict__ s) {
  const unsigned long long sel = s->prefix;
  unsigned long long le = 0, above = ~0ull;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const unsigned long long key = (unsigned long long)__double_as_longlong(v[k]);
    if (key <= sel) ++le;
    else if (key < above) above = key;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    le += __shfl_down_sync(0xffffffffu, le, o);
    const unsigned long long a = __shfl_down_sync(0xffffffffu, above, o);
    above = a < above ? a : above;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&s->count_le, le);
    atomicMin(&s->min_above, above);
  }
}

// np.percentile(image, q) with the linear method, then clip(image / peak, 0, 1).
__global__ void k_tm_finish(double *__restrict__ out, const double *__restrict__ image,
                            long long n, const SelectState *__restrict__ s, long long lo_rank,
                            double t) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double a = __longlong_as_double((long long)s->prefix);
  // rank lo + 1 is the selected value again when it repeats, else the next one up
  const double b = (s->count_le > (unsigned long long)lo_rank + 1ull || t == 0.0)
                       ? a
                       : __longlong_as_double((long long)s->min_above);
  // NumPy's _lerp: a + (b - a) t, or b - (b - a)(1 - t) for t >= 0.5
  const double diff = __dsub_rn(b, a);
  const double peak = t >= 0.5 ? __dsub_rn(b, __dmul_rn(diff, __dsub_rn(1.0, t)))
                               : __dadd_rn(a, __dmul_rn(diff, t));
  const double v = image[k] / fmax(peak, 1e-12);
  out[k] = fmin(fmax(v, 0.0), 1.0);
}

__global__ void k_select_init(SelectState *s, unsigned *hist, unsigned long long rank) {
  if (threadIdx.x == 0) {
    s->prefix = 0ull;
    s->mask = 0ull;
    s->rank = rank;
    s->count_le = 0ull;
    s->min_above = ~0ull;
  }
  for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0u;
}

struct TmScratch {
  double *part;       // kTmBlocks partials and their reduction
  SelectState *sel;
  unsigned *hist;     // 256 counters
};

TmScratch tm_scratch(void *base) {
  char *p = static_cast<char *>(base);
  TmScratch s;
  s.part = reinterpret_cast<double *>(p);
  s.sel = reinterpret_cast<SelectState *>(p + 4096);
  s.hist = reinterpret_cast<unsigned *>(p + 8192);
  return s;
}

}  // namespace
}  // namespace gd

using namespace gd;

extern "C" size_t gd_tm_scratch_bytes(void) { return 16384; }

extern "C" int gd_tm_log_luminance(double *logl, double *lum, const double *radiance, int32_t h,
                                   int32_t w, cudaStream_t st) {
  GD_REQUIRE(logl && lum && radiance && h > 0 && w > 0, GD_ERR_ARG,
             "gd_tm_log_luminance: bad arguments");
  const long long n = (long long)h * w;
  k_tm_luminance<<<blocks_for(n), kTmThreads, 0, st>>>(logl, lum, radiance, n);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_tm_downsample(double *out, const double *in, int32_t h, int32_t w,
                                cudaStream_t st) {
  GD_REQUIRE(out && in && h > 0 && w > 0, GD_ERR_ARG, "gd_tm_downsample: bad arguments");
  k_tm_downsample<<<blocks_for((long long)((h + 1) / 2) * ((w + 1) / 2)), kTmThreads, 0, st>>>(
      out, in, h, w);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_tm_level_factor(double *factor, const double *level, const double *coarse,
                                  int32_t h, int32_t w, int32_t ch, int32_t cw, double spacing,
                                  double alpha, double beta, double epsilon, void *scratch,
                                  cudaStream_t st) {
  GD_REQUIRE(factor && level && scratch && h > 0 && w > 0 && spacing > 0.0, GD_ERR_ARG,
             "gd_tm_level_factor: bad arguments");
  GD_REQUIRE(!coarse || (ch > 0 && cw > 0), GD_ERR_ARG, "gd_tm_level_factor: bad coarse level");
  const TmScratch s = tm_scratch(scratch);
  k_tm_mag_partials<<<kTmBlocks, kTmThreads, 0, st>>>(s.part, level, h, w, 2.0 * spacing);
  k_tm_finish_sum<<<1, 32, 0, st>>>(s.part);
  k_tm_factor<<<blocks_for((long long)h * w), kTmThreads, 0, st>>>(
      factor, level, coarse, s.part, h, w, ch, cw, 2.0 * spacing, alpha, beta, epsilon);
  GD_CHECK_LAUNCH();
  return GD_OK;
}

extern "C" int gd_tm_compose(double *out, double *image, const double *radiance,
                             const double *lum, const double *compressed, int32_t h, int32_t w,
                             double saturation, double percentile, void *scratch,
                             cudaStream_t st) {
  GD_REQUIRE(out && image && radiance && lum && compressed && scratch && h > 0 && w > 0,
             GD_ERR_ARG, "gd_tm_compose: bad arguments");
  GD_REQUIRE(percentile >= 0.0 && percentile <= 100.0, GD_ERR_ARG,
             "gd_tm_compose: percentile outside [0, 100]");
  const TmScratch s = tm_scratch(scratch);
  const long long n = (long long)h * w, n3 = 3 * n;
  k_tm_max_partials<<<kTmBlocks, kTmThreads, 0, st>>>(s.part, compressed, n);
  k_tm_finish_max<<<1, 32, 0, st>>>(s.part);
  k_tm_image<<<blocks_for(n), kTmThreads, 0, st>>>(image, radiance, lum, compressed, s.part, n,
                                                   saturation);
  // NumPy's linear percentile: index q/100 (n - 1), neighbours floor and floor + 1
  const double index = percentile / 100.0 * (double)(n3 - 1);
  const long long lo = (long long)index;
  const double t = index - (double)lo;
  k_select_init<<<1, kTmThreads, 0, st>>>(s.sel, s.hist, (unsigned long long)lo);
  for (int pass = 0; pass < 8; ++pass) {
    const int shift = 56 - 8 * pass;
    k_select_hist<<<kTmBlocks, kTmThreads, 0, st>>>(s.hist, image, n3, s.sel, shift);
    k_select_digit<<<1, 32, 0, st>>>(s.hist, s.sel, shift);
  }
  k_select_next<<<kTmBlocks, kTmThreads, 0, st>>>(image, n3, s.sel);
  k_tm_finish<<<blocks_for(n3), kTmThreads, 0, st>>>(out, image, n3, s.sel, lo, t);
  GD_CHECK_LAUNCH();
  return GD_OK;
}
