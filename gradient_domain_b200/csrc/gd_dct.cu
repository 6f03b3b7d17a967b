// Exact Neumann Poisson solve by the discrete cosine transform: the algorithm
// of solvers.py:224-262 (dctn type 2, division by the eigenvalues
// 2 cos(pi i / m) + 2 cos(pi j / n) - 4 with the constant mode dropped, idctn),
// on the device with this library's own FFT kernels.
//
// Three passes over HBM, each CTA working on two lines (rows or columns) at
// once, held in shared memory as one complex sequence z = a + i b:
//   rows:    load two rows of b, DCT-II along x, write the coefficients to T;
//   columns: load two columns of T, DCT-II along y, divide by the
//            eigenvalues, inverse transform (DCT-III) along y, write back;
//   rows:    load two rows of T, DCT-III along x, write u.
// so b is read once, u written once and T read and written twice: 48 bytes
// per cell against 16 for b and u alone.
//
// One DCT-II of length N is one complex FFT of length N (Makhoul's
// reordering v = (x0, x2, x4, ..., x5, x3, x1), X_k = Re(e^{-i pi k/2N} V_k));
// two real lines share one FFT and are separated from its output by the
// Hermitian symmetry of each.  The inverse forms
// W_k = e^{i pi k/2N} (X_k - i X_{N-k}) and takes an inverse FFT (scaled by
// 1/N) whose output, read back through the reordering, is the line.  The
// coefficients here are half those of scipy's unnormalised DCT-II; the
// forward / inverse pair is exact either way and the solve only divides by
// the eigenvalues in between.
//
// The FFT is a mixed-radix transform in place in shared memory: forward
// passes decimate in frequency (natural order in, digit-reversed order out),
// inverse passes decimate in time (digit-reversed in, natural out), so no
// reordering pass is needed between them.  Radices 8, 4 and 2 have dedicated
// butterflies, 3, 5 and 7 a small direct DFT per butterfly, and any larger
// prime factor a direct DFT computed one output per thread.  Twiddles come
// from per-plan tables of e^{-2 pi i m / N} computed with sincospi at bind.

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "gd_internal.cuh"

namespace gd {
namespace dct {

constexpr int kMaxLen = 8192;   // longest line (128 KB of complex values in shared memory)
constexpr int kMaxStages = 16;  // 8192 = 8^4 * 2
constexpr int kThreads = 256;
constexpr int kMaxPerThread = kMaxLen / kThreads;  // outputs per thread of a large-prime stage

// Radix sequence of one transform length, largest radices first.
struct Radices {
  int n = 0, count = 0;
  int r[kMaxStages] = {0};
};

inline Radices factor(int n) {
  Radices f;
  f.n = n;
  int m = n;
  auto push = [&](int r) { f.r[f.count++] = r; m /= r; };
  while (m % 8 == 0) push(8);
  if (m % 4 == 0) push(4);
  if (m % 2 == 0) push(2);
  for (int p = 3; m > 1; p += 2)
    while (m % p == 0) push(p);
  return f;
}

// Per-axis tables: FFT twiddles e^{-2 pi i m / N} (N entries), the DCT
// twiddles e^{-i pi k / 2N} (N entries) and the eigenvalue terms
// 2 cos(pi k / N) (N entries).  The eigenvalue of mode (i, j) is formed as
// (2 cos(pi i / m) + 2 cos(pi j / n)) - 4 with cos(pi k / N) evaluated from the
// rounded product pi k, as solvers.py:253-258 does: the smallest eigenvalues
// cancel most of their digits in that sum, and the solution's smoothest modes
// carry that rounding, so the same expression keeps the result within
// rounding of the reference's.
struct Axis {
  Radices rad;
  const double2 *tw;
  const double2 *post;
  const double *eig;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
// multiply by -i (forward, SIGN = -1) or +i (inverse, SIGN = +1)
template <int SIGN>
__device__ __forceinline__ double2 rot90(double2 a) {
  return SIGN < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

// In-register DFTs y_q = sum_j x_j e^{SIGN 2 pi i j q / R}, natural order.
template <int SIGN>
__device__ __forceinline__ void dft2(double2 &a, double2 &b) {
  const double2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int SIGN>
__device__ __forceinline__ void dft4(double2 (&x)[4]) {
  double2 a0 = cadd(x[0], x[2]), a1 = csub(x[0], x[2]);
  double2 b0 = cadd(x[1], x[3]), b1 = rot90<SIGN>(csub(x[1], x[3]));
  x[0] = cadd(a0, b0);
  x[2] = csub(a0, b0);
  x[1] = cadd(a1, b1);
  x[3] = csub(a1, b1);
}

template <int SIGN>
__device__ __forceinline__ void dft8(double2 (&x)[8]) {
  constexpr double h = 0.70710678118654752440;  // sqrt(1/2)
  // two DFT-4 of the even and odd samples, then the radix-2 combination
  double2 e[4] = {x[0], x[2], x[4], x[6]};
  double2 o[4] = {x[1], x[3], x[5], x[7]};
  dft4<SIGN>(e);
  dft4<SIGN>(o);
  // o_q *= e^{SIGN 2 pi i q / 8}
  o[1] = make_double2(h * (o[1].x - SIGN * o[1].y), h * (o[1].y + SIGN * o[1].x));
  o[2] = rot90<SIGN>(o[2]);
  o[3] = make_double2(h * (-o[3].x - SIGN * o[3].y), h * (-o[3].y + SIGN * o[3].x));
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    x[q] = cadd(e[q], o[q]);
    x[q + 4] = csub(e[q], o[q]);
  }
}

// Direct DFT of a small odd radix, roots of unity from the length-N table.
template <int R, int SIGN>
__device__ __forceinline__ void dft_odd(double2 (&x)[R], const double2 *tw, int n) {
  double2 y[R];
  const int s = n / R;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    double2 acc = x[0];
#pragma unroll
    for (int j = 1; j < R; ++j) {
      const double2 w = tw[((j * q) % R) * s];
      acc = cadd(acc, SIGN < 0 ? cmul(x[j], w) : cmulc(x[j], w));
    }
    y[q] = acc;
  }
#pragma unroll
  for (int q = 0; q < R; ++q) x[q] = y[q];
}

template <int R, int SIGN>
__device__ __forceinline__ void dft_small(double2 (&x)[R], const double2 *tw, int n) {
  if constexpr (R == 2) dft2<SIGN>(x[0], x[1]);
  else if constexpr (R == 4) dft4<SIGN>(x);
  else if constexpr (R == 8) dft8<SIGN>(x);
  else dft_odd<R, SIGN>(x, tw, n);
}

// One decimation-in-frequency pass of radix R on sub-transforms of length L:
// each butterfly reads R values spaced L/R apart, transforms them and
// multiplies output q by e^{-2 pi i q k / L}.  A thread owns whole butterflies,
// so the pass is in place.
template <int R>
__device__ void dif_pass(double2 *z, int n, int L, const double2 *tw) {
  const int m = L / R, step = n / L;
  for (int t = threadIdx.x; t < n / R; t += blockDim.x) {
    const int blk = t / m, k = t - blk * m;
    double2 *p = z + blk * L + k;
    double2 x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) x[j] = p[j * m];
    dft_small<R, -1>(x, tw, n);
    p[0] = x[0];
#pragma unroll
    for (int q = 1; q < R; ++q) p[q * m] = cmul(x[q], tw[q * k * step]);
  }
}

// The inverse: decimation in time on sub-transforms of length L = R m; input
// q is multiplied by e^{+2 pi i q k / L} before the DFT.
template <int R>
__device__ void dit_pass(double2 *z, int n, int L, const double2 *tw) {
  const int m = L / R, step = n / L;
  for (int t = threadIdx.x; t < n / R; t += blockDim.x) {
    const int blk = t / m, k = t - blk * m;
    double2 *p = z + blk * L + k;
    double2 x[R];
    x[0] = p[0];
#pragma unroll
    for (int q = 1; q < R; ++q) x[q] = cmulc(p[q * m], tw[q * k * step]);
    dft_small<R, 1>(x, tw, n);
#pragma unroll
    for (int j = 0; j < R; ++j) p[j * m] = x[j];
  }
}

// A pass of a prime radix above 7: one output per thread and step, computed
// into registers from the whole butterfly, then written back after a barrier.
template <int SIGN>
__device__ void prime_pass(double2 *z, int n, int L, int r, const double2 *tw) {
  const int m = L / r, step = n / L, s = n / r;
  double2 res[kMaxPerThread];
#pragma unroll
  for (int c = 0; c < kMaxPerThread; ++c) {
    const int o = threadIdx.x + c * kThreads;
    if (o < n) {
      const int blk = o / L, rem = o - blk * L;
      const int q = rem / m, k = rem - q * m;
      const double2 *p = z + blk * L + k;
      double2 acc = make_double2(0.0, 0.0);
      int e = 0;  // (j q) mod r
      for (int j = 0; j < r; ++j) {
        double2 v = p[j * m];
        if (SIGN > 0 && j) v = cmulc(v, tw[j * k * step]);  // DIT: input twiddle
        const double2 w = tw[e * s];
        acc = cadd(acc, SIGN < 0 ? cmul(v, w) : cmulc(v, w));
        e += q;
        if (e >= r) e -= r;
      }
      if (SIGN < 0 && q) acc = cmul(acc, tw[q * k * step]);  // DIF: output twiddle
      res[c] = acc;
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < kMaxPerThread; ++c) {
    const int o = threadIdx.x + c * kThreads;
    if (o < n) z[o] = res[c];
  }
}

template <int SIGN, bool PRIME>
__device__ void run_pass(double2 *z, int n, int L, int r, const double2 *tw) {
  switch (r) {
    case 8: SIGN < 0 ? dif_pass<8>(z, n, L, tw) : dit_pass<8>(z, n, L, tw); break;
    case 4: SIGN < 0 ? dif_pass<4>(z, n, L, tw) : dit_pass<4>(z, n, L, tw); break;
    case 2: SIGN < 0 ? dif_pass<2>(z, n, L, tw) : dit_pass<2>(z, n, L, tw); break;
    case 3: SIGN < 0 ? dif_pass<3>(z, n, L, tw) : dit_pass<3>(z, n, L, tw); break;
    case 5: SIGN < 0 ? dif_pass<5>(z, n, L, tw) : dit_pass<5>(z, n, L, tw); break;
    case 7: SIGN < 0 ? dif_pass<7>(z, n, L, tw) : dit_pass<7>(z, n, L, tw); break;
    default:
      if constexpr (PRIME) prime_pass<SIGN>(z, n, L, r, tw);
      break;
  }
}

// Any length: the radices of the plan, passes dispatched at run time.  PRIME:
// the length has a prime factor above 7 (a separate instantiation, so that the
// register buffer of prime_pass does not weigh on the common lengths).
template <bool PRIME>
struct GeneralFft {
  static constexpr int kMinBlocks = PRIME ? 1 : 3;
  const Axis &a;
  static constexpr size_t extra_smem(int) { return 0; }
  __device__ __forceinline__ GeneralFft(const Axis &ax, double2 *) : a(ax) {}
  __device__ __forceinline__ int n() const { return a.rad.n; }
  // shared-memory slot of element idx
  __device__ __forceinline__ int at(int idx) const { return idx; }

  // natural order in, digit-reversed order out
  __device__ void forward(double2 *z) const {
    int L = a.rad.n;
    for (int s = 0; s < a.rad.count; ++s) {
      __syncthreads();
      run_pass<-1, PRIME>(z, a.rad.n, L, a.rad.r[s], a.tw);
      L /= a.rad.r[s];
    }
    __syncthreads();
  }
  // unscaled inverse: digit-reversed order in, natural order out
  __device__ void inverse(double2 *z) const {
    int L = 1;
    for (int s = a.rad.count - 1; s >= 0; --s) {
      L *= a.rad.r[s];
      __syncthreads();
      run_pass<1, PRIME>(z, a.rad.n, L, a.rad.r[s], a.tw);
    }
    __syncthreads();
  }
  // position of frequency k in the forward output
  __device__ __forceinline__ int rev(int k) const {
    int pos = 0, L = a.rad.n;
    for (int s = 0; s < a.rad.count; ++s) {
      const int r = a.rad.r[s];
      const int q = k % r;
      k /= r;
      L /= r;
      pos += q * L;
    }
    return pos;
  }
};

// Lengths 2^LOG2N (64 .. 8192): radix-8 passes and one radix-2 or -4 pass,
// every index a shift or a mask known at compile time.
//
// Shared memory: a warp's 16-byte accesses are served eight lanes at a time,
// without conflict when those eight lanes hit eight different 128-byte bank
// rows' slots (idx & 7).  Butterflies of stride 4, 2 or 1 and the
// digit-reversed reads (strides N/8, N/64, ...) would all land on one slot, so
// element idx is stored at idx ^ fold(idx >> 3), fold = XOR of the octal
// digits: a permutation inside every aligned group of eight that gives
// distinct slots to any eight elements spaced by a power of eight, by four
// (with the pair offset of the radix-8 passes) or by one.
//
// Twiddles: one e^{-2 pi i m / N} per butterfly from two small shared tables,
// hi[m >> 6] * lo[m & 63], and its powers by multiplication (the butterfly of
// radix R needs w^q, q < R).
template <int LOG2N>
struct Pow2Fft {
  static constexpr int N = 1 << LOG2N;
  static constexpr int S8 = LOG2N / 3;            // radix-8 passes
  static constexpr int REM = LOG2N % 3;           // last pass radix 2^REM (none if 0)
  static constexpr int NST = S8 + (REM ? 1 : 0);
  static constexpr int HI = N >> 6;
  static constexpr int kMinBlocks = 3;
  static constexpr size_t extra_smem(int) { return (size_t)(HI + 64) * sizeof(double2); }
  const double2 *hi, *lo;

  // fill the tables from the plan's length-N table (every thread calls this)
  __device__ __forceinline__ Pow2Fft(const Axis &a, double2 *tables) {
    double2 *h = tables, *l = tables + HI;
    for (int j = threadIdx.x; j < HI + 64; j += blockDim.x)
      if (j < HI) h[j] = a.tw[j << 6];
      else l[j - HI] = a.tw[j - HI];
    hi = h;
    lo = l;
  }
  __device__ __forceinline__ int n() const { return N; }
  __device__ __forceinline__ double2 w(int m) const { return cmul(hi[m >> 6], lo[m & 63]); }
  __device__ __forceinline__ static int at(int idx) {
    int x = idx >> 3, f = x;
#pragma unroll
    for (int d = 3; d < LOG2N - 3; d += 3) f ^= x >> d;
    return idx ^ (f & 7);
  }

  __host__ __device__ static constexpr int lr(int s) { return s < S8 ? 3 : REM; }

  // w^q for q < R from w = e^{SIGN 2 pi i m / N}
  template <int R>
  __device__ __forceinline__ static void powers(double2 (&t)[R], double2 w1) {
    t[0] = make_double2(1.0, 0.0);
    if constexpr (R > 1) t[1] = w1;
    if constexpr (R > 2) t[2] = cmul(w1, w1);
    if constexpr (R > 3) t[3] = cmul(t[2], w1);
    if constexpr (R > 4) {
      t[4] = cmul(t[2], t[2]);
      t[5] = cmul(t[4], w1);
      t[6] = cmul(t[3], t[3]);
      t[7] = cmul(t[6], w1);
    }
  }

  template <int S, int SIGN>
  __device__ __forceinline__ void pass(double2 *z) const {
    constexpr int LR = lr(S), R = 1 << LR;
    constexpr int LL = LOG2N - 3 * S;  // log2 of the sub-transform length
    constexpr int LM = LL - LR;        // log2 of the butterfly stride
    for (int t = threadIdx.x; t < (N >> LR); t += blockDim.x) {
      const int k = t & ((1 << LM) - 1);
      const int base = ((t >> LM) << LL) + k;
      double2 x[R], tw[R];
      powers<R>(tw, w(k << (3 * S)));
      if constexpr (SIGN < 0) {
#pragma unroll
        for (int j = 0; j < R; ++j) x[j] = z[at(base + (j << LM))];
        dft_small<R, -1>(x, nullptr, N);
#pragma unroll
        for (int q = 0; q < R; ++q) z[at(base + (q << LM))] = q ? cmul(x[q], tw[q]) : x[q];
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const double2 v = z[at(base + (q << LM))];
          x[q] = q ? cmulc(v, tw[q]) : v;
        }
        dft_small<R, 1>(x, nullptr, N);
#pragma unroll
        for (int j = 0; j < R; ++j) z[at(base + (j << LM))] = x[j];
      }
    }
  }

  template <int S>
  __device__ __forceinline__ void fwd_from(double2 *z) const {
    if constexpr (S < NST) {
      __syncthreads();
      pass<S, -1>(z);
      fwd_from<S + 1>(z);
    }
  }
  template <int S>
  __device__ __forceinline__ void inv_from(double2 *z) const {
    if constexpr (S >= 0) {
      __syncthreads();
      pass<S, 1>(z);
      inv_from<S - 1>(z);
    }
  }
  __device__ void forward(double2 *z) const {
    fwd_from<0>(z);
    __syncthreads();
  }
  __device__ void inverse(double2 *z) const {
    inv_from<NST - 1>(z);
    __syncthreads();
  }
  // digit q_S of k (radix of pass S) lands at stride N / (r_0 ... r_S)
  __device__ __forceinline__ int rev(int k) const {
    int pos = 0;
#pragma unroll
    for (int S = 0; S < S8; ++S) pos |= ((k >> (3 * S)) & 7) << (LOG2N - 3 * S - 3);
    if constexpr (REM) pos |= (k >> (3 * S8)) & ((1 << REM) - 1);
    return pos;
  }
};

// Where sample j of a line sits in Makhoul's even/odd reordering.
__device__ __forceinline__ int mak(int j, int n) { return (j & 1) ? n - 1 - (j >> 1) : (j >> 1); }

// Forward DCT coefficients of the two lines packed in Z, at frequency k and
// its partner n - k (k in 1 .. n-1): X_a[k], X_b[k], X_a[n-k], X_b[n-k].
struct Coef4 {
  double ak, bk, an, bn;
};

__device__ __forceinline__ Coef4 split(double2 zk, double2 zn, double2 tk, double2 tn) {
  // A_k = (Z_k + conj Z_{n-k}) / 2, B_k = (Z_k - conj Z_{n-k}) / 2i; A_{n-k} = conj A_k
  const double2 A = make_double2(0.5 * (zk.x + zn.x), 0.5 * (zk.y - zn.y));
  const double2 B = make_double2(0.5 * (zk.y + zn.y), 0.5 * (zn.x - zk.x));
  Coef4 c;
  c.ak = tk.x * A.x - tk.y * A.y;  // Re(t_k A_k)
  c.bk = tk.x * B.x - tk.y * B.y;
  c.an = tn.x * A.x + tn.y * A.y;  // Re(t_{n-k} conj A_k)
  c.bn = tn.x * B.x + tn.y * B.y;
  return c;
}

// W_k = conj(t_k) (X_k - i X_{n-k}) for both lines, packed as W_a + i W_b.
__device__ __forceinline__ double2 pack_inverse(double xa, double xan, double xb, double xbn,
                                                double2 tk) {
  // conj(t) (x - i y) = (c + i s)(x - i y) with t = c - i s
  const double c = tk.x, s = -tk.y;
  const double2 wa = make_double2(c * xa + s * xan, s * xa - c * xan);
  const double2 wb = make_double2(c * xb + s * xbn, s * xb - c * xbn);
  return make_double2(wa.x - wb.y, wa.y + wb.x);
}

// The kernels below are bound by memory latency (two lines per CTA, a few
// CTAs per SM), so every loop that reads global memory first issues the loads
// of kLoads (kTables for table reads) iterations, then uses them.
constexpr int kLoads = 8;
constexpr int kTables = 4;

// Pass 1: rows r0, r0 + 1 of b -> their DCT-II coefficients along x in T.
template <class F>
__global__ void __launch_bounds__(kThreads, F::kMinBlocks) k_dct_rows(double *__restrict__ T,
                                                          long long tpitch,
                                                          const double *__restrict__ b,
                                                          long long bpitch, int h, Axis ax) {
  extern __shared__ double2 z[];
  const int n = ax.rad.n;
  const F fft(ax, z + n);
  const int r0 = 2 * blockIdx.x;
  const bool two = r0 + 1 < h;
  const double *ra = b + (long long)r0 * bpitch;
  const double *rb = ra + bpitch;
  for (int j0 = threadIdx.x; j0 < n; j0 += kLoads * kThreads) {
    double va[kLoads], vb[kLoads];
#pragma unroll
    for (int u = 0; u < kLoads; ++u) {
      const int j = j0 + u * kThreads;
      va[u] = j < n ? ra[j] : 0.0;
      vb[u] = (two && j < n) ? rb[j] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kLoads; ++u) {
      const int j = j0 + u * kThreads;
      if (j < n) z[fft.at(mak(j, n))] = make_double2(va[u], vb[u]);
    }
  }
  fft.forward(z);
  double *ta = T + (long long)r0 * tpitch;
  double *tb = ta + tpitch;
  for (int k0 = threadIdx.x; k0 < n; k0 += kTables * kThreads) {
    double2 tk[kTables], tn[kTables];
#pragma unroll
    for (int u = 0; u < kTables; ++u) {
      const int k = min(k0 + u * kThreads, n - 1);
      tk[u] = ax.post[k];
      tn[u] = ax.post[k ? n - k : 0];
    }
#pragma unroll
    for (int u = 0; u < kTables; ++u) {
      const int k = k0 + u * kThreads;
      if (k >= n) break;
      const Coef4 c = split(z[fft.at(fft.rev(k))], z[fft.at(fft.rev(k ? n - k : 0))], tk[u],
                            tn[u]);
      ta[k] = c.ak;
      if (two) tb[k] = c.bk;
    }
  }
}

// Pass 2: columns c0, c0 + 1 of T: DCT-II along y, division by the
// eigenvalues (the constant mode set to zero), DCT-III along y.
template <class F>
__global__ void __launch_bounds__(kThreads, F::kMinBlocks) k_dct_cols(double *__restrict__ T,
                                                          long long tpitch, int w, Axis ay,
                                                          const double *eig_w) {
  extern __shared__ double2 z[];
  const int n = ay.rad.n;
  const F fft(ay, z + n);
  const int c0 = 2 * blockIdx.x;
  const bool two = c0 + 1 < w;
  double *col = T + c0;
  for (int i0 = threadIdx.x; i0 < n; i0 += kLoads * kThreads) {
    double2 v[kLoads];
#pragma unroll
    for (int u = 0; u < kLoads; ++u) {
      const int i = i0 + u * kThreads;
      const double *p = col + (long long)min(i, n - 1) * tpitch;
      v[u] = two ? *reinterpret_cast<const double2 *>(p) : make_double2(p[0], 0.0);
    }
#pragma unroll
    for (int u = 0; u < kLoads; ++u) {
      const int i = i0 + u * kThreads;
      if (i < n) z[fft.at(mak(i, n))] = v[u];
    }
  }
  fft.forward(z);
  const double ew_a = eig_w[c0], ew_b = two ? eig_w[c0 + 1] : 0.0;
  for (int k0 = threadIdx.x; k0 <= n / 2; k0 += kTables * kThreads) {
    double2 tk[kTables], tn[kTables];
    double ek[kTables], en[kTables];
#pragma unroll
    for (int u = 0; u < kTables; ++u) {
      const int k = min(k0 + u * kThreads, n / 2);
      tk[u] = ay.post[k];
      tn[u] = ay.post[(n - k) % n];
      ek[u] = ay.eig[k];
      en[u] = ay.eig[(n - k) % n];
    }
#pragma unroll
    for (int u = 0; u < kTables; ++u) {
      const int k = k0 + u * kThreads;
      if (k > n / 2) break;
      const int pk = fft.at(fft.rev(k));
      if (k == 0) {
        const double2 z0 = z[pk];  // X_a[0] = Re Z_0, X_b[0] = Im Z_0; W_0 = X_0
        const double la = (ek[u] + ew_a) - 4.0, lb = (ek[u] + ew_b) - 4.0;
        // mode (0, 0) is the constant: zero (the zero-mean solution)
        z[pk] = make_double2(c0 == 0 ? 0.0 : z0.x / la, z0.y / lb);
        continue;
      }
      const int nk = n - k;
      const int pn = fft.at(fft.rev(nk));
      Coef4 c = split(z[pk], z[pn], tk[u], tn[u]);
      c.ak /= (ek[u] + ew_a) - 4.0;
      c.bk /= (ek[u] + ew_b) - 4.0;
      c.an /= (en[u] + ew_a) - 4.0;
      c.bn /= (en[u] + ew_b) - 4.0;
      z[pk] = pack_inverse(c.ak, c.an, c.bk, c.bn, tk[u]);
      if (nk != k) z[pn] = pack_inverse(c.an, c.ak, c.bn, c.bk, tn[u]);
    }
  }
  fft.inverse(z);
  const double inv_n = 1.0 / (double)n;
  for (int i = threadIdx.x; i < n; i += kThreads) {
    const double2 v = z[fft.at(mak(i, n))];
    double *p = col + (long long)i * tpitch;
    if (two) *reinterpret_cast<double2 *>(p) = make_double2(v.x * inv_n, v.y * inv_n);
    else p[0] = v.x * inv_n;
  }
}

// Pass 3: rows r0, r0 + 1 of T (coefficients along x) -> DCT-III -> u.
template <class F>
__global__ void __launch_bounds__(kThreads, F::kMinBlocks) k_idct_rows(double *__restrict__ u,
                                                           long long upitch,
                                                           const double *__restrict__ T,
                                                           long long tpitch, int h, Axis ax) {
  extern __shared__ double2 z[];
  const int n = ax.rad.n;
  const F fft(ax, z + n);
  const int r0 = 2 * blockIdx.x;
  const bool two = r0 + 1 < h;
  const double *ta = T + (long long)r0 * tpitch;
  const double *tb = two ? ta + tpitch : ta;  // a single row reads its own row twice
  for (int k0 = threadIdx.x; k0 <= n / 2; k0 += kTables * kThreads) {
    double xa[kTables], xb[kTables], xan[kTables], xbn[kTables];
    double2 tk[kTables], tn[kTables];
#pragma unroll
    for (int u = 0; u < kTables; ++u) {
      const int k = min(k0 + u * kThreads, n / 2);
      const int nk = (n - k) % n;
      xa[u] = ta[k];
      xb[u] = tb[k];
      xan[u] = ta[nk];
      xbn[u] = tb[nk];
      tk[u] = ax.post[k];
      tn[u] = ax.post[nk];
    }
#pragma unroll
    for (int u = 0; u < kTables; ++u) {
      const int k = k0 + u * kThreads;
      if (k > n / 2) break;
      const double b0 = two ? xb[u] : 0.0, bn = two ? xbn[u] : 0.0;
      if (k == 0) {
        z[fft.at(fft.rev(0))] = make_double2(xa[u], b0);  // W_0 = X_0 (X_n = 0)
        continue;
      }
      const int nk = n - k;
      z[fft.at(fft.rev(k))] = pack_inverse(xa[u], xan[u], b0, bn, tk[u]);
      if (nk != k) z[fft.at(fft.rev(nk))] = pack_inverse(xan[u], xa[u], bn, b0, tn[u]);
    }
  }
  fft.inverse(z);
  const double inv_n = 1.0 / (double)n;
  double *ua = u + (long long)r0 * upitch;
  double *ub = ua + upitch;
  for (int j = threadIdx.x; j < n; j += kThreads) {
    const double2 v = z[fft.at(mak(j, n))];
    ua[j] = v.x * inv_n;
    if (two) ub[j] = v.y * inv_n;
  }
}

__global__ void k_dct_tables(double2 *tw, double2 *post, double *eig, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double s, c;
  sincospi(2.0 * (double)k / (double)n, &s, &c);
  tw[k] = make_double2(c, -s);
  sincospi((double)k / (2.0 * (double)n), &s, &c);
  post[k] = make_double2(c, -s);
  eig[k] = 2.0 * cos(M_PI * (double)k / (double)n);
}

inline bool has_large_prime(const Radices &r) {
  for (int s = 0; s < r.count; ++s)
    if (r.r[s] > 8) return true;
  return false;
}

inline size_t a256(size_t v) { return (v + 255) & ~(size_t)255; }
inline size_t smem_bytes(int n) { return (size_t)n * sizeof(double2); }
// the most dynamic shared memory any DCT kernel launch asks for (a line of
// kMaxLen complex values and the power-of-two twiddle tables)
constexpr size_t kMaxSmemBytes = (size_t)kMaxLen * sizeof(double2) + Pow2Fft<13>::extra_smem(0);

template <class T>
struct Tag {
  using type = T;
};

// Call fn(Tag<F>{}) with the FFT policy of a length: the power-of-two kernels
// for 64 .. 8192, the general ones otherwise.
template <class Fn>
void with_fft(const Radices &r, Fn &&fn) {
  const int n = r.n;
  if (n >= 64 && (n & (n - 1)) == 0) {
    switch (__builtin_ctz((unsigned)n)) {
      case 6: fn(Tag<Pow2Fft<6>>{}); return;
      case 7: fn(Tag<Pow2Fft<7>>{}); return;
      case 8: fn(Tag<Pow2Fft<8>>{}); return;
      case 9: fn(Tag<Pow2Fft<9>>{}); return;
      case 10: fn(Tag<Pow2Fft<10>>{}); return;
      case 11: fn(Tag<Pow2Fft<11>>{}); return;
      case 12: fn(Tag<Pow2Fft<12>>{}); return;
      case 13: fn(Tag<Pow2Fft<13>>{}); return;
      default: break;
    }
  }
  if (has_large_prime(r)) fn(Tag<GeneralFft<true>>{});
  else fn(Tag<GeneralFft<false>>{});
}

}  // namespace dct
}  // namespace gd

using namespace gd;

struct gd_dct_plan_s {
  int h = 0, w = 0;
  long long tpitch = 0;  // row pitch of the coefficient buffer T (even: column pairs align)
  dct::Radices rh, rw;
  size_t o_t = 0, o_tab_w = 0, o_tab_h = 0, total = 0;
  char *ws = nullptr;
};

namespace {

struct AxisTables {
  double2 *tw, *post;
  double *eig;
};

AxisTables tables(gd_dct_plan p, size_t off, int n) {
  char *b = p->ws + off;
  AxisTables t;
  t.tw = reinterpret_cast<double2 *>(b);
  t.post = t.tw + n;
  t.eig = reinterpret_cast<double *>(t.post + n);
  return t;
}

dct::Axis axis(gd_dct_plan p, bool rows) {
  const int n = rows ? p->w : p->h;
  const AxisTables t = tables(p, rows ? p->o_tab_w : p->o_tab_h, n);
  dct::Axis a;
  a.rad = rows ? p->rw : p->rh;
  a.tw = t.tw;
  a.post = t.post;
  a.eig = t.eig;
  return a;
}

}  // namespace

extern "C" void gd_dct_plan_destroy(gd_dct_plan p) { delete p; }

extern "C" int gd_dct_plan_create(int32_t h, int32_t w, gd_dct_plan *out) {
  GD_REQUIRE(out && h > 1 && w > 1, GD_ERR_ARG,
             "gd_dct_plan_create: the grid needs at least 2 x 2 cells");
  GD_REQUIRE(h <= dct::kMaxLen && w <= dct::kMaxLen, GD_ERR_UNSUPPORTED,
             "gd_dct_plan_create: sides above %d are not supported (grid %d x %d)",
             dct::kMaxLen, h, w);
  *out = nullptr;
  gd_dct_plan p = new gd_dct_plan_s();
  p->h = h;
  p->w = w;
  p->tpitch = (w + 1) & ~1;
  p->rh = dct::factor(h);
  p->rw = dct::factor(w);
  size_t o = 0;
  p->o_t = o;
  o = dct::a256(o + (size_t)h * p->tpitch * sizeof(double));
  p->o_tab_w = o;
  o = dct::a256(o + (size_t)w * (2 * sizeof(double2) + sizeof(double)));
  p->o_tab_h = o;
  o = dct::a256(o + (size_t)h * (2 * sizeof(double2) + sizeof(double)));
  p->total = o;
  *out = p;
  return GD_OK;
}

extern "C" size_t gd_dct_workspace_bytes(gd_dct_plan p) { return p ? p->total : 0; }

extern "C" int gd_dct_plan_bind(gd_dct_plan p, void *ws, size_t bytes, cudaStream_t st) {
  GD_REQUIRE(p && ws, GD_ERR_ARG, "gd_dct_plan_bind: bad arguments");
  GD_REQUIRE(bytes >= p->total, GD_ERR_ARG, "gd_dct_plan_bind: workspace %zu < %zu bytes", bytes,
             p->total);
  GD_REQUIRE(((uintptr_t)ws & 255) == 0, GD_ERR_ARG, "gd_dct_plan_bind: workspace must be "
                                                     "256-byte aligned");
  p->ws = static_cast<char *>(ws);
  const AxisTables tw = tables(p, p->o_tab_w, p->w), th = tables(p, p->o_tab_h, p->h);
  dct::k_dct_tables<<<(p->w + 255) / 256, 256, 0, st>>>(tw.tw, tw.post, tw.eig, p->w);
  dct::k_dct_tables<<<(p->h + 255) / 256, 256, 0, st>>>(th.tw, th.post, th.eig, p->h);
  GD_CHECK_LAUNCH();
  // the tables must be complete before a solve on any stream (set-up, once per plan)
  GD_CHECK_CUDA(cudaStreamSynchronize(st));
  // Shared memory of the kernels this plan launches.  The limit is one value per
  // kernel for the whole process, so every plan sets the same value, the most any
  // length needs: a plan bound later for a shorter line must not lower the limit
  // under a plan of a longer one (its next launch would fail).
  cudaError_t err = cudaSuccess;
  auto allow = [&](const void *fn) {
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)dct::kMaxSmemBytes);
    if (e != cudaSuccess) err = e;
  };
  dct::with_fft(p->rw, [&](auto tag) {
    using F = typename decltype(tag)::type;
    allow((const void *)dct::k_dct_rows<F>);
    allow((const void *)dct::k_idct_rows<F>);
  });
  dct::with_fft(p->rh, [&](auto tag) {
    using F = typename decltype(tag)::type;
    allow((const void *)dct::k_dct_cols<F>);
  });
  GD_CHECK_CUDA(err);
  return GD_OK;
}

extern "C" int gd_dct_solve_neumann(gd_dct_plan p, const double *b_in, double *u, int32_t pitch,
                                    cudaStream_t st) {
  GD_REQUIRE(p && p->ws && b_in && u && pitch >= p->w, GD_ERR_ARG,
             "gd_dct_solve_neumann: bad arguments or unbound plan");
  const int h = p->h, w = p->w;
  double *T = reinterpret_cast<double *>(p->ws + p->o_t);
  const dct::Axis ax = axis(p, true), ay = axis(p, false);
  const unsigned rows = (unsigned)(h + 1) / 2, cols = (unsigned)(w + 1) / 2;
  dct::with_fft(p->rw, [&](auto tag) {
    using F = typename decltype(tag)::type;
    const size_t b = dct::smem_bytes(w) + F::extra_smem(w);
    dct::k_dct_rows<F><<<rows, dct::kThreads, b, st>>>(T, p->tpitch, b_in, pitch, h, ax);
  });
  dct::with_fft(p->rh, [&](auto tag) {
    using F = typename decltype(tag)::type;
    const size_t b = dct::smem_bytes(h) + F::extra_smem(h);
    dct::k_dct_cols<F><<<cols, dct::kThreads, b, st>>>(T, p->tpitch, w, ay, ax.eig);
  });
  dct::with_fft(p->rw, [&](auto tag) {
    using F = typename decltype(tag)::type;
    const size_t b = dct::smem_bytes(w) + F::extra_smem(w);
    dct::k_idct_rows<F><<<rows, dct::kThreads, b, st>>>(u, pitch, T, p->tpitch, h, ax);
  });
  GD_CHECK_LAUNCH();
  return GD_OK;
}
