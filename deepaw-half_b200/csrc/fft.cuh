// Shared-memory mixed-radix (4, 2, 3, 5) FFT engine for pencils of length
// n <= kMaxFFT, used by every transform in the library.
//
// Two in-place stage orders are provided and chosen per pass so that no
// explicit permutation pass is ever needed:
//   * DIF  (decimation in frequency): natural-order input, output X[k] left at
//     position pos(k) (mixed-radix digit reversal);
//   * DIT  (decimation in time, the transposed algorithm): input x[k] placed
//     at pos(k), natural-order output.
// The scatter into (and the gather out of) the transform is where the
// permutation is absorbed: sphere points are scattered straight to pos(k),
// and sphere points are gathered straight from pos(k).
// Sign convention: sign = -1 is exp(-2 pi i jk/n) (the reference's FORWARD),
// sign = +1 is the unnormalised inverse (CUFFT_INVERSE).
#pragma once

#include <vector>

#include "common.h"

namespace hb {

constexpr int kMaxFFT = 128;
constexpr int kMaxStages = 8;

struct FFTPlan {
  int n = 0;
  int nstages = 0;
  int radix[kMaxStages] = {};
  int span[kMaxStages] = {};   // block length entering stage s (DIF order)
};

inline bool fft_size_supported(int n) {
  if (n < 1 || n > kMaxFFT) return false;
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

inline FFTPlan make_fft_plan(int n) {
  if (!fft_size_supported(n))
    fail(kUnavailable, "FFT grid dimension " + std::to_string(n) + " is not a 2^a 3^b 5^c size up to " +
                           std::to_string(kMaxFFT));
  FFTPlan p;
  p.n = n;
  int m = n;
  auto push = [&](int r) { p.radix[p.nstages++] = r; m /= r; };
  while (m % 4 == 0) push(4);
  while (m % 2 == 0) push(2);
  while (m % 3 == 0) push(3);
  while (m % 5 == 0) push(5);
  int L = n;
  for (int s = 0; s < p.nstages; ++s) { p.span[s] = L; L /= p.radix[s]; }
  return p;
}

// pos[k]: storage position of X[k] after a DIF pass (= input slot of x[k] for DIT)
inline std::vector<int> fft_positions(const FFTPlan& p) {
  std::vector<int> pos(p.n);
  for (int k = 0; k < p.n; ++k) {
    int kk = k, q = 0;
    for (int s = 0; s < p.nstages; ++s) {
      int r = p.radix[s];
      q += (kk % r) * (p.span[s] / r);
      kk /= r;
    }
    pos[k] = q;
  }
  return pos;
}

#ifdef __CUDACC__

template <typename C>
__device__ __forceinline__ C mul_i(C a, int sign) {  // (sign * i) * a
  C r;
  r.x = -sign * a.y;
  r.y = sign * a.x;
  return r;
}

// y_p = sum_q x_q exp(sign 2 pi i p q / r), in place on x[0..r-1]
template <typename C, typename R>
__device__ __forceinline__ void butterfly(int r, C* x, int sign) {
  if (r == 4) {
    C a = cadd(x[0], x[2]), b = csub(x[0], x[2]), c = cadd(x[1], x[3]), d = mul_i(csub(x[1], x[3]), sign);
    x[0] = cadd(a, c); x[2] = csub(a, c); x[1] = cadd(b, d); x[3] = csub(b, d);
  } else if (r == 2) {
    C a = x[0];
    x[0] = cadd(a, x[1]); x[1] = csub(a, x[1]);
  } else if (r == 3) {
    const R c3 = R(-0.5), s3 = R(0.86602540378443864676372317075294);
    C t = cadd(x[1], x[2]);
    C u = mul_i(cscale(csub(x[1], x[2]), s3), sign);
    C base = cadd(x[0], cscale(t, c3));
    x[0] = cadd(x[0], t);
    x[1] = cadd(base, u);
    x[2] = csub(base, u);
  } else {  // r == 5
    const R c1 = R(0.30901699437494742410229341718282), s1 = R(0.95105651629515357211643933337938);
    const R c2 = R(-0.80901699437494742410229341718282), s2 = R(0.58778525229247312916870595463907);
    C t1 = cadd(x[1], x[4]), t2 = cadd(x[2], x[3]);
    C u1 = csub(x[1], x[4]), u2 = csub(x[2], x[3]);
    C a1 = cadd(x[0], cadd(cscale(t1, c1), cscale(t2, c2)));
    C a2 = cadd(x[0], cadd(cscale(t1, c2), cscale(t2, c1)));
    C b1 = mul_i(cadd(cscale(u1, s1), cscale(u2, s2)), sign);
    C b2 = mul_i(csub(cscale(u1, s2), cscale(u2, s1)), sign);
    x[0] = cadd(x[0], cadd(t1, t2));
    x[1] = cadd(a1, b1); x[4] = csub(a1, b1);
    x[2] = cadd(a2, b2); x[3] = csub(a2, b2);
  }
}

// Twiddle table exp(-2 pi i t / n), t < n, filled by the block.
template <typename C>
__device__ __forceinline__ void fill_twiddles(C* tw, int n) {
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    double s, c;
    sincospi(-2.0 * double(t) / double(n), &s, &c);
    tw[t].x = c;
    tw[t].y = s;
  }
}

// In-place batched transform of `npencils` pencils held in shared memory;
// element k of pencil p lives at buf[p * pstride + k * estride].  Threads of
// the block cooperate over (pencil, butterfly) pairs; the pencil index runs
// fastest for strided pencils so that a warp touches consecutive addresses.
// `rows`, when given, lists the pencils to transform (pencil p starts at
// rows[p] * pstride) so that all-zero pencils of a pruned transform are skipped.
template <bool DIT, typename C, typename R>
__device__ void fft_pencils(C* buf, int npencils, int pstride, int estride, const FFTPlan& plan,
                            const C* tw, int sign, const int* rows = nullptr) {
  const int n = plan.n;
  for (int si = 0; si < plan.nstages; ++si) {
    const int s = DIT ? plan.nstages - 1 - si : si;
    const int r = plan.radix[s], L = plan.span[s], m = L / r;
    const int per = n / r;
    const int total = npencils * per;
    const int tunit = n / L;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      int p, b;
      if (estride == 1) { p = t / per; b = t - p * per; }
      else { b = t / npencils; p = t - b * npencils; }
      const int blk = b / m, j = b - blk * m;
      C* base = buf + (rows ? rows[p] : p) * pstride + (blk * L + j) * estride;
      const int step = m * estride;
      C x[5];
#pragma unroll
      for (int q = 0; q < 5; ++q)
        if (q < r) x[q] = base[q * step];
      const int tj = j * tunit;
      if (DIT) {
#pragma unroll
        for (int q = 1; q < 5; ++q)
          if (q < r && tj) {
            C w = tw[q * tj];
            if (sign > 0) w.y = -w.y;
            x[q] = cmul(x[q], w);
          }
      }
      butterfly<C, R>(r, x, sign);
      if (!DIT) {
#pragma unroll
        for (int q = 1; q < 5; ++q)
          if (q < r && tj) {
            C w = tw[q * tj];
            if (sign > 0) w.y = -w.y;
            x[q] = cmul(x[q], w);
          }
      }
#pragma unroll
      for (int q = 0; q < 5; ++q)
        if (q < r) base[q * step] = x[q];
    }
    __syncthreads();
  }
}

// Plan + position table as kernel arguments (passed by value).
struct AxisPlan {
  FFTPlan plan;
  int pos[kMaxFFT];
};

inline AxisPlan make_axis_plan(int n) {
  AxisPlan a;
  a.plan = make_fft_plan(n);
  auto p = fft_positions(a.plan);
  for (int k = 0; k < n; ++k) a.pos[k] = p[k];
  for (int k = n; k < kMaxFFT; ++k) a.pos[k] = 0;
  return a;
}

#endif  // __CUDACC__

}  // namespace hb
