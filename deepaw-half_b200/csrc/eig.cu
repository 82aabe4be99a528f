// Small dense Hermitian eigensolvers for the ACC subspace problems, device
// resident and free of host synchronisation.
//
// The reference calls cuSOLVER zheevd (m x m metric) and zhegvd (2m x 2m
// Rayleigh-Ritz) once per iteration (src/half_cuda_iterative_solver.cuf:
// 242-275).  For the sizes the solver meets (m <= a few hundred) those calls
// are dominated by per-reflector back-transformation launches and a host
// round trip.  Here the same reduction is kept -- B = U^H U (Cholesky),
// C = U^-H A U^-1, Householder tridiagonalisation (cuSOLVER zhetrd) -- and
// the rest is done by two kernels of this file:
//
//   tridiag_eig_kernel   eigenvalues of the real symmetric tridiagonal T by
//                        multisection on Sturm counts (a group of warp lanes
//                        per eigenvalue), eigenvectors by inverse iteration on
//                        the pivoted tridiagonal LU; eigenvalues closer than
//                        1e-7 ||T|| form clusters whose members are iterated in
//                        order and Gram-Schmidt orthogonalised against each
//                        other (the strategy of LAPACK's dstebz/dstein);
//   back_transform_kernel V = Q Z with Q = H(n-1)...H(1) from zhetrd's
//                        reflectors, one warp per eigenvector.
//
// The eigenvectors are finally Y = U^-1 V (trsm), giving Y^H B Y = I, the
// same normalisation as zhegvd (itype 1, upper).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>

#include "blas.h"
#include "context.h"
#include "eig.h"

namespace hb {

namespace {

constexpr int kEigThreads = 512;
constexpr int kExtraEig = 8;   // eigenvalues located beyond the wanted ones (cluster at the cut)
constexpr int kMetricMax = 164;   // packed triangle + two m-vectors within kSmemMax
constexpr size_t kSmemMax = 226 * 1024;   // dynamic shared memory per CTA, leaving room for static

// Number of eigenvalues of T below x (Sylvester inertia of T - x I).  The
// pivots of the LDL^T factorisation are ratios q_i = p_i / p_{i-1} of the
// continuant p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2}, so the count is the
// number of sign changes along p_0 = 1, p_1, ..., p_n.  Carrying p instead of
// q keeps divisions off the dependent chain (one FMA per step).  A pivot of
// magnitude below kPivFloor is replaced by -kPivFloor (LAPACK dstebz does the
// same with its pivmin), and the pair (p_{i-1}, p_i) is rescaled by a power
// of two whenever p_i leaves [2^-300, 2^300], which changes no ratio.
constexpr double kPivFloor = 0x1p-400;

__device__ int sturm_count(const double* d, const double* e2, int n, double x) {
  double p0 = 1.0, p1 = d[0] - x;
  if (fabs(p1) < kPivFloor) p1 = -kPivFloor;
  int c = p1 < 0.0;
  for (int i = 1; i < n; ++i) {
    double p2 = fma(d[i] - x, p1, -e2[i - 1] * p0);
    const double lim = kPivFloor * fabs(p1);
    if (fabs(p2) < lim) p2 = p1 < 0.0 ? lim : -lim;
    c += (p2 < 0.0) != (p1 < 0.0);
    p0 = p1;
    p1 = p2;
    const double a = fabs(p1);
    if (a > 0x1p300 || a < 0x1p-300) {   // |p_i| in [2^-700, 2^330] here; bring it to [1, 2)
      const double sc = scalbn(1.0, -ilogb(p1));
      p0 *= sc;
      p1 *= sc;
    }
  }
  return c;
}

// LU factorisation with partial pivoting of T - lambda I (O(n)); the pivots
// are stored inverted so that the solves multiply.  ai, b1, b2, l and piv are
// per-thread scratch of n elements at stride st (the slots of a batch of
// threads are interleaved, so a warp touches consecutive words).
__device__ void tri_factor(const double* d, const double* e, int n, double lam, double tiny, double* ai, double* b1,
                           double* b2, double* l, unsigned char* piv, int st) {
  double diag = d[0] - lam, sup = n > 1 ? e[0] : 0.0;
  for (int i = 0; i < n - 1; ++i) {
    const double sub = e[i];
    const double nd = d[i + 1] - lam, ns = (i + 1 < n - 1) ? e[i + 1] : 0.0;
    const int o = i * st;
    if (fabs(diag) >= fabs(sub)) {
      if (fabs(diag) < tiny) diag = diag < 0 ? -tiny : tiny;
      const double r = 1.0 / diag, m = sub * r;
      ai[o] = r; b1[o] = sup; b2[o] = 0.0; l[o] = m; piv[o] = 0;
      diag = nd - m * sup;
      sup = ns;
    } else {
      const double r = 1.0 / sub, m = diag * r;
      ai[o] = r; b1[o] = nd; b2[o] = ns; l[o] = m; piv[o] = 1;
      diag = sup - m * nd;
      sup = -m * ns;
    }
  }
  if (fabs(diag) < tiny) diag = diag < 0 ? -tiny : tiny;
  const int o = (n - 1) * st;
  ai[o] = 1.0 / diag;
  b1[o] = 0.0;
  b2[o] = 0.0;
}

// The running values of both sweeps stay in registers, so the dependent
// chain of a step is one or two FMAs, not a shared-memory round trip.
__device__ void tri_solve(int n, const double* ai, const double* b1, const double* b2, const double* l,
                          const unsigned char* piv, double* x, int st) {
  double cur = x[0];
  for (int i = 0; i < n - 1; ++i) {   // forward: L^-1 with the row swaps
    const int o = i * st;
    const double nxt = x[o + st], li = l[o];
    if (piv[o]) {
      x[o] = nxt;
      cur = cur - li * nxt;
    } else {
      x[o] = cur;
      cur = nxt - li * cur;
    }
  }
  const int on = (n - 1) * st;
  double x1 = cur * ai[on];   // x(i+1)
  x[on] = x1;
  if (n == 1) return;
  const int om = (n - 2) * st;
  double x0 = (x[om] - b1[om] * x1) * ai[om];   // x(i)
  x[om] = x0;
  for (int i = n - 3; i >= 0; --i) {   // backward: U^-1
    const int o = i * st;
    const double xi = (x[o] - b1[o] * x0 - b2[o] * x1) * ai[o];
    x[o] = xi;
    x1 = x0;
    x0 = xi;
  }
}

// One CTA: eigenvalues 0..nev-1 of T (ascending) and their eigenvectors Z (n x nev).
__global__ void __launch_bounds__(kEigThreads) tridiag_eig_kernel(const double* __restrict__ d_in,
                                                                  const double* __restrict__ e_in, int n, int nev,
                                                                  double* __restrict__ w, double* __restrict__ Z,
                                                                  double* __restrict__ gscratch, int batch,
                                                                  int* __restrict__ status) {
  // Eigenvalues up to ne = nev + kExtraEig are located so that a cluster
  // straddling the last wanted index is computed (and orthogonalised) whole;
  // only the first nev pairs are returned.
  const int ne = min(n, nev + kExtraEig);
  extern __shared__ double sm[];
  double* d = sm;
  double* e = d + n;
  double* e2 = e + n;
  double* lam = e2 + n;
  int* cl_first = reinterpret_cast<int*>(lam + ne);
  __shared__ double s_gl, s_gu, s_norm;
  if (threadIdx.x == 0) *status = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = d_in[i];
    double ei = i < n - 1 ? e_in[i] : 0.0;
    e[i] = ei;
    e2[i] = ei * ei;
  }
  __syncthreads();
  if (threadIdx.x == 0) {   // Gershgorin interval and norm
    double gl = d[0], gu = d[0], nrm = 0;
    for (int i = 0; i < n; ++i) {
      double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
      gl = fmin(gl, d[i] - r);
      gu = fmax(gu, d[i] + r);
      nrm = fmax(nrm, fabs(d[i]) + r);
    }
    double pad = 2.0 * DBL_EPSILON * fmax(fabs(gl), fabs(gu)) * n + 1e-300;
    s_gl = gl - pad;
    s_gu = gu + pad;
    s_norm = fmax(nrm, DBL_MIN);
  }
  __syncthreads();
  const double tnorm = s_norm;
  // Multisection: a group of g lanes (a power of two, inside one warp) owns
  // one eigenvalue; each round its lanes count at g interior points, and the
  // bracket shrinks to the pair of neighbouring points whose counts straddle
  // the index, a factor g + 1 per round.  Brackets end at 2 eps |lambda| +
  // eps ||T|| (absolute accuracy eps ||T||, as bisection guarantees).
  {
    int g = 1;
    while (g < 32 && 2 * g * ne <= int(blockDim.x)) g *= 2;
    const int lane = threadIdx.x & 31, gl = lane & (g - 1), gbase = lane & ~(g - 1);
    const unsigned gmask = g == 32 ? 0xffffffffu : (((1u << g) - 1u) << gbase);
    const int groups = blockDim.x / g;
    const int slots = (ne + groups - 1) / groups;   // same trip count on every thread
    for (int sidx = 0; sidx < slots; ++sidx) {
      const int k = sidx * groups + int(threadIdx.x) / g;
      const bool active = k < ne;
      double lo = s_gl, hi = s_gu;
      bool done = !active;
      for (int round = 0; round < 200; ++round) {
        if (!done && hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + DBL_EPSILON * tnorm) done = true;
        if (__all_sync(0xffffffffu, done)) break;
        const double x = lo + (hi - lo) * double(gl + 1) / double(g + 1);
        const bool above = !done && sturm_count(d, e2, n, x) > k;   // lambda_k < x
        const unsigned b = __ballot_sync(0xffffffffu, above) & gmask;
        const int first = b ? (__ffs(b) - 1 - gbase) : g;          // first point above lambda_k
        const double xlo = __shfl_sync(0xffffffffu, x, gbase + (first > 0 ? first - 1 : 0));
        const double xhi = __shfl_sync(0xffffffffu, x, gbase + (first < g ? first : g - 1));
        if (!done) {
          const double nlo = first > 0 ? xlo : lo, nhi = first < g ? xhi : hi;
          if (!(nlo > lo || nhi < hi)) done = true;   // no progress left in floating point
          lo = nlo;
          hi = nhi;
        }
      }
      if (active && gl == 0) lam[k] = 0.5 * (lo + hi);
    }
  }
  __syncthreads();
  // Clusters: consecutive eigenvalues closer than 1e-7 ||T||.  Outside a cluster
  // inverse iteration alone keeps |<z_i, z_j>| <= eps ||T|| / gap <~ 1e-9;
  // inside, members are Gram-Schmidt orthogonalised against each other
  // (LAPACK's dstein uses 1e-3 ||T||, which would serialise the dense Ritz
  // spectra met here).
  const double ortol = 1.0e-7 * tnorm;
  if (threadIdx.x == 0) {
    int first = 0;
    for (int k = 0; k < ne; ++k) {
      if (k > 0 && lam[k] - lam[k - 1] > ortol) first = k;
      cl_first[k] = first;
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nev; k += blockDim.x) w[k] = lam[k];
  // Inverse iteration, in batches of `batch` threads whose scratch (five
  // n-vectors and the pivot flags, interleaved by thread) sits in shared
  // memory after the tables when it fits (gscratch == nullptr), else in
  // global memory.  The thread owning a cluster's first member computes the
  // whole cluster.
  const double tiny = DBL_EPSILON * tnorm;
  double* sbase = gscratch;
  if (!sbase) {
    size_t off = (3 * size_t(n) + ne) * sizeof(double) + size_t(ne) * sizeof(int);
    off = (off + 15) & ~size_t(15);
    sbase = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(sm) + off);
  }
  const int st = batch;
  for (int b0 = 0; b0 < nev; b0 += batch) {
    const int t = threadIdx.x;
    const int k0 = b0 + t;
    if (t < batch && k0 < nev && cl_first[k0] == k0) {
      double* ai = sbase + t;
      double* b1 = ai + size_t(n) * st;
      double* b2 = b1 + size_t(n) * st;
      double* l = b2 + size_t(n) * st;
      double* x = l + size_t(n) * st;
      unsigned char* piv = reinterpret_cast<unsigned char*>(sbase + 5 * size_t(n) * st) + t;
      int k1 = k0;
      while (k1 + 1 < ne && cl_first[k1 + 1] == k0) ++k1;
      double prev = -HUGE_VAL;
      for (int k = k0; k <= k1; ++k) {
        double lk = lam[k];
        // separate numerically equal eigenvalues of a cluster (dstein)
        double sep = 10.0 * DBL_EPSILON * fmax(fabs(lk), tnorm * 1e-3);
        if (k > k0 && lk - prev < sep) lk = prev + sep;
        prev = lk;
        tri_factor(d, e, n, lk, tiny, ai, b1, b2, l, piv, st);
        unsigned s = 0x9E3779B9u * (k + 1);
        for (int i = 0; i < n; ++i) {   // deterministic pseudo-random start vector
          s = s * 1664525u + 1013904223u;
          x[i * st] = 1.0 + 0.5 * (double(s >> 8) / 16777216.0 - 0.5);
        }
        // With an eigenvalue accurate to rounding each solve amplifies the
        // wanted direction by ~gap / (eps ||T||): two solves for an isolated
        // eigenvalue, three (each followed by Gram-Schmidt against the earlier
        // members) inside a cluster.
        const int steps = k1 > k0 ? 3 : 2;
        for (int it = 0; it < steps; ++it) {
          tri_solve(n, ai, b1, b2, l, piv, x, st);
          for (int j = k0; j < k; ++j) {
            const double* y = Z + (size_t)j * n;
            double dot = 0;
            for (int i = 0; i < n; ++i) dot += y[i] * x[i * st];
            for (int i = 0; i < n; ++i) x[i * st] -= dot * y[i];
          }
          double nrm = 0;
          for (int i = 0; i < n; ++i) nrm += x[i * st] * x[i * st];
          nrm = sqrt(nrm);
          if (!(nrm > 0) || !isfinite(nrm)) { atomicExch(status, 1); break; }
          const double inv = 1.0 / nrm;
          for (int i = 0; i < n; ++i) x[i * st] *= inv;
        }
        // sign convention: largest component positive
        double big = 0;
        for (int i = 0; i < n; ++i) if (fabs(x[i * st]) > fabs(big)) big = x[i * st];
        const double sg = big < 0 ? -1.0 : 1.0;
        double* z = Z + (size_t)k * n;
        for (int i = 0; i < n; ++i) z[i] = sg * x[i * st];
      }
    }
    __syncthreads();   // the next batch reuses the slots
  }
}

// V[:, j] = H(1) H(2) ... applied as Q z_j with Q = H(n-1) ... H(1)
// (LAPACK zhetrd, UPLO = 'U': v(i) = 1, v(1:i-1) = A(1:i-1, i+1), tau(i)).
__global__ void back_transform_kernel(const double2* __restrict__ A, const double2* __restrict__ tau,
                                      const double* __restrict__ Z, int n, int nev, double2* __restrict__ V) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + warp;
  if (j >= nev) return;
  extern __shared__ double2 xs[];
  double2* x = xs + (size_t)warp * n;
  for (int r = lane; r < n; r += 32) x[r] = make_double2(Z[(size_t)j * n + r], 0.0);
  __syncwarp();
  for (int i0 = 0; i0 <= n - 2; ++i0) {
    const double2* v = A + (size_t)(i0 + 1) * n;   // column i0+1, rows 0..i0-1; v[i0] = 1
    const double2 t = tau[i0];
    double wr = 0, wi = 0;
    for (int r = lane; r <= i0; r += 32) {
      double2 vr = r == i0 ? make_double2(1.0, 0.0) : v[r];
      double2 xr = x[r];
      wr += vr.x * xr.x + vr.y * xr.y;      // conj(v) . x
      wi += vr.x * xr.y - vr.y * xr.x;
    }
    for (int off = 16; off > 0; off >>= 1) {
      wr += __shfl_xor_sync(0xffffffffu, wr, off);
      wi += __shfl_xor_sync(0xffffffffu, wi, off);
    }
    // x -= tau * w * v
    double cr = t.x * wr - t.y * wi, ci = t.x * wi + t.y * wr;
    for (int r = lane; r <= i0; r += 32) {
      double2 vr = r == i0 ? make_double2(1.0, 0.0) : v[r];
      x[r].x -= cr * vr.x - ci * vr.y;
      x[r].y -= cr * vr.y + ci * vr.x;
    }
    __syncwarp();
  }
  for (int r = lane; r < n; r += 32) V[(size_t)j * n + r] = x[r];
}

// lower triangle from the upper one (Hermitian)
__global__ void hermitian_fill_kernel(double2* A, int n) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  int j = int(t / n), i = int(t - (long long)j * n);
  if (i > j) {
    double2 u = A[(long long)i * n + j];
    A[t] = make_double2(u.x, -u.y);
  } else if (i == j) {
    A[t].y = 0.0;
  }
}

// S-metric normalisation of the ACC correction block without an
// eigendecomposition.  Given M = P^H S P (m x m, upper triangle read), write
// U (m x m, upper triangular) with (P U)^H S (P U) = I up to the floor:
//   D = diag(M)^-1/2,  D M D = R^H R (Cholesky, pivots floored at 1e-14),
//   U = D R^-1.
// P U spans what P spans (the reference's eigenvector basis U Lambda^-1/2
// spans the same space), so the Rayleigh-Ritz step that follows sees the
// same subspace; the floor plays the role of the reference's 1e-14 floor on
// the metric eigenvalues for nearly dependent directions.  One CTA; the
// packed upper triangle of D M D lives in shared memory (m <= kMetricMax).
// *status = 1 if a pivot was not finite.
__global__ void __launch_bounds__(512) metric_cholesky_kernel(double2* __restrict__ M, int m,
                                                              int* __restrict__ status) {
  extern __shared__ double2 pk[];   // packed upper: (i, j), i <= j at j (j + 1) / 2 + i
  double* dsc = reinterpret_cast<double*>(pk + size_t(m) * (m + 1) / 2);
  double2* col = reinterpret_cast<double2*>(dsc + m);
  __shared__ double s_inv;
  __shared__ int s_bad;
  const int tid = threadIdx.x, nt = blockDim.x;
  auto at = [](int i, int j) { return j * (j + 1) / 2 + i; };
  if (tid == 0) s_bad = 0;
  for (int j = tid; j < m; j += nt) dsc[j] = 1.0 / sqrt(fmax(M[size_t(j) * m + j].x, DBL_MIN));
  __syncthreads();
  for (int q = tid; q < m * m; q += nt) {
    const int i = q % m, j = q / m;
    if (i <= j) {
      double2 v = M[size_t(j) * m + i];
      if (i == j) v.y = 0.0;
      pk[at(i, j)] = cscale(v, dsc[i] * dsc[j]);
    }
  }
  __syncthreads();
  // Right-looking Cholesky, row k of R overwrites row k of the triangle.  A
  // pivot at or below 1e-14 (of the unit scaled diagonal) marks a direction
  // dependent on the earlier ones to working precision: R(k,k) = 1e-7 and
  // the rest of its row is zero, so the direction stays in the span without
  // being eliminated from later columns (no growth from indefinite rounding).
  const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
  for (int k = 0; k < m; ++k) {
    if (tid == 0) {
      double p = pk[at(k, k)].x;
      if (!isfinite(p)) s_bad = 1;
      double r = 1.0e-7, inv = 0.0;
      if (p > 1.0e-14) { r = sqrt(p); inv = 1.0 / r; }
      pk[at(k, k)] = make_double2(r, 0.0);
      s_inv = inv;
    }
    __syncthreads();
    const double inv = s_inv;
    for (int j = k + 1 + tid; j < m; j += nt) {
      const double2 v = cscale(pk[at(k, j)], inv);
      pk[at(k, j)] = v;
      col[j] = v;
    }
    __syncthreads();
    if (inv != 0.0) {
      for (int j = k + 1 + warp; j < m; j += nw) {   // A(i,j) -= conj(R(k,i)) R(k,j), k < i <= j
        const double2 b = col[j];
        double2* cj = pk + j * (j + 1) / 2;
        for (int i = k + 1 + lane; i <= j; i += 32) {
          const double2 a = col[i];
          cj[i].x -= a.x * b.x + a.y * b.y;
          cj[i].y -= a.x * b.y - a.y * b.x;
        }
      }
    }
    __syncthreads();
  }
  // X = R^-1 column by column, in place: X(i,j) = -X(i, i:j-1) R(i:j-1, j) / R(j,j)
  for (int j = 0; j < m; ++j) {
    for (int i = tid; i <= j; i += nt) col[i] = pk[at(i, j)];
    __syncthreads();
    const double rjj = col[j].x;
    for (int i = warp; i < j; i += nw) {
      double sr = 0, si = 0;
      for (int k = i + lane; k < j; k += 32) {
        const double2 x = pk[at(i, k)], r = col[k];
        sr += x.x * r.x - x.y * r.y;
        si += x.x * r.y + x.y * r.x;
      }
      for (int off = 16; off > 0; off >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, off);
        si += __shfl_xor_sync(0xffffffffu, si, off);
      }
      if (lane == 0) pk[at(i, j)] = make_double2(-sr / rjj, -si / rjj);
    }
    if (tid == 0) pk[at(j, j)] = make_double2(1.0 / rjj, 0.0);
    __syncthreads();
  }
  // U = D X, lower triangle zero
  for (int q = tid; q < m * m; q += nt) {
    const int i = q % m, j = q / m;
    M[q] = i <= j ? cscale(pk[at(i, j)], dsc[i]) : make_double2(0.0, 0.0);
  }
  if (tid == 0) *status = s_bad;
}

// The same normalisation as metric_cholesky_kernel, blocked by 32 columns
// for m <= kBlockedMax (1024 threads): per block row K, one warp factors the
// diagonal block (shuffles, no CTA barrier per column), one warp per column
// solves the panel R_KK^H R_K,J = A_K,J, and the trailing Hermitian update
// is one warp-reduced dot product of two packed column segments per element.
// The inverse X = R^-1 is built the same way: diagonal blocks by one warp
// each, then block column J from T_KJ = sum_L X_KL R_LJ and X_KJ = -T_KJ X_JJ.
// Dependent pivots (<= 1e-14 of the unit scaled diagonal) get R(k,k) = 1e-7
// and a zero row, exactly as in the unblocked kernel.
constexpr int kBlockedMax = 144;   // packed triangle + T blocks ((m - 32) x 32) within kSmemMax

__global__ void __launch_bounds__(1024) metric_cholesky_blocked_kernel(double2* __restrict__ M, int m,
                                                                       int* __restrict__ status) {
  extern __shared__ double2 pk[];   // packed upper triangle, (i, j) at j (j + 1) / 2 + i
  double* dsc = reinterpret_cast<double*>(pk + size_t(m) * (m + 1) / 2);
  double* ipiv = dsc + m;                                   // 1 / R(k,k), 0 for a dependent pivot
  double2* tmp = reinterpret_cast<double2*>(ipiv + m);      // T blocks, [column c][row r], (m - 32) x 32
  __shared__ int s_bad;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
  auto at = [](int i, int j) { return j * (j + 1) / 2 + i; };
  if (tid == 0) s_bad = 0;
  for (int j = tid; j < m; j += nt) dsc[j] = 1.0 / sqrt(fmax(M[size_t(j) * m + j].x, DBL_MIN));
  __syncthreads();
  for (int j = warp; j < m; j += nw) {
    const double dj = dsc[j];
    for (int i = lane; i <= j; i += 32) {
      double2 v = M[size_t(j) * m + i];
      if (i == j) v.y = 0.0;
      pk[at(i, j)] = cscale(v, dsc[i] * dj);
    }
  }
  __syncthreads();
  const int nblk = (m + 31) / 32;
  for (int K = 0; K < nblk; ++K) {
    const int K0 = 32 * K, b = min(32, m - K0), E = K0 + b;
    if (warp == 0) {   // diagonal block: unblocked Cholesky by one warp, lane = column
      const int c = K0 + lane;
      for (int k = 0; k < b; ++k) {
        const int kk = K0 + k;
        const double p = pk[at(kk, kk)].x;
        __syncwarp();
        double r = 1.0e-7, inv = 0.0;
        if (p > 1.0e-14) { r = sqrt(p); inv = 1.0 / r; }
        if (lane == 0) {
          if (!isfinite(p)) s_bad = 1;
          ipiv[kk] = inv;
          pk[at(kk, kk)] = make_double2(r, 0.0);
        }
        if (lane > k && lane < b) pk[at(kk, c)] = cscale(pk[at(kk, c)], inv);
        __syncwarp();
        if (lane > k && lane < b && inv != 0.0) {
          const double2 rc = pk[at(kk, c)];
          for (int i = kk + 1; i <= c; ++i) {
            const double2 a = pk[at(kk, i)];
            double2& t = pk[at(i, c)];
            t.x -= a.x * rc.x + a.y * rc.y;
            t.y -= a.x * rc.y - a.y * rc.x;
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // panel: R(K0:E, c) = R_KK^-H A(K0:E, c) for c >= E; lane = row, forward substitution
    for (int c = E + warp; c < m; c += nw) {
      double2 a = lane < b ? pk[at(K0 + lane, c)] : make_double2(0.0, 0.0);
      for (int i = 0; i < b; ++i) {
        const double xi_r = __shfl_sync(0xffffffffu, a.x, i) * ipiv[K0 + i];
        const double xi_i = __shfl_sync(0xffffffffu, a.y, i) * ipiv[K0 + i];
        if (lane == i) a = make_double2(xi_r, xi_i);
        if (lane > i && lane < b) {
          const double2 r = pk[at(K0 + i, K0 + lane)];   // R(i, lane): a -= conj(r) x_i
          a.x -= r.x * xi_r + r.y * xi_i;
          a.y -= r.x * xi_i - r.y * xi_r;
        }
      }
      if (lane < b) pk[at(K0 + lane, c)] = a;
    }
    __syncthreads();
    // trailing update: A(i,j) -= sum_l conj(R(K0+l, i)) R(K0+l, j), E <= i <= j
    const int rem = m - E;
    const int npair = rem * (rem + 1) / 2;
    for (int q = warp; q < npair; q += nw) {
      // q -> (i, j) with column-major packed order inside the trailing triangle
      int j = int((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
      while ((j + 1) * (j + 2) / 2 <= q) ++j;
      while (j * (j + 1) / 2 > q) --j;
      const int i = q - j * (j + 1) / 2;
      const int gi = E + i, gj = E + j;
      double sr = 0, si = 0;
      if (lane < b) {
        const double2 x = pk[at(K0 + lane, gi)], y = pk[at(K0 + lane, gj)];
        sr = x.x * y.x + x.y * y.y;
        si = x.x * y.y - x.y * y.x;
      }
      for (int off = 16; off > 0; off >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, off);
        si += __shfl_xor_sync(0xffffffffu, si, off);
      }
      if (lane == 0) {
        pk[at(gi, gj)].x -= sr;
        pk[at(gi, gj)].y -= si;
      }
    }
    __syncthreads();
  }
  // inverse, diagonal blocks: warp K inverts R_KK in place (lane = row)
  for (int K = warp; K < nblk; K += nw) {
    const int K0 = 32 * K, b = min(32, m - K0);
    for (int c = 0; c < b; ++c) {
      const int gc = K0 + c;
      const double rcc = pk[at(gc, gc)].x;   // R(c, c); column c is still R here
      double sr = 0, si = 0;
      if (lane < c) {   // X(lane, c) = -sum_{k=lane}^{c-1} X(lane, k) R(k, c) / R(c, c)
        for (int k = lane; k < c; ++k) {
          const double2 x = pk[at(K0 + lane, K0 + k)], r = pk[at(K0 + k, gc)];
          sr += x.x * r.x - x.y * r.y;
          si += x.x * r.y + x.y * r.x;
        }
      }
      __syncwarp();
      if (lane < c) pk[at(K0 + lane, gc)] = make_double2(-sr / rcc, -si / rcc);
      if (lane == c) pk[at(gc, gc)] = make_double2(1.0 / rcc, 0.0);
      __syncwarp();
    }
  }
  __syncthreads();
  // block columns J = 1 .. nblk-1: T_KJ = sum_{k = row}^{J0-1} X(row, k) R(k, c), rows < J0
  for (int J = 1; J < nblk; ++J) {
    const int J0 = 32 * J, bJ = min(32, m - J0);
    for (int q = tid; q < J0 * bJ; q += nt) {
      const int r = q % J0, c = q / J0;
      double sr = 0, si = 0;
      for (int k = r; k < J0; ++k) {
        const double2 x = pk[at(r, k)], rr = pk[at(k, J0 + c)];
        sr += x.x * rr.x - x.y * rr.y;
        si += x.x * rr.y + x.y * rr.x;
      }
      tmp[c * J0 + r] = make_double2(sr, si);
    }
    __syncthreads();
    for (int q = tid; q < J0 * bJ; q += nt) {   // X(r, J0+c) = -sum_{l<=c} T(r, l) X(J0+l, J0+c)
      const int r = q % J0, c = q / J0;
      double sr = 0, si = 0;
      for (int l = 0; l <= c; ++l) {
        const double2 t = tmp[l * J0 + r], x = pk[at(J0 + l, J0 + c)];
        sr += t.x * x.x - t.y * x.y;
        si += t.x * x.y + t.y * x.x;
      }
      pk[at(r, J0 + c)] = make_double2(-sr, -si);
    }
    __syncthreads();
  }
  for (int j = warp; j < m; j += nw) {   // U = D X, lower triangle zero
    for (int i = lane; i < m; i += 32)
      M[size_t(j) * m + i] = i <= j ? cscale(pk[at(i, j)], dsc[i]) : make_double2(0.0, 0.0);
  }
  if (tid == 0) *status = s_bad;
}

// Block-wide sum of a (real, imaginary) pair; every thread gets the result.
__device__ double2 block_sum2(double a, double b, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, off);
    b += __shfl_xor_sync(0xffffffffu, b, off);
  }
  __syncthreads();   // red may still be read by a previous call
  if (lane == 0) { red[2 * warp] = a; red[2 * warp + 1] = b; }
  __syncthreads();
  double sa = 0, sb = 0;
  for (int w = 0; w < nw; ++w) { sa += red[2 * w]; sb += red[2 * w + 1]; }
  return make_double2(sa, sb);
}

// Householder reduction of a Hermitian A (n x n, upper triangle read) to the
// real tridiagonal T = Q^H A Q, in the storage convention of LAPACK zhetrd
// with UPLO = 'U' (the published zhetd2 algorithm): for i = n-2 .. 0 the
// reflector H(i) = I - tau_i v v^H with v(i) = 1 and v(0:i-1) left in
// A(0:i-1, i+1) annihilates A(0:i-1, i+1); d = diag(T), e = superdiagonal.
// One CTA; the packed upper triangle stays in shared memory for the whole
// reduction (n <= kMetricMax), replacing a launch pair per reflector.
__global__ void __launch_bounds__(512) hetrd_kernel(double2* __restrict__ A, int n, double* __restrict__ dout,
                                                    double* __restrict__ eout, double2* __restrict__ tauout) {
  extern __shared__ double2 pk[];
  double2* v = pk + size_t(n) * (n + 1) / 2;
  double2* y = v + n;
  __shared__ double red[64];
  __shared__ double2 s_tau, s_scale, s_alpha2;
  __shared__ double s_beta;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
  auto at = [](int i, int j) { return j * (j + 1) / 2 + i; };
  for (int q = tid; q < n * n; q += nt) {
    const int i = q % n, j = q / n;
    if (i <= j) {
      double2 a = A[q];
      if (i == j) a.y = 0.0;
      pk[at(i, j)] = a;
    }
  }
  __syncthreads();
  for (int i0 = n - 2; i0 >= 0; --i0) {
    const int L = i0 + 1, c = i0 + 1;
    // zlarfg on (alpha = A(i0, c), x = A(0:i0-1, c))
    double part = 0;
    for (int r = tid; r < i0; r += nt) {
      const double2 x = pk[at(r, c)];
      part += x.x * x.x + x.y * x.y;
    }
    const double xn2 = block_sum2(part, 0.0, red).x;
    if (tid == 0) {
      const double2 al = pk[at(i0, c)];
      if (xn2 == 0.0 && al.y == 0.0) {
        s_tau = make_double2(0.0, 0.0);
        s_beta = al.x;
        s_scale = make_double2(1.0, 0.0);
      } else {
        const double beta = -copysign(sqrt(al.x * al.x + al.y * al.y + xn2), al.x);
        s_tau = make_double2((beta - al.x) / beta, -al.y / beta);
        const double dr = al.x - beta, di = al.y, den = dr * dr + di * di;
        s_scale = make_double2(dr / den, -di / den);   // 1 / (alpha - beta)
        s_beta = beta;
      }
    }
    __syncthreads();
    const double2 tau = s_tau, sc = s_scale;
    for (int r = tid; r < L; r += nt) {
      double2 vr = make_double2(1.0, 0.0);
      if (r < i0) {
        const double2 x = pk[at(r, c)];
        vr = make_double2(x.x * sc.x - x.y * sc.y, x.x * sc.y + x.y * sc.x);
        pk[at(r, c)] = vr;
      }
      v[r] = vr;
    }
    __syncthreads();
    if (tau.x != 0.0 || tau.y != 0.0) {
      // y = tau A(0:i0, 0:i0) v: g = 2^k threads per row, partial sums over
      // s = p, p + g, ... combined by shuffles (deterministic order)
      {
        int lg = 0;
        while (lg < 5 && (2 << lg) * L <= nt) ++lg;
        const int g = 1 << lg, r = tid >> lg, p = tid & (g - 1);
        double sr = 0, si = 0;
        if (r < L) {
          const double2* cr = pk + r * (r + 1) / 2;   // column r: A(s, r), s <= r
          for (int s2 = p; s2 < L; s2 += g) {
            double2 a;
            if (r <= s2) a = pk[s2 * (s2 + 1) / 2 + r];
            else { a = cr[s2]; a.y = -a.y; }
            const double2 vv = v[s2];
            sr += a.x * vv.x - a.y * vv.y;
            si += a.x * vv.y + a.y * vv.x;
          }
        }
        for (int off = g >> 1; off > 0; off >>= 1) {
          sr += __shfl_xor_sync(0xffffffffu, sr, off);
          si += __shfl_xor_sync(0xffffffffu, si, off);
        }
        if (r < L && p == 0) y[r] = make_double2(tau.x * sr - tau.y * si, tau.x * si + tau.y * sr);
      }
      __syncthreads();
      // alpha2 = -tau (y^H v) / 2; w = y + alpha2 v
      double pr = 0, pi = 0;
      for (int r = tid; r < L; r += nt) {
        const double2 yy = y[r], vv = v[r];
        pr += yy.x * vv.x + yy.y * vv.y;   // conj(y) v
        pi += yy.x * vv.y - yy.y * vv.x;
      }
      const double2 dot = block_sum2(pr, pi, red);
      if (tid == 0) s_alpha2 = make_double2(-0.5 * (tau.x * dot.x - tau.y * dot.y), -0.5 * (tau.x * dot.y + tau.y * dot.x));
      __syncthreads();
      const double2 a2 = s_alpha2;
      for (int r = tid; r < L; r += nt) {
        const double2 vv = v[r];
        y[r].x += a2.x * vv.x - a2.y * vv.y;
        y[r].y += a2.x * vv.y + a2.y * vv.x;
      }
      __syncthreads();
      // A(0:i0, 0:i0) -= v w^H + w v^H (upper triangle), one warp per column
      for (int s2 = warp; s2 < L; s2 += nw) {
        const double2 ws = y[s2], vs = v[s2];
        double2* cs = pk + s2 * (s2 + 1) / 2;
        for (int r = lane; r <= s2; r += 32) {
          const double2 vr = v[r], wr = y[r];
          cs[r].x -= (vr.x * ws.x + vr.y * ws.y) + (wr.x * vs.x + wr.y * vs.y);
          cs[r].y -= (vr.y * ws.x - vr.x * ws.y) + (wr.y * vs.x - wr.x * vs.y);
        }
      }
      __syncthreads();
    }
    if (tid == 0) {
      eout[i0] = s_beta;
      dout[i0 + 1] = pk[at(i0 + 1, i0 + 1)].x;
      tauout[i0] = tau;
    }
  }
  __syncthreads();
  if (tid == 0) dout[0] = pk[at(0, 0)].x;
  for (int q = tid; q < n * n; q += nt) {   // reflector vectors back to A (strict upper triangle)
    const int i = q % n, j = q / n;
    if (i < j) A[q] = pk[at(i, j)];
  }
}

}  // namespace

void SmallEigen::reserve(Runtime& rt, int nmax) {
  if (nmax <= cap) return;
  cap = nmax;
  d.resize(nmax);
  e.resize(nmax);
  tau.resize(nmax);
  V.resize(size_t(nmax) * nmax);
  Z.resize(size_t(nmax) * nmax);
  scratch.resize(size_t(kEigThreads) * (5 * size_t(nmax) + (nmax + 7) / 8) + 16);
  info.resize(1);
  info.zero(rt.stream);
  int l1 = 0, l2 = 0;
  cusolver_check(cusolverDnZhetrd_bufferSize(rt.solver, CUBLAS_FILL_MODE_UPPER, nmax,
                                             reinterpret_cast<cuDoubleComplex*>(V.get()), nmax, d.get(), e.get(),
                                             reinterpret_cast<cuDoubleComplex*>(tau.get()), &l1),
                 "zhetrd buffer");
  cusolver_check(cusolverDnZpotrf_bufferSize(rt.solver, CUBLAS_FILL_MODE_UPPER, nmax,
                                             reinterpret_cast<cuDoubleComplex*>(V.get()), nmax, &l2),
                 "zpotrf buffer");
  work.resize(size_t(std::max({l1, l2, 1})));
}

// Hermitian eigenproblem of A (n x n, upper triangle used); the nev lowest
// eigenvectors overwrite A[:, :nev], eigenvalues go to w.
void SmallEigen::heev(Runtime& rt, double2* A, int n, int nev, double* w, int* status) {
  reserve(rt, n);
  cudaStream_t s = rt.stream;
  if (n <= kMetricMax) {   // whole reduction in one CTA
    const size_t tsm = (size_t(n) * (n + 1) / 2 + 2 * size_t(n)) * sizeof(double2);
    raise_smem_limit(hetrd_kernel, tsm);
    hetrd_kernel<<<1, 512, tsm, s>>>(A, n, d.get(), e.get(), tau.get());
    HALF_LAUNCH("Householder tridiagonalisation");
    rt.prof.launches += 1;
  } else {
    cusolver_check(cusolverDnZhetrd(rt.solver, CUBLAS_FILL_MODE_UPPER, n, reinterpret_cast<cuDoubleComplex*>(A), n,
                                    d.get(), e.get(), reinterpret_cast<cuDoubleComplex*>(tau.get()),
                                    reinterpret_cast<cuDoubleComplex*>(work.get()), int(work.size()), info.get()),
                   "zhetrd");
  }
  const int ne = std::min(n, nev + kExtraEig);
  size_t sm = (3 * size_t(n) + ne) * sizeof(double) + size_t(ne) * sizeof(int);
  if (sm > kSmemMax || size_t(n) * sizeof(double2) > kSmemMax)
    fail(kCapacity, "subspace eigenproblem too large for the tridiagonal solver: n=" + std::to_string(n));
  // inverse-iteration slots: in shared memory when at least 32 fit, else global
  sm = (sm + 15) & ~size_t(15);
  const size_t per_slot = 5 * size_t(n) * sizeof(double) + size_t(n);
  int batch = int(std::min<size_t>((kSmemMax - sm) / per_slot, size_t(kEigThreads)));
  batch = std::min(batch, (nev + 31) / 32 * 32) / 32 * 32;
  double* gs = nullptr;
  if (batch >= 32) {
    sm += size_t(batch) * per_slot;
  } else {
    batch = kEigThreads;
    gs = scratch.get();
  }
  raise_smem_limit(tridiag_eig_kernel, sm);
  tridiag_eig_kernel<<<1, kEigThreads, sm, s>>>(d.get(), e.get(), n, nev, w, Z.get(), gs, batch, status);
  HALF_LAUNCH("tridiagonal eigensolver");
  const int warps = n <= 384 ? 4 : 1;   // one n-vector of shared memory per warp
  raise_smem_limit(back_transform_kernel, size_t(warps) * n * sizeof(double2));
  back_transform_kernel<<<ceil_div(nev, warps), 32 * warps, size_t(warps) * n * sizeof(double2), s>>>(
      A, tau.get(), Z.get(), n, nev, V.get());
  HALF_LAUNCH("back transformation");
  HALF_CUDA(cudaMemcpyAsync(A, V.get(), size_t(n) * nev * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  rt.prof.launches += 2;
}

// Generalized problem A y = lambda B y (itype 1, upper triangles used), B HPD.
// The nev lowest eigenvectors (Y^H B Y = I) overwrite A[:, :nev].
void SmallEigen::hegv(Runtime& rt, double2* A, double2* B, int n, int nev, double* w, int* status, int* chol_status) {
  reserve(rt, n);
  cudaStream_t s = rt.stream;
  if (n <= kMetricMax) {
    // B -> X = D R^-1 with X^H B X = I (metric_cholesky_kernel), C = X^H A X,
    // C V = V Lambda, Y = X V: the same pencil reduction as zhegvd's
    // Cholesky / two triangular solves, with the factor inverted in shared
    // memory and the products done by three small GEMMs
    metric_normalize(rt, B, n, chol_status);
    hermitian_fill_kernel<<<ceil_div((long long)n * n, 256), 256, 0, s>>>(A, n);
    rt.prof.launches += 1;
    const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
    gemm(rt, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, one, A, n, B, n, zero, V.get(), n);
    gemm(rt, CUBLAS_OP_C, CUBLAS_OP_N, n, n, n, one, B, n, V.get(), n, zero, A, n);
    heev(rt, A, n, nev, w, status);
    gemm(rt, CUBLAS_OP_N, CUBLAS_OP_N, n, nev, n, one, B, n, A, n, zero, V.get(), n);
    HALF_CUDA(cudaMemcpyAsync(A, V.get(), size_t(n) * nev * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    return;
  }
  auto* Bc = reinterpret_cast<cuDoubleComplex*>(B);
  auto* Ac = reinterpret_cast<cuDoubleComplex*>(A);
  cusolver_check(cusolverDnZpotrf(rt.solver, CUBLAS_FILL_MODE_UPPER, n, Bc, n,
                                  reinterpret_cast<cuDoubleComplex*>(work.get()), int(work.size()), chol_status),
                 "zpotrf");
  hermitian_fill_kernel<<<ceil_div((long long)n * n, 256), 256, 0, s>>>(A, n);
  rt.prof.launches += 1;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  cublas_check(cublasZtrsm(rt.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, n, n,
                           &one, Bc, n, Ac, n),
               "ztrsm");
  cublas_check(cublasZtrsm(rt.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, n, n,
                           &one, Bc, n, Ac, n),
               "ztrsm");
  heev(rt, A, n, nev, w, status);
  cublas_check(cublasZtrsm(rt.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, n, nev,
                           &one, Bc, n, Ac, n),
               "ztrsm");
}

// U with (P U)^H S (P U) = I from M = P^H S P, overwriting M (see
// metric_cholesky_kernel); false when m is beyond the shared-memory kernel.
bool SmallEigen::metric_normalize(Runtime& rt, double2* M, int m, int* status) {
  if (m > kMetricMax) return false;
  if (m <= kBlockedMax) {
    const size_t bsm = size_t(m) * (m + 1) / 2 * sizeof(double2) + 2 * size_t(m) * sizeof(double) +
                       size_t(std::max(m - 32, 1)) * 32 * sizeof(double2);
    raise_smem_limit(metric_cholesky_blocked_kernel, bsm);
    metric_cholesky_blocked_kernel<<<1, 1024, bsm, rt.stream>>>(M, m, status);
    HALF_LAUNCH("metric Cholesky (blocked)");
    rt.prof.launches += 1;
    return true;
  }
  const size_t sm = (size_t(m) * (m + 1) / 2 + m) * sizeof(double2) + size_t(m) * sizeof(double);
  raise_smem_limit(metric_cholesky_kernel, sm);
  metric_cholesky_kernel<<<1, 512, sm, rt.stream>>>(M, m, status);
  HALF_LAUNCH("metric Cholesky");
  rt.prof.launches += 1;
  return true;
}

}  // namespace hb
