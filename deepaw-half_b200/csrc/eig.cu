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
//   tridiag_values_kernel  eigenvalues of the real symmetric tridiagonal T by
//                          multisection on Sturm counts (one warp per
//                          eigenvalue, CTAs across the GPU);
//   tridiag_vectors_kernel eigenvectors by inverse iteration on the pivoted
//                          tridiagonal LU (one thread per eigenvector);
//                          eigenvalues closer than 1e-7 ||T|| form clusters
//                          whose members are iterated in order and
//                          Gram-Schmidt orthogonalised against each other (the
//                          strategy of LAPACK's dstebz/dstein);
//   back_transform_kernel  V = Q Z with Q = H(n-1)...H(1) from zhetrd's
//                          reflectors staged in shared memory, one warp per
//                          eigenvector.
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
// per-thread scratch of n elements at stride st (the slots of a group of
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

// Padded Gershgorin interval of T and the norm max_i (|d_i| + |e_{i-1}| + |e_i|);
// both tridiagonal kernels evaluate it with this one routine, so they agree bit for bit.
__device__ void gershgorin(const double* d, const double* e, int n, double& lo, double& hi, double& nrm) {
  double gl = d[0], gu = d[0];
  nrm = 0;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    gl = fmin(gl, d[i] - r);
    gu = fmax(gu, d[i] + r);
    nrm = fmax(nrm, fabs(d[i]) + r);
  }
  const double pad = 2.0 * DBL_EPSILON * fmax(fabs(gl), fabs(gu)) * n + 1e-300;
  lo = gl - pad;
  hi = gu + pad;
  nrm = fmax(nrm, DBL_MIN);
}

constexpr int kValueWarps = 8;       // eigenvalues per CTA of the value kernel, one warp each
constexpr int kVectorThreads = 32;   // eigenvectors per CTA of the vector kernel, one thread each

// Eigenvalues 0..ne-1 of T (ascending) by multisection: the 32 lanes of a warp
// count at 32 interior points of its eigenvalue's bracket per round, which
// shrinks to the pair of neighbouring points whose counts straddle the index
// (33-fold per round).  Brackets end at 2 eps |lambda| + eps ||T|| (absolute
// accuracy eps ||T||, as bisection guarantees).  Also clears *status for the
// vector kernel that follows on the stream.
__global__ void __launch_bounds__(32 * kValueWarps) tridiag_values_kernel(const double* __restrict__ d_in,
                                                                          const double* __restrict__ e_in, int n,
                                                                          int ne, double* __restrict__ lam,
                                                                          int* __restrict__ status) {
  extern __shared__ double sm[];
  double* d = sm;
  double* e = d + n;
  double* e2 = e + n;
  __shared__ double s_gl, s_gu, s_norm;
  if (blockIdx.x == 0 && threadIdx.x == 0) *status = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = d_in[i];
    const double ei = i < n - 1 ? e_in[i] : 0.0;
    e[i] = ei;
    e2[i] = ei * ei;
  }
  __syncthreads();
  if (threadIdx.x == 0) gershgorin(d, e, n, s_gl, s_gu, s_norm);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * kValueWarps + (threadIdx.x >> 5);
  if (k >= ne) return;   // whole warps; no barrier follows
  const double tnorm = s_norm;
  double lo = s_gl, hi = s_gu;   // warp-uniform throughout
  for (int round = 0; round < 200; ++round) {
    if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + DBL_EPSILON * tnorm) break;
    const double x = lo + (hi - lo) * double(lane + 1) / 33.0;
    const unsigned b = __ballot_sync(0xffffffffu, sturm_count(d, e2, n, x) > k);   // lambda_k < x
    const int first = b ? __ffs(b) - 1 : 32;                                          // first point above
    const double xlo = __shfl_sync(0xffffffffu, x, first > 0 ? first - 1 : 0);
    const double xhi = __shfl_sync(0xffffffffu, x, first < 32 ? first : 31);
    const double nlo = first > 0 ? xlo : lo, nhi = first < 32 ? xhi : hi;
    if (!(nlo > lo || nhi < hi)) break;   // no progress left in floating point
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) lam[k] = 0.5 * (lo + hi);
}

// Eigenvectors of lam[0..nev) by inverse iteration on the pivoted LU of
// T - lambda I, one thread per eigenvector.  Eigenvalues (up to ne) closer
// than 1e-7 ||T|| form clusters; the thread of a cluster's first member
// computes the whole cluster in order, Gram-Schmidt orthogonalising each
// member against the earlier ones (the strategy of LAPACK's dstein with a
// tighter cluster threshold: dstein's 1e-3 ||T|| would serialise the dense
// Ritz spectra met here).  Outside a cluster inverse iteration alone keeps
// |<z_i, z_j>| <= eps ||T|| / gap <~ 1e-9.  Scratch: five n-vectors and the
// pivot flags per thread, interleaved by thread (a warp touches consecutive
// words), in shared memory after the tables when gscratch is null, else in
// global memory with one slot per thread of the grid.
__global__ void __launch_bounds__(kVectorThreads) tridiag_vectors_kernel(
    const double* __restrict__ d_in, const double* __restrict__ e_in, int n, int nev, int ne,
    const double* __restrict__ lam_g, double* __restrict__ w, double* __restrict__ Z, double* __restrict__ gscratch,
    int* __restrict__ status) {
  extern __shared__ double sm[];
  double* d = sm;
  double* e = d + n;
  double* lam = e + n;
  int* cl_first = reinterpret_cast<int*>(lam + ne);
  __shared__ double s_gl, s_gu, s_norm;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = d_in[i];
    e[i] = i < n - 1 ? e_in[i] : 0.0;
  }
  for (int i = threadIdx.x; i < ne; i += blockDim.x) lam[i] = lam_g[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    gershgorin(d, e, n, s_gl, s_gu, s_norm);
    const double ortol = 1.0e-7 * s_norm;
    int first = 0;
    for (int k = 0; k < ne; ++k) {
      if (k > 0 && lam[k] - lam[k - 1] > ortol) first = k;
      cl_first[k] = first;
    }
  }
  __syncthreads();
  const double tnorm = s_norm;
  const int k0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (k0 < nev) w[k0] = lam[k0];
  if (k0 >= nev || cl_first[k0] != k0) return;
  const double tiny = DBL_EPSILON * tnorm;
  double* ai;
  unsigned char* piv;
  int st;
  if (gscratch) {
    st = gridDim.x * blockDim.x;
    ai = gscratch + k0;
    piv = reinterpret_cast<unsigned char*>(gscratch + 5 * size_t(n) * st) + k0;
  } else {
    size_t off = (2 * size_t(n) + ne) * sizeof(double) + size_t(ne) * sizeof(int);
    off = (off + 15) & ~size_t(15);
    double* sbase = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(sm) + off);
    st = blockDim.x;
    ai = sbase + threadIdx.x;
    piv = reinterpret_cast<unsigned char*>(sbase + 5 * size_t(n) * st) + threadIdx.x;
  }
  double* b1 = ai + size_t(n) * st;
  double* b2 = b1 + size_t(n) * st;
  double* l = b2 + size_t(n) * st;
  double* x = l + size_t(n) * st;
  int k1 = k0;
  while (k1 + 1 < ne && cl_first[k1 + 1] == k0) ++k1;
  double prev = -HUGE_VAL;
  for (int k = k0; k <= k1; ++k) {
    double lk = lam[k];
    // separate numerically equal eigenvalues of a cluster (dstein)
    const double sep = 10.0 * DBL_EPSILON * fmax(fabs(lk), tnorm * 1e-3);
    if (k > k0 && lk - prev < sep) lk = prev + sep;
    prev = lk;
    tri_factor(d, e, n, lk, tiny, ai, b1, b2, l, piv, st);
    unsigned s = 0x9E3779B9u * (k + 1);
    for (int i = 0; i < n; ++i) {   // deterministic pseudo-random start vector
      s = s * 1664525u + 1013904223u;
      x[i * st] = 1.0 + 0.5 * (double(s >> 8) / 16777216.0 - 0.5);
    }
    // With an eigenvalue accurate to rounding each solve amplifies the wanted
    // direction by ~gap / (eps ||T||): two solves for an isolated eigenvalue,
    // three (each followed by Gram-Schmidt against the earlier members) inside
    // a cluster.
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
      if (!(nrm > 0) || !isfinite(nrm)) {
        atomicExch(status, 1);
        break;
      }
      const double inv = 1.0 / nrm;
      for (int i = 0; i < n; ++i) x[i * st] *= inv;
    }
    // sign convention: largest component positive
    double big = 0;
    for (int i = 0; i < n; ++i)
      if (fabs(x[i * st]) > fabs(big)) big = x[i * st];
    const double sg = big < 0 ? -1.0 : 1.0;
    double* z = Z + (size_t)k * n;
    for (int i = 0; i < n; ++i) z[i] = sg * x[i * st];
  }
}

constexpr int kBackWarps = 8;   // eigenvectors per CTA of the back-transformation, one warp each

// V[:, j] = H(1) H(2) ... applied as Q z_j with Q = H(n-1) ... H(1)
// (LAPACK zhetrd, UPLO = 'U': v(i) = 1, v(1:i-1) = A(1:i-1, i+1), tau(i)).
// The CTA's warps share the reflectors, staged in shared memory `chunk` at a
// time (v with its unit entry and zeros below, so the inner loops have no
// branch); each warp applies them to its eigenvector in order.
__global__ void __launch_bounds__(32 * kBackWarps) back_transform_kernel(const double2* __restrict__ A,
                                                                         const double2* __restrict__ tau,
                                                                         const double* __restrict__ Z, int n, int nev,
                                                                         int chunk, double2* __restrict__ V) {
  extern __shared__ double2 sv[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * kBackWarps + warp;
  const bool active = j < nev;
  double2* x = sv + (size_t)warp * n;
  double2* vs = sv + (size_t)kBackWarps * n;   // chunk x n
  double2* ts = vs + (size_t)chunk * n;        // chunk
  if (active)
    for (int r = lane; r < n; r += 32) x[r] = make_double2(Z[(size_t)j * n + r], 0.0);
  for (int c0 = 0; c0 <= n - 2; c0 += chunk) {
    const int cnt = min(chunk, n - 1 - c0);
    __syncthreads();   // the previous chunk is consumed
    for (int t = threadIdx.x; t < cnt * n; t += blockDim.x) {
      const int q = t / n, row = t - q * n, i0 = c0 + q;
      vs[t] = row < i0 ? A[(size_t)(i0 + 1) * n + row] : make_double2(row == i0 ? 1.0 : 0.0, 0.0);
    }
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) ts[t] = tau[c0 + t];
    __syncthreads();
    if (!active) continue;
    for (int q = 0; q < cnt; ++q) {
      const int i0 = c0 + q;
      const double2* v = vs + (size_t)q * n;
      const double2 t = ts[q];
      double wr = 0, wi = 0;
      for (int r = lane; r <= i0; r += 32) {
        const double2 vr = v[r], xr = x[r];
        wr += vr.x * xr.x + vr.y * xr.y;   // conj(v) . x
        wi += vr.x * xr.y - vr.y * xr.x;
      }
      for (int off = 16; off > 0; off >>= 1) {
        wr += __shfl_xor_sync(0xffffffffu, wr, off);
        wi += __shfl_xor_sync(0xffffffffu, wi, off);
      }
      // x -= tau * w * v
      const double cr = t.x * wr - t.y * wi, ci = t.x * wi + t.y * wr;
      for (int r = lane; r <= i0; r += 32) {
        const double2 vr = v[r];
        x[r].x -= cr * vr.x - ci * vr.y;
        x[r].y -= cr * vr.y + ci * vr.x;
      }
      __syncwarp();
    }
  }
  if (active)
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
// the metric eigenvalues for nearly dependent directions: a pivot at or below
// 1e-14 (of the unit scaled diagonal) gives R(k,k) = 1e-7 and a zero row, so
// the direction stays in the span without being eliminated from later
// columns.
//
// One CTA, the packed upper triangle in shared memory (m <= kMetricMax), and
// ONE right-looking sweep that builds R^-1 together with R.  With
// T(i,j) = sum_{l<j} X(i,l) R(l,j) for i < j (X = R^-1), step k is
//   W(i,j) -= conj(W(k,i)) W(k,j) / p_k    k < i <= j   (trailing Schur complement)
//   T(i,j) -= T(i,k) W(k,j) / p_k          i < k < j
//   T(k,j)  = W(k,j) / p_k                 j > k         (row k becomes X(k,k) R(k,j))
// with p_k = W(k,k): a rank-1 update of every stored column right of k.  The
// two index ranges occupy disjoint slots of one packed triangle (rows <= k
// hold T, rows > k hold W), and at the end X(i,j) = -T(i,j) / R(j,j),
// X(j,j) = 1 / R(j,j).  Two CTA barriers per step; the update's row factors
// are held in registers (lane-owned rows), its column factors broadcast from
// shared memory.  *status = 1 if a pivot was not finite.
constexpr int kFactorThreads = 1024;
constexpr int kFactorRows = (kMetricMax + 31) / 32;   // lane-owned rows per thread

__global__ void __launch_bounds__(kFactorThreads) metric_factor_kernel(double2* __restrict__ M, int m,
                                                                      int* __restrict__ status) {
  extern __shared__ double2 pk[];                  // packed upper triangle, (i, j) at j (j + 1) / 2 + i
  double2* av = pk + size_t(m) * (m + 1) / 2;      // row factors of the step (T(i,k) or conj W(k,i))
  double2* cv = av + m;                            // column factors W(k,j) / p_k
  double* dsc = reinterpret_cast<double*>(cv + m);   // D
  double* ir = dsc + m;                              // 1 / R(k,k)
  __shared__ int s_bad;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
  if (tid == 0) s_bad = 0;
  for (int j = tid; j < m; j += nt) dsc[j] = 1.0 / sqrt(fmax(M[size_t(j) * m + j].x, DBL_MIN));
  __syncthreads();
  for (int j = warp; j < m; j += nw) {
    const double dj = dsc[j];
    double2* col = pk + size_t(j) * (j + 1) / 2;
    for (int i = lane; i <= j; i += 32) {
      double2 v = M[size_t(j) * m + i];
      if (i == j) v.y = 0.0;
      col[i] = cscale(v, dsc[i] * dj);
    }
  }
  __syncthreads();
  for (int k = 0; k < m; ++k) {
    // phase A: pivot (every thread, same value) and the step's factor vectors
    const double p = pk[size_t(k) * (k + 1) / 2 + k].x;
    const bool dep = !(p > 1.0e-14);   // also true for NaN
    const double invp = dep ? 0.0 : 1.0 / p;
    if (tid == 0) {
      if (!isfinite(p)) s_bad = 1;
      ir[k] = dep ? 1.0e7 : 1.0 / sqrt(p);
    }
    const double2* colk = pk + size_t(k) * (k + 1) / 2;
    for (int i = tid; i < m; i += nt) {
      if (i < k) {
        av[i] = colk[i];                                     // T(i, k)
      } else if (i > k) {
        const double2 w = pk[size_t(i) * (i + 1) / 2 + k];   // W(k, i)
        av[i] = make_double2(w.x, -w.y);
        cv[i] = cscale(w, invp);
      }
    }
    __syncthreads();
    // phase B: columns j > k, one warp per column, lane-owned rows i = lane + 32 t
    double2 a[kFactorRows];
#pragma unroll
    for (int t = 0; t < kFactorRows; ++t) {
      const int i = lane + 32 * t;
      a[t] = i < m && i != k ? av[i] : make_double2(0.0, 0.0);
    }
    for (int j = k + 1 + warp; j < m; j += nw) {
      const double2 c = cv[j];
      double2* col = pk + size_t(j) * (j + 1) / 2;
#pragma unroll
      for (int t = 0; t < kFactorRows; ++t) {
        const int i = lane + 32 * t;
        if (i <= j) {
          if (i == k) {
            col[i] = c;
          } else if (!dep) {
            double2 x = col[i];
            x.x -= a[t].x * c.x - a[t].y * c.y;
            x.y -= a[t].x * c.y + a[t].y * c.x;
            col[i] = x;
          }
        }
      }
    }
    __syncthreads();
  }
  // U = D X with X(i,j) = -T(i,j) / R(j,j), X(j,j) = 1 / R(j,j); lower triangle zero
  for (int j = warp; j < m; j += nw) {
    const double2* col = pk + size_t(j) * (j + 1) / 2;
    const double irj = ir[j];
    for (int i = lane; i < m; i += 32) {
      double2 u = make_double2(0.0, 0.0);
      if (i < j) u = cscale(col[i], -irj * dsc[i]);
      else if (i == j) u = make_double2(irj * dsc[i], 0.0);
      M[size_t(j) * m + i] = u;
    }
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

__global__ void real_to_complex_block_kernel(const double* __restrict__ z, long long count, double2* __restrict__ out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < count) out[t] = make_double2(z[t], 0.0);
}

// Large orders (the dense solves): T stays in global memory, read through
// L1 with all lanes of a warp at the same index.  e2[i] = e[i]^2 and the
// Gershgorin bounds (lo, hi, norm) are formed once by the first kernel.
__global__ void tridiag_bounds_kernel(const double* __restrict__ d, const double* __restrict__ e, int n,
                                      double* __restrict__ e2, double* __restrict__ bounds) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) e2[i] = i < n - 1 ? e[i] * e[i] : 0.0;
  if (threadIdx.x == 0) gershgorin(d, e, n, bounds[0], bounds[1], bounds[2]);
}

// Eigenvalues k0 .. k0 + ne - 1 of T (ascending), one warp each, by the same
// multisection as tridiag_values_kernel.
__global__ void __launch_bounds__(32 * kValueWarps) tridiag_values_global_kernel(const double* __restrict__ d,
                                                                                 const double* __restrict__ e2, int n,
                                                                                 int k0, int ne,
                                                                                 const double* __restrict__ bounds,
                                                                                 double* __restrict__ lam) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * kValueWarps + (threadIdx.x >> 5);
  if (j >= ne) return;
  const int k = k0 + j;
  const double tnorm = bounds[2];
  double lo = bounds[0], hi = bounds[1];
  for (int round = 0; round < 200; ++round) {
    if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + DBL_EPSILON * tnorm) break;
    const double x = lo + (hi - lo) * double(lane + 1) / 33.0;
    const unsigned b = __ballot_sync(0xffffffffu, sturm_count(d, e2, n, x) > k);
    const int first = b ? __ffs(b) - 1 : 32;
    const double xlo = __shfl_sync(0xffffffffu, x, first > 0 ? first - 1 : 0);
    const double xhi = __shfl_sync(0xffffffffu, x, first < 32 ? first : 31);
    const double nlo = first > 0 ? xlo : lo, nhi = first < 32 ? xhi : hi;
    if (!(nlo > lo || nhi < hi)) break;
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) lam[j] = 0.5 * (lo + hi);
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
  // global inverse-iteration scratch: one slot per thread of the vector kernel's grid
  const size_t slots = size_t(ceil_div(nmax, kVectorThreads)) * kVectorThreads;
  scratch.resize(5 * size_t(nmax) * slots + (size_t(nmax) * slots + 7) / 8 + 16);
  lam.resize(nmax);
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
  int l3 = 0;
  cusolver_check(cusolverDnZunmtr_bufferSize(rt.solver, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, nmax,
                                             nmax, reinterpret_cast<cuDoubleComplex*>(V.get()), nmax,
                                             reinterpret_cast<cuDoubleComplex*>(tau.get()),
                                             reinterpret_cast<cuDoubleComplex*>(V.get()), nmax, &l3),
                 "zunmtr buffer");
  work.resize(size_t(std::max({l1, l2, l3, 1})));
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
  // Eigenvalues up to ne = nev + kExtraEig are located so that a cluster
  // straddling the last wanted index is computed (and orthogonalised) whole;
  // only the first nev pairs are returned.
  const int ne = std::min(n, nev + kExtraEig);
  const size_t vsm = 3 * size_t(n) * sizeof(double);
  raise_smem_limit(tridiag_values_kernel, vsm);
  tridiag_values_kernel<<<ceil_div(ne, kValueWarps), 32 * kValueWarps, vsm, s>>>(d.get(), e.get(), n, ne, lam.get(),
                                                                                  status);
  HALF_LAUNCH("tridiagonal eigenvalues");
  size_t tsm = (2 * size_t(n) + ne) * sizeof(double) + size_t(ne) * sizeof(int);
  if (tsm > kSmemMax) fail(kCapacity, "subspace eigenproblem too large for the tridiagonal solver: n=" + std::to_string(n));
  tsm = (tsm + 15) & ~size_t(15);
  const size_t slots_sm = size_t(kVectorThreads) * (5 * size_t(n) * sizeof(double) + size_t(n));
  double* gs = nullptr;
  if (tsm + slots_sm <= kSmemMax) tsm += slots_sm;
  else gs = scratch.get();
  raise_smem_limit(tridiag_vectors_kernel, tsm);
  tridiag_vectors_kernel<<<ceil_div(nev, kVectorThreads), kVectorThreads, tsm, s>>>(d.get(), e.get(), n, nev, ne,
                                                                                     lam.get(), w, Z.get(), gs, status);
  HALF_LAUNCH("tridiagonal eigenvectors");
  if (n > kMetricMax) {
    // large orders: cuSOLVER's blocked back-transformation (zunmtr, Q Z with
    // zhetrd's reflectors) on the complex copy of Z
    real_to_complex_block_kernel<<<ceil_div((long long)n * nev, 256), 256, 0, s>>>(Z.get(), (long long)n * nev,
                                                                                   V.get());
    HALF_LAUNCH("tridiagonal eigenvectors to complex");
    cusolver_check(cusolverDnZunmtr(rt.solver, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, n, nev,
                                    reinterpret_cast<cuDoubleComplex*>(A), n,
                                    reinterpret_cast<cuDoubleComplex*>(tau.get()),
                                    reinterpret_cast<cuDoubleComplex*>(V.get()), n,
                                    reinterpret_cast<cuDoubleComplex*>(work.get()), int(work.size()), info.get()),
                   "zunmtr");
    HALF_CUDA(cudaMemcpyAsync(A, V.get(), size_t(n) * nev * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    rt.prof.launches += 3;
    return;
  }
  // back-transformation: the reflectors in chunks that fit next to the warps' vectors
  const size_t vec_bytes = size_t(kBackWarps) * n * sizeof(double2);
  if (vec_bytes + (size_t(n) + 1) * sizeof(double2) > kSmemMax)
    fail(kCapacity, "subspace eigenproblem too large for the back-transformation: n=" + std::to_string(n));
  const int chunk = int(std::max<size_t>(1, std::min<size_t>(size_t(std::max(n - 1, 1)),
                                                             (kSmemMax - vec_bytes) / ((size_t(n) + 1) * sizeof(double2)))));
  const size_t bsm = vec_bytes + size_t(chunk) * (n + 1) * sizeof(double2);
  raise_smem_limit(back_transform_kernel, bsm);
  back_transform_kernel<<<ceil_div(nev, kBackWarps), 32 * kBackWarps, bsm, s>>>(A, tau.get(), Z.get(), n, nev, chunk,
                                                                                 V.get());
  HALF_LAUNCH("back transformation");
  HALF_CUDA(cudaMemcpyAsync(A, V.get(), size_t(n) * nev * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  rt.prof.launches += 3;
}

// Generalized problem A y = lambda B y (itype 1, upper triangles used), B HPD.
// The nev lowest eigenvectors (Y^H B Y = I) overwrite A[:, :nev].
void SmallEigen::hegv(Runtime& rt, double2* A, double2* B, int n, int nev, double* w, int* status, int* chol_status) {
  reserve(rt, n);
  cudaStream_t s = rt.stream;
  if (n <= kMetricMax) {
    // B -> X = D R^-1 with X^H B X = I (metric_factor_kernel), C = X^H A X,
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
// metric_factor_kernel); false when m is beyond the shared-memory kernel.
bool SmallEigen::metric_normalize(Runtime& rt, double2* M, int m, int* status) {
  if (m > kMetricMax) return false;
  const size_t sm = (size_t(m) * (m + 1) / 2 + 2 * size_t(m)) * sizeof(double2) + 2 * size_t(m) * sizeof(double);
  raise_smem_limit(metric_factor_kernel, sm);
  metric_factor_kernel<<<1, kFactorThreads, sm, rt.stream>>>(M, m, status);
  HALF_LAUNCH("metric factor");
  rt.prof.launches += 1;
  return true;
}

void hermitian_eigenvalues_large(Runtime& rt, double2* A, long long n, const std::vector<int>& k0s,
                                 const std::vector<int>& counts, double* lam) {
  if (n > INT32_MAX / 2) fail(kUnavailable, "dense order beyond the tridiagonalisation's range");
  cudaStream_t s = rt.stream;
  const int ni = int(n);
  DeviceBuffer<double> d(ni), e(ni), e2(ni), bounds(3);
  DeviceBuffer<double2> tau(ni);
  DeviceBuffer<int> info(1);
  int lwork = 0;
  cusolver_check(cusolverDnZhetrd_bufferSize(rt.solver, CUBLAS_FILL_MODE_UPPER, ni,
                                             reinterpret_cast<cuDoubleComplex*>(A), ni, d.get(), e.get(),
                                             reinterpret_cast<cuDoubleComplex*>(tau.get()), &lwork),
                 "zhetrd buffer (large)");
  DeviceBuffer<double2> work(size_t(std::max(lwork, 1)));
  cusolver_check(cusolverDnZhetrd(rt.solver, CUBLAS_FILL_MODE_UPPER, ni, reinterpret_cast<cuDoubleComplex*>(A), ni,
                                  d.get(), e.get(), reinterpret_cast<cuDoubleComplex*>(tau.get()),
                                  reinterpret_cast<cuDoubleComplex*>(work.get()), lwork, info.get()),
                 "zhetrd (large)");
  int hinfo = 0;
  HALF_CUDA(cudaMemcpyAsync(&hinfo, info.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  HALF_CUDA(cudaStreamSynchronize(s));
  if (hinfo != 0) fail(kInternal, "Householder tridiagonalisation failed");
  tridiag_bounds_kernel<<<1, 1024, 0, s>>>(d.get(), e.get(), ni, e2.get(), bounds.get());
  HALF_LAUNCH("tridiagonal bounds");
  int off = 0;
  for (size_t r = 0; r < k0s.size(); ++r) {
    const int k0 = k0s[r], ne = counts[r];
    if (k0 < 0 || ne < 0 || k0 + ne > ni) fail(kInvalidArgument, "eigenvalue index range outside the matrix");
    if (ne == 0) continue;
    tridiag_values_global_kernel<<<ceil_div(ne, kValueWarps), 32 * kValueWarps, 0, s>>>(d.get(), e2.get(), ni, k0, ne,
                                                                                       bounds.get(), lam + off);
    HALF_LAUNCH("tridiagonal eigenvalues (large)");
    off += ne;
  }
  HALF_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hb
