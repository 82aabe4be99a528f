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
// per-thread scratch of length n.
__device__ void tri_factor(const double* d, const double* e, int n, double lam, double tiny, double* ai, double* b1,
                           double* b2, double* l, unsigned char* piv) {
  double diag = d[0] - lam, sup = n > 1 ? e[0] : 0.0;
  for (int i = 0; i < n - 1; ++i) {
    const double sub = e[i];
    const double nd = d[i + 1] - lam, ns = (i + 1 < n - 1) ? e[i + 1] : 0.0;
    if (fabs(diag) >= fabs(sub)) {
      if (fabs(diag) < tiny) diag = diag < 0 ? -tiny : tiny;
      const double r = 1.0 / diag, m = sub * r;
      ai[i] = r; b1[i] = sup; b2[i] = 0.0; l[i] = m; piv[i] = 0;
      diag = nd - m * sup;
      sup = ns;
    } else {
      const double r = 1.0 / sub, m = diag * r;
      ai[i] = r; b1[i] = nd; b2[i] = ns; l[i] = m; piv[i] = 1;
      diag = sup - m * nd;
      sup = -m * ns;
    }
  }
  if (fabs(diag) < tiny) diag = diag < 0 ? -tiny : tiny;
  ai[n - 1] = 1.0 / diag;
  b1[n - 1] = 0.0;
  b2[n - 1] = 0.0;
}

__device__ void tri_solve(int n, const double* ai, const double* b1, const double* b2, const double* l,
                          const unsigned char* piv, double* x) {
  for (int i = 0; i < n - 1; ++i) {
    if (piv[i]) { double t = x[i]; x[i] = x[i + 1]; x[i + 1] = t - l[i] * x[i]; }
    else x[i + 1] -= l[i] * x[i];
  }
  x[n - 1] *= ai[n - 1];
  if (n > 1) x[n - 2] = (x[n - 2] - b1[n - 2] * x[n - 1]) * ai[n - 2];
  for (int i = n - 3; i >= 0; --i) x[i] = (x[i] - b1[i] * x[i + 1] - b2[i] * x[i + 2]) * ai[i];
}

// One CTA: eigenvalues 0..nev-1 of T (ascending) and their eigenvectors Z (n x nev).
__global__ void __launch_bounds__(kEigThreads) tridiag_eig_kernel(const double* __restrict__ d_in,
                                                                  const double* __restrict__ e_in, int n, int nev,
                                                                  double* __restrict__ w, double* __restrict__ Z,
                                                                  double* __restrict__ scratch, int* __restrict__ status) {
  extern __shared__ double sm[];
  double* d = sm;
  double* e = d + n;
  double* e2 = e + n;
  double* lam = e2 + n;
  int* cl_first = reinterpret_cast<int*>(lam + nev);
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
    while (g < 32 && 2 * g * nev <= int(blockDim.x)) g *= 2;
    const int lane = threadIdx.x & 31, gl = lane & (g - 1), gbase = lane & ~(g - 1);
    const unsigned gmask = g == 32 ? 0xffffffffu : (((1u << g) - 1u) << gbase);
    const int groups = blockDim.x / g;
    const int slots = (nev + groups - 1) / groups;   // same trip count on every thread
    for (int sidx = 0; sidx < slots; ++sidx) {
      const int k = sidx * groups + int(threadIdx.x) / g;
      const bool active = k < nev;
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
    for (int k = 0; k < nev; ++k) {
      if (k > 0 && lam[k] - lam[k - 1] > ortol) first = k;
      cl_first[k] = first;
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nev; k += blockDim.x) w[k] = lam[k];
  // inverse iteration: the thread owning a cluster's first member computes the whole cluster
  const double tiny = DBL_EPSILON * tnorm;
  double* ai = scratch + (size_t)threadIdx.x * 5 * n;
  double* b1 = ai + n;
  double* b2 = b1 + n;
  double* l = b2 + n;
  unsigned char* piv = reinterpret_cast<unsigned char*>(l + n);
  for (int k0 = threadIdx.x; k0 < nev; k0 += blockDim.x) {
    if (cl_first[k0] != k0) continue;
    int k1 = k0;
    while (k1 + 1 < nev && cl_first[k1 + 1] == k0) ++k1;
    double prev = -HUGE_VAL;
    for (int k = k0; k <= k1; ++k) {
      double lk = lam[k];
      // separate numerically equal eigenvalues of a cluster (dstein)
      double sep = 10.0 * DBL_EPSILON * fmax(fabs(lk), tnorm * 1e-3);
      if (k > k0 && lk - prev < sep) lk = prev + sep;
      prev = lk;
      tri_factor(d, e, n, lk, tiny, ai, b1, b2, l, piv);
      double* x = Z + (size_t)k * n;
      unsigned s = 0x9E3779B9u * (k + 1);
      for (int i = 0; i < n; ++i) {   // deterministic pseudo-random start vector
        s = s * 1664525u + 1013904223u;
        x[i] = 1.0 + 0.5 * (double(s >> 8) / 16777216.0 - 0.5);
      }
      // three steps: with an eigenvalue accurate to rounding, each solve
      // amplifies the wanted direction by ~1/eps
      for (int it = 0; it < 3; ++it) {
        tri_solve(n, ai, b1, b2, l, piv, x);
        for (int j = k0; j < k; ++j) {   // Gram-Schmidt against earlier members of the cluster
          const double* y = Z + (size_t)j * n;
          double dot = 0;
          for (int i = 0; i < n; ++i) dot += y[i] * x[i];
          for (int i = 0; i < n; ++i) x[i] -= dot * y[i];
        }
        double nrm = 0;
        for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
        nrm = sqrt(nrm);
        if (!(nrm > 0) || !isfinite(nrm)) { atomicExch(status, 1); break; }
        const double inv = 1.0 / nrm;
        for (int i = 0; i < n; ++i) x[i] *= inv;
      }
      // sign convention: largest component positive
      double big = 0;
      for (int i = 0; i < n; ++i) if (fabs(x[i]) > fabs(big)) big = x[i];
      if (big < 0) for (int i = 0; i < n; ++i) x[i] = -x[i];
    }
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

}  // namespace

void SmallEigen::reserve(Runtime& rt, int nmax) {
  if (nmax <= cap) return;
  cap = nmax;
  d.resize(nmax);
  e.resize(nmax);
  tau.resize(nmax);
  V.resize(size_t(nmax) * nmax);
  Z.resize(size_t(nmax) * nmax);
  scratch.resize(size_t(kEigThreads) * 5 * nmax + 16);
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
  cusolver_check(cusolverDnZhetrd(rt.solver, CUBLAS_FILL_MODE_UPPER, n, reinterpret_cast<cuDoubleComplex*>(A), n,
                                  d.get(), e.get(), reinterpret_cast<cuDoubleComplex*>(tau.get()),
                                  reinterpret_cast<cuDoubleComplex*>(work.get()), int(work.size()), info.get()),
                 "zhetrd");
  size_t sm = (3 * size_t(n) + nev) * sizeof(double) + size_t(nev) * sizeof(int);
  if (sm > 227 * 1024 || size_t(n) * sizeof(double2) > 227 * 1024) fail(kCapacity, "subspace eigenproblem too large for the tridiagonal solver: n=" + std::to_string(n));
  raise_smem_limit(tridiag_eig_kernel, sm);
  tridiag_eig_kernel<<<1, kEigThreads, sm, s>>>(d.get(), e.get(), n, nev, w, Z.get(), scratch.get(), status);
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

}  // namespace hb
