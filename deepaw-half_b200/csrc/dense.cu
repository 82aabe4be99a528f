// Dense H/S assembly and the dense generalized solves (evd, index-range).
//
// Reference: assemble_dense_gamma_cuda_full (src/half_cuda_assembly.cuf:
// 327-400) and solve_device_matrices (src/half_cuda_solver.cuf:97-181):
// H[i,j] = V(G_i - G_j) (circular box index) + T delta_ij + sum_I B_I D_I B_I^H,
// S = I + sum_I B_I Q B_I^H, hermitised; overlap extremes from zheevd(S);
// zhegvd for `evd`, zhegvdx with an index range for the VASP-like selector.
// Here the two projector sums are one GEMM each, (B . blockdiag(D)) B^H.
#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "blas.h"
#include "context.h"
#include "eig.h"

namespace hb {

const double2* projector_matrix64(KOperatorSet& ks);

namespace {

__global__ void local_dense_kernel(const double2* __restrict__ vg, const int* __restrict__ gvec,
                                   const double* __restrict__ kinetic, int n, int n1, int n2, int n3,
                                   double2* __restrict__ h, double2* __restrict__ s) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  int j = int(t / n), i = int(t - (long long)j * n);
  int a = ((gvec[3 * i] - gvec[3 * j]) % n1 + n1) % n1;
  int b = ((gvec[3 * i + 1] - gvec[3 * j + 1]) % n2 + n2) % n2;
  int c = ((gvec[3 * i + 2] - gvec[3 * j + 2]) % n3 + n3) % n3;
  double2 v = vg[((long long)a * n2 + b) * n3 + c];
  double2 one = make_double2(i == j ? 1.0 : 0.0, 0.0);
  if (i == j) v.x += kinetic[i];
  h[t] = v;
  s[t] = one;
}

// out[:, p] = sum_c B[:, base(p)+c] M[c][a(p)]
__global__ void right_blockdiag_kernel(const double2* __restrict__ B, int npw, const int* __restrict__ col_base,
                                       const int* __restrict__ col_a, const int* __restrict__ col_nlm,
                                       const int* __restrict__ col_ofs, const double* __restrict__ M,
                                       double2* __restrict__ out) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  int p = blockIdx.y;
  if (g >= npw) return;
  int base = col_base[p], a = col_a[p], nlm = col_nlm[p];
  const double* mat = M + col_ofs[p];
  double2 acc = make_double2(0, 0);
  for (int c = 0; c < nlm; ++c) {
    double w = mat[c * nlm + a];
    double2 b = B[(long long)(base + c) * npw + g];
    acc.x += w * b.x;
    acc.y += w * b.y;
  }
  out[(long long)p * npw + g] = acc;
}

__global__ void hermitize_kernel(double2* h, double2* s, int n) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  int j = int(t / n), i = int(t - (long long)j * n);
  if (i > j) return;
  long long ij = (long long)j * n + i, ji = (long long)i * n + j;
  double2 a = h[ij], b = h[ji];
  double2 z = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
  h[ij] = z;
  h[ji] = make_double2(z.x, -z.y);
  a = s[ij]; b = s[ji];
  z = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
  s[ij] = z;
  s[ji] = make_double2(z.x, -z.y);
}

__global__ void scale_kernel(double2* v, long long n, double s) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) v[i] = cscale(v[i], s);
}

__global__ void to_complex_kernel(const double* in, double2* out, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_double2(in[i], 0.0);
}

}  // namespace

void assemble_dense(Context& ctx, KOperatorSet& ks, double2* h, double2* s) {
  Runtime& rt = *ks.rt;
  cudaStream_t st = rt.stream;
  const Basis& b = ks.basis;
  const int n = int(b.npw());
  const long long nr = ctx.nr();
  DeviceBuffer<double2> vg(nr);
  to_complex_kernel<<<ceil_div(nr, 256), 256, 0, st>>>(ctx.veff.get(), vg.get(), nr);
  fft3d_inplace(vg.get(), b.shape, -1, st);
  scale_kernel<<<ceil_div(nr, 256), 256, 0, st>>>(vg.get(), nr, 1.0 / double(nr));
  DeviceBuffer<int> gv;
  gv.upload(b.gvec, st);
  DeviceBuffer<double> kin;
  kin.upload(b.kinetic, st);
  local_dense_kernel<<<ceil_div((long long)n * n, 256), 256, 0, st>>>(vg.get(), gv.get(), kin.get(), n, b.shape[0],
                                                                       b.shape[1], b.shape[2], h, s);
  HALF_LAUNCH("dense local");
  const int np = ks.np;
  if (np > 0) {
    std::vector<int> cb, ca, cn, cd, cq;
    std::vector<double> dall, qall;
    int col0 = 0, dofs = 0, qofs = 0;
    for (auto& sp : ctx.species) {
      for (int a = 0; a < sp.natoms; ++a)
        for (int i = 0; i < sp.nlm; ++i) {
          cb.push_back(col0 + a * sp.nlm);
          ca.push_back(i);
          cn.push_back(sp.nlm);
          cd.push_back(dofs + a * sp.nlm * sp.nlm);
          cq.push_back(qofs);
        }
      dall.insert(dall.end(), sp.dij_host.begin(), sp.dij_host.end());
      qall.insert(qall.end(), sp.qij_host.begin(), sp.qij_host.end());
      col0 += sp.natoms * sp.nlm;
      dofs += sp.natoms * sp.nlm * sp.nlm;
      qofs += sp.nlm * sp.nlm;
    }
    DeviceBuffer<int> dcb, dca, dcn, dcd, dcq;
    dcb.upload(cb, st); dca.upload(ca, st); dcn.upload(cn, st); dcd.upload(cd, st); dcq.upload(cq, st);
    DeviceBuffer<double> dd, dq;
    dd.upload(dall, st);
    dq.upload(qall, st);
    DeviceBuffer<double2> tmp((size_t)n * np);
    const double2* B = projector_matrix64(ks);
    const double2 one = make_double2(1, 0);
    right_blockdiag_kernel<<<dim3(ceil_div(n, 256), np), 256, 0, st>>>(B, n, dcb.get(), dca.get(), dcn.get(), dcd.get(),
                                                                        dd.get(), tmp.get());
    gemm(rt, CUBLAS_OP_N, CUBLAS_OP_C, n, n, np, one, tmp.get(), n, B, n, one, h, n);
    right_blockdiag_kernel<<<dim3(ceil_div(n, 256), np), 256, 0, st>>>(B, n, dcb.get(), dca.get(), dcn.get(), dcq.get(),
                                                                        dq.get(), tmp.get());
    gemm(rt, CUBLAS_OP_N, CUBLAS_OP_C, n, n, np, one, tmp.get(), n, B, n, one, s, n);
    HALF_LAUNCH("dense projectors");
  }
  hermitize_kernel<<<ceil_div((long long)n * n, 256), 256, 0, st>>>(h, s, n);
  HALF_LAUNCH("hermitize");
  HALF_CUDA(cudaStreamSynchronize(st));
}

namespace {

// Orders above this go through the 64-bit solver API: the workspace queries of
// zheevd / zhegvd return an int count of complex elements, which overflows near
// n = 2^15 (measured: the 38,089-plane-wave Gamma point of the 216-atom cell).
// HALF_DENSE_64BIT_ORDER lowers the switch point (tests exercise the 64-bit
// path at small orders with it).
long long dense_64bit_order() {
  const char* e = std::getenv("HALF_DENSE_64BIT_ORDER");
  if (e && *e) return std::atoll(e);
  return 16384;
}

struct DnParams {
  cusolverDnParams_t p = nullptr;
  DnParams() { cusolver_check(cusolverDnCreateParams(&p), "params"); }
  ~DnParams() { if (p) cusolverDnDestroyParams(p); }
  DnParams(const DnParams&) = delete;
  DnParams& operator=(const DnParams&) = delete;
};

struct Work64 {
  DeviceBuffer<unsigned char> dev;
  std::vector<unsigned char> host;
  void reserve(size_t d, size_t hb) {
    if (d > dev.size()) dev.resize(d);
    if (hb > host.size()) host.resize(hb);
  }
};

int read_info(const DeviceBuffer<int>& info, cudaStream_t st) {
  int h = 0;
  HALF_CUDA(cudaMemcpyAsync(&h, info.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  HALF_CUDA(cudaStreamSynchronize(st));
  return h;
}

// Eigenvalues (and, with vectors, eigenvectors in place) of the Hermitian
// matrix A through the 64-bit API; with index_range only the lowest nbands.
// Without vectors the lowest nbands come from the tridiagonal route of
// eig.cu instead: the 64-bit syevd's workspace query answered INVALID_VALUE
// at the 216-atom cell's Gamma point (n = 38,089), as the 32-bit one did.
void heevd64(Runtime& rt, const DnParams& prm, Work64& ws, bool vectors, bool index_range, long long n, int nbands,
             double2* A, double* w, DeviceBuffer<int>& info) {
  if (!vectors) {
    hermitian_eigenvalues_large(rt, A, n, {0}, {nbands}, w);
    return;
  }
  const cusolverEigMode_t jobz = CUSOLVER_EIG_MODE_VECTOR;
  size_t dbytes = 0, hbytes = 0;
  if (index_range) {
    double vl = 0, vu = 0;
    int64_t meig = 0;
    cusolver_check(cusolverDnXsyevdx_bufferSize(rt.solver, prm.p, jobz, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_UPPER, n,
                                                CUDA_C_64F, A, n, &vl, &vu, 1, nbands, &meig, CUDA_R_64F, w,
                                                CUDA_C_64F, &dbytes, &hbytes),
                   "Xsyevdx buffer");
    ws.reserve(dbytes, hbytes);
    cusolver_check(cusolverDnXsyevdx(rt.solver, prm.p, jobz, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_UPPER, n,
                                     CUDA_C_64F, A, n, &vl, &vu, 1, nbands, &meig, CUDA_R_64F, w, CUDA_C_64F,
                                     ws.dev.get(), ws.dev.size(), ws.host.data(), ws.host.size(), info.get()),
                   "Xsyevdx");
    if (read_info(info, rt.stream) != 0 || meig != nbands) fail(kInternal, "VASP-like generalized eigensolve failed");
    return;
  }
  cusolver_check(cusolverDnXsyevd_bufferSize(rt.solver, prm.p, jobz, CUBLAS_FILL_MODE_UPPER, n, CUDA_C_64F, A, n,
                                             CUDA_R_64F, w, CUDA_C_64F, &dbytes, &hbytes),
                 "Xsyevd buffer");
  ws.reserve(dbytes, hbytes);
  cusolver_check(cusolverDnXsyevd(rt.solver, prm.p, jobz, CUBLAS_FILL_MODE_UPPER, n, CUDA_C_64F, A, n, CUDA_R_64F, w,
                                  CUDA_C_64F, ws.dev.get(), ws.dev.size(), ws.host.data(), ws.host.size(), info.get()),
                 "Xsyevd");
  if (read_info(info, rt.stream) != 0) fail(kInternal, "eigensolve failed");
}

// The generalized problem H X = S X w at large order, the steps zhegvd takes:
// S = U^H U (Cholesky, upper), C = U^-H H U^-1 (two triangular solves),
// C Z = Z w, X = U^-1 Z.  H is overwritten by X, S by U.
void solve_dense_64(Runtime& rt, long long n, int nbands, bool index_range, bool vectors, double2* h, double2* s,
                    double* w, SolveOutput& out) {
  cudaStream_t st = rt.stream;
  DnParams prm;
  Work64 ws;
  DeviceBuffer<int> info(1);
  if (!index_range) {
    // overlap extremes from the eigenvalues of S (src/half_cuda_solver.cuf:146-150)
    DeviceBuffer<double2> s2((size_t)n * n);
    HALF_CUDA(cudaMemcpyAsync(s2.get(), s, (size_t)n * n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    hermitian_eigenvalues_large(rt, s2.get(), n, {0, int(n - 1)}, {1, 1}, w);
    double ext[2] = {0, 0};
    HALF_CUDA(cudaMemcpyAsync(ext, w, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaStreamSynchronize(st));
    out.overlap_min = ext[0];
    out.overlap_max = ext[1];
  } else {
    out.overlap_min = -1.0;
    out.overlap_max = -1.0;
  }
  size_t dbytes = 0, hbytes = 0;
  cusolver_check(cusolverDnXpotrf_bufferSize(rt.solver, prm.p, CUBLAS_FILL_MODE_UPPER, n, CUDA_C_64F, s, n, CUDA_C_64F,
                                             &dbytes, &hbytes),
                 "Xpotrf buffer");
  ws.reserve(dbytes, hbytes);
  cusolver_check(cusolverDnXpotrf(rt.solver, prm.p, CUBLAS_FILL_MODE_UPPER, n, CUDA_C_64F, s, n, CUDA_C_64F,
                                  ws.dev.get(), ws.dev.size(), ws.host.data(), ws.host.size(), info.get()),
                 "Xpotrf");
  if (read_info(info, st) != 0) fail(kInternal, "generalized eigensolve failed (overlap not positive definite)");
  const cuDoubleComplex one = make_cuDoubleComplex(1, 0);
  auto* H = reinterpret_cast<cuDoubleComplex*>(h);
  auto* U = reinterpret_cast<const cuDoubleComplex*>(s);
  cublas_check(cublasZtrsm_64(rt.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, n,
                              n, &one, U, n, H, n),
               "ztrsm U^-H H");
  cublas_check(cublasZtrsm_64(rt.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, n,
                              n, &one, U, n, H, n),
               "ztrsm H U^-1");
  heevd64(rt, prm, ws, vectors, index_range, n, nbands, h, w, info);
  if (vectors) {
    // only the first nbands columns of Z are kept
    cublas_check(cublasZtrsm_64(rt.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                                n, nbands, &one, U, n, H, n),
                 "ztrsm U^-1 Z");
  }
}

}  // namespace

void solve_dense(Context& ctx, KOperatorSet& ks, int nbands, bool index_range, bool want_vectors, SolveOutput& out) {
  Runtime& rt = *ks.rt;
  cudaStream_t st = rt.stream;
  const int n = int(ks.basis.npw());
  if (nbands < 1 || nbands > n) fail(kInvalidArgument, "invalid requested band count");
  DeviceBuffer<double2> h((size_t)n * n), s((size_t)n * n);
  assemble_dense(ctx, ks, h.get(), s.get());
  DeviceBuffer<double> w(n);
  DeviceBuffer<int> info(1);
  auto* H = reinterpret_cast<cuDoubleComplex*>(h.get());
  auto* S = reinterpret_cast<cuDoubleComplex*>(s.get());
  int lwork = 0, hinfo = 0;
  // eigenvectors are formed for the host copy or for a caller that keeps them on the device (forces)
  const bool compute_vectors = want_vectors || out.keep_device;
  if (n > dense_64bit_order()) {
    solve_dense_64(rt, n, nbands, index_range, compute_vectors, h.get(), s.get(), w.get(), out);
  } else if (index_range) {
    // src/half_cuda_solver.cuf:119-144: only the lowest nbands, no overlap solve
    int meig = 0;
    cusolverEigMode_t jobz = compute_vectors ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
    cusolver_check(cusolverDnZhegvdx_bufferSize(rt.solver, CUSOLVER_EIG_TYPE_1, jobz, CUSOLVER_EIG_RANGE_I,
                                                CUBLAS_FILL_MODE_UPPER, n, H, n, S, n, 0.0, 0.0, 1, nbands, &meig,
                                                w.get(), &lwork),
                   "zhegvdx buffer");
    DeviceBuffer<double2> work(std::max(lwork, 1));
    cusolver_check(cusolverDnZhegvdx(rt.solver, CUSOLVER_EIG_TYPE_1, jobz, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_UPPER,
                                     n, H, n, S, n, 0.0, 0.0, 1, nbands, &meig, w.get(),
                                     reinterpret_cast<cuDoubleComplex*>(work.get()), lwork, info.get()),
                   "zhegvdx");
    HALF_CUDA(cudaMemcpyAsync(&hinfo, info.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaStreamSynchronize(st));
    if (hinfo != 0 || meig != nbands) fail(kInternal, "VASP-like generalized eigensolve failed");
    out.overlap_min = -1.0;
    out.overlap_max = -1.0;
  } else {
    DeviceBuffer<double2> s2((size_t)n * n);
    HALF_CUDA(cudaMemcpyAsync(s2.get(), s.get(), (size_t)n * n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    auto* S2 = reinterpret_cast<cuDoubleComplex*>(s2.get());
    cusolver_check(cusolverDnZheevd_bufferSize(rt.solver, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_UPPER, n, S2, n,
                                               w.get(), &lwork),
                   "zheevd buffer");
    int lwork2 = 0;
    cusolverEigMode_t jobz = compute_vectors ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
    cusolver_check(cusolverDnZhegvd_bufferSize(rt.solver, CUSOLVER_EIG_TYPE_1, jobz, CUBLAS_FILL_MODE_UPPER, n, H, n, S,
                                               n, w.get(), &lwork2),
                   "zhegvd buffer");
    DeviceBuffer<double2> work(std::max({lwork, lwork2, 1}));
    cusolver_check(cusolverDnZheevd(rt.solver, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_UPPER, n, S2, n, w.get(),
                                    reinterpret_cast<cuDoubleComplex*>(work.get()), int(work.size()), info.get()),
                   "zheevd");
    std::vector<double> ov(n);
    HALF_CUDA(cudaMemcpyAsync(&hinfo, info.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaMemcpyAsync(ov.data(), w.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaStreamSynchronize(st));
    if (hinfo != 0) fail(kInternal, "overlap eigensolve failed");
    out.overlap_min = ov.front();
    out.overlap_max = ov.back();
    cusolver_check(cusolverDnZhegvd(rt.solver, CUSOLVER_EIG_TYPE_1, jobz, CUBLAS_FILL_MODE_UPPER, n, H, n, S, n, w.get(),
                                    reinterpret_cast<cuDoubleComplex*>(work.get()), int(work.size()), info.get()),
                   "zhegvd");
    HALF_CUDA(cudaMemcpyAsync(&hinfo, info.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaStreamSynchronize(st));
    if (hinfo != 0) fail(kInternal, "generalized eigensolve failed");
  }
  std::vector<double> ev(n);
  HALF_CUDA(cudaMemcpyAsync(ev.data(), w.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st));
  HALF_CUDA(cudaStreamSynchronize(st));
  out.eigenvalues.assign(ev.begin(), ev.begin() + nbands);
  if (compute_vectors) {
    out.dvectors.resize((size_t)n * nbands);
    HALF_CUDA(cudaMemcpyAsync(out.dvectors.get(), h.get(), (size_t)n * nbands * sizeof(double2),
                              cudaMemcpyDeviceToDevice, st));
  } else {
    out.dvectors.release();
  }
  if (want_vectors) {
    out.vectors.resize((size_t)2 * n * nbands);
    HALF_CUDA(cudaMemcpyAsync(out.vectors.data(), h.get(), (size_t)n * nbands * sizeof(double2), cudaMemcpyDeviceToHost, st));
  }
  HALF_CUDA(cudaStreamSynchronize(st));
}

}  // namespace hb
