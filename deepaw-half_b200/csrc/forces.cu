// Hellmann-Feynman band-energy (non-local PAW) force on the GPU.
//
// Reference: add_nonlocal_paw_forces (src/half_forces.F90:9-73), a host triple
// loop recomputing c = B_I^H psi_n and dc_alpha = B_I^H (i q_alpha psi_n) per
// atom and band, then
//   F_I,alpha -= 2 w f_n Re[((D_I - eps_n Q) c)^H dc_alpha] + w f_n Re[c^H dD_I/dR_alpha c].
// Here all c and dc for all atoms and bands come from ONE GEMM
//   B^H [psi | i q_x psi | i q_y psi | i q_z psi]   (N_p x 4m, K = N_pw),
// followed by an epilogue kernel (one block per atom, threads over bands,
// deterministic tree reduction).  Bands with zero occupation are skipped as
// in the reference.
#include <algorithm>

#include "blas.h"
#include "context.h"

namespace hb {

const double2* projector_matrix64(KOperatorSet& ks);

namespace {

constexpr int kMaxNlm = 32;

__global__ void build_qpsi_kernel(const double2* __restrict__ psi, long long ld, int npw, int nb,
                                  const double* __restrict__ q, double2* __restrict__ w) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)npw * nb) return;
  int b = int(t / npw), g = int(t - (long long)b * npw);
  double2 x = psi[(long long)b * ld + g];
  const long long blk = (long long)npw * nb;
  w[(long long)b * npw + g] = x;
  for (int a = 0; a < 3; ++a) {
    double qa = q[3 * g + a];
    w[(a + 1) * blk + (long long)b * npw + g] = make_double2(-qa * x.y, qa * x.x);   // i q_alpha psi
  }
}

struct AtomInfo {
  int col;     // first projector column of the atom
  int nlm;
  int dofs;    // offset of D_I (row-major nlm x nlm)
  int ddofs;   // offset of dD_I ([alpha][a][b])
  int qofs;    // offset of the species Q
};

__global__ void force_epilogue_kernel(const double2* __restrict__ cc, int np, int nb, const AtomInfo* __restrict__ atoms,
                                      const double* __restrict__ dall, const double* __restrict__ ddall,
                                      const double* __restrict__ qall, const double* __restrict__ eig,
                                      const double* __restrict__ occ, double kweight, double* __restrict__ out) {
  const int ion = blockIdx.x;
  const AtomInfo A = atoms[ion];
  const int nlm = A.nlm;
  const double* D = dall + A.dofs;
  const double* Q = qall + A.qofs;
  double f[3] = {0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    double fo = occ[b];
    if (fo == 0.0) continue;
    double e = eig[b];
    double2 c[kMaxNlm];
    for (int a = 0; a < nlm; ++a) c[a] = cc[(long long)b * np + A.col + a];
    double2 mc[kMaxNlm];
    for (int a = 0; a < nlm; ++a) {
      double2 acc = make_double2(0, 0);
      for (int k = 0; k < nlm; ++k) {
        double w = D[a * nlm + k] - e * Q[a * nlm + k];
        acc.x += w * c[k].x;
        acc.y += w * c[k].y;
      }
      mc[a] = acc;
    }
    for (int al = 0; al < 3; ++al) {
      const double2* dc = cc + (long long)(al + 1) * nb * np + (long long)b * np + A.col;
      double re = 0;
      for (int a = 0; a < nlm; ++a) re += mc[a].x * dc[a].x + mc[a].y * dc[a].y;   // Re(conj(mc) . dc)
      double t1 = -2.0 * kweight * fo * re;
      const double* dD = ddall + A.ddofs + al * nlm * nlm;
      double q = 0;
      for (int a = 0; a < nlm; ++a) {
        double2 acc = make_double2(0, 0);
        for (int k = 0; k < nlm; ++k) {
          acc.x += dD[a * nlm + k] * c[k].x;
          acc.y += dD[a * nlm + k] * c[k].y;
        }
        q += c[a].x * acc.x + c[a].y * acc.y;   // Re(conj(c) . dD c)
      }
      f[al] += t1 - kweight * fo * q;
    }
  }
  __shared__ double red[3][256];
  for (int al = 0; al < 3; ++al) red[al][threadIdx.x] = f[al];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int al = 0; al < 3; ++al) red[al][threadIdx.x] += red[al][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int al = 0; al < 3; ++al) out[3 * ion + al] = red[al][0];
}

}  // namespace

void nonlocal_forces_device(Context& ctx, KOperatorSet& ks, const double2* dvec, long long ld, int nb, const double* eig,
                            const double* occ, double kweight, double* forces_host) {
  Runtime& rt = *ks.rt;
  cudaStream_t st = rt.stream;
  const int npw = int(ks.basis.npw()), np = ks.np;
  const int nions = ctx.crystal.nions();
  if (np == 0 || nb == 0) return;
  std::vector<AtomInfo> atoms(nions);
  std::vector<double> dall, ddall, qall;
  int col0 = 0;
  for (auto& sp : ctx.species) {
    if (sp.nlm > kMaxNlm) fail(kUnavailable, "more than 32 projector functions per atom");
    auto ddh = sp.ddij.download(st);
    int qofs = int(qall.size());
    qall.insert(qall.end(), sp.qij_host.begin(), sp.qij_host.end());
    for (int a = 0; a < sp.natoms; ++a) {
      AtomInfo ai;
      ai.col = col0 + a * sp.nlm;
      ai.nlm = sp.nlm;
      ai.dofs = int(dall.size()) + a * sp.nlm * sp.nlm;
      ai.ddofs = int(ddall.size()) + a * 3 * sp.nlm * sp.nlm;
      ai.qofs = qofs;
      atoms[sp.first_ion + a] = ai;
    }
    dall.insert(dall.end(), sp.dij_host.begin(), sp.dij_host.end());
    ddall.insert(ddall.end(), ddh.begin(), ddh.end());
    col0 += sp.natoms * sp.nlm;
  }
  DeviceBuffer<AtomInfo> datoms;
  datoms.upload(atoms, st);
  DeviceBuffer<double> dd, ddd, dq, deig, docc, dout(size_t(nions) * 3);
  dd.upload(dall, st);
  ddd.upload(ddall, st);
  dq.upload(qall, st);
  deig.upload(eig, nb, st);
  docc.upload(occ, nb, st);
  DeviceBuffer<double2> w(size_t(4) * npw * nb), cc(size_t(4) * np * nb);
  Profile& pf = rt.prof;
  const int ev0 = pf.record(st);
  build_qpsi_kernel<<<ceil_div((long long)npw * nb, 256), 256, 0, st>>>(dvec, ld, npw, nb, ks.qvec.get(), w.get());
  HALF_LAUNCH("force qpsi");
  const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
  gemm(rt, CUBLAS_OP_C, CUBLAS_OP_N, np, 4 * nb, npw, one, projector_matrix64(ks), npw, w.get(), npw, zero, cc.get(), np);
  force_epilogue_kernel<<<nions, 256, 0, st>>>(cc.get(), np, nb, datoms.get(), dd.get(), ddd.get(), dq.get(), deig.get(),
                                               docc.get(), kweight, dout.get());
  HALF_LAUNCH("force epilogue");
  pf.span(Profile::kAdjoint, ev0, pf.record(st));
  pf.launches += 2;
  auto f = dout.download(st);
  for (int i = 0; i < nions * 3; ++i) forces_host[i] += f[i];
}

}  // namespace hb
