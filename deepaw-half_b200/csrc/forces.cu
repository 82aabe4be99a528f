// Hellmann-Feynman band-energy (non-local PAW) force on the GPU: a
// hand-written FP64 adjoint kernel.
//
// Reference: add_nonlocal_paw_forces (src/half_forces.F90:9-73), a host triple
// loop recomputing c = B_I^H psi_n and dc_alpha = B_I^H (i q_alpha psi_n) per
// atom and band, then
//   F_I,alpha -= 2 w f_n Re[((D_I - eps_n Q) c)^H dc_alpha] + w f_n Re[c^H dD_I/dR_alpha c].
//
// B200 design: one kernel, one CTA per (atom, tile of 128 bands; 64 or 32
// for atoms with more than 8 or 16 channels), 8 warps.  Per
// chunk of 32 plane waves the CTA stages psi (coalesced along g), the plane
// waves' q vectors, the atom's phase exp(+i q.R) (from the packed G indices and
// the atom's b_j.R / 2 pi, reduced to one turn in FP64) and the chunk of
// conj(B) = Omega^-1/2 beta_l(|q|) Y_lm(q^) i^l exp(+i q.R) generated from the
// k point's radial-angular table: B is never stored, and neither is the
// [psi | i q psi] block.  Thread = (band, group of up to four projector
// channels): every thread accumulates c and u_alpha = sum_g q_alpha conj(B)
// psi for its channels in FP64 registers (dc_alpha = i u_alpha).  The
// epilogue contracts them with D, Q and dD/dR per band and reduces the
// tile's bands with warp shuffles and one ordered sum; a second kernel
// adds the band tiles of each atom in order, so the result does not depend on
// scheduling.  Bands with zero occupation are skipped as in the reference.
#include <algorithm>

#include "context.h"

namespace hb {

namespace {

constexpr int kMaxNlm = 32;
constexpr int kAdjThreads = 256;
constexpr int kAdjPer = 4;                     // projector channels per thread
constexpr int kAdjG = 32;                      // plane waves per shared-memory chunk

struct AtomInfo {
  int col;     // first projector column of the atom
  int nlm;
  int dofs;    // offset of D_I (row-major nlm x nlm)
  int ddofs;   // offset of dD_I ([alpha][a][b])
  int qofs;    // offset of the species Q
};

// Shared memory of the kernel variant with BT bands per CTA (256 / BT
// channel groups): the chunk staging, or the epilogue's c and dc of every
// band of the tile, whichever is larger.
size_t adjoint_smem(int bt) {
  const int groups = kAdjThreads / bt;
  const size_t chunk = (size_t(kAdjG) * kMaxNlm + size_t(kAdjG) * (bt + 1)) * sizeof(double2) +
                       size_t(kAdjG) * 4 * sizeof(double);
  const size_t epilogue = size_t(4) * bt * groups * kAdjPer * sizeof(double2) + 8 * 3 * sizeof(double);
  return std::max(chunk, epilogue);
}

// One CTA per (atom, BT-band tile).  Thread = (band b = tid % BT, channel
// group grp = tid / BT); it owns channels grp, grp + G, ... (up to kAdjPer of
// them, G = 256 / BT groups, so atoms of up to 4 G channels).  A warp is 32
// consecutive bands of one group: psi loads from shared memory are
// conflict-free and the conj(B), q and phase loads are broadcasts.
template <int BT>
__global__ void __launch_bounds__(kAdjThreads)
    force_adjoint_kernel(const double2* __restrict__ psi, long long ld, int npw, int nb, const double* __restrict__ qv,
                         const double* __restrict__ ftab, const int* __restrict__ gpack, const int* __restrict__ pcol,
                         const double* __restrict__ afrac, double kf0, double kf1, double kf2,
                         const AtomInfo* __restrict__ atoms, const double* __restrict__ dall,
                         const double* __restrict__ ddall, const double* __restrict__ qall,
                         const double* __restrict__ eig, const double* __restrict__ occ, double kweight,
                         double* __restrict__ partial) {
  constexpr int G = kAdjThreads / BT;
  constexpr int NL = G * kAdjPer;   // channel slots of a band in the epilogue
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* sB = reinterpret_cast<double2*>(smem_raw);      // [kAdjG][kMaxNlm]  conj(B)
  // [kAdjG][BT + 1]: the row pad keeps the g-major staging stores and the
  // band-major reads free of bank conflicts
  constexpr int BP = BT + 1;
  double2* spsi = sB + kAdjG * kMaxNlm;
  double* sq = reinterpret_cast<double*>(spsi + kAdjG * BP);   // [kAdjG][4]: q_x, q_y, q_z
  __shared__ double2 sph[kAdjG];
  __shared__ int sfrow[kMaxNlm], sl[kMaxNlm];
  const int ion = blockIdx.x, bt = blockIdx.y;
  const AtomInfo A = atoms[ion];
  const int nlm = A.nlm;
  const int tid = threadIdx.x, bl = tid % BT, grp = tid / BT;
  const int n = bt * BT + bl;
  if (tid < nlm) {
    const int d = pcol[A.col + tid];
    sfrow[tid] = (d >> 2) & 0x3FFF;
    sl[tid] = d & 3;
  }
  const int atom = pcol[A.col] >> 16;
  const double f0 = afrac[3 * atom], f1 = afrac[3 * atom + 1], f2 = afrac[3 * atom + 2];
  double2 acc[4][kAdjPer];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int j = 0; j < kAdjPer; ++j) acc[q][j] = make_double2(0.0, 0.0);

  for (int g0 = 0; g0 < npw; g0 += kAdjG) {
    __syncthreads();   // the previous chunk has been consumed
    if (tid < kAdjG) {
      const int g = g0 + tid;
      double2 ph = make_double2(0.0, 0.0);
      if (g < npw) {
        const int gp = gpack[g];
        const double t = (double((gp << 22) >> 22) + kf0) * f0 + (double((gp << 12) >> 22) + kf1) * f1 +
                         (double((gp << 2) >> 22) + kf2) * f2;
        double s, c;
        sincospi(2.0 * (t - rint(t)), &s, &c);
        ph = make_double2(c, s);   // exp(+i q.R)
      }
      sph[tid] = ph;
    }
    for (int t = tid; t < kAdjG * BT; t += kAdjThreads) {
      const int gl = t % kAdjG, b = t / kAdjG, g = g0 + gl, nn = bt * BT + b;
      spsi[gl * BP + b] = (g < npw && nn < nb) ? psi[(long long)nn * ld + g] : make_double2(0.0, 0.0);
    }
    for (int t = tid; t < kAdjG * 3; t += kAdjThreads) {
      const int gl = t / 3, a = t - 3 * gl, g = g0 + gl;
      sq[4 * gl + a] = g < npw ? qv[3 * (long long)g + a] : 0.0;
    }
    __syncthreads();
    for (int t = tid; t < kAdjG * nlm; t += kAdjThreads) {
      const int gl = t / nlm, a = t - gl * nlm, g = g0 + gl;
      double2 v = make_double2(0.0, 0.0);
      if (g < npw) {
        const double f = ftab[(long long)sfrow[a] * npw + g];
        const double2 p = sph[gl];
        double re, im;   // i^l (c + i s)
        switch (sl[a]) {
          case 0: re = p.x; im = p.y; break;
          case 1: re = -p.y; im = p.x; break;
          case 2: re = -p.x; im = -p.y; break;
          default: re = p.y; im = -p.x; break;
        }
        v = make_double2(f * re, f * im);
      }
      sB[gl * kMaxNlm + a] = v;
    }
    __syncthreads();
    if (n < nb) {
#pragma unroll 4
      for (int gl = 0; gl < kAdjG; ++gl) {
        const double2 x = spsi[gl * BP + bl];
        const double qx = sq[4 * gl], qy = sq[4 * gl + 1], qz = sq[4 * gl + 2];
#pragma unroll
        for (int j = 0; j < kAdjPer; ++j) {
          const int a = grp + j * G;
          if (a < nlm) {
            const double2 b = sB[gl * kMaxNlm + a];
            const double tr = b.x * x.x - b.y * x.y, ti = b.x * x.y + b.y * x.x;
            acc[0][j].x += tr;
            acc[0][j].y += ti;
            acc[1][j].x = fma(qx, tr, acc[1][j].x);
            acc[1][j].y = fma(qx, ti, acc[1][j].y);
            acc[2][j].x = fma(qy, tr, acc[2][j].x);
            acc[2][j].y = fma(qy, ti, acc[2][j].y);
            acc[3][j].x = fma(qz, tr, acc[3][j].x);
            acc[3][j].y = fma(qz, ti, acc[3][j].y);
          }
        }
      }
    }
  }
  __syncthreads();
  // c and dc_alpha = i u_alpha of every band of the tile -> shared memory
  double2* sc = reinterpret_cast<double2*>(smem_raw);   // [4][BT][NL]
#pragma unroll
  for (int j = 0; j < kAdjPer; ++j) {
    const int a = grp + j * G;
    if (a < nlm) {
      sc[(0 * BT + bl) * NL + a] = acc[0][j];
      for (int al = 0; al < 3; ++al)
        sc[((1 + al) * BT + bl) * NL + a] = make_double2(-acc[1 + al][j].y, acc[1 + al][j].x);
    }
  }
  __syncthreads();
  double* wsum = reinterpret_cast<double*>(sc + 4 * BT * NL);   // [BT / 32][3]
  if (tid < BT) {
    double fsum[3] = {0.0, 0.0, 0.0};
    const double fo = n < nb ? occ[n] : 0.0;
    if (fo != 0.0) {
      const double e = eig[n];
      const double* D = dall + A.dofs;
      const double* Q = qall + A.qofs;
      const double2* c = sc + bl * NL;
      double2 mc[NL];
      for (int a = 0; a < nlm; ++a) {
        double2 s = make_double2(0.0, 0.0);
        for (int k = 0; k < nlm; ++k) {
          const double w = D[a * nlm + k] - e * Q[a * nlm + k];
          s.x += w * c[k].x;
          s.y += w * c[k].y;
        }
        mc[a] = s;
      }
      for (int al = 0; al < 3; ++al) {
        const double2* dc = sc + ((1 + al) * BT + bl) * NL;
        double re = 0.0;
        for (int a = 0; a < nlm; ++a) re += mc[a].x * dc[a].x + mc[a].y * dc[a].y;   // Re(conj(mc) . dc)
        const double* dD = ddall + A.ddofs + al * nlm * nlm;
        double q = 0.0;
        for (int a = 0; a < nlm; ++a) {
          double2 s = make_double2(0.0, 0.0);
          for (int k = 0; k < nlm; ++k) {
            s.x += dD[a * nlm + k] * c[k].x;
            s.y += dD[a * nlm + k] * c[k].y;
          }
          q += c[a].x * s.x + c[a].y * s.y;   // Re(conj(c) . dD c)
        }
        fsum[al] = -2.0 * kweight * fo * re - kweight * fo * q;
      }
    }
    for (int al = 0; al < 3; ++al) {
      double v = fsum[al];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if ((tid & 31) == 0) wsum[(tid >> 5) * 3 + al] = v;
    }
  }
  __syncthreads();
  if (tid < 3) {   // the tile's warps in order
    double v = 0.0;
    for (int w = 0; w < BT / 32; ++w) v += wsum[w * 3 + tid];
    partial[((long long)ion * gridDim.y + bt) * 3 + tid] = v;
  }
}

// out[ion][alpha] = sum over band tiles, in tile order.
__global__ void sum_tiles_kernel(const double* __restrict__ partial, int nions, int ntiles, double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nions * 3) return;
  const int ion = t / 3, al = t - 3 * ion;
  double s = 0.0;
  for (int b = 0; b < ntiles; ++b) s += partial[((long long)ion * ntiles + b) * 3 + al];
  out[t] = s;
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
  int nlm_max = 1;
  for (auto& sp : ctx.species) nlm_max = std::max(nlm_max, sp.nlm);
  // bands per CTA: 128 for atoms of up to 8 channels, 64 up to 16, 32 up to 32
  const int bt = nlm_max <= 2 * kAdjPer ? 128 : nlm_max <= 4 * kAdjPer ? 64 : 32;
  const int ntiles = (nb + bt - 1) / bt;
  DeviceBuffer<AtomInfo> datoms;
  datoms.upload(atoms, st);
  DeviceBuffer<double> dd, ddd, dq, deig, docc, dpart(size_t(nions) * ntiles * 3), dout(size_t(nions) * 3);
  dd.upload(dall, st);
  ddd.upload(ddall, st);
  dq.upload(qall, st);
  deig.upload(eig, nb, st);
  docc.upload(occ, nb, st);
  const size_t smem = adjoint_smem(bt);
  Profile& pf = rt.prof;
  const int ev0 = pf.record(st);
  auto launch = [&](auto kernel) {
    raise_smem_limit(kernel, smem);
    kernel<<<dim3(nions, ntiles), kAdjThreads, smem, st>>>(
        dvec, ld, npw, nb, ks.qvec.get(), ks.ftab64.get(), ks.gpack.get(), ks.pcol.get(), ks.afrac.get(), ks.kf[0],
        ks.kf[1], ks.kf[2], datoms.get(), dd.get(), ddd.get(), dq.get(), deig.get(), docc.get(), kweight, dpart.get());
  };
  if (bt == 128) launch(force_adjoint_kernel<128>);
  else if (bt == 64) launch(force_adjoint_kernel<64>);
  else launch(force_adjoint_kernel<32>);
  HALF_LAUNCH("force adjoint");
  sum_tiles_kernel<<<ceil_div(nions * 3, 128), 128, 0, st>>>(dpart.get(), nions, ntiles, dout.get());
  HALF_LAUNCH("force tiles");
  pf.span(Profile::kAdjoint, ev0, pf.record(st));
  pf.launches += 2;
  auto f = dout.download(st);
  for (int i = 0; i < nions * 3; ++i) forces_host[i] += f[i];
}

}  // namespace hb
