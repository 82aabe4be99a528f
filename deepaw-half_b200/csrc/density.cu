// Output density of solved states on the device: the smooth part
// sum_k w_k sum_n f_nk |psi_nk(r)|^2 (src/half_local_forces.F90:102-127) plus
// the MIMIC_US augmentation (src/half_uspp.F90:26-111):
//   rho_ij^I = sum_k w_k sum_n f_nk Re(conj(c_i) c_j),  c = B_I^H psi_n,
//   n_aug(r) = Omega sum_I sum_lm [sum_ij rho_ij^I M_ij,lm] g_l(|r - R_I|) Y_lm(r - R_I)
// over the box points within paw_rmax of each atom (minimum image).
//
// * The smooth part reuses the operator's sphere->planes pass and a density
//   variant of its x-line pass (hs.cu), so no band is ever scattered into a
//   full zeroed box.
// * All projector coefficients of a k point come from one GEMM B^H X.
// * The augmentation deposit is one thread per box point looping over the
//   species' atoms in order (the reference's per-point summation order), no
//   atomics.
#include <algorithm>
#include <cmath>

#include "blas.h"
#include "context.h"

namespace hb {

const double2* projector_matrix64(KOperatorSet& ks);   // hs.cu

namespace {

struct OccAtom {
  int col;   // first projector column of the atom
  int nlm;
  int ofs;   // offset of its nlm x nlm occupancy (row-major [a][b])
};

// occ[ofs + a*nlm + b] += sum_n bw[n] Re(conj(c[col+a, n]) c[col+b, n]), bands in order.
__global__ void occupancy_kernel(const double2* __restrict__ cc, int np, int nb, const OccAtom* __restrict__ atoms,
                                 const double* __restrict__ bw, double* __restrict__ occ) {
  const OccAtom A = atoms[blockIdx.x];
  const int npair = A.nlm * A.nlm;
  for (int t = threadIdx.x; t < npair; t += blockDim.x) {
    const int a = t / A.nlm, b = t - a * A.nlm;
    double acc = occ[A.ofs + t];
    for (int n = 0; n < nb; ++n) {
      const double2 ca = cc[(long long)n * np + A.col + a], cb = cc[(long long)n * np + A.col + b];
      acc += bw[n] * (ca.x * cb.x + ca.y * cb.y);
    }
    occ[A.ofs + t] = acc;
  }
}

struct BoxCell {
  double lat[9];   // rows a_i
};

// density_f (x fastest) += Omega * sum over the species' atoms within rmax of
// sum_k coeff[a*naug + k] g_{l_k}(r) Y_{l_k m_k}; shape = [l][z1, z2, c1, c2].
__global__ void augmentation_deposit_kernel(double* __restrict__ density_f, int n1, int n2, int n3,
                                            const double* __restrict__ frac, int natoms, BoxCell cell, double rmax,
                                            const double* __restrict__ coeff, int lmax,
                                            const double* __restrict__ shape, double volume) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n1 * n2 * n3) return;
  const int i1 = int(idx % n1);
  const long long t = idx / n1;
  const int i2 = int(t % n2), i3 = int(t / n2);
  const double f1 = double(i1) / n1, f2 = double(i2) / n2, f3 = double(i3) / n3;
  const int naug = (lmax + 1) * (lmax + 1);
  double total = density_f[idx];
  for (int a = 0; a < natoms; ++a) {
    double d1 = f1 - frac[3 * a], d2 = f2 - frac[3 * a + 1], d3 = f3 - frac[3 * a + 2];
    d1 -= round(d1);
    d2 -= round(d2);
    d3 -= round(d3);
    const double x = d1 * cell.lat[0] + d2 * cell.lat[3] + d3 * cell.lat[6];
    const double y = d1 * cell.lat[1] + d2 * cell.lat[4] + d3 * cell.lat[7];
    const double z = d1 * cell.lat[2] + d2 * cell.lat[5] + d3 * cell.lat[8];
    const double r = sqrt(x * x + y * y + z * z);
    if (r > rmax) continue;
    double ct = cos(0.0), phi = 0.0;
    if (r > 1.0e-14) {
      ct = cos(acos(fmax(-1.0, fmin(1.0, z / r))));
      phi = atan2(y, x);
    }
    double value = 0;
    int k = 0;
    for (int l = 0; l <= lmax; ++l) {
      const double* sc = shape + 4 * l;
      const double g = sc[2] * sph_bessel(l, sc[0] * r / rmax) + sc[3] * sph_bessel(l, sc[1] * r / rmax);
      for (int m = -l; m <= l; ++m, ++k) value += coeff[a * naug + k] * g * real_ylm(l, m, ct, phi);
    }
    total += volume * value;
  }
  density_f[idx] = total;
}

__global__ void reorder_c_to_f_kernel(const double* in, double* out, int n1, int n2, int n3) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)n1 * n2 * n3;
  if (i >= n) return;
  const int i3 = int(i % n3);
  const long long t = i / n3;
  const int i2 = int(t % n2), i1 = int(t / n2);
  out[i1 + (long long)n1 * (i2 + (long long)n2 * i3)] = in[i];
}

// part[block] = sum of the block's strided share of v (fixed order).
__global__ void box_sum_kernel(const double* v, long long n, double* part) {
  __shared__ double red[256];
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += v[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

double box_sum(const double* v, long long n, cudaStream_t s) {
  constexpr int kBlocks = 4 * 148;
  DeviceBuffer<double> part(kBlocks);
  box_sum_kernel<<<kBlocks, 256, 0, s>>>(v, n, part.get());
  HALF_LAUNCH("box sum");
  double total = 0;
  for (double p : part.download(s)) total += p;
  return total;
}

}  // namespace

void accumulate_band_density(KOperatorSet& ks, const double2* x, long long ld, int nb, const double* bw,
                             double* density_c, int chunk);   // hs.cu

void output_density_device(Context& ctx, int nk, const double* kpoints, const double* kweights, int nb,
                           const std::vector<const double2*>& vectors, const std::vector<long long>& ld,
                           const double* occupations, double* density_f, double* augmentation_charge) {
  Runtime& rt = *ctx.rt;
  cudaStream_t s = rt.stream;
  const auto& sh = ctx.charge.shape;
  const long long n = ctx.nr();
  const int nions = ctx.crystal.nions();
  // occupancy layout: atoms in the context's (type-major) order
  std::vector<OccAtom> atoms(nions);
  int col0 = 0, ofs = 0;
  for (auto& sp : ctx.species) {
    for (int a = 0; a < sp.natoms; ++a) {
      atoms[sp.first_ion + a] = OccAtom{col0 + a * sp.nlm, sp.nlm, ofs};
      ofs += sp.nlm * sp.nlm;
    }
    col0 += sp.natoms * sp.nlm;
  }
  DeviceBuffer<OccAtom> datoms;
  datoms.upload(atoms, s);
  DeviceBuffer<double> occ(std::max(ofs, 1)), density_c(n), bw(nb);
  occ.zero(s);
  density_c.zero(s);
  const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
  for (int ik = 0; ik < nk; ++ik) {
    auto ks = prepare_operator(ctx, rt, kpoints + 3 * ik, true, false);
    const int npw = int(ks->basis.npw());
    if (ld[ik] < npw) fail(kCapacity, "eigenvector leading dimension is too small");
    std::vector<double> w(nb);
    for (int b = 0; b < nb; ++b) w[b] = kweights[ik] * occupations[(size_t)ik * nb + b];
    bw.upload(w, s);
    accumulate_band_density(*ks, vectors[ik], ld[ik], nb, bw.get(), density_c.get(), ctx.acc.block);
    if (ks->np > 0 && nions > 0) {
      DeviceBuffer<double2> cc((size_t)ks->np * nb);
      gemm(rt, CUBLAS_OP_C, CUBLAS_OP_N, ks->np, nb, npw, one, projector_matrix64(*ks), npw, vectors[ik], ld[ik], zero,
           cc.get(), ks->np);
      occupancy_kernel<<<nions, 128, 0, s>>>(cc.get(), ks->np, nb, datoms.get(), bw.get(), occ.get());
      HALF_LAUNCH("augmentation occupancy");
      HALF_CUDA(cudaStreamSynchronize(s));
    }
    HALF_CUDA(cudaStreamSynchronize(s));   // the operator, its work buffer and cc are released here
  }
  reorder_c_to_f_kernel<<<ceil_div(n, 256), 256, 0, s>>>(density_c.get(), density_f, sh[0], sh[1], sh[2]);
  HALF_LAUNCH("reorder density");
  const double before = box_sum(density_f, n, s) / double(n);
  // augmentation deposit, species by species
  const std::vector<double> occ_h = occ.download(s);
  BoxCell cell{};
  for (int k = 0; k < 9; ++k) cell.lat[k] = ctx.crystal.lattice[k];
  for (size_t it = 0; it < ctx.species.size(); ++it) {
    const SpeciesDevice& sp = ctx.species[it];
    const QdepTables& t = sp.tables;
    if (sp.natoms == 0 || t.naug == 0) continue;
    std::vector<double> coeff((size_t)sp.natoms * t.naug, 0.0), frac;
    for (int a = 0; a < sp.natoms; ++a) {
      const double* o = occ_h.data() + atoms[sp.first_ion + a].ofs;
      for (int k = 0; k < t.naug; ++k) {
        double c = 0;
        for (int jb = 0; jb < t.nlm; ++jb)
          for (int ja = 0; ja < t.nlm; ++ja) c += o[ja * t.nlm + jb] * t.multipole[((size_t)ja * t.nlm + jb) * t.naug + k];
        coeff[(size_t)a * t.naug + k] = c;
      }
      for (int d = 0; d < 3; ++d) frac.push_back(ctx.crystal.positions[3 * (sp.first_ion + a) + d]);
    }
    DeviceBuffer<double> dcoeff, dfrac, dshape;
    dcoeff.upload(coeff, s);
    dfrac.upload(frac, s);
    dshape.upload(t.shape_coeff, s);
    augmentation_deposit_kernel<<<ceil_div(n, 256), 256, 0, s>>>(density_f, sh[0], sh[1], sh[2], dfrac.get(),
                                                                 sp.natoms, cell, ctx.pots[it].paw_rmax, dcoeff.get(),
                                                                 t.lmax, dshape.get(), ctx.crystal.volume());
    HALF_LAUNCH("augmentation deposit");
    HALF_CUDA(cudaStreamSynchronize(s));
  }
  const double after = box_sum(density_f, n, s) / double(n);
  if (augmentation_charge) *augmentation_charge = after - before;
}

}  // namespace hb
