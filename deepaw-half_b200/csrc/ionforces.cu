// Ion-position force terms of the reference's --forces path
// (app/half_cli.F90:947-955), on the device:
//
// * Ewald ion-ion energy and force (src/half_energy.F90:122-210);
// * local ionic force and energy on a density (src/half_local_forces.F90:11-56);
// * non-linear core correction force with the input density's V_xc (:58-100);
// * the frozen-input Harris response (:129-161) through the radial core-density
//   force (:163-191).
//
// The three density terms are one reciprocal-space contraction
//   F_I = - sum_G G * Im( w(G) e^{-i G.R_I} ),  E = sum_I sum_G Re( w(G) e^{-i G.R_I} ),
//   w(G) = scale * radial_s(|G|) * conj(f(G)),
// over the full charge box, with f the forward transform / N of a real field
// (density, V_xc or the Veff response).  w is formed once per species
// (radial_weight_kernel); the per-atom sums run as (chunk, atom) blocks that
// write partials, reduced over chunks in a fixed order, so results do not
// depend on scheduling.
#include <algorithm>
#include <cmath>

#include "context.h"
#include "grid.cuh"

namespace hb {

Grid3 charge_grid(const Context& ctx);   // setup.cu

namespace {

constexpr int kThreads = 256;

// Sum four per-thread values over a 256-thread block; thread 0 gets the totals.
__device__ void block_sum4(double v[4]) {
  __shared__ double red[kThreads / 32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = 0; c < 4; ++c)
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  if (lane == 0)
    for (int c = 0; c < 4; ++c) red[warp][c] = v[c];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int c = 0; c < 4; ++c) {
      double t = 0;
      for (int w = 0; w < kThreads / 32; ++w) t += red[w][c];
      v[c] = t;
    }
  }
}

// w(G) = scale * radial(|G|) * conj(f(G)) where the reference includes G, else 0.
// radial = spline(table) (minus 4 pi Z e^2 / G^2 for the local part); G = 0
// and |G| > gmax - cut_points * gmax / nrad are excluded.
__global__ void radial_weight_kernel(const double2* f, double2* w, const double* y, const double* m2, int nrad,
                                     double gmax, int cut_points, int coulomb, double zval, double scale, Grid3 g) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.size()) return;
  double qx, qy, qz;
  gvector(i, g, qx, qy, qz);
  const double g2 = qx * qx + qy * qy + qz * qz;
  double2 out = make_double2(0.0, 0.0);
  if (g2 > 1.0e-12) {
    const double gn = sqrt(g2);
    if (gn <= gmax - cut_points * gmax / nrad) {
      double radial = spline_eval(y, m2, nrad, gmax, gn);
      if (coulomb) radial -= 4 * kPi * zval * kFelect / g2;
      const double a = radial * scale;
      const double2 fv = f[i];
      out = make_double2(a * fv.x, -a * fv.y);
    }
  }
  w[i] = out;
}

// Block (c, a): box points [c*chunk, (c+1)*chunk) against atom a at cartesian
// pos[3a..3a+2]; part[(a * nchunk + c) * 4 + {x, y, z, energy}].
__global__ void phase_sum_kernel(const double2* w, Grid3 g, const double* pos, long long chunk, double* part) {
  const int c = blockIdx.x, a = blockIdx.y;
  const double rx = pos[3 * a], ry = pos[3 * a + 1], rz = pos[3 * a + 2];
  const long long n = g.size();
  const long long begin = c * chunk, end = min(n, begin + chunk);
  double v[4] = {0, 0, 0, 0};
  for (long long i = begin + threadIdx.x; i < end; i += blockDim.x) {
    const double2 wv = w[i];
    if (wv.x == 0.0 && wv.y == 0.0) continue;
    double qx, qy, qz;
    gvector(i, g, qx, qy, qz);
    double sn, cs;
    sincos(qx * rx + qy * ry + qz * rz, &sn, &cs);
    const double im = wv.y * cs - wv.x * sn;   // Im(w e^{-i phase})
    v[0] -= qx * im;
    v[1] -= qy * im;
    v[2] -= qz * im;
    v[3] += wv.x * cs + wv.y * sn;             // Re(w e^{-i phase})
  }
  block_sum4(v);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) part[((long long)a * gridDim.x + c) * 4 + k] = v[k];
}

// out[a * 4 + k] = sum over chunks (in chunk order) of part.
__global__ void reduce_chunks_kernel(const double* part, int nchunk, int natoms, double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= natoms * 4) return;
  const int a = t / 4, k = t - a * 4;
  double s = 0;
  for (int c = 0; c < nchunk; ++c) s += part[((long long)a * nchunk + c) * 4 + k];
  out[t] = s;
}

__global__ void harris_densities_kernel(const double* in_c, const double* out_c, double* plus, double* minus,
                                        long long n, double t) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double d = out_c[i] - in_c[i];
  plus[i] = in_c[i] + t * d;
  minus[i] = in_c[i] - t * d;
}

__global__ void central_difference_kernel(const double* vplus, const double* vminus, double* out, long long n,
                                          double t) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = (vplus[i] - vminus[i]) / (2 * t);
}

// ------------------------------------------------------------------ Ewald

struct Cell {
  double lat[9];   // rows a_i
  double rec[9];   // rows b_i
};

// Real-space sum for ion i = blockIdx.x over all (j, image) pairs within rcut:
// part[i*4 + {0,1,2}] = felect z_i sum z_j screen(d) d, part[i*4+3] = z_i sum z_j erfc(alpha d)/d.
__global__ void ewald_real_kernel(const double* pos, const double* z, int nions, Cell cell, int rb, double alpha,
                                  double rcut, double* part) {
  const int i = blockIdx.x;
  const int side = 2 * rb + 1;
  const long long nimg = (long long)side * side * side;
  const long long total = nimg * nions;
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
  double v[4] = {0, 0, 0, 0};
  for (long long t = threadIdx.x; t < total; t += blockDim.x) {
    const int j = int(t / nimg);
    const long long im = t - (long long)j * nimg;
    const int n1 = int(im / (side * side)) - rb;
    const int n2 = int((im / side) % side) - rb;
    const int n3 = int(im % side) - rb;
    const double dx = xi - pos[3 * j] + n1 * cell.lat[0] + n2 * cell.lat[3] + n3 * cell.lat[6];
    const double dy = yi - pos[3 * j + 1] + n1 * cell.lat[1] + n2 * cell.lat[4] + n3 * cell.lat[7];
    const double dz = zi - pos[3 * j + 2] + n1 * cell.lat[2] + n2 * cell.lat[5] + n3 * cell.lat[8];
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    if (dist > 1.0e-13 && dist <= rcut) {
      const double ec = erfc(alpha * dist);
      const double ad = alpha * dist;
      const double screen = ec / (dist * dist * dist) + 2 * alpha * exp(-ad * ad) / (sqrt(kPi) * dist * dist);
      v[0] += z[j] * screen * dx;
      v[1] += z[j] * screen * dy;
      v[2] += z[j] * screen * dz;
      v[3] += z[j] * ec / dist;
    }
  }
  block_sum4(v);
  if (threadIdx.x == 0) {
    part[4 * i + 0] = kFelect * z[i] * v[0];
    part[4 * i + 1] = kFelect * z[i] * v[1];
    part[4 * i + 2] = kFelect * z[i] * v[2];
    part[4 * i + 3] = z[i] * v[3];
  }
}

__device__ __forceinline__ void ewald_gvec(long long t, int gb, const Cell& cell, double& gx, double& gy, double& gz) {
  const int side = 2 * gb + 1;
  const int n1 = int(t / (side * side)) - gb;
  const int n2 = int((t / side) % side) - gb;
  const int n3 = int(t % side) - gb;
  gx = n1 * cell.rec[0] + n2 * cell.rec[3] + n3 * cell.rec[6];
  gy = n1 * cell.rec[1] + n2 * cell.rec[4] + n3 * cell.rec[7];
  gz = n1 * cell.rec[2] + n2 * cell.rec[5] + n3 * cell.rec[8];
}

// Structure factor S(G) = sum_j z_j e^{-i G.R_j} and exp(-G^2/4alpha^2)/G^2 on the
// reciprocal images within gcut (pref 0 elsewhere).
__global__ void ewald_structure_kernel(const double* pos, const double* z, int nions, Cell cell, int gb, double alpha,
                                       double gcut, double2* sf, double* pref) {
  const int side = 2 * gb + 1;
  const long long ng = (long long)side * side * side;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= ng) return;
  double gx, gy, gz;
  ewald_gvec(t, gb, cell, gx, gy, gz);
  const double gn = sqrt(gx * gx + gy * gy + gz * gz);
  double sr = 0, si = 0, p = 0;
  if (gn > 1.0e-13 && gn <= gcut) {
    for (int j = 0; j < nions; ++j) {
      double sn, cs;
      sincos(gx * pos[3 * j] + gy * pos[3 * j + 1] + gz * pos[3 * j + 2], &sn, &cs);
      sr += z[j] * cs;
      si -= z[j] * sn;
    }
    p = exp(-gn * gn / (4 * alpha * alpha)) / (gn * gn);
  }
  sf[t] = make_double2(sr, si);
  pref[t] = p;
}

// Blocks i < nions: reciprocal force on ion i (x 4 pi felect / Omega);
// block nions: the reciprocal energy sum (x 2 pi felect / Omega).
__global__ void ewald_recip_kernel(const double* pos, const double* z, int nions, Cell cell, int gb,
                                   const double2* sf, const double* pref, double volume, double* part) {
  const int i = blockIdx.x;
  const int side = 2 * gb + 1;
  const long long ng = (long long)side * side * side;
  double v[4] = {0, 0, 0, 0};
  for (long long t = threadIdx.x; t < ng; t += blockDim.x) {
    const double p = pref[t];
    if (p == 0.0) continue;
    const double2 s = sf[t];
    if (i == nions) {
      v[3] += p * (s.x * s.x + s.y * s.y);
      continue;
    }
    double gx, gy, gz;
    ewald_gvec(t, gb, cell, gx, gy, gz);
    double sn, cs;
    sincos(gx * pos[3 * i] + gy * pos[3 * i + 1] + gz * pos[3 * i + 2], &sn, &cs);
    const double w = p * z[i] * (s.x * sn + s.y * cs);
    v[0] += w * gx;
    v[1] += w * gy;
    v[2] += w * gz;
  }
  block_sum4(v);
  if (threadIdx.x == 0) {
    const double f = 4 * kPi * kFelect / volume;
    part[4 * i + 0] = f * v[0];
    part[4 * i + 1] = f * v[1];
    part[4 * i + 2] = f * v[2];
    part[4 * i + 3] = 2 * kPi * kFelect / volume * v[3];
  }
}

// Smallest singular value of a 3x3 matrix (rows m[0..2], m[3..5], m[6..8]):
// square root of the smallest eigenvalue of M M^T, by the closed-form
// trigonometric solution of the symmetric 3x3 characteristic cubic.
double smallest_singular(const double* m) {
  double a[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) a[r][c] = m[3 * r] * m[3 * c] + m[3 * r + 1] * m[3 * c + 1] + m[3 * r + 2] * m[3 * c + 2];
  const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
  double lo;
  if (off == 0.0) {
    lo = std::min(a[0][0], std::min(a[1][1], a[2][2]));
  } else {
    const double q = (a[0][0] + a[1][1] + a[2][2]) / 3;
    const double p2 = (a[0][0] - q) * (a[0][0] - q) + (a[1][1] - q) * (a[1][1] - q) + (a[2][2] - q) * (a[2][2] - q) +
                      2 * off;
    const double p = std::sqrt(p2 / 6);
    double b[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) b[r][c] = (a[r][c] - (r == c ? q : 0.0)) / p;
    const double det = b[0][0] * (b[1][1] * b[2][2] - b[1][2] * b[2][1]) -
                       b[0][1] * (b[1][0] * b[2][2] - b[1][2] * b[2][0]) +
                       b[0][2] * (b[1][0] * b[2][1] - b[1][1] * b[2][0]);
    const double hr = std::max(-1.0, std::min(1.0, det / 2));
    const double phi = std::acos(hr) / 3;
    lo = q + 2 * p * std::cos(phi + 2 * kPi / 3);   // the smallest of the three roots
  }
  return std::sqrt(std::max(0.0, lo));
}

void ewald_device(Context& ctx, cudaStream_t s, IonicForces& out) {
  const Crystal& c = ctx.crystal;
  const int nions = c.nions();
  const double volume = c.volume();
  const double tol = 1.0e-11;
  const double alpha = std::sqrt(kPi) / std::cbrt(volume);
  const double scale = std::sqrt(-std::log(tol));
  const double rcut = scale / alpha, gcut = 2 * alpha * scale;
  Cell cell{};
  auto rec = c.reciprocal();
  for (int k = 0; k < 9; ++k) {
    cell.lat[k] = c.lattice[k];
    cell.rec[k] = rec[k];
  }
  const int rb = int(std::ceil(rcut / smallest_singular(cell.lat))) + 1;
  const int gb = int(std::ceil(gcut / smallest_singular(cell.rec))) + 1;
  std::vector<double> pos, z;
  int ion = 0;
  for (size_t it = 0; it < ctx.pots.size(); ++it)
    for (int a = 0; a < c.counts[it]; ++a, ++ion) {
      auto r = c.cartesian(ion);
      pos.insert(pos.end(), r.begin(), r.end());
      z.push_back(ctx.pots[it].zval);
    }
  const long long ng = (long long)(2 * gb + 1) * (2 * gb + 1) * (2 * gb + 1);
  DeviceBuffer<double> dpos, dz, real_part(4 * (size_t)nions), recip_part(4 * (size_t)(nions + 1)), pref(ng);
  DeviceBuffer<double2> sf(ng);
  dpos.upload(pos, s);
  dz.upload(z, s);
  ewald_real_kernel<<<nions, kThreads, 0, s>>>(dpos.get(), dz.get(), nions, cell, rb, alpha, rcut, real_part.get());
  HALF_LAUNCH("ewald real");
  ewald_structure_kernel<<<blocks_for(ng), kThreads, 0, s>>>(dpos.get(), dz.get(), nions, cell, gb, alpha, gcut,
                                                              sf.get(), pref.get());
  HALF_LAUNCH("ewald structure");
  ewald_recip_kernel<<<nions + 1, kThreads, 0, s>>>(dpos.get(), dz.get(), nions, cell, gb, sf.get(), pref.get(),
                                                     volume, recip_part.get());
  HALF_LAUNCH("ewald reciprocal");
  const std::vector<double> rp = real_part.download(s), gp = recip_part.download(s);
  double re = 0, zz = 0, zsum = 0;
  out.ewald.assign(3 * (size_t)nions, 0.0);
  for (int i = 0; i < nions; ++i) {
    re += rp[4 * i + 3];
    zz += z[i] * z[i];
    zsum += z[i];
    for (int k = 0; k < 3; ++k) out.ewald[3 * i + k] = rp[4 * i + k] + gp[4 * i + k];
  }
  re *= 0.5 * kFelect;
  const double ge = gp[4 * nions + 3];
  const double se = -kFelect * alpha / std::sqrt(kPi) * zz;
  const double be = -kFelect * kPi * zsum * zsum / (2 * alpha * alpha * volume);
  out.ewald_energy[0] = re + ge + se + be;
  out.ewald_energy[1] = re;
  out.ewald_energy[2] = ge;
  out.ewald_energy[3] = se;
  out.ewald_energy[4] = be;
}

// The reciprocal-space contraction of the file header for every species
// with a table (local: psp_local with the Coulomb tail, 1/Omega, one grid
// point trimmed; core: pspcor, three points trimmed).  forces: nions*3.
void radial_forces(Context& ctx, cudaStream_t s, const double2* field_g, bool local, std::vector<double>& forces,
                   double* energy) {
  const Grid3 g = charge_grid(ctx);
  const long long n = g.size();
  const int nions = ctx.crystal.nions();
  forces.assign(3 * (size_t)nions, 0.0);
  double etotal = 0;
  DeviceBuffer<double2> w(n);
  int ion0 = 0;
  for (size_t it = 0; it < ctx.pots.size(); ++it) {
    const Potcar& p = ctx.pots[it];
    const int nat = ctx.crystal.counts[it];
    const std::vector<double>& table = local ? p.psp_local : p.pspcor;
    if (nat == 0 || table.empty()) {
      ion0 += nat;
      continue;
    }
    const int nrad = int(table.size());
    DeviceBuffer<double> dy, dm2, dpos;
    dy.upload(table, s);
    dm2.upload(spline_second(table, p.psp_gmax), s);
    std::vector<double> pos;
    for (int a = 0; a < nat; ++a) {
      auto r = ctx.crystal.cartesian(ion0 + a);
      pos.insert(pos.end(), r.begin(), r.end());
    }
    dpos.upload(pos, s);
    radial_weight_kernel<<<blocks_for(n), kThreads, 0, s>>>(field_g, w.get(), dy.get(), dm2.get(), nrad, p.psp_gmax,
                                                             local ? 1 : 3, local ? 1 : 0, p.zval,
                                                             local ? 1.0 / ctx.crystal.volume() : 1.0, g);
    HALF_LAUNCH("radial weight");
    // enough (chunk, atom) blocks to cover the SMs several times over
    const long long max_chunks = std::max(1LL, (n + kThreads - 1) / kThreads);
    const int nchunk = int(std::min<long long>(max_chunks, std::max(1, (4 * 148 + nat - 1) / nat)));
    const long long chunk = (n + nchunk - 1) / nchunk;
    DeviceBuffer<double> part((size_t)nat * nchunk * 4), sums((size_t)nat * 4);
    phase_sum_kernel<<<dim3(nchunk, nat), kThreads, 0, s>>>(w.get(), g, dpos.get(), chunk, part.get());
    HALF_LAUNCH("phase sum");
    reduce_chunks_kernel<<<blocks_for(4LL * nat), kThreads, 0, s>>>(part.get(), nchunk, nat, sums.get());
    HALF_LAUNCH("reduce chunks");
    const std::vector<double> h = sums.download(s);
    for (int a = 0; a < nat; ++a) {
      for (int k = 0; k < 3; ++k) forces[3 * (ion0 + a) + k] = h[4 * a + k];
      etotal += h[4 * a + 3];
    }
    ion0 += nat;
  }
  if (energy) *energy = etotal;
}

bool any_core(const Context& ctx) {
  for (const Potcar& p : ctx.pots)
    if (p.has_core()) return true;
  return false;
}

}  // namespace

void ionic_forces_device(Context& ctx, const double* output_f, bool output_on_device, bool want_ewald,
                         bool want_local, bool want_nlcc, bool want_harris, IonicForces& out) {
  cudaStream_t s = ctx.rt->stream;
  const auto& sh = ctx.charge.shape;
  const long long n = ctx.nr();
  const int nions = ctx.crystal.nions();
  DeviceBuffer<double> raw(n), in_c(n), out_c;
  DeviceBuffer<double2> freq(n);
  raw.upload(ctx.charge.values, s);
  density_to_c_order(raw.get(), in_c.get(), sh, s);
  const double* outc = in_c.get();
  if (output_f) {
    out_c.resize(n);
    const double* src = output_f;
    if (!output_on_device) {
      HALF_CUDA(cudaMemcpyAsync(raw.get(), output_f, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      src = raw.get();
    }
    density_to_c_order(src, out_c.get(), sh, s);
    outc = out_c.get();
  }
  if (want_local) {
    forward_transform(outc, freq.get(), sh, s);
    radial_forces(ctx, s, freq.get(), true, out.local, &out.local_energy);
  }
  const bool core = any_core(ctx);
  if (want_nlcc) {
    if (core) {
      DeviceBuffer<double> veff(n), vxc(n);
      build_potential(ctx, s, in_c.get(), veff.get(), vxc.get());
      forward_transform(vxc.get(), freq.get(), sh, s);
      radial_forces(ctx, s, freq.get(), false, out.nlcc, nullptr);
    } else {
      out.nlcc.assign(3 * (size_t)nions, 0.0);
    }
  }
  if (want_harris) {
    if (core && output_f) {
      const double t = 1.0e-4;
      DeviceBuffer<double> plus(n), minus(n), veff(n), vplus(n), vminus(n);
      harris_densities_kernel<<<blocks_for(n), kThreads, 0, s>>>(in_c.get(), outc, plus.get(), minus.get(), n, t);
      HALF_LAUNCH("harris densities");
      build_potential(ctx, s, plus.get(), veff.get(), vplus.get());
      build_potential(ctx, s, minus.get(), veff.get(), vminus.get());
      central_difference_kernel<<<blocks_for(n), kThreads, 0, s>>>(vplus.get(), vminus.get(), veff.get(), n, t);
      HALF_LAUNCH("harris response");
      forward_transform(veff.get(), freq.get(), sh, s);
      radial_forces(ctx, s, freq.get(), false, out.harris, nullptr);
    } else {
      // no partial core, or no density change: the response has nothing to act on
      out.harris.assign(3 * (size_t)nions, 0.0);
    }
  }
  if (want_ewald) ewald_device(ctx, s, out);
  HALF_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hb
