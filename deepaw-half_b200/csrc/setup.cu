// Context set-up on the device: the fixed-density effective potential and
// the MIMIC_US QDEP correction D_ij^I with its position derivative.
//
// * Veff restates the ACC path's builder src/half_cuda_potential.cuf:270-350
//   (Hartree + ionic local part in reciprocal space, PZ81 LDA or PBE with
//   spectral gradients and finite-difference functional derivatives).
// * D_ij^I and dD_ij^I/dR restate src/half_uspp.F90:112-241 (the CPU variant,
//   which also provides dD/dR and symmetrises both); the GPU D-only variant
//   src/half_cuda_uspp.cuf:124-195 is the same algorithm without symmetrising.
// All full-box transforms use the library's own shared-memory FFT engine.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>

#include "context.h"
#include "grid.cuh"

namespace hb {

// ------------------------------------------------------------------ runtime

Runtime::Runtime() {
  HALF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  cublas_check(cublasCreate(&blas), "create");
  cublas_check(cublasSetStream(blas, stream), "set stream");
  cusolver_check(cusolverDnCreate(&solver), "create");
  cusolver_check(cusolverDnSetStream(solver, stream), "set stream");
  int v = 0;
  cublasGetVersion(blas, &v);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  // FP32 emulation on BF16 tensor cores: cuBLAS >= 12.9 on compute capability 10.x.
  // The math mode only affects FP32 routines, i.e. the mixed-precision GEMMs.
  bf16x9 = (v >= 120900) && prop.major == 10;
  if (bf16x9 && cublasSetMathMode(blas, CUBLAS_FP32_EMULATED_BF16X9_MATH) != CUBLAS_STATUS_SUCCESS) bf16x9 = false;
  HALF_CUDA(cudaEventCreate(&prof.a));
  HALF_CUDA(cudaEventCreate(&prof.b));
  if (const char* tg = std::getenv("HALF_TC_GEMM")) tc_gemm = std::string(tg) != "0";
}

int Profile::record(cudaStream_t s) {
  if (used == pool.size()) {
    cudaEvent_t e = nullptr;
    HALF_CUDA(cudaEventCreate(&e));
    pool.push_back(e);
  }
  HALF_CUDA(cudaEventRecord(pool[used], s));
  return int(used++);
}

void Profile::collect() {
  for (const auto& sp : spans) {
    float ms = 0;
    HALF_CUDA(cudaEventElapsedTime(&ms, pool[sp.second.first], pool[sp.second.second]));
    if (sp.first == kLocal) local_ms += ms;
    else if (sp.first == kSweep) sweep_ms += ms;
    else if (sp.first == kTensor) tensor_ms += ms;
    else adjoint_ms += ms;
  }
  spans.clear();
  used = 0;
}

void Profile::destroy() {
  for (cudaEvent_t e : pool)
    if (e) cudaEventDestroy(e);
  pool.clear();
  for (cudaEvent_t e : {a, b})
    if (e) cudaEventDestroy(e);
  a = b = nullptr;
}

Runtime::~Runtime() {
  prof.destroy();
  if (solver) cusolverDnDestroy(solver);
  if (blas) cublasDestroy(blas);
  if (stream) cudaStreamDestroy(stream);
}

// ------------------------------------------------------------------ 3-D FFT

namespace {

constexpr int kTile = 16;   // pencils per block for strided axes

// FFT along the contiguous axis (i3): each block transforms `rows` pencils.
template <typename C, typename R>
__global__ void fft_rows_kernel(C* data, long long npencils, AxisPlan ap, int sign) {
  extern __shared__ unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int n = ap.plan.n;
  C* buf = tw + kMaxFFT;
  fill_twiddles(tw, n);
  const long long p0 = (long long)blockIdx.x * kTile;
  const int np = int(min((long long)kTile, npencils - p0));
  for (int t = threadIdx.x; t < np * n; t += blockDim.x) buf[t] = data[p0 * n + t];
  __syncthreads();
  fft_pencils<false, C, R>(buf, np, n, 1, ap.plan, tw, sign);
  for (int t = threadIdx.x; t < np * n; t += blockDim.x) {
    int p = t / n, k = t - p * n;
    data[(p0 + p) * n + k] = buf[p * n + ap.pos[k]];
  }
}

// FFT along a strided axis: pencil (o, c) starts at o*outer_stride + c and
// steps by axis_stride; a block takes kTile consecutive c (coalesced).
template <typename C, typename R>
__global__ void fft_strided_kernel(C* data, int ncols, long long axis_stride, long long outer_stride, AxisPlan ap,
                                   int sign) {
  extern __shared__ unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int n = ap.plan.n;
  C* buf = tw + kMaxFFT;   // [k][tz]
  fill_twiddles(tw, n);
  const int c0 = blockIdx.x * kTile;
  const int nc = min(kTile, ncols - c0);
  const long long base = (long long)blockIdx.y * outer_stride + c0;
  for (int t = threadIdx.x; t < n * kTile; t += blockDim.x) {
    int k = t / kTile, c = t - k * kTile;
    if (c < nc) buf[t] = data[base + k * axis_stride + c];
    else buf[t] = cmake(R(0), R(0));
  }
  __syncthreads();
  fft_pencils<false, C, R>(buf, kTile, 1, kTile, ap.plan, tw, sign);
  for (int t = threadIdx.x; t < n * kTile; t += blockDim.x) {
    int k = t / kTile, c = t - k * kTile;
    if (c < nc) data[base + k * axis_stride + c] = buf[ap.pos[k] * kTile + c];
  }
}

}  // namespace

void fft3d_inplace(double2* data, const std::array<int, 3>& shape, int sign, cudaStream_t s) {
  const int n1 = shape[0], n2 = shape[1], n3 = shape[2];
  AxisPlan a1 = make_axis_plan(n1), a2 = make_axis_plan(n2), a3 = make_axis_plan(n3);
  const long long rows = (long long)n1 * n2;
  size_t sm3 = (kMaxFFT + size_t(kTile) * n3) * sizeof(double2);
  fft_rows_kernel<double2, double><<<ceil_div(rows, kTile), 256, sm3, s>>>(data, rows, a3, sign);
  HALF_LAUNCH("fft rows");
  size_t sm2 = (kMaxFFT + size_t(kTile) * n2) * sizeof(double2);
  fft_strided_kernel<double2, double><<<dim3(ceil_div(n3, kTile), n1), 256, sm2, s>>>(data, n3, n3, (long long)n2 * n3,
                                                                                       a2, sign);
  HALF_LAUNCH("fft axis 2");
  size_t sm1 = (kMaxFFT + size_t(kTile) * n1) * sizeof(double2);
  fft_strided_kernel<double2, double><<<dim3(ceil_div((long long)n2 * n3, kTile), 1), 256, sm1, s>>>(
      data, n2 * n3, (long long)n2 * n3, 0, a1, sign);
  HALF_LAUNCH("fft axis 1");
}

// ------------------------------------------------------------------ Veff

namespace {

__global__ void reorder_f_to_c_kernel(const double* in, double* out, int n1, int n2, int n3) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long n = (long long)n1 * n2 * n3;
  if (i >= n) return;
  int i3 = int(i % n3);
  long long t = i / n3;
  int i2 = int(t % n2), i1 = int(t / n2);
  out[i] = in[i1 + (long long)n1 * (i2 + (long long)n2 * i3)];
}

__global__ void real_to_complex_kernel(const double* in, double2* out, long long n, double scale) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_double2(in[i] * scale, 0.0);
}

__global__ void hartree_kernel(const double2* rho_g, double2* local_g, double2* core_g, Grid3 g, double volume) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long n = (long long)g.n1 * g.n2 * g.n3;
  if (i >= n) return;
  double qx, qy, qz;
  gvector(i, g, qx, qy, qz);
  double g2 = qx * qx + qy * qy + qz * qz;
  double2 v = make_double2(0, 0);
  if (g2 > 1.0e-12) v = cscale(rho_g[i], kEdeps / (g2 * volume));
  local_g[i] = v;
  core_g[i] = make_double2(0, 0);
}

__global__ void ionic_species_kernel(double2* local_g, double2* core_g, const double* y, const double* m2,
                                     const double* cy, const double* cm2, int nrad, double gmax, double zval,
                                     const double* pos, int natoms, Grid3 g, double volume, int has_core) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long n = (long long)g.n1 * g.n2 * g.n3;
  if (i >= n) return;
  double qx, qy, qz;
  gvector(i, g, qx, qy, qz);
  double g2 = qx * qx + qy * qy + qz * qz, gn = sqrt(g2);
  double radial = spline_eval(y, m2, nrad, gmax, gn);
  if (g2 > 1.0e-12) radial -= 4 * kPi * zval * kFelect / g2;
  if (g2 <= 1.0e-12 || gn > gmax - gmax / nrad) radial = 0;
  double core = 0;
  if (has_core && gn <= gmax - 3 * gmax / nrad) core = spline_eval(cy, cm2, nrad, gmax, gn);
  double sr = 0, si = 0;
  for (int a = 0; a < natoms; ++a) {
    double ph = qx * pos[3 * a] + qy * pos[3 * a + 1] + qz * pos[3 * a + 2];
    double s, c;
    sincos(ph, &s, &c);
    sr += c;
    si -= s;
  }
  double2 l = local_g[i], cg = core_g[i];
  l.x += radial * sr / volume;
  l.y += radial * si / volume;
  cg.x += core * sr;
  cg.y += core * si;
  local_g[i] = l;
  core_g[i] = cg;
}

__global__ void extract_real_kernel(const double2* in, double* out, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i].x;
}

// PZ81 LDA (src/half_cuda_potential.cuf:236-259); vxc in eV.
__global__ void lda_kernel(const double* charge, const double* core, const double* local_r, double* veff,
                           double* vxc, long long n, double volume) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double density = (charge[i] + core[i]) / volume;
  double rhoau = density * kAutoa * kAutoa * kAutoa;
  if (rhoau <= 1.0e-30) {
    veff[i] = local_r[i];
    vxc[i] = 0.0;
    return;
  }
  double rs = cbrt(3.0 / (4 * kPi * rhoau));
  double vx = -(4.0 / 3.0) * 0.4582 / rs, vc;
  if (rs >= 1) {
    double sr = sqrt(rs), denom = 1 + 1.0529 * sr + 0.3334 * rs;
    double ec = -0.1423 / denom;
    vc = ec * (1 + (7.0 / 6.0) * 1.0529 * sr + (4.0 / 3.0) * 0.3334 * rs) / denom;
  } else {
    double lnrs = log(rs);
    vc = 0.0311 * lnrs + (-0.048 - 0.0311 / 3) + (2.0 / 3.0) * 0.002 * rs * lnrs + (-0.0232 - 0.002) * rs / 3;
  }
  const double v = (vx + vc) * kHatoev;
  vxc[i] = v;
  veff[i] = local_r[i] + v;
}

__device__ double pw92_ec(double rs) {
  const double a = .031091, a1 = .21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = .49294;
  double sr = sqrt(rs);
  double q = 2 * a * (b1 * sr + b2 * rs + b3 * rs * sr + b4 * rs * rs);
  return -2 * a * (1 + a1 * rs) * log(1 + 1 / q);
}

// PBE energy density per volume (src/half_xc.F90:94-107)
__device__ double pbe_energy_density(double density, double sigma) {
  const double mu = 0.2195149727645171, kappa = 0.804, beta = 0.06672455060314922;
  const double gamma = (1.0 - 0.69314718055994530942) / (kPi * kPi);
  double n = fmax(density, 1.0e-30), s = fmax(sigma, 0.0);
  double rs = cbrt(3 / (4 * kPi * n));
  double kf = cbrt(3 * kPi * kPi * n);
  double exlda = -3 * kf / (4 * kPi);
  double s2 = s / (4 * kf * kf * n * n);
  double fx = 1 + kappa - kappa / (1 + mu * s2 / kappa);
  double ec = pw92_ec(rs);
  double ks2 = 4 * kf / kPi;
  double t2 = s / (4 * ks2 * n * n);
  double aa = beta / gamma / (exp(-ec / gamma) - 1);
  double at2 = aa * t2, ratio;
  if (t2 == 0) ratio = 0;
  else if (at2 < 1.0e100) ratio = t2 * (1 + at2) / (1 + at2 + at2 * at2);
  else { double iv = 1 / at2; ratio = (1 / aa) * (1 + iv) / (1 + iv + iv * iv); }
  double hh = gamma * log(1 + beta / gamma * ratio);
  return n * (exlda * fx + ec + hh);
}

__global__ void pbe_density_kernel(const double* charge, const double* core, double* density, double2* work,
                                   long long n, double volume) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double total = charge[i] + core[i];
  density[i] = fmax(total / volume * kAutoa * kAutoa * kAutoa, 1.0e-20);
  work[i] = make_double2(total / volume, 0.0);
}

__global__ void spectral_derivative_kernel(const double2* freq, double2* deriv, Grid3 g, int alpha) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long n = (long long)g.n1 * g.n2 * g.n3;
  if (i >= n) return;
  double qx, qy, qz;
  gvector(i, g, qx, qy, qz);
  double q = alpha == 0 ? qx : (alpha == 1 ? qy : qz);
  double2 f = freq[i];
  deriv[i] = make_double2(-q * f.y, q * f.x);
}

__global__ void accumulate_gradient_kernel(const double2* work, double* grad, double* sigma, long long n, int alpha) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a4 = kAutoa * kAutoa * kAutoa * kAutoa;
  double gv = work[i].x / double(n) * a4;
  grad[alpha * n + i] = gv;
  sigma[i] = (alpha == 0 ? 0.0 : sigma[i]) + gv * gv;
}

__global__ void pbe_eval_kernel(const double* density, const double* sigma, double* fn, double* fs, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double d = density[i], s = sigma[i];
  double dn = fmax(fabs(d) * 2.0e-5, 1.0e-12), nm = fmax(d - dn, 1.0e-30), np = d + dn;
  fn[i] = (pbe_energy_density(np, s) - pbe_energy_density(nm, s)) / (np - nm);
  double ds = fmax(fabs(s) * 2.0e-5, 1.0e-14), sm = fmax(s - ds, 0.0), sp = s + ds;
  double f = (pbe_energy_density(d, sp) - pbe_energy_density(d, sm)) / (sp - sm);
  fs[i] = d <= 1.0e-20 ? 0.0 : f;
}

__global__ void flux_kernel(const double* fs, const double* grad, double2* work, long long n, int alpha) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) work[i] = make_double2(2 * fs[i] * grad[alpha * n + i], 0.0);
}

__global__ void subtract_divergence_kernel(const double2* work, double* fn, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) fn[i] -= kAutoa * work[i].x / double(n);
}

__global__ void finish_pbe_kernel(const double* density, const double* local_r, const double* fn, double* veff,
                                  double* vxc, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = (density[i] <= 1.0e-20 ? 0.0 : fn[i]) * kHatoev;
  vxc[i] = v;
  veff[i] = local_r[i] + v;
}

}  // namespace

Grid3 charge_grid(const Context& ctx) {
  const auto& sh = ctx.charge.shape;
  Grid3 g{sh[0], sh[1], sh[2], {}};
  auto rec = ctx.crystal.reciprocal();
  for (int i = 0; i < 9; ++i) g.rec[i] = rec[i];
  return g;
}

void density_to_c_order(const double* f_order, double* c_order, const std::array<int, 3>& shape, cudaStream_t s) {
  const long long n = (long long)shape[0] * shape[1] * shape[2];
  reorder_f_to_c_kernel<<<blocks_for(n), 256, 0, s>>>(f_order, c_order, shape[0], shape[1], shape[2]);
  HALF_LAUNCH("reorder density");
}

void forward_transform(const double* real_c, double2* freq, const std::array<int, 3>& shape, cudaStream_t s) {
  const long long n = (long long)shape[0] * shape[1] * shape[2];
  real_to_complex_kernel<<<blocks_for(n), 256, 0, s>>>(real_c, freq, n, 1.0 / double(n));
  HALF_LAUNCH("real to complex");
  fft3d_inplace(freq, shape, -1, s);
}

void build_potential(Context& ctx, cudaStream_t s, const double* charge, double* veff_out, double* vxc_out) {
  const auto& sh = ctx.charge.shape;
  const long long n = ctx.nr();
  const Grid3 g = charge_grid(ctx);
  const double vol = ctx.crystal.volume();
  DeviceBuffer<double> local_r(n), core_r(n), vxc_scratch;
  double* vxc = vxc_out;
  if (!vxc) {
    vxc_scratch.resize(n);
    vxc = vxc_scratch.get();
  }
  DeviceBuffer<double2> work(n), rho_g(n), local_g(n), core_g(n);
  real_to_complex_kernel<<<blocks_for(n), 256, 0, s>>>(charge, rho_g.get(), n, 1.0 / double(n));
  fft3d_inplace(rho_g.get(), sh, -1, s);
  hartree_kernel<<<blocks_for(n), 256, 0, s>>>(rho_g.get(), local_g.get(), core_g.get(), g, vol);
  HALF_LAUNCH("hartree");
  int ion0 = 0;
  std::vector<DeviceBuffer<double>> keep;
  for (size_t it = 0; it < ctx.pots.size(); ++it) {
    const Potcar& p = ctx.pots[it];
    int nat = ctx.crystal.counts[it];
    auto m2 = spline_second(p.psp_local, p.psp_gmax);
    std::vector<double> cy(p.psp_local.size(), 0.0), cm2(p.psp_local.size(), 0.0);
    if (p.has_core()) { cy = p.pspcor; cm2 = spline_second(p.pspcor, p.psp_gmax); }
    std::vector<double> pos;
    for (int a = 0; a < nat; ++a) {
      auto r = ctx.crystal.cartesian(ion0 + a);
      pos.insert(pos.end(), r.begin(), r.end());
    }
    keep.emplace_back(); keep.back().upload(p.psp_local, s);
    const double* dy = keep.back().get();
    keep.emplace_back(); keep.back().upload(m2, s);
    const double* dm2 = keep.back().get();
    keep.emplace_back(); keep.back().upload(cy, s);
    const double* dcy = keep.back().get();
    keep.emplace_back(); keep.back().upload(cm2, s);
    const double* dcm2 = keep.back().get();
    keep.emplace_back(); keep.back().upload(pos, s);
    const double* dpos = keep.back().get();
    ionic_species_kernel<<<blocks_for(n), 256, 0, s>>>(local_g.get(), core_g.get(), dy, dm2, dcy, dcm2,
                                                        int(p.psp_local.size()), p.psp_gmax, p.zval, dpos, nat, g, vol,
                                                        p.has_core() ? 1 : 0);
    HALF_LAUNCH("ionic species");
    ion0 += nat;
  }
  fft3d_inplace(local_g.get(), sh, +1, s);
  extract_real_kernel<<<blocks_for(n), 256, 0, s>>>(local_g.get(), local_r.get(), n);
  fft3d_inplace(core_g.get(), sh, +1, s);
  extract_real_kernel<<<blocks_for(n), 256, 0, s>>>(core_g.get(), core_r.get(), n);
  if (!ctx.use_pbe) {
    lda_kernel<<<blocks_for(n), 256, 0, s>>>(charge, core_r.get(), local_r.get(), veff_out, vxc, n, vol);
    HALF_LAUNCH("lda");
  } else {
    DeviceBuffer<double> density(n), sigma(n), grad(3 * n), fn(n), fs(n);
    DeviceBuffer<double2> freq(n), deriv(n);
    pbe_density_kernel<<<blocks_for(n), 256, 0, s>>>(charge, core_r.get(), density.get(), freq.get(), n, vol);
    fft3d_inplace(freq.get(), sh, -1, s);
    for (int a = 0; a < 3; ++a) {
      spectral_derivative_kernel<<<blocks_for(n), 256, 0, s>>>(freq.get(), deriv.get(), g, a);
      fft3d_inplace(deriv.get(), sh, +1, s);
      accumulate_gradient_kernel<<<blocks_for(n), 256, 0, s>>>(deriv.get(), grad.get(), sigma.get(), n, a);
    }
    pbe_eval_kernel<<<blocks_for(n), 256, 0, s>>>(density.get(), sigma.get(), fn.get(), fs.get(), n);
    for (int a = 0; a < 3; ++a) {
      flux_kernel<<<blocks_for(n), 256, 0, s>>>(fs.get(), grad.get(), work.get(), n, a);
      fft3d_inplace(work.get(), sh, -1, s);
      spectral_derivative_kernel<<<blocks_for(n), 256, 0, s>>>(work.get(), deriv.get(), g, a);
      fft3d_inplace(deriv.get(), sh, +1, s);
      subtract_divergence_kernel<<<blocks_for(n), 256, 0, s>>>(deriv.get(), fn.get(), n);
    }
    finish_pbe_kernel<<<blocks_for(n), 256, 0, s>>>(density.get(), local_r.get(), fn.get(), veff_out, vxc, n);
    HALF_LAUNCH("pbe");
  }
  // the scratch above is released on return: finish its users first
  HALF_CUDA(cudaStreamSynchronize(s));
}

void build_veff_device(Context& ctx) {
  cudaStream_t s = ctx.rt->stream;
  const long long n = ctx.nr();
  DeviceBuffer<double> raw(n), charge(n);
  raw.upload(ctx.charge.values, s);
  density_to_c_order(raw.get(), charge.get(), ctx.charge.shape, s);
  ctx.veff.resize(n);
  build_potential(ctx, s, charge.get(), ctx.veff.get(), nullptr);
}

// ------------------------------------------------------------------ QDEP

namespace {

__global__ void prefilter_kernel(double2* freq, int n1, int n2, int n3) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long n = (long long)n1 * n2 * n3;
  if (i >= n) return;
  int i3 = int(i % n3);
  long long t = i / n3;
  int i2 = int(t % n2), i1 = int(t / n2);
  double b1 = (2.0 + cospi(2.0 * i1 / n1)) / 3.0;
  double b2 = (2.0 + cospi(2.0 * i2 / n2)) / 3.0;
  double b3 = (2.0 + cospi(2.0 * i3 / n3)) / 3.0;
  freq[i] = cscale(freq[i], 1.0 / (b1 * b2 * b3));
}

__global__ void coeff_real_kernel(const double2* in, double* out, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i].x / double(n);
}

__device__ __forceinline__ void cubic_w(double t, double* w) {
  double u = 1 - t;
  w[0] = u * u * u / 6;
  w[1] = (3 * t * t * t - 6 * t * t + 4) / 6;
  w[2] = (-3 * t * t * t + 3 * t * t + 3 * t + 1) / 6;
  w[3] = t * t * t / 6;
}
__device__ __forceinline__ void cubic_dw(double t, double* w) {
  w[0] = -0.5 * (1 - t) * (1 - t);
  w[1] = 1.5 * t * t - 2.0 * t;
  w[2] = -1.5 * t * t + t + 0.5;
  w[3] = 0.5 * t * t;
}

struct SampleGeom {
  int n1, n2, n3;
  double inv[9];   // inverse lattice, row-major
};

// One sample per (atom, radial point, direction): value and Cartesian
// gradient of the cubic B-spline interpolant (src/half_uspp.F90:243-277).
__global__ void sample_kernel(const double* coeff, const double* pos, const double* rgrid, const double* dirs,
                              int natoms, int nrad, int nang, SampleGeom g, int gradient, double* out) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long total = (long long)natoms * nrad * nang;
  if (idx >= total) return;
  int ip = int(idx % nang);
  long long t = idx / nang;
  int ir = int(t % nrad), a = int(t / nrad);
  double cart[3], frac[3];
  for (int j = 0; j < 3; ++j) cart[j] = pos[3 * a + j] + rgrid[ir] * dirs[3 * ip + j];
  for (int j = 0; j < 3; ++j) {
    double f = cart[0] * g.inv[0 * 3 + j] + cart[1] * g.inv[1 * 3 + j] + cart[2] * g.inv[2 * 3 + j];
    frac[j] = f - floor(f);
  }
  int nn[3] = {g.n1, g.n2, g.n3};
  int ix[3];
  double w[3][4], dw[3][4];
  for (int j = 0; j < 3; ++j) {
    double c = frac[j] * nn[j];
    ix[j] = int(floor(c));
    cubic_w(c - ix[j], w[j]);
    cubic_dw(c - ix[j], dw[j]);
  }
  double v = 0, df0 = 0, df1 = 0, df2 = 0;
  for (int p = 0; p < 4; ++p) {
    int ia = ((ix[0] + p - 1) % g.n1 + g.n1) % g.n1;
    for (int q = 0; q < 4; ++q) {
      int ib = ((ix[1] + q - 1) % g.n2 + g.n2) % g.n2;
      const double* row = coeff + ((long long)ia * g.n2 + ib) * g.n3;
      for (int r = 0; r < 4; ++r) {
        int ic = ((ix[2] + r - 1) % g.n3 + g.n3) % g.n3;
        double c = row[ic];
        v += w[0][p] * w[1][q] * w[2][r] * c;
        if (gradient) {
          df0 += dw[0][p] * w[1][q] * w[2][r] * c * g.n1;
          df1 += w[0][p] * dw[1][q] * w[2][r] * c * g.n2;
          df2 += w[0][p] * w[1][q] * dw[2][r] * c * g.n3;
        }
      }
    }
  }
  out[idx] = v;
  if (gradient) {
    for (int al = 0; al < 3; ++al)
      out[(al + 1) * total + idx] = df0 * g.inv[al * 3 + 0] + df1 * g.inv[al * 3 + 1] + df2 * g.inv[al * 3 + 2];
  }
}

// radial[c][a][k] = sum_ir wr2g[k][ir] sum_ip samples[c][a][ir][ip] yweight[ip][k]
__global__ void project_radial_kernel(const double* samples, const double* yweight, const double* wr2g, int natoms,
                                      int nrad, int nang, int naug, int ncomp, double* radial) {
  int k = blockIdx.x, a = blockIdx.y, c = blockIdx.z;
  if (k >= naug || a >= natoms || c >= ncomp) return;
  long long total = (long long)natoms * nrad * nang;
  double acc = 0;
  for (int ir = threadIdx.x; ir < nrad; ir += blockDim.x) {
    const double* s = samples + c * total + ((long long)a * nrad + ir) * nang;
    double v = 0;
    for (int ip = 0; ip < nang; ++ip) v += s[ip] * yweight[ip * naug + k];
    acc += wr2g[(long long)k * nrad + ir] * v;
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) radial[((long long)c * natoms + a) * naug + k] = red[0];
}

// D = DION + multipole . radial_v (symmetrised); dD_alpha = multipole . radial_grad_alpha
__global__ void finish_dij_kernel(const double* dion, const double* mp, const double* radial, int natoms, int nlm,
                                  int naug, int ncomp, double* dij, double* ddij) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long total = (long long)natoms * nlm * nlm;
  if (idx >= total) return;
  int b = int(idx % nlm);
  long long t = idx / nlm;
  int a = int(t % nlm), at = int(t / nlm);
  for (int c = 0; c < ncomp; ++c) {
    const double* rv = radial + ((long long)c * natoms + at) * naug;
    double vab = 0, vba = 0;
    for (int k = 0; k < naug; ++k) {
      vab += mp[((long long)a * nlm + b) * naug + k] * rv[k];
      vba += mp[((long long)b * nlm + a) * naug + k] * rv[k];
    }
    if (c == 0) {
      vab += dion[a * nlm + b];
      vba += dion[b * nlm + a];
      dij[idx] = 0.5 * (vab + vba);
    } else {
      ddij[(((long long)at * 3 + (c - 1)) * nlm + a) * nlm + b] = 0.5 * (vab + vba);
    }
  }
}

}  // namespace

void build_dij_device(Context& ctx, bool gradient) {
  cudaStream_t s = ctx.rt->stream;
  const auto& sh = ctx.charge.shape;
  const long long n = ctx.nr();
  DeviceBuffer<double2> freq(n);
  DeviceBuffer<double> coeff(n);
  real_to_complex_kernel<<<blocks_for(n), 256, 0, s>>>(ctx.veff.get(), freq.get(), n, 1.0);
  fft3d_inplace(freq.get(), sh, -1, s);
  prefilter_kernel<<<blocks_for(n), 256, 0, s>>>(freq.get(), sh[0], sh[1], sh[2]);
  fft3d_inplace(freq.get(), sh, +1, s);
  coeff_real_kernel<<<blocks_for(n), 256, 0, s>>>(freq.get(), coeff.get(), n);
  HALF_LAUNCH("qdep prefilter");
  SampleGeom geom{sh[0], sh[1], sh[2], {}};
  auto inv = ctx.crystal.inverse_lattice();
  for (int i = 0; i < 9; ++i) geom.inv[i] = inv[i];
  const int ncomp = gradient ? 4 : 1;
  for (auto& sp : ctx.species) {
    const QdepTables& t = sp.tables;
    const int nang = int(t.dirs.size() / 3);
    std::vector<double> pos;
    for (int a = 0; a < sp.natoms; ++a) {
      auto r = ctx.crystal.cartesian(sp.first_ion + a);
      pos.insert(pos.end(), r.begin(), r.end());
    }
    DeviceBuffer<double> dpos, drg, ddirs, dyw, dwr, dmp, ddion, samples, radial;
    dpos.upload(pos, s);
    drg.upload(t.rgrid, s);
    ddirs.upload(t.dirs, s);
    dyw.upload(t.yweight, s);
    dwr.upload(t.wr2g, s);
    dmp.upload(t.multipole, s);
    ddion.upload(t.dion_lm, s);
    long long total = (long long)sp.natoms * t.nrad * nang;
    samples.resize(size_t(total) * ncomp);
    radial.resize(size_t(ncomp) * sp.natoms * t.naug);
    sample_kernel<<<blocks_for(total), 256, 0, s>>>(coeff.get(), dpos.get(), drg.get(), ddirs.get(), sp.natoms, t.nrad,
                                                     nang, geom, gradient ? 1 : 0, samples.get());
    HALF_LAUNCH("qdep sample");
    project_radial_kernel<<<dim3(t.naug, sp.natoms, ncomp), 256, 0, s>>>(samples.get(), dyw.get(), dwr.get(), sp.natoms,
                                                                          t.nrad, nang, t.naug, ncomp, radial.get());
    HALF_LAUNCH("qdep radial");
    sp.dij.resize(size_t(sp.natoms) * sp.nlm * sp.nlm);
    sp.ddij.resize(size_t(sp.natoms) * 3 * sp.nlm * sp.nlm);
    if (!gradient) sp.ddij.zero(s);
    long long npair = (long long)sp.natoms * sp.nlm * sp.nlm;
    finish_dij_kernel<<<blocks_for(npair), 256, 0, s>>>(ddion.get(), dmp.get(), radial.get(), sp.natoms, sp.nlm, t.naug,
                                                         ncomp, sp.dij.get(), sp.ddij.get());
    HALF_LAUNCH("qdep finish");
    HALF_CUDA(cudaStreamSynchronize(s));
    sp.dij_host = sp.dij.download(s);
  }
}

// ------------------------------------------------------------------ context

void Context::initialize() {
  if (!rt) rt = std::make_unique<Runtime>();
  if (const char* w = std::getenv("HALF_KPOINT_STREAMS")) kpoint_workers = std::max(1, std::atoi(w));
  for (int j = 0; j < 3; ++j) make_fft_plan(charge.shape[j]);   // validates the box
  species.clear();
  species.resize(pots.size());
  int ion0 = 0;
  for (size_t it = 0; it < pots.size(); ++it) {
    SpeciesDevice& sp = species[it];
    const Potcar& p = pots[it];
    sp.natoms = crystal.counts[it];
    sp.nlm = p.nlm();
    sp.first_ion = ion0;
    sp.lps = p.lps;
    sp.nchan = p.channels();
    sp.pspnl_gmax = p.pspnl_gmax;
    sp.tables = build_qdep_tables(p);
    sp.qij_host = sp.tables.qij_lm;
    sp.qij.upload(sp.qij_host, rt->stream);
    sp.radial_y.clear();
    sp.radial_m2.clear();
    for (int c = 0; c < sp.nchan; ++c) {
      std::vector<double> y(p.pspnl.begin() + c * 100, p.pspnl.begin() + (c + 1) * 100);
      auto m2 = spline_second(y, p.pspnl_gmax);
      sp.radial_y.insert(sp.radial_y.end(), y.begin(), y.end());
      sp.radial_m2.insert(sp.radial_m2.end(), m2.begin(), m2.end());
    }
    ion0 += sp.natoms;
  }
  build_veff_device(*this);
  rebuild_dij();
}

void Context::rebuild_dij() {
  if (use_uspp) {
    build_dij_device(*this, true);
    return;
  }
  for (auto& sp : species) {   // DION only, the same for every atom (src/half_cuda_assembly.cuf:443-446)
    sp.dij_host.clear();
    for (int a = 0; a < sp.natoms; ++a)
      sp.dij_host.insert(sp.dij_host.end(), sp.tables.dion_lm.begin(), sp.tables.dion_lm.end());
    sp.dij.upload(sp.dij_host, rt->stream);
    sp.ddij.resize(size_t(sp.natoms) * 3 * sp.nlm * sp.nlm);
    sp.ddij.zero(rt->stream);
  }
  HALF_CUDA(cudaStreamSynchronize(rt->stream));
}

// ------------------------------------------------- fixed-scratch D_ij rebuild

namespace {

// Device scratch of the allocation-free rebuild (half_set_positions_noalloc):
// a file-scope array, so the call needs no cudaMalloc/cudaFree.  It holds the
// B-spline coefficients of Veff (8 B per grid point) followed by a region that
// first holds the complex transform (16 B per point) and then, species by
// species, the QDEP tables, the atom positions and the samples and radial
// projections of a chunk of atoms.  Every word read is written earlier in the
// same call, so nothing in it has to start at zero.  All calls on one device
// share it: overlapping calls (any handle, any thread) race.
constexpr size_t kFixedScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;
static __device__ __align__(256) unsigned char g_fixed_scratch[kFixedScratchBytes];

std::mutex g_fixed_mutex;
unsigned char* g_fixed_addr[kMaxDevices] = {};

// Address of the scratch on the current device, resolved once per device.
// The cached address belongs to the device's primary context, which the
// library assumes lives as long as the process: after a cudaDeviceReset the
// next call would use a stale address.
unsigned char* fixed_scratch() {
  int dev = 0;
  HALF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) fail(kInternal, "device ordinal out of range: " + std::to_string(dev));
  std::lock_guard<std::mutex> lock(g_fixed_mutex);
  if (!g_fixed_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_fixed_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      fail(kInternal, std::string("cudaGetSymbolAddress of the fixed D_ij scratch failed: ") + cudaGetErrorString(e));
    }
    g_fixed_addr[dev] = static_cast<unsigned char*>(p);
  }
  return g_fixed_addr[dev];
}

constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Bump allocator over a slice of the scratch; sizes were checked by the plan.
struct Slice {
  unsigned char* base;
  size_t used = 0;
  template <typename T>
  T* take(size_t n) {
    T* p = reinterpret_cast<T*>(base + used);
    used += align256(n * sizeof(T));
    return p;
  }
};

// Atoms of one species that fit the region after its tables (0: not even one).
int fixed_chunk(const SpeciesDevice& sp, size_t region) {
  const QdepTables& t = sp.tables;
  const size_t nang = t.dirs.size() / 3, ncomp = 4;
  size_t fixed = align256(t.rgrid.size() * 8) + align256(t.dirs.size() * 8) + align256(t.yweight.size() * 8) +
                 align256(t.wr2g.size() * 8) + align256(t.multipole.size() * 8) + align256(t.dion_lm.size() * 8) +
                 align256(size_t(sp.natoms) * 3 * 8);
  if (fixed + 2 * 256 >= region) return 0;
  size_t per_atom = (size_t(t.nrad) * nang + t.naug) * ncomp * 8;
  size_t fit = (region - fixed - 2 * 256) / per_atom;
  return int(std::min<size_t>(fit, size_t(sp.natoms)));
}

}  // namespace

void Context::rebuild_dij_fixed_scratch(bool check_only) {
  cudaStream_t s = rt->stream;
  if (!use_uspp) {   // DION only: copies into the existing D buffers
    for (auto& sp : species) {
      const size_t nd = size_t(sp.natoms) * sp.tables.dion_lm.size();
      if (sp.dij.size() != nd || sp.ddij.size() != 3 * nd) fail(kInternal, "D_ij buffers were not set up");
    }
    if (check_only) return;
    for (auto& sp : species) {
      const size_t per = sp.tables.dion_lm.size(), nd = size_t(sp.natoms) * per;
      sp.dij_host.resize(nd);
      for (int a = 0; a < sp.natoms; ++a)
        std::copy(sp.tables.dion_lm.begin(), sp.tables.dion_lm.end(), sp.dij_host.begin() + a * per);
      HALF_CUDA(cudaMemcpyAsync(sp.dij.get(), sp.dij_host.data(), nd * sizeof(double), cudaMemcpyHostToDevice, s));
      sp.ddij.zero(s);
    }
    HALF_CUDA(cudaStreamSynchronize(s));
    return;
  }
  const long long n = nr();
  // The new D_ij and dD_ij/dR of every species are staged at the end of the
  // scratch and copied into the context only after every species succeeded.
  size_t stage_bytes = 0;
  for (auto& sp : species) stage_bytes += align256(size_t(sp.natoms) * sp.nlm * sp.nlm * 4 * sizeof(double));
  const size_t coeff_bytes = align256(size_t(n) * sizeof(double));
  const size_t need_fft = coeff_bytes + align256(size_t(n) * sizeof(double2)) + stage_bytes;
  if (need_fft > kFixedScratchBytes)
    fail(kCapacity, "the fixed D_ij scratch holds " + std::to_string(kFixedScratchBytes >> 20) + " MiB; a " +
                        std::to_string(n) + "-point grid needs " + std::to_string(need_fft) +
                        " bytes (24 B per point plus the staged D_ij): use half_set_positions");
  const size_t region = kFixedScratchBytes - coeff_bytes - stage_bytes;
  std::vector<int> chunk(species.size());
  for (size_t it = 0; it < species.size(); ++it) {
    chunk[it] = fixed_chunk(species[it], region);
    if (chunk[it] < 1)
      fail(kCapacity, "the QDEP tables of species " + std::to_string(it) + " do not fit the fixed " +
                          std::to_string(kFixedScratchBytes >> 20) + " MiB D_ij scratch: use half_set_positions");
    const SpeciesDevice& sp = species[it];
    const size_t nd = size_t(sp.natoms) * sp.nlm * sp.nlm;
    if (sp.dij.size() != nd || sp.ddij.size() != 3 * nd || sp.dij_host.size() != nd)
      fail(kInternal, "D_ij buffers were not set up");
  }
  if (check_only) return;

  unsigned char* base = fixed_scratch();
  double* coeff = reinterpret_cast<double*>(base);
  unsigned char* stage = base + kFixedScratchBytes - stage_bytes;
  std::vector<double*> stage_d(species.size());
  {
    size_t off = 0;
    for (size_t it = 0; it < species.size(); ++it) {
      stage_d[it] = reinterpret_cast<double*>(stage + off);
      off += align256(size_t(species[it].natoms) * species[it].nlm * species[it].nlm * 4 * sizeof(double));
    }
  }
  double2* freq = reinterpret_cast<double2*>(base + coeff_bytes);
  const auto& sh = charge.shape;
  real_to_complex_kernel<<<blocks_for(n), 256, 0, s>>>(veff.get(), freq, n, 1.0);
  fft3d_inplace(freq, sh, -1, s);
  prefilter_kernel<<<blocks_for(n), 256, 0, s>>>(freq, sh[0], sh[1], sh[2]);
  fft3d_inplace(freq, sh, +1, s);
  coeff_real_kernel<<<blocks_for(n), 256, 0, s>>>(freq, coeff, n);
  HALF_LAUNCH("qdep prefilter");
  SampleGeom geom{sh[0], sh[1], sh[2], {}};
  auto inv = crystal.inverse_lattice();
  for (int i = 0; i < 9; ++i) geom.inv[i] = inv[i];
  const int ncomp = 4;
  auto put = [&](double* dst, const std::vector<double>& v) {
    HALF_CUDA(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  };
  for (size_t it = 0; it < species.size(); ++it) {
    SpeciesDevice& sp = species[it];
    const QdepTables& t = sp.tables;
    const int nang = int(t.dirs.size() / 3), na_max = chunk[it];
    std::vector<double> pos;
    for (int a = 0; a < sp.natoms; ++a) {
      auto r = crystal.cartesian(sp.first_ion + a);
      pos.insert(pos.end(), r.begin(), r.end());
    }
    // The region is reused: the copies below are ordered after every earlier
    // kernel on this stream, including those still reading the transform.
    Slice sl{base + coeff_bytes};
    double* drg = sl.take<double>(t.rgrid.size());
    double* ddirs = sl.take<double>(t.dirs.size());
    double* dyw = sl.take<double>(t.yweight.size());
    double* dwr = sl.take<double>(t.wr2g.size());
    double* dmp = sl.take<double>(t.multipole.size());
    double* ddion = sl.take<double>(t.dion_lm.size());
    double* dpos = sl.take<double>(pos.size());
    double* samples = sl.take<double>(size_t(na_max) * t.nrad * nang * ncomp);
    double* radial = sl.take<double>(size_t(ncomp) * na_max * t.naug);
    if (sl.used > region) fail(kInternal, "fixed D_ij scratch plan overflow");
    put(drg, t.rgrid);
    put(ddirs, t.dirs);
    put(dyw, t.yweight);
    put(dwr, t.wr2g);
    put(dmp, t.multipole);
    put(ddion, t.dion_lm);
    put(dpos, pos);
    const size_t nd = size_t(sp.nlm) * sp.nlm;
    for (int a0 = 0; a0 < sp.natoms; a0 += na_max) {
      const int na = std::min(na_max, sp.natoms - a0);
      const long long total = (long long)na * t.nrad * nang;
      sample_kernel<<<blocks_for(total), 256, 0, s>>>(coeff, dpos + 3 * a0, drg, ddirs, na, t.nrad, nang, geom, 1,
                                                       samples);
      HALF_LAUNCH("qdep sample");
      project_radial_kernel<<<dim3(t.naug, na, ncomp), 256, 0, s>>>(samples, dyw, dwr, na, t.nrad, nang, t.naug,
                                                                     ncomp, radial);
      HALF_LAUNCH("qdep radial");
      const long long npair = (long long)na * nd;
      double* sd = stage_d[it];
      double* sdd = sd + size_t(sp.natoms) * nd;
      finish_dij_kernel<<<blocks_for(npair), 256, 0, s>>>(ddion, dmp, radial, na, sp.nlm, t.naug, ncomp,
                                                           sd + a0 * nd, sdd + 3 * a0 * nd);
      HALF_LAUNCH("qdep finish");
    }
  }
  // every species succeeded: commit the staged D_ij and dD_ij/dR
  HALF_CUDA(cudaStreamSynchronize(s));
  for (size_t it = 0; it < species.size(); ++it) {
    SpeciesDevice& sp = species[it];
    const size_t nd = size_t(sp.natoms) * sp.nlm * sp.nlm;
    HALF_CUDA(cudaMemcpyAsync(sp.dij.get(), stage_d[it], nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    HALF_CUDA(cudaMemcpyAsync(sp.ddij.get(), stage_d[it] + nd, 3 * nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    HALF_CUDA(cudaMemcpyAsync(sp.dij_host.data(), stage_d[it], nd * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  HALF_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hb
