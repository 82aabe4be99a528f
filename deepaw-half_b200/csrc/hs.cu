// The matrix-free MIMIC_US H/S operator of one k point.
//
// Reference: apply_hs_operator_cuda (src/half_cuda_assembly.cuf:468-519)
// scatters each band into a zeroed N_r box, runs one cuFFT per band inverse,
// multiplies by Veff/N_r, one cuFFT per band forward, gathers and adds T psi,
// then per species runs three ZGEMMs around a D/Q mixing kernel.
//
// B200 design: the local part is three fused kernels over x-planes of the box
// that never materialise empty data.  Planes are indexed by g1 in the
// sphere's x-extent only (about 40% of the box); within a plane only the rows
// that hold sphere points are transformed along z.
//   K1  sphere -> planes: scatter band points straight into the transform's
//       digit-reversed slots, inverse z FFT on occupied rows, inverse y FFT
//       on all columns, one coalesced plane store;
//   K2  x lines: gather the occupied x slots, inverse x FFT, multiply by
//       Veff/N_r, forward x FFT, store the occupied slots back;
//   K3  planes -> sphere: forward y FFT, forward z FFT on occupied rows,
//       gather sphere points, H psi = . + T psi, S psi = psi.
// Bands go through in chunks (the ACC block size) so the plane buffer of a
// chunk stays resident in the 126 MB L2 between the three kernels.  The
// projector part is one GEMM B^H X over all species and bands, a D/Q mixing
// kernel and the GEMMs accumulating B DY into H X and B QY into S X.  In FP64
// B is stored and the GEMMs are cuBLAS ZGEMM (the reference's calls); in FP32
// one pass per k point generates B from a radial-angular table
// (Omega^-1/2 beta_l(|q|) Y_lm, one row per species channel), the packed
// plane-wave indices and the ions' b_j.R / 2 pi straight into the bf16 planes
// of the tensor-core GEMM (tc_gemm.cu), in both orientations (conj(B)^T and
// B; 8 bytes per element each), and B [DY | QY] is one GEMM with a doubled N
// writing H X and S X.
#include <algorithm>
#include <cmath>
#include <map>

#include "blas.h"
#include "context.h"
#include "tune.h"

namespace hb {

template <typename R>
struct KOperator {
  using C = cplx_t<R>;
  int npw = 0, n1 = 0, n2 = 0, n3 = 0, g1min = 0, nplanes = 0, np = 0, max_rows = 0;
  AxisPlan ax, ay, az;
  DeviceBuffer<int> plane_start, spos, row_start, row_list, plane_xpos;
  DeviceBuffer<R> veff;      // Veff / N_r, C order
  DeviceBuffer<R> kinetic;
  DeviceBuffer<C> work;      // chunk x nplanes x n2 x n3
  int work_chunk = 0;
  DeviceBuffer<C> B;         // FP64: npw x np, column-major
  // FP32: the projector matrix is generated from these tables straight into
  // the bf16 planes of the tensor-core GEMM (tc_gemm.cu), once per k point,
  // in the two orientations the products use
  DeviceBuffer<float> ftab;  // [frow][npw] Omega^-1/2 beta_l(|q|) Y_lm(q^), frow = (species, channel, m)
  DeviceBuffer<int> gpack;   // npw packed (n1, n2, n3)
  DeviceBuffer<int> pcol;    // np: (ion << 16) | (frow << 2) | l
  DeviceBuffer<double> afrac;   // nions x 3: b_j . R / 2 pi
  double kf[3] = {0, 0, 0};
  DeviceBuffer<unsigned char> bh_store, b_store;
  TcOperand bh_planes;       // conj(B)^T: np x npw
  TcOperand b_planes;        // B: npw x np
  DeviceBuffer<R> dall, qall;            // D per atom, Q per species
  DeviceBuffer<int> col_base, col_a, col_nlm, col_dofs, col_qofs;
  DeviceBuffer<C> coeff, dy, qy;
  int ws_cols = 0;
};

KOperatorSet::~KOperatorSet() = default;

namespace {

constexpr int kXTile = 16;

template <typename C>
__device__ __forceinline__ C czero() { C c; c.x = 0; c.y = 0; return c; }

template <typename R>
__global__ void __launch_bounds__(512) k1_sphere_to_planes(const cplx_t<R>* __restrict__ psi, long long ld, int b0,
                                                           int n2, int n3, int nplanes, const int* __restrict__ plane_start,
                                                           const int* __restrict__ spos, const int* __restrict__ row_start,
                                                           const int* __restrict__ row_list, AxisPlan ay, AxisPlan az,
                                                           cplx_t<R>* __restrict__ work) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* twy = reinterpret_cast<C*>(smem_raw);
  C* twz = twy + kMaxFFT;
  C* plane = twz + kMaxFFT;
  int* rows = reinterpret_cast<int*>(plane + n2 * n3);
  const int j = blockIdx.x, b = blockIdx.y;
  fill_twiddles(twy, n2);
  fill_twiddles(twz, n3);
  const int npl = n2 * n3;
  for (int t = threadIdx.x; t < npl; t += blockDim.x) plane[t] = czero<C>();
  const int r0 = row_start[j], nrows = row_start[j + 1] - r0;
  for (int t = threadIdx.x; t < nrows; t += blockDim.x) rows[t] = row_list[r0 + t];
  __syncthreads();
  const C* col = psi + (long long)(b0 + b) * ld;
  const int p0 = plane_start[j], p1 = plane_start[j + 1];
  for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) plane[spos[p]] = col[p];
  __syncthreads();
  fft_pencils<true, C, R>(plane, nrows, n3, 1, az.plan, twz, +1, rows);
  fft_pencils<true, C, R>(plane, n3, 1, n3, ay.plan, twy, +1);
  C* dst = work + ((long long)b * nplanes + j) * npl;
  for (int t = threadIdx.x; t < npl; t += blockDim.x) dst[t] = plane[t];
}

template <typename R>
__global__ void __launch_bounds__(256) k2_xlines(cplx_t<R>* __restrict__ work, int n1, int n2, int n3, int nplanes,
                                                 const int* __restrict__ plane_xpos, AxisPlan ax,
                                                 const R* __restrict__ veff, int nb, int bands_per_cta) {
  // One CTA per (i2, z tile) and group of bands_per_cta of the chunk's nb
  // bands, looping over its bands: the twiddles, the occupied-slot map and
  // the tile's Veff are set up once per CTA.
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* X = tw + kMaxFFT;                                 // [i1][tz]
  R* vt = reinterpret_cast<R*>(X + n1 * kXTile);       // [i1][tz] Veff / N_r
  int* xpos = reinterpret_cast<int*>(vt + n1 * kXTile);
  const int tiles = (n3 + kXTile - 1) / kXTile;
  const int i2 = blockIdx.x / tiles, z0 = (blockIdx.x - i2 * tiles) * kXTile;
  const int nz = min(kXTile, n3 - z0);
  fill_twiddles(tw, n1);
  for (int t = threadIdx.x; t < nplanes; t += blockDim.x) xpos[t] = plane_xpos[t];
  for (int t = threadIdx.x; t < n1 * kXTile; t += blockDim.x) {
    const int i1 = t / kXTile, c = t - i1 * kXTile;
    vt[t] = c < nz ? veff[((long long)i1 * n2 + i2) * n3 + z0 + c] : R(0);
  }
  const long long npl = (long long)n2 * n3;
  const int bend = min(nb, (blockIdx.y + 1) * bands_per_cta);
  for (int b = blockIdx.y * bands_per_cta; b < bend; ++b) {
    for (int t = threadIdx.x; t < n1 * kXTile; t += blockDim.x) X[t] = czero<C>();
    __syncthreads();
    C* base = work + (long long)b * nplanes * npl + (long long)i2 * n3 + z0;
    for (int t = threadIdx.x; t < nplanes * kXTile; t += blockDim.x) {
      int jj = t / kXTile, c = t - jj * kXTile;
      if (c < nz) X[xpos[jj] * kXTile + c] = base[jj * npl + c];
    }
    __syncthreads();
    fft_pencils<true, C, R>(X, kXTile, 1, kXTile, ax.plan, tw, +1);
    for (int t = threadIdx.x; t < n1 * kXTile; t += blockDim.x) X[t] = cscale(X[t], vt[t]);
    __syncthreads();
    fft_pencils<false, C, R>(X, kXTile, 1, kXTile, ax.plan, tw, -1);
    for (int t = threadIdx.x; t < nplanes * kXTile; t += blockDim.x) {
      int jj = t / kXTile, c = t - jj * kXTile;
      if (c < nz) base[jj * npl + c] = X[xpos[jj] * kXTile + c];
    }
    __syncthreads();
  }
}

template <typename R>
__global__ void __launch_bounds__(512) k3_planes_to_sphere(const cplx_t<R>* __restrict__ work, int n2, int n3,
                                                           int nplanes, const int* __restrict__ plane_start,
                                                           const int* __restrict__ spos, const int* __restrict__ row_start,
                                                           const int* __restrict__ row_list, AxisPlan ay, AxisPlan az,
                                                           const cplx_t<R>* __restrict__ psi, long long ld, int b0,
                                                           const R* __restrict__ kinetic, cplx_t<R>* __restrict__ hpsi,
                                                           cplx_t<R>* __restrict__ spsi) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* twy = reinterpret_cast<C*>(smem_raw);
  C* twz = twy + kMaxFFT;
  C* plane = twz + kMaxFFT;
  int* rows = reinterpret_cast<int*>(plane + n2 * n3);
  const int j = blockIdx.x, b = blockIdx.y;
  fill_twiddles(twy, n2);
  fill_twiddles(twz, n3);
  const int npl = n2 * n3;
  const C* src = work + ((long long)b * nplanes + j) * npl;
  for (int t = threadIdx.x; t < npl; t += blockDim.x) plane[t] = src[t];
  const int r0 = row_start[j], nrows = row_start[j + 1] - r0;
  for (int t = threadIdx.x; t < nrows; t += blockDim.x) rows[t] = row_list[r0 + t];
  __syncthreads();
  fft_pencils<false, C, R>(plane, n3, 1, n3, ay.plan, twy, -1);
  fft_pencils<false, C, R>(plane, nrows, n3, 1, az.plan, twz, -1, rows);
  const long long off = (long long)(b0 + b) * ld;
  const int p0 = plane_start[j], p1 = plane_start[j + 1];
  for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    C x = psi[off + p];
    C h = plane[spos[p]];
    R kin = kinetic[p];
    h.x += kin * x.x;
    h.y += kin * x.y;
    hpsi[off + p] = h;
    spsi[off + p] = x;
  }
}

// Density variant of k2_xlines: the block owns the box points (all i1, its
// i2, its z tile) and runs the chunk's bands in order through the inverse x
// transform, accumulating bw[b] |psi_b(r)|^2; the chunk total is added to
// density (C order) once.  No atomics: each point has one owner.
__global__ void __launch_bounds__(256) k2_density(const double2* __restrict__ work, int n1, int n2, int n3,
                                                  int nplanes, const int* __restrict__ plane_xpos, AxisPlan ax,
                                                  const double* __restrict__ bw, int nb,
                                                  double* __restrict__ density) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  double2* X = tw + kMaxFFT;                                   // [i1][tz]
  double* acc = reinterpret_cast<double*>(X + n1 * kXTile);    // [i1][tz]
  int* xpos = reinterpret_cast<int*>(acc + n1 * kXTile);
  const int tiles = (n3 + kXTile - 1) / kXTile;
  const int i2 = blockIdx.x / tiles, z0 = (blockIdx.x - i2 * tiles) * kXTile;
  const int nz = min(kXTile, n3 - z0);
  fill_twiddles(tw, n1);
  for (int t = threadIdx.x; t < n1 * kXTile; t += blockDim.x) acc[t] = 0.0;
  for (int t = threadIdx.x; t < nplanes; t += blockDim.x) xpos[t] = plane_xpos[t];
  const long long npl = (long long)n2 * n3;
  for (int b = 0; b < nb; ++b) {
    for (int t = threadIdx.x; t < n1 * kXTile; t += blockDim.x) X[t] = czero<double2>();
    __syncthreads();
    const double2* base = work + (long long)b * nplanes * npl + (long long)i2 * n3 + z0;
    for (int t = threadIdx.x; t < nplanes * kXTile; t += blockDim.x) {
      int jj = t / kXTile, c = t - jj * kXTile;
      if (c < nz) X[xpos[jj] * kXTile + c] = base[jj * npl + c];
    }
    __syncthreads();
    fft_pencils<true, double2, double>(X, kXTile, 1, kXTile, ax.plan, tw, +1);
    const double w = bw[b];
    for (int t = threadIdx.x; t < n1 * kXTile; t += blockDim.x) {
      const double2 v = X[t];
      acc[t] += w * (v.x * v.x + v.y * v.y);
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < n1 * kXTile; t += blockDim.x) {
    int i1 = t / kXTile, c = t - i1 * kXTile;
    if (c < nz) density[((long long)i1 * n2 + i2) * n3 + z0 + c] += acc[t];
  }
}

// dy[:,b] = blockdiag(D_atom) coeff[:,b], qy[:,b] = blockdiag(Q_species) coeff[:,b]
// (src/half_cuda_assembly.cuf:220-237)
template <typename R>
__global__ void mix_kernel(const cplx_t<R>* __restrict__ coeff, int np, int nb, const int* __restrict__ col_base,
                           const int* __restrict__ col_a, const int* __restrict__ col_nlm,
                           const int* __restrict__ col_dofs, const int* __restrict__ col_qofs,
                           const R* __restrict__ dall, const R* __restrict__ qall, cplx_t<R>* __restrict__ dy,
                           cplx_t<R>* __restrict__ qy) {
  using C = cplx_t<R>;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)np * nb) return;
  int p = int(idx % np);
  long long b = idx / np;
  const int base = col_base[p], a = col_a[p], nlm = col_nlm[p];
  const R* drow = dall + col_dofs[p] + a * nlm;
  const R* qrow = qall + col_qofs[p] + a * nlm;
  const C* c = coeff + b * np + base;
  C zd = czero<C>(), zq = czero<C>();
  for (int k = 0; k < nlm; ++k) {
    C v = c[k];
    zd.x += drow[k] * v.x; zd.y += drow[k] * v.y;
    zq.x += qrow[k] * v.x; zq.y += qrow[k] * v.y;
  }
  dy[idx] = zd;
  qy[idx] = zq;
}

struct ProjCol {
  int chan;      // global channel index into the radial tables
  int l, m;
  int ion;
  double gmax;
};

// beta_l(|q|) Y_lm(q^) of one projector channel at one plane wave, with the
// reference's 0.99 gmax cut (src/half_paw.F90:52-65).
__device__ __forceinline__ double radial_angular(const ProjCol& col, double qx, double qy, double qz,
                                                 const double* __restrict__ ry, const double* __restrict__ rm2) {
  double qn = sqrt(qx * qx + qy * qy + qz * qz);
  double theta = 0, phi = 0;
  if (qn > 1.0e-10) {
    theta = acos(fmax(-1.0, fmin(1.0, qz / qn)));
    phi = atan2(qy, qx);
  }
  double rval = spline_eval(ry + col.chan * 100, rm2 + col.chan * 100, 100, col.gmax, qn);
  if (qn > 0.99 * col.gmax) rval = 0;
  return rval * real_ylm(col.l, col.m, cos(theta), phi);
}

// B[g, p] = Omega^-1/2 (-i)^l beta_l(|q|) Y_lm(q^) exp(-i q.R)   (src/half_paw.F90:52-65)
__global__ void projector_kernel(double2* __restrict__ B, int npw, const double* __restrict__ q,
                                 const ProjCol* __restrict__ cols, const double* __restrict__ ry,
                                 const double* __restrict__ rm2, const double* __restrict__ pos, double pref) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  int p = blockIdx.y;
  if (g >= npw) return;
  const ProjCol col = cols[p];
  double qx = q[3 * g], qy = q[3 * g + 1], qz = q[3 * g + 2];
  double ph = qx * pos[3 * col.ion] + qy * pos[3 * col.ion + 1] + qz * pos[3 * col.ion + 2];
  double s, c;
  sincos(ph, &s, &c);
  double amp = pref * radial_angular(col, qx, qy, qz, ry, rm2);
  // (-i)^l * (cos - i sin)
  double re = amp * c, im = -amp * s, tr, ti;
  switch (col.l & 3) {
    case 0: tr = re; ti = im; break;
    case 1: tr = im; ti = -re; break;
    case 2: tr = -re; ti = -im; break;
    default: tr = -im; ti = re; break;
  }
  B[(long long)p * npw + g] = make_double2(tr, ti);
}

// ftab[r][g] = Omega^-1/2 beta_l(|q|) Y_lm(q^) for the channel rows of the
// generated FP32 projector tiles (one row per (species, channel, m)).
__global__ void radial_angular_table_kernel(double* __restrict__ ftab, int npw, const double* __restrict__ q,
                                            const ProjCol* __restrict__ rows, const double* __restrict__ ry,
                                            const double* __restrict__ rm2, double pref) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (g >= npw) return;
  ftab[(long long)r * npw + g] = pref * radial_angular(rows[r], q[3 * g], q[3 * g + 1], q[3 * g + 2], ry, rm2);
}

template <typename R>
__global__ void scale_copy_kernel(const double* __restrict__ in, R* __restrict__ out, long long n, double s) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = R(in[i] * s);
}

template <typename R>
size_t plane_smem(int n2, int n3) {
  return (2 * kMaxFFT + size_t(n2) * n3) * sizeof(cplx_t<R>) + size_t(n2) * sizeof(int);
}
template <typename R>
size_t xline_smem(int n1, int nplanes) {
  return (kMaxFFT + size_t(n1) * kXTile) * sizeof(cplx_t<R>) + size_t(n1) * kXTile * sizeof(R) +
         size_t(nplanes) * sizeof(int);
}

struct HostGeom {
  int g1min = 0, nplanes = 0, max_rows = 0;
  std::vector<int> plane_start, spos, row_start, row_list, plane_xpos;
};

HostGeom plane_geometry(const Basis& b, const AxisPlan& ax, const AxisPlan& ay, const AxisPlan& az) {
  HostGeom h;
  const int n1 = b.shape[0], n2 = b.shape[1], n3 = b.shape[2];
  const long long npw = b.npw();
  int g1min = b.gvec[0], g1max = b.gvec[3 * (npw - 1)];
  h.g1min = g1min;
  h.nplanes = g1max - g1min + 1;
  if (h.nplanes > n1) fail(kInternal, "sphere x-extent exceeds the FFT box");
  h.plane_start.assign(h.nplanes + 1, 0);
  h.spos.resize(npw);
  long long p = 0;
  for (int j = 0; j < h.nplanes; ++j) {
    h.plane_start[j] = int(p);
    h.row_start.push_back(int(h.row_list.size()));
    int last_i2 = -1;
    while (p < npw && b.gvec[3 * p] == g1min + j) {
      int i2 = ((b.gvec[3 * p + 1] % n2) + n2) % n2, i3 = ((b.gvec[3 * p + 2] % n3) + n3) % n3;
      int row = ay.pos[i2];
      if (i2 != last_i2) { h.row_list.push_back(row); last_i2 = i2; }
      h.spos[p] = row * n3 + az.pos[i3];
      ++p;
    }
    int i1 = (((g1min + j) % n1) + n1) % n1;
    h.plane_xpos.push_back(ax.pos[i1]);
  }
  h.plane_start[h.nplanes] = int(p);
  h.row_start.push_back(int(h.row_list.size()));
  for (int j = 0; j < h.nplanes; ++j) h.max_rows = std::max(h.max_rows, h.row_start[j + 1] - h.row_start[j]);
  if (p != npw) fail(kInternal, "basis is not ordered by g1");
  return h;
}

// What the FP32 operator needs to generate projector tiles: one radial-angular
// row per (species, channel, m), the column descriptors, and the ions' b_j.R / 2 pi.
struct ProjGen {
  std::vector<ProjCol> frows;
  std::vector<int> pcol, gpack;
  std::vector<double> afrac;
  const double* ftab64 = nullptr;   // device [frow][npw], built by prepare_operator
  const double* qvec = nullptr;   // device npw x 3
  const double* ry = nullptr;     // device radial tables
  const double* rm2 = nullptr;
  double pref = 0;
};

template <typename R>
void fill_operator(Context& ctx, Runtime& rt, const Basis& basis, const HostGeom& hg, const DeviceBuffer<double2>& B64, int np,
                   const std::vector<int>& cb, const std::vector<int>& ca, const std::vector<int>& cn,
                   const std::vector<int>& cd, const std::vector<int>& cq, const ProjGen& gen, KOperator<R>& op) {
  cudaStream_t s = rt.stream;
  op.npw = int(basis.npw());
  op.n1 = basis.shape[0]; op.n2 = basis.shape[1]; op.n3 = basis.shape[2];
  op.ax = make_axis_plan(op.n1); op.ay = make_axis_plan(op.n2); op.az = make_axis_plan(op.n3);
  op.g1min = hg.g1min; op.nplanes = hg.nplanes; op.max_rows = hg.max_rows; op.np = np;
  if (plane_smem<R>(op.n2, op.n3) > 227 * 1024)
    fail(kUnavailable, "FFT plane " + std::to_string(op.n2) + "x" + std::to_string(op.n3) +
                           " exceeds the shared-memory capacity of one CTA at this precision");
  op.plane_start.upload(hg.plane_start, s);
  op.spos.upload(hg.spos, s);
  op.row_start.upload(hg.row_start, s);
  op.row_list.upload(hg.row_list, s);
  op.plane_xpos.upload(hg.plane_xpos, s);
  const long long nr = ctx.nr();
  op.veff.resize(nr);
  scale_copy_kernel<R><<<ceil_div(nr, 256), 256, 0, s>>>(ctx.veff.get(), op.veff.get(), nr, 1.0 / double(nr));
  DeviceBuffer<double> kin;
  kin.upload(basis.kinetic, s);
  op.kinetic.resize(basis.npw());
  scale_copy_kernel<R><<<ceil_div(basis.npw(), 256), 256, 0, s>>>(kin.get(), op.kinetic.get(), basis.npw(), 1.0);
  if constexpr (sizeof(R) == 8) {
    op.B.resize(B64.size());
    HALF_CUDA(cudaMemcpyAsync(op.B.get(), B64.get(), B64.size() * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  } else if (np > 0) {
    const long long nt = (long long)gen.frows.size() * basis.npw();
    op.ftab.resize(size_t(nt));
    scale_copy_kernel<float><<<ceil_div(nt, 256), 256, 0, s>>>(gen.ftab64, op.ftab.get(), nt, 1.0);
    HALF_LAUNCH("radial-angular table (FP32)");
    op.gpack.upload(gen.gpack, s);
    op.pcol.upload(gen.pcol, s);
    op.afrac.upload(gen.afrac, s);
    for (int j = 0; j < 3; ++j) op.kf[j] = basis.kpoint[j];
    TcOperand g;
    g.kind = TcOperand::kProjConj;
    g.rows = np;
    g.kdim = op.npw;
    g.ftab = op.ftab.get();
    g.gpack = op.gpack.get();
    g.pcol = op.pcol.get();
    g.afrac = op.afrac.get();
    g.kf0 = op.kf[0];
    g.kf1 = op.kf[1];
    g.kf2 = op.kf[2];
    g.npw = op.npw;
    op.bh_planes = tc_presplit_a(rt, g, op.bh_store);
    g.kind = TcOperand::kProj;
    g.rows = op.npw;
    g.kdim = np;
    op.b_planes = tc_presplit_a(rt, g, op.b_store);
  }
  std::vector<double> dall, qall;
  for (auto& sp : ctx.species) {
    dall.insert(dall.end(), sp.dij_host.begin(), sp.dij_host.end());
    qall.insert(qall.end(), sp.qij_host.begin(), sp.qij_host.end());
  }
  DeviceBuffer<double> dd, dq;
  dd.upload(dall, s);
  dq.upload(qall, s);
  op.dall.resize(dall.size());
  op.qall.resize(qall.size());
  scale_copy_kernel<R><<<ceil_div((long long)dall.size(), 256), 256, 0, s>>>(dd.get(), op.dall.get(), (long long)dall.size(), 1.0);
  scale_copy_kernel<R><<<ceil_div((long long)qall.size(), 256), 256, 0, s>>>(dq.get(), op.qall.get(), (long long)qall.size(), 1.0);
  op.col_base.upload(cb, s);
  op.col_a.upload(ca, s);
  op.col_nlm.upload(cn, s);
  op.col_dofs.upload(cd, s);
  op.col_qofs.upload(cq, s);
  HALF_LAUNCH("operator tables");
  HALF_CUDA(cudaStreamSynchronize(s));
  raise_smem_limit(k1_sphere_to_planes<R>, plane_smem<R>(op.n2, op.n3));
  raise_smem_limit(k3_planes_to_sphere<R>, plane_smem<R>(op.n2, op.n3));
  raise_smem_limit(k2_xlines<R>, xline_smem<R>(op.n1, op.nplanes));
}

}  // namespace

std::unique_ptr<KOperatorSet> prepare_operator(Context& ctx, Runtime& rt, const double k[3], bool fp64, bool fp32) {
  auto ks = std::make_unique<KOperatorSet>();
  ks->rt = &rt;
  ks->basis = build_basis(ctx.crystal, ctx.charge.shape, ctx.encut, k);
  const Basis& basis = ks->basis;
  const int npw = int(basis.npw());
  if (npw < 1) fail(kInvalidArgument, "empty plane-wave basis");
  cudaStream_t s = rt.stream;
  AxisPlan ax = make_axis_plan(basis.shape[0]), ay = make_axis_plan(basis.shape[1]), az = make_axis_plan(basis.shape[2]);
  HostGeom hg = plane_geometry(basis, ax, ay, az);
  // projector columns: species-major, atom-major, then (channel, m)
  std::vector<ProjCol> cols;
  std::vector<int> cb, ca, cn, cd, cq;
  std::vector<double> ry, rm2, pos;
  int chan0 = 0, dofs = 0, qofs = 0, col0 = 0;
  for (auto& sp : ctx.species) {
    for (int a = 0; a < sp.natoms; ++a) {
      int ilm = 0;
      for (int c = 0; c < sp.nchan; ++c) {
        int l = sp.lps[c];
        for (int m = -l; m <= l; ++m, ++ilm) {
          cols.push_back({chan0 + c, l, m, sp.first_ion + a, sp.pspnl_gmax});
          cb.push_back(col0 + a * sp.nlm);
          ca.push_back(ilm);
          cn.push_back(sp.nlm);
          cd.push_back(dofs + a * sp.nlm * sp.nlm);
          cq.push_back(qofs);
        }
      }
    }
    ry.insert(ry.end(), sp.radial_y.begin(), sp.radial_y.end());
    rm2.insert(rm2.end(), sp.radial_m2.begin(), sp.radial_m2.end());
    chan0 += sp.nchan;
    dofs += sp.natoms * sp.nlm * sp.nlm;
    qofs += sp.nlm * sp.nlm;
    col0 += sp.natoms * sp.nlm;
  }
  for (int i = 0; i < ctx.crystal.nions(); ++i) {
    auto r = ctx.crystal.cartesian(i);
    pos.insert(pos.end(), r.begin(), r.end());
  }
  const int np = int(cols.size());
  ks->np = np;
  // generated-tile tables for the FP32 operator: radial-angular rows are per
  // (species, channel, m), shared by the species' atoms
  ProjGen gen;
  {
    int chan = 0, frow0 = 0;
    size_t c = 0;
    for (auto& sp : ctx.species) {
      for (int ch = 0; ch < sp.nchan; ++ch) {
        int l = sp.lps[ch];
        for (int m = -l; m <= l; ++m) gen.frows.push_back({chan + ch, l, m, 0, sp.pspnl_gmax});
      }
      for (int a = 0; a < sp.natoms; ++a)
        for (int ilm = 0; ilm < sp.nlm; ++ilm, ++c) {
          if (cols[c].ion >= (1 << 15) || frow0 + ilm >= (1 << 14)) fail(kUnavailable, "too many ions or projector channels");
          gen.pcol.push_back((cols[c].ion << 16) | ((frow0 + ilm) << 2) | (cols[c].l & 3));
        }
      chan += sp.nchan;
      frow0 += sp.nlm;
    }
    auto rec = ctx.crystal.reciprocal();
    for (int i = 0; i < ctx.crystal.nions(); ++i) {
      auto r = ctx.crystal.cartesian(i);
      for (int j = 0; j < 3; ++j)
        gen.afrac.push_back((rec[3 * j] * r[0] + rec[3 * j + 1] * r[1] + rec[3 * j + 2] * r[2]) / (2.0 * kPi));
    }
  }
  for (size_t g = 0; g < basis.gvec.size(); ++g)
    if (basis.gvec[g] < -512 || basis.gvec[g] > 511) fail(kUnavailable, "plane-wave index beyond the packed range");
  ks->qvec.upload(basis.qvec, s);
  DeviceBuffer<ProjCol> dcols;
  dcols.upload(cols, s);
  DeviceBuffer<double> dry, drm2, dpos;
  dry.upload(ry, s);
  drm2.upload(rm2, s);
  dpos.upload(pos, s);
  DeviceBuffer<double2> B64((size_t)npw * np);
  gen.qvec = ks->qvec.get();
  gen.ry = dry.get();
  gen.rm2 = drm2.get();
  gen.pref = 1.0 / std::sqrt(ctx.crystal.volume());
  DeviceBuffer<ProjCol> drows;
  if (np > 0) {   // projector generation tables, shared by the FP32 operator's planes and the force adjoint
    const int nf = int(gen.frows.size());
    drows.upload(gen.frows, s);
    ks->ftab64.resize(size_t(nf) * npw);
    radial_angular_table_kernel<<<dim3(ceil_div(npw, 256), nf), 256, 0, s>>>(ks->ftab64.get(), npw, ks->qvec.get(),
                                                                            drows.get(), dry.get(), drm2.get(), gen.pref);
    HALF_LAUNCH("radial-angular table");
    gen.gpack.resize(npw);
    for (int g = 0; g < npw; ++g)
      gen.gpack[g] = (basis.gvec[3 * g] & 1023) | ((basis.gvec[3 * g + 1] & 1023) << 10) |
                     ((basis.gvec[3 * g + 2] & 1023) << 20);
    ks->gpack.upload(gen.gpack, s);
    ks->pcol.upload(gen.pcol, s);
    ks->afrac.upload(gen.afrac, s);
    for (int j = 0; j < 3; ++j) ks->kf[j] = basis.kpoint[j];
    gen.ftab64 = ks->ftab64.get();
  }
  if (np > 0) {
    projector_kernel<<<dim3(ceil_div(npw, 256), np), 256, 0, s>>>(B64.get(), npw, ks->qvec.get(), dcols.get(), dry.get(),
                                                                   drm2.get(), dpos.get(), 1.0 / std::sqrt(ctx.crystal.volume()));
    HALF_LAUNCH("projectors");
  }
  if (fp64) {
    ks->op64 = std::make_unique<KOperator<double>>();
    fill_operator<double>(ctx, rt, basis, hg, B64, np, cb, ca, cn, cd, cq, gen, *ks->op64);
  }
  if (fp32) {
    ks->op32 = std::make_unique<KOperator<float>>();
    fill_operator<float>(ctx, rt, basis, hg, B64, np, cb, ca, cn, cd, cq, gen, *ks->op32);
  }
  HALF_CUDA(cudaStreamSynchronize(s));
  return ks;
}

template <typename R>
KOperator<R>& pick(KOperatorSet& ks);
template <>
KOperator<double>& pick<double>(KOperatorSet& ks) {
  if (!ks.op64) fail(kInternal, "FP64 operator not prepared");
  return *ks.op64;
}
template <>
KOperator<float>& pick<float>(KOperatorSet& ks) {
  if (!ks.op32) fail(kInternal, "FP32 operator not prepared");
  return *ks.op32;
}

template <typename R>
void apply_nonlocal(Runtime& rt, KOperator<R>& op, const cplx_t<R>* x, long long ld, int nb, cplx_t<R>* hx,
                    cplx_t<R>* sx);

template <typename R>
void apply_hs(Context& ctx, KOperatorSet& ks, const cplx_t<R>* x, long long ld, int nb, cplx_t<R>* hx, cplx_t<R>* sx,
              int chunk) {
  using C = cplx_t<R>;
  KOperator<R>& op = pick<R>(ks);
  Runtime& rt = *ks.rt;
  cudaStream_t s = rt.stream;
  if (nb <= 0) return;
  // chunk <= 0: bands per chunk chosen by the autotuner (tune.h) per box,
  // sphere extent and precision; every choice gives bit-identical results
  int tune_token = 0;
  if (chunk <= 0) {
    static const std::vector<int> cand = {16, 8, 32, 64};
    const std::string key = "local " + std::to_string(op.n1) + "x" + std::to_string(op.n2) + "x" +
                            std::to_string(op.n3) + " planes " + std::to_string(op.nplanes) + " fp" +
                            std::to_string(8 * sizeof(R));
    const int idx = Tuner::pick(key, cand);
    chunk = cand[idx];
    tune_token = Tuner::begin(key, idx, s);
  }
  chunk = std::max(1, std::min(chunk, nb));
  if (op.work_chunk < chunk) {
    op.work.resize((size_t)chunk * op.nplanes * op.n2 * op.n3);
    op.work_chunk = chunk;
  }
  const size_t psm = plane_smem<R>(op.n2, op.n3), xsm = xline_smem<R>(op.n1, op.nplanes);
  const int tiles = (op.n3 + kXTile - 1) / kXTile;
  int sms = 148, dev = 0;
  HALF_CUDA(cudaGetDevice(&dev));
  HALF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  Profile& pf = rt.prof;
  const int ev_sweep = pf.record(s);
  const int ev_local = ev_sweep;
  for (int b0 = 0; b0 < nb; b0 += chunk) {
    int nbc = std::min(chunk, nb - b0);
    k1_sphere_to_planes<R><<<dim3(op.nplanes, nbc), 512, psm, s>>>(
        x, ld, b0, op.n2, op.n3, op.nplanes, op.plane_start.get(), op.spos.get(), op.row_start.get(), op.row_list.get(),
        op.ay, op.az, op.work.get());
    // bands per K2 CTA: as many as keep about eight CTAs per SM busy
    const int lines = op.n2 * tiles;
    const int groups = std::max(1, std::min(nbc, ceil_div(8 * sms, lines)));
    const int bpc = ceil_div(nbc, groups);
    k2_xlines<R><<<dim3(lines, ceil_div(nbc, bpc)), 256, xsm, s>>>(op.work.get(), op.n1, op.n2, op.n3, op.nplanes,
                                                                  op.plane_xpos.get(), op.ax, op.veff.get(), nbc, bpc);
    k3_planes_to_sphere<R><<<dim3(op.nplanes, nbc), 512, psm, s>>>(
        op.work.get(), op.n2, op.n3, op.nplanes, op.plane_start.get(), op.spos.get(), op.row_start.get(),
        op.row_list.get(), op.ay, op.az, x, ld, b0, op.kinetic.get(), hx, sx);
    pf.launches += 3;
  }
  HALF_LAUNCH("local operator");
  Tuner::finish(tune_token, s, double(nb));
  pf.span(Profile::kLocal, ev_local, pf.record(s));
  {
    // FFT-path algorithmic bytes per band: read psi, write H psi and S psi, two
    // transforms x two passes x (read + write) of the box; Veff once per call.
    const double sz = sizeof(C), rz = sizeof(R), nr = double(op.n1) * op.n2 * op.n3;
    pf.local_bytes += nb * (3.0 * sz * op.npw + 8.0 * sz * nr) + rz * nr;
    pf.local_columns += nb;
  }
  if (op.np > 0) {
    pf.launches += 1;
    apply_nonlocal<R>(rt, op, x, ld, nb, hx, sx);
  }
  pf.span(Profile::kSweep, ev_sweep, pf.record(s));
  pf.sweep_columns += nb;
}

// Projector part: H X += B blockdiag(D) B^H X, S X += B blockdiag(Q) B^H X
template <typename R>
void apply_nonlocal(Runtime& rt, KOperator<R>& op, const cplx_t<R>* x, long long ld, int nb, cplx_t<R>* hx,
                    cplx_t<R>* sx) {
  using C = cplx_t<R>;
  cudaStream_t s = rt.stream;
  if (op.ws_cols < nb) {
    op.coeff.resize((size_t)op.np * nb);
    op.dy.resize((size_t)op.np * nb);
    op.qy.resize((size_t)op.np * nb);
    op.ws_cols = nb;
  }
  const C one = cval<R>(1.0), zero = cval<R>(0.0);
  auto mix = [&]() {
    mix_kernel<R><<<ceil_div((long long)op.np * nb, 256), 256, 0, s>>>(op.coeff.get(), op.np, nb, op.col_base.get(),
                                                                       op.col_a.get(), op.col_nlm.get(), op.col_dofs.get(),
                                                                       op.col_qofs.get(), op.dall.get(), op.qall.get(),
                                                                       op.dy.get(), op.qy.get());
    HALF_LAUNCH("mix");
    ++rt.prof.launches;
  };
  if constexpr (sizeof(R) == 4) {
    // FP32: B in bf16 planes split once per k point (fill_operator).
    //   coeff = conj(B)^T X            (np x nb, K = npw)
    //   [H X | S X] += B [DY | QY]     (npw x 2nb, K = np; one GEMM, two outputs)
    tc_cgemm(rt, op.bh_planes, tc_dense_b(CUBLAS_OP_N, x, ld, op.npw, nb), op.np, nb, op.npw, make_double2(1, 0),
             make_double2(0, 0), op.coeff.get(), false, op.np);
    mix();
    TcOperand y = tc_dense_b(CUBLAS_OP_N, op.dy.get(), op.np, op.np, 2 * nb);
    y.p2 = op.qy.get();
    y.split = nb;
    tc_cgemm(rt, op.b_planes, y, op.npw, 2 * nb, op.np, make_double2(1, 0), make_double2(1, 0), hx, false, ld, sx, nb);
  } else {
    gemm(rt, CUBLAS_OP_C, CUBLAS_OP_N, op.np, nb, op.npw, one, op.B.get(), op.npw, x, ld, zero, op.coeff.get(), op.np);
    mix();
    gemm(rt, CUBLAS_OP_N, CUBLAS_OP_N, op.npw, nb, op.np, one, op.B.get(), op.npw, op.dy.get(), op.np, one, hx, ld);
    gemm(rt, CUBLAS_OP_N, CUBLAS_OP_N, op.npw, nb, op.np, one, op.B.get(), op.npw, op.qy.get(), op.np, one, sx, ld);
  }
}

template void apply_hs<double>(Context&, KOperatorSet&, const double2*, long long, int, double2*, double2*, int);
template void apply_hs<float>(Context&, KOperatorSet&, const float2*, long long, int, float2*, float2*, int);

namespace {
template <typename A, typename B>
__global__ void convert_complex_kernel(const A* __restrict__ in, B* __restrict__ out, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) {
    B v;
    v.x = in[i].x;
    v.y = in[i].y;
    out[i] = v;
  }
}
}  // namespace

void apply_hs_fp32(Context& ctx, KOperatorSet& ks, const double2* x, long long n, int nb, double2* hx, double2* sx,
                   int chunk) {
  cudaStream_t s = ks.rt->stream;
  const long long tot = n * nb;
  DeviceBuffer<float2> x32(tot), h32(tot), s32(tot);
  convert_complex_kernel<double2, float2><<<ceil_div(tot, 256), 256, 0, s>>>(x, x32.get(), tot);
  HALF_LAUNCH("to FP32");
  apply_hs<float>(ctx, ks, x32.get(), n, nb, h32.get(), s32.get(), chunk);
  convert_complex_kernel<float2, double2><<<ceil_div(tot, 256), 256, 0, s>>>(h32.get(), hx, tot);
  convert_complex_kernel<float2, double2><<<ceil_div(tot, 256), 256, 0, s>>>(s32.get(), sx, tot);
  HALF_LAUNCH("to FP64");
  HALF_CUDA(cudaStreamSynchronize(s));
}

void accumulate_band_density(KOperatorSet& ks, const double2* x, long long ld, int nb, const double* bw,
                             double* density_c, int chunk) {
  KOperator<double>& op = pick<double>(ks);
  cudaStream_t s = ks.rt->stream;
  if (nb <= 0) return;
  if (chunk <= 0) chunk = 16;
  chunk = std::max(1, std::min(chunk, nb));
  if (op.work_chunk < chunk) {
    op.work.resize((size_t)chunk * op.nplanes * op.n2 * op.n3);
    op.work_chunk = chunk;
  }
  const size_t psm = plane_smem<double>(op.n2, op.n3);
  const size_t dsm = xline_smem<double>(op.n1, op.nplanes);   // its accumulator takes the Veff tile's place
  raise_smem_limit(k2_density, dsm);
  const int tiles = (op.n3 + kXTile - 1) / kXTile;
  for (int b0 = 0; b0 < nb; b0 += chunk) {
    const int nbc = std::min(chunk, nb - b0);
    k1_sphere_to_planes<double><<<dim3(op.nplanes, nbc), 512, psm, s>>>(
        x, ld, b0, op.n2, op.n3, op.nplanes, op.plane_start.get(), op.spos.get(), op.row_start.get(),
        op.row_list.get(), op.ay, op.az, op.work.get());
    k2_density<<<op.n2 * tiles, 256, dsm, s>>>(op.work.get(), op.n1, op.n2, op.n3, op.nplanes, op.plane_xpos.get(),
                                                op.ax, bw + b0, nbc, density_c);
    ks.rt->prof.launches += 2;
  }
  HALF_LAUNCH("band density");
}

// Projector matrix of the prepared k point (used by the dense path and forces).
const double2* projector_matrix64(KOperatorSet& ks) { return pick<double>(ks).B.get(); }

}  // namespace hb
