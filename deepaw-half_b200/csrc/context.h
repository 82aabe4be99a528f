// Library context and the per-k operator objects of the B200 path.
#pragma once

#include <array>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "fft.cuh"
#include "io.h"
#include "radial.h"

namespace hb {

enum Precision : int { kFP64 = 0, kMixed = 1, kFP64Guarded = 2 };

// ACC controls; tolerance and iteration bound default to the reference's
// (src/half_cuda_iterative_solver.cuf:113-118).  block is the operator's bands
// per chunk (the reference's 16); 0, the default here, lets the autotuner
// choose it (tune.h), which changes no result.
struct AccControls {
  double tol = 1.0e-4;
  int max_iter = 40;
  int block = 0;
  int precision = kFP64;
};

struct SolveInfo {
  int iterations = 0, fp64_iterations = 0, converged = 0;
  long long npw = 0, operator_columns = 0;
  double max_residual = 0, setup_ms = 0, solve_ms = 0, operator_ms = 0;
  double device_ms = 0;          // CUDA-event span on the context stream, prepare -> eigenpairs
  double local_ms = 0;           // CUDA-event time inside the local-operator kernels
  double local_bytes = 0;        // their algorithmic bytes (per-band FFT-path figure)
  long long local_columns = 0;   // band columns through the local operator
  long long launches = 0;        // library kernels launched
  double sweep_ms = 0;           // CUDA-event time of whole H/S applications
  long long sweep_columns = 0;
  double adjoint_ms = 0;         // CUDA-event time of the force adjoint
  double tensor_ms = 0;          // CUDA-event time of the tensor-core GEMM kernels
  double tensor_flops = 0;       // their bf16 tensor flops (24 per complex multiply-add)
  long long tensor_launches = 0;
};

// Event-based accounting of the library's own kernels.
// Event-timed spans of one device call.  Spans are recorded without host
// synchronisation; their durations are read once, when the call ends and its
// stream has been synchronised (collect), so timing adds no bubbles.
struct Profile {
  enum Kind { kLocal = 0, kSweep = 1, kAdjoint = 2, kTensor = 3 };
  cudaEvent_t a = nullptr, b = nullptr;
  std::vector<cudaEvent_t> pool;                         // reused across calls
  std::vector<std::pair<int, std::pair<int, int>>> spans;   // (kind, (begin, end) pool slots)
  size_t used = 0;
  double local_ms = 0, local_bytes = 0, sweep_ms = 0, adjoint_ms = 0, tensor_ms = 0, tensor_flops = 0;
  long long local_columns = 0, launches = 0, sweep_columns = 0, tensor_launches = 0;
  void reset() {
    local_ms = local_bytes = sweep_ms = adjoint_ms = tensor_ms = tensor_flops = 0;
    local_columns = launches = sweep_columns = tensor_launches = 0;
    spans.clear();
    used = 0;
  }
  int record(cudaStream_t s);                // a pooled event recorded on s
  void span(Kind k, int begin, int end) { spans.push_back({int(k), {begin, end}}); }
  void collect();                            // after synchronisation: add the span durations
  void destroy();
};

// Per-stream library handles.
struct Runtime {
  cudaStream_t stream = nullptr;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  bool bf16x9 = false;   // cuBLAS offers FP32 emulation on BF16 tensor cores
  bool tc_gemm = true;   // complex FP32 GEMMs on the library's tcgen05 kernel (tc_gemm.cu)
  DeviceBuffer<unsigned char> tc_work;   // its split-K partial sums, grow-only
  DeviceBuffer<unsigned char> tc_planes; // its operands pre-split into bf16 planes, grow-only
  DeviceBuffer<int> tc_err;              // raised when one of its pipeline waits gave up
  Profile prof;
  Runtime();
  ~Runtime();
  Runtime(const Runtime&) = delete;
  Runtime& operator=(const Runtime&) = delete;
};

// Plane-wave basis (src/half_basis.F90:9-55); fft_index is 0-based C order.
struct Basis {
  std::array<int, 3> shape{};
  std::array<double, 3> kpoint{};
  std::vector<int> gvec;          // npw*3
  std::vector<double> qvec;       // npw*3, A^-1
  std::vector<double> kinetic;    // npw, eV
  std::vector<long long> fft_index;
  long long npw() const { return (long long)kinetic.size(); }
};
Basis build_basis(const Crystal& c, const std::array<int, 3>& shape, double encut, const double k[3]);

// Device copy of everything the projector/D stage needs for one species.
struct SpeciesDevice {
  int natoms = 0, nlm = 0, first_ion = 0, nchan = 0;
  std::vector<int> lps;
  QdepTables tables;                   // host tables (QDEP)
  DeviceBuffer<double> dij;            // natoms * nlm * nlm, row-major per atom
  DeviceBuffer<double> ddij;           // natoms * 3 * nlm * nlm
  std::vector<double> dij_host;        // mirror of dij
  DeviceBuffer<double> qij;            // nlm * nlm
  std::vector<double> qij_host;
  double pspnl_gmax = 0;
  std::vector<double> radial_y, radial_m2;   // [channel][100]
};

struct Context {
  Crystal crystal;
  ChargeGrid charge;
  std::vector<Potcar> pots;
  double encut = 0;
  bool use_pbe = true, use_uspp = true;
  int backend = 2, solver = 1;
  AccControls acc;
  SolveInfo last;
  // request geometry (deep copy, src/half_library.F90:227-247)
  bool has_request_geometry = false;
  int request_nions = 0, request_ntypes = 0;
  std::array<int, 3> request_grid{};
  std::array<double, 9> request_lattice{};
  std::vector<int> request_species;
  std::vector<double> request_positions;

  std::unique_ptr<Runtime> rt;
  std::vector<std::unique_ptr<Runtime>> workers;   // extra streams for concurrent k points
  int kpoint_workers = 4;
  DeviceBuffer<double> veff;           // C order, eV
  std::vector<SpeciesDevice> species;

  void initialize();                   // Veff + QDEP on the device
  void rebuild_dij();                  // QDEP at fixed Veff (positions changed)
  // The same rebuild with every device scratch buffer in one fixed,
  // statically allocated device array (no device allocation); check only
  // reports whether this system fits it.
  void rebuild_dij_fixed_scratch(bool check_only);
  long long nr() const { return (long long)charge.shape[0] * charge.shape[1] * charge.shape[2]; }
};

// ----------------------------------------------------------------- set-up
void build_veff_device(Context& ctx);                 // setup.cu
void build_dij_device(Context& ctx, bool gradient);   // setup.cu
void fft3d_inplace(double2* data, const std::array<int, 3>& shape, int sign, cudaStream_t s);
// Effective potential of a device density (C order, rho * Omega): veff = local + V_xc and,
// when vxc is not null, V_xc alone (both C order, eV; src/half_potential.F90:31-93).
// Synchronises s before returning.
void build_potential(Context& ctx, cudaStream_t s, const double* charge_c, double* veff, double* vxc);
void density_to_c_order(const double* f_order, double* c_order, const std::array<int, 3>& shape, cudaStream_t s);
// freq = FFT_forward(real_c) / N over the box (the reference's fft3_forward then /n)
void forward_transform(const double* real_c, double2* freq, const std::array<int, 3>& shape, cudaStream_t s);

// ----------------------------------------------------------------- ion-position forces (ionforces.cu)
struct IonicForces {
  std::vector<double> ewald, local, nlcc, harris;   // nions * 3 each, eV/A (empty when not requested)
  double ewald_energy[5] = {0, 0, 0, 0, 0};          // total, real, reciprocal, self, background
  double local_energy = 0;
};
// output_f: the output density in file order (x fastest, rho * Omega), host or device memory;
// null = the context's density.
void ionic_forces_device(Context& ctx, const double* output_f, bool output_on_device, bool want_ewald,
                         bool want_local, bool want_nlcc, bool want_harris, IonicForces& out);

// ----------------------------------------------------------------- VASP wave export (export.cu)
// Basis indices in VASP's plane-wave order (the box's x-fastest order).
std::vector<int> vasp_order(const Basis& b);
// out (device, nb x npw float2, band-major) = FP32 coefficients vec[b*ld + order[g]].
void pack_vasp_device(Runtime& rt, const double2* vec, long long ld, int npw, int nb, const std::vector<int>& order,
                      float2* out);

// ----------------------------------------------------------------- output density (density.cu)
// density_f (device, n, file order) = smooth density of the states plus the augmentation density;
// vectors[ik] (device, ld[ik] x nb column-major), occupations [nk][nb].
void output_density_device(Context& ctx, int nk, const double* kpoints, const double* kweights, int nb,
                           const std::vector<const double2*>& vectors, const std::vector<long long>& ld,
                           const double* occupations, double* density_f, double* augmentation_charge);

// ----------------------------------------------------------------- operator
template <typename R>
struct KOperator;   // hs.cu

struct KOperatorSet {
  Runtime* rt = nullptr;                      // stream and handles the operator runs on
  Basis basis;
  int np = 0;                                 // projector columns (all species)
  std::unique_ptr<KOperator<double>> op64;
  std::unique_ptr<KOperator<float>> op32;
  DeviceBuffer<double> qvec;                  // npw*3 (forces)
  // Tables that generate the projector matrix (the FP32 operator's bf16
  // planes and, in-tile, the FP64 force adjoint): B[g, col] = ftab64[frow][g] (-i)^l
  // exp(-2 pi i sum_j (n_j(g) + k_j) afrac[3 atom + j]), pcol[col] =
  // (atom << 16) | (frow << 2) | l, gpack[g] = (n1, n2, n3) as signed 10-bit fields.
  DeviceBuffer<double> ftab64, afrac;
  DeviceBuffer<int> gpack, pcol;
  double kf[3] = {0, 0, 0};
  ~KOperatorSet();
};

std::unique_ptr<KOperatorSet> prepare_operator(Context& ctx, Runtime& rt, const double k[3], bool fp64, bool fp32);

// H/S application on device blocks (column-major, leading dimension ld).
template <typename R>
void apply_hs(Context& ctx, KOperatorSet& ks, const cplx_t<R>* x, long long ld, int nb, cplx_t<R>* hx,
              cplx_t<R>* sx, int chunk);
// The mixed mode's FP32 operator on complex128 device blocks (ld = n): rounded
// to FP32, applied, widened back.  Synchronises the stream.
void apply_hs_fp32(Context& ctx, KOperatorSet& ks, const double2* x, long long n, int nb, double2* hx, double2* sx,
                   int chunk);

// ----------------------------------------------------------------- solvers
struct SolveOutput {
  std::vector<double> eigenvalues;
  std::vector<double> vectors;       // interleaved complex, npw x nbands (optional)
  double overlap_min = -1, overlap_max = -1;
  bool keep_device = false;          // request dvectors even without host vectors
  DeviceBuffer<double2> dvectors;    // device copy (kept for forces)
};
void solve_acc(Context& ctx, KOperatorSet& ks, int nbands, bool want_vectors, SolveOutput& out, SolveInfo& info);
void solve_dense(Context& ctx, KOperatorSet& ks, int nbands, bool index_range, bool want_vectors, SolveOutput& out);
void assemble_dense(Context& ctx, KOperatorSet& ks, double2* h, double2* s);   // device N x N

// ----------------------------------------------------------------- mapped hand-off
// host_dst (ld x nb, column-major) = rows of src (n x nb) in the order src_row
// (host row j takes HALF row src_row[j]); rows n..ld-1 zero.  mapped.cu.
void gather_rows_to_host(Runtime& rt, const double2* src, long long n, int nb, const std::vector<int>& src_row,
                         long long ld, double2* host_dst);

// ----------------------------------------------------------------- forces
void nonlocal_forces_device(Context& ctx, KOperatorSet& ks, const double2* dvec, long long ld, int nb,
                            const double* eig, const double* occ, double kweight, double* forces_host);

}  // namespace hb
