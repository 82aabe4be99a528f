// The libhalf C ABI (include/half.h, include/half_b200.h).
//
// Handle registry, status and error-string conventions follow
// src/half_c_api.F90: at most 32 live contexts, handle = generation*32 + slot
// (:13-16, 208-209, 627-634), "invalid HALF context handle" for stale or
// unknown handles (:636-640), error buffers cleared on entry and filled
// NUL-terminated and truncated to capacity-1 (:650-665), and the mapped
// solve's open-addressing G-vector hash with the same multipliers
// (:521-597).  Backend/solver validation follows src/half_library.F90:51-110:
// this build has the CUDA backend only (the reference's CPU backend needs
// oneMKL), so CPU contexts answer HALF_ERROR_UNAVAILABLE.  Device failures
// return HALF_ERROR_INTERNAL with a message instead of stopping the process.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>

#include "../../include/half_b200.h"
#include "context.h"
#include "devmem.h"
#include "tc_gemm.h"

using namespace hb;

namespace {

constexpr int kMaxContexts = 32;

struct Slot {
  bool used = false;
  long long generation = 0;
  std::unique_ptr<Context> ctx;
};
Slot g_slots[kMaxContexts];
std::mutex g_mutex;

void clear_error(char* e, int cap) {
  if (e && cap > 0) e[0] = '\0';
}

void export_error(const std::string& msg, char* e, int cap) {
  if (!e || cap <= 0) return;
  std::string m = msg;
  while (!m.empty() && m.back() == ' ') m.pop_back();
  size_t n = std::min(m.size(), size_t(cap - 1));
  std::memcpy(e, m.data(), n);
  e[n] = '\0';
}

int slot_of(half_handle h) {
  if (h <= 0) return -1;
  long long s = h % kMaxContexts;
  if (s == 0) s = kMaxContexts;
  long long g = (h - s) / kMaxContexts;
  int idx = int(s - 1);
  if (!g_slots[idx].used || g != g_slots[idx].generation) return -1;
  return idx;
}

Context* lookup(half_handle h) {
  int s = slot_of(h);
  return s < 0 ? nullptr : g_slots[s].ctx.get();
}

int bad_handle(char* e, int cap) {
  export_error("invalid HALF context handle", e, cap);
  return HALF_ERROR_INVALID_HANDLE;
}

template <typename F>
int guarded(char* e, int cap, F&& f) {
  try {
    return f();
  } catch (const Error& err) {
    export_error(err.what(), e, cap);
    return err.status;
  } catch (const std::bad_alloc&) {
    export_error("host allocation failed", e, cap);
    return HALF_ERROR_INTERNAL;
  } catch (const std::exception& ex) {
    export_error(std::string("internal error: ") + ex.what(), e, cap);
    return HALF_ERROR_INTERNAL;
  }
}

std::string cstr(const char* s) {
  if (!s) return std::string();
  size_t n = 0;
  while (n < 4096 && s[n]) ++n;
  return std::string(s, n);
}

bool finite3(const double k[3]) { return k && std::isfinite(k[0]) && std::isfinite(k[1]) && std::isfinite(k[2]); }

double det3(const double* a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}

bool cuda_available() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) { cudaGetLastError(); return false; }
  return n > 0;
}

int create_context(const std::string& charge, const std::string& potential, double encut, int xc, int use_uspp,
                   int backend, int solver, half_handle* handle, char* err, int cap) {
  if (handle) *handle = 0;
  return guarded(err, cap, [&]() -> int {
    std::lock_guard<std::mutex> lock(g_mutex);
    int slot = -1;
    for (int i = 0; i < kMaxContexts; ++i)
      if (!g_slots[i].used) { slot = i; break; }
    if (slot < 0) { export_error("HALF context registry is full", err, cap); return HALF_ERROR_INTERNAL; }
    // src/half_library.F90:62-95
    if (!(encut > 0) || !std::isfinite(encut)) fail(kInvalidArgument, "ENCUT must be positive and finite");
    int be = backend == HALF_BACKEND_AUTO ? HALF_BACKEND_CUDA : backend;
    if (be == HALF_BACKEND_CPU) fail(kUnavailable, "CPU API backend is not built in this B200 library; use CUDA");
    if (!cuda_available()) fail(kUnavailable, "CUDA backend: no CUDA device is available");
    if (!file_exists(charge)) fail(kIO, "charge input does not exist");
    if (!file_exists(potential)) fail(kIO, "potential input does not exist");
    auto ctx = std::make_unique<Context>();
    read_chgcar(charge, ctx->crystal, ctx->charge);
    ctx->pots = read_potcar(potential);
    validate_potcar_structure(ctx->pots, ctx->crystal);
    ctx->encut = encut;
    ctx->use_pbe = xc == HALF_XC_PBE;
    ctx->use_uspp = use_uspp != 0;
    ctx->backend = be;
    ctx->solver = solver;
    ctx->initialize();
    g_slots[slot].used = true;
    g_slots[slot].generation += 1;
    g_slots[slot].ctx = std::move(ctx);
    if (handle) *handle = g_slots[slot].generation * kMaxContexts + (slot + 1);
    return HALF_SUCCESS;
  });
}

// Event accounting around one device call (solve, H/S application, force).
void begin_call(Runtime& rt) {
  Profile& pf = rt.prof;
  pf.reset();
  HALF_CUDA(cudaEventRecord(pf.a, rt.stream));
}

void end_call(Runtime& rt, SolveInfo& info) {
  Profile& pf = rt.prof;
  HALF_CUDA(cudaEventRecord(pf.b, rt.stream));
  HALF_CUDA(cudaEventSynchronize(pf.b));
  float ms = 0;
  HALF_CUDA(cudaEventElapsedTime(&ms, pf.a, pf.b));
  pf.collect();
  info.device_ms = ms;
  info.local_ms = pf.local_ms;
  info.local_bytes = pf.local_bytes;
  info.local_columns = pf.local_columns;
  info.launches = pf.launches;
  info.sweep_ms = pf.sweep_ms;
  info.sweep_columns = pf.sweep_columns;
  info.adjoint_ms = pf.adjoint_ms;
  info.tensor_ms = pf.tensor_ms;
  info.tensor_flops = pf.tensor_flops;
  info.tensor_launches = pf.tensor_launches;
}

// Solve one k point with the context's solver on runtime rt; out holds device vectors.
void solve_one(Context& ctx, Runtime& rt, const double k[3], int nbands, bool want_vectors, SolveOutput& out,
               SolveInfo& info, std::unique_ptr<KOperatorSet>* keep = nullptr) {
  auto t0 = std::chrono::steady_clock::now();
  if (!finite3(k)) fail(kInvalidArgument, "k point must be finite");
  info = SolveInfo();
  begin_call(rt);
  bool mixed = ctx.solver == HALF_SOLVER_ACC && ctx.acc.precision == kMixed;
  auto ks = prepare_operator(ctx, rt, k, true, mixed);
  double setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (nbands < 1 || nbands > ks->basis.npw()) fail(kInvalidArgument, "invalid requested band count");
  switch (ctx.solver) {
    case HALF_SOLVER_ACC: solve_acc(ctx, *ks, nbands, want_vectors, out, info); break;
    case HALF_SOLVER_EVD: solve_dense(ctx, *ks, nbands, false, want_vectors, out); break;
    case HALF_SOLVER_VASP: solve_dense(ctx, *ks, nbands, true, want_vectors, out); break;
    default: fail(kUnavailable, "the EVJ (Jacobi) dense solver is not built in this B200 library; use EVD, VASP or ACC");
  }
  info.setup_ms = setup_ms;
  info.npw = ks->basis.npw();
  end_call(rt, info);
  if (keep) *keep = std::move(ks);
}

void solve_one(Context& ctx, const double k[3], int nbands, bool want_vectors, SolveOutput& out,
               std::unique_ptr<KOperatorSet>* keep = nullptr) {
  solve_one(ctx, *ctx.rt, k, nbands, want_vectors, out, ctx.last, keep);
}

void accumulate(SolveInfo& total, const SolveInfo& s, bool first) {
  total.iterations += s.iterations;
  total.fp64_iterations += s.fp64_iterations;
  total.converged = (first ? 1 : total.converged) & s.converged;
  total.operator_columns += s.operator_columns;
  total.max_residual = std::max(total.max_residual, s.max_residual);
  total.setup_ms += s.setup_ms;
  total.solve_ms += s.solve_ms;
  total.operator_ms += s.operator_ms;
  total.npw += s.npw;
  total.local_ms += s.local_ms;
  total.local_bytes += s.local_bytes;
  total.local_columns += s.local_columns;
  total.launches += s.launches;
  total.sweep_ms += s.sweep_ms;
  total.sweep_columns += s.sweep_columns;
  total.tensor_ms += s.tensor_ms;
  total.tensor_flops += s.tensor_flops;
  total.tensor_launches += s.tensor_launches;
}

}  // namespace

extern "C" {

int half_get_abi_version(void) { return HALF_ABI_VERSION; }

const char* half_get_version_string(void) { return "0.6.0"; }

int half_get_capabilities(void) { return cuda_available() ? HALF_CAP_CUDA : 0; }

int half_escn_health(const char*, int, char* error, int cap) {
  clear_error(error, cap);
  export_error("DeePAW-eSCN density service is not part of this build", error, cap);
  return HALF_ERROR_UNAVAILABLE;
}

int half_escn_predict(const char*, const half_escn_request_v1*, half_escn_result_v1*, int, char* error, int cap) {
  clear_error(error, cap);
  export_error("DeePAW-eSCN density service is not part of this build", error, cap);
  return HALF_ERROR_UNAVAILABLE;
}

int half_create_from_files(const char* charge, const char* potential, double encut, int xc, int use_uspp,
                           half_handle* handle, char* error, int cap) {
  clear_error(error, cap);
  if (handle) *handle = 0;
  std::string c = cstr(charge), p = cstr(potential);
  if (c.empty() || p.empty() || (xc != 1 && xc != 2)) {
    export_error("invalid path or XC selector", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return create_context(c, p, encut, xc, use_uspp, HALF_BACKEND_AUTO, HALF_SOLVER_EVD, handle, error, cap);
}

int half_create_from_files_backend(const char* charge, const char* potential, double encut, int xc, int use_uspp,
                                   int backend, int solver, half_handle* handle, char* error, int cap) {
  clear_error(error, cap);
  if (handle) *handle = 0;
  std::string c = cstr(charge), p = cstr(potential);
  if (c.empty() || p.empty() || (xc != 1 && xc != 2) || backend < 0 || backend > 2 || solver < 1 || solver > 4) {
    export_error("invalid path, XC, backend, or solver selector", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return create_context(c, p, encut, xc, use_uspp, backend, solver, handle, error, cap);
}

int half_create_from_escn(const char* url, const char* potential, const half_request_geometry_v1* geometry, double,
                          int xc, int, int backend, int solver, int normalization, int, half_handle* handle,
                          char* error, int cap) {
  clear_error(error, cap);
  if (handle) *handle = 0;
  if (cstr(url).empty() || cstr(potential).empty() || !geometry || (xc != 1 && xc != 2) || backend < 0 ||
      backend > 2 || solver < 1 || solver > 4 || (normalization != 0 && normalization != 1)) {
    export_error("invalid eSCN URL, path, geometry, execution policy, or normalization", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  export_error("DeePAW-eSCN density service is not part of this build", error, cap);
  return HALF_ERROR_UNAVAILABLE;
}

int half_destroy(half_handle handle, char* error, int cap) {
  clear_error(error, cap);
  std::lock_guard<std::mutex> lock(g_mutex);
  int s = slot_of(handle);
  if (s < 0) return bad_handle(error, cap);
  return guarded(error, cap, [&]() -> int {
    g_slots[s].ctx.reset();
    g_slots[s].used = false;
    bool any = false;
    for (const auto& sl : g_slots) any = any || sl.used;
    if (!any) device_cache_release();   // last context gone: cached device blocks back to the driver
    return HALF_SUCCESS;
  });
}

int half_set_request_geometry(half_handle handle, const half_request_geometry_v1* g, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (!g) { export_error("request geometry pointer is required", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  if (g->struct_size < sizeof(half_request_geometry_v1) || g->flags != 0) {
    export_error("unsupported request geometry structure size or flags", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  if (g->nions < 1 || g->ntypes < 1 || !g->species || !g->positions_fractional) {
    export_error("request geometry arrays and positive dimensions are required", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  // src/half_library.F90:227-247
  if (g->grid[0] < 1 || g->grid[1] < 1 || g->grid[2] < 1) {
    export_error("invalid request geometry dimensions", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < g->nions; ++i)
    if (g->species[i] < 1 || g->species[i] > g->ntypes) {
      export_error("invalid request geometry values", error, cap);
      return HALF_ERROR_INVALID_ARGUMENT;
    }
  for (int i = 0; i < 9; ++i)
    if (std::isnan(g->lattice[i])) { export_error("invalid request geometry values", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  for (int i = 0; i < 3 * g->nions; ++i)
    if (std::isnan(g->positions_fractional[i])) {
      export_error("invalid request geometry values", error, cap);
      return HALF_ERROR_INVALID_ARGUMENT;
    }
  if (std::fabs(det3(g->lattice)) < 1.0e-12) { export_error("request lattice is singular", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  ctx->request_nions = g->nions;
  ctx->request_ntypes = g->ntypes;
  for (int i = 0; i < 3; ++i) ctx->request_grid[i] = g->grid[i];
  for (int i = 0; i < 9; ++i) ctx->request_lattice[i] = g->lattice[i];
  ctx->request_species.assign(g->species, g->species + g->nions);
  ctx->request_positions.assign(g->positions_fractional, g->positions_fractional + 3 * g->nions);
  ctx->has_request_geometry = true;
  return HALF_SUCCESS;
}

int half_get_request_geometry(half_handle handle, int32_t* nions, int32_t* ntypes, int32_t grid[3], double lattice[9],
                              int64_t species_capacity, int32_t* species, int64_t positions_capacity,
                              double* positions, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (!ctx->has_request_geometry) { export_error("request geometry has not been set", error, cap); return HALF_ERROR_UNAVAILABLE; }
  if (!nions || !ntypes) { export_error("nions and ntypes output pointers are required", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  *nions = ctx->request_nions;
  *ntypes = ctx->request_ntypes;
  if (grid) for (int i = 0; i < 3; ++i) grid[i] = ctx->request_grid[i];
  if (lattice) for (int i = 0; i < 9; ++i) lattice[i] = ctx->request_lattice[i];
  if (species) {
    if (species_capacity < ctx->request_nions) { export_error("request species output capacity is too small", error, cap); return HALF_ERROR_CAPACITY; }
    std::copy(ctx->request_species.begin(), ctx->request_species.end(), species);
  }
  if (positions) {
    if (positions_capacity < 3LL * ctx->request_nions) { export_error("request positions output capacity is too small", error, cap); return HALF_ERROR_CAPACITY; }
    std::copy(ctx->request_positions.begin(), ctx->request_positions.end(), positions);
  }
  return HALF_SUCCESS;
}

int half_get_system_info(half_handle handle, int* nions, int* ntypes, int grid[3], double lattice[9], double* volume,
                         char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nions) *nions = ctx->crystal.nions();
  if (ntypes) *ntypes = ctx->crystal.ntypes();
  if (grid) for (int i = 0; i < 3; ++i) grid[i] = ctx->charge.shape[i];
  if (lattice) for (int i = 0; i < 9; ++i) lattice[i] = ctx->crystal.lattice[i];
  if (volume) *volume = ctx->crystal.volume();
  return HALF_SUCCESS;
}

int half_get_basis_size(half_handle handle, const double kpoint[3], int64_t* npw, char* error, int cap) {
  clear_error(error, cap);
  if (npw) *npw = 0;
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  return guarded(error, cap, [&]() -> int {
    if (!finite3(kpoint)) fail(kInvalidArgument, "k point must be finite");
    Basis b = build_basis(ctx->crystal, ctx->charge.shape, ctx->encut, kpoint);
    if (npw) *npw = b.npw();
    return HALF_SUCCESS;
  });
}

int half_get_basis(half_handle handle, const double kpoint[3], int64_t capacity, int32_t* gvec, double* kinetic,
                   char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  return guarded(error, cap, [&]() -> int {
    if (!finite3(kpoint)) fail(kInvalidArgument, "k point must be finite");
    Basis b = build_basis(ctx->crystal, ctx->charge.shape, ctx->encut, kpoint);
    if (capacity < b.npw()) fail(kCapacity, "basis output capacity is too small");
    for (long long i = 0; i < b.npw(); ++i) {
      if (gvec) for (int j = 0; j < 3; ++j) gvec[3 * i + j] = b.gvec[3 * i + j];
      if (kinetic) kinetic[i] = b.kinetic[i];
    }
    return HALF_SUCCESS;
  });
}

int half_assemble_hs(half_handle handle, const double kpoint[3], int64_t ld, HALF_C128* h, HALF_C128* s, char* error,
                     int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (!h || !s) { export_error("H and S output pointers are required", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  return guarded(error, cap, [&]() -> int {
    if (!finite3(kpoint)) fail(kInvalidArgument, "k point must be finite");
    auto ks = prepare_operator(*ctx, *ctx->rt, kpoint, true, false);
    long long n = ks->basis.npw();
    if (ld < n) fail(kCapacity, "matrix leading dimension is too small");
    DeviceBuffer<double2> dh((size_t)n * n), ds((size_t)n * n);
    assemble_dense(*ctx, *ks, dh.get(), ds.get());
    cudaStream_t st = ctx->rt->stream;
    HALF_CUDA(cudaMemcpy2DAsync(h, ld * sizeof(double2), dh.get(), n * sizeof(double2), n * sizeof(double2), n,
                                cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaMemcpy2DAsync(s, ld * sizeof(double2), ds.get(), n * sizeof(double2), n * sizeof(double2), n,
                                cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaStreamSynchronize(st));
    return HALF_SUCCESS;
  });
}

int half_apply_hs(half_handle handle, const double kpoint[3], int nstates, int64_t ld, const HALF_C128* psi,
                  HALF_C128* hpsi, HALF_C128* spsi, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nstates < 1 || !psi || !hpsi || !spsi) { export_error("invalid state block arguments", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  return guarded(error, cap, [&]() -> int {
    if (!finite3(kpoint)) fail(kInvalidArgument, "k point must be finite");
    bool fp32 = ctx->acc.precision == kMixed;
    auto ks = prepare_operator(*ctx, *ctx->rt, kpoint, true, fp32);
    long long n = ks->basis.npw();
    if (ld < n) fail(kCapacity, "state leading dimension is too small");
    cudaStream_t st = ctx->rt->stream;
    DeviceBuffer<double2> x((size_t)n * nstates), hx((size_t)n * nstates), sx((size_t)n * nstates);
    HALF_CUDA(cudaMemcpy2DAsync(x.get(), n * sizeof(double2), psi, ld * sizeof(double2), n * sizeof(double2), nstates,
                                cudaMemcpyHostToDevice, st));
    ctx->last = SolveInfo();
    begin_call(*ctx->rt);
    if (fp32) {
      apply_hs_fp32(*ctx, *ks, x.get(), n, nstates, hx.get(), sx.get(), ctx->acc.block);
      tc_check(*ctx->rt);
    } else {
      apply_hs<double>(*ctx, *ks, x.get(), n, nstates, hx.get(), sx.get(), ctx->acc.block);
    }
    end_call(*ctx->rt, ctx->last);
    HALF_CUDA(cudaMemcpy2DAsync(hpsi, ld * sizeof(double2), hx.get(), n * sizeof(double2), n * sizeof(double2), nstates,
                                cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaMemcpy2DAsync(spsi, ld * sizeof(double2), sx.get(), n * sizeof(double2), n * sizeof(double2), nstates,
                                cudaMemcpyDeviceToHost, st));
    HALF_CUDA(cudaStreamSynchronize(st));
    return HALF_SUCCESS;
  });
}

int half_solve_kpoint(half_handle handle, const double kpoint[3], int nbands, double* eigenvalues, HALF_C128* vectors,
                      int64_t ld, double* overlap_min, double* overlap_max, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nbands < 1) { export_error("band count must be positive", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  return guarded(error, cap, [&]() -> int {
    SolveOutput out;
    out.keep_device = vectors != nullptr;   // copied out below with the caller's leading dimension
    std::unique_ptr<KOperatorSet> ks;
    solve_one(*ctx, kpoint, nbands, false, out, &ks);
    long long n = ks->basis.npw();
    if (vectors && ld < n) fail(kCapacity, "eigenvector leading dimension is too small");
    if (eigenvalues) std::copy(out.eigenvalues.begin(), out.eigenvalues.end(), eigenvalues);
    if (overlap_min) *overlap_min = out.overlap_min;
    if (overlap_max) *overlap_max = out.overlap_max;
    if (vectors) {
      cudaStream_t st = ctx->rt->stream;
      HALF_CUDA(cudaMemcpy2DAsync(vectors, ld * sizeof(double2), out.dvectors.get(), n * sizeof(double2),
                                  n * sizeof(double2), nbands, cudaMemcpyDeviceToHost, st));
      HALF_CUDA(cudaStreamSynchronize(st));
    }
    return HALF_SUCCESS;
  });
}

namespace {
int g_hash(int32_t gx, int32_t gy, int32_t gz, int table_size) {   // src/half_c_api.F90:590-597 (0-based)
  long long v = (long long)gx * 73856093LL + (long long)gy * 19349663LL + (long long)gz * 83492791LL;
  long long m = v % table_size;
  if (m < 0) m += table_size;
  return int(m);
}
}  // namespace

int half_solve_kpoint_mapped(half_handle handle, const double kpoint[3], int nbands, int64_t host_npw,
                             const int32_t* host_gvec, double* eigenvalues, HALF_C128* vectors, int64_t ld,
                             double* overlap_min, double* overlap_max, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nbands < 1 || host_npw < 1 || ld < host_npw || !vectors || !host_gvec) {
    export_error("invalid mapped-solve band count, basis size, leading dimension, or output pointer", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    SolveOutput out;
    out.keep_device = true;   // the permutation runs on the device
    std::unique_ptr<KOperatorSet> ks;
    solve_one(*ctx, kpoint, nbands, false, out, &ks);
    const Basis& b = ks->basis;
    long long n = b.npw();
    if (host_npw != n) fail(kInvalidArgument, "host and HALF plane-wave bases have different sizes");
    int table_size = 1;
    while (table_size < 2 * n) table_size *= 2;
    std::vector<int> table(table_size, -1);
    for (long long hi = 0; hi < n; ++hi) {
      int p = g_hash(host_gvec[3 * hi], host_gvec[3 * hi + 1], host_gvec[3 * hi + 2], table_size);
      while (table[p] >= 0) {
        int i = table[p];
        if (host_gvec[3 * i] == host_gvec[3 * hi] && host_gvec[3 * i + 1] == host_gvec[3 * hi + 1] &&
            host_gvec[3 * i + 2] == host_gvec[3 * hi + 2])
          fail(kInvalidArgument, "host G-vector list contains a duplicate");
        p = (p + 1) % table_size;
      }
      table[p] = int(hi);
    }
    std::vector<int> src_row(n);   // host row perm[i] takes HALF row i
    for (long long i = 0; i < n; ++i) {
      int p = g_hash(b.gvec[3 * i], b.gvec[3 * i + 1], b.gvec[3 * i + 2], table_size), hit = -1;
      while (table[p] >= 0) {
        int j = table[p];
        if (host_gvec[3 * j] == b.gvec[3 * i] && host_gvec[3 * j + 1] == b.gvec[3 * i + 1] &&
            host_gvec[3 * j + 2] == b.gvec[3 * i + 2]) { hit = j; break; }
        p = (p + 1) % table_size;
      }
      if (hit < 0) fail(kInvalidArgument, "host and HALF plane-wave bases contain different G vectors");
      src_row[hit] = int(i);
    }
    gather_rows_to_host(*ctx->rt, out.dvectors.get(), n, nbands, src_row, ld, reinterpret_cast<double2*>(vectors));
    if (eigenvalues) std::copy(out.eigenvalues.begin(), out.eigenvalues.end(), eigenvalues);
    if (overlap_min) *overlap_min = out.overlap_min;
    if (overlap_max) *overlap_max = out.overlap_max;
    return HALF_SUCCESS;
  });
}

// ------------------------------------------------------------- extensions

int half_set_acc_controls(half_handle handle, double tol, int max_iterations, int block_size, int precision,
                          char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (!(tol > 0) || !std::isfinite(tol) || max_iterations < 1 || block_size < 0 ||
      (precision != HALF_PRECISION_FP64 && precision != HALF_PRECISION_MIXED &&
       precision != HALF_PRECISION_FP64_GUARDED)) {
    export_error("invalid ACC solver controls", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  ctx->acc.tol = tol;
  ctx->acc.max_iter = max_iterations;
  ctx->acc.block = block_size;
  ctx->acc.precision = precision;
  return HALF_SUCCESS;
}

int half_get_last_solve_info(half_handle handle, half_solve_info_v1* info, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (!info || info->struct_size < sizeof(half_solve_info_v1)) {
    export_error("solve info structure is missing or too small", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  const SolveInfo& s = ctx->last;
  info->iterations = s.iterations;
  info->fp64_iterations = s.fp64_iterations;
  info->converged = s.converged;
  info->npw = s.npw;
  info->operator_applications = s.operator_columns;
  info->max_residual_eV = s.max_residual;
  info->setup_ms = s.setup_ms;
  info->solve_ms = s.solve_ms;
  info->operator_ms = s.operator_ms;
  info->device_ms = s.device_ms;
  info->local_ms = s.local_ms;
  info->local_bytes = s.local_bytes;
  info->local_columns = s.local_columns;
  info->kernel_launches = s.launches;
  info->sweep_ms = s.sweep_ms;
  info->sweep_columns = s.sweep_columns;
  info->adjoint_ms = s.adjoint_ms;
  info->tensor_ms = s.tensor_ms;
  info->tensor_flops = s.tensor_flops;
  info->tensor_launches = s.tensor_launches;
  std::memset(info->reserved, 0, sizeof(info->reserved));
  return HALF_SUCCESS;
}

}  // extern "C"

namespace {

// Solve nk independent k points, up to ctx.kpoint_workers of them at a time,
// each worker on its own stream with its own cuBLAS/cuSOLVER handles (one k
// point's host-side solver latency overlaps another's device work).  sink(ik,
// out, rt) runs on the worker that solved k point ik, before its next solve;
// device work it enqueues on rt.stream is complete when this returns.
template <typename Sink>
void solve_batch(Context& ctx, int nk, const double* kpoints, int nbands, bool keep_device, Sink sink) {
  const int workers = std::max(1, std::min(nk, ctx.kpoint_workers));
  while ((int)ctx.workers.size() < workers - 1) ctx.workers.push_back(std::make_unique<Runtime>());
  std::vector<SolveInfo> infos(nk);
  std::vector<std::string> errors(workers);
  std::vector<int> codes(workers, 0);
  HALF_CUDA(cudaDeviceSynchronize());
  cudaEvent_t t0;
  HALF_CUDA(cudaEventCreate(&t0));
  HALF_CUDA(cudaEventRecord(t0, ctx.rt->stream));
  std::vector<cudaEvent_t> ends(workers);
  for (auto& e : ends) HALF_CUDA(cudaEventCreate(&e));
  auto body = [&](int w) {
    Runtime& rt = w == 0 ? *ctx.rt : *ctx.workers[w - 1];
    try {
      for (int ik = w; ik < nk; ik += workers) {
        SolveOutput out;
        out.keep_device = keep_device;
        solve_one(ctx, rt, kpoints + 3 * ik, nbands, false, out, infos[ik]);
        sink(ik, out, rt);
      }
    } catch (const Error& e) {
      codes[w] = e.status;
      errors[w] = e.what();
    } catch (const std::exception& e) {
      codes[w] = HALF_ERROR_INTERNAL;
      errors[w] = e.what();
    }
    cudaEventRecord(ends[w], rt.stream);
  };
  if (workers == 1) {
    body(0);
  } else {
    std::vector<std::thread> pool;
    for (int w = 0; w < workers; ++w) pool.emplace_back(body, w);
    for (auto& t : pool) t.join();
  }
  float span = 0;
  for (int w = 0; w < workers; ++w) {
    HALF_CUDA(cudaEventSynchronize(ends[w]));
    float ms = 0;
    HALF_CUDA(cudaEventElapsedTime(&ms, t0, ends[w]));
    span = std::max(span, ms);
    cudaEventDestroy(ends[w]);
  }
  cudaEventDestroy(t0);
  for (int w = 0; w < workers; ++w)
    if (codes[w] != 0) fail(codes[w], errors[w]);
  SolveInfo total;
  for (int ik = 0; ik < nk; ++ik) accumulate(total, infos[ik], ik == 0);
  total.device_ms = span;   // wall span on the device of the whole batch
  ctx.last = total;
}

bool device_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" {

int half_solve_kpoints(half_handle handle, int nk, const double* kpoints, int nbands, double* eigenvalues, char* error,
                       int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nk < 1 || !kpoints || nbands < 1 || !eigenvalues) {
    export_error("invalid k-point batch arguments", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    solve_batch(*ctx, nk, kpoints, nbands, false, [&](int ik, SolveOutput& out, Runtime&) {
      std::copy(out.eigenvalues.begin(), out.eigenvalues.end(), eigenvalues + (size_t)ik * nbands);
    });
    return HALF_SUCCESS;
  });
}

int half_solve_kpoints_device(half_handle handle, int nk, const double* kpoints, int nbands,
                              double* eigenvalues_device, HALF_C128* vectors_device, int64_t ld, char* error,
                              int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nk < 1 || !kpoints || nbands < 1 || !eigenvalues_device || (vectors_device && ld < 1)) {
    export_error("invalid k-point batch arguments", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    if (!device_pointer(eigenvalues_device) || (vectors_device && !device_pointer(vectors_device)))
      fail(kInvalidArgument, "eigenvalue and eigenvector buffers must be device memory");
    if (vectors_device)
      for (int ik = 0; ik < nk; ++ik) {
        if (!finite3(kpoints + 3 * ik)) fail(kInvalidArgument, "k point must be finite");
        if (build_basis(ctx->crystal, ctx->charge.shape, ctx->encut, kpoints + 3 * ik).npw() > ld)
          fail(kCapacity, "eigenvector leading dimension is smaller than a k point's basis");
      }
    double2* vec = reinterpret_cast<double2*>(vectors_device);
    solve_batch(*ctx, nk, kpoints, nbands, vectors_device != nullptr, [&](int ik, SolveOutput& out, Runtime& rt) {
      HALF_CUDA(cudaMemcpyAsync(eigenvalues_device + (size_t)ik * nbands, out.eigenvalues.data(),
                                size_t(nbands) * sizeof(double), cudaMemcpyHostToDevice, rt.stream));
      if (!vec) return;
      const size_t npw = out.dvectors.size() / size_t(nbands);
      double2* dst = vec + (size_t)ik * ld * nbands;
      HALF_CUDA(cudaMemcpy2DAsync(dst, ld * sizeof(double2), out.dvectors.get(), npw * sizeof(double2),
                                  npw * sizeof(double2), nbands, cudaMemcpyDeviceToDevice, rt.stream));
      if ((size_t)ld > npw)
        HALF_CUDA(cudaMemset2DAsync(dst + npw, ld * sizeof(double2), 0, (ld - npw) * sizeof(double2), nbands,
                                    rt.stream));
    });
    return HALF_SUCCESS;
  });
}

int half_set_positions(half_handle handle, const double* positions, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (!positions) { export_error("positions pointer is required", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  return guarded(error, cap, [&]() -> int {
    int n = ctx->crystal.nions();
    for (int i = 0; i < 3 * n; ++i)
      if (!std::isfinite(positions[i])) fail(kInvalidArgument, "positions must be finite");
    ctx->crystal.positions.assign(positions, positions + 3 * n);
    ctx->rebuild_dij();
    return HALF_SUCCESS;
  });
}

int half_set_positions_noalloc(half_handle handle, const double* positions, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (!positions) { export_error("positions pointer is required", error, cap); return HALF_ERROR_INVALID_ARGUMENT; }
  return guarded(error, cap, [&]() -> int {
    int n = ctx->crystal.nions();
    for (int i = 0; i < 3 * n; ++i)
      if (!std::isfinite(positions[i])) fail(kInvalidArgument, "positions must be finite");
    ctx->rebuild_dij_fixed_scratch(true);   // capacity errors leave the context unchanged
    // The rebuild stages the new D_ij and commits it only after every species
    // succeeded; on any error the old positions come back with it.
    std::vector<double> old = ctx->crystal.positions;
    ctx->crystal.positions.assign(positions, positions + 3 * n);
    try {
      ctx->rebuild_dij_fixed_scratch(false);
    } catch (...) {
      ctx->crystal.positions = std::move(old);
      throw;
    }
    return HALF_SUCCESS;
  });
}

int half_nonlocal_forces(half_handle handle, const double kpoint[3], int nbands, int64_t ld, const HALF_C128* vectors,
                         const double* eigenvalues, const double* occupations, double kweight, double* forces,
                         char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nbands < 1 || !vectors || !eigenvalues || !occupations || !forces) {
    export_error("invalid force arguments", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    if (!finite3(kpoint)) fail(kInvalidArgument, "k point must be finite");
    auto ks = prepare_operator(*ctx, *ctx->rt, kpoint, true, false);
    long long n = ks->basis.npw();
    if (ld < n) fail(kCapacity, "eigenvector leading dimension is too small");
    cudaStream_t st = ctx->rt->stream;
    DeviceBuffer<double2> dv((size_t)n * nbands);
    HALF_CUDA(cudaMemcpy2DAsync(dv.get(), n * sizeof(double2), vectors, ld * sizeof(double2), n * sizeof(double2),
                                nbands, cudaMemcpyHostToDevice, st));
    ctx->last = SolveInfo();
    begin_call(*ctx->rt);
    nonlocal_forces_device(*ctx, *ks, dv.get(), n, nbands, eigenvalues, occupations, kweight, forces);
    end_call(*ctx->rt, ctx->last);
    return HALF_SUCCESS;
  });
}

}  // extern "C"

// occupations (src/half_energy.F90:41-120), shared with half_band_forces
namespace hb {
void compute_occupations(const std::vector<double>& eig, int nk, int nb, const double* w, double nelect, double sigma,
                         int ismear, std::vector<double>& occ, double& mu, double& band, double& entropy);
}

extern "C" int half_band_forces(half_handle handle, int nk, const double* kpoints, const double* kweights, int nbands,
                                double nelect, double sigma, int ismear, double* forces, double* eig_out,
                                double* occ_out, double* energies, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nk < 1 || !kpoints || !kweights || nbands < 1 || !forces || !(sigma >= 0) || (ismear != -1 && ismear != 0)) {
    export_error("invalid band-force arguments", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    std::vector<SolveOutput> outs(nk);
    std::vector<std::unique_ptr<KOperatorSet>> ops(nk);   // each solve's operator, reused by its force
    std::vector<double> eig((size_t)nk * nbands);
    for (int ik = 0; ik < nk; ++ik) {
      outs[ik].keep_device = true;   // the force needs the eigenvectors on the device
      solve_one(*ctx, kpoints + 3 * ik, nbands, false, outs[ik], &ops[ik]);
      std::copy(outs[ik].eigenvalues.begin(), outs[ik].eigenvalues.end(), eig.begin() + (size_t)ik * nbands);
    }
    std::vector<double> occ;
    double mu = 0, band = 0, entropy = 0;
    compute_occupations(eig, nk, nbands, kweights, nelect, sigma, ismear, occ, mu, band, entropy);
    int nions = ctx->crystal.nions();
    std::fill(forces, forces + 3 * nions, 0.0);
    for (int ik = 0; ik < nk; ++ik) {
      KOperatorSet& ks = *ops[ik];
      nonlocal_forces_device(*ctx, ks, outs[ik].dvectors.get(), ks.basis.npw(), nbands, eig.data() + (size_t)ik * nbands,
                             occ.data() + (size_t)ik * nbands, kweights[ik], forces);
      ops[ik].reset();
    }
    if (eig_out) std::copy(eig.begin(), eig.end(), eig_out);
    if (occ_out) std::copy(occ.begin(), occ.end(), occ_out);
    if (energies) { energies[0] = band; energies[1] = entropy; energies[2] = mu; }
    return HALF_SUCCESS;
  });
}

extern "C" int half_ionic_forces(half_handle handle, const double* output_density, int64_t n, double* ewald,
                                 double* local, double* nlcc, double* harris, double* energies, char* error,
                                 int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (output_density && n != ctx->nr()) {
    export_error("output density size does not match the context's grid", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    const bool dens_dev = output_density && device_pointer(output_density);
    if (output_density && !dens_dev)
      for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(output_density[i])) fail(kInvalidArgument, "output density must be finite");
    IonicForces f;
    ctx->last = SolveInfo();
    begin_call(*ctx->rt);
    ionic_forces_device(*ctx, output_density, dens_dev, ewald || energies, local || energies, nlcc != nullptr,
                        harris != nullptr, f);
    end_call(*ctx->rt, ctx->last);
    if (ewald) std::copy(f.ewald.begin(), f.ewald.end(), ewald);
    if (local) std::copy(f.local.begin(), f.local.end(), local);
    if (nlcc) std::copy(f.nlcc.begin(), f.nlcc.end(), nlcc);
    if (harris) std::copy(f.harris.begin(), f.harris.end(), harris);
    if (energies) {
      std::copy(f.ewald_energy, f.ewald_energy + 5, energies);
      energies[5] = f.local_energy;
    }
    return HALF_SUCCESS;
  });
}

extern "C" int half_output_density(half_handle handle, int nk, const double* kpoints, const double* kweights,
                                   int nbands, int64_t ld, const HALF_C128* vectors, const double* occupations,
                                   double* density, int64_t n, double* augmentation_charge, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nk < 1 || !kpoints || !kweights || nbands < 1 || !vectors || !occupations || !density) {
    export_error("invalid output-density arguments", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  if (n != ctx->nr()) {
    export_error("density size does not match the context's grid", error, cap);
    return HALF_ERROR_CAPACITY;
  }
  return guarded(error, cap, [&]() -> int {
    for (int ik = 0; ik < nk; ++ik)
      if (!finite3(kpoints + 3 * ik)) fail(kInvalidArgument, "k point must be finite");
    cudaStream_t st = ctx->rt->stream;
    const bool vec_dev = device_pointer(vectors);   // device eigenvectors are read in place
    std::vector<DeviceBuffer<double2>> dv(nk);
    std::vector<const double2*> ptr(nk);
    std::vector<long long> lds(nk);
    for (int ik = 0; ik < nk; ++ik) {
      const Basis b = build_basis(ctx->crystal, ctx->charge.shape, ctx->encut, kpoints + 3 * ik);
      const long long npw = b.npw();
      if (ld < npw) fail(kCapacity, "eigenvector leading dimension is too small");
      const double2* src = reinterpret_cast<const double2*>(vectors) + (size_t)ik * ld * nbands;
      if (vec_dev) {
        ptr[ik] = src;
        lds[ik] = ld;
        continue;
      }
      dv[ik].resize((size_t)npw * nbands);
      HALF_CUDA(cudaMemcpy2DAsync(dv[ik].get(), npw * sizeof(double2), src, ld * sizeof(double2),
                                  npw * sizeof(double2), nbands, cudaMemcpyHostToDevice, st));
      ptr[ik] = dv[ik].get();
      lds[ik] = npw;
    }
    DeviceBuffer<double> out(ctx->nr());
    double aug = 0;
    ctx->last = SolveInfo();
    begin_call(*ctx->rt);
    output_density_device(*ctx, nk, kpoints, kweights, nbands, ptr, lds, occupations, out.get(), &aug);
    end_call(*ctx->rt, ctx->last);
    HALF_CUDA(cudaMemcpyAsync(density, out.get(), sizeof(double) * n, cudaMemcpyDefault, st));
    HALF_CUDA(cudaStreamSynchronize(st));
    if (augmentation_charge) *augmentation_charge = aug;
    return HALF_SUCCESS;
  });
}

extern "C" int half_forces(half_handle handle, int nk, const double* kpoints, const double* kweights, int nbands,
                           double nelect, double sigma, int ismear, double* forces, double* components,
                           double* output_density, double* energies, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nk < 1 || !kpoints || !kweights || nbands < 1 || !forces || !(sigma >= 0) || (ismear != -1 && ismear != 0)) {
    export_error("invalid force arguments", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    std::vector<SolveOutput> outs(nk);
    std::vector<std::unique_ptr<KOperatorSet>> ops(nk);   // each solve's operator, reused by its force
    std::vector<double> eig((size_t)nk * nbands);
    for (int ik = 0; ik < nk; ++ik) {
      outs[ik].keep_device = true;
      solve_one(*ctx, kpoints + 3 * ik, nbands, false, outs[ik], &ops[ik]);
      std::copy(outs[ik].eigenvalues.begin(), outs[ik].eigenvalues.end(), eig.begin() + (size_t)ik * nbands);
    }
    std::vector<double> occ;
    double mu = 0, band = 0, entropy = 0;
    compute_occupations(eig, nk, nbands, kweights, nelect, sigma, ismear, occ, mu, band, entropy);
    if (sigma > 0)   // app/half_cli.F90:897
      for (int ik = 0; ik < nk; ++ik)
        if (occ[(size_t)ik * nbands + nbands - 1] > 1e-6)
          fail(kInvalidArgument, "highest computed band is occupied; increase nbands");
    const int nions = ctx->crystal.nions();
    std::vector<double> nonlocal(3 * (size_t)nions, 0.0);
    std::vector<const double2*> ptr(nk);
    std::vector<long long> lds(nk);
    for (int ik = 0; ik < nk; ++ik) {
      KOperatorSet& ks = *ops[ik];
      nonlocal_forces_device(*ctx, ks, outs[ik].dvectors.get(), ks.basis.npw(), nbands,
                             eig.data() + (size_t)ik * nbands, occ.data() + (size_t)ik * nbands, kweights[ik],
                             nonlocal.data());
      ptr[ik] = outs[ik].dvectors.get();
      lds[ik] = ks.basis.npw();
      ops[ik].reset();
    }
    const long long n = ctx->nr();
    DeviceBuffer<double> rho_out(n);
    double aug = 0;
    output_density_device(*ctx, nk, kpoints, kweights, nbands, ptr, lds, occ.data(), rho_out.get(), &aug);
    IonicForces f;
    ionic_forces_device(*ctx, rho_out.get(), true, true, true, true, true, f);
    for (int i = 0; i < 3 * nions; ++i) forces[i] = f.ewald[i] + f.local[i] + nonlocal[i] + f.nlcc[i] + f.harris[i];
    if (components) {
      const std::vector<double>* parts[5] = {&f.ewald, &f.local, &nonlocal, &f.nlcc, &f.harris};
      for (int c = 0; c < 5; ++c) std::copy(parts[c]->begin(), parts[c]->end(), components + (size_t)c * 3 * nions);
    }
    if (output_density) {
      HALF_CUDA(cudaMemcpyAsync(output_density, rho_out.get(), sizeof(double) * n, cudaMemcpyDeviceToHost,
                                ctx->rt->stream));
      HALF_CUDA(cudaStreamSynchronize(ctx->rt->stream));
    }
    if (energies) {
      energies[0] = band;
      energies[1] = entropy;
      energies[2] = mu;
      energies[3] = f.ewald_energy[0];
      energies[4] = f.local_energy;
      energies[5] = aug;
    }
    return HALF_SUCCESS;
  });
}

extern "C" int half_pack_vasp_waves(half_handle handle, int nk, const double* kpoints, int nbands, int64_t ld,
                                    const HALF_C128* vectors, float* packed, int64_t capacity, int* npws,
                                    int64_t* offsets, char* error, int cap) {
  clear_error(error, cap);
  Context* ctx = lookup(handle);
  if (!ctx) return bad_handle(error, cap);
  if (nk < 1 || !kpoints || nbands < 1 || !npws || !offsets || (packed && !vectors) || capacity < 0) {
    export_error("invalid wave-export arguments", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    std::vector<Basis> bases;
    int64_t total = 0;
    for (int ik = 0; ik < nk; ++ik) {
      if (!finite3(kpoints + 3 * ik)) fail(kInvalidArgument, "k point must be finite");
      bases.push_back(build_basis(ctx->crystal, ctx->charge.shape, ctx->encut, kpoints + 3 * ik));
      if (bases.back().npw() > ld) fail(kCapacity, "eigenvector leading dimension is smaller than a k point's basis");
      npws[ik] = int(bases.back().npw());
      offsets[ik] = total;
      total += 2 * int64_t(npws[ik]) * nbands;
    }
    if (!packed) return HALF_SUCCESS;   // size query
    if (capacity < total) fail(kCapacity, "packed buffer is smaller than 2 * nbands * sum(npw)");
    Runtime& rt = *ctx->rt;
    cudaStream_t st = rt.stream;
    const bool vec_dev = device_pointer(vectors), out_dev = device_pointer(packed);
    ctx->last = SolveInfo();
    begin_call(rt);
    for (int ik = 0; ik < nk; ++ik) {
      const int npw = npws[ik];
      const double2* src = reinterpret_cast<const double2*>(vectors) + (size_t)ik * ld * nbands;
      DeviceBuffer<double2> dv;
      long long sld = ld;
      if (!vec_dev) {
        dv.resize((size_t)npw * nbands);
        HALF_CUDA(cudaMemcpy2DAsync(dv.get(), npw * sizeof(double2), src, ld * sizeof(double2), npw * sizeof(double2),
                                    nbands, cudaMemcpyHostToDevice, st));
        src = dv.get();
        sld = npw;
      }
      float2* dst = reinterpret_cast<float2*>(packed + offsets[ik]);
      DeviceBuffer<float2> dout;
      if (!out_dev) {
        dout.resize((size_t)npw * nbands);
        dst = dout.get();
      }
      pack_vasp_device(rt, src, sld, npw, nbands, vasp_order(bases[ik]), dst);
      if (!out_dev) {
        HALF_CUDA(cudaMemcpyAsync(packed + offsets[ik], dout.get(), sizeof(float2) * npw * nbands,
                                  cudaMemcpyDeviceToHost, st));
        HALF_CUDA(cudaStreamSynchronize(st));
      }
    }
    end_call(rt, ctx->last);
    return HALF_SUCCESS;
  });
}

extern "C" int half_occupations(int nk, int nbands, const double* eigenvalues, const double* kweights, double nelect,
                                double sigma, int ismear, double* occupations, double* energies, char* error,
                                int cap) {
  clear_error(error, cap);
  if (nk < 1 || nbands < 1 || !eigenvalues || !kweights || !occupations) {
    export_error("invalid occupation arguments", error, cap);
    return HALF_ERROR_INVALID_ARGUMENT;
  }
  return guarded(error, cap, [&]() -> int {
    for (long long i = 0; i < (long long)nk * nbands; ++i)
      if (!std::isfinite(eigenvalues[i])) fail(kInvalidArgument, "eigenvalues must be finite");
    std::vector<double> eig(eigenvalues, eigenvalues + (size_t)nk * nbands), occ;
    double mu = 0, band = 0, entropy = 0;
    compute_occupations(eig, nk, nbands, kweights, nelect, sigma, ismear, occ, mu, band, entropy);
    std::copy(occ.begin(), occ.end(), occupations);
    if (energies) {
      energies[0] = band;
      energies[1] = entropy;
      energies[2] = mu;
    }
    return HALF_SUCCESS;
  });
}

// ---- diagnostic: the tensor-core complex GEMM on caller device memory
namespace {

std::mutex g_diag_mutex;

// One runtime (stream + handles) per device for diagnostic calls; kept for
// the life of the process.
Runtime& diagnostic_runtime() {
  static Runtime* rts[64] = {};
  int dev = 0;
  HALF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) fail(kInternal, "device ordinal out of range");
  if (!rts[dev]) rts[dev] = new Runtime();
  return *rts[dev];
}

bool gemm_op(char c, cublasOperation_t& op) {
  switch (c) {
    case 'N': case 'n': op = CUBLAS_OP_N; return true;
    case 'T': case 't': op = CUBLAS_OP_T; return true;
    case 'C': case 'c': op = CUBLAS_OP_C; return true;
    default: return false;
  }
}

}  // namespace

extern "C" int half_tc_cgemm(char op_a, char op_b, int m, int n, int k, const double* alpha, const float* a,
                             int64_t lda, const float* b, int64_t ldb, const double* beta, void* c, int64_t ldc,
                             int c_fp64, char* error, int cap) {
  clear_error(error, cap);
  return guarded(error, cap, [&]() -> int {
    cublasOperation_t ta, tb;
    if (!gemm_op(op_a, ta) || !gemm_op(op_b, tb)) fail(kInvalidArgument, "operation must be 'N', 'T' or 'C'");
    if (m < 0 || n < 0 || k < 0 || !alpha || !beta) fail(kInvalidArgument, "invalid GEMM dimensions or scalars");
    if (m == 0 || n == 0) return HALF_SUCCESS;
    const long long arows = ta == CUBLAS_OP_N ? m : k, brows = tb == CUBLAS_OP_N ? k : n;
    if (lda < std::max(1LL, arows) || ldb < std::max(1LL, brows) || ldc < m)
      fail(kCapacity, "leading dimension is too small");
    if ((k > 0 && (!device_pointer(a) || !device_pointer(b))) || !device_pointer(c))
      fail(kInvalidArgument, "operands must be device memory");
    std::lock_guard<std::mutex> lock(g_diag_mutex);
    Runtime& rt = diagnostic_runtime();
    rt.prof.reset();   // the profiler's events are reused call after call
    const float2* A = reinterpret_cast<const float2*>(a);
    const float2* B = reinterpret_cast<const float2*>(b);
    tc_cgemm(rt, tc_dense_a(ta, A, lda, m, k), tc_dense_b(tb, B, ldb, k, n), m, n, k, make_double2(alpha[0], alpha[1]),
             make_double2(beta[0], beta[1]), c, c_fp64 != 0, ldc);
    tc_check(rt);
    return HALF_SUCCESS;
  });
}

extern "C" int half_get_allocation_counts(int64_t* requests, int64_t* driver_allocations, char* error, int cap) {
  clear_error(error, cap);
  long long r = 0, d = 0;
  device_alloc_counts(&r, &d);
  if (requests) *requests = r;
  if (driver_allocations) *driver_allocations = d;
  return HALF_SUCCESS;
}
