/* Additive extensions to libhalf ABI v1 (B200 build).
 *
 * None of these symbols exists in the reference; they are the "additive
 * extensions" its docs/API.md:111-112 anticipates.  Each comment names the
 * reference routine whose behaviour the call exposes.  All calls follow the
 * ABI v1 conventions of half.h (status return, caller-owned buffers, error
 * buffer cleared on entry, complex128 column-major).
 */
#ifndef DEEPAW_HALF_B200_H
#define DEEPAW_HALF_B200_H

#include "half.h"

#ifdef __cplusplus
extern "C" {
#endif

enum half_precision {
  HALF_PRECISION_FP64 = 0,         /* the reference's iteration, every step in FP64 */
  HALF_PRECISION_MIXED = 1,        /* FP32 operator / tensor-core GEMMs, FP64 refinement,
                                      guard bands */
  HALF_PRECISION_FP64_GUARDED = 2  /* FP64 throughout, with guard bands */
};
/* Guard bands: the block carries m/4 extra bands (at least 4, within NPL/2)
 * and convergence is decided on the requested m.  Without them the block
 * iteration converges on the last requested band at the rate set by its gap
 * to the first unrequested one, and when the band count cuts a degenerate
 * level it can converge to a higher level than the m-th eigenvalue (the
 * residual test accepts any converged eigenpairs); the reference's iteration
 * has the same property. */

/* ACC controls.  The reference's solve_block_harris_cuda_full takes
 * tolerance / max_iterations / block_size (src/half_cuda_iterative_solver.cuf:
 * 113-119; CLI --acc-tol, --acc-max-iter, --acc-block-size) but ABI v1 never
 * passes them, so the defaults 1e-4 eV / 40 / 16 apply (src/half_library.F90:
 * 343-367).  This setter keeps those defaults until it is called.
 * tolerance_eV > 0, max_iterations >= 1, block_size >= 0, precision one of
 * half_precision; otherwise HALF_ERROR_INVALID_ARGUMENT.  block_size is the
 * operator's bands per chunk; 0 (this library's default) lets its
 * autotuner choose it by measurement, which changes no result. */
int half_set_acc_controls(half_handle handle, double tolerance_eV,
                          int max_iterations, int block_size, int precision,
                          char *error, int error_capacity);

/* Diagnostics of the last device call on this context (solve, H/S
 * application or force); the reference reports the solver figures through its
 * CLI JSON: iterative_solver_iterations, final residual, phase seconds
 * (app/half_cli.F90:306-349).  Event times are measured on the library's
 * CUDA stream. */
typedef struct half_solve_info_v1 {
  uint32_t struct_size;        /* set to sizeof(half_solve_info_v1) */
  int32_t iterations;          /* ACC iterations (all phases) */
  int32_t fp64_iterations;     /* of which in the FP64 refinement phase */
  int32_t converged;           /* 1 when max residual <= tolerance */
  int64_t npw;
  int64_t operator_applications;  /* band-columns pushed through H/S */
  double max_residual_eV;
  double setup_ms;             /* basis, projectors, operator tables */
  double solve_ms;             /* iterations through eigenpairs */
  double operator_ms;          /* time inside H/S applications */
  double device_ms;            /* CUDA-event span on the library stream */
  double local_ms;             /* CUDA-event time of the local-operator kernels */
  double local_bytes;          /* their algorithmic bytes (FFT-path figure per band) */
  int64_t local_columns;       /* band columns through the local operator */
  int64_t kernel_launches;     /* library kernels launched by the call */
  double sweep_ms;             /* CUDA-event time of whole H/S applications */
  int64_t sweep_columns;       /* band columns of those applications */
  double adjoint_ms;           /* CUDA-event time of the force adjoint (GEMM + epilogue) */
  double tensor_ms;            /* CUDA-event time of the tensor-core GEMM kernels */
  double tensor_flops;         /* their bf16 tensor flops: 24 per complex multiply-add
                                  (four real products, three split terms) */
  int64_t tensor_launches;     /* tensor-core GEMM kernel launches */
  uint64_t reserved[1];
} half_solve_info_v1;
int half_get_last_solve_info(half_handle handle, half_solve_info_v1 *info,
                             char *error, int error_capacity);

/* Solve several k points in one call (eigenvalues only, row-major
 * [ik][band]).  Same per-k algorithm as half_solve_kpoint; the k points are
 * independent units (the reference distributes them cyclically over MPI
 * ranks, src/half_parallel.F90:62-65). */
int half_solve_kpoints(half_handle handle, int nk, const double *kpoints,
                       int nbands, double *eigenvalues_eV,
                       char *error, int error_capacity);

/* Batched solve with device-resident outputs: the additive "batched multi-k
 * solve on device pointers" for callers that keep the eigenpairs on the GPU
 * (no counterpart in ABI v1).  eigenvalues_device: device memory, nk x nbands
 * (row-major [ik][band]).  vectors_device: device memory or NULL (values
 * only); k point ik's eigenvectors are the column-major block at
 * vectors_device + ik * ld * nbands, npw_k rows used and rows npw_k .. ld-1
 * zeroed.  ld must be at least every k point's basis size, else
 * HALF_ERROR_CAPACITY; host pointers give HALF_ERROR_INVALID_ARGUMENT.  The
 * buffers are complete when the call returns.  Same per-k algorithm and
 * concurrency as half_solve_kpoints. */
int half_solve_kpoints_device(half_handle handle, int nk, const double *kpoints,
                              int nbands, double *eigenvalues_device,
                              HALF_C128 *vectors_device, int64_t ld,
                              char *error, int error_capacity);

/* Move the atoms at fixed Veff (positions fractional, atom-major, in the
 * context's type-major order).  Rebuilds the MIMIC_US D_ij and dD_ij/dR
 * (src/half_uspp.F90:137-241) and, at the next solve, the projector phases
 * (src/half_paw.F90:52-65).  This is the perturbation the finite-difference
 * force oracle applies. */
int half_set_positions(half_handle handle, const double *positions_fractional,
                       char *error, int error_capacity);

/* half_set_positions without device allocation (no counterpart in the
 * reference).  For callers that must not allocate device memory in this call:
 * a relaxation or MD driver that has reserved the rest of HBM for its own
 * pool, or that keeps other streams busy and cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree.  Results are identical to
 * half_set_positions.
 * Scratch: one fixed 32 MiB device array inside the library, shared by every
 * handle on a device.  It must hold 24 bytes per grid point, the new D_ij and
 * dD_ij/dR (32 bytes per atom and projector pair) and one atom's QDEP samples
 * (about 1.5 MB); larger systems get HALF_ERROR_CAPACITY.  The new D_ij is
 * staged in the scratch and copied into the context only when every species
 * succeeded, so on any error the context keeps its positions and D_ij.
 * Nothing in the scratch needs to start at zero.  Calls that overlap on one
 * device (any handles, any threads) race on the scratch: serialise them.  The
 * first call on each device resolves the scratch address
 * (cudaGetSymbolAddress) and must not be made while a stream capture is in
 * progress; the address is kept for the life of the process, which assumes the
 * device's primary context is not reset (cudaDeviceReset) meanwhile. */
int half_set_positions_noalloc(half_handle handle,
                               const double *positions_fractional,
                               char *error, int error_capacity);

/* Non-local PAW band-energy force for given eigenpairs at one k point
 * (src/half_forces.F90:9-73), accumulated into forces[nions*3] (atom-major,
 * eV/A).  vectors: npw x nbands, leading dimension ld >= npw; bands with zero
 * occupation are skipped exactly as in the reference. */
int half_nonlocal_forces(half_handle handle, const double kpoint[3], int nbands,
                         int64_t ld, const HALF_C128 *vectors,
                         const double *eigenvalues_eV,
                         const double *occupations, double kweight,
                         double *forces, char *error, int error_capacity);

/* The band-energy force workload end to end: solve nk k points with the
 * context's solver, compute occupations for nelect electrons with width
 * sigma (ismear -1 Fermi-Dirac, 0 Gaussian; src/half_energy.F90:41-120), then
 * the non-local force on the GPU.  Optional outputs may be NULL:
 * eigenvalues [nk][nbands], occupations [nk][nbands], energies[3] =
 * {band energy, entropy term, chemical potential}. */
int half_band_forces(half_handle handle, int nk, const double *kpoints,
                     const double *kweights, int nbands, double nelect,
                     double sigma, int ismear, double *forces,
                     double *eigenvalues_eV, double *occupations,
                     double *energies, char *error, int error_capacity);

/* The ion-position force terms that the reference's --forces path adds to
 * the non-local force (app/half_cli.F90:947-955), on the GPU.  Each force
 * output is [nions][3] (eV/A, atom-major), overwritten; NULL skips the term:
 *   ewald   ion-ion Ewald force (src/half_energy.F90:164-210);
 *   local   local ionic force on the output density
 *           (src/half_local_forces.F90:11-56);
 *   nlcc    non-linear core correction force with the XC potential of the
 *           context's density (:58-100); zero without a partial core;
 *   harris  frozen-input Harris response from the context's density to the
 *           output density (:129-161); zero without a partial core.
 * output_density: n values on the context's grid in the CHGCAR convention
 * (x fastest, rho * Omega), host or device memory, normally the smooth plus
 * augmentation density of the solved states; NULL = the context's own
 * density (Harris is then zero).
 * energies (NULL to skip) [6] = {Ewald total, real-space, reciprocal, self,
 * background (src/half_energy.F90:122-162), local ionic energy on the output
 * density}. */
int half_ionic_forces(half_handle handle, const double *output_density,
                      int64_t n, double *ewald, double *local, double *nlcc,
                      double *harris, double *energies, char *error,
                      int error_capacity);

/* Output density of given states on the GPU: the smooth density
 * sum_k w_k sum_n f_nk |psi_nk(r)|^2 (src/half_local_forces.F90:102-127) plus
 * the MIMIC_US augmentation density of the occupancies
 * rho_ij = sum w f Re(conj(c_i) c_j), c = B^H psi (src/half_uspp.F90:26-111).
 * vectors: nk consecutive blocks of ld x nbands (column-major, ld >= npw of
 * every k point), host or device memory (device blocks are read in place);
 * occupations [nk][nbands] (bands with f = 0 contribute nothing).  density:
 * n values on the context's grid in the CHGCAR convention (x fastest,
 * rho * Omega), host or device memory, overwritten; n must equal the grid
 * size, else HALF_ERROR_CAPACITY.  augmentation_charge (NULL to skip): the augmentation's
 * contribution to the grid average, the reference's integrated_charge. */
int half_output_density(half_handle handle, int nk, const double *kpoints,
                        const double *kweights, int nbands, int64_t ld,
                        const HALF_C128 *vectors, const double *occupations,
                        double *density, int64_t n,
                        double *augmentation_charge, char *error,
                        int error_capacity);

/* The reference's analytic --forces workload end to end on the GPU
 * (app/half_cli.F90:895-955): solve nk k points with the context's solver,
 * occupations (as half_band_forces), the non-local force, the output density
 * (as half_output_density), then the ion-position terms (as
 * half_ionic_forces with that density).
 *   forces [nions][3] = Ewald + local + non-local + NLCC + Harris, eV/A;
 *   components (NULL to skip) [5][nions][3] = {Ewald, local, non-local, NLCC,
 *     Harris};
 *   output_density (NULL to skip) [n] as half_output_density;
 *   energies (NULL to skip) [6] = {band energy, entropy term, chemical
 *     potential, Ewald energy, local ionic energy, augmentation charge}.
 * With sigma > 0 an occupied highest band (f > 1e-6 at any k) is an
 * HALF_ERROR_INVALID_ARGUMENT, as in the reference CLI. */
int half_forces(half_handle handle, int nk, const double *kpoints,
                const double *kweights, int nbands, double nelect,
                double sigma, int ismear, double *forces, double *components,
                double *output_density, double *energies, char *error,
                int error_capacity);

/* VASP wave-coefficient export (src/half_vaspwave.F90:94-154): each k
 * point's eigenvectors in VASP's plane-wave order (the box's x-fastest order,
 * vasp_permutation :143-154) as interleaved single precision, band-major:
 * packed[offsets[ik] + 2 * (ib * npws[ik] + ig) + {0, 1}] = (re, im), the
 * layout of /wave/spin_1/kpoint_<k>/wave [nb][npw][2] in vaspwave.h5 (the
 * HDF5 container itself is written by the caller's HDF5 library, as the
 * reference's src/half_hdf5_bridge.c does).
 * vectors: nk blocks of ld x nbands (column-major), host or device memory;
 * packed: host or device memory of capacity floats (>= 2 * nbands *
 * sum npw_k, else HALF_ERROR_CAPACITY), or NULL to query npws and offsets
 * only.  npws[nk] and offsets[nk] (in floats) are always written. */
int half_pack_vasp_waves(half_handle handle, int nk, const double *kpoints,
                         int nbands, int64_t ld, const HALF_C128 *vectors,
                         float *packed, int64_t capacity, int *npws,
                         int64_t *offsets, char *error, int error_capacity);

/* Band occupations for nelect electrons, restating compute_occupations
 * (src/half_energy.F90:41-120); a host routine that needs no context or GPU.
 * eigenvalues [nk][nbands] in eV, kweights summing to one (else
 * HALF_ERROR_INVALID_ARGUMENT), sigma >= 0: zero fills degenerate levels
 * fractionally in ascending order, otherwise ismear -1 (Fermi-Dirac) or 0
 * (Gaussian) with the chemical potential found by bisection.  occupations
 * [nk][nbands] in 0..2 are written; energies (NULL to skip) [3] = {band
 * energy, entropy term, chemical potential}.  The same routine sets the
 * occupations inside half_band_forces and half_forces; callers that shard
 * k points over processes use it on the gathered eigenvalues. */
int half_occupations(int nk, int nbands, const double *eigenvalues,
                     const double *kweights, double nelect, double sigma,
                     int ismear, double *occupations, double *energies,
                     char *error, int error_capacity);

/* Device-memory requests of this process since it loaded the library (a
 * diagnostic with no counterpart in the reference): *requests counts every
 * device buffer the library took, from its cache or from the driver, and
 * *driver_allocations the cudaMalloc calls among them.  Either pointer may be
 * NULL.  Comparing the counts around a call shows whether it allocated. */
int half_get_allocation_counts(int64_t *requests, int64_t *driver_allocations,
                               char *error, int error_capacity);

/* Complex FP32 GEMM on the library's tcgen05 tensor-core kernel, the kernel
 * behind the mixed mode's projector and subspace products (a diagnostic
 * entry; the reference's products are cuBLAS ZGEMM calls,
 * src/half_cuda_assembly.cuf:502-512, src/half_cuda_iterative_solver.cuf:
 * 148-194).  C = alpha op(A) op(B) + beta C with op(A) m x k, op(B) k x n;
 * op_a / op_b are 'N', 'T' or 'C'.  a, b: device memory, column-major
 * complex64 (interleaved float pairs); c: device memory, complex64, or
 * complex128 when c_fp64 != 0.  Every operand is split into bf16 hi/lo
 * parts and each real product taken as hi*hi + hi*lo + lo*hi with FP32
 * accumulation (relative error about 2^-16).  Returns when C is complete;
 * host pointers give HALF_ERROR_INVALID_ARGUMENT. */
int half_tc_cgemm(char op_a, char op_b, int m, int n, int k,
                  const double alpha[2], const float *a, int64_t lda,
                  const float *b, int64_t ldb, const double beta[2], void *c,
                  int64_t ldc, int c_fp64, char *error, int error_capacity);

#ifdef __cplusplus
}
#endif
#endif
