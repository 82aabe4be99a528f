/* libhalf ABI v1 -- B200 implementation.
 *
 * This header keeps DeePAW-HALF's published C ABI byte for byte: the same
 * enum values, struct layouts, symbol names and argument order as the
 * reference's include/half.h:11-189, so a caller built against the reference
 * links against this library unchanged.  Every entry point is implemented in
 * deepaw-half_b200/csrc/api.cpp; the line cited beside each declaration is
 * the reference declaration (or implementation) it replaces.
 *
 * Conventions (reference docs/API.md:54-67): matrices and state blocks are
 * complex128 column-major; energies in eV, lengths in Angstrom, k points in
 * fractional reciprocal coordinates; every call returns a status code and
 * writes a NUL-terminated message (truncated to capacity-1, cleared on
 * entry) into the caller's error buffer.
 */
#ifndef DEEPAW_HALF_H
#define DEEPAW_HALF_H

#include <stdint.h>
#ifndef __cplusplus
#include <complex.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define HALF_ABI_VERSION 1
#define HALF_VERSION_MAJOR 0
#define HALF_VERSION_MINOR 6
#define HALF_VERSION_PATCH 0

/* reference include/half.h:16-24 */
enum half_status {
  HALF_SUCCESS = 0,
  HALF_ERROR_INVALID_ARGUMENT = 1,
  HALF_ERROR_IO = 2,
  HALF_ERROR_INVALID_HANDLE = 3,
  HALF_ERROR_CAPACITY = 4,
  HALF_ERROR_UNAVAILABLE = 5,
  HALF_ERROR_INTERNAL = 6
};

/* reference include/half.h:26-38 */
enum half_xc { HALF_XC_LDA = 1, HALF_XC_PBE = 2 };
enum half_backend { HALF_BACKEND_AUTO = 0, HALF_BACKEND_CPU = 1, HALF_BACKEND_CUDA = 2 };
enum half_solver {
  HALF_SOLVER_EVD = 1,   /* dense generalized solve, all eigenpairs */
  HALF_SOLVER_EVJ = 2,   /* Jacobi variant (accepted; this build answers UNAVAILABLE) */
  HALF_SOLVER_VASP = 3,  /* dense index-range solve of the requested bands */
  HALF_SOLVER_ACC = 4    /* matrix-free all-band block solver */
};

/* reference include/half.h:40-53 */
enum half_capability {
  HALF_CAP_CPU = 1 << 0,
  HALF_CAP_CUDA = 1 << 1,
  HALF_CAP_MPI = 1 << 2,
  HALF_CAP_HDF5 = 1 << 3,
  HALF_CAP_SPGLIB = 1 << 4,
  HALF_CAP_ESCN_API = 1 << 5
};
enum half_escn_flag { HALF_ESCN_INCLUDE_UNCERTAINTY = 1 << 0 };
enum half_density_normalization {
  HALF_DENSITY_RAW = 0,
  HALF_DENSITY_NORMALIZE_VALENCE = 1
};

typedef int64_t half_handle;

/* reference include/half.h:62-73.  lattice is row-major [vector][xyz];
 * positions are atom-major fractional; species are one-based type indices. */
typedef struct half_request_geometry_v1 {
  uint32_t struct_size;
  uint32_t flags;
  int32_t nions;
  int32_t ntypes;
  int32_t grid[3];
  int32_t reserved_i32;
  double lattice[9];
  const int32_t *species;
  const double *positions_fractional;
  uint64_t reserved[8];
} half_request_geometry_v1;

/* reference include/half.h:78-88 */
typedef struct half_escn_request_v1 {
  uint32_t struct_size;
  uint32_t flags;
  int32_t nions;
  int32_t grid[3];
  int32_t reserved_i32;
  double cell[9];
  const int32_t *atomic_numbers;
  const double *positions_cartesian;
  uint64_t reserved[8];
} half_escn_request_v1;

/* reference include/half.h:94-107 */
typedef struct half_escn_result_v1 {
  uint32_t struct_size;
  uint32_t flags;
  int32_t grid[3];
  int32_t reserved_i32;
  int64_t capacity;
  float *density;
  float *nu;
  float *alpha;
  float *beta;
  float *risk;
  double elapsed_seconds;
  uint64_t reserved[8];
} half_escn_result_v1;

#ifdef __cplusplus
typedef struct { double re, im; } half_complex128;
#define HALF_C128 half_complex128
#else
#define HALF_C128 double _Complex
#endif

int half_get_abi_version(void);                 /* reference half.h:109 */
const char *half_get_version_string(void);      /* reference half.h:110 */
int half_get_capabilities(void);                /* reference half.h:111 */

/* reference half.h:113-118 (remote density service; this build answers
 * HALF_ERROR_UNAVAILABLE: the density service is outside the solver path) */
int half_escn_health(const char *base_url, int timeout_seconds,
                     char *error, int error_capacity);
int half_escn_predict(const char *base_url,
                      const half_escn_request_v1 *request,
                      half_escn_result_v1 *result, int timeout_seconds,
                      char *error, int error_capacity);

/* reference half.h:120-122: AUTO backend + EVD solver */
int half_create_from_files(const char *charge_path, const char *potential_path,
                           double encut_eV, int xc, int use_uspp_dij,
                           half_handle *handle, char *error, int error_capacity);
/* reference half.h:125-129 */
int half_create_from_files_backend(const char *charge_path,
                                   const char *potential_path,
                                   double encut_eV, int xc, int use_uspp_dij,
                                   int backend, int solver, half_handle *handle,
                                   char *error, int error_capacity);
/* reference half.h:134-139 (UNAVAILABLE in this build, see above) */
int half_create_from_escn(const char *base_url, const char *potential_path,
                          const half_request_geometry_v1 *geometry,
                          double encut_eV, int xc, int use_uspp_dij,
                          int backend, int solver, int normalization,
                          int timeout_seconds, half_handle *handle,
                          char *error, int error_capacity);
/* reference half.h:140 */
int half_destroy(half_handle handle, char *error, int error_capacity);

/* reference half.h:142-153 */
int half_set_request_geometry(half_handle handle,
                              const half_request_geometry_v1 *geometry,
                              char *error, int error_capacity);
int half_get_request_geometry(half_handle handle, int32_t *nions,
                              int32_t *ntypes, int32_t grid[3],
                              double lattice[9], int64_t species_capacity,
                              int32_t *species, int64_t positions_capacity,
                              double *positions_fractional,
                              char *error, int error_capacity);

/* reference half.h:155-157 */
int half_get_system_info(half_handle handle, int *nions, int *ntypes,
                         int grid[3], double lattice[9], double *volume_A3,
                         char *error, int error_capacity);

/* reference half.h:161-165: gvec[3*i+axis], kinetic_eV[i] */
int half_get_basis_size(half_handle handle, const double kpoint[3], int64_t *npw,
                        char *error, int error_capacity);
int half_get_basis(half_handle handle, const double kpoint[3], int64_t capacity,
                   int32_t *gvec, double *kinetic_eV,
                   char *error, int error_capacity);

/* reference half.h:168-174.  The reference's CUDA contexts answer UNAVAILABLE
 * here; this build evaluates both on the GPU (dense assembly for
 * half_assemble_hs, the matrix-free operator for half_apply_hs: FP64, or the
 * mixed mode's FP32 operator when half_set_acc_controls selected
 * HALF_PRECISION_MIXED). */
int half_assemble_hs(half_handle handle, const double kpoint[3], int64_t ld,
                     HALF_C128 *h, HALF_C128 *s,
                     char *error, int error_capacity);
int half_apply_hs(half_handle handle, const double kpoint[3], int nstates,
                  int64_t ld, const HALF_C128 *psi,
                  HALF_C128 *hpsi, HALF_C128 *spsi,
                  char *error, int error_capacity);
/* reference half.h:175-178 */
int half_solve_kpoint(half_handle handle, const double kpoint[3], int nbands,
                      double *eigenvalues_eV, HALF_C128 *eigenvectors,
                      int64_t ld, double *overlap_min, double *overlap_max,
                      char *error, int error_capacity);
/* reference half.h:183-189: eigenvectors permuted into the host's G order */
int half_solve_kpoint_mapped(half_handle handle, const double kpoint[3],
                            int nbands, int64_t host_npw,
                            const int32_t *host_gvec,
                            double *eigenvalues_eV,
                            HALF_C128 *eigenvectors, int64_t ld,
                            double *overlap_min, double *overlap_max,
                            char *error, int error_capacity);

#ifdef __cplusplus
}
#endif
#endif
