/*
 * kcfd.h -- C ABI of libkcfd.so, the B200-native (sm_100a) SIMPLE inner loop for
 * unstructured finite-volume meshes.
 *
 * Every entry point is extern "C", takes plain pointers and sizes and returns an
 * int status (KCFD_OK = 0). Device pointers are owned by the caller; handles own
 * only their internal scratch. kcfd_last_error() returns the text of the last
 * failure on the calling thread.
 *
 * Each declaration names the K-CFD reference interface it replaces
 * (paths relative to the reference checkout).
 */
#ifndef KCFD_H
#define KCFD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status ---- */
#define KCFD_OK          0  /* converged / done                                   */
#define KCFD_MAXITER     1  /* iteration cap reached (reference: prints, returns x) */
#define KCFD_BREAKDOWN   2  /* BiCGSTAB rho/omega breakdown                        */
#define KCFD_BAD_INPUT   3  /* malformed arguments (sizes, pointers, CSR)           */
#define KCFD_CUDA_ERROR  4  /* CUDA runtime error                                   */
#define KCFD_TIMEOUT     5  /* a bounded device-side wait ran out                   */

/* preconditioners (core/preconditioner.py:18-76 method names) */
#define KCFD_PREC_NONE   0
#define KCFD_PREC_JACOBI 1
#define KCFD_PREC_ILU0   2

/* stopping rules */
#define KCFD_STOP_SCIPY  0  /* scipy bicgstab: ||r|| < max(atol, rtol ||b||), eps^2 breakdown
                               (core/linear_solver.py:59 -> scipy.sparse.linalg.bicgstab) */
#define KCFD_STOP_GPU    1  /* core/gpu_solver.py:111-155: ||s||/||b||, ||r||/||b|| < tol,
                               1e-30 guards                                            */

/* precision modes */
#define KCFD_MODE_FP64   0  /* plain FP64                                            */
#define KCFD_MODE_MIXED  1  /* FP32 inner BiCGSTAB, FP64 residual + refinement + dots */

int  kcfd_version(void);
/* Copies the last error message of this thread into buf (NUL-terminated). */
int  kcfd_last_error(char* buf, int32_t len);
/* Number of SMs and compute capability of the current device (probe, no allocation). */
int  kcfd_device_info(int32_t* sm_count, int32_t* cc_major, int32_t* cc_minor);

/* ------------------------------------------------------- host mesh build ---- */
/* Face discovery, owner/neighbour, geometry, boundary tagging
 * (mesh/mesh_reader.py:141-323 build_fvmesh_from_arrays / _build_fvmesh_3d), plus
 * the canonical CSR pattern of FVMSystem.to_sparse() (core/fvm_operators.py:43-48),
 * the face -> CSR slot map, a face colouring for atomic-free scatter and a cell
 * colouring for ILU(0) level scheduling.
 *
 * 2D: cface_* are NULL; faces are the cell edges (cell_nodes[k], cell_nodes[k+1]).
 * 3D: cface_ptr[n_cells+1] indexes the per-cell face list; face q has cface_len[q]
 *     nodes starting at cface_off[q] in cface_nodes.
 * Boundary faces: n_bfaces node lists (bface_len, flattened bface_nodes), each with
 *     the index of its patch in the caller's patch-dict order (bface_patch).      */
typedef struct kcfd_host_mesh kcfd_host_mesh;

int kcfd_mesh_build(int32_t ndim, int64_t n_nodes, const double* nodes,
                    int64_t n_cells, const int64_t* cell_ptr, const int64_t* cell_nodes,
                    const int64_t* cface_ptr, const int64_t* cface_len, const int64_t* cface_off,
                    const int64_t* cface_nodes,
                    int64_t n_bfaces, const int64_t* bface_len, const int64_t* bface_nodes,
                    const int32_t* bface_patch, kcfd_host_mesh** out);

/* info[0..9] = n_faces, n_internal, nnz, max_face_nodes, max_cell_faces,
 *              n_int_colors, n_bnd_colors, n_cell_colors, n_levels_natural, ndim */
int kcfd_mesh_info(const kcfd_host_mesh* m, int64_t* info);

/* Caller-allocated host arrays; any pointer may be NULL to skip that output.
 * Face arrays are in reference face order. face_patch: -1 internal, else the
 * caller's patch index, or -2 when no boundary entry matched ("default").      */
typedef struct {
    int64_t* owner;        /* [F]                 */
    int64_t* neighbour;    /* [F]  -1 = boundary   */
    int64_t* face_nodes;   /* [F * max_face_nodes], -1 padded (first-discovery order) */
    int64_t* cell_faces;   /* [n * max_cell_faces], -1 padded (cell.faces order)      */
    double*  area;         /* [F]                 */
    double*  normal;       /* [F * ndim]          */
    double*  fcenter;      /* [F * ndim]          */
    double*  ccenter;      /* [n * ndim]          */
    double*  volume;       /* [n]                 */
    int32_t* face_patch;   /* [F]                 */
    int32_t* indptr;       /* [n + 1]             */
    int32_t* indices;      /* [nnz]               */
    int32_t* slot_on;      /* [F] CSR slot of (owner, neighbour), -1 on boundary */
    int32_t* slot_no;      /* [F] CSR slot of (neighbour, owner), -1 on boundary */
    int32_t* diag_slot;    /* [n]                 */
    int32_t* face_color;   /* [F] internal 0..Ci-1, boundary Ci..Ci+Cb-1          */
    int32_t* cell_color;   /* [n] greedy colouring of the cell adjacency graph    */
    int32_t* level_natural;/* [n] dependency level of row i in natural order      */
} kcfd_mesh_export_t;

int  kcfd_mesh_export(const kcfd_host_mesh* m, kcfd_mesh_export_t* out);
void kcfd_mesh_free(kcfd_host_mesh* m);

/* ------------------------------------------------------------- CSR / SpMV ---- */
/* Device CSR (int32 indices). vals64 and/or vals32 may be set; kernels read the
 * precision they are asked for.                                                   */
typedef struct {
    int32_t n;
    int32_t nnz;
    const int32_t* indptr;   /* [n+1] */
    const int32_t* indices;  /* [nnz] */
    const double*  vals64;   /* [nnz] or NULL */
    const float*   vals32;   /* [nnz] or NULL */
} kcfd_csr_t;

/* dst[i] = (float) src[i]: FP32 copy of FP64 matrix values for the MIXED inner solve. */
int kcfd_cast_f64_f32(int64_t m, const double* src, float* dst, void* stream);

/* y = A x (gpu_spmv, core/gpu_solver.py:55-79). nrhs vectors interleaved [n][nrhs]. */
int kcfd_spmv_f64(const kcfd_csr_t* A, const double* x, double* y, int32_t nrhs, void* stream);
int kcfd_spmv_f32(const kcfd_csr_t* A, const float* x, float* y, int32_t nrhs, void* stream);

/* ------------------------------------------------------------ BiCGSTAB ------ */
/* Solver handle: binds one CSR pattern (sizes), allocates the Krylov scratch for
 * nrhs right-hand sides in the requested mode, and carries the preconditioner set-up.
 * Replaces gpu_bicgstab (core/gpu_solver.py:82-108) and the bicgstab branch of
 * solve_linear_system (core/linear_solver.py:50-62) with create_preconditioner
 * (core/preconditioner.py:18-76, methods 'none' / 'jacobi' / 'ilu0').            */
typedef struct kcfd_solver kcfd_solver;

typedef struct {
    int32_t precond;     /* KCFD_PREC_*                                        */
    int32_t stop;        /* KCFD_STOP_*                                        */
    int32_t mode;        /* KCFD_MODE_*                                        */
    int32_t nrhs;        /* 1 or 3 (momentum components share one matrix)     */
    int32_t maxiter;     /* BiCGSTAB iterations (inner iterations in MIXED)   */
    int32_t team;        /* 0 auto, 1 one CTA per system, 2 whole grid         */
    int32_t lanes;       /* SpMV lanes per row: 0 auto, 1..32                  */
    int32_t block;       /* threads per CTA: 0 auto                            */
    double  rtol;        /* relative tolerance                                 */
    double  atol;        /* absolute tolerance (KCFD_STOP_SCIPY)               */
    double  inner_rtol;  /* MIXED: inner FP32 solve reduction per refinement   */
    int32_t max_refine;  /* MIXED: refinement steps                            */
    int32_t pad;
} kcfd_solver_opts_t;

/* ILU(0) ordering: perm/levels as produced by kcfd_mesh_export (cell_color or
 * level_natural). level_of_row == NULL -> natural-order levels computed here.  */
int kcfd_solver_create(const kcfd_csr_t* A, const kcfd_solver_opts_t* opts,
                       const int32_t* level_of_row_host, kcfd_solver** out);
void kcfd_solver_destroy(kcfd_solver* s);

/* Preconditioner set-up on the current values of A (Jacobi inverse diagonal or the
 * numeric ILU(0) factorisation). Device-side, no host sync.                       */
int kcfd_solver_setup(kcfd_solver* s, const kcfd_csr_t* A, void* stream);

/* Solve A x = b on the device. x holds x0 on entry. b, x interleaved [n][nrhs] in
 * FP64. Results (per rhs) are written to the device arrays iters/relres/status if
 * non-NULL; nothing is synchronised with the host.                               */
int kcfd_solver_solve(kcfd_solver* s, const kcfd_csr_t* A, const double* b, double* x,
                      int32_t* iters, double* relres, int32_t* status, void* stream);

/* Barrier error flag of the handle's last launch (KCFD_TIMEOUT when a bounded team
 * barrier wait expired, else 0). Synchronises the stream.                         */
int kcfd_solver_error(kcfd_solver* s, int32_t* err, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* KCFD_H */
