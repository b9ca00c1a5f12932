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
#define KCFD_PREC_AMG    3  /* smoothed-aggregation multigrid, one V(1,1) cycle per apply */

/* stopping rules */
#define KCFD_STOP_SCIPY  0  /* scipy bicgstab: ||r|| < max(atol, rtol ||b||), eps^2 breakdown
                               (core/linear_solver.py:59 -> scipy.sparse.linalg.bicgstab) */
#define KCFD_STOP_GPU    1  /* core/gpu_solver.py:111-155: ||s||/||b||, ||r||/||b|| < tol,
                               1e-30 guards                                            */

/* Krylov methods */
#define KCFD_METHOD_BICGSTAB 0  /* scipy bicgstab (core/linear_solver.py:59)             */
#define KCFD_METHOD_CG       1  /* scipy cg: solve_pressure_correction's iterative branch
                                   (core/linear_solver.py:90-92); one right-hand side,
                                   FP64, scipy stop, graph engine (team 0 or 3)          */

/* precision modes */
#define KCFD_MODE_FP64   0  /* plain FP64                                            */
#define KCFD_MODE_MIXED  1  /* FP32 inner BiCGSTAB, FP64 residual + refinement + dots */

int  kcfd_version(void);
/* Copies the last error message of this thread into buf (NUL-terminated). */
int  kcfd_last_error(char* buf, int32_t len);
/* Number of SMs and compute capability of the current device (probe, no allocation). */
int  kcfd_device_info(int32_t* sm_count, int32_t* cc_major, int32_t* cc_minor);

/* ------------------------------------------------------------ CUDA graphs ---- */
/* Capture the device work of a sequence of kcfd_* calls issued on one stream as a
 * CUDA graph and replay it (e.g. one SIMPLE outer iteration: assembly, solver set-up
 * and solves, with fixed pointers and sizes). No counterpart in the reference, whose
 * outer loop is host Python (models/single_phase.py:70-101).
 * kcfd_graph_capture_begin starts a thread-local capture on a non-default stream;
 * calls that allocate (kcfd_solver_create, kcfd_batch_create, kcfd_mesh_build) and a
 * handle's first solve on the graph engine must come before it (inside a capture an
 * engine handle solves on its persistent kernel). kcfd_graph_capture_end ends the
 * capture and instantiates the graph into *out; kcfd_graph_launch replays it on a
 * stream; kcfd_graph_destroy frees it.                                             */
/* Failure-detection self-test of the team barrier (no counterpart in the reference):
 * `ctas` CTAs meet at one barrier of a team that expects `team_size` members, on the
 * caller's zeroed counter `bar` (uint32) and error flag `err` (int32). With
 * team_size > ctas the barrier cannot complete; every wait gives up after
 * budget_cycles (clock64), records KCFD_TIMEOUT in *err and returns, as the solver's
 * barriers do, and the context stays usable. With team_size == ctas *err stays 0.  */
int  kcfd_selftest_barrier(int32_t ctas, int32_t team_size, int64_t budget_cycles, uint32_t* bar, int32_t* err,
                           void* stream);
typedef struct kcfd_graph kcfd_graph;
int  kcfd_graph_capture_begin(void* stream);
int  kcfd_graph_capture_end(void* stream, kcfd_graph** out);
int  kcfd_graph_launch(kcfd_graph* g, void* stream);
void kcfd_graph_destroy(kcfd_graph* g);

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
/* The build runs its independent passes on up to 16 host threads (KCFD_HOST_THREADS in
 * the environment, read once per process, caps the count); the result does not depend
 * on the thread count. */
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

/* Device face layout of a built mesh (host arrays in, host arrays out; no device
 * call). Faces are ordered colour by colour (internal colours first), by reference
 * face id inside a colour; per face, the geometric factors of the SIMPLE kernels with
 * the reference's formulas: gc = dN / (dO + dN) (0.5 when dO + dN <= 1e-30;
 * models/single_phase.py:380-388), dlen = |d_PN| on internal faces and |x_f - x_P| on
 * boundary faces (:197), dorth = max(|d_PN . n|, 0.1 |d_PN|) (:166-175); and the faces
 * of every cell in ascending reference id as device face indices. Row norms and dots
 * sum their components left to right. Inputs are the kcfd_mesh_export arrays in
 * reference face order; n_colors = internal + boundary face colours.               */
typedef struct {
    int64_t* order;      /* [F] reference face id of each device face                 */
    int32_t* color_ptr;  /* [n_colors + 1] device face range of each colour           */
    int32_t* owner;      /* [F]                                                       */
    int32_t* neigh;      /* [Fi]                                                      */
    double*  area;       /* [F]                                                       */
    double*  normal;     /* [F * ndim]                                                */
    double*  fcenter;    /* [F * ndim]                                                */
    double*  gc;         /* [Fi]                                                      */
    double*  dlen;       /* [F]                                                       */
    double*  dorth;      /* [Fi]                                                      */
    int32_t* slot_on;    /* [Fi]                                                      */
    int32_t* slot_no;    /* [Fi]                                                      */
    int32_t* cf_ptr;     /* [n + 1]                                                   */
    int32_t* cf_face;    /* [n * max_cell_faces]; the first cf_ptr[n] entries are set */
} kcfd_face_layout_t;

int kcfd_mesh_device_layout(int32_t ndim, int64_t n_cells, int64_t n_faces, int64_t n_internal,
                            int32_t n_colors, int32_t max_cell_faces, const int64_t* owner,
                            const int64_t* neighbour, const int32_t* face_color, const double* ccenter,
                            const double* fcenter, const double* normal, const double* area,
                            const int32_t* slot_on, const int32_t* slot_no, const int64_t* cell_faces,
                            kcfd_face_layout_t* out);

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
typedef struct kcfd_amg kcfd_amg;

typedef struct {
    int32_t precond;     /* KCFD_PREC_*                                        */
    int32_t stop;        /* KCFD_STOP_*                                        */
    int32_t mode;        /* KCFD_MODE_*                                        */
    int32_t nrhs;        /* 1, 2 or 3 (momentum components share one matrix)  */
    int32_t maxiter;     /* BiCGSTAB iterations (inner iterations in MIXED)   */
    int32_t team;        /* 0 auto, 1 one CTA per system, 2 whole grid (one
                            persistent cooperative kernel), 3 graph engine
                            (phase kernels in one CUDA graph per solve with a
                            device-side loop; inside a stream capture the solve
                            runs on the team-2 kernel; MIXED there: FP32 Krylov
                            vectors and values, FP64 iterate, residual
                            replacement against the FP64 matrix -- for well
                            conditioned systems, so only when asked for). Auto:
                            1 for n*nrhs <= 1024, 2 up to 40000 and for MIXED,
                            else 3.                                              
                            KCFD_ENGINE_EAGER=1 in the environment at creation
                            launches the engine's kernels from a host loop
                            instead (for profilers; same results);
                            KCFD_ENGINE_PDL=0 launches its phase kernels
                            without programmatic dependent launch.            */
    int32_t lanes;       /* SpMV lanes per row: 0 auto, 1..32                  */
    int32_t block;       /* threads per CTA: 0 auto (team 1: 512, team 2: 512) */
    double  rtol;        /* relative tolerance                                 */
    double  atol;        /* absolute tolerance (KCFD_STOP_SCIPY)               */
    double  inner_rtol;  /* MIXED: inner FP32 solve reduction per refinement   */
    int32_t max_refine;  /* MIXED: refinement steps                            */
    int32_t inner_maxiter; /* MIXED: inner iterations per refinement step (0: 400) */
    int32_t fill_level;  /* KCFD_PREC_ILU0 only: 0 ILU(0); k > 0 ILU(k), the
                            level-of-fill factorisation (core/preconditioner.py:
                            56-61 offers 'iluk' through SuperLU's threshold ILU;
                            this is the structural form)                        */
    int32_t amg_max_levels; /* KCFD_PREC_AMG: kcfd_amg_opts_t.max_levels (0: 12)    */
    int32_t amg_coarse_max; /* KCFD_PREC_AMG: kcfd_amg_opts_t.coarse_max (0: 128)   */
    int32_t method;      /* KCFD_METHOD_* (0: BiCGSTAB)                             */
} kcfd_solver_opts_t;
/* KCFD_PREC_AMG: one right-hand side, graph engine only (team 0 or 3). The handle
 * builds a kcfd_amg hierarchy on the pattern at creation and refreshes it in
 * kcfd_solver_setup; each preconditioner apply inside the engine's loop is one V-cycle
 * (its kernels are nodes of the engine's loop body). mode KCFD_MODE_MIXED keeps the
 * Krylov iteration FP64 and stores the multigrid hierarchy and cycle vectors in FP32
 * (FP64 arithmetic). Inside a stream capture an AMG handle does not solve (the
 * engine's graph is not nested): the call returns KCFD_BAD_INPUT.                 */

/* ILU(0) ordering: level_of_row_host gives each row's level (e.g. the mesh's cell
 * colouring, or natural-order dependency levels); NULL -> natural-order levels.
 * Coupled rows must lie on different levels. With ILU(0) the handle solves the
 * level-permuted system P A P^T (rows grouped by level), so every level is a
 * contiguous row range that all CTAs share evenly.
 * ILU(k), fill_level = k > 0: the rows are ordered by a greedy distance-(k+1)
 * colouring of A's (symmetrised) graph, which keeps every fill entry between rows of
 * different colours, so the colours are the levels (level_of_row_host is not used);
 * the factor's pattern (A's plus the fill of level <= k) is the handle's permuted
 * matrix, with zeros in the fill slots, so its products are A's.                  */
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

/* z = M^-1 r with the handle's set-up preconditioner (one right-hand side, FP64
 * handles): Jacobi, ILU(0) / ILU(k) (both sweeps on the level-permuted factors), one
 * AMG V-cycle, or a copy for KCFD_PREC_NONE. Device vectors, no host sync. This is
 * M.matvec of the LinearOperator that create_preconditioner returns
 * (core/preconditioner.py:18-76).                                                   */
int kcfd_solver_apply_precond(kcfd_solver* s, const kcfd_csr_t* A, const double* r, double* z, void* stream);
/* The multigrid hierarchy of a KCFD_PREC_AMG handle (owned by the handle; NULL for
 * other preconditioners), for kcfd_amg_info / kcfd_amg_export.                    */
int kcfd_solver_amg(const kcfd_solver* s, kcfd_amg** out);


/* ------------------------------------------------ algebraic multigrid ------ */
/* Smoothed-aggregation AMG (Vanek, Mandel and Brezina 1996), the device counterpart of
 * create_preconditioner(A, 'amg') (core/preconditioner.py:63-74: pyamg's
 * smoothed_aggregation_solver(A).aspreconditioner()). Aggregates from three greedy
 * passes over A's graph; P = (I - omega D^-1 A) T; A_c = P^T A P; omega = 4 / (3 rho)
 * with rho a Gershgorin bound on level 0 and a power-iteration estimate below; a
 * V(1,1) cycle with damped Jacobi; the coarsest level (<= 256 rows) by its dense
 * inverse. kcfd_amg_create builds every pattern and product map on the host from A's
 * pattern (device pointers; every row needs its diagonal entry); kcfd_amg_setup
 * refreshes all values from A's current values on the device (no host sync);
 * kcfd_amg_apply computes x = M^-1 b (one cycle) on the device.                   */
typedef struct {
    int32_t mode;         /* KCFD_MODE_FP64, or KCFD_MODE_MIXED: hierarchy values and cycle
                             vectors stored in FP32, arithmetic in FP64            */
    int32_t coarse_max;   /* stop coarsening at or below this many rows (0: 128, <= 256) */
    int32_t max_levels;   /* 0: 12 (at most 16)                                     */
    int32_t power_iters;  /* power iterations for rho(D^-1 A) below level 0 (0: 8)   */
} kcfd_amg_opts_t;
int  kcfd_amg_create(const kcfd_csr_t* A, const kcfd_amg_opts_t* opts, kcfd_amg** out);
int  kcfd_amg_setup(kcfd_amg* h, const kcfd_csr_t* A, void* stream);
int  kcfd_amg_apply(kcfd_amg* h, const double* b, double* x, void* stream);
/* nlevels; rows_nnz[2 l], rows_nnz[2 l + 1] = rows and entries of level l (room for 16
 * levels); device_bytes = memory the handle holds.                                */
int  kcfd_amg_info(const kcfd_amg* h, int32_t* nlevels, int64_t* rows_nnz, int64_t* device_bytes);
/* Copies one item of a level to host memory (synchronises the device), for tests:  */
#define KCFD_AMG_AGGREGATES     0  /* int32[n_l] aggregate of each row (not the coarsest) */
#define KCFD_AMG_INDPTR         1  /* int32[n_l + 1] A_l row pointers                     */
#define KCFD_AMG_INDICES        2  /* int32[nnz_l] A_l columns                            */
#define KCFD_AMG_VALUES         3  /* double[nnz_l] A_l values (levels >= 1)              */
#define KCFD_AMG_P_INDPTR       4  /* int32[n_l + 1] prolongator row pointers             */
#define KCFD_AMG_P_INDICES      5  /* int32[nnz(P_l)] prolongator columns                 */
#define KCFD_AMG_P_VALUES       6  /* double[nnz(P_l)] prolongator values                 */
#define KCFD_AMG_OMEGA          7  /* double[1] the level's omega                         */
#define KCFD_AMG_COARSE_INVERSE 8  /* double[n_l * n_l] dense inverse (coarsest level)    */
int  kcfd_amg_export(const kcfd_amg* h, int32_t level, int32_t what, void* out_host);
void kcfd_amg_destroy(kcfd_amg* h);

/* ------------------------------------------------------ batched systems ---- */
/* Many independent systems (e.g. the pressure-correction systems of many meshes) of
 * uneven sizes solved together over packed CSR with per-system offsets: each team
 * takes the next system from a largest-first queue and solves it alone (FP64 or MIXED
 * BiCGSTAB, Jacobi or no preconditioner; the scipy stopping rule per system). The
 * tiers run concurrently, one persistent launch each. Cluster tiers: a system is
 * solved by the CTAs of one thread-block cluster (512 threads each, one per SM, rows
 * split between them, bounded software barriers) -- graded (cluster_size 0): 8, 4 or
 * 2 CTAs for systems of at least 8R, 4R or 2R rows, R = cluster_rows (0: 16384), so
 * that the big systems get CTAs in proportion to their size; or one tier of
 * cluster_size CTAs from cluster_rows rows (0: 131072). Then systems of at least
 * big_rows rows are solved by one 512-thread CTA, the rest by one 256-thread CTA. A
 * system's tier depends only on its own size (and on whether a cluster of its size
 * can be resident at all), so its result is the same alone and in any mix. No
 * counterpart API in the reference, which solves one system per call
 * (core/linear_solver.py:14-70); results per system equal that path's semantics. */
typedef struct kcfd_batch kcfd_batch;
typedef struct {
    int32_t precond, stop, mode, maxiter, lanes, max_refine, inner_maxiter;
    int32_t big_rows;      /* tier threshold in rows: 0 default (16384), < 0 none      */
    int32_t cluster_rows;  /* graded: R (0: 16384); one tier: its threshold (0:
                              131072); < 0: no cluster tier                           */
    int32_t cluster_size;  /* CTAs per cluster team: 0 graded, 2..8 one tier           */
    double  rtol, atol, inner_rtol;
    int32_t restarts;      /* KCFD_STOP_SCIPY: a system whose rho or omega breaks down
                              (|.| < eps^2) restarts from its current iterate with
                              rhat = r, p = r, up to this many times; 0 stops there with
                              KCFD_BREAKDOWN as scipy does. With restarts > 0 (FP64) a
                              system that stops on its recursive residual is also
                              checked against b - A x: up to 3 more passes start from
                              the true residual (a pass that meets the tolerance at
                              once ends with no iteration)                            */
} kcfd_batch_opts_t;
/* indptr_host: per system n[s]+1 local row pointers, concatenated; indices_host:
 * local column indices, concatenated (host arrays, copied to the device).          */
int  kcfd_batch_create(int32_t nsys, const int32_t* n, const int32_t* nnz, const int32_t* indptr_host,
                       const int32_t* indices_host, const kcfd_batch_opts_t* opts, kcfd_batch** out);
/* The team each system of a batch would get on a device with sm_count SMs (host only, no
 * device call; every cluster size taken as resident): team[s] = CTAs of its thread-block
 * cluster (2, 4 or 8), 1 for one 512-thread CTA, 0 for one 256-thread CTA. The same rule
 * as kcfd_batch_create. No counterpart in the reference (batching is this library's).  */
int  kcfd_batch_plan(int32_t nsys, const int32_t* n, const kcfd_batch_opts_t* opts, int32_t sm_count, int32_t* team);
void kcfd_batch_destroy(kcfd_batch* b);
/* info[0..3] = nsys, total rows, total entries, CTAs per launch */
int  kcfd_batch_info(const kcfd_batch* b, int64_t* info);
/* tiers[5]: systems in the cluster, big and small tiers, clusters launched, CTAs
 * per cluster.                                                                     */
int  kcfd_batch_tiers(const kcfd_batch* b, int32_t* tiers);
/* vals64, rhs, x: packed device arrays (system s at its row / entry offset); x holds
 * x0 on entry. iters/relres/status: device arrays of nsys entries.                 */
int  kcfd_batch_solve(kcfd_batch* b, const double* vals64, const double* rhs, double* x, int32_t* iters,
                      double* relres, int32_t* status, void* stream);

/* ------------------------------------------------------- device mesh -------- */
/* Device-resident SoA mesh. Faces are stored colour by colour: internal faces first
 * (colours 0..n_colors_int-1), then boundary faces (n_colors_bnd colours); no two
 * faces of one colour share a cell, so the owner/neighbour scatter of a colour is
 * free of write conflicts (no atomics). face_ref maps a device face to its
 * reference face id. All pointers are device pointers except color_ptr (host).   */
typedef struct {
    int32_t ndim, n_cells, n_faces, n_internal;
    const int32_t* owner;      /* [F]  */
    const int32_t* neigh;      /* [Fi] */
    const double*  area;       /* [F]  */
    const double*  normal;     /* [F*ndim] unit, owner-outward */
    const double*  fcenter;    /* [F*ndim] */
    const double*  ccenter;    /* [n*ndim] */
    const double*  volume;     /* [n]  */
    const double*  gc;         /* [Fi] interpolation weight dN/(dO+dN) */
    const double*  dlen;       /* [F]  |d_PN| internal, |x_f - x_P| boundary */
    const double*  dorth;      /* [Fi] max(|d_PN . n|, 0.1 |d_PN|) */
    const int32_t* slot_on;    /* [Fi] CSR slot (owner, neighbour) */
    const int32_t* slot_no;    /* [Fi] CSR slot (neighbour, owner) */
    const int32_t* diag_slot;  /* [n]  */
    const int32_t* indptr;     /* [n+1] CSR row pointers */
    const int32_t* face_ref;   /* [F]  reference face id */
    const int32_t* color_ptr;  /* HOST [n_colors_int + n_colors_bnd + 1] face ranges */
    int32_t n_colors_int, n_colors_bnd;
    const int32_t* cf_ptr;     /* [n+1] faces of each cell (NULL: not provided)   */
    const int32_t* cf_face;    /* device faces of the cells, each cell's in ascending
                                  reference face id (the reference's summation order) */
} kcfd_dmesh_t;

/* Boundary conditions per boundary face (index = device face - n_internal).
 * type: 0 zero_gradient, 1 dirichlet, 2 neumann.                                */
typedef struct {
    const int8_t* u_type;   /* [Fb]        velocity BC type               */
    const double* u_val;    /* [Fb*ndim]   velocity boundary values       */
    const int8_t* p_type;   /* [Fb]        pressure BC type               */
    const double* p_val;    /* [Fb]        pressure boundary values       */
    int32_t has_p_dirichlet;
    int32_t pad;
} kcfd_bc_t;

#define KCFD_LIM_NONE       (-1)
#define KCFD_LIM_MINMOD       0
#define KCFD_LIM_SUPERBEE     1
#define KCFD_LIM_VAN_ALBADA   2
#define KCFD_LIM_VAN_LEER     3

typedef struct {
    double  rho, mu, alpha_u, dt;  /* dt > 0 adds the backward-Euler term (transient) */
    int32_t limiter;               /* KCFD_LIM_*: MUSCL deferred correction, NONE = upwind */
    int32_t nonorth;               /* 1: over-relaxed non-orthogonal correction           */
} kcfd_mom_params_t;


/* ------------------------------------------------ generic FVM operators ---- */
/* Each operator ADDS into a device system (vals64: CSR values on the mesh's
 * pattern, diag: the tracked diagonal of FVMSystem, rhs), like the reference's COO
 * triplets summed by to_sparse() (core/fvm_operators.py:13-56). Face operators run
 * one launch per face colour.                                                     */
/* diffusion_operator (core/fvm_operators.py:59-100): harmonic-mean gamma, |d_PN|. */
int kcfd_op_diffusion(const kcfd_dmesh_t* m, const double* gamma, double* vals, double* diag, void* stream);
/* convection_operator_upwind (core/fvm_operators.py:103-129); mf in device face order. */
int kcfd_op_convection_upwind(const kcfd_dmesh_t* m, const double* mf, double* vals, double* diag, void* stream);
/* apply_boundary_conditions (core/fvm_operators.py:178-225). Per boundary face:
 * btype 0 zero_gradient / 1 dirichlet / 2 neumann, bval = phi_b, bgrad = neumann value. */
int kcfd_op_boundary(const kcfd_dmesh_t* m, const int8_t* btype, const double* bval, const double* bgrad,
                     const double* gamma, const double* mf, double* vals, double* diag, double* rhs, void* stream);
/* Cell operators (core/fvm_operators.py:132-175, 228-240):
 *   kind 0 temporal_operator   a0 = rho, a1 = dt, p0 = phi_old
 *   kind 1 source_term         p0 = S
 *   kind 2 linearized_source   p0 = Sp, p1 = Su
 *   kind 3 under_relax         a0 = alpha, p0 = phi (reads the tracked diagonal)     */
int kcfd_op_cells(const kcfd_dmesh_t* m, int32_t kind, double a0, double a1, const double* p0, const double* p1,
                  double* vals, double* diag, double* rhs, void* stream);
/* muscl_deferred_correction (core/interpolation.py:227-303): corr[n] (overwritten)
 * from phi, mf (device face order) and grad [n][ndim]; limiter KCFD_LIM_*.        */
int kcfd_muscl_correction(const kcfd_dmesh_t* m, int32_t limiter, const double* phi, const double* mf,
                          const double* grad, double* corr, void* stream);

/* ------------------------------------------------ SIMPLE assembly kernels --- */
/* Face mass flux F = rho (u_f . n) A, u_f = gc U_O + (1-gc) U_N inside, the
 * dirichlet value (else U_O) on boundary faces. mf in device face order.
 * SIMPLESolver._face_mass_flux (models/single_phase.py:124-144);
 * compute_mass_flux (core/interpolation.py:163-182).                            */
int kcfd_mass_flux(const kcfd_dmesh_t* m, const kcfd_bc_t* bc, const double* U, double rho, double* mf,
                   void* stream);

/* Momentum matrix (shared by all velocity components) and ndim right-hand sides:
 * harmonic mu, d_orth diffusion, first-order upwind, boundary terms, face pressure
 * source, optional MUSCL deferred correction and non-orthogonal correction (gradU:
 * [n][ndim][ndim] Green-Gauss gradients of the components), optional time term,
 * under-relaxation. Writes vals64 (and vals32 if non-NULL), b [n][ndim],
 * aP_phys [n] (unrelaxed aP) and dP [n] = V / mean(aP).
 * SIMPLESolver._momentum_eq (models/single_phase.py:147-258);
 * muscl_deferred_correction (core/interpolation.py:227-303).                    */
int kcfd_momentum_assemble(const kcfd_dmesh_t* m, const kcfd_bc_t* bc, const kcfd_mom_params_t* prm,
                           const double* U, const double* U_old, const double* p, const double* mf,
                           const double* gradU, double* aP, double* vals64, float* vals32, double* b,
                           double* dP, void* stream);

/* Pressure-correction matrix and rhs (models/single_phase.py:274-348): df =
 * rho (dP_O+dP_N)/2 A / d_orth, rhs = -sum(+-mf), dirichlet-p boundary terms, and the
 * row-0 reference pin when no pressure patch is dirichlet.                        */
int kcfd_pressure_assemble(const kcfd_dmesh_t* m, const kcfd_bc_t* bc, double rho, const double* dP,
                           const double* mf, double* aP, double* vals64, float* vals32, double* b,
                           void* stream);

/* Green-Gauss gradient of ncomp cell fields phi [n][ncomp] -> grad [n][ncomp][ndim]
 * (core/gradient.py:12-48). Boundary face value: bval[bf*ncomp+k] where
 * btype[bf] == 1, else the owner value.                                            */
int kcfd_gg_gradient(const kcfd_dmesh_t* m, int32_t ncomp, const double* phi, const int8_t* btype,
                     const double* bval, double* grad, void* stream);

/* Reductions use a caller-provided scratch of KCFD_REDUCE_SCRATCH doubles.       */
#define KCFD_REDUCE_SCRATCH 8192

/* least_squares_gradient (core/gradient.py:51-99) of a scalar: phi [n], phi_b per
 * boundary face (the patch values), grad [n][ndim]; needs the cell-face list.      */
int kcfd_lsq_gradient(const kcfd_dmesh_t* m, const double* phi, const double* phi_b, double* grad, void* stream);

/* SIMPLE correction (models/single_phase.py:355-377): U -= dP grad(p'),
 * p += alpha_p p'; norms2[0] = ||p'||^2, norms2[1] = ||p||^2 (after the update),
 * summed in a fixed order. grad_pp: [n][ndim].                                     */
int kcfd_simple_correct(const kcfd_dmesh_t* m, double alpha_p, const double* pp, const double* grad_pp,
                        const double* dP, double* U, double* p, double* norms2, double* scratch, void* stream);

/* norms2[2c] = ||A x_c - b_c||^2, norms2[2c+1] = ||b_c||^2 for c < nrhs
 * (the post-solve residual of models/single_phase.py:270-271).                   */
int kcfd_residual_norms(const kcfd_csr_t* A, const double* x, const double* b, int32_t nrhs, double* norms2,
                        double* scratch, void* stream);

/* Outer residual bookkeeping of solve_steady (models/single_phase.py:86-92) on the
 * device: res = max(max_c ||r_c||/max(||b_c||,1e-15), ||p'||/max(||p||+1e-10,1e-10)),
 * normalised by the first residual above 1e-30 (state[0]); state[1] = raw residual;
 * hist[*it] = normalised residual when *it < max_hist; then *it += 1 (device counter,
 * so a captured CUDA graph can replay the step).                                   */
int kcfd_simple_residual(int32_t ndim, const double* mom_norms2, const double* p_norms2, double* state,
                         double* hist, int32_t* it, int32_t max_hist, void* stream);

/* out[c] = sum_i x[i*k + c]^2 for c < k (k <= 6), fixed-order sums; scratch as above. */
int kcfd_vec_norms2(int32_t n, int32_t k, const double* x, double* out2, double* scratch, void* stream);

/* Continuity residual history of served runs: chist[*it] = ||b_p'|| (from its
 * squared norm); call before kcfd_simple_residual advances *it.                    */
int kcfd_record_norm(const double* norm2, double* chist, const int32_t* it, int32_t max_hist, void* stream);

/* Barrier error flag of the handle's last launch (KCFD_TIMEOUT when a bounded team
 * barrier wait expired, else 0). Synchronises the stream.                         */
int kcfd_solver_error(kcfd_solver* s, int32_t* err, void* stream);

/* Launch shape the handle resolved at creation: info[0] team (1 one CTA, 2 whole
 * grid, 3 graph engine), info[1] lanes per row, info[2] threads per CTA, info[3]
 * ILU(0) levels (1 without ILU). No reference counterpart (diagnostics).         */
int kcfd_solver_info(const kcfd_solver* s, int32_t* info4);

/* ------------------------------------------------ two-fluid system set ----- */
/* The pieces of the Euler-Euler model (models/two_fluid.py, models/closure.py) that
 * are not generic FVM operators, for the device TwoFluidSolver. Cell arrays [n],
 * vectors [n][ndim]; face arrays in device face order; boundary arrays per boundary
 * face (device order), nc right-hand sides interleaved [n][nc]. Each call ADDS into
 * the system like the reference's FVMSystem; face terms run one launch per colour. */
typedef struct {
    double rho_l, rho_g, mu_l, mu_g, cp_l, cp_g, k_l, k_g, d_b;
    double g[3];                                 /* gravity (last axis -9.81)   */
    double h_i_coeff, a_i_coeff, T_sat, h_fg, r_phase_change;
    double dt;
} kcfd_tf_params_t;

/* K_drag (drag_coefficient_implicit, models/closure.py:72-92; Schiller-Naumann :13-34) */
int kcfd_tf_drag(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, const double* alpha_g, const double* U_g,
                 const double* U_l, double* K, void* stream);
/* h_i a_i V (Ranz-Marshall, models/two_fluid.py:395-410) */
int kcfd_tf_interfacial(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, const double* alpha_g, const double* U_g,
                        const double* U_l, double* hiaiV, void* stream);
/* Lee evaporation / condensation rate dot_m (models/two_fluid.py:334-360) */
int kcfd_tf_phase_change(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, const double* alpha_l,
                         const double* alpha_g, const double* T_l, const double* T_g, double* dot_m, void* stream);
/* gamma = alpha coef (kind 0), or alpha mu_l + alpha mu_BIT with Sato's bubble-induced
 * viscosity (kind 1; models/two_fluid.py:551-561, models/closure.py:146-164)      */
int kcfd_tf_gamma(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, int32_t kind, const double* alpha, double coef,
                  const double* alpha_g, const double* U_g, const double* U_l, double* gamma, void* stream);
/* face flux weighting: kind 0 mf alpha[owner] (models/two_fluid.py:566-568); kind 1
 * mf alpha_upwind cp (models/two_fluid.py:433-444)                                */
int kcfd_tf_face_flux(const kcfd_dmesh_t* m, int32_t kind, const double* mf, const double* alpha, double cp,
                      double* out, void* stream);
/* compute_mass_flux with per-boundary-face values U_b (core/interpolation.py:163-182) */
int kcfd_tf_mass_flux(const kcfd_dmesh_t* m, double rho, const double* U, const double* U_b, double* mf,
                      void* stream);
/* boundary values of masked (zero_gradient) faces := owner values
 * (_update_zero_gradient_boundaries, models/two_fluid.py:224-250)                 */
int kcfd_tf_zero_gradient(const kcfd_dmesh_t* m, const int8_t* mask, const double* field, int32_t nc, double* bval,
                          void* stream);
/* phase momentum terms for components comp0..comp0+nc-1 (models/two_fluid.py:570-598):
 * temporal (U_old may be NULL), pressure force -alpha grad p per face, implicit drag,
 * gravity                                                                           */
int kcfd_tf_momentum_sources(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, int32_t comp0, int32_t nc, double rho,
                             const double* alpha, const double* p, const double* K, const double* U_other,
                             const double* U_old, double* vals, double* diag, double* rhs, void* stream);
/* apply_boundary_conditions (core/fvm_operators.py:178-225) for nc rhs sharing one matrix */
int kcfd_tf_boundary(const kcfd_dmesh_t* m, const int8_t* btype, const double* bval, const double* bgrad, int32_t nc,
                     const double* gamma, const double* mf, double* vals, double* diag, double* rhs, void* stream);
/* diagonal floor (diag < 1e-20 -> 1e-10, if floor_diag) then under_relax for nc rhs */
int kcfd_tf_relax(const kcfd_dmesh_t* m, double alpha, const double* phi, int32_t nc, int32_t floor_diag, double* vals,
                  double* diag, double* rhs, void* stream);
/* aP = max(diag, 1e-20) (first) or max(aP, max(diag, 1e-20)) (models/two_fluid.py:620-633) */
int kcfd_tf_update_ap(const kcfd_dmesh_t* m, const double* diag, double* aP, int32_t first, void* stream);
/* two-phase p' system with the row-0 pin diag += 1e10 (models/two_fluid.py:641-689) */
int kcfd_tf_pressure_assemble(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, const double* alpha_l,
                              const double* alpha_g, const double* aP_l, const double* aP_g, const double* mf_l,
                              const double* mf_g, double* vals, double* diag, double* rhs, void* stream);
/* p += alpha_p p'; face-difference gradient of p'; U_k += alpha_p (-alpha_k V / aP_k) grad p'
 * (models/two_fluid.py:697-723); grad: [n][ndim] scratch                           */
int kcfd_tf_correct(const kcfd_dmesh_t* m, double alpha_p, const double* pp, const double* alpha_l,
                    const double* alpha_g, const double* aP_l, const double* aP_g, double* grad, double* U_l,
                    double* U_g, double* p, void* stream);
/* volume-fraction source dot_m / rho_g V where |dot_m| > 1e-30 (models/two_fluid.py:753-758) */
int kcfd_tf_alpha_source(const kcfd_dmesh_t* m, double rho_g, const double* dot_m, double* rhs, void* stream);
/* phase energy terms (models/two_fluid.py:446-496): temporal (T_old may be NULL),
 * interfacial exchange, latent heat of dm_sign * dot_m, wall heat flux q_b on the
 * boundary faces with qmask set, weighted by alpha_wall[owner]                      */
int kcfd_tf_energy_sources(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, double rho, double cp,
                           const double* alpha, const double* T_old, const double* T_other, const double* hiaiV,
                           const double* dot_m, double dm_sign, const int8_t* qmask, const double* q_b,
                           const double* alpha_wall, double* vals, double* diag, double* rhs, void* stream);
/* post-solve guards: mode 0 restore old if any NaN; 1 restore old if any NaN/inf,
 * else clip to [lo, hi]; 2 zero if any NaN. flag: one device int of scratch.       */
int kcfd_tf_guard(int64_t count, double* x, const double* old, int32_t mode, double lo, double hi, int32_t* flag,
                  void* stream);
/* alpha_g clipped to [0, 1], alpha_l = 1 - alpha_g, maxdiff = max |alpha_g - alpha_old| */
int kcfd_tf_alpha_finish(int32_t n, double* alpha_g, double* alpha_l, const double* alpha_old, double* maxdiff,
                         void* stream);
/* dst[i*dst_stride + dst_off + c] = src[i*src_stride + src_off + c], c < ncopy      */
int kcfd_tf_copy(int32_t n, int32_t ncopy, const double* src, int32_t src_stride, int32_t src_off, double* dst,
                 int32_t dst_stride, int32_t dst_off, void* stream);

/* ------------------------------------------- allocation-free solve ---------- */
/* No counterpart in the reference. For callers that cannot call cudaMalloc --
 * real-time loops that must not block on the device allocator, and host programs
 * whose device memory is owned and pre-reserved by someone else (a framework's
 * caching allocator, a fixed budget per tenant) -- this solves
 * one system of at most kcfd_noalloc_max_rows() rows (32768) with the single-CTA
 * FP64 BiCGSTAB (precond KCFD_PREC_NONE or KCFD_PREC_JACOBI, stop rule as in
 * kcfd_solver_create) and allocates nothing: its Krylov vectors live in a fixed
 * array inside libkcfd (about 2.6 MB held on every GPU that loads the library until
 * the process exits). Larger systems are rejected with KCFD_BAD_INPUT. The first
 * call on a device looks up the array's device address, so make that call before
 * any stream capture (a first call on a capturing stream returns KCFD_BAD_INPUT and
 * says so). All calls share the array and it keeps the last call's contents (each
 * call initialises what it reads): calls that overlap on the GPU (on different
 * streams) race. A, b, x (x0 on entry), iters, relres and status
 * are caller device memory, as in kcfd_solver_solve.                              */
int kcfd_noalloc_max_rows(void);
int kcfd_bicgstab_noalloc(const kcfd_csr_t* A, const double* b, double* x, int32_t precond, int32_t stop,
                          double rtol, double atol, int32_t maxiter, int32_t* iters, double* relres,
                          int32_t* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* KCFD_H */
