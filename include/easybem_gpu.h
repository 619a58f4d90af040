/*
 * easybem B200 — C ABI of the matrix-free Galerkin layer-potential apply.
 *
 * Plain pointers and sizes only. Every entry point returns an int status
 * (EB_OK on success); eb_last_error() returns a message for the last failure
 * on the calling thread. Elements are 1-based vertex triples, as in easybem.
 *
 * The reference exposes this path as process-global C++ functions
 * (include/BEM3dLaplaceGPU.h:8-18) bound to Python in python/bindings.cpp:
 * 186-253. This ABI is the handle-based form of the same operations; the
 * legacy C++ symbols (include/BEM3dLaplaceGPU.h of this project) are a thin
 * shim over one default handle.
 */
#ifndef EASYBEM_GPU_H
#define EASYBEM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define EB_OK 0
#define EB_ERR_INVALID 1        /* bad argument: null pointer, size, order index */
#define EB_ERR_MESH 2           /* vertex index out of range, repeated or degenerate triangle */
#define EB_ERR_CUDA 3           /* a CUDA runtime call failed */
#define EB_ERR_NOMEM 4          /* device memory exhausted or over a budget */
#define EB_ERR_TIMEOUT 5        /* a bounded device-side wait ran out */
#define EB_ERR_STATE 6          /* call out of order (no mesh, closed server) */
#define EB_ERR_NOT_CONVERGED 7  /* a solve stopped at its iteration limit */

/* Far-field arithmetic. The Sauter-Schwab near field is always FP64. */
#define EB_PREC_FP64 0  /* plain FP64: the default */
#define EB_PREC_MIXED 1 /* FP32 far field with compensated (two-sum) row sums */

typedef struct eb_mesh_s* eb_mesh;

const char* eb_version(void);
const char* eb_last_error(void);

/* Uploads a closed or open triangulated surface and precomputes, once, the
 * FP64 Sauter-Schwab near-field correction (coincident, edge- and
 * vertex-adjacent pairs) and the far-field quadrature points. `order` is the
 * easybem quadrature index (0..18, default 4). Replaces initGPU
 * (src/BEM3dLaplaceGPU.cu:830-921 with src/meshTopology.cpp:196-261). */
int eb_mesh_create(int nnodes, const double* nodes, int nelems, const int* elems, int order,
                   eb_mesh* out);
/* Releases a mesh. Replaces closeGPU (src/BEM3dLaplaceGPU.cu:924-957).
 * Work queued on caller streams with this mesh (the _device applies) must
 * have completed: its memory goes back to the memory pool at once. */
int eb_mesh_destroy(eb_mesh mesh);
/* Sizes: vertices, triangles, near pairs (incl. coincident) and the number of
 * regular quadrature-point pairs one far-field apply evaluates. */
int eb_mesh_info(eb_mesh mesh, int* nnodes, int* nelems, long long* near_pairs,
                 long long* far_quad_pairs);
/* The library allocates from each device's stream-ordered memory pool and
 * keeps freed memory there for reuse (cudaMalloc and cudaFree from a thread
 * preparing meshes were measured to wait for kernels other threads run).
 * eb_release_cached_memory returns the unused pool memory to the driver (it
 * waits for the devices); eb_cached_memory_bytes reports the unused pool
 * memory of the current device. No counterpart in the reference. */
int eb_release_cached_memory(void);
int eb_cached_memory_bytes(long long* bytes);

/* Algorithmic bytes one SL+DL finalize launch moves (near-field CSR, the
 * gathered densities, the far-field partial sums under the current plan and
 * the outputs): the numerator of its HBM roofline. No counterpart in the
 * reference. */
int eb_mesh_finalize_bytes(eb_mesh mesh, long long* bytes);
/* The same bytes split into the near-field SpMV of both operators (CSR row
 * pointers, columns and values, gathered densities, outputs) and the fold of
 * the far-field partial sums that the same launch performs. No counterpart
 * in the reference. */
int eb_mesh_near_field_bytes(eb_mesh mesh, long long* spmv_bytes, long long* fold_bytes);
/* (target item, source triangle) pairs of the far-field work (each warp of
 * 32 target items x each 32-triangle source cell) in source cells well
 * separated from the warp's items (centre distance above 1.6 x the sum of the
 * bounding radii: no vertex mask, expanded |x - y|^2) and in the other cells
 * (vertex mask and direct differences), as the CUDA-core far kernel splits
 * them. A target item is a triangle for rules of up to 7 points (then the sum
 * is nelems^2), a chunk of 8 of its points otherwise. No counterpart in the
 * reference. */
int eb_mesh_cell_pairs(eb_mesh mesh, long long* far_cell_tri_pairs, long long* near_cell_tri_pairs);
/* Meshes with at least nelems triangles build their near-pair topology (the
 * CSR lists of vertex-sharing triangle pairs and the double-layer vertex
 * columns of the Sauter-Schwab near field) on the GPU; smaller meshes, and a
 * mesh with a triangle that has more than 48 vertex-sharing neighbours
 * (counted with repeats), build it on the host. Both give the same lists.
 * Default 65,536; 0: every mesh; INT_MAX: none. Creating an L7 icosphere
 * (327,680 triangles) took 732 ms with it against 904 ms on the host. The
 * reference builds its
 * topology on the host (src/meshTopology.cpp:22-261). */
int eb_set_device_topology_min(int nelems);
int eb_get_device_topology_min(int* nelems);
/* 1 when the mesh's near-pair topology was built on the GPU, else 0. */
int eb_mesh_topology_on_device(eb_mesh mesh, int* on_device);

/* v = V t, the P0 single layer (Galerkin, kernel 1/(4 pi |x-y|)); t and v
 * have nelems entries, host memory. Replaces applyGPULaplace3d1Layer(t, v, 0)
 * (src/BEM3dLaplaceGPU.cu:985-1322). */
int eb_apply_sl_p0(eb_mesh mesh, int precision, const double* t, double* v);
/* q = K u, the double layer with P0 test and P1 trial functions; u has
 * nnodes entries, q nelems, host memory. Replaces applyGPULaplace3d2Layer
 * (src/BEM3dLaplaceGPU.cu:1325-1551). */
int eb_apply_dl_p1(eb_mesh mesh, int precision, const double* u, double* q);
/* Both applies in one pass over the pairs (shared distance evaluation). */
int eb_apply_sl_dl(eb_mesh mesh, int precision, const double* t, const double* u, double* v,
                   double* q);
/* Device-pointer form on a CUDA stream (cudaStream_t passed as void*; null
 * selects the legacy default stream). Any of t/v or u/q may be null to skip
 * that operator. Asynchronous: the caller synchronises the stream. */
int eb_apply_sl_dl_device(eb_mesh mesh, int precision, const double* d_t, const double* d_u,
                          double* d_v, double* d_q, void* stream);

/* eb_apply_sl_dl_device without any device allocation, for callers that
 * cannot call cudaMalloc when they apply the operator (memory owned by their
 * own pool or framework allocator, or a loop that must not enter the driver's
 * allocator). No counterpart in the reference. Device pointers in and out;
 * all per-apply scratch lives in one fixed 32 MiB device array that every GPU
 * loading the library keeps until exit. Meshes needing more scratch are
 * rejected (EB_ERR_INVALID, message gives the size). Calls share that array:
 * calls overlapping on the GPU race. The first call on a device looks up the
 * array's address and should come before any stream capture; under CUDA's
 * lazy module loading (the default) that first call is also where the 32 MiB
 * are placed on the device, so make it at start-up, before the caller's own
 * allocator fills the device (no room then: EB_ERR_CUDA). */
int eb_apply_sl_dl_noalloc(eb_mesh mesh, int precision, const double* d_t, const double* d_u,
                           double* d_v, double* d_q, void* stream);

/* v = V1 t, the single layer with P1 test and trial functions (t, v have
 * nnodes entries). Replaces applyGPULaplace3d1Layer(t, v, 1)
 * (src/BEM3dLaplaceGPU.cu:82-154, 211-320, 371-442, 491-557, host :1034-1313)
 * with the same Sauter-Schwab formulas in FP64, but trial indices taken from
 * the trial triangle (the reference scatters them onto the test triangle's
 * vertices off the diagonal, :1128, :1219, :1311, and drops a -1 at :1125). */
int eb_apply_sl_p1(eb_mesh mesh, int precision, const double* t, double* v);
/* Device-pointer form of eb_apply_sl_p1 on a stream (asynchronous). */
int eb_apply_sl_p1_device(eb_mesh mesh, int precision, const double* d_t, double* d_v, void* stream);
/* q = D u, the hypersingular operator in the curl form
 * D = sum_k C_k^T V C_k of getLaplace3d (src/BEM3dLaplace.cpp:767-771); u, q
 * have nnodes entries. Replaces the empty applyGPULaplace3dHyperSing
 * (src/BEM3dLaplaceGPU.cu:1554-1555). */
int eb_apply_hypersingular(eb_mesh mesh, int precision, const double* u, double* q);
/* Device-pointer form of eb_apply_hypersingular on a stream (asynchronous). */
int eb_apply_hypersingular_device(eb_mesh mesh, int precision, const double* d_u, double* d_q,
                                  void* stream);

/* u(x) = V t - W u at npts points off the surface (the representation formula
 * with the triangle rule of the mesh's order, any index): pts [npts][3],
 * t [nelems], u [nnodes], out [npts], host memory. Replaces evaluateLaplace3d
 * (src/BEM3dLaplace.cpp:784-843). */
int eb_evaluate_potential(eb_mesh mesh, int precision, int npts, const double* pts, const double* t,
                          const double* u, double* out);

/* ---- Batched apply (no counterpart in the reference): the P0 single layer
 * of many meshes, each with ncols (1..4) right-hand sides, in one persistent
 * far-field launch (captured once in a CUDA graph and replayed). d_t[i] and
 * d_v[i] are device arrays [ncols][nelems_i]. With a null stream the call
 * runs on the batch's own stream and returns when done; otherwise it is
 * asynchronous on `stream`. */
typedef struct eb_batch_s* eb_batch;
int eb_batch_create(int nmesh, const eb_mesh* meshes, int ncols, int precision, eb_batch* out);
int eb_batch_destroy(eb_batch batch);
int eb_batch_apply(eb_batch batch, const double* const* d_t, double* const* d_v, void* stream);
/* Regular quadrature-point pairs one batched apply evaluates (per column set). */
int eb_batch_info(eb_batch batch, long long* quad_pairs);
/* Batched single and double layer: v_i = V_i t_i and q_i = K_i u_i for every
 * mesh i in one persistent far-field pass (the fused variant of
 * eb_apply_sl_dl; each quadrature-pair distance serves both operators). d_t,
 * d_v, d_q hold device arrays of nelems_i entries, d_u of nnodes_i. Stream
 * semantics as eb_batch_apply; eb_batch_info counts each pair once. No
 * counterpart in the reference (one mesh per process, applyGPULaplace3d1Layer
 * and applyGPULaplace3d2Layer as separate passes, src/BEM3dLaplaceGPU.cu:
 * 985-1551). */
int eb_batch_create_sl_dl(int nmesh, const eb_mesh* meshes, int precision, eb_batch* out);
int eb_batch_apply_sl_dl(eb_batch batch, const double* const* d_t, const double* const* d_u,
                         double* const* d_v, double* const* d_q, void* stream);

/* ---- Solves: V x = b (P0 single layer) by GMRES with iterative refinement.
 * No counterpart in the reference (its drivers call SciPy CG on FP32 GPU
 * matvecs, python/examples/laplace3dDirichletGPU.py:64-81). Each restart
 * cycle of GMRES(restart) uses the `inner_precision` apply (mixed: FP32 far
 * field); the Arnoldi basis and Gram-Schmidt are FP64 on the GPU; every cycle
 * ends with the FP64 residual b - V x, and a system stops when
 * ||b - V x|| <= tol ||b||. Many systems (meshes x right-hand sides) advance in
 * lockstep through batched applies. */
typedef struct eb_solve_options {
  double tol;          /* FP64 relative residual target (default 1e-8) */
  double inner_tol;    /* relative reduction per GMRES cycle (default 1e-6) */
  int restart;         /* Krylov dimension (default 50) */
  int max_cycles;      /* refinement cycles per system (default 40) */
  int max_iterations;  /* GMRES iterations per system (default 4000) */
  int inner_precision; /* EB_PREC_MIXED (default) or EB_PREC_FP64 */
  int precond;         /* 1 (default): right preconditioner M, the sparse
                        * approximate inverse of the FP64 near field on its own
                        * pattern (column j minimises ||N m - e_j|| over the
                        * triangles sharing a vertex with j); 0: none. It changes
                        * the iteration count only: every cycle ends with the
                        * true FP64 residual of V x = b. */
  int rhs_precision;   /* the server's right-hand sides (1/2 M + K) g:
                        * EB_PREC_FP64 (default) or EB_PREC_MIXED (FP32 far
                        * field of K g, FP64 near field and mass term). For
                        * data harmonic inside the surface 1/2 M g and K g
                        * cancel (||K g|| / ||b|| ~ 20 on the serving tori), so
                        * the 1e-7 error of the FP32 K g grows to a few 1e-6 in
                        * b and the solution. The solvers take b as given. */
} eb_solve_options;

typedef struct eb_solve_stats {
  int converged;
  int cycles;
  int iterations;
  double rel_residual; /* final ||b - V x|| / ||b|| from the FP64 apply */
} eb_solve_stats;

void eb_solve_options_default(eb_solve_options* opt);
/* y = M x with the solver's near-field preconditioner (built on first use);
 * x and y have nelems entries, host memory. No counterpart in the reference. */
int eb_apply_near_precond(eb_mesh mesh, const double* x, double* y);
/* Solves sum(nrhs) systems at once: b[i] and x[i] are host arrays
 * [nrhs[i]][nelems of meshes[i]]; stats (optional) has one entry per system
 * in mesh-major order. All meshes need the same quadrature order. Returns
 * EB_ERR_NOT_CONVERGED if any system missed the tolerance (x still holds the
 * last iterate). */
int eb_solve_sl(int nmesh, const eb_mesh* meshes, const int* nrhs, const double* const* b, double* const* x,
                const eb_solve_options* opt, eb_solve_stats* stats);

/* Stepwise form for continuous batching: systems join and leave between
 * steps; one step advances every active system by one GMRES iteration or one
 * refinement residual. */
typedef struct eb_solver_s* eb_solver;
int eb_solver_create(const eb_solve_options* opt, eb_solver* out);
int eb_solver_destroy(eb_solver solver);
int eb_solver_add(eb_solver solver, eb_mesh mesh, int nrhs, const double* b, int* ids);
int eb_solver_step(eb_solver solver, int* nactive);
int eb_solver_done(eb_solver solver, int id, int* done);
int eb_solver_result(eb_solver solver, int id, double* x, eb_solve_stats* stats);
int eb_solver_remove(eb_solver solver, int id);
/* Device memory one system of this mesh holds in the solver (Krylov basis
 * and vectors), for admission control. */
int eb_solver_bytes_per_system(eb_solver solver, eb_mesh mesh, long long* bytes);

/* ---- Continuous-batching solve server (no counterpart in the reference).
 * A request is a mesh (1-based elements, quadrature order) with nrhs sets of
 * Dirichlet vertex data g ([nrhs][nnodes]); its answer is t ([nrhs][nelems])
 * with V t = (1/2 M + K) g, solved to the server's options. Requests are
 * admitted under a device-memory budget (resident mesh data plus Krylov
 * storage), prepared by a host worker thread while other requests run, and
 * join the shared lockstep solver as soon as they are ready and fewer than
 * max_systems right-hand sides are active; eb_server_step advances all of
 * them by one iteration. A request's result does not depend on what runs
 * beside it. Poll states: 0 queued, 1 preparing, 2 prepared, 3 solving,
 * 4 done, 5 failed. times_ms (optional, 4 entries): total latency, queue
 * wait, preparation, solve. */
typedef struct eb_server_s* eb_server;
int eb_server_create(long long budget_bytes, int max_systems, const eb_solve_options* opt, eb_server* out);
int eb_server_destroy(eb_server server);
int eb_server_submit(eb_server server, int nnodes, const double* nodes, int nelems, const int* elems, int order,
                     int nrhs, const double* g, long long* id);
int eb_server_step(eb_server server, int* nactive, int* nwaiting);
int eb_server_poll(eb_server server, long long id, int* state);
int eb_server_result(eb_server server, long long id, double* t, eb_solve_stats* stats, double* times_ms);
int eb_server_release(eb_server server, long long id);
int eb_server_usage(eb_server server, long long* used_bytes, long long* budget_bytes);
/* Operating counters, up to n of: steps, seconds spent in eb_server_step,
 * solver batch rebuilds (membership changes), seconds spent in them,
 * requests prepared, seconds the preparation worker was busy, and of those
 * the seconds in mesh creation, right-hand sides and preconditioner builds,
 * mesh creation split into topology, static tables and near field, and the
 * static tables' device allocation and copy.
 * No counterpart in the reference. */
int eb_server_stats(eb_server server, double* stats, int n);

/* Right-hand side of the direct (Green) formulation of the interior Dirichlet
 * problem, as the reference examples build it (python/examples/
 * laplace3dDirichletGPU.py:63): b = (1/2) M g + K g with M the P0 x P1 mass
 * matrix (src/BEM3dLaplace.cpp:448-486) and K the double layer, for nrhs
 * vertex data g ([nrhs][nnodes], host) into b ([nrhs][nelems], host). FP64. */
int eb_dirichlet_rhs(eb_mesh mesh, int nrhs, const double* g, double* b);

/* The same right-hand sides with K g in the given precision (EB_PREC_FP64 as
 * eb_dirichlet_rhs, or EB_PREC_MIXED: FP32 far field, FP64 near field and
 * mass term). No counterpart in the reference. */
int eb_dirichlet_rhs_prec(eb_mesh mesh, int precision, int nrhs, const double* g, double* b);

/* The quadrature rules behind index `order` (host only, no GPU needed):
 * the Gauss-Legendre rule on [0,1] (up to 64 points) and the triangle rule on
 * the reference triangle (up to 79 points, weights summing to 1/2). Mirrors
 * the tables LineQuadrature* / TriangleQuadrature* of src/quadrature.cpp:
 * 284-305, 1045-1070. Arrays must hold 64 and 79 entries. */
int eb_quadrature(int order, int* nline, double* lx, double* lw, int* ntri, double* tx, double* ty,
                  double* tw);

/* ---- Mesh ingestion (host only, no GPU needed). Readers of the two surface
 * formats the reference's drivers load: easybem's plain-text surface
 * (python/examples/surface3dMesh.py:51-83 load3dSurface: dimension, vertices
 * per element, vertex list, triangle list, then "index label" lines) and the
 * surface triangles of a Netgen .vol file (:86-146 load3dSurfaceFromNetgen:
 * sections "points" and "surfaceelementsgi", label = surface number).
 * nodes [nnodes][3], elems [nelems][3] 1-based, labels [nelems]; with null
 * arrays only the counts are written (call once for sizes, once to fill). */
int eb_read_surface_txt(const char* path, int* nnodes, double* nodes, int* nelems, int* elems, int* labels);
int eb_read_netgen_vol(const char* path, int* nnodes, double* nodes, int* nelems, int* elems, int* labels);
/* Uniform 1->4 refinement (:149-221 refineMesh): one midpoint per unique
 * edge, numbered after the old vertices in lexicographic order of the
 * edge's (smaller, larger) vertex pair; children of triangle k at k, m + k,
 * 2m + k, 3m + k (m = nelems): (v0, m01, m20), (m01, v1, m12),
 * (m20, m12, v2), (m01, m12, m20). Child labels are their parent's (the
 * reference repeats each label four times in a row instead, so its labels
 * do not follow its own child order). With null output arrays only the
 * counts are written. labels and labels_out may be null. */
int eb_mesh_refine(int nnodes, const double* nodes, int nelems, const int* elems, const int* labels,
                   int* nnodes_out, double* nodes_out, int* nelems_out, int* elems_out, int* labels_out);

/* Roofline calibration: sustained FP32 FFMA throughput of the current GPU in
 * TFLOP/s (FMA = 2 flops), from a register-only FMA-chain kernel. No
 * counterpart in the reference. */
int eb_measure_fp32_peak(double* tflops, double* seconds);
/* MUFU reciprocal-square-root throughput of the current GPU in Tops/s (one
 * rsqrt.approx.f32 per far-field quadrature pair), from a chain kernel. No
 * counterpart in the reference. */
int eb_measure_rsqrt_peak(double* tops, double* seconds);

/* Event timing of the far-field kernel and of the finalize kernel (which
 * includes the near-field SpMV) of the last apply on this mesh, recorded on
 * the apply's stream when profiling is on. Blocks until that apply ends.
 * No counterpart in the reference (which has no timing API). */
int eb_set_profiling(eb_mesh mesh, int on);
int eb_last_kernel_ms(eb_mesh mesh, double* far_ms, double* finalize_ms);

/* Launch plan of a mesh's far field: work items per SM (how finely the source
 * range of every 128-target tile is cut for the persistent CTAs' queue) and
 * source triangles per shared-memory tile (0 = the variant's default, at most
 * 64). eb_mesh_set_plan rebuilds the work list and drops the cached launch
 * descriptors; batches and solvers built later use the new plan. No work on
 * the mesh may be in flight (synchronise its streams first), and no other
 * call on the same mesh may run meanwhile. Results
 * change only by rounding (summation order). No counterpart in the reference,
 * whose launch shape is fixed (src/BEM3dLaplaceGPU.cu:985-1322, 256 threads). */
int eb_mesh_set_plan(eb_mesh mesh, int items_per_sm, int src_tile);
int eb_mesh_get_plan(eb_mesh mesh, int* items_per_sm, int* src_tile, int* nsplit, int* work_items);

/* Far-field engine of a mesh's fused FP32 SL+DL apply (EB_PREC_MIXED, both
 * operators, 7-point triangle rule = quadrature index 4):
 * EB_FAR_CUDA_CORES evaluates every quadrature pair on the FP32 pipes;
 * EB_FAR_TENSOR_CORES computes |x - y|^2 and the double-layer numerator
 * s (x - y).n of well-separated cells as split-TF32 GEMMs on the tensor
 * cores (tcgen05) and keeps the reciprocal square root and the sums on the
 * CUDA cores; EB_FAR_SYMMETRIC evaluates every unordered quadrature-point
 * pair once on the FP32 pipes and adds it to both rows of its triangle pair
 * (the test and trial rules are the same rule, so 1/|x-y| and 1/|x-y|^3
 * serve both orders), which halves the reciprocal square roots and cuts the
 * FMA-pipe work per pair from 8 to 4.5 operations. It needs one partial slot
 * per 128-triangle tile and row (16 bytes each: ne^2/8 bytes, 0.84 GB at
 * 81,920 triangles, 13.4 GB at 327,680), allocated on its first apply, and
 * takes meshes of up to 524,288 triangles (32 GiB of slots); larger meshes
 * use the CUDA cores. EB_FAR_SYMMETRIC is the default of a new mesh. Other
 * variants always use the CUDA cores; get reports the engine an apply in
 * `precision` with both operators would use. No counterpart in the
 * reference. */
#define EB_FAR_CUDA_CORES 0
#define EB_FAR_TENSOR_CORES 1
#define EB_FAR_SYMMETRIC 2
/* EB_FAR_SYMMETRIC for the FP64 applies too (every unordered pair once in
 * FP64: 7 instead of 13 FP64-pipe operations per pair for SL+DL, 5 instead
 * of 10 for the single layer). Opt-in: the FP64 default of the apply entry
 * points stays the plain ordered-pair kernel (the solver's internal FP64
 * residuals take the symmetric kernel on the default engine); get reports
 * EB_FAR_SYMMETRIC for an FP64 apply on this engine. */
#define EB_FAR_SYMMETRIC_ALL 3
int eb_mesh_set_far_engine(eb_mesh mesh, int engine);
int eb_mesh_get_far_engine(eb_mesh mesh, int precision, int* engine);
/* Pipe work per well-separated quadrature pair of the fused mixed SL+DL far
 * field on an engine, as this library was built: MUFU reciprocal square
 * roots, FMA-pipe lane operations (an FMA counts once) and tensor-core
 * flops (the numerators of the kernels' rooflines). */
int eb_far_engine_costs(int engine, double* mufu_per_pair, double* fma_ops_per_pair, double* tensor_flops_per_pair);
/* The symmetric engine's work list for a mesh of nelems triangles in sorted
 * order (host only, no GPU): *nitems work items as (first target row, first
 * source cell, end source cell, forward slot) quadruples in items[4 * k ..]
 * (cells of 32 triangles, target tiles of 128 rows; a source range after the
 * tile is evaluated in both orders and its transposed sums go to the tile's
 * slot, a range on the tile itself in forward order), the largest slot count
 * of a row in *nslots_max, and in row_slots[s] the slots row s holds (the
 * ones its finalize folds). cells_per_item 0 takes the single-mesh default,
 * 32 is the batches'. Pass null arrays to get the sizes. No counterpart in
 * the reference. */
int eb_sym_plan(int nelems, int cells_per_item, int* nitems, int* nslots_max, int* items, int* row_slots);

/* Times candidate plans (items_per_sm in {4,8,...,512} x source tile in
 * {default, 32, 16}) on this mesh with CUDA events, median of `reps` applies
 * each; operators: 1 = SL, 2 = DL, 3 = SL+DL. Keeps the fastest on the mesh
 * and records it in the process-wide plan table under (SM count,
 * floor(log2 nelems), triangle-rule points, precision); meshes created later
 * that match an entry start from it (mixed entries first). start_ms is the
 * time of the plan the mesh had. No counterpart in the reference. */
int eb_autotune(eb_mesh mesh, int precision, int operators, int reps, int* items_per_sm, int* src_tile,
                double* best_ms, double* start_ms);
/* Plan table as text: a header line, then "sms bucket points precision
 * items_per_sm src_tile ms" per entry. Load merges into the table. */
int eb_plan_table_save(const char* path);
int eb_plan_table_load(const char* path, int* loaded);
int eb_plan_table_clear(void);

#ifdef __cplusplus
}
#endif

#endif /* EASYBEM_GPU_H */
