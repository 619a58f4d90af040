// Device-resident mesh and the apply pipeline.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "farfield.cuh"
#include "mesh_host.h"

namespace eb {

// p1t selects P1 test functions (three outputs per item; NSL = 1, no DL).
cudaError_t far_launch(bool fp32, int NSL, int ND, int K, int Q, const FarMeshDesc* dm, const WorkItem* di, int n,
                       int* dc, size_t smem, int grid, cudaStream_t st, bool p1t = false);
int far_occupancy(bool fp32, int NSL, int ND, int K, int Q, size_t smem, bool p1t = false);
bool far_variant_supported(int NSL, int ND);
cudaError_t prep_launch(bool fp32, int NSL, int ND, const ApplyArgs& A, cudaStream_t st);
cudaError_t finalize_launch(int NSL, int ND, const ApplyArgs& A, cudaStream_t st);
cudaError_t prep_launch_batch(bool fp32, int NSL, int ND, const ApplyArgs* d_args, const int* d_off, int n,
                              int nblocks, cudaStream_t st);
cudaError_t finalize_launch_batch(int NSL, int ND, const ApplyArgs* d_args, const int* d_off, int n, int nblocks,
                                  cudaStream_t st);

// Blocking set-up copies and memset on the calling thread's non-blocking
// stream (host side through a pinned staging buffer): unlike cudaMemcpy and
// cudaMemset they do not go through the legacy default stream. The current
// device must own dst (or src).
int copy_h2d(void* dst, const void* src, size_t bytes);
int copy_d2h(void* dst, const void* src, size_t bytes);
int memset_sync(void* dst, int value, size_t bytes);

// Returns the pool memory of a device that no buffer uses to the driver
// (waits for the device); the bytes the pool holds unused.
int devmem_trim(int device);
size_t devmem_cached_bytes(int device);

// Temporary device buffer ordered on a stream (cudaMallocAsync /
// cudaFreeAsync): unlike cudaFree, releasing it does not wait for the whole
// device, so set-up work on a private stream does not stall behind kernels
// that other threads keep running. release() must come before the stream is
// destroyed.
struct TmpBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  explicit TmpBuf(cudaStream_t s) : st(s) {}
  TmpBuf(const TmpBuf&) = delete;
  TmpBuf& operator=(const TmpBuf&) = delete;
  ~TmpBuf() { release(); }
  void release()
  {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
  }
  int alloc(size_t n);
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

// Simple owning device buffer.
// Owning device buffer from the device's stream-ordered memory pool, which
// keeps freed memory for reuse (cudaFree waits for the whole device, so
// releasing a mesh or a solver system while other threads keep the GPU busy
// would stall them). Memory goes back to the driver only through
// devmem_trim(). Releasing a buffer is only allowed once no queued work uses
// it (every caller synchronises first).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int dev = 0;
  bool owns = true;  // false: a view into another buffer (not freed here)
  ~DevBuf() { release(); }
  void release();
  // A view of [base, base + n) of a buffer that outlives it.
  void view(void* base, size_t n)
  {
    release();
    p = base;
    bytes = n;
    owns = false;
  }
  int alloc(size_t n);  // no-op when already at least n bytes
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

// Launch plan of the far field for one mesh (tile shape and work split).
struct FarPlan {
  int engine = 2;         // 0: CUDA-core far kernel; 1: tensor-core kernel, 2: symmetric kernel, where the variant has one
  int items_per_sm = 32;  // work items per SM the source ranges are cut into (load balance)
  int tile = 0;           // source triangles per shared-memory tile (0: the variant's default)
  int src_tile = kTS;     // tile of the last launch
  int nsplit = 1;         // source ranges per target tile
  int grid = 0;           // persistent CTAs of the last launch
  size_t smem = 0;
};

struct Mesh {
  HostMesh h;
  int device = 0;

  // static geometry (sorted order), views into one allocation (arena)
  DevBuf arena;
  DevBuf pos32, pos64, wj, trin, svid, perm, iperm, bary;
  DevBuf tgt32, tgt64, tgtw32, tgtw64, tcent, tnrm, tvid, ccent, snrm, ttile, twarp, splane32, splane64;
  // P1 x P1 single layer near field (built on first use)
  DevBuf p1_rowptr, p1_col, p1_val;
  // near field
  DevBuf sl_rowptr, sl_col, sl_val, dl_rowptr, dl_col, dl_val;
  // near-field sparse approximate inverse of V (solver preconditioner, built on first use)
  DevBuf pc_val;
  long long npairs = 0;
  // per-apply scratch
  DevBuf rec, partial, counter, items;
  std::vector<WorkItem> items_host;
  DevBuf io_t, io_u, io_v, io_q;
  // hypersingular: curl coefficients, vertex -> (triangle, local) lists, work vectors
  DevBuf curl9, vtri_ptr, vtri_list, elems0, hs_x, hs_w;
  // potential evaluation: per-chunk partial sums and host-call staging
  DevBuf pot_partial, io_pts, io_pot, pot_rec64;
  int nitems_work = 0;
  FarPlan plan;
  // one immutable device descriptor and launch shape per far-field variant
  // (key = fp32 * 64 + nsl * 5 + nd), so a queued launch never sees it change
  struct Variant {
    DevBuf desc;
    int grid = 0;
    size_t smem = 0;
    int src_tile = 0;
  };
  Variant variants[128];
  // tensor-core far field (fused FP32 SL+DL, 7-point rule): source operands
  // per cell, SL charges, a bounded-wait error flag and its descriptor
  DevBuf tc_bd2, tc_be, tc_charge, tc_err;
  Variant tc_var;
  bool tc_static_ready = false;
  bool tc_used = false;  // the last apply ran the tensor-core kernel
  // symmetric far field (7-point rule): its own work list and partial slots
  // (per output, one per target tile and row; the finalize reads only the
  // slots a row's items write), descriptor and launch shape
  DevBuf sym_items, sym_partial;
  std::vector<WorkItem> sym_items_host;
  int sym_nitems = 0, sym_nsplit = 0;
  Variant sym_var;
  bool sym_used = false;  // the last apply ran the symmetric kernel
  // host seconds of mesh creation: topology and pairs, static tables, near
  // field, and within the tables their device allocation and copy
  double setup_s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  // optional event timing of the far-field kernel
  bool profile = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  float last_far_ms = 0.f, last_fin_ms = 0.f;

  ~Mesh();
};

int mesh_create(int nv, const double* nodes, int ne, const int* elems1, int order, Mesh** out);
// Prep/finalize arguments of mesh m for the given scratch and vectors.
ApplyArgs mesh_apply_args(const Mesh* m, bool fp32, void* rec, const double* partial, const double* t, int tstride,
                          const double* u, double* v, int vstride, double* q);
// Source triangles per shared-memory tile of a far-field variant.
int src_tile_for(int Q, bool fp32, int nsl, int nd);
// Far-field descriptor of mesh m for the given scratch.
FarMeshDesc mesh_far_desc(const Mesh* m, bool fp32, int nsl, int nd, void* rec, double* partial);
// True when mesh m applies the fused FP32 SL+DL far field with the
// tensor-core kernel (engine 1, 7-point rule).
bool tc_eligible(const Mesh* m, bool fp32, int nsl, int nd);
// True when mesh m applies this far-field variant with a symmetric kernel
// (engine 2 for FP32, engine 3 for both precisions; 7-point rule, one target
// item per triangle; SL+DL, or SL only with 1, 3 or 4 columns).
// fp64_internal: an FP64 apply inside the library (the solver's residuals),
// which takes the symmetric kernel on engine 2 too.
bool sym_eligible(const Mesh* m, bool fp32, int nsl, int nd, bool fp64_internal = false);
// Device bytes of the symmetric kernels' partial slots for nout outputs.
size_t sym_slot_bytes(const HostMesh& h, int nout);
// Partial slots (summed over the rows, per output) the finalize of the next
// apply in `precision` with nsl SL and nd DL columns would fold.
long long mesh_far_slots(const Mesh* m, bool fp32, int nsl, int nd);
// The tensor-core distance operand of m (built once, synchronously).
int ensure_tc_static(Mesh* m);
// EB_ERR_TIMEOUT (and the flag cleared) if the last tensor-core launch on m
// gave up a bounded wait; EB_OK otherwise. The stream must be synchronised.
int mesh_check_far_error(Mesh* m);
// Device-pointer apply: t has nsl columns (stride ne), v likewise; u has nd
// DL columns (stride nnodes), q likewise (stride ne).
int mesh_apply(Mesh* m, int precision, int nsl, int nd, const double* d_t, const double* d_u, double* d_v,
               double* d_q, cudaStream_t st);

// u(x) = V t - W u at npts points (device arrays: pts [npts][3], t [nelems], u [nnodes]).
int mesh_evaluate_potential(Mesh* m, int precision, int npts, const double* d_pts, const double* d_t,
                            const double* d_u, double* d_out, cudaStream_t st);
// v = V1 t, P1 x P1 single layer; t and v have nnodes entries (device).
int mesh_apply_sl_p1(Mesh* m, int precision, const double* d_t, double* d_v, cudaStream_t st);
// Replaces the launch plan (work split, source tile) of a mesh; later applies
// and batches use it. No work on the mesh may be in flight.
int mesh_set_plan(Mesh* m, int items_per_sm, int tile);
// The tuned plan recorded for meshes like m (returns false if none).
bool tuned_plan_for(const HostMesh& h, int* items_per_sm, int* tile);
// Sparse approximate inverse of the SL near field on its own pattern (built once).
int ensure_near_precond(Mesh* m);
// y = M x with that inverse (original triangle order, device vectors).
cudaError_t near_precond_apply(const Mesh* m, const double* d_x, double* d_y, cudaStream_t st);
// vertex -> (triangle, local index) lists on the device (built on first use)
int ensure_vertex_lists(Mesh* m);
// q = D u (hypersingular, curl form); u and q have nnodes entries (device).
int mesh_apply_hypersingular(Mesh* m, int precision, const double* d_u, double* d_q, cudaStream_t st);

}  // namespace eb
