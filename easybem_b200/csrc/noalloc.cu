// An apply entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they need a matvec: an
// application whose memory is owned by its own pool or framework allocator
// (so that a stray cudaMalloc would fragment or exceed a budget it enforces),
// or a real-time loop that must not hit the driver's allocator, which can
// synchronise the device. eb_apply_sl_dl_noalloc serves them: the caller
// passes device pointers for the densities and the results, the mesh must
// already exist (eb_mesh_create allocates its resident geometry once), and
// every per-apply scratch buffer (source records, partial row sums, the work
// counter and the launch descriptor) lives in one fixed device array defined
// in this file.
//
// That array has kNoAllocScratchBytes bytes and is held by every GPU that
// loads the library until the process exits. Meshes whose scratch would not
// fit are rejected with EB_ERR_INVALID and a message stating the size. All
// calls share the array and the last call's contents stay in it; the work
// counter is cleared by each call. Two calls whose work overlaps on the GPU
// (different streams, or different meshes at the same time) race on the
// array: issue them on one stream or wait in between.
//
// The first call on each device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture. With CUDA's lazy module loading (the default)
// the array is only placed in device memory at that first lookup, so the
// first call on a device is where its 32 MiB are taken: make it (or one
// warm-up call) at start-up, before the caller's own allocator fills the
// device; if no room is left then, it returns EB_ERR_CUDA. The looked-up
// address is kept for the life of the process, so after cudaDeviceReset the
// library must be loaded again.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <string>

#include "engine.h"

namespace eb {

constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 32 MiB
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device, looked up once under
// g_noalloc_mu (calls from several host threads may race to the first lookup).
static std::atomic<void*> g_noalloc_ptr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mu;

static size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Writes the launch descriptor (passed by value) into the scratch array.
__global__ void noalloc_store_desc(FarMeshDesc d, FarMeshDesc* dst)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = d;
}

}  // namespace eb

// The mesh behind a handle (defined with the handle in engine.cu).
eb::Mesh* eb_mesh_internal(eb_mesh handle);

extern "C" int eb_apply_sl_dl_noalloc(eb_mesh handle, int precision, const double* d_t, const double* d_u,
                                      double* d_v, double* d_q, void* stream)
{
  using namespace eb;
  if (!handle) return set_error(EB_ERR_INVALID, "null mesh");
  Mesh* m = eb_mesh_internal(handle);
  const HostMesh& h = m->h;
  if (precision != EB_PREC_FP64 && precision != EB_PREC_MIXED)
    return set_error(EB_ERR_INVALID, "precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  const bool sl = d_t && d_v, dl = d_u && d_q;
  if (!sl && !dl) return set_error(EB_ERR_INVALID, "nothing to apply: pass t/v and/or u/q");
  const int nsl = sl ? 1 : 0;
  const bool fp32 = precision == EB_PREC_MIXED;
  if (m->device < 0 || m->device >= kNoAllocMaxDevices)
    return set_error(EB_ERR_INVALID, "device index " + std::to_string(m->device) + " beyond the " +
                                         std::to_string(kNoAllocMaxDevices) + " devices eb_apply_sl_dl_noalloc serves");
  EB_CUDA(cudaSetDevice(m->device));

  // scratch layout: [counter | descriptor | source records | partial sums]
  const int nrec = rec_slots(nsl, dl);
  const size_t slot = fp32 ? sizeof(float4) : sizeof(dq);
  const size_t off_desc = 256;
  const size_t off_rec = off_desc + align256(sizeof(FarMeshDesc));
  const size_t rec_bytes = (size_t)h.ne * h.Q * nrec * slot;
  const size_t off_part = off_rec + align256(rec_bytes);
  const int nout = nsl + (dl ? 1 : 0);
  const size_t part_bytes = sizeof(double) * (size_t)nout * m->plan.nsplit * h.nitems;
  const size_t need = off_part + align256(part_bytes);
  if (need > kNoAllocScratchBytes)
    return set_error(EB_ERR_INVALID, "this mesh needs " + std::to_string(need) +
                                         " bytes of apply scratch; eb_apply_sl_dl_noalloc holds at most " +
                                         std::to_string(kNoAllocScratchBytes) + " bytes (use eb_apply_sl_dl_device)");

  // once per device, with that device current
  void* scratch = g_noalloc_ptr[m->device].load(std::memory_order_acquire);
  if (!scratch) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    scratch = g_noalloc_ptr[m->device].load(std::memory_order_relaxed);
    if (!scratch) {
      EB_CUDA(cudaGetSymbolAddress(&scratch, g_noalloc_scratch));
      g_noalloc_ptr[m->device].store(scratch, std::memory_order_release);
    }
  }
  unsigned char* base = static_cast<unsigned char*>(scratch);
  int* counter = reinterpret_cast<int*>(base);
  FarMeshDesc* d_desc = reinterpret_cast<FarMeshDesc*>(base + off_desc);
  void* rec = base + off_rec;
  double* partial = reinterpret_cast<double*>(base + off_part);
  cudaStream_t st = (cudaStream_t)stream;

  const FarMeshDesc desc = mesh_far_desc(m, fp32, nsl, dl, rec, partial);
  const size_t smem = far_smem_bytes(desc.src_tile, h.Q, nrec, fp32);
  int occ = far_occupancy(fp32, nsl, dl, h.K, h.Q, smem);
  if (occ < 1) occ = 1;
  int nsm = 148;
  EB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device));
  const int grid = std::min(nsm * occ, std::max(1, m->nitems_work));

  noalloc_store_desc<<<1, 32, 0, st>>>(desc, d_desc);
  EB_CUDA(cudaGetLastError());
  const ApplyArgs A = mesh_apply_args(m, fp32, rec, partial, d_t, h.ne, d_u, d_v, h.ne, d_q);
  EB_CUDA(prep_launch(fp32, nsl, dl, A, st));
  EB_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
  EB_CUDA(far_launch(fp32, nsl, dl, h.K, h.Q, d_desc, m->items.as<WorkItem>(), m->nitems_work, counter, smem, grid,
                     st));
  EB_CUDA(finalize_launch(nsl, dl, A, st));
  return EB_OK;
}
