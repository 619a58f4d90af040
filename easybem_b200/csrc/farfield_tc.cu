// Far field of the fused FP32 SL+DL apply with the pair distances on the
// tensor cores (sm_100a tcgen05).
//
// Per far quadrature pair the CUDA-core kernel (farfield.cu) spends 8
// FMA-pipe operations and one MUFU reciprocal square root, and the two pipes
// bound it together. Two of its terms are bilinear in the target point x and
// the source point y (both relative to the source cell's centre):
//
//   |x - y|^2       = x.(-2y) + |x|^2 + |y|^2
//   e = s (x - y).n = x.(s n) - s (P0 - c).n      (s: DL strength of y, n: normal
//                                                  of y's triangle, flat triangle)
//
// so for a tile of 128 target triangles (one target point index a at a time)
// against 112 source points they are two M=128 x N=112 GEMMs with the
// coordinates split into TF32 high and low parts (x y ~ xh yh + xl yh + xh yl,
// K = 16 with |x|^2, |y|^2 and the constants as extra columns). tcgen05.mma
// writes both into tensor memory; the threads read them back with
// tcgen05.ld and keep only the non-linear part on the CUDA cores:
//
//   r = rsqrt(d2),  sl += c r,  dl += e r^3      (1 MUFU + 4 FMA-pipe operations)
//
// which leaves MUFU as the only saturated pipe. Source operands are
// prepared in global memory in the UMMA K-major, no-swizzle layout (per cell
// of kCell triangles: 8-row groups of 512 bytes, four 16-byte K groups per
// row group), copied into shared memory per cell; the target operand of each
// point index is built per cell by the threads (cell-relative coordinates,
// FP64-formed offsets, as the CUDA-core kernel does). Cells that are not well
// separated from the target tile (shared vertices possible) run the
// CUDA-core code. Accumulation: per cell in FP32, per item in a two-sum
// (float-float) pair, FP64 partial sums, as in the CUDA-core kernel.
//
// Launch: one persistent CTA of 256 threads per SM (two warpgroups split
// every 112-column chunk into halves of 56 columns), 512 tensor-memory
// columns: two buffers x (d2, e) x 112. Round r = (chunk, point index) is
// issued by one thread into buffer r % 2 while the threads evaluate round
// r - 1. Every wait on an mbarrier is bounded; a wait that runs out sets an
// error flag, the CTA stops taking work, releases its tensor memory and
// exits, and the host reports EB_ERR_TIMEOUT.
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"
#include "farfield_eval.cuh"
#include "farfield_tc.h"

namespace eb {

namespace tc {

constexpr int kThreads = 256;
constexpr int kQ = 7;
constexpr int kChunk = kTcChunk;               // 112 source points per MMA
constexpr int kCellPts = kCell * kQ;           // 224 source points per cell
constexpr int kChunks = kCellPts / kChunk;     // 2
constexpr int kRounds = kChunks * kQ;          // 14 (chunk, point index) rounds per cell
constexpr int kHalf = kChunk / 2;              // 56 columns per warpgroup
constexpr int kRowBytes = 64;                  // 16 TF32 per operand row
constexpr int kABytes = 128 * kRowBytes;       // one target operand (128 rows)
constexpr int kCellBBytes = kCellPts * kRowBytes;  // 14,336: one source operand of a cell
constexpr int kTmemCols = 512;
constexpr unsigned kWaitLimit = 1u << 20;      // try_wait calls before a wait gives up

static_assert(kCellPts % kChunk == 0 && kChunk % 16 == 0, "chunk shape");
static_assert(kTT == 128, "one tensor-memory lane per target triangle");

// Source operands of the next well-separated cell of a work item are copied
// into a second set of buffers (cp.async) while the current cell's rounds run.
#ifndef EB_TC_PREFETCH
#define EB_TC_PREFETCH 1  // measured: 159.7 -> 146.4 ms at L6
#endif
constexpr int kSets = EB_TC_PREFETCH ? 2 : 1;

// dynamic shared memory layout (bytes); an operand set is (d2 operand, e
// operand, charges) of one cell
constexpr int kOffA = 0;                                   // 7 target operands
constexpr int kSetBytes = 2 * kCellBBytes + kCellPts * 4;  // 29,568
constexpr int kOffSets = kOffA + kQ * kABytes;
constexpr int kOffRec = kOffSets + kSets * kSetBytes;      // CUDA-core records of a near cell
constexpr int kOffEnd = kOffRec + kCellPts * 2 * 16;
// more than half of the SM's shared memory: one CTA per SM (it holds all
// 512 tensor-memory columns)
constexpr int kSmemBytes = kSets == 1 ? 120 * 1024 : 124 * 1024;
static_assert(kOffEnd <= kSmemBytes, "shared memory layout");
static_assert(kSetBytes % 16 == 0, "16-byte aligned operand sets");

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_rna(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// K-major, no-swizzle shared-memory matrix descriptor: 8-row core matrices of
// 16-byte rows, K groups LBO = 128 bytes apart, 8-row groups SBO = 512 bytes
// apart, descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)(128 >> 4) << 16;
  d |= (uint64_t)(512 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: D F32, A and B TF32, both K-major, N = kChunk, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kChunk >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Waits for phase `parity` of the mbarrier to complete; false if it did not
// within kWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 8 consecutive 32-bit columns of this thread's tensor-memory lane (the
// column offset is a multiple of 8)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v)
{
  uint32_t* r = reinterpret_cast<uint32_t*>(v);
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Copies cell `cell`'s d2 and e operands and charges into an operand set:
// synchronously (ASYNC false) or with cp.async (committed as one group).
template <bool ASYNC>
__device__ __forceinline__ void load_cell_operands(unsigned char* set, const FarMeshDesc& md, int cell, int tid)
{
  const float4* gB = reinterpret_cast<const float4*>(reinterpret_cast<const char*>(md.tc_bd2) + (size_t)cell * kCellBBytes);
  const float4* gE = reinterpret_cast<const float4*>(reinterpret_cast<const char*>(md.tc_be) + (size_t)cell * kCellBBytes);
  const float4* gC = reinterpret_cast<const float4*>(md.tc_charge + (size_t)cell * kCellPts);
  float4* sB = reinterpret_cast<float4*>(set);
  float4* sE = reinterpret_cast<float4*>(set + kCellBBytes);
  float4* sC = reinterpret_cast<float4*>(set + 2 * kCellBBytes);
  for (int k = tid; k < kCellBBytes / 16; k += kThreads) {
    if constexpr (ASYNC) {
      cp_async16(sB + k, gB + k);
      cp_async16(sE + k, gE + k);
    } else {
      sB[k] = gB[k];
      sE[k] = gE[k];
    }
  }
  for (int k = tid; k < kCellPts / 4; k += kThreads) {
    if constexpr (ASYNC) cp_async16(sC + k, gC + k);
    else sC[k] = gC[k];
  }
  if constexpr (ASYNC) cp_async_commit();
}

// Columns of every 16 whose reciprocal square root runs on the FMA pipe
// instead of MUFU (MUFU is the tensor-core kernel's only saturated pipe; the
// FMA pipe has half its time left).
#ifndef EB_TC_NEWTON
#define EB_TC_NEWTON 2  // measured best of 0, 2, 4 (L6: 146.4, 141.1, 145.7 ms with the prefetch)
#endif
constexpr int kNewtonPer16 = EB_TC_NEWTON;
// Tensor-memory columns read per wait (a multiple of 8).
#ifndef EB_TC_SUB
#define EB_TC_SUB 16
#endif
constexpr int kSubCols = EB_TC_SUB;
// Independent accumulators per product and thread within a round.
#ifndef EB_TC_ACC
#define EB_TC_ACC 1  // measured best of 1, 2, 4 (L6: 138.3, 141.3, 144.5 ms)
#endif
constexpr int kAcc = EB_TC_ACC;
static_assert(kSubCols % 8 == 0 && kSubCols >= 8 && kSubCols <= 56, "tensor-memory read block");
static_assert(kNewtonPer16 % 2 == 0 && kNewtonPer16 <= 16, "Newton columns come in pairs");

// 1/sqrt(x) of two values on the FMA pipe: the magic-constant seed of the
// "fast inverse square root" (constant 0x5f375a86 from C. Lomont, "Fast
// Inverse Square Root", 2003; relative error < 3.5e-2) and three Newton
// steps y <- y (3/2 - x/2 y^2), which square the error each time (below the
// FP32 rounding after the third). 2 integer and 10 FP32 lane operations per
// value.
__device__ __forceinline__ float2 rsqrt2_newton(float2 x)
{
  float2 y = make_float2(__int_as_float(0x5f375a86 - (__float_as_int(x.x) >> 1)),
                         __int_as_float(0x5f375a86 - (__float_as_int(x.y) >> 1)));
  const float2 hx = __fmul2_rn(make_float2(-0.5f, -0.5f), x);
  const float2 c15 = make_float2(1.5f, 1.5f);
#pragma unroll
  for (int k = 0; k < 3; ++k) y = __fmul2_rn(y, __ffma2_rn(hx, __fmul2_rn(y, y), c15));
  return y;
}

// byte offset of (row, 16-byte K group) in the UMMA K-major no-swizzle layout
__host__ __device__ constexpr int umma_off(int row, int kg) { return (row >> 3) * 512 + kg * 128 + (row & 7) * 16; }

}  // namespace tc

// ---------------------------------------------------------------------------
// Source operands. Row p of cell c (point p of the cell's kCell triangles):
//   d2: [-2y_h, -2y_h, -2y_l, 1, 1, |y|^2_h, |y|^2_l, 0, 0, 0]
//   e : [(s n)_h, (s n)_h, (s n)_l, 0, 0, (-s h)_h, (-s h)_l, 0, 0, 0]
// (h = (P0 - c).n the plane offset of the point's triangle). Points past the
// last triangle get d2 = |x|^2 + 1 and e = 0: finite and without effect.

__global__ void tc_prep_static_kernel(int ne, int ncells, const float4* __restrict__ pos32, float4* __restrict__ bd2)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ncells * tc::kCellPts) return;
  const int c = idx / tc::kCellPts, p = idx % tc::kCellPts;
  float row[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) row[k] = 0.f;
  if (idx < ne * tc::kQ) {
    const float4 y = pos32[idx];
    const float m[3] = {y.x, y.y, y.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float h = tc::tf32_rna(m[k]);
      row[k] = h;
      row[3 + k] = h;
      row[6 + k] = tc::tf32_rna(m[k] - h);
    }
    row[9] = 1.f;
    row[10] = 1.f;
    const float wh = tc::tf32_rna(y.w);
    row[11] = wh;
    row[12] = tc::tf32_rna(y.w - wh);
  } else {
    row[11] = 1.f;
  }
  char* base = reinterpret_cast<char*>(bd2) + (size_t)c * tc::kCellBBytes;
#pragma unroll
  for (int kg = 0; kg < 4; ++kg)
    *reinterpret_cast<float4*>(base + tc::umma_off(p, kg)) =
        make_float4(row[4 * kg], row[4 * kg + 1], row[4 * kg + 2], row[4 * kg + 3]);
}

// records of the fused SL+DL FP32 variant: slot1 = (s, c, 0, 0)
__device__ __forceinline__ void tc_prep_dl_point(int idx, int ne, int ncells, const float4* __restrict__ rec,
                                                 const float4* __restrict__ splane32, float4* __restrict__ be,
                                                 float* __restrict__ charges)
{
  if (idx >= ncells * tc::kCellPts) return;
  const int c = idx / tc::kCellPts, p = idx % tc::kCellPts;
  float row[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) row[k] = 0.f;
  float charge = 0.f;
  if (idx < ne * tc::kQ) {
    const float4 r1 = rec[(size_t)idx * 2 + 1];
    const float4 pl = splane32[idx / tc::kQ];
    const float g[3] = {r1.x * pl.x, r1.x * pl.y, r1.x * pl.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float h = tc::tf32_rna(g[k]);
      row[k] = h;
      row[3 + k] = h;
      row[6 + k] = tc::tf32_rna(g[k] - h);
    }
    const float kk = -r1.x * pl.w;
    const float kh = tc::tf32_rna(kk);
    row[11] = kh;
    row[12] = tc::tf32_rna(kk - kh);
    charge = r1.y;
  }
  char* base = reinterpret_cast<char*>(be) + (size_t)c * tc::kCellBBytes;
#pragma unroll
  for (int kg = 0; kg < 4; ++kg)
    *reinterpret_cast<float4*>(base + tc::umma_off(p, kg)) =
        make_float4(row[4 * kg], row[4 * kg + 1], row[4 * kg + 2], row[4 * kg + 3]);
  charges[idx] = charge;
}

__global__ void tc_prep_dl_kernel(int ne, int ncells, const float4* __restrict__ rec, const float4* __restrict__ splane32,
                                  float4* __restrict__ be, float* __restrict__ charges)
{
  tc_prep_dl_point(blockIdx.x * blockDim.x + threadIdx.x, ne, ncells, rec, splane32, be, charges);
}

__global__ void tc_prep_dl_batch_kernel(const TcPrepArgs* __restrict__ args, const int* __restrict__ off, int n)
{
  int lo = 0, hi = n;  // off[lo] <= blockIdx.x < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= (int)blockIdx.x) lo = mid;
    else hi = mid;
  }
  const TcPrepArgs A = args[lo];
  if (A.active && *A.active == 0) return;
  tc_prep_dl_point((blockIdx.x - off[lo]) * blockDim.x + threadIdx.x, A.ne, A.ncells, A.rec, A.splane32, A.be,
                   A.charges);
}

__global__ void __launch_bounds__(tc::kThreads, 1)
    far_tc_kernel(const FarMeshDesc* __restrict__ meshes, const WorkItem* __restrict__ items, int nitems,
                  int* __restrict__ counter, int* __restrict__ error_flag)
{
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t s_mbar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_item;
  __shared__ int s_stop;
  __shared__ int4 s_vid[kCell];
  __shared__ dq s_nrm[kCell];
  __shared__ float4 s_plane[kCell];
  __shared__ float s_comb[4][128];

  const int tid = threadIdx.x;
  const int wg = tid >> 7;          // warpgroup: columns [wg * 56, wg * 56 + 56) of every chunk
  const int row = tid & 127;        // target triangle of the tile = tensor-memory lane
  const int warp = tid >> 5;
  unsigned char* sA = smem + kOffA;
  float* sRec = reinterpret_cast<float*>(smem + kOffRec);
  int set_cur = 0;  // operand set of the current far cell (uniform)
  const uint32_t mbar0 = smem_u32(&s_mbar[0]);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(mbar0, 1);
    mbar_init(mbar0 + 8, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_stop = 0;
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = s_tmem;
  uint32_t phase_bits = 0u;  // bit b: parity of the next completion of mbarrier b

  for (;;) {
    if (tid == 0) s_item = s_stop ? nitems : atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const WorkItem w = items[it];
    const FarMeshDesc md = meshes[w.mesh];
    if (md.active && *md.active == 0) continue;
    const int ti = w.tgt0 + row;
    const bool active = ti < md.nitems;
    const int tsel = active ? ti : w.tgt0;
    const dq tile = md.ttile[w.tgt0 / kTT];
    double cen[3], nrm[3];
    {
      const dq c = md.tcent[tsel];
      cen[0] = c.x; cen[1] = c.y; cen[2] = c.z;
      const dq n = md.tnrm[tsel];
      nrm[0] = n.x; nrm[1] = n.y; nrm[2] = n.z;
    }
    const int4 tv = active ? md.tvid[tsel] : make_int4(-1, -1, -1, 0);
    float pw[kQ];
#pragma unroll
    for (int a = 0; a < kQ; ++a) pw[a] = md.tgt32[(size_t)tsel * kQ + a].w;
    float acc_hi[2] = {0.f, 0.f}, acc_lo[2] = {0.f, 0.f};  // SL, DL
    const float4* rec = reinterpret_cast<const float4*>(md.rec);
    auto is_far = [&](int c) {  // tile-level separation test: uniform across the CTA
      const dq cc = md.ccent[c];
      const double ddx = cc.x - tile.x, ddy = cc.y - tile.y, ddz = cc.z - tile.z;
      const double rr = kFarRatio * (cc.w + tile.w);
      return ddx * ddx + ddy * ddy + ddz * ddz > rr * rr;
    };
    int prefetched = -1;  // cell whose operands are in flight into set set_cur ^ 1

    for (int cell = w.cell0; cell < w.cell1; ++cell) {
      const int s0 = cell * kCell, s1 = min(md.ne, s0 + kCell);
      const dq cc = md.ccent[cell];
      const bool far = is_far(cell);
      const float o[3] = {(float)(cc.x - cen[0]), (float)(cc.y - cen[1]), (float)(cc.z - cen[2])};
      float xs[kQ], ys[kQ], zs[kQ], q2[kQ];
#pragma unroll
      for (int a = 0; a < kQ; ++a) {
        const float4 p = md.tgt32[(size_t)tsel * kQ + a];
        xs[a] = p.x - o[0]; ys[a] = p.y - o[1]; zs[a] = p.z - o[2];
        q2[a] = xs[a] * xs[a] + ys[a] * ys[a] + zs[a] * zs[a];
      }
      float part_sl = 0.f, part_dl = 0.f;
      if (!far) {
        // CUDA-core path: the two warpgroups take halves of the cell's triangles
        const int npt = (s1 - s0) * kQ;
        for (int k = tid; k < npt * 2; k += kThreads) reinterpret_cast<float4*>(sRec)[k] = rec[(size_t)s0 * kQ * 2 + k];
        for (int k = tid; k < s1 - s0; k += kThreads) {
          s_vid[k] = md.svid[s0 + k];
          s_nrm[k] = md.snrm[s0 + k];
          s_plane[k] = md.splane32[s0 + k];
        }
        __syncthreads();
        if (active) {
          const int mid = (s1 - s0 + 1) / 2;
          float sl[1][kQ], dl[1][kQ];
#pragma unroll
          for (int a = 0; a < kQ; ++a) sl[0][a] = dl[0][a] = 0.f;
          eval_cell_x2<kQ, kQ, 1, 1, false>(sRec, s_vid, s_nrm, s_plane, wg ? mid : 0, wg ? s1 - s0 : mid, kQ, tv,
                                            xs, ys, zs, q2, o, cen, nrm, sl, dl);
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
            part_sl += pw[a] * sl[0][a];
            part_dl += pw[a] * dl[0][a];
          }
        }
        __syncthreads();
      } else {
        // target operands: warpgroup 0 builds point indices 0..3, warpgroup 1 4..6
#pragma unroll
        for (int a = 0; a < kQ; ++a) {
          if ((a < 4) != (wg == 0)) continue;
          float v[16];
          const float x3[3] = {xs[a], ys[a], zs[a]};
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const float h = active ? tf32_rna(x3[k]) : 0.f;
            v[k] = h;
            v[3 + k] = active ? tf32_rna(x3[k] - h) : 0.f;
            v[6 + k] = h;
          }
          const float qh = active ? tf32_rna(q2[a]) : 0.f;
          v[9] = qh;
          v[10] = active ? tf32_rna(q2[a] - qh) : 0.f;
          v[11] = 1.f;
          v[12] = 1.f;
          v[13] = v[14] = v[15] = 0.f;
          unsigned char* dstA = sA + a * kABytes;
#pragma unroll
          for (int kg = 0; kg < 4; ++kg)
            *reinterpret_cast<float4*>(dstA + umma_off(row, kg)) =
                make_float4(v[4 * kg], v[4 * kg + 1], v[4 * kg + 2], v[4 * kg + 3]);
        }
        // source operands and charges of the cell: already in flight into
        // the other set, or copied now
        if (kSets == 2 && prefetched == cell) {
          set_cur ^= 1;
          cp_async_wait_all();
        } else {
          load_cell_operands<false>(smem + kOffSets + set_cur * kSetBytes, md, cell, tid);
        }
        prefetched = -1;
        unsigned char* set = smem + kOffSets + set_cur * kSetBytes;
        unsigned char* sB = set;
        unsigned char* sE = set + kCellBBytes;
        const float* sC = reinterpret_cast<const float*>(set + 2 * kCellBBytes);
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        // the next cell's operands into the other set while these rounds run
        // (that set's last reader, the previous far cell's MMAs, has completed)
        if (kSets == 2 && cell + 1 < w.cell1 && is_far(cell + 1)) {
          load_cell_operands<true>(smem + kOffSets + (set_cur ^ 1) * kSetBytes, md, cell + 1, tid);
          prefetched = cell + 1;
        }
        const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB), eBase = smem_u32(sE);
        auto issue = [&](int r) {
          const int a = r % kQ, ch = r / kQ;  // thread 0 only: runtime indices are fine here
          const uint32_t d2 = tmem + (uint32_t)((r & 1) * 2 * kChunk);
          const uint32_t de = d2 + kChunk;
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {  // two K steps of 8 TF32
            const uint64_t ad = umma_desc(aBase + a * kABytes + ks * 256);
            mma_tf32(d2, ad, umma_desc(bBase + ch * (kChunk / 8) * 512 + ks * 256), ks);
            mma_tf32(de, ad, umma_desc(eBase + ch * (kChunk / 8) * 512 + ks * 256), ks);
          }
          mma_commit(mbar0 + 8 * (r & 1));
        };
        if (tid == 0) issue(0);
        float2 slp[kQ], dlp[kQ];
#pragma unroll
        for (int a = 0; a < kQ; ++a) {
          slp[a] = make_float2(0.f, 0.f);
          dlp[a] = make_float2(0.f, 0.f);
        }
        bool ok = true;
#pragma unroll 1
        for (int ch = 0; ch < kChunks && ok; ++ch) {
#pragma unroll
        for (int a = 0; a < kQ; ++a) {
          const int r = ch * kQ + a;
          if (tid == 0 && r + 1 < kRounds) issue(r + 1);
          const int b = r & 1;
          const bool waited = mbar_wait(mbar0 + 8 * b, (phase_bits >> b) & 1u);
          phase_bits ^= 1u << b;
          fence_after_sync();
          const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;
          const uint32_t d2 = tmem + lane + (uint32_t)(b * 2 * kChunk + wg * kHalf);
          const uint32_t de = d2 + kChunk;
          const float* cc2 = sC + ch * kChunk + wg * kHalf;
          // kAcc independent accumulator pairs per product (column pairs taken
          // round-robin) so consecutive FFMA2s do not wait on each other
          float2 sl2[kAcc], dl2[kAcc];
#pragma unroll
          for (int k = 0; k < kAcc; ++k) sl2[k] = dl2[k] = make_float2(0.f, 0.f);
          // the warpgroup's 56 columns in blocks of kSubCols (the last one shorter)
#pragma unroll
          for (int h0 = 0; h0 < kHalf; h0 += kSubCols) {
            constexpr int kMax = kSubCols;
            const int nb = min(kSubCols, kHalf - h0) / 8;  // x8 loads per product (compile-time after unrolling)
            float vd[kMax], ve[kMax];
#pragma unroll
            for (int k = 0; k < kMax / 8; ++k)
              if (k < nb) {
                tmem_ld8(d2 + h0 + 8 * k, vd + 8 * k);
                tmem_ld8(de + h0 + 8 * k, ve + 8 * k);
              }
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < kMax; j += 2) {
              if (j >= 8 * nb) break;
              const float2 cj = *reinterpret_cast<const float2*>(cc2 + h0 + j);
              const float2 ri = (j % 16) >= 16 - kNewtonPer16 ? rsqrt2_newton(make_float2(vd[j], vd[j + 1]))
                                                              : make_float2(rsq(vd[j]), rsq(vd[j + 1]));
              const int k = ((h0 + j) / 2) % kAcc;
              sl2[k] = __ffma2_rn(cj, ri, sl2[k]);
              dl2[k] = __ffma2_rn(__fmul2_rn(ri, ri), __fmul2_rn(make_float2(ve[j], ve[j + 1]), ri), dl2[k]);
            }
          }
#pragma unroll
          for (int k = 0; k < kAcc; ++k) {
            slp[a] = __fadd2_rn(slp[a], sl2[k]);
            dlp[a] = __fadd2_rn(dlp[a], dl2[k]);
          }
          fence_before_sync();
          ok = __syncthreads_and(waited) != 0;  // buffer b is free for round r + 2; same verdict in every thread
          fence_after_sync();
          if (!ok) break;
        }
        }
        if (!ok) {
          if (tid == 0) atomicExch(error_flag, 1);
          s_stop = 1;
          cp_async_wait_all();
          // wait (bounded) for the MMAs already issued before the memory is released
          for (int b = 0; b < 2; ++b) mbar_wait(mbar0 + 8 * b, (phase_bits >> b) & 1u);
          break;
        }
        if (active) {
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
            part_sl += pw[a] * (slp[a].x + slp[a].y);
            part_dl += pw[a] * (dlp[a].x + dlp[a].y);
          }
        }
      }
      two_sum_add(acc_hi[0], acc_lo[0], part_sl);
      two_sum_add(acc_hi[1], acc_lo[1], part_dl);
    }
    // combine the warpgroups' sums and write the item's partial slots
    __syncthreads();
    if (wg == 1) {
      s_comb[0][row] = acc_hi[0];
      s_comb[1][row] = acc_lo[0];
      s_comb[2][row] = acc_hi[1];
      s_comb[3][row] = acc_lo[1];
    }
    __syncthreads();
    if (wg == 0 && active) {
      const size_t stride = (size_t)md.nsplit * md.nitems;
      double* out = md.partial + (size_t)w.split * md.nitems + ti;
      out[0] = ((double)acc_hi[0] + (double)acc_lo[0]) + ((double)s_comb[0][row] + (double)s_comb[1][row]);
      out[stride] = ((double)acc_hi[1] + (double)acc_lo[1]) + ((double)s_comb[2][row] + (double)s_comb[3][row]);
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

void far_tc_costs(double* mufu_per_pair, double* fma_ops_per_pair, double* tensor_flops_per_pair)
{
  // per warpgroup round: kHalf columns, of which 3 x kNewtonPer16 take the FMA-pipe root
  const double f = 3.0 * tc::kNewtonPer16 / tc::kHalf;
  if (mufu_per_pair) *mufu_per_pair = 1.0 - f;
  if (fma_ops_per_pair) *fma_ops_per_pair = 4.0 + 10.0 * f;  // SL 1, DL 3; Newton root 10
  if (tensor_flops_per_pair) *tensor_flops_per_pair = 2.0 * 2.0 * 16.0;  // two GEMMs, K = 16, FMA = 2 flops
}

cudaError_t far_tc_prep_static(int ne, int ncells, const float4* pos32, float4* bd2, cudaStream_t st)
{
  const int n = ncells * tc::kCellPts;
  tc_prep_static_kernel<<<(n + 255) / 256, 256, 0, st>>>(ne, ncells, pos32, bd2);
  return cudaGetLastError();
}

cudaError_t far_tc_prep_dl(int ne, int ncells, const float4* rec, const float4* splane32, float4* be, float* charges,
                           cudaStream_t st)
{
  const int n = ncells * tc::kCellPts;
  tc_prep_dl_kernel<<<(n + 255) / 256, 256, 0, st>>>(ne, ncells, rec, splane32, be, charges);
  return cudaGetLastError();
}

cudaError_t far_tc_prep_dl_batch(const TcPrepArgs* d_args, const int* d_off, int n, int nblocks, cudaStream_t st)
{
  if (nblocks > 0) tc_prep_dl_batch_kernel<<<nblocks, 256, 0, st>>>(d_args, d_off, n);
  return cudaGetLastError();
}

cudaError_t far_tc_launch(const FarMeshDesc* d_meshes, const WorkItem* d_items, int nitems, int* d_counter,
                          int* d_error, int grid, cudaStream_t st)
{
  cudaError_t e = cudaFuncSetAttribute(far_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes);
  if (e != cudaSuccess) return e;
  far_tc_kernel<<<grid, tc::kThreads, tc::kSmemBytes, st>>>(d_meshes, d_items, nitems, d_counter, d_error);
  return cudaGetLastError();
}

}  // namespace eb
