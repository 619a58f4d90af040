// Launch-plan tuning of the far field.
//
// A plan has two knobs: how many work items per SM the source range of every
// target tile is cut into (the persistent CTAs pull items from one queue, so
// more items balance better but add partial sums for the finalize kernel to
// add), and how many source triangles one shared-memory tile holds (fewer
// means less shared memory per CTA, more barriers). eb_autotune times every
// candidate on the mesh itself with CUDA events on a private stream, keeps
// the fastest on the mesh and records it in a process-wide table keyed by
// (SM count, size bucket = floor(log2 nelems), triangle-rule points,
// precision). Meshes created later in the same bucket start from the table,
// which can be written to and read from a text file. The reference has no
// counterpart (its launch shape is fixed at 256 threads per block).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "easybem_gpu.h"
#include "engine.h"

eb::Mesh* eb_mesh_internal(eb_mesh handle);

namespace eb {

namespace {

struct PlanRec {
  int items_per_sm = 32;
  int tile = 0;
  double ms = 0.0;
};
using PlanKey = std::tuple<int, int, int, int>;  // SMs, size bucket, rule points, precision

std::mutex g_plan_mu;
std::map<PlanKey, PlanRec> g_plans;

int size_bucket(int ne)
{
  int b = 0;
  while (b < 30 && (2 << b) <= ne) b++;
  return b;
}

int device_sms()
{
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nsm;
}

// deterministic densities for timing (values do not change the work done)
std::vector<double> timing_vector(size_t n, double phase)
{
  std::vector<double> x(n);
  for (size_t i = 0; i < n; i++) x[i] = std::sin(0.37 * (double)i + phase);
  return x;
}

}  // namespace

bool tuned_plan_for(const HostMesh& h, int* items_per_sm, int* tile)
{
  const int nsm = device_sms();
  std::lock_guard<std::mutex> g(g_plan_mu);
  for (int prec : {EB_PREC_MIXED, EB_PREC_FP64}) {
    auto it = g_plans.find(PlanKey(nsm, size_bucket(h.ne), h.Q, prec));
    if (it != g_plans.end()) {
      *items_per_sm = it->second.items_per_sm;
      *tile = it->second.tile;
      return true;
    }
  }
  return false;
}

static int time_plan(Mesh* m, int precision, int nsl, bool dl, int reps, const double* t, const double* u, double* v,
                     double* q, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, double* ms)
{
  EB_CHECK(mesh_apply(m, precision, nsl, dl, t, u, v, q, st));  // warm-up (builds the variant)
  std::vector<float> times;
  for (int r = 0; r < reps; r++) {
    EB_CUDA(cudaEventRecord(e0, st));
    EB_CHECK(mesh_apply(m, precision, nsl, dl, t, u, v, q, st));
    EB_CUDA(cudaEventRecord(e1, st));
    EB_CUDA(cudaEventSynchronize(e1));
    float x = 0.f;
    EB_CUDA(cudaEventElapsedTime(&x, e0, e1));
    times.push_back(x);
  }
  std::sort(times.begin(), times.end());
  *ms = times[times.size() / 2];
  return EB_OK;
}

int autotune(Mesh* m, int precision, int operators, int reps, int* best_ips, int* best_tile, double* best_ms,
             double* first_ms)
{
  if (precision != EB_PREC_MIXED && precision != EB_PREC_FP64)
    return set_error(EB_ERR_INVALID, "precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  if (operators < 1 || operators > 3) return set_error(EB_ERR_INVALID, "operators must be 1 (SL), 2 (DL) or 3 (both)");
  if (reps < 1 || reps > 100) return set_error(EB_ERR_INVALID, "reps must be in 1..100");
  const HostMesh& h = m->h;
  const int nsl = (operators & 1) ? 1 : 0;
  const bool dl = (operators & 2) != 0;
  DevBuf t, u, v, q;
  const std::vector<double> ht = timing_vector(h.ne, 0.0), hu = timing_vector(h.nv, 1.0);
  EB_CHECK(t.alloc(sizeof(double) * h.ne));
  EB_CHECK(v.alloc(sizeof(double) * h.ne));
  EB_CHECK(u.alloc(sizeof(double) * h.nv));
  EB_CHECK(q.alloc(sizeof(double) * h.ne));
  EB_CHECK(copy_h2d(t.p, ht.data(), sizeof(double) * h.ne));
  EB_CHECK(copy_h2d(u.p, hu.data(), sizeof(double) * h.nv));

  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  EB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const FarPlan start = m->plan;
  const int deft = src_tile_for(h.Q, precision == EB_PREC_MIXED, nsl, dl);
  std::vector<int> tiles{0};
  for (int c : {32, 16})
    if (c < deft) tiles.push_back(c);
  const int ips_list[] = {4, 8, 16, 32, 64, 128, 256, 512};

  int rc = EB_OK;
  PlanRec best{start.items_per_sm, start.tile, 1e300};
  double ms0 = 0.0;
  // the current plan first (its time is reported as the starting point)
  rc = time_plan(m, precision, nsl, dl, reps, t.as<double>(), u.as<double>(), v.as<double>(), q.as<double>(), st, e0,
                 e1, &ms0);
  if (rc == EB_OK) best.ms = ms0;
  for (int ips : ips_list) {
    for (int tile : tiles) {
      if (rc != EB_OK) break;
      if (ips == start.items_per_sm && tile == start.tile) continue;
      rc = mesh_set_plan(m, ips, tile);
      double ms = 0.0;
      if (rc == EB_OK)
        rc = time_plan(m, precision, nsl, dl, reps, t.as<double>(), u.as<double>(), v.as<double>(), q.as<double>(),
                       st, e0, e1, &ms);
      if (rc == EB_OK && ms < best.ms) best = PlanRec{ips, tile, ms};
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  // keep the winner (or put the starting plan back after a failure)
  const int rc2 = rc == EB_OK ? mesh_set_plan(m, best.items_per_sm, best.tile)
                              : mesh_set_plan(m, start.items_per_sm, start.tile);
  if (rc != EB_OK) return rc;
  EB_CHECK(rc2);
  {
    std::lock_guard<std::mutex> g(g_plan_mu);
    g_plans[PlanKey(device_sms(), size_bucket(h.ne), h.Q, precision)] = best;
  }
  if (best_ips) *best_ips = best.items_per_sm;
  if (best_tile) *best_tile = best.tile;
  if (best_ms) *best_ms = best.ms;
  if (first_ms) *first_ms = ms0;
  return EB_OK;
}

static const char kPlanHeader[] = "easybem-b200-plans 1";

int plan_table_save(const char* path)
{
  if (!path) return set_error(EB_ERR_INVALID, "null path");
  FILE* f = std::fopen(path, "w");
  if (!f) return set_error(EB_ERR_INVALID, std::string("cannot write ") + path);
  std::lock_guard<std::mutex> g(g_plan_mu);
  std::fprintf(f, "%s\n", kPlanHeader);
  for (const auto& kv : g_plans)
    std::fprintf(f, "%d %d %d %d %d %d %.6f\n", std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first),
                 std::get<3>(kv.first), kv.second.items_per_sm, kv.second.tile, kv.second.ms);
  const bool ok = std::fclose(f) == 0;
  return ok ? EB_OK : set_error(EB_ERR_INVALID, std::string("cannot write ") + path);
}

int plan_table_load(const char* path, int* loaded)
{
  if (!path) return set_error(EB_ERR_INVALID, "null path");
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error(EB_ERR_INVALID, std::string("cannot read ") + path);
  char line[256];
  if (!std::fgets(line, sizeof line, f) || std::string(line).rfind(kPlanHeader, 0) != 0) {
    std::fclose(f);
    return set_error(EB_ERR_INVALID, std::string("not a plan table: ") + path);
  }
  std::map<PlanKey, PlanRec> add;
  int sms, bucket, Q, prec, ips, tile;
  double ms;
  while (std::fgets(line, sizeof line, f)) {
    if (std::sscanf(line, "%d %d %d %d %d %d %lf", &sms, &bucket, &Q, &prec, &ips, &tile, &ms) != 7 || ips < 1 ||
        ips > 4096 || tile < 0 || tile > kTS || (prec != EB_PREC_MIXED && prec != EB_PREC_FP64)) {
      std::fclose(f);
      return set_error(EB_ERR_INVALID, std::string("bad plan table line in ") + path + ": " + line);
    }
    add[PlanKey(sms, bucket, Q, prec)] = PlanRec{ips, tile, ms};
  }
  std::fclose(f);
  std::lock_guard<std::mutex> g(g_plan_mu);
  for (const auto& kv : add) g_plans[kv.first] = kv.second;
  if (loaded) *loaded = (int)add.size();
  return EB_OK;
}

}  // namespace eb

// ---------------------------------------------------------------------------
// C ABI

using eb::set_error;

extern "C" {

int eb_mesh_set_plan(eb_mesh mesh, int items_per_sm, int src_tile)
{
  eb::Mesh* m = eb_mesh_internal(mesh);
  if (!m) return set_error(EB_ERR_INVALID, "null mesh");
  EB_CUDA(cudaSetDevice(m->device));
  return eb::mesh_set_plan(m, items_per_sm, src_tile);
}

int eb_mesh_get_plan(eb_mesh mesh, int* items_per_sm, int* src_tile, int* nsplit, int* work_items)
{
  eb::Mesh* m = eb_mesh_internal(mesh);
  if (!m) return set_error(EB_ERR_INVALID, "null mesh");
  if (items_per_sm) *items_per_sm = m->plan.items_per_sm;
  if (src_tile) *src_tile = m->plan.tile;
  if (nsplit) *nsplit = m->plan.nsplit;
  if (work_items) *work_items = m->nitems_work;
  return EB_OK;
}

int eb_autotune(eb_mesh mesh, int precision, int operators, int reps, int* items_per_sm, int* src_tile,
                double* best_ms, double* start_ms)
{
  eb::Mesh* m = eb_mesh_internal(mesh);
  if (!m) return set_error(EB_ERR_INVALID, "null mesh");
  EB_CUDA(cudaSetDevice(m->device));
  return eb::autotune(m, precision, operators, reps, items_per_sm, src_tile, best_ms, start_ms);
}

int eb_plan_table_save(const char* path) { return eb::plan_table_save(path); }

int eb_plan_table_load(const char* path, int* loaded) { return eb::plan_table_load(path, loaded); }

int eb_plan_table_clear(void)
{
  std::lock_guard<std::mutex> g(eb::g_plan_mu);
  eb::g_plans.clear();
  return EB_OK;
}

}  // extern "C"
