// The reference's process-global C++ GPU interface (include/BEM3dLaplaceGPU.h:
// 8-18, implemented in src/BEM3dLaplaceGPU.cu:830-1555) as a shim over one
// default eb_mesh handle. python/bindings.cpp:6 declares `extern int ne,
// nnodes;` and sizes its result arrays with them, so both are defined here.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/BEM3dLaplaceGPU.h"
#include "../../include/easybem_gpu.h"

int ne = 0;
int nnodes = 0;

static eb_mesh g_mesh = nullptr;

static int legacy_precision()
{
  const char* p = std::getenv("EASYBEM_PRECISION");
  if (p && (std::strcmp(p, "mixed") == 0 || std::strcmp(p, "fp32") == 0)) return EB_PREC_MIXED;
  return EB_PREC_FP64;
}

static void report(const char* what, int st)
{
  if (st != EB_OK) std::fprintf(stderr, "easybem: %s failed (%d): %s\n", what, st, eb_last_error());
}

void initGPU(int nNodes, const double* nodes, int nElements, const int* elements, int order, int nblocks,
             int nthreads)
{
  (void)nblocks;
  (void)nthreads;
  // The reference leaks the previous mesh unless closeGPU was called; here
  // the previous mesh is released.
  if (g_mesh) {
    eb_mesh_destroy(g_mesh);
    g_mesh = nullptr;
  }
  int st = eb_mesh_create(nNodes, nodes, nElements, elements, order, &g_mesh);
  report("initGPU", st);
  if (st == EB_OK) {
    ne = nElements;
    nnodes = nNodes;
  } else {
    ne = nnodes = 0;
  }
}

void closeGPU()
{
  if (g_mesh) eb_mesh_destroy(g_mesh);
  g_mesh = nullptr;
}

void applyGPULaplace3d1Layer(const double* t, double* v, int ansatz)
{
  if (!g_mesh) {
    std::fprintf(stderr, "easybem: applyGPULaplace3d1Layer called before initGPU\n");
    return;
  }
  if (ansatz == 0) {
    report("applyGPULaplace3d1Layer", eb_apply_sl_p0(g_mesh, legacy_precision(), t, v));
  } else {
    report("applyGPULaplace3d1Layer(ansatz=1)", eb_apply_sl_p1(g_mesh, legacy_precision(), t, v));
  }
}

void applyGPULaplace3d2Layer(const double* u, double* q)
{
  if (!g_mesh) {
    std::fprintf(stderr, "easybem: applyGPULaplace3d2Layer called before initGPU\n");
    return;
  }
  report("applyGPULaplace3d2Layer", eb_apply_dl_p1(g_mesh, legacy_precision(), u, q));
}

void applyGPULaplace3dHyperSing(const double* u, double* q)
{
  if (!g_mesh) {
    std::fprintf(stderr, "easybem: applyGPULaplace3dHyperSing called before initGPU\n");
    return;
  }
  report("applyGPULaplace3dHyperSing", eb_apply_hypersingular(g_mesh, legacy_precision(), u, q));
}
