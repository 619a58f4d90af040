// C wrappers over the reference's own GPU path (include/BEM3dLaplaceGPU.h:8-18,
// src/BEM3dLaplaceGPU.cu:830-1555), compiled from the reference sources where
// they lie by `make -C oracle refgpu`. Test infrastructure only:
// tests/test_gpu_vs_reference_gpu.py compares it with this library's applies
// (results and time) on the same mesh; the product never loads it. Linked with -Bsymbolic so the reference's C++ entry
// points and globals (same names as this project's legacy shim) bind inside
// this library.
#include "BEM3dLaplaceGPU.h"

extern "C" {

// elements 1-based, as the reference takes them; the examples use 240 blocks
// of 32 threads (python/examples/laplace3dDirichletGPU.py:62)
void refgpu_init(int nnodes, const double* nodes, int nelems, const int* elems, int order)
{
  initGPU(nnodes, nodes, nelems, elems, order, 240, 32);
}

void refgpu_apply_sl(const double* t, double* v) { applyGPULaplace3d1Layer(t, v, 0); }

void refgpu_apply_dl(const double* u, double* q) { applyGPULaplace3d2Layer(u, q); }

void refgpu_close() { closeGPU(); }

}  // extern "C"
