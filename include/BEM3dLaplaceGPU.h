// easybem B200 — the legacy C++ GPU interface, declared exactly as the
// reference declares it (include/BEM3dLaplaceGPU.h:8-18), so code written
// against easybem (python/bindings.cpp included) compiles and links unchanged
// against libeasybem_gpu.so. The library also defines the process-global
// `int ne, nnodes` that python/bindings.cpp:6 declares extern.
//
// Semantics kept from the reference: one process-global mesh; initGPU
// replaces it; outputs are overwritten; `elements` are 1-based; nblocks and
// nthreads are accepted and ignored (the launch shape is chosen by the
// library). FP64 is the default arithmetic; EASYBEM_PRECISION=mixed selects
// the FP32 far field. Errors are reported on stderr and via eb_last_error().

#ifndef BEM3DLAPLACEGPU_H
#define BEM3DLAPLACEGPU_H


void initGPU (int nNodes, const double *nodes,
              int nElements, const int *elements, int order,
              int nblocks, int nthreads);

void closeGPU ();

void applyGPULaplace3d1Layer (const double *t, double *v, int ansatz=0);

void applyGPULaplace3d2Layer (const double *u, double *q);

void applyGPULaplace3dHyperSing (const double *u, double *q);


#endif
