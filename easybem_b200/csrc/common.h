// Shared definitions of the easybem B200 library: status codes, error
// plumbing and small vector helpers used by host and device code.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/easybem_gpu.h"

namespace eb {

// Records a message for eb_last_error() and returns the status code.
int set_error(int status, const std::string& msg);
const char* last_error();

#define EB_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t err_ = (call);                                                          \
    if (err_ != cudaSuccess)                                                            \
      return ::eb::set_error(EB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_)); \
  } while (0)

#define EB_CHECK(status_expr)              \
  do {                                     \
    int st_ = (status_expr);               \
    if (st_ != EB_OK) return st_;          \
  } while (0)

struct d3 { double x, y, z; };

__host__ __device__ inline d3 mk3(double x, double y, double z) { return d3{x, y, z}; }
__host__ __device__ inline d3 operator+(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline d3 operator-(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline d3 operator*(double s, d3 a) { return d3{s * a.x, s * a.y, s * a.z}; }
__host__ __device__ inline double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline d3 cross3(d3 a, d3 b)
{
  return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

}  // namespace eb
