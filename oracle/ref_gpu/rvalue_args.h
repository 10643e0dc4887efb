// Pre-included ahead of the reference's GPU_kernel.cu when it is built as a
// checker (TEST INFRASTRUCTURE ONLY).  That file passes temporaries such as
// make_double4(...) to functions taking non-const references (accepted by the
// compiler it was written for, rejected by nvcc's front end).  These overloads
// take the temporaries and forward them as lvalues to the file's own
// definitions, declared here ahead of it; no definition of the file changes.
#pragma once
#include <cuda_runtime.h>

__device__ double compute_r(double4 &r1, double4 &r2);
double cpu_compute_r(double4 &r1, double4 &r2);
__device__ double3 cross_uxv(double3 &u, double3 &v);
__device__ double my_dot(double3 &a, double3 &b);

__device__ inline double compute_r(double4 &&r1, double4 &&r2) { return compute_r(r1, r2); }
inline double cpu_compute_r(double4 &&r1, double4 &&r2) { return cpu_compute_r(r1, r2); }
__device__ inline double3 cross_uxv(double3 &u, double3 &&v) { return cross_uxv(u, v); }
__device__ inline double my_dot(double3 &a, double3 &&b) { return my_dot(a, b); }
