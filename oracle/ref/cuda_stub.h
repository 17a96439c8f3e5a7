/*
 * cuda_stub.h -- lets the reference's thrust-based entry files (Union.cu, Difference.cu,
 * Unique.cu, Reduce.cu, Sort.cu) compile as host C++ against their vendored thrust 1.7
 * with the CPP device system.  "Device" memory is host memory here, so the runtime
 * calls they make reduce to memmove / no-ops.  Used only to build oracle/_ref, the
 * reference-code cross-check for the oracle; never linked into the product.
 */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define THRUST_DEVICE_SYSTEM THRUST_DEVICE_SYSTEM_CPP
typedef int cudaError_t;
enum { cudaSuccess = 0 };
enum { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3 };
typedef void* cudaEvent_t;
static inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, int) { std::memmove(d, s, n); return 0; }
static inline cudaError_t cudaEventCreate(cudaEvent_t*) { return 0; }
static inline cudaError_t cudaEventRecord(cudaEvent_t, int = 0) { return 0; }
static inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return 0; }
static inline cudaError_t cudaEventElapsedTime(float* t, cudaEvent_t, cudaEvent_t) { *t = 0; return 0; }
static inline cudaError_t cudaEventDestroy(cudaEvent_t) { return 0; }
static inline const char* cudaGetErrorString(cudaError_t) { return ""; }
static inline cudaError_t cudaMalloc(void** p, size_t n) { *p = std::malloc(n); return 0; }
static inline cudaError_t cudaFree(void* p) { std::free(p); return 0; }
/* The device templates of Project.h name the launch built-ins at definition time. */
struct rfx_stub_dim3 { unsigned x, y, z; };
static const rfx_stub_dim3 gridDim = {1, 1, 1}, blockDim = {1, 1, 1}, threadIdx = {0, 0, 0}, blockIdx = {0, 0, 0};
