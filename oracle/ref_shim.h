/*
 * ref_shim.h -- lets the reference's CUDA kernel templates compile as host
 * C++ (TEST INFRASTRUCTURE ONLY; used by oracle/build_ref.py).
 *
 * The reference kernels (CHANS-HiPIMS/hipims/cuda/*_Kernel.cu) are plain
 * one-thread-per-cell SIMT code.  With the CUDA qualifiers defined away,
 * threadIdx/blockIdx/blockDim as thread-local variables and CUDA's
 * fmin/fmax-style min/max overloads, each kernel body is an ordinary C++
 * function that a host loop calls once per "thread".
 */
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __syncthreads() ((void)0)

struct hb_ref_uint3 {
  unsigned int x, y, z;
};
static thread_local hb_ref_uint3 threadIdx, blockIdx, blockDim;

using std::abs;
using std::fabs;
using std::pow;
using std::sqrt;

/* CUDA's device min/max on floating types are fmin/fmax. */
static inline double max(double a, double b) { return std::fmax(a, b); }
static inline double min(double a, double b) { return std::fmin(a, b); }
static inline float max(float a, float b) { return std::fmax(a, b); }
static inline float min(float a, float b) { return std::fmin(a, b); }
static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
