/*
 * ref_cuda_shim.h -- what the reference's HiPIMS kernel files expect from
 * their dropped #include lines when their kernels are compiled with nvcc for
 * the GPU without torch (used by baseline/build_ref_cuda.py only): the CUDA
 * runtime and math headers, fixed-width integers, and the launch-size helpers
 * of the reference's gpu.cuh (1024 threads per block, ceil(N / 1024) blocks).
 */
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

constexpr int CUDA_NUM_THREADS = 1024;
inline int GET_BLOCKS(const int N) { return (N - 1) / CUDA_NUM_THREADS + 1; }
