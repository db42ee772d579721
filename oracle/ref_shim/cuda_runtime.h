/*
 * cuda_runtime.h -- TEST INFRASTRUCTURE ONLY: lets the reference's
 * __host__ __device__ headers compile as plain host C++ with g++ for the
 * known-answer vectors (oracle/Makefile `ref`).  The CUDA execution-space
 * qualifiers become nothing; no CUDA runtime is involved.
 */
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>

#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
