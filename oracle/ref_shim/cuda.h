/*
 * cuda.h -- TEST INFRASTRUCTURE ONLY: the one driver-API type the reference
 * headers compiled for the known-answer vectors name (CuBufferView.h).  A
 * CUdeviceptr there holds a host address.
 */
#pragma once

#include <cstdint>

typedef unsigned long long CUdeviceptr;
