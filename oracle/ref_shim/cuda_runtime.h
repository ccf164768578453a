// Host-only stand-in for the CUDA runtime header, used ONLY to compile the
// reference LIMA_MD engine (Quantom/Quantom/Engine.cu and the headers it
// includes) as plain host C++ for the oracle in oracle/_ref.  Test
// infrastructure: nothing in the product links this.
//
// What it provides:
//  * CUDA qualifiers as no-ops; `__shared__` becomes a per-OS-thread static so
//    that every fiber (emulated CUDA thread) of one emulated block sees the same
//    object, as CUDA shared memory does.
//  * threadIdx/blockIdx/blockDim/gridDim as thread_local variables that the
//    block emulator in oracle/ref_emu.cpp sets before it resumes each fiber.
//  * __syncthreads() implemented by the emulator (a fiber yield).
//  * cudaMemcpy / cudaMallocManaged / cudaMemcpyToSymbol over host memory.
#pragma once

#include <cstdint>
#include <cstddef>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <algorithm>
#include <iostream>
#include <vector>
#include <string>
#include <memory>
#include <stdexcept>
#include <thread>
#include <chrono>
#include <fstream>
#include <sstream>
#include <climits>

#define __host__
#define __device__
#define __global__
#define __constant__
#define __forceinline__ inline
#define __shared__ static thread_local

struct uint3 { unsigned int x, y, z; };
struct dim3 {
    unsigned int x, y, z;
    dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

void __syncthreads();

// The reference calls exit() on capacity overflow and on some errors.  Inside
// the oracle library that would kill the test process, so exit() is routed to
// a handler that records the code and unwinds to the C API boundary.
[[noreturn]] void lima_ref_exit(int code);
#define exit(code) lima_ref_exit(code)

// Force hook: the build script inserts one call to this at the top of the
// reference's integratePosition() (Engine.cu:849) so the oracle can report the
// total force each particle was integrated with.  Defined in ref_emu.cpp.
struct Float3;
void lima_ref_force_hook(int p_index, const Float3* force);

typedef int cudaError_t;
static const cudaError_t cudaSuccess = 0;
enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3,
    cudaMemcpyDefault = 4
};

inline cudaError_t cudaMemcpy(void* dst, const void* src, size_t n, cudaMemcpyKind) {
    if (n) std::memmove(dst, src, n);
    return cudaSuccess;
}
inline cudaError_t cudaMemcpyToSymbol(const void* sym, const void* src, size_t n, size_t off = 0,
                                      cudaMemcpyKind = cudaMemcpyHostToDevice) {
    std::memcpy(static_cast<char*>(const_cast<void*>(sym)) + off, src, n);
    return cudaSuccess;
}
template <typename T>
inline cudaError_t cudaMallocManaged(T** p, size_t n) {
    *p = static_cast<T*>(std::calloc(1, n ? n : 1));
    return cudaSuccess;
}
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
