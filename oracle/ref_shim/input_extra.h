// Host stand-ins the reference's box builder needs beyond cuda_runtime.h
// (BoxBuilder::buildBox allocates the next-step state with cudaMalloc).  Test
// infrastructure only: used by oracle/build_ref_input.sh.
#pragma once
#include <cstdlib>
template <typename T>
inline int cudaMalloc(T** p, size_t n) {
    *p = static_cast<T*>(std::calloc(1, n ? n : 1));
    return 0;
}
inline int cudaFree(void* p) {
    std::free(p);
    return 0;
}
