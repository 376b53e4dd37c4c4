// Interface stand-in (test infrastructure): raw device pointer of a thrust vector, the
// launch-check helper and integer ceil-division the reference's sources call.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#include <thrust/device_vector.h>

template<class T>
inline T* rawPtr(thrust::device_vector<T>& v) { return thrust::raw_pointer_cast(v.data()); }
template<class T>
inline const T* rawPtr(const thrust::device_vector<T>& v) { return thrust::raw_pointer_cast(v.data()); }

inline void checkGpuErrors(cudaError_t e)
{
    if (e != cudaSuccess)
    {
        std::fprintf(stderr, "reference probe: CUDA error %s\n", cudaGetErrorString(e));
        std::abort();
    }
}

template<class I>
__host__ __device__ constexpr I iceil(I a, I b) { return (a + b - 1) / b; }
