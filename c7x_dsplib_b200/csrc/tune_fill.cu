// Scratch contents for the autotuner's measurements: a hashed pattern of 32-bit words
// (floats in [-0.5, 0.5) for float buffers, any bits for integer ones).  Zero-filled
// scratch would not do: HBM traffic of constant data can be cheaper than that of real
// signals, which moves the best launch shape of the memory-bound kernels.
#include <cuda_runtime.h>

#include "dsplib_internal.h"

namespace dsplib {
namespace {

__global__ void tune_fill_kernel(uint32_t *p, size_t words, int asFloat)
{
   for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < words; i += (size_t) gridDim.x * blockDim.x) {
      uint32_t h = (uint32_t) i * 0x9E3779B1u;
      h ^= h >> 15;
      h *= 0x85EBCA77u;
      h ^= h >> 13;
      p[i] = asFloat ? __float_as_uint(((float) (h >> 8) * (1.0f / 16777216.0f)) - 0.5f) : h;
   }
}

} // namespace

cudaError_t launchTuneFill(void *p, size_t bytes, bool asFloat, cudaStream_t s)
{
   const size_t words = bytes / 4;
   if (words == 0) return cudaSuccess;
   const int blocks = (int) ((words + 255) / 256 < 4096 ? (words + 255) / 256 : 4096);
   tune_fill_kernel<<<blocks, 256, 0, s>>>((uint32_t *) p, words, asFloat ? 1 : 0);
   return cudaGetLastError();
}

} // namespace dsplib
