// Tensor-core (tcgen05) FIR kernels for sm_100a.
#include <cuda_runtime.h>

#include "dsplib_internal.h"

namespace dsplib {

cudaError_t launchFirBf16x3(const FirLaunch &a, cudaStream_t s)
{
   (void) a;
   (void) s;
   return cudaErrorNotSupported;
}

} // namespace dsplib
