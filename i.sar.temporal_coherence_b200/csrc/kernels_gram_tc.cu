/* Tensor-core (tcgen05) masked coherence-matrix accumulation: placeholder
   until the kernel lands; reports itself unavailable. */
#include "tcoh_internal.h"

bool tc_gram_tensor_supported(const TcStrip &) { return false; }

cudaError_t tc_launch_gram_tensor(const TcStrip &, const TcChunk &, int, const float *,
                                  const uint32_t *, float2 *, cudaStream_t)
{
    return cudaErrorNotSupported;
}
