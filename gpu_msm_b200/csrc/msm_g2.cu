// G2 instantiation of the MSM launch sequence.
#include "msm_host.cuh"

namespace gm {
template int msm_launch<Fp2>(cudaStream_t, int, const uint4 *, const uint64_t *, int, const uint64_t *, int, int64_t,
                             uint64_t *, int, uint32_t *);
}  // namespace gm
