// G2 instantiation of the MSM launch sequence.
#include "msm_batch.cuh"

namespace gm {
template int msm_launch<Fp2>(cudaStream_t, int, const uint4 *, const uint64_t *, int, const uint64_t *, int, int64_t,
                             uint64_t *, int, uint32_t *, cudaEvent_t, TailHandoff *);
template int batch_layouts<Fp2>(BatchPlan &, int);
template int batch_run<Fp2>(const BatchPlan &, cudaStream_t, const uint64_t *, uint64_t *);
template int batch_queue_setup<Fp2>(BatchPlan &);
template int window_table_launch<Fp2>(cudaStream_t, const uint4 *, int64_t, int, int, uint4 *);
}  // namespace gm
