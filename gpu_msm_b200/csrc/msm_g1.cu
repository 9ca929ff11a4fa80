// G1 instantiation of the MSM launch sequence.
#include "msm_batch.cuh"

namespace gm {
template int msm_launch<Fp>(cudaStream_t, int, const uint4 *, const uint64_t *, int, const uint64_t *, int, int64_t,
                            uint64_t *, int, uint32_t *, cudaEvent_t, TailHandoff *);
template int msm_plan<Fp>(MsmLayout<Fp> &, int, int64_t, int, int, bool, int64_t);
template int msm_run<Fp>(cudaStream_t, const MsmLayout<Fp> &, char *, const uint4 *, const uint64_t *, int,
                         const uint64_t *, uint64_t *, bool, uint32_t *, cudaEvent_t, TailHandoff *);
template int batch_layouts<Fp>(BatchPlan &, int);
template int batch_run<Fp>(const BatchPlan &, cudaStream_t, const uint64_t *, uint64_t *);
template int batch_queue_setup<Fp>(BatchPlan &);
template int window_table_launch<Fp>(cudaStream_t, const uint4 *, int64_t, int, int, uint4 *);
}  // namespace gm
