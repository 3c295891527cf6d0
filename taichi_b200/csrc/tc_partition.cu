// tc_partition.cu -- GPU partitioner (thumbnail, morphology, contours,
// dense-diagonal extraction).  Being written; fails loudly until then.
#include "tc_internal.h"

namespace tc {
tc_status gpu_partition(int, int, int64_t, const int *, const int *, const float *,
                        const tc_params &, bool, bool, cudaStream_t, PartitionOut &)
{
    return fail(TC_ERR_UNSUPPORTED, "GPU partitioner not available in this build");
}
}  // namespace tc

extern "C" tc_status tc_getsdf(int, int, const int *, const int *, const tc_params *, int *, int *,
                               int *, int, int *, unsigned char *, void *)
{
    return tc::fail(TC_ERR_UNSUPPORTED, "GPU partitioner not available in this build");
}

extern "C" tc_status tc_trace_contours(const unsigned char *, int, int, int *, int *, int, int *)
{
    return tc::fail(TC_ERR_UNSUPPORTED, "GPU partitioner not available in this build");
}
