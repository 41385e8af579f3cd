// queue_fp64.cu -- instantiation of the persistent queue sweep with double butterflies (one
// translation unit per precision so that nvcc compiles them in parallel).
#include "queue_launch.cuh"

namespace hm {
template int launch_queue_kernel<double, QS_Q2>(hm_ctx *, const QArgs &, int, long long, int *);
template int launch_queue_kernel<double, QS_Q23>(hm_ctx *, const QArgs &, int, long long, int *);
template int launch_queue_kernel<double, QS_GEN>(hm_ctx *, const QArgs &, int, long long, int *);
template int queue_warps<double, QS_Q2>(hm_ctx *, int, long long, int *);
template int queue_warps<double, QS_Q23>(hm_ctx *, int, long long, int *);
template int queue_warps<double, QS_GEN>(hm_ctx *, int, long long, int *);
}  // namespace hm
