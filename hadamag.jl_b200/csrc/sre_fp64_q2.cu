// sre_fp64_q2.cu -- instantiation of the exact-SRE launchers: double butterflies, moment set QS_Q2
// (one translation unit per combination so that nvcc compiles them in parallel).
#include "sre_launch.cuh"

namespace hm {
template int launch_sre_qs<double, 32, QS_Q2>(hm_ctx *, const void *, int, uint64_t, uint64_t, const QParams &, int *);
}
