// gr_single_clear.cu -- the single-scene transport kernels specialised for clear
// isotropic stones (no birefringence, no absorption data) in each environment kind:
// the c1 / c2 brilliant's class.  Their kernels contain no walk-off, mode-coupling,
// Beer-Lambert or other-environment code.
#include "gr_single.cuh"

namespace grh {

gr_status launch_single_clear(int K, const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R,
                              float *xyz, cudaStream_t stream, const StagedLaunch *st, unsigned int *sorted_work,
                              int sm_count) {
    constexpr int IC = grd::K_ISO | grd::K_CLEAR;
    if (sorted_work) {
        switch (K) {
        case IC | grd::k_env(GR_ENV_UNIFORM):
            return launch_sorted_k<IC | grd::k_env(GR_ENV_UNIFORM)>(S, B, R, xyz, stream, sorted_work, sm_count);
        case IC | grd::k_env(GR_ENV_STUDIO):
            return launch_sorted_k<IC | grd::k_env(GR_ENV_STUDIO)>(S, B, R, xyz, stream, sorted_work, sm_count);
        case IC | grd::k_env(GR_ENV_LATLONG):
            return launch_sorted_k<IC | grd::k_env(GR_ENV_LATLONG)>(S, B, R, xyz, stream, sorted_work, sm_count);
        default: return fail(GR_EINVAL, "scene class %d has no sorted kernel", K);
        }
    }
    switch (K) {
    case IC | grd::k_env(GR_ENV_UNIFORM): return launch_single_k<IC | grd::k_env(GR_ENV_UNIFORM)>(S, B, R, xyz, stream, st);
    case IC | grd::k_env(GR_ENV_STUDIO): return launch_single_k<IC | grd::k_env(GR_ENV_STUDIO)>(S, B, R, xyz, stream, st);
    case IC | grd::k_env(GR_ENV_LATLONG): return launch_single_k<IC | grd::k_env(GR_ENV_LATLONG)>(S, B, R, xyz, stream, st);
    default: return fail(GR_EINVAL, "scene class %d has no clear-stone kernel", K);
    }
}

}  // namespace grh
