// gr_single_general.cu -- the single-scene transport kernels for stones with
// birefringence or absorption (uniaxial, dichroic, tinted) in each environment kind:
// the c3 emerald's class.  The environment kind is fixed at compile time; the material
// checks stay at run time.
#include "gr_single.cuh"

namespace grh {

gr_status launch_single_general(int K, const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R,
                                float *xyz, cudaStream_t stream, const StagedLaunch *st) {
    switch (K) {
    case grd::k_env(GR_ENV_UNIFORM): return launch_single_k<grd::k_env(GR_ENV_UNIFORM)>(S, B, R, xyz, stream, st);
    case grd::k_env(GR_ENV_STUDIO): return launch_single_k<grd::k_env(GR_ENV_STUDIO)>(S, B, R, xyz, stream, st);
    case grd::k_env(GR_ENV_LATLONG): return launch_single_k<grd::k_env(GR_ENV_LATLONG)>(S, B, R, xyz, stream, st);
    default: return fail(GR_EINVAL, "scene class %d has no general kernel", K);
    }
}

}  // namespace grh
