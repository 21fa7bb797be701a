// pending.cu — entry points whose kernels are not built yet report
// AUR_ERR_UNSUPPORTED instead of falling back to any other path.
#include "aur_capi_internal.h"

namespace aur {
aur_status render_wavefront(aur_scene*, const aur_render_opts*, float*, aur_render_stats*) {
    return fail(AUR_ERR_UNSUPPORTED, "aur_render: wavefront mode is not available in this build");
}
}  // namespace aur

extern "C" {
aur_status aur_render_batch(aur_scene* const*, const aur_render_opts*, uint32_t, float* const*, aur_render_stats*) {
    return aur::fail(AUR_ERR_UNSUPPORTED, "aur_render_batch is not available in this build");
}
aur_status aur_render_adjoint(aur_scene*, const aur_render_opts*, const float*, float*, float*, aur_render_stats*) {
    return aur::fail(AUR_ERR_UNSUPPORTED, "aur_render_adjoint is not available in this build");
}
aur_status aur_scene_load_json(aur_ctx*, const char*, aur_scene**) {
    return aur::fail(AUR_ERR_UNSUPPORTED, "aur_scene_load_json is not available in this build");
}
}
