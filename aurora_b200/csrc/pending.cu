// pending.cu — entry points whose kernels are not built yet report
// AUR_ERR_UNSUPPORTED instead of falling back to any other path.
#include "aur_capi_internal.h"

extern "C" {
aur_status aur_render_adjoint(aur_scene*, const aur_render_opts*, const float*, float*, float*, aur_render_stats*) {
    return aur::fail(AUR_ERR_UNSUPPORTED, "aur_render_adjoint is not available in this build");
}
aur_status aur_scene_load_json(aur_ctx*, const char*, aur_scene**) {
    return aur::fail(AUR_ERR_UNSUPPORTED, "aur_scene_load_json is not available in this build");
}
}
