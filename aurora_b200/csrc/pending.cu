// pending.cu — entry points whose kernels are not built yet report
// AUR_ERR_UNSUPPORTED instead of falling back to any other path.
#include "aur_capi_internal.h"

extern "C" {
aur_status aur_scene_load_json(aur_ctx*, const char*, aur_scene**) {
    return aur::fail(AUR_ERR_UNSUPPORTED, "aur_scene_load_json is not available in this build");
}
}
