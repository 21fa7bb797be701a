// aur_image_io.h — host-side image readers for textures and environment maps.
#pragma once
#include <string>
#include <vector>
#include "aurora_b200.h"

namespace aur {

// RGB floats of an OpenEXR file's data window, top row first (Texture2D's pixel buffer,
// Aurora/src/frontend/texture2D.cpp:23-46). Returns AUR_OK, AUR_ERR_IO, AUR_ERR_PARSE or
// AUR_ERR_UNSUPPORTED with a message in *err.
aur_status read_exr_rgb(const std::string& path, std::vector<float>* rgb, int* w, int* h, std::string* err);

}  // namespace aur
