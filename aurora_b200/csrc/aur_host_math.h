// aur_host_math.h — host-side FP32 matrix helpers shared by the scene loader and scene
// creation.
#pragma once
#include <cmath>
#include <cstring>
#include <utility>

namespace aur {

// Gauss-Jordan elimination with full pivoting in FP32 on a row-major 4x4 matrix (the
// published algorithm Matrix4x4::inverse of the reference follows, core/matrix4x4.cpp:
// 77-150). Returns false for a singular matrix.
inline bool invert4_gj(const float in[16], float out[16]) {
    int indxc[4], indxr[4], ipiv[4] = {0, 0, 0, 0};
    float a[4][4];
    memcpy(a, in, sizeof(a));
    for (int i = 0; i < 4; ++i) {
        int irow = -1, icol = -1;
        float big = 0.f;
        for (int j = 0; j < 4; ++j) {
            if (ipiv[j] == 1) continue;
            for (int k = 0; k < 4; ++k) {
                if (ipiv[k] == 0) {
                    if (fabsf(a[j][k]) >= big) { big = fabsf(a[j][k]); irow = j; icol = k; }
                } else if (ipiv[k] > 1) {
                    return false;
                }
            }
        }
        if (icol < 0) return false;
        ++ipiv[icol];
        if (irow != icol)
            for (int k = 0; k < 4; ++k) std::swap(a[irow][k], a[icol][k]);
        indxr[i] = irow;
        indxc[i] = icol;
        if (a[icol][icol] == 0.f) return false;
        const float pivinv = 1.f / a[icol][icol];
        a[icol][icol] = 1.f;
        for (int j = 0; j < 4; ++j) a[icol][j] *= pivinv;
        for (int j = 0; j < 4; ++j) {
            if (j == icol) continue;
            const float save = a[j][icol];
            a[j][icol] = 0.f;
            for (int k = 0; k < 4; ++k) a[j][k] -= a[icol][k] * save;
        }
    }
    for (int j = 3; j >= 0; --j) {
        if (indxr[j] == indxc[j]) continue;
        for (int k = 0; k < 4; ++k) std::swap(a[k][indxr[j]], a[k][indxc[j]]);
    }
    memcpy(out, a, sizeof(a));
    return true;
}

}  // namespace aur
