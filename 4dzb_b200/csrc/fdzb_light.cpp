// fdzb_light.cpp -- host light setup: FD::FDsetAreaLight (FS/api.cpp:303-400).
//
// Built with -ffp-contract=off: every float expression is a sequence of single
// IEEE binary32 operations in the reference's order, so the matrix, corners and
// deltas are bit-identical to the reference's (its helper_math float3 operators
// and GLM 0.9.8 lookAtRH / infinitePerspectiveRH / mat4 product,
// 4DZB/glm/gtc/matrix_transform.inl:378-393,521-546,
// 4DZB/glm/detail/type_mat4x4.inl:595-614).
#include <cmath>
#include <cstring>

#include "fdzb_internal.h"

namespace fdzb {
namespace {

struct V3 {
    float x, y, z;
};
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
// v * (1 / sqrt(dot(v, v))): the host rsqrtf of the vector helpers and GLM's
// inversesqrt are both 1/sqrt.
inline V3 normalize(V3 v)
{
    const float inv = 1.0f / std::sqrt(dot(v, v));
    return v * inv;
}
inline void put(float *d, V3 a)
{
    d[0] = a.x;
    d[1] = a.y;
    d[2] = a.z;
}

}  // namespace

void light_setup(const float rightRadius, const float topRadius, const float position[3],
                 const float viewDir[3], const float upDir[3], int resW, int resH, LightParams *L)
{
    std::memset(L, 0, sizeof(*L));
    L->N = resW;
    L->NC = resH;
    L->full = resH >= 32 ? 0xffffffffu : ((1u << resH) - 1u);
    L->fullRows = resW >= 64 ? ~0ull : ((1ull << resW) - 1ull);
    L->fullCols = resH >= 64 ? ~0ull : ((1ull << resH) - 1ull);

    const V3 pos = v3(position[0], position[1], position[2]);
    const V3 up = normalize(v3(upDir[0], upDir[1], upDir[2]));
    const V3 view = normalize(v3(viewDir[0], viewDir[1], viewDir[2]));
    const V3 right = normalize(cross(view, up));
    const V3 top = normalize(cross(right, view));

    put(L->xd, right * (rightRadius * -2.0f / (float)resW));
    put(L->yd, top * (topRadius * -2.0f / (float)resH));

    const float xf = ((float)resW - 1.0f) / (float)resW;
    const float yf = ((float)resH - 1.0f) / (float)resH;
    const V3 nr = right * -1.0f, nt = top * -1.0f;
    const V3 ur = pos + right * xf * rightRadius + top * yf * topRadius;
    put(L->ur, ur);
    put(L->ul, pos + nr * xf * rightRadius + top * yf * topRadius);
    put(L->dl, pos + nr * xf * rightRadius + nt * yf * topRadius);
    put(L->dr, pos + right * xf * rightRadius + nt * yf * topRadius);

    // lookAtRH(eye = ur, center = ur + 10 * view, up)
    const V3 center = ur + v3(10.0f * view.x, 10.0f * view.y, 10.0f * view.z);
    const V3 f = normalize(center - ur);
    const V3 s = normalize(cross(f, up));
    const V3 u = cross(s, f);
    float mv[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};  // [column][row]
    mv[0][0] = s.x; mv[1][0] = s.y; mv[2][0] = s.z;
    mv[0][1] = u.x; mv[1][1] = u.y; mv[2][1] = u.z;
    mv[0][2] = -f.x; mv[1][2] = -f.y; mv[2][2] = -f.z;
    mv[3][0] = -dot(s, ur);
    mv[3][1] = -dot(u, ur);
    mv[3][2] = dot(f, ur);

    // infinitePerspectiveRH(fovy = 120 (radians in GLM 0.9.8), aspect 1, zNear 0.1)
    // tan(fovy / 2) is taken correctly rounded to binary32 (evaluated in double):
    // 0.32004037f.  C runtimes differ in the last bit here -- glibc's tanf(60.0f)
    // returns 0.3200404f -- and this constant scales the whole projection.
    const float fovy = 120.0f, aspect = 1.0f, zNear = 0.1f;
    const float range = (float)std::tan((double)(fovy / 2.0f)) * zNear;
    const float left = -range * aspect, rgt = range * aspect, bottom = -range, tp = range;
    float P[4][4] = {};
    P[0][0] = (2.0f * zNear) / (rgt - left);
    P[1][1] = (2.0f * zNear) / (tp - bottom);
    P[2][2] = -1.0f;
    P[2][3] = -1.0f;
    P[3][2] = -2.0f * zNear;

    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) {
            const float a0 = P[0][r] * mv[c][0];
            const float a1 = P[1][r] * mv[c][1];
            const float a2 = P[2][r] * mv[c][2];
            const float a3 = P[3][r] * mv[c][3];
            L->mat[c * 4 + r] = ((a0 + a1) + a2) + a3;
        }
    L->RF[0] = rightRadius * 2.0f * xf * P[0][0] * 0.5f;
    L->RF[1] = topRadius * 2.0f * yf * P[1][1] * 0.5f;
}

}  // namespace fdzb
