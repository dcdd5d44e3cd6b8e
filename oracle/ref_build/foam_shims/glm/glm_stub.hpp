// Minimal stand-ins for the glm types and functions named in the reference's
// manager/source/math_func.cpp, so that file compiles on a box without glm.
// Only the shapes matter: the OpenFOAM export reaches none of the four helpers
// that use them (dotClamp, getQuat, getNormalizedDeviceCoords, scaleMat4).
#pragma once
namespace glm {
struct vec2 {
    float x = 0.f, y = 0.f;
    vec2() = default;
    vec2(float a, float b) : x(a), y(b) {}
};
struct vec3 {
    float x = 0.f, y = 0.f, z = 0.f;
    vec3() = default;
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
};
struct vec4 {
    float x = 0.f, y = 0.f, z = 0.f, w = 0.f;
};
struct quat {
    float w = 1.f, x = 0.f, y = 0.f, z = 0.f;
};
struct mat4 {
    float m[16] = {};
};
inline float clamp(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline vec3 normalize(const vec3& a) { return a; }
inline quat angleAxis(float, const vec3&) { return quat{}; }
inline mat4 scale(const mat4& m, const vec3&) { return m; }
}  // namespace glm
