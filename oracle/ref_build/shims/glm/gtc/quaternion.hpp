// Forward declarations standing in for the glm types named in declarations of
// printer.h / math_func.h (no glm type is used on the solve path).
#pragma once
namespace glm {
struct vec2;
struct vec3;
struct vec4;
struct quat;
struct mat4;
}  // namespace glm
