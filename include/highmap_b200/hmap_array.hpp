/*
 * hmap_array.hpp - minimal hmap::Array for callers that do not include
 * HighMap's own headers.
 *
 * Same members, in the same order, as hmap::Array of
 * HighMap/include/highmap/array.hpp:31-44 (glm::ivec2 shape, then
 * std::vector<float> vector; element (i, j) at vector[j * shape.x + i],
 * array.hpp:236-252), so code built against either header calls the same
 * hmap::gpu functions of libhm_erosion.so.  glm is used when present;
 * otherwise a two-int glm::ivec2 of the same layout is declared.
 */
#ifndef HMAP_B200_ARRAY_HPP
#define HMAP_B200_ARRAY_HPP

#include <vector>

#if defined(__has_include)
#if __has_include(<glm/vec2.hpp>)
#include <glm/vec2.hpp>
#define HMAP_B200_HAVE_GLM 1
#endif
#endif

#ifndef HMAP_B200_HAVE_GLM
namespace glm
{
struct ivec2
{
  int x = 0, y = 0;
  ivec2() = default;
  ivec2(int x_, int y_) : x(x_), y(y_) {}
};
} // namespace glm
#endif

namespace hmap
{

class Array
{
public:
  glm::ivec2         shape = glm::ivec2(0, 0);
  std::vector<float> vector;

  Array() = default;
  explicit Array(glm::ivec2 s) : shape(s), vector((size_t)s.x * (size_t)s.y, 0.f) {}
  Array(glm::ivec2 s, float value) : shape(s), vector((size_t)s.x * (size_t)s.y, value) {}

  float       &operator()(int i, int j) { return vector[(size_t)j * shape.x + i]; }
  const float &operator()(int i, int j) const { return vector[(size_t)j * shape.x + i]; }
  size_t       size() const { return vector.size(); }
};

} // namespace hmap

#endif
