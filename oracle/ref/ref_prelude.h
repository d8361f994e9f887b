/*
 * Force-included (g++ -include) ahead of every reference translation unit compiled by
 * oracle/Makefile. It makes the reference compile with GCC 13 without editing it:
 *  - <algorithm> for std::sort in color/spectrumoperations.cpp:21;
 *  - FILIANORE_INLINE (core/elemental.h:20, always_inline) is redefined empty, because
 *    functions carrying it are defined in other translation units (sampling/sampling.h:14-16);
 *  - Vector2 min/max, which Rect (maths/geometry.h:388-401) calls but the reference only
 *    declares for Vector3. Declared here against the forward declaration of Vector2.
 * Test infrastructure only.
 */
#pragma once
#include <algorithm>
#include "filianore/core/elemental.h"
#undef FILIANORE_INLINE
#define FILIANORE_INLINE
namespace filianore {
template <typename T>
Vector2<T> min(const Vector2<T> &a, const Vector2<T> &b) { return Vector2<T>(std::min(a.x, b.x), std::min(a.y, b.y)); }
template <typename T>
Vector2<T> max(const Vector2<T> &a, const Vector2<T> &b) { return Vector2<T>(std::max(a.x, b.x), std::max(a.y, b.y)); }
} // namespace filianore
