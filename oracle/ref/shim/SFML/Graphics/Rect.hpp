// Minimal stand-in for sf::Rect (position + size, centre) as used by the
// reference quadtree.
#pragma once

#include "SFML/System/Vector2.hpp"

namespace sf {

template <typename T>
struct Rect {
    Vector2<T> position{}, size{};
    constexpr Rect() = default;
    constexpr Rect(Vector2<T> p, Vector2<T> s) : position(p), size(s) {}
    constexpr Vector2<T> getCenter() const { return position + size / T(2); }
};

}  // namespace sf
