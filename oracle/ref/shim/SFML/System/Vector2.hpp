// Minimal stand-in for the one SFML type the reference's simulation code
// uses (a 2-component vector with arithmetic), so the reference CPU backend
// compiles without SFML.  Only the members those sources call are provided.
#pragma once

#include <cmath>

namespace sf {

template <typename T>
struct Vector2 {
    T x{}, y{};
    constexpr Vector2() = default;
    constexpr Vector2(T x_, T y_) : x(x_), y(y_) {}
    constexpr T lengthSquared() const { return x * x + y * y; }
    T length() const { return std::sqrt(lengthSquared()); }
    constexpr Vector2& operator+=(const Vector2& o) { x += o.x; y += o.y; return *this; }
    constexpr Vector2& operator-=(const Vector2& o) { x -= o.x; y -= o.y; return *this; }
};

template <typename T>
constexpr Vector2<T> operator+(const Vector2<T>& a, const Vector2<T>& b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
constexpr Vector2<T> operator-(const Vector2<T>& a, const Vector2<T>& b) { return {a.x - b.x, a.y - b.y}; }
template <typename T>
constexpr Vector2<T> operator*(const Vector2<T>& a, T s) { return {a.x * s, a.y * s}; }
template <typename T>
constexpr Vector2<T> operator*(T s, const Vector2<T>& a) { return {a.x * s, a.y * s}; }
template <typename T>
constexpr Vector2<T> operator/(const Vector2<T>& a, T s) { return {a.x / s, a.y / s}; }
template <typename T>
constexpr bool operator==(const Vector2<T>& a, const Vector2<T>& b) { return a.x == b.x && a.y == b.y; }
template <typename T>
constexpr bool operator!=(const Vector2<T>& a, const Vector2<T>& b) { return !(a == b); }

using Vector2u = Vector2<unsigned int>;
using Vector2f = Vector2<float>;

}  // namespace sf
