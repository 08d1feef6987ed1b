// Minimal stand-in for sf::Color (constexpr RGBA) named by the reference's
// constants header.
#pragma once

#include <cstdint>

namespace sf {

struct Color {
    std::uint8_t r = 0, g = 0, b = 0, a = 255;
    constexpr Color() = default;
    constexpr Color(std::uint8_t r_, std::uint8_t g_, std::uint8_t b_, std::uint8_t a_ = 255)
        : r(r_), g(g_), b(b_), a(a_) {}
};

}  // namespace sf
