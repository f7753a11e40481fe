// 2-vector of the drop-in API (the reference's struct vec2, src/vec2.cuh:7-96).
#pragma once

#include <cmath>

// Symbols of the C++ drop-in classes are exported from libcuplast.so.
#if defined(__GNUC__)
#define CUPLAST_CXX_API __attribute__((visibility("default")))
#else
#define CUPLAST_CXX_API
#endif

namespace cuplast {

struct vec2 {
    double x = 0., y = 0.;
    vec2() = default;
    vec2(double _x, double _y) : x(_x), y(_y) {}
    double operator*(const vec2& v) const { return x * v.x + y * v.y; }
    vec2 operator*(double k) const { return {x * k, y * k}; }
    vec2 operator/(double k) const { return {x / k, y / k}; }
    vec2 operator+(const vec2& v) const { return {x + v.x, y + v.y}; }
    vec2 operator-(const vec2& v) const { return {x - v.x, y - v.y}; }
    vec2 operator-() const { return {-x, -y}; }
    vec2& operator+=(const vec2& v) { x += v.x; y += v.y; return *this; }
    vec2& operator-=(const vec2& v) { x -= v.x; y -= v.y; return *this; }
    vec2& operator*=(double k) { x *= k; y *= k; return *this; }
    vec2& operator/=(double k) { x /= k; y /= k; return *this; }
    double crossZ(const vec2& v) const { return x * v.y - y * v.x; }
    double norm() const { return std::sqrt(x * x + y * y); }
    vec2 normalize() const { return *this * (1. / norm()); }
};

inline vec2 operator*(double k, const vec2& v) { return v * k; }

}  // namespace cuplast
