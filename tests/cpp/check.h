// check.h -- assertion helpers shared by the C++ API test programs.
#pragma once

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

namespace check {

inline void require(bool condition, const std::string& message)
{
    if (!condition) throw std::runtime_error(message);
}

// fn() must throw an exception of type E whose what() contains `fragment`.
template <class E = std::runtime_error, class Fn>
void expect_throw(Fn&& fn, const std::string& fragment)
{
    try {
        fn();
    } catch (const E& e) {
        require(std::string(e.what()).find(fragment) != std::string::npos,
                "unexpected error text: '" + std::string(e.what()) + "', wanted '" + fragment + "'");
        return;
    }
    throw std::runtime_error("expected a failure containing '" + fragment + "'");
}

inline uint32_t bits(float f)
{
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b;
}

inline float from_bits(uint32_t b)
{
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

// Deterministic 64-bit generator (splitmix64) for test inputs.
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    uint32_t below(uint32_t n) { return n ? static_cast<uint32_t>(next() % n) : 0u; }
    float uniform() { return static_cast<float>(next() >> 40) / static_cast<float>(1u << 24); }
};

}  // namespace check
