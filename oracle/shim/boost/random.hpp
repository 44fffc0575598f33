// Test infrastructure only: std-only stand-in for the parts of Boost.Random
// that the reference CPU oracles name (mt19937 and uniform_int_distribution).
#pragma once
#include <cstdint>
#include <ctime>
#include <random>

namespace boost {
namespace random {
using mt19937 = std::mt19937;
template <class I = int>
using uniform_int_distribution = std::uniform_int_distribution<I>;
}  // namespace random
}  // namespace boost
