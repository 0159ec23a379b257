// Compatibility header for compiling the reference's CPU sources without Boost.
// Only the one facility those sources use: boost::array as std::array.
#pragma once
#include <array>
#include <cstddef>
namespace boost { template <class T, std::size_t N> using array = std::array<T, N>; }
