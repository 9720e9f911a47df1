// Test-infrastructure shim (oracle build only): boost is not installed; the
// reference's headers use boost::array as a fixed-size array with assign().
#pragma once
#include <array>
#include <cstddef>
namespace boost {
template <typename T, std::size_t N>
struct array : public std::array<T, N> {
    void assign(const T& value) { this->fill(value); }
};
} // namespace boost
