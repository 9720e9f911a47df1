// Test-infrastructure shim (oracle build only): hex rendering of a value, used
// only inside disabled debug log statements of the reference.
#pragma once
#include <string>
namespace tlx {
template <typename T>
std::string hexdump_type(const T& t) {
    static const char digits[] = "0123456789ABCDEF";
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&t);
    std::string out;
    for (size_t i = 0; i < sizeof(T); ++i) {
        out += digits[p[i] >> 4];
        out += digits[p[i] & 15];
    }
    return out;
}
} // namespace tlx
