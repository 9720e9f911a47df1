// Test-infrastructure shim (oracle build only): size strings for psstest's
// -s/-S options: a number with an optional SI (k, m, g, t: powers of 1000) or
// IEC (ki, mi, gi, ti: powers of 1024) unit, an optional trailing 'b'.
#pragma once
#include <cctype>
#include <cstdint>
#include <cstdlib>
#include <string>
namespace tlx {
static inline bool parse_si_iec_units(const std::string& str, uint64_t* out, char default_unit = 0)
{
    const char* s = str.c_str();
    char* end = nullptr;
    double v = std::strtod(s, &end);
    if (end == s) return false;
    while (*end == ' ') ++end;
    char unit = *end ? (char)std::tolower(*end) : (char)std::tolower(default_unit);
    if (*end) ++end;
    bool iec = false;
    if (*end == 'i' || *end == 'I') { iec = true; ++end; }
    if (*end == 'b' || *end == 'B') ++end;
    if (*end != 0) return false;
    const double base = iec ? 1024.0 : 1000.0;
    double mul = 1.0;
    switch (unit) {
    case 0: case 'b': break;
    case 'k': mul = base; break;
    case 'm': mul = base * base; break;
    case 'g': mul = base * base * base; break;
    case 't': mul = base * base * base * base; break;
    default: return false;
    }
    *out = (uint64_t)(v * mul);
    return true;
}
} // namespace tlx
