// Test-infrastructure shim (oracle build only): the reference includes tlx's
// logger, whose submodule is empty in the reference tree. Every LOG statement
// compiles to a discarded stream, matching the reference's release builds in
// which the debug flags are static const false.
#pragma once
#include <ostream>
namespace oracle_shim {
struct NullStream {
    template <typename T>
    NullStream& operator << (const T&) { return *this; }
};
} // namespace oracle_shim
#define LOG while (false) ::oracle_shim::NullStream()
#define LOG0 LOG
#define LOG1 LOG
#define LOGC(cond) LOG
#define sLOG LOG
#define sLOG0 LOG
#define sLOG1 LOG
#define sLOGC(cond) LOG
