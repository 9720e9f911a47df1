// Test-infrastructure shim (oracle build only): boost is not installed.
#pragma once
#include <type_traits>
namespace boost {
using std::integral_constant;
using std::true_type;
using std::false_type;
} // namespace boost
