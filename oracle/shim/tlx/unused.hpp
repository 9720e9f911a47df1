// Test-infrastructure shim (oracle build only): marks values as used.
#pragma once
namespace tlx {
template <typename... Types>
void unused(Types&&...) {}
} // namespace tlx
