// Test-infrastructure shim (oracle build only): boost is not installed.
#pragma once
#define BOOST_STATIC_ASSERT(x) static_assert((x), #x)
