// Test-infrastructure shim (oracle build only): branch hints.
#pragma once
#define TLX_LIKELY(c) __builtin_expect(!!(c), 1)
#define TLX_UNLIKELY(c) __builtin_expect(!!(c), 0)
