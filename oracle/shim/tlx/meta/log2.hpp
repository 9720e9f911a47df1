// Test-infrastructure shim (oracle build only): included by the reference but
// none of its templates are used on the pS5 path.
#pragma once
