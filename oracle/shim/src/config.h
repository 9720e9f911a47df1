/* Test-infrastructure shim (oracle build only): replaces the CMake-generated
 * src/config.h of the reference. */
#pragma once
#define HAVE_ATOMIC_H 1
