// Test-infrastructure shim (oracle build only): abort-on-failure macros used by
// the reference's verifying wrappers.
#pragma once
#include <cstdlib>
#include <iostream>
#define die(msg) do { std::cerr << "DIE: " << msg << std::endl; std::abort(); } while (0)
#define die_unless(X) do { if (!(X)) { std::cerr << "DIE: " #X << std::endl; std::abort(); } } while (0)
#define die_if(X) do { if ((X)) { std::cerr << "DIE: " #X << std::endl; std::abort(); } } while (0)
