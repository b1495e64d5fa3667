// Debug logging of the public API (the reference's axhel/util/debug.hpp
// interface): AXHEL_LOG(stream expression) writes one "[AXHEL] ..." line to
// std::cerr when the library is built with AXHEL_DEBUG defined
// (python -m axhel_b200.build --debug-log), and compiles to nothing otherwise.
#pragma once

#include "axhel/util/defines.hpp"

#ifdef AXHEL_DEBUG
#include <iostream>
#define AXHEL_LOG(message)                             \
    do {                                               \
        std::cerr << "[AXHEL] " << message << '\n';    \
    } while (false)
#else
#define AXHEL_LOG(message) \
    do {                   \
    } while (false)
#endif
