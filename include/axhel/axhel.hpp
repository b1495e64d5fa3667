// Umbrella header of the AXHEL drop-in API (namespace unipi::axhel), same
// layout as the reference's axhel/include/axhel/axhel.hpp:6-12.  The
// implementation runs on the GPU through the C-ABI in axhel_cuda.h.
#pragma once

#include "axhel/util/defines.hpp"
#include "axhel/eltwise/eltwise-add-mod.hpp"
#include "axhel/eltwise/eltwise-sub-mod.hpp"
#include "axhel/eltwise/eltwise-mul-mod.hpp"
#include "axhel/eltwise/eltwise-fma-mod.hpp"
#include "axhel/eltwise/eltwise-reduce-mod.hpp"
#include "axhel/ntt/ntt.hpp"
