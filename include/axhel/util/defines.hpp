// Configuration header of the B200 build (the reference generates its own
// from axhel/include/axhel/util/defines.hpp.in).  AXHEL_HAS_SVE is never
// defined: the element-wise and NTT kernels run on an sm_100a GPU.
#pragma once

#define AXHEL_HAS_CUDA 1

// Avoid unused variable warnings
#define AXHEL_UNUSED(x) (void)(x)
