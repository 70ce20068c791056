// Drop-in path of the reference's header (include/function/SIMDRecSplit.hpp): SIMDRecSplit
// builds the same function as GPURecSplit, here on the GPU (include/rsb/GPURecSplit.hpp).
#pragma once
#include "../rsb/GPURecSplit.hpp"
