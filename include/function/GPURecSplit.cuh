// Drop-in path of the reference's header (include/function/GPURecSplit.cuh): the class is
// implemented by the B200 engine behind the C ABI (include/rsb/GPURecSplit.hpp). Plain C++;
// no CUDA compiler is needed to include it.
#pragma once
#include "../rsb/GPURecSplit.hpp"
