/* Test infrastructure: host stand-in, see cuda_runtime.h beside it. */
#include "cuda_runtime.h"
