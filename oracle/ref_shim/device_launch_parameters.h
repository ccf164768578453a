// Host-only stand-in (oracle build of the reference engine): everything the
// reference expects from this header is provided by ref_shim/cuda_runtime.h.
#pragma once
#include "cuda_runtime.h"
