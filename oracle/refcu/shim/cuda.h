// cuda.h (host shim) -- TEST INFRASTRUCTURE ONLY; see cuda_runtime.h.
#pragma once
#include "cuda_runtime.h"
