// nvToolsExt.h (host shim) -- TEST INFRASTRUCTURE ONLY: profiling ranges are no-ops.
#pragma once
inline int nvtxRangePushA(const char *) { return 0; }
inline int nvtxRangePop() { return 0; }
