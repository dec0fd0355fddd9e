// nvToolsExt.h (stub) -- TEST INFRASTRUCTURE ONLY: the reference's NVTX
// profiling ranges are no-ops (no NVTX library is linked).
#pragma once
inline int nvtxRangePushA(const char *) { return 0; }
inline int nvtxRangePop() { return 0; }
