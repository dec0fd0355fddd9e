// dg_net_impl.h -- internal entry points of the correction network for the
// other sources of the library (the learned coarse step).
#pragma once
#include <cuda_runtime.h>

struct dg_net;

namespace dg {
// Inference forward pass on the given stream (asynchronous; the first call
// for a shape allocates the activation workspace and synchronises).
int net_forward_stream(dg_net *net, const void *feat, int n, int x, int y, int z, float *out, cudaStream_t st);
int net_inputs(const dg_net *net);
int net_device(const dg_net *net);
int net_outputs(const dg_net *net);
unsigned *net_status(dg_net *net);
const char *net_error(const dg_net *net);
}  // namespace dg
