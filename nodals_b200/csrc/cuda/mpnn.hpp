// Host interface of the learned pressure stage (mpnn.cu) used by the solver.
#pragma once
#include <cuda_runtime.h>

#include <memory>

#include "../../../include/nodals_b200.h"

namespace nds {

struct MpnnImpl;
struct MpnnDeleter {
  void operator()(MpnnImpl* m) const;
};
using MpnnPtr = std::unique_ptr<MpnnImpl, MpnnDeleter>;

// device state for graphs of up to n_max nodes, launching on stream st
MpnnPtr make_mpnn(int n_max, bool training, cudaStream_t st);
void mpnn_set_params(MpnnImpl& m, const float* host_params);
// z = N(v) on one graph segment; launches only (no host synchronisation, no
// host-to-device copy), so it can be captured in a CUDA graph
void mpnn_forward(MpnnImpl& m, const nds_mpnn_graph& g, const float* v, float* z);
// throws when a tensor-core wait of an earlier launch ran out
void mpnn_check(MpnnImpl& m);

}  // namespace nds
