// Compiled configurations of order 4 (precision, fused runs, relaxation mechanisms).
#include "kernel_impl.cuh"

namespace edge_b200 {
KernelSet *makeKernelSet_o4(int precision, int order, int runs, int rms) {
#include "inst_o4.inc"
  return nullptr;
}
}  // namespace edge_b200
