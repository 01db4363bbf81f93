// Compiled configurations of order 2 (precision, fused runs, relaxation mechanisms).
#include "kernel_impl.cuh"

namespace edge_b200 {
KernelSet *makeKernelSet_o2(int precision, int order, int runs, int rms) {
#include "inst_o2.inc"
  return nullptr;
}
}  // namespace edge_b200
