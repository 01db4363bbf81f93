// Compiled configurations of order 6 (precision, fused runs, relaxation mechanisms).
#include "kernel_impl.cuh"

namespace edge_b200 {
KernelSet *makeKernelSet_o6(int precision, int order, int runs, int rms) {
#include "inst_o6.inc"
  return nullptr;
}

// process-wide instances, one per device, for callers that must not allocate
// (edge_b200_step_noalloc); device < kStaticDevices
KernelSet *staticKernelSet_o6(int precision, int order, int runs, int rms, int device) {
#undef EDGE_B200_CFG
#define EDGE_B200_CFG(T, O, R, RM, prec)                          \
  if (precision == prec && order == O && runs == R && rms == RM) { \
    static KernelSetImpl<T, O, R, RM> inst[kStaticDevices];       \
    return &inst[device];                                         \
  }
#include "inst_o6.inc"
  return nullptr;
}
}  // namespace edge_b200
