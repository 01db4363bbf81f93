// Kernel-set factories of one order (EDGE_B200_ORDER, configurations listed in EDGE_B200_INC),
// split over four objects: the order's inst_oN.cu is compiled once per part with
// -DEDGE_B200_PART=p, and each object instantiates only every fourth configuration of the list
// (from the p-th on), so the configurations of one order compile in parallel. Part 0 also holds
// the order's entry points, which ask the parts in turn.
#pragma once
#include "kernel_impl.cuh"

#ifndef EDGE_B200_PART
#define EDGE_B200_PART 0
#endif
#define EDGE_B200_CAT2(a, b) a##b
#define EDGE_B200_CAT(a, b) EDGE_B200_CAT2(a, b)
#define EDGE_B200_FN(base, p) EDGE_B200_CAT(EDGE_B200_CAT(EDGE_B200_CAT(base, EDGE_B200_ORDER), _p), p)

namespace edge_b200 {
constexpr int kInstParts = 4;
static_assert(EDGE_B200_PART >= 0 && EDGE_B200_PART < kInstParts, "part index");

// configuration I of the list, when it belongs to this part and matches the request
template <int I, typename T, int O, int R, int RM>
KernelSet *pickKernelSet(int precision, int order, int runs, int rms, int prec) {
  if constexpr (I % kInstParts == EDGE_B200_PART) {
    if (precision == prec && order == O && runs == R && rms == RM) return new KernelSetImpl<T, O, R, RM>();
  }
  return nullptr;
}
// the same as process-wide instances, one per device, for callers that must not allocate
// (edge_b200_step_noalloc); device < kStaticDevices
template <int I, typename T, int O, int R, int RM>
KernelSet *pickStaticKernelSet(int precision, int order, int runs, int rms, int prec, int device) {
  if constexpr (I % kInstParts == EDGE_B200_PART) {
    if (precision == prec && order == O && runs == R && rms == RM) {
      static KernelSetImpl<T, O, R, RM> inst[kStaticDevices];
      return &inst[device];
    }
  }
  return nullptr;
}

KernelSet *EDGE_B200_FN(makeKernelSet_o, EDGE_B200_PART)(int precision, int order, int runs, int rms) {
  enum { kBase = __COUNTER__ };
#undef EDGE_B200_CFG
#define EDGE_B200_CFG(T, O, R, RM, prec)                                                               \
  if (KernelSet *k = pickKernelSet<__COUNTER__ - kBase - 1, T, O, R, RM>(precision, order, runs, rms, prec)) \
    return k;
#include EDGE_B200_INC
  return nullptr;
}

KernelSet *EDGE_B200_FN(staticKernelSet_o, EDGE_B200_PART)(int precision, int order, int runs, int rms,
                                                          int device) {
  enum { kBase = __COUNTER__ };
#undef EDGE_B200_CFG
#define EDGE_B200_CFG(T, O, R, RM, prec)                                                                  \
  if (KernelSet *k =                                                                                      \
          pickStaticKernelSet<__COUNTER__ - kBase - 1, T, O, R, RM>(precision, order, runs, rms, prec, device)) \
    return k;
#include EDGE_B200_INC
  return nullptr;
}

#if EDGE_B200_PART == 0
KernelSet *EDGE_B200_FN(makeKernelSet_o, 1)(int, int, int, int);
KernelSet *EDGE_B200_FN(makeKernelSet_o, 2)(int, int, int, int);
KernelSet *EDGE_B200_FN(makeKernelSet_o, 3)(int, int, int, int);
KernelSet *EDGE_B200_FN(staticKernelSet_o, 1)(int, int, int, int, int);
KernelSet *EDGE_B200_FN(staticKernelSet_o, 2)(int, int, int, int, int);
KernelSet *EDGE_B200_FN(staticKernelSet_o, 3)(int, int, int, int, int);
static_assert(kInstParts == 4, "the entry points ask parts 0-3");

KernelSet *EDGE_B200_CAT(makeKernelSet_o, EDGE_B200_ORDER)(int precision, int order, int runs, int rms) {
  KernelSet *k = EDGE_B200_FN(makeKernelSet_o, 0)(precision, order, runs, rms);
  if (!k) k = EDGE_B200_FN(makeKernelSet_o, 1)(precision, order, runs, rms);
  if (!k) k = EDGE_B200_FN(makeKernelSet_o, 2)(precision, order, runs, rms);
  if (!k) k = EDGE_B200_FN(makeKernelSet_o, 3)(precision, order, runs, rms);
  return k;
}

KernelSet *EDGE_B200_CAT(staticKernelSet_o, EDGE_B200_ORDER)(int precision, int order, int runs, int rms,
                                                             int device) {
  KernelSet *k = EDGE_B200_FN(staticKernelSet_o, 0)(precision, order, runs, rms, device);
  if (!k) k = EDGE_B200_FN(staticKernelSet_o, 1)(precision, order, runs, rms, device);
  if (!k) k = EDGE_B200_FN(staticKernelSet_o, 2)(precision, order, runs, rms, device);
  if (!k) k = EDGE_B200_FN(staticKernelSet_o, 3)(precision, order, runs, rms, device);
  return k;
}
#endif
}  // namespace edge_b200
