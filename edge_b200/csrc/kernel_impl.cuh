// KernelSet implementation for one configuration; included by the inst_*.cu translation units.
#pragma once
#include "kernel_set.h"
#include "kernels.cuh"

namespace edge_b200 {

template <typename T, int O, int R, int RM>
class KernelSetImpl final : public KernelSet {
  using G = Geo<T, O, R, RM>;
  int numSms_ = 0, occLocal_ = 1, occNeigh_ = 1, occRecv_ = 1, occLocalLts_ = 1, occLocalSum_ = 1,
      capLocal_ = 0, capNeigh_ = 0;

  static StepArgs<T> cast(const StepArgsRaw &a) {
    StepArgs<T> b;
    b.dofsE = static_cast<T *>(a.dofsE);
    b.dofsA = static_cast<T *>(a.dofsA);
    b.tDofs = static_cast<T *>(a.tDofs);
    b.face = static_cast<T *>(a.face);
    b.starE = a.starE;
    b.starA = a.starA;
    b.srcA = a.srcA;
    b.fsE = a.fsE;
    b.fsA = a.fsA;
    b.elFaEl = a.elFaEl;
    b.fId = a.fId;
    b.vId = a.vId;
    b.faType = a.faType;
    b.nEl = a.nEl;
    b.elFirst = a.elFirst;
    b.elCount = a.elCount;
    b.dt = a.dt;
    for (int i = 0; i < 3; i++) b.omega[i] = a.omega[i];
    b.faceSum = static_cast<T *>(a.faceSum);
    b.faceHalf1 = static_cast<T *>(a.faceHalf1);
    b.faceHalf2 = static_cast<T *>(a.faceHalf2);
    b.ltsFlags = a.ltsFlags;
    b.ltsRel = a.ltsRel;
    b.sumIdx = a.sumIdx;
    b.halfIdx = a.halfIdx;
    b.firstTs = a.firstTs;
    b.fsLR = static_cast<const T *>(a.fsLR);
    b.fsChar = a.fsChar;
    b.faceIn = static_cast<const T *>(a.faceIn);
    b.grpDt = a.grpDt;
    return b;
  }
  static constexpr size_t smemLocal() { return G::smemLocalGts; }
  static constexpr size_t smemNeigh() { return G::smemNeigh; }
  static constexpr size_t smemRecv() { return G::smemLocal; }

 public:
  cudaError_t init(int device) override {
    cudaError_t e;
    if ((e = cudaDeviceGetAttribute(&numSms_, cudaDevAttrMultiProcessorCount, device))) return e;
    if ((e = cudaFuncSetAttribute(kLocal<T, O, R, RM, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemLocal())))
      return e;
    if ((e = cudaFuncSetAttribute(kNeigh<T, O, R, RM, G::premix>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemNeigh())))
      return e;
    if ((e = cudaFuncSetAttribute(kRecv<T, O, R, RM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemRecv())))
      return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occLocal_, kLocal<T, O, R, RM, 0>, G::NT, smemLocal())))
      return e;
    if constexpr (G::premix) {
      if ((e = cudaFuncSetAttribute(kLocal<T, O, R, RM, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smemLocal())))
        return e;
    }
    if constexpr (G::charMix) {
      if ((e = cudaFuncSetAttribute(kLocal<T, O, R, RM, 0, false, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemLocal())))
        return e;
      if ((e = cudaFuncSetAttribute(kLocal<T, O, R, RM, 0, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smemLocal())))
        return e;
    }
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occNeigh_, kNeigh<T, O, R, RM, G::premix>, G::NT, smemNeigh())))
      return e;
    if constexpr (G::premixLts != G::premix) {
      if ((e = cudaFuncSetAttribute(kNeigh<T, O, R, RM, G::premixLts>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smemNeigh())))
        return e;
    }
    if constexpr (G::ltsOk) {
      if ((e = cudaFuncSetAttribute(kLocal<T, O, R, RM, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)G::smemLocalLts)))
        return e;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occLocalLts_, kLocal<T, O, R, RM, 2>, G::NT,
                                                             G::smemLocalLts)))
        return e;
      occLocalLts_ = occLocalLts_ < 1 ? 1 : occLocalLts_;
      if ((e = cudaFuncSetAttribute(kLocal<T, O, R, RM, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)G::smemLocalSums)))
        return e;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occLocalSum_, kLocal<T, O, R, RM, 1>, G::NT,
                                                             G::smemLocalSums)))
        return e;
      occLocalSum_ = occLocalSum_ < 1 ? 1 : occLocalSum_;
      if constexpr (G::charMixLts) {
        if ((e = cudaFuncSetAttribute(kLocal<T, O, R, RM, 2, false, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smemLocalLts)))
          return e;
        if ((e = cudaFuncSetAttribute(kLocal<T, O, R, RM, 1, false, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smemLocalSums)))
          return e;
      }
    }
    occLocal_ = occLocal_ < 1 ? 1 : occLocal_;
    occNeigh_ = occNeigh_ < 1 ? 1 : occNeigh_;
    return cudaSuccess;
  }
  int elementsPerCta() const override { return G::E; }
  int ctasLocal() const override { return capLocal_ > 0 ? capLocal_ : numSms_ * occLocal_; }
  int ctasNeigh() const override { return capNeigh_ > 0 ? capNeigh_ : numSms_ * occNeigh_; }
  void setGridCaps(int local, int neigh) override {
    capLocal_ = local;
    capNeigh_ = neigh;
  }

  static int grid(int64_t nEl, int cap) {
    int64_t groups = (nEl + G::E - 1) / G::E;
    return (int)(groups < cap ? (groups < 1 ? 1 : groups) : cap);
  }

  cudaError_t local(const StepArgsRaw &a, cudaStream_t s) override {
    if (a.elCount < 1) return cudaSuccess;
    if constexpr (G::charMix) {
      if (a.fsChar) {
        kLocal<T, O, R, RM, 0, false, true><<<grid(a.elCount, ctasLocal()), G::NT, smemLocal(), s>>>(cast(a));
        return cudaGetLastError();
      }
    }
    kLocal<T, O, R, RM, 0><<<grid(a.elCount, ctasLocal()), G::NT, smemLocal(), s>>>(cast(a));
    return cudaGetLastError();
  }
  cudaError_t localFused(const StepArgsRaw &a, cudaStream_t s) override {
    if constexpr (G::premix) {
      if (a.elCount < 1) return cudaSuccess;
      if constexpr (G::charMix) {
        if (a.fsChar) {
          kLocal<T, O, R, RM, 0, true, true><<<grid(a.elCount, ctasLocal()), G::NT, smemLocal(), s>>>(cast(a));
          return cudaGetLastError();
        }
      }
      kLocal<T, O, R, RM, 0, true><<<grid(a.elCount, ctasLocal()), G::NT, smemLocal(), s>>>(cast(a));
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  bool fusedSupported() const override { return G::premix; }
  cudaError_t localLts(const StepArgsRaw &a, cudaStream_t s) override {
    if constexpr (G::ltsOk) {
      if (a.elCount < 1) return cudaSuccess;
      if constexpr (G::charMixLts) {
        if (a.fsChar) {
          kLocal<T, O, R, RM, 2, false, true>
              <<<grid(a.elCount, numSms_ * occLocalLts_), G::NT, G::smemLocalLts, s>>>(cast(a));
          return cudaGetLastError();
        }
      }
      kLocal<T, O, R, RM, 2><<<grid(a.elCount, numSms_ * occLocalLts_), G::NT, G::smemLocalLts, s>>>(cast(a));
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  cudaError_t localLtsSums(const StepArgsRaw &a, cudaStream_t s) override {
    if constexpr (G::ltsOk) {
      if (a.elCount < 1) return cudaSuccess;
      if constexpr (G::charMixLts) {
        if (a.fsChar) {
          kLocal<T, O, R, RM, 1, false, true>
              <<<grid(a.elCount, numSms_ * occLocalSum_), G::NT, G::smemLocalSums, s>>>(cast(a));
          return cudaGetLastError();
        }
      }
      kLocal<T, O, R, RM, 1><<<grid(a.elCount, numSms_ * occLocalSum_), G::NT, G::smemLocalSums, s>>>(cast(a));
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  bool ltsSupported() const override { return G::ltsOk; }
  bool premix() const override { return G::premix; }
  int fsPairStride() const override { return G::FSP; }
  bool charMix() const override { return G::charMix; }
  bool charMixLts() const override { return G::charMixLts; }
  cudaError_t neigh(const StepArgsRaw &a, cudaStream_t s) override {
    if (a.elCount < 1) return cudaSuccess;
    kNeigh<T, O, R, RM, G::premix><<<grid(a.elCount, ctasNeigh()), G::NT, smemNeigh(), s>>>(cast(a));
    return cudaGetLastError();
  }
  cudaError_t neighLts(const StepArgsRaw &a, cudaStream_t s) override {
    if (a.elCount < 1) return cudaSuccess;
    kNeigh<T, O, R, RM, G::premixLts><<<grid(a.elCount, ctasNeigh()), G::NT, smemNeigh(), s>>>(cast(a));
    return cudaGetLastError();
  }
  cudaError_t recv(const StepArgsRaw &a, const RecvArgs &r, cudaStream_t s) override {
    const int g = (r.nGrp + G::E - 1) / G::E;
    if (g == 0) return cudaSuccess;
    kRecv<T, O, R, RM><<<g, G::NT, smemRecv(), s>>>(cast(a), r);
    return cudaGetLastError();
  }
  cudaError_t sources(void *dofsE, const SrcArgs &sa, cudaStream_t s) override {
    if (sa.nGrp == 0) return cudaSuccess;
    kSources<T, O, R><<<sa.nGrp, 128, 0, s>>>(static_cast<T *>(dofsE), sa);
    return cudaGetLastError();
  }
};

}  // namespace edge_b200

// registry of one translation unit: a function returning the matching configuration
#define EDGE_B200_CFG(T, O, R, RM, prec)                                    \
  if (precision == prec && order == O && runs == R && rms == RM)           \
    return new edge_b200::KernelSetImpl<T, O, R, RM>();
