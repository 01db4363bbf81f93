// Type-erased launchers of one compiled configuration (precision, order, runs, mechanisms).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace edge_b200 {

struct RecvArgs;
struct SrcArgs;

// StepArgs with the DOF pointers untyped; the concrete KernelSet casts to its precision.
struct StepArgsRaw {
  void *dofsE = nullptr, *dofsA = nullptr, *tDofs = nullptr, *face = nullptr;
  const double *starE = nullptr, *starA = nullptr, *srcA = nullptr, *fsE = nullptr, *fsA = nullptr;
  const int32_t *elFaEl = nullptr;
  const uint8_t *fId = nullptr, *vId = nullptr, *faType = nullptr;
  int64_t nEl = 0;
  int64_t elFirst = 0, elCount = 0;  // element range of the launch (a time group, or all)
  double dt = 0;
  double omega[3] = {0, 0, 0};
  // rate-2 LTS (all null for GTS): see StepArgs
  void *faceSum = nullptr, *faceHalf1 = nullptr, *faceHalf2 = nullptr;
  const uint8_t *ltsFlags = nullptr, *ltsRel = nullptr;
  const int32_t *sumIdx = nullptr, *halfIdx = nullptr;
  int firstTs = 0;
  // per element face fsE[0] and the face reader's fsE[1] in the configuration's precision, each
  // padded to 16 bytes: [nEl][4][2][fsPairStride()] (premix); fsChar: their characteristic
  // factors instead (charMix)
  const void *fsLR = nullptr;
  int fsChar = 0;
  // fused GTS steps: the previous step's face projections whose neighbour step is still pending
  const void *faceIn = nullptr;
  // per element group time steps of the GTS local step (merged simulations), or null
  const double *grpDt = nullptr;
};

class KernelSet {
 public:
  virtual ~KernelSet() {}
  virtual cudaError_t init(int device) = 0;  // sets smem attributes, sizes the persistent grids
  virtual cudaError_t local(const StepArgsRaw &a, cudaStream_t s) = 0;
  // the local step with the pending neighbour step of the previous one folded in (a.faceIn)
  virtual cudaError_t localFused(const StepArgsRaw &a, cudaStream_t s) = 0;
  virtual bool fusedSupported() const = 0;
  // local step with the LTS face buffers (the half-step time integral needs one more tile)
  virtual cudaError_t localLts(const StepArgsRaw &a, cudaStream_t s) = 0;
  // the same without half-step integrals, for elements without a smaller neighbour (no extra tile)
  virtual cudaError_t localLtsSums(const StepArgsRaw &a, cudaStream_t s) = 0;
  virtual bool ltsSupported() const = 0;
  // GTS face projections leave the local kernel mixed with the reader's flux solver (fsLR)
  virtual bool premix() const = 0;
  virtual int fsPairStride() const = 0;
  // the GTS local kernel mixes face projections through the rank-3 factors of the flux-solver
  // pairs when fsLR holds them (StepArgsRaw::fsChar)
  virtual bool charMix() const = 0;
  // the LTS local kernels do the same (both of their tiles of characteristic rows fit)
  virtual bool charMixLts() const = 0;
  virtual cudaError_t neigh(const StepArgsRaw &a, cudaStream_t s) = 0;
  // the neighbour step over the buffers the LTS local kernels wrote (pre-mixed where those
  // kernels have room for it)
  virtual cudaError_t neighLts(const StepArgsRaw &a, cudaStream_t s) = 0;
  virtual cudaError_t recv(const StepArgsRaw &a, const RecvArgs &r, cudaStream_t s) = 0;
  virtual cudaError_t sources(void *dofsE, const SrcArgs &sa, cudaStream_t s) = 0;
  virtual int elementsPerCta() const = 0;
  virtual int ctasLocal() const = 0;
  virtual int ctasNeigh() const = 0;
  // caps on the persistent grids of the GTS local / neighbour kernels (0: resident CTAs per SM x
  // SMs, the default; a larger cap gives one CTA per element group up to it)
  virtual void setGridCaps(int local, int neigh) = 0;
  // static instances only: init() has run on their device (edge_b200_step_noalloc, under its lock)
  bool staticReady = false;
};

// returns nullptr when the configuration is not compiled in
KernelSet *makeKernelSet(int precision, int order, int runs, int rms);

// devices the allocation-free entry point serves (one static kernel set per device and configuration)
constexpr int kStaticDevices = 64;

}  // namespace edge_b200
