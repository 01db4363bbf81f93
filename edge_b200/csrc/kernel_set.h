// Type-erased launchers of one compiled configuration (precision, order, runs, mechanisms).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace edge_b200 {

struct RecvArgs;
struct SrcArgs;

// StepArgs with the DOF pointers untyped; the concrete KernelSet casts to its precision.
struct StepArgsRaw {
  void *dofsE, *dofsA, *tDofs, *face;
  const double *starE, *starA, *srcA, *fsE, *fsA;
  const int32_t *elFaEl;
  const uint8_t *fId, *vId, *faType;
  int64_t nEl;
  double dt;
  double omega[3];
};

class KernelSet {
 public:
  virtual ~KernelSet() {}
  virtual cudaError_t init(int device) = 0;  // sets smem attributes, sizes the persistent grids
  virtual cudaError_t local(const StepArgsRaw &a, cudaStream_t s) = 0;
  virtual cudaError_t neigh(const StepArgsRaw &a, cudaStream_t s) = 0;
  virtual cudaError_t recv(const StepArgsRaw &a, const RecvArgs &r, cudaStream_t s) = 0;
  virtual cudaError_t sources(void *dofsE, const SrcArgs &sa, cudaStream_t s) = 0;
  virtual int elementsPerCta() const = 0;
  virtual int ctasLocal() const = 0;
  virtual int ctasNeigh() const = 0;
};

// returns nullptr when the configuration is not compiled in
KernelSet *makeKernelSet(int precision, int order, int runs, int rms);

}  // namespace edge_b200
