// edge_b200_step_noalloc: the GTS step over caller-owned device arrays with its scratch (the face
// projections the local kernel writes and the neighbour kernel reads, and the DOFs converted to the
// kernels' row layout) in a static device array, for callers that cannot allocate device memory
// while they run.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/edge_b200.h"
#include "kernel_set.h"
#include "kernels.cuh"
#include "layout.cuh"

namespace edge_b200 {
KernelSet *staticKernelSet_o2(int, int, int, int, int);
KernelSet *staticKernelSet_o3(int, int, int, int, int);
KernelSet *staticKernelSet_o4(int, int, int, int, int);
KernelSet *staticKernelSet_o5(int, int, int, int, int);
KernelSet *staticKernelSet_o6(int, int, int, int, int);
}  // namespace edge_b200

using namespace edge_b200;

namespace {

constexpr size_t kScratchBytes = EDGE_B200_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = kStaticDevices;

// Held by every GPU that loads the library, until the process exits.
__device__ __align__(256) unsigned char g_faceScratch[kScratchBytes];

// per device: the array's device address (host code only sees a stand-in symbol); per device and
// configuration: whether that kernel set's launch attributes and grid sizes were set (each device
// has kernel sets of its own, so devices with different SM counts do not share grid sizes)
std::mutex g_setupMutex;
void *g_scratchPtr[kMaxDevices] = {};

KernelSet *staticKernelSet(int precision, int order, int runs, int rms, int device) {
  switch (order) {
    case 2: return staticKernelSet_o2(precision, order, runs, rms, device);
    case 3: return staticKernelSet_o3(precision, order, runs, rms, device);
    case 4: return staticKernelSet_o4(precision, order, runs, rms, device);
    case 5: return staticKernelSet_o5(precision, order, runs, rms, device);
    case 6: return staticKernelSet_o6(precision, order, runs, rms, device);
    default: return nullptr;
  }
}

// makes `device` current for the call and gives the caller's current device back on every return
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) return;
    ok = prev == device || cudaSetDevice(device) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (ok && prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int edge_b200_step_noalloc(const edge_b200_cfg *cfg, int64_t n_el, double dt, int n_steps,
                                      void *dofs_e, void *dofs_a, const double *star_e, const double *fs_e,
                                      const double *star_a, const double *src_a, const double *fs_a,
                                      const double *omega, const int32_t *el_fa_el,
                                      const uint8_t *fid_el_fa_el, const uint8_t *vid_el_fa_el,
                                      const uint8_t *el_fa_type) {
  if (!cfg || n_el < 1 || !(dt > 0) || n_steps < 0) return EDGE_B200_EINVAL;
  if (cfg->precision != 32 && cfg->precision != 64) return EDGE_B200_EINVAL;
  if (cfg->n_rms < 0 || cfg->n_rms > 3 || cfg->n_runs < 1 || 32 % cfg->n_runs) return EDGE_B200_EINVAL;
  if (cfg->device < 0 || cfg->device >= kMaxDevices) return EDGE_B200_EINVAL;
  if (!dofs_e || !star_e || !fs_e || !el_fa_el || !fid_el_fa_el || !vid_el_fa_el || !el_fa_type)
    return EDGE_B200_EINVAL;
  if (cfg->n_rms && (!dofs_a || !star_a || !src_a || !fs_a || !omega)) return EDGE_B200_EINVAL;
  // the neighbour kernel reads an element's four connectivity entries with one vector load
  if (reinterpret_cast<uintptr_t>(el_fa_el) % 16 || reinterpret_cast<uintptr_t>(fid_el_fa_el) % 4 ||
      reinterpret_cast<uintptr_t>(vid_el_fa_el) % 4 || reinterpret_cast<uintptr_t>(el_fa_type) % 4)
    return EDGE_B200_EINVAL;
  const size_t realSize = cfg->precision == 64 ? 8 : 4;
  // scratch: face projections, then the DOFs in the device-resident row layout (256-byte aligned);
  // n_el is checked against the per-element size first, so the products below cannot wrap
  const int B = nModes(cfg->order), GB = rowPad(B, cfg->precision);
  const int GF = rowPad(nFaceModes(cfg->order), cfg->precision);
  const size_t perEl = ((size_t)4 * 9 * GF + (size_t)(9 + 6 * cfg->n_rms) * GB) * cfg->n_runs * realSize;
  if ((uint64_t)n_el > kScratchBytes / perEl) return EDGE_B200_ESCRATCH;
  auto align = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t faceBytes = align((size_t)n_el * 4 * 9 * cfg->n_runs * GF * realSize);
  const size_t dofsBytes = align((size_t)n_el * 9 * cfg->n_runs * GB * realSize);
  const size_t dofsABytes = align((size_t)n_el * 6 * cfg->n_rms * cfg->n_runs * GB * realSize);
  if (faceBytes + dofsBytes + dofsABytes > kScratchBytes) return EDGE_B200_ESCRATCH;
  KernelSet *ks = staticKernelSet(cfg->precision, cfg->order, cfg->n_runs, cfg->n_rms, cfg->device);
  if (!ks) return EDGE_B200_ENOTSUP;

  DeviceGuard dev(cfg->device);
  if (!dev.ok) return EDGE_B200_EDEVICE;
  void *scratch = nullptr;
  {
    // set-up once per device (the scratch address) and once per device and configuration (the
    // kernels' dynamic shared-memory limits and persistent grid sizes), with that device current
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchPtr[cfg->device]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_faceScratch) != cudaSuccess || !p) return EDGE_B200_EDEVICE;
      g_scratchPtr[cfg->device] = p;
    }
    scratch = g_scratchPtr[cfg->device];
    if (!ks->staticReady) {
      if (ks->init(cfg->device) != cudaSuccess) return EDGE_B200_EDEVICE;
      ks->staticReady = true;
    }
  }

  StepArgsRaw a;
  unsigned char *sc = static_cast<unsigned char *>(scratch);
  a.dofsE = sc + faceBytes;
  a.dofsA = cfg->n_rms ? sc + faceBytes + dofsBytes : nullptr;
  a.tDofs = nullptr;
  a.face = sc;
  a.starE = star_e;
  a.starA = cfg->n_rms ? star_a : nullptr;
  a.srcA = cfg->n_rms ? src_a : nullptr;
  a.fsE = fs_e;
  a.fsA = cfg->n_rms ? fs_a : nullptr;
  a.elFaEl = el_fa_el;
  a.fId = fid_el_fa_el;
  a.vId = vid_el_fa_el;
  a.faType = el_fa_type;
  a.nEl = n_el;
  a.elFirst = 0;
  a.elCount = n_el;
  a.dt = dt;
  for (int m = 0; m < 3; m++) a.omega[m] = (cfg->n_rms && m < cfg->n_rms) ? omega[m] : 0.0;
  cudaStream_t s = (cudaStream_t)cfg->stream;
  // the caller's DOFs (reference layout) into the scratch rows, the steps, and back
  const int R = cfg->n_runs, P = cfg->precision;
  if (convertLayout(true, P, dofs_e, a.dofsE, n_el * 9, B, R, GB, s) != cudaSuccess) return EDGE_B200_EDEVICE;
  if (cfg->n_rms && convertLayout(true, P, dofs_a, a.dofsA, n_el * 6 * cfg->n_rms, B, R, GB, s) != cudaSuccess)
    return EDGE_B200_EDEVICE;
  for (int st = 0; st < n_steps; st++) {
    if (ks->local(a, s) != cudaSuccess) return EDGE_B200_EDEVICE;
    if (ks->neigh(a, s) != cudaSuccess) return EDGE_B200_EDEVICE;
  }
  if (convertLayout(false, P, a.dofsE, dofs_e, n_el * 9, B, R, GB, s) != cudaSuccess) return EDGE_B200_EDEVICE;
  if (cfg->n_rms && convertLayout(false, P, a.dofsA, dofs_a, n_el * 6 * cfg->n_rms, B, R, GB, s) != cudaSuccess)
    return EDGE_B200_EDEVICE;
  return EDGE_B200_OK;
}
