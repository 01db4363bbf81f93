// C ABI of the device element update (include/edge_b200.h): context, uploads, the GTS step loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/edge_b200.h"
#include "kernel_set.h"
#include "kernels.cuh"
#include "layout.cuh"

namespace edge_b200 {
KernelSet *makeKernelSet_o2(int, int, int, int);
KernelSet *makeKernelSet_o3(int, int, int, int);
KernelSet *makeKernelSet_o4(int, int, int, int);
KernelSet *makeKernelSet_o5(int, int, int, int);
KernelSet *makeKernelSet_o6(int, int, int, int);

KernelSet *makeKernelSet(int precision, int order, int runs, int rms) {
  switch (order) {
    case 2: return makeKernelSet_o2(precision, order, runs, rms);
    case 3: return makeKernelSet_o3(precision, order, runs, rms);
    case 4: return makeKernelSet_o4(precision, order, runs, rms);
    case 5: return makeKernelSet_o5(precision, order, runs, rms);
    case 6: return makeKernelSet_o6(precision, order, runs, rms);
    default: return nullptr;
  }
}
}  // namespace edge_b200

using namespace edge_b200;

namespace {
constexpr double kTolTime = 1e-9;  // TOL.TIME of the FP64 build (src/constants.hpp:289-309)

template <typename P>
void dfree(P *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

// A device array that keeps its allocation while later contents fit (cudaFree synchronises the
// device, which would stall the other contexts' streams on every re-set of sources or receivers).
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  cudaError_t fit(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    dfree(p);
    cap = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
  cudaError_t put(const void *src, size_t bytes, cudaStream_t s) {
    cudaError_t e = fit(bytes ? bytes : 1);
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, s);
    return e;
  }
  template <typename T>
  T *as() const { return static_cast<T *>(p); }
  ~DevBuf() { dfree(p); }
};

// flux-solver pairs of the pre-mixed face projections: per element face fsE[0] of the element and
// the fsE[1] block its face reader applies (the face neighbour's at its own face id for inner faces,
// the element's own for a free surface, zeros for outflow), 81 values padded to P, in the
// configuration's precision: out[nEl][4][2][P]
template <typename T>
__global__ void kBuildFsLR(const double *fsE, const int32_t *elFaEl, const uint8_t *fId, const uint8_t *faType,
                           int64_t nEl, int P, T *out) {
  const int64_t total = nEl * 4 * 2 * P;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t ef = i / (2 * P);
    const int w = int(i % (2 * P)) / P, j = int(i % P);
    double v = 0;
    if (j < 81) {
      if (w == 0) {
        v = fsE[ef * 81 + j];
      } else {
        const int ty = faType[ef];
        const int64_t e = ef / 4;
        const int fa = int(ef % 4);
        if (ty == EDGE_FACE_INNER)
          v = fsE[((nEl + elFaEl[ef]) * 4 + fId[ef]) * 81 + j];
        else if (ty == EDGE_FACE_FREE_SURFACE)
          v = fsE[((nEl + e) * 4 + fa) * 81 + j];
      }
    }
    out[i] = T(v);
  }
}

// characteristic factors of the same pairs (Geo::charMix): per element face the stacked flux
// solvers S = [fsE[0]; the reader's fsE[1]] (18 x 9, zeros for an outflow reader) have rank 3 --
// the waves leaving the element through the face -- so S = U V^T with U 18 x 3 and V 9 x 3. The
// columns of S (inputs: stresses and velocities, whose scales differ by the impedances) are
// scaled to unit maximum, c; Gram-Schmidt with pivoting over the 18 scaled rows (each new
// direction orthogonalised twice) gives Q (3 orthonormal directions); then U = (S / c) Q^T and
// V = c Q. out[nEl][4][2][P]: V [9][4] (column 3 zero), then per quantity q {U0[q][0..2],
// U1[q][0..2], 0, 0}, the rest zero; a face whose scaled rows keep more than 1e-9 of the largest
// row's norm outside the three directions counts in *bad (its pair is not of rank 3).
template <typename T>
__global__ void kBuildFsChar(const double *fsE, const int32_t *elFaEl, const uint8_t *fId, const uint8_t *faType,
                             int64_t nEl, int P, T *out, int *bad) {
  for (int64_t ef = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; ef < nEl * 4;
       ef += int64_t(gridDim.x) * blockDim.x) {
    const double *A = fsE + ef * 81;
    const double *Bm = nullptr;
    const int ty = faType[ef];
    if (ty == EDGE_FACE_INNER)
      Bm = fsE + ((nEl + elFaEl[ef]) * 4 + fId[ef]) * 81;
    else if (ty == EDGE_FACE_FREE_SURFACE)
      Bm = fsE + (nEl * 4 + ef) * 81;
    auto entry = [&](int i, int j) { return i < 9 ? A[i * 9 + j] : (Bm ? Bm[(i - 9) * 9 + j] : 0.0); };
    double c[9];
    for (int j = 0; j < 9; j++) {
      double m = 0;
      for (int i = 0; i < 18; i++) m = fmax(m, fabs(entry(i, j)));
      c[j] = m > 0 ? m : 1.0;
    }
    double rs[18][9], nrm0 = 0;
    for (int i = 0; i < 18; i++) {
      double n2 = 0;
      for (int j = 0; j < 9; j++) {
        rs[i][j] = entry(i, j) / c[j];
        n2 += rs[i][j] * rs[i][j];
      }
      nrm0 = fmax(nrm0, n2);
    }
    double Q[3][9];
    for (int k = 0; k < 3; k++) {
      int piv = 0;
      double best = -1;
      for (int i = 0; i < 18; i++) {
        double n2 = 0;
        for (int j = 0; j < 9; j++) n2 += rs[i][j] * rs[i][j];
        if (n2 > best) {
          best = n2;
          piv = i;
        }
      }
      double v[9];
      for (int j = 0; j < 9; j++) v[j] = rs[piv][j];
      for (int pass = 0; pass < 2; pass++)
        for (int kk = 0; kk < k; kk++) {
          double d = 0;
          for (int j = 0; j < 9; j++) d += v[j] * Q[kk][j];
          for (int j = 0; j < 9; j++) v[j] -= d * Q[kk][j];
        }
      double n2 = 0;
      for (int j = 0; j < 9; j++) n2 += v[j] * v[j];
      const double inv = n2 > 1e-60 * nrm0 && n2 > 0 ? 1.0 / sqrt(n2) : 0.0;
      for (int j = 0; j < 9; j++) Q[k][j] = v[j] * inv;
      for (int i = 0; i < 18; i++) {
        double d = 0;
        for (int j = 0; j < 9; j++) d += rs[i][j] * Q[k][j];
        for (int j = 0; j < 9; j++) rs[i][j] -= d * Q[k][j];
      }
    }
    double res = 0;
    for (int i = 0; i < 18; i++) {
      double n2 = 0;
      for (int j = 0; j < 9; j++) n2 += rs[i][j] * rs[i][j];
      res = fmax(res, n2);
    }
    if (res > 1e-18 * nrm0) atomicAdd(bad, 1);
    T *o = out + ef * 2 * P;
    for (int j = 0; j < 2 * P; j++) o[j] = T(0);
    for (int j = 0; j < 9; j++)
      for (int k = 0; k < 3; k++) o[4 * j + k] = T(c[j] * Q[k][j]);
    for (int i = 0; i < 18; i++)
      for (int k = 0; k < 3; k++) {
        double u = 0;
        for (int j = 0; j < 9; j++) u += entry(i, j) / c[j] * Q[k][j];
        o[36 + (i % 9) * 8 + (i / 9) * 3 + k] = T(u);
      }
  }
}

// halo exchange: blocks [9][R][GF] of face slots (element * 4 + face) to / from a packed buffer,
// 16 bytes per thread; slots outside the face buffer are skipped
__global__ void kFacePack(uint4 *face, uint4 *buf, const int32_t *slots, int n, int64_t blk16, int64_t nSlots,
                          bool pack) {
  const int64_t total = (int64_t)n * blk16;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t k = i / blk16, w = i % blk16;
    const int64_t sl = slots[k];
    if (sl < 0 || sl >= nSlots) continue;
    if (pack)
      buf[i] = face[sl * blk16 + w];
    else
      face[sl * blk16 + w] = buf[i];
  }
}

// Error norms against plane waves. Thread (q, r) of a CTA holds the DOF row of quantity q, run r
// of an element, evaluates it at the quadrature points (basis values in shared memory) and the
// reference sum of plane waves at the physical points; L1 / squared L2 accumulate with the
// physical weights, Linf as a maximum; one atomic per thread and norm at the end.
struct PlaneWave {
  double k[3], omega, phase;
  double amp[9];
  int run;  // -1: every run
};
template <typename T>
__global__ void kErrorNorms(const T *dofsE, const double *geom, int64_t nEl, int B, int R, int G, int nQp,
                            const double *quad /* [nQp][3 + 1 + B]: xi, w, basis */, const PlaneWave *waves,
                            int nWaves, double t, double *norms /* [3][9][R] */) {
  extern __shared__ double sq[];
  const int stride = 4 + B;
  for (int i = threadIdx.x; i < nQp * stride; i += blockDim.x) sq[i] = quad[i];
  __syncthreads();
  const int q = threadIdx.x / R, r = threadIdx.x % R;
  if (q >= 9) return;
  double l1 = 0, l2 = 0, li = 0;
  double row[64];
  for (int64_t e = blockIdx.x; e < nEl; e += gridDim.x) {
    const T *p = dofsE + ((e * 9 + q) * R + r) * int64_t(G);
    for (int b = 0; b < B; b++) row[b] = double(p[b]);
    const double *v = geom + e * 12;
    double j[3][3];
    for (int a = 0; a < 3; a++)
      for (int d = 0; d < 3; d++) j[a][d] = v[3 * (a + 1) + d] - v[d];
    const double det = fabs(j[0][0] * (j[1][1] * j[2][2] - j[1][2] * j[2][1]) -
                            j[0][1] * (j[1][0] * j[2][2] - j[1][2] * j[2][0]) +
                            j[0][2] * (j[1][0] * j[2][1] - j[1][1] * j[2][0]));
    for (int k = 0; k < nQp; k++) {
      const double *qp = sq + k * stride;
      double uh = 0;
      for (int b = 0; b < B; b++) uh += qp[4 + b] * row[b];
      double x[3];
      for (int d = 0; d < 3; d++) x[d] = v[d] + qp[0] * j[0][d] + qp[1] * j[1][d] + qp[2] * j[2][d];
      double ur = 0;
      for (int w = 0; w < nWaves; w++) {
        const PlaneWave &pw = waves[w];
        if (pw.run >= 0 && pw.run != r) continue;
        ur += pw.amp[q] * sin(pw.k[0] * x[0] + pw.k[1] * x[1] + pw.k[2] * x[2] - pw.omega * t + pw.phase);
      }
      const double diff = fabs(uh - ur), wt = qp[3] * det;
      l1 += diff * wt;
      l2 += diff * diff * wt;
      li = fmax(li, diff);
    }
  }
  atomicAdd(norms + q * R + r, l1);
  atomicAdd(norms + (9 + q) * R + r, l2);
  // non-negative doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long *>(norms + (18 + q) * R + r), __double_as_longlong(li));
}

// wave-field snapshot: the mode-0 coefficient (the element mean of the orthogonal basis) of every
// quantity and run as FP32, out[run][q][el]
template <typename T>
__global__ void kWaveField(const T *dofsE, int64_t nEl, int R, int G, float *out) {
  const int64_t total = nEl * 9 * R;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t e = i % nEl, qr = i / nEl;
    const int q = int(qr % 9), r = int(qr / 9);
    out[i] = float(dofsE[((e * 9 + q) * R + r) * int64_t(G)]);
  }
}

// rows [nRows][R][G] <- src [nRows][B] for one run (zeros when src is null)
template <typename T>
__global__ void kSetRun(T *rows, const T *src, int64_t nRows, int B, int R, int G, int run) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nRows * G) return;
  const int64_t row = i / G;
  const int n = int(i % G);
  rows[(row * R + run) * G + n] = (src && n < B) ? src[row * B + n] : T(0);
}
}  // namespace

struct edge_b200_ctx {
  edge_b200_cfg cfg{};
  int64_t nEl = 0;
  int64_t nOwned = 0;  // the kernels update elements [0, nOwned); the rest are halo ghosts
  // halo parts: owned elements [0, nSend) have a face neighbour in another part; the local step
  // can run on them first (their face rows packed and sent while the rest run)
  int64_t nSend = 0;
  // local-step range of the next runSteps call (phases 2 / 3 of edge_b200_step_phase)
  int64_t rangeFirst = 0, rangeCount = -1;
  bool rangeRecv = true, rangeSrc = true;
  int B = 0, F = 0;
  size_t realSize = 8;
  cudaStream_t stream = nullptr;
  KernelSet *ks = nullptr;
  // resident device data
  void *dofsE = nullptr, *dofsA = nullptr, *tDofs = nullptr, *face = nullptr;
  double *starE = nullptr, *starA = nullptr, *srcA = nullptr, *fsE = nullptr, *fsA = nullptr;
  int32_t *elFaEl = nullptr;
  uint8_t *fId = nullptr, *vId = nullptr, *faType = nullptr;
  double omega[3] = {0, 0, 0};
  bool meshSet = false, dataSet = false, keepTDofs = false;
  // flux-solver pairs of the pre-mixed face projections (configurations with KernelSet::premix),
  // rebuilt before the next GTS step after the mesh or the element data changed
  DevBuf fsLR;
  bool fsLRStale = true;
  bool fsLRChar = false;      // fsLR holds the characteristic factors of the pairs
  DevBuf charBad;             // device counter of the factor build's rank check
  bool charRejected = false;  // some face's pair is not of rank 3 (until the element data changes)
  // fused GTS steps (pre-mixing configurations, no halo): within one multi-step call each local
  // step also runs the previous step's neighbour step, so the face projections alternate between
  // two buffers (faceCur holds the last written); the last step's neighbour step runs on its own at
  // the end of the call (flush), so between calls nothing is pending
  DevBuf faceAlt;
  int faceCur = 0;
  bool pending = false, fusedOn = true;
  void *faceBuf(int i) const { return i ? faceAlt.p : face; }
  // sources
  SrcArgs src{};
  DevBuf srcMem[10];
  // per-source clocks and per-group time steps of merged simulations (edge_b200_set_source_clocks,
  // edge_b200_set_group_dt); srcStep counts the steps since the clocks were set
  DevBuf srcClk0, srcClkDt, grpDt;
  bool srcClocks = false, grpDtOn = false;
  int64_t srcStep = 0;
  int nSrc = 0;
  // merged simulations still running: elements [0, nActive) (the rest share no face with them)
  int64_t nActive = INT64_MAX;
  // receivers
  int nRecv = 0, nRecvGrp = 0, maxBuf = 0;
  double recvTime = 0, period = 0;
  int32_t recvCount = 0;
  DevBuf grpEl, grpOff, basis, recvBuf;
  std::vector<double> hBufTime;
  std::vector<int64_t> hRecvGrpEl;  // element of each receiver group (ascending)
  std::vector<int32_t> hRecvOff;    // receivers of group g: hRecvOff[g] .. hRecvOff[g+1]
  bool lastLts = false;             // the receivers were last advanced by edge_b200_step_lts
  std::vector<int64_t> hSrcGrpEl;   // element of each source group (ascending)
  // host copy of the connectivity (LTS relations are derived from it)
  std::vector<int32_t> hElFaEl;
  std::vector<uint8_t> hFId, hFaType;
  // rate-2 LTS: time groups are element ranges [tgFirst[g], tgFirst[g+1]); per-group receiver
  // clocks; compact face buffers of the elements at group interfaces
  int nTg = 0;
  std::vector<int64_t> tgFirst;
  std::vector<int64_t> tgHalfEnd;  // group g: elements [tgFirst[g], tgHalfEnd[g]) hold every one with a smaller neighbour
  std::vector<double> tgRecvTime;
  std::vector<int32_t> tgRecvCount;
  DevBuf ltsFlags, ltsRel, sumIdx, halfIdx, faceSum, faceHalf1, faceHalf2;
  // element vertex coordinates [nEl][4][3] (error norms), plane waves and norm accumulators
  DevBuf geom, waves, quad, norms;
  int groupOf(int64_t el) const {
    int g = 0;
    while (g + 1 < nTg && el >= tgFirst[g + 1]) g++;
    return g;
  }
  double *dTau = nullptr;
  int32_t *dSlot = nullptr;
  size_t tauCap = 0;
  int64_t launches = 0;
  std::string err;
  // optional per-kernel event timing: pairs of events per launch, resolved lazily
  bool timing = false;
  struct Timed { int kind; cudaEvent_t a, b; };
  std::vector<Timed> timed;
  std::vector<cudaEvent_t> eventPool;
  double kernMs[4] = {0, 0, 0, 0};
  int64_t kernN[4] = {0, 0, 0, 0};

  cudaEvent_t takeEvent() {
    if (!eventPool.empty()) {
      cudaEvent_t e = eventPool.back();
      eventPool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  void resolveTimes() {
    for (auto &t : timed) {
      float ms = 0;
      cudaEventSynchronize(t.b);
      cudaEventElapsedTime(&ms, t.a, t.b);
      kernMs[t.kind] += ms;
      kernN[t.kind]++;
      eventPool.push_back(t.a);
      eventPool.push_back(t.b);
    }
    timed.clear();
  }
  template <typename F>
  cudaError_t launch(int kind, F &&f) {
    if (!timing) return f();
    cudaEvent_t a = takeEvent(), b = takeEvent();
    cudaEventRecord(a, stream);
    cudaError_t e = f();
    cudaEventRecord(b, stream);
    timed.push_back({kind, a, b});
    if (timed.size() > 4096) resolveTimes();
    return e;
  }

  // device-resident row layout (padded rows of GB / GF elements) and the reference layout
  int GB = 0, GF = 0;
  void *stage = nullptr;  // reference-layout staging for uploads / downloads, allocated on first use
  size_t dofsCount() const { return (size_t)nEl * 9 * cfg.n_runs * GB; }
  size_t dofsACount() const { return (size_t)nEl * cfg.n_rms * 6 * cfg.n_runs * GB; }
  size_t faceCount() const { return (size_t)nEl * 4 * 9 * cfg.n_runs * GF; }
  size_t refCount(int rows) const { return (size_t)nEl * rows * B * cfg.n_runs; }
  cudaError_t ensureStage() {
    if (stage) return cudaSuccess;
    const size_t n = std::max(refCount(9), refCount(6 * cfg.n_rms));
    return cudaMalloc(&stage, n * realSize);
  }
  // host (reference layout) -> device rows
  cudaError_t uploadRows(void *rows, const void *host, int rowsPerEl) {
    cudaError_t e;
    if ((e = ensureStage())) return e;
    if ((e = cudaMemcpyAsync(stage, host, refCount(rowsPerEl) * realSize, cudaMemcpyHostToDevice, stream))) return e;
    return convertLayout(true, cfg.precision, stage, rows, nEl * rowsPerEl, B, cfg.n_runs, GB, stream);
  }
  // device rows -> host (reference layout); synchronises the stream
  cudaError_t downloadRows(void *host, const void *rows, int rowsPerEl) {
    cudaError_t e;
    if ((e = ensureStage())) return e;
    if ((e = convertLayout(false, cfg.precision, rows, stage, nEl * rowsPerEl, B, cfg.n_runs, GB, stream))) return e;
    if ((e = cudaMemcpyAsync(host, stage, refCount(rowsPerEl) * realSize, cudaMemcpyDeviceToHost, stream))) return e;
    return cudaStreamSynchronize(stream);
  }

  // asynchronous transfers on their own copy streams. Uploads move element chunks of about
  // kChunkBytes through a ring of kSlots staging slots: per chunk the copy and its layout kernel (on
  // the context stream) are ordered by events, and a slot is reused once the kernel of its previous
  // chunk read it, so the copies run back to back while the layout kernels trail them. Downloads
  // convert all rows at once (the next step rewrites them) into one of two full-size buffers and
  // copy that out; a buffer is reused once its copy from two downloads back finished, so the context
  // stream never waits for the copy of the step just before.
  static constexpr int kSlots = 3;
  static constexpr size_t kChunkBytes = size_t(1) << 30;
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t evH2D[kSlots] = {}, evToRows[kSlots] = {}, evFromRows[2] = {}, evD2H[2] = {};
  cudaEvent_t evMark = nullptr;
  void *slotIn[kSlots] = {}, *bufOut[2] = {};
  bool toRowsPending[kSlots] = {}, d2hPending[2] = {};
  int inNext = 0, outNext = 0, outLast = -1;
  int64_t chunkEls = 1;
  cudaError_t ensureAsync() {
    cudaError_t e;
    if (h2d) return cudaSuccess;
    const size_t perEl = size_t(std::max(9, 6 * cfg.n_rms)) * B * cfg.n_runs * realSize;
    chunkEls = std::max<int64_t>(1, std::min<int64_t>(nEl, int64_t(kChunkBytes / perEl)));
    for (int i = 0; i < kSlots; i++) {
      if ((e = cudaMalloc(&slotIn[i], chunkEls * perEl))) return e;
      for (cudaEvent_t *ev : {&evH2D[i], &evToRows[i]})
        if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming))) return e;
    }
    for (int i = 0; i < 2; i++) {
      if ((e = cudaMalloc(&bufOut[i], nEl * perEl))) return e;
      for (cudaEvent_t *ev : {&evFromRows[i], &evD2H[i]})
        if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming))) return e;
    }
    if ((e = cudaEventCreateWithFlags(&evMark, cudaEventDisableTiming))) return e;
    if ((e = cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking))) return e;
    return cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking);
  }
  cudaError_t uploadRowsAsync(void *rows, const void *host, int rowsPerEl) {
    cudaError_t e;
    const size_t refEl = size_t(rowsPerEl) * B * cfg.n_runs * realSize;
    const size_t rowEl = size_t(rowsPerEl) * cfg.n_runs * GB * realSize;
    for (int64_t e0 = 0; e0 < nEl; e0 += chunkEls) {
      const int64_t n = std::min(chunkEls, nEl - e0);
      const int k = inNext;
      inNext = (inNext + 1) % kSlots;
      // the slot is free once the layout kernel of its previous chunk read it
      if (toRowsPending[k] && (e = cudaStreamWaitEvent(h2d, evToRows[k], 0))) return e;
      if ((e = cudaMemcpyAsync(slotIn[k], static_cast<const char *>(host) + e0 * refEl, n * refEl,
                               cudaMemcpyHostToDevice, h2d)))
        return e;
      if ((e = cudaEventRecord(evH2D[k], h2d))) return e;
      if ((e = cudaStreamWaitEvent(stream, evH2D[k], 0))) return e;
      if ((e = convertLayout(true, cfg.precision, slotIn[k], static_cast<char *>(rows) + e0 * rowEl,
                             n * rowsPerEl, B, cfg.n_runs, GB, stream)))
        return e;
      toRowsPending[k] = true;
      if ((e = cudaEventRecord(evToRows[k], stream))) return e;
    }
    return cudaSuccess;
  }
  cudaError_t downloadRowsAsync(void *host, const void *rows, int rowsPerEl) {
    cudaError_t e;
    const int k = outNext;
    outNext ^= 1;
    // the buffer is free once its copy to the host from two downloads back finished
    if (d2hPending[k] && (e = cudaStreamWaitEvent(stream, evD2H[k], 0))) return e;
    if ((e = convertLayout(false, cfg.precision, rows, bufOut[k], nEl * rowsPerEl, B, cfg.n_runs, GB, stream)))
      return e;
    if ((e = cudaEventRecord(evFromRows[k], stream))) return e;
    if ((e = cudaStreamWaitEvent(d2h, evFromRows[k], 0))) return e;
    if ((e = cudaMemcpyAsync(host, bufOut[k], refCount(rowsPerEl) * realSize, cudaMemcpyDeviceToHost, d2h)))
      return e;
    d2hPending[k] = true;
    outLast = k;
    return cudaEventRecord(evD2H[k], d2h);
  }

  // runs the pending neighbour step of the last fused step
  cudaError_t flush() {
    if (!pending) return cudaSuccess;
    StepArgsRaw a = args(0);
    cudaError_t e = launch(1, [&] { return ks->neigh(a, stream); });
    if (e) return e;
    pending = false;
    return cudaSuccess;
  }

  // the flux-solver pairs of the pre-mixed projections, as characteristic factors for the steps of
  // a configuration whose kernels (GTS, or LTS for lts) mix through them (unless some face's pair is
  // not of rank 3, found when the factors are built: the pairs themselves from then on until the
  // element data changes), else as the pairs themselves
  cudaError_t ensureFsLR(bool lts = false) {
    if (!ks->premix()) return cudaSuccess;
    const bool wantChar = (lts ? ks->charMixLts() : ks->charMix()) && !charRejected;
    if (!fsLRStale && fsLRChar == wantChar) return cudaSuccess;
    const int P = ks->fsPairStride();
    cudaError_t e = fsLR.fit(size_t(nEl) * 4 * 2 * P * realSize);
    if (e) return e;
    if (wantChar) {
      // the count of faces whose pair is not of rank 3, read back once (no allocation or device-wide
      // synchronisation on the way: pools of a server set themselves up while others run)
      if ((e = charBad.fit(sizeof(int)))) return e;
      int *bad = charBad.as<int>();
      int nBad = 0;
      e = cudaMemsetAsync(bad, 0, sizeof(int), stream);
      if (!e) {
        const int grid = (int)std::min<int64_t>((nEl * 4 + 127) / 128, 148 * 8);
        if (cfg.precision == 64)
          kBuildFsChar<double><<<grid, 128, 0, stream>>>(fsE, elFaEl, fId, faType, nEl, P, fsLR.as<double>(), bad);
        else
          kBuildFsChar<float><<<grid, 128, 0, stream>>>(fsE, elFaEl, fId, faType, nEl, P, fsLR.as<float>(), bad);
        e = cudaGetLastError();
      }
      if (!e) e = cudaMemcpyAsync(&nBad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream);
      if (!e) e = cudaStreamSynchronize(stream);
      if (e) return e;
      if (nBad == 0) {
        fsLRStale = false;
        fsLRChar = true;
        return cudaSuccess;
      }
      charRejected = true;
    }
    const int64_t total = nEl * 4 * 2 * P;
    const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
    if (cfg.precision == 64)
      kBuildFsLR<double><<<grid, 256, 0, stream>>>(fsE, elFaEl, fId, faType, nEl, P, fsLR.as<double>());
    else
      kBuildFsLR<float><<<grid, 256, 0, stream>>>(fsE, elFaEl, fId, faType, nEl, P, fsLR.as<float>());
    if ((e = cudaGetLastError())) return e;
    fsLRStale = false;
    fsLRChar = false;
    return cudaSuccess;
  }

  int fail(cudaError_t e, const char *what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return EDGE_B200_EDEVICE;
  }
  StepArgsRaw args(double dt) const {
    StepArgsRaw a;
    a.dofsE = dofsE;
    a.dofsA = dofsA;
    a.tDofs = keepTDofs ? tDofs : nullptr;
    a.face = faceBuf(faceCur);
    a.starE = starE;
    a.starA = starA;
    a.srcA = srcA;
    a.fsE = fsE;
    a.fsA = fsA;
    a.elFaEl = elFaEl;
    a.fId = fId;
    a.vId = vId;
    a.faType = faType;
    a.fsLR = (ks->premix() && !fsLRStale) ? fsLR.p : nullptr;
    a.fsChar = (a.fsLR && fsLRChar) ? 1 : 0;
    a.grpDt = grpDtOn ? grpDt.as<double>() : nullptr;
    a.nEl = nEl;
    a.elFirst = 0;
    a.elCount = std::min(nOwned, nActive);
    a.dt = dt;
    for (int i = 0; i < 3; i++) a.omega[i] = omega[i];
    return a;
  }
  // element data borrowed from another context (edge_b200_share_element_data): not freed here
  bool sharedData = false;
  ~edge_b200_ctx() {
    dfree(dofsE); dfree(dofsA); dfree(tDofs); dfree(face);
    if (!sharedData) {
      dfree(starE); dfree(starA); dfree(srcA); dfree(fsE); dfree(fsA);
    }
    dfree(elFaEl); dfree(fId); dfree(vId); dfree(faType);
    dfree(dTau); dfree(dSlot); dfree(stage);
    for (int i = 0; i < kSlots; i++) dfree(slotIn[i]);
    for (int i = 0; i < 2; i++) dfree(bufOut[i]);
    if (h2d) cudaStreamSynchronize(h2d), cudaStreamDestroy(h2d);
    if (d2h) cudaStreamSynchronize(d2h), cudaStreamDestroy(d2h);
    for (int i = 0; i < kSlots; i++)
      for (cudaEvent_t ev : {evH2D[i], evToRows[i]})
        if (ev) cudaEventDestroy(ev);
    for (int i = 0; i < 2; i++)
      for (cudaEvent_t ev : {evFromRows[i], evD2H[i]})
        if (ev) cudaEventDestroy(ev);
    if (evMark) cudaEventDestroy(evMark);
    for (auto &t : timed) {
      cudaEventDestroy(t.a);
      cudaEventDestroy(t.b);
    }
    for (auto e : eventPool) cudaEventDestroy(e);
    delete ks;
  }
};

#define EDGE_CUDA(call, what)                 \
  do {                                        \
    cudaError_t e_ = (call);                  \
    if (e_ != cudaSuccess) return ctx->fail(e_, what); \
  } while (0)

template <typename P>
static cudaError_t upload(P *&dst, const void *src, size_t bytes, cudaStream_t s) {
  cudaError_t e;
  if (!dst && (e = cudaMalloc((void **)&dst, bytes ? bytes : 1))) return e;
  if (bytes && (e = cudaMemcpyAsync((void *)dst, src, bytes, cudaMemcpyHostToDevice, s))) return e;
  return cudaSuccess;
}

extern "C" {

int edge_b200_create(const edge_b200_cfg *cfg, int64_t n_el, edge_b200_ctx **out) {
  if (!cfg || !out || n_el < 1) return EDGE_B200_EINVAL;
  if (cfg->precision != 32 && cfg->precision != 64) return EDGE_B200_EINVAL;
  if (cfg->n_rms < 0 || cfg->n_rms > 3 || cfg->n_runs < 1 || 32 % cfg->n_runs) return EDGE_B200_EINVAL;
  KernelSet *ks = makeKernelSet(cfg->precision, cfg->order, cfg->n_runs, cfg->n_rms);
  if (!ks) return EDGE_B200_ENOTSUP;
  edge_b200_ctx *ctx = new (std::nothrow) edge_b200_ctx();
  if (!ctx) {
    delete ks;
    return EDGE_B200_ENOMEM;
  }
  ctx->cfg = *cfg;
  ctx->ks = ks;
  ctx->nEl = n_el;
  ctx->nOwned = n_el;
  ctx->B = nModes(cfg->order);
  ctx->F = nFaceModes(cfg->order);
  ctx->realSize = cfg->precision == 64 ? 8 : 4;
  ctx->GB = rowPad(ctx->B, cfg->precision);
  ctx->GF = rowPad(ctx->F, cfg->precision);
  ctx->stream = (cudaStream_t)cfg->stream;
  cudaError_t e;
  if ((e = cudaSetDevice(cfg->device)) != cudaSuccess || (e = ks->init(cfg->device)) != cudaSuccess) {
    delete ctx;
    return EDGE_B200_EDEVICE;
  }
  size_t rs = ctx->realSize;
  if ((e = cudaMalloc(&ctx->dofsE, ctx->dofsCount() * rs)) ||
      (cfg->n_rms && (e = cudaMalloc(&ctx->dofsA, ctx->dofsACount() * rs))) ||
      (e = cudaMalloc(&ctx->face, ctx->faceCount() * rs))) {
    delete ctx;
    return e == cudaErrorMemoryAllocation ? EDGE_B200_ENOMEM : EDGE_B200_EDEVICE;
  }
  cudaMemsetAsync(ctx->dofsE, 0, ctx->dofsCount() * rs, ctx->stream);
  if (cfg->n_rms) cudaMemsetAsync(ctx->dofsA, 0, ctx->dofsACount() * rs, ctx->stream);
  cudaMemsetAsync(ctx->face, 0, ctx->faceCount() * rs, ctx->stream);
  *out = ctx;
  return EDGE_B200_OK;
}

int edge_b200_destroy(edge_b200_ctx *ctx) {
  if (!ctx) return EDGE_B200_EINVAL;
  cudaStreamSynchronize(ctx->stream);
  delete ctx;
  return EDGE_B200_OK;
}

int edge_b200_upload_mesh(edge_b200_ctx *ctx, const int32_t *el_fa_el, const uint8_t *fid_el_fa_el,
                          const uint8_t *vid_el_fa_el, const uint8_t *el_fa_type) {
  if (!ctx || !el_fa_el || !fid_el_fa_el || !vid_el_fa_el || !el_fa_type) return EDGE_B200_EINVAL;
  const int64_t n = ctx->nEl * 4;
  for (int64_t i = 0; i < n; i++) {
    const int ty = el_fa_type[i];
    if (ty > EDGE_FACE_OUTFLOW) return EDGE_B200_EINVAL;
    if (ty == EDGE_FACE_INNER &&
        (el_fa_el[i] < 0 || el_fa_el[i] >= ctx->nEl || fid_el_fa_el[i] > 3 || vid_el_fa_el[i] > 2))
      return EDGE_B200_EMESH;
  }
  cudaStream_t s = ctx->stream;
  EDGE_CUDA(upload(ctx->elFaEl, el_fa_el, n * sizeof(int32_t), s), "upload elFaEl");
  EDGE_CUDA(upload(ctx->fId, fid_el_fa_el, n, s), "upload fId");
  EDGE_CUDA(upload(ctx->vId, vid_el_fa_el, n, s), "upload vId");
  EDGE_CUDA(upload(ctx->faType, el_fa_type, n, s), "upload faType");
  EDGE_CUDA(cudaStreamSynchronize(s), "upload mesh");
  ctx->hElFaEl.assign(el_fa_el, el_fa_el + n);
  ctx->hFId.assign(fid_el_fa_el, fid_el_fa_el + n);
  ctx->hFaType.assign(el_fa_type, el_fa_type + n);
  ctx->meshSet = true;
  ctx->fsLRStale = true;
  ctx->charRejected = false;
  return EDGE_B200_OK;
}

int edge_b200_upload_element_data(edge_b200_ctx *ctx, const double *star_e, const double *fs_e,
                                  const double *star_a, const double *src_a, const double *fs_a,
                                  const double *omega) {
  if (!ctx || !star_e || !fs_e) return EDGE_B200_EINVAL;
  const int rm = ctx->cfg.n_rms;
  if (rm && (!star_a || !src_a || !fs_a || !omega)) return EDGE_B200_EINVAL;
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->nEl;
  if (ctx->sharedData) {  // stop borrowing: this context gets arrays of its own
    ctx->starE = ctx->starA = ctx->srcA = ctx->fsE = ctx->fsA = nullptr;
    ctx->sharedData = false;
  }
  EDGE_CUDA(upload(ctx->starE, star_e, n * 72 * sizeof(double), s), "upload starE");
  EDGE_CUDA(upload(ctx->fsE, fs_e, n * 2 * 4 * 81 * sizeof(double), s), "upload fsE");
  if (rm) {
    EDGE_CUDA(upload(ctx->starA, star_a, n * 27 * sizeof(double), s), "upload starA");
    EDGE_CUDA(upload(ctx->srcA, src_a, n * rm * 12 * sizeof(double), s), "upload srcA");
    EDGE_CUDA(upload(ctx->fsA, fs_a, n * 2 * 4 * 54 * sizeof(double), s), "upload fsA");
    for (int m = 0; m < rm; m++) ctx->omega[m] = omega[m];
  }
  EDGE_CUDA(cudaStreamSynchronize(s), "upload element data");
  ctx->dataSet = true;
  ctx->fsLRStale = true;
  ctx->charRejected = false;
  return EDGE_B200_OK;
}

int edge_b200_share_element_data(edge_b200_ctx *dst, const edge_b200_ctx *src) {
  if (!dst || !src || dst == src || !src->dataSet) return EDGE_B200_EINVAL;
  if (dst->nEl != src->nEl || dst->cfg.n_rms != src->cfg.n_rms || dst->cfg.device != src->cfg.device)
    return EDGE_B200_EINVAL;
  edge_b200_ctx *ctx = dst;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  EDGE_CUDA(cudaStreamSynchronize(ctx->stream), "share element data");
  if (!ctx->sharedData) {
    dfree(ctx->starE); dfree(ctx->starA); dfree(ctx->srcA); dfree(ctx->fsE); dfree(ctx->fsA);
  }
  ctx->starE = src->starE;
  ctx->starA = src->starA;
  ctx->srcA = src->srcA;
  ctx->fsE = src->fsE;
  ctx->fsA = src->fsA;
  for (int m = 0; m < 3; m++) ctx->omega[m] = src->omega[m];
  ctx->sharedData = true;
  ctx->dataSet = true;
  ctx->fsLRStale = true;
  ctx->charRejected = false;
  return EDGE_B200_OK;
}

int edge_b200_upload_dofs(edge_b200_ctx *ctx, const void *dofs_e, const void *dofs_a) {
  if (!ctx || !dofs_e || (ctx->cfg.n_rms && !dofs_a)) return EDGE_B200_EINVAL;
  ctx->pending = false;  // the new DOFs replace the ones a pending neighbour step would complete
  EDGE_CUDA(ctx->uploadRows(ctx->dofsE, dofs_e, 9), "upload dofsE");
  if (ctx->cfg.n_rms) EDGE_CUDA(ctx->uploadRows(ctx->dofsA, dofs_a, 6 * ctx->cfg.n_rms), "upload dofsA");
  return EDGE_B200_OK;
}

int edge_b200_download_dofs(edge_b200_ctx *ctx, void *dofs_e, void *dofs_a) {
  if (!ctx || !dofs_e) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  EDGE_CUDA(ctx->downloadRows(dofs_e, ctx->dofsE, 9), "download dofsE");
  if (ctx->cfg.n_rms && dofs_a) EDGE_CUDA(ctx->downloadRows(dofs_a, ctx->dofsA, 6 * ctx->cfg.n_rms), "download dofsA");
  return EDGE_B200_OK;
}

int edge_b200_upload_dofs_async(edge_b200_ctx *ctx, const void *dofs_e, const void *dofs_a) {
  if (!ctx || !dofs_e || (ctx->cfg.n_rms && !dofs_a)) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->ensureAsync(), "async transfers");
  ctx->pending = false;
  EDGE_CUDA(ctx->uploadRowsAsync(ctx->dofsE, dofs_e, 9), "upload dofsE");
  if (ctx->cfg.n_rms) EDGE_CUDA(ctx->uploadRowsAsync(ctx->dofsA, dofs_a, 6 * ctx->cfg.n_rms), "upload dofsA");
  return EDGE_B200_OK;
}

int edge_b200_download_dofs_async(edge_b200_ctx *ctx, void *dofs_e, void *dofs_a) {
  if (!ctx || !dofs_e) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->ensureAsync(), "async transfers");
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  EDGE_CUDA(ctx->downloadRowsAsync(dofs_e, ctx->dofsE, 9), "download dofsE");
  if (ctx->cfg.n_rms && dofs_a)
    EDGE_CUDA(ctx->downloadRowsAsync(dofs_a, ctx->dofsA, 6 * ctx->cfg.n_rms), "download dofsA");
  return EDGE_B200_OK;
}

int edge_b200_join_transfers(edge_b200_ctx *ctx, int after_stream) {
  if (!ctx) return EDGE_B200_EINVAL;
  if (after_stream) {
    // the copy streams start after what the context stream holds now
    EDGE_CUDA(ctx->ensureAsync(), "join transfers");
    EDGE_CUDA(cudaEventRecord(ctx->evMark, ctx->stream), "join transfers");
    EDGE_CUDA(cudaStreamWaitEvent(ctx->h2d, ctx->evMark, 0), "join transfers");
    EDGE_CUDA(cudaStreamWaitEvent(ctx->d2h, ctx->evMark, 0), "join transfers");
  } else if (ctx->outLast >= 0) {
    // the copies to the host run in order on one stream: the last one covers the others
    EDGE_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->evD2H[ctx->outLast], 0), "join transfers");
  }
  return EDGE_B200_OK;
}

int edge_b200_set_run_dofs(edge_b200_ctx *ctx, int run, const void *dofs_e, const void *dofs_a) {
  if (!ctx || run < 0 || run >= ctx->cfg.n_runs) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  EDGE_CUDA(ctx->ensureStage(), "set run dofs");
  const int rm = ctx->cfg.n_rms;
  for (int part = 0; part < (rm ? 2 : 1); part++) {
    const void *src = part == 0 ? dofs_e : dofs_a;
    void *rows = part == 0 ? ctx->dofsE : ctx->dofsA;
    const int64_t nRows = ctx->nEl * (part == 0 ? 9 : 6 * rm);
    if (src)
      EDGE_CUDA(cudaMemcpyAsync(ctx->stage, src, nRows * ctx->B * ctx->realSize, cudaMemcpyHostToDevice,
                                ctx->stream), "set run dofs");
    const int64_t n = nRows * ctx->GB;
    const int grid = (int)((n + 255) / 256);
    if (ctx->cfg.precision == 64)
      kSetRun<double><<<grid, 256, 0, ctx->stream>>>((double *)rows, src ? (const double *)ctx->stage : nullptr,
                                                     nRows, ctx->B, ctx->cfg.n_runs, ctx->GB, run);
    else
      kSetRun<float><<<grid, 256, 0, ctx->stream>>>((float *)rows, src ? (const float *)ctx->stage : nullptr,
                                                    nRows, ctx->B, ctx->cfg.n_runs, ctx->GB, run);
    EDGE_CUDA(cudaGetLastError(), "set run dofs");
  }
  return EDGE_B200_OK;
}

int edge_b200_copy_run(edge_b200_ctx *dst, int dst_run, edge_b200_ctx *src, int src_run) {
  if (!dst || !src || dst_run < 0 || dst_run >= dst->cfg.n_runs || src_run < 0 || src_run >= src->cfg.n_runs)
    return EDGE_B200_EINVAL;
  if (dst->nEl != src->nEl || dst->cfg.order != src->cfg.order || dst->cfg.n_rms != src->cfg.n_rms ||
      dst->cfg.precision != src->cfg.precision || dst->cfg.device != src->cfg.device || dst->GB != src->GB)
    return EDGE_B200_EINVAL;
  if (dst == src && dst_run == src_run) return EDGE_B200_OK;
  edge_b200_ctx *ctx = dst;  // errors are recorded on the destination
  EDGE_CUDA(src->flush(), "pending neighbour step");
  EDGE_CUDA(dst->flush(), "pending neighbour step");
  // the source's stream reaches this point before the destination's copies start
  cudaEvent_t ev;
  EDGE_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "copy run");
  cudaError_t e = cudaEventRecord(ev, src->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(dst->stream, ev, 0);
  cudaEventDestroy(ev);
  EDGE_CUDA(e, "copy run");
  // one padded row [GB] per (element, quantity row) of the run: a strided 2D copy per DOF array
  const size_t row = (size_t)dst->GB * dst->realSize;
  for (int part = 0; part < (dst->cfg.n_rms ? 2 : 1); part++) {
    const int64_t nRows = dst->nEl * (part == 0 ? 9 : 6 * dst->cfg.n_rms);
    char *d = static_cast<char *>(part == 0 ? dst->dofsE : dst->dofsA) + dst_run * row;
    const char *sp = static_cast<const char *>(part == 0 ? src->dofsE : src->dofsA) + src_run * row;
    EDGE_CUDA(cudaMemcpy2DAsync(d, dst->cfg.n_runs * row, sp, src->cfg.n_runs * row, row, (size_t)nRows,
                                cudaMemcpyDeviceToDevice, dst->stream),
              "copy run");
  }
  return EDGE_B200_OK;
}

int edge_b200_keep_tdofs(edge_b200_ctx *ctx, int enable) {
  if (!ctx) return EDGE_B200_EINVAL;
  if (enable && !ctx->tDofs) {
    cudaError_t e = cudaMalloc(&ctx->tDofs, ctx->dofsCount() * ctx->realSize);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? EDGE_B200_ENOMEM : ctx->fail(e, "keep tDofs");
    EDGE_CUDA(cudaMemsetAsync(ctx->tDofs, 0, ctx->dofsCount() * ctx->realSize, ctx->stream), "keep tDofs");
  }
  ctx->keepTDofs = enable != 0;
  return EDGE_B200_OK;
}

int edge_b200_download_tdofs(edge_b200_ctx *ctx, void *tdofs) {
  if (!ctx || !tdofs || !ctx->tDofs) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->downloadRows(tdofs, ctx->tDofs, 9), "download tDofs");
  return EDGE_B200_OK;
}

int edge_b200_set_sources(edge_b200_ctx *ctx, int n, const int64_t *el, const int32_t *run,
                          const double *scal, const double *b_eval, const double *t0,
                          const double *dt, const int64_t *ts_off, const int64_t *n_pts,
                          int64_t n_ts, const double *ts) {
  if (!ctx || n < 0) return EDGE_B200_EINVAL;
  ctx->src = SrcArgs{};
  ctx->hSrcGrpEl.clear();
  ctx->nSrc = 0;
  ctx->srcClocks = false;  // clocks belong to a source list
  if (n == 0) return EDGE_B200_OK;
  if (!el || !run || !scal || !b_eval || !t0 || !dt || !ts_off || !n_pts || !ts) return EDGE_B200_EINVAL;
  std::vector<int32_t> off{0};
  for (int i = 0; i < n; i++) {
    if (el[i] < 0 || el[i] >= ctx->nEl || run[i] < 0 || run[i] >= ctx->cfg.n_runs || n_pts[i] < 1 ||
        ts_off[i] < 0 || ts_off[i] + n_pts[i] > n_ts || !(dt[i] > 0))
      return EDGE_B200_EINVAL;
    if (i > 0 && (el[i] < el[i - 1] || (el[i] == el[i - 1] && run[i] < run[i - 1]))) return EDGE_B200_EINVAL;
    if (i > 0 && (el[i] != el[i - 1] || run[i] != run[i - 1])) off.push_back(i);
  }
  off.push_back(n);
  cudaStream_t s = ctx->stream;
  const int B = ctx->B;
  DevBuf *m = ctx->srcMem;
  EDGE_CUDA(m[0].put(off.data(), off.size() * sizeof(int32_t), s), "sources");
  EDGE_CUDA(m[1].put(el, n * sizeof(int64_t), s), "sources");
  EDGE_CUDA(m[2].put(run, n * sizeof(int32_t), s), "sources");
  EDGE_CUDA(m[3].put(scal, n * 9 * sizeof(double), s), "sources");
  EDGE_CUDA(m[4].put(b_eval, (size_t)n * B * sizeof(double), s), "sources");
  EDGE_CUDA(m[5].put(t0, n * sizeof(double), s), "sources");
  EDGE_CUDA(m[6].put(dt, n * sizeof(double), s), "sources");
  EDGE_CUDA(m[7].put(ts_off, n * sizeof(int64_t), s), "sources");
  EDGE_CUDA(m[8].put(n_pts, n * sizeof(int64_t), s), "sources");
  EDGE_CUDA(m[9].put(ts, n_ts * sizeof(double), s), "sources");
  ctx->src.nGrp = (int)off.size() - 1;
  for (int g = 0; g + 1 < (int)off.size(); g++) ctx->hSrcGrpEl.push_back(el[off[g]]);
  ctx->src.grpOff = m[0].as<int32_t>();
  ctx->src.el = m[1].as<int64_t>();
  ctx->src.run = m[2].as<int32_t>();
  ctx->src.scal = m[3].as<double>();
  ctx->src.bEval = m[4].as<double>();
  ctx->src.t0 = m[5].as<double>();
  ctx->src.dts = m[6].as<double>();
  ctx->src.tsOff = m[7].as<int64_t>();
  ctx->src.nPts = m[8].as<int64_t>();
  ctx->src.ts = m[9].as<double>();
  ctx->src.tol = kTolTime;
  ctx->nSrc = n;
  EDGE_CUDA(cudaStreamSynchronize(s), "sources");
  return EDGE_B200_OK;
}

int edge_b200_set_source_clocks(edge_b200_ctx *ctx, const double *t0, const double *dt) {
  if (!ctx) return EDGE_B200_EINVAL;
  ctx->srcStep = 0;
  if (!t0 || !dt) {
    ctx->srcClocks = false;
    return EDGE_B200_OK;
  }
  const int n = ctx->nSrc;
  if (n == 0) return EDGE_B200_EINVAL;
  for (int i = 0; i < n; i++)
    if (!(dt[i] > 0)) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->srcClk0.put(t0, n * sizeof(double), ctx->stream), "source clocks");
  EDGE_CUDA(ctx->srcClkDt.put(dt, n * sizeof(double), ctx->stream), "source clocks");
  EDGE_CUDA(cudaStreamSynchronize(ctx->stream), "source clocks");
  ctx->srcClocks = true;
  return EDGE_B200_OK;
}

int edge_b200_set_active_elements(edge_b200_ctx *ctx, int64_t n_active) {
  if (!ctx || n_active < 0 || n_active > ctx->nEl || ctx->nTg > 1) return EDGE_B200_EINVAL;
  // the pending neighbour step of a fused call covers the old range
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  ctx->nActive = n_active;
  return EDGE_B200_OK;
}

int edge_b200_set_group_dt(edge_b200_ctx *ctx, const double *dt_group) {
  if (!ctx) return EDGE_B200_EINVAL;
  if (!dt_group) {
    ctx->grpDtOn = false;
    return EDGE_B200_OK;
  }
  if (ctx->nTg > 1) return EDGE_B200_EINVAL;  // GTS only
  const int64_t E = ctx->ks->elementsPerCta(), n = (ctx->nEl + E - 1) / E;
  for (int64_t g = 0; g < n; g++)
    if (!(dt_group[g] > 0)) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  EDGE_CUDA(ctx->grpDt.put(dt_group, n * sizeof(double), ctx->stream), "group time steps");
  EDGE_CUDA(cudaStreamSynchronize(ctx->stream), "group time steps");
  ctx->grpDtOn = true;
  return EDGE_B200_OK;
}

int edge_b200_set_receivers(edge_b200_ctx *ctx, int n, const int64_t *el, const double *basis,
                            double t_first, double period, int max_buf) {
  if (!ctx || n < 0) return EDGE_B200_EINVAL;
  ctx->nRecv = ctx->nRecvGrp = 0;
  if (n == 0) return EDGE_B200_OK;
  if (!el || !basis || !(period > 0) || max_buf < 1) return EDGE_B200_EINVAL;
  std::vector<int64_t> gEl;
  std::vector<int32_t> gOff;
  for (int i = 0; i < n; i++) {
    if (el[i] < 0 || el[i] >= ctx->nEl || (i > 0 && el[i] < el[i - 1])) return EDGE_B200_EINVAL;
    if (i == 0 || el[i] != el[i - 1]) {
      gEl.push_back(el[i]);
      gOff.push_back(i);
    }
  }
  gOff.push_back(n);
  cudaStream_t s = ctx->stream;
  EDGE_CUDA(ctx->grpEl.put(gEl.data(), gEl.size() * sizeof(int64_t), s), "receivers");
  EDGE_CUDA(ctx->grpOff.put(gOff.data(), gOff.size() * sizeof(int32_t), s), "receivers");
  EDGE_CUDA(ctx->basis.put(basis, (size_t)n * ctx->B * sizeof(double), s), "receivers");
  const size_t bufCount = (size_t)n * max_buf * 9 * ctx->cfg.n_runs;
  EDGE_CUDA(ctx->recvBuf.fit(bufCount * sizeof(double)), "receivers");
  EDGE_CUDA(cudaMemsetAsync(ctx->recvBuf.p, 0, bufCount * sizeof(double), s), "receivers");
  EDGE_CUDA(cudaStreamSynchronize(s), "receivers");
  ctx->nRecv = n;
  ctx->nRecvGrp = (int)gEl.size();
  ctx->maxBuf = max_buf;
  ctx->recvTime = t_first;
  ctx->period = period;
  ctx->recvCount = 0;
  ctx->hBufTime.assign(max_buf, 0.0);
  ctx->hRecvGrpEl = gEl;
  ctx->hRecvOff = gOff;
  ctx->tgRecvTime.assign(ctx->nTg, t_first);
  ctx->tgRecvCount.assign(ctx->nTg, 0);
  return EDGE_B200_OK;
}

int edge_b200_rewind_receivers(edge_b200_ctx *ctx, double t_first) {
  if (!ctx) return EDGE_B200_EINVAL;
  ctx->recvTime = t_first;
  ctx->recvCount = 0;
  std::fill(ctx->hBufTime.begin(), ctx->hBufTime.end(), 0.0);
  ctx->tgRecvTime.assign(ctx->nTg, t_first);
  ctx->tgRecvCount.assign(ctx->nTg, 0);
  return EDGE_B200_OK;
}

// n_steps GTS steps; phases selects the halves of each step (1: receivers, local, sources;
// 2: neighbour; 3: both)
static int runSteps(edge_b200_ctx *ctx, double t, double dt, int n_steps, int phases) {
  if (!ctx || !(dt > 0) || n_steps < 0) return EDGE_B200_EINVAL;
  if (!ctx->meshSet || !ctx->dataSet) return EDGE_B200_EINVAL;
  ctx->lastLts = false;
  cudaStream_t s = ctx->stream;
  EDGE_CUDA(ctx->ensureFsLR(), "flux-solver pairs");
  // whole GTS steps of a pre-mixing configuration without halo parts fold each neighbour step
  // into the next local step; the split phases run the neighbour step on its own
  const bool fused = phases == 3 && ctx->fusedOn && ctx->ks->fusedSupported() && ctx->nOwned == ctx->nEl;
  if (fused) {
    if (!ctx->faceAlt.p) {
      EDGE_CUDA(ctx->faceAlt.fit(ctx->faceCount() * ctx->realSize), "second face buffer");
      EDGE_CUDA(cudaMemsetAsync(ctx->faceAlt.p, 0, ctx->faceCount() * ctx->realSize, s), "second face buffer");
    }
  } else {
    EDGE_CUDA(ctx->flush(), "pending neighbour step");
  }
  // receiver samples of every step (Receivers::getRecvTimeRel, io/Receivers.cpp:235-248)
  std::vector<int> stepFirst(n_steps + 1, 0);
  std::vector<double> tau;
  std::vector<int32_t> slot;
  {
    double ts = t;
    for (int st = 0; st < n_steps; st++) {
      stepFirst[st] = (int)tau.size();
      if (ctx->nRecv && (phases & 1) && ctx->rangeRecv) {
        while (ctx->recvTime > ts - kTolTime && ctx->recvTime < ts + dt - kTolTime) {
          if (ctx->recvCount >= ctx->maxBuf) return EDGE_B200_EOVERFLOW;
          tau.push_back(std::abs(ctx->recvTime - ts));
          slot.push_back(ctx->recvCount);
          ctx->hBufTime[ctx->recvCount] = ctx->recvTime;
          ctx->recvCount++;
          ctx->recvTime += ctx->period;
        }
      }
      ts += dt;
    }
    stepFirst[n_steps] = (int)tau.size();
  }
  if (!tau.empty()) {
    if (tau.size() > ctx->tauCap) {
      dfree(ctx->dTau);
      dfree(ctx->dSlot);
      ctx->tauCap = std::max(tau.size(), (size_t)1024);
      EDGE_CUDA(cudaMalloc(&ctx->dTau, ctx->tauCap * sizeof(double)), "receiver schedule");
      EDGE_CUDA(cudaMalloc(&ctx->dSlot, ctx->tauCap * sizeof(int32_t)), "receiver schedule");
    }
    EDGE_CUDA(cudaMemcpyAsync(ctx->dTau, tau.data(), tau.size() * sizeof(double), cudaMemcpyHostToDevice, s),
              "receiver schedule");
    EDGE_CUDA(cudaMemcpyAsync(ctx->dSlot, slot.data(), slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s),
              "receiver schedule");
  }
  ctx->launches = 0;
  StepArgsRaw a = ctx->args(dt);
  if (ctx->rangeCount >= 0) {
    a.elFirst = ctx->rangeFirst;
    a.elCount = ctx->rangeCount;
  }
  double ts = t;
  for (int st = 0; st < n_steps; st++) {
    const int ns = stepFirst[st + 1] - stepFirst[st];
    if (fused) {
      // the previous step's projections (their neighbour step still pending) in, this step's out
      a.faceIn = ctx->pending ? ctx->faceBuf(ctx->faceCur) : nullptr;
      a.face = ctx->faceBuf(ctx->faceCur ^ 1);
    }
    if ((phases & 1) && ns > 0 && ctx->nRecvGrp > 0) {
      RecvArgs r;
      r.grpEl = ctx->grpEl.as<int64_t>();
      r.grpOff = ctx->grpOff.as<int32_t>();
      r.basis = ctx->basis.as<double>();
      r.tau = ctx->dTau + stepFirst[st];
      r.slot = ctx->dSlot + stepFirst[st];
      r.nSamples = ns;
      r.nGrp = ctx->nRecvGrp;
      r.maxBuf = ctx->maxBuf;
      r.buf = ctx->recvBuf.as<double>();
      EDGE_CUDA(ctx->launch(3, [&] { return ctx->ks->recv(a, r, s); }), "receiver kernel");
      ctx->launches++;
    }
    if (phases & 1) {
      EDGE_CUDA(ctx->launch(0, [&] { return fused ? ctx->ks->localFused(a, s) : ctx->ks->local(a, s); }),
                "local kernel");
      ctx->launches++;
      if (ctx->src.nGrp > 0 && ctx->rangeSrc) {
        SrcArgs sa = ctx->src;
        sa.t = ts;
        sa.elLimit = std::min(ctx->nOwned, ctx->nActive);
        if (ctx->srcClocks) {
          sa.clk0 = ctx->srcClk0.as<double>();
          sa.clkDt = ctx->srcClkDt.as<double>();
          sa.step = ctx->srcStep;
        }
        sa.dt = dt;
        EDGE_CUDA(ctx->launch(2, [&] { return ctx->ks->sources(ctx->dofsE, sa, s); }), "source kernel");
        ctx->launches++;
      }
    }
    if ((phases & 1) && ctx->rangeSrc) ctx->srcStep++;
    if (fused) {
      ctx->faceCur ^= 1;
      ctx->pending = true;
    } else if (phases & 2) {
      EDGE_CUDA(ctx->launch(1, [&] { return ctx->ks->neigh(a, s); }), "neighbour kernel");
      ctx->launches++;
    }
    ts += dt;
  }
  // the last step's neighbour step on its own: the DOFs are complete when the call returns
  if (fused && ctx->pending) {
    EDGE_CUDA(ctx->flush(), "neighbour kernel");
    ctx->launches++;
  }
  return EDGE_B200_OK;
}

int edge_b200_set_fused(edge_b200_ctx *ctx, int enable) {
  if (!ctx) return EDGE_B200_EINVAL;
  if (!enable) EDGE_CUDA(ctx->flush(), "pending neighbour step");
  ctx->fusedOn = enable != 0;
  return EDGE_B200_OK;
}

int edge_b200_step(edge_b200_ctx *ctx, double t, double dt, int n_steps) {
  return runSteps(ctx, t, dt, n_steps, 3);
}

int edge_b200_step_phase(edge_b200_ctx *ctx, double t, double dt, int phase) {
  if (!ctx || phase < 0 || phase > 3) return EDGE_B200_EINVAL;
  if (phase < 2) return runSteps(ctx, t, dt, 1, phase == 0 ? 1 : 2);
  // 2: receivers and local step of the send elements; 3: local step of the others and the sources
  const int64_t nSend = std::min(ctx->nSend, ctx->nOwned);
  ctx->rangeFirst = phase == 2 ? 0 : nSend;
  ctx->rangeCount = phase == 2 ? nSend : ctx->nOwned - nSend;
  ctx->rangeRecv = phase == 2;
  ctx->rangeSrc = phase == 3;
  const int rc = runSteps(ctx, t, dt, 1, 1);
  ctx->rangeCount = -1;
  ctx->rangeRecv = ctx->rangeSrc = true;
  return rc;
}

int edge_b200_set_send_count(edge_b200_ctx *ctx, int64_t n_send) {
  if (!ctx || n_send < 0 || n_send > ctx->nOwned) return EDGE_B200_EINVAL;
  ctx->nSend = n_send;
  return EDGE_B200_OK;
}

int edge_b200_set_owned(edge_b200_ctx *ctx, int64_t n_owned) {
  if (!ctx || n_owned < 0 || n_owned > ctx->nEl || ctx->nTg > 1) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  ctx->nOwned = n_owned;
  return EDGE_B200_OK;
}

int64_t edge_b200_face_block_bytes(const edge_b200_ctx *ctx) {
  return ctx ? (int64_t)9 * ctx->cfg.n_runs * ctx->GF * (int64_t)ctx->realSize : -1;
}

static int packFaces(edge_b200_ctx *ctx, int n, const int32_t *slots, void *buf, bool pack) {
  if (!ctx || n < 0 || (n && (!slots || !buf))) return EDGE_B200_EINVAL;
  if (n == 0) return EDGE_B200_OK;
  const int64_t blk16 = edge_b200_face_block_bytes(ctx) / 16;
  const int64_t total = (int64_t)n * blk16;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  kFacePack<<<grid, 256, 0, ctx->stream>>>(static_cast<uint4 *>(ctx->faceBuf(ctx->faceCur)), static_cast<uint4 *>(buf), slots,
                                             n, blk16, ctx->nEl * 4, pack);
  EDGE_CUDA(cudaGetLastError(), pack ? "pack faces" : "unpack faces");
  return EDGE_B200_OK;
}

int edge_b200_pack_faces(edge_b200_ctx *ctx, int n, const int32_t *slots, void *out) {
  return packFaces(ctx, n, slots, out, true);
}

int edge_b200_unpack_faces(edge_b200_ctx *ctx, int n, const int32_t *slots, const void *in) {
  return packFaces(ctx, n, slots, const_cast<void *>(in), false);
}

int edge_b200_set_time_groups(edge_b200_ctx *ctx, int n_groups, const int64_t *group_first) {
  if (!ctx || !ctx->meshSet || n_groups < 1 || n_groups > 16 || !group_first) return EDGE_B200_EINVAL;
  if (ctx->nOwned != ctx->nEl || ctx->nActive < ctx->nEl) return EDGE_B200_EINVAL;  // time groups cover the whole mesh
  if (group_first[0] != 0 || group_first[n_groups] != ctx->nEl) return EDGE_B200_EINVAL;
  for (int g = 0; g < n_groups; g++)
    if (group_first[g + 1] < group_first[g]) return EDGE_B200_EINVAL;
  if (n_groups > 1 && !ctx->ks->ltsSupported()) return EDGE_B200_ENOTSUP;
  const int64_t nEl = ctx->nEl;
  std::vector<uint8_t> grp(nEl);
  for (int g = 0; g < n_groups; g++)
    for (int64_t e = group_first[g]; e < group_first[g + 1]; e++) grp[e] = (uint8_t)g;
  // relation per inner face (rate 2: face neighbours differ by at most one group), element flags
  std::vector<uint8_t> rel(4 * nEl, LTS_EQ), flags(nEl, 0);
  for (int64_t e = 0; e < nEl; e++)
    for (int f = 0; f < 4; f++) {
      if (ctx->hFaType[4 * e + f] != EDGE_FACE_INNER) continue;
      const int64_t ne = ctx->hElFaEl[4 * e + f];
      const int d = int(grp[e]) - int(grp[ne]);
      if (d > 1 || d < -1) return EDGE_B200_EINVAL;
      rel[4 * e + f] = d > 0 ? LTS_GT : d < 0 ? LTS_LT : LTS_EQ;
      if (d < 0) flags[e] |= LTS_HAS_LARGER;
      if (d > 0) flags[e] |= LTS_HAS_SMALLER;
    }
  std::vector<int32_t> sIdx(nEl, -1), hIdx(nEl, -1);
  int32_t nSum = 0, nHalf = 0;
  for (int64_t e = 0; e < nEl; e++) {
    if (flags[e] & LTS_HAS_LARGER) sIdx[e] = nSum++;
    if (flags[e] & LTS_HAS_SMALLER) hIdx[e] = nHalf++;
  }
  cudaStream_t s = ctx->stream;
  const size_t slotBytes = (size_t)4 * 9 * ctx->cfg.n_runs * ctx->GF * ctx->realSize;
  EDGE_CUDA(ctx->ltsFlags.put(flags.data(), flags.size(), s), "time groups");
  EDGE_CUDA(ctx->ltsRel.put(rel.data(), rel.size(), s), "time groups");
  EDGE_CUDA(ctx->sumIdx.put(sIdx.data(), sIdx.size() * sizeof(int32_t), s), "time groups");
  EDGE_CUDA(ctx->halfIdx.put(hIdx.data(), hIdx.size() * sizeof(int32_t), s), "time groups");
  EDGE_CUDA(ctx->faceSum.fit(std::max<size_t>(nSum * slotBytes, 16)), "time groups");
  EDGE_CUDA(ctx->faceHalf1.fit(std::max<size_t>(nHalf * slotBytes, 16)), "time groups");
  EDGE_CUDA(ctx->faceHalf2.fit(std::max<size_t>(nHalf * slotBytes, 16)), "time groups");
  EDGE_CUDA(cudaMemsetAsync(ctx->faceSum.p, 0, nSum * slotBytes, s), "time groups");
  EDGE_CUDA(cudaMemsetAsync(ctx->faceHalf1.p, 0, nHalf * slotBytes, s), "time groups");
  EDGE_CUDA(cudaMemsetAsync(ctx->faceHalf2.p, 0, nHalf * slotBytes, s), "time groups");
  EDGE_CUDA(cudaStreamSynchronize(s), "time groups");
  ctx->nTg = n_groups;
  ctx->tgFirst.assign(group_first, group_first + n_groups + 1);
  // the local step needs the half-step tile only up to the last element with a smaller neighbour
  // of each group (a group sorted with those elements first keeps the rest on the faster kernel)
  ctx->tgHalfEnd.assign(n_groups, 0);
  for (int g = 0; g < n_groups; g++) {
    int64_t end = group_first[g];
    for (int64_t e = group_first[g]; e < group_first[g + 1]; e++)
      if (flags[e] & LTS_HAS_SMALLER) end = e + 1;
    ctx->tgHalfEnd[g] = end;
  }
  ctx->tgRecvTime.assign(n_groups, ctx->recvTime);
  ctx->tgRecvCount.assign(n_groups, ctx->recvCount);
  return EDGE_B200_OK;
}

int edge_b200_step_lts(edge_b200_ctx *ctx, double t, double dt_fun, int n_cycles) {
  if (!ctx || !(dt_fun > 0) || n_cycles < 0 || ctx->nTg < 1) return EDGE_B200_EINVAL;
  if (!ctx->meshSet || !ctx->dataSet) return EDGE_B200_EINVAL;
  if (!ctx->ks->ltsSupported()) return EDGE_B200_ENOTSUP;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  EDGE_CUDA(ctx->ensureFsLR(true), "flux-solver pairs");
  ctx->lastLts = true;
  const int G = ctx->nTg;
  const int64_t nFun = int64_t(1) << (G - 1);  // fundamental steps per cycle (largest group's step)
  cudaStream_t s = ctx->stream;
  // the work regions of the call, in the order of the rate-2 schedule: at fundamental step k the
  // groups starting a step (k % 2^g == 0) run local + sources, then the groups ending one
  // ((k+1) % 2^g == 0) run neigh (TimeGroupStatic / man_sched.inc dependencies, sequentialised)
  struct Work { int kind, g, firstTs; double t, dt; int s0, s1; };
  std::vector<Work> work;
  std::vector<double> tau;
  std::vector<int32_t> slot;
  // receiver groups and source groups of each time group (both sorted by element)
  std::vector<int> rB(G), rE(G), sB(G), sE(G);
  for (int g = 0; g < G; g++) {
    auto lo = ctx->tgFirst[g], hi = ctx->tgFirst[g + 1];
    rB[g] = int(std::lower_bound(ctx->hRecvGrpEl.begin(), ctx->hRecvGrpEl.end(), lo) - ctx->hRecvGrpEl.begin());
    rE[g] = int(std::lower_bound(ctx->hRecvGrpEl.begin(), ctx->hRecvGrpEl.end(), hi) - ctx->hRecvGrpEl.begin());
    sB[g] = int(std::lower_bound(ctx->hSrcGrpEl.begin(), ctx->hSrcGrpEl.end(), lo) - ctx->hSrcGrpEl.begin());
    sE[g] = int(std::lower_bound(ctx->hSrcGrpEl.begin(), ctx->hSrcGrpEl.end(), hi) - ctx->hSrcGrpEl.begin());
  }
  for (int64_t c = 0; c < n_cycles; c++)
    for (int64_t k = 0; k < nFun; k++) {
      const int64_t kk = c * nFun + k;  // fundamental step since t
      for (int g = 0; g < G; g++) {
        if (k % (int64_t(1) << g)) continue;
        const double tg = t + double(kk) * dt_fun, dtg = dt_fun * double(int64_t(1) << g);
        const int firstTs = ((kk >> g) & 1) == 0;
        Work w{0, g, firstTs, tg, dtg, (int)tau.size(), 0};
        if (ctx->nRecv && rE[g] > rB[g]) {
          double &rt = ctx->tgRecvTime[g];
          int32_t &rc = ctx->tgRecvCount[g];
          while (rt > tg - kTolTime && rt < tg + dtg - kTolTime) {
            if (rc >= ctx->maxBuf) return EDGE_B200_EOVERFLOW;
            tau.push_back(std::abs(rt - tg));
            slot.push_back(rc);
            ctx->hBufTime[rc] = rt;
            rc++;
            rt += ctx->period;
          }
        }
        w.s1 = (int)tau.size();
        work.push_back(w);
      }
      for (int g = 0; g < G; g++) {
        const int64_t span = int64_t(1) << g;
        if ((k + 1) % span) continue;
        const int64_t k0 = kk + 1 - span;  // the step that ends now started at k0
        work.push_back(Work{1, g, ((k0 >> g) & 1) == 0, t + double(k0) * dt_fun, dt_fun * double(span), 0, 0});
      }
    }
  if (!tau.empty()) {
    if (tau.size() > ctx->tauCap) {
      dfree(ctx->dTau);
      dfree(ctx->dSlot);
      ctx->tauCap = std::max(tau.size(), (size_t)1024);
      EDGE_CUDA(cudaMalloc(&ctx->dTau, ctx->tauCap * sizeof(double)), "receiver schedule");
      EDGE_CUDA(cudaMalloc(&ctx->dSlot, ctx->tauCap * sizeof(int32_t)), "receiver schedule");
    }
    EDGE_CUDA(cudaMemcpyAsync(ctx->dTau, tau.data(), tau.size() * sizeof(double), cudaMemcpyHostToDevice, s),
              "receiver schedule");
    EDGE_CUDA(cudaMemcpyAsync(ctx->dSlot, slot.data(), slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s),
              "receiver schedule");
  }
  ctx->launches = 0;
  for (const Work &w : work) {
    StepArgsRaw a = ctx->args(w.dt);
    a.elFirst = ctx->tgFirst[w.g];
    a.elCount = ctx->tgFirst[w.g + 1] - ctx->tgFirst[w.g];
    a.faceSum = ctx->faceSum.p;
    a.faceHalf1 = ctx->faceHalf1.p;
    a.faceHalf2 = ctx->faceHalf2.p;
    a.ltsFlags = ctx->ltsFlags.as<uint8_t>();
    a.ltsRel = ctx->ltsRel.as<uint8_t>();
    a.sumIdx = ctx->sumIdx.as<int32_t>();
    a.halfIdx = ctx->halfIdx.as<int32_t>();
    a.firstTs = w.firstTs;
    if (a.elCount == 0) continue;
    if (w.kind == 0) {
      const int ns = w.s1 - w.s0;
      if (ns > 0) {
        RecvArgs r;
        r.grpEl = ctx->grpEl.as<int64_t>() + rB[w.g];
        r.grpOff = ctx->grpOff.as<int32_t>() + rB[w.g];
        r.basis = ctx->basis.as<double>();
        r.tau = ctx->dTau + w.s0;
        r.slot = ctx->dSlot + w.s0;
        r.nSamples = ns;
        r.nGrp = rE[w.g] - rB[w.g];
        r.maxBuf = ctx->maxBuf;
        r.buf = ctx->recvBuf.as<double>();
        EDGE_CUDA(ctx->launch(3, [&] { return ctx->ks->recv(a, r, s); }), "receiver kernel");
        ctx->launches++;
      }
      StepArgsRaw aHalf = a, aSums = a;
      aHalf.elCount = ctx->tgHalfEnd[w.g] - a.elFirst;
      aSums.elFirst = ctx->tgHalfEnd[w.g];
      aSums.elCount = a.elFirst + a.elCount - aSums.elFirst;
      if (aHalf.elCount > 0) {
        EDGE_CUDA(ctx->launch(0, [&] { return ctx->ks->localLts(aHalf, s); }), "local kernel");
        ctx->launches++;
      }
      if (aSums.elCount > 0) {
        EDGE_CUDA(ctx->launch(0, [&] { return ctx->ks->localLtsSums(aSums, s); }), "local kernel");
        ctx->launches++;
      }
      if (sE[w.g] > sB[w.g]) {
        SrcArgs sa = ctx->src;
        sa.grpOff += sB[w.g];
        sa.nGrp = sE[w.g] - sB[w.g];
        sa.t = w.t;
        sa.dt = w.dt;
        EDGE_CUDA(ctx->launch(2, [&] { return ctx->ks->sources(ctx->dofsE, sa, s); }), "source kernel");
        ctx->launches++;
      }
    } else {
      EDGE_CUDA(ctx->launch(1, [&] { return ctx->ks->neighLts(a, s); }), "neighbour kernel");
      ctx->launches++;
    }
  }
  return EDGE_B200_OK;
}

int edge_b200_read_receivers(edge_b200_ctx *ctx, double *buf, double *buf_time, int32_t *counts) {
  if (!ctx) return EDGE_B200_EINVAL;
  if (ctx->nRecv == 0) return EDGE_B200_OK;
  const size_t bufCount = (size_t)ctx->nRecv * ctx->maxBuf * 9 * ctx->cfg.n_runs;
  if (buf)
    EDGE_CUDA(cudaMemcpyAsync(buf, ctx->recvBuf.p, bufCount * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
              "read receivers");
  EDGE_CUDA(cudaStreamSynchronize(ctx->stream), "read receivers");
  for (int gi = 0; gi < ctx->nRecvGrp; gi++) {
    const int64_t el = ctx->hRecvGrpEl[gi];
    // receivers of one element share its group's clock (the GTS clock without time groups)
    const int32_t cnt = ctx->lastLts ? ctx->tgRecvCount[ctx->groupOf(el)] : ctx->recvCount;
    for (int i = ctx->hRecvOff[gi]; i < ctx->hRecvOff[gi + 1]; i++) {
      if (counts) counts[i] = cnt;
      if (buf_time)
        for (int j = 0; j < ctx->maxBuf; j++) buf_time[(size_t)i * ctx->maxBuf + j] = j < cnt ? ctx->hBufTime[j] : 0.0;
    }
  }
  return EDGE_B200_OK;
}

int edge_b200_upload_geometry(edge_b200_ctx *ctx, const double *el_ve_crds) {
  if (!ctx || !el_ve_crds) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->geom.put(el_ve_crds, (size_t)ctx->nEl * 12 * sizeof(double), ctx->stream), "upload geometry");
  EDGE_CUDA(cudaStreamSynchronize(ctx->stream), "upload geometry");
  return EDGE_B200_OK;
}

int edge_b200_error_norms(edge_b200_ctx *ctx, double t, int n_waves, const double *waves, int n_qp,
                          const double *qp_xi, const double *qp_w, const double *qp_basis, double *l1, double *l2,
                          double *linf) {
  if (!ctx || !ctx->geom.p || n_waves < 0 || n_waves > 64 || (n_waves && !waves) || n_qp < 1 || n_qp > 512 ||
      !qp_xi || !qp_w || !qp_basis || ctx->B > 64)
    return EDGE_B200_EINVAL;
  const int B = ctx->B, R = ctx->cfg.n_runs;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  std::vector<PlaneWave> pw(std::max(n_waves, 1));
  for (int w = 0; w < n_waves; w++) {
    const double *src = waves + 15 * w;  // k[3], omega, phase, amp[9], run
    for (int d = 0; d < 3; d++) pw[w].k[d] = src[d];
    pw[w].omega = src[3];
    pw[w].phase = src[4];
    for (int q = 0; q < 9; q++) pw[w].amp[q] = src[5 + q];
    pw[w].run = (int)src[14];
    if (pw[w].run >= R) return EDGE_B200_EINVAL;
  }
  std::vector<double> quad((size_t)n_qp * (4 + B));
  for (int k = 0; k < n_qp; k++) {
    double *d = &quad[(size_t)k * (4 + B)];
    for (int i = 0; i < 3; i++) d[i] = qp_xi[3 * k + i];
    d[3] = qp_w[k];
    for (int b = 0; b < B; b++) d[4 + b] = qp_basis[(size_t)k * B + b];
  }
  cudaStream_t s = ctx->stream;
  const size_t smem = quad.size() * sizeof(double);
  if (smem > 200 * 1024) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->waves.put(pw.data(), pw.size() * sizeof(PlaneWave), s), "error norms");
  EDGE_CUDA(ctx->quad.put(quad.data(), smem, s), "error norms");
  EDGE_CUDA(ctx->norms.fit(27 * R * sizeof(double)), "error norms");
  EDGE_CUDA(cudaMemsetAsync(ctx->norms.p, 0, 27 * R * sizeof(double), s), "error norms");
  const int threads = ((9 * R + 31) / 32) * 32;
  const int grid = (int)std::min<int64_t>(ctx->nEl, 148 * 8);
  if (ctx->cfg.precision == 64) {
    EDGE_CUDA(cudaFuncSetAttribute(kErrorNorms<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
              "error norms");
    kErrorNorms<double><<<grid, threads, smem, s>>>((const double *)ctx->dofsE, ctx->geom.as<double>(), ctx->nOwned,
                                                    B, R, ctx->GB, n_qp, ctx->quad.as<double>(),
                                                    ctx->waves.as<PlaneWave>(), n_waves, t, ctx->norms.as<double>());
  } else {
    EDGE_CUDA(cudaFuncSetAttribute(kErrorNorms<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
              "error norms");
    kErrorNorms<float><<<grid, threads, smem, s>>>((const float *)ctx->dofsE, ctx->geom.as<double>(), ctx->nOwned,
                                                   B, R, ctx->GB, n_qp, ctx->quad.as<double>(),
                                                   ctx->waves.as<PlaneWave>(), n_waves, t, ctx->norms.as<double>());
  }
  EDGE_CUDA(cudaGetLastError(), "error norms");
  std::vector<double> h(27 * R);
  EDGE_CUDA(cudaMemcpyAsync(h.data(), ctx->norms.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s),
            "error norms");
  EDGE_CUDA(cudaStreamSynchronize(s), "error norms");
  for (int i = 0; i < 9 * R; i++) {
    if (l1) l1[i] = h[i];
    if (l2) l2[i] = std::sqrt(h[9 * R + i]);
    if (linf) linf[i] = h[18 * R + i];
  }
  return EDGE_B200_OK;
}

int edge_b200_wavefield(edge_b200_ctx *ctx, float *out) {
  if (!ctx || !out) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  const size_t n = (size_t)ctx->nEl * 9 * ctx->cfg.n_runs;
  cudaStream_t s = ctx->stream;
  EDGE_CUDA(ctx->norms.fit(n * sizeof(float)), "wave field");
  const int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  if (ctx->cfg.precision == 64)
    kWaveField<double><<<grid, 256, 0, s>>>((const double *)ctx->dofsE, ctx->nEl, ctx->cfg.n_runs, ctx->GB,
                                            ctx->norms.as<float>());
  else
    kWaveField<float><<<grid, 256, 0, s>>>((const float *)ctx->dofsE, ctx->nEl, ctx->cfg.n_runs, ctx->GB,
                                           ctx->norms.as<float>());
  EDGE_CUDA(cudaGetLastError(), "wave field");
  EDGE_CUDA(cudaMemcpyAsync(out, ctx->norms.p, n * sizeof(float), cudaMemcpyDeviceToHost, s), "wave field");
  EDGE_CUDA(cudaStreamSynchronize(s), "wave field");
  return EDGE_B200_OK;
}

int edge_b200_sync(edge_b200_ctx *ctx) {
  if (!ctx) return EDGE_B200_EINVAL;
  if (ctx->h2d) EDGE_CUDA(cudaStreamSynchronize(ctx->h2d), "sync");
  if (ctx->d2h) EDGE_CUDA(cudaStreamSynchronize(ctx->d2h), "sync");
  EDGE_CUDA(cudaStreamSynchronize(ctx->stream), "sync");
  return EDGE_B200_OK;
}

int edge_b200_device_dofs(edge_b200_ctx *ctx, void **dofs_e, void **dofs_a, void **tdofs) {
  if (!ctx) return EDGE_B200_EINVAL;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  if (dofs_e) *dofs_e = ctx->dofsE;
  if (dofs_a) *dofs_a = ctx->dofsA;
  if (tdofs) *tdofs = ctx->tDofs;
  return EDGE_B200_OK;
}

int64_t edge_b200_last_launches(const edge_b200_ctx *ctx) { return ctx ? ctx->launches : -1; }

int edge_b200_kernel_config(const edge_b200_ctx *ctx, int32_t info[6]) {
  if (!ctx || !info) return EDGE_B200_EINVAL;
  info[5] = (ctx->fusedOn && ctx->ks->fusedSupported() && ctx->nOwned == ctx->nEl) ? 1 : 0;
  info[0] = ctx->ks->elementsPerCta();
  info[1] = ctx->ks->premix() ? ((ctx->ks->charMix() && !ctx->charRejected) ? 2 : 1) : 0;
  info[2] = ctx->ks->fsPairStride();
  info[3] = ctx->ks->ctasLocal();
  info[4] = ctx->ks->ctasNeigh();
  return EDGE_B200_OK;
}

int edge_b200_set_timing(edge_b200_ctx *ctx, int enable) {
  if (!ctx) return EDGE_B200_EINVAL;
  ctx->resolveTimes();
  ctx->timing = enable != 0;
  for (int i = 0; i < 4; i++) {
    ctx->kernMs[i] = 0;
    ctx->kernN[i] = 0;
  }
  return EDGE_B200_OK;
}

int edge_b200_kernel_times(edge_b200_ctx *ctx, double *ms, int64_t *launches) {
  if (!ctx) return EDGE_B200_EINVAL;
  ctx->resolveTimes();
  for (int i = 0; i < 4; i++) {
    if (ms) ms[i] = ctx->kernMs[i];
    if (launches) launches[i] = ctx->kernN[i];
  }
  return EDGE_B200_OK;
}

const char *edge_b200_last_error(const edge_b200_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// batches of contexts stepped together through one captured CUDA graph, and the launch-shape
// autotuner
// ------------------------------------------------------------------------------------------------
namespace {
__global__ void kAdvanceSteps(int64_t *steps, const int32_t *active, int n, int by) {
  for (int k = threadIdx.x; k < n; k += blockDim.x)
    if (active[k]) steps[k] += by;
}
}  // namespace

struct edge_b200_batch {
  std::vector<edge_b200_ctx *> ctxs;
  std::vector<double> t0, dt;
  std::vector<int32_t> active;
  std::vector<cudaStream_t> streams;  // one per context, forked from `origin` inside the capture
  std::vector<cudaEvent_t> joins;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr;
  int64_t *steps = nullptr;    // device: steps taken per context
  int32_t *activeDev = nullptr;
  cudaGraphExec_t exec = nullptr;  // two batch steps
  std::vector<char> fu;            // per context: fused steps, fixed when the graph is captured
  bool dirty = true;
  std::string err;
  ~edge_b200_batch() {
    if (origin) cudaStreamSynchronize(origin);
    if (exec) cudaGraphExecDestroy(exec);
    for (cudaStream_t s : streams)
      if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : joins)
      if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (origin) cudaStreamDestroy(origin);
    dfree(steps);
    dfree(activeDev);
  }
  // contexts whose GTS steps fold each neighbour step into the next local step (as edge_b200_step
  // does): within a call their steps alternate between the two face buffers
  static bool fused(const edge_b200_ctx *c) { return c->fusedOn && c->ks->fusedSupported(); }
  // one GTS step of context k on its stream, its sources at t0 + tOff + steps[k] * dt. kind 0: a
  // call's first step (fused contexts: nothing pending, projections out to faceAlt); 1: fused,
  // pending projections in faceAlt, out to face; 2: in face, out to faceAlt. Other contexts take
  // a whole separate-kernel step (local, sources, neighbour) in each kind.
  cudaError_t issueStep(size_t k, int kind, double tOff) {
    edge_b200_ctx *ctx = ctxs[k];
    cudaStream_t s = streams[k];
    StepArgsRaw a = ctx->args(dt[k]);
    cudaError_t c;
    if (fu[k]) {
      a.faceIn = kind == 0 ? nullptr : ctx->faceBuf(kind == 1 ? 1 : 0);
      a.face = ctx->faceBuf(kind == 1 ? 0 : 1);
      c = ctx->ks->localFused(a, s);
    } else {
      c = ctx->ks->local(a, s);
    }
    if (c) return c;
    if (ctx->src.nGrp > 0) {
      SrcArgs sa = ctx->src;
      sa.t = t0[k] + tOff;
      if (ctx->srcClocks) {
        sa.clk0 = ctx->srcClk0.as<double>();
        sa.clkDt = ctx->srcClkDt.as<double>();
      }
      sa.dt = dt[k];
      sa.stepDev = steps + k;
      if ((c = ctx->ks->sources(ctx->dofsE, sa, s))) return c;
    }
    return fu[k] ? cudaSuccess : ctx->ks->neigh(a, s);
  }
  // body(k) on every active context's stream, forked from and joined back into `origin`
  template <class F>
  cudaError_t forkJoin(F body) {
    cudaError_t c = cudaEventRecord(fork, origin);
    for (size_t k = 0; k < ctxs.size() && !c; k++) {
      if (!active[k]) continue;
      cudaStream_t s = streams[k];
      if ((c = cudaStreamWaitEvent(s, fork, 0))) break;
      if ((c = body(k))) break;
      if ((c = cudaEventRecord(joins[k], s))) break;
      c = cudaStreamWaitEvent(origin, joins[k], 0);
    }
    return c;
  }
  cudaError_t advance(int by) {
    kAdvanceSteps<<<1, 256, 0, origin>>>(steps, activeDev, (int)ctxs.size(), by);
    return cudaGetLastError();
  }
  // the replayed unit: two GTS steps of every active context (fused ones: kinds 1 then 2, which
  // leaves the pending projections where they were), each context on its own stream
  cudaError_t capture() {
    cudaError_t e;
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    if ((e = cudaMemcpyAsync(activeDev, active.data(), active.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                             origin)))
      return e;
    if ((e = cudaStreamSynchronize(origin))) return e;
    // each context's step form for this graph and the direct launches around it (a context switched
    // to fused steps after the batch was created, without its second face buffer, stays separate)
    fu.assign(ctxs.size(), 0);
    for (size_t k = 0; k < ctxs.size(); k++) fu[k] = fused(ctxs[k]) && ctxs[k]->faceAlt.p != nullptr;
    if ((e = cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal))) return e;
    cudaError_t c = forkJoin([&](size_t k) {
      cudaError_t r = issueStep(k, 1, 0.0);
      return r ? r : issueStep(k, 2, dt[k]);
    });
    if (!c) c = advance(2);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(origin, &graph);
    if (c) {
      if (graph) cudaGraphDestroy(graph);
      return c;
    }
    if (e) return e;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e) return e;
    dirty = false;
    return cudaSuccess;
  }
  // n GTS steps of every active context: the first launched directly (kind 0), then pairs by
  // graph, an odd one left directly (kind 1), then the fused contexts' last neighbour step, so
  // that nothing is pending when the call returns
  cudaError_t run(int n) {
    cudaError_t c;
    if (dirty && (c = capture())) return c;
    for (size_t k = 0; k < ctxs.size(); k++)
      if (active[k] && fu[k]) ctxs[k]->faceCur = 0;  // nothing pending: only a relabelling
    if ((c = forkJoin([&](size_t k) { return issueStep(k, 0, 0.0); }))) return c;
    if ((c = advance(1))) return c;
    for (int i = 0; i < (n - 1) / 2; i++)
      if ((c = cudaGraphLaunch(exec, origin))) return c;
    const bool odd = (n - 1) % 2 == 1;
    if (odd) {
      if ((c = forkJoin([&](size_t k) { return issueStep(k, 1, 0.0); }))) return c;
      if ((c = advance(1))) return c;
    }
    // last written: faceAlt after kinds 0 and 2, face after kind 1
    const int last = odd ? 0 : 1;
    c = forkJoin([&](size_t k) {
      edge_b200_ctx *ctx = ctxs[k];
      if (!fu[k]) return cudaSuccess;
      StepArgsRaw a = ctx->args(dt[k]);
      a.face = ctx->faceBuf(last);
      return ctx->ks->neigh(a, streams[k]);
    });
    if (c) return c;
    for (size_t k = 0; k < ctxs.size(); k++)
      if (active[k] && fu[k]) ctxs[k]->faceCur = last;
    return cudaSuccess;
  }
};

#define EDGE_BATCH_CUDA(call, what)                                 \
  do {                                                              \
    cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) {                                        \
      b->err = std::string(what) + ": " + cudaGetErrorString(e_);   \
      return EDGE_B200_EDEVICE;                                     \
    }                                                               \
  } while (0)

int edge_b200_batch_create(edge_b200_ctx *const *ctxs, int n, const double *t0, const double *dt,
                           edge_b200_batch **out) {
  if (!ctxs || n < 1 || !t0 || !dt || !out) return EDGE_B200_EINVAL;
  for (int k = 0; k < n; k++) {
    edge_b200_ctx *c = ctxs[k];
    if (!c || !c->meshSet || !c->dataSet || !(dt[k] > 0)) return EDGE_B200_EINVAL;
    if (c->nRecv > 0 || c->nOwned != c->nEl || c->timing) return EDGE_B200_ENOTSUP;
    if (c->cfg.device != ctxs[0]->cfg.device) return EDGE_B200_EINVAL;
    for (int j = 0; j < k; j++)
      if (ctxs[j] == c) return EDGE_B200_EINVAL;
  }
  edge_b200_batch *b = new (std::nothrow) edge_b200_batch();
  if (!b) return EDGE_B200_ENOMEM;
  b->ctxs.assign(ctxs, ctxs + n);
  b->t0.assign(t0, t0 + n);
  b->dt.assign(dt, dt + n);
  b->active.assign(n, 1);
  b->streams.assign(n, nullptr);
  b->joins.assign(n, nullptr);
  cudaError_t e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking);
  if (!e) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int k = 0; k < n && !e; k++) {
    e = cudaStreamCreateWithFlags(&b->streams[k], cudaStreamNonBlocking);
    if (!e) e = cudaEventCreateWithFlags(&b->joins[k], cudaEventDisableTiming);
  }
  if (!e) e = cudaMalloc(&b->steps, n * sizeof(int64_t));
  if (!e) e = cudaMalloc(&b->activeDev, n * sizeof(int32_t));
  if (!e) e = cudaMemsetAsync(b->steps, 0, n * sizeof(int64_t), b->origin);
  // the contexts' pending work (uploads) and their flux-solver pairs come before the first step
  for (int k = 0; k < n && !e; k++) {
    edge_b200_ctx *c = ctxs[k];
    e = c->flush();
    if (!e) e = c->ensureFsLR();
    if (!e && edge_b200_batch::fused(c) && !c->faceAlt.p) {
      e = c->faceAlt.fit(c->faceCount() * c->realSize);
      if (!e) e = cudaMemsetAsync(c->faceAlt.p, 0, c->faceCount() * c->realSize, c->stream);
    }
    if (!e) e = cudaEventRecord(b->joins[k], c->stream);
    if (!e) e = cudaStreamWaitEvent(b->origin, b->joins[k], 0);
  }
  if (e) {
    delete b;
    return e == cudaErrorMemoryAllocation ? EDGE_B200_ENOMEM : EDGE_B200_EDEVICE;
  }
  *out = b;
  return EDGE_B200_OK;
}

int edge_b200_batch_set_active(edge_b200_batch *b, const int32_t *active) {
  if (!b || !active) return EDGE_B200_EINVAL;
  for (size_t k = 0; k < b->active.size(); k++) {
    const int32_t v = active[k] ? 1 : 0;
    if (v != b->active[k]) b->dirty = true;
    b->active[k] = v;
  }
  return EDGE_B200_OK;
}

int edge_b200_batch_step(edge_b200_batch *b, int n_steps) {
  if (!b || n_steps < 0) return EDGE_B200_EINVAL;
  if (n_steps == 0) return EDGE_B200_OK;
  EDGE_BATCH_CUDA(b->run(n_steps), "batch steps");
  return EDGE_B200_OK;
}

int edge_b200_batch_sync(edge_b200_batch *b, int64_t *steps) {
  if (!b) return EDGE_B200_EINVAL;
  EDGE_BATCH_CUDA(cudaStreamSynchronize(b->origin), "batch sync");
  if (steps)
    EDGE_BATCH_CUDA(cudaMemcpy(steps, b->steps, b->ctxs.size() * sizeof(int64_t), cudaMemcpyDeviceToHost),
                    "batch steps");
  return EDGE_B200_OK;
}

const char *edge_b200_batch_last_error(const edge_b200_batch *b) { return b ? b->err.c_str() : ""; }

int edge_b200_batch_destroy(edge_b200_batch *b) {
  if (!b) return EDGE_B200_EINVAL;
  delete b;
  return EDGE_B200_OK;
}

int edge_b200_autotune(edge_b200_ctx *ctx, double dt, int32_t caps[2]) {
  if (!ctx || !(dt > 0)) return EDGE_B200_EINVAL;
  if (!ctx->meshSet || !ctx->dataSet || ctx->timing) return EDGE_B200_EINVAL;
  cudaStream_t s = ctx->stream;
  EDGE_CUDA(ctx->flush(), "pending neighbour step");
  EDGE_CUDA(ctx->ensureFsLR(), "flux-solver pairs");
  const size_t rs = ctx->realSize;
  const size_t bytesE = ctx->dofsCount() * rs, bytesA = ctx->dofsACount() * rs;
  DevBuf save;
  if (save.fit(bytesE + bytesA) != cudaSuccess) return EDGE_B200_ENOMEM;
  EDGE_CUDA(cudaMemcpyAsync(save.p, ctx->dofsE, bytesE, cudaMemcpyDeviceToDevice, s), "autotune save");
  if (bytesA)
    EDGE_CUDA(cudaMemcpyAsync(static_cast<char *>(save.p) + bytesE, ctx->dofsA, bytesA, cudaMemcpyDeviceToDevice, s),
              "autotune save");
  KernelSet *ks = ctx->ks;
  ks->setGridCaps(0, 0);
  const int64_t groups = (ctx->nOwned + ks->elementsPerCta() - 1) / ks->elementsPerCta();
  const int defL = ks->ctasLocal(), defN = ks->ctasNeigh();
  cudaEvent_t ev[2];
  EDGE_CUDA(cudaEventCreate(&ev[0]), "autotune");
  EDGE_CUDA(cudaEventCreate(&ev[1]), "autotune");
  StepArgsRaw a = ctx->args(dt);
  int best[2] = {0, 0};
  cudaError_t err = cudaSuccess;
  for (int kind = 0; kind < 2 && !err; kind++) {
    const int def = kind == 0 ? defL : defN;
    // candidates: the persistent default, half of it, one CTA per element group (when more)
    const int64_t cand[3] = {0, def / 2, groups > def ? std::min<int64_t>(groups, 1 << 30) : 0};
    float bestMs = 1e30f;
    for (int c = 0; c < 3 && !err; c++) {
      if (c > 0 && cand[c] <= 0) continue;
      if (kind == 0)
        ks->setGridCaps((int)cand[c], 0);
      else
        ks->setGridCaps(best[0], (int)cand[c]);
      float ms = 1e30f;
      for (int rep = 0; rep < 4 && !err; rep++) {
        if ((err = cudaEventRecord(ev[0], s))) break;
        err = kind == 0 ? ks->local(a, s) : ks->neigh(a, s);
        if (!err) err = cudaEventRecord(ev[1], s);
        if (!err) err = cudaEventSynchronize(ev[1]);
        float t = 0;
        if (!err) err = cudaEventElapsedTime(&t, ev[0], ev[1]);
        if (rep > 0) ms = std::min(ms, t);  // the first launch warms up
      }
      if (!err && ms < bestMs) {
        bestMs = ms;
        best[kind] = (int)cand[c];
      }
    }
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  EDGE_CUDA(err, "autotune");
  ks->setGridCaps(best[0], best[1]);
  EDGE_CUDA(cudaMemcpyAsync(ctx->dofsE, save.p, bytesE, cudaMemcpyDeviceToDevice, s), "autotune restore");
  if (bytesA)
    EDGE_CUDA(cudaMemcpyAsync(ctx->dofsA, static_cast<char *>(save.p) + bytesE, bytesA, cudaMemcpyDeviceToDevice, s),
              "autotune restore");
  EDGE_CUDA(cudaStreamSynchronize(s), "autotune restore");
  if (caps) {
    caps[0] = best[0];
    caps[1] = best[1];
  }
  return EDGE_B200_OK;
}
