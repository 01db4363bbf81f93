// sm_100a kernels of the tet4 ADER-DG element update (elastic + viscoelastic, fused runs).
//
// Thread layout shared by all element kernels: a CTA has 9 "quantity" warps (warp q owns stress /
// velocity quantity q) plus, with attenuation, 6 "anelastic" warps (warp 9+s owns the anelastic
// stress component s of every mechanism). Lane l of every warp is the pair (element l / R, run
// l % R), so a CTA covers E = 32 / R elements; quantity-mixing reads go through shared memory,
// mode products (the global DG matrices) run in registers as compile-time sparse FMA sequences
// (gen/dg_sparse.cuh). CTAs are persistent and loop over element groups.
//
// Data per element, device-resident layout (a contiguous row of modes per quantity and run, padded
// to 16 bytes: GB = B, GF = F rounded up): dofsE [9][R][GB], dofsA [RM*6][R][GB], face buffer
// [4][9][R][GF] = tInt * fluxL_f (the time-integrated DOFs projected on each face, read by the
// neighbours); star [3][24] / starA [3][9] / srcA [RM][12] / fsE [2][.][4][81] / fsA [2][.][4][54]
// in FP64, converted to the kernel precision on load.
#pragma once
#include <cstdint>

#include "gen/dg_sparse.cuh"

namespace edge_b200 {

__host__ __device__ constexpr int nModes(int o) { return o <= 0 ? 0 : o * (o + 1) * (o + 2) / 6; }
__host__ __device__ constexpr int nFaceModes(int o) { return o * (o + 1) / 2; }

enum { FT_INNER = 0, FT_FREE = 1, FT_OUTFLOW = 2 };

template <typename T>
struct StepArgs {
  T *dofsE;             // [nEl][9][R][GB]
  T *dofsA;             // [nEl][RM*6][R][GB]
  T *tDofs;             // [nEl][9][R][GB] or null
  T *face;              // [nEl][4][9][R][GF]
  const double *starE;  // [nEl][3][24]
  const double *starA;  // [nEl][3][9]
  const double *srcA;   // [nEl][RM][12]
  const double *fsE;    // [2][nEl][4][81]
  const double *fsA;    // [2][nEl][4][54]
  const int32_t *elFaEl;
  const uint8_t *fId, *vId, *faType;
  int64_t nEl;
  int64_t elFirst, elCount;  // the launch covers elements [elFirst, elFirst + elCount)
  double dt;
  double omega[3];
  // rate-2 LTS (AderDg.hpp:384-417, 620-674), null for GTS. Elements with a larger neighbour keep
  // the face projections of their time integrals summed over two steps (faceSum, compact slot
  // sumIdx[el]); elements with a smaller neighbour those of the half-step integrals over [0, dt/2]
  // and [dt/2, dt] (faceHalf1 / faceHalf2, slot halfIdx[el]). Each compact buffer is
  // [slots][4][9][R][GF] like face.
  T *faceSum, *faceHalf1, *faceHalf2;
  const uint8_t *ltsFlags;  // [nEl] bit 0: a larger neighbour, bit 1: a smaller neighbour
  const uint8_t *ltsRel;    // [nEl][4] 0 equal, 1 this element larger, 2 this element smaller
  const int32_t *sumIdx, *halfIdx;
  int firstTs;              // first step of a rate-2 pair of this group
  // elastic GTS (Geo::premix): per element face the element's own flux solver fsE[0] and the one
  // its face reader applies (fsE[1] of the face neighbour at its face, or the element's own for a
  // free surface; zeros for outflow) in T, each padded to 16 bytes (Geo::FSP): [nEl][4][2][FSP];
  // null: gathered through the connectivity. fsChar: fsLR holds the characteristic factors of
  // those pairs instead (Geo::charMix: V [9][4], then per quantity {U0[q][0..2], U1[q][0..2], 0, 0})
  const T *fsLR;
  int fsChar;
  // fused GTS steps (kLocal<..., FUSED>, kRecv): the previous step's pre-mixed face projections,
  // whose neighbour fluxes are added to the DOF rows before the recursion (the previous step's
  // neighbour step runs here), or null when none are pending
  const T *faceIn;
  // GTS local step with a time step per element group (g = 0 .. of the launch range: E elements
  // each) instead of dt, or null: several simulations merged into one context step together
  const double *grpDt;
};
enum { LTS_HAS_LARGER = 1, LTS_HAS_SMALLER = 2 };
enum { LTS_EQ = 0, LTS_GT = 1, LTS_LT = 2 };

// sparse patterns (row-major non-zeros): elastic star rows -> (index into the 24, column);
// missing third entries use index -1 (coefficient 0) and a valid column.
__constant__ int8_t kStarIdx[9][3] = {{0, 1, 2}, {3, 4, 5}, {6, 7, 8}, {9, 10, -1}, {11, 12, -1},
                                      {13, 14, -1}, {15, 16, 17}, {18, 19, 20}, {21, 22, 23}};
__constant__ int8_t kStarCol[9][3] = {{6, 7, 8}, {6, 7, 8}, {6, 7, 8}, {6, 7, 6}, {7, 8, 7},
                                      {6, 8, 6}, {0, 3, 5}, {1, 3, 4}, {2, 4, 5}};
// anelastic star rows s -> (index into the 9, velocity column 0..2)
__constant__ int8_t kStarAIdx[6][2] = {{0, -1}, {1, -1}, {2, -1}, {3, 4}, {5, 6}, {7, 8}};
__constant__ int8_t kStarACol[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 2}, {0, 2}};
// anelastic source rows (stress q < 6) -> (index into the 12, anelastic column)
__constant__ int8_t kSrcIdx[6][3] = {{0, 1, 2}, {3, 4, 5}, {6, 7, 8}, {9, -1, -1}, {10, -1, -1}, {11, -1, -1}};
__constant__ int8_t kSrcCol[6][3] = {{0, 1, 2}, {0, 1, 2}, {0, 1, 2}, {3, 3, 3}, {4, 4, 4}, {5, 5, 5}};

template <typename T>
__device__ __forceinline__ T ldd(const double *p, int i) {
  return i < 0 ? T(0) : T(__ldg(p + i));
}

// ------------------------------------------------------------------------------------------------
// shared-memory layout: one contiguous, padded row per (quantity, lane)
// ------------------------------------------------------------------------------------------------
// A tile [rows][32 lanes][S] keeps each lane's modes contiguous so a thread moves four modes with
// one 128-bit access. S is padded so that the eight lanes of a 128-bit phase hit distinct bank
// groups (S / (16 / sizeof(T)) odd) and rows can be read in groups of four past their end.
template <typename T>
__host__ __device__ constexpr int padRow(int n) {
  const int w = 16 / int(sizeof(T));  // elements per 128-bit access
  int m = (((n + 3) / 4) * 4 + w - 1) / w;
  if (m % 2 == 0) m++;
  return m * w;
}
// the same without the odd-chunk padding (rows of four-mode groups only), for tiles that would not
// fit shared memory otherwise; 128-bit accesses then meet two-way bank conflicts
template <typename T>
__host__ __device__ constexpr int padRowTight(int n) {
  const int w = 16 / int(sizeof(T));
  return ((((n + 3) / 4) * 4 + w - 1) / w) * w;
}

template <typename T>
__device__ __forceinline__ void ld4(const T *p, T (&v)[4]);
template <>
__device__ __forceinline__ void ld4<float>(const float *p, float (&v)[4]) {
  const float4 t = *reinterpret_cast<const float4 *>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
template <>
__device__ __forceinline__ void ld4<double>(const double *p, double (&v)[4]) {
  const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
template <typename T>
__device__ __forceinline__ void st4(T *p, const T *v);
template <>
__device__ __forceinline__ void st4<float>(float *p, const float *v) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
template <>
__device__ __forceinline__ void st4<double>(double *p, const double *v) {
  *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2 *>(p + 2) = make_double2(v[2], v[3]);
}
// v[0..N) -> row (128-bit stores, scalar tail)
template <typename T, int N>
__device__ __forceinline__ void stRow(T *p, const T *v) {
#pragma unroll
  for (int n = 0; n + 4 <= N; n += 4) st4<T>(p + n, v + n);
#pragma unroll
  for (int n = (N / 4) * 4; n < N; n++) p[n] = v[n];
}
template <typename T, int N>
__device__ __forceinline__ void ldRow(const T *p, T *v) {
#pragma unroll
  for (int n = 0; n + 4 <= N; n += 4) {
    T t[4];
    ld4<T>(p + n, t);
#pragma unroll
    for (int i = 0; i < 4; i++) v[n + i] = t[i];
  }
#pragma unroll
  for (int n = (N / 4) * 4; n < N; n++) v[n] = p[n];
}

// ------------------------------------------------------------------------------------------------
// device-resident layout: one contiguous row of modes per (element, quantity, run)
// ------------------------------------------------------------------------------------------------
// dofsE [nEl][9][R][GB], dofsA [nEl][RM*6][R][GB], tDofs like dofsE, face [nEl][4][9][R][GF]:
// rows padded to 16 bytes so a thread moves its row with 128-bit accesses. The reference layout
// [nEl][9][B][R] exists only at the C ABI (uploads and downloads transpose on the device).
template <typename T>
__host__ __device__ constexpr int padGlobal(int n) {
  const int w = 16 / int(sizeof(T));
  return ((n + w - 1) / w) * w;
}
// row r of quantity row q of element e, with nRows quantity rows per element
template <typename T, int R, int G>
__device__ __forceinline__ T *gRow(T *base, int64_t e, int nRows, int q, int r) {
  return base + ((e * nRows + q) * R + r) * int64_t(G);
}
template <typename T, int R, int G>
__device__ __forceinline__ const T *gRow(const T *base, int64_t e, int nRows, int q, int r) {
  return base + ((e * nRows + q) * R + r) * int64_t(G);
}
// v[0..N) <- global row (128-bit loads; the row is padded to a multiple of four elements)
template <typename T, int N>
__device__ __forceinline__ void ldRowG(const T *p, T *v, bool valid) {
  constexpr int G = padGlobal<T>(N);
  if (!valid) {
#pragma unroll
    for (int n = 0; n < N; n++) v[n] = T(0);
    return;
  }
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int n = 0; n < G; n += 4) {
      const float4 t = *reinterpret_cast<const float4 *>(p + n);
      const T u[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (n + i < N) v[n + i] = u[i];
    }
  } else {
#pragma unroll
    for (int n = 0; n < G; n += 2) {
      const double2 t = *reinterpret_cast<const double2 *>(p + n);
      v[n] = t.x;
      if (n + 1 < N) v[n + 1] = t.y;
    }
  }
}
// global row <- v[0..N) (128-bit stores; padding is written as zero)
template <typename T, int N>
__device__ __forceinline__ void stRowG(T *p, const T *v) {
  constexpr int G = padGlobal<T>(N);
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int n = 0; n < G; n += 4) {
      float4 t;
      t.x = v[n];
      t.y = n + 1 < N ? v[n + 1] : T(0);
      t.z = n + 2 < N ? v[n + 2] : T(0);
      t.w = n + 3 < N ? v[n + 3] : T(0);
      *reinterpret_cast<float4 *>(p + n) = t;
    }
  } else {
#pragma unroll
    for (int n = 0; n < G; n += 2) {
      double2 t;
      t.x = v[n];
      t.y = n + 1 < N ? v[n + 1] : T(0);
      *reinterpret_cast<double2 *>(p + n) = t;
    }
  }
}

// asynchronous global -> shared copies (cp.async: no registers held while in flight)
__device__ __forceinline__ void cpAsync16(void *dst, const void *src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsync8(void *dst, const void *src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// cooperative copy of the rows [R][GB] of quantity row q (of nRows per element) of element e into
// the tile rows (q, eo * R + row) with stride S, consecutive lanes moving consecutive 16-byte chunks
template <typename T, int R, int GB, int S>
__device__ __forceinline__ void copyRows(T *tile, const T *base, int64_t e, int nRows, int q, int eo, int r) {
  constexpr int W = 16 / int(sizeof(T)), CPRB = GB / W;
  const T *blk = base + (e * nRows + q) * int64_t(R * GB);
  T *dst = tile + (q * 32 + eo * R) * S;
#pragma unroll
  for (int it = 0; it < CPRB; it++) {
    const int k = it * R + r;
    const int row = k / CPRB, col = k % CPRB;
    cpAsync16(dst + row * S + col * W, blk + row * GB + col * W);
  }
}

// cooperative copy of the DOF rows [R][GB] of quantity q of an element into the tile rows
// (q, eo * R + row) with stride S: warp q moves its quantity's rows, consecutive lanes consecutive
// 16-byte chunks
template <typename T, int R, int GB, int S>
__device__ __forceinline__ void copyDofRows(T *tile, const T *dofsE, int64_t e, int q, int eo, int r) {
  copyRows<T, R, GB, S>(tile, dofsE, e, 9, q, eo, r);
}

// the reverse for results: tile rows (q, eo * R + row), stride S -> the [R][G] rows of row block
// blk in global memory, consecutive lanes storing consecutive 16-byte chunks (the caller orders the
// tile rows before, e.g. with __syncwarp when warp q wrote them)
template <typename T, int R, int G, int S>
__device__ __forceinline__ void storeRowsCoalesced(const T *tile, T *blk, int q, int eo, int r) {
  constexpr int W = 16 / int(sizeof(T)), CPR = G / W;
  const T *src = tile + (q * 32 + eo * R) * S;
#pragma unroll
  for (int it = 0; it < CPR; it++) {
    const int k = it * R + r;
    const int row = k / CPR, col = k % CPR;
    T v[4];
    if constexpr (sizeof(T) == 4) {
      ld4<T>(src + row * S + col * W, v);
      *reinterpret_cast<float4 *>(blk + row * G + col * W) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
      const double2 d = *reinterpret_cast<const double2 *>(src + row * S + col * W);
      *reinterpret_cast<double2 *>(blk + row * G + col * W) = d;
    }
  }
}

template <typename T, int O, int R, int RM>
struct Geo {
  static constexpr int GB = padGlobal<T>(nModes(O)), GF = padGlobal<T>(nFaceModes(O));
  static constexpr int B = nModes(O), F = nFaceModes(O), E = 32 / R;
  static constexpr int NW = 9 + (RM ? 6 : 0);
  static constexpr int NT = NW * 32;
  // rows padded for conflict-free 128-bit accesses, unless the derivative, anelastic and face tiles
  // would then exceed the 227 KB of a CTA (order 6 with attenuation): tight rows instead
  static constexpr bool tightRows =
      (size_t(9) * 32 * padRow<T>(B) * (1 + 2 * RM) + size_t(9) * 32 * padRow<T>(F)) * sizeof(T) > 227 * 1024;
  static constexpr int SB = tightRows ? padRowTight<T>(B) : padRow<T>(B);
  static constexpr int SF = tightRows ? padRowTight<T>(F) : padRow<T>(F);
  // X [9][32][SB]   derivatives during the CK recursion
  // TI [9][32][SB]  time-integrated DOFs
  // XA / TIA [RM][6][32][SB]  anelastic derivatives / time integrals
  // S0 [9][32][SF]  face tiles
  static constexpr size_t nX = size_t(9) * 32 * SB;
  static constexpr size_t nXA = size_t(RM) * 6 * 32 * SB;
  static constexpr size_t nS0 = size_t(9) * 32 * SF;
  // The time integrals live in shared memory when that fits (227 KB per CTA); the face tiles
  // then reuse X. Otherwise they stay in registers during the recursion and are copied into X /
  // XA afterwards, with the face tiles behind X.
  static constexpr bool tiSmem = (2 * nX + 2 * nXA) * sizeof(T) <= 227 * 1024;
  static constexpr size_t nTI = tiSmem ? nX : nS0;
  static constexpr size_t nTIA = tiSmem ? nXA : 0;
  // With room for the face tiles in a region of their own, X is free after the recursion: the
  // local kernel then copies the DOF rows into X asynchronously (the current group's again after
  // the recursion, for the volume integral, and the next group's during the face integrals)
  static constexpr size_t baseLocal = (nX + nTI + nXA + nTIA) * sizeof(T);
  static constexpr size_t localBudget =
      (sizeof(T) == 4 && RM == 0 && baseLocal <= 110 * 1024) ? 110 * 1024 : 227 * 1024;
  static constexpr bool asyncLocal = tiSmem && baseLocal + nS0 * sizeof(T) <= localBudget;
  static constexpr size_t smemLocal = baseLocal + (asyncLocal ? nS0 * sizeof(T) : 0);
  // elastic GTS: the local kernel stores each face projection already mixed with the reading
  // element's flux solver (fsE[1] of the face neighbour, or its own for a free surface), so the
  // neighbour kernel only rotates its own quantity row and applies fluxT (no shared mix, no
  // barrier). The two flux-solver blocks of every face arrive one face ahead by cp.async into two
  // buffers [E][2][FSP] behind the face tile; configurations without room for them keep the mix in
  // the neighbour kernel.
  static constexpr int FSP = padGlobal<T>(81);  // a 9x9 block padded to 16 bytes
  static constexpr size_t premixBytes = size_t(2) * E * 2 * FSP * sizeof(T);
  static constexpr bool premix = RM == 0 && asyncLocal && smemLocal + premixBytes <= localBudget;
  // configurations that mix in the neighbour kernel (attenuation among them): the local flux-solver
  // blocks fsE[0] (and fsA[0]) of every face arrive one face ahead by cp.async into two buffers
  // [E][NFL] of doubles behind the face tile, where they fit
  static constexpr int NFL = 81 + (RM ? 54 : 0);
  static constexpr size_t fsLocalBytes = size_t(2) * E * NFL * sizeof(double);
  static constexpr bool fsLocal = !premix && asyncLocal && smemLocal + fsLocalBytes <= localBudget;
  // with attenuation the next group's element coefficients (star, starA, srcA: NCO doubles per
  // element) arrive by cp.async as well, into a buffer behind those
  static constexpr int NCO = 72 + 27 + 12 * RM;
  static constexpr size_t coefBytes = size_t(E) * NCO * sizeof(double);
  static constexpr bool coefSmem = fsLocal && RM > 0 && smemLocal + fsLocalBytes + coefBytes <= localBudget;
  // and the anelastic warps compute the anelastic source terms of the elastic rows, handed over in a
  // tile [9][32][SB] behind the coefficients (srcShare)
  static constexpr size_t srcOff = (smemLocal + fsLocalBytes + coefBytes + 15) / 16 * 16;
  static constexpr size_t srcBytes = size_t(9) * 32 * SB * sizeof(T);
  static constexpr bool srcSplit = coefSmem && srcOff + srcBytes <= localBudget;
  // and the group's 36 face projections (9 rows x 4 faces) are spread over all fifteen warps into
  // four face tiles (the face tile, X, and two behind the source tile), with the flux-solver blocks
  // of all four faces at hand (faces 2 and 3 behind the source tile): one barrier before the four
  // faces' mixes instead of one per face (facesSplit)
  static constexpr size_t fsExtraOff = srcOff + srcBytes;
  static constexpr size_t tilesOff = (fsExtraOff + fsLocalBytes + 15) / 16 * 16;
  static constexpr bool projSplit = srcSplit && tilesOff + 2 * nS0 * sizeof(T) <= localBudget;
  // characteristic mix (elastic GTS, pre-mixing): the two flux solvers a face projection P meets
  // -- fsE[0] of the element and the reader's fsE[1] -- stacked (18 x 9) have rank 3, the three
  // waves that leave the element through the face: [fsE0; fsE1] = [U0; U1] V^T. The nine warps
  // first compute the three characteristic rows W = V^T P (a four-mode chunk each), then every
  // warp its two output rows from W: 3 x 9 + 2 x 9 x 3 products per face mode instead of 2 x 81.
  // W [3][32][SF] lives in X behind the face rows it holds during the faces, or behind the
  // flux-solver buffers
  static constexpr size_t nW = size_t(3) * 32 * SF;
  static constexpr bool wInX = nW <= nX - nS0;
  static constexpr bool charMix =
      premix && (F + 3) / 4 <= 9 && (wInX || smemLocal + premixBytes + nW * sizeof(T) <= localBudget);
  // LTS local kernels: the characteristic rows (and, in mode 2, those of the half-step projections)
  // behind X's face rows, where both tiles fit there
  static constexpr bool w2InX = 2 * nW <= nX - nS0;
  static constexpr size_t smemLocalGts = premix      ? smemLocal + premixBytes +
                                                      (charMix && !wInX ? nW * sizeof(T) : 0)
                                         : projSplit ? tilesOff + 2 * nS0 * sizeof(T)
                                         : srcSplit  ? srcOff + srcBytes
                                         : fsLocal  ? smemLocal + fsLocalBytes + (coefSmem ? coefBytes : 0)
                                                    : smemLocal;
  // the local kernel's shared-memory regions: in order, 16-byte aligned where 128-bit accesses or
  // 16-byte copies reach them, within the 227 KB a CTA may hold
  static_assert(smemLocal % 16 == 0, "buffers behind the tiles start on 16-byte boundaries");
  static_assert(!srcSplit || (srcOff % 16 == 0 && srcOff >= smemLocal + fsLocalBytes + coefBytes),
                "source tile behind the coefficients");
  static_assert(!projSplit || (tilesOff % 16 == 0 && tilesOff >= fsExtraOff + fsLocalBytes),
                "face tiles behind the flux-solver blocks of faces 2 and 3");
  static_assert(smemLocalGts <= 227 * 1024, "local kernel within a CTA's shared memory");
  // elastic CK with ping-pong derivatives between X and the separate face tile
  static constexpr bool ckPingPong = asyncLocal && RM == 0 && nModes(O - 1) <= SF;
  // LTS local step: one more [9][32][SB] tile for the half-step time integral (behind the rest)
  // and, pre-mixing, the flux-solver buffers and two face tiles for the half-step projections;
  // configurations whose time integrals do not fit shared memory have no LTS kernels
  static constexpr bool premixLts =
      premix && smemLocal + nX * sizeof(T) + premixBytes + 2 * nS0 * sizeof(T) <= 227 * 1024;
  static constexpr size_t smemLocalLts =
      smemLocal + nX * sizeof(T) + (premixLts ? premixBytes + 2 * nS0 * sizeof(T) : 0);
  // the LTS local kernel without half-step integrals (mode 1)
  static constexpr size_t smemLocalSums = smemLocal + (premixLts ? premixBytes : 0);
  static constexpr bool ltsOk = tiSmem && smemLocalLts <= 227 * 1024;
  static constexpr bool charMixLts = premixLts && charMix && ltsOk && w2InX;
  // neighbour kernel: a ring of NSN slots, each [9][32][SF] face rows and, for E <= 4, the E
  // elements' flux-solver blocks (81 + 54 doubles); as many slots (2..4) as fit the shared memory
  // of minCtasNeigh CTAs per SM (228 KB, 1 KB reserved per CTA)
  static constexpr int minCtasNeigh = (sizeof(T) == 4 && RM == 0) ? 2 : 1;
  static constexpr bool fsSmem = E <= 4;
  static constexpr size_t slotNeigh =
      (nS0 * sizeof(T) + 15) / 16 * 16 + (fsSmem ? size_t(E) * (81 + (RM ? 54 : 0)) * 8 : 0);
  static constexpr size_t budgetNeigh = (228 * 1024) / minCtasNeigh - 1024;
  // the next group's DOF rows [9][32][SB] are prefetched into a tile behind the slots when that
  // leaves room for at least three slots
  static constexpr size_t dofTileBytes = size_t(9) * 32 * SB * sizeof(T);
  static constexpr bool dofTile = budgetNeigh >= dofTileBytes + 3 * slotNeigh;
  static constexpr size_t slotRoom = budgetNeigh - (dofTile ? dofTileBytes : 0);
  static constexpr int NSN = slotRoom / slotNeigh >= 4 ? 4 : int(slotRoom / slotNeigh);
  static_assert(NSN >= 2, "neighbour kernel needs two slots");
  static_assert(slotNeigh % 16 == 0, "slots start on 16-byte boundaries (cp.async targets)");
  // with attenuation the group's anelastic rows [RM * 6][32][SB] arrive in a tile of their own
  // (with the DOF rows, one group ahead) where it fits
  static constexpr size_t dofATileBytes = size_t(RM) * 6 * 32 * SB * sizeof(T);
  static constexpr bool dofATile =
      RM > 0 && dofTile && NSN * slotNeigh + dofTileBytes + dofATileBytes <= budgetNeigh;
  static constexpr size_t smemNeigh =
      NSN * slotNeigh + (dofTile ? dofTileBytes : 0) + (dofATile ? dofATileBytes : 0);
  // resident CTAs per SM the register allocation targets (65,536 registers per SM): FP32 keeps
  // two 288-thread CTAs of each kernel (<= 113 registers); FP64 rows need twice the registers
  // and keep one
  static constexpr int minCtasLocal = (sizeof(T) == 4 && RM == 0 && smemLocal <= 110 * 1024) ? 2 : 1;
};

// per-thread element coefficients
template <typename T, int RM>
struct ElemCoef {
  T cs[3][3];     // star row q, 3 slots, per derivative direction (kStarDir)
  int cols[3];
  T ca[3][2];     // anelastic star row s, per derivative direction
  int colsA[2];
  T csrc[3][3];   // source matrices row q (< 6), per mechanism
  int colsSrc[3];

  __device__ __forceinline__ void load(const StepArgs<T> &a, int64_t e, bool valid, int q) {
    loadFrom<true>(a.starE + e * 72, a.starA + e * 27, a.srcA + e * (RM * 12), valid, q);
  }
  template <bool GLOBAL>
  __device__ __forceinline__ static double rd(const double *p) {
    if constexpr (GLOBAL)
      return __ldg(p);
    else
      return *p;
  }
  // from the element's blocks star [3][24], starA [3][9], srcA [RM][12] (global memory, or a copy in
  // shared memory)
  // SPLIT: the anelastic warps compute the anelastic source terms of the elastic rows (srcShare)
  // and hold their coefficients; the elastic warps hold none
  template <bool GLOBAL, bool SPLIT = false>
  __device__ __forceinline__ void loadFrom(const double *sE, const double *sA, const double *sS, bool valid,
                                           int q) {
    if (q < 9) {
#pragma unroll
      for (int i = 0; i < 3; i++) cols[i] = kStarCol[q][i];
      // star_dim -> star of the derivative directions of the generated stiffness products (FP64)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int idx = kStarIdx[q][i];
        double v[3] = {0, 0, 0};
        if (valid && idx >= 0)
#pragma unroll
          for (int d = 0; d < 3; d++) v[d] = rd<GLOBAL>(sE + d * 24 + idx);
#pragma unroll
        for (int d = 0; d < 3; d++) cs[d][i] = T(kStarDir[0][d] * v[0] + kStarDir[1][d] * v[1] + kStarDir[2][d] * v[2]);
      }
      if (RM && q < 6 && !SPLIT) {
#pragma unroll
        for (int i = 0; i < 3; i++) colsSrc[i] = kSrcCol[q][i];
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
          for (int i = 0; i < 3; i++) {
            int idx = kSrcIdx[q][i];
            csrc[m][i] = valid && m < RM && idx >= 0 ? T(rd<GLOBAL>(sS + m * 12 + idx)) : T(0);
          }
      } else {
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
          for (int i = 0; i < 3; i++) csrc[m][i] = T(0);
#pragma unroll
        for (int i = 0; i < 3; i++) colsSrc[i] = 0;
      }
    } else {
      const int s = q - 9;
#pragma unroll
      for (int i = 0; i < 2; i++) colsA[i] = kStarACol[s][i];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int idx = kStarAIdx[s][i];
        double v[3] = {0, 0, 0};
        if (valid && idx >= 0)
#pragma unroll
          for (int d = 0; d < 3; d++) v[d] = rd<GLOBAL>(sA + d * 9 + idx);
#pragma unroll
        for (int d = 0; d < 3; d++) ca[d][i] = T(kStarDir[0][d] * v[0] + kStarDir[1][d] * v[1] + kStarDir[2][d] * v[2]);
      }
      if constexpr (SPLIT && RM > 0) {
        // s < 3: srcA_m[s][i] of mechanisms m < RM - 1 (csrc[m][i]); s >= 3: srcA_{RM-1}[s - 3][i]
        // (csrc[0][i]) and srcA_m[s][s] of every mechanism (csrc[1][m])
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
          for (int i = 0; i < 3; i++) csrc[m][i] = T(0);
        if (s < 3) {
#pragma unroll
          for (int m = 0; m + 1 < RM; m++)
#pragma unroll
            for (int i = 0; i < 3; i++) csrc[m][i] = valid ? T(rd<GLOBAL>(sS + m * 12 + kSrcIdx[s][i])) : T(0);
        } else {
#pragma unroll
          for (int i = 0; i < 3; i++) csrc[0][i] = valid ? T(rd<GLOBAL>(sS + (RM - 1) * 12 + kSrcIdx[s - 3][i])) : T(0);
#pragma unroll
          for (int m = 0; m < RM; m++) csrc[1][m] = valid ? T(rd<GLOBAL>(sS + m * 12 + kSrcIdx[s][0])) : T(0);
        }
      }
    }
  }
};

// operand of the stiffness products: star mix of three source rows, shared by the three directions
// zz[dim][i] = sum_s c[dim][s] * X[col_s][l][k0 + i]
template <typename T, int S>
struct Mix3 {
  const T *r0, *r1, *r2;  // source rows of this lane
  const T (*c)[3];
  template <int K0>
  __device__ __forceinline__ void load(T (&zz)[3][4]) const {
    T v0[4], v1[4], v2[4];
    ld4<T>(r0 + K0, v0);
    ld4<T>(r1 + K0, v1);
    ld4<T>(r2 + K0, v2);
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int i = 0; i < 4; i++) zz[d][i] = fmaT(c[d][2], v2[i], fmaT(c[d][1], v1[i], c[d][0] * v0[i]));
  }
};
// FP32: the same products on packed pairs of modes (sm_100 FFMA2: half the issue slots; each lane
// of a pair rounds as the scalar chain does, so the results are bit-identical)
template <int S>
struct Mix3<float, S> {
  const float *r0, *r1, *r2;
  const float (*c)[3];
  template <int K0>
  __device__ __forceinline__ void load(float (&zz)[3][4]) const {
    const float4 a = *reinterpret_cast<const float4 *>(r0 + K0);
    const float4 b = *reinterpret_cast<const float4 *>(r1 + K0);
    const float4 e = *reinterpret_cast<const float4 *>(r2 + K0);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float2 k0 = make_float2(c[d][0], c[d][0]), k1 = make_float2(c[d][1], c[d][1]),
                   k2 = make_float2(c[d][2], c[d][2]);
      float2 lo = __fmul2_rn(k0, make_float2(a.x, a.y));
      float2 hi = __fmul2_rn(k0, make_float2(a.z, a.w));
      lo = __ffma2_rn(k1, make_float2(b.x, b.y), lo);
      hi = __ffma2_rn(k1, make_float2(b.z, b.w), hi);
      lo = __ffma2_rn(k2, make_float2(e.x, e.y), lo);
      hi = __ffma2_rn(k2, make_float2(e.z, e.w), hi);
      zz[d][0] = lo.x;
      zz[d][1] = lo.y;
      zz[d][2] = hi.x;
      zz[d][3] = hi.y;
    }
  }
};
// anelastic star: two velocity rows
template <typename T, int S>
struct Mix2 {
  const T *r0, *r1;
  const T (*c)[2];
  template <int K0>
  __device__ __forceinline__ void load(T (&zz)[3][4]) const {
    T v0[4], v1[4];
    ld4<T>(r0 + K0, v0);
    ld4<T>(r1 + K0, v1);
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int i = 0; i < 4; i++) zz[d][i] = fmaT(c[d][1], v1[i], c[d][0] * v0[i]);
  }
};
template <int S>
struct Mix2<float, S> {
  const float *r0, *r1;
  const float (*c)[2];
  template <int K0>
  __device__ __forceinline__ void load(float (&zz)[3][4]) const {
    const float4 a = *reinterpret_cast<const float4 *>(r0 + K0);
    const float4 b = *reinterpret_cast<const float4 *>(r1 + K0);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float2 k0 = make_float2(c[d][0], c[d][0]), k1 = make_float2(c[d][1], c[d][1]);
      float2 lo = __fmul2_rn(k0, make_float2(a.x, a.y));
      float2 hi = __fmul2_rn(k0, make_float2(a.z, a.w));
      lo = __ffma2_rn(k1, make_float2(b.x, b.y), lo);
      hi = __ffma2_rn(k1, make_float2(b.z, b.w), hi);
      zz[d][0] = lo.x;
      zz[d][1] = lo.y;
      zz[d][2] = hi.x;
      zz[d][3] = hi.y;
    }
  }
};
// the thread's own row
template <typename T>
struct OwnRow {
  const T *r;
  template <int K0>
  __device__ __forceinline__ void load(T (&zz)[1][4]) const { ld4<T>(r + K0, zz[0]); }
};

template <typename T, int S>
__device__ __forceinline__ const T *rowPtr(const T *base, int row, int l) {
  return base + (row * 32 + l) * S;
}
template <typename T, int S>
__device__ __forceinline__ T *rowPtr(T *base, int row, int l) {
  return base + (row * 32 + l) * S;
}

// dofs rows 0..5 += sum_m srcA_m * Y_m (anelastic source matrices, all B modes)
template <typename T, int B, int S, int RM>
__device__ __forceinline__ void addSrc(const ElemCoef<T, RM> &c, const T *Y, int l, T *acc) {
#pragma unroll
  for (int m = 0; m < RM; m++)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      T y[B];
      ldRow<T, B>(rowPtr<T, S>(Y, m * 6 + c.colsSrc[i], l), y);
#pragma unroll
      for (int n = 0; n < B; n++) acc[n] = fmaT(c.csrc[m][i], y[n], acc[n]);
    }
}

// the same source terms computed by the anelastic warps (ElemCoef SPLIT), into the rows of SRC
// [9][32][S]: warp s < 3 the terms of mechanisms m < RM - 1 of elastic row s (row s); warp s >= 3
// those of elastic row s (row s) and the last mechanism's of elastic row s - 3 (row s + 3). Elastic
// row q < 6 then adds row q, and q < 3 row q + 6 too: six source rows per anelastic warp instead of
// nine per elastic warp 0-2.
template <typename T, int B, int S, int RM>
__device__ __forceinline__ void srcShare(const ElemCoef<T, RM> &c, const T *Y, int l, int s, T *SRC) {
  T o[B], y[B];
#pragma unroll
  for (int n = 0; n < B; n++) o[n] = T(0);
  if (s < 3) {
#pragma unroll
    for (int m = 0; m + 1 < RM; m++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        ldRow<T, B>(rowPtr<T, S>(Y, m * 6 + i, l), y);
#pragma unroll
        for (int n = 0; n < B; n++) o[n] = fmaT(c.csrc[m][i], y[n], o[n]);
      }
    stRow<T, B>(rowPtr<T, S>(SRC, s, l), o);
  } else {
#pragma unroll
    for (int i = 0; i < 3; i++) {
      ldRow<T, B>(rowPtr<T, S>(Y, (RM - 1) * 6 + i, l), y);
#pragma unroll
      for (int n = 0; n < B; n++) o[n] = fmaT(c.csrc[0][i], y[n], o[n]);
    }
    stRow<T, B>(rowPtr<T, S>(SRC, s + 3, l), o);
#pragma unroll
    for (int n = 0; n < B; n++) o[n] = T(0);
#pragma unroll
    for (int m = 0; m < RM; m++) {
      ldRow<T, B>(rowPtr<T, S>(Y, m * 6 + s, l), y);
#pragma unroll
      for (int n = 0; n < B; n++) o[n] = fmaT(c.csrc[1][m], y[n], o[n]);
    }
    stRow<T, B>(rowPtr<T, S>(SRC, s, l), o);
  }
}
// elastic row q < 6: acc += its source rows of SRC
template <typename T, int B, int S>
__device__ __forceinline__ void addSrcRows(const T *SRC, int q, int l, T *acc) {
  T y[B];
  ldRow<T, B>(rowPtr<T, S>(SRC, q, l), y);
#pragma unroll
  for (int n = 0; n < B; n++) acc[n] += y[n];
  if (q < 3) {
    ldRow<T, B>(rowPtr<T, S>(SRC, q + 6, l), y);
#pragma unroll
    for (int n = 0; n < B; n++) acc[n] += y[n];
  }
}

// ---------------------------------------- CK recursion -----------------------------------------
// derivative D of TimePredVanilla::ck (TimePredVanilla.hpp:229-303) with the star matrix applied
// before the stiffness product; der[D] replaces der[D-1] in X, TI += sca * der[D] (rows owned by
// their warp), the anelastic warps update XA and TIA.
// PP (ping-pong, elastic only): the derivatives alternate between X (even D, stride SB) and the
// face tile XP (odd D, stride SF), so a level reads one buffer and writes the other and needs one
// barrier instead of two (the truncated derivatives of levels >= 1 fit the face tile's rows)
template <typename T, int O, int R, int RM, int D, bool H = false, bool PP = false>
struct CkStep {
  using G = Geo<T, O, R, RM>;
  static constexpr int B = G::B, S = G::SB;
  static constexpr int NN = RM ? nModes(O - 1) : nModes(O - D);  // output modes of the product
  static constexpr int DK = RM ? 1 : D;                           // truncation of the product
  static constexpr bool IN_P = PP && (D - 1) % 2 == 1, OUT_P = PP && D % 2 == 1;
  static constexpr int SI = IN_P ? G::SF : S, SO = OUT_P ? G::SF : S;
  static_assert(!PP || (RM == 0 && NN <= G::SF), "ping-pong derivatives must fit the face tile");

  // H: also TIh += scaH * der[D] (the time integral over the first half of the step, for LTS)
  // SRC (attenuation, ElemCoef SPLIT): the anelastic warps compute the source terms (srcShare)
  __device__ __forceinline__ static void run(T *X, T *TI, T *XA, T *TIA, int q, int l, const ElemCoef<T, RM> &c,
                                             const double *omega, T sca, T *tIr, T (*tIAr)[B], T *TIh = nullptr,
                                             T scaH = T(0), T *XP = nullptr, T *SRC = nullptr) {
    T *Xin = IN_P ? XP : X;
    T *Xout = OUT_P ? XP : X;
    T acc[B];
#pragma unroll
    for (int n = 0; n < B; n++) acc[n] = T(0);
    if (q < 9) {
      Mix3<T, SI> z{rowPtr<T, SI>(Xin, c.cols[0], l), rowPtr<T, SI>(Xin, c.cols[1], l),
                    rowPtr<T, SI>(Xin, c.cols[2], l), c.cs};
      CkMul<O, DK>::template run<T>(z, acc);
      if constexpr (RM > 0)
        if (q < 6 && !SRC) addSrc<T, B, S, RM>(c, XA, l, acc);
    } else if constexpr (RM > 0) {
      if (SRC) srcShare<T, B, S, RM>(c, XA, l, q - 9, SRC);
      Mix2<T, S> z{rowPtr<T, S>(X, 6 + c.colsA[0], l), rowPtr<T, S>(X, 6 + c.colsA[1], l), c.ca};
      CkMul<O, DK>::template run<T>(z, acc);
    }
    if constexpr (!PP) __syncthreads();
    if constexpr (RM > 0)
      if (SRC && q < 6) addSrcRows<T, B, S>(SRC, q, l, acc);
    if (q < 9) {
      constexpr int NW = RM ? B : NN;  // modes beyond NN stay zero without anelasticity
      stRow<T, NW>(rowPtr<T, SO>(Xout, q, l), acc);
      if constexpr (G::tiSmem) {
        T t[NW];
        T *p = rowPtr<T, S>(TI, q, l);
        ldRow<T, NW>(p, t);
#pragma unroll
        for (int n = 0; n < NW; n++) t[n] = fmaT(sca, acc[n], t[n]);
        stRow<T, NW>(p, t);
        if constexpr (H) {
          T *ph = rowPtr<T, S>(TIh, q, l);
          ldRow<T, NW>(ph, t);
#pragma unroll
          for (int n = 0; n < NW; n++) t[n] = fmaT(scaH, acc[n], t[n]);
          stRow<T, NW>(ph, t);
        }
      } else {
#pragma unroll
        for (int n = 0; n < NW; n++) tIr[n] = fmaT(sca, acc[n], tIr[n]);
      }
    } else if constexpr (RM > 0) {
      const int s = q - 9;
#pragma unroll
      for (int m = 0; m < RM; m++) {
        const T om = T(omega[m]);
        T *px = rowPtr<T, S>(XA, m * 6 + s, l);
        T v[B];
        ldRow<T, B>(px, v);
#pragma unroll
        for (int n = 0; n < B; n++) v[n] = om * (acc[n] + v[n]);
        stRow<T, B>(px, v);
        if constexpr (G::tiSmem) {
          T *pt = rowPtr<T, S>(TIA, m * 6 + s, l);
          T t[B];
          ldRow<T, B>(pt, t);
#pragma unroll
          for (int n = 0; n < B; n++) t[n] = fmaT(sca, v[n], t[n]);
          stRow<T, B>(pt, t);
        } else {
#pragma unroll
          for (int n = 0; n < B; n++) tIAr[m][n] = fmaT(sca, v[n], tIAr[m][n]);
        }
      }
    }
    __syncthreads();
  }
};

template <typename T, int O, int R, int RM, int D, bool H = false, bool PP = false>
__device__ __forceinline__ void ckAll(T *X, T *TI, T *XA, T *TIA, int q, int l, const ElemCoef<T, RM> &c,
                                      const double *omega, T dt, T sca, T *tIr, T (*tIAr)[nModes(O)],
                                      T *TIh = nullptr, T scaH = T(0), T *XP = nullptr, T *SRC = nullptr) {
  if constexpr (D < O) {
    sca = sca * dt / T(D + 1);
    if constexpr (H) scaH = scaH * (dt * T(0.5)) / T(D + 1);
    CkStep<T, O, R, RM, D, H, PP>::run(X, TI, XA, TIA, q, l, c, omega, sca, tIr, tIAr, TIh, scaH, XP, SRC);
    ckAll<T, O, R, RM, D + 1, H, PP>(X, TI, XA, TIA, q, l, c, omega, dt, sca, tIr, tIAr, TIh, scaH, XP, SRC);
  }
}

// s1[j] = sum_i fr[i] * S0[i][l][j] for j < F (128-bit loads over j)
template <typename T, int F, int SF>
__device__ __forceinline__ void faceMix(const T *S0, int l, const T (&fr)[9], T *s) {
#pragma unroll
  for (int j0 = 0; j0 < F; j0 += 4) {
    T v[4];
    ld4<T>(rowPtr<T, SF>(S0, 0, l) + j0, v);
    T o[4];
#pragma unroll
    for (int u = 0; u < 4; u++) o[u] = fr[0] * v[u];
#pragma unroll
    for (int i = 1; i < 9; i++) {
      ld4<T>(rowPtr<T, SF>(S0, i, l) + j0, v);
#pragma unroll
      for (int u = 0; u < 4; u++) o[u] = fmaT(fr[i], v[u], o[u]);
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (j0 + u < F) s[j0 + u] = o[u];
  }
}

// two mixes of the same rows: s[j] = sum_i fr[i] S0[i][l][j] into registers, t[j] = sum_i fr1[i]
// S0[i][l][j] written to tRow[0, G) chunk by chunk (skipped when tRow is null); S0's rows are zero
// in [F, G), so is t there
template <typename T, int F, int SF, int G>
__device__ __forceinline__ void faceMix2(const T *S0, int l, const T (&fr)[9], const T (&fr1)[9], T *s,
                                         T *tRow) {
#pragma unroll
  for (int j0 = 0; j0 < F; j0 += 4) {
    T v[4];
    ld4<T>(rowPtr<T, SF>(S0, 0, l) + j0, v);
    // modes past F (the zero padding of the last chunk) are not mixed: t is zero there
    T o[4], p[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      o[u] = j0 + u < F ? fr[0] * v[u] : T(0);
      p[u] = j0 + u < F ? fr1[0] * v[u] : T(0);
    }
#pragma unroll
    for (int i = 1; i < 9; i++) {
      ld4<T>(rowPtr<T, SF>(S0, i, l) + j0, v);
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (j0 + u < F) {
          o[u] = fmaT(fr[i], v[u], o[u]);
          p[u] = fmaT(fr1[i], v[u], p[u]);
        }
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (j0 + u < F) s[j0 + u] = o[u];
    if (tRow) {
      if (j0 + 4 <= G) {
        st4<T>(tRow + j0, p);
      } else {
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (j0 + u < G) tRow[j0 + u] = p[u];
      }
    }
  }
}

// one mix of the characteristic rows: h[j] = sum_k u[k] W[k][j] for j < F (u: three values)
template <typename T, int F, int SF>
__device__ __forceinline__ void charMixOne(const T *Wt, int l, const T *u, T *h) {
  const T u0 = u[0], u1 = u[1], u2 = u[2];
#pragma unroll
  for (int j0 = 0; j0 < F; j0 += 4) {
    T w0[4], w1[4], w2[4];
    ld4<T>(rowPtr<T, SF>(Wt, 0, l) + j0, w0);
    ld4<T>(rowPtr<T, SF>(Wt, 1, l) + j0, w1);
    ld4<T>(rowPtr<T, SF>(Wt, 2, l) + j0, w2);
#pragma unroll
    for (int v = 0; v < 4; v++)
      if (j0 + v < F) h[j0 + v] = fmaT(u2, w2[v], fmaT(u1, w1[v], u0 * w0[v]));
  }
}

// the flux-solver blocks of face FA of group g's elements (pre-mixed projections) into buf
// [E][2][FSP]: 16-byte copies from fsLR, or (without it) loads gathered through the connectivity
// and stored in T, visible after the next barrier like the copies
template <typename T>
struct MixFs {
  T *buf;  // two buffers [2][E][2][FSP]
  int64_t g, nGroups;
  T *w = nullptr;   // characteristic rows [3][32][SF] (Geo::charMix)
  T *wh = nullptr;  // those of the half-step projections (LTS mode 2, Geo::charMixLts)
};

// characteristic rows of a face (Geo::charMix), first half: warp q < ceil(F / 4) computes modes
// [4q, 4q + 4) of W[k] = sum_i V[i][k] S0[i] (k < 3) into Wt; fb = this lane's element's factors
// (V [9][4] first). Modes past F read whatever the row holds there and count as zero.
template <typename T, int F, int SF>
__device__ __forceinline__ void charRows(const T *S0, const T *fb, int q, int l, T *Wt) {
  if (q >= (F + 3) / 4) return;
  const int j0 = 4 * q;
  T w[3][4];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int u = 0; u < 4; u++) w[k][u] = T(0);
#pragma unroll
  for (int i = 0; i < 9; i++) {
    T v[4], vk[4];
    ld4<T>(rowPtr<T, SF>(S0, i, l) + j0, v);
    ld4<T>(fb + 4 * i, vk);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const T x = j0 + u < F ? v[u] : T(0);
#pragma unroll
      for (int k = 0; k < 3; k++) w[k][u] = fmaT(vk[k], x, w[k][u]);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++) st4<T>(rowPtr<T, SF>(Wt, k, l) + j0, w[k]);
}

// second half: s[j] = sum_k uu[k] W[k][j] into registers, t[j] = sum_k uu[3 + k] W[k][j] written to
// tRow[0, G) chunk by chunk; W is zero past F, so is t
template <typename T, int F, int SF, int G>
__device__ __forceinline__ void charMix2(const T *Wt, int l, const T *uu, T *s, T *tRow) {
  T u[8];
  {
    T a[4], b[4];
    ld4<T>(uu, a);
    ld4<T>(uu + 4, b);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      u[i] = a[i];
      u[4 + i] = b[i];
    }
  }
#pragma unroll
  for (int j0 = 0; j0 < F; j0 += 4) {
    T w0[4], w1[4], w2[4], o[4], p[4];
    ld4<T>(rowPtr<T, SF>(Wt, 0, l) + j0, w0);
    ld4<T>(rowPtr<T, SF>(Wt, 1, l) + j0, w1);
    ld4<T>(rowPtr<T, SF>(Wt, 2, l) + j0, w2);
#pragma unroll
    for (int v = 0; v < 4; v++) {
      o[v] = fmaT(u[2], w2[v], fmaT(u[1], w1[v], u[0] * w0[v]));
      p[v] = fmaT(u[5], w2[v], fmaT(u[4], w1[v], u[3] * w0[v]));
    }
#pragma unroll
    for (int v = 0; v < 4; v++)
      if (j0 + v < F) s[j0 + v] = o[v];
    if (j0 + 4 <= G) {
      st4<T>(tRow + j0, p);
    } else {
#pragma unroll
      for (int v = 0; v < 4; v++)
        if (j0 + v < G) tRow[j0 + v] = p[v];
    }
  }
}
// CHAR: only the characteristic factors (the first 108 values: V [9][4], then {U0, U1} [9][8])
template <typename T, int O, int R, int RM, int FA, bool CHAR = false>
__device__ __forceinline__ void issueMixFs(const StepArgs<T> &a, T *buf, int64_t g, int64_t nGroups) {
  using G = Geo<T, O, R, RM>;
  constexpr int E = G::E, FSP = G::FSP, W = 16 / int(sizeof(T)), NC = FSP / W;
  constexpr int NCP = CHAR ? 108 / W : 2 * NC;  // chunks copied per element face
  static_assert(108 % W == 0 && 108 <= 2 * FSP, "factor entries of whole chunks within the pair stride");
  if (g >= nGroups) return;
  if (a.fsLR) {
    for (int i = threadIdx.x; i < E * NCP; i += G::NT) {
      const int eo = i / NCP, k = i % NCP;
      if (g * E + eo >= a.elCount) continue;
      const int64_t e = a.elFirst + g * E + eo;
      cpAsync16(buf + eo * 2 * FSP + k * W, a.fsLR + (e * 4 + FA) * (2 * FSP) + k * W);
    }
  } else {
    for (int i = threadIdx.x; i < E * 2 * 81; i += G::NT) {
      const int eo = i / 162, k = i % 162, w = k / 81, j = k % 81;
      if (g * E + eo >= a.elCount) continue;
      const int64_t e = a.elFirst + g * E + eo;
      int64_t src = (e * 4 + FA) * 81 + j;
      if (w == 1) {
        const int ty = a.faType[e * 4 + FA];
        if (ty == FT_OUTFLOW) continue;
        const int64_t rd = ty == FT_INNER ? int64_t(a.elFaEl[e * 4 + FA]) : e;
        const int rf = ty == FT_INNER ? int(a.fId[e * 4 + FA]) : FA;
        src = ((a.nEl + rd) * 4 + rf) * 81 + j;
      }
      buf[eo * 2 * FSP + w * FSP + j] = T(__ldg(a.fsE + src));
    }
  }
}

// local flux-solver blocks fsE[0] (and fsA[0]) of face FA of group g's elements into buf [E][NFL]
// (Geo::fsLocal)
struct LocalFs {
  double *buf;  // two buffers [2][E][NFL]
  int64_t g, nGroups;
};
template <typename T, int O, int R, int RM, int FA>
__device__ __forceinline__ void issueLocalFs(const StepArgs<T> &a, double *buf, int64_t g, int64_t nGroups) {
  using G = Geo<T, O, R, RM>;
  constexpr int E = G::E, NFL = G::NFL;
  if (g >= nGroups) return;
  for (int i = threadIdx.x; i < E * NFL; i += G::NT) {
    const int eo = i / NFL, j = i % NFL;
    if (g * E + eo >= a.elCount) continue;
    const int64_t e = a.elFirst + g * E + eo;
    cpAsync8(buf + i, j < 81 ? a.fsE + (e * 4 + FA) * 81 + j : a.fsA + (e * 4 + FA) * 54 + (j - 81));
  }
}

// element coefficients of group g's elements into buf [E][NCO]: star [3][24], starA [3][9],
// srcA [RM][12] (Geo::coefSmem)
template <typename T, int O, int R, int RM>
__device__ __forceinline__ void issueCoef(const StepArgs<T> &a, double *buf, int64_t g, int64_t nGroups) {
  using G = Geo<T, O, R, RM>;
  constexpr int E = G::E, NCO = G::NCO;
  if (g >= nGroups) return;
  for (int i = threadIdx.x; i < E * NCO; i += G::NT) {
    const int eo = i / NCO, j = i % NCO;
    if (g * E + eo >= a.elCount) continue;
    const int64_t e = a.elFirst + g * E + eo;
    cpAsync8(buf + i, j < 72   ? a.starE + e * 72 + j
                      : j < 99 ? a.starA + e * 27 + (j - 72)
                               : a.srcA + e * (RM * 12) + (j - 99));
  }
}

// face connectivity of one element (all four faces): the face slot each face gathers from
// (neighbour * 4 + its face id, or a compact LTS slot * 4 + face id), and one byte per face for the
// buffer (LTS relation), the vertex id and the face type
struct FaceMeta {
  int32_t src[4];
  uint32_t rel, vi, ty;
  template <typename T>
  __device__ __forceinline__ void load(const StepArgs<T> &a, int64_t e, bool valid) {
    if (valid) {
      const int4 n = __ldg(reinterpret_cast<const int4 *>(a.elFaEl) + e);
      const uint32_t fo = __ldg(reinterpret_cast<const uint32_t *>(a.fId) + e);
      vi = __ldg(reinterpret_cast<const uint32_t *>(a.vId) + e);
      ty = __ldg(reinterpret_cast<const uint32_t *>(a.faType) + e);
      rel = a.ltsRel ? __ldg(reinterpret_cast<const uint32_t *>(a.ltsRel) + e) : 0u;
      const int32_t ne[4] = {n.x, n.y, n.z, n.w};
#pragma unroll
      for (int f = 0; f < 4; f++) {
        int32_t slotEl = ne[f];
        const int rf = (rel >> (8 * f)) & 0xff;
        if (((ty >> (8 * f)) & 0xff) == FT_INNER && rf != LTS_EQ)
          slotEl = __ldg((rf == LTS_GT ? a.sumIdx : a.halfIdx) + ne[f]);
        src[f] = slotEl * 4 + int32_t((fo >> (8 * f)) & 0xff);
      }
    } else {
      src[0] = src[1] = src[2] = src[3] = 0;
      rel = vi = 0;
      ty = 0x02020202u;  // outflow on every face: nothing to gather or add
    }
  }
  __device__ __forceinline__ int type(int f) const { return (ty >> (8 * f)) & 0xff; }
  __device__ __forceinline__ int relation(int f) const { return (rel >> (8 * f)) & 0xff; }
  __device__ __forceinline__ int vert(int f) const { return (vi >> (8 * f)) & 0xff; }
};

// the reflection (OriMul index) taking the neighbour's projection at its face fo (in that face's
// basis) to this element's face FA basis, for the neighbour's vertex id at FA (kFacePerm)
template <int O, int FA>
__device__ __forceinline__ int neighOri(const FaceMeta &m) {
  return kFacePerm[O - 2][m.src[FA] & 3][FA][m.vert(FA)];
}


// the neighbour flux of face FA through pre-mixed projections read straight from global memory
// (this warp's quantity row, this lane's run): the arithmetic of the neighbour kernel's
// neighApplyMixed, for kernels that fold a pending neighbour step into their DOF rows
template <typename T, int O, int R, int RM, int FA>
__device__ __forceinline__ void neighFluxFace(const T *faceIn, const FaceMeta &m, int64_t e, int q, int r,
                                              bool valid, T *acc) {
  using G = Geo<T, O, R, RM>;
  constexpr int F = G::F;
  const int ty = m.type(FA);
  if (!valid || ty == FT_OUTFLOW || q >= 9) return;
  const int64_t src = ty == FT_INNER ? int64_t(m.src[FA]) : e * 4 + FA;
  T x[F];
  ldRowG<T, F>(gRow<T, R, G::GF>(faceIn, src, 9, q, r), x, true);
  if (ty == FT_INNER) {
    T o[F];
#pragma unroll
    for (int j = 0; j < F; j++) o[j] = T(0);
    const int v = neighOri<O, FA>(m);
    if (v == 0)
      OriMul<O, 0>::template run<T>(x, o);
    else if (v == 1)
      OriMul<O, 1>::template run<T>(x, o);
    else
      OriMul<O, 2>::template run<T>(x, o);
    FluxTMul<O, FA>::template run<T>(o, acc);
  } else {
    FluxTMul<O, FA>::template run<T>(x, acc);
  }
}
template <typename T, int O, int R, int RM>
__device__ __forceinline__ void neighFluxDirect(const StepArgs<T> &a, const T *faceIn, int64_t e, int q, int r,
                                                bool valid, T *acc) {
  FaceMeta m;
  m.load(a, e, valid);
  neighFluxFace<T, O, R, RM, 0>(faceIn, m, e, q, r, valid, acc);
  neighFluxFace<T, O, R, RM, 1>(faceIn, m, e, q, r, valid, acc);
  neighFluxFace<T, O, R, RM, 2>(faceIn, m, e, q, r, valid, acc);
  neighFluxFace<T, O, R, RM, 3>(faceIn, m, e, q, r, valid, acc);
}

// ------------------------------------------------------------------------------------------------
// local step: CK, volume, local surface, face projections (AderDg::local, AderDg.hpp:338-534)
// ------------------------------------------------------------------------------------------------
// TAIL: a barrier after the quantity mix, before the face tile is written again (not needed when
// consecutive faces alternate between two tiles)
// LTS: 0 none, 1 the two-step sums of elements with a larger neighbour, 2 also the half-step
// projections of elements with a smaller neighbour (needs TIh)
// pre-mixed projections (LTS 0, Geo::premix): S0alt is a tile free for this warp's own rows,
// through which the mixed projection leaves as coalesced stores; mf the flux-solver buffers
// CHAR: the pre-mixed projections mix through the characteristic factors in mf.buf (Geo::charMix)
template <typename T, int O, int R, int RM, int FA, int LTS = 0, bool TAIL = true, bool CHAR = false>
__device__ __forceinline__ void localFace(const StepArgs<T> &a, const T *TI, T *S0, int q, int l, int64_t e,
                                          int r, bool valid, T *acc, T *upA, const T *TIh = nullptr,
                                          T *S0alt = nullptr, const MixFs<T> &mf = MixFs<T>{nullptr, 0, 0},
                                          T *Sh = nullptr, const LocalFs &lf = LocalFs{nullptr, 0, 0}) {
  using G = Geo<T, O, R, RM>;
  constexpr int F = G::F, SF = G::SF, SB = G::SB;
  constexpr bool PM = LTS == 0 ? G::premix : G::premixLts;
  // pre-mixing LTS mode 2: the half-step projection rows of elements with a smaller neighbour go
  // through a face tile of their own (two, alternating with the faces) for their quantity mix
  T *ShF = (PM && LTS == 2) ? Sh + (FA % 2) * G::nS0 : nullptr;
  const bool half = LTS == 2 && valid && (a.ltsFlags[e] & LTS_HAS_SMALLER);
  T s[F];
  if (q < 9) {
#pragma unroll
    for (int j = 0; j < F; j++) s[j] = T(0);
    FluxLMul<O, FA>::template run<T>(OwnRow<T>{rowPtr<T, SB>(TI, q, l)}, s);
    {
      // the row padded to GF with zeros (for the coalesced stores of the warp's rows)
      T *p = rowPtr<T, SF>(S0, q, l);
      stRow<T, F>(p, s);
#pragma unroll
      for (int j = F; j < G::GF; j++) p[j] = T(0);
    }
    if constexpr (!PM) {
      __syncwarp();
      if (valid)
        storeRowsCoalesced<T, R, G::GF, SF>(S0, a.face + ((e * 4 + FA) * 9 + q) * int64_t(R * G::GF), q, l / R,
                                            l % R);
    }
    if constexpr (PM && LTS == 2) {
      if (half) {
        T h[F];
#pragma unroll
        for (int j = 0; j < F; j++) h[j] = T(0);
        FluxLMul<O, FA>::template run<T>(OwnRow<T>{rowPtr<T, SB>(TIh, q, l)}, h);
        stRow<T, F>(rowPtr<T, SF>(ShF, q, l), h);
      }
    }
    if constexpr (LTS && !PM) {
      if (valid) {
        const int fl = a.ltsFlags[e];
        if (fl & LTS_HAS_LARGER) {
          // face projection of the time integral summed over the two steps of a pair
          T *p = gRow<T, R, G::GF>(a.faceSum, int64_t(a.sumIdx[e]) * 4 + FA, 9, q, r);
          T v[F];
          ldRowG<T, F>(p, v, !a.firstTs);
#pragma unroll
          for (int j = 0; j < F; j++) v[j] += s[j];
          stRowG<T, F>(p, v);
        }
        if (LTS == 2 && (fl & LTS_HAS_SMALLER)) {
          // face projections of the integrals over [0, dt/2] and [dt/2, dt]
          T h[F];
#pragma unroll
          for (int j = 0; j < F; j++) h[j] = T(0);
          FluxLMul<O, FA>::template run<T>(OwnRow<T>{rowPtr<T, SB>(TIh, q, l)}, h);
          const int64_t slot = int64_t(a.halfIdx[e]) * 4 + FA;
          stRowG<T, F>(gRow<T, R, G::GF>(a.faceHalf1, slot, 9, q, r), h);
#pragma unroll
          for (int j = 0; j < F; j++) h[j] = s[j] - h[j];
          stRowG<T, F>(gRow<T, R, G::GF>(a.faceHalf2, slot, 9, q, r), h);
        }
      }
    }
  }
  if constexpr (PM) {
    constexpr int E = G::E, FSP = G::FSP;
    // this face's flux-solver blocks (issued one face ahead) for every thread after the barrier
    cpAsyncWait<0>();
    const int ty = valid ? a.faType[e * 4 + FA] : FT_OUTFLOW;
    __syncthreads();
    // the next face's blocks into the other buffer, whose readers (two faces back) all passed the
    // barrier; after the last face the next group's first
    if constexpr (FA < 3)
      issueMixFs<T, O, R, RM, FA + 1, CHAR>(a, mf.buf + ((FA + 1) % 2) * (E * 2 * FSP), mf.g, mf.nGroups);
    else
      issueMixFs<T, O, R, RM, 0, CHAR>(a, mf.buf, mf.g + gridDim.x, mf.nGroups);
    cpAsyncCommit();
    const T *fbE = mf.buf + (FA % 2) * (E * 2 * FSP) + (l / R) * (2 * FSP);
    static_assert(!CHAR || (LTS == 0 ? G::charMix : G::charMixLts),
                  "characteristic mix: configurations with room for its rows");
    // the mixed projection t of this warp's row: through the characteristic rows of all warps'
    // projections (CHAR; it leaves through this warp's own row of S0, which no warp reads after the
    // second barrier), else through the pair blocks (through the warp's row of S0alt)
    T *tile = CHAR ? S0 : S0alt;
    T *tRow = rowPtr<T, SF>(tile, q, l);
    T fr1[CHAR ? 1 : 9];
    if constexpr (CHAR) {
      charRows<T, F, SF>(S0, fbE, q, l, mf.w);
      // with half-step projections (LTS 2) their characteristic rows too
      if constexpr (LTS == 2) charRows<T, F, SF>(ShF, fbE, q, l, mf.wh);
      __syncthreads();
      charMix2<T, F, SF, G::GF>(mf.w, l, fbE + 36 + q * 8, s, tRow);
    } else {
      T fr[9];
#pragma unroll
      for (int i = 0; i < 9; i++) {
        fr[i] = fbE[q * 9 + i];
        fr1[i] = fbE[FSP + q * 9 + i];
      }
      faceMix2<T, F, SF, G::GF>(S0, l, fr, fr1, s, tRow);
    }
    __syncwarp();
    if (ty != FT_OUTFLOW)
      storeRowsCoalesced<T, R, G::GF, SF>(tile, a.face + ((e * 4 + FA) * 9 + q) * int64_t(R * G::GF), q, l / R,
                                          l % R);
    if constexpr (LTS) {
      // the LTS buffers of the (pre-mixed) projection t: its sum over the two steps of a pair for a
      // larger neighbour, the half-step projections (mixed alike) for a smaller one
      if (valid) {
        const int fl = a.ltsFlags[e];
        if (fl & LTS_HAS_LARGER) {
          T *p = gRow<T, R, G::GF>(a.faceSum, int64_t(a.sumIdx[e]) * 4 + FA, 9, q, r);
          T v[F], t[F];
          ldRowG<T, F>(p, v, !a.firstTs);
          ldRow<T, F>(tRow, t);
#pragma unroll
          for (int j = 0; j < F; j++) v[j] += t[j];
          stRowG<T, F>(p, v);
        }
        if (LTS == 2 && half) {
          T h[F], t[F];
          if constexpr (CHAR)
            charMixOne<T, F, SF>(mf.wh, l, fbE + 36 + q * 8 + 3, h);
          else
            faceMix<T, F, SF>(ShF, l, fr1, h);
          const int64_t slot = int64_t(a.halfIdx[e]) * 4 + FA;
          stRowG<T, F>(gRow<T, R, G::GF>(a.faceHalf1, slot, 9, q, r), h);
          ldRow<T, F>(tRow, t);
#pragma unroll
          for (int j = 0; j < F; j++) h[j] = t[j] - h[j];
          stRowG<T, F>(gRow<T, R, G::GF>(a.faceHalf2, slot, 9, q, r), h);
        }
      }
    }
    // the next face writes this warp's rows of the tile again
    __syncwarp();
    FluxTMul<O, FA>::template run<T>(s, acc);
    if constexpr (TAIL) __syncthreads();
    return;
  }
  // flux-solver row of this thread (elastic 9x9 or anelastic 6x9): from the buffer filled one face
  // ahead (Geo::fsLocal), else loaded before the barrier
  T fr[9];
  if constexpr (LTS == 0 && G::fsLocal) {
    constexpr int E = G::E, NFL = G::NFL;
    cpAsyncWait<0>();
    __syncthreads();
    // the next face's blocks into the other buffer, whose readers (one face back) all passed the
    // barrier; after the last face the next group's first
    if constexpr (FA < 3)
      issueLocalFs<T, O, R, RM, FA + 1>(a, lf.buf + ((FA + 1) % 2) * (E * NFL), lf.g, lf.nGroups);
    else
      issueLocalFs<T, O, R, RM, 0>(a, lf.buf, lf.g + gridDim.x, lf.nGroups);
    cpAsyncCommit();
    const double *fp = lf.buf + (FA % 2) * (E * NFL) + (l / R) * NFL + (q < 9 ? q * 9 : 81 + (q - 9) * 9);
#pragma unroll
    for (int i = 0; i < 9; i++) fr[i] = valid ? T(fp[i]) : T(0);
  } else {
    if (q < 9) {
      const double *fp = a.fsE + ((e * 4 + FA) * 81 + q * 9);
#pragma unroll
      for (int i = 0; i < 9; i++) fr[i] = valid ? T(__ldg(fp + i)) : T(0);
    } else if constexpr (RM > 0) {
      const double *fp = a.fsA + ((e * 4 + FA) * 54 + (q - 9) * 9);
#pragma unroll
      for (int i = 0; i < 9; i++) fr[i] = valid ? T(__ldg(fp + i)) : T(0);
    }
    __syncthreads();
  }
  faceMix<T, F, SF>(S0, l, fr, s);
  if (q < 9)
    FluxTMul<O, FA>::template run<T>(s, acc);
  else if constexpr (RM > 0)
    FluxTMul<O, FA>::template run<T>(s, upA);
  if constexpr (TAIL) __syncthreads();
}

// quantity mix of face FA's tile with this thread's flux-solver row fp, lifted into acc (elastic
// rows) or upA (anelastic rows)
template <typename T, int O, int R, int RM, int FA>
__device__ __forceinline__ void faceLift(const T *tile, const double *fp, int q, int l, bool valid, T *acc,
                                         T *upA) {
  using G = Geo<T, O, R, RM>;
  constexpr int F = G::F, SF = G::SF;
  T fr[9];
#pragma unroll
  for (int i = 0; i < 9; i++) fr[i] = valid ? T(fp[i]) : T(0);
  T s[F];
  faceMix<T, F, SF>(tile, l, fr, s);
  if (q < 9)
    FluxTMul<O, FA>::template run<T>(s, acc);
  else if constexpr (RM > 0)
    FluxTMul<O, FA>::template run<T>(s, upA);
}

// the four local faces with the projections spread over all warps (Geo::projSplit, attenuation,
// GTS): elastic warp q projects its row onto faces 0 and 1, anelastic warp s takes tasks 18 + s,
// 24 + s and 30 + s of the 18 (face 2 and 3) row projections (task t: row t % 9, face t / 9); each
// projection goes to its face tile and to the face buffer. A barrier after every warp's first task
// keeps the face-1 projections out of X until all DOF rows there have been read; after one more
// barrier every warp mixes and lifts its own row for the four faces (fs4: the flux-solver blocks of
// the four faces). A barrier at the end orders the tiles' readers before X is written again.
template <typename T, int O, int R, int RM>
__device__ __forceinline__ void facesSplit(const StepArgs<T> &a, const T *TI, T *const (&tiles)[4],
                                           const double *const (&fs4)[4], int q, int l, int64_t e, bool valid,
                                           T *acc, T *upA) {
  using G = Geo<T, O, R, RM>;
  constexpr int F = G::F, SF = G::SF, SB = G::SB, NFL = G::NFL;
  const int eo = l / R, r = l % R;
  const int nTasks = q < 9 ? 2 : 3;
  for (int j = 0; j < nTasks; j++) {
    // face 1's tile is X, where the elastic warps have just reloaded and read their DOF rows (row
    // stride SB, not SF): every warp passes this barrier after its first task, so no projection
    // reaches X while another warp's DOF rows are still arriving there or being read
    if (j == 1) __syncthreads();
    const int t = q < 9 ? q + 9 * j : 18 + (q - 9) + 6 * j;
    const int row = t % 9, fa = t / 9;
    T s[F];
#pragma unroll
    for (int i = 0; i < F; i++) s[i] = T(0);
    const OwnRow<T> src{rowPtr<T, SB>(TI, row, l)};
    if (fa == 0)
      FluxLMul<O, 0>::template run<T>(src, s);
    else if (fa == 1)
      FluxLMul<O, 1>::template run<T>(src, s);
    else if (fa == 2)
      FluxLMul<O, 2>::template run<T>(src, s);
    else
      FluxLMul<O, 3>::template run<T>(src, s);
    T *tile = fa == 0 ? tiles[0] : fa == 1 ? tiles[1] : fa == 2 ? tiles[2] : tiles[3];
    T *p = rowPtr<T, SF>(tile, row, l);
    stRow<T, F>(p, s);
#pragma unroll
    for (int i = F; i < G::GF; i++) p[i] = T(0);
    __syncwarp();
    if (valid)
      storeRowsCoalesced<T, R, G::GF, SF>(tile, a.face + ((e * 4 + fa) * 9 + row) * int64_t(R * G::GF), row, eo,
                                          r);
  }
  cpAsyncWait<0>();
  __syncthreads();
  const int fo = (l / R) * NFL + (q < 9 ? q * 9 : 81 + (q - 9) * 9);
  faceLift<T, O, R, RM, 0>(tiles[0], fs4[0] + fo, q, l, valid, acc, upA);
  faceLift<T, O, R, RM, 1>(tiles[1], fs4[1] + fo, q, l, valid, acc, upA);
  faceLift<T, O, R, RM, 2>(tiles[2], fs4[2] + fo, q, l, valid, acc, upA);
  faceLift<T, O, R, RM, 3>(tiles[3], fs4[3] + fo, q, l, valid, acc, upA);
  __syncthreads();
}

// LTS as in localFace; mode 2 keeps the half-step integral in one more tile (one CTA per SM), mode
// 1 runs on the elements of a time group without a smaller neighbour
// FUSED (GTS, pre-mixing configurations): the previous step's neighbour fluxes (a.faceIn, when
// pending) are added to each group's DOF rows first, and the completed rows stored back
template <typename T, int O, int R, int RM, int LTS, bool FUSED = false, bool CHAR = false>
__global__ void __launch_bounds__(Geo<T, O, R, RM>::NT, LTS == 2 ? 1 : Geo<T, O, R, RM>::minCtasLocal)
    kLocal(StepArgs<T> a) {
  using G = Geo<T, O, R, RM>;
  constexpr int B = G::B, E = G::E, SB = G::SB;
  extern __shared__ __align__(16) unsigned char smem[];
  T *X = reinterpret_cast<T *>(smem);
  T *XA = X + G::nX + G::nTI;
  // see Geo: time integrals in shared memory (TI behind X, TIA behind XA, face tiles reuse X) or
  // in registers (copied into X / XA after the recursion, face tiles behind X); with LTS the
  // half-step integral TIh behind everything
  // AS (G::asyncLocal): the DOF rows arrive by cp.async (the next group's into this warp's TI rows
  // at the end of a group, the current group's into X again after the recursion) and the faces
  // alternate between a separate face tile (even faces) and X (odd faces): one barrier per face
  // instead of two (the last face keeps both)
  constexpr bool AS = G::asyncLocal;
  T *TI = G::tiSmem ? X + G::nX : X;
  T *TIA = G::tiSmem ? XA + G::nXA : XA;
  T *S0 = AS ? TIA + G::nTIA : (G::tiSmem ? X : X + G::nX);
  T *TIh = LTS == 2 ? reinterpret_cast<T *>(smem + G::smemLocal) : nullptr;
  // pre-mixed face projections: flux-solver buffers behind the face tile (behind TIh with LTS
  // mode 2, followed by its two half-step face tiles)
  constexpr bool PM = LTS == 0 ? G::premix : G::premixLts;
  constexpr size_t fsOff = G::smemLocal + (LTS == 2 ? G::nX * sizeof(T) : 0);
  T *fsb = PM ? reinterpret_cast<T *>(smem + fsOff) : nullptr;
  T *Sh = (PM && LTS == 2) ? reinterpret_cast<T *>(smem + fsOff + G::premixBytes) : nullptr;
  // local flux-solver buffers one face ahead (Geo::fsLocal) in the same place
  constexpr bool FL = LTS == 0 && G::fsLocal;
  double *fsl = FL ? reinterpret_cast<double *>(smem + G::smemLocal) : nullptr;
  // AP (GTS): the anelastic rows arrive by cp.async too (the next group's into this warp's TIA
  // rows at the end of a group, the current group's into its XA rows after the recursion, for the
  // update)
  constexpr bool AP = AS && RM > 0 && LTS == 0;
  // element coefficients one group ahead (Geo::coefSmem), behind the flux-solver buffers
  constexpr bool CS = FL && G::coefSmem;
  double *coefBuf = CS ? fsl + 2 * E * G::NFL : nullptr;
  // anelastic source terms from the anelastic warps (Geo::srcSplit)
  constexpr bool SS = CS && G::srcSplit;
  T *srcBuf = SS ? reinterpret_cast<T *>(smem + G::srcOff) : nullptr;
  // projections spread over all warps (Geo::projSplit): the flux-solver blocks of the four faces of
  // a group arrive together, one group ahead
  constexpr bool PSP = SS && G::projSplit;
  double *fsExtra = PSP ? reinterpret_cast<double *>(smem + G::fsExtraOff) : nullptr;
  const int q = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int eo = l / R, r = l % R;
  const int64_t nGroups = (a.elCount + E - 1) / E;
  const T dt0 = T(a.dt);
  if constexpr (AS) {
    // the first group's DOF rows (and flux-solver blocks of its first face)
    const int64_t g0 = blockIdx.x;
    if (q < 9 && g0 < nGroups && g0 * E + eo < a.elCount)
      copyDofRows<T, R, G::GB, SB>(TI, a.dofsE, a.elFirst + g0 * E + eo, q, eo, r);
    if constexpr (AP) {
      if (q >= 9 && g0 < nGroups && g0 * E + eo < a.elCount)
#pragma unroll
        for (int m = 0; m < RM; m++)
          copyRows<T, R, G::GB, SB>(TIA, a.dofsA, a.elFirst + g0 * E + eo, RM * 6, m * 6 + q - 9, eo, r);
    }
    if constexpr (PM) issueMixFs<T, O, R, RM, 0, CHAR>(a, fsb, g0, nGroups);
    if constexpr (FL) issueLocalFs<T, O, R, RM, 0>(a, fsl, g0, nGroups);
    if constexpr (PSP) {
      issueLocalFs<T, O, R, RM, 1>(a, fsl + E * G::NFL, g0, nGroups);
      issueLocalFs<T, O, R, RM, 2>(a, fsExtra, g0, nGroups);
      issueLocalFs<T, O, R, RM, 3>(a, fsExtra + E * G::NFL, g0, nGroups);
    }
    if constexpr (CS) issueCoef<T, O, R, RM>(a, coefBuf, g0, nGroups);
    cpAsyncCommit();
  }
  for (int64_t g = blockIdx.x; g < nGroups; g += gridDim.x) {
    const int64_t e = a.elFirst + g * E + eo;
    const bool valid = g * E + eo < a.elCount;
    const int64_t ev = valid ? e : 0;
    const T dt = (LTS == 0 && a.grpDt) ? T(a.grpDt[g]) : dt0;
    T tIr[G::tiSmem ? 1 : B];
    T tIAr[(G::tiSmem || RM == 0) ? 1 : RM][B];
    // DOFs -> X, dt * DOFs -> TI (and the anelastic counterparts)
    if (q < 9) {
      T v[B];
      if constexpr (AS) {
        cpAsyncWait<0>();
        __syncwarp();
        if (valid)
          ldRow<T, B>(rowPtr<T, SB>(TI, q, l), v);
        else
#pragma unroll
          for (int n = 0; n < B; n++) v[n] = T(0);
        if constexpr (FUSED) {
          if (a.faceIn) {
            neighFluxDirect<T, O, R, RM>(a, a.faceIn, ev, q, r, valid, v);
            // the completed rows back to the DOFs (the volume integral reads them again)
            T *p = rowPtr<T, SB>(X, q, l);
            stRow<T, B>(p, v);
#pragma unroll
            for (int n = B; n < G::GB; n++) p[n] = T(0);
            __syncwarp();
            if (valid)
              storeRowsCoalesced<T, R, G::GB, SB>(X, a.dofsE + (e * 9 + q) * int64_t(R * G::GB), q, eo, r);
            __syncwarp();
          }
        }
        stRow<T, B>(rowPtr<T, SB>(X, q, l), v);
      } else {
        ldRowG<T, B>(gRow<T, R, G::GB>(a.dofsE, ev, 9, q, r), v, valid);
        stRow<T, B>(rowPtr<T, SB>(X, q, l), v);
      }
      if constexpr (LTS == 2) {
        T h[B];
#pragma unroll
        for (int n = 0; n < B; n++) h[n] = (dt * T(0.5)) * v[n];
        stRow<T, B>(rowPtr<T, SB>(TIh, q, l), h);
      }
#pragma unroll
      for (int n = 0; n < B; n++) v[n] = dt * v[n];
      if constexpr (G::tiSmem)
        stRow<T, B>(rowPtr<T, SB>(TI, q, l), v);
      else {
#pragma unroll
        for (int n = 0; n < B; n++) tIr[n] = v[n];
      }
    } else if constexpr (RM > 0) {
      const int s = q - 9;
      if constexpr (AP) {
        cpAsyncWait<0>();
        __syncwarp();
      }
#pragma unroll
      for (int m = 0; m < RM; m++) {
        T v[B];
        if constexpr (AP) {
          if (valid)
            ldRow<T, B>(rowPtr<T, SB>(TIA, m * 6 + s, l), v);
          else
#pragma unroll
            for (int n = 0; n < B; n++) v[n] = T(0);
        } else {
          ldRowG<T, B>(gRow<T, R, G::GB>(a.dofsA, ev, RM * 6, m * 6 + s, r), v, valid);
        }
        stRow<T, B>(rowPtr<T, SB>(XA, m * 6 + s, l), v);
#pragma unroll
        for (int n = 0; n < B; n++) v[n] = dt * v[n];
        if constexpr (G::tiSmem)
          stRow<T, B>(rowPtr<T, SB>(TIA, m * 6 + s, l), v);
        else {
#pragma unroll
          for (int n = 0; n < B; n++) tIAr[m][n] = v[n];
        }
      }
    }
    ElemCoef<T, RM> c;
    if constexpr (CS) {
      // every thread waited for its copies above; the barrier makes all of them visible
      __syncthreads();
      const double *cb = coefBuf + eo * G::NCO;
      c.template loadFrom<false, SS>(cb, cb + 72, cb + 99, valid, q);
    } else {
      c.load(a, ev, valid, q);
      __syncthreads();
    }
    // Cauchy-Kowalevski (TimePredVanilla::ck, TimePredVanilla.hpp:200-306)
    ckAll<T, O, R, RM, 1, LTS == 2, G::ckPingPong>(X, TI, XA, TIA, q, l, c, a.omega, dt, dt, tIr, tIAr, TIh,
                                              dt * T(0.5), S0, srcBuf);
    if constexpr (!G::tiSmem) {
      if (q < 9) {
        stRow<T, B>(rowPtr<T, SB>(X, q, l), tIr);
      } else if constexpr (RM > 0) {
        const int s = q - 9;
#pragma unroll
        for (int m = 0; m < RM; m++) stRow<T, B>(rowPtr<T, SB>(XA, m * 6 + s, l), tIAr[m]);
      }
      __syncthreads();
    }
    if (a.tDofs && valid && q < 9) {
      T t[B];
      ldRow<T, B>(rowPtr<T, SB>(TI, q, l), t);
      stRowG<T, B>(gRow<T, R, G::GB>(a.tDofs, e, 9, q, r), t);
    }
    // volume integral (VolIntVanilla::apply, VolIntVanilla.hpp:189-241)
    T acc[B];
    T upA[RM ? B : 1];
    if (q < 9) {
      if constexpr (AS) {
        // the DOF rows again (X is free after the recursion; L2-resident since the group start)
        if (valid) copyDofRows<T, R, G::GB, SB>(X, a.dofsE, e, q, eo, r);
        cpAsyncCommit();
        cpAsyncWait<0>();
        __syncwarp();
        if (valid)
          ldRow<T, B>(rowPtr<T, SB>(X, q, l), acc);
        else
#pragma unroll
          for (int n = 0; n < B; n++) acc[n] = T(0);
      } else {
        ldRowG<T, B>(gRow<T, R, G::GB>(a.dofsE, ev, 9, q, r), acc, valid);
      }
      Mix3<T, SB> z{rowPtr<T, SB>(TI, c.cols[0], l), rowPtr<T, SB>(TI, c.cols[1], l),
                    rowPtr<T, SB>(TI, c.cols[2], l), c.cs};
      VolMul<O>::template run<T>(z, acc);
      if constexpr (RM > 0 && !SS)
        if (q < 6) addSrc<T, B, SB, RM>(c, TIA, l, acc);
    } else if constexpr (RM > 0) {
      // (SS: the source terms of the time integrals, added to the elastic rows after the faces)
      if constexpr (SS) srcShare<T, B, SB, RM>(c, TIA, l, q - 9, srcBuf);
      if constexpr (AP) {
        // this group's anelastic rows into this warp's XA rows (free after the recursion)
        if (valid)
#pragma unroll
          for (int m = 0; m < RM; m++) copyRows<T, R, G::GB, SB>(XA, a.dofsA, e, RM * 6, m * 6 + q - 9, eo, r);
        cpAsyncCommit();
      }
#pragma unroll
      for (int n = 0; n < B; n++) {
        acc[n] = T(0);
        upA[n] = T(0);
      }
      Mix2<T, SB> z{rowPtr<T, SB>(TI, 6 + c.colsA[0], l), rowPtr<T, SB>(TI, 6 + c.colsA[1], l), c.ca};
      VolMul<O>::template run<T>(z, acc);
    }
    // local surface integral (SurfIntVanilla::local, SurfIntVanilla.hpp:212-262) + face projections
    if constexpr (AS) {
      // characteristic rows: behind the face rows of X, or behind the flux-solver buffers
      T *const wTile =
          CHAR ? (G::wInX ? X + G::nS0 : reinterpret_cast<T *>(smem + G::smemLocal + G::premixBytes)) : nullptr;
      const MixFs<T> mf{fsb, g, nGroups, wTile, (CHAR && LTS == 2) ? X + G::nS0 + G::nW : nullptr};
      const LocalFs lf{fsl, g, nGroups};
      if constexpr (PSP) {
        T *const tiles[4] = {S0, X, reinterpret_cast<T *>(smem + G::tilesOff),
                             reinterpret_cast<T *>(smem + G::tilesOff) + G::nS0};
        const double *const fs4[4] = {fsl, fsl + E * G::NFL, fsExtra, fsExtra + E * G::NFL};
        facesSplit<T, O, R, RM>(a, TI, tiles, fs4, q, l, ev, valid, acc, upA);
        // the next group's flux-solver blocks (every thread read this group's before the barrier)
        const int64_t gn = g + gridDim.x;
        issueLocalFs<T, O, R, RM, 0>(a, fsl, gn, nGroups);
        issueLocalFs<T, O, R, RM, 1>(a, fsl + E * G::NFL, gn, nGroups);
        issueLocalFs<T, O, R, RM, 2>(a, fsExtra, gn, nGroups);
        issueLocalFs<T, O, R, RM, 3>(a, fsExtra + E * G::NFL, gn, nGroups);
        cpAsyncCommit();
      } else {
        localFace<T, O, R, RM, 0, LTS, false, CHAR>(a, TI, S0, q, l, ev, r, valid, acc, upA, TIh, X, mf, Sh, lf);
        localFace<T, O, R, RM, 1, LTS, false, CHAR>(a, TI, X, q, l, ev, r, valid, acc, upA, TIh, S0, mf, Sh, lf);
        localFace<T, O, R, RM, 2, LTS, false, CHAR>(a, TI, S0, q, l, ev, r, valid, acc, upA, TIh, X, mf, Sh, lf);
        // the barrier after the last face orders its readers of X (and of the characteristic rows
        // behind its face rows) before the next group writes X
        localFace<T, O, R, RM, 3, LTS, true, CHAR>(a, TI, X, q, l, ev, r, valid, acc, upA, TIh, S0, mf, Sh, lf);
      }
      if constexpr (SS)
        if (q < 6) addSrcRows<T, B, SB>(srcBuf, q, l, acc);
      if constexpr (CS) {
        // the next group's coefficients (every thread read this group's before the barriers above)
        issueCoef<T, O, R, RM>(a, coefBuf, g + gridDim.x, nGroups);
        cpAsyncCommit();
      }
    } else {
      localFace<T, O, R, RM, 0, LTS>(a, TI, S0, q, l, ev, r, valid, acc, upA, TIh);
      localFace<T, O, R, RM, 1, LTS>(a, TI, S0, q, l, ev, r, valid, acc, upA, TIh);
      localFace<T, O, R, RM, 2, LTS>(a, TI, S0, q, l, ev, r, valid, acc, upA, TIh);
      localFace<T, O, R, RM, 3, LTS>(a, TI, S0, q, l, ev, r, valid, acc, upA, TIh);
    }
    if constexpr (G::tiSmem) {
      // the updated rows through the (now unused) time-integral tile, stored coalesced
      if (q < 9) {
        T *p = rowPtr<T, SB>(TI, q, l);
        stRow<T, B>(p, acc);
#pragma unroll
        for (int n = B; n < G::GB; n++) p[n] = T(0);
        __syncwarp();
        if (valid)
          storeRowsCoalesced<T, R, G::GB, SB>(TI, a.dofsE + (e * 9 + q) * int64_t(R * G::GB), q, eo, r);
        if constexpr (AS) {
          // the next group's DOF rows into this warp's TI rows
          __syncwarp();
          const int64_t gn = g + gridDim.x;
          if (gn < nGroups && gn * E + eo < a.elCount)
            copyDofRows<T, R, G::GB, SB>(TI, a.dofsE, a.elFirst + gn * E + eo, q, eo, r);
        }
      }
      if constexpr (AS) cpAsyncCommit();
    }
    if constexpr (AP) {
      if (q >= 9) {
        cpAsyncWait<0>();
        __syncwarp();
      }
    }
    if (valid) {
      if (q < 9) {
        if constexpr (!G::tiSmem) stRowG<T, B>(gRow<T, R, G::GB>(a.dofsE, e, 9, q, r), acc);
      } else if constexpr (RM > 0) {
        // dofsA_m += omega_m * (Psi_vol - tIntA_m) + omega_m * upA_surf
        const int s = q - 9;
#pragma unroll
        for (int m = 0; m < RM; m++) {
          const T om = T(a.omega[m]);
          T ti[B];
          ldRow<T, B>(rowPtr<T, SB>(TIA, m * 6 + s, l), ti);
          T *dst = gRow<T, R, G::GB>(a.dofsA, e, RM * 6, m * 6 + s, r);
          T v[B];
          if constexpr (AP)
            ldRow<T, B>(rowPtr<T, SB>(XA, m * 6 + s, l), v);
          else
            ldRowG<T, B>(dst, v, true);
#pragma unroll
          for (int n = 0; n < B; n++) {
            v[n] = fmaT(om, acc[n] - ti[n], v[n]);
            v[n] = fmaT(om, upA[n], v[n]);
          }
          stRowG<T, B>(dst, v);
        }
      }
    }
    if constexpr (AP) {
      // the next group's anelastic rows into this warp's TIA rows (read above by their lanes)
      if (q >= 9) {
        __syncwarp();
        const int64_t gn = g + gridDim.x;
        if (gn < nGroups && gn * E + eo < a.elCount)
#pragma unroll
          for (int m = 0; m < RM; m++)
            copyRows<T, R, G::GB, SB>(TIA, a.dofsA, a.elFirst + gn * E + eo, RM * 6, m * 6 + q - 9, eo, r);
        cpAsyncCommit();
      }
    }
  }
  if constexpr (AS) cpAsyncWait<0>();
}

// ------------------------------------------------------------------------------------------------
// neighbour step (AderDg::neigh, AderDg.hpp:553-722)
// ------------------------------------------------------------------------------------------------
// The face rows a CTA reads (the neighbours' face projections, or its own for free-surface faces)
// and the flux-solver blocks are gathered with asynchronous copies (cp.async, no registers held)
// into a ring of NSN shared-memory slots, one slot per (element group, face) item, NSN - 1 items
// ahead of the one being processed. Where a DOF tile fits, the updated DOF rows leave through it as
// coalesced stores and the next group's DOF rows arrive in it asynchronously. Per item: wait for its copies, rotate the neighbour's rows into this element's face
// orientation in place, one CTA barrier, issue the copies of the item NSN - 1 ahead into the slot
// the previous item released, then mix quantities and apply fluxT.

template <typename T, int O, int R, int RM>
struct NeighSlots {
  using G = Geo<T, O, R, RM>;
  static constexpr int E = G::E, SF = G::SF, GF = G::GF, NT = G::NT;
  static constexpr int W = 16 / int(sizeof(T));  // elements per 16-byte chunk
  static constexpr int CPR = GF / W;             // 16-byte chunks per face row
  static constexpr int CPRB = G::GB / W;         // 16-byte chunks per DOF row
  static constexpr int NFS = 81 + (RM ? 54 : 0); // flux-solver doubles per element and face
  static constexpr size_t rowsBytes = (G::nS0 * sizeof(T) + 15) / 16 * 16;
  __device__ __forceinline__ static T *rows(unsigned char *base, int slot) {
    return reinterpret_cast<T *>(base + slot * G::slotNeigh);
  }
  __device__ __forceinline__ static double *fs(unsigned char *base, int slot) {
    return reinterpret_cast<double *>(base + slot * G::slotNeigh + rowsBytes);
  }
  __device__ __forceinline__ static T *dofTile(unsigned char *base) {
    return reinterpret_cast<T *>(base + G::NSN * G::slotNeigh);
  }

  // the DOF rows of group g into the tile behind the slots (warp q copies quantity q's rows)
  __device__ __forceinline__ static void issueDofs(const StepArgs<T> &a, unsigned char *base, int q, int l,
                                                   int64_t g, bool groupValid) {
    if constexpr (G::dofTile) {
      const int eo = l / R, r = l % R;
      const int64_t e = a.elFirst + g * E + eo;
      if (!groupValid || q >= 9 || g * E + eo >= a.elCount) return;
      const T *blk = a.dofsE + (e * 9 + q) * int64_t(R * G::GB);
      T *dst = dofTile(base) + (q * 32 + eo * R) * G::SB;
#pragma unroll
      for (int it = 0; it < CPRB; it++) {
        const int k = it * R + r;
        const int row = k / CPRB, col = k % CPRB;
        cpAsync16(dst + row * G::SB + col * W, blk + row * G::GB + col * W);
      }
    }
  }

  __device__ __forceinline__ static T *dofATile(unsigned char *base) {
    return reinterpret_cast<T *>(base + G::NSN * G::slotNeigh + G::dofTileBytes);
  }
  // the anelastic rows of group g into their tile (anelastic warp s copies rows m * 6 + s)
  __device__ __forceinline__ static void issueDofsA(const StepArgs<T> &a, unsigned char *base, int q, int l,
                                                    int64_t g, bool groupValid) {
    if constexpr (G::dofATile) {
      const int eo = l / R, r = l % R;
      if (!groupValid || q < 9 || g * E + eo >= a.elCount) return;
      const int64_t e = a.elFirst + g * E + eo;
#pragma unroll
      for (int m = 0; m < RM; m++)
        copyRows<T, R, G::GB, G::SB>(dofATile(base), a.dofsA, e, RM * 6, m * 6 + q - 9, eo, r);
    }
  }

  // copies of item (group g, face FA) into `slot`; m = connectivity of this lane's element; PM: the
  // rows are pre-mixed (no flux-solver blocks)
  template <int FA, bool PM>
  __device__ __forceinline__ static void issue(const StepArgs<T> &a, unsigned char *base, int slot, int q, int l,
                                               int64_t g, bool groupValid, const FaceMeta &m) {
    if (groupValid) {
      const int eo = l / R, r = l % R;
      const int64_t e = a.elFirst + g * E + eo;
      const int ty = m.type(FA);
      if (q < 9 && g * E + eo < a.elCount && ty != FT_OUTFLOW) {
        // inner faces: the neighbour's projection over this element's step (its own face buffer,
        // or with LTS its two-step sum / half-step buffer); free surface: this element's own
        const T *buf = a.face;
        if (ty == FT_INNER) {
          const int rf = m.relation(FA);
          buf = rf == LTS_EQ ? a.face : rf == LTS_GT ? a.faceSum : (a.firstTs ? a.faceHalf1 : a.faceHalf2);
        }
        const int64_t srcFace = ty == FT_INNER ? int64_t(m.src[FA]) : e * 4 + FA;
        const T *blk = buf + (srcFace * 9 + q) * int64_t(R * GF);
        T *dst = rows(base, slot) + (q * 32 + eo * R) * SF;
#pragma unroll
        for (int it = 0; it < CPR; it++) {
          const int k = it * R + r;  // consecutive lanes move consecutive 16-byte chunks
          const int row = k / CPR, col = k % CPR;
          cpAsync16(dst + row * SF + col * W, blk + row * GF + col * W);
        }
      }
      if constexpr (G::fsSmem && !PM) {
        // flux-solver blocks fsE[1][e][FA] (and fsA[1][e][FA]) of the group's elements
        double *fsDst = fs(base, slot);
        for (int i = threadIdx.x; i < E * NFS; i += NT) {
          const int eo2 = i / NFS, j = i % NFS;
          if (g * E + eo2 >= a.elCount) continue;
          const int64_t e2 = a.elFirst + g * E + eo2;
          const double *src = j < 81 ? a.fsE + ((a.nEl + e2) * 4 + FA) * 81 + j
                                     : a.fsA + ((a.nEl + e2) * 4 + FA) * 54 + (j - 81);
          cpAsync8(fsDst + i, src);
        }
      }
    }
    cpAsyncCommit();
  }
};

// the neighbour's rows of this item, rotated into this element's face orientation in place
template <typename T, int O, int R, int RM, int FA>
__device__ __forceinline__ void neighOrient(T *S, int q, int l, bool valid, const FaceMeta &m) {
  using G = Geo<T, O, R, RM>;
  constexpr int F = G::F, SF = G::SF;
  if (q < 9 && valid && m.type(FA) == FT_INNER) {
    T x[F], s[F];
    ldRow<T, F>(rowPtr<T, SF>(S, q, l), x);
#pragma unroll
    for (int j = 0; j < F; j++) s[j] = T(0);
    const int v = neighOri<O, FA>(m);
    if (v == 0)
      OriMul<O, 0>::template run<T>(x, s);
    else if (v == 1)
      OriMul<O, 1>::template run<T>(x, s);
    else
      OriMul<O, 2>::template run<T>(x, s);
    stRow<T, F>(rowPtr<T, SF>(S, q, l), s);
  }
}

template <typename T, int O, int R, int RM, int FA>
__device__ __forceinline__ void neighApply(const StepArgs<T> &a, const T *S, const double *fs, int q, int l,
                                           int64_t e, bool valid, const FaceMeta &m, T *acc, T *upA) {
  using G = Geo<T, O, R, RM>;
  using NS = NeighSlots<T, O, R, RM>;
  constexpr int F = G::F, SF = G::SF;
  if (!valid || m.type(FA) == FT_OUTFLOW) return;
  T fr[9];
  if constexpr (G::fsSmem) {
    const int eo = l / R;
    const double *fp = q < 9 ? fs + eo * NS::NFS + q * 9 : fs + eo * NS::NFS + 81 + (q - 9) * 9;
#pragma unroll
    for (int i = 0; i < 9; i++) fr[i] = T(fp[i]);
  } else {
    const double *fp = q < 9 ? a.fsE + ((a.nEl + e) * 4 + FA) * 81 + q * 9
                             : a.fsA + ((a.nEl + e) * 4 + FA) * 54 + (q - 9) * 9;
#pragma unroll
    for (int i = 0; i < 9; i++) fr[i] = T(__ldg(fp + i));
  }
  T s[F];
  faceMix<T, F, SF>(S, l, fr, s);
  if (q < 9)
    FluxTMul<O, FA>::template run<T>(s, acc);
  else if constexpr (RM > 0)
    FluxTMul<O, FA>::template run<T>(s, upA);
}

// pre-mixed rows: this warp's own quantity row of the neighbour's projection, rotated into this
// element's face orientation (inner faces), then fluxT
template <typename T, int O, int R, int RM, int FA>
__device__ __forceinline__ void neighApplyMixed(const T *S, int q, int l, bool valid, const FaceMeta &m, T *acc) {
  using G = Geo<T, O, R, RM>;
  constexpr int F = G::F, SF = G::SF;
  const int ty = m.type(FA);
  if (!valid || ty == FT_OUTFLOW || q >= 9) return;
  T x[F];
  ldRow<T, F>(rowPtr<T, SF>(S, q, l), x);
  if (ty == FT_INNER) {
    T o[F];
#pragma unroll
    for (int j = 0; j < F; j++) o[j] = T(0);
    const int v = neighOri<O, FA>(m);
    if (v == 0)
      OriMul<O, 0>::template run<T>(x, o);
    else if (v == 1)
      OriMul<O, 1>::template run<T>(x, o);
    else
      OriMul<O, 2>::template run<T>(x, o);
    FluxTMul<O, FA>::template run<T>(o, acc);
  } else {
    FluxTMul<O, FA>::template run<T>(x, acc);
  }
}

// item (local group k, face FA): item index i = 4k + FA lives in slot i % NSN; after the barrier the
// item i + NSN - 1 is issued into slot (i - 1) % NSN, which the barrier has released. PM: every warp
// touches only its own quantity rows, so a warp-level order replaces the barrier.
template <typename T, int O, int R, int RM, int FA, bool PM>
__device__ __forceinline__ void neighItem(const StepArgs<T> &a, unsigned char *base, int q, int l, int64_t e,
                                          bool valid, const FaceMeta &cur, const FaceMeta &nxt, int64_t g,
                                          bool nextValid, int64_t k, T *acc, T *upA) {
  using NS = NeighSlots<T, O, R, RM>;
  constexpr int NSN = Geo<T, O, R, RM>::NSN;
  if constexpr (PM) {
    cpAsyncWait<NSN - 2>();
    __syncwarp();
    const int64_t item = k * 4 + FA;
    const int slot = int(item % NSN);
    T *S = NS::rows(base, slot);
    neighApplyMixed<T, O, R, RM, FA>(S, q, l, valid, cur, acc);
    __syncwarp();
    constexpr int AHEAD = FA + NSN - 1;
    const int slotNext = int((item + NSN - 1) % NSN);
    if constexpr (AHEAD < 4)
      NS::template issue<AHEAD, true>(a, base, slotNext, q, l, g, true, cur);
    else
      NS::template issue<AHEAD - 4, true>(a, base, slotNext, q, l, g + gridDim.x, nextValid, nxt);
    return;
  }
  cpAsyncWait<NSN - 2>();
  __syncwarp();
  const int64_t item = k * 4 + FA;
  const int slot = int(item % NSN);
  T *S = NS::rows(base, slot);
  neighOrient<T, O, R, RM, FA>(S, q, l, valid, cur);
  __syncthreads();
  constexpr int AHEAD = FA + NSN - 1;
  const int slotNext = int((item + NSN - 1) % NSN);
  // the next group's DOF rows join the copies committed now (the barrier ordered this group's
  // reads of the tile before them)
  if constexpr (AHEAD < 4)
    NS::template issue<AHEAD, false>(a, base, slotNext, q, l, g, true, cur);
  else
    NS::template issue<AHEAD - 4, false>(a, base, slotNext, q, l, g + gridDim.x, nextValid, nxt);
  neighApply<T, O, R, RM, FA>(a, S, NS::fs(base, slot), q, l, e, valid, cur, acc, upA);
}

// PM: the face buffers hold projections pre-mixed with this element's flux solvers (the local
// kernels write them so where their buffers fit); otherwise the mix happens here (attenuation,
// configurations without room for pre-mixing)
template <typename T, int O, int R, int RM, bool PM>
__global__ void __launch_bounds__(Geo<T, O, R, RM>::NT, Geo<T, O, R, RM>::minCtasNeigh) kNeigh(StepArgs<T> a) {
  using G = Geo<T, O, R, RM>;
  using NS = NeighSlots<T, O, R, RM>;
  constexpr int B = G::B, E = G::E, NSN = G::NSN;
  extern __shared__ __align__(16) unsigned char smem[];
  const int q = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int eo = l / R, r = l % R;
  const int64_t nGroups = (a.elCount + E - 1) / E;
  int64_t g = blockIdx.x;
  FaceMeta cur, nxt;
  cur.load(a, a.elFirst + g * E + eo, g * E + eo < a.elCount);
  // prologue: the first group's DOF rows and items 0 .. NSN-2 (its first faces)
  NS::issueDofs(a, smem, q, l, g, g < nGroups);
  NS::issueDofsA(a, smem, q, l, g, g < nGroups);
  NS::template issue<0, PM>(a, smem, 0, q, l, g, g < nGroups, cur);
  if constexpr (NSN > 2) NS::template issue<1, PM>(a, smem, 1, q, l, g, g < nGroups, cur);
  if constexpr (NSN > 3) NS::template issue<2, PM>(a, smem, 2, q, l, g, g < nGroups, cur);
  for (int64_t k = 0; g < nGroups; g += gridDim.x, k++) {
    const int64_t e = a.elFirst + g * E + eo;
    const bool valid = g * E + eo < a.elCount;
    const int64_t gn = g + gridDim.x;
    const bool nextValid = gn < nGroups;
    nxt.load(a, a.elFirst + gn * E + eo, nextValid && gn * E + eo < a.elCount);
    T acc[B];
    T upA[RM ? B : 1];
    if (q < 9) {
      if constexpr (G::dofTile) {
        // the group's DOF rows (committed last, at the end of the previous group)
        cpAsyncWait<0>();
        __syncwarp();
        if (valid)
          ldRow<T, B>(rowPtr<T, G::SB>(NS::dofTile(smem), q, l), acc);
        else
#pragma unroll
          for (int n = 0; n < B; n++) acc[n] = T(0);
      } else {
        ldRowG<T, B>(gRow<T, R, G::GB>(a.dofsE, valid ? e : 0, 9, q, r), acc, valid);
      }
    } else if constexpr (RM > 0) {
      if constexpr (G::dofATile) {
        // the group's anelastic rows (committed with the DOF rows), read back at the group's end
        cpAsyncWait<0>();
        __syncwarp();
      }
#pragma unroll
      for (int n = 0; n < B; n++) upA[n] = T(0);
    }
    neighItem<T, O, R, RM, 0, PM>(a, smem, q, l, e, valid, cur, nxt, g, nextValid, k, acc, upA);
    neighItem<T, O, R, RM, 1, PM>(a, smem, q, l, e, valid, cur, nxt, g, nextValid, k, acc, upA);
    neighItem<T, O, R, RM, 2, PM>(a, smem, q, l, e, valid, cur, nxt, g, nextValid, k, acc, upA);
    neighItem<T, O, R, RM, 3, PM>(a, smem, q, l, e, valid, cur, nxt, g, nextValid, k, acc, upA);
    if constexpr (RM > 0) {
      if (q >= 9) {
        if (valid) {
          // scatterUpdateA (SurfInt.hpp:139-156)
          const int s = q - 9;
#pragma unroll
          for (int m = 0; m < RM; m++) {
            const T om = T(a.omega[m]);
            T *dst = gRow<T, R, G::GB>(a.dofsA, e, RM * 6, m * 6 + s, r);
            T v[B];
            if constexpr (G::dofATile)
              ldRow<T, B>(rowPtr<T, G::SB>(NS::dofATile(smem), m * 6 + s, l), v);
            else
              ldRowG<T, B>(dst, v, true);
#pragma unroll
            for (int n = 0; n < B; n++) v[n] = fmaT(om, upA[n], v[n]);
            stRowG<T, B>(dst, v);
          }
        }
        // the tile rows read above before the next group's copies into them
        if constexpr (G::dofATile) __syncwarp();
      }
    }
    if constexpr (G::dofTile) {
      // the updated rows through the DOF tile (this warp's rows only), stored coalesced; then the
      // next group's DOF rows into the tile
      if (q < 9) {
        T *p = rowPtr<T, G::SB>(NS::dofTile(smem), q, l);
        stRow<T, B>(p, acc);
#pragma unroll
        for (int n = B; n < G::GB; n++) p[n] = T(0);
        __syncwarp();
        if (valid)
          storeRowsCoalesced<T, R, G::GB, G::SB>(NS::dofTile(smem), a.dofsE + (e * 9 + q) * int64_t(R * G::GB), q,
                                                 eo, r);
        __syncwarp();
      }
      NS::issueDofs(a, smem, q, l, g + gridDim.x, nextValid);
      NS::issueDofsA(a, smem, q, l, g + gridDim.x, nextValid);
      cpAsyncCommit();
    }
    if constexpr (!G::dofTile)
      if (valid && q < 9) stRowG<T, B>(gRow<T, R, G::GB>(a.dofsE, e, 9, q, r), acc);
    cur = nxt;
  }
  cpAsyncWait<0>();
}

// ------------------------------------------------------------------------------------------------
// receivers: recompute the time prediction of receiver elements and sample the Taylor expansion
// (AderDg.hpp:476-494, TimePred::evalTimePrediction TimePred.hpp:130-156, Receivers.cpp:250-290)
// ------------------------------------------------------------------------------------------------
struct RecvArgs {
  const int64_t *grpEl;    // [nGrp] element of each receiver group
  const int32_t *grpOff;   // [nGrp+1] receivers of group g: grpOff[g]..grpOff[g+1]
  const double *basis;     // [nRecv][B]
  const double *tau;       // [nSamples] relative times of this step's samples
  const int32_t *slot;     // [nSamples] buffer slot of each sample
  int nSamples;
  int nGrp;
  int maxBuf;
  double *buf;             // [nRecv][maxBuf][9][R]
};

template <typename T, int O, int R, int RM, int D>
__device__ __forceinline__ void recvAll(T *X, T *TI, T *XA, T *TIA, int q, int l, const ElemCoef<T, RM> &c,
                                        const double *omega, T dt, T sca, const RecvArgs &rv, int i0, int i1,
                                        bool valid, int r, T *tIr, T (*tIAr)[nModes(O)]) {
  constexpr int B = nModes(O), SB = Geo<T, O, R, RM>::SB;
  // value[i][j][q][r] += tau_j^D / D! * sum_{n < B(O-D)} basis_i[n] der_D[q][n]  (CK modes only,
  // even with anelasticity: TimePred.hpp:149)
  if (q < 9 && valid) {
    constexpr int NCK = nModes(O - D);
    const T *xr = rowPtr<T, SB>(X, q, l);
    for (int i = i0; i < i1; i++) {
      double dotv = 0;
#pragma unroll
      for (int n = 0; n < NCK; n++) dotv += rv.basis[i * B + n] * double(xr[n]);
      for (int j = 0; j < rv.nSamples; j++) {
        double cf = 1.0;
        for (int k = 1; k <= D; k++) cf *= rv.tau[j] / k;
        double *o = rv.buf + ((int64_t(i) * rv.maxBuf + rv.slot[j]) * 9 + q) * R + r;
        *o = (D == 0 ? 0.0 : *o) + cf * dotv;
      }
    }
  }
  if constexpr (D + 1 < O) {
    sca = sca * dt / T(D + 2);
    CkStep<T, O, R, RM, D + 1>::run(X, TI, XA, TIA, q, l, c, omega, sca, tIr, tIAr);
    recvAll<T, O, R, RM, D + 1>(X, TI, XA, TIA, q, l, c, omega, dt, sca, rv, i0, i1, valid, r, tIr, tIAr);
  }
}

template <typename T, int O, int R, int RM>
__global__ void __launch_bounds__(Geo<T, O, R, RM>::NT) kRecv(StepArgs<T> a, RecvArgs rv) {
  using G = Geo<T, O, R, RM>;
  constexpr int B = G::B, E = G::E, SB = G::SB;
  extern __shared__ __align__(16) unsigned char smem[];
  T *X = reinterpret_cast<T *>(smem);
  T *XA = X + G::nX + G::nTI;
  // time integrals are carried along but unused here (only the derivatives are sampled)
  T *TI = X + G::nX;
  T *TIA = G::tiSmem ? XA + G::nXA : XA;
  const int q = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int eo = l / R, r = l % R;
  const int64_t grp = int64_t(blockIdx.x) * E + eo;
  const bool valid = grp < rv.nGrp;
  const int64_t ev = valid ? rv.grpEl[grp] : 0;
  const T dt = T(a.dt);
  T tIr[G::tiSmem ? 1 : B];
  T tIAr[(G::tiSmem || RM == 0) ? 1 : RM][B];
  T zero[B];
#pragma unroll
  for (int n = 0; n < B; n++) zero[n] = T(0);
  if (q < 9) {
    T v[B];
    ldRowG<T, B>(gRow<T, R, G::GB>(a.dofsE, ev, 9, q, r), v, valid);
    // a pending neighbour step (fused GTS steps) completes the rows first
    if constexpr (RM == 0)
      if (a.faceIn) neighFluxDirect<T, O, R, RM>(a, a.faceIn, ev, q, r, valid, v);
    stRow<T, B>(rowPtr<T, SB>(X, q, l), v);
    if constexpr (G::tiSmem)
      stRow<T, B>(rowPtr<T, SB>(TI, q, l), zero);
    else {
#pragma unroll
      for (int n = 0; n < B; n++) tIr[n] = T(0);
    }
  } else if constexpr (RM > 0) {
    const int s = q - 9;
#pragma unroll
    for (int m = 0; m < RM; m++) {
      T v[B];
      ldRowG<T, B>(gRow<T, R, G::GB>(a.dofsA, ev, RM * 6, m * 6 + s, r), v, valid);
      stRow<T, B>(rowPtr<T, SB>(XA, m * 6 + s, l), v);
      if constexpr (G::tiSmem)
        stRow<T, B>(rowPtr<T, SB>(TIA, m * 6 + s, l), zero);
      else {
#pragma unroll
        for (int n = 0; n < B; n++) tIAr[m][n] = T(0);
      }
    }
  }
  ElemCoef<T, RM> c;
  c.load(a, ev, valid, q);
  __syncthreads();
  const int i0 = valid ? rv.grpOff[grp] : 0, i1 = valid ? rv.grpOff[grp + 1] : 0;
  recvAll<T, O, R, RM, 0>(X, TI, XA, TIA, q, l, c, a.omega, dt, dt, rv, i0, i1, valid, r, tIr, tIAr);
}

// ------------------------------------------------------------------------------------------------
// point sources (PointSources::apply, PointSources.hpp:887-931; Series<1>::integrate, Series.hpp:59-134)
// ------------------------------------------------------------------------------------------------
struct SrcArgs {
  int nGrp;                 // groups of sources sharing (element, run)
  const int32_t *grpOff;    // [nGrp+1]
  const int64_t *el;        // [nSrc]
  const int32_t *run;       // [nSrc]
  const double *scal;       // [nSrc][9]
  const double *bEval;      // [nSrc][B]
  const double *t0, *dts;   // [nSrc]
  const int64_t *tsOff, *nPts;
  const double *ts;
  double t, dt, tol;
  // replayed launches (a captured batch step): the step starts at t + (*stepDev) * dt, the step
  // counter advancing on the device after each step; null: at t
  const int64_t *stepDev;
  // per-source clocks (merged simulations with their own time steps), or null: source i's step k
  // (k = *stepDev, or `step`) covers [clk0[i] + k clkDt[i], clk0[i] + (k + 1) clkDt[i]]
  const double *clk0 = nullptr, *clkDt = nullptr;
  int64_t step = 0;
  // sources in elements at or beyond elLimit (not stepped) are skipped
  int64_t elLimit = 0x7fffffffffffffffLL;
};

__device__ inline double seriesIntegral(double dx, double xStart, int64_t nPts, const double *vals, double x1,
                                        double x2, double tol) {
  const double dxH = dx * 0.5;
  double out = 0;
  double f = (x1 - xStart + dx) / dx, lf = (x2 - xStart) / dx;
  int64_t first = (int64_t)(f > 0 ? f : 0), last = (int64_t)(lf > 0 ? lf : 0);
  if (last > nPts - 1) last = nPts - 1;
  if (first > last) first = last;
  for (int64_t p = first + 1; p < last + 1; p++) {
    out += dxH * (vals[p] - vals[p - 1]);
    out += vals[p - 1] * dx;
  }
  const double tEnd = xStart + (nPts - 1) * dx;
  const bool bL = x1 + tol > xStart && x1 - tol < tEnd;
  const bool bR = x2 + tol > xStart && x2 - tol < tEnd;
  double diff = xStart + first * dx - x1;
  if (first > 0 && bL) {
    out += 0.5 * diff * (diff / dx) * (vals[first - 1] - vals[first]);
    out += vals[first] * diff;
  }
  diff = x2 - (xStart + last * dx);
  if (last < nPts - 1 && bR) {
    out += 0.5 * diff * (diff / dx) * (vals[last + 1] - vals[last]);
    out += vals[last] * diff;
  }
  return out;
}

template <typename T, int O, int R>
__global__ void kSources(T *dofsE, SrcArgs s) {
  constexpr int B = nModes(O);
  const int g = blockIdx.x;
  if (g >= s.nGrp) return;
  const double k = s.stepDev ? double(*s.stepDev) : double(s.step);
  const double t1 = s.stepDev ? s.t + k * s.dt : s.t;
  if (s.el[s.grpOff[g]] >= s.elLimit) return;
  for (int t = threadIdx.x; t < 9 * B; t += blockDim.x) {
    const int q = t / B, md = t % B;
    for (int i = s.grpOff[g]; i < s.grpOff[g + 1]; i++) {
      const double a1 = s.clk0 ? s.clk0[i] + k * s.clkDt[i] : t1;
      const double a2 = s.clk0 ? a1 + s.clkDt[i] : t1 + s.dt;
      const double in = seriesIntegral(s.dts[i], s.t0[i], s.nPts[i], s.ts + s.tsOff[i], a1, a2, s.tol);
      const double sc = in * s.scal[i * 9 + q];
      T *p = dofsE + ((s.el[i] * 9 + q) * R + s.run[i]) * int64_t(padGlobal<T>(B)) + md;
      *p = T(double(*p) + sc * s.bEval[i * B + md]);
    }
  }
}

}  // namespace edge_b200
