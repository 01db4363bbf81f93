// sm_100a kernels of the tet4 ADER-DG element update (elastic + viscoelastic, fused runs).
//
// Thread layout shared by all element kernels: a CTA has 9 "quantity" warps (warp q owns stress /
// velocity quantity q) plus, with attenuation, 6 "anelastic" warps (warp 9+s owns the anelastic
// stress component s of every mechanism). Lane l of every warp is the pair (element l / R, run
// l % R), so a CTA covers E = 32 / R elements; quantity-mixing reads go through shared memory,
// mode products (the global DG matrices) run in registers as compile-time sparse FMA sequences
// (gen/dg_sparse.cuh). CTAs are persistent and loop over element groups.
//
// Data per element (runs fastest): dofsE [9][B][R], dofsA [RM][6][B][R], face buffer
// [4][9][F][R] = tInt * fluxL_f (the time-integrated DOFs projected on each face, read by the
// neighbours), star [3][24] / starA [3][9] / srcA [RM][12] / fsE [2][.][4][81] / fsA [2][.][4][54] in
// FP64, converted to the kernel precision on load.
#pragma once
#include <cstdint>

#include "gen/dg_sparse.cuh"

namespace edge_b200 {

__host__ __device__ constexpr int nModes(int o) { return o <= 0 ? 0 : o * (o + 1) * (o + 2) / 6; }
__host__ __device__ constexpr int nFaceModes(int o) { return o * (o + 1) / 2; }

enum { FT_INNER = 0, FT_FREE = 1, FT_OUTFLOW = 2 };

template <typename T>
struct StepArgs {
  T *dofsE;             // [nEl][9][B][R]
  T *dofsA;             // [nEl][RM][6][B][R]
  T *tDofs;             // [nEl][9][B][R] or null
  T *face;              // [nEl][4][9][F][R]
  const double *starE;  // [nEl][3][24]
  const double *starA;  // [nEl][3][9]
  const double *srcA;   // [nEl][RM][12]
  const double *fsE;    // [2][nEl][4][81]
  const double *fsA;    // [2][nEl][4][54]
  const int32_t *elFaEl;
  const uint8_t *fId, *vId, *faType;
  int64_t nEl;
  double dt;
  double omega[3];
};

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
// compile-time loops over derivatives / dimensions / faces
// ------------------------------------------------------------------------------------------------
template <int O, int D, int DIM, typename T>
__device__ __forceinline__ void ckMul(const T *z, T *acc) { CkMul<O, D, DIM>::template run<T>(z, acc); }

template <typename T, int O, int R, int RM>
struct Geo {
  static constexpr int B = nModes(O), F = nFaceModes(O), E = 32 / R;
  static constexpr int NW = 9 + (RM ? 6 : 0);
  static constexpr int NT = NW * 32;
  // shared memory: X [9][B][32], XA [RM][6][B][32], S0 [9][F][32]
  static constexpr size_t smemX = size_t(9) * B * 32;
  static constexpr size_t smemXA = size_t(RM) * 6 * B * 32;
  static constexpr size_t smemS0 = size_t(9) * F * 32;
  static constexpr size_t smemBytes = (smemX + smemXA + smemS0) * sizeof(T);
};

// z[k] = sum_i c[i] * X[col_i][k][l] for k < nK
template <typename T, int B, int NK, int NS>
__device__ __forceinline__ void mix(const T *X, int l, const int (&col)[NS], const T (&c)[NS], T *z) {
#pragma unroll
  for (int k = 0; k < NK; k++) {
    T v = T(0);
#pragma unroll
    for (int i = 0; i < NS; i++) v = fmaT(c[i], X[(col[i] * B + k) * 32 + l], v);
    z[k] = v;
  }
}

// ---------------------------------------- CK recursion -----------------------------------------
template <typename T, int O, int R, int RM, int D>
struct CkStep {
  static constexpr int B = nModes(O);
  // elastic derivative D (no anelasticity): in B(O-D+1) modes, out B(O-D) modes
  static constexpr int NK = RM ? B : nModes(O - D + 1);
  static constexpr int NN = RM ? nModes(O - 1) : nModes(O - D);
  static constexpr int DK = RM ? 1 : D;  // which truncation of the stiffness product applies

  __device__ __forceinline__ static void run(T *X, T *XA, int q, int l, const T (&cs)[3][3],
                                             const int (&cols)[3], const T (&ca)[3][2],
                                             const int (&colsA)[2], const T (&csrc)[3][3],
                                             const int (&colsSrc)[3], const double *omega,
                                             T sca, T *tI, T (*tIA)[B]) {
    T acc[B];
    T z[B];
#pragma unroll
    for (int n = 0; n < B; n++) acc[n] = T(0);
    if (q < 9) {
      const T c0[3] = {cs[0][0], cs[0][1], cs[0][2]}, c1[3] = {cs[1][0], cs[1][1], cs[1][2]},
              c2[3] = {cs[2][0], cs[2][1], cs[2][2]};
      mix<T, B, NK, 3>(X, l, cols, c0, z);
      ckMul<O, DK, 0, T>(z, acc);
      mix<T, B, NK, 3>(X, l, cols, c1, z);
      ckMul<O, DK, 1, T>(z, acc);
      mix<T, B, NK, 3>(X, l, cols, c2, z);
      ckMul<O, DK, 2, T>(z, acc);
      if (RM && q < 6) {
        // der[d] += srcA_m * derA_m[d-1] (all B modes)
#pragma unroll
        for (int m = 0; m < RM; m++)
#pragma unroll
          for (int n = 0; n < B; n++) {
            T v = acc[n];
#pragma unroll
            for (int i = 0; i < 3; i++) v = fmaT(csrc[m][i], XA[((m * 6 + colsSrc[i]) * B + n) * 32 + l], v);
            acc[n] = v;
          }
      }
    } else {
      // anelastic strain-rate part Psi = sum_dim (starA_dim * der[d-1][u,v,w]) * (-K^T_dim)
      int cv[2] = {6 + colsA[0], 6 + colsA[1]};
      const T a0[2] = {ca[0][0], ca[0][1]}, a1[2] = {ca[1][0], ca[1][1]}, a2[2] = {ca[2][0], ca[2][1]};
      mix<T, B, NK, 2>(X, l, cv, a0, z);
      ckMul<O, DK, 0, T>(z, acc);
      mix<T, B, NK, 2>(X, l, cv, a1, z);
      ckMul<O, DK, 1, T>(z, acc);
      mix<T, B, NK, 2>(X, l, cv, a2, z);
      ckMul<O, DK, 2, T>(z, acc);
    }
    __syncthreads();
    if (q < 9) {
      constexpr int NW = RM ? B : NN;  // rows beyond NN are zero without anelasticity
#pragma unroll
      for (int n = 0; n < NW; n++) {
        X[(q * B + n) * 32 + l] = acc[n];
        tI[n] = fmaT(sca, acc[n], tI[n]);
      }
    } else if (RM) {
      const int s = q - 9;
#pragma unroll
      for (int m = 0; m < RM; m++) {
        const T om = T(omega[m]);
#pragma unroll
        for (int n = 0; n < B; n++) {
          T *p = &XA[((m * 6 + s) * B + n) * 32 + l];
          T v = om * (acc[n] + *p);
          *p = v;
          tIA[m][n] = fmaT(sca, v, tIA[m][n]);
        }
      }
    }
    __syncthreads();
  }
};

template <typename T, int O, int R, int RM, int D>
__device__ __forceinline__ void ckAll(T *X, T *XA, int q, int l, const T (&cs)[3][3], const int (&cols)[3],
                                      const T (&ca)[3][2], const int (&colsA)[2], const T (&csrc)[3][3],
                                      const int (&colsSrc)[3], const double *omega, T dt, T sca, T *tI,
                                      T (*tIA)[nModes(O)]) {
  if constexpr (D < O) {
    sca = sca * dt / T(D + 1);
    CkStep<T, O, R, RM, D>::run(X, XA, q, l, cs, cols, ca, colsA, csrc, colsSrc, omega, sca, tI, tIA);
    ckAll<T, O, R, RM, D + 1>(X, XA, q, l, cs, cols, ca, colsA, csrc, colsSrc, omega, dt, sca, tI, tIA);
  }
}

template <int O, int DIM, typename T>
__device__ __forceinline__ void volMul(const T *z, T *acc) { VolMul<O, DIM>::template run<T>(z, acc); }
template <int O, int FA, typename T>
__device__ __forceinline__ void fluxLMul(const T *x, T *s) { FluxLMul<O, FA>::template run<T>(x, s); }
template <int O, int FA, typename T>
__device__ __forceinline__ void fluxTMul(const T *s, T *acc) { FluxTMul<O, FA>::template run<T>(s, acc); }

// per-thread element coefficients
template <typename T, int RM>
struct ElemCoef {
  T cs[3][3];     // star row q, 3 slots, per dim
  int cols[3];
  T ca[3][2];     // anelastic star row s, per dim
  int colsA[2];
  T csrc[3][3];   // source matrices row q (< 6), per mechanism
  int colsSrc[3];

  __device__ __forceinline__ void load(const StepArgs<T> &a, int64_t e, bool valid, int q) {
    if (q < 9) {
#pragma unroll
      for (int i = 0; i < 3; i++) cols[i] = kStarCol[q][i];
#pragma unroll
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int i = 0; i < 3; i++) {
          int idx = kStarIdx[q][i];
          cs[d][i] = valid && idx >= 0 ? T(__ldg(&a.starE[(e * 3 + d) * 24 + idx])) : T(0);
        }
      if (RM && q < 6) {
#pragma unroll
        for (int i = 0; i < 3; i++) colsSrc[i] = kSrcCol[q][i];
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
          for (int i = 0; i < 3; i++) {
            int idx = kSrcIdx[q][i];
            csrc[m][i] = valid && m < RM && idx >= 0 ? T(__ldg(&a.srcA[(e * RM + m) * 12 + idx])) : T(0);
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
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int i = 0; i < 2; i++) {
          int idx = kStarAIdx[s][i];
          ca[d][i] = valid && idx >= 0 ? T(__ldg(&a.starA[(e * 3 + d) * 9 + idx])) : T(0);
        }
    }
  }
};

// ------------------------------------------------------------------------------------------------
// local step: CK, volume, local surface, face projections (AderDg::local, AderDg.hpp:338-534)
// ------------------------------------------------------------------------------------------------
template <typename T, int O, int R, int RM, int FA>
__device__ __forceinline__ void localFace(const StepArgs<T> &a, T *X, T *S0, int q, int l, int64_t e,
                                          int r, bool valid, const T *tI, T *acc, T *upA) {
  using G = Geo<T, O, R, RM>;
  constexpr int B = G::B, F = G::F;
  T s[F];
  if (q < 9) {
#pragma unroll
    for (int j = 0; j < F; j++) s[j] = T(0);
    fluxLMul<O, FA, T>(tI, s);
#pragma unroll
    for (int j = 0; j < F; j++) S0[(q * F + j) * 32 + l] = s[j];
    if (valid) {
      T *fb = a.face + ((((e * 4 + FA) * 9 + q) * F) * R) + r;
#pragma unroll
      for (int j = 0; j < F; j++) fb[j * R] = s[j];
    }
  }
  __syncthreads();
  // s1[j] = sum_q' fs[q][q'] * S0[q'][j]
  T fr[9];
  if (q < 9) {
    const double *fp = a.fsE + ((e * 4 + FA) * 81 + q * 9);
#pragma unroll
    for (int i = 0; i < 9; i++) fr[i] = valid ? T(__ldg(fp + i)) : T(0);
  } else {
    const double *fp = a.fsA + ((e * 4 + FA) * 54 + (q - 9) * 9);
#pragma unroll
    for (int i = 0; i < 9; i++) fr[i] = valid ? T(__ldg(fp + i)) : T(0);
  }
#pragma unroll
  for (int j = 0; j < F; j++) {
    T v = T(0);
#pragma unroll
    for (int i = 0; i < 9; i++) v = fmaT(fr[i], S0[(i * F + j) * 32 + l], v);
    s[j] = v;
  }
  if (q < 9)
    fluxTMul<O, FA, T>(s, acc);
  else if constexpr (RM > 0)
    fluxTMul<O, FA, T>(s, upA);
  __syncthreads();
}

template <typename T, int O, int R, int RM>
__global__ void __launch_bounds__(Geo<T, O, R, RM>::NT) kLocal(StepArgs<T> a) {
  using G = Geo<T, O, R, RM>;
  constexpr int B = G::B, E = G::E;
  extern __shared__ __align__(16) unsigned char smem[];
  T *X = reinterpret_cast<T *>(smem);
  T *XA = X + G::smemX;
  T *S0 = XA + G::smemXA;
  const int q = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int eo = l / R, r = l % R;
  const int64_t nGroups = (a.nEl + E - 1) / E;
  const T dt = T(a.dt);
  for (int64_t g = blockIdx.x; g < nGroups; g += gridDim.x) {
    const int64_t e = g * E + eo;
    const bool valid = e < a.nEl;
    const int64_t ev = valid ? e : 0;
    T tI[B];
    T tIA[RM ? RM : 1][B];
    // load DOFs
    if (q < 9) {
      const T *src = a.dofsE + ((ev * 9 + q) * B) * R + r;
#pragma unroll
      for (int n = 0; n < B; n++) {
        T v = valid ? src[n * R] : T(0);
        X[(q * B + n) * 32 + l] = v;
        tI[n] = dt * v;
      }
    } else if (RM) {
      const int s = q - 9;
#pragma unroll
      for (int m = 0; m < RM; m++) {
        const T *src = a.dofsA + (((ev * RM + m) * 6 + s) * B) * R + r;
#pragma unroll
        for (int n = 0; n < B; n++) {
          T v = valid ? src[n * R] : T(0);
          XA[((m * 6 + s) * B + n) * 32 + l] = v;
          tIA[m][n] = dt * v;
        }
      }
    }
    ElemCoef<T, RM> c;
    c.load(a, ev, valid, q);
    __syncthreads();
    // Cauchy-Kowalevski (TimePredVanilla::ck, TimePredVanilla.hpp:200-306)
    ckAll<T, O, R, RM, 1>(X, XA, q, l, c.cs, c.cols, c.ca, c.colsA, c.csrc, c.colsSrc, a.omega, dt, dt,
                          tI, tIA);
    // time-integrated DOFs to shared memory (and global for callers that keep them)
    if (q < 9) {
#pragma unroll
      for (int n = 0; n < B; n++) X[(q * B + n) * 32 + l] = tI[n];
      if (a.tDofs && valid) {
        T *dst = a.tDofs + ((e * 9 + q) * B) * R + r;
#pragma unroll
        for (int n = 0; n < B; n++) dst[n * R] = tI[n];
      }
    } else if (RM) {
      const int s = q - 9;
#pragma unroll
      for (int m = 0; m < RM; m++)
#pragma unroll
        for (int n = 0; n < B; n++) XA[((m * 6 + s) * B + n) * 32 + l] = tIA[m][n];
    }
    __syncthreads();
    // volume integral (VolIntVanilla::apply, VolIntVanilla.hpp:189-241)
    T acc[B];
    T upA[RM ? B : 1];
    {
      constexpr int NK = nModes(O - 1);
      T z[NK > 0 ? NK : 1];
      if (q < 9) {
        const T *src = a.dofsE + ((ev * 9 + q) * B) * R + r;
#pragma unroll
        for (int n = 0; n < B; n++) acc[n] = valid ? src[n * R] : T(0);
        const T c0[3] = {c.cs[0][0], c.cs[0][1], c.cs[0][2]}, c1[3] = {c.cs[1][0], c.cs[1][1], c.cs[1][2]},
                c2[3] = {c.cs[2][0], c.cs[2][1], c.cs[2][2]};
        mix<T, B, NK, 3>(X, l, c.cols, c0, z);
        volMul<O, 0, T>(z, acc);
        mix<T, B, NK, 3>(X, l, c.cols, c1, z);
        volMul<O, 1, T>(z, acc);
        mix<T, B, NK, 3>(X, l, c.cols, c2, z);
        volMul<O, 2, T>(z, acc);
        if (RM && q < 6) {
#pragma unroll
          for (int m = 0; m < RM; m++)
#pragma unroll
            for (int n = 0; n < B; n++) {
              T v = acc[n];
#pragma unroll
              for (int i = 0; i < 3; i++) v = fmaT(c.csrc[m][i], XA[((m * 6 + c.colsSrc[i]) * B + n) * 32 + l], v);
              acc[n] = v;
            }
        }
      } else if constexpr (RM > 0) {
#pragma unroll
        for (int n = 0; n < B; n++) acc[n] = T(0);
        int cv[2] = {6 + c.colsA[0], 6 + c.colsA[1]};
        const T a0[2] = {c.ca[0][0], c.ca[0][1]}, a1[2] = {c.ca[1][0], c.ca[1][1]}, a2[2] = {c.ca[2][0], c.ca[2][1]};
        mix<T, B, NK, 2>(X, l, cv, a0, z);
        volMul<O, 0, T>(z, acc);
        mix<T, B, NK, 2>(X, l, cv, a1, z);
        volMul<O, 1, T>(z, acc);
        mix<T, B, NK, 2>(X, l, cv, a2, z);
        volMul<O, 2, T>(z, acc);
#pragma unroll
        for (int n = 0; n < B; n++) upA[n] = T(0);
      }
    }
    // local surface integral (SurfIntVanilla::local, SurfIntVanilla.hpp:212-262) + face projections
    localFace<T, O, R, RM, 0>(a, X, S0, q, l, ev, r, valid, tI, acc, upA);
    localFace<T, O, R, RM, 1>(a, X, S0, q, l, ev, r, valid, tI, acc, upA);
    localFace<T, O, R, RM, 2>(a, X, S0, q, l, ev, r, valid, tI, acc, upA);
    localFace<T, O, R, RM, 3>(a, X, S0, q, l, ev, r, valid, tI, acc, upA);
    if (valid) {
      if (q < 9) {
        T *dst = a.dofsE + ((e * 9 + q) * B) * R + r;
#pragma unroll
        for (int n = 0; n < B; n++) dst[n * R] = acc[n];
      } else if (RM) {
        // dofsA_m += omega_m * (Psi_vol - tIntA_m) + omega_m * upA_surf
        const int s = q - 9;
#pragma unroll
        for (int m = 0; m < RM; m++) {
          const T om = T(a.omega[m]);
          T *dst = a.dofsA + (((e * RM + m) * 6 + s) * B) * R + r;
#pragma unroll
          for (int n = 0; n < B; n++) {
            T v = dst[n * R];
            v = fmaT(om, acc[n] - tIA[m][n], v);
            v = fmaT(om, upA[n], v);
            dst[n * R] = v;
          }
        }
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// neighbour step (AderDg::neigh, AderDg.hpp:553-722)
// ------------------------------------------------------------------------------------------------
template <int O, int V, typename T>
__device__ __forceinline__ void oriMul(const T *x, T *s) { OriMul<O, V>::template run<T>(x, s); }

template <typename T, int O, int R, int RM, int FA>
__device__ __forceinline__ void neighFace(const StepArgs<T> &a, T *S0, int q, int l, int64_t e, int r,
                                          bool valid, T *acc, T *upA) {
  using G = Geo<T, O, R, RM>;
  constexpr int F = G::F;
  const int ty = valid ? a.faType[e * 4 + FA] : FT_OUTFLOW;
  if (q < 9) {
    T s[F];
#pragma unroll
    for (int j = 0; j < F; j++) s[j] = T(0);
    if (ty == FT_FREE) {
      // own face projection with the local flux matrix; the mirror is in fsE[1]
      const T *fb = a.face + ((((e * 4 + FA) * 9 + q) * F) * R) + r;
#pragma unroll
      for (int j = 0; j < F; j++) s[j] = fb[j * R];
    } else if (ty == FT_INNER) {
      const int64_t ne = a.elFaEl[e * 4 + FA];
      const int fo = a.fId[e * 4 + FA], v = a.vId[e * 4 + FA];
      const T *fb = a.face + ((((ne * 4 + fo) * 9 + q) * F) * R) + r;
      T x[F];
#pragma unroll
      for (int j = 0; j < F; j++) x[j] = fb[j * R];
      if (v == 0)
        oriMul<O, 0, T>(x, s);
      else if (v == 1)
        oriMul<O, 1, T>(x, s);
      else
        oriMul<O, 2, T>(x, s);
    }
#pragma unroll
    for (int j = 0; j < F; j++) S0[(q * F + j) * 32 + l] = s[j];
  }
  __syncthreads();
  if (ty != FT_OUTFLOW) {
    T fr[9];
    if (q < 9) {
      const double *fp = a.fsE + ((a.nEl + e) * 4 + FA) * 81 + q * 9;
#pragma unroll
      for (int i = 0; i < 9; i++) fr[i] = T(__ldg(fp + i));
    } else {
      const double *fp = a.fsA + ((a.nEl + e) * 4 + FA) * 54 + (q - 9) * 9;
#pragma unroll
      for (int i = 0; i < 9; i++) fr[i] = T(__ldg(fp + i));
    }
    T s[F];
#pragma unroll
    for (int j = 0; j < F; j++) {
      T v = T(0);
#pragma unroll
      for (int i = 0; i < 9; i++) v = fmaT(fr[i], S0[(i * F + j) * 32 + l], v);
      s[j] = v;
    }
    if (q < 9)
      fluxTMul<O, FA, T>(s, acc);
    else if constexpr (RM > 0)
      fluxTMul<O, FA, T>(s, upA);
  }
  __syncthreads();
}

template <typename T, int O, int R, int RM>
__global__ void __launch_bounds__(Geo<T, O, R, RM>::NT) kNeigh(StepArgs<T> a) {
  using G = Geo<T, O, R, RM>;
  constexpr int B = G::B, E = G::E;
  extern __shared__ __align__(16) unsigned char smem[];
  T *S0 = reinterpret_cast<T *>(smem);
  const int q = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int eo = l / R, r = l % R;
  const int64_t nGroups = (a.nEl + E - 1) / E;
  for (int64_t g = blockIdx.x; g < nGroups; g += gridDim.x) {
    const int64_t e = g * E + eo;
    const bool valid = e < a.nEl;
    const int64_t ev = valid ? e : 0;
    T acc[B];
    T upA[RM ? B : 1];
    if (q < 9) {
      const T *src = a.dofsE + ((ev * 9 + q) * B) * R + r;
#pragma unroll
      for (int n = 0; n < B; n++) acc[n] = valid ? src[n * R] : T(0);
    } else if constexpr (RM > 0) {
#pragma unroll
      for (int n = 0; n < B; n++) upA[n] = T(0);
    }
    neighFace<T, O, R, RM, 0>(a, S0, q, l, ev, r, valid, acc, upA);
    neighFace<T, O, R, RM, 1>(a, S0, q, l, ev, r, valid, acc, upA);
    neighFace<T, O, R, RM, 2>(a, S0, q, l, ev, r, valid, acc, upA);
    neighFace<T, O, R, RM, 3>(a, S0, q, l, ev, r, valid, acc, upA);
    if (valid) {
      if (q < 9) {
        T *dst = a.dofsE + ((e * 9 + q) * B) * R + r;
#pragma unroll
        for (int n = 0; n < B; n++) dst[n * R] = acc[n];
      } else if (RM) {
        // scatterUpdateA (SurfInt.hpp:139-156)
        const int s = q - 9;
#pragma unroll
        for (int m = 0; m < RM; m++) {
          const T om = T(a.omega[m]);
          T *dst = a.dofsA + (((e * RM + m) * 6 + s) * B) * R + r;
#pragma unroll
          for (int n = 0; n < B; n++) dst[n * R] = fmaT(om, upA[n], dst[n * R]);
        }
      }
    }
  }
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

template <typename T, int O, int R, int RM>
__global__ void __launch_bounds__(Geo<T, O, R, RM>::NT) kRecv(StepArgs<T> a, RecvArgs rv) {
  using G = Geo<T, O, R, RM>;
  constexpr int B = G::B, E = G::E;
  extern __shared__ __align__(16) unsigned char smem[];
  T *X = reinterpret_cast<T *>(smem);
  T *XA = X + G::smemX;
  const int q = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int eo = l / R, r = l % R;
  const int64_t grp = int64_t(blockIdx.x) * E + eo;
  const bool valid = grp < rv.nGrp;
  const int64_t ev = valid ? rv.grpEl[grp] : 0;
  const T dt = T(a.dt);
  T tI[B];
  T tIA[RM ? RM : 1][B];
  if (q < 9) {
    const T *src = a.dofsE + ((ev * 9 + q) * B) * R + r;
#pragma unroll
    for (int n = 0; n < B; n++) X[(q * B + n) * 32 + l] = valid ? src[n * R] : T(0);
  } else if (RM) {
    const int s = q - 9;
#pragma unroll
    for (int m = 0; m < RM; m++) {
      const T *src = a.dofsA + (((ev * RM + m) * 6 + s) * B) * R + r;
#pragma unroll
      for (int n = 0; n < B; n++) XA[((m * 6 + s) * B + n) * 32 + l] = valid ? src[n * R] : T(0);
    }
  }
  ElemCoef<T, RM> c;
  c.load(a, ev, valid, q);
  __syncthreads();
  // accumulate value[i][j][q][r] = sum_d tau_j^d / d! * sum_{n < B(O-d)} basis_i[n] der_d[q][n]
  const int i0 = valid ? rv.grpOff[grp] : 0, i1 = valid ? rv.grpOff[grp + 1] : 0;
  auto addDerivative = [&](int d) {
    if (q >= 9 || !valid) return;
    const int nck = nModes(O - d);
    for (int i = i0; i < i1; i++) {
      double dotv = 0;
      for (int n = 0; n < nck; n++) dotv += rv.basis[i * B + n] * double(X[(q * B + n) * 32 + l]);
      for (int j = 0; j < rv.nSamples; j++) {
        double cf = 1.0;
        for (int k = 1; k <= d; k++) cf *= rv.tau[j] / k;
        double *o = rv.buf + ((int64_t(i) * rv.maxBuf + rv.slot[j]) * 9 + q) * R + r;
        *o = (d == 0 ? 0.0 : *o) + cf * dotv;
      }
    }
  };
  addDerivative(0);
  T sca = dt;
  // derivative by derivative; the CK step writes der[d] into X
#define EDGE_RECV_STEP(D)                                                                              \
  if constexpr (D < O) {                                                                              \
    sca = sca * dt / T(D + 1);                                                                        \
    CkStep<T, O, R, RM, D>::run(X, XA, q, l, c.cs, c.cols, c.ca, c.colsA, c.csrc, c.colsSrc, a.omega, \
                                sca, tI, tIA);                                                        \
    addDerivative(D);                                                                                 \
    __syncthreads();                                                                                  \
  }
  for (int n = 0; n < B; n++) tI[n] = T(0);
  for (int m = 0; m < (RM ? RM : 1); m++)
    for (int n = 0; n < B; n++) tIA[m][n] = T(0);
  EDGE_RECV_STEP(1)
  EDGE_RECV_STEP(2)
  EDGE_RECV_STEP(3)
  EDGE_RECV_STEP(4)
  EDGE_RECV_STEP(5)
#undef EDGE_RECV_STEP
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
  for (int t = threadIdx.x; t < 9 * B; t += blockDim.x) {
    const int q = t / B, md = t % B;
    for (int i = s.grpOff[g]; i < s.grpOff[g + 1]; i++) {
      const double in = seriesIntegral(s.dts[i], s.t0[i], s.nPts[i], s.ts + s.tsOff[i], s.t, s.t + s.dt, s.tol);
      const double sc = in * s.scal[i * 9 + q];
      T *p = dofsE + ((s.el[i] * 9 + q) * B + md) * R + s.run[i];
      *p = T(double(*p) + sc * s.bEval[i * B + md]);
    }
  }
}

}  // namespace edge_b200
