/*
 * CPU oracle for the tet4 ADER-DG elastic / viscoelastic element update.
 *
 * TEST INFRASTRUCTURE ONLY. This file restates, in plain C and FP64, the reference's GTS element
 * update so that tests, smoke() and the bench's CPU-baseline leg can check the CUDA path against
 * it. Nothing in the product links, calls or ships this code.
 *
 * Layouts (runs fastest, row-major):
 *   dofsE  [nEl][9][B][R]          dofsA [nEl][rm][6][B][R]        tDofs [nEl][9][B][R]
 *   starE  [nEl][3][24]  (row-major non-zeros of the elastic star matrices, Elasticity.cpp:254-300)
 *   starA  [nEl][3][9]   (row-major non-zeros of the 6x3 anelastic star, ViscoElasticity.cpp:295-316)
 *   srcA   [nEl][rm][12] (row-major non-zeros of the 6x6 anelastic source, ViscoElasticity.h:460-508)
 *   fsE    [2][nEl][4][81] (row-major 9x9 flux solvers; [0] local, [1] neighbour, AderDgInit.hpp:394-665)
 *   fsA    [2][nEl][4][54] (row-major 6x9 anelastic flux solvers)
 *   stiffT [3][B][B] = K_d^T M^-1 (NOT negated; negated on use like dg/TimePred.hpp:86)
 *   stiffV [3][B][B] = K_d M^-1,  fluxL [4][B][F], fluxN [12][B][F] (id 4v+f), fluxT [4][F][B]
 *
 * Functions follow (reference file:line):
 *   oracle_ck          TimePredVanilla::ck            src/impl/seismic/kernels/TimePredVanilla.hpp:200-306
 *   oracle_eval_pred   TimePred::evalTimePrediction   src/impl/seismic/kernels/TimePred.hpp:130-156
 *   oracle_volint      VolIntVanilla::apply           src/impl/seismic/kernels/VolIntVanilla.hpp:189-241
 *   oracle_surf_local  SurfIntVanilla::local          src/impl/seismic/kernels/SurfIntVanilla.hpp:212-262
 *   oracle_surf_neigh  SurfIntVanilla::neigh(+FluxInt) src/impl/seismic/kernels/SurfIntVanilla.hpp:274-357
 *   oracle_series_int  Series<1>::integrate           src/linalg/Series.hpp:59-134
 *   oracle_integrate   TimePred::integrate            src/impl/seismic/kernels/TimePred.hpp:165-202
 *   oracle_step        steps 0/1/2 of one GTS step    src/impl/seismic/steps.inc:24-77 with
 *                      AderDg::local (AderDg.hpp:338-534), PointSources::apply (PointSources.hpp:887-931),
 *                      AderDg::neigh (AderDg.hpp:553-722), Receivers (io/Receivers.cpp:235-290)
 *   oracle_lts_local / oracle_lts_neigh  the same work regions of one rate-2 LTS time group
 *                      (AderDg.hpp:384-417 and 620-674, TimeGroupStatic.cpp:46-111)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* sparsity patterns: row-major non-zeros (Elasticity.cpp:254-300, ViscoElasticity.cpp:295-316,
 * ViscoElasticity.h:484-507) */
static const int SE_R[24] = {0,0,0,1,1,1,2,2,2,3,3,4,4,5,5,6,6,6,7,7,7,8,8,8};
static const int SE_C[24] = {6,7,8,6,7,8,6,7,8,6,7,7,8,6,8,0,3,5,1,3,4,2,4,5};
static const int SA_R[9]  = {0,1,2,3,3,4,4,5,5};
static const int SA_C[9]  = {0,1,2,0,1,1,2,0,2}; /* column within the velocities (6+c) */
static const int SR_R[12] = {0,0,0,1,1,1,2,2,2,3,4,5};
static const int SR_C[12] = {0,1,2,0,1,2,0,1,2,3,4,5};

static int nmodes(int o) { return o <= 0 ? 0 : o * (o + 1) * (o + 2) / 6; }

/* Operand rounding of the products with the global DG matrices (mm_ac), for measuring what tensor
 * cores would do to the results: 0 none (FP64), 1 both operands rounded to tf32 (10-bit mantissa,
 * round to nearest with ties away from zero, as cvt.rna.tf32.f32 does after the FP32 value), 2 the
 * three-product split a_hi b_hi + a_hi b_lo + a_lo b_hi of tf32 parts, 3 both operands rounded to
 * bf16 (8-bit mantissa, round to nearest even, as cvt.rn.bf16.f32), 4 the three-product split of
 * bf16 parts. The star and flux-solver mixes (mm_bc) stay exact. Test infrastructure only. */
static int g_mmMode = 0;
void oracle_set_mm_mode(int mode) { g_mmMode = mode; }

static double tf32(double x) {
  float f = (float)x;
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  memcpy(&f, &u, 4);
  return (double)f;
}

static double bf16(double x) {
  float f = (float)x;
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x7fffu + ((u >> 16) & 1u)) & 0xffff0000u;
  memcpy(&f, &u, 4);
  return (double)f;
}

static double mmProd(double a, double b) {
  double (*rnd)(double) = g_mmMode >= 3 ? bf16 : tf32;
  if (g_mmMode == 1 || g_mmMode == 3) return rnd(a) * rnd(b);
  const double ah = rnd(a), bh = rnd(b);
  const double al = rnd((double)((float)a - (float)ah)), bl = rnd((double)((float)b - (float)bh));
  return ah * bh + (ah * bl + al * bh);
}

/* C[m][n][r] (+)= sum_k A[m][k][r] * B[k][n]   (MmVanilla fused-AC, Matrix.h:296-330) */
static void mm_ac(int R, int M, int N, int K, int ldA, int ldB, int ldC, double beta,
                  const double *A, const double *Bm, double *C) {
  for (int m = 0; m < M; m++)
    for (int n = 0; n < N; n++)
      for (int r = 0; r < R; r++) {
        double *c = &C[((size_t)m * ldC + n) * R + r];
        *c = (beta != 0.0) ? *c * beta : 0.0;
      }
  for (int k = 0; k < K; k++)
    for (int m = 0; m < M; m++)
      for (int n = 0; n < N; n++) {
        double b = Bm[(size_t)k * ldB + n];
        if (b == 0.0) continue; /* exact: adding a zero product changes nothing */
        if (g_mmMode) {
          for (int r = 0; r < R; r++)
            C[((size_t)m * ldC + n) * R + r] += mmProd(A[((size_t)m * ldA + k) * R + r], b);
          continue;
        }
        for (int r = 0; r < R; r++)
          C[((size_t)m * ldC + n) * R + r] += A[((size_t)m * ldA + k) * R + r] * b;
      }
}

/* C[m][n][r] += sum_k A[m][k] * B[k][n][r] with A dense MxK (fused-BC, Matrix.h:332-378) */
static void mm_bc(int R, int M, int N, int K, int ldB, int ldC, const double *A,
                  const double *Bm, double *C) {
  for (int k = 0; k < K; k++)
    for (int m = 0; m < M; m++) {
      double a = A[m * K + k];
      if (a == 0.0) continue;
      for (int n = 0; n < N; n++)
        for (int r = 0; r < R; r++)
          C[((size_t)m * ldC + n) * R + r] += a * Bm[((size_t)k * ldB + n) * R + r];
    }
}

static void dense_star(const double *sp, double *d) {
  memset(d, 0, 81 * sizeof(double));
  for (int i = 0; i < 24; i++) d[SE_R[i] * 9 + SE_C[i]] = sp[i];
}
static void dense_starA(const double *sp, double *d) { /* 6x3 acting on velocities */
  memset(d, 0, 18 * sizeof(double));
  for (int i = 0; i < 9; i++) d[SA_R[i] * 3 + SA_C[i]] = sp[i];
}
static void dense_src(const double *sp, double *d) {
  memset(d, 0, 36 * sizeof(double));
  for (int i = 0; i < 12; i++) d[SR_R[i] * 6 + SR_C[i]] = sp[i];
}

void oracle_ck(int O, int R, int rm, double dt, const double *stiffT, const double *starE,
               const double *starA, const double *srcA, const double *omega,
               const double *dofsE, const double *dofsA, double *derE, double *tIntE,
               double *tIntA) {
  const int B = nmodes(O);
  const size_t szE = (size_t)9 * B * R, szM = (size_t)6 * B * R;
  double *scr = calloc(szE, sizeof(double));
  double *scrA = calloc(szM, sizeof(double));
  double *derA = rm ? calloc((size_t)rm * O * szM, sizeof(double)) : NULL;
  double *kT = malloc((size_t)3 * B * B * sizeof(double));
  double st[3][81], sa[3][18], sr[6 * 6];
  for (size_t i = 0; i < (size_t)3 * B * B; i++) kT[i] = -stiffT[i];
  for (int d = 0; d < 3; d++) {
    dense_star(starE + 24 * d, st[d]);
    if (rm) dense_starA(starA + 9 * d, sa[d]);
  }
  double sca = dt;
  for (size_t i = 0; i < szE; i++) {
    derE[i] = dofsE[i];
    tIntE[i] = sca * dofsE[i];
  }
  for (int m = 0; m < rm; m++)
    for (size_t i = 0; i < szM; i++) {
      derA[(size_t)m * O * szM + i] = dofsA[m * szM + i];
      tIntA[m * szM + i] = sca * dofsA[m * szM + i];
    }
  for (int de = 1; de < O; de++) {
    const int re = rm == 0 ? de : 1;
    const int nN = nmodes(O - re), nK = nmodes(O - re + 1);
    double *dCur = derE + (size_t)de * szE, *dPrv = derE + (size_t)(de - 1) * szE;
    memset(dCur, 0, szE * sizeof(double));
    memset(scrA, 0, szM * sizeof(double));
    for (int di = 0; di < 3; di++) {
      mm_ac(R, 9, nN, nK, B, B, B, 0.0, dPrv, kT + (size_t)di * B * B, scr);
      mm_bc(R, 9, nN, 9, B, B, st[di], scr, dCur);
      if (rm) mm_bc(R, 6, nN, 3, B, B, sa[di], scr + (size_t)6 * B * R, scrA);
    }
    sca *= dt / (de + 1);
    for (int m = 0; m < rm; m++) {
      double *aPrv = derA + ((size_t)m * O + de - 1) * szM, *aCur = aPrv + szM;
      dense_src(srcA + 12 * m, sr);
      mm_bc(R, 6, B, 6, B, B, sr, aPrv, dCur);
      for (size_t i = 0; i < szM; i++) {
        aCur[i] = omega[m] * (scrA[i] + aPrv[i]);
        tIntA[m * szM + i] += sca * aCur[i];
      }
    }
    const int nCp = rm == 0 ? nmodes(O - de) : B;
    for (int q = 0; q < 9; q++)
      for (int md = 0; md < nCp; md++)
        for (int r = 0; r < R; r++) {
          size_t i = ((size_t)q * B + md) * R + r;
          tIntE[i] += sca * dCur[i];
        }
  }
  free(scr);
  free(scrA);
  free(derA);
  free(kT);
}

void oracle_eval_pred(int O, int R, double tau, const double *derE, double *pred) {
  const int B = nmodes(O);
  const size_t szE = (size_t)9 * B * R;
  memcpy(pred, derE, szE * sizeof(double));
  double sca = 1.0;
  for (int de = 1; de < O; de++) {
    sca *= tau / de;
    const int nCk = nmodes(O - de); /* CK modes even with anelasticity (TimePred.hpp:149) */
    for (int q = 0; q < 9; q++)
      for (int md = 0; md < nCk; md++)
        for (int r = 0; r < R; r++) {
          size_t i = ((size_t)q * B + md) * R + r;
          pred[i] += sca * derE[(size_t)de * szE + i];
        }
  }
}

void oracle_volint(int O, int R, int rm, const double *stiffV, const double *starE,
                   const double *starA, const double *srcA, const double *omega,
                   const double *tIntE, const double *tIntA, double *dofsE, double *dofsA) {
  const int B = nmodes(O), Bk = nmodes(O - 1);
  const size_t szE = (size_t)9 * B * R, szM = (size_t)6 * B * R;
  double *scr = malloc(szE * sizeof(double));
  double *scrA = calloc(szM, sizeof(double));
  double st[81], sa[18], sr[36];
  for (int di = 0; di < 3; di++) {
    mm_ac(R, 9, B, Bk, B, B, B, 0.0, tIntE, stiffV + (size_t)di * B * B, scr);
    dense_star(starE + 24 * di, st);
    mm_bc(R, 9, B, 9, B, B, st, scr, dofsE);
    if (rm) {
      dense_starA(starA + 9 * di, sa);
      mm_bc(R, 6, B, 3, B, B, sa, scr + (size_t)6 * B * R, scrA);
    }
  }
  for (int m = 0; m < rm; m++) {
    dense_src(srcA + 12 * m, sr);
    mm_bc(R, 6, B, 6, B, B, sr, tIntA + m * szM, dofsE);
    for (size_t i = 0; i < szM; i++) dofsA[m * szM + i] += omega[m] * (scrA[i] - tIntA[m * szM + i]);
  }
  free(scr);
  free(scrA);
}

/* one face of the surface integral: dofsE += fluxT_f^T-apply((fs * (tInt * flux)));  upA likewise */
static void surf_face(int O, int R, int rm, const double *flux, const double *fluxTf,
                      const double *fsE, const double *fsA, const double *tInt, double *dofsE,
                      double *upA, double *s0, double *s1) {
  const int B = nmodes(O), F = O * (O + 1) / 2;
  mm_ac(R, 9, F, B, B, F, F, 0.0, tInt, flux, s0);
  memset(s1, 0, (size_t)9 * F * R * sizeof(double));
  mm_bc(R, 9, F, 9, F, F, fsE, s0, s1);
  mm_ac(R, 9, B, F, F, B, B, 1.0, s1, fluxTf, dofsE);
  if (rm) {
    memset(s1, 0, (size_t)6 * F * R * sizeof(double));
    mm_bc(R, 6, F, 9, F, F, fsA, s0, s1);
    mm_ac(R, 6, B, F, F, B, B, 1.0, s1, fluxTf, upA);
  }
}

static void scatter_upA(int B, int R, int rm, const double *omega, const double *upA,
                        double *dofsA) {
  const size_t szM = (size_t)6 * B * R;
  for (int m = 0; m < rm; m++)
    for (size_t i = 0; i < szM; i++) dofsA[m * szM + i] += omega[m] * upA[i];
}

void oracle_surf_local(int O, int R, int rm, const double *fluxL, const double *fluxT,
                       const double *fsE4, const double *fsA4, const double *omega,
                       const double *tIntE, double *dofsE, double *dofsA) {
  const int B = nmodes(O), F = O * (O + 1) / 2;
  double *s0 = malloc((size_t)9 * F * R * sizeof(double));
  double *s1 = malloc((size_t)9 * F * R * sizeof(double));
  double *upA = calloc((size_t)6 * B * R, sizeof(double));
  for (int f = 0; f < 4; f++)
    surf_face(O, R, rm, fluxL + (size_t)f * B * F, fluxT + (size_t)f * F * B, fsE4 + 81 * f,
              rm ? fsA4 + 54 * f : NULL, tIntE, dofsE, upA, s0, s1);
  if (rm) scatter_upA(B, R, rm, omega, upA, dofsA);
  free(s0);
  free(s1);
  free(upA);
}

/* vId < 0 selects the local flux matrix of face fa (free surface); otherwise fluxN[4*vId+fId] */
void oracle_surf_neigh(int O, int R, int rm, int fa, int vId, int fId, const double *fluxL,
                       const double *fluxN, const double *fluxT, const double *fsE,
                       const double *fsA, const double *tIntNe, double *dofsE, double *upA) {
  const int B = nmodes(O), F = O * (O + 1) / 2;
  double *s0 = malloc((size_t)9 * F * R * sizeof(double));
  double *s1 = malloc((size_t)9 * F * R * sizeof(double));
  const double *flux = vId < 0 ? fluxL + (size_t)fa * B * F : fluxN + (size_t)(4 * vId + fId) * B * F;
  surf_face(O, R, rm, flux, fluxT + (size_t)fa * F * B, fsE, fsA, tIntNe, dofsE, upA, s0, s1);
  free(s0);
  free(s1);
}

double oracle_series_int(double dx, double xStart, long nPts, const double *vals, double x1,
                         double x2, double na, double tol) {
  const double dxH = dx * 0.5;
  double out = 0;
  double f = (x1 - xStart + dx) / dx, l = (x2 - xStart) / dx;
  size_t first = (size_t)(f > 0 ? f : 0), last = (size_t)(l > 0 ? l : 0);
  if (last > (size_t)(nPts - 1)) last = nPts - 1;
  if (first > last) first = last;
  for (size_t p = first + 1; p < last + 1; p++) {
    out += dxH * (vals[p] - vals[p - 1]);
    out += vals[p - 1] * dx;
  }
  int bL = 0, bR = 0;
  double tEnd = xStart + (nPts - 1) * dx;
  if (x1 + tol > xStart && x1 - tol < tEnd) bL = 1;
  if (x2 + tol > xStart && x2 - tol < tEnd) bR = 1;
  double diff = xStart + first * dx - x1;
  if (first > 0 && bL) {
    out += 0.5 * diff * (diff / dx) * (vals[first - 1] - vals[first]);
    out += vals[first] * diff;
  } else
    out += na * diff;
  diff = x2 - (xStart + last * dx);
  if (last < (size_t)(nPts - 1) && bR) {
    out += 0.5 * diff * (diff / dx) * (vals[last + 1] - vals[last]);
    out += vals[last] * diff;
  } else
    out += na * diff;
  return out;
}

/* TimePred::integrate (TimePred.hpp:165-202): tIntE = int_0^dt of the Taylor expansion of the
 * elastic derivatives derE [O][9][B][R]; all modes with anelasticity, CK modes without */
void oracle_integrate(int O, int R, int rm, double dt, const double *derE, double *tIntE) {
  const int B = nmodes(O);
  const size_t szE = (size_t)9 * B * R;
  double sca = dt;
  for (size_t i = 0; i < szE; i++) tIntE[i] = sca * derE[i];
  for (int de = 1; de < O; de++) {
    sca *= dt / (de + 1);
    const int nCp = rm == 0 ? nmodes(O - de) : B;
    for (int q = 0; q < 9; q++)
      for (int md = 0; md < nCp; md++)
        for (int r = 0; r < R; r++) {
          size_t k = ((size_t)q * B + md) * R + r;
          tIntE[k] += sca * derE[(size_t)de * szE + k];
        }
  }
}

/* face types of the per-element face table */
enum { FT_INNER = 0, FT_FREE = 1, FT_OUTFLOW = 2 };
/* rate-2 LTS: element flags (AderDg.hpp:384-417) and relation to the face neighbour (622-674) */
enum { LTS_HAS_LARGER = 1, LTS_HAS_SMALLER = 2 };
enum { LTS_EQ = 0, LTS_GT = 1, LTS_LT = 2 };

/*
 * Local step (CK, receivers, volume, local surface) of the elements [first, first+n).
 * Receivers: nRe receivers grouped by element (recvEl ascending, equal elements adjacent); each
 * has basis values recvBasis[nRe][B] and its next output time recvTime[nRe] (updated). Output:
 * recvBuf[nRe][maxBuf][9][R], recvBufTime[nRe][maxBuf], recvCount[nRe] (updated). A group of
 * receivers in one element is evaluated at the first receiver's time (Receivers.cpp:250-290).
 * LTS (ltsFlags != NULL): elements with a larger neighbour add their time integral to tDofs1
 * (reset when firstTs), elements with a smaller neighbour store the integral over [0, dt/2] in
 * tDofs2 (AderDg.hpp:384-417).
 */
static int local_range(int O, int R, int rm, long first, long n, double t, double dt,
                       const double *stiffT, const double *stiffV, const double *fluxL,
                       const double *fluxT, const double *starE, const double *starA,
                       const double *srcA, const double *omega, const double *fsE, const double *fsA,
                       double *dofsE, double *dofsA, double *tDofs, const unsigned char *ltsFlags,
                       int firstTs, double *tDofs1, double *tDofs2, int nRe, const long *recvEl,
                       const double *recvBasis, double *recvTime, double period, int maxBuf,
                       double *recvBuf, double *recvBufTime, int *recvCount, double tolTime) {
  const int B = nmodes(O);
  const size_t szE = (size_t)9 * B * R, szM = (size_t)6 * B * R;
  int overflow = 0;
#pragma omp parallel reduction(| : overflow)
  {
  double *der = malloc((size_t)O * szE * sizeof(double));
  double *tIntA = rm ? malloc((size_t)rm * szM * sizeof(double)) : NULL;
  double *pred = malloc(szE * sizeof(double));
#pragma omp for schedule(dynamic, 16)
  for (long el = first; el < first + n; el++) {
    double *dE = dofsE + el * szE, *dA = rm ? dofsA + el * rm * szM : NULL;
    double *tD = tDofs + el * szE;
    oracle_ck(O, R, rm, dt, stiffT, starE + el * 72, rm ? starA + el * 27 : NULL,
              rm ? srcA + el * 12 * rm : NULL, omega, dE, dA, der, tD, tIntA);
    if (ltsFlags && (ltsFlags[el] & LTS_HAS_LARGER)) {
      double *t1 = tDofs1 + el * szE;
      if (firstTs) memset(t1, 0, szE * sizeof(double));
      for (size_t i = 0; i < szE; i++) t1[i] += tD[i];
    }
    if (ltsFlags && (ltsFlags[el] & LTS_HAS_SMALLER)) oracle_integrate(O, R, rm, 0.5 * dt, der, tDofs2 + el * szE);
    int lo = 0, hi = nRe;
    while (lo < hi) {
      int mid = (lo + hi) / 2;
      if (recvEl[mid] < el) lo = mid + 1; else hi = mid;
    }
    const int re = lo;
    if (re < nRe && recvEl[re] == el) {
      for (;;) {
        double tr = recvTime[re];
        if (!(tr > t - tolTime && tr < t + dt - tolTime)) break;
        oracle_eval_pred(O, R, fabs(tr - t), der, pred);
        for (int r2 = re; r2 < nRe && recvEl[r2] == el; r2++) {
          if (recvCount[r2] >= maxBuf) { overflow = 1; recvTime[re] = t + dt; break; }
          double *buf = recvBuf + ((size_t)r2 * maxBuf + recvCount[r2]) * 9 * R;
          for (int q = 0; q < 9; q++) {
            for (int r = 0; r < R; r++) buf[q * R + r] = 0;
            for (int md = 0; md < B; md++)
              for (int r = 0; r < R; r++)
                buf[q * R + r] += recvBasis[(size_t)r2 * B + md] * pred[((size_t)q * B + md) * R + r];
          }
          recvBufTime[(size_t)r2 * maxBuf + recvCount[r2]] = recvTime[r2];
          recvTime[r2] += period;
          recvCount[r2]++;
        }
      }
    }
    oracle_volint(O, R, rm, stiffV, starE + el * 72, rm ? starA + el * 27 : NULL,
                  rm ? srcA + el * 12 * rm : NULL, omega, tD, tIntA, dE, dA);
    oracle_surf_local(O, R, rm, fluxL, fluxT, fsE + el * 4 * 81,
                      rm ? fsA + el * 4 * 54 : NULL, omega, tD, dE, dA);
  }
  free(der);
  free(tIntA);
  free(pred);
  }
  return overflow ? -1 : 0;
}

/* Point sources of the elements [first, first+n) over [t, t+dt] (PointSources::apply,
 * PointSources.hpp:887-931). Sources are sorted by (element, run); source s adds
 * int_{t}^{t+dt} series * srcScal[s][q] * srcBEval[s][md] to run srcRun[s] of element srcEl[s].
 * Series s has srcNPts[s] samples at srcTsOff[s] in srcTs, start time srcT0[s], spacing srcDt[s]. */
static void sources_range(int O, int R, long first, long n, double t, double dt, double *dofsE,
                          int nSrc, const long *srcEl, const int *srcRun, const double *srcScal,
                          const double *srcBEval, const double *srcT0, const double *srcDt,
                          const long *srcTsOff, const long *srcNPts, const double *srcTs,
                          double tolTime) {
  const int B = nmodes(O);
  const size_t szE = (size_t)9 * B * R;
  for (int s = 0; s < nSrc; s++) {
    if (srcEl[s] < first || srcEl[s] >= first + n) continue;
    double in = oracle_series_int(srcDt[s], srcT0[s], srcNPts[s], srcTs + srcTsOff[s], t, t + dt,
                                  0.0, tolTime);
    double *dE = dofsE + srcEl[s] * szE;
    for (int q = 0; q < 9; q++) {
      double sc = in * srcScal[(size_t)s * 9 + q];
      for (int md = 0; md < B; md++)
        dE[((size_t)q * B + md) * R + srcRun[s]] += sc * srcBEval[(size_t)s * B + md];
    }
  }
}

/* Neighbour step of the elements [first, first+n) (AderDg::neigh, AderDg.hpp:553-722). With LTS
 * (ltsRel != NULL, [nEl][4]) the neighbour's time integral over this element's step is tDofs of
 * an equal neighbour, tDofs1 of a smaller one (two steps summed) and, for a larger neighbour,
 * tDofs2 (first half) on the first step of a pair, tDofs - tDofs2 (second half) otherwise. */
static void neigh_range(int O, int R, int rm, long first, long n, long nEl, const double *fluxL,
                        const double *fluxN, const double *fluxT, const double *fsE, const double *fsA,
                        const double *omega, const int *elFaEl, const unsigned char *fIdElFaEl,
                        const unsigned char *vIdElFaEl, const unsigned char *faType,
                        const double *tDofs, const unsigned char *ltsRel, int firstTs,
                        const double *tDofs1, const double *tDofs2, double *dofsE, double *dofsA) {
  const int B = nmodes(O);
  const size_t szE = (size_t)9 * B * R, szM = (size_t)6 * B * R;
  const double *fsE1 = fsE + (size_t)nEl * 4 * 81;
  const double *fsA1 = rm ? fsA + (size_t)nEl * 4 * 54 : NULL;
#pragma omp parallel
  {
  double *upA = rm ? malloc(szM * sizeof(double)) : NULL;
  double *diff = malloc(szE * sizeof(double));
#pragma omp for schedule(dynamic, 16)
  for (long el = first; el < first + n; el++) {
    if (rm) memset(upA, 0, szM * sizeof(double));
    for (int f = 0; f < 4; f++) {
      int ty = faType[el * 4 + f];
      if (ty == FT_OUTFLOW) continue;
      long ne = ty == FT_FREE ? el : elFaEl[el * 4 + f];
      int vId = ty == FT_FREE ? -1 : vIdElFaEl[el * 4 + f];
      int fId = ty == FT_FREE ? -1 : fIdElFaEl[el * 4 + f];
      const double *tNe = tDofs + ne * szE;
      const int rel = (ltsRel && ty == FT_INNER) ? ltsRel[el * 4 + f] : LTS_EQ;
      if (rel == LTS_GT) {
        tNe = tDofs1 + ne * szE;
      } else if (rel == LTS_LT) {
        if (firstTs) {
          tNe = tDofs2 + ne * szE;
        } else {
          for (size_t i = 0; i < szE; i++) diff[i] = tDofs[ne * szE + i] - tDofs2[ne * szE + i];
          tNe = diff;
        }
      }
      oracle_surf_neigh(O, R, rm, f, vId, fId, fluxL, fluxN, fluxT, fsE1 + (el * 4 + f) * 81,
                        rm ? fsA1 + (el * 4 + f) * 54 : NULL, tNe, dofsE + el * szE, upA);
    }
    if (rm) scatter_upA(B, R, rm, omega, upA, dofsA + el * rm * szM);
  }
  free(upA);
  free(diff);
  }
}

/* One GTS time step over the whole mesh: local -> point sources -> neighbour (steps 0/1/2 of
 * src/impl/seismic/steps.inc:24-77). Returns -1 when a receiver buffer is full. */
int oracle_step(int O, int R, int rm, long nEl, double t, double dt, const double *stiffT,
                const double *stiffV, const double *fluxL, const double *fluxN,
                const double *fluxT, const double *starE, const double *starA,
                const double *srcA, const double *omega, const double *fsE, const double *fsA,
                const int *elFaEl, const unsigned char *fIdElFaEl,
                const unsigned char *vIdElFaEl, const unsigned char *faType, double *dofsE,
                double *dofsA, double *tDofs,
                /* receivers */ int nRe, const long *recvEl, const double *recvBasis,
                double *recvTime, double period, int maxBuf, double *recvBuf,
                double *recvBufTime, int *recvCount,
                /* sources */ int nSrc, const long *srcEl, const int *srcRun,
                const double *srcScal, const double *srcBEval, const double *srcT0,
                const double *srcDt, const long *srcTsOff, const long *srcNPts,
                const double *srcTs, double tolTime) {
  if (local_range(O, R, rm, 0, nEl, t, dt, stiffT, stiffV, fluxL, fluxT, starE, starA, srcA, omega, fsE,
                  fsA, dofsE, dofsA, tDofs, NULL, 0, NULL, NULL, nRe, recvEl, recvBasis, recvTime, period,
                  maxBuf, recvBuf, recvBufTime, recvCount, tolTime))
    return -1;
  sources_range(O, R, 0, nEl, t, dt, dofsE, nSrc, srcEl, srcRun, srcScal, srcBEval, srcT0, srcDt, srcTsOff,
                srcNPts, srcTs, tolTime);
  neigh_range(O, R, rm, 0, nEl, nEl, fluxL, fluxN, fluxT, fsE, fsA, omega, elFaEl, fIdElFaEl, vIdElFaEl,
              faType, tDofs, NULL, 0, NULL, NULL, dofsE, dofsA);
  return 0;
}

/* Rate-2 LTS work regions of one time group (the elements [first, first+n)): local with the
 * tDofs1 / tDofs2 bookkeeping, then its sources, and later its neighbour step (TimeGroupStatic
 * computeStep with steps.inc:24-77; the order across groups is the caller's). */
int oracle_lts_local(int O, int R, int rm, long first, long n, int firstTs, double t, double dt,
                     const double *stiffT, const double *stiffV, const double *fluxL, const double *fluxT,
                     const double *starE, const double *starA, const double *srcA, const double *omega,
                     const double *fsE, const double *fsA, const unsigned char *ltsFlags, double *dofsE,
                     double *dofsA, double *tDofs, double *tDofs1, double *tDofs2, int nRe,
                     const long *recvEl, const double *recvBasis, double *recvTime, double period,
                     int maxBuf, double *recvBuf, double *recvBufTime, int *recvCount, int nSrc,
                     const long *srcEl, const int *srcRun, const double *srcScal, const double *srcBEval,
                     const double *srcT0, const double *srcDt, const long *srcTsOff, const long *srcNPts,
                     const double *srcTs, double tolTime) {
  if (local_range(O, R, rm, first, n, t, dt, stiffT, stiffV, fluxL, fluxT, starE, starA, srcA, omega, fsE,
                  fsA, dofsE, dofsA, tDofs, ltsFlags, firstTs, tDofs1, tDofs2, nRe, recvEl, recvBasis,
                  recvTime, period, maxBuf, recvBuf, recvBufTime, recvCount, tolTime))
    return -1;
  sources_range(O, R, first, n, t, dt, dofsE, nSrc, srcEl, srcRun, srcScal, srcBEval, srcT0, srcDt, srcTsOff,
                srcNPts, srcTs, tolTime);
  return 0;
}

void oracle_lts_neigh(int O, int R, int rm, long first, long n, long nEl, int firstTs, const double *fluxL,
                      const double *fluxN, const double *fluxT, const double *fsE, const double *fsA,
                      const double *omega, const int *elFaEl, const unsigned char *fIdElFaEl,
                      const unsigned char *vIdElFaEl, const unsigned char *faType,
                      const unsigned char *ltsRel, const double *tDofs, const double *tDofs1,
                      const double *tDofs2, double *dofsE, double *dofsA) {
  neigh_range(O, R, rm, first, n, nEl, fluxL, fluxN, fluxT, fsE, fsA, omega, elFaEl, fIdElFaEl, vIdElFaEl,
              faType, tDofs, ltsRel, firstTs, tDofs1, tDofs2, dofsE, dofsA);
}
