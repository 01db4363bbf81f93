// Test harness around the reference's own code (compiled from the reference checkout into
// oracle/_ref by oracle/ref.mk; TEST INFRASTRUCTURE ONLY).
//
// It drives, unchanged:
//   * TimePredVanilla / VolIntVanilla / SurfIntVanilla (src/impl/seismic/kernels/*Vanilla.hpp) over
//     one GTS step, restating the loop of AderDg::local (AderDg.hpp:338-534, receivers omitted)
//     and AderDg::neigh (AderDg.hpp:553-722) with OpenMP over element ranges as EDGE's work
//     regions do (src/parallel/Shared.h:179-260);
//   * Elasticity::star / Elasticity::fs (src/impl/seismic/setups/Elasticity.cpp:167-441) and
//     seismic::common::setupTrafo3d / setupTrafoInv3d (src/impl/seismic/common.hpp:314-343);
//   * ViscoElasticity::frequencies (ViscoElasticity.h:168-183);
//   * linalg::Series<1>::integrate (src/linalg/Series.hpp:59-134).
// The global DG matrices the reference links as edge::pre::dg::g_* (src/dg/Basis.h:38-59) are
// provided from this repository's generator, which reproduces the reference pre-processor's values.
#include <cstddef>
#include <cstring>
#include <iostream>
#include <vector>

#include "impl/seismic/kernels/TimePredVanilla.hpp"
#include "impl/seismic/kernels/VolIntVanilla.hpp"
#include "impl/seismic/kernels/SurfIntVanilla.hpp"
#include "impl/seismic/setups/Elasticity.h"
#include "impl/seismic/setups/ViscoElasticity.h"
#include "impl/seismic/common.hpp"
#include "linalg/Series.hpp"
#include "linalg/Mappings.hpp"
#include "linalg/Matrix.h"
#include "dg/Basis.h"
#include "data/Dynamic.h"

#include "edge_b200/csrc/gen/dg_tet.h"

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define DGM(name) CAT(CAT(edge_dg_, name), CAT(_O, PP_ORDER))

static const unsigned short O = PP_ORDER;
static const unsigned short R = PP_N_CRUNS;
static const unsigned short RM = PP_N_RELAXATION_MECHANISMS;
static const unsigned short B = CE_N_ELEMENT_MODES(TET4, PP_ORDER);
static const unsigned short F = CE_N_ELEMENT_MODES(TRIA3, PP_ORDER);

// ---- the pre-processed DG matrices the reference links against ---------------------------------
static std::vector<double> makeMass() {
  std::vector<double> m((size_t)B * B, 0.0);
  for (int i = 0; i < B; i++) m[(size_t)i * B + i] = DGM(mass)[i];
  return m;
}
static std::vector<double> g_massStore = makeMass();
namespace edge { namespace pre { namespace dg {
double const *g_massRaw = g_massStore.data();
std::size_t const g_massSize = (std::size_t)B * B;
double const *g_stiffVRaw = DGM(stiffV);
std::size_t const g_stiffVSize = (std::size_t)3 * B * B;
double const *g_stiffTRaw = DGM(stiffT);
std::size_t const g_stiffTSize = (std::size_t)3 * B * B;
double const *g_fluxLRaw = DGM(fluxL);
std::size_t const g_fluxLSize = (std::size_t)4 * B * F;
double const *g_fluxNRaw = DGM(fluxN);
std::size_t const g_fluxNSize = (std::size_t)12 * B * F;
double const *g_fluxTRaw = DGM(fluxT);
std::size_t const g_fluxTSize = (std::size_t)4 * B * F;
}}}

using TP = edge::seismic::kernels::TimePredVanilla<double, RM, TET4, O, O, R>;
using VI = edge::seismic::kernels::VolIntVanilla<double, RM, TET4, O, R>;
using SI = edge::seismic::kernels::SurfIntVanilla<double, RM, TET4, O, R>;

struct Kernels {
  edge::data::Dynamic mem;
  TP *tp;
  VI *vi;
  SI *si;
  explicit Kernels(const double *omega) {
    double w[RM > 0 ? RM : 1] = {0};
    for (int i = 0; i < RM; i++) w[i] = omega[i];
    // without easylogging the reference's verbose logs go to std::cout (io/logging.h:66-78);
    // silence them while the kernels are generated
    std::streambuf *saved = std::cout.rdbuf(nullptr);
    tp = new TP(RM ? w : nullptr, mem);
    vi = new VI(RM ? w : nullptr, mem);
    si = new SI(RM ? w : nullptr, mem);
    std::cout.rdbuf(saved);
    std::cout.clear();
  }
  ~Kernels() { delete tp; delete vi; delete si; }
};

static const int SE_R[24] = {0,0,0,1,1,1,2,2,2,3,3,4,4,5,5,6,6,6,7,7,7,8,8,8};
static const int SE_C[24] = {6,7,8,6,7,8,6,7,8,6,7,7,8,6,8,0,3,5,1,3,4,2,4,5};
static const int SA_R[9] = {0,1,2,3,3,4,4,5,5};
static const int SA_C[9] = {0,1,2,0,1,1,2,0,2};
static const int SR_R[12] = {0,0,0,1,1,1,2,2,2,3,4,5};
static const int SR_C[12] = {0,1,2,0,1,2,0,1,2,3,4,5};

typedef double tDofs_t[9][B][R];

extern "C" {

int ref_config(int *o, int *r, int *rm) {
  *o = O; *r = R; *rm = RM;
  return 0;
}

// one GTS step of the reference kernels: local -> (sources applied by the caller) -> neigh.
// Arrays as in oracle.c; phase = 0 runs the local step, 1 the neighbour step.
int ref_step_phase(int phase, long nEl, double dt, const double *starE, const double *starA,
                   const double *srcA, const double *omega, const double *fsE, const double *fsA,
                   const int *elFaEl, const unsigned char *fId, const unsigned char *vId,
                   const unsigned char *faType, double *dofsE, double *dofsA, double *tDofs) {
  static Kernels *k = nullptr;
  if (!k) k = new Kernels(omega);
  const size_t szE = (size_t)9 * B * R, szM = (size_t)6 * B * R;
  if (phase == 0) {
#pragma omp parallel
    {
      std::vector<double> der((size_t)O * szE), scr(szE), tmpFa(2 * (size_t)9 * F * R);
      std::vector<double> tA((size_t)(RM ? RM : 1) * szM), dA((size_t)(RM ? RM : 1) * O * szM);
#pragma omp for schedule(static)
      for (long el = 0; el < nEl; el++) {
        double st[3][81] = {{0}}, sa[3][18] = {{0}}, sr[RM ? RM : 1][36];
        for (int d = 0; d < 3; d++) {
          for (int i = 0; i < 24; i++) st[d][SE_R[i] * 9 + SE_C[i]] = starE[(el * 3 + d) * 24 + i];
          if (RM) for (int i = 0; i < 9; i++) sa[d][SA_R[i] * 3 + SA_C[i]] = starA[(el * 3 + d) * 9 + i];
        }
        for (int m = 0; m < RM; m++) {
          std::memset(sr[m], 0, sizeof(sr[m]));
          for (int i = 0; i < 12; i++) sr[m][SR_R[i] * 6 + SR_C[i]] = srcA[(el * RM + m) * 12 + i];
        }
        double (*dE)[B][R] = (double (*)[B][R])(dofsE + el * szE);
        double (*dAe)[6][B][R] = RM ? (double (*)[6][B][R])(dofsA + el * RM * szM) : nullptr;
        double (*tD)[B][R] = (double (*)[B][R])(tDofs + el * szE);
        k->tp->ck(dt, st, RM ? sa : nullptr, RM ? sr : nullptr, dE, dAe,
                  (double (*)[B][R])scr.data(), (double (*)[9][B][R])der.data(),
                  RM ? (double (*)[O][6][B][R])dA.data() : nullptr, tD,
                  RM ? (double (*)[6][B][R])tA.data() : nullptr);
        k->vi->apply(st, RM ? sa : nullptr, RM ? sr : nullptr, tD,
                     RM ? (double (*)[6][B][R])tA.data() : nullptr, dE, dAe,
                     (double (*)[B][R])scr.data());
        double fl[4][81], fa[4][54];
        for (int f = 0; f < 4; f++) {
          std::memcpy(fl[f], fsE + (el * 4 + f) * 81, sizeof(fl[f]));
          if (RM) std::memcpy(fa[f], fsA + (el * 4 + f) * 54, sizeof(fa[f]));
        }
        k->si->local(fl, RM ? fa : nullptr, tD, dE, dAe, (double (*)[9][F][R])tmpFa.data());
      }
    }
    return 0;
  }
  const double *fsE1 = fsE + (size_t)nEl * 4 * 81;
  const double *fsA1 = RM ? fsA + (size_t)nEl * 4 * 54 : nullptr;
#pragma omp parallel
  {
    std::vector<double> tmpFa(2 * (size_t)9 * F * R), upA(szM), tNe(szE);
#pragma omp for schedule(static)
    for (long el = 0; el < nEl; el++) {
      std::fill(upA.begin(), upA.end(), 0.0);
      for (int f = 0; f < 4; f++) {
        if (faType[el * 4 + f] == 2) continue;  // outflow
        bool fs = faType[el * 4 + f] == 1;
        long ne = fs ? el : elFaEl[el * 4 + f];
        unsigned short v = fs ? std::numeric_limits<unsigned short>::max() : vId[el * 4 + f];
        unsigned short fi = fs ? std::numeric_limits<unsigned short>::max() : fId[el * 4 + f];
        std::memcpy(tNe.data(), tDofs + ne * szE, szE * sizeof(double));
        k->si->neigh(f, v, fi, fsE1 + (el * 4 + f) * 81, RM ? fsA1 + (el * 4 + f) * 54 : nullptr,
                     (double (*)[B][R])tNe.data(), nullptr, (double (*)[B][R])(dofsE + el * szE),
                     (double (*)[B][R])upA.data(), (double (*)[9][F][R])tmpFa.data());
      }
      if (RM)
        k->si->scatterUpdateA((double (*)[B][R])upA.data(),
                              (double (*)[6][B][R])(dofsA + el * RM * szM));
    }
  }
  return 0;
}

void ref_star(double rho, double lam, double mu, const double *jacInv, double *out24x3) {
  double ji[3][3];
  for (int i = 0; i < 9; i++) ji[i / 3][i % 3] = jacInv[i];
  double o[3][24];
  edge::seismic::setups::Elasticity::star(rho, lam, mu, ji, o);
  std::memcpy(out24x3, o, sizeof(o));
}

void ref_trafo(const double *n, const double *s, const double *t, double *T, double *Ti) {
  double a[9][9], b[9][9];
  edge::seismic::common::setupTrafo3d(n[0], n[1], n[2], s[0], s[1], s[2], t[0], t[1], t[2], a);
  edge::seismic::common::setupTrafoInv3d(n[0], n[1], n[2], s[0], s[1], s[2], t[0], t[1], t[2], b);
  std::memcpy(T, a, sizeof(a));
  std::memcpy(Ti, b, sizeof(b));
}

void ref_fs(double rhoL, double rhoR, double lamL, double lamR, double muL, double muR,
            const double *n, const double *s, const double *t, int freeSurface, double *fsl,
            double *fsr) {
  double a[9][9], b[9][9];
  edge::seismic::common::setupTrafo3d(n[0], n[1], n[2], s[0], s[1], s[2], t[0], t[1], t[2], a);
  edge::seismic::common::setupTrafoInv3d(n[0], n[1], n[2], s[0], s[1], s[2], t[0], t[1], t[2], b);
  edge::seismic::setups::Elasticity::fs(rhoL, rhoR, lamL, lamR, muL, muR, a, b, fsl, fsr,
                                        freeSurface != 0);
}

void ref_frequencies(int n, double fc, double fr, double *out) {
  edge::seismic::setups::ViscoElasticity::frequencies(n, fc, fr, out);
}

// a point in a tet's reference coordinates (linalg::Mappings::phyToRefTet4; ves [3 dims][4 vertices]),
// the element basis there (dg::Basis::evalBasis) and the determinant of the element's Jacobian
// (Mappings::evalJac, Matrix::det): the steps receivers and point sources take to their basis
// values (Receivers.cpp:127-143; PointSources.hpp:458-495, which also scales by the inverse mass
// matrix and divides by the determinant)
void ref_locate_eval(const double *ves, const double *x, double *ref, double *basis, double *jacDet) {
  edge::linalg::Mappings::phyToRefTet4((const double (*)[4])ves, x, ref);
  for (int md = 0; md < B; md++) basis[md] = edge::dg::Basis::evalBasis(md, TET4, ref[0], ref[1], ref[2]);
  double jac[3][3];
  edge::linalg::Mappings::evalJac(TET4, ves, jac[0]);
  *jacDet = edge::linalg::Matrix::det(3, jac[0]);
}

double ref_series_int(double dx, double x0, long n, const double *vals, double x1, double x2) {
  double o[1];
  edge::linalg::Series<1>::integrate(dx, x0, (std::size_t)n, (const double (*)[1])vals, x1, x2, o, 0.0);
  return o[0];
}

}  // extern "C"
