// Test harness around the reference's own AderDg class (compiled from the reference checkout into
// oracle/_ref by oracle/ref.mk; TEST INFRASTRUCTURE ONLY).
//
// It calls, unchanged, edge::seismic::solvers::AderDg<double, 0, TET4, O, O, R, false>::local and
// ::neigh (src/impl/seismic/solvers/AderDg.hpp:338-534 and 553-722) with their rate-2 LTS branches
// (summed time integrals 384-417, half-step integrals through TimePred::integrate, the "=", "<" and
// ">" gathers 620-674) on the vanilla kernels, so that the oracle's restatement of those branches
// (oracle.c oracle_lts_local / oracle_lts_neigh) is checked against the reference's code.
//
// The class keeps its element data in private members filled by its constructor from the mesh
// geometry; the harness fills the same members from the caller's star matrices and flux solvers
// (AderDgInit's layouts), which is why the header is included with private access opened. The
// receiver output the local step would write goes through io::Receivers, whose source needs a
// geometry library absent here; no element carries the RECEIVER flag, so the two methods below
// are never called and only satisfy the linker.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#define private public
#include "impl/seismic/solvers/AderDg.hpp"
#undef private

#include "edge_b200/csrc/gen/dg_tet.h"

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define DGM(name) CAT(CAT(edge_dg_, name), CAT(_O, PP_ORDER))

static const unsigned short O = PP_ORDER;
static const unsigned short R = PP_N_CRUNS;
static const unsigned short B = CE_N_ELEMENT_MODES(TET4, PP_ORDER);

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
std::size_t const g_fluxLSize = (std::size_t)4 * B * CE_N_ELEMENT_MODES(TRIA3, PP_ORDER);
double const *g_fluxNRaw = DGM(fluxN);
std::size_t const g_fluxNSize = (std::size_t)12 * B * CE_N_ELEMENT_MODES(TRIA3, PP_ORDER);
double const *g_fluxTRaw = DGM(fluxT);
std::size_t const g_fluxTSize = (std::size_t)4 * B * CE_N_ELEMENT_MODES(TRIA3, PP_ORDER);
}}}

// link-only definitions (see the header comment)
double edge::io::Receivers::getRecvTimeRel(std::size_t, double, double) { return -1; }
void edge::io::Receivers::writeRecvAll(std::size_t, double const (*)[N_ELEMENT_MODES][N_CRUNS]) {}

using AD = edge::seismic::solvers::AderDg<double, 0, TET4, O, O, R, false>;
typedef double tDofsE_t[9][B][R];
typedef double tBlk_t[B][R];

namespace {
struct State {
  edge::data::Dynamic mem;
  alignas(AD) unsigned char obj[sizeof(AD)];
  AD *ad = nullptr;
  long nEl = 0;
  std::vector<double> starDense, fs0, fs1;
  std::vector<t_elementChars> elChars;
  std::vector<t_faceChars> faChars;
  std::vector<long> elFa, elFaEl;
  std::vector<unsigned short> fIdElFaEl, vIdElFaEl;
  std::vector<tBlk_t *> tPtr[3];
  t_scratchMem *scratch = nullptr;
};
State *g = nullptr;

const int SE_R[24] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 6, 7, 7, 7, 8, 8, 8};
const int SE_C[24] = {6, 7, 8, 6, 7, 8, 6, 7, 8, 6, 7, 7, 8, 6, 8, 0, 3, 5, 1, 3, 4, 2, 4, 5};
}  // namespace

extern "C" {

int ref_lts_config(int *o, int *r) {
  *o = O;
  *r = R;
  return 0;
}

// Element data and connectivity of the mesh (layouts of oracle.c: starE [nEl][3][24] sparse,
// fsE [2][nEl][4][81], elFaEl / fId / vId / faType [nEl][4] with faType 0 inner, 1 free surface,
// 2 outflow), the LTS relations (flags [nEl]: 1 a neighbour with a larger step, 2 one with a
// smaller step; rel [nEl][4]: 0 equal, 1 this element's step larger, 2 smaller) and the three
// time-integral buffers tDofs, tDofs1, tDofs2 [nEl][9][B][R] the calls below write and read.
int ref_lts_setup(long nEl, const double *starE, const double *fsE, const int *elFaEl, const unsigned char *fId,
                  const unsigned char *vId, const unsigned char *faType, const unsigned char *flags,
                  const unsigned char *rel, double *tDofs, double *tDofs1, double *tDofs2) {
  delete g;
  g = new State();
  g->nEl = nEl;
  std::streambuf *saved = std::cout.rdbuf(nullptr);
  AD *ad = reinterpret_cast<AD *>(g->obj);
  std::memset(g->obj, 0, sizeof(g->obj));
  ad->m_kernels = new edge::seismic::kernels::Kernels<double, 0, TET4, O, O, R>(nullptr, g->mem);
  std::cout.rdbuf(saved);
  std::cout.clear();
  g->starDense.assign((size_t)nEl * 3 * 81, 0.0);
  for (long e = 0; e < nEl; e++)
    for (int d = 0; d < 3; d++)
      for (int i = 0; i < 24; i++) g->starDense[(e * 3 + d) * 81 + SE_R[i] * 9 + SE_C[i]] = starE[(e * 3 + d) * 24 + i];
  g->fs0.assign(fsE, fsE + (size_t)nEl * 4 * 81);
  g->fs1.assign(fsE + (size_t)nEl * 4 * 81, fsE + (size_t)2 * nEl * 4 * 81);
  ad->m_starE = reinterpret_cast<double(*)[3][81]>(g->starDense.data());
  ad->m_fsE[0] = reinterpret_cast<double(*)[4][81]>(g->fs0.data());
  ad->m_fsE[1] = reinterpret_cast<double(*)[4][81]>(g->fs1.data());
  g->ad = ad;
  // element and face characteristics: one face record per element face (4 e + f)
  g->elChars.assign(nEl, t_elementChars{});
  g->faChars.assign((size_t)nEl * 4, t_faceChars{});
  g->elFa.resize((size_t)nEl * 4);
  g->elFaEl.resize((size_t)nEl * 4);
  g->fIdElFaEl.resize((size_t)nEl * 4);
  g->vIdElFaEl.resize((size_t)nEl * 4);
  for (long e = 0; e < nEl; e++) {
    int_spType sp = 0;
    if (flags[e] & 1) sp |= C_LTS_EL[EL_INT_LT];
    if (flags[e] & 2) sp |= C_LTS_EL[EL_INT_GT];
    for (int f = 0; f < 4; f++) {
      const size_t i = (size_t)e * 4 + f;
      const int r = rel[i];
      sp |= C_LTS_AD[f][r == 0 ? AD_EQ : r == 1 ? AD_GT : AD_LT];
      g->elFa[i] = (long)i;
      g->faChars[i].spType = faType[i] == 1 ? FREE_SURFACE : faType[i] == 2 ? OUTFLOW : 0;
      g->elFaEl[i] = elFaEl[i] < 0 ? std::numeric_limits<long>::max() : elFaEl[i];
      g->fIdElFaEl[i] = fId[i];
      g->vIdElFaEl[i] = vId[i];
    }
    g->elChars[e].spType = sp;
  }
  double *buf[3] = {tDofs, tDofs1, tDofs2};
  for (int k = 0; k < 3; k++) {
    g->tPtr[k].resize(nEl);
    for (long e = 0; e < nEl; e++) g->tPtr[k][e] = reinterpret_cast<tBlk_t *>(buf[k] + (size_t)e * 9 * B * R);
  }
  // the per-thread scratch of the reference's work regions (data/Internal.hpp:449), aligned
  const size_t scratchBytes = (sizeof(t_scratchMem) + 4095) / 4096 * 4096;
  g->scratch = static_cast<t_scratchMem *>(aligned_alloc(4096, scratchBytes));
  if (!g->scratch) return -2;
  std::memset(static_cast<void *>(g->scratch), 0, scratchBytes);
  edge::parallel::g_scratchMem = g->scratch;
  return 0;
}

// AderDg::local over the elements [first, first + n) (no receivers, no MPI send faces)
int ref_lts_local(long first, long n, int firstTs, double t, double dt, double *dofsE) {
  if (!g) return -1;
  tBlk_t *const *tp[3] = {g->tPtr[0].data(), g->tPtr[1].data(), g->tPtr[2].data()};
  // storage standing in for the receiver object, which the local step does not touch here
  alignas(edge::io::Receivers) static unsigned char recvStore[sizeof(edge::io::Receivers)];
  edge::io::Receivers *noRecv = reinterpret_cast<edge::io::Receivers *>(recvStore);
  g->ad->local(first, n, firstTs != 0, t, dt, (long)0, g->elChars.data(),
               reinterpret_cast<unsigned short const(*)[4]>(g->vIdElFaEl.data()),
               reinterpret_cast<tDofsE_t *>(dofsE), (tBlk_t *)nullptr, tp, (double(*const *)[CE_N_ELEMENT_MODES(TRIA3, PP_ORDER)][R]) nullptr,
               *noRecv);
  return 0;
}

// AderDg::neigh over the elements [first, first + n)
int ref_lts_neigh(long first, long n, int firstTs, double *dofsE) {
  if (!g) return -1;
  tBlk_t *const *tp[3] = {g->tPtr[0].data(), g->tPtr[1].data(), g->tPtr[2].data()};
  g->ad->neigh(first, n, firstTs != 0, g->faChars.data(), g->elChars.data(),
               reinterpret_cast<long const(*)[4]>(g->elFa.data()), reinterpret_cast<long const(*)[4]>(g->elFaEl.data()),
               reinterpret_cast<unsigned short const(*)[4]>(g->fIdElFaEl.data()),
               reinterpret_cast<unsigned short const(*)[4]>(g->vIdElFaEl.data()), tp,
               reinterpret_cast<tDofsE_t *>(dofsE), (tBlk_t *)nullptr,
               (double const(*const *)[CE_N_ELEMENT_MODES(TRIA3, PP_ORDER)][R]) nullptr);
  return 0;
}

}  // extern "C"
