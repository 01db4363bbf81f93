// Host-side setup of the tet4 ADER-DG element update, keeping EDGE's semantics:
// box meshes with EDGE-V's vertex / face / neighbour conventions, star matrices, Godunov flux
// solvers, attenuation, CFL time step, and point location for sources and receivers.
// Everything here runs once per simulation in FP64; the time loop lives on the device.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <vector>

#include "../../include/edge_b200.h"
#include "gen/dg_tet.h"

namespace {

constexpr double kTolMesh = 1e-9;  // TOL.MESH of the FP64 build (src/constants.hpp:289-309)

// -------------------------------------------------------------------------------------------------
// small dense helpers
// -------------------------------------------------------------------------------------------------
double det3(const double a[3][3]) {
  return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
         a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
         a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}

void inv3(const double a[3][3], double o[3][3]) {
  double d = det3(a);
  o[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / d;
  o[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / d;
  o[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / d;
  o[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / d;
  o[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / d;
  o[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / d;
  o[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / d;
  o[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / d;
  o[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / d;
}

void cross(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
double dot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double norm(const double a[3]) { return std::sqrt(dot(a, a)); }

// C = A * B for row-major dense matrices (M x K) * (K x N)
void matmul(int M, int N, int K, const double *A, const double *B, double *C) {
  for (int m = 0; m < M; m++)
    for (int n = 0; n < N; n++) {
      double s = 0;
      for (int k = 0; k < K; k++) s += A[m * K + k] * B[k * N + n];
      C[m * N + n] = s;
    }
}

// splitmix64: seeded, platform-independent random numbers for mesh jitter
struct Rng {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
};

}  // namespace

// -------------------------------------------------------------------------------------------------
// mesh
// -------------------------------------------------------------------------------------------------
struct edge_mesh {
  std::vector<double> ve;        // [nVe][3]
  std::vector<int64_t> elVe;     // [nEl][4]
  std::vector<int64_t> elFa;     // [nEl][4]
  std::vector<int64_t> faVe;     // [nFa][3] ascending vertex ids
  std::vector<int64_t> faEl;     // [nFa][2] ascending, -1 = none (left is always present)
  std::vector<uint8_t> faType;   // [nFa] EDGE_FACE_*
  std::vector<int64_t> faPartner; // [nFa] element across a periodic boundary face, -1 otherwise
  std::vector<double> faNormal;  // [nFa][3]
  std::vector<double> faTangent; // [nFa][2][3]
  std::vector<double> faArea;    // [nFa]
  std::vector<double> elVol, elInDia;
  std::vector<int32_t> elFaEl;   // [nEl][4]
  std::vector<uint8_t> fIdElFaEl, vIdElFaEl, elFaType;  // [nEl][4]
  // point-location grid over element bounding boxes
  double lo[3], hi[3];
  int ng[3];
  std::vector<int64_t> cellOff, cellEl;
  int64_t nVe() const { return (int64_t)ve.size() / 3; }
  int64_t nEl() const { return (int64_t)elVe.size() / 4; }
  int64_t nFa() const { return (int64_t)faVe.size() / 3; }
  void veCrds(int64_t el, double v[4][3]) const {
    for (int i = 0; i < 4; i++)
      for (int d = 0; d < 3; d++) v[i][d] = ve[3 * elVe[4 * el + i] + d];
  }
  // jac[d1][d2] = d x_{d2} / d xi_{d1} (linalg/Mappings.hpp:189-230)
  void jac(int64_t el, double j[3][3]) const {
    double v[4][3];
    veCrds(el, v);
    for (int a = 0; a < 3; a++)
      for (int d = 0; d < 3; d++) j[a][d] = v[a + 1][d] - v[0][d];
  }
};

namespace {

// tangents / normal of a triangle, oriented away from point np (geom/Tria3.cpp:48-120)
void triaFrame(const double v[3][3], const double np[3], double t0[3], double t1[3], double n[3]) {
  double d0[3], d1[3];
  for (int i = 0; i < 3; i++) {
    d0[i] = v[1][i] - v[0][i];
    d1[i] = v[2][i] - v[0][i];
  }
  double alpha = -dot(d0, d1) / dot(d0, d0);
  double n0[3];
  for (int i = 0; i < 3; i++) n0[i] = d1[i] + alpha * d0[i];
  double l0 = norm(d0), l1 = norm(n0);
  for (int i = 0; i < 3; i++) {
    d0[i] /= l0;
    n0[i] /= l1;
  }
  double n1[3], dn[3];
  cross(d0, n0, n1);
  for (int i = 0; i < 3; i++) dn[i] = np[i] - v[0][i];
  if (dot(n1, dn) > 0) std::swap(d0, n0);
  for (int i = 0; i < 3; i++) {
    t0[i] = d0[i];
    t1[i] = n0[i];
  }
  cross(t0, t1, n);
}

// local faces of the unit tet by their vertices, in face-parameter order: face 0 = (0,2,1),
// face 1 = (0,1,3), face 2 = (0,3,2), face 3 = (1,2,3) (edge_pre types/Tet.py:89-97)
const int kFaVe[4][3] = {{0, 2, 1}, {0, 1, 3}, {0, 3, 2}, {1, 2, 3}};

void buildLocateGrid(edge_mesh &m) {
  for (int d = 0; d < 3; d++) {
    m.lo[d] = std::numeric_limits<double>::max();
    m.hi[d] = -std::numeric_limits<double>::max();
  }
  const int64_t nVe = m.nVe(), nEl = m.nEl();
  for (int64_t v = 0; v < nVe; v++)
    for (int d = 0; d < 3; d++) {
      m.lo[d] = std::min(m.lo[d], m.ve[3 * v + d]);
      m.hi[d] = std::max(m.hi[d], m.ve[3 * v + d]);
    }
  int64_t per = std::max<int64_t>(1, (int64_t)std::cbrt((double)nEl / 4.0));
  for (int d = 0; d < 3; d++) m.ng[d] = (int)std::min<int64_t>(per, 512);
  auto cell = [&](int d, double x) {
    double f = (x - m.lo[d]) / (m.hi[d] - m.lo[d] + 1e-300) * m.ng[d];
    int c = (int)std::floor(f);
    return std::max(0, std::min(m.ng[d] - 1, c));
  };
  int64_t nCell = (int64_t)m.ng[0] * m.ng[1] * m.ng[2];
  std::vector<int64_t> cnt(nCell + 1, 0);
  std::vector<std::array<int, 6>> box(nEl);
  for (int64_t e = 0; e < nEl; e++) {
    double v[4][3];
    m.veCrds(e, v);
    for (int d = 0; d < 3; d++) {
      double a = std::min(std::min(v[0][d], v[1][d]), std::min(v[2][d], v[3][d]));
      double b = std::max(std::max(v[0][d], v[1][d]), std::max(v[2][d], v[3][d]));
      box[e][d] = cell(d, a - kTolMesh);
      box[e][3 + d] = cell(d, b + kTolMesh);
    }
    for (int i = box[e][0]; i <= box[e][3]; i++)
      for (int j = box[e][1]; j <= box[e][4]; j++)
        for (int k = box[e][2]; k <= box[e][5]; k++) cnt[((int64_t)k * m.ng[1] + j) * m.ng[0] + i + 1]++;
  }
  for (int64_t c = 0; c < nCell; c++) cnt[c + 1] += cnt[c];
  m.cellOff = cnt;
  m.cellEl.assign(cnt[nCell], 0);
  std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
  for (int64_t e = 0; e < nEl; e++)
    for (int i = box[e][0]; i <= box[e][3]; i++)
      for (int j = box[e][1]; j <= box[e][4]; j++)
        for (int k = box[e][2]; k <= box[e][5]; k++) m.cellEl[pos[((int64_t)k * m.ng[1] + j) * m.ng[0] + i]++] = e;
}

// EDGE-V normalisation: sort element vertices, then fix the orientation (mesh/Mesh.cpp:312-313,
// geom/Tet4.cpp:80-112); faces of an element with ascending vertices a<b<c<d are {abc},{abd},
// {acd},{bcd}, i.e. local face f omits local vertex 3-f. An element whose volume is below
// TOL.MESH relative to its longest edge cubed is degenerate.
int normalizeElements(edge_mesh &m) {
  const int64_t nEl = m.nEl();
  for (int64_t e = 0; e < nEl; e++) {
    int64_t *ev = &m.elVe[4 * e];
    std::sort(ev, ev + 4);
    double v[4][3];
    m.veCrds(e, v);
    double lMax = 0;
    for (int a = 0; a < 4; a++)
      for (int b = a + 1; b < 4; b++) {
        double d[3] = {v[b][0] - v[a][0], v[b][1] - v[a][1], v[b][2] - v[a][2]};
        lMax = std::max(lMax, norm(d));
      }
    double j3[3][3];
    m.jac(e, j3);
    const double d = det3(j3);
    if (!(std::abs(d) > kTolMesh * lMax * lMax * lMax)) return EDGE_B200_EMESH;
    if (d < 0) std::swap(ev[2], ev[3]);
  }
  return EDGE_B200_OK;
}

// unique faces in order of first appearance (element order, local face order), faEl ascending
// with "none" last (std::sort of faEl with none = max, Mesh.cpp:306); a face shared by more than
// two elements is an error
int buildFaces(edge_mesh &m) {
  const int64_t nEl = m.nEl();
  std::map<std::array<int64_t, 3>, int64_t> faceIds;
  m.elFa.assign(4 * nEl, -1);
  m.faVe.clear();
  m.faEl.clear();
  for (int64_t e = 0; e < nEl; e++) {
    const int64_t *ev = &m.elVe[4 * e];
    for (int f = 0; f < 4; f++) {
      std::array<int64_t, 3> key = {ev[kFaVe[f][0]], ev[kFaVe[f][1]], ev[kFaVe[f][2]]};
      std::sort(key.begin(), key.end());
      auto it = faceIds.find(key);
      int64_t fa;
      if (it == faceIds.end()) {
        fa = (int64_t)faceIds.size();
        faceIds.emplace(key, fa);
        m.faVe.insert(m.faVe.end(), key.begin(), key.end());
        m.faEl.push_back(e);
        m.faEl.push_back(-1);
      } else {
        fa = it->second;
        if (m.faEl[2 * fa + 1] != -1) return EDGE_B200_EMESH;
        m.faEl[2 * fa + 1] = e;
      }
      m.elFa[4 * e + f] = fa;
    }
  }
  const int64_t nFa = m.nFa();
  for (int64_t fa = 0; fa < nFa; fa++) {
    int64_t a = m.faEl[2 * fa], b = m.faEl[2 * fa + 1];
    if (b != -1 && b < a) std::swap(m.faEl[2 * fa], m.faEl[2 * fa + 1]);
  }
  m.faType.assign(nFa, EDGE_FACE_INNER);
  m.faPartner.assign(nFa, -1);
  return EDGE_B200_OK;
}

// neighbour and type per element face (from faEl and faType)
void buildNeighbours(edge_mesh &m) {
  const int64_t nEl = m.nEl();
  m.elFaEl.assign(4 * nEl, -1);
  m.elFaType.assign(4 * nEl, EDGE_FACE_INNER);
  for (int64_t e = 0; e < nEl; e++)
    for (int f = 0; f < 4; f++) {
      int64_t fa = m.elFa[4 * e + f];
      int64_t a = m.faEl[2 * fa], b = m.faEl[2 * fa + 1];
      m.elFaEl[4 * e + f] = (int32_t)(a == e ? b : a);
      m.elFaType[4 * e + f] = m.faType[fa];
    }
}

// neighbour face ids (geom/Generic.cpp:92-116) and vertex ids (geom/Tet4.cpp:114-229). perFo
// holds the neighbour's local face across a periodic face (-1 elsewhere); partnerVe maps this
// element's vertex to the neighbour's matching vertex across such a face.
template <typename PartnerVe>
int buildFaceIds(edge_mesh &m, const std::vector<int> &perFo, PartnerVe partnerVe) {
  const int64_t nEl = m.nEl();
  m.fIdElFaEl.assign(4 * nEl, 255);
  m.vIdElFaEl.assign(4 * nEl, 255);
  for (int64_t e = 0; e < nEl; e++)
    for (int f = 0; f < 4; f++) {
      int64_t ne = m.elFaEl[4 * e + f];
      if (ne < 0) continue;
      const bool per = !perFo.empty() && perFo[4 * e + f] >= 0;
      int fAd = -1;
      if (per) {
        fAd = perFo[4 * e + f];
      } else {
        for (int g = 0; g < 4; g++)
          if (m.elFaEl[4 * ne + g] == e && m.elFa[4 * ne + g] == m.elFa[4 * e + f]) {
            fAd = g;
            break;
          }
      }
      int64_t ve0 = f <= 2 ? m.elVe[4 * e + 0] : m.elVe[4 * e + 1];
      if (per) ve0 = partnerVe(e, f, ve0);
      int veAd = -1;
      for (int g = 0; g < 4; g++)
        if (m.elVe[4 * ne + g] == ve0) veAd = g;
      int vId = -1;
      if (fAd >= 0)
        for (int i = 0; i < 3; i++)
          if (kFaVe[fAd][i] == veAd) vId = i;
      if (fAd < 0 || vId < 0) return EDGE_B200_EMESH;
      m.fIdElFaEl[4 * e + f] = (uint8_t)fAd;
      m.vIdElFaEl[4 * e + f] = (uint8_t)vId;
    }
  return EDGE_B200_OK;
}

// face normals (away from the left element's vertex opposite the face), tangents and areas;
// element volumes and in-diameters 6V/S (geom/Tet4.cpp:30-78); the point-location grid
void buildGeometry(edge_mesh &m) {
  const int64_t nFa = m.nFa(), nEl = m.nEl();
  m.faNormal.resize(3 * nFa);
  m.faTangent.resize(6 * nFa);
  m.faArea.resize(nFa);
  for (int64_t fa = 0; fa < nFa; fa++) {
    double v[3][3];
    for (int i = 0; i < 3; i++)
      for (int d = 0; d < 3; d++) v[i][d] = m.ve[3 * m.faVe[3 * fa + i] + d];
    int64_t el = m.faEl[2 * fa];
    int64_t np = -1;
    for (int a = 0; a < 4; a++) {
      int64_t x = m.elVe[4 * el + a];
      if (x != m.faVe[3 * fa] && x != m.faVe[3 * fa + 1] && x != m.faVe[3 * fa + 2]) np = x;
    }
    triaFrame(v, &m.ve[3 * np], &m.faTangent[6 * fa], &m.faTangent[6 * fa + 3], &m.faNormal[3 * fa]);
    double d0[3], d1[3], c[3];
    for (int d = 0; d < 3; d++) {
      d0[d] = v[1][d] - v[0][d];
      d1[d] = v[2][d] - v[0][d];
    }
    cross(d0, d1, c);
    m.faArea[fa] = norm(c) / 2;
  }
  m.elVol.resize(nEl);
  m.elInDia.resize(nEl);
  for (int64_t e = 0; e < nEl; e++) {
    double j3[3][3];
    m.jac(e, j3);
    double vol = std::abs(det3(j3)) / 6;
    double s = 0;
    for (int f = 0; f < 4; f++) s += 2 * m.faArea[m.elFa[4 * e + f]];
    m.elVol[e] = vol;
    m.elInDia[e] = 12 * vol / s;
  }
  buildLocateGrid(m);
}

// Morton (Z-order) key of a point in the unit cube, 21 bits per axis
uint64_t mortonKey(const double x[3]) {
  uint64_t k = 0;
  uint32_t c[3];
  for (int d = 0; d < 3; d++) c[d] = (uint32_t)std::min(std::max(x[d], 0.0) * 2097151.0, 2097151.0);
  for (int b = 20; b >= 0; b--)
    for (int d = 0; d < 3; d++) k = (k << 1) | ((c[d] >> b) & 1u);
  return k;
}

// reference coordinates of a physical point (linalg/Mappings.hpp phyToRef)
void phyToRef(const edge_mesh &m, int64_t el, const double x[3], double xi[3]) {
  double j[3][3], ji[3][3], v[4][3];
  m.jac(el, j);
  inv3(j, ji);
  m.veCrds(el, v);
  double dx[3] = {x[0] - v[0][0], x[1] - v[0][1], x[2] - v[0][2]};
  // x = v0 + sum_a xi_a * jac[a]  ->  xi = dx * jac^-1
  for (int a = 0; a < 3; a++) xi[a] = dx[0] * ji[0][a] + dx[1] * ji[1][a] + dx[2] * ji[2][a];
}

}  // namespace

extern "C" {

int edge_mesh_box(int nx, int ny, int nz, const double ext[3], double jitter, uint64_t seed,
                  int bc_top, int bc_sides, edge_mesh **out) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || !ext || jitter < 0 || jitter >= 0.5) return EDGE_B200_EINVAL;
  const bool periodic = bc_top == EDGE_FACE_PERIODIC && bc_sides == EDGE_FACE_PERIODIC;
  if (!periodic && ((bc_top != EDGE_FACE_FREE_SURFACE && bc_top != EDGE_FACE_OUTFLOW) ||
                    (bc_sides != EDGE_FACE_FREE_SURFACE && bc_sides != EDGE_FACE_OUTFLOW)))
    return EDGE_B200_EINVAL;
  if (periodic && (nx < 2 || ny < 2 || nz < 2)) return EDGE_B200_EINVAL;
  edge_mesh *m = new (std::nothrow) edge_mesh();
  if (!m) return EDGE_B200_ENOMEM;
  const int64_t vx = nx + 1, vy = ny + 1, vz = nz + 1;
  const double h[3] = {ext[0] / nx, ext[1] / ny, ext[2] / nz};
  auto vid = [&](int64_t i, int64_t j, int64_t k) { return i + vx * (j + vy * k); };
  m->ve.resize(3 * vx * vy * vz);
  for (int64_t k = 0; k < vz; k++)
    for (int64_t j = 0; j < vy; j++)
      for (int64_t i = 0; i < vx; i++) {
        int64_t v = vid(i, j, k);
        m->ve[3 * v + 0] = i * h[0];
        m->ve[3 * v + 1] = j * h[1];
        m->ve[3 * v + 2] = k * h[2];
      }
  // 6 tets per cube along the main diagonal (0,0,0)-(1,1,1): one per axis permutation
  const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  const int64_t nEl = 6ll * nx * ny * nz;
  m->elVe.resize(4 * nEl);
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++)
      for (int64_t i = 0; i < nx; i++) {
        int64_t c = i + nx * (j + (int64_t)ny * k);
        for (int p = 0; p < 6; p++) {
          int64_t idx[3] = {i, j, k};
          int64_t *ev = &m->elVe[4 * (6 * c + p)];
          ev[0] = vid(idx[0], idx[1], idx[2]);
          for (int s = 0; s < 3; s++) {
            idx[perm[p][s]]++;
            ev[s + 1] = vid(idx[0], idx[1], idx[2]);
          }
        }
      }
  // jitter interior vertices; redraw the vertices of inverted tets
  if (jitter > 0) {
    Rng rng{seed};
    std::vector<double> base = m->ve;
    auto interior = [&](int64_t v) {
      int64_t i = v % vx, j = (v / vx) % vy, k = v / (vx * vy);
      return i > 0 && i < nx && j > 0 && j < ny && k > 0 && k < nz;
    };
    auto draw = [&](int64_t v) {
      for (int d = 0; d < 3; d++) m->ve[3 * v + d] = base[3 * v + d] + (2 * rng.uniform() - 1) * jitter * h[d];
    };
    // orientation of every tet before the jitter (the six tets of a cube alternate in sign; the
    // element normalisation orients them later): a jittered tet is inverted when its sign flips
    std::vector<int8_t> sign0(nEl);
    for (int64_t e = 0; e < nEl; e++) {
      double j3[3][3];
      m->jac(e, j3);
      sign0[e] = det3(j3) > 0 ? 1 : -1;
    }
    for (int64_t v = 0; v < vx * vy * vz; v++)
      if (interior(v)) draw(v);
    for (int it = 0; it < 64; it++) {
      std::vector<int64_t> bad;
      for (int64_t e = 0; e < nEl; e++) {
        double j3[3][3];
        m->jac(e, j3);
        const double sv = sign0[e] * det3(j3);
        if (sv <= 1e-3 * h[0] * h[1] * h[2])
          for (int a = 0; a < 4; a++)
            if (interior(m->elVe[4 * e + a])) bad.push_back(m->elVe[4 * e + a]);
      }
      if (bad.empty()) break;
      std::sort(bad.begin(), bad.end());
      bad.erase(std::unique(bad.begin(), bad.end()), bad.end());
      for (int64_t v : bad) {
        if (it < 48) draw(v);
        else for (int d = 0; d < 3; d++) m->ve[3 * v + d] = base[3 * v + d];
      }
    }
  }
  int rc;
  if ((rc = normalizeElements(*m)) || (rc = buildFaces(*m))) {
    delete m;
    return rc;
  }
  const int64_t nFa = m->nFa();
  // boundary types
  for (int64_t fa = 0; fa < nFa; fa++) {
    if (m->faEl[2 * fa + 1] != -1) continue;
    bool top = true;
    for (int i = 0; i < 3; i++) top = top && std::abs(m->ve[3 * m->faVe[3 * fa + i] + 2] - ext[2]) < 1e-9 * ext[2];
    m->faType[fa] = (uint8_t)(periodic ? EDGE_FACE_INNER : (top ? bc_top : bc_sides));
  }
  buildNeighbours(*m);
  // periodic boxes: pair each boundary face with its translate on the opposite side (grid
  // indices of boundary vertices are exact, jitter moves interior vertices only), as EDGE-V
  // pairs periodic faces by matching coordinates (mesh/Mesh.cpp:190-286)
  const int64_t nGrid[3] = {nx, ny, nz};
  auto gridIdx = [&](int64_t v, int64_t g[3]) {
    g[0] = v % vx;
    g[1] = (v / vx) % vy;
    g[2] = v / (vx * vy);
  };
  std::vector<int> perFo, perDir;
  if (periodic) {
    perFo.assign(4 * nEl, -1);
    perDir.assign(4 * nEl, -1);
    std::map<std::array<int64_t, 7>, std::pair<int64_t, int>> open;  // key -> (element, local face)
    for (int64_t e = 0; e < nEl; e++)
      for (int f = 0; f < 4; f++) {
        if (m->elFaEl[4 * e + f] != -1) continue;
        int64_t fa = m->elFa[4 * e + f];
        int64_t g[3][3];
        for (int i = 0; i < 3; i++) gridIdx(m->faVe[3 * fa + i], g[i]);
        int dir = -1;
        for (int d = 0; d < 3; d++)
          if (g[0][d] == g[1][d] && g[1][d] == g[2][d] && (g[0][d] == 0 || g[0][d] == nGrid[d])) dir = d;
        if (dir < 0) {
          delete m;
          return EDGE_B200_EMESH;
        }
        std::array<int64_t, 7> key{};
        key[0] = dir;
        std::array<std::pair<int64_t, int64_t>, 3> other;
        for (int i = 0; i < 3; i++) other[i] = {g[i][(dir + 1) % 3], g[i][(dir + 2) % 3]};
        std::sort(other.begin(), other.end());
        for (int i = 0; i < 3; i++) {
          key[1 + 2 * i] = other[i].first;
          key[2 + 2 * i] = other[i].second;
        }
        auto it = open.find(key);
        if (it == open.end()) {
          open.emplace(key, std::make_pair(e, f));
        } else {
          const int64_t e1 = it->second.first;
          const int f1 = it->second.second;
          perFo[4 * e + f] = f1;
          perDir[4 * e + f] = dir;
          perFo[4 * e1 + f1] = f;
          perDir[4 * e1 + f1] = dir;
          m->elFaEl[4 * e + f] = (int32_t)e1;
          m->elFaEl[4 * e1 + f1] = (int32_t)e;
          m->faPartner[m->elFa[4 * e + f]] = e1;
          m->faPartner[m->elFa[4 * e1 + f1]] = e;
          open.erase(it);
        }
      }
    if (!open.empty()) {
      delete m;
      return EDGE_B200_EMESH;
    }
  }
  // across a periodic face the matching vertex of the neighbour sits on the opposite side
  auto partnerVe = [&](int64_t e, int f, int64_t ve0) {
    const int d = perDir[4 * e + f];
    int64_t g[3];
    gridIdx(ve0, g);
    g[d] = g[d] == 0 ? nGrid[d] : 0;
    return vid(g[0], g[1], g[2]);
  };
  if ((rc = buildFaceIds(*m, perFo, partnerVe))) {
    delete m;
    return rc;
  }
  buildGeometry(*m);
  *out = m;
  return EDGE_B200_OK;
}

int edge_mesh_from_arrays(int64_t n_ve, const double *ve, int64_t n_el, const int64_t *el_ve, int64_t n_bf,
                          const int64_t *bf_ve, const int32_t *bf_tag, int default_type, int reorder,
                          int64_t *el_perm, edge_mesh **out) {
  if (!out || n_ve < 4 || !ve || n_el < 1 || !el_ve || n_bf < 0 || (n_bf && (!bf_ve || !bf_tag)))
    return EDGE_B200_EINVAL;
  if (n_el > std::numeric_limits<int32_t>::max()) return EDGE_B200_EINVAL;
  if (default_type != -1 && default_type != EDGE_FACE_FREE_SURFACE && default_type != EDGE_FACE_OUTFLOW)
    return EDGE_B200_EINVAL;
  for (int64_t i = 0; i < 4 * n_el; i++)
    if (el_ve[i] < 0 || el_ve[i] >= n_ve) return EDGE_B200_EINVAL;
  // boundary tags by sorted vertex triple: EDGE's physical groups 101 (free surface), 105 (outflow)
  std::map<std::array<int64_t, 3>, uint8_t> tagged;
  for (int64_t i = 0; i < n_bf; i++) {
    std::array<int64_t, 3> key = {bf_ve[3 * i], bf_ve[3 * i + 1], bf_ve[3 * i + 2]};
    for (int64_t k : key)
      if (k < 0 || k >= n_ve) return EDGE_B200_EINVAL;
    std::sort(key.begin(), key.end());
    uint8_t ty;
    if (bf_tag[i] == 101) ty = EDGE_FACE_FREE_SURFACE;
    else if (bf_tag[i] == 105) ty = EDGE_FACE_OUTFLOW;
    else return EDGE_B200_ENOTSUP;
    tagged[key] = ty;
  }
  edge_mesh *m = new (std::nothrow) edge_mesh();
  if (!m) return EDGE_B200_ENOMEM;
  m->ve.assign(ve, ve + 3 * n_ve);
  std::vector<int64_t> perm(n_el);
  for (int64_t e = 0; e < n_el; e++) perm[e] = e;
  if (reorder) {
    // elements along a Z-order curve of their centroids, for neighbour locality in the device
    // gathers (EDGE-V reorders elements for its partitions and time groups instead)
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t v = 0; v < n_ve; v++)
      for (int d = 0; d < 3; d++) {
        lo[d] = std::min(lo[d], ve[3 * v + d]);
        hi[d] = std::max(hi[d], ve[3 * v + d]);
      }
    double span = 0;
    for (int d = 0; d < 3; d++) span = std::max(span, hi[d] - lo[d]);
    std::vector<uint64_t> key(n_el);
    for (int64_t e = 0; e < n_el; e++) {
      double c[3] = {0, 0, 0};
      for (int a = 0; a < 4; a++)
        for (int d = 0; d < 3; d++) c[d] += ve[3 * el_ve[4 * e + a] + d] / 4;
      for (int d = 0; d < 3; d++) c[d] = (c[d] - lo[d]) / (span > 0 ? span : 1.0);
      key[e] = mortonKey(c);
    }
    std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
  }
  m->elVe.resize(4 * n_el);
  for (int64_t e = 0; e < n_el; e++)
    for (int a = 0; a < 4; a++) m->elVe[4 * e + a] = el_ve[4 * perm[e] + a];
  int rc;
  if ((rc = normalizeElements(*m)) || (rc = buildFaces(*m))) {
    delete m;
    return rc;
  }
  const int64_t nFa = m->nFa();
  for (int64_t fa = 0; fa < nFa; fa++) {
    if (m->faEl[2 * fa + 1] != -1) continue;
    std::array<int64_t, 3> key = {m->faVe[3 * fa], m->faVe[3 * fa + 1], m->faVe[3 * fa + 2]};
    auto it = tagged.find(key);
    if (it != tagged.end()) {
      m->faType[fa] = it->second;
    } else if (default_type >= 0) {
      m->faType[fa] = (uint8_t)default_type;
    } else {
      delete m;
      return EDGE_B200_EMESH;
    }
  }
  buildNeighbours(*m);
  if ((rc = buildFaceIds(*m, std::vector<int>(), [](int64_t, int, int64_t v) { return v; }))) {
    delete m;
    return rc;
  }
  buildGeometry(*m);
  if (el_perm) std::copy(perm.begin(), perm.end(), el_perm);
  *out = m;
  return EDGE_B200_OK;
}

int edge_mesh_sizes(const edge_mesh *m, int64_t *n_ve, int64_t *n_fa, int64_t *n_el) {
  if (!m) return EDGE_B200_EINVAL;
  if (n_ve) *n_ve = m->nVe();
  if (n_fa) *n_fa = m->nFa();
  if (n_el) *n_el = m->nEl();
  return EDGE_B200_OK;
}

int edge_mesh_arrays(const edge_mesh *m, double *ve, int64_t *el_ve, int64_t *el_fa,
                     int64_t *fa_el, double *fa_normal, double *fa_tangent, double *fa_area,
                     uint8_t *fa_type, double *el_vol, double *el_india, int32_t *el_fa_el,
                     uint8_t *fid_el_fa_el, uint8_t *vid_el_fa_el, uint8_t *el_fa_type) {
  if (!m) return EDGE_B200_EINVAL;
  auto cp = [](auto *dst, const auto &src) {
    if (dst) std::copy(src.begin(), src.end(), dst);
  };
  cp(ve, m->ve);
  cp(el_ve, m->elVe);
  cp(el_fa, m->elFa);
  cp(fa_el, m->faEl);
  cp(fa_normal, m->faNormal);
  cp(fa_tangent, m->faTangent);
  cp(fa_area, m->faArea);
  cp(fa_type, m->faType);
  cp(el_vol, m->elVol);
  cp(el_india, m->elInDia);
  cp(el_fa_el, m->elFaEl);
  cp(fid_el_fa_el, m->fIdElFaEl);
  cp(vid_el_fa_el, m->vIdElFaEl);
  cp(el_fa_type, m->elFaType);
  return EDGE_B200_OK;
}

void edge_mesh_free(edge_mesh *m) { delete m; }

// -------------------------------------------------------------------------------------------------
// physics setup
// -------------------------------------------------------------------------------------------------

// dense 9x9 elastic star matrix of one reference direction, row-major
static void starDense(double rho, double lam, double mu, const double ji[3][3], int di, double o[81]) {
  std::fill(o, o + 81, 0.0);
  // Jacobians A_1, A_2, A_3 of q_t + A_j q_{x_j} = 0, stresses xx,yy,zz,xy,yz,xz, velocities u,v,w
  const double lp = -lam - 2 * mu, l = -lam, m = -mu, r = -1 / rho;
  const double a = ji[0][di], b = ji[1][di], c = ji[2][di];
  o[0 * 9 + 6] += lp * a; o[1 * 9 + 6] += l * a; o[2 * 9 + 6] += l * a;
  o[3 * 9 + 7] += m * a;  o[5 * 9 + 8] += m * a;
  o[6 * 9 + 0] += r * a;  o[7 * 9 + 3] += r * a; o[8 * 9 + 5] += r * a;
  o[0 * 9 + 7] += l * b;  o[1 * 9 + 7] += lp * b; o[2 * 9 + 7] += l * b;
  o[3 * 9 + 6] += m * b;  o[4 * 9 + 8] += m * b;
  o[6 * 9 + 3] += r * b;  o[7 * 9 + 1] += r * b; o[8 * 9 + 4] += r * b;
  o[0 * 9 + 8] += l * c;  o[1 * 9 + 8] += l * c; o[2 * 9 + 8] += lp * c;
  o[4 * 9 + 7] += m * c;  o[5 * 9 + 6] += m * c;
  o[6 * 9 + 5] += r * c;  o[7 * 9 + 4] += r * c; o[8 * 9 + 2] += r * c;
}

static const int kSE_R[24] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 6, 7, 7, 7, 8, 8, 8};
static const int kSE_C[24] = {6, 7, 8, 6, 7, 8, 6, 7, 8, 6, 7, 7, 8, 6, 8, 0, 3, 5, 1, 3, 4, 2, 4, 5};
static const int kSA_R[9] = {0, 1, 2, 3, 3, 4, 4, 5, 5};
static const int kSA_C[9] = {0, 1, 2, 0, 1, 1, 2, 0, 2};

int edge_setup_star(const edge_mesh *m, const double *rho, const double *lam, const double *mu,
                    double *star_e) {
  if (!m || !rho || !lam || !mu || !star_e) return EDGE_B200_EINVAL;
  const int64_t nEl = m->nEl();
  for (int64_t e = 0; e < nEl; e++) {
    double j[3][3], ji[3][3], d[81];
    m->jac(e, j);
    inv3(j, ji);
    for (int di = 0; di < 3; di++) {
      starDense(rho[e], lam[e], mu[e], ji, di, d);
      for (int i = 0; i < 24; i++) star_e[(e * 3 + di) * 24 + i] = d[kSE_R[i] * 9 + kSE_C[i]];
    }
  }
  return EDGE_B200_OK;
}

int edge_setup_star_anelastic(const edge_mesh *m, double *star_a) {
  if (!m || !star_a) return EDGE_B200_EINVAL;
  const int64_t nEl = m->nEl();
  for (int64_t e = 0; e < nEl; e++) {
    double j[3][3], ji[3][3];
    m->jac(e, j);
    inv3(j, ji);
    for (int di = 0; di < 3; di++) {
      // anelastic Jacobians: the strain rates the mechanisms relax (6 x 3 acting on u, v, w)
      double o[18] = {0};
      const double a = ji[0][di], b = ji[1][di], c = ji[2][di];
      o[0 * 3 + 0] += -1.0 * a; o[3 * 3 + 1] += -0.5 * a; o[5 * 3 + 2] += -0.5 * a;
      o[1 * 3 + 1] += -1.0 * b; o[3 * 3 + 0] += -0.5 * b; o[4 * 3 + 2] += -0.5 * b;
      o[2 * 3 + 2] += -1.0 * c; o[4 * 3 + 1] += -0.5 * c; o[5 * 3 + 0] += -0.5 * c;
      for (int i = 0; i < 9; i++) star_a[(e * 3 + di) * 9 + i] = o[kSA_R[i] * 3 + kSA_C[i]];
    }
  }
  return EDGE_B200_OK;
}

// Quantity transform from the face-aligned frame (x' = n, y' = s, z' = t) to xyz: the stress
// tensor rotates as R S' R^T, the velocity as R u' with R = [n s t]; T_inv uses R^T.
static void trafo(const double n[3], const double s[3], const double t[3], bool inverse, double T[81]) {
  double R[3][3];
  for (int i = 0; i < 3; i++) {
    const double col[3] = {n[i], s[i], t[i]};
    for (int k = 0; k < 3; k++) R[i][k] = inverse ? 0 : col[k];
  }
  if (inverse)
    for (int i = 0; i < 3; i++) {
      R[0][i] = n[i];
      R[1][i] = s[i];
      R[2][i] = t[i];
    }
  // Voigt pairs of xx, yy, zz, xy, yz, xz
  const int vi[6] = {0, 1, 2, 0, 1, 0}, vj[6] = {0, 1, 2, 1, 2, 2};
  std::fill(T, T + 81, 0.0);
  for (int I = 0; I < 6; I++)
    for (int J = 0; J < 6; J++) {
      int i = vi[I], j = vj[I], k = vi[J], l = vj[J];
      T[I * 9 + J] = (k == l) ? R[i][k] * R[j][k] : R[i][k] * R[j][l] + R[i][l] * R[j][k];
    }
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) T[(6 + i) * 9 + 6 + k] = R[i][k];
}

// Godunov middle-state flux of the face-aligned 1D Riemann problem: F = A_L q*, with q* the
// interface state of left state qL and right state qR. Returns dF/dqL and dF/dqR (9x9), and the
// anelastic counterparts (6x9) that use the anelastic Jacobian's normal part instead of A_L.
// Impedances Zp = rho cp, Zs = rho cs; with D = ZL + ZR:
//   u*  = (ZL uL + ZR uR + sR - sL) / D,   s* = (ZR sL + ZL sR + ZL ZR (uR - uL)) / D
// for the pairs (sxx, u) with P impedances and (sxy, v), (sxz, w) with S impedances.
static void middleStates(double rhoL, double rhoR, double lamL, double lamR, double muL, double muR,
                         double FL[81], double FR[81], double AL[54], double AR[54]) {
  const double cpL = std::sqrt((lamL + 2 * muL) / rhoL), cpR = std::sqrt((lamR + 2 * muR) / rhoR);
  const double csL = std::sqrt(muL / rhoL), csR = std::sqrt(muR / rhoR);
  const double zpL = rhoL * cpL, zpR = rhoR * cpR, zsL = rhoL * csL, zsR = rhoR * csR;
  // d(u*, s*)/d(sL, uL, sR, uR) for one characteristic pair
  struct Pair { double du[4], ds[4]; };
  auto pair = [](double zL, double zR) {
    Pair p;
    const double D = zL + zR;
    p.du[0] = -1 / D; p.du[1] = zL / D; p.du[2] = 1 / D; p.du[3] = zR / D;
    p.ds[0] = zR / D; p.ds[1] = -zL * zR / D; p.ds[2] = zL / D; p.ds[3] = zL * zR / D;
    return p;
  };
  Pair P = pair(zpL, zpR), S = pair(zsL, zsR);
  // q* rows needed: sxx*(0), sxy*(3), sxz*(5), u*(6), v*(7), w*(8); columns: quantities of qL / qR
  double dqL[9][9] = {{0}}, dqR[9][9] = {{0}};
  const int sIdx[3] = {0, 3, 5}, uIdx[3] = {6, 7, 8};
  for (int c = 0; c < 3; c++) {
    const Pair &p = c == 0 ? P : S;
    int si = sIdx[c], ui = uIdx[c];
    dqL[si][si] = p.ds[0]; dqL[si][ui] = p.ds[1]; dqR[si][si] = p.ds[2]; dqR[si][ui] = p.ds[3];
    dqL[ui][si] = p.du[0]; dqL[ui][ui] = p.du[1]; dqR[ui][si] = p.du[2]; dqR[ui][ui] = p.du[3];
  }
  // normal Jacobian of the left material in the face-aligned frame
  double A[81] = {0};
  A[0 * 9 + 6] = -lamL - 2 * muL; A[1 * 9 + 6] = -lamL; A[2 * 9 + 6] = -lamL;
  A[3 * 9 + 7] = -muL; A[5 * 9 + 8] = -muL;
  A[6 * 9 + 0] = -1 / rhoL; A[7 * 9 + 3] = -1 / rhoL; A[8 * 9 + 5] = -1 / rhoL;
  matmul(9, 9, 9, A, &dqL[0][0], FL);
  matmul(9, 9, 9, A, &dqR[0][0], FR);
  double Aa[54] = {0};
  Aa[0 * 9 + 6] = -1.0; Aa[3 * 9 + 7] = -0.5; Aa[5 * 9 + 8] = -0.5;
  matmul(6, 9, 9, Aa, &dqL[0][0], AL);
  matmul(6, 9, 9, Aa, &dqR[0][0], AR);
}

int edge_setup_trafo(const double n[3], const double s[3], const double t[3], double *t_mat,
                     double *t_inv) {
  if (!n || !s || !t) return EDGE_B200_EINVAL;
  if (t_mat) trafo(n, s, t, false, t_mat);
  if (t_inv) trafo(n, s, t, true, t_inv);
  return EDGE_B200_OK;
}

int edge_setup_fs_pair(double rho_l, double rho_r, double lam_l, double lam_r, double mu_l,
                       double mu_r, const double n[3], const double s[3], const double t[3],
                       int free_surface, double *fs_el, double *fs_er, double *fs_al,
                       double *fs_ar) {
  if (!n || !s || !t || !fs_el || !fs_er) return EDGE_B200_EINVAL;
  if (!(mu_l > 0 && mu_r > 0 && rho_l > 0 && rho_r > 0)) return EDGE_B200_EINVAL;
  double T[81], Ti[81], FL[81], FR[81], AL[54], AR[54], tmp[81];
  trafo(n, s, t, false, T);
  trafo(n, s, t, true, Ti);
  middleStates(rho_l, rho_r, lam_l, lam_r, mu_l, mu_r, FL, FR, AL, AR);
  if (free_surface) {
    // mirror the right state: traction-free face (Elasticity.cpp:421-433)
    for (int r = 0; r < 9; r++) {
      FR[r * 9 + 0] *= -1; FR[r * 9 + 3] *= -1; FR[r * 9 + 5] *= -1;
    }
    for (int r = 0; r < 6; r++) {
      AR[r * 9 + 0] *= -1; AR[r * 9 + 3] *= -1; AR[r * 9 + 5] *= -1;
    }
  }
  matmul(9, 9, 9, T, FL, tmp);
  matmul(9, 9, 9, tmp, Ti, fs_el);
  matmul(9, 9, 9, T, FR, tmp);
  matmul(9, 9, 9, tmp, Ti, fs_er);
  if (fs_al && fs_ar) {
    double TA[36];
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) TA[i * 6 + j] = T[i * 9 + j];
    matmul(6, 9, 6, TA, AL, tmp);
    matmul(6, 9, 9, tmp, Ti, fs_al);
    matmul(6, 9, 6, TA, AR, tmp);
    matmul(6, 9, 9, tmp, Ti, fs_ar);
  }
  return EDGE_B200_OK;
}

int edge_setup_flux_solvers(const edge_mesh *m, int n_rms, const double *rho, const double *lam,
                            const double *mu, double *fs_e, double *fs_a) {
  if (!m || !rho || !lam || !mu || !fs_e || (n_rms > 0 && !fs_a)) return EDGE_B200_EINVAL;
  const int64_t nEl = m->nEl(), nFa = m->nFa();
  double *fsE[2] = {fs_e, fs_e + nEl * 4 * 81};
  double *fsA[2] = {n_rms ? fs_a : nullptr, n_rms ? fs_a + nEl * 4 * 54 : nullptr};
  for (int64_t fa = 0; fa < nFa; fa++) {
    int64_t elL = m->faEl[2 * fa], elR = m->faEl[2 * fa + 1];
    int fIdL = -1, fIdR = -1;
    for (int f = 0; f < 4; f++) {
      if (m->elFa[4 * elL + f] == fa) fIdL = f;
      if (elR >= 0 && m->elFa[4 * elR + f] == fa) fIdR = f;
    }
    if (fIdL < 0 || (elR >= 0 && fIdR < 0)) return EDGE_B200_EMESH;
    const int ty = m->faType[fa];
    // boundaries: right material = left (AderDgInit.hpp:490-493); periodic faces: the partner's
    const int64_t mR = elR >= 0 ? elR : (m->faPartner[fa] >= 0 ? m->faPartner[fa] : elL);
    const double *n = &m->faNormal[3 * fa], *s = &m->faTangent[6 * fa], *t = &m->faTangent[6 * fa + 3];
    double el[81], er[81], al[54], ar[54];
    int rc = edge_setup_fs_pair(rho[elL], rho[mR], lam[elL], lam[mR], mu[elL], mu[mR], n, s, t,
                                ty == EDGE_FACE_FREE_SURFACE, el, er, al, ar);
    if (rc) return rc;
    // scaling -2 * area / detJ (AderDgInit.hpp:621-646)
    double j3[3][3];
    m->jac(elL, j3);
    double dL = det3(j3);
    if (!(dL > 0)) return EDGE_B200_EMESH;
    double sc = -m->faArea[fa] / dL * 2;
    for (int i = 0; i < 81; i++) {
      fsE[0][(elL * 4 + fIdL) * 81 + i] = el[i] * sc;
      fsE[1][(elL * 4 + fIdL) * 81 + i] = er[i] * sc;
    }
    if (n_rms)
      for (int i = 0; i < 54; i++) {
        fsA[0][(elL * 4 + fIdL) * 54 + i] = al[i] * sc;
        fsA[1][(elL * 4 + fIdL) * 54 + i] = ar[i] * sc;
      }
    if (elR >= 0) {
      const double nm[3] = {-n[0], -n[1], -n[2]};
      rc = edge_setup_fs_pair(rho[elR], rho[elL], lam[elR], lam[elL], mu[elR], mu[elL], nm, s, t, 0,
                              el, er, al, ar);
      if (rc) return rc;
      m->jac(elR, j3);
      double dR = det3(j3);
      if (!(dR > 0)) return EDGE_B200_EMESH;
      double scR = -m->faArea[fa] / dR * 2;
      for (int i = 0; i < 81; i++) {
        fsE[0][(elR * 4 + fIdR) * 81 + i] = el[i] * scR;
        fsE[1][(elR * 4 + fIdR) * 81 + i] = er[i] * scR;
      }
      if (n_rms)
        for (int i = 0; i < 54; i++) {
          fsA[0][(elR * 4 + fIdR) * 54 + i] = al[i] * scR;
          fsA[1][(elR * 4 + fIdR) * 54 + i] = ar[i] * scR;
        }
    }
  }
  return EDGE_B200_OK;
}

int edge_setup_frequencies(int n_rms, double freq_cen, double freq_rat, double *freqs) {
  if (n_rms < 1 || !freqs || !(freq_cen > 0) || !(freq_rat > 0)) return EDGE_B200_EINVAL;
  freqs[0] = 2 * M_PI * freq_cen;
  freqs[0] /= std::sqrt(freq_rat);
  for (int f = 1; f < 2 * n_rms - 1; f++) {
    freqs[f] = std::log(freqs[0]);
    freqs[f] += (f * std::log(freq_rat)) / (2 * (n_rms - 1));
    freqs[f] = std::exp(freqs[f]);
  }
  return EDGE_B200_OK;
}

// Least squares min ||A x - b|| by Householder QR in long double; A is (2n-1) x n, full column rank.
int edge_setup_anelastic_coeffs(int n_rms, double quality, const double *freqs, double *coeffs) {
  if (n_rms < 1 || !freqs || !coeffs || !(quality > 0)) return EDGE_B200_EINVAL;
  const int nF = 2 * n_rms - 1, n = n_rms;
  std::vector<long double> A(nF * n), b(nF);
  const long double qInv = 1.0L / quality;
  for (int f = 0; f < nF; f++) {
    for (int me = 0; me < n; me++) {
      long double mf = freqs[2 * me];
      A[f * n + me] = (mf * freqs[f] + mf * mf * qInv) / ((long double)freqs[f] * freqs[f] + mf * mf);
    }
    b[f] = qInv;
  }
  for (int k = 0; k < n; k++) {
    long double nrm = 0;
    for (int i = k; i < nF; i++) nrm += A[i * n + k] * A[i * n + k];
    nrm = std::sqrt(nrm);
    if (nrm == 0) return EDGE_B200_EINVAL;
    long double alpha = A[k * n + k] > 0 ? -nrm : nrm;
    std::vector<long double> v(nF, 0);
    for (int i = k; i < nF; i++) v[i] = A[i * n + k];
    v[k] -= alpha;
    long double vv = 0;
    for (int i = k; i < nF; i++) vv += v[i] * v[i];
    if (vv == 0) continue;
    for (int j = k; j < n; j++) {
      long double s = 0;
      for (int i = k; i < nF; i++) s += v[i] * A[i * n + j];
      s = 2 * s / vv;
      for (int i = k; i < nF; i++) A[i * n + j] -= s * v[i];
    }
    long double s = 0;
    for (int i = k; i < nF; i++) s += v[i] * b[i];
    s = 2 * s / vv;
    for (int i = k; i < nF; i++) b[i] -= s * v[i];
  }
  for (int k = n - 1; k >= 0; k--) {
    long double s = b[k];
    for (int j = k + 1; j < n; j++) s -= A[k * n + j] * coeffs[j];
    coeffs[k] = (double)(s / A[k * n + k]);
  }
  return EDGE_B200_OK;
}

int edge_setup_elastic_lame(int n_rms, double freq_ref, const double *freqs,
                            const double *coeffs_kappa, const double *coeffs_mu, double lam_phase,
                            double mu_phase, double *lam_el, double *mu_el) {
  if (n_rms < 1 || !freqs || !coeffs_kappa || !coeffs_mu || !lam_el || !mu_el) return EDGE_B200_EINVAL;
  double th1[2] = {1, 1}, th2[2] = {0, 0};
  for (int me = 0; me < n_rms; me++) {
    double fr = freq_ref / freqs[me * 2];
    double sc = 1.0 / (1 + fr * fr);
    th1[0] -= coeffs_kappa[me] * sc;
    th1[1] -= coeffs_mu[me] * sc;
    th2[0] += coeffs_kappa[me] * fr * sc;
    th2[1] += coeffs_mu[me] * fr * sc;
  }
  double r[2];
  for (int i = 0; i < 2; i++) r[i] = std::sqrt(th1[i] * th1[i] + th2[i] * th2[i]);
  *mu_el = mu_phase * (r[1] + th1[1]) / (2 * r[1] * r[1]);
  double kappa = (lam_phase + 2 * mu_phase) * (r[0] + th1[0]) / (2 * r[0] * r[0]);
  *lam_el = kappa - 2 * *mu_el;
  return EDGE_B200_OK;
}

int edge_setup_attenuation(int n_rms, double freq_cen, double freq_rat, int64_t n_el,
                           const double *qp, const double *qs, double *lam, double *mu,
                           double *src_a, double *omega) {
  if (n_rms < 1 || !qp || !qs || !lam || !mu || !src_a || !omega) return EDGE_B200_EINVAL;
  std::vector<double> freqs(2 * n_rms - 1), co(2 * n_rms);
  int rc = edge_setup_frequencies(n_rms, freq_cen, freq_rat, freqs.data());
  if (rc) return rc;
  for (int me = 0; me < n_rms; me++) omega[me] = freqs[2 * me];
  const double fRef = 2 * M_PI * freq_cen;
  for (int64_t e = 0; e < n_el; e++) {
    // anelasticCoeffLame (ViscoElasticity.cpp:130-176)
    if ((rc = edge_setup_anelastic_coeffs(n_rms, qp[e], freqs.data(), co.data()))) return rc;
    if ((rc = edge_setup_anelastic_coeffs(n_rms, qs[e], freqs.data(), co.data() + n_rms))) return rc;
    double lamE, muE;
    edge_setup_elastic_lame(n_rms, fRef, freqs.data(), co.data(), co.data() + n_rms, lam[e], mu[e],
                            &lamE, &muE);
    for (int me = 0; me < n_rms; me++) {
      double sc = 2.0 * muE / lamE;
      co[me] = (1.0 + sc) * co[me];
      co[me] -= sc * co[n_rms + me];
    }
    // source matrices (ViscoElasticity.h:379-508), 12 row-major non-zeros
    for (int me = 0; me < n_rms; me++) {
      double nz0 = -lamE * co[me];
      nz0 -= 2 * muE * co[n_rms + me];
      double nz1 = -2 * muE * co[n_rms + me];
      double nz2 = -lamE * co[me];
      double *o = &src_a[(e * n_rms + me) * 12];
      o[0] = nz0; o[1] = nz2; o[2] = nz2;
      o[3] = nz2; o[4] = nz0; o[5] = nz2;
      o[6] = nz2; o[7] = nz2; o[8] = nz0;
      o[9] = nz1; o[10] = nz1; o[11] = nz1;
    }
    lam[e] = lamE;
    mu[e] = muE;
  }
  return EDGE_B200_OK;
}

int edge_setup_dt_cfl(const edge_mesh *m, int order, const double *rho, const double *lam,
                      const double *mu, double *dt_min) {
  if (!m || order < 1 || !rho || !lam || !mu || !dt_min) return EDGE_B200_EINVAL;
  double best = std::numeric_limits<double>::max();
  for (int64_t e = 0; e < m->nEl(); e++) {
    double cp = std::sqrt((lam[e] + 2.0 * mu[e]) / rho[e]);
    double dt = m->elInDia[e];
    dt *= 0.5;  // SCALE_CFL (src/impl/seismic/const.inc:135-137)
    dt /= cp;
    dt /= 2.0 * order - 1;
    best = std::min(best, dt);
  }
  *dt_min = best;
  return EDGE_B200_OK;
}

int edge_setup_dt_cfl_el(const edge_mesh *m, int order, const double *rho, const double *lam,
                         const double *mu, double *dt_el) {
  if (!m || order < 1 || !rho || !lam || !mu || !dt_el) return EDGE_B200_EINVAL;
  for (int64_t e = 0; e < m->nEl(); e++) {
    double cp = std::sqrt((lam[e] + 2.0 * mu[e]) / rho[e]);
    double dt = m->elInDia[e];
    dt *= 0.5;  // SCALE_CFL (src/impl/seismic/const.inc:135-137)
    dt /= cp;
    dt /= 2.0 * order - 1;
    dt_el[e] = dt;
  }
  return EDGE_B200_OK;
}

int edge_setup_time_groups(const edge_mesh *m, const double *dt_el, int n_groups, double fun_dt, uint8_t *el_tg,
                           int64_t *n_norm) {
  if (!m || !dt_el || !el_tg || n_groups < 1 || n_groups > 16 || !(fun_dt > 0) || fun_dt > 1)
    return EDGE_B200_EINVAL;
  const int64_t nEl = m->nEl();
  double dtMin = std::numeric_limits<double>::max();
  for (int64_t e = 0; e < nEl; e++) {
    if (!(dt_el[e] > 0)) return EDGE_B200_EINVAL;
    dtMin = std::min(dtMin, dt_el[e]);
  }
  // group boundaries fun_dt * 2^g of the relative steps (Groups::setElTg, time/Groups.cpp:84-100)
  for (int64_t e = 0; e < nEl; e++) {
    const double ts = dt_el[e] / dtMin;
    int g = n_groups - 1;
    double upper = fun_dt * 2;
    for (int k = 0; k < n_groups - 1; k++, upper *= 2)
      if (ts < upper) {
        g = k;
        break;
      }
    el_tg[e] = (uint8_t)g;
  }
  // face neighbours differ by at most one group (Groups::normalizeElTgs, time/Groups.cpp:47-82)
  int64_t changes = 0;
  for (;;) {
    int64_t it = 0;
    for (int64_t e = 0; e < nEl; e++)
      for (int f = 0; f < 4; f++) {
        const int64_t ad = m->elFaEl[4 * e + f];
        if (ad < 0) continue;
        if (el_tg[e] > el_tg[ad] + 1) {
          el_tg[e] = (uint8_t)(el_tg[ad] + 1);
          it++;
        }
      }
    changes += it;
    if (it == 0) break;
  }
  if (n_norm) *n_norm = changes;
  return EDGE_B200_OK;
}

int edge_setup_eval_basis(int order, const double ref[3], double *vals) {
  edge_dg_tables t;
  if (!ref || !vals || edge_dg_get(order, &t)) return EDGE_B200_EINVAL;
  const int B = order * (order + 1) * (order + 2) / 6;
  for (int b = 0; b < B; b++) {
    double s = 0;
    for (int i = t.basisOff[b]; i < t.basisOff[b + 1]; i++) {
      const unsigned char *e = &t.basisExp[3 * i];
      s += t.basisCoef[i] * std::pow(ref[0], e[0]) * std::pow(ref[1], e[1]) * std::pow(ref[2], e[2]);
    }
    vals[b] = s;
  }
  return EDGE_B200_OK;
}

int edge_setup_locate(const edge_mesh *m, int order, int n, const double *xyz, int64_t *el,
                      double *ref, double *basis, int scale_mass_jac) {
  edge_dg_tables t;
  if (!m || !xyz || n < 0 || edge_dg_get(order, &t)) return EDGE_B200_EINVAL;
  const int B = order * (order + 1) * (order + 2) / 6;
  for (int p = 0; p < n; p++) {
    const double *x = &xyz[3 * p];
    int c[3];
    for (int d = 0; d < 3; d++) {
      double f = (x[d] - m->lo[d]) / (m->hi[d] - m->lo[d] + 1e-300) * m->ng[d];
      c[d] = std::max(0, std::min(m->ng[d] - 1, (int)std::floor(f)));
    }
    int64_t cell = ((int64_t)c[2] * m->ng[1] + c[1]) * m->ng[0] + c[0];
    int64_t found = -1;
    double best = -std::numeric_limits<double>::max(), bestXi[3] = {0, 0, 0};
    // the element whose smallest barycentric coordinate is largest (exactly one contains x,
    // ties on shared faces go to the lowest id)
    for (int64_t i = m->cellOff[cell]; i < m->cellOff[cell + 1]; i++) {
      int64_t e = m->cellEl[i];
      double xi[3];
      phyToRef(*m, e, x, xi);
      double bmin = std::min(std::min(xi[0], xi[1]), std::min(xi[2], 1 - xi[0] - xi[1] - xi[2]));
      if (bmin > best + 1e-14 || (std::abs(bmin - best) <= 1e-14 && e < found)) {
        best = bmin;
        found = e;
        std::copy(xi, xi + 3, bestXi);
      }
    }
    if (found < 0 || best < -kTolMesh) return EDGE_B200_ENOTFOUND;
    if (el) el[p] = found;
    if (ref) std::copy(bestXi, bestXi + 3, &ref[3 * p]);
    if (basis) {
      double *bv = &basis[(int64_t)p * B];
      edge_setup_eval_basis(order, bestXi, bv);
      if (scale_mass_jac) {
        double j3[3][3];
        m->jac(found, j3);
        double jdi = 1.0 / det3(j3);
        for (int b = 0; b < B; b++) bv[b] *= t.massInv[b];
        for (int b = 0; b < B; b++) bv[b] *= jdi;
      }
    }
  }
  return EDGE_B200_OK;
}

}  // extern "C"
