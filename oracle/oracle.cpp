// TEST INFRASTRUCTURE ONLY (see oracle.h): FP64 CPU restatement of the reference's solver. Each
// function cites the reference file:line it restates; the reference is TypeScript, so this is a
// restatement in C++ of its arithmetic, kept in the reference's operation order where that order
// decides a branch.

#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

constexpr double INF = std::numeric_limits<double>::infinity();

double hyp3(double a, double b, double c) { return std::sqrt(a * a + b * b + c * c); }
double sq3(double a, double b, double c) { return a * a + b * b + c * c; }

// ---------------------------------------------------------------------------- axial.ts

struct Yarn {
  double eaLow, eaHigh, crimpStrain, eaCompress, axialViscosity, bendRigidity, bendViscosity;
  double softening;
  int yarnsPerSpan;  // 1 when the reference leaves it undefined
};

// axialTension (axial.ts:16-22).
double axialTension(const Yarn& p, double eps) {
  if (eps <= 0) return p.eaCompress * eps;
  double ec = p.crimpStrain, dk = p.eaHigh - p.eaLow;
  if (eps <= ec) return p.eaLow * eps + (dk * eps * eps) / (2 * ec);
  return p.eaLow * ec + (dk * ec) / 2 + p.eaHigh * (eps - ec);
}
// axialStiffness (axial.ts:25-30).
double axialStiffness(const Yarn& p, double eps) {
  if (eps <= 0) return p.eaCompress;
  double ec = p.crimpStrain;
  if (eps <= ec) return p.eaLow + ((p.eaHigh - p.eaLow) * eps) / ec;
  return p.eaHigh;
}
// axialEnergyDensity (axial.ts:33-42).
double axialEnergyDensity(const Yarn& p, double eps) {
  if (eps <= 0) return 0.5 * p.eaCompress * eps * eps;
  double ec = p.crimpStrain, dk = p.eaHigh - p.eaLow;
  if (eps <= ec) return 0.5 * p.eaLow * eps * eps + (dk * eps * eps * eps) / (6 * ec);
  double tc = p.eaLow * ec + (dk * ec) / 2;
  double ecEnergy = 0.5 * p.eaLow * ec * ec + (dk * ec * ec) / 6;
  double d = eps - ec;
  return ecEnergy + tc * d + 0.5 * p.eaHigh * d * d;
}
// strainAtTension (axial.ts:45-53).
double strainAtTension(const Yarn& p, double t) {
  double ec = p.crimpStrain, dk = p.eaHigh - p.eaLow;
  double tc = p.eaLow * ec + (dk * ec) / 2;
  if (t >= tc) return ec + (t - tc) / p.eaHigh;
  double a = dk / (2 * ec);
  return (2 * t) / (p.eaLow + std::sqrt(p.eaLow * p.eaLow + 4 * a * t));
}
// yarnDamage (axial.ts:63-70).
double yarnDamage(const Yarn& p, double yarns, double area, double peakYarn, double softStrain, double eps) {
  double ep = strainAtTension(p, (peakYarn * yarns) / area);
  if (eps <= ep) return 0;
  if (eps >= ep + softStrain) return 1;
  double tEnv = peakYarn * (1 - (eps - ep) / softStrain);
  double tEl = (area * axialTension(p, eps)) / yarns;
  return std::min(1.0, std::max(0.0, 1 - tEnv / std::max(tEl, 1e-12)));
}

// ---------------------------------------------------------------------------- laws.ts

constexpr double BEND_S0 = 0.85;
// bendPsi (laws.ts:17-30): [Psi, Psi', Psi''].
void bendPsi(double q, double a, double* out) {
  double s = q / a;
  if (s < BEND_S0) {
    double d = 1 - s;
    out[0] = q / d;
    out[1] = 1 / (d * d);
    out[2] = 2 / (a * d * d * d);
    return;
  }
  double d0 = 1 - BEND_S0, q0 = BEND_S0 * a;
  double p1 = 1 / (d0 * d0), p2 = 2 / (a * d0 * d0 * d0);
  double t = q - q0;
  out[0] = q0 / d0 + p1 * t + 0.5 * p2 * t * t;
  out[1] = p1 + p2 * t;
  out[2] = p2;
}
struct BendGeometry {
  double wa, wc, kPerB, fold;
};
// bendGeometry (laws.ts:54-58).
BendGeometry bendGeometry(double La, double Lc) {
  double s = La + Lc;
  double lh = (2 * La * Lc) / s;
  return {(2 * Lc) / s, (2 * La) / s, 1 / (lh * lh * 0.5 * s), 4 * lh * lh};
}
int popcount32(uint32_t v) { return __builtin_popcount(v); }
// bendScale (laws.ts:67-74).
double bendScale(double ia, double ic, uint32_t maskA, uint32_t maskC, int B) {
  uint32_t full = B >= 32 ? 0xffffffffu : ((1u << B) - 1u);
  int cont = popcount32(~(maskA | maskC) & full);
  if (cont == 0) return 0;
  int ua = popcount32(~maskA & full), uc = popcount32(~maskC & full);
  return (static_cast<double>(cont) / B) * std::min(ua > 0 ? (ia * B) / ua : 0.0, uc > 0 ? (ic * B) / uc : 0.0);
}
// bendPsiDelta (laws.ts:89-103).
double bendPsiDelta(double q0, double q1, double dq, double a) {
  double s0 = q0 / a, s1 = q1 / a;
  if (s0 < BEND_S0 && s1 < BEND_S0) return dq / ((1 - s0) * (1 - s1));
  double qb = BEND_S0 * a, d0 = 1 - BEND_S0;
  double p1 = 1 / (d0 * d0), p2 = 2 / (a * d0 * d0 * d0);
  if (s0 >= BEND_S0 && s1 >= BEND_S0) return dq * (p1 + 0.5 * p2 * (q0 - qb + (q1 - qb)));
  double lo = std::min(q0, q1);
  double t = std::max(q0, q1) - qb;
  double up = (qb - lo) / ((1 - lo / a) * d0) + t * (p1 + 0.5 * p2 * t);
  return q1 >= q0 ? up : -up;
}
constexpr double SHEAR_JAM = 0.16, SHEAR_RAMP = 0.08, SHEAR_LOCK = 40;
const double SHEAR_COS0 = std::sqrt(1 - std::pow(1 - (1 - SHEAR_JAM) * (1 - SHEAR_JAM), 2));
// shearJam (laws.ts:126-129).
double shearJam(double area) {
  double c = SHEAR_COS0 * std::sqrt(std::min(1.0, std::max(0.02, area)));
  return 1 - std::sqrt(1 - std::sqrt(1 - c * c));
}
double cellArea(double cu, double tu, double cv, double rv) { return std::max(0.5 * (cu + tu), 0.5 * (cv + rv)); }
// shearLaw (laws.ts:140-159): [force, tangent, energy].
void shearLaw(double ks, double Ld, double l, double jam, double* out) {
  double d = l - Ld;
  double f = ks * d, k = ks, e = 0.5 * ks * d * d;
  double c = -d / Ld - jam;
  if (c > 0) {
    double extra = ks * (SHEAR_LOCK - 1);
    if (c < SHEAR_RAMP) {
      f -= (extra * Ld * c * c) / (2 * SHEAR_RAMP);
      k += (extra * c) / SHEAR_RAMP;
      e += (extra * Ld * Ld * c * c * c) / (6 * SHEAR_RAMP);
    } else {
      f -= extra * Ld * (c - 0.5 * SHEAR_RAMP);
      k += extra;
      e += extra * Ld * Ld *
           ((SHEAR_RAMP * SHEAR_RAMP) / 6 + 0.5 * (c - SHEAR_RAMP) * (c - SHEAR_RAMP) + 0.5 * SHEAR_RAMP * (c - SHEAR_RAMP));
    }
  }
  out[0] = f;
  out[1] = k;
  out[2] = e;
}

// ---------------------------------------------------------------------------- lattice.ts

struct LatticeLayer {
  int nx, ny, offset;
};
int coarseCount(int n) { return (n - 1 + 1) / 2 + 1; }  // Math.ceil((n - 1) / 2) + 1
int coarseToFine(int I, int n) { return std::min(2 * I, n - 1); }
// bracket (lattice.ts:30-41): up to two (coarse index, weight).
int bracket(int i, int n, int* idx, double* w) {
  int nc = coarseCount(n);
  int lo = std::min(nc - 1, i >> 1);
  if (coarseToFine(lo, n) > i) lo--;
  int a = coarseToFine(lo, n);
  if (a == i) {
    idx[0] = lo;
    w[0] = 1;
    return 1;
  }
  int b = coarseToFine(lo + 1, n);
  idx[0] = lo;
  w[0] = static_cast<double>(b - i) / (b - a);
  idx[1] = lo + 1;
  w[1] = static_cast<double>(i - a) / (b - a);
  return 2;
}
std::vector<LatticeLayer> coarsenLayers(const std::vector<LatticeLayer>& fine) {
  std::vector<LatticeLayer> out;
  int off = 0;
  for (auto& L : fine) {
    LatticeLayer C{coarseCount(L.nx), coarseCount(L.ny), off};
    off += C.nx * C.ny;
    out.push_back(C);
  }
  return out;
}
bool shouldCoarsen(const std::vector<LatticeLayer>& layers, int minNodes = 48) {
  for (auto& L : layers)
    if (!(L.nx * L.ny > minNodes && L.nx >= 5 && L.ny >= 5)) return false;
  return true;
}

// ---------------------------------------------------------------------------- newtonMultigrid.ts

constexpr int STENCIL = 25, CENTER = 12;
int offsetIndex(int di, int dj) { return (dj + 2) * 5 + (di + 2); }

struct Solver;

// StencilOperator (newtonMultigrid.ts:44-125).
struct StencilOperator {
  int N = 0;
  std::vector<LatticeLayer> layers;
  std::vector<double> A;
  std::vector<uint8_t> fixed;
  std::vector<int> ij;
  const Solver* linkSolver = nullptr;  // fine lattice: connectivity from the spans (A.link)
  explicit StencilOperator(const std::vector<LatticeLayer>& L) : layers(L) {
    for (auto& l : L) N += l.nx * l.ny;
    A.assign(static_cast<size_t>(N) * STENCIL * 9, 0.0);
    fixed.assign(N, 0);
    ij.assign(3 * static_cast<size_t>(N), 0);
    for (size_t l = 0; l < L.size(); ++l)
      for (int j = 0; j < L[l].ny; ++j)
        for (int i = 0; i < L[l].nx; ++i) {
          int n = L[l].offset + j * L[l].nx + i;
          ij[3 * n] = i;
          ij[3 * n + 1] = j;
          ij[3 * n + 2] = static_cast<int>(l);
        }
  }
  int nbr(int n, int di, int dj) const {
    int i = ij[3 * n] + di, j = ij[3 * n + 1] + dj;
    const LatticeLayer& L = layers[ij[3 * n + 2]];
    if (i < 0 || j < 0 || i >= L.nx || j >= L.ny) return -1;
    return L.offset + j * L.nx + i;
  }
  void addBlock(int row, int o, double s, const double* B) {
    double* p = &A[(static_cast<size_t>(row) * STENCIL + o) * 9];
    for (int q = 0; q < 9; ++q) p[q] += s * B[q];
  }
  // y = A x, fixed rows give y = x (newtonMultigrid.ts:95-124).
  void apply(const double* x, double* y) const {
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n) {
      if (fixed[n]) {
        y[3 * n] = x[3 * n];
        y[3 * n + 1] = x[3 * n + 1];
        y[3 * n + 2] = x[3 * n + 2];
        continue;
      }
      double a0 = 0, a1 = 0, a2 = 0;
      for (int dj = -2; dj <= 2; ++dj)
        for (int di = -2; di <= 2; ++di) {
          int m = nbr(n, di, dj);
          if (m < 0 || fixed[m]) continue;
          const double* b = &A[(static_cast<size_t>(n) * STENCIL + offsetIndex(di, dj)) * 9];
          double x0 = x[3 * m], x1 = x[3 * m + 1], x2 = x[3 * m + 2];
          a0 += b[0] * x0 + b[1] * x1 + b[2] * x2;
          a1 += b[3] * x0 + b[4] * x1 + b[5] * x2;
          a2 += b[6] * x0 + b[7] * x1 + b[8] * x2;
        }
      y[3 * n] = a0;
      y[3 * n + 1] = a1;
      y[3 * n + 2] = a2;
    }
  }
};

struct Prolongation {
  std::vector<int> idx;
  std::vector<double> w;
};
struct MGLevel {
  std::shared_ptr<StencilOperator> A;
  std::shared_ptr<Prolongation> P;
};

// ---------------------------------------------------------------------------- learned coarse correction
// Extension with no counterpart in the reference (the reference's coarsest level is two alternating
// line sweeps, newtonMultigrid.ts:495-502): a learned coarse space on the coarsest level. A per-node MLP
// maps features of each coarsest node to LC_K basis values per coordinate; with the node's diagonal
// block D_i = L_i L_i^T the basis is Phi_i = L_i^-T Psi_i (Psi_i the network's 3 x LC_K output). Half-way
// through the coarsest sweeps the V-cycle adds the Galerkin correction on that basis,
//   x += Phi (Phi^T A Phi)^-1 Phi^T (b - A x),
// an A-orthogonal projection; the sweeps around it are mirror images, so the V-cycle stays symmetric
// and PCG keeps its plain form. Inputs per node (LC_IN = 20), none of them depending on the residual:
//   10  lattice position u = i / (nx - 1), v = j / (ny - 1), sin/cos(pi u), sin/cos(pi v),
//       sin/cos(2 pi u), sin/cos(2 pi v);
//    6  D_i / tr(D_i): entries 00, 11, 22, 01, 02, 12;
//    1  log(tr(D_i) / mean tr(D));
//    1  fraction of the 8 window neighbours that are fixed or outside the lattice;
//    2  damage flag (a span at the node exists but is broken or not fully intact), contact flag (contact
//       terms on the node), each the maximum over the fine nodes its prolongation weights reach.
// The basis is built once per PCG solve. A solve whose mean contraction per iteration
// (||r_k|| / ||r_0||)^(1/k) exceeds the guard after three iterations restarts from its iterate with the
// plain V-cycle (the fallback). Logging records the training material: per coarsest operator the
// whitened operator L^-1 A L^-T over its free unknowns and the node inputs, and per call the whitened
// residual L^-1 r and exact correction L^T A^-1 r (dense Cholesky of the coarsest level).
// Network: tanh(x W1 + b1) -> tanh(. W2 + b2) -> . W3 + b3; W row-major [in][out]; output 3 k + c is
// coordinate c of basis vector k.
constexpr int LC_IN = 20, LC_HID = 64, LC_K = 8, LC_OUT = 3 * LC_K;
constexpr int LC_WEIGHTS = LC_IN * LC_HID + LC_HID + LC_HID * LC_HID + LC_HID + LC_HID * LC_OUT + LC_OUT;

void lcForward(const double* w, const double* in, double* out) {
  const double *W1 = w, *b1 = W1 + LC_IN * LC_HID, *W2 = b1 + LC_HID, *b2 = W2 + LC_HID * LC_HID, *W3 = b2 + LC_HID,
               *b3 = W3 + LC_HID * LC_OUT;
  double h1[LC_HID], h2[LC_HID];
  for (int h = 0; h < LC_HID; ++h) {
    double s = b1[h];
    for (int i = 0; i < LC_IN; ++i) s += in[i] * W1[i * LC_HID + h];
    h1[h] = std::tanh(s);
  }
  for (int h = 0; h < LC_HID; ++h) {
    double s = b2[h];
    for (int i = 0; i < LC_HID; ++i) s += h1[i] * W2[i * LC_HID + h];
    h2[h] = std::tanh(s);
  }
  for (int o = 0; o < LC_OUT; ++o) {
    double s = b3[o];
    for (int i = 0; i < LC_HID; ++i) s += h2[i] * W3[i * LC_OUT + o];
    out[o] = s;
  }
}

struct LearnedOp {  // one logged coarsest operator
  int nodes = 0;              // free unknowns / 3
  std::vector<double> At, X;  // whitened operator (3 nodes)^2, inputs nodes x LC_IN
};
struct LearnedCall {
  int op = 0;
  std::vector<double> r, d;  // whitened residual and exact correction, 3 nodes each
};

struct LearnedCoarse {
  bool on = false;       // add the learned coarse space on the coarsest level of every V-cycle
  bool active = false;   // this solve: on and not fallen back
  double guard = 0.9;    // mean contraction per PCG iteration above which a solve falls back
  std::vector<double> w; // LC_WEIGHTS
  std::vector<float> flags;  // 2 per coarsest node, set at the start of each PCG solve
  // the basis of the current solve: Phi (3 N x K), the Cholesky factor of Phi^T A Phi, dropped columns
  const StencilOperator* basisOp = nullptr;
  std::vector<double> phi, G;
  std::vector<uint8_t> dead;
  // logging
  bool log = false;
  size_t logCap = 0;  // calls
  std::vector<LearnedOp> ops;
  std::vector<LearnedCall> calls;
  std::shared_ptr<const StencilOperator> denseOp;  // coarsest operator whose dense factor is cached
  std::vector<double> denseL, nodeL;
  std::vector<int> denseFree;
  size_t denseDim = 0;
  bool denseOk = false;
  long long applied = 0, fallbacks = 0, solves = 0;
};

constexpr double LINK_MIN_INTACT = 0.02;
constexpr double PIVOT_SHIFT = 2e-6;
const double LINE_ALPHAS[4] = {1, 0.5, 0.25, 0.125};
constexpr double LINE_NOISE = 4e-6;

// ---------------------------------------------------------------------------- yarnField.ts

constexpr int DAMAGE_CUT = 255, DAMAGE_PULLED = 254, DAMAGE_SEPARATED = 254;
constexpr int RECOIL_MAX = 12;
constexpr double SHARE_FRACTION = 0.6, SHARE_REACH = 1.2e-3;
constexpr int SHARE_MAXRUN = 6;
constexpr uint16_t SEG_EXISTS = 1, SEG_BROKEN = 2, SEG_SLIPPED = 8;

struct Layer {
  int index, nx, ny, nodeOffset;
  int fOffset, K, M, bu, bv;  // FieldLayer
  Yarn yarns[2];
  double pitchU, pitchV, weavePitchU, weavePitchV;
  double shearStiffness, crossingFriction, crossingNormal0, crossingWrap, airDrag, thickness;
};

int bundleOf(const Layer& fl, int f) { return f == 1 ? fl.bu : fl.bv; }
int spanLength(const Layer& fl, int f) { return f == 1 ? fl.bv : fl.bu; }
double areaOf(int code) { return std::max(0.02, code / 255.0); }
int damageCode(double d) { return d >= 1 ? DAMAGE_CUT : std::min(DAMAGE_PULLED - 1, static_cast<int>(std::floor(d * DAMAGE_CUT))); }

// recoilLength (yarnField.ts:109-115).
double recoilLength(const Yarn& y, double B, double area, double peak, double eps, double mu, double n0, double wrap,
                    double tCross, double pitch) {
  if (!(eps > 0)) return 0;
  double share = area / B;
  double e = std::min(eps, strainAtTension(y, peak / share));
  double comp = share * (axialTension(y, e) * e - axialEnergyDensity(y, e));
  return (comp * pitch) / (mu * (n0 + wrap * std::max(0.0, tCross)));
}
// breakDistance (yarnField.ts:158-177).
int breakDistance(const Layer& fl, const uint8_t* damage, int f, int k, int m) {
  int pos = f == 0 ? k : m, len = f == 0 ? fl.K : fl.M, stride = f == 0 ? 1 : fl.K;
  int c = fl.fOffset + m * fl.K + k;
  int best = -1;
  for (int dir = -1; dir <= 1; dir += 2) {
    for (int d = 1; d <= RECOIL_MAX; ++d) {
      int p = pos + dir * d;
      if (p < 0 || p >= len) break;
      int code = damage[2 * (c + dir * d * stride) + f];
      if (code == DAMAGE_CUT) {
        if (best < 0 || d < best) best = d;
        break;
      }
      if (code != DAMAGE_PULLED) break;
    }
  }
  return best;
}
int nodeOfCrossing(const Layer& L, int k, int m) {
  int i = std::min(L.nx - 1, k / L.bu), j = std::min(L.ny - 1, m / L.bv);
  return L.nodeOffset + j * L.nx + i;
}
// spanCrossing (yarnField.ts:201-204).
int spanCrossing(const Layer& fl, int i, int j, int f, int q, int p) {
  if (f == 1) return fl.fOffset + (j * fl.bv + fl.bv / 2 + p) * fl.K + i * fl.bu + q;
  return fl.fOffset + (j * fl.bv + q) * fl.K + i * fl.bu + fl.bu / 2 + p;
}
// interpolatedStrain (yarnField.ts:216-240).
double interpolatedStrain(const Layer& L, int f, int k, int m, const double* strain) {
  double s = f == 1 ? (k - (L.bu - 1) / 2.0) / L.bu : (k - (L.bu - 0.5)) / L.bu;
  double t = f == 1 ? (m - (L.bv - 0.5)) / L.bv : (m - (L.bv - 1) / 2.0) / L.bv;
  int i0 = static_cast<int>(std::floor(s)), j0 = static_cast<int>(std::floor(t));
  double fu = s - i0, fv = t - j0;
  int imax = f == 1 ? L.nx - 1 : L.nx - 2;
  int jmax = f == 1 ? L.ny - 2 : L.ny - 1;
  double num = 0, den = 0;
  for (int dj = 0; dj < 2; ++dj)
    for (int di = 0; di < 2; ++di) {
      int i = i0 + di, j = j0 + dj;
      if (i < 0 || j < 0 || i > imax || j > jmax) continue;
      double e = strain[2 * (L.nodeOffset + j * L.nx + i) + f];
      if (!std::isfinite(e)) continue;
      double w = (di ? fu : 1 - fu) * (dj ? fv : 1 - fv);
      num += w * e;
      den += w;
    }
  return den > 1e-6 ? num / den : NAN;
}
int shareReach(const Layer& L, int f) {
  return std::max(1, static_cast<int>(std::round(SHARE_REACH / (f == 1 ? L.weavePitchV : L.weavePitchU))));
}
double shareCap(int reach, double mu, double n0, double wrap, double tCross, double peak) {
  return ((2 * reach + 1) * mu * (n0 + wrap * tCross)) / peak;
}
// shareFactor (yarnField.ts:303-321).
double shareFactor(const Layer& fl, const uint8_t* sep, int f, int k, int m, int reach, double cap) {
  int along = f == 1 ? m : k, lenAlong = f == 1 ? fl.M : fl.K;
  int across = f == 1 ? k : m, lenAcross = f == 1 ? fl.K : fl.M;
  auto at = [&](int y, int a) { return fl.fOffset + (f == 1 ? a * fl.K + y : y * fl.K + a); };
  int runs = 0;
  for (int dir = -1; dir <= 1; dir += 2) {
    for (int d = 1; d <= SHARE_MAXRUN; ++d) {
      int y = across + dir * d;
      if (y < 0 || y >= lenAcross) break;
      bool broken = false;
      for (int a = std::max(0, along - reach); a <= std::min(lenAlong - 1, along + reach) && !broken; ++a)
        broken = sep[2 * at(y, a) + f] == 1;
      if (!broken) break;
      runs++;
    }
  }
  return 1 + std::min((SHARE_FRACTION * runs) / 2, cap);
}
// partSpanYarns (yarnField.ts:422-434).
void partSpanYarns(const Layer& fl, uint8_t* damage, int i, int j, int f, int slipEnd) {
  int P = spanLength(fl, f), half = P - P / 2;
  for (int q = 0; q < bundleOf(fl, f); ++q) {
    bool ofA = slipEnd != 0;
    for (int p = 0; p < P; ++p) {
      int e = 2 * spanCrossing(fl, i, j, f, q, p) + f;
      if (damage[e] >= DAMAGE_SEPARATED) {
        if (slipEnd < 0) ofA = false;
      } else if (ofA != (p < half)) {
        damage[e] = DAMAGE_PULLED;
      }
    }
  }
}

// ---------------------------------------------------------------------------- solver.ts (reference)

struct Grip {
  std::vector<int> nodes;
  std::vector<double> w, offset;
  double goal[3];
  double k;
};

struct FloorParams {
  bool on = false;
  double z = 0, bulge = 0.3e-3, stiffness = 1300, friction = 0.35, frictionSpeed = 0.002;
};

struct Solver {
  ora_params prm;
  int N = 0, C = 0;
  std::vector<Layer> layers;
  std::vector<double> mass, crossingNormal0, softening;
  std::vector<uint8_t> pinned;
  std::vector<float> fieldStrength;
  std::vector<uint8_t> fieldArea;
  std::vector<double> x, v, dx, pred, restLength, intact, failSite, strain, tails, lastUpdate;
  std::vector<uint32_t> cutMask;
  std::vector<uint16_t> segFlags;
  std::vector<uint8_t> fieldDamage;
  // per (crossing, family), the last damage update's relative distance to the separation threshold of
  // the yarn acting there: eps / (eps_peak + eps_soft) - 1 for a cut (yarnDamage reaches 1), delta /
  // ((d - 1/2) pitch) - 1 for a pull-out; +inf where nothing was evaluated (test instrumentation)
  std::vector<double> breakMargin;
  std::vector<int> nbr;
  std::vector<int> layerOf;
  std::vector<Grip> grips;
  std::vector<std::vector<std::pair<int, int>>> gripOf;  // per node: (grip, entry)
  FloorParams floor;
  // self-contact (selfcontact.wgsl restated in FP64): K candidate faces per node, the bounds (8 per
  // node: own normal + share, reciprocal direction + share; share >= 1e8: none), the terms of the
  // current Newton iterate (3 gradient + 6 symmetric Hessian per node)
  bool contactOn = false;
  std::vector<int> ctCand;
  std::vector<double> ctBound, extG, extH;
  bool historyEnabled = true;
  int brokenCount = 0, pulledOutCount = 0;
  std::vector<MGLevel> lagged;      // lagged coarse levels (newtonMultigrid.ts:579)
  std::vector<MGLevel> stageLevels; // levels built by ora_build_levels / the last Newton step

  const Layer& layer(int n) const { return layers[layerOf[n]]; }
  int seg(int n, int f, int dir) const {
    if (dir > 0) return nbr[4 * n + 2 * f + 1] >= 0 ? 2 * n + f : -1;
    int p = nbr[4 * n + 2 * f];
    return p >= 0 ? 2 * p + f : -1;
  }
  bool segActive(int s) const { return s >= 0 && (segFlags[s] & (SEG_EXISTS | SEG_BROKEN)) == SEG_EXISTS; }
  int segOther(int s) const { return nbr[4 * (s >> 1) + 2 * (s & 1) + 1]; }

  // diagActive (solver.ts(ref):232-241).
  bool diagActive(int c, int d) const {
    int r = nbr[4 * c + 1], t = nbr[4 * c + 3];
    if (r < 0 || t < 0) return false;
    bool cu = segActive(2 * c), cv = segActive(2 * c + 1), rv = segActive(2 * r + 1), tu = segActive(2 * t);
    return d == 0 ? (cu && rv) || (cv && tu) : (cu && cv) || (rv && tu);
  }

  // airDrag (solver.ts(ref):132-165): row-major 3x3.
  void airDrag(int n, double* D) const {
    std::fill(D, D + 9, 0.0);
    const Layer& m = layer(n);
    if (!(m.airDrag > 0)) return;
    double k = (m.airDrag * m.pitchU * m.pitchV) / prm.h;
    auto tangent = [&](int f, double* t) {
      int a = n, b = n;
      if (segActive(seg(n, f, -1))) a = nbr[4 * n + 2 * f];
      if (segActive(seg(n, f, 1))) b = nbr[4 * n + 2 * f + 1];
      for (int q = 0; q < 3; ++q) t[q] = x[3 * b + q] - x[3 * a + q];
    };
    double tu[3], tv[3];
    tangent(0, tu);
    tangent(1, tv);
    double lu = hyp3(tu[0], tu[1], tu[2]), lv = hyp3(tv[0], tv[1], tv[2]);
    auto outer = [&](const double* e, double kPar, double kPerp) {
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) D[3 * r + c] = (kPar - kPerp) * e[r] * e[c] + (r == c ? kPerp : 0);
    };
    if (lu > 0 && lv > 0) {
      double c[3] = {tu[1] * tv[2] - tu[2] * tv[1], tu[2] * tv[0] - tu[0] * tv[2], tu[0] * tv[1] - tu[1] * tv[0]};
      double lc = hyp3(c[0], c[1], c[2]);
      if (lc > 1e-3 * lu * lv) {
        double e[3] = {c[0] / lc, c[1] / lc, c[2] / lc};
        outer(e, k, 0);
        return;
      }
    }
    if (lu > 0 || lv > 0) {
      double t[3];
      for (int q = 0; q < 3; ++q) t[q] = lu >= lv ? tu[q] / lu : tv[q] / lv;
      outer(t, 0, k);
      return;
    }
    double e[3] = {1, 0, 0};
    outer(e, k, k);
  }
  static void dragMul(const double* D, const double* v, double* o) {
    o[0] = D[0] * v[0] + D[1] * v[1] + D[2] * v[2];
    o[1] = D[3] * v[0] + D[4] * v[1] + D[5] * v[2];
    o[2] = D[6] * v[0] + D[7] * v[1] + D[8] * v[2];
  }

  // gripTerm (solver.ts(ref):173-180), summed over every grip holding the node.
  double gripTerm(int n, double* g) const {
    double ktot = 0;
    for (auto& ge : gripOf[n]) {
      const Grip& G = grips[ge.first];
      int k = ge.second;
      double kg = G.k * G.w[k];
      for (int q = 0; q < 3; ++q) g[q] += kg * (x[3 * n + q] + dx[3 * n + q] - (G.goal[q] + G.offset[3 * k + q]));
      ktot += kg;
    }
    return ktot;
  }
  double gripEnergy(int n) const {
    double E = 0;
    for (auto& ge : gripOf[n]) {
      const Grip& G = grips[ge.first];
      int k = ge.second;
      double l2 = 0;
      for (int q = 0; q < 3; ++q) {
        double d = x[3 * n + q] + dx[3 * n + q] - (G.goal[q] + G.offset[3 * k + q]);
        l2 += d * d;
      }
      E += 0.5 * G.k * G.w[k] * l2;
    }
    return E;
  }

  // response (solver.ts(ref):641-644) = spanResponse (axial.ts:78-80).
  void response(int s, double eps, double* T, double* K) const {
    const Yarn& y = layer(s >> 1).yarns[s & 1];
    *T = intact[s] * axialTension(y, eps);
    *K = intact[s] * axialStiffness(y, eps);
  }

  // segForce (solver.ts(ref):254-277): [fs, kPar, kPerp, l], e = unit vector owner -> far end.
  void segForce(int s, double* out, double* e) const {
    int a = s >> 1, f = s & 1, b = segOther(s);
    double en[3], ee[3];
    for (int q = 0; q < 3; ++q) {
      en[q] = x[3 * b + q] - x[3 * a + q];
      ee[q] = en[q] + (dx[3 * b + q] - dx[3 * a + q]);
    }
    double l = hyp3(ee[0], ee[1], ee[2]), ln = hyp3(en[0], en[1], en[2]);
    for (int q = 0; q < 3; ++q) e[q] = ee[q] / l;
    double L = restLength[s];
    const Yarn& y = layer(a).yarns[f];
    double T, K;
    response(s, l / L - 1, &T, &K);
    double c = y.axialViscosity / (L * prm.h);
    double fs = T + c * (l - ln);
    out[0] = fs;
    out[1] = std::max(K, 0.0) / L + c;
    out[2] = std::max(fs, 0.0) / l;
    out[3] = l;
  }

  // bendCoeffs (solver.ts(ref):284-291): [kb, kd, fold, wa, wc].
  void bendCoeffs(int b, int f, int s0, int s1, double* o) const {
    const Yarn& y = layer(b).yarns[f];
    BendGeometry geo = bendGeometry(restLength[s0], restLength[s1]);
    double scale = bendScale(intact[s0], intact[s1], cutMask[s0], cutMask[s1], y.yarnsPerSpan);
    double kb = y.bendRigidity * scale * geo.kPerB;
    o[0] = kb;
    o[1] = (kb * y.bendViscosity) / prm.h;
    o[2] = geo.fold;
    o[3] = geo.wa;
    o[4] = geo.wc;
  }
  // triple (solver.ts(ref):311-316).
  void triple(int a, int b, int c, double wa, double wc, double* r, double* rn) const {
    for (int k = 0; k < 3; ++k) {
      rn[k] = wa * x[3 * a + k] - 2 * x[3 * b + k] + wc * x[3 * c + k];
      r[k] = rn[k] + wa * dx[3 * a + k] - 2 * dx[3 * b + k] + wc * dx[3 * c + k];
    }
  }
  // bendGradCoeff + bendViscCoeff (solver.ts(ref):294-308).
  static double bendCoeffSum(double kb, double kd, double fold, const double* r, const double* rn) {
    double ps[3];
    bendPsi(r[0] * r[0] + r[1] * r[1] + r[2] * r[2], fold, ps);
    double ke = kb * ps[1];
    double lr = hyp3(r[0], r[1], r[2]);
    return ke + (kd * (lr - hyp3(rn[0], rn[1], rn[2]))) / std::max(lr, 1e-12);
  }
  // addBendingGradient (solver.ts(ref):319-352).
  void addBendingGradient(int n, int f, double* g) const {
    int prev = nbr[4 * n + 2 * f], nxt = nbr[4 * n + 2 * f + 1];
    int sPrev = prev >= 0 ? 2 * prev + f : -1, sNext = nxt >= 0 ? 2 * n + f : -1;
    double c[5], r[3], rn[3];
    if (segActive(sPrev) && segActive(sNext)) {
      bendCoeffs(n, f, sPrev, sNext, c);
      triple(prev, n, nxt, c[3], c[4], r, rn);
      double kv = bendCoeffSum(c[0], c[1], c[2], r, rn);
      for (int k = 0; k < 3; ++k) g[k] += -2 * kv * r[k];
    }
    if (segActive(sNext)) {
      int nxt2 = nbr[4 * nxt + 2 * f + 1];
      int sNext2 = nxt2 >= 0 ? 2 * nxt + f : -1;
      if (segActive(sNext2)) {
        bendCoeffs(nxt, f, sNext, sNext2, c);
        triple(n, nxt, nxt2, c[3], c[4], r, rn);
        double kv = bendCoeffSum(c[0], c[1], c[2], r, rn);
        for (int k = 0; k < 3; ++k) g[k] += c[3] * kv * r[k];
      }
    }
    if (segActive(sPrev)) {
      int prev2 = nbr[4 * prev + 2 * f];
      int sPrev2 = prev2 >= 0 ? 2 * prev2 + f : -1;
      if (segActive(sPrev2)) {
        bendCoeffs(prev, f, sPrev2, sPrev, c);
        triple(prev2, prev, n, c[3], c[4], r, rn);
        double kv = bendCoeffSum(c[0], c[1], c[2], r, rn);
        for (int k = 0; k < 3; ++k) g[k] += c[4] * kv * r[k];
      }
    }
  }

  // cellShear (solver.ts(ref):374-380): [ks, jam].
  void cellShear(int cell, double* ks, double* jam) const {
    int r = nbr[4 * cell + 1], t = nbr[4 * cell + 3];
    auto io = [&](int s) { return segActive(s) ? intact[s] : 0.0; };
    const Layer& m = layer(cell);
    *ks = (m.shearStiffness * crossingNormal0[cell]) / m.crossingNormal0;
    *jam = shearJam(cellArea(io(2 * cell), io(2 * t), io(2 * cell + 1), io(2 * r + 1)));
  }
  double shearRest(int cell) const {
    double a = restLength[2 * cell], b = restLength[2 * cell + 1];
    return std::sqrt(a * a + b * b);
  }

  // Floor terms of a node at its iterate (assemble.wgsl:191-209): gradient, diagonal Hessian,
  // whether the node sits at the hard limit.
  bool floorTerm(int n, double* g, double* H, bool* core) const {
    *core = false;
    if (!floor.on) return false;
    double half = 0.5 * layer(n).thickness;
    double delta = half + floor.bulge;
    double zc = x[3 * n + 2] + dx[3 * n + 2];
    double s = delta - (zc - floor.z);
    if (!(s > 0)) return false;
    double kc = floor.stiffness;
    double lam = kc * s * s / delta;
    double ut0 = dx[3 * n], ut1 = dx[3 * n + 1];
    double kf = floor.friction * lam / std::max(std::sqrt(ut0 * ut0 + ut1 * ut1), floor.frictionSpeed * prm.h);
    g[0] += kf * ut0;
    g[1] += kf * ut1;
    g[2] += -lam;
    H[0] = kf;
    H[1] = kf;
    H[2] = 2 * kc * s / delta;
    *core = zc <= floor.z + half * (1 + 1e-3);
    return true;
  }

  // The z step of node n bounded against the floor from its iterate step linz (floorLowest,
  // common.wgsl:262-265; floorBound, step.wgsl:78-86): a node comes down at most to where its weight
  // alone would sink it into the penalty (or twice its current depth), never below half thickness.
  double floorBoundZ(int n, double linz, double dz) const {
    if (!floor.on) return dz;
    double half = 0.5 * layer(n).thickness;
    double delta = half + floor.bulge;
    double gmag = std::sqrt(prm.gravity[0] * prm.gravity[0] + prm.gravity[1] * prm.gravity[1] + prm.gravity[2] * prm.gravity[2]);
    double sWeight = std::sqrt(mass[n] * gmag * delta / floor.stiffness);
    double z0 = x[3 * n + 2], zLin = z0 + linz;
    double s = std::max(delta - (zLin - floor.z), 0.0);
    double lowest = std::min(std::max(floor.z + delta - std::max(sWeight, 2 * s), floor.z + half), zLin);
    return std::max(dz, lowest - z0);
  }


  // ---------------------------------------------------------------- self-contact (selfcontact.wgsl)
  // SELF_CONTACT (selfcontact.ts:7-33) and the shader's constants (selfcontact.wgsl:21-31).
  static constexpr double CT_CELL = 12e-3, CT_REACH = 3e-3, CT_DELTA = 1.0e-3, CT_K_PEN = 500, CT_MU = 0.45,
                          CT_FRICTION_SPEED = 0.002, CT_BOUND_FRACTION = 0.45, CT_HARD_CORE = 0.3e-3, CT_RECIP_UNIT = 1e-5;
  static constexpr int CT_KC = 4, CT_WINDOW = 3;
  static constexpr unsigned CT_MASK = (1u << 17) - 1u;

  void coordOf(int n, int* i, int* j, int* l) const {
    *l = layerOf[n];
    const Layer& L = layers[*l];
    int k = n - L.nodeOffset;
    *i = k % L.nx, *j = k / L.nx;
  }
  void curOf(int n, double* p) const {
    for (int q = 0; q < 3; ++q) p[q] = x[3 * n + q] + dx[3 * n + q];
  }
  // faceValid (selfcontact.wgsl:78-88)
  bool faceValid(int f) const {
    int i, j, l;
    coordOf(f, &i, &j, &l);
    const Layer& L = layers[l];
    if (i + 1 >= L.nx || j + 1 >= L.ny) return false;
    int c00 = f, c10 = f + 1, c01 = f + L.nx;
    return segActive(2 * c00) && segActive(2 * c00 + 1) && segActive(2 * c10 + 1) && segActive(2 * c01);
  }
  void faceCorners(int f, int* c) const {
    int nx = layer(f).nx;
    c[0] = f, c[1] = f + 1, c[2] = f + nx, c[3] = f + nx + 1;
  }
  static unsigned hashCell(long cx, long cy, long cz) {
    unsigned h = (static_cast<unsigned>(cx) * 73856093u) ^ (static_cast<unsigned>(cy) * 19349663u) ^ (static_cast<unsigned>(cz) * 83492791u);
    return h & CT_MASK;
  }
  static void cellOf(const double* p, long* c) {
    for (int q = 0; q < 3; ++q) c[q] = static_cast<long>(std::floor(p[q] / CT_CELL));
  }
  // Closest point of triangle (a, b, c) to p (Ericson 5.1.5): weights w[3], squared distance.
  static double closestTri(const double* p, const double* a, const double* b, const double* c, double* w) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int q = 0; q < 3; ++q) ab[q] = b[q] - a[q], ac[q] = c[q] - a[q], ap[q] = p[q] - a[q], bp[q] = p[q] - b[q], cp[q] = p[q] - c[q];
    auto dot = [](const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    w[0] = 1, w[1] = 0, w[2] = 0;
    if (!(d1 <= 0 && d2 <= 0)) {
      double d3 = dot(ab, bp), d4 = dot(ac, bp), d5 = dot(ab, cp), d6 = dot(ac, cp);
      double vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
      if (d3 >= 0 && d4 <= d3) {
        w[0] = 0, w[1] = 1, w[2] = 0;
      } else if (d6 >= 0 && d5 <= d6) {
        w[0] = 0, w[1] = 0, w[2] = 1;
      } else if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        double v = d1 / (d1 - d3);
        w[0] = 1 - v, w[1] = v, w[2] = 0;
      } else if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        double v = d2 / (d2 - d6);
        w[0] = 1 - v, w[1] = 0, w[2] = v;
      } else if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        double v = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        w[0] = 0, w[1] = 1 - v, w[2] = v;
      } else {
        double den = 1 / (va + vb + vc), wb = vb * den, wc = vc * den;
        w[0] = 1 - wb - wc, w[1] = wb, w[2] = wc;
      }
    }
    double e[3];
    for (int q = 0; q < 3; ++q) e[q] = p[q] - (w[0] * a[q] + w[1] * b[q] + w[2] * c[q]);
    return dot(e, e);
  }
  // faceHitP (selfcontact.wgsl:159-172): corner weights w4 (c00 c10 c01 c11), closest point q, distance.
  static double faceHitP(const double* p, const double* p00, const double* p10, const double* p01, const double* p11, double* w4, double* q) {
    double w1[3], w2[3];
    double t1 = closestTri(p, p00, p10, p11, w1), t2 = closestTri(p, p00, p11, p01, w2);
    double d;
    if (t1 <= t2) {
      w4[0] = w1[0], w4[1] = w1[1], w4[2] = 0, w4[3] = w1[2];
      d = std::sqrt(t1);
    } else {
      w4[0] = w2[0], w4[1] = 0, w4[2] = w2[2], w4[3] = w2[1];
      d = std::sqrt(t2);
    }
    for (int k = 0; k < 3; ++k) q[k] = w4[0] * p00[k] + w4[1] * p10[k] + w4[2] * p01[k] + w4[3] * p11[k];
    return d;
  }
  double faceHit(const double* p, const int* c, bool start, double* w4, double* q) const {
    double P[4][3];
    for (int k = 0; k < 4; ++k)
      for (int z = 0; z < 3; ++z) P[k][z] = x[3 * c[k] + z] + (start ? 0.0 : dx[3 * c[k] + z]);
    return faceHitP(p, P[0], P[1], P[2], P[3], w4, q);
  }
  static double segDist(const double* q, const double* a, const double* b) {
    double e[3], qa[3];
    for (int k = 0; k < 3; ++k) e[k] = b[k] - a[k], qa[k] = q[k] - a[k];
    double ee = std::max(e[0] * e[0] + e[1] * e[1] + e[2] * e[2], 1e-20);
    double t = std::min(std::max((qa[0] * e[0] + qa[1] * e[1] + qa[2] * e[2]) / ee, 0.0), 1.0);
    return hyp3(qa[0] - t * e[0], qa[1] - t * e[1], qa[2] - t * e[2]);
  }
  static void cross3(const double* u, const double* v, double* o) {
    o[0] = u[1] * v[2] - u[2] * v[1], o[1] = u[2] * v[0] - u[0] * v[2], o[2] = u[0] * v[1] - u[1] * v[0];
  }
  // Segment (o, o + d) against triangle (a, b, c) (Moeller-Trumbore): parameter of the crossing or 2.
  static double segTri(const double* o, const double* d, const double* a, const double* b, const double* c) {
    double e1[3], e2[3], p[3], sv[3], qv[3];
    for (int k = 0; k < 3; ++k) e1[k] = b[k] - a[k], e2[k] = c[k] - a[k], sv[k] = o[k] - a[k];
    cross3(d, e2, p);
    double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
    if (std::fabs(det) < 1e-18) return 2;
    double inv = 1 / det;
    double u = (sv[0] * p[0] + sv[1] * p[1] + sv[2] * p[2]) * inv;
    if (u < 0 || u > 1) return 2;
    cross3(sv, e1, qv);
    double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv;
    if (v < 0 || u + v > 1) return 2;
    double t = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv;
    return t >= 0 && t <= 1 ? t : 2;
  }
  double pathCrossing(const double* o, const double* d, const int* c) const {
    double A0[3], B0[3], E0[3], G0[3], A1[3], B1[3], E1[3], G1[3];
    for (int z = 0; z < 3; ++z) {
      A0[z] = x[3 * c[0] + z], B0[z] = x[3 * c[1] + z], E0[z] = x[3 * c[2] + z], G0[z] = x[3 * c[3] + z];
      A1[z] = A0[z] + dx[3 * c[0] + z], B1[z] = B0[z] + dx[3 * c[1] + z], E1[z] = E0[z] + dx[3 * c[2] + z], G1[z] = G0[z] + dx[3 * c[3] + z];
    }
    double t = std::min(segTri(o, d, A0, B0, G0), segTri(o, d, A0, G0, E0));
    return std::min(t, std::min(segTri(o, d, A1, B1, G1), segTri(o, d, A1, G1, E1)));
  }
  bool rowHolds(const Layer& L, int j, int i0, int i1) const {
    for (int i = std::min(i0, i1); i < std::max(i0, i1); ++i)
      if (!segActive(2 * (L.nodeOffset + j * L.nx + i))) return false;
    return true;
  }
  bool columnHolds(const Layer& L, int i, int j0, int j1) const {
    for (int j = std::min(j0, j1); j < std::max(j0, j1); ++j)
      if (!segActive(2 * (L.nodeOffset + j * L.nx + i) + 1)) return false;
    return true;
  }
  // latticeLinked (selfcontact.wgsl:290-296)
  bool latticeLinked(const Layer& L, int ni, int nj, int fi, int fj) const {
    int ci = std::min(std::max(ni, fi), fi + 1), cj = std::min(std::max(nj, fj), fj + 1);
    if (rowHolds(L, nj, ni, ci) && columnHolds(L, ci, nj, cj)) return true;
    return columnHolds(L, ni, nj, cj) && rowHolds(L, cj, ni, ci);
  }

  // faceCount / scan / faceFill, damageRow, detect, resolveBounds (selfcontact.wgsl:186-478), with
  // the same hash and table, so that hash collisions bring the same extra faces.
  void contactDetect() {
    const size_t T = size_t(CT_MASK) + 1;
    std::vector<std::vector<int>> cells(T);
    struct Item { double m1[3], r, m0[3]; };
    std::vector<Item> items(N);
    for (int f = 0; f < N; ++f) {
      if (!faceValid(f)) continue;
      int c[4];
      faceCorners(f, c);
      double P0[4][3], P1[4][3];
      Item& it = items[f];
      for (int z = 0; z < 3; ++z) it.m0[z] = it.m1[z] = 0;
      for (int k = 0; k < 4; ++k)
        for (int z = 0; z < 3; ++z) {
          P0[k][z] = x[3 * c[k] + z];
          P1[k][z] = P0[k][z] + dx[3 * c[k] + z];
          it.m0[z] += 0.25 * P0[k][z];
          it.m1[z] += 0.25 * P1[k][z];
        }
      double r0 = 0, r1 = 0;
      for (int k = 0; k < 4; ++k) {
        r0 = std::max(r0, sq3(P0[k][0] - it.m0[0], P0[k][1] - it.m0[1], P0[k][2] - it.m0[2]));
        r1 = std::max(r1, sq3(P1[k][0] - it.m1[0], P1[k][1] - it.m1[1], P1[k][2] - it.m1[2]));
      }
      it.r = std::sqrt(std::max(r0, r1));
      long k1[3], k0[3];
      cellOf(it.m1, k1);
      cellOf(it.m0, k0);
      unsigned h1 = hashCell(k1[0], k1[1], k1[2]);
      cells[h1].push_back(f);
      if (!(k0[0] == k1[0] && k0[1] == k1[1] && k0[2] == k1[2])) cells[hashCell(k0[0], k0[1], k0[2])].push_back(f);
    }
    std::vector<uint8_t> rowMark(N, 0);
    for (int n = 0; n < N; ++n) {
      int i, j, l;
      coordOf(n, &i, &j, &l);
      const Layer& L = layers[l];
      for (int a = std::max(i - CT_WINDOW, 0); a <= std::min(i + CT_WINDOW, L.nx - 1); ++a) {
        int m = L.nodeOffset + j * L.nx + a;
        if ((segFlags[2 * m] & SEG_BROKEN) || (segFlags[2 * m + 1] & SEG_BROKEN)) rowMark[n] = 1;
      }
    }
    ctCand.assign(CT_KC * size_t(N), -1);
    ctBound.assign(8 * size_t(N), 0.0);
    std::vector<unsigned long long> recipKey(N, 0);
    for (int n = 0; n < N; ++n) {
      ctBound[8 * n + 3] = 1e9;
      ctBound[8 * n + 7] = 1e9;
      if (pinned[n]) continue;
      double p[3], p0[3], path[3];
      curOf(n, p);
      for (int z = 0; z < 3; ++z) p0[z] = x[3 * n + z], path[z] = p[z] - p0[z];
      bool moving = sq3(path[0], path[1], path[2]) > CT_HARD_CORE * CT_HARD_CORE;
      int best[CT_KC];
      double bestD[CT_KC];
      for (int k = 0; k < CT_KC; ++k) best[k] = -1, bestD[k] = 1e9;
      double d0min = 1e9, n0[3] = {0, 0, 0};
      int f0 = -1;
      double tc = 2;
      int fc = -1;
      long lo[3], hi[3];
      for (int z = 0; z < 3; ++z) {
        lo[z] = static_cast<long>(std::floor(std::min(p[z], p0[z]) / CT_CELL - 0.5));
        hi[z] = std::min(static_cast<long>(std::floor(std::max(p[z], p0[z]) / CT_CELL + 0.5)), lo[z] + 3);
      }
      int ni, nj, nl;
      coordOf(n, &ni, &nj, &nl);
      const Layer& NL = layers[nl];
      bool damaged = false;
      for (int b = std::max(nj - CT_WINDOW, 0); b <= std::min(nj + CT_WINDOW, NL.ny - 1); ++b)
        if (rowMark[NL.nodeOffset + b * NL.nx + ni]) damaged = true;
      // ties on a shared edge go to the lower face index (an unsigned comparison: -1 is none)
      auto lowerIdx = [](int a, int b) { return static_cast<unsigned>(a) < static_cast<unsigned>(b); };
      for (long cz = lo[2]; cz <= hi[2]; ++cz)
        for (long cy = lo[1]; cy <= hi[1]; ++cy)
          for (long cx = lo[0]; cx <= hi[0]; ++cx)
            for (int f : cells[hashCell(cx, cy, cz)]) {
              const Item& it = items[f];
              bool nearNow = hyp3(p[0] - it.m1[0], p[1] - it.m1[1], p[2] - it.m1[2]) - it.r < CT_REACH;
              bool nearStart = hyp3(p0[0] - it.m0[0], p0[1] - it.m0[1], p0[2] - it.m0[2]) - it.r < std::min(d0min, 0.5 * CT_CELL);
              bool onPath = moving && std::min(segDist(it.m0, p0, p), segDist(it.m1, p0, p)) < it.r;
              if (!nearNow && !nearStart && !onPath) continue;
              int fi, fj, fl;
              coordOf(f, &fi, &fj, &fl);
              int di = fi - ni, dj = fj - nj;
              if (fl == nl && di >= -3 && di <= 2 && dj >= -3 && dj <= 2 && (!damaged || latticeLinked(NL, ni, nj, ni + di, nj + dj)))
                continue;
              int cf[4];
              faceCorners(f, cf);
              double w4[4], q[3];
              if (nearStart) {
                double d = faceHit(p0, cf, true, w4, q);
                if ((d < d0min || (d == d0min && lowerIdx(f, f0))) && d > 1e-9) {
                  d0min = d;
                  for (int z = 0; z < 3; ++z) n0[z] = (p0[z] - q[z]) / d;
                  f0 = f;
                }
              }
              if (onPath) {
                double t = pathCrossing(p0, path, cf);
                if (t < tc || (t == tc && t <= 1 && lowerIdx(f, fc))) tc = t, fc = f;
              }
              if (!nearNow) continue;
              double d = faceHit(p, cf, false, w4, q);
              if (d >= CT_REACH) continue;
              int cand = f;
              double cd = d;
              for (int k = 0; k < CT_KC; ++k) {
                if (cand == best[k]) break;
                if (cd < bestD[k] || (cd == bestD[k] && lowerIdx(cand, best[k]))) {
                  std::swap(best[k], cand);
                  std::swap(bestD[k], cd);
                }
              }
            }
      for (int k = 0; k < CT_KC; ++k) ctCand[CT_KC * n + k] = best[k];
      double nb[3] = {n0[0], n0[1], n0[2]}, db = d0min;
      int fb = f0;
      if (fc >= 0 && fc != f0) {
        int c[4];
        faceCorners(fc, c);
        double e1[3], e2[3], nrm[3];
        for (int z = 0; z < 3; ++z) e1[z] = x[3 * c[1] + z] - x[3 * c[0] + z], e2[z] = x[3 * c[2] + z] - x[3 * c[0] + z];
        cross3(e1, e2, nrm);
        double ln = hyp3(nrm[0], nrm[1], nrm[2]);
        if (ln > 1e-12) {
          for (int z = 0; z < 3; ++z) nrm[z] /= ln;
          double side = (p0[0] - x[3 * c[0]]) * nrm[0] + (p0[1] - x[3 * c[0] + 1]) * nrm[1] + (p0[2] - x[3 * c[0] + 2]) * nrm[2];
          for (int z = 0; z < 3; ++z) nb[z] = side >= 0 ? nrm[z] : -nrm[z];
          db = std::fabs(side);
          fb = fc;
        }
      }
      if (fb < 0 || (fb == f0 && db >= 0.5 * CT_CELL)) continue;
      double share = CT_BOUND_FRACTION * std::max(db - CT_HARD_CORE, 0.0);
      for (int z = 0; z < 3; ++z) ctBound[8 * n + z] = nb[z];
      ctBound[8 * n + 3] = share;
      // reciprocal key: the tightest share quantised to 10 um wins (ties: the higher node)
      unsigned long long qs = 4095u - std::min<unsigned long long>(4095u, static_cast<unsigned long long>(share / CT_RECIP_UNIT));
      unsigned long long key = (qs << 20) | static_cast<unsigned long long>(n + 1);
      int c[4];
      faceCorners(fb, c);
      for (int k = 0; k < 4; ++k) recipKey[c[k]] = std::max(recipKey[c[k]], key);
    }
    for (int n = 0; n < N; ++n) {
      unsigned long long key = recipKey[n];
      if (key == 0) continue;
      int j = static_cast<int>(key & 0xFFFFFu) - 1;
      double share = static_cast<double>(4095u - (key >> 20)) * CT_RECIP_UNIT;
      for (int z = 0; z < 3; ++z) ctBound[8 * n + 4 + z] = -ctBound[8 * j + z];
      ctBound[8 * n + 7] = share;
    }
  }

  // terms (selfcontact.wgsl:493-545): penalty and friction at the current iterate into extG/extH
  // (node stiffness doubled, each corner's 2 w H), and the trust region of the own bound.
  void contactTerms() {
    extG.assign(3 * size_t(N), 0.0);
    extH.assign(6 * size_t(N), 0.0);
    const double gmag = hyp3(prm.gravity[0], prm.gravity[1], prm.gravity[2]);
    auto addTerm = [&](int m, const double* g, const double* H, double s) {
      for (int z = 0; z < 3; ++z) extG[3 * m + z] += s * g[z];
      for (int z = 0; z < 6; ++z) extH[6 * m + z] += H[z];
    };
    for (int n = 0; n < N; ++n) {
      double p[3];
      curOf(n, p);
      const double* own = &ctBound[8 * n];
      double reach = 1e9;
      double sWeight = std::sqrt(mass[n] * gmag * CT_DELTA / CT_K_PEN);
      for (int k = 0; k < CT_KC; ++k) {
        int f = ctCand[CT_KC * n + k];
        if (f < 0) continue;
        int c[4];
        faceCorners(f, c);
        double w4[4], q[3];
        double d = faceHit(p, c, false, w4, q);
        if (d <= 1e-9) continue;
        double nn[3] = {(p[0] - q[0]) / d, (p[1] - q[1]) / d, (p[2] - q[2]) / d};
        double al = nn[0] * own[0] + nn[1] * own[1] + nn[2] * own[2];
        if (al > 0.1) reach = std::min(reach, (d - CT_DELTA + std::max(sWeight, 2 * std::max(CT_DELTA - d, 0.0))) / al);
        if (d >= CT_DELTA) continue;
        double sd = CT_DELTA - d;
        double lam = CT_K_PEN * sd * sd / CT_DELTA;
        double rel[3];
        for (int z = 0; z < 3; ++z)
          rel[z] = dx[3 * n + z] - (w4[0] * dx[3 * c[0] + z] + w4[1] * dx[3 * c[1] + z] + w4[2] * dx[3 * c[2] + z] + w4[3] * dx[3 * c[3] + z]);
        double rn = rel[0] * nn[0] + rel[1] * nn[1] + rel[2] * nn[2];
        double ut[3] = {rel[0] - rn * nn[0], rel[1] - rn * nn[1], rel[2] - rn * nn[2]};
        double kf = CT_MU * lam / std::max(hyp3(ut[0], ut[1], ut[2]), CT_FRICTION_SPEED * prm.h);
        double g[3] = {-lam * nn[0] + kf * ut[0], -lam * nn[1] + kf * ut[1], -lam * nn[2] + kf * ut[2]};
        double kn = 2 * CT_K_PEN * sd / CT_DELTA;
        double H[6] = {kn * nn[0] * nn[0] + kf * (1 - nn[0] * nn[0]), (kn - kf) * nn[0] * nn[1], (kn - kf) * nn[0] * nn[2],
                       kn * nn[1] * nn[1] + kf * (1 - nn[1] * nn[1]), (kn - kf) * nn[1] * nn[2], kn * nn[2] * nn[2] + kf * (1 - nn[2] * nn[2])};
        double H2[6];
        for (int z = 0; z < 6; ++z) H2[z] = 2 * H[z];
        addTerm(n, g, H2, 1.0);
        for (int k2 = 0; k2 < 4; ++k2) {
          if (w4[k2] <= 0) continue;
          double Hw[6];
          for (int z = 0; z < 6; ++z) Hw[z] = 2 * w4[k2] * H[z];
          addTerm(c[k2], g, Hw, -w4[k2]);
        }
      }
      // (a node's terms read only its own bound, so it is tightened in place)
      if (reach < 1e9 && (own[0] != 0 || own[1] != 0 || own[2] != 0)) {
        double approach = -(dx[3 * n] * own[0] + dx[3 * n + 1] * own[1] + dx[3 * n + 2] * own[2]);
        ctBound[8 * n + 3] = std::min(own[3], approach + reach);
      }
    }
  }

  // ---- cross-layer contact (contact.ts:7-19, contact.wgsl): a scene of several layers gets node-node
  // contact between its layers in place of self-contact (solver.ts:364), when crossLayer is set.
  // Detection once per substep on a (cell, layer) hash with the same hash and table as the shader
  // (so collisions bring the same extra candidates), the K nearest foreign nodes within the contact
  // distance and a quarter cell, and a directional bound; terms per Newton iterate from the pairs.
  bool crossLayer = false;
  static constexpr double XC_CELL = 1.0e-3, XC_K_PEN = 3000, XC_MU = 0.45, XC_FRICTION_SPEED = 0.002, XC_BOUND_FRACTION = 0.45;
  static constexpr unsigned XC_MASK = (1u << 20) - 1u;
  double xcDist[4] = {0, 0, 0, 0};  // midsurface contact distance of layer pairs 0-1, 0-2, 1-2; same layer
  // hashCell (contact.wgsl:31-34)
  static unsigned xcHash(long cx, long cy, long cz, unsigned l) {
    unsigned h = (static_cast<unsigned>(cx) * 73856093u) ^ (static_cast<unsigned>(cy) * 19349663u) ^
                 (static_cast<unsigned>(cz) * 83492791u) ^ (l * 2654435761u);
    return h & XC_MASK;
  }
  // pairDistance (contact.wgsl:36-42)
  double xcPair(int la, int lb) const {
    if (la == lb) return xcDist[3];
    const int s = la + lb;
    return s == 1 ? xcDist[0] : s == 2 ? xcDist[1] : xcDist[2];
  }
  // hashCount / scan / hashFill / detect (contact.wgsl:46-129), the cells filled in node order
  void crossDetect() {
    const size_t T = size_t(XC_MASK) + 1;
    std::vector<unsigned> key(N);
    std::vector<unsigned> start(T + 1, 0);
    for (int n = 0; n < N; ++n) {
      double p[3];
      curOf(n, p);
      long c[3];
      for (int q = 0; q < 3; ++q) c[q] = static_cast<long>(std::floor(p[q] / XC_CELL));
      key[n] = xcHash(c[0], c[1], c[2], static_cast<unsigned>(layerOf[n]));
      ++start[key[n] + 1];
    }
    for (size_t h = 0; h < T; ++h) start[h + 1] += start[h];
    std::vector<int> items(N);
    std::vector<unsigned> fill(start.begin(), start.end() - 1);
    for (int n = 0; n < N; ++n) items[fill[key[n]]++] = n;
    ctCand.assign(CT_KC * size_t(N), -1);
    ctBound.assign(8 * size_t(N), 0.0);
    for (int n = 0; n < N; ++n) {
      double p[3];
      curOf(n, p);
      const int ln = layerOf[n];
      int best[CT_KC];
      double bestD[CT_KC];
      for (int k = 0; k < CT_KC; ++k) best[k] = -1, bestD[k] = 1e9;
      double dmin = 1e9, nmin[3] = {0, 0, 0};
      long c[3];
      for (int q = 0; q < 3; ++q) c[q] = static_cast<long>(std::floor(p[q] / XC_CELL));
      for (int lo = 0; lo < static_cast<int>(layers.size()); ++lo) {
        if (lo == ln) continue;
        const double r = xcPair(ln, lo);
        for (int dz = -1; dz <= 1; ++dz)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dxc = -1; dxc <= 1; ++dxc) {
              const unsigned h = xcHash(c[0] + dxc, c[1] + dy, c[2] + dz, static_cast<unsigned>(lo));
              for (unsigned q = start[h]; q < start[h + 1]; ++q) {
                const int m = items[q];
                if (layerOf[m] != lo) continue;
                double pm[3];
                curOf(m, pm);
                const double d = hyp3(p[0] - pm[0], p[1] - pm[1], p[2] - pm[2]);
                if (d - r < dmin && d > 1e-9) {
                  dmin = d - r;
                  for (int z = 0; z < 3; ++z) nmin[z] = (p[z] - pm[z]) / d;
                }
                if (d >= r + 0.25 * XC_CELL) continue;
                int cand = m;
                double cd = d - r;
                for (int k = 0; k < CT_KC; ++k)
                  if (cd < bestD[k]) std::swap(best[k], cand), std::swap(bestD[k], cd);
              }
            }
      }
      for (int k = 0; k < CT_KC; ++k) ctCand[CT_KC * n + k] = best[k];
      // the directional bound: approach the nearest foreign node by a share of its clearance plus
      // half the contact distance (of the 0-1 pair, as the shader takes it); no reciprocal bound
      if (dmin < 1e8) {
        for (int z = 0; z < 3; ++z) ctBound[8 * n + z] = nmin[z];
        ctBound[8 * n + 3] = XC_BOUND_FRACTION * (std::max(0.0, dmin) + 0.5 * xcDist[0]);
      } else {
        ctBound[8 * n + 3] = 1e9;
      }
      ctBound[8 * n + 7] = 1e9;
    }
  }
  // terms (contact.wgsl:131-164): linear penalty and lagged-normal regularised Coulomb friction on the
  // relative tangential step, each node's own terms into extG / extH
  void crossTerms() {
    extG.assign(3 * size_t(N), 0.0);
    extH.assign(6 * size_t(N), 0.0);
    const double epsU = XC_FRICTION_SPEED * prm.h;
    for (int n = 0; n < N; ++n) {
      double p[3];
      curOf(n, p);
      double g[3] = {0, 0, 0}, H[6] = {0, 0, 0, 0, 0, 0};
      for (int k = 0; k < CT_KC; ++k) {
        const int m = ctCand[CT_KC * n + k];
        if (m < 0) continue;
        double pm[3];
        curOf(m, pm);
        const double dv[3] = {p[0] - pm[0], p[1] - pm[1], p[2] - pm[2]};
        const double d = hyp3(dv[0], dv[1], dv[2]);
        const double r = xcPair(layerOf[n], layerOf[m]);
        if (d >= r || d <= 1e-9) continue;
        const double nn[3] = {dv[0] / d, dv[1] / d, dv[2] / d};
        const double lam = XC_K_PEN * (r - d);
        double rel[3];
        for (int z = 0; z < 3; ++z) rel[z] = dx[3 * n + z] - dx[3 * m + z];
        const double rn = rel[0] * nn[0] + rel[1] * nn[1] + rel[2] * nn[2];
        const double ut[3] = {rel[0] - rn * nn[0], rel[1] - rn * nn[1], rel[2] - rn * nn[2]};
        const double kf = XC_MU * lam / std::max(hyp3(ut[0], ut[1], ut[2]), epsU);
        for (int z = 0; z < 3; ++z) g[z] += -lam * nn[z] + kf * ut[z];
        const int idx[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
        for (int q = 0; q < 6; ++q) {
          const int a = idx[q][0], b = idx[q][1];
          H[q] += XC_K_PEN * nn[a] * nn[b] + kf * ((a == b ? 1.0 : 0.0) - nn[a] * nn[b]);
        }
      }
      for (int z = 0; z < 3; ++z) extG[3 * n + z] = g[z];
      for (int z = 0; z < 6; ++z) extH[6 * n + z] = H[z];
    }
  }

  // ---- detached pieces' rigid modes (rigid_frame.wgsl, rigid_apply.wgsl, rigid_spin.wgsl; solver.ts:612-716).
  // A detached piece's rigid motion is resisted by its inertia, drag and contact alone, against yarn
  // couplings far stiffer, and the multigrid hierarchy does not carry those near-null modes. Each
  // piece's six rigid modes Z (translation, rotation about its mass centroid) give PCG an exact start
  // x0 = Z E^-1 Z^T b with E = Z^T A Z built from what each term puts on a rigid motion (the external
  // blocks fully, the internal terms only on rotation as their tension's geometric stiffness); the
  // line search and update move a piece's nodes along the rotation of that start rather than its
  // tangent, and each substep starts a spinning piece on its rotation continued over the substep.
  // Pieces are set from outside (Topology.setPieces); with none, nothing here runs.
  static constexpr uint32_t NO_PIECE = 0xFFFFFFFFu;
  static constexpr int MAX_PIECES = 4096;  // solver.ts:86
  std::vector<uint32_t> pieceOf, pieceStart, pieceNodes;
  int pieceCount = 0;
  std::vector<double> pieceFrame;  // 40 per piece: centroid (3), valid, E^-1 row-major (36)
  std::vector<double> pieceStep;   // 6 per piece: rigid step (t, w), or (centroid, spin rotation) in the predictor
  std::vector<double> curveW, curveR;  // 3 per node: the piece's rotation in the direction and the node's arm
  std::vector<uint8_t> curveOn;
  bool inPiece(int n) const { return pieceCount > 0 && pieceOf[n] < static_cast<uint32_t>(pieceCount); }
  void rigidRotation(std::vector<double>& kr) const;
  void rigidFrame(const std::vector<double>& kx);
  void rigidStart(const double* b, double* x0);
  void curveSet();
  void spinStart();
  // rotationCurve (common.wgsl:274-283): R(th) r - r - th x r, what rotating r by th adds to its tangent step
  static void rotationCurve(const double* th, const double* r, double* out) {
    const double phi = hyp3(th[0], th[1], th[2]);
    if (phi < 1e-9) {
      out[0] = out[1] = out[2] = 0;
      return;
    }
    const double k[3] = {th[0] / phi, th[1] / phi, th[2] / phi};
    double kr[3], kkr[3];
    cross3(k, r, kr);
    cross3(k, kr, kkr);
    const double a = std::sin(phi) - phi, c = 1 - std::cos(phi);
    for (int z = 0; z < 3; ++z) out[z] = a * kr[z] + c * kkr[z];
  }

  // A half-space bound: the step may move against m by at most m[3] (step.wgsl:62-65).
  static void boundStep(double* d, const double* m) {
    double approach = -(d[0] * m[0] + d[1] * m[1] + d[2] * m[2]);
    if (approach > m[3])
      for (int z = 0; z < 3; ++z) d[z] += (approach - m[3]) * m[z];
  }
  // feasible (step.wgsl:67-75): own, reciprocal, own.
  void feasible(int n, double* d) const {
    if (!contactOn) return;
    boundStep(d, &ctBound[8 * n]);
    boundStep(d, &ctBound[8 * n + 4]);
    boundStep(d, &ctBound[8 * n]);
  }

  // nodeGradient (solver.ts(ref):387-422).
  void nodeGradient(int n, double* g) const {
    g[0] = g[1] = g[2] = 0;
    if (pinned[n]) return;
    double h = prm.h;
    double w = mass[n] / (h * h);
    for (int q = 0; q < 3; ++q) g[q] += w * (dx[3 * n + q] - pred[3 * n + q]);
    gripTerm(n, g);
    if (contactOn && !extG.empty())
      for (int q = 0; q < 3; ++q) g[q] += extG[3 * n + q];
    double D[9], Dg[3];
    airDrag(n, D);
    dragMul(D, &dx[3 * n], Dg);
    for (int q = 0; q < 3; ++q) g[q] += Dg[q];
    double Hf[3];
    bool core;
    floorTerm(n, g, Hf, &core);
    double sf[4], e[3];
    for (int f = 0; f < 2; ++f) {
      int sPrev = seg(n, f, -1), sNext = seg(n, f, 1);
      if (segActive(sPrev)) {
        segForce(sPrev, sf, e);
        for (int q = 0; q < 3; ++q) g[q] += sf[0] * e[q];
      }
      if (segActive(sNext)) {
        segForce(sNext, sf, e);
        for (int q = 0; q < 3; ++q) g[q] -= sf[0] * e[q];
      }
      addBendingGradient(n, f, g);
    }
    // shearPartners (solver.ts(ref):355-367)
    int left = nbr[4 * n], right = nbr[4 * n + 1], down = nbr[4 * n + 2], up = nbr[4 * n + 3];
    int cand[4][3];
    int nc = 0;
    if (right >= 0 && up >= 0) cand[nc][0] = n, cand[nc][1] = nbr[4 * up + 1], cand[nc++][2] = 0;
    if (left >= 0 && down >= 0) cand[nc][0] = nbr[4 * down], cand[nc][1] = nbr[4 * down], cand[nc++][2] = 0;
    if (left >= 0 && up >= 0) cand[nc][0] = left, cand[nc][1] = nbr[4 * up], cand[nc++][2] = 1;
    if (right >= 0 && down >= 0) cand[nc][0] = down, cand[nc][1] = nbr[4 * down + 1], cand[nc++][2] = 1;
    for (int k = 0; k < nc; ++k) {
      int cell = cand[k][0], partner = cand[k][1];
      if (partner < 0 || !diagActive(cell, cand[k][2])) continue;
      double ks, jam, sl[3];
      cellShear(cell, &ks, &jam);
      double d0 = (x[3 * partner] + dx[3 * partner]) - (x[3 * n] + dx[3 * n]);
      double d1 = (x[3 * partner + 1] + dx[3 * partner + 1]) - (x[3 * n + 1] + dx[3 * n + 1]);
      double d2 = (x[3 * partner + 2] + dx[3 * partner + 2]) - (x[3 * n + 2] + dx[3 * n + 2]);
      double l = hyp3(d0, d1, d2);
      shearLaw(ks, shearRest(cell), l, jam, sl);
      g[0] -= (sl[0] * d0) / l;
      g[1] -= (sl[0] * d1) / l;
      g[2] -= (sl[0] * d2) / l;
    }
  }

  // energyChange (solver.ts(ref):430-534), plus the floor's quadratic model (energy.wgsl:116-125).
  void energyChange(const double* d, double* out, double* mag) const {
    const int NA = 4;
    double h = prm.h;
    std::vector<double> eacc(static_cast<size_t>(N) * 8, 0.0);
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n) {
      double* o = &eacc[8 * static_cast<size_t>(n)];
      double* mg = o + 4;
      auto add = [&](int k, double v) {
        o[k] += v;
        mg[k] += std::fabs(v);
      };
      auto quad = [&](double gd, double q) {
        for (int k = 0; k < NA; ++k) {
          double a = LINE_ALPHAS[k];
          o[k] += a * gd + 0.5 * a * a * q;
          mg[k] += std::fabs(a * gd) + std::fabs(0.5 * a * a * q);
        }
      };
      auto dirOf = [&](int m, double* o3) {
        for (int q = 0; q < 3; ++q) o3[q] = pinned[m] ? 0.0 : d[3 * m + q];
      };
      auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
      // node m's step at step length k (steps, energy.wgsl:63-72): alpha d, plus on a detached piece the
      // rotation curve of its rigid part (alpha being a power of two, alpha d is exact, so a node off
      // every piece steps exactly as alpha times its direction)
      const bool curves = !curveOn.empty();
      auto stepAt = [&](int m, int k, double* o3) {
        const double a = LINE_ALPHAS[k];
        for (int q = 0; q < 3; ++q) o3[q] = pinned[m] ? 0.0 : a * d[3 * m + q];
        if (curves && curveOn[m] && !pinned[m]) {
          const double th[3] = {a * curveW[3 * m], a * curveW[3 * m + 1], a * curveW[3 * m + 2]};
          double c[3];
          rotationCurve(th, &curveR[3 * m], c);
          for (int q = 0; q < 3; ++q) o3[q] += c[q];
        }
      };
      // |e0 + D| - |e0| without cancellation, and |e0 + D|
      auto lenChange = [&](const double* e0, const double* D, double l0, double* la) {
        double ea[3] = {e0[0] + D[0], e0[1] + D[1], e0[2] + D[2]};
        *la = hyp3(ea[0], ea[1], ea[2]);
        return (2 * dot(e0, D) + dot(D, D)) / std::max(*la + l0, 1e-12);
      };
      double sn[4][3];
      for (int k = 0; k < NA; ++k) stepAt(n, k, sn[k]);
      // a quadratic node term (gradient g, Hessian applied by Hs) over the steps
      auto quadS = [&](const double* g, auto Hs) {
        for (int k = 0; k < NA; ++k) {
          double hs[3];
          Hs(sn[k], hs);
          const double lin = dot(g, sn[k]), q = 0.5 * dot(sn[k], hs);
          o[k] += lin + q;
          mg[k] += std::fabs(lin) + std::fabs(q);
        }
      };
      double d0[3] = {dx[3 * n], dx[3 * n + 1], dx[3 * n + 2]};
      const bool curved = curves && curveOn[n] && !pinned[n];
      if (!pinned[n] && !curved) {
        double dn[3];
        dirOf(n, dn);
        double w = mass[n] / (h * h);
        double dp[3] = {d0[0] - pred[3 * n], d0[1] - pred[3 * n + 1], d0[2] - pred[3 * n + 2]};
        quad(w * dot(dn, dp), w * dot(dn, dn));
        double g[3] = {0, 0, 0};
        double kg = gripTerm(n, g);
        if (kg > 0) quad(dot(g, dn), kg * dot(dn, dn));
        if (contactOn && !extG.empty()) {
          const double* eg = &extG[3 * n];
          const double* eh = &extH[6 * n];
          double Hd[3] = {eh[0] * dn[0] + eh[1] * dn[1] + eh[2] * dn[2], eh[1] * dn[0] + eh[3] * dn[1] + eh[4] * dn[2],
                          eh[2] * dn[0] + eh[4] * dn[1] + eh[5] * dn[2]};
          if (eg[0] != 0 || eg[1] != 0 || eg[2] != 0 || eh[0] != 0 || eh[3] != 0 || eh[5] != 0) quad(dot(eg, dn), dot(dn, Hd));
        }
        double Dd[9], t1[3], t2[3];
        airDrag(n, Dd);
        dragMul(Dd, d0, t1);
        dragMul(Dd, dn, t2);
        quad(dot(t1, dn), dot(dn, t2));
        double gf[3] = {0, 0, 0}, Hf[3];
        bool core;
        if (floorTerm(n, gf, Hf, &core)) quad(dot(gf, dn), Hf[0] * dn[0] * dn[0] + Hf[1] * dn[1] * dn[1] + Hf[2] * dn[2] * dn[2]);
      }
      if (curved) {
        // the same node terms along the curved steps
        double w = mass[n] / (h * h);
        double gi[3] = {w * (d0[0] - pred[3 * n]), w * (d0[1] - pred[3 * n + 1]), w * (d0[2] - pred[3 * n + 2])};
        quadS(gi, [&](const double* v3, double* o3) { for (int q = 0; q < 3; ++q) o3[q] = w * v3[q]; });
        double g[3] = {0, 0, 0};
        double kg = gripTerm(n, g);
        if (kg > 0) quadS(g, [&](const double* v3, double* o3) { for (int q = 0; q < 3; ++q) o3[q] = kg * v3[q]; });
        if (contactOn && !extG.empty()) {
          const double* eg = &extG[3 * n];
          const double* eh = &extH[6 * n];
          if (eg[0] != 0 || eg[1] != 0 || eg[2] != 0 || eh[0] != 0 || eh[3] != 0 || eh[5] != 0)
            quadS(eg, [&](const double* v, double* o3) {
              o3[0] = eh[0] * v[0] + eh[1] * v[1] + eh[2] * v[2];
              o3[1] = eh[1] * v[0] + eh[3] * v[1] + eh[4] * v[2];
              o3[2] = eh[2] * v[0] + eh[4] * v[1] + eh[5] * v[2];
            });
        }
        double Dd[9], t1[3];
        airDrag(n, Dd);
        dragMul(Dd, d0, t1);
        quadS(t1, [&](const double* v3, double* o3) { dragMul(Dd, v3, o3); });
        double gf[3] = {0, 0, 0}, Hf[3];
        bool core;
        if (floorTerm(n, gf, Hf, &core))
          quadS(gf, [&](const double* v3, double* o3) { for (int q = 0; q < 3; ++q) o3[q] = Hf[q] * v3[q]; });
      }
      const Layer& mat = layer(n);
      for (int f = 0; f < 2; ++f) {
        const Yarn& y = mat.yarns[f];
        int next = nbr[4 * n + 2 * f + 1];
        int s = 2 * n + f;
        if (next >= 0 && segActive(s)) {
          double L = restLength[s];
          double en[3], ec[3];
          for (int q = 0; q < 3; ++q) {
            en[q] = x[3 * next + q] - x[3 * n + q];
            ec[q] = en[q] + dx[3 * next + q] - d0[q];
          }
          double l0 = hyp3(ec[0], ec[1], ec[2]), ln = hyp3(en[0], en[1], en[2]);
          double T0, K0;
          response(s, l0 / L - 1, &T0, &K0);
          double c = y.axialViscosity / (L * h);
          for (int k = 0; k < NA; ++k) {
            double la, sb[3], de[3];
            stepAt(next, k, sb);
            for (int q = 0; q < 3; ++q) de[q] = sb[q] - sn[k][q];
            double dl = lenChange(ec, de, l0, &la);
            double Ta, Ka;
            response(s, la / L - 1, &Ta, &Ka);
            add(k, 0.5 * (T0 + Ta) * dl);
            add(k, 0.5 * c * dl * (la + l0 - 2 * ln));
          }
        }
        int prev = nbr[4 * n + 2 * f];
        if (prev >= 0 && next >= 0 && segActive(2 * prev + f) && segActive(s)) {
          double cf[5];
          bendCoeffs(n, f, 2 * prev + f, s, cf);
          double kb = cf[0], kd = cf[1], ab = cf[2], wa = cf[3], wc = cf[4];
          double rn[3], r0[3];
          for (int q = 0; q < 3; ++q) {
            rn[q] = wa * x[3 * prev + q] - 2 * x[3 * n + q] + wc * x[3 * next + q];
            r0[q] = rn[q] + wa * dx[3 * prev + q] - 2 * d0[q] + wc * dx[3 * next + q];
          }
          double q0 = dot(r0, r0), l0 = std::sqrt(q0), lrn = hyp3(rn[0], rn[1], rn[2]);
          for (int k = 0; k < NA; ++k) {
            double dp[3], dq[3], dr[3];
            stepAt(prev, k, dp);
            stepAt(next, k, dq);
            for (int q = 0; q < 3; ++q) dr[q] = wa * dp[q] - 2 * sn[k][q] + wc * dq[q];
            double dqa = 2 * dot(r0, dr) + dot(dr, dr);
            add(k, 0.5 * kb * bendPsiDelta(q0, q0 + dqa, dqa, ab));
            double la;
            double dl = lenChange(r0, dr, l0, &la);
            add(k, 0.5 * kd * dl * (la + l0 - 2 * lrn));
          }
        }
      }
      if (nbr[4 * n + 1] >= 0 && nbr[4 * n + 3] >= 0) {
        int r = nbr[4 * n + 1], t = nbr[4 * n + 3], rt = nbr[4 * r + 3];
        double Ld = shearRest(n), ks, jam;
        cellShear(n, &ks, &jam);
        int pq[2][3] = {{n, rt, 0}, {r, t, 1}};
        for (auto& e : pq) {
          int p = e[0], q = e[1];
          if (!diagActive(n, e[2])) continue;
          double ec[3];
          for (int z = 0; z < 3; ++z) ec[z] = x[3 * q + z] + dx[3 * q + z] - x[3 * p + z] - dx[3 * p + z];
          double l0 = hyp3(ec[0], ec[1], ec[2]), sl0[3], sla[3];
          shearLaw(ks, Ld, l0, jam, sl0);
          for (int k = 0; k < NA; ++k) {
            double la, dq[3], dp[3], de[3];
            stepAt(q, k, dq);
            stepAt(p, k, dp);
            for (int z = 0; z < 3; ++z) de[z] = dq[z] - dp[z];
            double dl = lenChange(ec, de, l0, &la);
            shearLaw(ks, Ld, la, jam, sla);
            add(k, 0.5 * (sl0[0] + sla[0]) * dl);
          }
        }
      }
    }
    for (int k = 0; k < 4; ++k) out[k] = mag[k] = 0;
    for (int n = 0; n < N; ++n)
      for (int k = 0; k < 4; ++k) {
        out[k] += eacc[8 * static_cast<size_t>(n) + k];
        mag[k] += eacc[8 * static_cast<size_t>(n) + 4 + k];
      }
  }

  double segLength(int s) const {
    int a = s >> 1, b = segOther(s);
    return hyp3(x[3 * b] - x[3 * a], x[3 * b + 1] - x[3 * a + 1], x[3 * b + 2] - x[3 * a + 2]);
  }

  // potential (solver.ts(ref):537-595): the undamaged (history-free) potential, for verification.
  double potential() const {
    double h = prm.h, E = 0;
    for (int n = 0; n < N; ++n) {
      if (pinned[n]) continue;
      double w = mass[n] / (2 * h * h);
      for (int q = 0; q < 3; ++q) {
        double dd = dx[3 * n + q] - pred[3 * n + q];
        E += w * dd * dd;
      }
      E += gripEnergy(n);
      double D[9], Ddx[3];
      airDrag(n, D);
      dragMul(D, &dx[3 * n], Ddx);
      E += 0.5 * (dx[3 * n] * Ddx[0] + dx[3 * n + 1] * Ddx[1] + dx[3 * n + 2] * Ddx[2]);
    }
    for (int s = 0; s < 2 * N; ++s) {
      if (!segActive(s)) continue;
      int a = s >> 1, f = s & 1, b = segOther(s);
      double pa[3], pb[3];
      for (int q = 0; q < 3; ++q) {
        pa[q] = x[3 * a + q] + dx[3 * a + q];
        pb[q] = x[3 * b + q] + dx[3 * b + q];
      }
      double l = hyp3(pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]);
      double ln = segLength(s);
      double L = restLength[s];
      const Yarn& y = layer(a).yarns[f];
      E += L * axialEnergyDensity(y, l / L - 1);
      double c = y.axialViscosity / (L * h);
      E += 0.5 * c * (l - ln) * (l - ln);
      int nb = nbr[4 * b + 2 * f + 1];
      if (nb >= 0 && segActive(2 * b + f)) {
        double cf[5], r[3], rn[3], ps[3];
        bendCoeffs(b, f, s, 2 * b + f, cf);
        triple(a, b, nb, cf[3], cf[4], r, rn);
        bendPsi(r[0] * r[0] + r[1] * r[1] + r[2] * r[2], cf[2], ps);
        E += 0.5 * cf[0] * ps[0];
        double dv = hyp3(r[0], r[1], r[2]) - hyp3(rn[0], rn[1], rn[2]);
        E += 0.5 * cf[1] * dv * dv;
      }
    }
    for (int n = 0; n < N; ++n) {
      if (nbr[4 * n + 1] < 0 || nbr[4 * n + 3] < 0) continue;
      int r = nbr[4 * n + 1], t = nbr[4 * n + 3], rt = nbr[4 * r + 3];
      double ks, jam, sl[3];
      cellShear(n, &ks, &jam);
      double Ld = shearRest(n);
      int pq[2][3] = {{n, rt, 0}, {r, t, 1}};
      for (auto& e : pq) {
        if (!diagActive(n, e[2])) continue;
        int p = e[0], q = e[1];
        double l = hyp3(x[3 * q] + dx[3 * q] - x[3 * p] - dx[3 * p], x[3 * q + 1] + dx[3 * q + 1] - x[3 * p + 1] - dx[3 * p + 1],
                        x[3 * q + 2] + dx[3 * q + 2] - x[3 * p + 2] - dx[3 * p + 2]);
        shearLaw(ks, Ld, l, jam, sl);
        E += sl[2];
      }
    }
    return E;
  }

  // predict (solver.ts(ref):602-613).
  void predict() {
    lagged.clear();
    double h = prm.h;
    for (int n = 0; n < N; ++n)
      for (int q = 0; q < 3; ++q) {
        double hv = pinned[n] ? 0 : h * v[3 * n + q];
        pred[3 * n + q] = pinned[n] ? 0 : hv + h * h * prm.gravity[q];
        dx[3 * n + q] = hv;
      }
    // detached pieces start from their rotation over the substep (encodePredict, solver.ts:698-704)
    if (pieceCount > 0) spinStart();
    // contact detection at the predicted iterate (SelfContact.encodeDetect, solver.ts:743)
    if (contactOn) crossLayer ? crossDetect() : contactDetect();
    // projectStart (step.wgsl:90-95): the predicted start made feasible and bounded against the floor
    if (floor.on || contactOn)
      for (int n = 0; n < N; ++n) {
        if (pinned[n]) continue;
        feasible(n, &dx[3 * n]);
        dx[3 * n + 2] = floorBoundZ(n, 0.0, dx[3 * n + 2]);
      }
  }

  // segTension (solver.ts(ref):647-652).
  void segTension(int s, double* T, double* k) const {
    double L = restLength[s], l = segLength(s), K;
    response(s, l / L - 1, T, &K);
    *k = std::max(K, 0.0) * (l / (L * L));
  }

  void updateField();
  int pullOut();
  int coupleSpans();
  void updateDamage();
  void slipNode(int n, int f);
  void updateSlip();
  void finalize();

  double yarnMaterialLength() const {
    double total = 0;
    for (int s = 0; s < 2 * N; ++s)
      if (segActive(s)) total += restLength[s];
    for (int q = 0; q < 4 * N; ++q) total += tails[q];
    return total;
  }

  // multigrid
  std::shared_ptr<StencilOperator> assembleFineOperator(std::vector<double>* kx = nullptr) const;
  void rhs(double* b) const;
  std::vector<MGLevel> buildHierarchy(std::shared_ptr<StencilOperator> fine) const;
  void vcycle(const std::vector<MGLevel>& levels, int k, double* x, const double* b) const;
  std::shared_ptr<StencilOperator> pcgOp;  // precision study (fp32_rows 3): PCG's operator apart from the hierarchy's
  void pcg(const std::vector<MGLevel>& levels, const double* b, double* x, int iterations, double tol, int* done,
           double* rel) const;
  double newtonStep(int* pcgDone, double* rel, double* alphaOut);

  // learned coarse correction (extension; no counterpart in the reference)
  mutable LearnedCoarse lc;
  void learnedFlags(const std::vector<MGLevel>& levels) const;
  bool learnedInputs(const StencilOperator& A, std::vector<double>& L, std::vector<uint8_t>& ok,
                     std::vector<double>& X) const;
  void learnedBasis(const std::vector<MGLevel>& levels) const;
  void learnedCorrection(const std::vector<MGLevel>& levels, int k, double* x, const double* b) const;
};

// updateField (yarnField.ts:338-410).
void Solver::updateField() {
  if (breakMargin.size() != fieldDamage.size()) breakMargin.assign(fieldDamage.size(), INFINITY);
  std::vector<uint8_t> sep(fieldDamage.size());
  for (size_t q = 0; q < fieldDamage.size(); ++q) sep[q] = fieldDamage[q] >= DAMAGE_SEPARATED ? 1 : 0;
  for (const Layer& L : layers) {
    for (int j = 0; j < L.ny; ++j)
      for (int i = 0; i < L.nx; ++i)
        for (int f = 0; f < 2; ++f) {
          if ((f == 0 && i >= L.nx - 1) || (f == 1 && j >= L.ny - 1)) continue;
          int s = 2 * (L.nodeOffset + j * L.nx + i) + f;
          if (!segActive(s)) continue;
          const Yarn& y = L.yarns[f];
          int B = bundleOf(L, f), P = spanLength(L, f);
          double soft = softening[s] / restLength[s];
          int reach = shareReach(L, f);
          for (int q = 0; q < B; ++q) {
            if ((cutMask[s] >> q) & 1) continue;
            int mid = spanCrossing(L, i, j, f, q, P >> 1) - L.fOffset;
            double eps = interpolatedStrain(L, f, mid % L.K, mid / L.K, strain.data());
            if (!std::isfinite(eps)) continue;
            double minPeak = INF;
            for (int p = 0; p < P; ++p) {
              int c = spanCrossing(L, i, j, f, q, p);
              minPeak = std::min(minPeak, strainAtTension(y, (static_cast<double>(fieldStrength[2 * c + f]) * B) / areaOf(fieldArea[2 * c + f])));
            }
            if (eps * (1 + SHARE_FRACTION * SHARE_MAXRUN) <= minPeak) continue;
            int g = 1 - f;
            int kM = mid % L.K, mM = mid / L.K;
            double ec = interpolatedStrain(L, g, kM, mM, strain.data());
            double tCross = std::isfinite(ec)
                                ? (std::max(0.0, axialTension(L.yarns[g], ec)) * areaOf(fieldArea[2 * (mid + L.fOffset) + g])) / bundleOf(L, g)
                                : 0;
            double transfer = shareCap(reach, L.crossingFriction, crossingNormal0[s >> 1] / (L.bu * L.bv), L.crossingWrap, tCross, 1);
            int best = -1, soft0 = -1, softCode = 0;
            double bestScore = -INF, bestOmega = 1;
            for (int p = 0; p < P; ++p) {
              int c = spanCrossing(L, i, j, f, q, p);
              int local = c - L.fOffset;
              double omega = shareFactor(L, sep.data(), f, local % L.K, local / L.K, reach, transfer / fieldStrength[2 * c + f]);
              double peak = strainAtTension(y, (static_cast<double>(fieldStrength[2 * c + f]) * B) / areaOf(fieldArea[2 * c + f]));
              double score = omega / peak;
              if (score > bestScore) best = c, bestScore = score, bestOmega = omega;
              if (fieldDamage[2 * c + f] > softCode) soft0 = c, softCode = fieldDamage[2 * c + f];
            }
            if (soft0 >= 0) {
              best = soft0;
              int local = best - L.fOffset;
              bestOmega = shareFactor(L, sep.data(), f, local % L.K, local / L.K, reach, transfer / fieldStrength[2 * best + f]);
            }
            int code = damageCode(yarnDamage(y, B, areaOf(fieldArea[2 * best + f]), fieldStrength[2 * best + f], soft, eps * bestOmega));
            {
              const double ep = strainAtTension(y, (static_cast<double>(fieldStrength[2 * best + f]) * B) / areaOf(fieldArea[2 * best + f]));
              const double m = eps * bestOmega / (ep + soft) - 1;
              double& bm = breakMargin[2 * best + f];
              if (std::fabs(m) < std::fabs(bm)) bm = m;
            }
            if (code > fieldDamage[2 * best + f]) fieldDamage[2 * best + f] = static_cast<uint8_t>(code);
          }
        }
  }
}

// pullOut (yarnField.ts:125-152).
int Solver::pullOut() {
  if (breakMargin.size() != fieldDamage.size()) breakMargin.assign(fieldDamage.size(), INFINITY);
  std::vector<int> marked;
  for (const Layer& L : layers)
    for (int m = 0; m < L.M; ++m)
      for (int k = 0; k < L.K; ++k) {
        int c = L.fOffset + m * L.K + k;
        for (int f = 0; f < 2; ++f) {
          if (fieldDamage[2 * c + f] >= DAMAGE_SEPARATED) continue;
          int d = breakDistance(L, fieldDamage.data(), f, k, m);
          if (d < 0) continue;
          double eps = interpolatedStrain(L, f, k, m, strain.data());
          if (!std::isfinite(eps)) continue;
          int g = 1 - f;
          double ec = interpolatedStrain(L, g, k, m, strain.data());
          double tCross = std::isfinite(ec) ? (std::max(0.0, axialTension(L.yarns[g], ec)) * areaOf(fieldArea[2 * c + g])) / bundleOf(L, g) : 0;
          int n = nodeOfCrossing(L, k, m);
          double pitch = f == 1 ? L.weavePitchV : L.weavePitchU;
          double delta = recoilLength(L.yarns[f], bundleOf(L, f), areaOf(fieldArea[2 * c + f]), fieldStrength[2 * c + f], eps,
                                      L.crossingFriction, crossingNormal0[n] / (L.bu * L.bv), L.crossingWrap, tCross, pitch);
          if (delta >= (d - 0.5) * pitch) marked.push_back(2 * c + f);
          {
            const double m = delta / ((d - 0.5) * pitch) - 1;
            double& bm = breakMargin[2 * c + f];
            if (std::fabs(m) < std::fabs(bm)) bm = m;
          }
        }
      }
  for (int q : marked) fieldDamage[q] = DAMAGE_PULLED;
  return static_cast<int>(marked.size());
}

// coupleSpans (yarnField.ts:443-499).
int Solver::coupleSpans() {
  int ruptures = 0;
  for (const Layer& L : layers)
    for (int j = 0; j < L.ny; ++j)
      for (int i = 0; i < L.nx; ++i)
        for (int f = 0; f < 2; ++f) {
          if ((f == 0 && i >= L.nx - 1) || (f == 1 && j >= L.ny - 1)) continue;
          int n = L.nodeOffset + j * L.nx + i;
          int s = 2 * n + f;
          if (segFlags[s] & SEG_SLIPPED) {
            partSpanYarns(L, fieldDamage.data(), i, j, f, failSite[s] < 0.5 ? 0 : 1);
            segFlags[s] &= static_cast<uint16_t>(~SEG_SLIPPED);
            continue;
          }
          if (!segActive(s)) continue;
          int B = bundleOf(L, f), P = spanLength(L, f);
          double sum = 0, site = 0;
          uint32_t mask = 0;
          for (int q = 0; q < B; ++q) {
            int dmax = 0, first = -1;
            double compliance = 0;
            for (int p = 0; p < P; ++p) {
              int c = spanCrossing(L, i, j, f, q, p);
              int d = fieldDamage[2 * c + f];
              if (d > dmax) dmax = d;
              if (d >= DAMAGE_SEPARATED && first < 0) first = p;
              compliance += 1 / areaOf(fieldArea[2 * c + f]);
            }
            sum += (dmax >= DAMAGE_SEPARATED ? 0 : 1 - static_cast<double>(dmax) / DAMAGE_CUT) * (P / compliance);
            if (dmax >= DAMAGE_SEPARATED) {
              mask |= 1u << q;
              site += (first + 0.5) / P;
            }
          }
          intact[s] = sum / B;
          cutMask[s] = mask;
          uint32_t full = B >= 32 ? 0xffffffffu : ((1u << B) - 1u);
          if (mask == full) {
            double phi = site / B, rest = restLength[s];
            int b = f == 0 ? n + 1 : n + L.nx;
            segFlags[s] |= SEG_BROKEN;
            failSite[s] = phi;
            tails[4 * n + 2 * f + 1] += rest * phi;
            tails[4 * b + 2 * f] += rest * (1 - phi);
            ruptures++;
            partSpanYarns(L, fieldDamage.data(), i, j, f, -1);
          }
        }
  return ruptures;
}

// updateDamage (solver.ts(ref):659-666).
void Solver::updateDamage() {
  breakMargin.assign(fieldDamage.size(), INFINITY);
  for (int q = 0; q < 2 * N; ++q) strain[q] = segActive(q) ? segLength(q) / restLength[q] - 1 : NAN;
  updateField();
  pullOut();
  brokenCount += coupleSpans();
}

// slipNode (solver.ts(ref):685-740).
void Solver::slipNode(int n, int f) {
  if (pinned[n]) return;
  int sL = seg(n, f, -1), sR = seg(n, f, 1);
  if (sL < 0 || sR < 0) return;
  bool actL = segActive(sL), actR = segActive(sR);
  if (!actL && !actR) return;
  int tailL = 4 * n + 2 * f, tailR = 4 * n + 2 * f + 1;
  double TL = 0, kL = 0, TR = 0, kR = 0;
  if (actL) segTension(sL, &TL, &kL);
  if (actR) segTension(sR, &TR, &kR);
  double tc = 0;
  int cnt = 0;
  for (int dir = -1; dir <= 1; dir += 2) {
    int s = seg(n, 1 - f, dir);
    if (segActive(s)) {
      double T, k;
      segTension(s, &T, &k);
      tc += std::max(0.0, T);
      cnt++;
    }
  }
  if (cnt == 0) return;
  tc /= cnt;
  const Layer& mat = layer(n);
  double Fc = mat.crossingFriction * (crossingNormal0[n] + mat.crossingWrap * mat.yarns[f].yarnsPerSpan * tc);
  double dT = std::max(TR, 0.0) - std::max(TL, 0.0);
  if (std::fabs(dT) <= Fc) return;
  bool highR = dT > 0;
  double kHigh = highR ? kR : kL;
  bool lowActive = highR ? actL : actR;
  double kLow = lowActive ? (highR ? kL : kR) : 0;
  double dl = (std::fabs(dT) - Fc) / std::max(kHigh + kLow, 1e-9);
  double pitch = f == 0 ? mat.pitchU : mat.pitchV;
  int sHigh = highR ? sR : sL, sLow = highR ? sL : sR;
  if (lowActive) {
    dl = std::min(dl, std::max(0.0, restLength[sLow] - 0.55 * pitch));
    restLength[sLow] -= dl;
    restLength[sHigh] += dl;
  } else {
    int tIdx = highR ? tailL : tailR;
    dl = std::min(dl, tails[tIdx]);
    tails[tIdx] -= dl;
    restLength[sHigh] += dl;
    if (tails[tIdx] <= 1e-9) {
      tails[tIdx] = 0;
      int far = highR ? segOther(sHigh) : sHigh >> 1;
      int farTail = highR ? 4 * far + 2 * f : 4 * far + 2 * f + 1;
      tails[farTail] += restLength[sHigh];
      segFlags[sHigh] |= SEG_BROKEN | SEG_SLIPPED;
      failSite[sHigh] = highR ? 0 : 1;
      pulledOutCount++;
    }
  }
}

// updateSlip (solver.ts(ref):669-683).
void Solver::updateSlip() {
  for (int f = 0; f < 2; ++f)
    for (int parity = 0; parity < 2; ++parity)
      for (const Layer& L : layers)
        for (int j = 0; j < L.ny; ++j)
          for (int i = 0; i < L.nx; ++i) {
            int along = f == 0 ? i : j;
            if ((along & 1) != parity) continue;
            slipNode(L.nodeOffset + j * L.nx + i, f);
          }
}

// finalize (solver.ts(ref):622-632).
void Solver::finalize() {
  double h = prm.h;
  for (int q = 0; q < 3 * N; ++q) {
    v[q] = dx[q] / h;
    x[q] += dx[q];
    dx[q] = 0;
  }
  if (!historyEnabled) return;
  updateDamage();
  updateSlip();
}

// ---------------------------------------------------------------------------- assembly

void axialBlock(double kPar, double kPerp, const double* e, double* out) {
  double d = kPar - kPerp;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[r * 3 + c] = d * e[r] * e[c] + (r == c ? kPerp : 0);
}
// scatterPair (newtonMultigrid.ts:133-146).
void scatterPair(StencilOperator& A, int a, int b, const double* H) {
  int ia = A.ij[3 * a], ja = A.ij[3 * a + 1], ib = A.ij[3 * b], jb = A.ij[3 * b + 1];
  if (!A.fixed[a]) {
    A.addBlock(a, CENTER, 1, H);
    if (!A.fixed[b]) A.addBlock(a, offsetIndex(ib - ia, jb - ja), -1, H);
  }
  if (!A.fixed[b]) {
    A.addBlock(b, CENTER, 1, H);
    if (!A.fixed[a]) A.addBlock(b, offsetIndex(ia - ib, ja - jb), -1, H);
  }
}
const double I3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};

// assembleFineOperator (newtonMultigrid.ts:169-274), plus the floor's diagonal Hessian and its hard
// limit (assemble.wgsl:191-209, 318-322) when the floor is on.
std::shared_ptr<StencilOperator> Solver::assembleFineOperator(std::vector<double>* kx) const {
  std::vector<LatticeLayer> ll;
  for (auto& L : layers) ll.push_back({L.nx, L.ny, L.nodeOffset});
  auto Ap = std::make_shared<StencilOperator>(ll);
  StencilOperator& A = *Ap;
  A.linkSolver = this;
  double h = prm.h;
  for (int n = 0; n < N; ++n)
    if (pinned[n]) {
      A.fixed[n] = 1;
      A.addBlock(n, CENTER, 1, I3);
    }
  double gTmp[3];
  for (int n = 0; n < N; ++n) {
    if (A.fixed[n]) continue;
    gTmp[0] = gTmp[1] = gTmp[2] = 0;
    A.addBlock(n, CENTER, mass[n] / (h * h) + gripTerm(n, gTmp), I3);
    double D[9];
    airDrag(n, D);
    A.addBlock(n, CENTER, 1, D);
  }
  double H[9], e[3];
  for (int s = 0; s < 2 * N; ++s) {
    if (!segActive(s)) continue;
    int a = s >> 1, f = s & 1, b = segOther(s);
    double l = 0;
    for (int q = 0; q < 3; ++q) {
      e[q] = x[3 * b + q] + dx[3 * b + q] - x[3 * a + q] - dx[3 * a + q];
      l += e[q] * e[q];
    }
    l = std::sqrt(l);
    for (int q = 0; q < 3; ++q) e[q] /= l;
    double L = restLength[s];
    const Yarn& y = layer(a).yarns[f];
    double T, K;
    response(s, l / L - 1, &T, &K);
    double ln = segLength(s);
    double c = y.axialViscosity / (L * h);
    double fs = T + c * (l - ln);
    axialBlock(std::max(K, 0.0) / L + c, std::max(fs, 0.0) / l, e, H);
    scatterPair(A, a, b, H);
  }
  for (int b = 0; b < N; ++b)
    for (int f = 0; f < 2; ++f) {
      int a = nbr[4 * b + 2 * f], c = nbr[4 * b + 2 * f + 1];
      if (a < 0 || c < 0) continue;
      int s0 = 2 * a + f, s1 = 2 * b + f;
      if (!segActive(s0) || !segActive(s1)) continue;
      const Yarn& y = layer(b).yarns[f];
      double cf[5];
      bendCoeffs(b, f, s0, s1, cf);
      double kb = cf[0], fold = cf[2], wa = cf[3], wc = cf[4];
      double q2 = 0;
      for (int z = 0; z < 3; ++z) {
        double rz = wa * (x[3 * a + z] + dx[3 * a + z]) - 2 * (x[3 * b + z] + dx[3 * b + z]) + wc * (x[3 * c + z] + dx[3 * c + z]);
        q2 += rz * rz;
      }
      double ps[3];
      bendPsi(q2, fold, ps);
      double k = kb * (ps[1] + 2 * ps[2] * q2) + (kb * y.bendViscosity) / h;
      int nodes[3] = {a, b, c};
      double w[3] = {wa, -2, wc};
      for (int p = 0; p < 3; ++p) {
        int r = nodes[p];
        if (A.fixed[r]) continue;
        for (int q = 0; q < 3; ++q) {
          int m = nodes[q];
          if (A.fixed[m]) continue;
          int o = offsetIndex(A.ij[3 * m] - A.ij[3 * r], A.ij[3 * m + 1] - A.ij[3 * r + 1]);
          A.addBlock(r, o, k * w[p] * w[q], I3);
        }
      }
    }
  for (int n = 0; n < N; ++n) {
    int r = nbr[4 * n + 1], t = nbr[4 * n + 3];
    if (r < 0 || t < 0) continue;
    int rt = nbr[4 * r + 3];
    double ks, jam;
    cellShear(n, &ks, &jam);
    double Ld = std::sqrt(restLength[2 * n] * restLength[2 * n] + restLength[2 * n + 1] * restLength[2 * n + 1]);
    int pq[2][3] = {{n, rt, 0}, {r, t, 1}};
    for (auto& pe : pq) {
      int p = pe[0], q = pe[1];
      if (!diagActive(n, pe[2])) continue;
      double pa[3], l = 0, sl[3];
      for (int z = 0; z < 3; ++z) {
        pa[z] = x[3 * q + z] + dx[3 * q + z] - x[3 * p + z] - dx[3 * p + z];
        l += pa[z] * pa[z];
      }
      l = std::sqrt(l);
      for (int z = 0; z < 3; ++z) pa[z] /= l;
      shearLaw(ks, Ld, l, jam, sl);
      axialBlock(sl[1], std::max(sl[0], 0.0) / l, pa, H);
      scatterPair(A, p, q, H);
    }
  }
  // the external block of each node of a detached piece (assemble.wgsl:172-190, 323-327): its
  // inertia, grip and drag here, its contact and floor blocks and active bounds below
  if (kx) {
    kx->assign(9 * static_cast<size_t>(N), 0.0);
    for (int n = 0; n < N; ++n) {
      if (A.fixed[n] || !inPiece(n)) continue;
      double* K = &(*kx)[9 * static_cast<size_t>(n)];
      double gT[3] = {0, 0, 0};
      const double w = mass[n] / (h * h) + gripTerm(n, gT);
      double D[9];
      airDrag(n, D);
      for (int z = 0; z < 9; ++z) K[z] = D[z] + (z % 4 == 0 ? w : 0.0);
    }
  }
  // contact's diagonal blocks, the floor's, then the active bounds (contact and the floor's hard
  // limit) where the forces still press on, at ACTIVE_BOUND times the block's trace
  // (assemble.wgsl:142, 191-209, 304-322)
  if (floor.on || contactOn) {
    for (int n = 0; n < N; ++n) {
      if (A.fixed[n]) continue;
      double g[3], Hf[3];
      nodeGradient(n, g);
      double* Dn = &A.A[(static_cast<size_t>(n) * STENCIL + CENTER) * 9];
      double* K = kx && inPiece(n) ? &(*kx)[9 * static_cast<size_t>(n)] : nullptr;
      if (contactOn && !extH.empty()) {
        const double* eh = &extH[6 * n];
        double B[9] = {eh[0], eh[1], eh[2], eh[1], eh[3], eh[4], eh[2], eh[4], eh[5]};
        for (int z = 0; z < 9; ++z) Dn[z] += B[z];
        if (K)
          for (int z = 0; z < 9; ++z) K[z] += B[z];
      }
      double gg[3] = {0, 0, 0};
      bool core = false;
      if (floorTerm(n, gg, Hf, &core)) {
        Dn[0] += Hf[0];
        Dn[4] += Hf[1];
        Dn[8] += Hf[2];
        if (K) K[0] += Hf[0], K[4] += Hf[1], K[8] += Hf[2];
      }
      const double kAct = 100.0 * (Dn[0] + Dn[4] + Dn[8]);
      if (contactOn && !ctBound.empty())
        for (int b = 0; b < 2; ++b) {
          const double* m = &ctBound[8 * n + 4 * b];
          if (m[3] >= 1e8 || (m[0] == 0 && m[1] == 0 && m[2] == 0)) continue;
          double app = -(dx[3 * n] * m[0] + dx[3 * n + 1] * m[1] + dx[3 * n + 2] * m[2]);
          if (app >= m[3] - 1e-3 * std::fabs(m[3]) && g[0] * m[0] + g[1] * m[1] + g[2] * m[2] > 0)
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) {
                Dn[3 * r + c] += kAct * m[r] * m[c];
                if (K) K[3 * r + c] += kAct * m[r] * m[c];
              }
        }
      if (core && g[2] > 0) {
        Dn[8] += kAct;
        if (K) K[8] += kAct;
      }
    }
  }
  return Ap;
}

void Solver::rhs(double* b) const {
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    double g[3];
    if (pinned[n]) {
      b[3 * n] = b[3 * n + 1] = b[3 * n + 2] = 0;
      continue;
    }
    nodeGradient(n, g);
    b[3 * n] = -g[0];
    b[3 * n + 1] = -g[1];
    b[3 * n + 2] = -g[2];
  }
}

// linked (newtonMultigrid.ts:287-295) with the fine lattice's A.link (newtonMultigrid.ts:172-175).
bool linked(const StencilOperator& A, int a, int di, int dj) {
  int b = A.nbr(a, di, dj);
  if (b < 0) return false;
  if (A.linkSolver) {
    const Solver& S = *A.linkSolver;
    int s = S.seg(a, di != 0 ? 0 : 1, di + dj > 0 ? 1 : -1);
    return S.segActive(s) && S.intact[s] > LINK_MIN_INTACT;
  }
  if (A.fixed[b]) return true;
  const double* p = &A.A[(static_cast<size_t>(a) * STENCIL + offsetIndex(di, dj)) * 9];
  for (int q = 0; q < 9; ++q)
    if (p[q] != 0) return true;
  return false;
}

// buildProlongation (newtonMultigrid.ts:305-342).
std::shared_ptr<Prolongation> buildProlongation(const StencilOperator& fine, std::vector<LatticeLayer>* coarseOut) {
  std::vector<LatticeLayer> coarse = coarsenLayers(fine.layers);
  auto P = std::make_shared<Prolongation>();
  P->idx.assign(4 * static_cast<size_t>(fine.N), -1);
  P->w.assign(4 * static_cast<size_t>(fine.N), 0.0);
  for (size_t l = 0; l < fine.layers.size(); ++l) {
    const LatticeLayer& L = fine.layers[l];
    const LatticeLayer& C = coarse[l];
    for (int j = 0; j < L.ny; ++j) {
      int bjI[2];
      double bjW[2];
      int nbj = bracket(j, L.ny, bjI, bjW);
      for (int i = 0; i < L.nx; ++i) {
        int f = L.offset + j * L.nx + i;
        if (fine.fixed[f]) continue;
        int biI[2];
        double biW[2];
        int nbi = bracket(i, L.nx, biI, biW);
        int k = 0;
        double sum = 0;
        for (int a = 0; a < nbj; ++a) {
          int J = bjI[a];
          double wj = bjW[a];
          int dj = coarseToFine(J, L.ny) - j;
          for (int b = 0; b < nbi; ++b) {
            int I = biI[b];
            double wi = biW[b];
            int di = coarseToFine(I, L.nx) - i;
            bool ok = true;
            if (di != 0 && dj != 0) {
              int m1 = fine.nbr(f, di, 0), m2 = fine.nbr(f, 0, dj);
              ok = (linked(fine, f, di, 0) && linked(fine, m1, 0, dj)) || (linked(fine, f, 0, dj) && linked(fine, m2, di, 0));
            } else if (di != 0 || dj != 0) {
              ok = linked(fine, f, di, dj);
            }
            P->idx[4 * f + k] = C.offset + J * C.nx + I;
            P->w[4 * f + k] = ok ? wi * wj : 0;
            sum += P->w[4 * f + k];
            k++;
          }
        }
        for (int q = 0; q < k; ++q) P->w[4 * f + q] = sum > 0 ? P->w[4 * f + q] / sum : 0;
      }
    }
  }
  *coarseOut = coarse;
  return P;
}

// galerkin (newtonMultigrid.ts:345-387).
std::shared_ptr<StencilOperator> galerkin(const StencilOperator& A, const std::vector<LatticeLayer>& coarseLayers,
                                          const Prolongation& P) {
  auto Cp = std::make_shared<StencilOperator>(coarseLayers);
  StencilOperator& C = *Cp;
  double blk[9];
  for (int a = 0; a < A.N; ++a) {
    if (A.fixed[a]) continue;
    for (int dj = -2; dj <= 2; ++dj)
      for (int di = -2; di <= 2; ++di) {
        int b = A.nbr(a, di, dj);
        if (b < 0 || A.fixed[b]) continue;
        const double* src = &A.A[(static_cast<size_t>(a) * STENCIL + offsetIndex(di, dj)) * 9];
        bool nz = false;
        for (int q = 0; q < 9; ++q) {
          blk[q] = src[q];
          nz = nz || blk[q] != 0;
        }
        if (!nz) continue;
        for (int ka = 0; ka < 4; ++ka) {
          int I = P.idx[4 * a + ka];
          if (I < 0) continue;
          double wa = P.w[4 * a + ka];
          for (int kb = 0; kb < 4; ++kb) {
            int J = P.idx[4 * b + kb];
            if (J < 0) continue;
            double w = wa * P.w[4 * b + kb];
            int oi = C.ij[3 * J] - C.ij[3 * I], oj = C.ij[3 * J + 1] - C.ij[3 * I + 1];
            if (std::abs(oi) > 2 || std::abs(oj) > 2) throw std::runtime_error("Galerkin stencil exceeds radius 2");
            C.addBlock(I, offsetIndex(oi, oj), w, blk);
          }
        }
      }
  }
  for (int I = 0; I < C.N; ++I) {
    double* base = &C.A[(static_cast<size_t>(I) * STENCIL + CENTER) * 9];
    if (base[0] + base[4] + base[8] <= 0) {
      C.fixed[I] = 1;
      std::fill(&C.A[static_cast<size_t>(I) * STENCIL * 9], &C.A[static_cast<size_t>(I + 1) * STENCIL * 9], 0.0);
      base[0] = base[4] = base[8] = 1;
    }
  }
  return Cp;
}

// inv3 / pivotInv3 (newtonMultigrid.ts:391-423).
void inv3(const double* a, double* out) {
  double a00 = a[0], a01 = a[1], a02 = a[2], a10 = a[3], a11 = a[4], a12 = a[5], a20 = a[6], a21 = a[7], a22 = a[8];
  double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
  double det = a00 * c00 + a01 * c01 + a02 * c02;
  double id = 1 / det;
  out[0] = c00 * id;
  out[1] = (a02 * a21 - a01 * a22) * id;
  out[2] = (a01 * a12 - a02 * a11) * id;
  out[3] = c01 * id;
  out[4] = (a00 * a22 - a02 * a20) * id;
  out[5] = (a02 * a10 - a00 * a12) * id;
  out[6] = c02 * id;
  out[7] = (a01 * a20 - a00 * a21) * id;
  out[8] = (a00 * a11 - a01 * a10) * id;
}

// rotationOfSpring (assemble.wgsl:20-26): a rigid rotation w moves the ends of a term's vector d by
// w x d, which a spring block of transverse stiffness kPerp (or a scalar stencil k on d) resists with
// kPerp (|d|^2 I - d d^T).
static void addRotationOfSpring(double kPerp, const double* d, double* K) {
  const double l2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) K[3 * r + c] += kPerp * ((r == c ? l2 : 0.0) - d[r] * d[c]);
}

// The stiffness the internal terms a node of a detached piece owns put on a rigid rotation
// (assemble.wgsl:245, 255, 301): its span to the next node along each family (the span's transverse
// stiffness, its tension over its length), the bending triple centred on it, and the two shear
// diagonals it is the lower end of (of its own cell, and of the cell below, to that cell's +u corner).
void Solver::rigidRotation(std::vector<double>& kr) const {
  kr.assign(9 * static_cast<size_t>(N), 0.0);
  const double h = prm.h;
  auto pos = [&](int m, int z) { return x[3 * m + z] + dx[3 * m + z]; };
  for (int n = 0; n < N; ++n) {
    if (!inPiece(n) || pinned[n]) continue;
    double* K = &kr[9 * static_cast<size_t>(n)];
    for (int f = 0; f < 2; ++f) {
      const int prev = nbr[4 * n + 2 * f], next = nbr[4 * n + 2 * f + 1];
      const int s = 2 * n + f;
      if (next >= 0 && segActive(s)) {
        double e[3], l = 0;
        for (int z = 0; z < 3; ++z) e[z] = pos(next, z) - pos(n, z), l += e[z] * e[z];
        l = std::sqrt(l);
        const double L = restLength[s];
        double T, Kt;
        response(s, l / L - 1, &T, &Kt);
        const double fs = T + layer(n).yarns[f].axialViscosity / (L * h) * (l - segLength(s));
        addRotationOfSpring(std::max(fs, 0.0) / l, e, K);
      }
      if (prev >= 0 && next >= 0 && segActive(2 * prev + f) && segActive(s)) {
        double cf[5];
        bendCoeffs(n, f, 2 * prev + f, s, cf);
        const double kb = cf[0], fold = cf[2], wa = cf[3], wc = cf[4];
        double r[3], q2 = 0;
        for (int z = 0; z < 3; ++z) r[z] = wa * pos(prev, z) - 2 * pos(n, z) + wc * pos(next, z), q2 += r[z] * r[z];
        double ps[3];
        bendPsi(q2, fold, ps);
        const double k = kb * (ps[1] + 2 * ps[2] * q2) + (kb * layer(n).yarns[f].bendViscosity) / h;
        addRotationOfSpring(k, r, K);
      }
    }
    // shear diagonal 0 of cell n (n to its +u+v corner) and diagonal 1 of the cell below (its +u
    // corner to n)
    const int below = nbr[4 * n + 2];
    const int cells[2][2] = {{n, 0}, {below, 1}};
    for (auto& cd : cells) {
      const int c = cd[0];
      if (c < 0) continue;
      const int r = nbr[4 * c + 1], t = nbr[4 * c + 3];
      if (r < 0 || t < 0 || !diagActive(c, cd[1])) continue;
      const int other = cd[1] == 0 ? nbr[4 * r + 3] : r;
      double ks, jam, sl[3], e[3], l = 0;
      cellShear(c, &ks, &jam);
      const double Ld = std::sqrt(restLength[2 * c] * restLength[2 * c] + restLength[2 * c + 1] * restLength[2 * c + 1]);
      for (int z = 0; z < 3; ++z) e[z] = pos(other, z) - pos(n, z), l += e[z] * e[z];
      l = std::sqrt(l);
      shearLaw(ks, Ld, l, jam, sl);
      addRotationOfSpring(std::max(sl[0], 0.0) / l, e, K);
    }
  }
}

// rigidFrame (rigid_frame.wgsl:56-161): per piece its mass centroid at the iterate and E = Z^T K Z
// over its nodes' external blocks, plus their internal rotation stiffness on the rotation block; the
// rotation block regularised relative to its scale, then E^-1 through a Cholesky factor (zero when E
// is not positive definite).
void Solver::rigidFrame(const std::vector<double>& kx) {
  std::vector<double> kr;
  rigidRotation(kr);
  pieceFrame.assign(40 * static_cast<size_t>(pieceCount), 0.0);
  auto tri = [](int i, int j) { return i * 6 - (i * (i + 1)) / 2 + j; };
  for (int p = 0; p < pieceCount; ++p) {
    const uint32_t a = pieceStart[p], b = pieceStart[p + 1];
    double m[4] = {0, 0, 0, 0};
    for (uint32_t k = a; k < b; ++k) {
      const int n = static_cast<int>(pieceNodes[k]);
      for (int z = 0; z < 3; ++z) m[z] += mass[n] * (x[3 * n + z] + dx[3 * n + z]);
      m[3] += mass[n];
    }
    double c[3] = {0, 0, 0};
    if (m[3] > 0)
      for (int z = 0; z < 3; ++z) c[z] = m[z] / m[3];
    double e[21] = {0};
    for (uint32_t k = a; k < b; ++k) {
      const int n = static_cast<int>(pieceNodes[k]);
      const double* K = &kx[9 * static_cast<size_t>(n)];
      double r[3];
      for (int z = 0; z < 3; ++z) r[z] = x[3 * n + z] + dx[3 * n + z] - c[z];
      double Z[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
      for (int i = 0; i < 3; ++i) cross3(Z[i], r, Z[3 + i]);
      for (int i = 0; i < 6; ++i) {
        double KZ[3];
        for (int row = 0; row < 3; ++row) KZ[row] = K[3 * row] * Z[i][0] + K[3 * row + 1] * Z[i][1] + K[3 * row + 2] * Z[i][2];
        for (int j = i; j < 6; ++j) e[tri(i, j)] += Z[j][0] * KZ[0] + Z[j][1] * KZ[1] + Z[j][2] * KZ[2];
      }
      const double* R = &kr[9 * static_cast<size_t>(n)];
      for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) e[tri(3 + i, 3 + j)] += R[3 * i + j];
    }
    double* F = &pieceFrame[40 * static_cast<size_t>(p)];
    F[0] = c[0], F[1] = c[1], F[2] = c[2], F[3] = m[3] > 0 ? 1 : 0;
    const double st = (e[tri(0, 0)] + e[tri(1, 1)] + e[tri(2, 2)]) / 3;
    const double sr = (e[tri(3, 3)] + e[tri(4, 4)] + e[tri(5, 5)]) / 3;
    const double eps = 1e-6 * std::max(sr, 1e-8 * st) + 1e-30;
    double A6[6][6], Lc[6][6] = {{0}};
    for (int i = 0; i < 6; ++i) {
      for (int j = 0; j < 6; ++j) A6[i][j] = e[tri(std::min(i, j), std::max(i, j))];
      if (i >= 3) A6[i][i] += eps;
    }
    bool ok = st > 0;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j <= i; ++j) {
        double sum = A6[i][j];
        for (int k = 0; k < j; ++k) sum -= Lc[i][k] * Lc[j][k];
        if (i == j) {
          if (sum <= 0) ok = false, sum = 1;
          Lc[i][i] = std::sqrt(sum);
        } else {
          Lc[i][j] = sum / Lc[j][j];
        }
      }
    for (int col = 0; col < 6; ++col) {
      double y[6], z6[6];
      for (int i = 0; i < 6; ++i) {
        double sum = i == col ? 1 : 0;
        for (int k = 0; k < i; ++k) sum -= Lc[i][k] * y[k];
        y[i] = sum / Lc[i][i];
      }
      for (int i = 5; i >= 0; --i) {
        double sum = y[i];
        for (int k = i + 1; k < 6; ++k) sum -= Lc[k][i] * z6[k];
        z6[i] = sum / Lc[i][i];
      }
      for (int i = 0; i < 6; ++i) F[4 + 6 * i + col] = ok ? z6[i] : 0.0;
    }
  }
}

// rigidReduce / rigidApply (rigid_apply.wgsl:37-87): per piece the rhs force and torque about its
// centroid and its rigid step (t, w) = E^-1 (force, torque); x0 = t + w x r on its nodes, zero elsewhere.
void Solver::rigidStart(const double* b, double* x0) {
  pieceStep.assign(6 * static_cast<size_t>(pieceCount), 0.0);
  for (int p = 0; p < pieceCount; ++p) {
    const double* F = &pieceFrame[40 * static_cast<size_t>(p)];
    double g[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t k = pieceStart[p]; k < pieceStart[p + 1]; ++k) {
      const int n = static_cast<int>(pieceNodes[k]);
      double r[3], t[3];
      for (int z = 0; z < 3; ++z) r[z] = x[3 * n + z] + dx[3 * n + z] - F[z], g[z] += b[3 * n + z];
      cross3(r, &b[3 * n], t);
      for (int z = 0; z < 3; ++z) g[3 + z] += t[z];
    }
    for (int i = 0; i < 6; ++i) {
      double sum = 0;
      for (int j = 0; j < 6; ++j) sum += F[4 + 6 * i + j] * g[j];
      pieceStep[6 * p + i] = F[3] > 0.5 ? sum : 0.0;
    }
  }
  for (int n = 0; n < N; ++n) {
    if (!inPiece(n)) continue;
    const int p = static_cast<int>(pieceOf[n]);
    const double* F = &pieceFrame[40 * static_cast<size_t>(p)];
    const double* q = &pieceStep[6 * p];
    double r[3], wr[3];
    for (int z = 0; z < 3; ++z) r[z] = x[3 * n + z] + dx[3 * n + z] - F[z];
    cross3(q + 3, r, wr);
    for (int z = 0; z < 3; ++z) x0[3 * n + z] = q[z] + wr[z];
  }
}

// curveSet (rigid_spin.wgsl:138-154): per node of a piece with a valid frame, the rotation of the
// direction's rigid start and the node's arm from the centroid at the iterate.
void Solver::curveSet() {
  curveOn.assign(N, 0);
  curveW.assign(3 * static_cast<size_t>(N), 0.0);
  curveR.assign(3 * static_cast<size_t>(N), 0.0);
  for (int n = 0; n < N; ++n) {
    if (!inPiece(n)) continue;
    const int p = static_cast<int>(pieceOf[n]);
    const double* F = &pieceFrame[40 * static_cast<size_t>(p)];
    if (!(F[3] > 0.5)) continue;
    curveOn[n] = 1;
    for (int z = 0; z < 3; ++z) {
      curveW[3 * n + z] = pieceStep[6 * p + 3 + z];
      curveR[3 * n + z] = x[3 * n + z] + dx[3 * n + z] - F[z];
    }
  }
}

// spinReduce / spinApply (rigid_spin.wgsl:44-136): a piece's rotation over the last substep, from its
// angular momentum about its centroid (w = I^-1 L, regularised as the rigid frame), continued over
// this one: the start moves by (R + R^T - 2 I) r = -2 (1 - cos th) r_perp about the centroid.
void Solver::spinStart() {
  pieceStep.assign(6 * static_cast<size_t>(pieceCount), 0.0);
  for (int p = 0; p < pieceCount; ++p) {
    const uint32_t a = pieceStart[p], b = pieceStart[p + 1];
    double M = 0, mx[3] = {0, 0, 0}, mv[3] = {0, 0, 0};
    for (uint32_t k = a; k < b; ++k) {
      const int n = static_cast<int>(pieceNodes[k]);
      M += mass[n];
      for (int z = 0; z < 3; ++z) mx[z] += mass[n] * x[3 * n + z], mv[z] += mass[n] * v[3 * n + z];
    }
    double c[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
    if (M > 0)
      for (int z = 0; z < 3; ++z) c[z] = mx[z] / M, vc[z] = mv[z] / M;
    double L[3] = {0, 0, 0}, I[6] = {0, 0, 0, 0, 0, 0};  // xx yy zz xy xz yz
    for (uint32_t k = a; k < b; ++k) {
      const int n = static_cast<int>(pieceNodes[k]);
      const double m = mass[n];
      double r[3], u[3], t[3];
      for (int z = 0; z < 3; ++z) r[z] = x[3 * n + z] - c[z], u[z] = v[3 * n + z] - vc[z];
      cross3(r, u, t);
      for (int z = 0; z < 3; ++z) L[z] += m * t[z];
      const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      I[0] += m * (rr - r[0] * r[0]);
      I[1] += m * (rr - r[1] * r[1]);
      I[2] += m * (rr - r[2] * r[2]);
      I[3] -= m * r[0] * r[1];
      I[4] -= m * r[0] * r[2];
      I[5] -= m * r[1] * r[2];
    }
    const double eps = 1e-6 * (I[0] + I[1] + I[2]) / 3 + 1e-30;
    const double T[9] = {I[0] + eps, I[3], I[4], I[3], I[1] + eps, I[5], I[4], I[5], I[2] + eps};
    double Ti[9], th[3];
    inv3(T, Ti);
    for (int z = 0; z < 3; ++z) th[z] = (Ti[3 * z] * L[0] + Ti[3 * z + 1] * L[1] + Ti[3 * z + 2] * L[2]) * prm.h;
    if (!(M > 0) || !std::isfinite(th[0]) || !std::isfinite(th[1]) || !std::isfinite(th[2])) th[0] = th[1] = th[2] = 0;
    for (int z = 0; z < 3; ++z) pieceStep[6 * p + z] = c[z], pieceStep[6 * p + 3 + z] = th[z];
  }
  for (int n = 0; n < N; ++n) {
    if (!inPiece(n) || pinned[n]) continue;
    const double* q = &pieceStep[6 * static_cast<size_t>(pieceOf[n])];
    const double phi = hyp3(q[3], q[4], q[5]);
    if (phi < 1e-9) continue;
    const double k[3] = {q[3] / phi, q[4] / phi, q[5] / phi};
    double r[3], kr[3], kkr[3];
    for (int z = 0; z < 3; ++z) r[z] = x[3 * n + z] - q[z];
    cross3(k, r, kr);
    cross3(k, kr, kkr);
    for (int z = 0; z < 3; ++z) dx[3 * n + z] += 2 * (1 - std::cos(phi)) * kkr[z];
  }
}
void pivotInv3(const double* a, double* out, double shift) {
  double e = shift * std::max(std::max(std::fabs(a[0]), std::fabs(a[4])), std::fabs(a[8]));
  double sh[9];
  for (int q = 0; q < 9; ++q) sh[q] = a[q];
  sh[0] += e;
  sh[4] += e;
  sh[8] += e;
  inv3(sh, out);
}
void mul3(const double* a, const double* b, double* out) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[r * 3 + c] = a[r * 3] * b[c] + a[r * 3 + 1] * b[3 + c] + a[r * 3 + 2] * b[6 + c];
}

// solvePenta (newtonMultigrid.ts:435-473).
void solvePenta(int n, const double* D, const double* E, const double* F, const double* r, double* x, double shift) {
  std::vector<double> Dk(D, D + 9 * n), U1(E, E + 9 * n), L1(9 * static_cast<size_t>(n), 0.0), rk(r, r + 3 * n);
  for (int k = 1; k < n; ++k)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) L1[9 * k + a * 3 + b] = E[9 * (k - 1) + b * 3 + a];
  double inv[9], Lm[9], t[9], Amk[9];
  for (int k = 0; k < n; ++k) {
    pivotInv3(&Dk[9 * k], inv, shift);
    for (int m = k + 1; m <= k + 2 && m < n; ++m) {
      if (m == k + 1)
        std::memcpy(Amk, &L1[9 * m], sizeof Amk);
      else
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) Amk[a * 3 + b] = F[9 * k + b * 3 + a];
      mul3(Amk, inv, Lm);
      if (k + 1 < n) {
        mul3(Lm, &U1[9 * k], t);
        double* dst = m == k + 1 ? Dk.data() : L1.data();
        for (int q = 0; q < 9; ++q) dst[9 * m + q] -= t[q];
      }
      if (k + 2 < n) {
        mul3(Lm, &F[9 * k], t);
        double* dst = m == k + 1 ? U1.data() : Dk.data();
        for (int q = 0; q < 9; ++q) dst[9 * m + q] -= t[q];
      }
      for (int q = 0; q < 3; ++q) rk[3 * m + q] -= Lm[q * 3] * rk[3 * k] + Lm[q * 3 + 1] * rk[3 * k + 1] + Lm[q * 3 + 2] * rk[3 * k + 2];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    double b0[3] = {rk[3 * k], rk[3 * k + 1], rk[3 * k + 2]};
    for (int q = 0; q < 3; ++q) {
      if (k + 1 < n) b0[q] -= U1[9 * k + q * 3] * x[3 * (k + 1)] + U1[9 * k + q * 3 + 1] * x[3 * (k + 1) + 1] + U1[9 * k + q * 3 + 2] * x[3 * (k + 1) + 2];
      if (k + 2 < n) b0[q] -= F[9 * k + q * 3] * x[3 * (k + 2)] + F[9 * k + q * 3 + 1] * x[3 * (k + 2) + 1] + F[9 * k + q * 3 + 2] * x[3 * (k + 2) + 2];
    }
    pivotInv3(&Dk[9 * k], inv, shift);
    for (int q = 0; q < 3; ++q) x[3 * k + q] = inv[q * 3] * b0[0] + inv[q * 3 + 1] * b0[1] + inv[q * 3 + 2] * b0[2];
  }
}

// smoothLines (newtonMultigrid.ts:659-733).
void smoothLines(const StencilOperator& A, double* x, const double* b, bool reverse, int colors) {
  int maxLen = 0;
  for (auto& L : A.layers) maxLen = std::max(maxLen, std::max(L.nx, L.ny));
  std::vector<std::pair<int, int>> order;
  for (int family : {1, 0})
    for (int c = 0; c < colors; ++c) order.push_back({family, c});
  if (reverse) std::reverse(order.begin(), order.end());
  std::vector<double> xOld(3 * static_cast<size_t>(A.N));
  for (auto& fc : order) {
    int family = fc.first, color = fc.second;
    std::copy(x, x + 3 * static_cast<size_t>(A.N), xOld.begin());
    for (const LatticeLayer& L : A.layers) {
      int lines = family == 0 ? L.ny : L.nx;
      int len = family == 0 ? L.nx : L.ny;
      int nlines = lines > color ? (lines - color + colors - 1) / colors : 0;
#pragma omp parallel
      {
        std::vector<double> D(9 * static_cast<size_t>(maxLen)), E(D.size()), F(D.size()), r(3 * static_cast<size_t>(maxLen)),
            sol(r.size());
#pragma omp for schedule(dynamic, 1)
        for (int li = 0; li < nlines; ++li) {
          int line = color + li * colors;
          auto node = [&](int k) { return family == 0 ? L.offset + line * L.nx + k : L.offset + k * L.nx + line; };
          std::fill(D.begin(), D.begin() + 9 * len, 0.0);
          std::fill(E.begin(), E.begin() + 9 * len, 0.0);
          for (int k = 0; k < len; ++k) {
            int n = node(k);
            r[3 * k] = b[3 * n];
            r[3 * k + 1] = b[3 * n + 1];
            r[3 * k + 2] = b[3 * n + 2];
            if (A.fixed[n]) {
              D[9 * k] = D[9 * k + 4] = D[9 * k + 8] = 1;
              continue;
            }
            double maj = 0;
            for (int dj = -2; dj <= 2; ++dj)
              for (int di = -2; di <= 2; ++di) {
                int m = A.nbr(n, di, dj);
                if (m < 0 || (A.fixed[m] && !(di == 0 && dj == 0))) continue;
                const double* B = &A.A[(static_cast<size_t>(n) * STENCIL + offsetIndex(di, dj)) * 9];
                int along = family == 0 ? di : dj, across = family == 0 ? dj : di;
                if (across == 0 && along == 0) {
                  for (int q = 0; q < 9; ++q) D[9 * k + q] += B[q];
                  continue;
                }
                if (across == 0 && along == 1) {
                  for (int q = 0; q < 9; ++q) E[9 * k + q] = B[q];
                  continue;
                }
                if (across == 0 && along == -1) continue;
                if (across == 0 || std::abs(across) == colors) {
                  double s = 0;
                  for (int q = 0; q < 9; ++q) s += B[q] * B[q];
                  maj += std::sqrt(s);
                }
                double x0 = xOld[3 * m], x1 = xOld[3 * m + 1], x2 = xOld[3 * m + 2];
                r[3 * k] -= B[0] * x0 + B[1] * x1 + B[2] * x2;
                r[3 * k + 1] -= B[3] * x0 + B[4] * x1 + B[5] * x2;
                r[3 * k + 2] -= B[6] * x0 + B[7] * x1 + B[8] * x2;
              }
            D[9 * k] += maj;
            D[9 * k + 4] += maj;
            D[9 * k + 8] += maj;
            r[3 * k] += maj * xOld[3 * n];
            r[3 * k + 1] += maj * xOld[3 * n + 1];
            r[3 * k + 2] += maj * xOld[3 * n + 2];
          }
          std::fill(F.begin(), F.begin() + 9 * len, 0.0);
          solvePenta(len, D.data(), E.data(), F.data(), r.data(), sol.data(), PIVOT_SHIFT);
          for (int k = 0; k < len; ++k) {
            int n = node(k);
            if (A.fixed[n]) continue;
            x[3 * n] = sol[3 * k];
            x[3 * n + 1] = sol[3 * k + 1];
            x[3 * n + 2] = sol[3 * k + 2];
          }
        }
      }
    }
  }
}

// Precision study: the operator as float32 storage would hold it (ora_params.fp32_rows).
void roundRows(StencilOperator& A, int mode) {
  if (mode == 0) return;
  auto rnd = [](double v) { return static_cast<double>(static_cast<float>(v)); };
  for (int n = 0; n < A.N; ++n) {
    double* row = &A.A[static_cast<size_t>(n) * STENCIL * 9];
    if (mode == 1) {
      for (int q = 0; q < STENCIL * 9; ++q) row[q] = rnd(row[q]);
      continue;
    }
    double sum[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int o = 0; o < STENCIL; ++o)
      for (int q = 0; q < 9; ++q) sum[q] += row[9 * o + q];
    for (int q = 0; q < 9; ++q) sum[q] = rnd(sum[q]);
    for (int o = 0; o < STENCIL; ++o) {
      if (o == CENTER) continue;
      for (int q = 0; q < 9; ++q) {
        row[9 * o + q] = rnd(row[9 * o + q]);
        sum[q] -= row[9 * o + q];
      }
    }
    for (int q = 0; q < 9; ++q) row[9 * CENTER + q] = sum[q];
  }
}

// buildHierarchy (newtonMultigrid.ts:480-491).
std::vector<MGLevel> Solver::buildHierarchy(std::shared_ptr<StencilOperator> fine) const {
  std::vector<MGLevel> levels;
  levels.push_back({fine, nullptr});
  std::shared_ptr<StencilOperator> cur = fine;
  while (cur->N > prm.max_coarsest_nodes && shouldCoarsen(cur->layers)) {
    std::vector<LatticeLayer> coarse;
    auto P = buildProlongation(*cur, &coarse);
    auto C = galerkin(*cur, coarse, *P);
    roundRows(*C, prm.fp32_rows / 10);
    if (prm.coarse_bf16)  // precision study: the coarse rows as BF16 storage would hold them
      for (size_t q = 0; q < C->A.size(); ++q) {
        // 2: the 24 coupling blocks only, the diagonal block kept
        if (prm.coarse_bf16 == 2 && (q / 9) % STENCIL == CENTER) continue;
        double& v = C->A[q];
        float f = static_cast<float>(v);
        uint32_t u;
        std::memcpy(&u, &f, 4);
        u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
        std::memcpy(&f, &u, 4);
        v = f;
      }
    levels.back().P = P;
    levels.push_back({C, nullptr});
    cur = C;
  }
  return levels;
}

// vcycle (newtonMultigrid.ts:495-528).
void Solver::vcycle(const std::vector<MGLevel>& levels, int k, double* x, const double* b) const {
  const StencilOperator& A = *levels[k].A;
  int colors = prm.line_colors;
  if (!levels[k].P) {
    if (lc.active || lc.log) {
      // the learned coarse space (extension) half-way through the sweeps, which mirror around it
      const int half = prm.coarse_sweeps / 2;
      for (int s = 0; s < half; ++s) smoothLines(A, x, b, (s & 1) == 1, colors);
      learnedCorrection(levels, k, x, b);
      for (int s = half; s < prm.coarse_sweeps; ++s) smoothLines(A, x, b, (s & 1) == 1, colors);
      return;
    }
    for (int s = 0; s < prm.coarse_sweeps; ++s) smoothLines(A, x, b, (s & 1) == 1, colors);
    return;
  }
  const Prolongation& P = *levels[k].P;
  smoothLines(A, x, b, false, colors);
  std::vector<double> Ax(3 * static_cast<size_t>(A.N));
  A.apply(x, Ax.data());
  const StencilOperator& C = *levels[k + 1].A;
  std::vector<double> rc(3 * static_cast<size_t>(C.N), 0.0);
  for (int f = 0; f < A.N; ++f) {
    if (A.fixed[f]) continue;
    for (int kk = 0; kk < 4; ++kk) {
      int c = P.idx[4 * f + kk];
      if (c < 0) continue;
      double w = P.w[4 * f + kk];
      for (int q = 0; q < 3; ++q) rc[3 * c + q] += w * (b[3 * f + q] - Ax[3 * f + q]);
    }
  }
  for (int c = 0; c < C.N; ++c)
    if (C.fixed[c]) rc[3 * c] = rc[3 * c + 1] = rc[3 * c + 2] = 0;
  std::vector<double> xc(3 * static_cast<size_t>(C.N), 0.0);
  vcycle(levels, k + 1, xc.data(), rc.data());
  for (int f = 0; f < A.N; ++f) {
    if (A.fixed[f]) continue;
    for (int kk = 0; kk < 4; ++kk) {
      int c = P.idx[4 * f + kk];
      if (c < 0) continue;
      double w = P.w[4 * f + kk];
      for (int q = 0; q < 3; ++q) x[3 * f + q] += w * xc[3 * c + q];
    }
  }
  smoothLines(A, x, b, true, colors);
}

// Lower Cholesky factor of a symmetric 3 x 3 block; false unless positive definite.
static bool chol3(const double* D, double* L) {
  double a = D[0];
  if (!(a > 0)) return false;
  L[0] = std::sqrt(a);
  L[1] = L[2] = L[5] = 0;
  L[3] = D[3] / L[0];
  L[6] = D[6] / L[0];
  double c = D[4] - L[3] * L[3];
  if (!(c > 0)) return false;
  L[4] = std::sqrt(c);
  L[7] = (D[7] - L[6] * L[3]) / L[4];
  double e = D[8] - L[6] * L[6] - L[7] * L[7];
  if (!(e > 0)) return false;
  L[8] = std::sqrt(e);
  return true;
}

// Damage and contact flags of the coarsest nodes: on the fine lattice a node is damaged when a span at it
// exists but is broken or not fully intact, in contact when contact terms act on it; a coarse node takes
// the maximum over the fine nodes its prolongation weights reach.
void Solver::learnedFlags(const std::vector<MGLevel>& levels) const {
  const int F = levels[0].A->N;
  std::vector<float> f(2 * static_cast<size_t>(F), 0.f);
  if (F == N) {
    bool ct = contactOn && extH.size() == 6 * static_cast<size_t>(N);
    for (int n = 0; n < N; ++n) {
      for (int fam = 0; fam < 2; ++fam)
        for (int dir = -1; dir <= 1; dir += 2) {
          int s = seg(n, fam, dir);
          if (s >= 0 && (segFlags[s] & SEG_EXISTS) && ((segFlags[s] & SEG_BROKEN) || intact[s] < 1)) f[2 * n] = 1;
        }
      if (ct)
        for (int z = 0; z < 6; ++z)
          if (extH[6 * n + z] != 0) f[2 * n + 1] = 1;
    }
  }
  for (size_t k = 0; k + 1 < levels.size(); ++k) {
    const Prolongation& P = *levels[k].P;
    const int Fk = levels[k].A->N, Ck = levels[k + 1].A->N;
    std::vector<float> c(2 * static_cast<size_t>(Ck), 0.f);
    for (int n = 0; n < Fk; ++n)
      for (int q = 0; q < 4; ++q) {
        int m = P.idx[4 * n + q];
        if (m < 0 || !(P.w[4 * n + q] > 0)) continue;
        c[2 * m] = std::max(c[2 * m], f[2 * n]);
        c[2 * m + 1] = std::max(c[2 * m + 1], f[2 * n + 1]);
      }
    f.swap(c);
  }
  lc.flags.swap(f);
}

// The network inputs of every coarsest node (see LearnedCoarse) with the Cholesky factors of the
// diagonal blocks; ok marks the free nodes whose block is positive definite.
bool Solver::learnedInputs(const StencilOperator& A, std::vector<double>& L, std::vector<uint8_t>& ok,
                           std::vector<double>& X) const {
  const int M = A.N;
  L.assign(9 * static_cast<size_t>(M), 0.0);
  ok.assign(M, 0);
  X.assign(static_cast<size_t>(M) * LC_IN, 0.0);
  std::vector<double> tr(M, 0.0);
  double trSum = 0;
  int nOk = 0;
  for (int n = 0; n < M; ++n) {
    if (A.fixed[n]) continue;
    const double* D = &A.A[(static_cast<size_t>(n) * STENCIL + CENTER) * 9];
    if (!chol3(D, &L[9 * static_cast<size_t>(n)])) continue;
    ok[n] = 1;
    tr[n] = D[0] + D[4] + D[8];
    trSum += tr[n];
    nOk++;
  }
  if (!nOk) return false;
  const double trMean = trSum / nOk, PI = 3.14159265358979323846;
  const bool haveFlags = lc.flags.size() == 2 * static_cast<size_t>(M);
  for (int n = 0; n < M; ++n) {
    if (!ok[n]) continue;
    double* in = &X[static_cast<size_t>(n) * LC_IN];
    const LatticeLayer& Ly = A.layers[A.ij[3 * n + 2]];
    double u = Ly.nx > 1 ? static_cast<double>(A.ij[3 * n]) / (Ly.nx - 1) : 0.0;
    double v = Ly.ny > 1 ? static_cast<double>(A.ij[3 * n + 1]) / (Ly.ny - 1) : 0.0;
    int q = 0;
    in[q++] = u;
    in[q++] = v;
    for (int f = 1; f <= 2; ++f) {
      in[q++] = std::sin(f * PI * u);
      in[q++] = std::cos(f * PI * u);
      in[q++] = std::sin(f * PI * v);
      in[q++] = std::cos(f * PI * v);
    }
    const double* D = &A.A[(static_cast<size_t>(n) * STENCIL + CENTER) * 9];
    in[q++] = D[0] / tr[n];
    in[q++] = D[4] / tr[n];
    in[q++] = D[8] / tr[n];
    in[q++] = D[1] / tr[n];
    in[q++] = D[2] / tr[n];
    in[q++] = D[5] / tr[n];
    in[q++] = std::log(tr[n] / trMean);
    int held = 0;
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        if (!di && !dj) continue;
        int m = A.nbr(n, di, dj);
        if (m < 0 || A.fixed[m]) held++;
      }
    in[q++] = held / 8.0;
    in[q++] = haveFlags ? lc.flags[2 * n] : 0.0;
    in[q++] = haveFlags ? lc.flags[2 * n + 1] : 0.0;
  }
  return true;
}

// The basis of this solve on the coarsest level: Phi = L^-T Psi from the network, A Phi, and the
// Cholesky factor of G = Phi^T A Phi; a column whose pivot falls below 1e-10 of the largest diagonal
// entry (dependent on the others) is dropped.
void Solver::learnedBasis(const std::vector<MGLevel>& levels) const {
  lc.basisOp = nullptr;
  const StencilOperator& A = *levels.back().A;
  const int M = A.N;
  std::vector<double> L, X;
  std::vector<uint8_t> ok;
  if (!learnedInputs(A, L, ok, X)) return;
  const size_t n3 = 3 * static_cast<size_t>(M);
  lc.phi.assign(n3 * LC_K, 0.0);
#pragma omp parallel for schedule(static)
  for (int n = 0; n < M; ++n) {
    if (!ok[n]) continue;
    double o[LC_OUT];
    lcForward(lc.w.data(), &X[static_cast<size_t>(n) * LC_IN], o);
    const double* Ln = &L[9 * static_cast<size_t>(n)];
    for (int k = 0; k < LC_K; ++k) {  // L^T phi = psi
      double p2 = o[3 * k + 2] / Ln[8];
      double p1 = (o[3 * k + 1] - Ln[7] * p2) / Ln[4];
      double p0 = (o[3 * k] - Ln[3] * p1 - Ln[6] * p2) / Ln[0];
      lc.phi[(3 * static_cast<size_t>(n)) * LC_K + k] = p0;
      lc.phi[(3 * static_cast<size_t>(n) + 1) * LC_K + k] = p1;
      lc.phi[(3 * static_cast<size_t>(n) + 2) * LC_K + k] = p2;
    }
  }
  std::vector<double> col(n3), Acol(n3), G(LC_K * LC_K, 0.0);
  std::vector<std::vector<double>> AP(LC_K);
  for (int k = 0; k < LC_K; ++k) {
    for (size_t q = 0; q < n3; ++q) col[q] = lc.phi[q * LC_K + k];
    A.apply(col.data(), Acol.data());
    for (int n = 0; n < M; ++n)
      if (A.fixed[n]) Acol[3 * n] = Acol[3 * n + 1] = Acol[3 * n + 2] = 0;
    AP[k] = Acol;
  }
  for (int a = 0; a < LC_K; ++a)
    for (int c = 0; c < LC_K; ++c) {
      double s = 0;
      for (size_t q = 0; q < n3; ++q) s += lc.phi[q * LC_K + a] * AP[c][q];
      G[a * LC_K + c] = s;
    }
  for (int a = 0; a < LC_K; ++a)  // symmetrise
    for (int c = 0; c < a; ++c) G[a * LC_K + c] = G[c * LC_K + a] = 0.5 * (G[a * LC_K + c] + G[c * LC_K + a]);
  double gmax = 0;
  for (int a = 0; a < LC_K; ++a) gmax = std::max(gmax, G[a * LC_K + a]);
  if (!(gmax > 0) || !std::isfinite(gmax)) return;
  lc.dead.assign(LC_K, 0);
  for (int j = 0; j < LC_K; ++j) {
    double d = G[j * LC_K + j];
    for (int q = 0; q < j; ++q) d -= G[j * LC_K + q] * G[j * LC_K + q];
    if (!(d > 1e-10 * gmax)) {
      lc.dead[j] = 1;
      for (int i = j; i < LC_K; ++i) G[i * LC_K + j] = 0;
      G[j * LC_K + j] = 1;
      continue;
    }
    d = std::sqrt(d);
    G[j * LC_K + j] = d;
    for (int i = j + 1; i < LC_K; ++i) {
      double v = G[i * LC_K + j];
      for (int q = 0; q < j; ++q) v -= G[i * LC_K + q] * G[j * LC_K + q];
      G[i * LC_K + j] = v / d;
    }
  }
  lc.G = G;
  lc.basisOp = &A;
}

// The learned coarse space on the coarsest level k, half-way through its sweeps (see LearnedCoarse):
// logs the training material when logging, adds the Galerkin correction on the basis when active.
void Solver::learnedCorrection(const std::vector<MGLevel>& levels, int k, double* x, const double* b) const {
  const StencilOperator& A = *levels[k].A;
  const int M = A.N;
  const size_t n3 = 3 * static_cast<size_t>(M);
  std::vector<double> r(n3);
  A.apply(x, r.data());
  for (int n = 0; n < M; ++n)
    for (int q = 0; q < 3; ++q) r[3 * n + q] = A.fixed[n] ? 0.0 : b[3 * n + q] - r[3 * n + q];

  if (lc.log && lc.calls.size() < lc.logCap) {
    if (lc.denseOp.get() != &A) {  // a new coarsest operator: dense whitened copy and its factor
      lc.denseOp = levels[k].A;
      std::vector<double> X;
      std::vector<uint8_t> ok;
      lc.denseOk = learnedInputs(A, lc.nodeL, ok, X);
      lc.denseFree.assign(M, -1);
      int nf = 0;
      for (int n = 0; n < M; ++n) {
        if (A.fixed[n]) continue;
        if (!ok[n]) lc.denseOk = false;
        lc.denseFree[n] = nf++;
      }
      const size_t D3 = 3 * static_cast<size_t>(nf);
      lc.denseDim = D3;
      lc.denseOk = lc.denseOk && nf > 0 && D3 <= 6000;
      lc.denseL.assign(lc.denseOk ? D3 * D3 : 0, 0.0);
      if (lc.denseOk) {
        double* Dm = lc.denseL.data();
        const double* NL = lc.nodeL.data();
        // whitened blocks L_n^-1 B L_m^-T
        for (int n = 0; n < M; ++n) {
          int a = lc.denseFree[n];
          if (a < 0) continue;
          for (int dj = -2; dj <= 2; ++dj)
            for (int di = -2; di <= 2; ++di) {
              int m = A.nbr(n, di, dj);
              if (m < 0 || lc.denseFree[m] < 0) continue;
              const double* B = &A.A[(static_cast<size_t>(n) * STENCIL + offsetIndex(di, dj)) * 9];
              const double *Ln = &NL[9 * static_cast<size_t>(n)], *Lm = &NL[9 * static_cast<size_t>(m)];
              double T[9], W[9];
              for (int c = 0; c < 3; ++c) {  // T = L_n^-1 B, column c
                T[c] = B[c] / Ln[0];
                T[3 + c] = (B[3 + c] - Ln[3] * T[c]) / Ln[4];
                T[6 + c] = (B[6 + c] - Ln[6] * T[c] - Ln[7] * T[3 + c]) / Ln[8];
              }
              for (int rr = 0; rr < 3; ++rr) {  // W = T L_m^-T: row rr solves L_m w = T[rr]
                W[3 * rr] = T[3 * rr] / Lm[0];
                W[3 * rr + 1] = (T[3 * rr + 1] - Lm[3] * W[3 * rr]) / Lm[4];
                W[3 * rr + 2] = (T[3 * rr + 2] - Lm[6] * W[3 * rr] - Lm[7] * W[3 * rr + 1]) / Lm[8];
              }
              for (int rr = 0; rr < 3; ++rr)
                for (int cc = 0; cc < 3; ++cc) Dm[(3 * a + rr) * D3 + 3 * lc.denseFree[m] + cc] = W[3 * rr + cc];
            }
        }
        LearnedOp op;
        op.nodes = nf;
        op.At.assign(Dm, Dm + D3 * D3);
        for (int n = 0; n < M; ++n)
          if (lc.denseFree[n] >= 0) op.X.insert(op.X.end(), &X[static_cast<size_t>(n) * LC_IN], &X[static_cast<size_t>(n + 1) * LC_IN]);
        lc.ops.push_back(std::move(op));
        for (size_t j = 0; j < D3 && lc.denseOk; ++j) {  // in-place lower Cholesky of the whitened operator
          double d = Dm[j * D3 + j];
          for (size_t q = 0; q < j; ++q) d -= Dm[j * D3 + q] * Dm[j * D3 + q];
          if (!(d > 0)) {
            lc.denseOk = false;
            lc.ops.pop_back();
            break;
          }
          d = std::sqrt(d);
          Dm[j * D3 + j] = d;
#pragma omp parallel for schedule(static)
          for (size_t i = j + 1; i < D3; ++i) {
            double v = Dm[i * D3 + j];
            for (size_t q = 0; q < j; ++q) v -= Dm[i * D3 + q] * Dm[j * D3 + q];
            Dm[i * D3 + j] = v / d;
          }
        }
      }
    }
    if (lc.denseOk) {
      const size_t D3 = lc.denseDim;
      const double* Dm = lc.denseL.data();
      LearnedCall call;
      call.op = static_cast<int>(lc.ops.size()) - 1;
      call.r.assign(D3, 0.0);
      for (int n = 0; n < M; ++n) {
        int a = lc.denseFree[n];
        if (a < 0) continue;
        const double* Ln = &lc.nodeL[9 * static_cast<size_t>(n)];
        const double* rn = &r[3 * n];
        double* g = &call.r[3 * a];
        g[0] = rn[0] / Ln[0];
        g[1] = (rn[1] - Ln[3] * g[0]) / Ln[4];
        g[2] = (rn[2] - Ln[6] * g[0] - Ln[7] * g[1]) / Ln[8];
      }
      std::vector<double> d(call.r);
      for (size_t i = 0; i < D3; ++i) {
        double v = d[i];
        for (size_t q = 0; q < i; ++q) v -= Dm[i * D3 + q] * d[q];
        d[i] = v / Dm[i * D3 + i];
      }
      for (size_t i = D3; i-- > 0;) {
        double v = d[i];
        for (size_t q = i + 1; q < D3; ++q) v -= Dm[q * D3 + i] * d[q];
        d[i] = v / Dm[i * D3 + i];
      }
      call.d = std::move(d);
      lc.calls.push_back(std::move(call));
    }
  }
  if (!lc.active || lc.basisOp != &A) return;

  double u[LC_K], c[LC_K];
  for (int a = 0; a < LC_K; ++a) {
    double s = 0;
    for (size_t q = 0; q < n3; ++q) s += lc.phi[q * LC_K + a] * r[q];
    u[a] = lc.dead[a] ? 0.0 : s;
  }
  for (int i = 0; i < LC_K; ++i) {  // G c = u with G = R R^T (R lower)
    double v = u[i];
    for (int q = 0; q < i; ++q) v -= lc.G[i * LC_K + q] * c[q];
    c[i] = lc.dead[i] ? 0.0 : v / lc.G[i * LC_K + i];
  }
  for (int i = LC_K; i-- > 0;) {
    double v = c[i];
    for (int q = i + 1; q < LC_K; ++q) v -= lc.G[q * LC_K + i] * c[q];
    c[i] = lc.dead[i] ? 0.0 : v / lc.G[i * LC_K + i];
  }
  for (size_t q = 0; q < n3; ++q) {
    double s = 0;
    for (int a = 0; a < LC_K; ++a) s += lc.phi[q * LC_K + a] * c[a];
    x[q] += s;
  }
  lc.applied++;
}

// Deterministic dot product: fixed 64 chunks summed in order, independent of the thread count.
double dotv(const double* a, const double* b, size_t n) {
  const int CH = 64;
  double part[CH];
#pragma omp parallel for schedule(static)
  for (int c = 0; c < CH; ++c) {
    size_t lo = n * c / CH, hi = n * (c + 1) / CH;
    double s = 0;
    for (size_t q = lo; q < hi; ++q) s += a[q] * b[q];
    part[c] = s;
  }
  double s = 0;
  for (int c = 0; c < CH; ++c) s += part[c];
  return s;
}

// pcg (newtonMultigrid.ts:537-576) with the relative-residual stop (extension).
void Solver::pcg(const std::vector<MGLevel>& levels, const double* b, double* x, int iterations, double tol, int* done,
                 double* relOut) const {
  const StencilOperator& A = pcgOp ? *pcgOp : *levels[0].A;
  size_t n = 3 * static_cast<size_t>(A.N);
  std::vector<double> r(n), Ap(n), z(n, 0.0), p(n);
  A.apply(x, Ap.data());
  for (size_t q = 0; q < n; ++q) r[q] = b[q] - Ap[q];
  for (int m = 0; m < A.N; ++m)
    if (A.fixed[m]) r[3 * m] = r[3 * m + 1] = r[3 * m + 2] = 0;
  double r0 = std::sqrt(dotv(r.data(), r.data(), n));
  double rel = 1;
  int it = 0;
  if (tol > 0 && !(r0 > 0)) {
    if (done) *done = 0;
    if (relOut) *relOut = 0;
    return;
  }
  // learned coarse correction (extension): on for this solve until the guard trips
  lc.active = lc.on && lc.w.size() == static_cast<size_t>(LC_WEIGHTS);
  if (lc.active || lc.log) learnedFlags(levels);
  if (lc.active) {
    lc.solves++;
    learnedBasis(levels);
  }
  vcycle(levels, 0, z.data(), r.data());
  p = z;
  double rz = dotv(r.data(), z.data(), n);
  for (it = 0; it < iterations; ++it) {
    A.apply(p.data(), Ap.data());
    for (int m = 0; m < A.N; ++m)
      if (A.fixed[m]) Ap[3 * m] = Ap[3 * m + 1] = Ap[3 * m + 2] = 0;
    double pAp = dotv(p.data(), Ap.data(), n);
    if (!(pAp > 0)) break;
    double alpha = rz / pAp;
    for (size_t q = 0; q < n; ++q) {
      x[q] += alpha * p[q];
      r[q] -= alpha * Ap[q];
    }
    if (tol > 0) {
      rel = std::sqrt(dotv(r.data(), r.data(), n)) / r0;
      if (rel <= tol) {
        it++;
        break;
      }
    }
    if (it + 1 == iterations) {
      it++;
      break;
    }
    // guard: mean contraction per iteration above lc.guard after three iterations -> plain V-cycle,
    // PCG restarted from the current iterate
    bool restart = false;
    if (lc.active && it + 1 >= 3) {
      double relNow = tol > 0 ? rel : std::sqrt(dotv(r.data(), r.data(), n)) / r0;
      if (!(std::pow(relNow, 1.0 / (it + 1)) <= lc.guard)) {
        lc.active = false;
        lc.fallbacks++;
        restart = true;
      }
    }
    std::fill(z.begin(), z.end(), 0.0);
    vcycle(levels, 0, z.data(), r.data());
    double rz2 = dotv(r.data(), z.data(), n);
    double beta = restart ? 0.0 : rz2 / rz;
    rz = rz2;
    for (size_t q = 0; q < n; ++q) p[q] = z[q] + beta * p[q];
  }
  lc.active = false;
  if (tol <= 0 && r0 > 0) rel = std::sqrt(dotv(r.data(), r.data(), n)) / r0;
  if (done) *done = it;
  if (relOut) *relOut = rel;
}

// chooseStep (newtonMultigrid.ts:597-603).
double chooseStep(const double* e, const double* m) {
  int best = 0;
  for (int k = 1; k < 4; ++k)
    if (e[k] < e[best]) best = k;
  if (e[best] < -LINE_NOISE * m[best]) return LINE_ALPHAS[best];
  bool all = true;
  for (int k = 0; k < 4; ++k) all = all && e[k] > LINE_NOISE * m[k];
  if (all) return 0;
  return 1;
}

// newtonStepPCG (newtonMultigrid.ts:610-645).
double Solver::newtonStep(int* pcgDone, double* rel, double* alphaOut) {
  if (contactOn) crossLayer ? crossTerms() : contactTerms();
  std::vector<double> kx;
  auto A = assembleFineOperator(pieceCount > 0 ? &kx : nullptr);
  // precision study: 3 keeps the operator PCG solves with exact and rounds the preconditioner's copy
  pcgOp = nullptr;
  if (prm.fp32_rows % 10 == 3) {
    pcgOp = A;
    A = std::make_shared<StencilOperator>(*A);
    roundRows(*A, 1);
  } else {
    roundRows(*A, prm.fp32_rows % 10);
  }
  // the detached pieces' rigid modes at this iterate (encodeAssemble, solver.ts:615-616)
  if (pieceCount > 0) rigidFrame(kx);
  std::vector<double> b(3 * static_cast<size_t>(N));
  rhs(b.data());
  std::vector<MGLevel> levels;
  if (prm.lag_coarse && !lagged.empty()) {
    levels = lagged;
    levels[0] = {A, lagged[0].P};
  } else {
    levels = buildHierarchy(A);
    if (prm.lag_coarse) lagged = levels;
  }
  stageLevels = levels;
  std::vector<double> d(3 * static_cast<size_t>(N), 0.0);
  // PCG starts from each piece's rigid response (encodeRigidStart, solver.ts:651-657)
  if (pieceCount > 0) rigidStart(b.data(), d.data());
  pcg(levels, b.data(), d.data(), prm.pcg_iterations, prm.pcg_rel_tol, pcgDone, rel);
  // pieces step along the rotation of that start (encodeLineSearch, solver.ts:680-681)
  if (pieceCount > 0) curveSet();
  double alpha = 1;
  if (prm.line_search) {
    double e[4], mag[4];
    energyChange(d.data(), e, mag);
    alpha = chooseStep(e, mag);
  }
  // curveApply (energy.wgsl:293-302): delta bent so that alpha delta moves them along that path
  if (pieceCount > 0 && alpha > 0)
    for (int n = 0; n < N; ++n) {
      if (pinned[n] || !curveOn[n]) continue;
      const double th[3] = {alpha * curveW[3 * n], alpha * curveW[3 * n + 1], alpha * curveW[3 * n + 2]};
      double c[3];
      rotationCurve(th, &curveR[3 * n], c);
      for (int z = 0; z < 3; ++z) d[3 * n + z] += c[z] / alpha;
    }
  curveOn.clear();
  double m = 0;
  for (size_t q = 0; q < d.size(); ++q) d[q] *= alpha;
  // newtonApply's contact and floor bounds (step.wgsl:97-112): the applied step is what is left of it
  if (floor.on || contactOn)
    for (int n = 0; n < N; ++n) {
      if (pinned[n]) continue;
      double nd[3] = {dx[3 * n] + d[3 * n], dx[3 * n + 1] + d[3 * n + 1], dx[3 * n + 2] + d[3 * n + 2]};
      feasible(n, nd);
      nd[2] = floorBoundZ(n, dx[3 * n + 2], nd[2]);
      for (int z = 0; z < 3; ++z) d[3 * n + z] = nd[z] - dx[3 * n + z];
    }
  for (size_t q = 0; q < d.size(); ++q) {
    dx[q] += d[q];
    m = std::max(m, std::fabs(d[q]));
  }
  for (int n = 0; n < N; ++n) lastUpdate[n] = hyp3(d[3 * n], d[3 * n + 1], d[3 * n + 2]);
  if (alphaOut) *alphaOut = alpha;
  return m;
}

Yarn toYarn(const btd_yarn& y) {
  return {y.ea_low, y.ea_high, y.crimp_strain, y.ea_compress, y.axial_viscosity, y.bend_rigidity, y.bend_viscosity,
          y.softening_opening, y.yarns_per_span > 0 ? y.yarns_per_span : 1};
}

}  // namespace

struct ora_solver {
  Solver s;
};

extern "C" {

const char* ora_last_error(void) { return g_err.c_str(); }

ora_solver* ora_create(const btd_scene* sc, const ora_params* p) {
  try {
    if (!sc || !p) throw std::runtime_error("null scene or params");
    auto* o = new ora_solver();
    Solver& S = o->s;
    S.prm = *p;
    S.contactOn = p->self_contact != 0;
    S.crossLayer = p->cross_layer != 0 && sc->n_layers > 1;
    {
      // contact distance of a layer pair: the mean of their thicknesses (contact.ts:49-50)
      auto thick = [&](int l) { return l < sc->n_layers ? sc->layers[l].material.thickness : 0.0; };
      S.xcDist[0] = 0.5 * (thick(0) + thick(1));
      S.xcDist[1] = 0.5 * (thick(0) + thick(2));
      S.xcDist[2] = 0.5 * (thick(1) + thick(2));
      S.xcDist[3] = 0.0;
    }
    if (p->threads > 0) omp_set_num_threads(p->threads);
    int N = sc->node_count, C = sc->crossing_count;
    S.N = N;
    S.C = C;
    for (int l = 0; l < sc->n_layers; ++l) {
      const btd_layer_info& L = sc->layers[l];
      Layer o2{};
      o2.index = L.index;
      o2.nx = L.nx;
      o2.ny = L.ny;
      o2.nodeOffset = L.node_offset;
      o2.fOffset = L.field_offset;
      o2.K = L.field_k;
      o2.M = L.field_m;
      o2.bu = L.bundle[0];
      o2.bv = L.bundle[1];
      o2.yarns[0] = toYarn(L.material.yarns[0]);
      o2.yarns[1] = toYarn(L.material.yarns[1]);
      o2.pitchU = L.material.pitch_u;
      o2.pitchV = L.material.pitch_v;
      o2.weavePitchU = L.weave.pitch_u;
      o2.weavePitchV = L.weave.pitch_v;
      o2.shearStiffness = L.material.shear_stiffness;
      o2.crossingFriction = L.material.crossing_friction;
      o2.crossingNormal0 = L.material.crossing_normal0;
      o2.crossingWrap = L.material.crossing_wrap;
      o2.airDrag = L.material.air_drag;
      o2.thickness = L.material.thickness;
      S.layers.push_back(o2);
    }
    S.mass.assign(sc->mass, sc->mass + N);
    S.crossingNormal0.assign(sc->crossing_normal0, sc->crossing_normal0 + N);
    S.softening.assign(sc->softening, sc->softening + 2 * size_t(N));
    S.pinned.assign(sc->pinned, sc->pinned + N);
    S.fieldStrength.assign(sc->field_strength, sc->field_strength + 2 * size_t(C));
    S.fieldArea.assign(sc->field_area, sc->field_area + 2 * size_t(C));
    S.fieldDamage.assign(sc->field_damage, sc->field_damage + 2 * size_t(C));
    S.x.assign(sc->position, sc->position + 3 * size_t(N));
    S.v.assign(3 * size_t(N), 0.0);
    S.dx.assign(3 * size_t(N), 0.0);
    S.pred.assign(3 * size_t(N), 0.0);
    S.restLength.assign(sc->rest_length, sc->rest_length + 2 * size_t(N));
    S.intact.assign(sc->intact, sc->intact + 2 * size_t(N));
    S.cutMask.assign(sc->cut_mask, sc->cut_mask + 2 * size_t(N));
    S.failSite.assign(sc->fail_site, sc->fail_site + 2 * size_t(N));
    S.segFlags.assign(sc->seg_flags, sc->seg_flags + 2 * size_t(N));
    S.tails.assign(sc->tails, sc->tails + 4 * size_t(N));
    S.strain.assign(2 * size_t(N), 0.0);
    S.lastUpdate.assign(N, 0.0);
    S.nbr.assign(4 * size_t(N), -1);
    S.layerOf.assign(N, 0);
    S.gripOf.assign(N, {});
    for (size_t l = 0; l < S.layers.size(); ++l) {
      const Layer& L = S.layers[l];
      for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
          int n = L.nodeOffset + j * L.nx + i;
          S.layerOf[n] = static_cast<int>(l);
          if (i > 0) S.nbr[4 * n + 0] = n - 1;
          if (i < L.nx - 1) S.nbr[4 * n + 1] = n + 1;
          if (j > 0) S.nbr[4 * n + 2] = n - L.nx;
          if (j < L.ny - 1) S.nbr[4 * n + 3] = n + L.nx;
        }
    }
    return o;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void ora_destroy(ora_solver* s) { delete s; }

int ora_set_state(ora_solver* o, const double* x, const double* v) {
  Solver& S = o->s;
  if (x) std::copy(x, x + 3 * size_t(S.N), S.x.begin());
  if (v)
    std::copy(v, v + 3 * size_t(S.N), S.v.begin());
  else
    std::fill(S.v.begin(), S.v.end(), 0.0);
  return 0;
}
int ora_get_state(ora_solver* o, double* x, double* v, double* dx, double* pred) {
  Solver& S = o->s;
  if (x) std::copy(S.x.begin(), S.x.end(), x);
  if (v) std::copy(S.v.begin(), S.v.end(), v);
  if (dx) std::copy(S.dx.begin(), S.dx.end(), dx);
  if (pred) std::copy(S.pred.begin(), S.pred.end(), pred);
  return 0;
}
int ora_set_dx(ora_solver* o, const double* dx, const double* pred) {
  Solver& S = o->s;
  if (dx) std::copy(dx, dx + 3 * size_t(S.N), S.dx.begin());
  if (pred) std::copy(pred, pred + 3 * size_t(S.N), S.pred.begin());
  return 0;
}
int ora_set_segments(ora_solver* o, const double* rest, const double* intact, const uint32_t* cut, const uint16_t* flags,
                     const double* fail, const double* tails) {
  Solver& S = o->s;
  size_t n2 = 2 * size_t(S.N);
  if (rest) std::copy(rest, rest + n2, S.restLength.begin());
  if (intact) std::copy(intact, intact + n2, S.intact.begin());
  if (cut) std::copy(cut, cut + n2, S.cutMask.begin());
  if (flags) std::copy(flags, flags + n2, S.segFlags.begin());
  if (fail) std::copy(fail, fail + n2, S.failSite.begin());
  if (tails) std::copy(tails, tails + 4 * size_t(S.N), S.tails.begin());
  return 0;
}
int ora_get_segments(ora_solver* o, double* rest, double* intact, uint32_t* cut, uint16_t* flags, double* fail,
                     double* tails) {
  Solver& S = o->s;
  if (rest) std::copy(S.restLength.begin(), S.restLength.end(), rest);
  if (intact) std::copy(S.intact.begin(), S.intact.end(), intact);
  if (cut) std::copy(S.cutMask.begin(), S.cutMask.end(), cut);
  if (flags) std::copy(S.segFlags.begin(), S.segFlags.end(), flags);
  if (fail) std::copy(S.failSite.begin(), S.failSite.end(), fail);
  if (tails) std::copy(S.tails.begin(), S.tails.end(), tails);
  return 0;
}
int ora_set_field(ora_solver* o, const uint8_t* d) {
  std::copy(d, d + o->s.fieldDamage.size(), o->s.fieldDamage.begin());
  return 0;
}
int ora_get_field(ora_solver* o, uint8_t* d) {
  std::copy(o->s.fieldDamage.begin(), o->s.fieldDamage.end(), d);
  return 0;
}
int ora_break_margins(ora_solver* o, double* out) {
  if (o->s.breakMargin.size() != o->s.fieldDamage.size()) {
    std::fill(out, out + o->s.fieldDamage.size(), INFINITY);
    return 0;
  }
  std::copy(o->s.breakMargin.begin(), o->s.breakMargin.end(), out);
  return 0;
}
int ora_set_history(ora_solver* o, int32_t on) {
  o->s.historyEnabled = on != 0;
  return 0;
}
int ora_counts(ora_solver* o, int32_t* broken, int32_t* pulled) {
  if (broken) *broken = o->s.brokenCount;
  if (pulled) *pulled = o->s.pulledOutCount;
  return 0;
}
int ora_clear_grips(ora_solver* o) {
  o->s.grips.clear();
  for (auto& g : o->s.gripOf) g.clear();
  return 0;
}
int ora_add_grip(ora_solver* o, const int32_t* nodes, const double* w, const double* offset, int32_t count, const double* goal,
                 double k) {
  Solver& S = o->s;
  Grip G;
  G.nodes.assign(nodes, nodes + count);
  G.w.assign(w, w + count);
  G.offset.assign(offset, offset + 3 * size_t(count));
  for (int q = 0; q < 3; ++q) G.goal[q] = goal[q];
  G.k = k;
  int gi = static_cast<int>(S.grips.size());
  for (int e = 0; e < count; ++e) {
    if (nodes[e] < 0 || nodes[e] >= S.N) return -1;
    S.gripOf[nodes[e]].push_back({gi, e});
  }
  S.grips.push_back(G);
  return gi;
}
int ora_set_grip_goal(ora_solver* o, int32_t grip, const double* goal) {
  if (grip < 0 || grip >= static_cast<int>(o->s.grips.size())) return -1;
  for (int q = 0; q < 3; ++q) o->s.grips[grip].goal[q] = goal[q];
  return 0;
}
int ora_set_pieces(ora_solver* o, const uint32_t* piece_of, const uint32_t* start, int32_t count, const uint32_t* nodes) {
  Solver& S = o->s;
  if (count < 0 || (count > 0 && (!piece_of || !start || !nodes))) {
    g_err = "ora_set_pieces: bad arguments";
    return -1;
  }
  // setPieces (solver.ts:664-677): pieces beyond MAX_PIECES go without the correction
  const int kept = std::min(count, Solver::MAX_PIECES);
  S.pieceCount = kept;
  S.pieceOf.assign(S.N, Solver::NO_PIECE);
  S.pieceStart.assign(start, start + (kept > 0 ? kept + 1 : 0));
  S.pieceNodes.clear();
  if (kept > 0) {
    for (int n = 0; n < S.N; ++n) S.pieceOf[n] = piece_of[n] < static_cast<uint32_t>(kept) ? piece_of[n] : Solver::NO_PIECE;
    S.pieceNodes.assign(nodes, nodes + start[kept]);
    for (uint32_t k = 0; k < start[kept]; ++k)
      if (nodes[k] >= static_cast<uint32_t>(S.N)) {
        g_err = "ora_set_pieces: node out of range";
        S.pieceCount = 0;
        return -1;
      }
  }
  return 0;
}

int ora_set_floor(ora_solver* o, int32_t enabled, double z, double bulge, double stiffness, double friction,
                  double friction_speed) {
  FloorParams& F = o->s.floor;
  F.on = enabled != 0;
  F.z = z;
  F.bulge = bulge;
  F.stiffness = stiffness;
  F.friction = friction;
  F.frictionSpeed = friction_speed;
  return 0;
}
int ora_predict(ora_solver* o) {
  o->s.predict();
  return 0;
}
int ora_newton_step(ora_solver* o, double* maxUpdate, int32_t* pcgIt, double* rel, double* alpha) {
  try {
    int done = 0;
    double r = 0, a = 1;
    double m = o->s.newtonStep(&done, &r, &a);
    if (maxUpdate) *maxUpdate = m;
    if (pcgIt) *pcgIt = done;
    if (rel) *rel = r;
    if (alpha) *alpha = a;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
int ora_finalize(ora_solver* o) {
  o->s.finalize();
  return 0;
}
int ora_update_damage(ora_solver* o) {
  o->s.updateDamage();
  return 0;
}
int ora_substep(ora_solver* o) {
  try {
    o->s.predict();
    for (int it = 0; it < o->s.prm.newton_iterations; ++it) {
      int d;
      double r, a;
      o->s.newtonStep(&d, &r, &a);
    }
    o->s.finalize();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
int ora_node_gradient(ora_solver* o, int32_t n, double* g) {
  o->s.nodeGradient(n, g);
  return 0;
}
double ora_potential(ora_solver* o) { return o->s.potential(); }
int ora_energy_change(ora_solver* o, const double* d, double* e4, double* m4) {
  o->s.energyChange(d, e4, m4);
  return 0;
}
double ora_yarn_material_length(ora_solver* o) { return o->s.yarnMaterialLength(); }

int ora_assemble(ora_solver* o, double* A, uint8_t* fixed, double* b) {
  try {
    auto op = o->s.assembleFineOperator();
    if (A) std::copy(op->A.begin(), op->A.end(), A);
    if (fixed) std::copy(op->fixed.begin(), op->fixed.end(), fixed);
    if (b) o->s.rhs(b);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
int ora_build_levels(ora_solver* o, const double* A) {
  try {
    auto op = o->s.assembleFineOperator();
    if (A) std::copy(A, A + op->A.size(), op->A.begin());
    o->s.stageLevels = o->s.buildHierarchy(op);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
int ora_level_count(ora_solver* o) { return static_cast<int>(o->s.stageLevels.size()); }
int ora_level_nodes(ora_solver* o, int32_t k) {
  if (k < 0 || k >= static_cast<int>(o->s.stageLevels.size())) return -1;
  return o->s.stageLevels[k].A->N;
}
int ora_read_level(ora_solver* o, int32_t k, double* A, uint8_t* fixed) {
  if (k < 0 || k >= static_cast<int>(o->s.stageLevels.size())) return -1;
  const StencilOperator& op = *o->s.stageLevels[k].A;
  if (A) std::copy(op.A.begin(), op.A.end(), A);
  if (fixed) std::copy(op.fixed.begin(), op.fixed.end(), fixed);
  return 0;
}
int ora_read_prolongation(ora_solver* o, int32_t k, int32_t* idx, double* w) {
  if (k < 0 || k >= static_cast<int>(o->s.stageLevels.size()) || !o->s.stageLevels[k].P) return -1;
  const Prolongation& P = *o->s.stageLevels[k].P;
  if (idx) std::copy(P.idx.begin(), P.idx.end(), idx);
  if (w) std::copy(P.w.begin(), P.w.end(), w);
  return 0;
}
int ora_apply(ora_solver* o, int32_t k, const double* x, double* y) {
  if (k < 0 || k >= static_cast<int>(o->s.stageLevels.size())) return -1;
  o->s.stageLevels[k].A->apply(x, y);
  return 0;
}
int ora_smooth(ora_solver* o, int32_t k, double* x, const double* b, int32_t reverse) {
  if (k < 0 || k >= static_cast<int>(o->s.stageLevels.size())) return -1;
  smoothLines(*o->s.stageLevels[k].A, x, b, reverse != 0, o->s.prm.line_colors);
  return 0;
}
int ora_vcycle(ora_solver* o, const double* b, double* z) {
  if (o->s.stageLevels.empty()) return -1;
  o->s.vcycle(o->s.stageLevels, 0, z, b);
  return 0;
}
int ora_pcg(ora_solver* o, const double* b, double* x, int32_t iterations, double tol, int32_t* done, double* rel) {
  if (o->s.stageLevels.empty()) return -1;
  int d = 0;
  double r = 0;
  o->s.pcg(o->s.stageLevels, b, x, iterations, tol, &d, &r);
  if (done) *done = d;
  if (rel) *rel = r;
  return 0;
}
int ora_solve_penta(int32_t n, const double* D, const double* E, const double* F, const double* r, double* x, double shift) {
  solvePenta(n, D, E, F, r, x, shift);
  return 0;
}

// ---- the constitutive laws on their own (axial.ts, laws.ts), so the reference's unit-test properties
// can be checked on the restatement; yarn = {eaLow, eaHigh, crimpStrain, eaCompress}.
static Yarn lawYarn(const double* y) {
  Yarn p{};
  p.eaLow = y[0], p.eaHigh = y[1], p.crimpStrain = y[2], p.eaCompress = y[3];
  p.yarnsPerSpan = 1;
  return p;
}
void ora_law_axial(const double* y, double eps, double* tke) {
  const Yarn p = lawYarn(y);
  tke[0] = axialTension(p, eps), tke[1] = axialStiffness(p, eps), tke[2] = axialEnergyDensity(p, eps);
}
double ora_law_strain_at_tension(const double* y, double t) { return strainAtTension(lawYarn(y), t); }
double ora_law_yarn_damage(const double* y, double yarns, double area, double peak, double soft, double eps) {
  return yarnDamage(lawYarn(y), yarns, area, peak, soft, eps);
}
void ora_law_bend_psi(double q, double a, double* out3) { bendPsi(q, a, out3); }
double ora_law_bend_psi_delta(double q0, double q1, double dq, double a) { return bendPsiDelta(q0, q1, dq, a); }
void ora_law_bend_geometry(double La, double Lc, double* out4) {
  const BendGeometry g = bendGeometry(La, Lc);
  out4[0] = g.wa, out4[1] = g.wc, out4[2] = g.kPerB, out4[3] = g.fold;
}
double ora_law_bend_scale(double ia, double ic, uint32_t maskA, uint32_t maskC, int32_t B) { return bendScale(ia, ic, maskA, maskC, B); }
double ora_law_shear_jam(double area) { return shearJam(area); }
double ora_law_cell_area(double cu, double tu, double cv, double rv) { return cellArea(cu, tu, cv, rv); }
void ora_law_shear(double ks, double Ld, double l, double jam, double* fke) { shearLaw(ks, Ld, l, jam, fke); }
void ora_law_constants(double* out3) { out3[0] = BEND_S0, out3[1] = SHEAR_JAM, out3[2] = SHEAR_RAMP; }

// ---- the yarn damage field's steps on a solver's own field and spans (yarnField.ts), so the
// reference's unit-test properties can be checked on the restatement.
// layer info: fOffset, K, M, bu, bv, nx, ny, nodeOffset
int ora_field_layer(ora_solver* o, int32_t l, int32_t* out8) {
  if (l < 0 || l >= (int)o->s.layers.size()) {
    g_err = "layer out of range";
    return -1;
  }
  const Layer& L = o->s.layers[l];
  const int32_t v[8] = {L.fOffset, L.K, L.M, L.bu, L.bv, L.nx, L.ny, L.nodeOffset};
  std::copy(v, v + 8, out8);
  return 0;
}
int32_t ora_field_span_crossing(ora_solver* o, int32_t l, int32_t i, int32_t j, int32_t f, int32_t q, int32_t p) {
  return spanCrossing(o->s.layers[l], i, j, f, q, p);
}
// ownSpan (yarnField.ts:187-196): the span (i, j) of family f that crossing (k, m) of the layer's
// field belongs to; returns 0 when it belongs to none.
int32_t ora_field_own_span(ora_solver* o, int32_t l, int32_t k, int32_t m, int32_t f, int32_t* ij) {
  const Layer& L = o->s.layers[l];
  auto fdiv = [](int a, int b) { return static_cast<int>(std::floor(static_cast<double>(a) / b)); };
  int i, j;
  bool ok;
  if (f == 1) {
    i = fdiv(k, L.bu), j = fdiv(m - L.bv / 2, L.bv);
    ok = i < L.nx && j >= 0 && j <= L.ny - 2;
  } else {
    j = fdiv(m, L.bv), i = fdiv(k - L.bu / 2, L.bu);
    ok = j < L.ny && i >= 0 && i <= L.nx - 2;
  }
  ij[0] = i, ij[1] = j;
  return ok ? 1 : 0;
}
double ora_field_interpolated_strain(ora_solver* o, int32_t l, int32_t f, int32_t k, int32_t m, const double* strain) {
  return interpolatedStrain(o->s.layers[l], f, k, m, strain);
}
int32_t ora_field_couple(ora_solver* o) { return o->s.coupleSpans(); }
int ora_field_update(ora_solver* o, const double* strain) {
  std::copy(strain, strain + o->s.strain.size(), o->s.strain.begin());
  o->s.updateField();
  return 0;
}
int32_t ora_field_pull_out(ora_solver* o, const double* strain) {
  std::copy(strain, strain + o->s.strain.size(), o->s.strain.begin());
  return o->s.pullOut();
}
double ora_field_recoil_length(const double* yarn, double B, double area, double peak, double eps, double mu, double n0, double wrap,
                               double tCross, double pitch) {
  return recoilLength(lawYarn(yarn), B, area, peak, eps, mu, n0, wrap, tCross, pitch);
}
int32_t ora_field_share_reach(ora_solver* o, int32_t l, int32_t f) { return shareReach(o->s.layers[l], f); }
double ora_field_share_factor(ora_solver* o, int32_t l, const uint8_t* sep, int32_t f, int32_t k, int32_t m, int32_t reach, double cap) {
  return shareFactor(o->s.layers[l], sep, f, k, m, reach, cap);
}
double ora_field_share_cap(int32_t reach, double mu, double n0, double wrap, double tCross, double peak) {
  return shareCap(reach, mu, n0, wrap, tCross, peak);
}
// SHARE_FRACTION, DAMAGE_CUT, DAMAGE_PULLED
void ora_field_constants(double* out3) { out3[0] = SHARE_FRACTION, out3[1] = DAMAGE_CUT, out3[2] = DAMAGE_PULLED; }

// Learned coarse correction (extension; no counterpart in the reference).
int32_t ora_learned_size(void) { return LC_WEIGHTS; }
int32_t ora_learned_dims(int32_t* in_hidden_basis) {
  in_hidden_basis[0] = LC_IN, in_hidden_basis[1] = LC_HID, in_hidden_basis[2] = LC_K;
  return 0;
}
int ora_learned_set(ora_solver* o, const double* w, int32_t count, int32_t on, double guard) {
  if (!o || (on && (!w || count != LC_WEIGHTS))) {
    g_err = "ora_learned_set: weights must hold ora_learned_size() values";
    return -1;
  }
  if (w && count == LC_WEIGHTS) o->s.lc.w.assign(w, w + LC_WEIGHTS);
  o->s.lc.on = on != 0;
  o->s.lc.guard = guard;
  return 0;
}
int ora_learned_log(ora_solver* o, int32_t on, int64_t capacity) {
  auto& lc = o->s.lc;
  lc.log = on != 0;
  lc.logCap = capacity > 0 ? static_cast<size_t>(capacity) : 0;
  lc.ops.clear();
  lc.calls.clear();
  lc.denseOp.reset();
  lc.denseL.clear();
  return 0;
}
int32_t ora_learned_ops(ora_solver* o) { return static_cast<int32_t>(o->s.lc.ops.size()); }
int32_t ora_learned_op_nodes(ora_solver* o, int32_t k) {
  if (k < 0 || k >= static_cast<int32_t>(o->s.lc.ops.size())) {
    g_err = "ora_learned_op_nodes: operator out of range";
    return -1;
  }
  return o->s.lc.ops[k].nodes;
}
int ora_learned_op(ora_solver* o, int32_t k, double* At, double* X) {
  if (k < 0 || k >= static_cast<int32_t>(o->s.lc.ops.size())) {
    g_err = "ora_learned_op: operator out of range";
    return -1;
  }
  const LearnedOp& op = o->s.lc.ops[k];
  std::copy(op.At.begin(), op.At.end(), At);
  std::copy(op.X.begin(), op.X.end(), X);
  return 0;
}
int32_t ora_learned_calls(ora_solver* o) { return static_cast<int32_t>(o->s.lc.calls.size()); }
int ora_learned_call(ora_solver* o, int32_t q, int32_t* op, double* r, double* d) {
  if (q < 0 || q >= static_cast<int32_t>(o->s.lc.calls.size())) {
    g_err = "ora_learned_call: call out of range";
    return -1;
  }
  const LearnedCall& c = o->s.lc.calls[q];
  *op = c.op;  // r and d may be null to ask for the operator (and so the size) first
  if (r) std::copy(c.r.begin(), c.r.end(), r);
  if (d) std::copy(c.d.begin(), c.d.end(), d);
  return 0;
}
int ora_learned_stats(ora_solver* o, int64_t* applied_fallbacks_solves) {
  applied_fallbacks_solves[0] = o->s.lc.applied;
  applied_fallbacks_solves[1] = o->s.lc.fallbacks;
  applied_fallbacks_solves[2] = o->s.lc.solves;
  return 0;
}
int ora_learned_forward(const double* w, const double* X, int64_t rows, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < rows; ++q) lcForward(w, X + q * LC_IN, out + q * LC_OUT);
  return 0;
}

// The learned basis of a given coarsest operator (one nx x ny layer, A in the 25-offset layout, fixed
// flags, 2 input flags per node: damage, contact): the node inputs X (M x LC_IN, zero rows for nodes
// without a positive definite block), Phi (3 M x LC_K), the Cholesky factor of Phi^T A Phi (LC_K^2) and
// its dropped columns; returns -1 if no basis could be built. Checks the CUDA path's basis kernel.
int ora_learned_basis_of(ora_solver* o, const double* w, const double* A, const uint8_t* fixed, int32_t nx, int32_t ny,
                         const float* flags, double* X, double* phi, double* G, int32_t* dead) {
  try {
    Solver& s = o->s;
    auto op = std::make_shared<StencilOperator>(std::vector<LatticeLayer>{{nx, ny, 0}});
    std::copy(A, A + op->A.size(), op->A.begin());
    std::copy(fixed, fixed + op->N, op->fixed.begin());
    const LearnedCoarse saved = s.lc;
    s.lc.w.assign(w, w + LC_WEIGHTS);
    s.lc.flags.assign(flags, flags + 2 * static_cast<size_t>(op->N));
    std::vector<double> L, Xv;
    std::vector<uint8_t> ok;
    s.learnedInputs(*op, L, ok, Xv);
    if (X) std::copy(Xv.begin(), Xv.end(), X);
    std::vector<MGLevel> levels{{op, nullptr}};
    s.learnedBasis(levels);
    const bool built = s.lc.basisOp == op.get();
    if (built) {
      if (phi) std::copy(s.lc.phi.begin(), s.lc.phi.end(), phi);
      if (G) std::copy(s.lc.G.begin(), s.lc.G.end(), G);
      if (dead)
        for (int k = 0; k < LC_K; ++k) dead[k] = s.lc.dead[k];
    }
    s.lc = saved;
    return built ? 0 : -1;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

}  // extern "C"
