// Per-node kernels of a substep outside the linear solve: predictor, fine-level assembly of the
// projected Newton system, bounded Newton update and commit.
//   predict      step.wgsl:46-59, ReferenceSolver.predict (solver.ts(ref):602-613)
//   assemble     assemble.wgsl:152-334 + drag.wgsl:344-391, assembleFineOperator/nodeGradient
//                (newtonMultigrid.ts:169-274, solver.ts(ref):387-422)
//   newtonApply  step.wgsl:97-112 (line-search step, non-finite firewall, floor bound)
//   commit       step.wgsl:128-147, ReferenceSolver.finalize (solver.ts(ref):622-628)
#pragma once

#include "common.cuh"

namespace btd {

struct StepArgs {
  const SimParams* P;
  int N;
  const NodeStatic* __restrict__ nodes;
  const uint32_t* __restrict__ pinned;  // fine-level fixed flags
  const DLayer* __restrict__ layers;
  float4* x;
  float4* v;
  float4* dx;
  float4* pred;
  const Seg* __restrict__ segs;
  const float4* __restrict__ ext;    // 3 per node: gradient, H (xx xy xz yy), H (yz zz)
  const float4* __restrict__ cmeta;  // 2 per node: contact bounds (own, reciprocal); nullptr: none
  uint32_t* counters;
  Scalars* scal;
  // detached pieces (pieceCount 0: none): the assembly writes each piece node's external block into kx
  int pieceCount;
  const uint32_t* __restrict__ pieceOf;
  float* kx;
  // the rotation curves of the pieces' nodes for the update (null: none)
  const float4* __restrict__ curveW;
  const float4* __restrict__ curveR;
};

__global__ void k_predict(StepArgs a) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  const SimParams P = *a.P;
  if (a.pinned[n]) {
    a.pred[n] = make_float4(0, 0, 0, 0);
    a.dx[n] = make_float4(0, 0, 0, 0);
    return;
  }
  float3 hv = P.h * f3(a.v[n]);
  float h2 = P.h * P.h;
  a.pred[n] = make_float4(hv.x + h2 * P.gx, hv.y + h2 * P.gy, hv.z + h2 * P.gz, 0.f);
  a.dx[n] = make_float4(hv.x, hv.y, hv.z, 0.f);
}

__device__ __forceinline__ int nodeAt(const DLayer& L, int i, int j) {
  if (i < 0 || j < 0 || i >= L.nx || j >= L.ny) return -1;
  return L.offset + j * L.nx + i;
}
__device__ __forceinline__ bool activeSpan(const Seg* __restrict__ segs, int owner, int f) {
  if (owner < 0) return false;
  return segActive(segs[2 * owner + f]);
}

struct SegForce {
  float fs, kPar, kPerp;
  float3 e;
  float l, L;
};
// Axial response of the span owned by a toward b (family f) at the current iterate (segForce,
// assemble.wgsl:53-65; solver.ts(ref):254-277).
__device__ __forceinline__ SegForce segForce(const StepArgs& A, int a, int b, int f, const DLayer& mat, float h) {
  float3 en = f3(A.x[b]) - f3(A.x[a]);
  float3 e = en + (f3(A.dx[b]) - f3(A.dx[a]));
  float l = len3(e), ln = len3(en);
  Seg s = A.segs[2 * a + f];
  const DYarn& y = mat.yarn[f];
  float L = s.rest;
  float eps = l / L - 1.f;
  float T = s.intact * axialTension(y, eps), K = s.intact * axialStiffness(y, eps);
  float c = y.axialVisc / (L * h);
  float fs = T + c * (l - ln);
  return {fs, fmaxf(K, 0.f) / L + c, fmaxf(fs, 0.f) / l, (1.f / l) * e, l, L};
}

struct Triple {
  float ke, kd, k, wa, wc;
  float3 r, rn;
};
// Bending triple (a, b, c) centred at b (triple, assemble.wgsl:84-97; bendCoeffs solver.ts(ref):284-291).
__device__ __forceinline__ Triple tripleAt(const StepArgs& A, int a, int b, int c, int f, const DLayer& mat, float h) {
  Seg sa = A.segs[2 * a + f], sb = A.segs[2 * b + f];
  float4 geo = bendGeometry(sa.rest, sb.rest);
  const DYarn& y = mat.yarn[f];
  float kb = y.bendRigidity * bendScale(sa.intact, sb.intact, sa.cutMask, sb.cutMask, (uint32_t)y.yarnsPerSpan) * geo.z;
  float kd = kb * y.bendVisc / h;
  float3 rn = geo.x * f3(A.x[a]) - 2.f * f3(A.x[b]) + geo.y * f3(A.x[c]);
  float3 r = rn + geo.x * f3(A.dx[a]) - 2.f * f3(A.dx[b]) + geo.y * f3(A.dx[c]);
  float q = dot3(r, r);
  float3 ps = bendPsi(q, geo.w);
  return {kb * ps.y, kd, kb * (ps.y + 2.f * ps.z * q) + kd, geo.x, geo.y, r, rn};
}
__device__ __forceinline__ float3 tripleGrad(const Triple& t) {
  float lr = len3(t.r);
  return (t.ke + t.kd * (lr - len3(t.rn)) / fmaxf(lr, 1e-12f)) * t.r;
}

// Shear diagonal d of the cell with lower-left corner (ci, cj) acts while one of its triangles is
// intact (diagActive, assemble.wgsl:108-119).
__device__ __forceinline__ bool diagActive(const Seg* __restrict__ segs, const DLayer& L, int ci, int cj, int d) {
  int c = nodeAt(L, ci, cj), r = nodeAt(L, ci + 1, cj), t = nodeAt(L, ci, cj + 1);
  if (c < 0 || r < 0 || t < 0) return false;
  bool cu = activeSpan(segs, c, 0), cv = activeSpan(segs, c, 1), rv = activeSpan(segs, r, 1), tu = activeSpan(segs, t, 0);
  if (d == 0) return (cu && rv) || (cv && tu);
  return (cu && cv) || (rv && tu);
}
__device__ __forceinline__ float intactOf(const Seg* __restrict__ segs, int owner, int f) {
  if (owner < 0) return 0.f;
  Seg s = segs[2 * owner + f];
  return segActive(s) ? s.intact : 0.f;
}
// Shear stiffness and jam strain of a cell (cellShear, assemble.wgsl:125-131).
__device__ __forceinline__ float2 cellShear(const StepArgs& A, const DLayer& L, int ci, int cj) {
  int c = nodeAt(L, ci, cj), r = nodeAt(L, ci + 1, cj), t = nodeAt(L, ci, cj + 1);
  float ar = cellArea(intactOf(A.segs, c, 0), intactOf(A.segs, t, 0), intactOf(A.segs, c, 1), intactOf(A.segs, r, 1));
  return make_float2(L.shearStiffness * A.nodes[c].n0 / L.crossingNormal0, shearJam(ar));
}
__device__ __forceinline__ float shearRest(const StepArgs& A, const DLayer& L, int ci, int cj) {
  int c = nodeAt(L, ci, cj);
  float s0 = A.segs[2 * c].rest, s1 = A.segs[2 * c + 1].rest;
  return sqrtf(s0 * s0 + s1 * s1);
}

// Implicit air drag block from the accepted state (airDragBlock, drag.wgsl:368-391).
__device__ __forceinline__ Sym airDragBlock(const StepArgs& A, int n, const DLayer& L, int i, int j, float h) {
  if (!(L.airDrag > 0.f)) return symZero();
  float k = L.airDrag * L.pitchU * L.pitchV / h;
  float3 t[2];
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    int du = f == 0 ? 1 : 0, dv = f == 1 ? 1 : 0;
    int prev = nodeAt(L, i - du, j - dv), next = nodeAt(L, i + du, j + dv);
    float3 a = f3(A.x[n]), b = a;
    if (activeSpan(A.segs, prev, f)) a = f3(A.x[prev]);
    if (next >= 0 && activeSpan(A.segs, n, f)) b = f3(A.x[next]);
    t[f] = b - a;
  }
  float lu = len3(t[0]), lv = len3(t[1]);
  if (lu > 0.f && lv > 0.f) {
    float3 c = cross3(t[0], t[1]);
    float lc = len3(c);
    if (lc > 1e-3f * lu * lv) return axialBlock(k, 0.f, (1.f / lc) * c);
  }
  if (lu > 0.f || lv > 0.f) {
    float3 tt = lu >= lv ? (1.f / lu) * t[0] : (1.f / lv) * t[1];
    return axialBlock(0.f, k, tt);
  }
  return symId(k);
}

// ------------------------------------------------------------------ the gradient in FP64
// The Newton right-hand side -grad(Phi) sums large elastic terms (span tensions of whole rows of the
// sheet) to a small net force. In FP32 the strain of a span is only known to ~6e-8 (l / L - 1 rounded),
// i.e. EA x 6e-8 of tension - a few per cent of a node's weight in the hanging patch - and that floor
// stays in the Newton iterate however far PCG converges. This evaluates the same terms in FP64 from the
// FP32 state (differences of positions formed before any rounding), so each Newton iteration is an
// iterative-refinement step: FP64 residual, FP32 correction (the operator and the solve stay FP32).
struct Dv {
  double x, y, z;
};
__device__ __forceinline__ Dv dv(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ Dv operator+(Dv a, Dv b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ Dv operator-(Dv a, Dv b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ Dv operator*(double s, Dv a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dotD(Dv a, Dv b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double lenD(Dv a) { return sqrt(dotD(a, a)); }
__device__ __forceinline__ Dv symVecD(const Sym& A, Dv v) {
  return {A.xx * v.x + A.xy * v.y + A.xz * v.z, A.xy * v.x + A.yy * v.y + A.yz * v.z, A.xz * v.x + A.yz * v.y + A.zz * v.z};
}
__device__ __forceinline__ double axialTensionD(const DYarn& y, double eps) {
  if (eps <= 0.0) return (double)y.eaCompress * eps;
  const double ec = y.crimpStrain, lo = y.eaLow, hi = y.eaHigh, dk = hi - lo;
  if (eps <= ec) return lo * eps + dk * eps * eps / (2.0 * ec);
  return lo * ec + dk * ec * 0.5 + hi * (eps - ec);
}
__device__ __forceinline__ double bendPsiSlopeD(double q, double a) {
  const double s = q / a, s0 = BEND_S0;
  if (s < s0) {
    const double d = 1.0 - s;
    return 1.0 / (d * d);
  }
  const double d0 = 1.0 - s0;
  return 1.0 / (d0 * d0) + 2.0 / (a * d0 * d0 * d0) * (q - s0 * a);
}
__device__ __forceinline__ double shearForceD(double ks, double jam, double Ld, double l) {
  double f = ks * (l - Ld);
  const double c = (Ld - l) / Ld - jam, ramp = SHEAR_RAMP;
  if (c > 0.0) {
    const double extra = ks * ((double)SHEAR_LOCK - 1.0);
    f -= c < ramp ? extra * Ld * c * c / (2.0 * ramp) : extra * Ld * (c - 0.5 * ramp);
  }
  return f;
}
// Axial force vector of the span owned by a toward b (fs e / l), FP64.
__device__ __forceinline__ Dv segForceD(const StepArgs& A, int a, int b, int f, const DLayer& mat, double h) {
  const Dv en = dv(A.x[b]) - dv(A.x[a]);
  const Dv e = en + (dv(A.dx[b]) - dv(A.dx[a]));
  const double l = lenD(e), ln = lenD(en);
  const Seg s = A.segs[2 * a + f];
  const DYarn& y = mat.yarn[f];
  const double L = s.rest;
  const double T = (double)s.intact * axialTensionD(y, l / L - 1.0);
  const double c = (double)y.axialVisc / (L * h);
  return ((T + c * (l - ln)) / l) * e;
}
// Bending gradient vector of the triple (a, b, c) centred at b, FP64 (tripleGrad).
__device__ __forceinline__ Dv tripleGradD(const StepArgs& A, int a, int b, int c, int f, const DLayer& mat, double h) {
  const Seg sa = A.segs[2 * a + f], sb = A.segs[2 * b + f];
  const double La = sa.rest, Lc = sb.rest, sum = La + Lc, lh = 2.0 * La * Lc / sum;
  const double wa = 2.0 * Lc / sum, wc = 2.0 * La / sum, gz = 1.0 / (lh * lh * 0.5 * sum), fold = 4.0 * lh * lh;
  const DYarn& y = mat.yarn[f];
  const double kb = (double)y.bendRigidity * bendScale(sa.intact, sb.intact, sa.cutMask, sb.cutMask, (uint32_t)y.yarnsPerSpan) * gz;
  const double kd = kb * (double)y.bendVisc / h;
  const Dv xb = dv(A.x[b]);
  const Dv rn = wa * (dv(A.x[a]) - xb) + wc * (dv(A.x[c]) - xb) + (wa + wc - 2.0) * xb;
  const Dv r = rn + wa * dv(A.dx[a]) - 2.0 * dv(A.dx[b]) + wc * dv(A.dx[c]);
  const double q = dotD(r, r), lr = sqrt(q);
  const double ke = kb * bendPsiSlopeD(q, fold);
  return (ke + kd * (lr - lenD(rn)) / fmax(lr, 1e-12)) * r;
}

// The gradient of node n in FP64: the same terms as k_assemble's FP32 g (inertia, drag, external,
// floor, axial, bending, shear).
__device__ Dv gradientD(const StepArgs& A, int n, const SimParams& P, const NodeStatic& st, const DLayer& L, int i, int j,
                        const Sym& Dd) {
  const double h = P.h, w = (double)st.mass / (h * h);
  const Dv dxn = dv(A.dx[n]);
  Dv g = w * (dxn - dv(A.pred[n]));
  g = g + symVecD(Dd, dxn);
  g = g + dv(A.ext[3 * n]);
  if (P.floorOn) {
    const double half = 0.5 * (double)L.thickness, delta = half + (double)P.floorBulge;
    const double zc = (double)A.x[n].z + dxn.z, s = delta - (zc - (double)P.floorZ);
    if (s > 0.0) {
      const double kc = P.floorStiffness, lam = kc * s * s / delta;
      const double kf = (double)P.floorFriction * lam / fmax(sqrt(dxn.x * dxn.x + dxn.y * dxn.y), (double)P.floorFrictionSpeed * h);
      g = g + Dv{kf * dxn.x, kf * dxn.y, -lam};
    }
  }
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    const int du = f == 0 ? 1 : 0, dv_ = f == 1 ? 1 : 0;
    const int prev = nodeAt(L, i - du, j - dv_), next = nodeAt(L, i + du, j + dv_);
    const int prev2 = nodeAt(L, i - 2 * du, j - 2 * dv_), next2 = nodeAt(L, i + 2 * du, j + 2 * dv_);
    const bool actPrev = activeSpan(A.segs, prev, f);
    const bool actNext = activeSpan(A.segs, n, f) && next >= 0;
    if (actPrev) g = g + segForceD(A, prev, n, f, L, h);
    if (actNext) g = g - segForceD(A, n, next, f, L, h);
    if (actPrev && actNext) g = g - 2.0 * tripleGradD(A, prev, n, next, f, L, h);
    if (actNext && activeSpan(A.segs, next, f) && next2 >= 0) {
      const Seg s0 = A.segs[2 * n + f], s1 = A.segs[2 * next + f];
      const double wa = 2.0 * (double)s1.rest / ((double)s0.rest + s1.rest);
      g = g + wa * tripleGradD(A, n, next, next2, f, L, h);
    }
    if (actPrev && activeSpan(A.segs, prev2, f)) {
      const Seg s0 = A.segs[2 * prev2 + f], s1 = A.segs[2 * prev + f];
      const double wc = 2.0 * (double)s0.rest / ((double)s0.rest + s1.rest);
      g = g + wc * tripleGradD(A, prev2, prev, n, f, L, h);
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int ci = i, cj = j, pi = i + 1, pj = j + 1;
    if (c == 1) ci = i - 1, cj = j - 1, pi = i - 1, pj = j - 1;
    if (c == 2) ci = i - 1, cj = j, pi = i - 1, pj = j + 1;
    if (c == 3) ci = i, cj = j - 1, pi = i + 1, pj = j - 1;
    const int p = nodeAt(L, pi, pj);
    if (p < 0 || !diagActive(A.segs, L, ci, cj, c < 2 ? 0 : 1)) continue;
    const Dv d = (dv(A.x[p]) - dv(A.x[n])) + (dv(A.dx[p]) - dxn);
    const double len = lenD(d);
    const float2 cs = cellShear(A, L, ci, cj);
    const int cn = nodeAt(L, ci, cj);
    const double r0 = A.segs[2 * cn].rest, r1 = A.segs[2 * cn + 1].rest;
    const double fsh = shearForceD(cs.x, cs.y, sqrt(r0 * r0 + r1 * r1), len);
    g = g - (fsh / len) * d;
  }
  return g;
}

// PSD block of a spring element (an axial span a -> b, or a shear diagonal): the closed-form projection
// kPar e e^T + kPerp (I - e e^T) (newtonMultigrid.ts:127-130, 154-157), except for a near-degenerate
// element - collapsed below 1 % of its rest length - whose block is the FP64 eigen-clamp of its exact
// Hessian (springBlockFP64).
constexpr float DEGENERATE_LENGTH = 1e-2f;
__device__ __forceinline__ Sym springBlock(const StepArgs& A, int a, int b, float K, float f, float kPerp, float3 e, float l, float L) {
  if (l >= DEGENERATE_LENGTH * L) return axialBlock(K, kPerp, e);
  const float4 xa = A.x[a], xb = A.x[b], da = A.dx[a], db = A.dx[b];
  const double dx = ((double)xb.x - xa.x) + ((double)db.x - da.x), dy = ((double)xb.y - xa.y) + ((double)db.y - da.y),
               dz = ((double)xb.z - xa.z) + ((double)db.z - da.z);
  return springBlockFP64(K, f, dx, dy, dz);
}

// The same block in FP64 for the FP64 row: the element's direction from its FP64 vector, so that the
// block is PSD in FP64 whatever the ratio of kPar to kPerp (its FP32 entries round by ~6e-8 kPar, which
// for a slack span exceeds kPerp and the inertia of a loose strand).
__device__ __forceinline__ SymD springBlockD(const StepArgs& A, int a, int b, float K, float f, float kPerp, float l, float L) {
  const float4 xa = A.x[a], xb = A.x[b], da = A.dx[a], db = A.dx[b];
  const double dx = ((double)xb.x - xa.x) + ((double)db.x - da.x), dy = ((double)xb.y - xa.y) + ((double)db.y - da.y),
               dz = ((double)xb.z - xa.z) + ((double)db.z - da.z);
  if (l < DEGENERATE_LENGTH * L) return springBlockFP64D(K, f, dx, dy, dz);
  const double ld = sqrt(dx * dx + dy * dy + dz * dz);
  return axialBlockD(K, kPerp, dx / ld, dy / ld, dz / ld);
}

// Normal stiffness of an active contact bound relative to the node's own diagonal (assemble.wgsl:142).
constexpr float ACTIVE_BOUND = 100.f;

__global__ void __launch_bounds__(128) k_assemble(StepArgs A, float4* __restrict__ op, float4* __restrict__ rhs,
                                                  double2* __restrict__ op64) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= A.N) return;
  const int N = A.N;
  float row[60];
#pragma unroll
  for (int q = 0; q < 60; ++q) row[q] = 0.f;
  if (A.pinned[n]) {
    storeSymAt(row, 0, symId(1.f));
#pragma unroll
    for (int p = 0; p < FINE_PLANES; ++p) op[(size_t)p * N + n] = make_float4(row[4 * p], row[4 * p + 1], row[4 * p + 2], row[4 * p + 3]);
    if (op64)
      for (int q = 0; q < FINE64_PLANES; ++q)  // the identity block: values 0, 3 and 5
        op64[(size_t)q * N + n] = make_double2(q == 0 ? 1.0 : 0.0, q == 1 || q == 2 ? 1.0 : 0.0);
    rhs[n] = make_float4(0, 0, 0, 0);
    return;
  }
  const SimParams P = *A.P;
  const NodeStatic st = A.nodes[n];
  const int i = st.ij & 0xFFFF, j = st.ij >> 16;
  const DLayer& L = A.layers[st.layer];
  const float h = P.h;
  const float w = st.mass / (h * h);
  Sym D = symId(w);
  const float3 dxn = f3(A.dx[n]);
  float3 g = w * (dxn - f3(A.pred[n]));
  Sym Dd = airDragBlock(A, n, L, i, j, h);
  g += Dd * dxn;
  D = D + Dd;
  {
    float4 e0 = A.ext[3 * n], e1 = A.ext[3 * n + 1], e2 = A.ext[3 * n + 2];
    g += f3(e0);
    D = D + Sym{e1.x, e1.y, e1.z, e1.w, e2.x, e2.y};
  }
  bool onFloorCore = false;
  if (P.floorOn) {
    float half = 0.5f * L.thickness;
    float delta = half + P.floorBulge;
    float zc = A.x[n].z + dxn.z;
    float s = delta - (zc - P.floorZ);
    if (s > 0.f) {
      float kc = P.floorStiffness;
      float lam = kc * s * s / delta;
      float kf = P.floorFriction * lam / fmaxf(sqrtf(dxn.x * dxn.x + dxn.y * dxn.y), P.floorFrictionSpeed * h);
      g += make_float3(kf * dxn.x, kf * dxn.y, -lam);
      D = D + Sym{kf, 0, 0, kf, 0, 2.f * kc * s / delta};
      onFloorCore = zc <= P.floorZ + half * (1.f + 1e-3f);
    }
  }
  // a detached piece's node: its external block (inertia, drag, contact, grips, floor; the active bounds
  // below) for the rigid frame (assemble.wgsl:172-190, 323-327)
  const bool pieceNode = A.pieceCount > 0 && A.pieceOf[n] < (uint32_t)A.pieceCount;
  Sym Dext = D;
  // the FP64 row (op64): the same terms summed in FP64, the spans' blocks formed in FP64
  SymD D64 = symD(D);
  SymD C1d[4] = {symZeroD(), symZeroD(), symZeroD(), symZeroD()};

  // couplings [+u, -u, +v, -v] axial/bending, scalars [+2u, -2u, +2v, -2v]
  Sym C1[4] = {symZero(), symZero(), symZero(), symZero()};
  float C2[4] = {0, 0, 0, 0};
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    const int du = f == 0 ? 1 : 0, dv = f == 1 ? 1 : 0;
    const int prev = nodeAt(L, i - du, j - dv), next = nodeAt(L, i + du, j + dv);
    const int prev2 = nodeAt(L, i - 2 * du, j - 2 * dv), next2 = nodeAt(L, i + 2 * du, j + 2 * dv);
    const bool actPrev = activeSpan(A.segs, prev, f);
    const bool actNext = activeSpan(A.segs, n, f) && next >= 0;
    const bool freeNext = next >= 0 && !A.pinned[next];
    const bool freePrev = prev >= 0 && !A.pinned[prev];
    const int kp = 2 * f, km = 2 * f + 1;
    if (actPrev) {
      SegForce s = segForce(A, prev, n, f, L, h);
      g += s.fs * s.e;
      Sym H = springBlock(A, prev, n, s.kPar, s.fs, s.kPerp, s.e, s.l, s.L);
      D = D + H;
      if (freePrev) C1[km] = C1[km] + H * -1.f;
      if (op64) {
        const SymD Hd = springBlockD(A, prev, n, s.kPar, s.fs, s.kPerp, s.l, s.L);
        D64 = D64 + Hd;
        if (freePrev) C1d[km] = C1d[km] + Hd * -1.0;
      }
    }
    if (actNext) {
      SegForce s = segForce(A, n, next, f, L, h);
      g -= s.fs * s.e;
      Sym H = springBlock(A, n, next, s.kPar, s.fs, s.kPerp, s.e, s.l, s.L);
      D = D + H;
      if (freeNext) C1[kp] = C1[kp] + H * -1.f;
      if (op64) {
        const SymD Hd = springBlockD(A, n, next, s.kPar, s.fs, s.kPerp, s.l, s.L);
        D64 = D64 + Hd;
        if (freeNext) C1d[kp] = C1d[kp] + Hd * -1.0;
      }
    }
    if (actPrev && actNext) {
      Triple t = tripleAt(A, prev, n, next, f, L, h);
      g += -2.f * tripleGrad(t);
      D = D + symId(4.f * t.k);
      if (freeNext) C1[kp] = C1[kp] + symId(-2.f * t.wc * t.k);
      if (freePrev) C1[km] = C1[km] + symId(-2.f * t.wa * t.k);
      D64 = D64 + symIdD(4.0 * t.k);
      if (freeNext) C1d[kp] = C1d[kp] + symIdD(-2.0 * t.wc * t.k);
      if (freePrev) C1d[km] = C1d[km] + symIdD(-2.0 * t.wa * t.k);
    }
    if (actNext && activeSpan(A.segs, next, f) && next2 >= 0) {
      Triple t = tripleAt(A, n, next, next2, f, L, h);
      g += t.wa * tripleGrad(t);
      D = D + symId(t.wa * t.wa * t.k);
      if (freeNext) C1[kp] = C1[kp] + symId(-2.f * t.wa * t.k);
      D64 = D64 + symIdD((double)t.wa * t.wa * t.k);
      if (freeNext) C1d[kp] = C1d[kp] + symIdD(-2.0 * t.wa * t.k);
      if (!A.pinned[next2]) C2[kp] += t.wa * t.wc * t.k;
    }
    if (actPrev && activeSpan(A.segs, prev2, f)) {
      Triple t = tripleAt(A, prev2, prev, n, f, L, h);
      g += t.wc * tripleGrad(t);
      D = D + symId(t.wc * t.wc * t.k);
      if (freePrev) C1[km] = C1[km] + symId(-2.f * t.wc * t.k);
      D64 = D64 + symIdD((double)t.wc * t.wc * t.k);
      if (freePrev) C1d[km] = C1d[km] + symIdD(-2.0 * t.wc * t.k);
      if (!A.pinned[prev2]) C2[km] += t.wa * t.wc * t.k;
    }
  }

  // shear diagonals around n; partner order +u+v, -u-v, -u+v, +u-v
  Sym CD[4] = {symZero(), symZero(), symZero(), symZero()};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int ci = i, cj = j, pi = i + 1, pj = j + 1;
    if (c == 1) ci = i - 1, cj = j - 1, pi = i - 1, pj = j - 1;
    if (c == 2) ci = i - 1, cj = j, pi = i - 1, pj = j + 1;
    if (c == 3) ci = i, cj = j - 1, pi = i + 1, pj = j - 1;
    int p = nodeAt(L, pi, pj);
    if (p < 0 || !diagActive(A.segs, L, ci, cj, c < 2 ? 0 : 1)) continue;
    float3 d = (f3(A.x[p]) - f3(A.x[n])) + (f3(A.dx[p]) - dxn);
    float len = len3(d);
    float3 e = (1.f / len) * d;
    float2 cs = cellShear(A, L, ci, cj);
    float2 sl = shearLaw(cs.x, cs.y, shearRest(A, L, ci, cj), len);
    g -= sl.x * e;
    const float Ld = shearRest(A, L, ci, cj);
    Sym H = springBlock(A, n, p, sl.y, sl.x, fmaxf(sl.x, 0.f) / len, e, len, Ld);
    D = D + H;
    D64 = D64 + symD(H);
    if (!A.pinned[p]) CD[c] = H * -1.f;
  }

  // active contact bounds and the floor's hard limit, where the forces still press on
  const float kAct = ACTIVE_BOUND * (D.xx + D.yy + D.zz);
  if (A.cmeta) {
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      float4 m = A.cmeta[2 * n + b];
      if (m.w >= 1e8f || (m.x == 0.f && m.y == 0.f && m.z == 0.f)) continue;
      float3 mv = f3(m);
      if (-dot3(dxn, mv) >= m.w - 1e-3f * fabsf(m.w) && dot3(g, mv) > 0.f) {
        D = D + axialBlock(kAct, 0.f, mv);
        D64 = D64 + symD(axialBlock(kAct, 0.f, mv));
        Dext = Dext + axialBlock(kAct, 0.f, mv);
      }
    }
  }
  if (onFloorCore && g.z > 0.f) {
    D = D + axialBlock(kAct, 0.f, make_float3(0, 0, 1));
    D64 = D64 + symD(axialBlock(kAct, 0.f, make_float3(0, 0, 1)));
    Dext = Dext + axialBlock(kAct, 0.f, make_float3(0, 0, 1));
  }
  if (op64) {
    double r64[58];
    auto put = [&](int f, const SymD& b) {
      r64[f] = b.xx, r64[f + 1] = b.xy, r64[f + 2] = b.xz, r64[f + 3] = b.yy, r64[f + 4] = b.yz, r64[f + 5] = b.zz;
    };
    put(0, D64);
#pragma unroll
    for (int k = 0; k < 4; ++k) put(6 * (k + 1), C1d[k]);
#pragma unroll
    for (int k = 0; k < 4; ++k) put(6 * (k + 5), symD(CD[k]));
#pragma unroll
    for (int k = 0; k < 4; ++k) r64[54 + k] = C2[k];
#pragma unroll
    for (int q = 0; q < FINE64_PLANES; ++q) op64[(size_t)q * N + n] = make_double2(r64[2 * q], r64[2 * q + 1]);
  }
  if (pieceNode) storeSymAt(A.kx + 6 * (size_t)n, 0, Dext);

  storeSymAt(row, 0, D);
#pragma unroll
  for (int k = 0; k < 4; ++k) storeSymAt(row, 6 * (k + 1), C1[k]);
#pragma unroll
  for (int k = 0; k < 4; ++k) storeSymAt(row, 6 * (k + 5), CD[k]);
  row[54] = C2[0], row[55] = C2[1], row[56] = C2[2], row[57] = C2[3];
#pragma unroll
  for (int p = 0; p < FINE_PLANES; ++p) op[(size_t)p * N + n] = make_float4(row[4 * p], row[4 * p + 1], row[4 * p + 2], row[4 * p + 3]);
  if (P.gradFp64) {
    const Dv gd = gradientD(A, n, P, st, L, i, j, Dd);
    rhs[n] = make_float4((float)-gd.x, (float)-gd.y, (float)-gd.z, 0.f);
    return;
  }
  rhs[n] = make_float4(-g.x, -g.y, -g.z, 0.f);
}

// A half-space bound: the step may move against m.xyz by at most m.w (step.wgsl:62-65).
__device__ __forceinline__ float3 boundStep(float3 d, float4 m) {
  float approach = -dot3(d, f3(m));
  return approach > m.w ? d + (approach - m.w) * f3(m) : d;
}
// floorLowest (common.wgsl:262-265).
__device__ __forceinline__ float floorLowest(float zLin, float fz, float delta, float half, float sWeight) {
  float s = fmaxf(delta - (zLin - fz), 0.f);
  return fminf(fmaxf(fz + delta - fmaxf(sWeight, 2.f * s), fz + half), zLin);
}
// The step d of node n bounded against the floor, from its iterate step lin (floorBound, step.wgsl:78-86).
__device__ __forceinline__ float3 floorBound(const StepArgs& A, const SimParams& P, int n, float3 lin, float3 d) {
  if (!P.floorOn) return d;
  const DLayer& L = A.layers[A.nodes[n].layer];
  float half = 0.5f * L.thickness;
  float delta = half + P.floorBulge;
  float gmag = sqrtf(P.gx * P.gx + P.gy * P.gy + P.gz * P.gz);
  float sWeight = sqrtf(A.nodes[n].mass * gmag * delta / P.floorStiffness);
  float z0 = A.x[n].z;
  float lowest = floorLowest(z0 + lin.z, P.floorZ, delta, half, sWeight);
  return make_float3(d.x, d.y, fmaxf(d.z, lowest - z0));
}
__device__ __forceinline__ float3 feasible(const StepArgs& A, int n, float3 d) {
  if (!A.cmeta) return d;
  float4 own = A.cmeta[2 * n], recip = A.cmeta[2 * n + 1];
  return boundStep(boundStep(boundStep(d, own), recip), own);
}

// After contact detection: the predicted step made feasible (projectStart, step.wgsl:90-95).
__global__ void k_project_start(StepArgs A) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= A.N || A.pinned[n]) return;
  const SimParams P = *A.P;
  float4 d = A.dx[n];
  float3 nd = floorBound(A, P, n, make_float3(0, 0, 0), feasible(A, n, f3(d)));
  A.dx[n] = make_float4(nd.x, nd.y, nd.z, d.w);
}

__global__ void k_newton_apply(StepArgs A, const float4* __restrict__ delta, int iteration) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n == 0) atomicAdd(&A.counters[CNT_NEWTON], 1u);
  if (n >= A.N || A.pinned[n]) return;
  const SimParams P = *A.P;
  float3 old = f3(A.dx[n]);
  float alpha = A.scal->lineAlpha;
  float3 dl = f3(delta[n]);
  float3 dn = (finite3(dl) && finite1(alpha)) ? dl : make_float3(0, 0, 0);
  float3 step = alpha * dn;
  // curveApply (energy.wgsl:293-302): a detached piece's node moves along the rotation of its rigid start
  if (A.curveW && alpha > 0.f) {
    const float4 w = A.curveW[n];
    if (w.w > 0.f) step += rotationCurve(alpha * f3(w), f3(A.curveR[n]));
  }
  float3 nd = floorBound(A, P, n, old, feasible(A, n, old + step));
  float upd = len3(nd - old);
  A.dx[n] = make_float4(nd.x, nd.y, nd.z, upd);
  atomicMax(&A.counters[CNT_UPDATE + iteration], __float_as_uint(upd));
}

__global__ void k_commit(StepArgs A) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= A.N) return;
  const SimParams P = *A.P;
  float4 d = A.dx[n];
  A.dx[n] = make_float4(0, 0, 0, 0);
  float4 xn = A.x[n];
  A.v[n] = make_float4(d.x / P.h, d.y / P.h, d.z / P.h, d.w);
  atomicMax(&A.counters[CNT_MAXSPEED], __float_as_uint(len3(f3(d)) / P.h));
  A.x[n] = make_float4(xn.x + d.x, xn.y + d.y, xn.z + d.z, xn.w);
}

// gate (gate.wgsl:12-23): the next optional Newton iteration runs only while iteration `prev` moved
// some node by more than the tolerance (the graph's conditional node reads the decision).
__global__ void k_gate(const uint32_t* __restrict__ counters, int prev, const SimParams* __restrict__ P, cudaGraphConditionalHandle h) {
  const float moved = __uint_as_float(counters[CNT_UPDATE + prev]);
  cudaGraphSetConditional(h, moved > P->newtonTol ? 1u : 0u);
}

}  // namespace btd
