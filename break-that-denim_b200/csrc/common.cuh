// Device-side definitions shared by the solve's kernels: HBM layouts, symmetric 3x3 block algebra,
// the constitutive laws in FP32 (the reference's GPU precision), and lattice helpers.
//
// Layouts (all arrays live in HBM, structure-of-arrays so a warp's loads are contiguous):
//   node state   x, v, dx, pred: float4 per node (x.w: 0; v.w / dx.w: last Newton update)
//   node static  NodeStatic per node (lattice coordinate, layer, mass, crossing normal force)
//   spans        Seg per span 2 n + f (rest, intact, cut mask, flags) + cold arrays (softening, fail site)
//   fine rows    15 float4 planes, plane p of node n at op[p * N + n]: 9 symmetric blocks (6 floats:
//                xx xy xz yy yz zz) in the order diag, +u, -u, +v, -v, +u+v, -u-v, -u+v, +u-v, then the
//                four scalar bending couplings +2u, -2u, +2v, -2v (232 algorithmic bytes per node)
//   coarse rows  38 float4 planes: 25 symmetric blocks in offset order (dj + 2) * 5 + (di + 2)
//                (600 algorithmic bytes per node)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace btd {

constexpr uint32_t SEG_EXISTS = 1u, SEG_BROKEN = 2u, SEG_SLIPPED = 8u;
constexpr int FINE_PLANES = 15;
constexpr int COARSE_PLANES = 38;
constexpr int MAX_NEWTON = 8;

struct DYarn {
  float eaLow, eaHigh, crimpStrain, eaCompress, axialVisc, bendRigidity, bendVisc, yarnsPerSpan;
};

// One layer of the fine lattice: extents, bundled material (LayerMat, common.wgsl:15-23) and its
// yarn-field layout (yarnField.ts:47-66).
struct DLayer {
  int offset, nx, ny, nodeCount;
  DYarn yarn[2];
  float shearStiffness, crossingFriction, crossingWrap, pitchU;
  float pitchV, airDrag, crossingNormal0, thickness;
  int fOffset, K, M, bu;
  int bv, reachU, reachV, pad0;
  float weavePitchU, weavePitchV, pad1, pad2;
};

struct DLevelLayer {
  int offset, nx, ny, pad;
};

struct NodeStatic {
  uint32_t ij;     // i | j << 16
  uint32_t layer;  // layer index
  float mass;
  float n0;        // crossing normal force at zero tension (wear-reduced), N
};

struct Seg {
  float rest;
  float intact;
  uint32_t cutMask;
  uint32_t flags;
};

// Uniform parameters read by every kernel (device memory, so host setters need no re-capture).
struct SimParams {
  float h, gx, gy, gz;
  int historyOn;
  float historyTol;
  int floorOn;
  float floorZ;
  float floorBulge, floorStiffness, floorFriction, floorFrictionSpeed;
  int pcgMax;
  int lineSearch;
  double pcgTol;
  float newtonTol;
  int gradFp64;  // the nonlinear residual (the Newton right-hand side) evaluated in FP64
  int pcgFlex;   // PCG's beta in the flexible (Polak-Ribiere) form, robust to an inexact preconditioner
  int pad2;
};

// Device-side scalars of one Newton iteration (FP64 dots, alpha/beta, convergence state).
struct Scalars {
  double rz, rzNew, pAp, alpha, beta, r0, rr, rel;
  double e[4], m[4];
  int pcgIt, converged, lineAlphaIdx, pad;
  int check;    // the recurrence residual met the tolerance: the true residual decides
  int restart;  // the residual was replaced by the true one: the next direction starts afresh
  int pad4, pad5;
  float lineAlpha;
  float pad1, pad2, pad3;
};

// Counters slots (include/btd.h): [0] ruptures [1] pulled [2] max speed [3] alpha [4+k] max update,
// [12] rejections, [16] PCG iterations last, [17] PCG iterations total, [18] Newton iterations,
// [19] last relative residual (f32 bits), [20] device error flags.
constexpr int CNT_RUPTURES = 0, CNT_PULLED = 1, CNT_MAXSPEED = 2, CNT_ALPHA = 3, CNT_UPDATE = 4, CNT_REJECT = 12,
              CNT_PCG_LAST = 16, CNT_PCG_TOTAL = 17, CNT_NEWTON = 18, CNT_REL = 19, CNT_ERROR = 20, CNT_REL_MAX = 21,
              CNT_PCG_MISSED = 22, CNT_SIZE = 32;

// ---------------------------------------------------------------------------------------------- Sym

struct Sym {
  float xx, xy, xz, yy, yz, zz;
};

__device__ __forceinline__ Sym symZero() { return {0, 0, 0, 0, 0, 0}; }
__device__ __forceinline__ Sym symId(float s) { return {s, 0, 0, s, 0, s}; }
__device__ __forceinline__ Sym operator+(Sym a, Sym b) {
  return {a.xx + b.xx, a.xy + b.xy, a.xz + b.xz, a.yy + b.yy, a.yz + b.yz, a.zz + b.zz};
}
__device__ __forceinline__ Sym operator*(Sym a, float s) { return {a.xx * s, a.xy * s, a.xz * s, a.yy * s, a.yz * s, a.zz * s}; }
__device__ __forceinline__ float3 operator*(Sym a, float3 v) {
  return make_float3(a.xx * v.x + a.xy * v.y + a.xz * v.z, a.xy * v.x + a.yy * v.y + a.yz * v.z,
                     a.xz * v.x + a.yz * v.y + a.zz * v.z);
}
__device__ __forceinline__ bool symIsZero(Sym a) {
  return a.xx == 0.f && a.xy == 0.f && a.xz == 0.f && a.yy == 0.f && a.yz == 0.f && a.zz == 0.f;
}
__device__ __forceinline__ float symFrob(Sym a) {
  return sqrtf(a.xx * a.xx + a.yy * a.yy + a.zz * a.zz + 2.f * (a.xy * a.xy + a.xz * a.xz + a.yz * a.yz));
}
// kPar e e^T + kPerp (I - e e^T)
__device__ __forceinline__ Sym axialBlock(float kPar, float kPerp, float3 e) {
  float d = kPar - kPerp;
  return {d * e.x * e.x + kPerp, d * e.x * e.y, d * e.x * e.z, d * e.y * e.y + kPerp, d * e.y * e.z, d * e.z * e.z + kPerp};
}

// PSD projection of a symmetric 3 x 3 block by eigen-clamping in FP64: the cyclic Jacobi method (Golub
// and Van Loan, Matrix Computations, section 8.5: plane rotations zeroing the off-diagonal entries in
// row order, repeated until they vanish against the diagonal) gives A = V diag(l) V^T; the projection is
// V diag(max(l, 0)) V^T. a and out: xx xy xz yy yz zz.
__device__ __forceinline__ void eigenClamp3(const double (&a)[6], double (&out)[6]) {
  double A[3][3] = {{a[0], a[1], a[2]}, {a[1], a[3], a[4]}, {a[2], a[4], a[5]}};
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 12; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (!(off > 1e-32 * dia)) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (A[p][q] == 0.0) continue;
        // rotation (c, s) with t = tan of the angle that zeroes A[p][q]
        const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {  // A <- A J (columns p, q)
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {  // A <- J^T A (rows p, q)
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {  // V <- V J
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  const double l[3] = {fmax(A[0][0], 0.0), fmax(A[1][1], 0.0), fmax(A[2][2], 0.0)};
  auto e = [&](int r, int c) { return V[r][0] * l[0] * V[c][0] + V[r][1] * l[1] * V[c][1] + V[r][2] * l[2] * V[c][2]; };
  out[0] = e(0, 0), out[1] = e(0, 1), out[2] = e(0, 2), out[3] = e(1, 1), out[4] = e(1, 2), out[5] = e(2, 2);
}

// Symmetric 3 x 3 block in FP64 (xx xy xz yy yz zz).
struct SymD {
  double xx, xy, xz, yy, yz, zz;
};
__device__ __forceinline__ SymD symD(const Sym& a) { return {a.xx, a.xy, a.xz, a.yy, a.yz, a.zz}; }
__device__ __forceinline__ SymD symZeroD() { return {0, 0, 0, 0, 0, 0}; }
__device__ __forceinline__ SymD symIdD(double s) { return {s, 0, 0, s, 0, s}; }
__device__ __forceinline__ SymD operator+(SymD a, SymD b) {
  return {a.xx + b.xx, a.xy + b.xy, a.xz + b.xz, a.yy + b.yy, a.yz + b.yz, a.zz + b.zz};
}
__device__ __forceinline__ SymD operator*(SymD a, double s) { return {a.xx * s, a.xy * s, a.xz * s, a.yy * s, a.yz * s, a.zz * s}; }
__device__ __forceinline__ Sym symF(const SymD& a) {
  return {(float)a.xx, (float)a.xy, (float)a.xz, (float)a.yy, (float)a.yz, (float)a.zz};
}
// kPar e e^T + kPerp (I - e e^T) with e a unit vector, in FP64: exactly PSD for kPar, kPerp >= 0.
__device__ __forceinline__ SymD axialBlockD(double kPar, double kPerp, double ex, double ey, double ez) {
  const double d = kPar - kPerp;
  return {d * ex * ex + kPerp, d * ex * ey, d * ex * ez, d * ey * ey + kPerp, d * ey * ez, d * ez * ez + kPerp};
}

// The spring block of a near-degenerate element (a span or shear diagonal collapsed to under 1 % of its
// rest length, where the closed-form projection's FP32 direction loses its digits or is undefined): the
// exact Hessian K e e^T + (f / l) (I - e e^T) of the spring energy, formed in FP64 from the element
// vector d (FP64) and eigen-clamped; a zero-length element gets max(K, 0) I.
__device__ __forceinline__ SymD springBlockFP64D(double K, double f, double dx, double dy, double dz) {
  const double l = sqrt(dx * dx + dy * dy + dz * dz);
  if (!(l > 0.0)) return symIdD(fmax(K, 0.0));
  const double ex = dx / l, ey = dy / l, ez = dz / l, kp = f / l, d = K - kp;
  const double a[6] = {d * ex * ex + kp, d * ex * ey, d * ex * ez, d * ey * ey + kp, d * ey * ez, d * ez * ez + kp};
  double o[6];
  eigenClamp3(a, o);
  return {o[0], o[1], o[2], o[3], o[4], o[5]};
}
__device__ __forceinline__ Sym springBlockFP64(double K, double f, double dx, double dy, double dz) {
  return symF(springBlockFP64D(K, f, dx, dy, dz));
}

// ---------------------------------------------------------------------------------------------- float3

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3& operator+=(float3& a, float3 b) {
  a.x += b.x, a.y += b.y, a.z += b.z;
  return a;
}
__device__ __forceinline__ float3& operator-=(float3& a, float3 b) {
  a.x -= b.x, a.y -= b.y, a.z -= b.z;
  return a;
}
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ bool finite1(float v) { return (__float_as_uint(v) & 0x7f800000u) != 0x7f800000u; }
__device__ __forceinline__ bool finite3(float3 v) { return finite1(v.x) && finite1(v.y) && finite1(v.z); }

// Programmatic dependent launch. A kernel launched with programmatic stream serialisation may start
// while the kernel before it on the stream still runs; pdlWait() returns once that kernel has
// completed and its writes are visible (at once for a kernel launched without the attribute), and
// pdlLaunchNext() lets the next kernel start. Every kernel of the PCG loop calls them in that order,
// first, so what a kernel may read before its own wait is what kernels two or more launches back
// wrote (the smoother's line factors), never its predecessor's output.
__device__ __forceinline__ void pdlWait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdlLaunchNext() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// rotationCurve (common.wgsl:274-283): R(th) r - r - th x r, what rotating r by th adds to its tangent step.
__device__ __forceinline__ float3 rotationCurve(float3 th, float3 r) {
  const float phi = len3(th);
  if (phi < 1e-9f) return make_float3(0, 0, 0);
  const float3 k = (1.f / phi) * th;
  const float3 kr = cross3(k, r), kkr = cross3(k, kr);
  return (sinf(phi) - phi) * kr + (1.f - cosf(phi)) * kkr;
}

// ---------------------------------------------------------------------------------------------- M3

// General 3x3 (row-major) for the line solves.
struct M3 {
  float a[9];
};
__device__ __forceinline__ M3 m3Zero() { return {{0, 0, 0, 0, 0, 0, 0, 0, 0}}; }
__device__ __forceinline__ M3 m3Id() { return {{1, 0, 0, 0, 1, 0, 0, 0, 1}}; }
__device__ __forceinline__ M3 m3FromSym(Sym s) { return {{s.xx, s.xy, s.xz, s.xy, s.yy, s.yz, s.xz, s.yz, s.zz}}; }
__device__ __forceinline__ M3 m3Mul(const M3& x, const M3& y) {
  M3 o;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) o.a[3 * r + c] = x.a[3 * r] * y.a[c] + x.a[3 * r + 1] * y.a[3 + c] + x.a[3 * r + 2] * y.a[6 + c];
  return o;
}
__device__ __forceinline__ M3 m3Sub(const M3& x, const M3& y) {
  M3 o;
#pragma unroll
  for (int q = 0; q < 9; ++q) o.a[q] = x.a[q] - y.a[q];
  return o;
}
__device__ __forceinline__ M3 m3Neg(const M3& x) {
  M3 o;
#pragma unroll
  for (int q = 0; q < 9; ++q) o.a[q] = -x.a[q];
  return o;
}
__device__ __forceinline__ float3 m3Vec(const M3& x, float3 v) {
  return make_float3(x.a[0] * v.x + x.a[1] * v.y + x.a[2] * v.z, x.a[3] * v.x + x.a[4] * v.y + x.a[5] * v.z,
                     x.a[6] * v.x + x.a[7] * v.y + x.a[8] * v.z);
}
// Inverse of a pivot block shifted by 2e-6 of its largest diagonal entry, with the diagonal fallback
// for a non-finite result (pivotInverse, common.wgsl:140-150; PIVOT_SHIFT, newtonMultigrid.ts:414).
__device__ __forceinline__ M3 pivotInverse(const M3& m) {
  float s = fmaxf(fmaxf(fabsf(m.a[0]), fabsf(m.a[4])), fabsf(m.a[8]));
  float e = 2e-6f * s + 1e-30f;
  float a00 = m.a[0] + e, a01 = m.a[1], a02 = m.a[2];
  float a10 = m.a[3], a11 = m.a[4] + e, a12 = m.a[5];
  float a20 = m.a[6], a21 = m.a[7], a22 = m.a[8] + e;
  float c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
  float det = a00 * c00 + a01 * c01 + a02 * c02;
  float id = __frcp_rn(det);
  M3 o = {{c00 * id, (a02 * a21 - a01 * a22) * id, (a01 * a12 - a02 * a11) * id, c01 * id, (a00 * a22 - a02 * a20) * id,
           (a02 * a10 - a00 * a12) * id, c02 * id, (a01 * a20 - a00 * a21) * id, (a00 * a11 - a01 * a10) * id}};
  bool ok = true;
#pragma unroll
  for (int q = 0; q < 9; ++q) ok = ok && finite1(o.a[q]);
  if (!ok) {
    float d = 1.f / fmaxf(s, 1e-30f);
    o = {{d, 0, 0, 0, d, 0, 0, 0, d}};
  }
  return o;
}

// ---------------------------------------------------------------------------------------------- laws

// Axial J-curve (axial.ts:16-42; common.wgsl:80-104).
__device__ __forceinline__ float axialTension(const DYarn& y, float eps) {
  if (eps <= 0.f) return y.eaCompress * eps;
  float ec = y.crimpStrain, dk = y.eaHigh - y.eaLow;
  if (eps <= ec) return y.eaLow * eps + dk * eps * eps / (2.f * ec);
  return y.eaLow * ec + dk * ec * 0.5f + y.eaHigh * (eps - ec);
}
__device__ __forceinline__ float axialStiffness(const DYarn& y, float eps) {
  if (eps <= 0.f) return y.eaCompress;
  float ec = y.crimpStrain;
  if (eps <= ec) return y.eaLow + (y.eaHigh - y.eaLow) * eps / ec;
  return y.eaHigh;
}
__device__ __forceinline__ float axialEnergyDensity(const DYarn& y, float eps) {
  if (eps <= 0.f) return 0.5f * y.eaCompress * eps * eps;
  float ec = y.crimpStrain, dk = y.eaHigh - y.eaLow;
  if (eps <= ec) return 0.5f * y.eaLow * eps * eps + dk * eps * eps * eps / (6.f * ec);
  float tc = y.eaLow * ec + dk * ec * 0.5f;
  float d = eps - ec;
  return 0.5f * y.eaLow * ec * ec + dk * ec * ec / 6.f + tc * d + 0.5f * y.eaHigh * d * d;
}
__device__ __forceinline__ float strainAtTension(const DYarn& y, float t) {
  float ec = y.crimpStrain, dk = y.eaHigh - y.eaLow;
  float tc = y.eaLow * ec + dk * ec * 0.5f;
  if (t >= tc) return ec + (t - tc) / y.eaHigh;
  float a = dk / (2.f * ec);
  return 2.f * t / (y.eaLow + sqrtf(y.eaLow * y.eaLow + 4.f * a * t));
}
__device__ __forceinline__ float yarnDamage(const DYarn& y, float B, float area, float peakY, float softStrain, float eps) {
  float ep = strainAtTension(y, peakY * B / area);
  if (eps <= ep) return 0.f;
  if (eps >= ep + softStrain) return 1.f;
  float tEnv = peakY * (1.f - (eps - ep) / softStrain);
  float tEl = area * axialTension(y, eps) / B;
  return fminf(fmaxf(1.f - tEnv / fmaxf(tEl, 1e-12f), 0.f), 1.f);
}

// Fold-stiffening bending (laws.ts:15-103; common.wgsl:156-210).
constexpr float BEND_S0 = 0.85f;
__device__ __forceinline__ float3 bendPsi(float q, float a) {
  float s = q / a;
  if (s < BEND_S0) {
    float d = 1.f - s;
    return make_float3(q / d, 1.f / (d * d), 2.f / (a * d * d * d));
  }
  float d0 = 1.f - BEND_S0, q0 = BEND_S0 * a;
  float p1 = 1.f / (d0 * d0), p2 = 2.f / (a * d0 * d0 * d0);
  float t = q - q0;
  return make_float3(q0 / d0 + p1 * t + 0.5f * p2 * t * t, p1 + p2 * t, p2);
}
// (wa, wc, 1 / (Lh^2 l), fold scale 4 Lh^2)
__device__ __forceinline__ float4 bendGeometry(float La, float Lc) {
  float s = La + Lc;
  float lh = 2.f * La * Lc / s;
  return make_float4(2.f * Lc / s, 2.f * La / s, 1.f / (lh * lh * 0.5f * s), 4.f * lh * lh);
}
__device__ __forceinline__ float bendScale(float ia, float ic, uint32_t maskA, uint32_t maskC, uint32_t B) {
  uint32_t full = B >= 32u ? 0xFFFFFFFFu : ((1u << B) - 1u);
  int cont = __popc(~(maskA | maskC) & full);
  if (cont == 0) return 0.f;
  int ua = __popc(~maskA & full), uc = __popc(~maskC & full);
  float fb = float(B);
  float ma = ua > 0 ? ia * fb / float(ua) : 0.f;
  float mc = uc > 0 ? ic * fb / float(uc) : 0.f;
  return float(cont) / fb * fminf(ma, mc);
}
__device__ __forceinline__ float bendPsiDelta(float q0, float q1, float dq, float a) {
  float s0 = q0 / a, s1 = q1 / a;
  if (s0 < BEND_S0 && s1 < BEND_S0) return dq / ((1.f - s0) * (1.f - s1));
  float qb = BEND_S0 * a, d0 = 1.f - BEND_S0;
  float p1 = 1.f / (d0 * d0), p2 = 2.f / (a * d0 * d0 * d0);
  if (s0 >= BEND_S0 && s1 >= BEND_S0) return dq * (p1 + 0.5f * p2 * ((q0 - qb) + (q1 - qb)));
  float lo = fminf(q0, q1);
  float t = fmaxf(q0, q1) - qb;
  float up = (qb - lo) / ((1.f - lo / a) * d0) + t * (p1 + 0.5f * p2 * t);
  return q1 >= q0 ? up : -up;
}

// Shear-locking diagonal (laws.ts:197-244; common.wgsl:212-242).
constexpr float SHEAR_JAM = 0.16f, SHEAR_RAMP = 0.08f, SHEAR_LOCK = 40.f;
__device__ __forceinline__ float shearJam(float area) {
  // SHEAR_COS0 = sqrt(1 - (1 - (1 - JAM)^2)^2)
  const float j1 = (1.f - SHEAR_JAM) * (1.f - SHEAR_JAM);
  const float cos0 = sqrtf(1.f - (1.f - j1) * (1.f - j1));
  float c = cos0 * sqrtf(fminf(fmaxf(area, 0.02f), 1.f));
  return 1.f - sqrtf(1.f - sqrtf(1.f - c * c));
}
__device__ __forceinline__ float cellArea(float cu, float tu, float cv, float rv) {
  return fmaxf(0.5f * (cu + tu), 0.5f * (cv + rv));
}
// (force, tangent)
__device__ __forceinline__ float2 shearLaw(float ks, float jam, float Ld, float l) {
  float f = ks * (l - Ld), k = ks;
  float c = (Ld - l) / Ld - jam;
  if (c > 0.f) {
    float extra = ks * (SHEAR_LOCK - 1.f);
    if (c < SHEAR_RAMP) {
      f -= extra * Ld * c * c / (2.f * SHEAR_RAMP);
      k += extra * c / SHEAR_RAMP;
    } else {
      f -= extra * Ld * (c - 0.5f * SHEAR_RAMP);
      k += extra;
    }
  }
  return make_float2(f, k);
}

__device__ __forceinline__ bool segActive(const Seg& s) { return (s.flags & (SEG_EXISTS | SEG_BROKEN)) == SEG_EXISTS; }

// ---------------------------------------------------------------------------------------------- rows

// Offsets of the fine row's couplings 0..11 (+u, -u, +v, -v, +u+v, -u-v, -u+v, +u-v, +2u, -2u, +2v, -2v).
__device__ __forceinline__ int2 fineOffset(int k) {
  const int di[12] = {1, -1, 0, 0, 1, -1, -1, 1, 2, -2, 0, 0};
  const int dj[12] = {0, 0, 1, -1, 1, -1, 1, -1, 0, 0, 2, -2};
  return make_int2(di[k], dj[k]);
}
// Coupling index of a fine offset, or -1 outside the fine stencil.
__device__ __forceinline__ int fineCoupling(int di, int dj) {
  if (dj == 0) {
    if (di == 1) return 0;
    if (di == -1) return 1;
    if (di == 2) return 8;
    if (di == -2) return 9;
    return -1;
  }
  if (di == 0) {
    if (dj == 1) return 2;
    if (dj == -1) return 3;
    if (dj == 2) return 10;
    if (dj == -2) return 11;
    return -1;
  }
  if (di == 1 && dj == 1) return 4;
  if (di == -1 && dj == -1) return 5;
  if (di == -1 && dj == 1) return 6;
  if (di == 1 && dj == -1) return 7;
  return -1;
}

// Symmetric block starting at float index f of a plane-major row (planes of N float4).
__device__ __forceinline__ Sym loadSymAt(const float4* __restrict__ op, int N, int n, int f) {
  const float4 a = __ldg(&op[(size_t)(f >> 2) * N + n]);
  const float4 b = __ldg(&op[(size_t)((f >> 2) + 1) * N + n]);
  if ((f & 3) == 0) return {a.x, a.y, a.z, a.w, b.x, b.y};
  return {a.z, a.w, b.x, b.y, b.z, b.w};
}

// Fine row: block k (0 diag, 1..8 couplings 0..7), scalars k = 8..11.
__device__ __forceinline__ Sym fineBlock(const float4* __restrict__ op, int N, int n, int b) { return loadSymAt(op, N, n, 6 * b); }
__device__ __forceinline__ float fineScalar(const float4* __restrict__ op, int N, int n, int s) {
  // floats 54..57: plane 13 .zw, plane 14 .xy
  if (s < 2) {
    float4 a = __ldg(&op[(size_t)13 * N + n]);
    return s == 0 ? a.z : a.w;
  }
  float4 a = __ldg(&op[(size_t)14 * N + n]);
  return s == 2 ? a.x : a.y;
}
// Coupling k (0..11) of a fine row as a symmetric block.
__device__ __forceinline__ Sym fineCouplingBlock(const float4* __restrict__ op, int N, int n, int k) {
  if (k < 8) return fineBlock(op, N, n, k + 1);
  return symId(fineScalar(op, N, n, k - 8));
}
// Coarse row: block of offset index o = (dj + 2) * 5 + (di + 2).
__device__ __forceinline__ Sym coarseBlock(const float4* __restrict__ op, int N, int n, int o) { return loadSymAt(op, N, n, 6 * o); }

// The fine row in FP64, the operator PCG solves with: the same 58 values as the fp32 row (value v in
// plane v / 2 of N double2), its element blocks exactly PSD in FP64 and summed in FP64, so that a row's
// stiff terms cancel on a rigid translation as they do in exact arithmetic.
constexpr int FINE64_PLANES = 29;
__device__ __forceinline__ SymD loadSymD(const double2* __restrict__ op, int N, int n, int f) {
  const double2 a = __ldg(&op[(size_t)(f >> 1) * N + n]), b = __ldg(&op[(size_t)((f >> 1) + 1) * N + n]),
                c = __ldg(&op[(size_t)((f >> 1) + 2) * N + n]);
  return {a.x, a.y, b.x, b.y, c.x, c.y};
}
// Coupling k (0..11) of an FP64 fine row; k = -1 the diagonal block.
__device__ __forceinline__ SymD fine64Block(const double2* __restrict__ op, int N, int n, int k) {
  if (k < 8) return loadSymD(op, N, n, 6 * (k + 1));
  const double2 a = __ldg(&op[(size_t)(27 + ((k - 8) >> 1)) * N + n]);
  return symIdD(((k - 8) & 1) ? a.y : a.x);
}
__device__ __forceinline__ void symDVecAdd(const SymD& A, const double* x, double& y0, double& y1, double& y2) {
  y0 += A.xx * x[0] + A.xy * x[1] + A.xz * x[2];
  y1 += A.xy * x[0] + A.yy * x[1] + A.yz * x[2];
  y2 += A.xz * x[0] + A.yz * x[1] + A.zz * x[2];
}

__device__ __forceinline__ void storeSymAt(float* row, int f, Sym s) {
  row[f] = s.xx, row[f + 1] = s.xy, row[f + 2] = s.xz, row[f + 3] = s.yy, row[f + 4] = s.yz, row[f + 5] = s.zz;
}

// Lower Cholesky factor of a symmetric 3 x 3 block (6 entries xx xy xz yy yz zz) in FP64: L00, L10, L11,
// L20, L21, L22; false unless positive definite.
__device__ __forceinline__ bool chol3d(const Sym& D, double (&L)[6]) {
  const double a = D.xx;
  if (!(a > 0.0)) return false;
  L[0] = sqrt(a);
  L[1] = D.xy / L[0];
  L[3] = D.xz / L[0];
  const double c = D.yy - L[1] * L[1];
  if (!(c > 0.0)) return false;
  L[2] = sqrt(c);
  L[4] = (D.yz - L[3] * L[1]) / L[2];
  const double e = D.zz - L[3] * L[3] - L[4] * L[4];
  if (!(e > 0.0)) return false;
  L[5] = sqrt(e);
  return true;
}

// Level geometry passed by value to kernels.
struct DLevel {
  int N;
  int nLayers;
  DLevelLayer one;  // the level's layer when it has a single one (nx = 0 otherwise): positions follow
                    // from the node index, with no table lookup
  const DLevelLayer* __restrict__ layers;
  const uint2* __restrict__ coord;  // (i | j << 16, layer)
  float4* op;
  uint32_t* fixed;
  float4* X;
  float4* B;
  float4* R;
  float4* pw;  // prolongation weights to the next coarser level (slot ki + 2 kj)
};

__device__ __forceinline__ int levelNode(const DLevelLayer& L, int i, int j) {
  if (i < 0 || j < 0 || i >= L.nx || j >= L.ny) return -1;
  return L.offset + j * L.nx + i;
}

// Coarse index set of one coarsening: every second index plus the last (lattice.ts:12-41).
__device__ __forceinline__ int coarseCount(int n) { return n / 2 + 1; }
__device__ __forceinline__ int coarseToFine(int I, int n) { return min(2 * I, n - 1); }
struct Bracket {
  int lo, hi;
  float wlo, whi;
};
__device__ __forceinline__ Bracket bracketOf(int i, int n) {
  int nc = coarseCount(n);
  int lo = min(nc - 1, i >> 1);
  if (coarseToFine(lo, n) > i) lo--;
  int a = coarseToFine(lo, n);
  if (a == i) return {lo, lo, 1.f, 0.f};
  int b = coarseToFine(lo + 1, n);
  float inv = 1.f / float(b - a);
  return {lo, lo + 1, float(b - i) * inv, float(i - a) * inv};
}

}  // namespace btd
