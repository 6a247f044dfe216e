// Detached pieces' rigid modes (rigid_frame.wgsl, rigid_apply.wgsl, rigid_spin.wgsl; solver.ts:612-716).
// A detached piece's rigid motion is resisted only by its inertia, drag and contact, against yarn
// couplings far stiffer, and the multigrid hierarchy does not carry those near-null modes. Each piece's
// six rigid modes Z (translation, rotation about its mass centroid) give PCG an exact start
// x0 = Z E^-1 Z^T b, E = Z^T A Z built from what each term puts on a rigid motion (the external blocks
// fully, the internal terms only on rotation through their tension's geometric stiffness); the line
// search and the update move a piece's nodes along the rotation of that start instead of its tangent;
// each substep starts a spinning piece on its rotation continued over the substep. Pieces come from the
// host (the topology analysis); with none, nothing here runs.
//
// Kernels: k_rigid_rotation (per node: the rotation stiffness of the internal terms it owns),
// k_rigid_frame (a CTA per piece: mass centroid, E in FP64, its regularised inverse), k_rigid_start
// (a CTA per piece: force and torque of the right-hand side, the rigid step), the PCG start itself in
// k_pcg_init_rigid (k_pcg.cuh), k_rigid_curves (per node: the rotation its step bends along),
// k_spin_reduce / k_spin_apply (the spin start of a substep).
#pragma once

#include "common.cuh"
#include "k_step.cuh"

namespace btd {

constexpr uint32_t NO_PIECE = 0xFFFFFFFFu;
constexpr int MAX_PIECES = 4096;  // solver.ts:86
constexpr int RIGID_THREADS = 256;

struct RigidArgs {
  int count;
  const uint32_t* __restrict__ pieceOf;  // N: piece of each node or NO_PIECE
  const uint32_t* __restrict__ start;    // count + 1
  const uint32_t* __restrict__ nodes;    // start[count]
  float* kx;       // 6 per node: external block (xx xy xz yy yz zz), written by the assembly
  float* kr;       // 6 per node: rotation stiffness of the internal terms it owns
  double* frame;   // 40 per piece: centroid (3), valid, E^-1 row-major (36)
  double* step;    // 6 per piece: rigid step (t, w); in the predictor (centroid, spin rotation)
  float4* curveW;  // per node: the piece's rotation of the direction (w: 1 on, 0 off)
  float4* curveR;  // per node: the arm from the centroid at the iterate
};

__device__ __forceinline__ bool inPiece(const RigidArgs& R, int n) { return R.count > 0 && R.pieceOf[n] < (uint32_t)R.count; }

// kPerp (|d|^2 I - d d^T): a rigid rotation w moves the ends of a term's vector d by w x d, which a
// spring block of transverse stiffness kPerp resists so (rotationOfSpring, assemble.wgsl:20-26).
__device__ __forceinline__ void addRotationOfSpring(float k, float3 d, float (&K)[6]) {
  const float l2 = dot3(d, d);
  K[0] += k * (l2 - d.x * d.x);
  K[1] -= k * d.x * d.y;
  K[2] -= k * d.x * d.z;
  K[3] += k * (l2 - d.y * d.y);
  K[4] -= k * d.y * d.z;
  K[5] += k * (l2 - d.z * d.z);
}

// The rotation stiffness of the internal terms node n owns (assemble.wgsl:245, 255, 301): its span to
// the next node along each family, the bending triple centred on it, and the two shear diagonals it is
// the lower end of (of its own cell, to the +u+v corner; of the cell below, to that cell's +u corner).
__global__ void k_rigid_rotation(StepArgs A, RigidArgs R) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= A.N || !inPiece(R, n) || A.pinned[n]) return;
  const SimParams P = *A.P;
  const NodeStatic st = A.nodes[n];
  const int i = st.ij & 0xFFFF, j = st.ij >> 16;
  const DLayer& L = A.layers[st.layer];
  float K[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    const int du = f == 0 ? 1 : 0, dv = f == 1 ? 1 : 0;
    const int prev = nodeAt(L, i - du, j - dv), next = nodeAt(L, i + du, j + dv);
    if (next >= 0 && activeSpan(A.segs, n, f)) {
      const SegForce s = segForce(A, n, next, f, L, P.h);
      addRotationOfSpring(fmaxf(s.fs, 0.f) / s.l, s.l * s.e, K);
    }
    if (prev >= 0 && next >= 0 && activeSpan(A.segs, prev, f) && activeSpan(A.segs, n, f)) {
      const Triple t = tripleAt(A, prev, n, next, f, L, P.h);
      addRotationOfSpring(t.k, t.r, K);
    }
  }
  const int cells[2][3] = {{i, j, 0}, {i, j - 1, 1}};
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int ci = cells[q][0], cj = cells[q][1], d = cells[q][2];
    if (cj < 0 || !diagActive(A.segs, L, ci, cj, d)) continue;
    const int other = d == 0 ? nodeAt(L, ci + 1, cj + 1) : nodeAt(L, ci + 1, cj);
    const float3 e = (f3(A.x[other]) - f3(A.x[n])) + (f3(A.dx[other]) - f3(A.dx[n]));
    const float len = len3(e);
    const float2 cs = cellShear(A, L, ci, cj);
    const float2 sl = shearLaw(cs.x, cs.y, shearRest(A, L, ci, cj), len);
    addRotationOfSpring(fmaxf(sl.x, 0.f) / len, e, K);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) R.kr[6 * n + q] = K[q];
}

// Block sum of NV doubles over a CTA of RIGID_THREADS; the totals in thread 0.
template <int NV>
__device__ __forceinline__ void rigidBlockSum(double (&v)[NV], double (*sh)[NV]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    if (lane == 0) sh[warp][q] = v[q];
  }
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int w = 0; w < RIGID_THREADS / 32; ++w) s += sh[w][q];
      v[q] = s;
    }
  __syncthreads();
}

__device__ __forceinline__ int triIdx(int i, int j) { return i * 6 - (i * (i + 1)) / 2 + j; }

// rigidFrame (rigid_frame.wgsl:56-161): per piece the mass centroid at the iterate and E = Z^T K Z over
// its nodes' external blocks, plus their internal rotation stiffness on the rotation block; the rotation
// block regularised relative to its scale, then E^-1 through a Cholesky factor (zero when E is not
// positive definite). One CTA per piece.
__global__ void __launch_bounds__(RIGID_THREADS) k_rigid_frame(StepArgs A, RigidArgs R) {
  __shared__ double sh4[RIGID_THREADS / 32][4];
  __shared__ double sh21[RIGID_THREADS / 32][21];
  __shared__ double cen[4];
  const int p = blockIdx.x;
  const uint32_t a = R.start[p], b = R.start[p + 1];
  double m[4] = {0, 0, 0, 0};
  for (uint32_t k = a + threadIdx.x; k < b; k += RIGID_THREADS) {
    const int n = (int)R.nodes[k];
    const double mass = A.nodes[n].mass;
    const float4 x = A.x[n], d = A.dx[n];
    m[0] += mass * ((double)x.x + d.x);
    m[1] += mass * ((double)x.y + d.y);
    m[2] += mass * ((double)x.z + d.z);
    m[3] += mass;
  }
  rigidBlockSum<4>(m, sh4);
  if (threadIdx.x == 0) {
    for (int z = 0; z < 3; ++z) cen[z] = m[3] > 0.0 ? m[z] / m[3] : 0.0;
    cen[3] = m[3];
  }
  __syncthreads();
  double e[21];
#pragma unroll
  for (int q = 0; q < 21; ++q) e[q] = 0.0;
  for (uint32_t k = a + threadIdx.x; k < b; k += RIGID_THREADS) {
    const int n = (int)R.nodes[k];
    if (A.pinned[n]) continue;
    const float* kx = R.kx + 6 * n;
    const double K[9] = {kx[0], kx[1], kx[2], kx[1], kx[3], kx[4], kx[2], kx[4], kx[5]};
    const float4 x = A.x[n], d = A.dx[n];
    const double r[3] = {(double)x.x + d.x - cen[0], (double)x.y + d.y - cen[1], (double)x.z + d.z - cen[2]};
    // Z columns: unit translations, then e_i x r
    double Z[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, -r[2], r[1]}, {r[2], 0, -r[0]}, {-r[1], r[0], 0}};
    for (int i = 0; i < 6; ++i) {
      const double KZ[3] = {K[0] * Z[i][0] + K[1] * Z[i][1] + K[2] * Z[i][2], K[3] * Z[i][0] + K[4] * Z[i][1] + K[5] * Z[i][2],
                            K[6] * Z[i][0] + K[7] * Z[i][1] + K[8] * Z[i][2]};
      for (int j = i; j < 6; ++j) e[triIdx(i, j)] += Z[j][0] * KZ[0] + Z[j][1] * KZ[1] + Z[j][2] * KZ[2];
    }
    const float* kr = R.kr + 6 * n;
    e[triIdx(3, 3)] += kr[0], e[triIdx(3, 4)] += kr[1], e[triIdx(3, 5)] += kr[2];
    e[triIdx(4, 4)] += kr[3], e[triIdx(4, 5)] += kr[4], e[triIdx(5, 5)] += kr[5];
  }
  rigidBlockSum<21>(e, sh21);
  if (threadIdx.x != 0) return;
  double* F = R.frame + 40 * (size_t)p;
  F[0] = cen[0], F[1] = cen[1], F[2] = cen[2], F[3] = cen[3] > 0.0 ? 1.0 : 0.0;
  const double st = (e[triIdx(0, 0)] + e[triIdx(1, 1)] + e[triIdx(2, 2)]) / 3;
  const double sr = (e[triIdx(3, 3)] + e[triIdx(4, 4)] + e[triIdx(5, 5)]) / 3;
  const double eps = 1e-6 * fmax(sr, 1e-8 * st) + 1e-30;
  double A6[6][6], Lc[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      A6[i][j] = e[triIdx(min(i, j), max(i, j))];
      Lc[i][j] = 0.0;
    }
  for (int i = 3; i < 6; ++i) A6[i][i] += eps;
  bool ok = st > 0.0;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      double sum = A6[i][j];
      for (int k = 0; k < j; ++k) sum -= Lc[i][k] * Lc[j][k];
      if (i == j) {
        if (sum <= 0.0) ok = false, sum = 1.0;
        Lc[i][i] = sqrt(sum);
      } else {
        Lc[i][j] = sum / Lc[j][j];
      }
    }
  for (int col = 0; col < 6; ++col) {
    double y[6], z6[6];
    for (int i = 0; i < 6; ++i) {
      double sum = i == col ? 1.0 : 0.0;
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

// rigidReduce (rigid_apply.wgsl:37-64): per piece the right-hand side's force and torque about the
// centroid and the rigid step (t, w) = E^-1 (force, torque). One CTA per piece.
__global__ void __launch_bounds__(RIGID_THREADS) k_rigid_start(StepArgs A, RigidArgs R, const float4* __restrict__ b) {
  __shared__ double sh6[RIGID_THREADS / 32][6];
  const int p = blockIdx.x;
  const double* F = R.frame + 40 * (size_t)p;
  double g[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t k = R.start[p] + threadIdx.x; k < R.start[p + 1]; k += RIGID_THREADS) {
    const int n = (int)R.nodes[k];
    const float4 x = A.x[n], d = A.dx[n], bn = b[n];
    const double r[3] = {(double)x.x + d.x - F[0], (double)x.y + d.y - F[1], (double)x.z + d.z - F[2]};
    g[0] += bn.x, g[1] += bn.y, g[2] += bn.z;
    g[3] += r[1] * bn.z - r[2] * bn.y;
    g[4] += r[2] * bn.x - r[0] * bn.z;
    g[5] += r[0] * bn.y - r[1] * bn.x;
  }
  rigidBlockSum<6>(g, sh6);
  if (threadIdx.x != 0) return;
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
    for (int j = 0; j < 6; ++j) s += F[4 + 6 * i + j] * g[j];
    R.step[6 * p + i] = F[3] > 0.5 ? s : 0.0;
  }
}

// The rigid start of node n (t + w x r on a piece, zero elsewhere; rigidApply, rigid_apply.wgsl:66-87).
__device__ __forceinline__ Dv rigidStartAt(const StepArgs& A, const RigidArgs& R, int n) {
  if (!inPiece(R, n)) return {0.0, 0.0, 0.0};
  const int p = (int)R.pieceOf[n];
  const double* F = R.frame + 40 * (size_t)p;
  const double* q = R.step + 6 * (size_t)p;
  const float4 x = A.x[n], d = A.dx[n];
  const double r[3] = {(double)x.x + d.x - F[0], (double)x.y + d.y - F[1], (double)x.z + d.z - F[2]};
  return {q[0] + q[4] * r[2] - q[5] * r[1], q[1] + q[5] * r[0] - q[3] * r[2], q[2] + q[3] * r[1] - q[4] * r[0]};
}

// curveSet (rigid_spin.wgsl:138-154): per node of a piece with a valid frame, the rotation of the
// direction's rigid start and the node's arm from the centroid at the iterate.
__global__ void k_rigid_curves(StepArgs A, RigidArgs R) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= A.N) return;
  float4 w = make_float4(0, 0, 0, 0), r = make_float4(0, 0, 0, 0);
  if (inPiece(R, n)) {
    const int p = (int)R.pieceOf[n];
    const double* F = R.frame + 40 * (size_t)p;
    if (F[3] > 0.5) {
      const double* q = R.step + 6 * (size_t)p;
      const float4 x = A.x[n], d = A.dx[n];
      w = make_float4((float)q[3], (float)q[4], (float)q[5], 1.f);
      r = make_float4((float)((double)x.x + d.x - F[0]), (float)((double)x.y + d.y - F[1]), (float)((double)x.z + d.z - F[2]), 0.f);
    }
  }
  R.curveW[n] = w;
  R.curveR[n] = r;
}

// spinReduce (rigid_spin.wgsl:44-112): a piece's rotation over the last substep from its angular
// momentum about its centroid, w = I^-1 L (I regularised as the rigid frame), continued over this one:
// step = (centroid, h w). One CTA per piece, on the committed state.
__global__ void __launch_bounds__(RIGID_THREADS) k_spin_reduce(StepArgs A, RigidArgs R) {
  __shared__ double sh7[RIGID_THREADS / 32][7];
  __shared__ double sh9[RIGID_THREADS / 32][9];
  __shared__ double cv[6];
  const int p = blockIdx.x;
  const uint32_t a = R.start[p], b = R.start[p + 1];
  double m[7] = {0, 0, 0, 0, 0, 0, 0};
  for (uint32_t k = a + threadIdx.x; k < b; k += RIGID_THREADS) {
    const int n = (int)R.nodes[k];
    const double mass = A.nodes[n].mass;
    const float4 x = A.x[n], v = A.v[n];
    m[0] += mass;
    m[1] += mass * x.x, m[2] += mass * x.y, m[3] += mass * x.z;
    m[4] += mass * v.x, m[5] += mass * v.y, m[6] += mass * v.z;
  }
  rigidBlockSum<7>(m, sh7);
  if (threadIdx.x == 0)
    for (int z = 0; z < 3; ++z) {
      cv[z] = m[0] > 0.0 ? m[1 + z] / m[0] : 0.0;
      cv[3 + z] = m[0] > 0.0 ? m[4 + z] / m[0] : 0.0;
    }
  __syncthreads();
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // L (3), I xx yy zz xy xz yz
  for (uint32_t k = a + threadIdx.x; k < b; k += RIGID_THREADS) {
    const int n = (int)R.nodes[k];
    const double mass = A.nodes[n].mass;
    const float4 x = A.x[n], v = A.v[n];
    const double r[3] = {x.x - cv[0], x.y - cv[1], x.z - cv[2]}, u[3] = {v.x - cv[3], v.y - cv[4], v.z - cv[5]};
    s[0] += mass * (r[1] * u[2] - r[2] * u[1]);
    s[1] += mass * (r[2] * u[0] - r[0] * u[2]);
    s[2] += mass * (r[0] * u[1] - r[1] * u[0]);
    const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    s[3] += mass * (rr - r[0] * r[0]);
    s[4] += mass * (rr - r[1] * r[1]);
    s[5] += mass * (rr - r[2] * r[2]);
    s[6] -= mass * r[0] * r[1];
    s[7] -= mass * r[0] * r[2];
    s[8] -= mass * r[1] * r[2];
  }
  rigidBlockSum<9>(s, sh9);
  if (threadIdx.x != 0) return;
  const double eps = 1e-6 * (s[3] + s[4] + s[5]) / 3 + 1e-30;
  const double T[9] = {s[3] + eps, s[6], s[7], s[6], s[4] + eps, s[8], s[7], s[8], s[5] + eps};
  // inverse by cofactors
  const double c00 = T[4] * T[8] - T[5] * T[7], c01 = T[5] * T[6] - T[3] * T[8], c02 = T[3] * T[7] - T[4] * T[6];
  const double det = T[0] * c00 + T[1] * c01 + T[2] * c02;
  const double Ti[9] = {c00 / det, (T[2] * T[7] - T[1] * T[8]) / det, (T[1] * T[5] - T[2] * T[4]) / det,
                        c01 / det, (T[0] * T[8] - T[2] * T[6]) / det, (T[2] * T[3] - T[0] * T[5]) / det,
                        c02 / det, (T[1] * T[6] - T[0] * T[7]) / det, (T[0] * T[4] - T[1] * T[3]) / det};
  const double h = A.P->h;
  double th[3];
  for (int z = 0; z < 3; ++z) th[z] = (Ti[3 * z] * s[0] + Ti[3 * z + 1] * s[1] + Ti[3 * z + 2] * s[2]) * h;
  if (!(m[0] > 0.0) || !isfinite(th[0]) || !isfinite(th[1]) || !isfinite(th[2])) th[0] = th[1] = th[2] = 0.0;
  double* q = R.step + 6 * (size_t)p;
  for (int z = 0; z < 3; ++z) q[z] = cv[z], q[3 + z] = th[z];
}

// spinApply (rigid_spin.wgsl:114-136): the start moves by (R + R^T - 2 I) r = 2 (1 - cos phi) k x (k x r)
// about the centroid, r from the committed position.
__global__ void k_spin_apply(StepArgs A, RigidArgs R) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= A.N || !inPiece(R, n) || A.pinned[n]) return;
  const double* q = R.step + 6 * (size_t)R.pieceOf[n];
  const double phi = sqrt(q[3] * q[3] + q[4] * q[4] + q[5] * q[5]);
  if (phi < 1e-9) return;
  const double k[3] = {q[3] / phi, q[4] / phi, q[5] / phi};
  const float4 x = A.x[n];
  const double r[3] = {x.x - q[0], x.y - q[1], x.z - q[2]};
  const double kr[3] = {k[1] * r[2] - k[2] * r[1], k[2] * r[0] - k[0] * r[2], k[0] * r[1] - k[1] * r[0]};
  const double kkr[3] = {k[1] * kr[2] - k[2] * kr[1], k[2] * kr[0] - k[0] * kr[2], k[0] * kr[1] - k[1] * kr[0]};
  const double c = 2.0 * (1.0 - cos(phi));
  float4 d = A.dx[n];
  A.dx[n] = make_float4((float)(d.x + c * kkr[0]), (float)(d.y + c * kkr[1]), (float)(d.z + c * kkr[2]), d.w);
}

}  // namespace btd
