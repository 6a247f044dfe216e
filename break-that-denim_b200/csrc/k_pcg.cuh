// PCG on the fine level with scalars kept on the device (pcg.wgsl; pcg(), newtonMultigrid.ts:537-576)
// and the Newton line search (energy.wgsl:89-290; energyChange/chooseStep, solver.ts(ref):430-534,
// newtonMultigrid.ts:597-603).
//
// Reductions: each block reduces in FP64 and writes one partial; the last block to finish (ticket
// counter) sums the partials in block order. The grid size is fixed per solver, so every sum is
// bitwise reproducible. The last block also does the scalar work (alpha, beta, convergence test)
// and, in a captured graph, sets the PCG while-node's condition.
#pragma once

#include "common.cuh"
#include "k_learned.cuh"
#include "k_mg.cuh"
#include "k_rigid.cuh"
#include "k_step.cuh"

namespace btd {

constexpr int RED_THREADS = 256;

struct Reduce {
  double* partials;    // [blocks * 8]
  unsigned* ticket;    // zero between launches
};

// Block-sum NV doubles; returns true in the last finished block, whose threads then hold the grid
// totals in out[] (thread 0 only is guaranteed to hold them).
template <int NV>
__device__ bool gridReduce(const Reduce& R, double (&v)[NV], double (&out)[NV]) {
  __shared__ double wsum[RED_THREADS / 32][NV];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) wsum[warp][q] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0;
      for (int w = 0; w < RED_THREADS / 32; ++w) s += wsum[w][q];
      R.partials[(size_t)blockIdx.x * 8 + q] = s;
    }
    __threadfence();
    unsigned t = atomicAdd(R.ticket, 1u);
    last = t == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += RED_THREADS) s += ((volatile double*)R.partials)[(size_t)b * 8 + q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) wsum[warp][q] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0;
      for (int w = 0; w < RED_THREADS / 32; ++w) s += wsum[w][q];
      out[q] = s;
    }
    *R.ticket = 0u;
  }
  return true;
}

struct PcgArgs {
  DLevel F;  // fine level: B = r, X = z
  float4* p;
  float4* Ap;
  float4* delta;
  float4* b0;  // the right-hand side PCG started from (the true residual's b)
  double* dd;  // the iterate accumulated in FP64, 3 per node (delta is its fp32 copy)
  Scalars* scal;
  const SimParams* P;
  uint32_t* counters;
  Reduce red;
  cudaGraphConditionalHandle cond;  // PCG while-node condition
  int useCond;
  LcState* lc;  // the learned coarse correction's state (null: not enabled)
  // the fine operator in FP64 (null: the fp32 rows): the operator PCG solves with - its products, the
  // true residual and the rigid start's residual - while the V-cycle keeps the fp32 rows
  const double2* op64;
  float4* zPrev;  // the previous preconditioned residual (the flexible beta's)
};

__device__ __forceinline__ double safeDiv(double a, double b) {
  double q = a / b;
  return (b > 0.0 && isfinite(q)) ? q : 0.0;
}

// delta = 0, z = 0; r0 = ||r|| (r = b: the solve starts from zero).
__global__ void __launch_bounds__(RED_THREADS) k_pcg_init(PcgArgs a) {
  pdlWait();
  pdlLaunchNext();
  double v[1] = {0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.F.N; n += gridDim.x * blockDim.x) {
    a.delta[n] = make_float4(0, 0, 0, 0);
    a.dd[3 * n] = a.dd[3 * n + 1] = a.dd[3 * n + 2] = 0.0;
    a.F.X[n] = make_float4(0, 0, 0, 0);
    a.b0[n] = a.F.B[n];
    float3 r = f3(a.F.B[n]);
    v[0] += (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
  }
  double out[1];
  if (gridReduce<1>(a.red, v, out) && threadIdx.x == 0) {
    Scalars& s = *a.scal;
    s.r0 = sqrt(out[0]);
    s.rr = out[0];
    s.rel = s.r0 > 0.0 ? 1.0 : 0.0;
    s.pcgIt = 0;
    s.converged = 0;
    s.check = 0;
    s.restart = 0;
  }
}

// Symmetric fp32 block times an FP64 vector, in FP64.
__device__ __forceinline__ void symVecAddD(const Sym& A, const double* x, double& y0, double& y1, double& y2) {
  y0 += (double)A.xx * x[0] + (double)A.xy * x[1] + (double)A.xz * x[2];
  y1 += (double)A.xy * x[0] + (double)A.yy * x[1] + (double)A.yz * x[2];
  y2 += (double)A.xz * x[0] + (double)A.yz * x[1] + (double)A.zz * x[2];
}

// y += (row n of the operator PCG solves with) x, in FP64: the FP64 row when there is one, else the fp32
// row's products summed in FP64. xAt(m, q) puts node m's x in q and returns false for a node whose x is
// zero (skipped).
template <class XAt>
__device__ __forceinline__ void pcgRowApply(const PcgArgs& a, int n, XAt xAt, double& y0, double& y1, double& y2) {
  const DLevel& F = a.F;
  int i, j, l;
  nodeAt(F, n, &i, &j, &l);
  const DLevelLayer L = layerOf(F, l);
  double q[3];
  if (xAt(n, q)) {
    if (a.op64)
      symDVecAdd(loadSymD(a.op64, F.N, n, 0), q, y0, y1, y2);
    else
      symVecAddD(FineRows::diag(F.op, F.N, n), q, y0, y1, y2);
  }
#pragma unroll
  for (int k = 0; k < FineRows::NC; ++k) {
    const int2 off = FineRows::offset(k);
    const int m = levelNode(L, i + off.x, j + off.y);
    if (m < 0 || !xAt(m, q)) continue;
    if (a.op64)
      symDVecAdd(fine64Block(a.op64, F.N, n, k), q, y0, y1, y2);
    else
      symVecAddD(FineRows::coupling(F.op, F.N, n, k), q, y0, y1, y2);
  }
}

// The PCG start from the detached pieces' rigid modes (encodeRigidStart, solver.ts:651-657): delta = x0
// (t + w x r on each piece's nodes, zero elsewhere), r = b - A x0 in FP64 (fixed rows 0), z = 0.
__global__ void __launch_bounds__(RED_THREADS) k_pcg_init_rigid(PcgArgs a, StepArgs S, RigidArgs R) {
  pdlWait();
  pdlLaunchNext();
  double v[1] = {0.0};
  const DLevel& F = a.F;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < F.N; n += gridDim.x * blockDim.x) {
    const Dv x0 = rigidStartAt(S, R, n);
    a.dd[3 * n] = x0.x, a.dd[3 * n + 1] = x0.y, a.dd[3 * n + 2] = x0.z;
    a.delta[n] = make_float4((float)x0.x, (float)x0.y, (float)x0.z, 0.f);
    a.F.X[n] = make_float4(0, 0, 0, 0);
    const float4 b = F.B[n];
    a.b0[n] = b;
    float3 r = make_float3(0, 0, 0);
    if (!F.fixed[n]) {
      double y0 = 0.0, y1 = 0.0, y2 = 0.0;
      pcgRowApply(
          a, n,
          [&](int m, double* q) {
            if (!inPiece(R, m)) return false;
            const Dv xm = rigidStartAt(S, R, m);
            q[0] = xm.x, q[1] = xm.y, q[2] = xm.z;
            return true;
          },
          y0, y1, y2);
      r = make_float3((float)(b.x - y0), (float)(b.y - y1), (float)(b.z - y2));
    }
    F.B[n] = make_float4(r.x, r.y, r.z, 0.f);
    v[0] += (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
  }
  double out[1];
  if (gridReduce<1>(a.red, v, out) && threadIdx.x == 0) {
    Scalars& s = *a.scal;
    s.r0 = sqrt(out[0]);
    s.rr = out[0];
    s.rel = s.r0 > 0.0 ? 1.0 : 0.0;
    s.pcgIt = 0;
    s.converged = 0;
    s.check = 0;
    s.restart = 0;
  }
}

// rz' = r . z; first: rz = rz', beta unused; else beta = rz' / rz, rz = rz'.
// With P.pcgFlex, beta = max(r' . (z' - z), 0) / rz (the flexible, Polak-Ribiere form: equal to the
// plain one in exact arithmetic with a fixed SPD preconditioner, and robust to one that is applied
// inexactly), z kept for the next iteration.
__global__ void __launch_bounds__(RED_THREADS) k_pcg_dot_rz(PcgArgs a, int first) {
  pdlWait();
  pdlLaunchNext();
  const bool flex = a.P->pcgFlex != 0;
  double v[2] = {0.0, 0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.F.N; n += gridDim.x * blockDim.x) {
    const float4 z4 = a.F.X[n];
    float3 r = f3(a.F.B[n]), z = f3(z4);
    v[0] += (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
    if (flex) {
      const float3 zp = f3(a.zPrev[n]);
      v[1] += (double)r.x * zp.x + (double)r.y * zp.y + (double)r.z * zp.z;
      a.zPrev[n] = z4;
    }
  }
  double out[2];
  if (gridReduce<2>(a.red, v, out) && threadIdx.x == 0) {
    Scalars& s = *a.scal;
    if (first || s.restart) {
      s.beta = 0.0;
      s.rz = out[0];
      s.restart = 0;
    } else {
      s.beta = flex ? fmax(safeDiv(out[0] - out[1], s.rz), 0.0) : safeDiv(out[0], s.rz);
      s.rz = out[0];
    }
  }
}

// p = z + beta p (first: p = z).
__global__ void k_pcg_update_p(PcgArgs a, int first) {
  pdlWait();
  pdlLaunchNext();
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.F.N) return;
  float3 z = f3(a.F.X[n]);
  if (first) {
    a.p[n] = make_float4(z.x, z.y, z.z, 0.f);
    return;
  }
  float beta = (float)a.scal->beta;
  float3 p = z + beta * f3(a.p[n]);
  a.p[n] = make_float4(p.x, p.y, p.z, 0.f);
}

// Ap = A p (fixed rows 0), p . Ap; alpha = rz / pAp (0 and stop when pAp <= 0, as pcg() breaks).
__global__ void __launch_bounds__(RED_THREADS) k_pcg_matvec(PcgArgs a) {
  pdlWait();
  pdlLaunchNext();
  double v[1] = {0.0};
  const DLevel& F = a.F;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < F.N; n += gridDim.x * blockDim.x) {
    // the row's loads do not wait for its fixed flag (a fixed row's product is dropped)
    float3 y = make_float3(0, 0, 0);
    const uint32_t fixedRow = F.fixed[n];
    {
      // products summed in FP64: the recurrence residual then drifts from the true one by the rounding
      // of the stored Ap only
      double y0 = 0.0, y1 = 0.0, y2 = 0.0;
      pcgRowApply(
          a, n,
          [&](int m, double* q) {
            const float4 pm = a.p[m];
            q[0] = pm.x, q[1] = pm.y, q[2] = pm.z;
            return true;
          },
          y0, y1, y2);
      if (!fixedRow) y = make_float3((float)y0, (float)y1, (float)y2);
    }
    a.Ap[n] = make_float4(y.x, y.y, y.z, 0.f);
    float3 p = f3(a.p[n]);
    v[0] += (double)y.x * p.x + (double)y.y * p.y + (double)y.z * p.z;
  }
  double out[1];
  if (gridReduce<1>(a.red, v, out) && threadIdx.x == 0) {
    Scalars& s = *a.scal;
    s.pAp = out[0];
    if (out[0] > 0.0) {
      s.alpha = safeDiv(s.rz, out[0]);
    } else {
      s.alpha = 0.0;
      s.converged = 2;  // breakdown: the reference's pcg() stops here
    }
  }
}

__device__ __forceinline__ void pcgStop(const PcgArgs& a, Scalars& s) {
  a.counters[CNT_PCG_LAST] = (uint32_t)s.pcgIt;
  atomicAdd(&a.counters[CNT_PCG_TOTAL], (uint32_t)s.pcgIt);
  a.counters[CNT_REL] = __float_as_uint((float)s.rel);
  // the worst relative residual a solve stopped at (non-negative floats order as their bits; NaN above
  // all) and the solves that stopped short of the tolerance (cap or breakdown)
  atomicMax(&a.counters[CNT_REL_MAX], __float_as_uint((float)s.rel));
  if (a.P->pcgTol > 0.0 && !(s.rel <= a.P->pcgTol)) atomicAdd(&a.counters[CNT_PCG_MISSED], 1u);
}

// delta += alpha p (accumulated in FP64, kept in fp32 too); r -= alpha Ap; z = 0; ||r||. The
// iteration cap, a breakdown or a zero right-hand side stop the loop (the while condition); the
// recurrence residual meeting the tolerance hands the decision to k_pcg_true_residual.
__global__ void __launch_bounds__(RED_THREADS) k_pcg_update_xr(PcgArgs a) {
  pdlWait();
  pdlLaunchNext();
  double v[1] = {0.0};
  const double alphaD = a.scal->alpha;
  const float alpha = (float)alphaD;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.F.N; n += gridDim.x * blockDim.x) {
    const float3 pn = f3(a.p[n]);
    const double d0 = a.dd[3 * n] + alphaD * pn.x, d1 = a.dd[3 * n + 1] + alphaD * pn.y, d2 = a.dd[3 * n + 2] + alphaD * pn.z;
    a.dd[3 * n] = d0, a.dd[3 * n + 1] = d1, a.dd[3 * n + 2] = d2;
    float3 r = f3(a.F.B[n]) - alpha * f3(a.Ap[n]);
    a.delta[n] = make_float4((float)d0, (float)d1, (float)d2, 0.f);
    a.F.B[n] = make_float4(r.x, r.y, r.z, 0.f);
    a.F.X[n] = make_float4(0, 0, 0, 0);
    v[0] += (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z;
  }
  double out[1];
  if (gridReduce<1>(a.red, v, out) && threadIdx.x == 0) {
    Scalars& s = *a.scal;
    const SimParams& P = *a.P;
    s.rr = out[0];
    s.rel = s.r0 > 0.0 ? sqrt(out[0]) / s.r0 : 0.0;
    s.pcgIt += 1;
    const bool met = P.pcgTol > 0.0 && s.rel <= P.pcgTol;
    const bool stop = s.converged != 0 || s.pcgIt >= P.pcgMax || !(s.r0 > 0.0);
    if (stop && s.converged == 0) s.converged = 1;
    s.check = !stop && met ? 1 : 0;
    if (stop) pcgStop(a, s);
    // guard of the learned coarse correction: a solve whose mean contraction per iteration
    // (||r_k|| / ||r_0||)^(1/k) exceeds the guard after three iterations goes on with the plain
    // V-cycle, PCG restarted from its iterate (the next direction starts afresh)
    if (a.lc && a.lc->active && !stop && !met && s.pcgIt >= 3) {
      const double rel = P.pcgTol > 0.0 ? s.rel : sqrt(out[0]) / s.r0;
      if (!(pow(rel, 1.0 / s.pcgIt) <= (double)a.lc->guard)) {
        a.lc->active = 0;
        a.lc->fallbacks += 1;
        s.restart = 1;
      }
    }
    if (a.useCond) cudaGraphSetConditional(a.cond, stop ? 0u : 1u);
  }
}


// The outer residual, when the recurrence residual met the tolerance: r = b0 - A delta with the
// FP64 iterate, every product and sum in FP64, ||r|| in FP64. Met: PCG stops. Not met (the fp32
// recurrence drifted): r replaces the recurrence residual (stored fp32) and the next direction starts
// afresh (keeping the old one stalls: measured ~10x more iterations), so the fp32 iterations solve
// for a correction that accumulates into the FP64 iterate - iterative refinement.
__global__ void __launch_bounds__(RED_THREADS) k_pcg_true_residual(PcgArgs a) {
  pdlWait();
  pdlLaunchNext();
  if (!a.scal->check) return;
  double v[1] = {0.0};
  const DLevel& F = a.F;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < F.N; n += gridDim.x * blockDim.x) {
    const float3 b = f3(a.b0[n]);
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    const uint32_t fixedRow = F.fixed[n];
    pcgRowApply(
        a, n,
        [&](int m, double* q) {
          q[0] = a.dd[3 * m], q[1] = a.dd[3 * m + 1], q[2] = a.dd[3 * m + 2];
          return true;
        },
        y0, y1, y2);
    if (fixedRow) y0 = y1 = y2 = 0.0;
    const double r0 = (double)b.x - y0, r1 = (double)b.y - y1, r2 = (double)b.z - y2;
    a.F.B[n] = make_float4((float)r0, (float)r1, (float)r2, 0.f);
    v[0] += r0 * r0 + r1 * r1 + r2 * r2;
  }
  double out[1];
  if (gridReduce<1>(a.red, v, out) && threadIdx.x == 0) {
    Scalars& s = *a.scal;
    const SimParams& P = *a.P;
    s.rr = out[0];
    s.rel = s.r0 > 0.0 ? sqrt(out[0]) / s.r0 : 0.0;
    s.check = 0;
    const bool stop = s.rel <= P.pcgTol || s.pcgIt >= P.pcgMax;
    if (stop) {
      s.converged = 1;
      pcgStop(a, s);
    } else {
      s.restart = 1;
    }
    if (a.useCond) cudaGraphSetConditional(a.cond, stop ? 0u : 1u);
  }
}

// y = A x and x . y for a fine-level operator (the PCG matvec of pcg.wgsl:268-287 without its scalar
// bookkeeping). `coord` may be null for a single-layer lattice, whose coordinates follow from nx.
struct MatvecArgs {
  int N, nx, ny;
  const uint2* __restrict__ coord;
  const DLevelLayer* __restrict__ layers;
  const float4* __restrict__ op;
  const uint32_t* __restrict__ fixed;
  const float4* __restrict__ x;
  float4* y;
  double* xy;
  Reduce red;
};

__global__ void __launch_bounds__(RED_THREADS) k_matvec_dot(MatvecArgs a) {
  double v[1] = {0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.N; n += gridDim.x * blockDim.x) {
    float3 y = make_float3(0, 0, 0);
    if (!a.fixed[n]) {
      int i, j;
      DLevelLayer L;
      if (a.coord) {
        const uint2 c = a.coord[n];
        i = c.x & 0xFFFF, j = c.x >> 16;
        L = a.layers[c.y];
      } else {
        i = n % a.nx, j = n / a.nx;
        L = {0, a.nx, a.ny, 0};
      }
      y = FineRows::diag(a.op, a.N, n) * f3(a.x[n]);
#pragma unroll
      for (int k = 0; k < FineRows::NC; ++k) {
        int2 off = FineRows::offset(k);
        int m = levelNode(L, i + off.x, j + off.y);
        if (m < 0) continue;
        y += FineRows::coupling(a.op, a.N, n, k) * f3(a.x[m]);
      }
    }
    a.y[n] = make_float4(y.x, y.y, y.z, 0.f);
    float3 x = f3(a.x[n]);
    v[0] += (double)y.x * x.x + (double)y.y * x.y + (double)y.z * x.z;
  }
  double out[1];
  if (gridReduce<1>(a.red, v, out) && threadIdx.x == 0) *a.xy = out[0];
}

// ------------------------------------------------------------------------------------ line search

constexpr float LINE_NOISE = 4e-6f;

struct EnergyArgs {
  StepArgs S;
  const float4* __restrict__ delta;
  Reduce red;
  // detached pieces (null: none): a node of a piece with a valid frame steps along the rotation of its
  // piece's rigid start (curveW.xyz the rotation, w 1 when on; curveR the arm from the centroid)
  const float4* __restrict__ curveW;
  const float4* __restrict__ curveR;
};

__device__ __forceinline__ float3 dirOf(const EnergyArgs& a, int n) {
  return a.S.pinned[n] ? make_float3(0, 0, 0) : f3(a.delta[n]);
}
__device__ __forceinline__ float2 lenChange(float3 e0, float3 s, float l0) {
  float la = len3(e0 + s);
  return make_float2((2.f * dot3(e0, s) + dot3(s, s)) / fmaxf(la + l0, 1e-12f), la);
}

// Per-node energy changes at alpha in {1, 1/2, 1/4, 1/8} and their magnitude sums (nodeDelta,
// energy.wgsl:89-218). A node owns its inertia/external/drag terms, its "+" spans, the bending
// triples centred on it and the shear diagonals of the cell it is the lower-left corner of.
__device__ void nodeDelta(const EnergyArgs& a, int n, float* acc, float* mag) {
  const StepArgs& A = a.S;
  const float ALPHA[4] = {1.f, 0.5f, 0.25f, 0.125f};
  auto add1 = [&](int k, float v) {
    acc[k] += v;
    mag[k] += fabsf(v);
  };
  // node m's step at step length k (steps, energy.wgsl:63-72): alpha d, plus on a detached piece the
  // rotation curve of its rigid part; alpha being a power of two, alpha d is exact, so the differences
  // of steps below equal alpha times the differences of directions bit for bit when no piece is set
  auto stepAt = [&](int m, int k) -> float3 {
    float3 sk = ALPHA[k] * dirOf(a, m);
    if (a.curveW && !a.S.pinned[m]) {
      const float4 w = a.curveW[m];
      if (w.w > 0.f) sk += rotationCurve(ALPHA[k] * f3(w), f3(a.curveR[m]));
    }
    return sk;
  };
  auto quad = [&](float3 g, Sym H, int m) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float3 sk = stepAt(m, k);
      add1(k, dot3(g, sk));
      add1(k, 0.5f * dot3(sk, H * sk));
    }
  };
  const SimParams P = *A.P;
  const NodeStatic st = A.nodes[n];
  const int i = st.ij & 0xFFFF, j = st.ij >> 16;
  const DLayer& L = A.layers[st.layer];
  const float h = P.h;
  const float3 d0 = f3(A.dx[n]);
  if (!A.pinned[n]) {
    float w = st.mass / (h * h);
    quad(w * (d0 - f3(A.pred[n])), symId(w), n);
    float4 e0 = A.ext[3 * n], e1 = A.ext[3 * n + 1], e2 = A.ext[3 * n + 2];
    quad(f3(e0), Sym{e1.x, e1.y, e1.z, e1.w, e2.x, e2.y}, n);
    if (P.floorOn) {
      float reach = 0.5f * L.thickness + P.floorBulge;
      float s0 = reach - (A.x[n].z + d0.z - P.floorZ);
      if (s0 > 0.f) {
        float kc = P.floorStiffness;
        float lam = kc * s0 * s0 / reach;
        float kf = P.floorFriction * lam / fmaxf(sqrtf(d0.x * d0.x + d0.y * d0.y), P.floorFrictionSpeed * h);
        quad(make_float3(kf * d0.x, kf * d0.y, -lam), Sym{kf, 0, 0, kf, 0, 2.f * kc * s0 / reach}, n);
      }
    }
    Sym Dd = airDragBlock(A, n, L, i, j, h);
    quad(Dd * d0, Dd, n);
  }
#pragma unroll
  for (int f = 0; f < 2; ++f) {
    const int du = f == 0 ? 1 : 0, dv = f == 1 ? 1 : 0;
    const DYarn& y = L.yarn[f];
    const int next = nodeAt(L, i + du, j + dv);
    if (next >= 0 && activeSpan(A.segs, n, f)) {
      const Seg s = A.segs[2 * n + f];
      const float Lr = s.rest;
      const float3 en = f3(A.x[next]) - f3(A.x[n]);
      const float3 ec = en + f3(A.dx[next]) - d0;
      const float l0 = len3(ec), ln = len3(en);
      const float T0 = s.intact * axialTension(y, l0 / Lr - 1.f);
      const float c = y.axialVisc / (Lr * h);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float2 r = lenChange(ec, stepAt(next, k) - stepAt(n, k), l0);
        float Ta = s.intact * axialTension(y, r.y / Lr - 1.f);
        add1(k, 0.5f * (T0 + Ta) * r.x);
        add1(k, 0.5f * c * r.x * (r.y + l0 - 2.f * ln));
      }
    }
    const int prev = nodeAt(L, i - du, j - dv);
    if (prev >= 0 && next >= 0 && activeSpan(A.segs, prev, f) && activeSpan(A.segs, n, f)) {
      const Seg sa = A.segs[2 * prev + f], sn = A.segs[2 * n + f];
      const float4 geo = bendGeometry(sa.rest, sn.rest);
      const float ke = y.bendRigidity * bendScale(sa.intact, sn.intact, sa.cutMask, sn.cutMask, (uint32_t)y.yarnsPerSpan) * geo.z;
      const float kd = ke * y.bendVisc / h;
      const float3 rn = geo.x * f3(A.x[prev]) - 2.f * f3(A.x[n]) + geo.y * f3(A.x[next]);
      const float3 r0 = rn + geo.x * f3(A.dx[prev]) - 2.f * d0 + geo.y * f3(A.dx[next]);
      const float q0 = dot3(r0, r0), l0 = sqrtf(q0), lrn = len3(rn);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float3 dr = geo.x * stepAt(prev, k) - 2.f * stepAt(n, k) + geo.y * stepAt(next, k);
        float dq = 2.f * dot3(r0, dr) + dot3(dr, dr);
        add1(k, 0.5f * ke * bendPsiDelta(q0, q0 + dq, dq, geo.w));
        float2 rl = lenChange(r0, dr, l0);
        add1(k, 0.5f * kd * rl.x * (rl.y + l0 - 2.f * lrn));
      }
    }
  }
  const int r = nodeAt(L, i + 1, j), t = nodeAt(L, i, j + 1), rt = nodeAt(L, i + 1, j + 1);
  if (r >= 0 && t >= 0) {
    const bool cu = activeSpan(A.segs, n, 0), cv = activeSpan(A.segs, n, 1), rv = activeSpan(A.segs, r, 1),
               tu = activeSpan(A.segs, t, 0);
    const bool on[2] = {(cu && rv) || (cv && tu), (cu && cv) || (rv && tu)};
    const float s0 = A.segs[2 * n].rest, s1 = A.segs[2 * n + 1].rest;
    const float Ld = sqrtf(s0 * s0 + s1 * s1);
    const float ar = cellArea(cu ? A.segs[2 * n].intact : 0.f, tu ? A.segs[2 * t].intact : 0.f, cv ? A.segs[2 * n + 1].intact : 0.f,
                              rv ? A.segs[2 * r + 1].intact : 0.f);
    const float ks = L.shearStiffness * st.n0 / L.crossingNormal0;
    const float jam = shearJam(ar);
    const int pa[2] = {n, r}, pb[2] = {rt, t};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (!on[q]) continue;
      const int p = pa[q], o = pb[q];
      const float3 ec = (f3(A.x[o]) + f3(A.dx[o])) - (f3(A.x[p]) + f3(A.dx[p]));
      const float l0 = len3(ec);
      const float f0 = shearLaw(ks, jam, Ld, l0).x;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float2 rr = lenChange(ec, stepAt(o, k) - stepAt(p, k), l0);
        add1(k, 0.5f * (f0 + shearLaw(ks, jam, Ld, rr.y).x) * rr.x);
      }
    }
  }
}

// Sum of the per-node changes (non-finite nodes excluded: the firewall) and the step choice.
__global__ void __launch_bounds__(RED_THREADS) k_energy(EnergyArgs a) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.S.N; n += gridDim.x * blockDim.x) {
    float acc[4] = {0, 0, 0, 0}, mag[4] = {0, 0, 0, 0};
    nodeDelta(a, n, acc, mag);
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 4; ++k) ok = ok && finite1(acc[k]) && finite1(mag[k]);
    if (ok) {
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] += acc[k], v[4 + k] += mag[k];
    }
  }
  double out[8];
  if (gridReduce<8>(a.red, v, out) && threadIdx.x == 0) {
    Scalars& s = *a.S.scal;
    const float ALPHA[4] = {1.f, 0.5f, 0.25f, 0.125f};
    for (int k = 0; k < 4; ++k) s.e[k] = out[k], s.m[k] = out[4 + k];
    int best = 0;
    for (int k = 1; k < 4; ++k)
      if (out[k] < out[best]) best = k;
    float alpha = 1.f;
    bool allUp = true;
    for (int k = 0; k < 4; ++k) allUp = allUp && out[k] > (double)LINE_NOISE * out[4 + k];
    if (out[best] < -(double)LINE_NOISE * out[4 + best]) {
      alpha = ALPHA[best];
    } else if (allUp) {
      alpha = 0.f;
      atomicAdd(&a.S.counters[CNT_REJECT], 1u);
    }
    s.lineAlpha = alpha;
    a.S.counters[CNT_ALPHA] = __float_as_uint(alpha);
  }
}

__global__ void k_set_alpha(Scalars* s, uint32_t* counters, float alpha) {
  s->lineAlpha = alpha;
  counters[CNT_ALPHA] = __float_as_uint(alpha);
}

}  // namespace btd
