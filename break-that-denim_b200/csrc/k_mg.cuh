// Galerkin multigrid kernels on the lattice stencils (multigrid.wgsl; newtonMultigrid.ts:282-528).
// Each kernel is a template over the row layout of the level it reads (fine: 12 couplings with
// scalar +-2 bending entries; coarse: the 24-coupling radius-2 stencil); coarse rows are always
// written in the coarse layout.
#pragma once

#include "common.cuh"

namespace btd {

struct FineRows {
  static constexpr int NC = 12;
  __device__ static int2 offset(int k) { return fineOffset(k); }
  __device__ static Sym diag(const float4* op, int N, int n) { return fineBlock(op, N, n, 0); }
  __device__ static Sym coupling(const float4* op, int N, int n, int k) { return fineCouplingBlock(op, N, n, k); }
  // coupling index of a unit offset (prolongation connectivity)
  __device__ static int index(int di, int dj) { return fineCoupling(di, dj); }
};
struct CoarseRows {
  static constexpr int NC = 24;
  __device__ static int2 offset(int k) {
    int o = k >= 12 ? k + 1 : k;
    return make_int2(o % 5 - 2, o / 5 - 2);
  }
  __device__ static Sym diag(const float4* op, int N, int n) { return coarseBlock(op, N, n, 12); }
  __device__ static Sym coupling(const float4* op, int N, int n, int k) { return coarseBlock(op, N, n, k >= 12 ? k + 1 : k); }
  __device__ static int index(int di, int dj) {
    int o = (dj + 2) * 5 + (di + 2);
    return o > 12 ? o - 1 : o;
  }
};

__device__ __forceinline__ void nodeCoord(const DLevel& L, int n, int* i, int* j, int* l) {
  uint2 c = L.coord[n];
  *i = c.x & 0xFFFF;
  *j = c.x >> 16;
  *l = c.y;
}
// Node n's position and layer index: by arithmetic on a single-layer level, else from the table.
__device__ __forceinline__ void nodeAt(const DLevel& L, int n, int* i, int* j, int* l) {
  if (L.one.nx > 0) {
    const int m = n - L.one.offset;
    *j = m / L.one.nx;
    *i = m - *j * L.one.nx;
    *l = 0;
  } else {
    nodeCoord(L, n, i, j, l);
  }
}
__device__ __forceinline__ DLevelLayer layerOf(const DLevel& L, int l) { return L.one.nx > 0 ? L.one : L.layers[l]; }

constexpr float LINK_MIN_INTACT = 0.02f;

// Whether node (i, j) of level F and its unit-offset neighbour are connected (linked,
// multigrid.wgsl:44-56; newtonMultigrid.ts:287-295): an intact span on the fine lattice; on coarse
// levels a nonzero Galerkin coupling or a fixed neighbour.
template <class Rows, bool FINE>
__device__ __forceinline__ bool linked(const DLevel& F, const Seg* __restrict__ segs, const DLevelLayer& L, int i, int j, int di, int dj) {
  int a = levelNode(L, i, j), b = levelNode(L, i + di, j + dj);
  if (a < 0 || b < 0) return false;
  if (FINE) {
    int f = di != 0 ? 0 : 1;
    int owner = di + dj > 0 ? a : b;
    Seg sg = segs[2 * owner + f];
    return segActive(sg) && sg.intact > LINK_MIN_INTACT;
  }
  if (F.fixed[b]) return true;
  return !symIsZero(Rows::coupling(F.op, F.N, a, Rows::index(di, dj)));
}

// Masked, renormalised bilinear weights (prolongWeights, multigrid.wgsl:62-102; buildProlongation,
// newtonMultigrid.ts:305-342).
template <class Rows, bool FINE>
__global__ void k_prolong_weights(DLevel F, const Seg* __restrict__ segs) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= F.N) return;
  if (F.fixed[a]) {
    F.pw[a] = make_float4(0, 0, 0, 0);
    return;
  }
  int i, j, l;
  nodeCoord(F, a, &i, &j, &l);
  const DLevelLayer L = F.layers[l];
  Bracket bi = bracketOf(i, L.nx), bj = bracketOf(j, L.ny);
  float w[4] = {0, 0, 0, 0};
  float sum = 0.f;
  for (int kj = 0; kj < 2; ++kj) {
    int J = kj ? bj.hi : bj.lo;
    float wj = kj ? bj.whi : bj.wlo;
    if (wj == 0.f) continue;
    int dj = coarseToFine(J, L.ny) - j;
    for (int ki = 0; ki < 2; ++ki) {
      int I = ki ? bi.hi : bi.lo;
      float wi = ki ? bi.whi : bi.wlo;
      if (wi == 0.f) continue;
      int di = coarseToFine(I, L.nx) - i;
      bool ok = true;
      if (di != 0 && dj != 0) {
        ok = (linked<Rows, FINE>(F, segs, L, i, j, di, 0) && linked<Rows, FINE>(F, segs, L, i + di, j, 0, dj)) ||
             (linked<Rows, FINE>(F, segs, L, i, j, 0, dj) && linked<Rows, FINE>(F, segs, L, i, j + dj, di, 0));
      } else if (di != 0 || dj != 0) {
        ok = linked<Rows, FINE>(F, segs, L, i, j, di, dj);
      }
      if (ok) {
        w[ki + 2 * kj] = wi * wj;
        sum += wi * wj;
      }
    }
  }
  F.pw[a] = sum > 0.f ? make_float4(w[0] / sum, w[1] / sum, w[2] / sum, w[3] / sum) : make_float4(0, 0, 0, 0);
}

// Bilinear (unmasked) weight of fine index i in coarse index I, 0 outside its bracket.
__device__ __forceinline__ float weightOf(int i, int I, int n) {
  Bracket b = bracketOf(i, n);
  if (b.lo == I) return b.wlo;
  if (b.hi == I && b.whi > 0.f) return b.whi;
  return 0.f;
}
__device__ __forceinline__ float pwSlot(float4 w, int s) { return s == 0 ? w.x : s == 1 ? w.y : s == 2 ? w.z : w.w; }

constexpr int RAP_THREADS = 64;

// Galerkin coarse row P^T A P of coarse node I (rap, multigrid.wgsl:115-178; galerkin,
// newtonMultigrid.ts:345-387). One thread per coarse node; its 25 accumulators live in shared memory.
template <class Rows>
__global__ void __launch_bounds__(RAP_THREADS) k_rap(DLevel F, DLevel C) {
  __shared__ float acc[RAP_THREADS][153];  // odd stride: conflict-free per-thread rows
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= C.N) return;
  float* a25 = acc[threadIdx.x];
  for (int q = 0; q < 150; ++q) a25[q] = 0.f;
  int ci, cj, l;
  nodeCoord(C, I, &ci, &cj, &l);
  const DLevelLayer Lf = F.layers[l];
  const int nxf = Lf.nx, nyf = Lf.ny;
  const int fi0 = coarseToFine(ci, nxf), fj0 = coarseToFine(cj, nyf);
  for (int aj = fj0 - 1; aj <= fj0 + 1; ++aj) {
    if (aj < 0 || aj >= nyf) continue;
    if (weightOf(aj, cj, nyf) == 0.f) continue;
    for (int ai = fi0 - 1; ai <= fi0 + 1; ++ai) {
      if (ai < 0 || ai >= nxf) continue;
      if (weightOf(ai, ci, nxf) == 0.f) continue;
      int a = levelNode(Lf, ai, aj);
      if (F.fixed[a]) continue;
      Bracket bai = bracketOf(ai, nxf), baj = bracketOf(aj, nyf);
      float wa = pwSlot(F.pw[a], (bai.lo == ci ? 0 : 1) + 2 * (baj.lo == cj ? 0 : 1));
      if (wa == 0.f) continue;
      for (int k = 0; k <= Rows::NC; ++k) {
        int2 off = make_int2(0, 0);
        Sym Ab;
        if (k == Rows::NC) {
          Ab = Rows::diag(F.op, F.N, a);
        } else {
          off = Rows::offset(k);
          Ab = Rows::coupling(F.op, F.N, a, k);
        }
        if (symIsZero(Ab)) continue;
        int bi = ai + off.x, bj = aj + off.y;
        if (bi < 0 || bj < 0 || bi >= nxf || bj >= nyf) continue;
        Bracket bri = bracketOf(bi, nxf), brj = bracketOf(bj, nyf);
        float4 wb = F.pw[levelNode(Lf, bi, bj)];
        for (int kj = 0; kj < 2; ++kj) {
          int J = kj ? brj.hi : brj.lo;
          for (int ki = 0; ki < 2; ++ki) {
            int Ii = ki ? bri.hi : bri.lo;
            float wJ = pwSlot(wb, ki + 2 * kj);
            if (wJ == 0.f) continue;
            const int oj = J - cj + 2, oi = Ii - ci + 2;
            if ((unsigned)oj > 4u || (unsigned)oi > 4u) continue;  // radius-2 closure (galerkin throws there)
            int o = oj * 5 + oi;
            float s = wa * wJ;
            float* p = a25 + 6 * o;
            p[0] += Ab.xx * s, p[1] += Ab.xy * s, p[2] += Ab.xz * s, p[3] += Ab.yy * s, p[4] += Ab.yz * s, p[5] += Ab.zz * s;
          }
        }
      }
    }
  }
  const float* c = a25 + 6 * 12;
  bool fixedRow = c[0] + c[3] + c[5] <= 0.f;
  if (fixedRow) {
    for (int q = 0; q < 150; ++q) a25[q] = 0.f;
    a25[72] = 1.f, a25[75] = 1.f, a25[77] = 1.f;
  }
  for (int p = 0; p < COARSE_PLANES; ++p) {
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = 4 * p + q < 150 ? a25[4 * p + q] : 0.f;
    C.op[(size_t)p * C.N + I] = make_float4(v[0], v[1], v[2], v[3]);
  }
  C.fixed[I] = fixedRow ? 1u : 0u;
}

// r = b - A x on the fine level (residual, multigrid.wgsl:182-199); fixed rows give 0. Loads are
// issued unconditionally (neighbour index clamped, outside couplings zero) so they overlap: the
// whole row in one round trip.
__global__ void k_residual_fine(DLevel F) {
  pdlWait();
  pdlLaunchNext();
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= F.N) return;
  int i, j, l;
  nodeAt(F, n, &i, &j, &l);
  const DLevelLayer L = layerOf(F, l);
  const uint32_t fixedRow = F.fixed[n];
  float3 r = f3(F.B[n]);
  float4 pl[FINE_PLANES];
#pragma unroll
  for (int p = 0; p < FINE_PLANES; ++p) pl[p] = __ldg(&F.op[(size_t)p * F.N + n]);
  float3 xm[12];
  bool ok[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    const int2 o = fineOffset(q);
    const int ii = i + o.x, jj = j + o.y;
    ok[q] = ii >= 0 && jj >= 0 && ii < L.nx && jj < L.ny;
    xm[q] = f3(F.X[ok[q] ? L.offset + jj * L.nx + ii : n]);
  }
  const float3 xn = f3(F.X[n]);
  const float* row = reinterpret_cast<const float*>(pl);
  r -= Sym{row[0], row[1], row[2], row[3], row[4], row[5]} * xn;
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    if (!ok[q]) continue;
    if (q < 8) {
      const float* b = row + 6 * q + 6;
      r -= Sym{b[0], b[1], b[2], b[3], b[4], b[5]} * xm[q];
    } else {
      r -= row[54 + q - 8] * xm[q];
    }
  }
  F.R[n] = fixedRow ? make_float4(0, 0, 0, 0) : make_float4(r.x, r.y, r.z, 0.f);
}

// The same residual from the FP64 fine rows (the operator PCG solves with), every product and sum in
// FP64: on torn cloth the FP32 row's stiff terms cancel on a loose strand's rigid motion only to ~6e-8
// of their size, which is larger than the strand's inertia, so the V-cycle would restrict noise there.
__global__ void k_residual_fine64(DLevel F, const double2* __restrict__ op64) {
  pdlWait();
  pdlLaunchNext();
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= F.N) return;
  int i, j, l;
  nodeAt(F, n, &i, &j, &l);
  const DLevelLayer L = layerOf(F, l);
  const uint32_t fixedRow = F.fixed[n];
  const float4 b = F.B[n], xn4 = F.X[n];
  double y0 = 0.0, y1 = 0.0, y2 = 0.0;
  {
    const double xn[3] = {xn4.x, xn4.y, xn4.z};
    symDVecAdd(loadSymD(op64, F.N, n, 0), xn, y0, y1, y2);
  }
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    const int2 o = fineOffset(q);
    const int ii = i + o.x, jj = j + o.y;
    if (ii < 0 || jj < 0 || ii >= L.nx || jj >= L.ny) continue;
    const float4 xm = F.X[L.offset + jj * L.nx + ii];
    const double x[3] = {xm.x, xm.y, xm.z};
    symDVecAdd(fine64Block(op64, F.N, n, q), x, y0, y1, y2);
  }
  F.R[n] = fixedRow ? make_float4(0, 0, 0, 0) : make_float4((float)(b.x - y0), (float)(b.y - y1), (float)(b.z - y2), 0.f);
}

// Row dj = R - 2 of the coarse stencil at node n = (i, j): sum over di of A(n, di, dj) x (di = -2..2).
template <int R>
__device__ __forceinline__ float3 coarseRowSum(const DLevel& F, const DLevelLayer& L, int n, int i, int j) {
  constexpr int f0 = 30 * R, p0 = f0 >> 2, sh = f0 & 3, dj = R - 2;
  float4 pl[9];
#pragma unroll
  for (int p = 0; p < 9; ++p) pl[p] = p0 + p < COARSE_PLANES ? __ldg(&F.op[(size_t)(p0 + p) * F.N + n]) : make_float4(0, 0, 0, 0);
  float3 xm[5];
  bool ok[5];
#pragma unroll
  for (int di = -2; di <= 2; ++di) {
    const int ii = i + di, jj = j + dj;
    ok[di + 2] = ii >= 0 && jj >= 0 && ii < L.nx && jj < L.ny;
    xm[di + 2] = f3(F.X[ok[di + 2] ? L.offset + jj * L.nx + ii : n]);
  }
  const float* row = reinterpret_cast<const float*>(pl) + sh;
  float3 s = make_float3(0, 0, 0);
#pragma unroll
  for (int di = -2; di <= 2; ++di) {
    if (!ok[di + 2]) continue;
    const float* bk = row + 6 * (di + 2);
    s += Sym{bk[0], bk[1], bk[2], bk[3], bk[4], bk[5]} * xm[di + 2];
  }
  return s;
}

// The same on a coarse level, eight lanes a node: lane dj + 2 (dj = -2..2) sums stencil row dj
// (5 blocks: 9 row planes and 5 unknowns, one round trip), lanes 5-7 hold zero, the group adds its
// partial sums by shuffles in a fixed order and lane 0 writes b minus the sum (0 on a fixed row).
// Every lane of the warp calls it (the shuffles); `valid` is false past the level's last node.
__device__ __forceinline__ void coarseResidualLane(const DLevel& F, const DLevelLayer& L, int n, int i, int j, int lane8, bool valid) {
  float3 s = make_float3(0, 0, 0);
  float4 b = make_float4(0, 0, 0, 0);
  uint32_t fx = 0u;
  if (valid && lane8 == 0) b = F.B[n], fx = F.fixed[n];
  if (valid) switch (lane8) {
      case 0: s = coarseRowSum<0>(F, L, n, i, j); break;
      case 1: s = coarseRowSum<1>(F, L, n, i, j); break;
      case 2: s = coarseRowSum<2>(F, L, n, i, j); break;
      case 3: s = coarseRowSum<3>(F, L, n, i, j); break;
      case 4: s = coarseRowSum<4>(F, L, n, i, j); break;
      default: break;
    }
#pragma unroll
  for (int m = 4; m >= 1; m >>= 1) {
    s.x += __shfl_xor_sync(0xffffffffu, s.x, m);
    s.y += __shfl_xor_sync(0xffffffffu, s.y, m);
    s.z += __shfl_xor_sync(0xffffffffu, s.z, m);
  }
  if (valid && lane8 == 0) F.R[n] = fx ? make_float4(0, 0, 0, 0) : make_float4(b.x - s.x, b.y - s.y, b.z - s.z, 0.f);
}

// Eight threads a node (blockDim a multiple of 32).
__global__ void k_residual_coarse(DLevel F) {
  pdlWait();
  pdlLaunchNext();
  const int it = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = it < 8 * F.N;
  const int n = valid ? it >> 3 : 0;
  int i = 0, j = 0, l = 0;
  if (valid) nodeAt(F, n, &i, &j, &l);
  coarseResidualLane(F, layerOf(F, l), n, i, j, it & 7, valid);
}

// b_c = P^T r_f and x_c = 0 (restrictResidual, multigrid.wgsl:204-232) for coarse node I at (ci, cj)
// of its layer, whose fine layer is Lf: the up to 3 x 3 fine nodes, all loads issued together.
__device__ __forceinline__ void restrictAt(const DLevel& F, const DLevel& C, const DLevelLayer& Lf, int I, int ci, int cj) {
  C.X[I] = make_float4(0, 0, 0, 0);
  const uint32_t fixedRow = C.fixed[I];
  const int fi0 = coarseToFine(ci, Lf.nx), fj0 = coarseToFine(cj, Lf.ny);
  float4 w4[9], r4[9];
  uint32_t fx[9];
  bool use[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const int ai = fi0 - 1 + q % 3, aj = fj0 - 1 + q / 3;
    use[q] = ai >= 0 && ai < Lf.nx && aj >= 0 && aj < Lf.ny && weightOf(ai, ci, Lf.nx) != 0.f && weightOf(aj, cj, Lf.ny) != 0.f;
    const int a = use[q] ? levelNode(Lf, ai, aj) : levelNode(Lf, fi0, fj0);
    w4[q] = F.pw[a];
    r4[q] = F.R[a];
    fx[q] = F.fixed[a];
  }
  float3 s = make_float3(0, 0, 0);
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    if (!use[q] || fx[q]) continue;
    const int ai = fi0 - 1 + q % 3, aj = fj0 - 1 + q / 3;
    const Bracket bai = bracketOf(ai, Lf.nx), baj = bracketOf(aj, Lf.ny);
    s += pwSlot(w4[q], (bai.lo == ci ? 0 : 1) + 2 * (baj.lo == cj ? 0 : 1)) * f3(r4[q]);
  }
  C.B[I] = fixedRow ? make_float4(0, 0, 0, 0) : make_float4(s.x, s.y, s.z, 0.f);
}

__global__ void k_restrict(DLevel F, DLevel C) {
  pdlWait();
  pdlLaunchNext();
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= C.N) return;
  int ci, cj, l;
  nodeAt(C, I, &ci, &cj, &l);
  restrictAt(F, C, layerOf(F, l), I, ci, cj);
}

// x_f += P x_c (prolongAdd, multigrid.wgsl:237-258) at fine node a = (i, j) of layers Lf / Lc.
__device__ __forceinline__ void prolongAt(const DLevel& F, const DLevel& C, const DLevelLayer& Lf, const DLevelLayer& Lc, int a, int i, int j) {
  const uint32_t fixedRow = F.fixed[a];
  const Bracket bi = bracketOf(i, Lf.nx), bj = bracketOf(j, Lf.ny);
  const float4 w = F.pw[a];
  const float4 x = F.X[a];
  float3 xc[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) xc[q] = f3(C.X[levelNode(Lc, (q & 1) ? bi.hi : bi.lo, (q & 2) ? bj.hi : bj.lo)]);
  float3 s = make_float3(0, 0, 0);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float wk = pwSlot(w, q);
    if (wk != 0.f) s += wk * xc[q];
  }
  if (!fixedRow) F.X[a] = make_float4(x.x + s.x, x.y + s.y, x.z + s.z, 0.f);
}

__global__ void k_prolong(DLevel F, DLevel C) {
  pdlWait();
  pdlLaunchNext();
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= F.N) return;
  int i, j, l;
  nodeAt(F, a, &i, &j, &l);
  prolongAt(F, C, layerOf(F, l), layerOf(C, l), a, i, j);
}

}  // namespace btd
