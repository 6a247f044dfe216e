// Cross-layer contact (contact.ts:7-19, 49-50; contact.wgsl:31-164): a scene of several layers gets
// node-node contact between its layers in place of self-contact (solver.ts:364). Detection once per
// substep at the predicted iterate on a (cell, layer) hash with the reference's hash function and table
// size (so hash collisions bring the same extra candidates): count, scan, fill, then per node the
// CT_K nearest nodes of other layers within the pair's contact distance and a quarter cell, and a
// directional bound toward the nearest one. Terms per Newton iterate: a linear penalty and
// lagged-normal regularised Coulomb friction on the relative tangential step, each node's own terms
// written into its external block (no scatter: a pair acts on both nodes through both their lists).
#pragma once

#include "common.cuh"
#include "k_contact.cuh"

namespace btd {

constexpr unsigned XC_MASK = (1u << 20) - 1u;
constexpr float XC_CELL = 1.0e-3f, XC_K_PEN = 3000.f, XC_MU = 0.45f, XC_FRICTION_SPEED = 0.002f, XC_BOUND_FRACTION = 0.45f;

struct XcArgs {
  int N;
  const NodeStatic* __restrict__ nodes;
  const SimParams* __restrict__ P;
  const float4* __restrict__ x;
  const float4* __restrict__ dx;
  unsigned* cells;  // 2 (XC_MASK + 1): cell starts (scanned counts), then fill counters
  int* items;       // N: nodes by cell
  int* cand;        // CT_K per node
  float4* cmeta;    // 2 per node: the directional bound, the (absent) reciprocal one
  float4* ext;      // 3 per node
  uint8_t* flag;    // per node: contact terms act on it (or null)
  float dist[4];    // contact distance of layer pairs 0-1, 0-2, 1-2 (mean thickness), same layer
};

// hashCell (contact.wgsl:31-34)
__device__ __forceinline__ unsigned xcHash(int cx, int cy, int cz, unsigned l) {
  return (((unsigned)cx * 73856093u) ^ ((unsigned)cy * 19349663u) ^ ((unsigned)cz * 83492791u) ^ (l * 2654435761u)) & XC_MASK;
}
// pairDistance (contact.wgsl:36-42)
__device__ __forceinline__ float xcPair(const XcArgs& a, unsigned la, unsigned lb) {
  if (la == lb) return a.dist[3];
  const unsigned s = la + lb;
  return s == 1 ? a.dist[0] : s == 2 ? a.dist[1] : a.dist[2];
}
// The node's position at the iterate and its cell (floor of the position over the cell size, in FP64).
__device__ __forceinline__ void xcCell(const XcArgs& a, int n, float3* p, int* c) {
  const float4 x = a.x[n], d = a.dx[n];
  const double px = (double)x.x + d.x, py = (double)x.y + d.y, pz = (double)x.z + d.z;
  *p = make_float3((float)px, (float)py, (float)pz);
  c[0] = (int)floor(px / 1.0e-3), c[1] = (int)floor(py / 1.0e-3), c[2] = (int)floor(pz / 1.0e-3);
}

__global__ void k_xc_count(XcArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  float3 p;
  int c[3];
  xcCell(a, n, &p, c);
  atomicAdd(&a.cells[xcHash(c[0], c[1], c[2], a.nodes[n].layer)], 1u);
}

__global__ void k_xc_fill(XcArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  float3 p;
  int c[3];
  xcCell(a, n, &p, c);
  const unsigned h = xcHash(c[0], c[1], c[2], a.nodes[n].layer);
  a.items[a.cells[h] + atomicAdd(&a.cells[XC_MASK + 1u + h], 1u)] = n;
}

// detect (contact.wgsl:46-129): the CT_K nearest foreign nodes within the pair distance and a quarter
// cell, and the directional bound: approach the nearest foreign node by a share of its clearance plus
// half the contact distance (of the 0-1 pair, as the shader takes it); no reciprocal bound.
__global__ void k_xc_detect(XcArgs a, int nLayers) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  float3 p;
  int c[3];
  xcCell(a, n, &p, c);
  const unsigned ln = a.nodes[n].layer;
  int best[CT_K];
  float bestD[CT_K];
#pragma unroll
  for (int k = 0; k < CT_K; ++k) best[k] = -1, bestD[k] = 1e9f;
  float dmin = 1e9f;
  float3 nmin = make_float3(0, 0, 0);
  for (int lo = 0; lo < nLayers; ++lo) {
    if ((unsigned)lo == ln) continue;
    const float r = xcPair(a, ln, (unsigned)lo);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dxc = -1; dxc <= 1; ++dxc) {
          const unsigned h = xcHash(c[0] + dxc, c[1] + dy, c[2] + dz, (unsigned)lo);
          const unsigned s0 = a.cells[h], s1 = s0 + a.cells[XC_MASK + 1u + h];
          for (unsigned q = s0; q < s1; ++q) {
            const int m = a.items[q];
            if (a.nodes[m].layer != (unsigned)lo) continue;
            const float4 xm = a.x[m], dm = a.dx[m];
            const float3 pm = make_float3(xm.x + dm.x, xm.y + dm.y, xm.z + dm.z);
            const float3 dv = p - pm;
            const float d = len3(dv);
            if (d - r < dmin && d > 1e-9f) {
              dmin = d - r;
              nmin = (1.f / d) * dv;
            }
            if (d >= r + 0.25f * XC_CELL) continue;
            int cnd = m;
            float cd = d - r;
#pragma unroll
            for (int k = 0; k < CT_K; ++k)
              if (cd < bestD[k]) {
                const int ti = best[k];
                const float td = bestD[k];
                best[k] = cnd, bestD[k] = cd;
                cnd = ti, cd = td;
              }
          }
        }
  }
#pragma unroll
  for (int k = 0; k < CT_K; ++k) a.cand[CT_K * n + k] = best[k];
  a.cmeta[2 * n] = dmin < 1e8f ? make_float4(nmin.x, nmin.y, nmin.z, XC_BOUND_FRACTION * (fmaxf(0.f, dmin) + 0.5f * a.dist[0]))
                               : make_float4(0, 0, 0, 1e9f);
  a.cmeta[2 * n + 1] = make_float4(0, 0, 0, 1e9f);
}

// terms (contact.wgsl:131-164): per candidate within its pair distance, the penalty k (r - d) along the
// normal and regularised Coulomb friction mu lambda on the relative tangential step; the node's own
// gradient and Hessian block into ext.
__global__ void k_xc_terms(XcArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  const float4 xn = a.x[n], dn = a.dx[n];
  const float3 p = make_float3(xn.x + dn.x, xn.y + dn.y, xn.z + dn.z);
  const float epsU = XC_FRICTION_SPEED * a.P->h;
  const unsigned ln = a.nodes[n].layer;
  float3 g = make_float3(0, 0, 0);
  Sym H = symZero();
#pragma unroll
  for (int k = 0; k < CT_K; ++k) {
    const int m = a.cand[CT_K * n + k];
    if (m < 0) continue;
    const float4 xm = a.x[m], dm = a.dx[m];
    const float3 dv = p - make_float3(xm.x + dm.x, xm.y + dm.y, xm.z + dm.z);
    const float d = len3(dv), r = xcPair(a, ln, a.nodes[m].layer);
    if (d >= r || d <= 1e-9f) continue;
    const float3 nn = (1.f / d) * dv;
    const float lam = XC_K_PEN * (r - d);
    const float3 rel = f3(dn) - f3(dm);
    const float rn = dot3(rel, nn);
    const float3 ut = rel - rn * nn;
    const float kf = XC_MU * lam / fmaxf(len3(ut), epsU);
    g += -lam * nn + kf * ut;
    H = H + axialBlock(XC_K_PEN, kf, nn);
  }
  a.ext[3 * n] = make_float4(g.x, g.y, g.z, 0.f);
  a.ext[3 * n + 1] = make_float4(H.xx, H.xy, H.xz, H.yy);
  a.ext[3 * n + 2] = make_float4(H.yz, H.zz, 0.f, 0.f);
  if (a.flag) a.flag[n] = (H.xx != 0.f || H.yy != 0.f || H.zz != 0.f) ? 1 : 0;
}

}  // namespace btd
