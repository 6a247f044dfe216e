// Self-contact of a cloth layer: a node against a face, an intact lattice cell taken as the two
// triangles (c00 c10 c11) and (c00 c11 c01) (SelfContact, selfcontact.ts:55-163; selfcontact.wgsl).
//
// Penalty E = k (delta - d)^3 / (3 delta) on the node-face distance d (force k s^2 / delta, stiffness
// 2 k s / delta at depth s = delta - d), lagged-normal regularised Coulomb friction on the step
// relative to the face's material point, the reaction on the face's corners by the closest point's
// barycentric weights. Contributions are scattered with fixed-point integer atomics (deterministic
// sums whatever the order) and gathered into ext, the operator seeing them as diagonal blocks.
//
// Once per substep, at the predicted iterate: faces are hashed by centroid (and by their centroid
// at the substep's start when that is another cell) into a 2^17-slot table - count, exclusive scan,
// fill - and each node keeps its K nearest faces within reach plus a directional bound (against the
// first face its predicted path crosses, else the nearest face at the substep's start) that lets its
// step close only a share of the clearance down to a hard core; the face's corners take the
// reciprocal bound. Faces within two lattice cells of a node and still linked to it through
// surviving spans are its own cloth and skipped. Every Newton iteration: terms, then gather.
#pragma once

#include "common.cuh"

namespace btd {

constexpr int CT_K = 4;
constexpr unsigned CT_NONE = 0xFFFFFFFFu;
constexpr float CT_GS = 1e8f;  // fixed-point scale of the gradient (N)
constexpr float CT_HS = 1e3f;  // of the Hessian (N/m)
constexpr int CT_ACC = 9;      // accumulator words per node: gradient xyz, Hessian xx xy xz yy yz zz
constexpr float CT_HARD_CORE = 0.3e-3f;
constexpr int CT_WINDOW = 3;
constexpr float CT_RECIP_UNIT = 1e-5f;
constexpr int CT_TABLE_BITS = 17;

// SELF_CONTACT (selfcontact.ts:7-33).
struct ContactLaw {
  float cell, reach, delta, stiffness, friction, frictionSpeed, boundFraction;
  unsigned mask;  // table slots - 1
};

struct ContactArgs {
  int N;
  const NodeStatic* __restrict__ nodes;
  const DLayer* __restrict__ layers;
  const SimParams* __restrict__ P;
  const uint32_t* __restrict__ pinned;
  const float4* __restrict__ x;
  const float4* __restrict__ dx;
  const Seg* __restrict__ segs;
  unsigned* cells;  // [0, T) counts then start offsets, [T, 2T) fill cursors
  float4* items;    // 2 per hashed face: centroid now + radius, centroid at the start + face index
  unsigned* pairs;  // K per node, then reciprocal keys (N), then row damage marks (N)
  float4* cmeta;    // 2 per node: own bound, reciprocal bound (unit normal, largest approach)
  int* acc;         // CT_ACC per node
  float4* ext;      // 3 per node
  uint8_t* flag;    // per node: contact terms act on it (the learned correction's input), or null
  ContactLaw law;
};

__device__ __forceinline__ float3 ctCur(const ContactArgs& a, int n) { return f3(a.x[n]) + f3(a.dx[n]); }
__device__ __forceinline__ bool ctCloth(const ContactArgs& a, int n) { return a.x[n].w < 1.5f; }
__device__ __forceinline__ void ctCoord(const ContactArgs& a, int n, int* i, int* j, int* l) {
  const NodeStatic s = a.nodes[n];
  *i = s.ij & 0xFFFF, *j = s.ij >> 16, *l = s.layer;
}

// Spatial hash of a cell (the three-prime XOR hash of Teschner et al. 2003).
__device__ __forceinline__ unsigned ctHash(const ContactArgs& a, int cx, int cy, int cz) {
  const unsigned h = ((unsigned)cx * 73856093u) ^ ((unsigned)cy * 19349663u) ^ ((unsigned)cz * 83492791u);
  return h & a.law.mask;
}
__device__ __forceinline__ int3 ctCell(const ContactArgs& a, float3 p) {
  return make_int3((int)floorf(p.x / a.law.cell), (int)floorf(p.y / a.law.cell), (int)floorf(p.z / a.law.cell));
}

// Corners (c00, c10, c01, c11) of the face whose lower-left node is f.
__device__ __forceinline__ int4 ctCorners(const ContactArgs& a, int f) {
  const int nx = a.layers[a.nodes[f].layer].nx;
  return make_int4(f, f + 1, f + nx, f + nx + 1);
}

// An intact cell of the cloth: its four spans hold and its corners are in the solve (faceValid).
__device__ __forceinline__ bool ctFaceValid(const ContactArgs& a, int f) {
  int i, j, l;
  ctCoord(a, f, &i, &j, &l);
  const DLayer& L = a.layers[l];
  if (i + 1 >= L.nx || j + 1 >= L.ny) return false;
  const int4 c = ctCorners(a, f);
  if (!ctCloth(a, c.x) || !ctCloth(a, c.y) || !ctCloth(a, c.z) || !ctCloth(a, c.w)) return false;
  return segActive(a.segs[2 * c.x]) && segActive(a.segs[2 * c.x + 1]) && segActive(a.segs[2 * c.y + 1]) &&
         segActive(a.segs[2 * c.z]);
}

// Closest point of triangle (A, B, C) to p by Voronoi regions (Ericson, Real-Time Collision
// Detection, 5.1.5): barycentric weights and squared distance.
__device__ __forceinline__ float4 ctClosestTri(float3 p, float3 A, float3 B, float3 C) {
  const float3 ab = B - A, ac = C - A, ap = p - A;
  const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  float3 w = make_float3(1.f, 0.f, 0.f);
  if (!(d1 <= 0.f && d2 <= 0.f)) {
    const float3 bp = p - B;
    const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    const float3 cp = p - C;
    const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    const float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
    if (d3 >= 0.f && d4 <= d3) {
      w = make_float3(0.f, 1.f, 0.f);
    } else if (d6 >= 0.f && d5 <= d6) {
      w = make_float3(0.f, 0.f, 1.f);
    } else if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
      const float v = d1 / (d1 - d3);
      w = make_float3(1.f - v, v, 0.f);
    } else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
      const float v = d2 / (d2 - d6);
      w = make_float3(1.f - v, 0.f, v);
    } else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
      const float v = (d4 - d3) / ((d4 - d3) + (d5 - d6));
      w = make_float3(0.f, 1.f - v, v);
    } else {
      const float den = 1.f / (va + vb + vc);
      const float wb = vb * den, wc = vc * den;
      w = make_float3(1.f - wb - wc, wb, wc);
    }
  }
  const float3 q = w.x * A + w.y * B + w.z * C;
  const float3 e = p - q;
  return make_float4(w.x, w.y, w.z, dot3(e, e));
}

struct FaceHit {
  float4 w;  // corner weights (c00, c10, c01, c11)
  float3 q;
  float d;
};

__device__ __forceinline__ FaceHit ctHitP(float3 p, float3 p00, float3 p10, float3 p01, float3 p11) {
  const float4 t1 = ctClosestTri(p, p00, p10, p11), t2 = ctClosestTri(p, p00, p11, p01);
  FaceHit o;
  if (t1.w <= t2.w) {
    o.w = make_float4(t1.x, t1.y, 0.f, t1.z);
    o.d = sqrtf(t1.w);
  } else {
    o.w = make_float4(t2.x, 0.f, t2.z, t2.y);
    o.d = sqrtf(t2.w);
  }
  o.q = o.w.x * p00 + o.w.y * p10 + o.w.z * p01 + o.w.w * p11;
  return o;
}
__device__ __forceinline__ FaceHit ctHit(const ContactArgs& a, float3 p, int4 c) {
  return ctHitP(p, ctCur(a, c.x), ctCur(a, c.y), ctCur(a, c.z), ctCur(a, c.w));
}
__device__ __forceinline__ FaceHit ctHitStart(const ContactArgs& a, float3 p, int4 c) {
  return ctHitP(p, f3(a.x[c.x]), f3(a.x[c.y]), f3(a.x[c.z]), f3(a.x[c.w]));
}

// The face's slots: its predicted centroid's cell, and its start centroid's when that differs.
__device__ __forceinline__ uint2 ctHashFace(const ContactArgs& a, int f) {
  const int4 c = ctCorners(a, f);
  const float3 m1 = 0.25f * (ctCur(a, c.x) + ctCur(a, c.y) + ctCur(a, c.z) + ctCur(a, c.w));
  const float3 m0 = 0.25f * (f3(a.x[c.x]) + f3(a.x[c.y]) + f3(a.x[c.z]) + f3(a.x[c.w]));
  const int3 k1 = ctCell(a, m1), k0 = ctCell(a, m0);
  const unsigned h1 = ctHash(a, k1.x, k1.y, k1.z);
  const bool same = k0.x == k1.x && k0.y == k1.y && k0.z == k1.z;
  return make_uint2(h1, same ? CT_NONE : ctHash(a, k0.x, k0.y, k0.z));
}

// faceCount (selfcontact.wgsl:186-193).
__global__ void k_ct_face_count(ContactArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.N || !ctFaceValid(a, f)) return;
  const uint2 h = ctHashFace(a, f);
  atomicAdd(&a.cells[h.x], 1u);
  if (h.y != CT_NONE) atomicAdd(&a.cells[h.y], 1u);
}

// Exclusive scan of the T cell counts in place (scan.wgsl's result), over the whole GPU in two
// launches: k_ct_scan_tiles sums each tile of 4,096 cells (a CTA of 1,024 threads, four consecutive
// cells a thread, so a warp reads 512 contiguous bytes), then k_ct_scan_apply scans each tile with the
// sum of the tiles before it as its offset. Integer sums: the same result as any order.
constexpr int CT_SCAN_THREADS = 1024, CT_SCAN_ITEMS = 4, CT_SCAN_TILE = CT_SCAN_THREADS * CT_SCAN_ITEMS;
constexpr int CT_SCAN_MAX_TILES = (1 << 20) / CT_SCAN_TILE;  // the largest table (cross-layer, 2^20 cells)

// Exclusive scan of v over the CTA; *total gets the CTA's sum.
__device__ __forceinline__ unsigned ctBlockScan(unsigned v, unsigned* warpSum, unsigned* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned w = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned u = __shfl_up_sync(0xffffffffu, w, o);
    if (lane >= o) w += u;
  }
  if (lane == 31) warpSum[warp] = w;
  __syncthreads();
  if (warp == 0) {
    unsigned x = warpSum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    warpSum[lane] = x;
  }
  __syncthreads();
  *total = warpSum[31];
  return w - v + (warp > 0 ? warpSum[warp - 1] : 0u);
}

__global__ void __launch_bounds__(CT_SCAN_THREADS) k_ct_scan_tiles(const unsigned* __restrict__ cells, int T, unsigned* __restrict__ tileSum) {
  __shared__ unsigned warpSum[32];
  const int base = blockIdx.x * CT_SCAN_TILE + threadIdx.x * CT_SCAN_ITEMS;
  unsigned v = 0;
#pragma unroll
  for (int q = 0; q < CT_SCAN_ITEMS; ++q)
    if (base + q < T) v += cells[base + q];
  unsigned total;
  ctBlockScan(v, warpSum, &total);
  if (threadIdx.x == 0) tileSum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(CT_SCAN_THREADS) k_ct_scan_apply(unsigned* cells, int T, const unsigned* __restrict__ tileSum) {
  __shared__ unsigned warpSum[32];
  __shared__ unsigned tileOff;
  if (threadIdx.x < 32) {
    unsigned o = 0;
    for (int k = threadIdx.x; k < (int)blockIdx.x; k += 32) o += tileSum[k];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) o += __shfl_down_sync(0xffffffffu, o, d);
    if (threadIdx.x == 0) tileOff = o;
  }
  const int base = blockIdx.x * CT_SCAN_TILE + threadIdx.x * CT_SCAN_ITEMS;
  unsigned c[CT_SCAN_ITEMS], v = 0;
#pragma unroll
  for (int q = 0; q < CT_SCAN_ITEMS; ++q) {
    c[q] = base + q < T ? cells[base + q] : 0u;
    v += c[q];
  }
  unsigned total;
  unsigned off = ctBlockScan(v, warpSum, &total);  // its barriers also publish tileOff
  off += tileOff;
#pragma unroll
  for (int q = 0; q < CT_SCAN_ITEMS; ++q) {
    if (base + q < T) cells[base + q] = off;
    off += c[q];
  }
}

// faceFill (selfcontact.wgsl:195-224).
__global__ void k_ct_face_fill(ContactArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.N || !ctFaceValid(a, f)) return;
  const int4 c = ctCorners(a, f);
  const float3 a0 = f3(a.x[c.x]), b0 = f3(a.x[c.y]), e0 = f3(a.x[c.z]), g0 = f3(a.x[c.w]);
  const float3 a1 = a0 + f3(a.dx[c.x]), b1 = b0 + f3(a.dx[c.y]), e1 = e0 + f3(a.dx[c.z]), g1 = g0 + f3(a.dx[c.w]);
  const float3 m0 = 0.25f * (a0 + b0 + e0 + g0), m1 = 0.25f * (a1 + b1 + e1 + g1);
  const float r0 = fmaxf(fmaxf(dot3(a0 - m0, a0 - m0), dot3(b0 - m0, b0 - m0)), fmaxf(dot3(e0 - m0, e0 - m0), dot3(g0 - m0, g0 - m0)));
  const float r1 = fmaxf(fmaxf(dot3(a1 - m1, a1 - m1), dot3(b1 - m1, b1 - m1)), fmaxf(dot3(e1 - m1, e1 - m1), dot3(g1 - m1, g1 - m1)));
  const float4 i1 = make_float4(m1.x, m1.y, m1.z, sqrtf(fmaxf(r0, r1)));
  const float4 i0 = make_float4(m0.x, m0.y, m0.z, (float)f);
  const uint2 h = ctHashFace(a, f);
  const unsigned T = a.law.mask + 1u;
  const unsigned slot = a.cells[h.x] + atomicAdd(&a.cells[T + h.x], 1u);
  a.items[2 * slot] = i1;
  a.items[2 * slot + 1] = i0;
  if (h.y != CT_NONE) {
    const unsigned s0 = a.cells[h.y] + atomicAdd(&a.cells[T + h.y], 1u);
    a.items[2 * s0] = i1;
    a.items[2 * s0 + 1] = i0;
  }
}

__device__ __forceinline__ float ctSegDist(float3 q, float3 A, float3 B) {
  const float3 e = B - A;
  const float s = fminf(fmaxf(dot3(q - A, e) / fmaxf(dot3(e, e), 1e-20f), 0.f), 1.f);
  return len3(q - A - s * e);
}
__device__ __forceinline__ float3 ctCross(float3 u, float3 v) {
  return make_float3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
}
// Segment (o, o + d) against triangle (A, B, C) (Moeller-Trumbore): the crossing's parameter, or 2.
__device__ __forceinline__ float ctSegTri(float3 o, float3 d, float3 A, float3 B, float3 C) {
  const float3 e1 = B - A, e2 = C - A, p = ctCross(d, e2);
  const float det = dot3(e1, p);
  if (fabsf(det) < 1e-18f) return 2.f;
  const float inv = 1.f / det;
  const float3 s = o - A;
  const float u = dot3(s, p) * inv;
  if (u < 0.f || u > 1.f) return 2.f;
  const float3 q = ctCross(s, e1);
  const float v = dot3(d, q) * inv;
  if (v < 0.f || u + v > 1.f) return 2.f;
  const float t = dot3(e2, q) * inv;
  return t >= 0.f && t <= 1.f ? t : 2.f;
}
__device__ __forceinline__ float ctPathCrossing(const ContactArgs& a, float3 o, float3 d, int4 c) {
  const float3 a0 = f3(a.x[c.x]), b0 = f3(a.x[c.y]), e0 = f3(a.x[c.z]), g0 = f3(a.x[c.w]);
  float t = fminf(ctSegTri(o, d, a0, b0, g0), ctSegTri(o, d, a0, g0, e0));
  const float3 a1 = ctCur(a, c.x), b1 = ctCur(a, c.y), e1 = ctCur(a, c.z), g1 = ctCur(a, c.w);
  return fminf(t, fminf(ctSegTri(o, d, a1, b1, g1), ctSegTri(o, d, a1, g1, e1)));
}

// Surviving material along a lattice row / column of layer L between two positions.
__device__ __forceinline__ bool ctRowHolds(const ContactArgs& a, const DLayer& L, int j, int i0, int i1) {
  for (int i = min(i0, i1); i < max(i0, i1); ++i) {
    const int m = L.offset + j * L.nx + i;
    if (!segActive(a.segs[2 * m]) || !ctCloth(a, m) || !ctCloth(a, m + 1)) return false;
  }
  return true;
}
__device__ __forceinline__ bool ctColumnHolds(const ContactArgs& a, const DLayer& L, int i, int j0, int j1) {
  for (int j = min(j0, j1); j < max(j0, j1); ++j) {
    const int m = L.offset + j * L.nx + i;
    if (!segActive(a.segs[2 * m + 1]) || !ctCloth(a, m) || !ctCloth(a, m + L.nx)) return false;
  }
  return true;
}
// latticeLinked (selfcontact.wgsl:290-296).
__device__ __forceinline__ bool ctLinked(const ContactArgs& a, const DLayer& L, int ni, int nj, int fi, int fj) {
  const int ci = min(max(ni, fi), fi + 1), cj = min(max(nj, fj), fj + 1);
  if (ctRowHolds(a, L, nj, ni, ci) && ctColumnHolds(a, L, ci, nj, cj)) return true;
  return ctColumnHolds(a, L, ni, nj, cj) && ctRowHolds(a, L, cj, ni, ci);
}

// damageRow (selfcontact.wgsl:304-320).
__global__ void k_ct_damage_row(ContactArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  int i, j, l;
  ctCoord(a, n, &i, &j, &l);
  const DLayer& L = a.layers[l];
  unsigned mark = 0u;
  for (int q = max(i - CT_WINDOW, 0); q <= min(i + CT_WINDOW, L.nx - 1); ++q) {
    const int m = L.offset + j * L.nx + q;
    if (a.x[m].w > 0.5f || (a.segs[2 * m].flags & SEG_BROKEN) || (a.segs[2 * m + 1].flags & SEG_BROKEN)) mark = 1u;
  }
  a.pairs[(CT_K + 1) * a.N + n] = mark;
}

// detect (selfcontact.wgsl:326-461).
__global__ void __launch_bounds__(128) k_ct_detect(ContactArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  for (int k = 0; k < CT_K; ++k) a.pairs[CT_K * n + k] = CT_NONE;
  if (a.pinned[n] || a.x[n].w > 1.5f) {
    a.cmeta[2 * n] = make_float4(0.f, 0.f, 0.f, 1e9f);
    return;
  }
  const float3 p = ctCur(a, n), p0 = f3(a.x[n]);
  const float3 path = p - p0;
  const bool moving = dot3(path, path) > CT_HARD_CORE * CT_HARD_CORE;
  const float reach = a.law.reach, cell = a.law.cell;
  const unsigned T = a.law.mask + 1u;
  unsigned best[CT_K];
  float bestD[CT_K];
#pragma unroll
  for (int k = 0; k < CT_K; ++k) best[k] = CT_NONE, bestD[k] = 1e9f;
  float d0min = 1e9f;
  float3 n0 = make_float3(0.f, 0.f, 0.f);
  unsigned f0 = CT_NONE;
  float tc = 2.f;
  unsigned fc = CT_NONE;
  const float3 pmin = make_float3(fminf(p.x, p0.x), fminf(p.y, p0.y), fminf(p.z, p0.z));
  const float3 pmax = make_float3(fmaxf(p.x, p0.x), fmaxf(p.y, p0.y), fmaxf(p.z, p0.z));
  const int3 lo = make_int3((int)floorf(pmin.x / cell - 0.5f), (int)floorf(pmin.y / cell - 0.5f), (int)floorf(pmin.z / cell - 0.5f));
  const int3 hi = make_int3(min((int)floorf(pmax.x / cell + 0.5f), lo.x + 3), min((int)floorf(pmax.y / cell + 0.5f), lo.y + 3),
                            min((int)floorf(pmax.z / cell + 0.5f), lo.z + 3));
  int ni, nj, nl;
  ctCoord(a, n, &ni, &nj, &nl);
  const DLayer& NL = a.layers[nl];
  bool damaged = false;
  for (int b = max(nj - CT_WINDOW, 0); b <= min(nj + CT_WINDOW, NL.ny - 1); ++b)
    if (a.pairs[(CT_K + 1) * a.N + NL.offset + b * NL.nx + ni] != 0u) damaged = true;
  for (int cz = lo.z; cz <= hi.z; ++cz)
    for (int cy = lo.y; cy <= hi.y; ++cy)
      for (int cx = lo.x; cx <= hi.x; ++cx) {
        const unsigned h = ctHash(a, cx, cy, cz);
        const unsigned start = a.cells[h], count = a.cells[T + h];
        for (unsigned q = 0; q < count; ++q) {
          const float4 i1 = a.items[2 * (start + q)], i0 = a.items[2 * (start + q) + 1];
          const bool nearNow = len3(p - f3(i1)) - i1.w < reach;
          const bool nearStart = len3(p0 - f3(i0)) - i1.w < fminf(d0min, 0.5f * cell);
          const bool onPath = moving && fminf(ctSegDist(f3(i0), p0, p), ctSegDist(f3(i1), p0, p)) < i1.w;
          if (!nearNow && !nearStart && !onPath) continue;
          const unsigned f = (unsigned)i0.w;
          int fi, fj, fl;
          ctCoord(a, (int)f, &fi, &fj, &fl);
          const int di = fi - ni, dj = fj - nj;
          if (fl == nl && di >= -3 && di <= 2 && dj >= -3 && dj <= 2 && (!damaged || ctLinked(a, NL, ni, nj, ni + di, nj + dj)))
            continue;
          const int4 cf = ctCorners(a, (int)f);
          if (nearStart) {
            const FaceHit s0 = ctHitStart(a, p0, cf);
            if ((s0.d < d0min || (s0.d == d0min && f < f0)) && s0.d > 1e-9f) {
              d0min = s0.d;
              n0 = (1.f / s0.d) * (p0 - s0.q);
              f0 = f;
            }
          }
          if (onPath) {
            const float t = ctPathCrossing(a, p0, path, cf);
            if (t < tc || (t == tc && t <= 1.f && f < fc)) tc = t, fc = f;
          }
          if (!nearNow) continue;
          const FaceHit hit = ctHit(a, p, cf);
          if (hit.d >= reach) continue;
          unsigned cand = f;
          float cd = hit.d;
#pragma unroll
          for (int k = 0; k < CT_K; ++k) {
            if (cand == best[k]) break;
            if (cd < bestD[k] || (cd == bestD[k] && cand < best[k])) {
              const unsigned ts = best[k];
              const float td = bestD[k];
              best[k] = cand, bestD[k] = cd;
              cand = ts, cd = td;
            }
          }
        }
      }
#pragma unroll
  for (int k = 0; k < CT_K; ++k) a.pairs[CT_K * n + k] = best[k];
  float3 nb = n0;
  float db = d0min;
  unsigned fb = f0;
  if (fc != CT_NONE && fc != f0) {
    const int4 c = ctCorners(a, (int)fc);
    const float3 A = f3(a.x[c.x]);
    float3 nrm = ctCross(f3(a.x[c.y]) - A, f3(a.x[c.z]) - A);
    const float ln = len3(nrm);
    if (ln > 1e-12f) {
      nrm = (1.f / ln) * nrm;
      const float side = dot3(p0 - A, nrm);
      nb = side >= 0.f ? nrm : -nrm;
      db = fabsf(side);
      fb = fc;
    }
  }
  if (fb == CT_NONE || (fb == f0 && db >= 0.5f * cell)) {
    a.cmeta[2 * n] = make_float4(0.f, 0.f, 0.f, 1e9f);
    return;
  }
  const float share = a.law.boundFraction * fmaxf(db - CT_HARD_CORE, 0.f);
  a.cmeta[2 * n] = make_float4(nb.x, nb.y, nb.z, share);
  const unsigned key = ((4095u - min(4095u, (unsigned)(share / CT_RECIP_UNIT))) << 20) | (unsigned)(n + 1);
  const int4 c = ctCorners(a, (int)fb);
  unsigned* recip = a.pairs + CT_K * a.N;
  atomicMax(&recip[c.x], key);
  atomicMax(&recip[c.y], key);
  atomicMax(&recip[c.z], key);
  atomicMax(&recip[c.w], key);
}

// resolveBounds (selfcontact.wgsl:463-478): the reciprocal bound of a face corner; clears the keys.
__global__ void k_ct_resolve(ContactArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  unsigned* recip = a.pairs + CT_K * a.N;
  const unsigned key = recip[n];
  recip[n] = 0u;
  if (key == 0u) {
    a.cmeta[2 * n + 1] = make_float4(0.f, 0.f, 0.f, 1e9f);
    return;
  }
  const int j = (int)(key & 0xFFFFFu) - 1;
  const float share = (float)(4095u - (key >> 20)) * CT_RECIP_UNIT;
  const float4 own = a.cmeta[2 * j];
  a.cmeta[2 * n + 1] = make_float4(-own.x, -own.y, -own.z, share);
}

__device__ __forceinline__ int ctFixed(float v) { return (int)fminf(fmaxf(v, -2e9f), 2e9f); }
__device__ __forceinline__ void ctAddTerm(const ContactArgs& a, int n, float3 g, Sym H) {
  int* b = a.acc + CT_ACC * n;
  atomicAdd(b, ctFixed(g.x * CT_GS));
  atomicAdd(b + 1, ctFixed(g.y * CT_GS));
  atomicAdd(b + 2, ctFixed(g.z * CT_GS));
  atomicAdd(b + 3, ctFixed(H.xx * CT_HS));
  atomicAdd(b + 4, ctFixed(H.xy * CT_HS));
  atomicAdd(b + 5, ctFixed(H.xz * CT_HS));
  atomicAdd(b + 6, ctFixed(H.yy * CT_HS));
  atomicAdd(b + 7, ctFixed(H.yz * CT_HS));
  atomicAdd(b + 8, ctFixed(H.zz * CT_HS));
}

// terms (selfcontact.wgsl:493-545): penalty and friction of each candidate pair, the node's
// stiffness doubled and each corner's split by its weight (the pair's closure shared between the
// independent diagonal corrections); the bound's trust region of the linearised penalty.
__global__ void k_ct_terms(ContactArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  const SimParams P = *a.P;
  const float3 p = ctCur(a, n);
  const float delta = a.law.delta, kc = a.law.stiffness, mu = a.law.friction;
  const float epsU = a.law.frictionSpeed * P.h;
  const float4 own = a.cmeta[2 * n];
  float reach = 1e9f;
  const float gmag = sqrtf(P.gx * P.gx + P.gy * P.gy + P.gz * P.gz);
  const float sWeight = sqrtf(a.nodes[n].mass * gmag * delta / kc);
  for (int k = 0; k < CT_K; ++k) {
    const unsigned f = a.pairs[CT_K * n + k];
    if (f == CT_NONE) continue;
    const int4 c = ctCorners(a, (int)f);
    const FaceHit hit = ctHit(a, p, c);
    if (hit.d <= 1e-9f) continue;
    const float3 nn = (1.f / hit.d) * (p - hit.q);
    const float al = dot3(nn, f3(own));
    if (al > 0.1f) reach = fminf(reach, (hit.d - delta + fmaxf(sWeight, 2.f * fmaxf(delta - hit.d, 0.f))) / al);
    if (hit.d >= delta) continue;
    const float s = delta - hit.d;
    const float lam = kc * s * s / delta;
    const float3 rel = f3(a.dx[n]) - (hit.w.x * f3(a.dx[c.x]) + hit.w.y * f3(a.dx[c.y]) + hit.w.z * f3(a.dx[c.z]) + hit.w.w * f3(a.dx[c.w]));
    const float3 ut = rel - dot3(rel, nn) * nn;
    const float kf = mu * lam / fmaxf(len3(ut), epsU);
    const float3 g = -lam * nn + kf * ut;
    const float kn = 2.f * kc * s / delta;
    // H = kn nn^T + kf (I - nn^T)
    const Sym H = {kn * nn.x * nn.x + kf * (1.f - nn.x * nn.x), (kn - kf) * nn.x * nn.y, (kn - kf) * nn.x * nn.z,
                   kn * nn.y * nn.y + kf * (1.f - nn.y * nn.y), (kn - kf) * nn.y * nn.z, kn * nn.z * nn.z + kf * (1.f - nn.z * nn.z)};
    ctAddTerm(a, n, g, H * 2.f);
    const int cs[4] = {c.x, c.y, c.z, c.w};
    const float ws[4] = {hit.w.x, hit.w.y, hit.w.z, hit.w.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (ws[q] <= 0.f) continue;
      ctAddTerm(a, cs[q], -ws[q] * g, H * (2.f * ws[q]));
    }
  }
  if (reach < 1e9f && (own.x != 0.f || own.y != 0.f || own.z != 0.f)) {
    const float approach = -dot3(f3(a.dx[n]), f3(own));
    a.cmeta[2 * n] = make_float4(own.x, own.y, own.z, fminf(own.w, approach + reach));
  }
}

// gather (selfcontact.wgsl:547-564): the accumulated terms into ext (grips add theirs afterwards);
// the accumulator is cleared.
__global__ void k_ct_gather(ContactArgs a) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.N) return;
  int* b = a.acc + CT_ACC * n;
  float v[CT_ACC];
#pragma unroll
  for (int k = 0; k < CT_ACC; ++k) {
    v[k] = (float)b[k] / (k < 3 ? CT_GS : CT_HS);
    b[k] = 0;
  }
  a.ext[3 * n] = make_float4(v[0], v[1], v[2], 0.f);
  a.ext[3 * n + 1] = make_float4(v[3], v[4], v[5], v[6]);
  a.ext[3 * n + 2] = make_float4(v[7], v[8], 0.f, 0.f);
  if (a.flag) a.flag[n] = (v[3] != 0.f || v[4] != 0.f || v[5] != 0.f || v[6] != 0.f || v[7] != 0.f || v[8] != 0.f) ? 1 : 0;
}

}  // namespace btd
