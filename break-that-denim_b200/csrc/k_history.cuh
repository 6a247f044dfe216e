// History after each committed substep: the yarn damage field (yarnField.ts:109-499; yarnfield.wgsl)
// and friction-limited crossing slip (slipNode, solver.ts(ref):685-740; step.wgsl:149-233).
//
// Field arrays per crossing c and family f at 2 c + f: damage code (u8, 255 cut, 254 pulled out),
// cross-section code (u8) and peak tension (f32). Passes, in the reference's order: strain snapshot
// per span; separated-state snapshot; per (span, yarn) damage update (each writes only its own
// crossings); pull-out marks then their application; span coupling and rupture (each span writes
// only its own crossings and tails); then four slip passes (family, parity), whose nodes in one
// pass touch disjoint spans.
#pragma once

#include "common.cuh"
#include "k_step.cuh"

namespace btd {

constexpr int DAMAGE_CUT = 255, DAMAGE_PULLED = 254, DAMAGE_SEPARATED = 254;
constexpr int RECOIL_MAX = 12, SHARE_MAXRUN = 6;
constexpr float SHARE_FRACTION = 0.6f;

struct HistArgs {
  StepArgs S;
  int nSpans;
  int nCross;
  int nLayers;
  float* strain;          // per span (NaN: carries none)
  float* softening;       // per span
  float* failSite;        // per span
  float* tails;           // 4 per node
  uint8_t* damage;        // 2 per crossing
  const uint8_t* __restrict__ area;
  const float* __restrict__ strength;
  uint8_t* sep;           // 2 per crossing
  uint8_t* marks;         // 2 per crossing
  Seg* segsW;             // writable alias of S.segs
};

__device__ __forceinline__ int layerOfNode(const HistArgs& a, int n) { return a.S.nodes[n].layer; }
__device__ __forceinline__ int bundleOfL(const DLayer& L, int f) { return f == 1 ? L.bu : L.bv; }
__device__ __forceinline__ int spanLengthL(const DLayer& L, int f) { return f == 1 ? L.bv : L.bu; }
__device__ __forceinline__ float areaOfCode(int code) { return fmaxf(0.02f, float(code) / 255.f); }
__device__ __forceinline__ int damageCodeOf(float d) { return d >= 1.f ? DAMAGE_CUT : min(DAMAGE_PULLED - 1, (int)floorf(d * 255.f)); }
__device__ __forceinline__ int spanCrossingL(const DLayer& L, int i, int j, int f, int q, int p) {
  if (f == 1) return L.fOffset + (j * L.bv + L.bv / 2 + p) * L.K + i * L.bu + q;
  return L.fOffset + (j * L.bv + q) * L.K + i * L.bu + L.bu / 2 + p;
}

// interpolatedStrain (yarnField.ts:216-240).
__device__ float interpStrain(const DLayer& L, int f, int k, int m, const float* __restrict__ strain) {
  float s = f == 1 ? (k - (L.bu - 1) * 0.5f) / L.bu : (k - (L.bu - 0.5f)) / L.bu;
  float t = f == 1 ? (m - (L.bv - 0.5f)) / L.bv : (m - (L.bv - 1) * 0.5f) / L.bv;
  int i0 = (int)floorf(s), j0 = (int)floorf(t);
  float fu = s - i0, fv = t - j0;
  int imax = f == 1 ? L.nx - 1 : L.nx - 2;
  int jmax = f == 1 ? L.ny - 2 : L.ny - 1;
  float num = 0.f, den = 0.f;
  for (int dj = 0; dj < 2; ++dj)
    for (int di = 0; di < 2; ++di) {
      int i = i0 + di, j = j0 + dj;
      if (i < 0 || j < 0 || i > imax || j > jmax) continue;
      float e = strain[2 * (L.offset + j * L.nx + i) + f];
      if (!finite1(e)) continue;
      float w = (di ? fu : 1.f - fu) * (dj ? fv : 1.f - fv);
      num += w * e;
      den += w;
    }
  return den > 1e-6f ? num / den : __int_as_float(0x7fc00000);
}

// shareFactor (yarnField.ts:303-321) from the separated-state snapshot.
__device__ float shareFactor(const DLayer& L, const uint8_t* __restrict__ sep, int f, int k, int m, int reach, float cap) {
  int along = f == 1 ? m : k, lenAlong = f == 1 ? L.M : L.K;
  int across = f == 1 ? k : m, lenAcross = f == 1 ? L.K : L.M;
  int runs = 0;
  for (int dir = -1; dir <= 1; dir += 2) {
    for (int d = 1; d <= SHARE_MAXRUN; ++d) {
      int yy = across + dir * d;
      if (yy < 0 || yy >= lenAcross) break;
      bool broken = false;
      for (int aa = max(0, along - reach); aa <= min(lenAlong - 1, along + reach) && !broken; ++aa) {
        int c = L.fOffset + (f == 1 ? aa * L.K + yy : yy * L.K + aa);
        broken = sep[2 * c + f] == 1;
      }
      if (!broken) break;
      runs++;
    }
  }
  return 1.f + fminf(SHARE_FRACTION * runs / 2.f, cap);
}

// Strain snapshot per span at the committed positions (updateDamage, solver.ts(ref):661).
__global__ void k_span_strain(HistArgs a) {
  if (!a.S.P->historyOn) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.nSpans) return;
  Seg sg = a.S.segs[s];
  float e = __int_as_float(0x7fc00000);
  if (segActive(sg)) {
    int n = s >> 1, f = s & 1;
    const DLayer& L = a.S.layers[a.S.nodes[n].layer];
    int b = n + (f == 0 ? 1 : L.nx);
    e = len3(f3(a.S.x[b]) - f3(a.S.x[n])) / sg.rest - 1.f;
  }
  a.strain[s] = e;
}

__global__ void k_sep_snapshot(HistArgs a) {
  if (!a.S.P->historyOn) return;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2 * a.nCross) return;
  a.sep[q] = a.damage[q] >= DAMAGE_SEPARATED ? 1 : 0;
}

// updateField (yarnField.ts:338-410): one thread per span, looping over its yarns.
__global__ void k_field_update(HistArgs a) {
  if (!a.S.P->historyOn) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.nSpans) return;
  const Seg sg = a.S.segs[s];
  if (!segActive(sg)) return;
  const int n = s >> 1, f = s & 1;
  const NodeStatic st = a.S.nodes[n];
  const DLayer& L = a.S.layers[st.layer];
  const int i = st.ij & 0xFFFF, j = st.ij >> 16;
  if ((f == 0 && i >= L.nx - 1) || (f == 1 && j >= L.ny - 1)) return;
  const DYarn& y = L.yarn[f];
  const int B = bundleOfL(L, f), P = spanLengthL(L, f);
  const float soft = a.softening[s] / sg.rest;
  const int reach = f == 1 ? L.reachV : L.reachU;
  for (int q = 0; q < B; ++q) {
    if ((sg.cutMask >> q) & 1u) continue;
    const int mid = spanCrossingL(L, i, j, f, q, P >> 1) - L.fOffset;
    const float eps = interpStrain(L, f, mid % L.K, mid / L.K, a.strain);
    if (!finite1(eps)) continue;
    float minPeak = __int_as_float(0x7f800000);
    for (int p = 0; p < P; ++p) {
      int c = spanCrossingL(L, i, j, f, q, p);
      minPeak = fminf(minPeak, strainAtTension(y, a.strength[2 * c + f] * B / areaOfCode(a.area[2 * c + f])));
    }
    if (eps * (1.f + SHARE_FRACTION * SHARE_MAXRUN) <= minPeak) continue;
    const int g = 1 - f;
    const int kM = mid % L.K, mM = mid / L.K;
    const float ec = interpStrain(L, g, kM, mM, a.strain);
    const float tCross = finite1(ec) ? fmaxf(0.f, axialTension(L.yarn[g], ec)) * areaOfCode(a.area[2 * (mid + L.fOffset) + g]) / bundleOfL(L, g) : 0.f;
    const float transfer = ((2 * reach + 1) * L.crossingFriction * (st.n0 / (L.bu * L.bv) + L.crossingWrap * tCross)) / 1.f;
    int best = -1, soft0 = -1, softCode = 0;
    float bestScore = -__int_as_float(0x7f800000), bestOmega = 1.f;
    for (int p = 0; p < P; ++p) {
      int c = spanCrossingL(L, i, j, f, q, p);
      int local = c - L.fOffset;
      float omega = shareFactor(L, a.sep, f, local % L.K, local / L.K, reach, transfer / a.strength[2 * c + f]);
      float peak = strainAtTension(y, a.strength[2 * c + f] * B / areaOfCode(a.area[2 * c + f]));
      float score = omega / peak;
      if (score > bestScore) best = c, bestScore = score, bestOmega = omega;
      if (a.damage[2 * c + f] > softCode) soft0 = c, softCode = a.damage[2 * c + f];
    }
    if (soft0 >= 0) {
      best = soft0;
      int local = best - L.fOffset;
      bestOmega = shareFactor(L, a.sep, f, local % L.K, local / L.K, reach, transfer / a.strength[2 * best + f]);
    }
    int code = damageCodeOf(yarnDamage(y, (float)B, areaOfCode(a.area[2 * best + f]), a.strength[2 * best + f], soft, eps * bestOmega));
    if (code > a.damage[2 * best + f]) a.damage[2 * best + f] = (uint8_t)code;
  }
}

// recoilLength (yarnField.ts:109-115).
__device__ float recoilLength(const DYarn& y, float B, float area, float peak, float eps, float mu, float n0, float wrap,
                              float tCross, float pitch) {
  if (!(eps > 0.f)) return 0.f;
  float share = area / B;
  float e = fminf(eps, strainAtTension(y, peak / share));
  float comp = share * (axialTension(y, e) * e - axialEnergyDensity(y, e));
  return comp * pitch / (mu * (n0 + wrap * fmaxf(0.f, tCross)));
}

// pullOut marks (yarnField.ts:125-152): one thread per crossing, both families.
__global__ void k_pull_mark(HistArgs a, int layer) {
  if (!a.S.P->historyOn) return;
  const DLayer& L = a.S.layers[layer];
  int local = blockIdx.x * blockDim.x + threadIdx.x;
  if (local >= L.K * L.M) return;
  const int k = local % L.K, m = local / L.K;
  const int c = L.fOffset + local;
  for (int f = 0; f < 2; ++f) {
    a.marks[2 * c + f] = 0;
    if (a.damage[2 * c + f] >= DAMAGE_SEPARATED) continue;
    // breakDistance (yarnField.ts:158-177)
    int pos = f == 0 ? k : m, len = f == 0 ? L.K : L.M, stride = f == 0 ? 1 : L.K;
    int best = -1;
    for (int dir = -1; dir <= 1; dir += 2) {
      for (int d = 1; d <= RECOIL_MAX; ++d) {
        int p = pos + dir * d;
        if (p < 0 || p >= len) break;
        int code = a.damage[2 * (c + dir * d * stride) + f];
        if (code == DAMAGE_CUT) {
          if (best < 0 || d < best) best = d;
          break;
        }
        if (code != DAMAGE_PULLED) break;
      }
    }
    if (best < 0) continue;
    float eps = interpStrain(L, f, k, m, a.strain);
    if (!finite1(eps)) continue;
    int g = 1 - f;
    float ec = interpStrain(L, g, k, m, a.strain);
    float tCross = finite1(ec) ? fmaxf(0.f, axialTension(L.yarn[g], ec)) * areaOfCode(a.area[2 * c + g]) / bundleOfL(L, g) : 0.f;
    int ni = min(L.nx - 1, k / L.bu), nj = min(L.ny - 1, m / L.bv);
    int node = L.offset + nj * L.nx + ni;
    float pitch = f == 1 ? L.weavePitchV : L.weavePitchU;
    float delta = recoilLength(L.yarn[f], (float)bundleOfL(L, f), areaOfCode(a.area[2 * c + f]), a.strength[2 * c + f], eps,
                               L.crossingFriction, a.S.nodes[node].n0 / (L.bu * L.bv), L.crossingWrap, tCross, pitch);
    if (delta >= (best - 0.5f) * pitch) a.marks[2 * c + f] = 1;
  }
}

__global__ void k_pull_apply(HistArgs a) {
  if (!a.S.P->historyOn) return;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2 * a.nCross) return;
  if (a.marks[q]) a.damage[q] = DAMAGE_PULLED;
}

// partSpanYarns (yarnField.ts:422-434).
__device__ void partSpanYarns(const DLayer& L, uint8_t* damage, int i, int j, int f, int slipEnd) {
  int P = spanLengthL(L, f), half = P - P / 2;
  for (int q = 0; q < bundleOfL(L, f); ++q) {
    bool ofA = slipEnd != 0;
    for (int p = 0; p < P; ++p) {
      int e = 2 * spanCrossingL(L, i, j, f, q, p) + f;
      if (damage[e] >= DAMAGE_SEPARATED) {
        if (slipEnd < 0) ofA = false;
      } else if (ofA != (p < half)) {
        damage[e] = DAMAGE_PULLED;
      }
    }
  }
}

// coupleSpans (yarnField.ts:443-499): one thread per span.
__global__ void k_couple(HistArgs a) {
  if (!a.S.P->historyOn) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.nSpans) return;
  const int n = s >> 1, f = s & 1;
  const NodeStatic st = a.S.nodes[n];
  const DLayer& L = a.S.layers[st.layer];
  const int i = st.ij & 0xFFFF, j = st.ij >> 16;
  if ((f == 0 && i >= L.nx - 1) || (f == 1 && j >= L.ny - 1)) return;
  Seg sg = a.segsW[s];
  if (sg.flags & SEG_SLIPPED) {
    partSpanYarns(L, a.damage, i, j, f, a.failSite[s] < 0.5f ? 0 : 1);
    a.segsW[s].flags = sg.flags & ~SEG_SLIPPED;
    return;
  }
  if (!segActive(sg)) return;
  const int B = bundleOfL(L, f), P = spanLengthL(L, f);
  float sum = 0.f, site = 0.f;
  uint32_t mask = 0;
  for (int q = 0; q < B; ++q) {
    int dmax = 0, firstSep = -1;
    float compliance = 0.f;
    for (int p = 0; p < P; ++p) {
      int c = spanCrossingL(L, i, j, f, q, p);
      int d = a.damage[2 * c + f];
      if (d > dmax) dmax = d;
      if (d >= DAMAGE_SEPARATED && firstSep < 0) firstSep = p;
      compliance += 1.f / areaOfCode(a.area[2 * c + f]);
    }
    sum += (dmax >= DAMAGE_SEPARATED ? 0.f : 1.f - float(dmax) / 255.f) * (P / compliance);
    if (dmax >= DAMAGE_SEPARATED) {
      mask |= 1u << q;
      site += (firstSep + 0.5f) / P;
    }
  }
  sg.intact = sum / B;
  sg.cutMask = mask;
  uint32_t full = B >= 32 ? 0xFFFFFFFFu : ((1u << B) - 1u);
  if (mask == full) {
    float phi = site / B;
    float rest = sg.rest;
    int b = f == 0 ? n + 1 : n + L.nx;
    sg.flags |= SEG_BROKEN;
    a.failSite[s] = phi;
    a.tails[4 * n + 2 * f + 1] += rest * phi;
    a.tails[4 * b + 2 * f] += rest * (1.f - phi);
    atomicAdd(&a.S.counters[CNT_RUPTURES], 1u);
    partSpanYarns(L, a.damage, i, j, f, -1);
  }
  a.segsW[s] = sg;
}

// Tension of an active span at committed positions and dT/dL at fixed length (segTension,
// solver.ts(ref):647-652).
__device__ __forceinline__ float2 spanTension(const HistArgs& a, int owner, int f) {
  Seg sg = a.segsW[2 * owner + f];
  const DLayer& L = a.S.layers[a.S.nodes[owner].layer];
  int b = owner + (f == 0 ? 1 : L.nx);
  float l = len3(f3(a.S.x[b]) - f3(a.S.x[owner]));
  float Lr = sg.rest;
  float eps = l / Lr - 1.f;
  float T = sg.intact * axialTension(L.yarn[f], eps), K = sg.intact * axialStiffness(L.yarn[f], eps);
  return make_float2(T, fmaxf(K, 0.f) * (l / (Lr * Lr)));
}
__device__ __forceinline__ bool spanOnW(const HistArgs& a, int owner, int f) {
  if (owner < 0) return false;
  return segActive(a.segsW[2 * owner + f]);
}

// slipNode (solver.ts(ref):685-740) for the nodes of one (family, parity) pass.
__global__ void k_slip(HistArgs a, int f, int parity) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= a.S.N) return;
  const SimParams P = *a.S.P;
  if (!P.historyOn) return;
  if (a.S.v[n].w > P.historyTol) return;
  const NodeStatic st = a.S.nodes[n];
  const int i = st.ij & 0xFFFF, j = st.ij >> 16;
  const int along = f == 0 ? i : j;
  if ((along & 1) != parity) return;
  if (a.S.pinned[n]) return;
  const DLayer& L = a.S.layers[st.layer];
  const int du = f == 0 ? 1 : 0, dv = f == 1 ? 1 : 0;
  const int prev = nodeAt(L, i - du, j - dv), next = nodeAt(L, i + du, j + dv);
  if (prev < 0 || next < 0) return;
  const bool actL = spanOnW(a, prev, f), actR = spanOnW(a, n, f);
  if (!actL && !actR) return;
  float2 tl = make_float2(0, 0), tr = make_float2(0, 0);
  if (actL) tl = spanTension(a, prev, f);
  if (actR) tr = spanTension(a, n, f);
  const int g = 1 - f;
  const int cp = nodeAt(L, i - (g == 0 ? 1 : 0), j - (g == 1 ? 1 : 0));
  const int cn = nodeAt(L, i + (g == 0 ? 1 : 0), j + (g == 1 ? 1 : 0));
  float tc = 0.f;
  int cnt = 0;
  if (spanOnW(a, cp, g)) tc += fmaxf(0.f, spanTension(a, cp, g).x), cnt++;
  if (cn >= 0 && spanOnW(a, n, g)) tc += fmaxf(0.f, spanTension(a, n, g).x), cnt++;
  if (cnt == 0) return;
  tc /= cnt;
  const float Fc = L.crossingFriction * (st.n0 + L.crossingWrap * L.yarn[f].yarnsPerSpan * tc);
  const float dT = fmaxf(tr.x, 0.f) - fmaxf(tl.x, 0.f);
  if (fabsf(dT) <= Fc) return;
  const bool highR = dT > 0.f;
  const float kHigh = highR ? tr.y : tl.y;
  const bool lowActive = highR ? actL : actR;
  const float kLow = lowActive ? (highR ? tl.y : tr.y) : 0.f;
  float dl = (fabsf(dT) - Fc) / fmaxf(kHigh + kLow, 1e-9f);
  const float pitch = f == 0 ? L.pitchU : L.pitchV;
  const int sHigh = highR ? 2 * n + f : 2 * prev + f;
  const int sLow = highR ? 2 * prev + f : 2 * n + f;
  if (lowActive) {
    dl = fminf(dl, fmaxf(0.f, a.segsW[sLow].rest - 0.55f * pitch));
    a.segsW[sLow].rest -= dl;
    a.segsW[sHigh].rest += dl;
  } else {
    const int tIdx = highR ? 4 * n + 2 * f : 4 * n + 2 * f + 1;
    dl = fminf(dl, a.tails[tIdx]);
    a.tails[tIdx] -= dl;
    a.segsW[sHigh].rest += dl;
    if (a.tails[tIdx] <= 1e-9f) {
      a.tails[tIdx] = 0.f;
      const int farTail = highR ? 4 * next + 2 * f : 4 * prev + 2 * f + 1;
      a.tails[farTail] += a.segsW[sHigh].rest;
      a.segsW[sHigh].flags |= SEG_BROKEN | SEG_SLIPPED;
      a.failSite[sHigh] = highR ? 0.f : 1.f;
      atomicAdd(&a.S.counters[CNT_PULLED], 1u);
    }
  }
}

}  // namespace btd
