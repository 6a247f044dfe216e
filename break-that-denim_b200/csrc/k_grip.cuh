// Grips: finite material patches held by quadratic springs to a handle (interact.wgsl:96-197;
// ReferenceGrip / gripTerm, solver.ts(ref):29-37, 172-206). Up to GRIPS grips hold disjoint patches
// of at most GRIP_ENTRIES entries, so every ext entry has a single writer.
//   gripLead  once per substep from committed positions: the closing axis of a two-pad pinch, the
//             weighted patch centroid, slip-out of entries torn away from it, and the effective
//             handle = requested handle clamped to within maxLead of the centroid (bounded force)
//   gripTerms every Newton iteration: gradient k w (y - target) and stiffness k w I into ext
//   gripInit  at attach: entry offsets from the picked node and the handle's origin
#pragma once

#include "common.cuh"

namespace btd {

constexpr int GRIPS = 4;
constexpr int GRIP_ENTRIES = 512;

struct GripSlot {
  float4 goal;    // requested handle (xyz, in the frame of anchor), entry count (w)
  float4 params;  // stiffness per unit weight (N/m), largest lead (m), picked node (bits), pinch scale
  float4 anchor;  // where the host took the picked material to be (xyz), pad pitch (w)
  float4 hold;    // slip distance of an entry (x, m; 0: the hold does not slip)
};

struct GripEntry {
  uint32_t node;
  float w;
  float side;  // pad along the closing axis (-1, +1), 0 in a radial pinch
  float pad;
  float4 offset;
};

struct GripArgs {
  const GripSlot* slots;
  GripEntry* entries;  // GRIPS * GRIP_ENTRIES
  float4* goal;        // 3 per grip: effective handle, origin, closing axis
  const float4* x;
  const float4* dx;
  float4* ext;
  int adds;  // 1: add to ext (contact terms wrote it this iteration); 0: the grips own ext and overwrite
};

// A retired node (out of the scene: x.w >= 0.5) is never held (live, interact.wgsl:79).
__device__ __forceinline__ bool liveNode(const float4* x, uint32_t n) { return x[n].w < 0.5f; }

// Target offset of an entry from the handle at pinch scale s (gathered, interact.wgsl:85-90).
__device__ __forceinline__ float3 gathered(const GripEntry& e, const GripSlot& S, float3 axis) {
  const float s = S.params.w;
  if (e.side == 0.f) return s * f3(e.offset);
  return f3(e.offset) - (e.side * (1.f - s) * S.anchor.w) * axis;
}

__device__ __forceinline__ float4 blockSum4(float4 v, float4* red) {
  const int t = threadIdx.x;
  red[t] = v;
  __syncthreads();
  for (int r = blockDim.x / 2; r > 0; r >>= 1) {
    if (t < r) {
      float4 a = red[t], b = red[t + r];
      red[t] = make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
    }
    __syncthreads();
  }
  float4 out = red[0];
  __syncthreads();
  return out;
}

// One block of 256 threads per grip (gripLead, interact.wgsl:96-157).
__global__ void __launch_bounds__(256) k_grip_lead(GripArgs a) {
  __shared__ float4 red[256];
  const int g = blockIdx.x, t = threadIdx.x;
  const GripSlot S = a.slots[g];
  const int count = (int)S.goal.w;
  if (count == 0) return;
  float4 dir = make_float4(0, 0, 0, 0);
  for (int k = t; k < count; k += 256) {
    const GripEntry e = a.entries[g * GRIP_ENTRIES + k];
    const float sw = e.side * e.w;
    dir = make_float4(dir.x + sw * e.offset.x, dir.y + sw * e.offset.y, dir.z + sw * e.offset.z, 0.f);
  }
  const float4 ds = blockSum4(dir, red);
  const float ld = len3(f3(ds));
  const float3 axis = ld > 1e-12f ? (1.f / fmaxf(ld, 1e-20f)) * f3(ds) : make_float3(0, 0, 0);
  float4 acc = make_float4(0, 0, 0, 0);
  for (int k = t; k < count; k += 256) {
    const GripEntry e = a.entries[g * GRIP_ENTRIES + k];
    if (!liveNode(a.x, e.node)) continue;
    const float3 p = f3(a.x[e.node]) - gathered(e, S, axis);
    acc = make_float4(acc.x + e.w * p.x, acc.y + e.w * p.y, acc.z + e.w * p.z, acc.w + e.w);
  }
  const float4 held = blockSum4(acc, red);
  if (held.w > 0.f && S.hold.x > 0.f) {
    const float3 c = (1.f / held.w) * f3(held);
    for (int k = t; k < count; k += 256) {
      const GripEntry e = a.entries[g * GRIP_ENTRIES + k];
      if (e.w > 0.f && liveNode(a.x, e.node) && len3(f3(a.x[e.node]) - gathered(e, S, axis) - c) > S.hold.x) a.entries[g * GRIP_ENTRIES + k].w = 0.f;
    }
  }
  if (t == 0) {
    a.goal[3 * g + 2] = make_float4(axis.x, axis.y, axis.z, 0.f);
    if (held.w <= 0.f) {
      a.goal[3 * g] = make_float4(a.goal[3 * g + 1].x, a.goal[3 * g + 1].y, a.goal[3 * g + 1].z, 0.f);
      return;
    }
    const float3 c = (1.f / held.w) * f3(held);
    const float3 requested = f3(a.goal[3 * g + 1]) + f3(S.goal) - f3(S.anchor);
    float3 lead = requested - c;
    const float l = len3(lead);
    if (l > S.params.y) lead = (S.params.y / l) * lead;
    const float3 h = c + lead;
    a.goal[3 * g] = make_float4(h.x, h.y, h.z, 0.f);
  }
}

// Grip gradient and stiffness into ext (gripTerms, interact.wgsl:159-181).
__global__ void k_grip_terms(GripArgs a) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = id / GRIP_ENTRIES, k = id % GRIP_ENTRIES;
  if (g >= GRIPS) return;
  const GripSlot S = a.slots[g];
  if (k >= (int)S.goal.w) return;
  const GripEntry e = a.entries[id];
  if (!liveNode(a.x, e.node)) return;
  const float3 y = f3(a.x[e.node]) + f3(a.dx[e.node]);
  const float3 d = y - (f3(a.goal[3 * g]) + gathered(e, S, f3(a.goal[3 * g + 2])));
  const float kg = S.params.x * e.w;
  const int b = 3 * e.node;
  float4 e0 = make_float4(0, 0, 0, 0), e1 = e0, e2 = e0;
  if (a.adds) e0 = a.ext[b], e1 = a.ext[b + 1], e2 = a.ext[b + 2];
  a.ext[b] = make_float4(e0.x + kg * d.x, e0.y + kg * d.y, e0.z + kg * d.z, e0.w);
  a.ext[b + 1] = make_float4(e1.x + kg, e1.y, e1.z, e1.w + kg);
  a.ext[b + 2] = make_float4(e2.x, e2.y + kg, e2.z, e2.w);
}

// Offsets from the picked node at attach time and the handle's origin (gripInit, interact.wgsl:185-197).
__global__ void k_grip_init(GripArgs a, int g) {
  const GripSlot S = a.slots[g];
  const uint32_t picked = __float_as_uint(S.params.z);
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id == 0) {
    a.goal[3 * g + 1] = make_float4(a.x[picked].x, a.x[picked].y, a.x[picked].z, 0.f);
    a.goal[3 * g] = a.goal[3 * g + 1];
  }
  if (id >= (int)S.goal.w) return;
  GripEntry& e = a.entries[g * GRIP_ENTRIES + id];
  const float3 o = f3(a.x[e.node]) - f3(a.x[picked]);
  e.offset = make_float4(o.x, o.y, o.z, 0.f);
}

// A grip slot's new value, carried as a launch argument (stream-ordered, no host buffer to keep
// alive or stage).
__global__ void k_grip_set_slot(GripSlot* slots, int g, GripSlot v) { slots[g] = v; }

}  // namespace btd
