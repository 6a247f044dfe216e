// The bottom of the V-cycle in one launch of a thread-block cluster: the level above the coarsest
// (pre-sweep, residual, restriction), the coarsest level's sweeps, then the way back up (prolongation,
// post-sweep) - 27 dependent launches of small grids (one CTA a line, 6-11 lines a colour at 256 x 256)
// become one, with a cluster barrier between the passes in place of a launch boundary.
//
// CTA b of the cluster solves line b of every colour pass (sweepLine, the same device code and the same
// arithmetic as k_smooth, so the result is the same bit for bit); the residual, restriction and
// prolongation run over the cluster's threads with the kernels' per-node device code. Every CTA takes
// every barrier: the passes and their line counts are kernel parameters, the same for all CTAs, and no
// CTA leaves early. The unknowns one pass writes reach the next pass's CTAs through global memory (L2;
// the staging loads bypass L1), ordered by a device-scope fence and the barrier's release/acquire.
#pragma once

#include "common.cuh"
#include "k_mg.cuh"
#include "k_smooth.cuh"

namespace btd {

constexpr int TAIL_MAX_CTAS = 16;  // a non-portable cluster size (16 CTAs on B200)

// One level of the tail: its device view, per colour the launch geometry and line count, the line
// factors and the staging tile.
struct TailLevel {
  DLevel L;
  LineGeom geom[6];
  int count[6];
  const float4* fac;
  int T;
};

struct TailArgs {
  TailLevel up;      // the level above the coarsest
  TailLevel bottom;  // the coarsest level
  int down;          // run the way down: pre-sweep of `up`, its residual, the restriction
  int sweepsFrom, sweepsTo;  // the coarsest level's sweeps [from, to) (odd ones reversed)
  int upward;        // run the way up: prolongation into `up`, its post-sweep (reversed)
  uint32_t* err;
};

__device__ __forceinline__ unsigned tailRank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned tailCtas() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(r));
  return r;
}
// Every thread of the cluster: this pass's global writes ordered before the next pass's reads.
__device__ __forceinline__ void tailSync() {
  __syncwarp();
  __threadfence();
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

__device__ __forceinline__ void tailSweep(const TailLevel& t, bool reverse, float4* sm4, uint64_t* bar, unsigned& phase, uint32_t* err) {
  const int b = (int)tailRank();
  for (int q = 0; q < 6; ++q) {
    const int c = reverse ? 5 - q : q;
    if (t.count[c] == 0) continue;
    if (b < t.count[c]) {
      const LineAt a = lineAt(t.geom[c], b);
      if (c < 3)
        sweepLine<CoarseRows, 1>(t.L, a, t.fac, t.T, err, sm4, bar, phase, false);
      else
        sweepLine<CoarseRows, 0>(t.L, a, t.fac, t.T, err, sm4, bar, phase, false);
    }
    tailSync();
  }
}

__global__ void __launch_bounds__(SM_SWEEP_THREADS, 1) k_vtail(TailArgs a) {
  __shared__ uint64_t bar;
  extern __shared__ float4 sm4[];
  if (threadIdx.x == 0) mbarInit(&bar, 1);
  pdlWait();
  pdlLaunchNext();
  __syncthreads();
  unsigned phase = 0;
  const int nt = (int)(blockDim.x * tailCtas());
  const int me = (int)(tailRank() * blockDim.x + threadIdx.x);
  const DLevel& F = a.up.L;
  const DLevel& C = a.bottom.L;
  if (a.down) {
    tailSweep(a.up, false, sm4, &bar, phase, a.err);
    // residual of the upper level, eight threads a node (whole warps in every round)
    for (int it0 = 0; it0 < 8 * F.N; it0 += nt) {
      const int it = it0 + me;
      const bool valid = it < 8 * F.N;
      const int n = valid ? it >> 3 : 0;
      int i = 0, j = 0, l = 0;
      if (valid) nodeAt(F, n, &i, &j, &l);
      coarseResidualLane(F, layerOf(F, l), n, i, j, it & 7, valid);
    }
    tailSync();
    for (int I = me; I < C.N; I += nt) {
      int ci, cj, l;
      nodeAt(C, I, &ci, &cj, &l);
      restrictAt(F, C, layerOf(F, l), I, ci, cj);
    }
    tailSync();
  }
  for (int sw = a.sweepsFrom; sw < a.sweepsTo; ++sw) tailSweep(a.bottom, (sw & 1) == 1, sm4, &bar, phase, a.err);
  if (a.upward) {
    for (int n = me; n < F.N; n += nt) {
      int i, j, l;
      nodeAt(F, n, &i, &j, &l);
      prolongAt(F, C, layerOf(F, l), layerOf(C, l), n, i, j);
    }
    tailSync();
    tailSweep(a.up, true, sm4, &bar, phase, a.err);
  }
}

}  // namespace btd
