// The bottom of the V-cycle in one launch of a thread-block cluster: the level above the coarsest
// (pre-sweep, residual, restriction), the coarsest level's sweeps, then the way back up (prolongation,
// post-sweep) - 27 dependent launches of small grids (one CTA a line, 6-11 lines a colour at 256 x 256)
// become one, with a cluster barrier between the passes in place of a launch boundary.
//
// A cluster of 16 CTAs: CTA b solves line b of every colour pass (sweepLine, the same device code and the
// same arithmetic as k_smooth, so the result is the same bit for bit; CTAs past a colour's line count
// wait), and the residual, restriction and prolongation run over all the cluster's threads with the
// kernels' per-node device code. The pass list is a kernel parameter, the same for every CTA, and no CTA
// leaves early, so every CTA takes every barrier. The unknowns one pass writes reach the next pass's CTAs
// through global memory (L2; the staging loads bypass L1), ordered by the barrier's release / acquire;
// each CTA issues its next line's factor copies before the barrier, as k_smooth does before its
// programmatic-launch wait. Off by default (btd_set_vcycle_tail): measured slower than the launches.
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

// A pass of the tail: a colour pass of one level's sweep, or a transfer over the cluster's threads.
enum TailKind : int { TAIL_SWEEP = 0, TAIL_RESIDUAL = 1, TAIL_RESTRICT = 2, TAIL_PROLONG = 3 };
constexpr int TAIL_MAX_PASSES = 64;

struct TailArgs {
  TailLevel lv[2];  // 0: the level above the coarsest, 1: the coarsest level
  int passes;
  int8_t kind[TAIL_MAX_PASSES], level[TAIL_MAX_PASSES], colour[TAIL_MAX_PASSES];
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
// Every thread of the cluster; the barrier's release / acquire order each pass's global writes (the
// unknowns, residuals, restricted right-hand sides) before the next pass's reads in any CTA.
__device__ __forceinline__ void tailSync() {
  __syncwarp();
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

__global__ void __launch_bounds__(SM_SWEEP_THREADS, 1) k_vtail(TailArgs a) {
  __shared__ uint64_t bar;
  extern __shared__ float4 sm4[];
  const int b = (int)tailRank();
  // the first pass's line copies (factors and couplings are the factorisation's, launches back) are
  // issued before waiting for the preceding kernel, as k_smooth does
  bool prefetched = false;
  if (threadIdx.x == 0) {
    mbarInit(&bar, 1);
    if (a.passes > 0 && a.kind[0] == TAIL_SWEEP && b < a.lv[a.level[0]].count[a.colour[0]]) {
      const TailLevel& t = a.lv[a.level[0]];
      issueLineCopies<CoarseRows>(lineAt(t.geom[a.colour[0]], b), t.fac, t.T, sm4, &bar);
    }
  }
  prefetched = a.passes > 0 && a.kind[0] == TAIL_SWEEP && b < a.lv[a.level[0]].count[a.colour[0]];
  pdlWait();
  pdlLaunchNext();
  __syncthreads();
  unsigned phase = 0;
  const int nt = (int)(blockDim.x * tailCtas());
  const int me = (int)(b * blockDim.x + threadIdx.x);
  const DLevel& F = a.lv[0].L;
  const DLevel& C = a.lv[1].L;
  for (int p = 0; p < a.passes; ++p) {
    const int kind = a.kind[p];
    if (kind == TAIL_SWEEP) {
      const TailLevel& t = a.lv[a.level[p]];
      const int c = a.colour[p];
      if (b < t.count[c]) {
        const LineAt ln = lineAt(t.geom[c], b);
        if (c < 3)
          sweepLine<CoarseRows, 1>(t.L, ln, t.fac, t.T, a.err, sm4, &bar, phase, prefetched);
        else
          sweepLine<CoarseRows, 0>(t.L, ln, t.fac, t.T, a.err, sm4, &bar, phase, prefetched);
      }
    } else if (kind == TAIL_RESIDUAL) {
      // eight threads a node, whole warps in every round
      for (int it0 = 0; it0 < 8 * F.N; it0 += nt) {
        const int it = it0 + me;
        const bool valid = it < 8 * F.N;
        const int n = valid ? it >> 3 : 0;
        int i = 0, j = 0, l = 0;
        if (valid) nodeAt(F, n, &i, &j, &l);
        coarseResidualLane(F, layerOf(F, l), n, i, j, it & 7, valid);
      }
    } else if (kind == TAIL_RESTRICT) {
      for (int I = me; I < C.N; I += nt) {
        int ci, cj, l;
        nodeAt(C, I, &ci, &cj, &l);
        restrictAt(F, C, layerOf(F, l), I, ci, cj);
      }
    } else {
      for (int n = me; n < F.N; n += nt) {
        int i, j, l;
        nodeAt(F, n, &i, &j, &l);
        prolongAt(F, C, layerOf(F, l), layerOf(C, l), n, i, j);
      }
    }
    // the next pass's line copies into this CTA's shared memory before the barrier (they read only the
    // factorisation's output), once every thread is done with the current contents
    prefetched = false;
    if (p + 1 < a.passes && a.kind[p + 1] == TAIL_SWEEP && b < a.lv[a.level[p + 1]].count[a.colour[p + 1]]) {
      __syncthreads();
      if (threadIdx.x == 0) {
        const TailLevel& t = a.lv[a.level[p + 1]];
        issueLineCopies<CoarseRows>(lineAt(t.geom[a.colour[p + 1]], b), t.fac, t.T, sm4, &bar);
      }
      prefetched = true;
    }
    tailSync();
  }
}

}  // namespace btd
