// Learned coarse correction on the coarsest V-cycle level. No counterpart in the reference: its
// coarsest level is two alternating line sweeps (newtonMultigrid.ts:495-502, solver.ts:584-598); this
// adds, half-way through those sweeps, the Galerkin correction on a basis that a small network builds
// from each coarsest node's local data:
//   x += Phi (Phi^T A Phi)^-1 Phi^T (b - A x),  Phi_i = L_i^-T Psi_i,  D_i = L_i L_i^T,
// with D_i the node's diagonal block and Psi_i the network's 3 x 8 output at the node. It is an
// A-orthogonal projection between mirror-image sweeps, so the V-cycle stays symmetric and PCG keeps
// its plain form. Inputs per coarsest node (20, none depending on the residual): lattice position
// u, v with sin/cos(pi u), sin/cos(pi v), sin/cos(2 pi u), sin/cos(2 pi v); D_i / tr D_i (entries 00,
// 11, 22, 01, 02, 12); log(tr D_i / mean tr D); the fraction of the 8 window neighbours fixed or
// outside the lattice; a damage flag and a contact flag restricted from the fine lattice (a coarse
// node takes the OR over the fine nodes its prolongation weights reach).
//
// Kernels: k_lc_flags_fine (per fine node), k_lc_flags_restrict (per coarse node of each level), then
// once per PCG solve k_lc_basis (one CTA: Cholesky of the diagonal blocks and the inputs in FP64, the
// network on the tensor cores, Phi, A Phi, the 8 x 8 Galerkin matrix and its Cholesky factor in
// FP64), and once per V-cycle k_lc_correct (one CTA: residual, Phi^T r in FP64, the small solve, the
// update). The guard lives in the PCG kernels: a solve whose mean contraction per iteration exceeds
// the guard after three iterations turns the correction off and restarts PCG from its iterate.
#pragma once

#include "common.cuh"
#include "k_mg.cuh"
#include "k_mlp.cuh"
#include "k_step.cuh"

namespace btd {

constexpr int LC_THREADS = 512;
constexpr uint8_t LC_DAMAGE = 1, LC_CONTACT = 2;

// Device state of the learned correction (one per solver).
struct LcState {
  int on;         // the correction is enabled for every PCG solve
  int active;     // this solve: on and not fallen back
  int basisOk;    // this solve's basis was built (false: no correction, the guard still counts)
  float guard;    // mean contraction per PCG iteration above which a solve falls back
  int solves, applied, fallbacks;
  int basisGen;   // hierarchy generation of the current basis (-1: none; the weights changed)
  int dead[LC_K];
  double G[LC_K * LC_K];  // Cholesky factor of Phi^T A Phi (lower, row-major), dead columns set to identity
  // logging of training material (the coarsest operators and the residuals at the correction)
  int log;         // logging on
  int gen;         // hierarchy generation (bumped by every Galerkin build)
  int loggedGen;   // generation of the last logged operator
  int curOp;       // logged operator of the current solve (-1: none)
  int nOps, nCalls, capOps, capCalls;
};

struct LcLog {
  float4* rows;     // capOps x COARSE_PLANES x M
  uint32_t* fixed;  // capOps x M
  float* X;         // capOps x M x LC_IN
  float* R;         // capCalls x 3 M
  int* opOf;        // capCalls
};

struct LcArgs {
  LcState* st;
  const MlpPacked* net;
  float* phi;  // 3 M x LC_K
  LcLog log;
  uint8_t* basisFlags;  // M: the coarsest flags the current basis was built with
};

// ---- flags

// Damage flag of fine node n: a span at it exists but is broken or not fully intact; contact flag:
// contact terms act on it (the Hessian of its contact accumulators is nonzero).
__global__ void k_lc_flags_fine(int N, const NodeStatic* __restrict__ nodes, const DLayer* __restrict__ layers,
                                const Seg* __restrict__ segs, const uint8_t* __restrict__ ctFlag, uint8_t* __restrict__ flags) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const NodeStatic st = nodes[n];
  const int i = st.ij & 0xFFFF, j = st.ij >> 16;
  const DLayer& L = layers[st.layer];
  uint8_t f = 0;
#pragma unroll
  for (int fam = 0; fam < 2; ++fam) {
    const int du = fam == 0 ? 1 : 0, dv = fam == 1 ? 1 : 0;
    const int next = nodeAt(L, i + du, j + dv), prev = nodeAt(L, i - du, j - dv);
    const int sp[2] = {next >= 0 ? 2 * n + fam : -1, prev >= 0 ? 2 * prev + fam : -1};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (sp[q] < 0) continue;
      const Seg s = segs[sp[q]];
      if ((s.flags & SEG_EXISTS) && ((s.flags & SEG_BROKEN) || s.intact < 1.f)) f |= LC_DAMAGE;
    }
  }
  if (ctFlag && ctFlag[n]) f |= LC_CONTACT;
  flags[n] = f;
}

// Coarse node I takes the OR of the fine nodes with a nonzero prolongation weight to it.
__global__ void k_lc_flags_restrict(DLevel F, DLevel C, const uint8_t* __restrict__ ff, uint8_t* __restrict__ cf) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= C.N) return;
  int ci, cj, l;
  nodeAt(C, I, &ci, &cj, &l);
  const DLevelLayer Lf = layerOf(F, l);
  const int fi0 = coarseToFine(ci, Lf.nx), fj0 = coarseToFine(cj, Lf.ny);
  uint8_t f = 0;
  for (int q = 0; q < 9; ++q) {
    const int ai = fi0 - 1 + q % 3, aj = fj0 - 1 + q / 3;
    if (ai < 0 || ai >= Lf.nx || aj < 0 || aj >= Lf.ny) continue;
    if (weightOf(ai, ci, Lf.nx) == 0.f || weightOf(aj, cj, Lf.ny) == 0.f) continue;
    const int a = levelNode(Lf, ai, aj);
    const Bracket bai = bracketOf(ai, Lf.nx), baj = bracketOf(aj, Lf.ny);
    if (pwSlot(F.pw[a], (bai.lo == ci ? 0 : 1) + 2 * (baj.lo == cj ? 0 : 1)) > 0.f) f |= ff[a];
  }
  cf[I] = f;
}

__global__ void k_mlp_pack(const float* __restrict__ w, MlpPacked* out) { mlpPack(w, out, threadIdx.x, blockDim.x); }

// A new Galerkin hierarchy was built: its coarsest operator is a new one for logging.
__global__ void k_lc_bump(LcState* st) { st->gen += 1; }

// ---- basis

// Shared-memory layout of k_lc_basis for M coarsest nodes (dynamic; the weights are static).
__host__ __device__ inline size_t lcBasisSmem(int M) {
  const int T = (M + 15) / 16 * 16;  // rows padded to whole MMA tiles
  return (size_t)M * sizeof(double) * 6           // L
         + (size_t)M * LC_OUT * sizeof(float) * 2  // Phi, network output / A Phi
         + (size_t)T * LC_XSTRIDE * 2              // inputs (bf16)
         + (size_t)M * sizeof(float)               // trace
         + (size_t)M;                              // ok
}

// One CTA on the coarsest level C (one layer). Builds this solve's basis; sets st->active = st->on
// and st->basisOk; with logging on and a new operator, also records the operator and its inputs.
__global__ void __launch_bounds__(LC_THREADS) k_lc_basis(DLevel C, const uint8_t* __restrict__ cflags, LcArgs a) {
  extern __shared__ __align__(16) unsigned char lcSmem[];
  __shared__ __align__(16) MlpPacked net;
  __shared__ double red[LC_THREADS / 32][2];
  __shared__ double Gs[LC_K * LC_K];
  __shared__ double trMean;
  const int M = C.N, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int T = (M + 15) / 16 * 16;
  double* sL = reinterpret_cast<double*>(lcSmem);
  float* sPhi = reinterpret_cast<float*>(sL + 6 * M);
  float* sOut = sPhi + (size_t)M * LC_OUT;  // network output, then A Phi
  __nv_bfloat16* sX = reinterpret_cast<__nv_bfloat16*>(sOut + (size_t)M * LC_OUT);
  float* sTr = reinterpret_cast<float*>(sX + (size_t)T * LC_XSTRIDE);
  uint8_t* sOk = reinterpret_cast<uint8_t*>(sTr + M);
  LcState& st = *a.st;
  // the basis is a function of the coarsest operator and its flags alone: when neither changed since
  // it was built (a hierarchy lagged over a substep's Newton iterations, the same contacts), the solve
  // reuses it (every thread reads the same state; not while logging, which records each solve)
  int same = (!st.log && st.basisGen == st.gen) ? 1 : 0;
  if (same) {
    int d = 0;
    for (int n = tid; n < M; n += LC_THREADS) d |= cflags[n] != a.basisFlags[n];
    same = !__syncthreads_or(d);
  }
  if (same) {
    if (tid == 0) {
      st.active = st.on;
      if (st.on) st.solves += 1;
    }
    return;
  }
  for (int q = tid; q < (int)(sizeof(MlpPacked) / 16); q += LC_THREADS)
    reinterpret_cast<float4*>(&net)[q] = reinterpret_cast<const float4*>(a.net)[q];
  const DLevelLayer Ly = C.one;  // the coarsest level of a single-layer lattice

  // diagonal blocks: Cholesky factors and traces (FP64)
  double trSum = 0.0, nOk = 0.0;
  for (int n = tid; n < M; n += LC_THREADS) {
    double L[6] = {0, 0, 0, 0, 0, 0};
    const Sym D = coarseBlock(C.op, M, n, 12);
    const bool ok = !C.fixed[n] && chol3d(D, L);
    for (int q = 0; q < 6; ++q) sL[6 * n + q] = L[q];
    sOk[n] = ok ? 1 : 0;
    const double tr = (double)D.xx + D.yy + D.zz;
    sTr[n] = (float)tr;
    if (ok) trSum += tr, nOk += 1.0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    trSum += __shfl_down_sync(0xffffffffu, trSum, o);
    nOk += __shfl_down_sync(0xffffffffu, nOk, o);
  }
  if (lane == 0) red[warp][0] = trSum, red[warp][1] = nOk;
  __syncthreads();
  __shared__ int freshOp;
  if (tid == 0) {
    double s = 0, c = 0;
    for (int w = 0; w < LC_THREADS / 32; ++w) s += red[w][0], c += red[w][1];
    trMean = c > 0 ? s / c : 0.0;
    // logging: a hierarchy built since the last logged operator gives a new one (while there is room);
    // the solves on the same operator log their calls against it
    freshOp = -1;
    if (!st.log) {
      st.curOp = -1;
    } else if (st.gen != st.loggedGen) {
      st.loggedGen = st.gen;
      st.curOp = st.nOps < st.capOps ? st.nOps++ : -1;
      freshOp = st.curOp;
    }
  }
  __syncthreads();
  const double mean = trMean;
  const int logOp = freshOp;
  const bool fresh = logOp >= 0;

  // inputs (FP64, stored as BF16 for the network; FP32 into the log)
  const double PI = 3.14159265358979323846;
  for (int n = tid; n < T; n += LC_THREADS) {
    double in[LC_IN];
    for (int q = 0; q < LC_IN; ++q) in[q] = 0.0;
    if (n < M && sOk[n] && mean > 0.0) {
      const int i = (n - Ly.offset) % Ly.nx, j = (n - Ly.offset) / Ly.nx;
      const double u = Ly.nx > 1 ? (double)i / (Ly.nx - 1) : 0.0, v = Ly.ny > 1 ? (double)j / (Ly.ny - 1) : 0.0;
      int q = 0;
      in[q++] = u;
      in[q++] = v;
      for (int f = 1; f <= 2; ++f) {
        in[q++] = sin(f * PI * u);
        in[q++] = cos(f * PI * u);
        in[q++] = sin(f * PI * v);
        in[q++] = cos(f * PI * v);
      }
      const Sym D = coarseBlock(C.op, M, n, 12);
      const double tr = (double)D.xx + D.yy + D.zz;
      in[q++] = D.xx / tr;
      in[q++] = D.yy / tr;
      in[q++] = D.zz / tr;
      in[q++] = D.xy / tr;
      in[q++] = D.xz / tr;
      in[q++] = D.yz / tr;
      in[q++] = log(tr / mean);
      int held = 0;
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          if (!di && !dj) continue;
          const int m = levelNode(Ly, i + di, j + dj);
          if (m < 0 || C.fixed[m]) held++;
        }
      in[q++] = held / 8.0;
      const uint8_t fl = cflags ? cflags[n] : 0;
      in[q++] = (fl & LC_DAMAGE) ? 1.0 : 0.0;
      in[q++] = (fl & LC_CONTACT) ? 1.0 : 0.0;
    }
    for (int q = 0; q < LC_IN_PAD; ++q) sX[n * LC_XSTRIDE + q] = __float2bfloat16_rn(q < LC_IN ? (float)in[q] : 0.f);
    if (fresh && n < M)
      for (int q = 0; q < LC_IN; ++q) a.log.X[((size_t)logOp * M + n) * LC_IN + q] = (float)in[q];
  }
  if (fresh) {
    for (int q = tid; q < COARSE_PLANES * M; q += LC_THREADS) a.log.rows[(size_t)logOp * COARSE_PLANES * M + q] = C.op[q];
    for (int n = tid; n < M; n += LC_THREADS) a.log.fixed[(size_t)logOp * M + n] = C.fixed[n];
  }
  __syncthreads();

  // the network: one warp per 16-row tile
  for (int tile = warp; tile < T / 16; tile += LC_THREADS / 32) {
    float out[3][4];
    mlpForwardTile(net, sX + tile * 16 * LC_XSTRIDE, lane, out);
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 3; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = tile * 16 + g + 8 * h;
        if (r < M) {
          sOut[r * LC_OUT + 8 * nt + 2 * t] = out[nt][2 * h];
          sOut[r * LC_OUT + 8 * nt + 2 * t + 1] = out[nt][2 * h + 1];
        }
      }
  }
  __syncthreads();

  // Phi_n = L_n^-T Psi_n (rows 3 n + c, column k at sPhi[(3 n + c) LC_K + k])
  for (int n = tid; n < M; n += LC_THREADS) {
    const double* L = sL + 6 * n;
    for (int k = 0; k < LC_K; ++k) {
      double p0 = 0, p1 = 0, p2 = 0;
      if (sOk[n]) {
        const float* o = sOut + (size_t)n * LC_OUT;
        p2 = (double)o[3 * k + 2] / L[5];
        p1 = ((double)o[3 * k + 1] - L[4] * p2) / L[2];
        p0 = ((double)o[3 * k] - L[1] * p1 - L[3] * p2) / L[0];
      }
      sPhi[(3 * n) * LC_K + k] = (float)p0;
      sPhi[(3 * n + 1) * LC_K + k] = (float)p1;
      sPhi[(3 * n + 2) * LC_K + k] = (float)p2;
    }
  }
  __syncthreads();

  // A Phi (fixed rows zero) into sOut
  for (int n = tid; n < M; n += LC_THREADS) {
    float y[3][LC_K];
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < LC_K; ++k) y[c][k] = 0.f;
    if (!C.fixed[n]) {
      const int i = (n - Ly.offset) % Ly.nx, j = (n - Ly.offset) / Ly.nx;
      for (int o = 0; o < 25; ++o) {
        const int m = levelNode(Ly, i + o % 5 - 2, j + o / 5 - 2);
        if (m < 0) continue;
        const Sym B = coarseBlock(C.op, M, n, o);
        const float* pm = sPhi + (size_t)3 * m * LC_K;
        for (int k = 0; k < LC_K; ++k) {
          const float v0 = pm[k], v1 = pm[LC_K + k], v2 = pm[2 * LC_K + k];
          y[0][k] += B.xx * v0 + B.xy * v1 + B.xz * v2;
          y[1][k] += B.xy * v0 + B.yy * v1 + B.yz * v2;
          y[2][k] += B.xz * v0 + B.yz * v1 + B.zz * v2;
        }
      }
    }
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < LC_K; ++k) sOut[(3 * n + c) * LC_K + k] = y[c][k];
  }
  __syncthreads();

  // G = Phi^T A Phi (FP64 sums), a warp per entry
  for (int e = warp; e < LC_K * LC_K; e += LC_THREADS / 32) {
    const int r = e / LC_K, c = e % LC_K;
    double s = 0.0;
    for (int q = lane; q < 3 * M; q += 32) s += (double)sPhi[q * LC_K + r] * (double)sOut[q * LC_K + c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) Gs[e] = s;
  }
  for (int q = tid; q < 3 * M * LC_K; q += LC_THREADS) a.phi[q] = sPhi[q];
  for (int n = tid; n < M; n += LC_THREADS) a.basisFlags[n] = cflags[n];
  __syncthreads();

  // symmetrise; Cholesky with dependent columns (pivot below 1e-10 of the largest diagonal) dropped
  if (tid == 0) {
    double G[LC_K * LC_K];
    for (int r = 0; r < LC_K; ++r)
      for (int c = 0; c < LC_K; ++c) G[r * LC_K + c] = 0.5 * (Gs[r * LC_K + c] + Gs[c * LC_K + r]);
    double gmax = 0.0;
    for (int r = 0; r < LC_K; ++r) gmax = fmax(gmax, G[r * LC_K + r]);
    bool ok = gmax > 0.0 && isfinite(gmax);
    for (int jc = 0; jc < LC_K && ok; ++jc) {
      double d = G[jc * LC_K + jc];
      for (int q = 0; q < jc; ++q) d -= G[jc * LC_K + q] * G[jc * LC_K + q];
      if (!(d > 1e-10 * gmax)) {
        st.dead[jc] = 1;
        for (int r = jc; r < LC_K; ++r) G[r * LC_K + jc] = 0.0;
        G[jc * LC_K + jc] = 1.0;
        continue;
      }
      st.dead[jc] = 0;
      d = sqrt(d);
      G[jc * LC_K + jc] = d;
      for (int r = jc + 1; r < LC_K; ++r) {
        double v = G[r * LC_K + jc];
        for (int q = 0; q < jc; ++q) v -= G[r * LC_K + q] * G[jc * LC_K + q];
        G[r * LC_K + jc] = v / d;
      }
    }
    for (int q = 0; q < LC_K * LC_K; ++q) st.G[q] = G[q];
    st.basisOk = ok ? 1 : 0;
    st.basisGen = st.gen;
    st.active = st.on;
    if (st.on) st.solves += 1;
  }
}

// ---- correction (between the coarsest sweeps, every V-cycle)

// One CTA: r = b - A x on the coarsest level (fixed rows 0), u = Phi^T r (FP64, dead columns 0),
// G c = u, x += Phi c. Skipped when the solve fell back or its basis failed. Logs r when logging.
__global__ void __launch_bounds__(LC_THREADS) k_lc_correct(DLevel C, LcArgs a) {
  pdlWait();
  pdlLaunchNext();
  __shared__ double red[LC_THREADS / 32][LC_K];
  __shared__ float cs[LC_K];
  LcState& st = *a.st;
  const bool apply = st.active && st.basisOk;
  const int logOp = st.log ? st.curOp : -1;
  __shared__ int slot;
  if (threadIdx.x == 0) {
    slot = -1;
    if (logOp >= 0 && st.nCalls < st.capCalls) {
      slot = st.nCalls++;
      a.log.opOf[slot] = logOp;
    }
  }
  __syncthreads();
  if (!apply && slot < 0) return;
  const int M = C.N, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const DLevelLayer Ly = C.one;
  double u[LC_K];
  for (int k = 0; k < LC_K; ++k) u[k] = 0.0;
  for (int n = tid; n < M; n += LC_THREADS) {
    float3 r = make_float3(0, 0, 0);
    if (!C.fixed[n]) {
      const int i = (n - Ly.offset) % Ly.nx, j = (n - Ly.offset) / Ly.nx;
      r = f3(C.B[n]);
      // unrolled: the 25 blocks' loads are independent and go out together (the sums keep their order)
#pragma unroll
      for (int o = 0; o < 25; ++o) {
        const int m = levelNode(Ly, i + o % 5 - 2, j + o / 5 - 2);
        if (m < 0) continue;
        r -= coarseBlock(C.op, M, n, o) * f3(C.X[m]);
      }
    }
    if (slot >= 0) {
      float* R = a.log.R + (size_t)slot * 3 * M + 3 * n;
      R[0] = r.x, R[1] = r.y, R[2] = r.z;
    }
    const float* p = a.phi + (size_t)3 * n * LC_K;
    for (int k = 0; k < LC_K; ++k) u[k] += (double)p[k] * r.x + (double)p[LC_K + k] * r.y + (double)p[2 * LC_K + k] * r.z;
  }
  if (!apply) return;
#pragma unroll
  for (int k = 0; k < LC_K; ++k) {
    double s = u[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp][k] = s;
  }
  __syncthreads();
  if (tid == 0) {
    double uu[LC_K], c[LC_K];
    for (int k = 0; k < LC_K; ++k) {
      double s = 0.0;
      for (int w = 0; w < LC_THREADS / 32; ++w) s += red[w][k];
      uu[k] = st.dead[k] ? 0.0 : s;
    }
    for (int i = 0; i < LC_K; ++i) {  // G c = u with G = R R^T (R lower)
      double v = uu[i];
      for (int q = 0; q < i; ++q) v -= st.G[i * LC_K + q] * c[q];
      c[i] = st.dead[i] ? 0.0 : v / st.G[i * LC_K + i];
    }
    for (int i = LC_K - 1; i >= 0; --i) {
      double v = c[i];
      for (int q = i + 1; q < LC_K; ++q) v -= st.G[q * LC_K + i] * c[q];
      c[i] = st.dead[i] ? 0.0 : v / st.G[i * LC_K + i];
    }
    for (int k = 0; k < LC_K; ++k) cs[k] = (float)c[k];
    st.applied += 1;
  }
  __syncthreads();
  for (int n = tid; n < M; n += LC_THREADS) {
    const float* p = a.phi + (size_t)3 * n * LC_K;
    float3 d = make_float3(0, 0, 0);
    for (int k = 0; k < LC_K; ++k) d += cs[k] * make_float3(p[k], p[LC_K + k], p[2 * LC_K + k]);
    const float4 x = C.X[n];
    C.X[n] = make_float4(x.x + d.x, x.y + d.y, x.z + d.z, x.w);
  }
}

}  // namespace btd
