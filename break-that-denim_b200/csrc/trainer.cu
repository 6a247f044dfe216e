// Training of the learned coarse space's network on the GPU (no counterpart in the reference: an
// extension of its coarsest V-cycle level, newtonMultigrid.ts:495-502). The material is what the
// solver logs (btd_learned_log): per coarsest operator its rows and its nodes' network inputs, per
// correction call the coarsest residual. Ingestion whitens each operator by its diagonal blocks
// (At = L^-1 A L^-T over the free unknowns, D_i = L_i L_i^T), factors it (dense Cholesky, FP64) and
// solves every call's exact correction d = At^-1 r of its whitened residual r.
//
// Objective (per call): the share of the call's error energy that the Galerkin correction on the
// network's basis Psi (3 n x 8, whitened frame) captures,
//   q = u^T G^-1 u / (r^T d),  u = Psi^T r,  G = Psi^T At Psi (+ 1e-8 tr(G) / 8 I),
// the loss the mean of 1 - q over a minibatch's calls, dq/dPsi = 2 (r - At Psi c) c^T / (r^T d) with
// c = G^-1 u. A step: the network forward over the minibatch's nodes (BF16 MMAs, FP32 accumulation),
// one CTA per operator for At Psi, G, the calls' u, c, q and dPsi (FP32 products, FP64 sums and small
// solves), the backward pass (BF16 MMAs, FP32 accumulation; weight gradients per CTA, summed in a fixed
// order), then Adam on FP32 master weights and the repacking of the BF16 fragments.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "btd.h"
#include "common.cuh"
#include "k_mlp.cuh"

namespace btd {
void setError(const std::string& msg);
}
using namespace btd;

namespace {

struct TrError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define TK(call)                                                                                       \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) throw TrError(std::string(#call) + ": " + cudaGetErrorString(e_));          \
  } while (0)

constexpr int TR_ROWS = 64;        // network rows per CTA (4 warps x 16)
inline int blocksOf(int n, int t) { return (n + t - 1) / t; }
constexpr int TR_OP_THREADS = 512; // per-operator CTA
constexpr double TR_RIDGE = 1e-8;
constexpr int TR_MAX_BATCH = 16;
constexpr int TR_MAX_NODES = LC_MAX_NODES;

// One operator of the training material on the device.
struct TrOp {
  const float* At;  // D3 x D3 (symmetric)
  const float* X;   // n x LC_IN
  const float* R;   // calls x D3 whitened residuals
  const float* D;   // calls x D3 exact corrections
  const double* E;  // calls: r . d
  int n, D3, calls, pad;
};

// ------------------------------------------------------------------------------------------- forward

// Row r of a minibatch (its operators' nodes in order) -> (operator slot, node).
__device__ __forceinline__ int batchSlot(const int* rowStart, int nb, int r) {
  int b = 0;
  while (b + 1 < nb && r >= rowStart[b + 1]) ++b;
  return b;
}

// Loads a 16-row input tile (bf16, stride LC_XSTRIDE, padded columns zero) of minibatch rows row0.. .
__device__ void loadInputTile(const TrOp* ops, const int* batch, const int* rowStart, int nb, int rows, int row0,
                              __nv_bfloat16* X, int lane) {
  for (int q = lane; q < 16 * LC_IN_PAD; q += 32) {
    const int r = q / LC_IN_PAD, c = q % LC_IN_PAD, row = row0 + r;
    float v = 0.f;
    if (row < rows && c < LC_IN) {
      const int b = batchSlot(rowStart, nb, row);
      const TrOp& o = ops[batch[b]];
      v = o.X[(size_t)(row - rowStart[b]) * LC_IN + c];
    }
    X[r * LC_XSTRIDE + c] = __float2bfloat16_rn(v);
  }
  __syncwarp();
}

__global__ void __launch_bounds__(128) k_tr_forward(const TrOp* __restrict__ ops, const int* __restrict__ batch,
                                                    const int* __restrict__ rowStart, int nb, const MlpPacked* __restrict__ P,
                                                    float* __restrict__ out) {
  __shared__ __align__(16) __nv_bfloat16 X[4][16 * LC_XSTRIDE];
  __shared__ __align__(16) MlpPacked net;
  for (int q = threadIdx.x; q < (int)(sizeof(MlpPacked) / 16); q += blockDim.x)
    reinterpret_cast<float4*>(&net)[q] = reinterpret_cast<const float4*>(P)[q];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, rows = rowStart[nb];
  const int row0 = blockIdx.x * TR_ROWS + 16 * warp;
  if (row0 >= rows) return;
  loadInputTile(ops, batch, rowStart, nb, rows, row0, X[warp], lane);
  float o[3][4];
  mlpForwardTile(net, X[warp], lane, o);
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 3; ++nt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = row0 + g + 8 * h;
      if (r < rows) {
        out[(size_t)r * LC_OUT + 8 * nt + 2 * t] = o[nt][2 * h];
        out[(size_t)r * LC_OUT + 8 * nt + 2 * t + 1] = o[nt][2 * h + 1];
      }
    }
}

// ------------------------------------------------------------------------------- per-operator algebra

__host__ __device__ inline size_t trOpSmem(int D3) { return (size_t)3 * D3 * LC_K * sizeof(float); }

// One CTA per operator of the minibatch: Psi from the network output, At Psi, G (+ ridge) and its
// Cholesky factor, then per call u = Psi^T r, c = G^-1 u, q = u . c / E (loss 1 - q) and
// dPsi += (r - At Psi c) c^T / E; finally dOut = -2 scale dPsi in the output layout.
__global__ void __launch_bounds__(TR_OP_THREADS) k_tr_operator(const TrOp* __restrict__ ops, const int* __restrict__ batch,
                                                               const int* __restrict__ rowStart, const float* __restrict__ out,
                                                               float* __restrict__ dOut, double* __restrict__ lossOut, double scale) {
  extern __shared__ __align__(16) float trSmem[];
  __shared__ double red[TR_OP_THREADS / 32][LC_K];
  __shared__ double Gs[LC_K * LC_K];
  __shared__ double cc[LC_K];
  __shared__ int gok;
  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const TrOp o = ops[batch[b]];
  const int D3 = o.D3, r0 = rowStart[b];
  float* Psi = trSmem;                  // D3 x 8
  float* AP = Psi + (size_t)D3 * LC_K;  // D3 x 8
  float* dPsi = AP + (size_t)D3 * LC_K; // D3 x 8
  for (int q = tid; q < D3 * LC_K; q += TR_OP_THREADS) {
    const int row = q / LC_K, k = q % LC_K;  // row 3 i + c
    Psi[q] = out[(size_t)(r0 + row / 3) * LC_OUT + 3 * k + row % 3];
    dPsi[q] = 0.f;
  }
  __syncthreads();
  // At Psi: At is symmetric, so row q of the product reads column q of At (coalesced across threads)
  for (int q = tid; q < D3; q += TR_OP_THREADS) {
    float s[LC_K] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int p = 0; p < D3; ++p) {
      const float a = o.At[(size_t)p * D3 + q];
      const float4 u0 = *reinterpret_cast<const float4*>(Psi + p * LC_K), u1 = *reinterpret_cast<const float4*>(Psi + p * LC_K + 4);
      s[0] += a * u0.x, s[1] += a * u0.y, s[2] += a * u0.z, s[3] += a * u0.w;
      s[4] += a * u1.x, s[5] += a * u1.y, s[6] += a * u1.z, s[7] += a * u1.w;
    }
    for (int k = 0; k < LC_K; ++k) AP[q * LC_K + k] = s[k];
  }
  __syncthreads();
  for (int e = warp; e < LC_K * LC_K; e += TR_OP_THREADS / 32) {
    const int r = e / LC_K, c = e % LC_K;
    double s = 0.0;
    for (int q = lane; q < D3; q += 32) s += (double)Psi[q * LC_K + r] * AP[q * LC_K + c];
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) s += __shfl_down_sync(0xffffffffu, s, w);
    if (lane == 0) Gs[e] = s;
  }
  __syncthreads();
  if (tid == 0) {  // symmetrise, ridge, Cholesky (lower, in place)
    double G[LC_K * LC_K], tr = 0.0;
    for (int r = 0; r < LC_K; ++r)
      for (int c = 0; c < LC_K; ++c) G[r * LC_K + c] = 0.5 * (Gs[r * LC_K + c] + Gs[c * LC_K + r]);
    for (int r = 0; r < LC_K; ++r) tr += G[r * LC_K + r];
    for (int r = 0; r < LC_K; ++r) G[r * LC_K + r] += TR_RIDGE * tr / LC_K;
    bool ok = tr > 0.0 && isfinite(tr);
    for (int j = 0; j < LC_K && ok; ++j) {
      double d = G[j * LC_K + j];
      for (int q = 0; q < j; ++q) d -= G[j * LC_K + q] * G[j * LC_K + q];
      if (!(d > 0.0)) {
        ok = false;
        break;
      }
      d = sqrt(d);
      G[j * LC_K + j] = d;
      for (int i = j + 1; i < LC_K; ++i) {
        double v = G[i * LC_K + j];
        for (int q = 0; q < j; ++q) v -= G[i * LC_K + q] * G[j * LC_K + q];
        G[i * LC_K + j] = v / d;
      }
    }
    for (int q = 0; q < LC_K * LC_K; ++q) Gs[q] = G[q];
    gok = ok ? 1 : 0;
  }
  __syncthreads();
  double loss = 0.0;
  if (!gok) {
    if (tid == 0) lossOut[b] = nan("");
    return;
  }
  for (int call = 0; call < o.calls; ++call) {
    const float* r = o.R + (size_t)call * D3;
    // u = Psi^T r (FP64)
    double u[LC_K] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int q = tid; q < D3; q += TR_OP_THREADS) {
      const double rv = r[q];
      for (int k = 0; k < LC_K; ++k) u[k] += (double)Psi[q * LC_K + k] * rv;
    }
#pragma unroll
    for (int k = 0; k < LC_K; ++k) {
      double s = u[k];
#pragma unroll
      for (int w = 16; w > 0; w >>= 1) s += __shfl_down_sync(0xffffffffu, s, w);
      if (lane == 0) red[warp][k] = s;
    }
    __syncthreads();
    if (tid == 0) {
      double uu[LC_K], c[LC_K];
      for (int k = 0; k < LC_K; ++k) {
        double s = 0.0;
        for (int w = 0; w < TR_OP_THREADS / 32; ++w) s += red[w][k];
        uu[k] = s;
      }
      for (int i = 0; i < LC_K; ++i) {
        double v = uu[i];
        for (int q = 0; q < i; ++q) v -= Gs[i * LC_K + q] * c[q];
        c[i] = v / Gs[i * LC_K + i];
      }
      for (int i = LC_K - 1; i >= 0; --i) {
        double v = c[i];
        for (int q = i + 1; q < LC_K; ++q) v -= Gs[q * LC_K + i] * c[q];
        c[i] = v / Gs[i * LC_K + i];
      }
      double qv = 0.0;
      for (int k = 0; k < LC_K; ++k) qv += uu[k] * c[k], cc[k] = c[k];
      loss += 1.0 - qv / o.E[call];
    }
    __syncthreads();
    const float invE = (float)(1.0 / o.E[call]);
    float ck[LC_K];
    for (int k = 0; k < LC_K; ++k) ck[k] = (float)cc[k];
    for (int q = tid; q < D3; q += TR_OP_THREADS) {
      float w = r[q];
      for (int k = 0; k < LC_K; ++k) w -= AP[q * LC_K + k] * ck[k];
      w *= invE;
      for (int k = 0; k < LC_K; ++k) dPsi[q * LC_K + k] += w * ck[k];
    }
    __syncthreads();  // red and cc are reused by the next call
  }
  const float sc = (float)(-2.0 * scale);
  for (int q = tid; q < D3 * LC_K; q += TR_OP_THREADS) {
    const int row = q / LC_K, k = q % LC_K;
    dOut[(size_t)(r0 + row / 3) * LC_OUT + 3 * k + row % 3] = sc * dPsi[q];
  }
  if (tid == 0) lossOut[b] = loss;
}

// ------------------------------------------------------------------------------------------- backward

// Fragment helpers over FP32 tiles in shared memory (row-major, stride ld), converted to BF16.
// A fragment (16 x 16) of the matrix element (m, k) = T[m][k] at (m0, k0).
__device__ __forceinline__ void fragA(const float* T, int ld, int m0, int k0, int lane, uint32_t (&a)[4]) {
  const int g = lane >> 2, t = lane & 3;
  const float* r0 = T + (m0 + g) * ld + k0 + 2 * t;
  const float* r1 = T + (m0 + g + 8) * ld + k0 + 2 * t;
  a[0] = packBf16(r0[0], r0[1]);
  a[1] = packBf16(r1[0], r1[1]);
  a[2] = packBf16(r0[8], r0[9]);
  a[3] = packBf16(r1[8], r1[9]);
}
// A fragment of the transpose: element (m, k) = T[k][m].
__device__ __forceinline__ void fragAT(const float* T, int ld, int m0, int k0, int lane, uint32_t (&a)[4]) {
  const int g = lane >> 2, t = lane & 3;
  auto e = [&](int m, int k) { return T[(k0 + k) * ld + m0 + m]; };
  a[0] = packBf16(e(g, 2 * t), e(g, 2 * t + 1));
  a[1] = packBf16(e(g + 8, 2 * t), e(g + 8, 2 * t + 1));
  a[2] = packBf16(e(g, 2 * t + 8), e(g, 2 * t + 9));
  a[3] = packBf16(e(g + 8, 2 * t + 8), e(g + 8, 2 * t + 9));
}
// B fragment (16 x 8), element (k, n) = T[k][n] at (k0, n0).
__device__ __forceinline__ uint2 fragBs(const float* T, int ld, int k0, int n0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  auto e = [&](int k) { return T[(k0 + k) * ld + n0 + g]; };
  return make_uint2(packBf16(e(2 * t), e(2 * t + 1)), packBf16(e(2 * t + 8), e(2 * t + 9)));
}
// Writes a 16 x 8 accumulator tile into T (row-major, stride ld) at (m0, n0).
__device__ __forceinline__ void storeAcc(float* T, int ld, int m0, int n0, const float (&c)[4], int lane) {
  const int g = lane >> 2, t = lane & 3;
  T[(m0 + g) * ld + n0 + 2 * t] = c[0];
  T[(m0 + g) * ld + n0 + 2 * t + 1] = c[1];
  T[(m0 + g + 8) * ld + n0 + 2 * t] = c[2];
  T[(m0 + g + 8) * ld + n0 + 2 * t + 1] = c[3];
}

constexpr int TR_LD = 68;  // FP32 tile row stride (64 + 4 against bank conflicts)

struct BackSmem {
  __nv_bfloat16 X[4][16 * LC_XSTRIDE];
  float Xf[TR_ROWS * 36];          // inputs as FP32, stride 36 (20 used, 32 read by fragments)
  float h1[TR_ROWS * TR_LD];
  float h2[TR_ROWS * TR_LD];
  float g2[TR_ROWS * TR_LD];       // dL/d(pre-activation of layer 2)
  float g1[TR_ROWS * TR_LD];       // dL/d(pre-activation of layer 1)
  float dO[TR_ROWS * 36];          // dL/d(output), stride 36 (24 used, 32 read)
};

// Recomputes the forward pass of the CTA's 64 rows and back-propagates dOut: weight and bias gradients
// of these rows into partial[blockIdx.x][LC_WEIGHTS] (the flat layout).
__global__ void __launch_bounds__(128) k_tr_backward(const TrOp* __restrict__ ops, const int* __restrict__ batch,
                                                     const int* __restrict__ rowStart, int nb, const MlpPacked* __restrict__ P,
                                                     const MlpPackedT* __restrict__ PT, const float* __restrict__ dOut,
                                                     float* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char trBack[];
  BackSmem& S = *reinterpret_cast<BackSmem*>(trBack);
  __shared__ __align__(16) MlpPacked net;
  for (int q = threadIdx.x; q < (int)(sizeof(MlpPacked) / 16); q += blockDim.x)
    reinterpret_cast<float4*>(&net)[q] = reinterpret_cast<const float4*>(P)[q];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, rows = rowStart[nb];
  const int base = blockIdx.x * TR_ROWS, row0 = base + 16 * warp, m0 = 16 * warp;
  const int g = lane >> 2, t = lane & 3;
  __syncthreads();
  // forward of this warp's 16 rows (rows past the minibatch: zero inputs and zero output gradients)
  loadInputTile(ops, batch, rowStart, nb, rows, row0, S.X[warp], lane);
  for (int q = lane; q < 16 * 36; q += 32) {
    const int r = q / 36, c = q % 36;
    S.Xf[(m0 + r) * 36 + c] = c < LC_IN_PAD ? __bfloat162float(S.X[warp][r * LC_XSTRIDE + c]) : 0.f;
    S.dO[(m0 + r) * 36 + c] = (c < LC_OUT && row0 + r < rows) ? dOut[(size_t)(row0 + r) * LC_OUT + c] : 0.f;
  }
  __syncwarp();
  // the hidden activations (the forward pass's fragments and rounding), stored per row
  {
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const float b0 = net.bias[8 * nt + 2 * t], b1 = net.bias[8 * nt + 2 * t + 1];
      acc[nt][0] = b0, acc[nt][1] = b1, acc[nt][2] = b0, acc[nt][3] = b1;
    }
#pragma unroll
    for (int kc = 0; kc < 2; ++kc) {
      uint32_t a[4];
      fragAFromSmem(S.X[warp], kc, lane, a);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) mma16816(acc[nt], a, net.frag[LC_F1 + (kc * 8 + nt) * 32 + lane]);
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[nt][q] = bf16Round(tanhf(acc[nt][q]));
      storeAcc(S.h1, TR_LD, m0, 8 * nt, acc[nt], lane);
    }
    uint32_t ah[4][4];
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) fragAFromAcc(acc[2 * kc], acc[2 * kc + 1], ah[kc]);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const float b0 = net.bias[LC_HID + 8 * nt + 2 * t], b1 = net.bias[LC_HID + 8 * nt + 2 * t + 1];
      acc[nt][0] = b0, acc[nt][1] = b1, acc[nt][2] = b0, acc[nt][3] = b1;
    }
#pragma unroll
    for (int kc = 0; kc < 4; ++kc)
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) mma16816(acc[nt], ah[kc], net.frag[LC_F2 + (kc * 8 + nt) * 32 + lane]);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[nt][q] = bf16Round(tanhf(acc[nt][q]));
      storeAcc(S.h2, TR_LD, m0, 8 * nt, acc[nt], lane);
    }
  }
  __syncwarp();
  // g2 = (dO W3^T) * (1 - h2^2)
  {
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int kc = 0; kc < 2; ++kc) {
      uint32_t a[4];
      fragA(S.dO, 36, m0, 16 * kc, lane, a);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) mma16816(acc[nt], a, PT->frag[LC_T3 + (kc * 8 + nt) * 32 + lane]);
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = 8 * nt + 2 * t;
      const float* h = S.h2;
      acc[nt][0] *= 1.f - h[(m0 + g) * TR_LD + c] * h[(m0 + g) * TR_LD + c];
      acc[nt][1] *= 1.f - h[(m0 + g) * TR_LD + c + 1] * h[(m0 + g) * TR_LD + c + 1];
      acc[nt][2] *= 1.f - h[(m0 + g + 8) * TR_LD + c] * h[(m0 + g + 8) * TR_LD + c];
      acc[nt][3] *= 1.f - h[(m0 + g + 8) * TR_LD + c + 1] * h[(m0 + g + 8) * TR_LD + c + 1];
      storeAcc(S.g2, TR_LD, m0, 8 * nt, acc[nt], lane);
    }
  }
  __syncwarp();
  // g1 = (g2 W2^T) * (1 - h1^2)
  {
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      uint32_t a[4];
      fragA(S.g2, TR_LD, m0, 16 * kc, lane, a);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) mma16816(acc[nt], a, PT->frag[LC_T2 + (kc * 8 + nt) * 32 + lane]);
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = 8 * nt + 2 * t;
      const float* h = S.h1;
      acc[nt][0] *= 1.f - h[(m0 + g) * TR_LD + c] * h[(m0 + g) * TR_LD + c];
      acc[nt][1] *= 1.f - h[(m0 + g) * TR_LD + c + 1] * h[(m0 + g) * TR_LD + c + 1];
      acc[nt][2] *= 1.f - h[(m0 + g + 8) * TR_LD + c] * h[(m0 + g + 8) * TR_LD + c];
      acc[nt][3] *= 1.f - h[(m0 + g + 8) * TR_LD + c + 1] * h[(m0 + g + 8) * TR_LD + c + 1];
      storeAcc(S.g1, TR_LD, m0, 8 * nt, acc[nt], lane);
    }
  }
  __syncthreads();
  float* part = partial + (size_t)blockIdx.x * LC_WEIGHTS;
  // weight gradients over the CTA's 64 rows (K = rows): warp w takes output rows 16 w .. of each
  // dW3[h][o] = sum_r h2[r][h] dO[r][o]   (M = 64 hidden, N = 24 outputs)
  {
    float acc[3][4];
#pragma unroll
    for (int nt = 0; nt < 3; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      uint32_t a[4];
      fragAT(S.h2, TR_LD, m0, 16 * kc, lane, a);
#pragma unroll
      for (int nt = 0; nt < 3; ++nt) mma16816(acc[nt], a, fragBs(S.dO, 36, 16 * kc, 8 * nt, lane));
    }
#pragma unroll
    for (int nt = 0; nt < 3; ++nt) {
      const int c = 8 * nt + 2 * t;
      part[LC_W3 + (m0 + g) * LC_OUT + c] = acc[nt][0];
      part[LC_W3 + (m0 + g) * LC_OUT + c + 1] = acc[nt][1];
      part[LC_W3 + (m0 + g + 8) * LC_OUT + c] = acc[nt][2];
      part[LC_W3 + (m0 + g + 8) * LC_OUT + c + 1] = acc[nt][3];
    }
  }
  // dW2[i][j] = sum_r h1[r][i] g2[r][j]   (M = 64, N = 64)
  {
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      uint32_t a[4];
      fragAT(S.h1, TR_LD, m0, 16 * kc, lane, a);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) mma16816(acc[nt], a, fragBs(S.g2, TR_LD, 16 * kc, 8 * nt, lane));
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = 8 * nt + 2 * t;
      part[LC_W2 + (m0 + g) * LC_HID + c] = acc[nt][0];
      part[LC_W2 + (m0 + g) * LC_HID + c + 1] = acc[nt][1];
      part[LC_W2 + (m0 + g + 8) * LC_HID + c] = acc[nt][2];
      part[LC_W2 + (m0 + g + 8) * LC_HID + c + 1] = acc[nt][3];
    }
  }
  // dW1[f][i] = sum_r X[r][f] g1[r][i]   (M = 32 padded inputs, N = 64): warps 0, 1 take m-tiles,
  // warps 2, 3 the bias gradients
  if (warp < 2) {
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      uint32_t a[4];
      fragAT(S.Xf, 36, 16 * warp, 16 * kc, lane, a);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) mma16816(acc[nt], a, fragBs(S.g1, TR_LD, 16 * kc, 8 * nt, lane));
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = 8 * nt + 2 * t, f0 = 16 * warp + g, f1 = f0 + 8;
      if (f0 < LC_IN) part[LC_W1 + f0 * LC_HID + c] = acc[nt][0], part[LC_W1 + f0 * LC_HID + c + 1] = acc[nt][1];
      if (f1 < LC_IN) part[LC_W1 + f1 * LC_HID + c] = acc[nt][2], part[LC_W1 + f1 * LC_HID + c + 1] = acc[nt][3];
    }
  } else {
    for (int c = threadIdx.x - 64; c < LC_BIAS; c += 64) {
      const float* src = c < LC_HID ? S.g1 + c : c < 2 * LC_HID ? S.g2 + (c - LC_HID) : S.dO + (c - 2 * LC_HID);
      const int ld = c < 2 * LC_HID ? TR_LD : 36;
      float s = 0.f;
      for (int r = 0; r < TR_ROWS; ++r) s += src[r * ld];
      const int dst = c < LC_HID ? LC_B1 + c : c < 2 * LC_HID ? LC_B2 + (c - LC_HID) : LC_B3 + (c - 2 * LC_HID);
      part[dst] = s;
    }
  }
}

// Sums the CTAs' partial gradients in order; optionally writes the gradient, applies an Adam step
// to the FP32 master weights and repacks the BF16 fragments. One CTA.
struct AdamArgs {
  float* w;       // master weights (LC_WEIGHTS)
  float* m;
  float* v;
  float* grad;    // optional gradient output
  MlpPacked* P;
  MlpPackedT* PT;
  const float* partial;
  int parts;
  int adam;       // apply the step
  int t;          // step number (1-based)
  float lr;
  const double* lossParts;
  int nb;
  double invCalls;
  float* lossHist;  // per step (or null)
};

__global__ void __launch_bounds__(1024) k_tr_adam(AdamArgs a) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int q = threadIdx.x; q < LC_WEIGHTS; q += blockDim.x) {
    float g = 0.f;
    for (int p = 0; p < a.parts; ++p) g += a.partial[(size_t)p * LC_WEIGHTS + q];
    if (a.grad) a.grad[q] = g;
    if (a.adam) {
      const float m = b1 * a.m[q] + (1.f - b1) * g, v = b2 * a.v[q] + (1.f - b2) * g * g;
      a.m[q] = m, a.v[q] = v;
      const float mh = m / (1.f - powf(b1, (float)a.t)), vh = v / (1.f - powf(b2, (float)a.t));
      a.w[q] -= a.lr * mh / (sqrtf(vh) + eps);
    }
  }
  if (threadIdx.x == 0 && a.lossHist) {
    double l = 0.0;
    for (int b = 0; b < a.nb; ++b) l += a.lossParts[b];
    a.lossHist[a.t - 1] = (float)(l * a.invCalls);
  }
  __syncthreads();
  if (a.adam) {
    mlpPack(a.w, a.P, threadIdx.x, blockDim.x);
    mlpPackT(a.w, a.PT, threadIdx.x, blockDim.x);
  }
}

__global__ void k_tr_pack(const float* w, MlpPacked* P, MlpPackedT* PT) {
  mlpPack(w, P, threadIdx.x, blockDim.x);
  mlpPackT(w, PT, threadIdx.x, blockDim.x);
}

// ------------------------------------------------------------------------------------------ ingestion

// Per logged operator: the diagonal blocks' Cholesky factors, which free nodes have a positive definite
// block (all must), and the free nodes' dense index. One CTA per operator.
__global__ void k_tr_scan(const float4* __restrict__ rows, const uint32_t* __restrict__ fixed, int M, int* __restrict__ freeIdx,
                          int* __restrict__ info /* [op][2]: free count, all ok */) {
  const int op = blockIdx.x;
  const float4* R = rows + (size_t)op * COARSE_PLANES * M;
  const uint32_t* F = fixed + (size_t)op * M;
  int* idx = freeIdx + (size_t)op * M;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int n = threadIdx.x; n < M; n += blockDim.x) {
    double L[6];
    if (!F[n] && !chol3d(coarseBlock(R, M, n, 12), L)) atomicOr(&bad, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int c = 0;
    for (int n = 0; n < M; ++n) idx[n] = F[n] ? -1 : c++;
    info[2 * op] = c;
    info[2 * op + 1] = bad ? 0 : 1;
  }
}

// Whitened dense operator At = L^-1 A L^-T over the free unknowns of one layer nx x ny: FP64 (for the
// factorisation) and FP32 (for training). One CTA per operator row block: thread per (node n, offset).
__global__ void k_tr_whiten(const float4* __restrict__ rows, int M, int nx, const int* __restrict__ freeIdx, int D3,
                            double* __restrict__ Ad, float* __restrict__ Af) {
  const int n = blockIdx.x;
  const int a = freeIdx[n];
  if (a < 0) return;
  const int i = n % nx, j = n / nx, ny = M / nx;
  double Ln[6], Lm[6];
  chol3d(coarseBlock(rows, M, n, 12), Ln);
  for (int o = threadIdx.x; o < 25; o += blockDim.x) {
    const int di = o % 5 - 2, dj = o / 5 - 2, ii = i + di, jj = j + dj;
    if (ii < 0 || jj < 0 || ii >= nx || jj >= ny) continue;
    const int m = jj * nx + ii, b = freeIdx[m];
    if (b < 0) continue;
    chol3d(coarseBlock(rows, M, m, 12), Lm);
    const Sym s = coarseBlock(rows, M, n, o);
    const double B[9] = {s.xx, s.xy, s.xz, s.xy, s.yy, s.yz, s.xz, s.yz, s.zz};
    // T = Ln^-1 B (column by column), W = T Lm^-T (row by row)
    double T[9], W[9];
    for (int c = 0; c < 3; ++c) {
      T[c] = B[c] / Ln[0];
      T[3 + c] = (B[3 + c] - Ln[1] * T[c]) / Ln[2];
      T[6 + c] = (B[6 + c] - Ln[3] * T[c] - Ln[4] * T[3 + c]) / Ln[5];
    }
    for (int r = 0; r < 3; ++r) {
      W[3 * r] = T[3 * r] / Lm[0];
      W[3 * r + 1] = (T[3 * r + 1] - Lm[1] * W[3 * r]) / Lm[2];
      W[3 * r + 2] = (T[3 * r + 2] - Lm[3] * W[3 * r] - Lm[4] * W[3 * r + 1]) / Lm[5];
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        const size_t q = (size_t)(3 * a + r) * D3 + 3 * b + c;
        Ad[q] = W[3 * r + c];
        Af[q] = (float)W[3 * r + c];
      }
  }
}

// In-place lower Cholesky factor of a dense SPD matrix (FP64, row-major D x D), one CTA; ok = 0 on a
// non-positive pivot. Right-looking: for each column, scale it, then update the trailing lower triangle.
__global__ void __launch_bounds__(1024) k_tr_cholesky(double* __restrict__ A, int D, int* __restrict__ ok) {
  __shared__ double piv;
  __shared__ int good;
  if (threadIdx.x == 0) good = 1;
  __syncthreads();
  for (int j = 0; j < D; ++j) {
    if (threadIdx.x == 0) {
      const double d = A[(size_t)j * D + j];
      if (!(d > 0.0) || !isfinite(d)) good = 0;
      piv = good ? sqrt(d) : 1.0;
      A[(size_t)j * D + j] = piv;
    }
    __syncthreads();
    if (!good) break;
    for (int i = j + 1 + threadIdx.x; i < D; i += blockDim.x) A[(size_t)i * D + j] /= piv;
    __syncthreads();
    // trailing update A[i][k] -= A[i][j] A[k][j] for j < k <= i: a thread per column k, rows in
    // order, so a warp's lanes touch consecutive columns of one row
    for (int k = j + 1 + threadIdx.x; k < D; k += blockDim.x) {
      const double akj = A[(size_t)k * D + j];
      for (int i = k; i < D; ++i) A[(size_t)i * D + k] -= A[(size_t)i * D + j] * akj;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *ok = good;
}

// The free nodes' network inputs of one logged operator, in dense order.
__global__ void k_tr_gather_x(const float* __restrict__ X, const int* __restrict__ freeIdx, int M, float* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < M * LC_IN; q += gridDim.x * blockDim.x) {
    const int n = q / LC_IN, a = freeIdx[n];
    if (a >= 0) out[(size_t)a * LC_IN + q % LC_IN] = X[q];
  }
}

// Per logged call (one CTA each): whitened residual r_w = L^-1 r over the free nodes, exact correction
// d = At^-1 r_w by forward and back substitution with the dense factor (FP64), E = r_w . d.
__global__ void __launch_bounds__(256) k_tr_solve(const float* __restrict__ Rraw, const int* __restrict__ callOp,
                                                  const int* __restrict__ opSlot, const float4* __restrict__ rows, int M,
                                                  const int* __restrict__ freeIdx, const int* __restrict__ opD3,
                                                  double* const* __restrict__ factors, double* __restrict__ work, float* const* __restrict__ Rout,
                                                  float* const* __restrict__ Dout, double* const* __restrict__ Eout,
                                                  const int* __restrict__ callSlot) {
  const int call = blockIdx.x;
  const int op = callOp[call], slot = opSlot[op];
  if (slot < 0 || callSlot[call] < 0) return;
  const int D3 = opD3[op];
  const double* Lf = factors[slot];
  const int* idx = freeIdx + (size_t)op * M;
  const float4* R = rows + (size_t)op * COARSE_PLANES * M;
  double* y = work + (size_t)call * 3 * M;
  const float* rr = Rraw + (size_t)call * 3 * M;
  for (int n = threadIdx.x; n < M; n += blockDim.x) {
    const int a = idx[n];
    if (a < 0) continue;
    double L[6];
    chol3d(coarseBlock(R, M, n, 12), L);
    const double g0 = rr[3 * n] / L[0];
    const double g1 = (rr[3 * n + 1] - L[1] * g0) / L[2];
    const double g2 = (rr[3 * n + 2] - L[3] * g0 - L[4] * g1) / L[5];
    y[3 * a] = g0, y[3 * a + 1] = g1, y[3 * a + 2] = g2;
  }
  __syncthreads();
  float* ro = Rout[slot] + (size_t)callSlot[call] * D3;
  for (int q = threadIdx.x; q < D3; q += blockDim.x) ro[q] = (float)y[q];
  __syncthreads();
  __shared__ double yj;
  // forward: L z = y (column-oriented)
  for (int j = 0; j < D3; ++j) {
    if (threadIdx.x == 0) {
      y[j] /= Lf[(size_t)j * D3 + j];
      yj = y[j];
    }
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < D3; i += blockDim.x) y[i] -= Lf[(size_t)i * D3 + j] * yj;
    __syncthreads();
  }
  // back: L^T d = z (row j of L^T is column j of L)
  for (int j = D3 - 1; j >= 0; --j) {
    if (threadIdx.x == 0) {
      y[j] /= Lf[(size_t)j * D3 + j];
      yj = y[j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < j; i += blockDim.x) y[i] -= Lf[(size_t)j * D3 + i] * yj;
    __syncthreads();
  }
  float* dout = Dout[slot] + (size_t)callSlot[call] * D3;
  __shared__ double part[8];
  double e = 0.0;
  for (int q = threadIdx.x; q < D3; q += blockDim.x) {
    dout[q] = (float)y[q];
    e += (double)ro[q] * y[q];
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w];
    Eout[slot][callSlot[call]] = s;
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------- the trainer

struct btd_trainer {
  cudaStream_t stream = nullptr;
  struct Op {
    int n = 0, D3 = 0, calls = 0;
    float *At = nullptr, *X = nullptr, *R = nullptr, *D = nullptr;
    double* E = nullptr;
    int group = 0;
  };
  std::vector<Op> ops;
  std::vector<void*> allocs;
  TrOp* dOps = nullptr;
  size_t dOpsCap = 0;
  // network state
  float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
  MlpPacked* P = nullptr;
  MlpPackedT* PT = nullptr;
  // per-step scratch
  float *out = nullptr, *dOut = nullptr, *partial = nullptr;
  size_t rowsCap = 0, partsCap = 0;
  double* lossParts = nullptr;
  int* dBatch = nullptr;   // per step: batch op indices then row starts
  size_t batchCap = 0;
  float* lossHist = nullptr;
  size_t histCap = 0;

  template <class T>
  T* alloc(size_t count) {
    void* p = nullptr;
    TK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    allocs.push_back(p);
    return static_cast<T*>(p);
  }
  void release(void* p) {
    if (!p) return;
    allocs.erase(std::remove(allocs.begin(), allocs.end(), p), allocs.end());
    cudaFree(p);
  }
  ~btd_trainer() {
    if (stream) cudaStreamSynchronize(stream);
    for (void* p : allocs) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
  void sync() { TK(cudaStreamSynchronize(stream)); }

  void uploadOps() {
    std::vector<TrOp> h(ops.size());
    for (size_t k = 0; k < ops.size(); ++k) h[k] = TrOp{ops[k].At, ops[k].X, ops[k].R, ops[k].D, ops[k].E, ops[k].n, ops[k].D3, ops[k].calls, 0};
    if (ops.size() > dOpsCap) {
      release(dOps);
      dOpsCap = std::max<size_t>(2 * ops.size(), 16);
      dOps = alloc<TrOp>(dOpsCap);
    }
    TK(cudaMemcpyAsync(dOps, h.data(), sizeof(TrOp) * h.size(), cudaMemcpyHostToDevice, stream));
    sync();
  }

  void ensureNet() {
    if (w) return;
    w = alloc<float>(LC_WEIGHTS);
    m = alloc<float>(LC_WEIGHTS);
    v = alloc<float>(LC_WEIGHTS);
    grad = alloc<float>(LC_WEIGHTS);
    P = alloc<MlpPacked>(1);
    PT = alloc<MlpPackedT>(1);
    lossParts = alloc<double>(TR_MAX_BATCH);
    static bool attr = false;
    if (!attr) {
      int dev = 0, optin = 0;
      TK(cudaGetDevice(&dev));
      TK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
      cudaFuncAttributes fa;
      TK(cudaFuncGetAttributes(&fa, (const void*)k_tr_operator));
      TK(cudaFuncSetAttribute((const void*)k_tr_operator, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
      TK(cudaFuncGetAttributes(&fa, (const void*)k_tr_backward));
      TK(cudaFuncSetAttribute((const void*)k_tr_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
      attr = true;
    }
  }

  // Scratch for minibatches of at most `rows` network rows.
  void ensureRows(size_t rows) {
    const size_t parts = (rows + TR_ROWS - 1) / TR_ROWS;
    if (rows > rowsCap) {
      release(out);
      release(dOut);
      rowsCap = std::max(rows, rowsCap * 2);
      out = alloc<float>(rowsCap * LC_OUT);
      dOut = alloc<float>(rowsCap * LC_OUT);
    }
    if (parts > partsCap) {
      release(partial);
      partsCap = std::max(parts, partsCap * 2);
      partial = alloc<float>(partsCap * LC_WEIGHTS);
    }
  }

  // One forward/backward over the minibatch `batch` (op indices) whose int block (batch, row starts)
  // sits at dBatchStep; returns the CTA count of the backward pass.
  int launchStep(const std::vector<int>& batch, const int* dB, int rows, double invCalls) {
    const int nb = (int)batch.size();
    const int* dRow = dB + TR_MAX_BATCH;
    const int parts = (rows + TR_ROWS - 1) / TR_ROWS;
    k_tr_forward<<<parts, 128, 0, stream>>>(dOps, dB, dRow, nb, P, out);
    int maxD3 = 0;
    for (int b : batch) maxD3 = std::max(maxD3, ops[b].D3);
    k_tr_operator<<<nb, TR_OP_THREADS, trOpSmem(maxD3), stream>>>(dOps, dB, dRow, out, dOut, lossParts, invCalls);
    k_tr_backward<<<parts, 128, sizeof(BackSmem), stream>>>(dOps, dB, dRow, nb, P, PT, dOut, partial);
    TK(cudaGetLastError());
    return parts;
  }
};

namespace {

int trFail(const std::exception& e) {
  btd::setError(e.what());
  if (dynamic_cast<const TrError*>(&e)) return BTD_E_CUDA;
  return BTD_E_INVALID;
}
#define TGUARD(...)                    \
  try {                                \
    __VA_ARGS__;                       \
    return BTD_OK;                     \
  } catch (const std::exception& e) {  \
    return trFail(e);                  \
  }

void checkTrainer(btd_trainer* t) {
  if (!t) throw std::invalid_argument("null trainer");
}

}  // namespace

extern "C" int btd_trainer_create(btd_trainer** out) {
  if (!out) {
    btd::setError("btd_trainer_create: null output");
    return BTD_E_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    btd::setError("btd_trainer_create: no CUDA device (training has no CPU fallback)");
    return BTD_E_NO_DEVICE;
  }
  std::unique_ptr<btd_trainer> t(new btd_trainer());
  TGUARD({
    TK(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking));
    t->ensureNet();
    *out = t.release();
  });
}

extern "C" int btd_trainer_destroy(btd_trainer* t) {
  delete t;
  return BTD_OK;
}

extern "C" int btd_trainer_add_op(btd_trainer* t, int32_t nodes, const double* At, const double* X, int32_t calls, const double* R,
                                  const double* D, int32_t group) {
  TGUARD({
    checkTrainer(t);
    if (nodes < 1 || nodes > TR_MAX_NODES) throw std::invalid_argument("btd_trainer_add_op: 1.." + std::to_string(TR_MAX_NODES) + " nodes");
    if (calls < 0 || !At || !X || (calls > 0 && (!R || !D))) throw std::invalid_argument("btd_trainer_add_op: null material");
    btd_trainer::Op o;
    o.n = nodes;
    o.D3 = 3 * nodes;
    o.calls = calls;
    o.group = group;
    const size_t D3 = o.D3;
    std::vector<float> at(D3 * D3), x((size_t)nodes * LC_IN), r(std::max<size_t>(1, (size_t)calls * D3)), d(r.size());
    std::vector<double> e(std::max(1, (int)calls));
    for (size_t q = 0; q < at.size(); ++q) at[q] = (float)At[q];
    for (size_t q = 0; q < x.size(); ++q) x[q] = (float)X[q];
    for (int c = 0; c < calls; ++c) {
      double s = 0.0;
      for (size_t q = 0; q < D3; ++q) {
        r[c * D3 + q] = (float)R[c * D3 + q];
        d[c * D3 + q] = (float)D[c * D3 + q];
        s += R[c * D3 + q] * D[c * D3 + q];
      }
      e[c] = s;
    }
    o.At = t->alloc<float>(at.size());
    o.X = t->alloc<float>(x.size());
    o.R = t->alloc<float>(r.size());
    o.D = t->alloc<float>(d.size());
    o.E = t->alloc<double>(e.size());
    TK(cudaMemcpyAsync(o.At, at.data(), sizeof(float) * at.size(), cudaMemcpyHostToDevice, t->stream));
    TK(cudaMemcpyAsync(o.X, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice, t->stream));
    TK(cudaMemcpyAsync(o.R, r.data(), sizeof(float) * r.size(), cudaMemcpyHostToDevice, t->stream));
    TK(cudaMemcpyAsync(o.D, d.data(), sizeof(float) * d.size(), cudaMemcpyHostToDevice, t->stream));
    TK(cudaMemcpyAsync(o.E, e.data(), sizeof(double) * e.size(), cudaMemcpyHostToDevice, t->stream));
    t->ops.push_back(o);
    t->uploadOps();
  });
}

// The solver's log (btd_learned_log) as training material. Declared in solver.cu.
namespace btd {
struct LearnedLogView {
  const float4* rows;
  const uint32_t* fixed;
  const float* X;
  const float* R;
  const int* opOf;
  int M, nx, ny, ops, calls;
  cudaStream_t stream;
};
int learnedLogView(btd_solver* s, LearnedLogView* v);
}  // namespace btd

extern "C" int btd_trainer_add_log(btd_trainer* t, btd_solver* s, int32_t group, int32_t* ops_added) {
  TGUARD({
    checkTrainer(t);
    LearnedLogView lv;
    if (btd::learnedLogView(s, &lv) != 0) throw std::invalid_argument("btd_trainer_add_log: the solver has no learned log");
    TK(cudaStreamSynchronize(lv.stream));
    const int M = lv.M, nOps = lv.ops, nCalls = lv.calls;
    if (ops_added) *ops_added = 0;
    if (nOps == 0) return BTD_OK;
    // 1. free nodes and positive definite blocks per operator
    int* freeIdx = t->alloc<int>((size_t)nOps * M);
    int* info = t->alloc<int>(2 * nOps);
    k_tr_scan<<<nOps, 256, 0, t->stream>>>(lv.rows, lv.fixed, M, freeIdx, info);
    std::vector<int> hinfo(2 * nOps);
    TK(cudaMemcpyAsync(hinfo.data(), info, sizeof(int) * 2 * nOps, cudaMemcpyDeviceToHost, t->stream));
    std::vector<int> hfree((size_t)nOps * M);
    TK(cudaMemcpyAsync(hfree.data(), freeIdx, sizeof(int) * hfree.size(), cudaMemcpyDeviceToHost, t->stream));
    std::vector<int> hop(nCalls);
    if (nCalls) TK(cudaMemcpyAsync(hop.data(), lv.opOf, sizeof(int) * nCalls, cudaMemcpyDeviceToHost, t->stream));
    t->sync();
    // 2. whitened dense operators and their factors (FP64), one slot per usable operator
    std::vector<int> slot(nOps, -1), d3(nOps, 0);
    std::vector<double*> fac;
    std::vector<int> facOp;
    for (int op = 0; op < nOps; ++op) {
      d3[op] = 3 * hinfo[2 * op];
      if (!hinfo[2 * op + 1] || d3[op] == 0) continue;
      slot[op] = (int)fac.size();
      fac.push_back(t->alloc<double>((size_t)d3[op] * d3[op]));
      facOp.push_back(op);
    }
    std::vector<btd_trainer::Op> added(fac.size());
    std::vector<int> okFac(fac.size(), 0);
    int* dOk = t->alloc<int>(std::max<size_t>(1, fac.size()));
    for (size_t k = 0; k < fac.size(); ++k) {
      const int op = facOp[k], D3 = d3[op];
      btd_trainer::Op& o = added[k];
      o.n = D3 / 3;
      o.D3 = D3;
      o.group = group;
      o.At = t->alloc<float>((size_t)D3 * D3);
      TK(cudaMemsetAsync(fac[k], 0, sizeof(double) * D3 * D3, t->stream));
      TK(cudaMemsetAsync(o.At, 0, sizeof(float) * D3 * D3, t->stream));
      k_tr_whiten<<<M, 32, 0, t->stream>>>(lv.rows + (size_t)op * COARSE_PLANES * M, M, lv.nx, freeIdx + (size_t)op * M, D3, fac[k], o.At);
      k_tr_cholesky<<<1, 1024, 0, t->stream>>>(fac[k], D3, dOk + k);
      // the free nodes' inputs
      o.X = t->alloc<float>((size_t)o.n * LC_IN);
      k_tr_gather_x<<<blocksOf(M * LC_IN, 256), 256, 0, t->stream>>>(lv.X + (size_t)op * M * LC_IN, freeIdx + (size_t)op * M, M, o.X);
    }
    TK(cudaGetLastError());
    TK(cudaMemcpyAsync(okFac.data(), dOk, sizeof(int) * fac.size(), cudaMemcpyDeviceToHost, t->stream));
    t->sync();
    for (size_t k = 0; k < fac.size(); ++k)
      if (!okFac[k]) slot[facOp[k]] = -1;
    // 3. every call's whitened residual and exact correction
    std::vector<int> callSlot(nCalls, -1);
    for (int c = 0; c < nCalls; ++c) {
      const int op = hop[c];
      if (op < 0 || op >= nOps || slot[op] < 0) continue;
      callSlot[c] = added[slot[op]].calls++;
    }
    std::vector<float*> Rp(fac.size()), Dp(fac.size());
    std::vector<double*> Ep(fac.size());
    for (size_t k = 0; k < fac.size(); ++k) {
      btd_trainer::Op& o = added[k];
      o.R = t->alloc<float>((size_t)std::max(1, o.calls) * o.D3);
      o.D = t->alloc<float>((size_t)std::max(1, o.calls) * o.D3);
      o.E = t->alloc<double>(std::max(1, o.calls));
      Rp[k] = o.R, Dp[k] = o.D, Ep[k] = o.E;
    }
    if (nCalls > 0) {
      int* dCallOp = t->alloc<int>(nCalls);
      int* dSlot = t->alloc<int>(nOps);
      int* dD3 = t->alloc<int>(nOps);
      int* dCallSlot = t->alloc<int>(nCalls);
      double** dFac = t->alloc<double*>(fac.size());
      float** dR = t->alloc<float*>(fac.size());
      float** dD = t->alloc<float*>(fac.size());
      double** dE = t->alloc<double*>(fac.size());
      double* work = t->alloc<double>((size_t)nCalls * 3 * M);
      // calls of unusable operators are skipped through their slot (-1) in the kernel
      // (and calls marked -1 in callSlot)
      for (int c = 0; c < nCalls; ++c)
        if (hop[c] < 0 || hop[c] >= nOps) hop[c] = 0;
      TK(cudaMemcpyAsync(dCallOp, hop.data(), sizeof(int) * nCalls, cudaMemcpyHostToDevice, t->stream));
      TK(cudaMemcpyAsync(dSlot, slot.data(), sizeof(int) * nOps, cudaMemcpyHostToDevice, t->stream));
      TK(cudaMemcpyAsync(dD3, d3.data(), sizeof(int) * nOps, cudaMemcpyHostToDevice, t->stream));
      TK(cudaMemcpyAsync(dCallSlot, callSlot.data(), sizeof(int) * nCalls, cudaMemcpyHostToDevice, t->stream));
      if (!fac.empty()) {
        TK(cudaMemcpyAsync(dFac, fac.data(), sizeof(double*) * fac.size(), cudaMemcpyHostToDevice, t->stream));
        TK(cudaMemcpyAsync(dR, Rp.data(), sizeof(float*) * fac.size(), cudaMemcpyHostToDevice, t->stream));
        TK(cudaMemcpyAsync(dD, Dp.data(), sizeof(float*) * fac.size(), cudaMemcpyHostToDevice, t->stream));
        TK(cudaMemcpyAsync(dE, Ep.data(), sizeof(double*) * fac.size(), cudaMemcpyHostToDevice, t->stream));
        k_tr_solve<<<nCalls, 256, 0, t->stream>>>(lv.R, dCallOp, dSlot, lv.rows, M, freeIdx, dD3, dFac, work, dR, dD, dE, dCallSlot);
        TK(cudaGetLastError());
      }
      t->sync();
      for (void* p : {(void*)dCallOp, (void*)dSlot, (void*)dD3, (void*)dCallSlot, (void*)dFac, (void*)dR, (void*)dD, (void*)dE, (void*)work})
        t->release(p);
    }
    for (double* f : fac) t->release(f);
    t->release(freeIdx);
    t->release(info);
    t->release(dOk);
    int n = 0;
    for (size_t k = 0; k < fac.size(); ++k) {
      if (!okFac[k] || added[k].calls == 0) {
        for (void* p : {(void*)added[k].At, (void*)added[k].X, (void*)added[k].R, (void*)added[k].D, (void*)added[k].E}) t->release(p);
        continue;
      }
      t->ops.push_back(added[k]);
      ++n;
    }
    t->uploadOps();
    if (ops_added) *ops_added = n;
  });
}

extern "C" int btd_trainer_counts(btd_trainer* t, int32_t* ops, int32_t* calls) {
  TGUARD({
    checkTrainer(t);
    int c = 0;
    for (auto& o : t->ops) c += o.calls;
    if (ops) *ops = (int32_t)t->ops.size();
    if (calls) *calls = c;
  });
}

extern "C" int btd_trainer_read_op(btd_trainer* t, int32_t op, int32_t* nodes, int32_t* calls, float* At, float* X, float* R, float* D,
                                   double* E) {
  TGUARD({
    checkTrainer(t);
    if (op < 0 || op >= (int)t->ops.size()) throw std::invalid_argument("btd_trainer_read_op: operator out of range");
    const auto& o = t->ops[op];
    if (nodes) *nodes = o.n;
    if (calls) *calls = o.calls;
    const size_t D3 = o.D3;
    if (At) TK(cudaMemcpyAsync(At, o.At, sizeof(float) * D3 * D3, cudaMemcpyDeviceToHost, t->stream));
    if (X) TK(cudaMemcpyAsync(X, o.X, sizeof(float) * o.n * LC_IN, cudaMemcpyDeviceToHost, t->stream));
    if (R) TK(cudaMemcpyAsync(R, o.R, sizeof(float) * D3 * o.calls, cudaMemcpyDeviceToHost, t->stream));
    if (D) TK(cudaMemcpyAsync(D, o.D, sizeof(float) * D3 * o.calls, cudaMemcpyDeviceToHost, t->stream));
    if (E) TK(cudaMemcpyAsync(E, o.E, sizeof(double) * o.calls, cudaMemcpyDeviceToHost, t->stream));
    t->sync();
  });
}

namespace {
// Uploads one minibatch's int block: op indices [TR_MAX_BATCH] then row starts [TR_MAX_BATCH + 1].
std::vector<int> batchBlock(const btd_trainer* t, const std::vector<int>& batch, int* rows, int* calls) {
  std::vector<int> blk(2 * TR_MAX_BATCH + 1, 0);
  int r = 0, c = 0;
  for (size_t b = 0; b < batch.size(); ++b) {
    blk[b] = batch[b];
    blk[TR_MAX_BATCH + b] = r;
    r += t->ops[batch[b]].n;
    c += t->ops[batch[b]].calls;
  }
  blk[TR_MAX_BATCH + batch.size()] = r;
  *rows = r;
  *calls = c;
  return blk;
}
}  // namespace

extern "C" int btd_trainer_loss_grad(btd_trainer* t, const float* weights, const int32_t* op_list, int32_t n_ops, double* loss, float* grad) {
  TGUARD({
    checkTrainer(t);
    if (!weights || !op_list || n_ops < 1 || n_ops > TR_MAX_BATCH)
      throw std::invalid_argument("btd_trainer_loss_grad: 1.." + std::to_string(TR_MAX_BATCH) + " operators and the weights");
    std::vector<int> batch(op_list, op_list + n_ops);
    for (int b : batch)
      if (b < 0 || b >= (int)t->ops.size()) throw std::invalid_argument("btd_trainer_loss_grad: operator out of range");
    int rows = 0, calls = 0;
    const std::vector<int> blk = batchBlock(t, batch, &rows, &calls);
    if (calls == 0) throw std::invalid_argument("btd_trainer_loss_grad: the operators have no calls");
    t->ensureRows(rows);
    if (t->batchCap < blk.size()) {
      t->release(t->dBatch);
      t->batchCap = blk.size();
      t->dBatch = t->alloc<int>(t->batchCap);
    }
    TK(cudaMemcpyAsync(t->w, weights, sizeof(float) * LC_WEIGHTS, cudaMemcpyHostToDevice, t->stream));
    TK(cudaMemcpyAsync(t->dBatch, blk.data(), sizeof(int) * blk.size(), cudaMemcpyHostToDevice, t->stream));
    k_tr_pack<<<1, 256, 0, t->stream>>>(t->w, t->P, t->PT);
    const double inv = 1.0 / calls;
    const int parts = t->launchStep(batch, t->dBatch, rows, inv);
    if (!t->lossHist) {
      t->histCap = 1;
      t->lossHist = t->alloc<float>(1);
    }
    AdamArgs a{t->w, t->m, t->v, t->grad, t->P, t->PT, t->partial, parts, 0, 1, 0.f, t->lossParts, n_ops, inv, nullptr};
    k_tr_adam<<<1, 1024, 0, t->stream>>>(a);
    TK(cudaGetLastError());
    std::vector<double> lp(n_ops);
    TK(cudaMemcpyAsync(lp.data(), t->lossParts, sizeof(double) * n_ops, cudaMemcpyDeviceToHost, t->stream));
    if (grad) TK(cudaMemcpyAsync(grad, t->grad, sizeof(float) * LC_WEIGHTS, cudaMemcpyDeviceToHost, t->stream));
    t->sync();
    double l = 0.0;
    for (double v : lp) l += v;
    if (loss) *loss = l * inv;
  });
}

extern "C" int btd_trainer_train(btd_trainer* t, float* weights, int32_t steps, int32_t batch_ops, float lr, uint64_t seed,
                                 const float* group_weights, int32_t n_groups, float* loss_history) {
  TGUARD({
    checkTrainer(t);
    if (!weights || steps < 1 || batch_ops < 1 || batch_ops > TR_MAX_BATCH || !(lr > 0.f))
      throw std::invalid_argument("btd_trainer_train: weights, steps >= 1, 1 <= batch_ops <= 16 and lr > 0");
    std::vector<int> usable;
    for (int k = 0; k < (int)t->ops.size(); ++k)
      if (t->ops[k].calls > 0) usable.push_back(k);
    if (usable.empty()) throw std::invalid_argument("btd_trainer_train: no training material");
    // operators drawn in proportion to their group's weight divided by the group's size, so that each
    // group weighs the same when its weight is the same, whatever its number of operators
    std::vector<double> prob(usable.size(), 1.0);
    if (group_weights && n_groups > 0) {
      std::vector<int> count(n_groups, 0);
      for (int k : usable)
        if (t->ops[k].group >= 0 && t->ops[k].group < n_groups) count[t->ops[k].group]++;
      for (size_t q = 0; q < usable.size(); ++q) {
        const int g = t->ops[usable[q]].group;
        prob[q] = (g >= 0 && g < n_groups && count[g] > 0) ? group_weights[g] / count[g] : 0.0;
      }
    }
    std::mt19937_64 rng(seed);
    const int nb = std::min<int>(batch_ops, (int)usable.size());
    // every step's minibatch (without replacement within a step), drawn up front
    std::vector<std::vector<int>> batches(steps);
    std::vector<int> allBlk;
    std::vector<int> stepRows(steps), stepCalls(steps);
    int maxRows = 0;
    for (int s = 0; s < steps; ++s) {
      std::vector<double> p(prob);
      for (int b = 0; b < nb; ++b) {
        std::discrete_distribution<int> pick(p.begin(), p.end());
        const int q = pick(rng);
        batches[s].push_back(usable[q]);
        p[q] = 0.0;
      }
      const std::vector<int> blk = batchBlock(t, batches[s], &stepRows[s], &stepCalls[s]);
      allBlk.insert(allBlk.end(), blk.begin(), blk.end());
      maxRows = std::max(maxRows, stepRows[s]);
    }
    const size_t blkSize = 2 * TR_MAX_BATCH + 1;
    t->ensureRows(maxRows);
    if (t->batchCap < allBlk.size()) {
      t->release(t->dBatch);
      t->batchCap = allBlk.size();
      t->dBatch = t->alloc<int>(t->batchCap);
    }
    if (t->histCap < (size_t)steps) {
      t->release(t->lossHist);
      t->histCap = steps;
      t->lossHist = t->alloc<float>(steps);
    }
    TK(cudaMemcpyAsync(t->dBatch, allBlk.data(), sizeof(int) * allBlk.size(), cudaMemcpyHostToDevice, t->stream));
    TK(cudaMemcpyAsync(t->w, weights, sizeof(float) * LC_WEIGHTS, cudaMemcpyHostToDevice, t->stream));
    TK(cudaMemsetAsync(t->m, 0, sizeof(float) * LC_WEIGHTS, t->stream));
    TK(cudaMemsetAsync(t->v, 0, sizeof(float) * LC_WEIGHTS, t->stream));
    k_tr_pack<<<1, 256, 0, t->stream>>>(t->w, t->P, t->PT);
    for (int s = 0; s < steps; ++s) {
      const int* dB = t->dBatch + (size_t)s * blkSize;
      const double inv = 1.0 / std::max(1, stepCalls[s]);
      const int parts = t->launchStep(batches[s], dB, stepRows[s], inv);
      const float lrs = lr * std::pow(0.1f, (float)(s + 1) / steps);  // decays tenfold over the run
      AdamArgs a{t->w, t->m, t->v, nullptr, t->P, t->PT, t->partial, parts, 1, s + 1, lrs, t->lossParts, nb, inv, t->lossHist};
      k_tr_adam<<<1, 1024, 0, t->stream>>>(a);
    }
    TK(cudaGetLastError());
    TK(cudaMemcpyAsync(weights, t->w, sizeof(float) * LC_WEIGHTS, cudaMemcpyDeviceToHost, t->stream));
    if (loss_history) TK(cudaMemcpyAsync(loss_history, t->lossHist, sizeof(float) * steps, cudaMemcpyDeviceToHost, t->stream));
    t->sync();
  });
}
