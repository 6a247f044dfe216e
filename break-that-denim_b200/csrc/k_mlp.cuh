// The learned coarse space's network on the tensor cores: a 3-layer MLP (20 -> 64 -> 64 -> 24, tanh
// after both hidden layers) with BF16 weights and activations and FP32 accumulation, evaluated by
// warp-level BF16 MMAs (m16n8k16). No counterpart in the reference (an extension of its coarsest
// V-cycle level, newtonMultigrid.ts:495-502).
//
// Weights arrive as the flat FP32 layout W1[20][64], b1[64], W2[64][64], b2[64], W3[64][24], b3[24]
// (row-major [in][out]); output 3 k + c is coordinate c of basis vector k at a node. On the device
// the matrices are kept rounded to BF16 and packed in MMA fragment order (k_mlp_pack), so that a lane
// loads its B fragment of one (k-chunk, n-tile) as a single 8-byte word; the biases stay FP32 (they
// are BF16-rounded values, like every weight).
//
// Layer shapes in MMA tiles: layer 1 K = 20 padded to 32 (2 k-chunks of 16) x N = 64 (8 n-tiles of 8);
// layer 2 K = 64 (4) x N = 64 (8); layer 3 K = 64 (4) x N = 24 (3). A warp evaluates 16 rows; the
// accumulators of two adjacent n-tiles are exactly the A fragment of one k-chunk of the next layer, so
// the hidden activations stay in registers.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace btd {

constexpr int LC_IN = 20, LC_HID = 64, LC_K = 8, LC_OUT = 3 * LC_K;
constexpr int LC_IN_PAD = 32;
constexpr int LC_MAX_NODES = 576;  // coarsest nodes the one-CTA basis holds in shared memory (215 KB at 576)
constexpr int LC_WEIGHTS = LC_IN * LC_HID + LC_HID + LC_HID * LC_HID + LC_HID + LC_HID * LC_OUT + LC_OUT;  // 7064
// flat offsets
constexpr int LC_W1 = 0, LC_B1 = LC_W1 + LC_IN * LC_HID, LC_W2 = LC_B1 + LC_HID, LC_B2 = LC_W2 + LC_HID * LC_HID,
              LC_W3 = LC_B2 + LC_HID, LC_B3 = LC_W3 + LC_HID * LC_OUT;
// packed fragments (uint2 per lane per (k-chunk, n-tile))
constexpr int LC_F1 = 0, LC_F2 = LC_F1 + 2 * 8 * 32, LC_F3 = LC_F2 + 4 * 8 * 32, LC_FRAGS = LC_F3 + 4 * 3 * 32;  // uint2 count
constexpr int LC_BIAS = LC_HID + LC_HID + LC_OUT;

struct MlpPacked {
  uint2 frag[LC_FRAGS];   // 1920 uint2 = 15 KB
  float bias[LC_BIAS];    // b1, b2, b3
};

__device__ __forceinline__ uint32_t packBf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low 16 bits), .y = hi
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float bf16Round(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// D += A B for one m16n8k16 tile: BF16 operands, FP32 accumulators.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// B fragment of lane `lane` for k-chunk kc, n-tile nt of a row-major [K][N] matrix W (rows >= K zero):
// (k = 16 kc + 2 t + {0, 1}, n = 8 nt + g) and (k + 8, n), g = lane / 4, t = lane % 4.
__device__ __forceinline__ uint2 fragB(const float* W, int K, int N, int kc, int nt, int lane) {
  const int g = lane >> 2, t = lane & 3, n = 8 * nt + g, k0 = 16 * kc + 2 * t;
  auto w = [&](int k) { return k < K && n < N ? W[k * N + n] : 0.f; };
  return make_uint2(packBf16(w(k0), w(k0 + 1)), packBf16(w(k0 + 8), w(k0 + 9)));
}

// Packs flat FP32 weights (rounded to BF16) into fragment order, threads tid of nthreads of one CTA.
__device__ __forceinline__ void mlpPack(const float* __restrict__ w, MlpPacked* out, int tid, int nthreads) {
  for (int q = tid; q < LC_FRAGS; q += nthreads) {
    const int lane = q & 31;
    uint2 f;
    if (q < LC_F2) {
      const int s = q >> 5, kc = s / 8, nt = s % 8;
      f = fragB(w + LC_W1, LC_IN, LC_HID, kc, nt, lane);
    } else if (q < LC_F3) {
      const int s = (q - LC_F2) >> 5, kc = s / 8, nt = s % 8;
      f = fragB(w + LC_W2, LC_HID, LC_HID, kc, nt, lane);
    } else {
      const int s = (q - LC_F3) >> 5, kc = s / 3, nt = s % 3;
      f = fragB(w + LC_W3, LC_HID, LC_OUT, kc, nt, lane);
    }
    out->frag[q] = f;
  }
  for (int q = tid; q < LC_BIAS; q += nthreads) {
    const float v = q < LC_HID ? w[LC_B1 + q] : q < 2 * LC_HID ? w[LC_B2 + q - LC_HID] : w[LC_B3 + q - 2 * LC_HID];
    out->bias[q] = bf16Round(v);
  }
}

// The transposed weight fragments the backward pass multiplies by: W3^T (K = 24 padded to 32, N = 64)
// and W2^T (K = 64, N = 64), element (k, n) = W[n][k].
constexpr int LC_T3 = 0, LC_T2 = LC_T3 + 2 * 8 * 32, LC_TFRAGS = LC_T2 + 4 * 8 * 32;
struct MlpPackedT {
  uint2 frag[LC_TFRAGS];
};

// B fragment of the transpose of a row-major [N][K] matrix W: element (k, n) = W[n][k].
__device__ __forceinline__ uint2 fragBT(const float* W, int K, int N, int kc, int nt, int lane) {
  const int g = lane >> 2, t = lane & 3, n = 8 * nt + g, k0 = 16 * kc + 2 * t;
  auto w = [&](int k) { return k < K && n < N ? W[n * K + k] : 0.f; };
  return make_uint2(packBf16(w(k0), w(k0 + 1)), packBf16(w(k0 + 8), w(k0 + 9)));
}

__device__ __forceinline__ void mlpPackT(const float* __restrict__ w, MlpPackedT* out, int tid, int nthreads) {
  for (int q = tid; q < LC_TFRAGS; q += nthreads) {
    const int lane = q & 31;
    if (q < LC_T2) {
      const int s = q >> 5, kc = s / 8, nt = s % 8;
      out->frag[q] = fragBT(w + LC_W3, LC_OUT, LC_HID, kc, nt, lane);
    } else {
      const int s = (q - LC_T2) >> 5, kc = s / 8, nt = s % 8;
      out->frag[q] = fragBT(w + LC_W2, LC_HID, LC_HID, kc, nt, lane);
    }
  }
}

// Row stride (bf16 elements) of the input tile in shared memory: 40 keeps a fragment load free of bank
// conflicts (8 rows x 20 words land on distinct banks).
constexpr int LC_XSTRIDE = 40;

// A fragment of k-chunk kc from a bf16 row-major tile X (16 rows, stride LC_XSTRIDE) in shared memory.
__device__ __forceinline__ void fragAFromSmem(const __nv_bfloat16* X, int kc, int lane, uint32_t (&a)[4]) {
  const int g = lane >> 2, t = lane & 3, c = 16 * kc + 2 * t;
  const uint32_t* r0 = reinterpret_cast<const uint32_t*>(X + g * LC_XSTRIDE);
  const uint32_t* r1 = reinterpret_cast<const uint32_t*>(X + (g + 8) * LC_XSTRIDE);
  a[0] = r0[c >> 1];
  a[1] = r1[c >> 1];
  a[2] = r0[(c + 8) >> 1];
  a[3] = r1[(c + 8) >> 1];
}

// A fragments of the next layer from the accumulators of 2 adjacent n-tiles (after the activation).
__device__ __forceinline__ void fragAFromAcc(const float (&lo)[4], const float (&hi)[4], uint32_t (&a)[4]) {
  a[0] = packBf16(lo[0], lo[1]);
  a[1] = packBf16(lo[2], lo[3]);
  a[2] = packBf16(hi[0], hi[1]);
  a[3] = packBf16(hi[2], hi[3]);
}

// Forward pass of one 16-row tile by one warp. X: the tile's inputs (bf16, stride LC_XSTRIDE, columns
// 20..31 zero). On return out[nt][4] holds the output accumulators of n-tile nt (rows g, g + 8; columns
// 8 nt + 2 t + {0, 1}); when h1/h2 are given, the hidden activations (after tanh, as the BF16 values
// the next layer used) are stored there row-major [16][64] in FP32 for a backward pass.
__device__ __forceinline__ void mlpForwardTile(const MlpPacked& P, const __nv_bfloat16* X, int lane, float (&out)[3][4],
                                               float* h1 = nullptr, float* h2 = nullptr) {
  const int g = lane >> 2, t = lane & 3;
  float acc[8][4];
  // layer 1
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = P.bias[8 * nt + 2 * t], b1 = P.bias[8 * nt + 2 * t + 1];
    acc[nt][0] = b0, acc[nt][1] = b1, acc[nt][2] = b0, acc[nt][3] = b1;
  }
#pragma unroll
  for (int kc = 0; kc < 2; ++kc) {
    uint32_t a[4];
    fragAFromSmem(X, kc, lane, a);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) mma16816(acc[nt], a, P.frag[LC_F1 + (kc * 8 + nt) * 32 + lane]);
  }
  uint32_t ah[4][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = bf16Round(tanhf(acc[nt][q]));
  if (h1)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = 8 * nt + 2 * t;
      h1[g * 64 + c] = acc[nt][0], h1[g * 64 + c + 1] = acc[nt][1];
      h1[(g + 8) * 64 + c] = acc[nt][2], h1[(g + 8) * 64 + c + 1] = acc[nt][3];
    }
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) fragAFromAcc(acc[2 * kc], acc[2 * kc + 1], ah[kc]);
  // layer 2
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = P.bias[LC_HID + 8 * nt + 2 * t], b1 = P.bias[LC_HID + 8 * nt + 2 * t + 1];
    acc[nt][0] = b0, acc[nt][1] = b1, acc[nt][2] = b0, acc[nt][3] = b1;
  }
#pragma unroll
  for (int kc = 0; kc < 4; ++kc)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) mma16816(acc[nt], ah[kc], P.frag[LC_F2 + (kc * 8 + nt) * 32 + lane]);
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = bf16Round(tanhf(acc[nt][q]));
  if (h2)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int c = 8 * nt + 2 * t;
      h2[g * 64 + c] = acc[nt][0], h2[g * 64 + c + 1] = acc[nt][1];
      h2[(g + 8) * 64 + c] = acc[nt][2], h2[(g + 8) * 64 + c + 1] = acc[nt][3];
    }
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) fragAFromAcc(acc[2 * kc], acc[2 * kc + 1], ah[kc]);
  // layer 3
#pragma unroll
  for (int nt = 0; nt < 3; ++nt) {
    const float b0 = P.bias[2 * LC_HID + 8 * nt + 2 * t], b1 = P.bias[2 * LC_HID + 8 * nt + 2 * t + 1];
    out[nt][0] = b0, out[nt][1] = b1, out[nt][2] = b0, out[nt][3] = b1;
  }
#pragma unroll
  for (int kc = 0; kc < 4; ++kc)
#pragma unroll
    for (int nt = 0; nt < 3; ++nt) mma16816(out[nt], ah[kc], P.frag[LC_F3 + (kc * 3 + nt) * 32 + lane]);
}

}  // namespace btd
