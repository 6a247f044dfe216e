// Yarn-line smoother: every line of one colour solved exactly as a block-tridiagonal system
// (smoothLines + solvePenta, newtonMultigrid.ts:659-733 / 435-473; smooth.wgsl:49-233).
//
// One CTA per line. Phase 1 (all threads, one node each): the line rows - diagonal block plus the
// Frobenius majorisation of the +-2 along-line couplings, the +1 coupling, and the rhs with every
// off-line and +-2 coupling lagged at the previous iterate (Jacobi within a colour). Lines of one
// colour are three apart, so they never read each other's unknowns. Phase 2 (P <= 64 threads): the
// partition method - each thread eliminates the interior of its chunk, expressing it through the
// chunk's end unknowns. Phase 3: the 2P end equations by odd-even cyclic reduction in shared memory
// (Gaussian elimination in a symmetric order, as accurate as the serial solve on these SPD
// systems). Phase 4: interior recovery and write-back. Every pivot is regularised by pivotInverse.
// The lower block of row k is the +1 block of row k - 1 (symmetric), as solvePenta takes it.
#pragma once

#include "common.cuh"
#include "k_mg.cuh"

namespace btd {

constexpr int SM_THREADS = 128;
constexpr int SM_PMAX = 64;
constexpr int SM_MAX_LINE = 1024;

// Shared-memory floats for a line of length len: rows (B 6, C 6, r 3), chunk data (G 9, h 3, V 9,
// W 9) per node, and the 2 * SM_PMAX reduced rows (L, D, U 9 each; r, x 3 each).
__host__ __device__ constexpr int smoothSmemFloats(int len) { return 45 * len + 2 * SM_PMAX * 33; }

__device__ __forceinline__ Sym ldSym(const float* p) { return {p[0], p[1], p[2], p[3], p[4], p[5]}; }
__device__ __forceinline__ void stSym(float* p, Sym s) {
  p[0] = s.xx, p[1] = s.xy, p[2] = s.xz, p[3] = s.yy, p[4] = s.yz, p[5] = s.zz;
}
__device__ __forceinline__ M3 ldM3(const float* p) {
  M3 m;
#pragma unroll
  for (int q = 0; q < 9; ++q) m.a[q] = p[q];
  return m;
}
__device__ __forceinline__ void stM3(float* p, const M3& m) {
#pragma unroll
  for (int q = 0; q < 9; ++q) p[q] = m.a[q];
}
__device__ __forceinline__ float3 ld3(const float* p) { return make_float3(p[0], p[1], p[2]); }
__device__ __forceinline__ void st3(float* p, float3 v) { p[0] = v.x, p[1] = v.y, p[2] = v.z; }
__device__ __forceinline__ M3 m3Add(const M3& x, const M3& y) {
  M3 o;
#pragma unroll
  for (int q = 0; q < 9; ++q) o.a[q] = x.a[q] + y.a[q];
  return o;
}

template <class Rows>
__global__ void __launch_bounds__(SM_THREADS) k_smooth(DLevel L, const int4* __restrict__ lines, int first) {
  extern __shared__ float sm[];
  const int4 line = lines[first + blockIdx.x];  // (start node, stride, length, family)
  const int n0 = line.x, st = line.y, len = line.z, fam = line.w;
  const int tid = threadIdx.x;
  float* sB = sm;              // 6 per node
  float* sC = sB + 6 * len;    // 6 per node
  float* sR = sC + 6 * len;    // 3 per node
  float* sG = sR + 3 * len;    // 9 per node
  float* sH = sG + 9 * len;    // 3 per node (h, then v)
  float* sV = sH + 3 * len;    // 9 per node (Hs, then V)
  float* sW = sV + 9 * len;    // 9 per node (He, then W)
  float* qL = sW + 9 * len;    // 9 per reduced row
  float* qD = qL + 9 * 2 * SM_PMAX;
  float* qU = qD + 9 * 2 * SM_PMAX;
  float* qr = qU + 9 * 2 * SM_PMAX;
  float* qx = qr + 3 * 2 * SM_PMAX;

  // ---- phase 1: line rows
  for (int k = tid; k < len; k += SM_THREADS) {
    const int n = n0 + k * st;
    Sym Bk = symId(1.f), Ck = symZero();
    float3 r = make_float3(0, 0, 0);
    if (!L.fixed[n]) {
      int i, j, l;
      nodeCoord(L, n, &i, &j, &l);
      const DLevelLayer Ly = L.layers[l];
      Sym D = Rows::diag(L.op, L.N, n);
      r = f3(L.B[n]);
      float maj = 0.f;
      for (int c = 0; c < Rows::NC; ++c) {
        const int2 off = Rows::offset(c);
        const int along = fam == 0 ? off.x : off.y;
        const int across = fam == 0 ? off.y : off.x;
        if (across == 0 && along == -1) continue;
        if (across == 0 && along == 1) {
          if (k + 1 < len) Ck = Rows::coupling(L.op, L.N, n, c);
          continue;
        }
        const int m = levelNode(Ly, i + off.x, j + off.y);
        if (m < 0) continue;
        const Sym Bc = Rows::coupling(L.op, L.N, n, c);
        if (across == 0) maj += symFrob(Bc);
        r -= Bc * f3(L.X[m]);
      }
      Bk = D + symId(maj);
      r += maj * f3(L.X[n]);
    }
    stSym(sB + 6 * k, Bk);
    stSym(sC + 6 * k, Ck);
    st3(sR + 3 * k, r);
  }
  __syncthreads();

  const int P = max(1, min(SM_PMAX, len / 2));
  const int base = len / P, extra = len % P;
  const int ks = tid * base + min(tid, extra);
  const int mlen = base + (tid < extra ? 1 : 0);
  const int ke = ks + mlen - 1;

  // ---- phase 2: chunk-interior elimination, right-hand sides [r | x_s | x_e]
  if (tid < P) {
    M3 Gp = m3Zero(), Hsp = m3Id(), Hep = m3Zero();
    float3 hp = make_float3(0, 0, 0);
    for (int k = ks + 1; k < ke; ++k) {
      const M3 Ak = m3FromSym(ldSym(sC + 6 * (k - 1)));
      const M3 Bk = m3FromSym(ldSym(sB + 6 * k));
      const M3 Ck = m3FromSym(ldSym(sC + 6 * k));
      const M3 Minv = pivotInverse(m3Sub(Bk, m3Mul(Ak, Gp)));
      M3 G = m3Zero(), Cext = m3Zero();
      if (k + 1 < ke)
        G = m3Mul(Minv, Ck);
      else
        Cext = Ck;
      const float3 h = m3Vec(Minv, ld3(sR + 3 * k) - m3Vec(Ak, hp));
      const M3 Hs = m3Mul(Minv, m3Neg(m3Mul(Ak, Hsp)));
      const M3 He = m3Mul(Minv, m3Sub(m3Neg(m3Mul(Ak, Hep)), Cext));
      stM3(sG + 9 * k, G);
      st3(sH + 3 * k, h);
      stM3(sV + 9 * k, Hs);
      stM3(sW + 9 * k, He);
      Gp = G, hp = h, Hsp = Hs, Hep = He;
    }
    // back substitution inside the chunk: x_k = v_k + V_k x_s + W_k x_e
    float3 vS = make_float3(0, 0, 0), vE = make_float3(0, 0, 0);
    M3 VS = m3Zero(), WS = m3Id(), VE = m3Id(), WE = m3Zero();
    if (mlen >= 3) {
      float3 vn = make_float3(0, 0, 0);
      M3 Vn = m3Zero(), Wn = m3Zero();
      for (int k = ke - 1; k > ks; --k) {
        const M3 G = ldM3(sG + 9 * k);
        const float3 v = ld3(sH + 3 * k) - m3Vec(G, vn);
        const M3 V = m3Sub(ldM3(sV + 9 * k), m3Mul(G, Vn));
        const M3 W = m3Sub(ldM3(sW + 9 * k), m3Mul(G, Wn));
        st3(sH + 3 * k, v);
        stM3(sV + 9 * k, V);
        stM3(sW + 9 * k, W);
        if (k == ke - 1) vE = v, VE = V, WE = W;
        vn = v, Vn = V, Wn = W;
      }
      vS = vn, VS = Vn, WS = Wn;
    }
    // reduced equations for x_s (row 2 tid) and x_e (row 2 tid + 1)
    const M3 As = ks > 0 ? m3FromSym(ldSym(sC + 6 * (ks - 1))) : m3Zero();
    const M3 Bs = m3FromSym(ldSym(sB + 6 * ks)), Cs = m3FromSym(ldSym(sC + 6 * ks));
    const M3 Ae = m3FromSym(ldSym(sC + 6 * (ke - 1))), Be = m3FromSym(ldSym(sB + 6 * ke));
    const M3 Ce = m3FromSym(ldSym(sC + 6 * ke));
    stM3(qL + 9 * (2 * tid), As);
    stM3(qD + 9 * (2 * tid), m3Add(Bs, m3Mul(Cs, VS)));
    stM3(qU + 9 * (2 * tid), m3Mul(Cs, WS));
    st3(qr + 3 * (2 * tid), ld3(sR + 3 * ks) - m3Vec(Cs, vS));
    stM3(qL + 9 * (2 * tid + 1), m3Mul(Ae, VE));
    stM3(qD + 9 * (2 * tid + 1), m3Add(Be, m3Mul(Ae, WE)));
    stM3(qU + 9 * (2 * tid + 1), Ce);
    st3(qr + 3 * (2 * tid + 1), ld3(sR + 3 * ke) - m3Vec(Ae, vE));
  }
  __syncthreads();

  // ---- phase 3: odd-even cyclic reduction of the 2P reduced rows. At stride s the rows with
  // (q + 1) % 2s == 0 eliminate their neighbours q -+ s, which no longer change.
  const int Q = 2 * P;
  int stride = 1;
  while (2 * stride <= Q) {
    const int q = tid;
    if (q < Q && (q + 1) % (2 * stride) == 0) {
      const int lo = q - stride;
      const M3 al = m3Mul(ldM3(qL + 9 * q), pivotInverse(ldM3(qD + 9 * lo)));
      M3 D = m3Sub(ldM3(qD + 9 * q), m3Mul(al, ldM3(qU + 9 * lo)));
      float3 r = ld3(qr + 3 * q) - m3Vec(al, ld3(qr + 3 * lo));
      const M3 Lq = m3Neg(m3Mul(al, ldM3(qL + 9 * lo)));
      M3 Uq = m3Zero();
      if (q + stride < Q) {
        const int hi = q + stride;
        const M3 ga = m3Mul(ldM3(qU + 9 * q), pivotInverse(ldM3(qD + 9 * hi)));
        D = m3Sub(D, m3Mul(ga, ldM3(qL + 9 * hi)));
        r = r - m3Vec(ga, ld3(qr + 3 * hi));
        Uq = m3Neg(m3Mul(ga, ldM3(qU + 9 * hi)));
      }
      stM3(qD + 9 * q, D);
      st3(qr + 3 * q, r);
      stM3(qL + 9 * q, Lq);
      stM3(qU + 9 * q, Uq);
    }
    __syncthreads();
    stride *= 2;
  }
  while (stride > 0) {
    const int q = tid;
    if (q < Q && (q + 1) % stride == 0 && (q + 1) % (2 * stride) != 0) {
      float3 r = ld3(qr + 3 * q);
      if (q >= stride) r = r - m3Vec(ldM3(qL + 9 * q), ld3(qx + 3 * (q - stride)));
      if (q + stride < Q) r = r - m3Vec(ldM3(qU + 9 * q), ld3(qx + 3 * (q + stride)));
      st3(qx + 3 * q, m3Vec(pivotInverse(ldM3(qD + 9 * q)), r));
    }
    __syncthreads();
    stride /= 2;
  }

  // ---- phase 4: recovery and write-back
  if (tid < P) {
    const float3 xs = ld3(qx + 3 * (2 * tid)), xe = ld3(qx + 3 * (2 * tid + 1));
    const int ns = n0 + ks * st, ne = n0 + ke * st;
    if (!L.fixed[ns]) L.X[ns] = make_float4(xs.x, xs.y, xs.z, 0.f);
    if (!L.fixed[ne]) L.X[ne] = make_float4(xe.x, xe.y, xe.z, 0.f);
    for (int k = ks + 1; k < ke; ++k) {
      const int n = n0 + k * st;
      if (L.fixed[n]) continue;
      const float3 x = ld3(sH + 3 * k) + m3Vec(ldM3(sV + 9 * k), xs) + m3Vec(ldM3(sW + 9 * k), xe);
      L.X[n] = make_float4(x.x, x.y, x.z, 0.f);
    }
  }
}

}  // namespace btd
