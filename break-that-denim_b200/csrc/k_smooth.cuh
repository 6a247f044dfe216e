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

// Line row of node n (k-th on its line, family fam) from a fine row: diagonal plus the Frobenius
// majorisation of the +-2 along-line couplings, the +1 along-line block, and the rhs with every other
// coupling lagged at the current iterate (lineRow, smooth.wgsl:49-84; smoothLines,
// newtonMultigrid.ts:676-720). All loads are issued before any use.
__device__ __forceinline__ void fineLineRow(const DLevel& L, int n, int k, int len, int fam, Sym* Bk, Sym* Ck, float3* rr) {
  float4 pl[FINE_PLANES];
#pragma unroll
  for (int p = 0; p < FINE_PLANES; ++p) pl[p] = __ldg(&L.op[(size_t)p * L.N + n]);
  const uint2 cc = L.coord[n];
  const int i = cc.x & 0xFFFF, j = cc.x >> 16;
  const DLevelLayer ly = L.layers[cc.y];
  float3 xm[12];
  bool ok[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    const int2 o = fineOffset(q);
    const int ii = i + o.x, jj = j + o.y;
    ok[q] = ii >= 0 && jj >= 0 && ii < ly.nx && jj < ly.ny;
    const int m = ok[q] ? ly.offset + jj * ly.nx + ii : n;
    xm[q] = f3(L.X[m]);
  }
  const float3 xn = f3(L.X[n]);
  float3 r = f3(L.B[n]);
  const float* row = reinterpret_cast<const float*>(pl);
  auto blk = [&](int b) { return Sym{row[6 * b], row[6 * b + 1], row[6 * b + 2], row[6 * b + 3], row[6 * b + 4], row[6 * b + 5]}; };
  // along-line couplings: u-lines use +u (0), -u (1), +-2u scalars (8, 9); v-lines +v (2), -v (3), +-2v (10, 11)
  const int qNext = fam == 0 ? 0 : 2, qPrev = fam == 0 ? 1 : 3, qS = fam == 0 ? 8 : 10;
  float maj = 0.f;
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    if (q == qPrev) continue;
    if (q == qNext) {
      if (k + 1 < len) *Ck = blk(q + 1);
      continue;
    }
    if (!ok[q]) continue;
    if (q < 8) {
      r -= blk(q + 1) * xm[q];
    } else {
      const float sc = row[54 + (q - 8)];
      if (q == qS || q == qS + 1) maj += 1.7320508075688772f * fabsf(sc);
      r -= sc * xm[q];
    }
  }
  *Bk = blk(0) + symId(maj);
  *rr = r + maj * xn;
}

// The same from a coarse (25-block) row, one stencil row of 5 blocks (30 floats) at a time.
__device__ __forceinline__ void coarseLineRow(const DLevel& L, int n, int k, int len, int fam, Sym* Bk, Sym* Ck, float3* rr) {
  const uint2 cc = L.coord[n];
  const int i = cc.x & 0xFFFF, j = cc.x >> 16;
  const DLevelLayer ly = L.layers[cc.y];
  const float3 xn = f3(L.X[n]);
  float3 r = f3(L.B[n]);
  float maj = 0.f;
  Sym D = symZero();
#pragma unroll
  for (int dj = -2; dj <= 2; ++dj) {
    // floats 30 (dj + 2) .. + 29 live in planes p0 .. p0 + 8
    const int f0 = 30 * (dj + 2), p0 = f0 >> 2, sh = f0 & 3;
    float4 pl[9];
#pragma unroll
    for (int p = 0; p < 9; ++p) pl[p] = p0 + p < COARSE_PLANES ? __ldg(&L.op[(size_t)(p0 + p) * L.N + n]) : make_float4(0, 0, 0, 0);
    float3 xm[5];
    bool ok[5];
#pragma unroll
    for (int di = -2; di <= 2; ++di) {
      const int ii = i + di, jj = j + dj;
      ok[di + 2] = ii >= 0 && jj >= 0 && ii < ly.nx && jj < ly.ny;
      const int m = ok[di + 2] ? ly.offset + jj * ly.nx + ii : n;
      xm[di + 2] = f3(L.X[m]);
    }
    const float* row = reinterpret_cast<const float*>(pl) + sh;
#pragma unroll
    for (int di = -2; di <= 2; ++di) {
      const float* b = row + 6 * (di + 2);
      const Sym B = {b[0], b[1], b[2], b[3], b[4], b[5]};
      const int along = fam == 0 ? di : dj, across = fam == 0 ? dj : di;
      if (across == 0 && along == 0) {
        D = B;
        continue;
      }
      if (across == 0 && along == -1) continue;
      if (across == 0 && along == 1) {
        if (k + 1 < len) *Ck = B;
        continue;
      }
      if (!ok[di + 2]) continue;
      if (across == 0) maj += symFrob(B);
      r -= B * xm[di + 2];
    }
  }
  *Bk = D + symId(maj);
  *rr = r + maj * xn;
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

  // ---- phase 1: line rows (each thread issues its row's and its neighbours' loads together)
  for (int k = tid; k < len; k += SM_THREADS) {
    const int n = n0 + k * st;
    Sym Bk = symId(1.f), Ck = symZero();
    float3 r = make_float3(0, 0, 0);
    if (!L.fixed[n]) {
      if constexpr (Rows::NC == 12)
        fineLineRow(L, n, k, len, fam, &Bk, &Ck, &r);
      else
        coarseLineRow(L, n, k, len, fam, &Bk, &Ck, &r);
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
