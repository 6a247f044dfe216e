// Yarn-line smoother: every line of one colour solved exactly as a block-tridiagonal system
// (smoothLines + solvePenta, newtonMultigrid.ts:659-733 / 435-473; smooth.wgsl:49-233).
//
// One CTA per line; the kernel is a latency chain, so each phase is built to keep that chain short.
// Phase 1 (one thread per node, in tiles of SM_THREADS nodes): the thread stages its row planes, the
// unknowns of its stencil neighbours and its rhs into its own shared-memory slot with cp.async -
// all copies in flight at once, one round trip - then builds its line row from the slot: diagonal
// block plus the Frobenius majorisation of the +-2 along-line couplings, the +1 along-line block,
// and the rhs with every off-line and +-2 coupling lagged at the current iterate (Jacobi within a
// colour: lines of one colour are three apart and never read each other's unknowns).
// Phase 2 (P <= 64 threads): the partition method - each thread eliminates its chunk's interior,
// expressing it through the chunk's end unknowns. Phase 3: the 2P end equations by odd-even cyclic
// reduction in shared memory (Gaussian elimination in a symmetric order: the accuracy of the serial
// solve on these SPD systems). Phase 4: interior recovery and write-back. Every pivot is regularised
// by pivotInverse. The lower block of row k is the +1 block of row k - 1 (symmetric), as solvePenta
// takes it.
#pragma once

#include "common.cuh"
#include "k_mg.cuh"

namespace btd {

constexpr int SM_THREADS = 128;
constexpr int SM_PMAX = 64;
constexpr int SM_MAX_LINE = 512;

template <class Rows>
struct SlotOf;
template <>
struct SlotOf<FineRows> {
  static constexpr int PLANES = FINE_PLANES, NC = 12;
};
template <>
struct SlotOf<CoarseRows> {
  static constexpr int PLANES = COARSE_PLANES, NC = 24;
};

// Shared memory (float4 units) of a line of length len: per-thread staging slots (row planes,
// neighbour unknowns, own unknown, rhs), per node the line row (B 2, C 2, r 1) and chunk data
// (G 3, h 1, V 3, W 3), and the 2 * SM_PMAX reduced rows (L, D, U 3 each; r, x 1 each).
template <class Rows>
__host__ __device__ constexpr int smoothSlotF4() {
  return SlotOf<Rows>::PLANES + SlotOf<Rows>::NC + 2;
}
template <class Rows>
__host__ __device__ constexpr size_t smoothSmemBytes(int len) {
  return 16 * ((size_t)SM_THREADS * smoothSlotF4<Rows>() + (size_t)len * 15 + (size_t)2 * SM_PMAX * 11);
}

__device__ __forceinline__ void cpAsync16(void* smem, const void* gmem, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cpAsyncWaitAll() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// 3x3 blocks in shared memory padded to 12 floats (three float4).
__device__ __forceinline__ M3 ldM(const float4* p) {
  const float4 a = p[0], b = p[1], c = p[2];
  return {{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x}};
}
__device__ __forceinline__ void stM(float4* p, const M3& m) {
  p[0] = make_float4(m.a[0], m.a[1], m.a[2], m.a[3]);
  p[1] = make_float4(m.a[4], m.a[5], m.a[6], m.a[7]);
  p[2] = make_float4(m.a[8], 0.f, 0.f, 0.f);
}
__device__ __forceinline__ Sym ldS(const float4* p) {
  const float4 a = p[0], b = p[1];
  return {a.x, a.y, a.z, a.w, b.x, b.y};
}
__device__ __forceinline__ void stS(float4* p, Sym s) {
  p[0] = make_float4(s.xx, s.xy, s.xz, s.yy);
  p[1] = make_float4(s.yz, s.zz, 0.f, 0.f);
}
__device__ __forceinline__ float3 ldV(const float4* p) { return f3(*p); }
__device__ __forceinline__ void stV(float4* p, float3 v) { *p = make_float4(v.x, v.y, v.z, 0.f); }
__device__ __forceinline__ M3 m3Add(const M3& x, const M3& y) {
  M3 o;
#pragma unroll
  for (int q = 0; q < 9; ++q) o.a[q] = x.a[q] + y.a[q];
  return o;
}

// Line row of the node staged in `slot` (row planes, then neighbour unknowns in coupling order,
// own unknown, rhs): diagonal + majorisation, +1 along-line block, lagged rhs (lineRow,
// smooth.wgsl:49-84; smoothLines, newtonMultigrid.ts:676-720).
template <class Rows>
__device__ __forceinline__ void lineRowFromSlot(const float4* slot, int i, int j, const DLevelLayer& ly, int k, int len, int fam,
                                                Sym* Bk, Sym* Ck, float3* rr) {
  constexpr int PL = SlotOf<Rows>::PLANES, NC = SlotOf<Rows>::NC;
  const float* row = reinterpret_cast<const float*>(slot);
  const float3 xn = f3(slot[PL + NC]);
  float3 r = f3(slot[PL + NC + 1]);
  float maj = 0.f;
  Sym D;
  if constexpr (NC == 12) {
    D = {row[0], row[1], row[2], row[3], row[4], row[5]};
    const int qNext = fam == 0 ? 0 : 2, qPrev = fam == 0 ? 1 : 3, qS = fam == 0 ? 8 : 10;
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      if (q == qPrev) continue;
      const int2 o = fineOffset(q);
      if (q == qNext) {
        if (k + 1 < len) *Ck = Sym{row[6 * q + 6], row[6 * q + 7], row[6 * q + 8], row[6 * q + 9], row[6 * q + 10], row[6 * q + 11]};
        continue;
      }
      const int ii = i + o.x, jj = j + o.y;
      if (ii < 0 || jj < 0 || ii >= ly.nx || jj >= ly.ny) continue;
      const float3 xm = f3(slot[PL + q]);
      if (q < 8) {
        const float* b = row + 6 * q + 6;
        r -= Sym{b[0], b[1], b[2], b[3], b[4], b[5]} * xm;
      } else {
        const float sc = row[54 + (q - 8)];
        if (q == qS || q == qS + 1) maj += 1.7320508075688772f * fabsf(sc);
        r -= sc * xm;
      }
    }
  } else {
    D = {row[72], row[73], row[74], row[75], row[76], row[77]};
#pragma unroll
    for (int q = 0; q < 24; ++q) {
      const int o = q >= 12 ? q + 1 : q;
      const int di = o % 5 - 2, dj = o / 5 - 2;
      const int along = fam == 0 ? di : dj, across = fam == 0 ? dj : di;
      if (across == 0 && along == -1) continue;
      const float* b = row + 6 * o;
      const Sym B = {b[0], b[1], b[2], b[3], b[4], b[5]};
      if (across == 0 && along == 1) {
        if (k + 1 < len) *Ck = B;
        continue;
      }
      const int ii = i + di, jj = j + dj;
      if (ii < 0 || jj < 0 || ii >= ly.nx || jj >= ly.ny) continue;
      if (across == 0) maj += symFrob(B);
      r -= B * f3(slot[PL + q]);
    }
  }
  *Bk = D + symId(maj);
  *rr = r + maj * xn;
}

template <class Rows>
__global__ void __launch_bounds__(SM_THREADS) k_smooth(DLevel L, const int4* __restrict__ lines, int first) {
  constexpr int PL = SlotOf<Rows>::PLANES, NC = SlotOf<Rows>::NC, SLOT = smoothSlotF4<Rows>();
  extern __shared__ float4 sm4[];
  const int4 line = lines[first + blockIdx.x];  // (start node, stride, length, family | layer << 1)
  const int n0 = line.x, st = line.y, len = line.z, fam = line.w & 1;
  const DLevelLayer ly = L.layers[line.w >> 1];
  const int tid = threadIdx.x;
  float4* slots = sm4;
  float4* sB = slots + SM_THREADS * SLOT;  // 2 per node
  float4* sC = sB + 2 * len;               // 2 per node
  float4* sR = sC + 2 * len;               // 1 per node
  float4* sG = sR + len;                   // 3 per node
  float4* sH = sG + 3 * len;               // 1 per node (h, then v)
  float4* sV = sH + len;                   // 3 per node (Hs, then V)
  float4* sW = sV + 3 * len;               // 3 per node (He, then W)
  float4* qL = sW + 3 * len;               // 3 per reduced row
  float4* qD = qL + 3 * 2 * SM_PMAX;
  float4* qU = qD + 3 * 2 * SM_PMAX;
  float4* qr = qU + 3 * 2 * SM_PMAX;
  float4* qx = qr + 2 * SM_PMAX;
  const int local0 = n0 - ly.offset;
  const int i0 = local0 % ly.nx, j0 = local0 / ly.nx;

  // ---- phase 1: stage (one cp.async round trip per tile), then build the line rows
  for (int k = tid; k < len; k += SM_THREADS) {
    const int n = n0 + k * st;
    const int i = fam == 0 ? i0 + k : i0, j = fam == 0 ? j0 : j0 + k;
    float4* slot = slots + tid * SLOT;
    const bool fixedNode = L.fixed[n] != 0u;
#pragma unroll
    for (int p = 0; p < PL; ++p) cpAsync16(slot + p, L.op + (size_t)p * L.N + n, true);
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const int2 o = Rows::offset(q);
      const int ii = i + o.x, jj = j + o.y;
      const bool ok = ii >= 0 && jj >= 0 && ii < ly.nx && jj < ly.ny;
      const int m = ok ? ly.offset + jj * ly.nx + ii : n;
      cpAsync16(slot + PL + q, L.X + m, ok);
    }
    cpAsync16(slot + PL + NC, L.X + n, true);
    cpAsync16(slot + PL + NC + 1, L.B + n, true);
    cpAsyncWaitAll();
    Sym Bk = symId(1.f), Ck = symZero();
    float3 r = make_float3(0, 0, 0);
    if (!fixedNode) lineRowFromSlot<Rows>(slot, i, j, ly, k, len, fam, &Bk, &Ck, &r);
    stS(sB + 2 * k, Bk);
    stS(sC + 2 * k, Ck);
    stV(sR + k, r);
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
      const M3 Ak = m3FromSym(ldS(sC + 2 * (k - 1)));
      const M3 Bk = m3FromSym(ldS(sB + 2 * k));
      const M3 Ck = m3FromSym(ldS(sC + 2 * k));
      const M3 Minv = pivotInverse(m3Sub(Bk, m3Mul(Ak, Gp)));
      M3 G = m3Zero(), Cext = m3Zero();
      if (k + 1 < ke)
        G = m3Mul(Minv, Ck);
      else
        Cext = Ck;
      const float3 h = m3Vec(Minv, ldV(sR + k) - m3Vec(Ak, hp));
      const M3 Hs = m3Mul(Minv, m3Neg(m3Mul(Ak, Hsp)));
      const M3 He = m3Mul(Minv, m3Sub(m3Neg(m3Mul(Ak, Hep)), Cext));
      stM(sG + 3 * k, G);
      stV(sH + k, h);
      stM(sV + 3 * k, Hs);
      stM(sW + 3 * k, He);
      Gp = G, hp = h, Hsp = Hs, Hep = He;
    }
    // back substitution inside the chunk: x_k = v_k + V_k x_s + W_k x_e
    float3 vS = make_float3(0, 0, 0), vE = make_float3(0, 0, 0);
    M3 VS = m3Zero(), WS = m3Id(), VE = m3Id(), WE = m3Zero();
    if (mlen >= 3) {
      float3 vn = make_float3(0, 0, 0);
      M3 Vn = m3Zero(), Wn = m3Zero();
      for (int k = ke - 1; k > ks; --k) {
        const M3 G = ldM(sG + 3 * k);
        const float3 v = ldV(sH + k) - m3Vec(G, vn);
        const M3 V = m3Sub(ldM(sV + 3 * k), m3Mul(G, Vn));
        const M3 W = m3Sub(ldM(sW + 3 * k), m3Mul(G, Wn));
        stV(sH + k, v);
        stM(sV + 3 * k, V);
        stM(sW + 3 * k, W);
        if (k == ke - 1) vE = v, VE = V, WE = W;
        vn = v, Vn = V, Wn = W;
      }
      vS = vn, VS = Vn, WS = Wn;
    }
    // reduced equations for x_s (row 2 tid) and x_e (row 2 tid + 1)
    const M3 As = ks > 0 ? m3FromSym(ldS(sC + 2 * (ks - 1))) : m3Zero();
    const M3 Bs = m3FromSym(ldS(sB + 2 * ks)), Cs = m3FromSym(ldS(sC + 2 * ks));
    const M3 Ae = m3FromSym(ldS(sC + 2 * (ke - 1))), Be = m3FromSym(ldS(sB + 2 * ke));
    const M3 Ce = m3FromSym(ldS(sC + 2 * ke));
    stM(qL + 3 * (2 * tid), As);
    stM(qD + 3 * (2 * tid), m3Add(Bs, m3Mul(Cs, VS)));
    stM(qU + 3 * (2 * tid), m3Mul(Cs, WS));
    stV(qr + 2 * tid, ldV(sR + ks) - m3Vec(Cs, vS));
    stM(qL + 3 * (2 * tid + 1), m3Mul(Ae, VE));
    stM(qD + 3 * (2 * tid + 1), m3Add(Be, m3Mul(Ae, WE)));
    stM(qU + 3 * (2 * tid + 1), Ce);
    stV(qr + 2 * tid + 1, ldV(sR + ke) - m3Vec(Ae, vE));
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
      const M3 al = m3Mul(ldM(qL + 3 * q), pivotInverse(ldM(qD + 3 * lo)));
      M3 D = m3Sub(ldM(qD + 3 * q), m3Mul(al, ldM(qU + 3 * lo)));
      float3 r = ldV(qr + q) - m3Vec(al, ldV(qr + lo));
      const M3 Lq = m3Neg(m3Mul(al, ldM(qL + 3 * lo)));
      M3 Uq = m3Zero();
      if (q + stride < Q) {
        const int hi = q + stride;
        const M3 ga = m3Mul(ldM(qU + 3 * q), pivotInverse(ldM(qD + 3 * hi)));
        D = m3Sub(D, m3Mul(ga, ldM(qL + 3 * hi)));
        r = r - m3Vec(ga, ldV(qr + hi));
        Uq = m3Neg(m3Mul(ga, ldM(qU + 3 * hi)));
      }
      stM(qD + 3 * q, D);
      stV(qr + q, r);
      stM(qL + 3 * q, Lq);
      stM(qU + 3 * q, Uq);
    }
    __syncthreads();
    stride *= 2;
  }
  while (stride > 0) {
    const int q = tid;
    if (q < Q && (q + 1) % stride == 0 && (q + 1) % (2 * stride) != 0) {
      float3 r = ldV(qr + q);
      if (q >= stride) r = r - m3Vec(ldM(qL + 3 * q), ldV(qx + q - stride));
      if (q + stride < Q) r = r - m3Vec(ldM(qU + 3 * q), ldV(qx + q + stride));
      stV(qx + q, m3Vec(pivotInverse(ldM(qD + 3 * q)), r));
    }
    __syncthreads();
    stride /= 2;
  }

  // ---- phase 4: recovery and write-back
  if (tid < P) {
    const float3 xs = ldV(qx + 2 * tid), xe = ldV(qx + 2 * tid + 1);
    const int ns = n0 + ks * st, ne = n0 + ke * st;
    if (!L.fixed[ns]) L.X[ns] = make_float4(xs.x, xs.y, xs.z, 0.f);
    if (!L.fixed[ne]) L.X[ne] = make_float4(xe.x, xe.y, xe.z, 0.f);
    for (int k = ks + 1; k < ke; ++k) {
      const int n = n0 + k * st;
      if (L.fixed[n]) continue;
      const float3 x = ldV(sH + k) + m3Vec(ldM(sV + 3 * k), xs) + m3Vec(ldM(sW + 3 * k), xe);
      L.X[n] = make_float4(x.x, x.y, x.z, 0.f);
    }
  }
}

}  // namespace btd
