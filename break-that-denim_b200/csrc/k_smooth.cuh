// Yarn-line smoother: every line of one colour solved exactly as a block-tridiagonal system
// (smoothLines + solvePenta, newtonMultigrid.ts:659-733 / 435-473; smooth.wgsl:49-233).
//
// The line matrices depend on the operator only, which stays fixed over every PCG iteration of a
// Newton iteration, so the solve is split in two kernels:
//
//   k_line_factor  once per operator (after assembly on the fine level, after the Galerkin product on
//                  a coarse one), every line of the level in one launch: line rows (diagonal block
//                  plus the Frobenius majorisation of the +-2 along-line couplings, and the +1 block),
//                  then the partition method - the line cut into P chunks, each chunk's interior
//                  eliminated in terms of the chunk's end unknowns - and odd-even cyclic reduction of
//                  the 2P end equations. It stores every pivot inverse and multiplier a solve needs.
//   k_smooth       every sweep, one CTA per line of one colour: the lagged right-hand side (b minus the
//                  off-line and +-2 couplings at the current iterate, plus the majorisation term), then
//                  the same elimination applied to the right-hand side only - a short chain of 3x3
//                  matrix-vector products - and the write-back.
//
// Both kernels stage with cp.async: a thread's row planes and stencil unknowns land in shared-memory
// columns (element p of thread t at p * SM_THREADS + t, so a warp's accesses fall in distinct banks),
// all copies in flight at once. Lines of one colour are three apart and never read each other's
// unknowns (Jacobi within a colour). Every pivot is regularised by pivotInverse. The lower block of
// row k is the +1 block of row k - 1 (symmetric), as solvePenta takes it.
//
// Factor layout per line (float4 units, from the line's base): node planes p = 0..14 of node k at
// p * len + k - planes 0-2 the pivot inverse Minv (padded 3x3; .y of plane 2 holds the majorisation
// coefficient), 3-5 Minv A (A the lower block), 6-8 G = Minv C, 9-11 V, 12-14 W (interior k:
// x_k = v_k + V_k x_s + W_k x_e); at a chunk's ends planes 0-2 hold the coupling into the chunk. Then
// per cyclic-reduction elimination (level by level) the multipliers al, ga (6 float4), then per
// reduced row Dinv, Dinv L, Dinv U (9 float4).
#pragma once

#include "common.cuh"
#include "k_mg.cuh"

namespace btd {

constexpr int SM_THREADS = 128;
constexpr int SM_PMAX = 32;
constexpr int SM_MAX_LINE = 512;
constexpr int FAC_NODE = 15;
constexpr int FAC_DOWN = 6;
constexpr int FAC_BACK = 9;

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

__host__ __device__ constexpr int linePartitions(int len) {
  return len / 2 < 1 ? 1 : (len / 2 < SM_PMAX ? len / 2 : SM_PMAX);
}
// float4 count of one line's factor region
__host__ __device__ constexpr int lineFactorF4(int len) {
  return FAC_NODE * len + (FAC_DOWN + FAC_BACK) * 2 * linePartitions(len);
}

// Shared memory (bytes) of the two kernels for lines up to len nodes.
template <class Rows>
__host__ __device__ constexpr size_t smoothSmemBytes(int len) {
  // staging columns (row planes, stencil unknowns, own unknown, rhs), factors, r, v, reduced r and x
  return 16 * ((size_t)SM_THREADS * (SlotOf<Rows>::PLANES + SlotOf<Rows>::NC + 2) + (size_t)lineFactorF4(len) + 2 * (size_t)len +
               4 * (size_t)SM_PMAX);
}
template <class Rows>
__host__ __device__ constexpr size_t factorSmemBytes(int len) {
  // staging columns (row planes), line rows B and C, factors, reduced L, D, U
  return 16 * ((size_t)SM_THREADS * SlotOf<Rows>::PLANES + 4 * (size_t)len + (size_t)lineFactorF4(len) + 9 * 2 * (size_t)SM_PMAX);
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

// 3x3 blocks padded to 12 floats (three float4, strided by `s` float4).
__device__ __forceinline__ M3 ldM(const float4* p, int s = 1) {
  const float4 a = p[0], b = p[s], c = p[2 * s];
  return {{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x}};
}
__device__ __forceinline__ void stM(float4* p, const M3& m, int s = 1, float extra = 0.f) {
  p[0] = make_float4(m.a[0], m.a[1], m.a[2], m.a[3]);
  p[s] = make_float4(m.a[4], m.a[5], m.a[6], m.a[7]);
  p[2 * s] = make_float4(m.a[8], extra, 0.f, 0.f);
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

// Float f of a row staged in a shared-memory column (plane f / 4, stride SM_THREADS).
__device__ __forceinline__ float colF(const float4* col, int f) {
  return reinterpret_cast<const float*>(col + (f >> 2) * SM_THREADS)[f & 3];
}
__device__ __forceinline__ Sym colSym(const float4* col, int f) {
  return {colF(col, f), colF(col, f + 1), colF(col, f + 2), colF(col, f + 3), colF(col, f + 4), colF(col, f + 5)};
}

// Coupling q of a row: its float offset in the row, its lattice offset, and its role in a line of
// family fam: 1 the +1 along-line block (into the line matrix), -1 the -1 block (the previous row's
// +1 block, by symmetry), 2 a +-2 along-line coupling (majorised), 0 an off-line coupling.
template <class Rows>
struct Coupling;
template <>
struct Coupling<FineRows> {
  __device__ static int diagF() { return 0; }
  __device__ static bool scalar(int q) { return q >= 8; }
  __device__ static int floatAt(int q) { return q < 8 ? 6 * q + 6 : 54 + (q - 8); }
  __device__ static int role(int q, int fam) {
    if (q == (fam == 0 ? 0 : 2)) return 1;
    if (q == (fam == 0 ? 1 : 3)) return -1;
    if (q == (fam == 0 ? 8 : 10) || q == (fam == 0 ? 9 : 11)) return 2;
    return 0;
  }
};
template <>
struct Coupling<CoarseRows> {
  __device__ static int diagF() { return 72; }
  __device__ static bool scalar(int) { return false; }
  __device__ static int floatAt(int q) { return 6 * (q >= 12 ? q + 1 : q); }
  __device__ static int role(int q, int fam) {
    const int o = q >= 12 ? q + 1 : q;
    const int di = o % 5 - 2, dj = o / 5 - 2;
    const int along = fam == 0 ? di : dj, across = fam == 0 ? dj : di;
    if (across != 0) return 0;
    return along == 1 ? 1 : along == -1 ? -1 : 2;
  }
};

// Line row of node (i, j) from its staged row planes: B = D + maj I, C the +1 block (zero at the
// line's end), maj = sqrt(3) |s| per scalar or ||B||_F per block +-2 along-line coupling with an
// in-bounds neighbour (lineRow, smooth.wgsl:49-84; smoothLines, newtonMultigrid.ts:676-720).
template <class Rows>
__device__ __forceinline__ void lineMatrixFromCol(const float4* col, int i, int j, const DLevelLayer& ly, int k, int len, int fam,
                                                  Sym* Bk, Sym* Ck, float* majOut) {
  using Cp = Coupling<Rows>;
  float maj = 0.f;
  *Ck = symZero();
#pragma unroll
  for (int q = 0; q < SlotOf<Rows>::NC; ++q) {
    const int role = Cp::role(q, fam);
    if (role == 1) {
      if (k + 1 < len) *Ck = Cp::scalar(q) ? symId(colF(col, Cp::floatAt(q))) : colSym(col, Cp::floatAt(q));
      continue;
    }
    if (role != 2) continue;
    const int2 o = Rows::offset(q);
    const int ii = i + o.x, jj = j + o.y;
    if (ii < 0 || jj < 0 || ii >= ly.nx || jj >= ly.ny) continue;
    maj += Cp::scalar(q) ? 1.7320508075688772f * fabsf(colF(col, Cp::floatAt(q))) : symFrob(colSym(col, Cp::floatAt(q)));
  }
  *Bk = colSym(col, Cp::diagF()) + symId(maj);
  *majOut = maj;
}

// Lagged right-hand side of the same row: b - sum over off-line and +-2 couplings of A x, plus
// maj x_n. Staged columns: row planes, then the stencil unknowns in coupling order, own, rhs.
template <class Rows>
__device__ __forceinline__ float3 lineRhsFromCol(const float4* col, int i, int j, const DLevelLayer& ly, int fam, float maj) {
  using Cp = Coupling<Rows>;
  constexpr int PL = SlotOf<Rows>::PLANES, NC = SlotOf<Rows>::NC;
  const float3 xn = f3(col[(PL + NC) * SM_THREADS]);
  float3 r = f3(col[(PL + NC + 1) * SM_THREADS]);
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    const int role = Cp::role(q, fam);
    if (role == 1 || role == -1) continue;
    const int2 o = Rows::offset(q);
    const int ii = i + o.x, jj = j + o.y;
    if (ii < 0 || jj < 0 || ii >= ly.nx || jj >= ly.ny) continue;
    const float3 xm = f3(col[(PL + q) * SM_THREADS]);
    if (Cp::scalar(q))
      r -= colF(col, Cp::floatAt(q)) * xm;
    else
      r -= colSym(col, Cp::floatAt(q)) * xm;
  }
  return r + maj * xn;
}

// Chunk t of a line of len nodes cut into P chunks: [ks, ke].
struct Chunks {
  int P, base, extra;
  __device__ Chunks(int len) : P(linePartitions(len)), base(len / linePartitions(len)), extra(len % linePartitions(len)) {}
  __device__ int start(int t) const { return t * base + min(t, extra); }
  __device__ int size(int t) const { return base + (t < extra ? 1 : 0); }
  __device__ int of(int k) const {
    const int cut = extra * (base + 1);
    return k < cut ? k / (base + 1) : extra + (k - cut) / base;
  }
};

// Elimination slots of cyclic reduction over Q rows: at stride s the rows q with (q + 1) % 2s == 0;
// slot = (rows of the smaller strides) + (q + 1) / 2s - 1.
__device__ __forceinline__ int crSlot(int Q, int stride, int q) {
  int off = 0;
  for (int s = 1; s < stride; s *= 2) off += Q / (2 * s);
  return off + (q + 1) / (2 * stride) - 1;
}

// ------------------------------------------------------------------------------------------ factor

template <class Rows>
__global__ void __launch_bounds__(SM_THREADS) k_line_factor(DLevel L, const int4* __restrict__ lines, const int* __restrict__ base,
                                                            float4* __restrict__ fac) {
  constexpr int PL = SlotOf<Rows>::PLANES;
  extern __shared__ float4 sm4[];
  const int4 line = lines[blockIdx.x];  // (start node, stride, length, family | layer << 1)
  const int n0 = line.x, st = line.y, len = line.z, fam = line.w & 1;
  const DLevelLayer ly = L.layers[line.w >> 1];
  const int tid = threadIdx.x;
  const Chunks ch(len);
  const int P = ch.P, Q = 2 * P;
  float4* cols = sm4;
  float4* sB = cols + SM_THREADS * PL;  // 2 per node
  float4* sC = sB + 2 * len;            // 2 per node
  float4* sF = sC + 2 * len;            // the line's factor region
  float4* qL = sF + lineFactorF4(len);  // 3 per reduced row
  float4* qD = qL + 3 * 2 * SM_PMAX;
  float4* qU = qD + 3 * 2 * SM_PMAX;
  float4* fDown = sF + FAC_NODE * len;
  float4* fBack = fDown + FAC_DOWN * Q;
  const int local0 = n0 - ly.offset;
  const int i0 = local0 % ly.nx, j0 = local0 / ly.nx;

  // ---- line rows
  for (int k = tid; k < len; k += SM_THREADS) {
    const int n = n0 + k * st;
    const int i = fam == 0 ? i0 + k : i0, j = fam == 0 ? j0 : j0 + k;
    float4* col = cols + tid;
#pragma unroll
    for (int p = 0; p < PL; ++p) cpAsync16(col + p * SM_THREADS, L.op + (size_t)p * L.N + n, true);
    cpAsyncWaitAll();
    Sym Bk = symId(1.f), Ck = symZero();
    float maj = 0.f;
    if (!L.fixed[n]) lineMatrixFromCol<Rows>(col, i, j, ly, k, len, fam, &Bk, &Ck, &maj);
    stS(sB + 2 * k, Bk);
    stS(sC + 2 * k, Ck);
    sF[2 * len + k] = make_float4(0.f, maj, 0.f, 0.f);
  }
  __syncthreads();

  // ---- chunk interiors: Minv, Minv A, G; then V, W by the backward pass; reduced rows
  if (tid < P) {
    const int ks = ch.start(tid), mlen = ch.size(tid), ke = ks + mlen - 1;
    M3 Gp = m3Zero(), Hsp = m3Id(), Hep = m3Zero();
    for (int k = ks + 1; k < ke; ++k) {
      const M3 Ak = m3FromSym(ldS(sC + 2 * (k - 1)));
      const M3 Bk = m3FromSym(ldS(sB + 2 * k));
      const M3 Ck = m3FromSym(ldS(sC + 2 * k));
      const M3 Minv = pivotInverse(m3Sub(Bk, m3Mul(Ak, Gp)));
      const M3 QA = m3Mul(Minv, Ak);
      M3 G = m3Zero(), Cext = m3Zero();
      if (k + 1 < ke)
        G = m3Mul(Minv, Ck);
      else
        Cext = Ck;
      const M3 Hs = m3Neg(m3Mul(QA, Hsp));
      const M3 He = m3Sub(m3Neg(m3Mul(QA, Hep)), m3Mul(Minv, Cext));
      const float maj = sF[2 * len + k].y;
      stM(sF + k, Minv, len, maj);
      stM(sF + 3 * len + k, QA, len);
      stM(sF + 6 * len + k, G, len);
      stM(sF + 9 * len + k, Hs, len);
      stM(sF + 12 * len + k, He, len);
      Gp = G, Hsp = Hs, Hep = He;
    }
    M3 VS = m3Zero(), WS = m3Id(), VE = m3Id(), WE = m3Zero();
    if (mlen >= 3) {
      M3 Vn = m3Zero(), Wn = m3Zero();
      for (int k = ke - 1; k > ks; --k) {
        const M3 G = ldM(sF + 6 * len + k, len);
        const M3 V = m3Sub(ldM(sF + 9 * len + k, len), m3Mul(G, Vn));
        const M3 W = m3Sub(ldM(sF + 12 * len + k, len), m3Mul(G, Wn));
        stM(sF + 9 * len + k, V, len);
        stM(sF + 12 * len + k, W, len);
        if (k == ke - 1) VE = V, WE = W;
        Vn = V, Wn = W;
      }
      VS = Vn, WS = Wn;
    }
    const M3 As = ks > 0 ? m3FromSym(ldS(sC + 2 * (ks - 1))) : m3Zero();
    const M3 Bs = m3FromSym(ldS(sB + 2 * ks)), Cs = m3FromSym(ldS(sC + 2 * ks));
    const M3 Ae = m3FromSym(ldS(sC + 2 * (ke - 1))), Be = m3FromSym(ldS(sB + 2 * ke));
    const M3 Ce = m3FromSym(ldS(sC + 2 * ke));
    // couplings the reduced right-hand sides need: Cs at the chunk's start, Ae at its end
    const float majS = sF[2 * len + ks].y, majE = sF[2 * len + ke].y;
    stM(sF + ks, Cs, len, majS);
    if (ke != ks) stM(sF + ke, Ae, len, majE);
    stM(qL + 3 * (2 * tid), As);
    stM(qD + 3 * (2 * tid), m3Add(Bs, m3Mul(Cs, VS)));
    stM(qU + 3 * (2 * tid), m3Mul(Cs, WS));
    stM(qL + 3 * (2 * tid + 1), m3Mul(Ae, VE));
    stM(qD + 3 * (2 * tid + 1), m3Add(Be, m3Mul(Ae, WE)));
    stM(qU + 3 * (2 * tid + 1), Ce);
  }
  __syncthreads();

  // ---- odd-even cyclic reduction of the 2P reduced rows. At stride s the rows with
  // (q + 1) % 2s == 0 eliminate their neighbours q -+ s, which no longer change.
  int stride = 1;
  while (2 * stride <= Q) {
    const int q = tid;
    if (q < Q && (q + 1) % (2 * stride) == 0) {
      const int lo = q - stride;
      const M3 al = m3Mul(ldM(qL + 3 * q), pivotInverse(ldM(qD + 3 * lo)));
      M3 D = m3Sub(ldM(qD + 3 * q), m3Mul(al, ldM(qU + 3 * lo)));
      const M3 Lq = m3Neg(m3Mul(al, ldM(qL + 3 * lo)));
      M3 Uq = m3Zero(), ga = m3Zero();
      if (q + stride < Q) {
        const int hi = q + stride;
        ga = m3Mul(ldM(qU + 3 * q), pivotInverse(ldM(qD + 3 * hi)));
        D = m3Sub(D, m3Mul(ga, ldM(qL + 3 * hi)));
        Uq = m3Neg(m3Mul(ga, ldM(qU + 3 * hi)));
      }
      const int slot = crSlot(Q, stride, q);
      stM(fDown + FAC_DOWN * slot, al);
      stM(fDown + FAC_DOWN * slot + 3, ga);
      stM(qD + 3 * q, D);
      stM(qL + 3 * q, Lq);
      stM(qU + 3 * q, Uq);
    }
    __syncthreads();
    stride *= 2;
  }
  while (stride > 0) {
    const int q = tid;
    if (q < Q && (q + 1) % stride == 0 && (q + 1) % (2 * stride) != 0) {
      const M3 Dinv = pivotInverse(ldM(qD + 3 * q));
      const M3 DL = q >= stride ? m3Mul(Dinv, ldM(qL + 3 * q)) : m3Zero();
      const M3 DU = q + stride < Q ? m3Mul(Dinv, ldM(qU + 3 * q)) : m3Zero();
      stM(fBack + FAC_BACK * q, Dinv);
      stM(fBack + FAC_BACK * q + 3, DL);
      stM(fBack + FAC_BACK * q + 6, DU);
    }
    __syncthreads();
    stride /= 2;
  }

  // ---- the region out, coalesced
  float4* out = fac + base[blockIdx.x];
  const int total = lineFactorF4(len);
  for (int e = tid; e < total; e += SM_THREADS) out[e] = sF[e];
}

// ------------------------------------------------------------------------------------------ sweep

template <class Rows>
__global__ void __launch_bounds__(SM_THREADS) k_smooth(DLevel L, const int4* __restrict__ lines, const int* __restrict__ base,
                                                       const float4* __restrict__ fac, int first) {
  constexpr int PL = SlotOf<Rows>::PLANES, NC = SlotOf<Rows>::NC, SLOT = PL + NC + 2;
  extern __shared__ float4 sm4[];
  const int li = first + blockIdx.x;
  const int4 line = lines[li];
  const int n0 = line.x, st = line.y, len = line.z, fam = line.w & 1;
  const DLevelLayer ly = L.layers[line.w >> 1];
  const int tid = threadIdx.x;
  const Chunks ch(len);
  const int P = ch.P, Q = 2 * P;
  const int total = lineFactorF4(len);
  float4* cols = sm4;
  float4* sF = cols + SM_THREADS * SLOT;
  float4* sR = sF + total;  // r, then the reduced solution's recovery reads it
  float4* sV = sR + len;    // h, then v
  float4* qr = sV + len;
  float4* qx = qr + 2 * SM_PMAX;
  const float4* fDown = sF + FAC_NODE * len;
  const float4* fBack = fDown + FAC_DOWN * Q;
  const int local0 = n0 - ly.offset;
  const int i0 = local0 % ly.nx, j0 = local0 / ly.nx;

  // ---- stage the factors and, tile by tile, each node's row planes and stencil unknowns; build r
  const float4* src = fac + base[li];
  for (int e = tid; e < total; e += SM_THREADS) cpAsync16(sF + e, src + e, true);
  for (int k = tid; k < len; k += SM_THREADS) {
    const int n = n0 + k * st;
    const int i = fam == 0 ? i0 + k : i0, j = fam == 0 ? j0 : j0 + k;
    float4* col = cols + tid;
#pragma unroll
    for (int p = 0; p < PL; ++p) cpAsync16(col + p * SM_THREADS, L.op + (size_t)p * L.N + n, true);
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const int2 o = Rows::offset(q);
      const int ii = i + o.x, jj = j + o.y;
      const bool ok = ii >= 0 && jj >= 0 && ii < ly.nx && jj < ly.ny;
      cpAsync16(col + (PL + q) * SM_THREADS, L.X + (ok ? ly.offset + jj * ly.nx + ii : n), ok);
    }
    cpAsync16(col + (PL + NC) * SM_THREADS, L.X + n, true);
    cpAsync16(col + (PL + NC + 1) * SM_THREADS, L.B + n, true);
    cpAsyncWaitAll();
    float3 r = make_float3(0, 0, 0);
    if (!L.fixed[n]) r = lineRhsFromCol<Rows>(col, i, j, ly, fam, sF[2 * len + k].y);
    stV(sR + k, r);
  }
  cpAsyncWaitAll();
  __syncthreads();

  // ---- chunk interiors: h_k = Minv_k r_k - (Minv A)_k h_{k-1}, v_k = h_k - G_k v_{k+1}; reduced r
  if (tid < P) {
    const int ks = ch.start(tid), mlen = ch.size(tid), ke = ks + mlen - 1;
    float3 h = make_float3(0, 0, 0);
    for (int k = ks + 1; k < ke; ++k) {
      h = m3Vec(ldM(sF + k, len), ldV(sR + k)) - m3Vec(ldM(sF + 3 * len + k, len), h);
      stV(sV + k, h);
    }
    float3 v = make_float3(0, 0, 0), vS = v, vE = v;
    for (int k = ke - 1; k > ks; --k) {
      v = ldV(sV + k) - m3Vec(ldM(sF + 6 * len + k, len), v);
      stV(sV + k, v);
      if (k == ke - 1) vE = v;
    }
    if (mlen >= 3) vS = v;
    stV(qr + 2 * tid, ldV(sR + ks) - m3Vec(ldM(sF + ks, len), vS));
    stV(qr + 2 * tid + 1, ldV(sR + ke) - m3Vec(ldM(sF + ke, len), vE));
  }
  __syncthreads();

  // ---- cyclic reduction of the reduced right-hand sides, then the reduced solution
  int stride = 1;
  while (2 * stride <= Q) {
    const int q = tid;
    if (q < Q && (q + 1) % (2 * stride) == 0) {
      const float4* f = fDown + FAC_DOWN * crSlot(Q, stride, q);
      float3 r = ldV(qr + q) - m3Vec(ldM(f), ldV(qr + q - stride));
      if (q + stride < Q) r = r - m3Vec(ldM(f + 3), ldV(qr + q + stride));
      stV(qr + q, r);
    }
    __syncthreads();
    stride *= 2;
  }
  while (stride > 0) {
    const int q = tid;
    if (q < Q && (q + 1) % stride == 0 && (q + 1) % (2 * stride) != 0) {
      const float4* f = fBack + FAC_BACK * q;
      float3 x = m3Vec(ldM(f), ldV(qr + q));
      if (q >= stride) x = x - m3Vec(ldM(f + 3), ldV(qx + q - stride));
      if (q + stride < Q) x = x - m3Vec(ldM(f + 6), ldV(qx + q + stride));
      stV(qx + q, x);
    }
    __syncthreads();
    stride /= 2;
  }

  // ---- recovery and write-back, every node in parallel
  for (int k = tid; k < len; k += SM_THREADS) {
    const int n = n0 + k * st;
    if (L.fixed[n]) continue;
    const int t = ch.of(k);
    const int ks = ch.start(t), ke = ks + ch.size(t) - 1;
    const float3 xs = ldV(qx + 2 * t), xe = ldV(qx + 2 * t + 1);
    float3 x;
    if (k == ks)
      x = xs;
    else if (k == ke)
      x = xe;
    else
      x = ldV(sV + k) + m3Vec(ldM(sF + 9 * len + k, len), xs) + m3Vec(ldM(sF + 12 * len + k, len), xe);
    L.X[n] = make_float4(x.x, x.y, x.z, 0.f);
  }
}

}  // namespace btd
