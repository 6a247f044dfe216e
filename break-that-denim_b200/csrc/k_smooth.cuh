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
//                  eliminated in terms of the chunk's end unknowns - and the inverse of the system
//                  of the 2P end equations (block LU, then one column per thread). It stores every
//                  pivot inverse and multiplier a solve needs, and a line-contiguous copy of each
//                  row's right-hand-side couplings.
//   k_smooth       every sweep, one CTA per line of one colour: the lagged right-hand side (b minus the
//                  off-line and +-2 couplings at the current iterate, plus the majorisation term), then
//                  the same elimination applied to the right-hand side only - a short chain of 3x3
//                  matrix-vector products per chunk, one dense product for the end unknowns - and the
//                  write-back.
//
// A sweep stages with cp.async, all copies of a tile in flight at once: the line's factors, its rows'
// coupling copies (contiguous along the line whatever the family, so every 32-byte sector fetched is
// used) and five columns of unknowns - the line itself and two lines either side - from which every
// stencil neighbour is read. Lines of one colour are three apart and never read each other's
// unknowns (Jacobi within a colour). Every pivot is regularised by pivotInverse. The lower block of
// row k is the +1 block of row k - 1 (symmetric), as solvePenta takes it.
//
// Factor region of a line (float4 units, from the line's base):
//   node planes p = 0..14, node k at p * NP + (its padded position, see chunkSlot): 0-2 the pivot
//     inverse Minv (padded 3x3; .y and .z of plane 2 hold the majorisation coefficient and whether
//     the row is fixed), 3-5 Minv A (A the lower block), 6-8 G = Minv C, 9-11 V, 12-14 W (interior k:
//     x_k = v_k + V_k x_s + W_k x_e); at a chunk's ends planes 0-2 hold the coupling into the chunk;
//   the inverse of the 2P x 2P block-tridiagonal system of the chunks' end unknowns, dense (see
//     denseStride);
//   coupling planes p = 0..RC-1 of node k at p * len + k: the row's couplings other than the +-1
//     along-line blocks, in coupling order (6 floats a block, 1 a scalar), zero where the neighbour is
//     outside the layer or the row is fixed, then the rhs scale (0 on a fixed row, else 1) and the
//     majorisation coefficient.
#pragma once

#include "common.cuh"
#include "k_mg.cuh"

namespace btd {

constexpr int SM_THREADS = 128;
constexpr int SM_PMAX = 16;
constexpr int SM_MAX_LINE = 512;
constexpr int FAC_NODE = 15;

template <class Rows>
struct SlotOf;
template <>
struct SlotOf<FineRows> {
  // 6 off-line blocks and 4 scalars (40 floats), rhs scale, majorisation
  static constexpr int PLANES = FINE_PLANES, NC = 12, COEF_FLOATS = 40, RC = 11;
};
template <>
struct SlotOf<CoarseRows> {
  // 22 blocks (132 floats), rhs scale, majorisation
  static constexpr int PLANES = COARSE_PLANES, NC = 24, COEF_FLOATS = 132, RC = 34;
};

__host__ __device__ constexpr int linePartitions(int len) {
  return len / 2 < 1 ? 1 : (len / 2 < SM_PMAX ? len / 2 : SM_PMAX);
}
// Per-node arrays of the solve keep each chunk in a slot of an odd number S >= its size of float4,
// node k of chunk t at t S + (k - start of t): the chunk threads, one per chunk, then step through
// distinct shared-memory banks. A line's node arrays hold P S entries.
__host__ __device__ constexpr int chunkSlot(int len) { return (len / linePartitions(len) + 1) | 1; }
__host__ __device__ constexpr int lineNodesPadded(int len) { return linePartitions(len) * chunkSlot(len); }
// The reduced system's inverse: 3Q x 3Q floats, column j at j (3Q + 1) (an odd stride: the threads
// that build one column each, and those that read one row each, fall in distinct banks).
__host__ __device__ constexpr int denseStride(int Q) { return 3 * Q + 1; }
__host__ __device__ constexpr int denseF4(int Q) { return (3 * Q * denseStride(Q) + 3) / 4; }
// float4 count of the factors of a line (node planes and the reduced system's inverse)
__host__ __device__ constexpr int lineSolveF4(int len) {
  return FAC_NODE * lineNodesPadded(len) + denseF4(2 * linePartitions(len));
}
template <class Rows>
__host__ __device__ constexpr int lineFactorF4(int len) {
  return lineSolveF4(len) + SlotOf<Rows>::RC * len;
}

// Shared memory (bytes) of a sweep over lines up to len nodes staged in tiles of T nodes: factors,
// coupling planes of a tile, five columns of unknowns (tile plus two either side), b of a tile, r, v,
// reduced r and x.
template <class Rows>
__host__ __device__ constexpr size_t smoothSmemBytes(int len, int T) {
  return 16 * ((size_t)lineSolveF4(len) + (size_t)SlotOf<Rows>::RC * T + 5 * ((size_t)T + 4) + (size_t)T +
               2 * (size_t)lineNodesPadded(len) + 4 * (size_t)SM_PMAX);
}
// Tile of a level whose lines reach len nodes: the whole line when it fits, else 256 or 128 nodes.
template <class Rows>
__host__ inline int smoothTile(int len) {
  constexpr size_t cap = 226 * 1024;  // the opt-in 227 KB less the kernel's static shared memory
  if (smoothSmemBytes<Rows>(len, len) <= cap) return len;
  if (len > 256 && smoothSmemBytes<Rows>(len, 256) <= cap) return 256;
  return 128;
}
template <class Rows>
__host__ __device__ constexpr size_t factorSmemBytes(int len) {
  // staging columns (row planes), line rows B and C, node planes and reduced system, reduced L, D, U
  return 16 * ((size_t)SM_THREADS * SlotOf<Rows>::PLANES + 4 * (size_t)len + (size_t)lineSolveF4(len) + 9 * 2 * (size_t)SM_PMAX);
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

// Bulk copies (the TMA engine, no tensor map, no multicast) into this CTA's shared memory, completed
// on an mbarrier: a few large requests instead of one per 16 bytes, which keeps an SM's L2 traffic
// near its bandwidth.
__device__ __forceinline__ unsigned smemAddr(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbarInit(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbarExpectTx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulkCopy(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smemAddr(dst)),
               "l"(src), "r"(bytes), "r"(smemAddr(bar))
               : "memory");
}
// Generic-proxy accesses to shared memory before this point are ordered before later bulk copies.
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smemAddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of an mbarrier (each try suspends the thread for a while). If the
// first bound runs out, the error flag is raised and the wait gets a second bound of its own, so that
// copies still in flight land before the CTA goes on and exits; either way the kernel goes on (with
// garbage, flagged) instead of hanging. The copies waited on are this CTA's own bulk copies from
// global memory (tens of KB, microseconds), so the second bound (2^20 tries, seconds) runs out only
// when the expected transaction bytes exceed the bytes issued - a bug, with no copy left in flight.
// The first bound is a device variable so that a test can make it run out (btd_set_wait_bound): with
// zero tries the flag is raised at once and the copies land under the second bound.
constexpr int MBAR_TRIES = 1 << 20;
constexpr uint32_t ERR_COPY_TIMEOUT = 1u;
__device__ int g_mbarFirstTries = MBAR_TRIES;
__device__ __forceinline__ void mbarWaitBounded(uint64_t* bar, unsigned parity, uint32_t* err) {
  const int first = g_mbarFirstTries;
  for (int i = 0; i < first; ++i)
    if (mbarTryWait(bar, parity)) return;
  if (err) atomicOr(err, ERR_COPY_TIMEOUT);
  for (int i = 0; i < MBAR_TRIES; ++i)
    if (mbarTryWait(bar, parity)) return;
}

// 3x3 blocks padded to 12 floats (three float4, strided by `s` float4).
__device__ __forceinline__ M3 ldM(const float4* p, int s = 1) {
  const float4 a = p[0], b = p[s], c = p[2 * s];
  return {{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x}};
}
__device__ __forceinline__ void stM(float4* p, const M3& m, int s = 1, float extra = 0.f, float extra2 = 0.f) {
  p[0] = make_float4(m.a[0], m.a[1], m.a[2], m.a[3]);
  p[s] = make_float4(m.a[4], m.a[5], m.a[6], m.a[7]);
  p[2 * s] = make_float4(m.a[8], extra, extra2, 0.f);
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

// Float f of planes strided by `stride` float4 (plane f / 4).
// Float f of a row staged as float4 planes (plane f / 4, stride `stride`): the whole float4 is loaded
// (one conflict-free 128-bit access a lane; the loads of a plane's other floats are the same load),
// where a 32-bit load of one float of each lane's float4 would meet a 4-way bank conflict.
__device__ __forceinline__ float colF(const float4* col, int f, int stride = SM_THREADS) {
  const float4 v = col[(f >> 2) * stride];
  const int c = f & 3;
  return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}
__device__ __forceinline__ Sym colSym(const float4* col, int f, int stride = SM_THREADS) {
  return {colF(col, f, stride), colF(col, f + 1, stride), colF(col, f + 2, stride),
          colF(col, f + 3, stride), colF(col, f + 4, stride), colF(col, f + 5, stride)};
}
__device__ __forceinline__ void putF(float4* col, int f, int stride, float v) {
  reinterpret_cast<float*>(col + (f >> 2) * stride)[f & 3] = v;
}

// Coupling q of a row: its float offset in the row, and its role in a line of family fam: 1 the +1
// along-line block (into the line matrix), -1 the -1 block (the previous row's +1 block, by
// symmetry), 2 a +-2 along-line coupling (majorised), 0 an off-line coupling.
template <class Rows>
struct Coupling;
template <>
struct Coupling<FineRows> {
  __device__ static constexpr int diagF() { return 0; }
  __device__ static constexpr bool scalar(int q) { return q >= 8; }
  __device__ static constexpr int width(int q) { return q >= 8 ? 1 : 6; }
  __device__ static constexpr int floatAt(int q) { return q < 8 ? 6 * q + 6 : 54 + (q - 8); }
  __device__ static constexpr int role(int q, int fam) {
    return q == (fam == 0 ? 0 : 2)                                 ? 1
           : q == (fam == 0 ? 1 : 3)                               ? -1
           : (q == (fam == 0 ? 8 : 10) || q == (fam == 0 ? 9 : 11)) ? 2
                                                                    : 0;
  }
};
template <>
struct Coupling<CoarseRows> {
  __device__ static constexpr int diagF() { return 72; }
  __device__ static constexpr bool scalar(int) { return false; }
  __device__ static constexpr int width(int) { return 6; }
  __device__ static constexpr int floatAt(int q) { return 6 * (q >= 12 ? q + 1 : q); }
  __device__ static constexpr int role(int q, int fam) {
    return (fam == 0 ? (q >= 12 ? q + 1 : q) / 5 - 2 : (q >= 12 ? q + 1 : q) % 5 - 2) != 0 ? 0
           : (fam == 0 ? (q >= 12 ? q + 1 : q) % 5 - 2 : (q >= 12 ? q + 1 : q) / 5 - 2) == 1  ? 1
           : (fam == 0 ? (q >= 12 ? q + 1 : q) % 5 - 2 : (q >= 12 ? q + 1 : q) / 5 - 2) == -1 ? -1
                                                                                              : 2;
  }
};

// Chunk t of a line of len nodes cut into P chunks: [ks, ke]; idx is a node's padded position.
// The chunk of node k is found by multiplying with rounded reciprocals: for k < 2^12, (k + 1/2) / m
// lies at least 1/(2m) from an integer and the rounding error of the product is below 1e-4, so the
// truncation is exact (an integer division would cost a dependent instruction sequence per node).
struct Chunks {
  int P, base, extra, S;
  float rb1, rb;  // 1 / (base + 1), 1 / base
  __host__ __device__ Chunks(int len) : Chunks(linePartitions(len), len / linePartitions(len), len % linePartitions(len), chunkSlot(len)) {}
  __host__ __device__ Chunks(int P_, int base_, int extra_, int S_)
      : P(P_), base(base_), extra(extra_), S(S_), rb1(1.0f / (float)(base_ + 1)), rb(1.0f / (float)base_) {}
  __host__ __device__ Chunks() : Chunks(1, 1, 0, 1) {}
  __device__ int start(int t) const { return t * base + min(t, extra); }
  __device__ int size(int t) const { return base + (t < extra ? 1 : 0); }
  __device__ int of(int k) const {
    const int cut = extra * (base + 1);
    return k < cut ? (int)(((float)k + 0.5f) * rb1) : extra + (int)(((float)(k - cut) + 0.5f) * rb);
  }
  __device__ int idx(int k) const {
    const int t = of(k);
    return t * S + (k - start(t));
  }
};

// ------------------------------------------------------------------------------------------ factor

// Line row of node (i, j) from its staged row planes: B = D + maj I, C the +1 block (zero at the
// line's end), maj = sqrt(3) |s| per scalar or ||B||_F per block +-2 along-line coupling with an
// in-bounds neighbour (lineRow, smooth.wgsl:49-84; smoothLines, newtonMultigrid.ts:676-720); and the
// row's coupling copy written to `cp` (planes strided by cstride).
template <class Rows>
__device__ __forceinline__ void lineRowFromCol(const float4* col, int i, int j, const DLevelLayer& ly, int k, int len, int fam,
                                               bool fixedNode, Sym* Bk, Sym* Ck, float* majOut, float4* cp, int cstride) {
  using Cp = Coupling<Rows>;
  constexpr int CF = SlotOf<Rows>::COEF_FLOATS;
  float maj = 0.f;
  *Ck = symZero();
  int pos = 0;
#pragma unroll
  for (int q = 0; q < SlotOf<Rows>::NC; ++q) {
    const int role = Cp::role(q, fam);
    const int2 o = Rows::offset(q);
    const int ii = i + o.x, jj = j + o.y;
    const bool in = !fixedNode && ii >= 0 && jj >= 0 && ii < ly.nx && jj < ly.ny;
    if (role == 1) {
      if (!fixedNode && k + 1 < len) *Ck = Cp::scalar(q) ? symId(colF(col, Cp::floatAt(q))) : colSym(col, Cp::floatAt(q));
      continue;
    }
    if (role == -1) continue;
#pragma unroll
    for (int w = 0; w < Cp::width(q); ++w) putF(cp, pos + w, cstride, in ? colF(col, Cp::floatAt(q) + w) : 0.f);
    pos += Cp::width(q);
    if (role == 2 && in)
      maj += Cp::scalar(q) ? 1.7320508075688772f * fabsf(colF(col, Cp::floatAt(q))) : symFrob(colSym(col, Cp::floatAt(q)));
  }
  putF(cp, CF, cstride, fixedNode ? 0.f : 1.f);
  putF(cp, CF + 1, cstride, maj);
#pragma unroll
  for (int w = CF + 2; w < 4 * SlotOf<Rows>::RC; ++w) putF(cp, w, cstride, 0.f);
  *Bk = fixedNode ? symId(1.f) : colSym(col, Cp::diagF()) + symId(maj);
  *majOut = maj;
}

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
  const int P = ch.P, Q = 2 * P, NP = lineNodesPadded(len), S = ch.S;
  float4* cols = sm4;
  float4* sB = cols + SM_THREADS * PL;  // 2 per node
  float4* sC = sB + 2 * len;            // 2 per node
  float4* sF = sC + 2 * len;            // node planes and reduced system
  float4* qL = sF + lineSolveF4(len);   // 3 per reduced row
  float4* qD = qL + 3 * 2 * SM_PMAX;
  float4* qU = qD + 3 * 2 * SM_PMAX;
  float* dense = reinterpret_cast<float*>(sF + FAC_NODE * NP);
  float4* out = fac + base[blockIdx.x];
  const int local0 = n0 - ly.offset;
  const int i0 = local0 % ly.nx, j0 = local0 / ly.nx;

  // ---- line rows and the coupling copy
  for (int k = tid; k < len; k += SM_THREADS) {
    const int n = n0 + k * st;
    const int i = fam == 0 ? i0 + k : i0, j = fam == 0 ? j0 : j0 + k;
    float4* col = cols + tid;
#pragma unroll
    for (int p = 0; p < PL; ++p) cpAsync16(col + p * SM_THREADS, L.op + (size_t)p * L.N + n, true);
    cpAsyncWaitAll();
    Sym Bk, Ck;
    float maj;
    if (fam == 0)
      lineRowFromCol<Rows>(col, i, j, ly, k, len, 0, L.fixed[n] != 0u, &Bk, &Ck, &maj, out + lineSolveF4(len) + k, len);
    else
      lineRowFromCol<Rows>(col, i, j, ly, k, len, 1, L.fixed[n] != 0u, &Bk, &Ck, &maj, out + lineSolveF4(len) + k, len);
    stS(sB + 2 * k, Bk);
    stS(sC + 2 * k, Ck);
    sF[2 * NP + ch.idx(k)] = make_float4(0.f, maj, L.fixed[n] != 0u ? 1.f : 0.f, 0.f);
  }
  __syncthreads();

  // ---- chunk interiors: Minv, Minv A, G; then V, W by the backward pass; reduced rows. Node k of
  // chunk t sits at t S + (k - ks) in the node planes.
  if (tid < P) {
    const int ks = ch.start(tid), mlen = ch.size(tid), ke = ks + mlen - 1;
    float4* nd = sF + tid * S - ks;  // node k's entry of plane p: nd[p * NP + k]
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
      const float4 mf = nd[2 * NP + k];
      stM(nd + k, Minv, NP, mf.y, mf.z);
      stM(nd + 3 * NP + k, QA, NP);
      stM(nd + 6 * NP + k, G, NP);
      stM(nd + 9 * NP + k, Hs, NP);
      stM(nd + 12 * NP + k, He, NP);
      Gp = G, Hsp = Hs, Hep = He;
    }
    M3 VS = m3Zero(), WS = m3Id(), VE = m3Id(), WE = m3Zero();
    if (mlen >= 3) {
      M3 Vn = m3Zero(), Wn = m3Zero();
      for (int k = ke - 1; k > ks; --k) {
        const M3 G = ldM(nd + 6 * NP + k, NP);
        const M3 V = m3Sub(ldM(nd + 9 * NP + k, NP), m3Mul(G, Vn));
        const M3 W = m3Sub(ldM(nd + 12 * NP + k, NP), m3Mul(G, Wn));
        stM(nd + 9 * NP + k, V, NP);
        stM(nd + 12 * NP + k, W, NP);
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
    const float4 mS = nd[2 * NP + ks], mE = nd[2 * NP + ke];
    stM(nd + ks, Cs, NP, mS.y, mS.z);
    stM(nd + ke, Ae, NP, mE.y, mE.z);
    stM(qL + 3 * (2 * tid), As);
    stM(qD + 3 * (2 * tid), m3Add(Bs, m3Mul(Cs, VS)));
    stM(qU + 3 * (2 * tid), m3Mul(Cs, WS));
    stM(qL + 3 * (2 * tid + 1), m3Mul(Ae, VE));
    stM(qD + 3 * (2 * tid + 1), m3Add(Be, m3Mul(Ae, WE)));
    stM(qU + 3 * (2 * tid + 1), Ce);
  }
  __syncthreads();

  // ---- the reduced system's inverse. Block LU by one thread (rows q of L, D, U: pivot inverses
  // Dinv_q of D_q - L_q G_{q-1}, G_q = Dinv_q U_q, in place of D and U), then column j of the inverse
  // by thread j: forward y_q = Dinv_q (e_j - L_q y_{q-1}), back x_q = y_q - G_q x_{q+1}, in place.
  if (tid == 0) {
    M3 G = m3Zero();
    for (int q = 0; q < Q; ++q) {
      const M3 Lq = ldM(qL + 3 * q);
      const M3 Dinv = pivotInverse(m3Sub(ldM(qD + 3 * q), m3Mul(Lq, G)));
      G = m3Mul(Dinv, ldM(qU + 3 * q));
      stM(qD + 3 * q, Dinv);
      stM(qU + 3 * q, G);
    }
  }
  __syncthreads();
  const int QS = denseStride(Q);
  for (int j = tid; j < 3 * Q; j += SM_THREADS) {
    float* col = dense + j * QS;
    float3 y = make_float3(0, 0, 0);
    for (int q = 0; q < Q; ++q) {
      float3 b = make_float3(q == j / 3 && j % 3 == 0 ? 1.f : 0.f, q == j / 3 && j % 3 == 1 ? 1.f : 0.f,
                             q == j / 3 && j % 3 == 2 ? 1.f : 0.f);
      y = m3Vec(ldM(qD + 3 * q), b - m3Vec(ldM(qL + 3 * q), y));
      col[3 * q] = y.x, col[3 * q + 1] = y.y, col[3 * q + 2] = y.z;
    }
    float3 x = y;
    for (int q = Q - 2; q >= 0; --q) {
      x = make_float3(col[3 * q], col[3 * q + 1], col[3 * q + 2]) - m3Vec(ldM(qU + 3 * q), x);
      col[3 * q] = x.x, col[3 * q + 1] = x.y, col[3 * q + 2] = x.z;
    }
  }
  __syncthreads();

  // ---- node planes and reduced system out, coalesced
  const int total = lineSolveF4(len);
  for (int e = tid; e < total; e += SM_THREADS) out[e] = sF[e];
}

// ------------------------------------------------------------------------------------------ sweep

// The lines of one colour launch: either each line from the line table (scenes of several layers),
// or, in a single layer, line b at start0 + b startStep with its factors at base0 + b baseStep.
struct LineGeom {
  int first;  // table index of block 0
  int table;
  int start0, startStep, stride, len, base0, baseStep;
  int across0;  // position of line 0 across its family (line b at across0 + 3 b)
  int P, chunkBase, chunkExtra, S;  // the lines' chunks (Chunks(len))
  DLevelLayer ly;
};

// One CTA per line, blockDim.x threads (a multiple of 32, up to SM_SWEEP_THREADS).
constexpr int SM_SWEEP_THREADS = 256;
// At least 128: the dense end-unknown product has 3Q <= 96 outputs, one a thread, in one round.
__host__ inline int sweepThreads(int maxLine) { return std::min(SM_SWEEP_THREADS, std::max(128, (maxLine + 31) / 32 * 32)); }

// One line of a sweep, its geometry resolved.
struct LineAt {
  int n0, st, len, fb, across0;
  DLevelLayer ly;
  Chunks ch;
};
__device__ __forceinline__ LineAt lineAt(const LineGeom& g, int b) {
  return LineAt{g.start0 + b * g.startStep, g.stride,  g.len, g.base0 + b * g.baseStep, g.across0 + 3 * b,
                g.ly,                       Chunks(g.P, g.chunkBase, g.chunkExtra, g.S)};
}

// Thread 0: the first tile's bulk copies of a line (its factors and coupling planes), completing
// the mbarrier's current phase.
template <class Rows>
__device__ __forceinline__ void issueLineCopies(const LineAt& a, const float4* __restrict__ fac, int T, float4* sm4, uint64_t* bar) {
  constexpr int RC = SlotOf<Rows>::RC;
  const int Q = 2 * a.ch.P, NP = a.ch.P * a.ch.S;
  const int solveF4 = FAC_NODE * NP + denseF4(Q);
  const int tn = min(T, a.len);
  const float4* src = fac + a.fb;
  float4* sCp = sm4 + solveF4;
  fenceProxyAsync();
  const unsigned coefBytes = 16u * RC * tn;
  mbarExpectTx(bar, coefBytes + 16u * solveF4);
  bulkCopy(sm4, src, 16u * solveF4, bar);
  if (tn == a.len && a.len == T)
    bulkCopy(sCp, src + solveF4, coefBytes, bar);
  else
    for (int p = 0; p < RC; ++p) bulkCopy(sCp + p * T, src + solveF4 + p * a.len, 16u * tn, bar);
}

// Solve line `a` in place of its unknowns. The mbarrier `bar` is initialised; `phase` is the parity
// its next phase completes with; with `prefetched` thread 0 already issued the first tile's copies.
template <class Rows, int FAM>
__device__ __forceinline__ void sweepLine(const DLevel& L, const LineAt& a, const float4* __restrict__ fac, int T, uint32_t* err,
                                          float4* sm4, uint64_t* bar, unsigned& phase, bool prefetched) {
  using Cp = Coupling<Rows>;
  constexpr int RC = SlotOf<Rows>::RC, CF = SlotOf<Rows>::COEF_FLOATS;
  const int n0 = a.n0, st = a.st, len = a.len, across0 = a.across0;
  const DLevelLayer ly = a.ly;
  const Chunks ch = a.ch;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int P = ch.P, Q = 2 * P, S = ch.S, NP = P * S;
  const int QS = denseStride(Q);
  const int solveF4 = FAC_NODE * NP + denseF4(Q);
  const int TX = T + 4;
  float4* sF = sm4;
  float4* sCp = sF + solveF4;  // coupling planes of the tile, plane stride T
  float4* sX = sCp + RC * T;   // 5 columns of TX unknowns
  float4* sBt = sX + 5 * TX;   // b of the tile
  float4* sR = sBt + T;        // r (padded node positions)
  float4* sV = sR + NP;        // h, then v
  float4* qr = sV + NP;
  float4* qx = qr + 2 * SM_PMAX;
  const float* dense = reinterpret_cast<const float*>(sF + FAC_NODE * NP);
  const float4* src = fac + a.fb;
  // lines across the family, and the node step to the neighbouring line
  const int nAcross = FAM == 0 ? ly.ny : ly.nx, acrossStep = FAM == 0 ? ly.nx : 1;

  // ---- stage: the factors and, tile by tile, the coupling planes by bulk copies (thread 0), the
  // unknowns and b by cp.async (strided along a v-line); then build r
  for (int k0 = 0; k0 < len; k0 += T) {
    const int tn = min(T, len - k0);
    if (tid == 0 && k0 == 0 && !prefetched) issueLineCopies<Rows>(a, fac, T, sm4, bar);
    if (tid == 0 && k0 > 0) {
      fenceProxyAsync();
      mbarExpectTx(bar, 16u * RC * tn);
      for (int p = 0; p < RC; ++p) bulkCopy(sCp + p * T, src + solveF4 + p * len + k0, 16u * tn, bar);
    }
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const int c = across0 + a - 2;
      for (int kk = tid; kk < tn + 4; kk += nt) {
        const int k = k0 + kk - 2;
        const bool ok = k >= 0 && k < len && c >= 0 && c < nAcross;
        cpAsync16(sX + a * TX + kk, L.X + (ok ? n0 + k * st + (a - 2) * acrossStep : n0), ok);
      }
    }
    for (int kk = tid; kk < tn; kk += nt) cpAsync16(sBt + kk, L.B + n0 + (k0 + kk) * st, true);
    cpAsyncWaitAll();
    mbarWaitBounded(bar, phase, err);
    phase ^= 1u;
    __syncthreads();
    for (int kk = tid; kk < tn; kk += nt) {
      const float4* cp = sCp + kk;
      const float4* xc = sX + kk + 2;
      float3 r = colF(cp, CF, T) * f3(sBt[kk]);
      int pos = 0;
#pragma unroll
      for (int q = 0; q < SlotOf<Rows>::NC; ++q) {
        const int role = Cp::role(q, FAM);
        if (role == 1 || role == -1) continue;
        const int2 o = Rows::offset(q);
        const int along = FAM == 0 ? o.x : o.y, across = FAM == 0 ? o.y : o.x;
        const float3 xm = f3(xc[(across + 2) * TX + along]);
        if (Cp::scalar(q))
          r -= colF(cp, pos, T) * xm;
        else
          r -= colSym(cp, pos, T) * xm;
        pos += Cp::width(q);
      }
      r = r + colF(cp, CF + 1, T) * f3(xc[2 * TX]);
      // interior nodes of a chunk keep Minv r, the chain's independent half
      const int k = k0 + kk, t = ch.of(k), ks = ch.start(t), ix = t * S + (k - ks);
      if (k != ks && k != ks + ch.size(t) - 1) r = m3Vec(ldM(sF + ix, NP), r);
      stV(sR + ix, r);
    }
    __syncthreads();
  }

  // ---- chunk interiors, lane t of warp 0 on chunk t: h_k = (Minv r)_k - (Minv A)_k h_{k-1},
  // v_k = h_k - G_k v_{k+1} (each step's matrices loaded a step ahead, off the dependent chain);
  // then the reduced right-hand sides
  if (tid < P) {
    const int lane = tid;
    const int ks = ch.start(lane), mlen = ch.size(lane), ke = ks + mlen - 1;
    const int o = lane * S - ks;  // padded position of node k: o + k
    float3 h = make_float3(0, 0, 0);
    if (ks + 1 < ke) {
      M3 Qa = ldM(sF + 3 * NP + o + ks + 1, NP);
      float3 tk = ldV(sR + o + ks + 1);
      for (int k = ks + 1; k < ke; ++k) {
        M3 QaN = Qa;
        float3 tN = tk;
        if (k + 1 < ke) QaN = ldM(sF + 3 * NP + o + k + 1, NP), tN = ldV(sR + o + k + 1);
        h = tk - m3Vec(Qa, h);
        stV(sV + o + k, h);
        Qa = QaN, tk = tN;
      }
    }
    float3 v = make_float3(0, 0, 0), vS = v, vE = v;
    if (ks + 1 < ke) {
      M3 Gk = ldM(sF + 6 * NP + o + ke - 1, NP);
      float3 hk = ldV(sV + o + ke - 1);
      for (int k = ke - 1; k > ks; --k) {
        M3 GN = Gk;
        float3 hN = hk;
        if (k - 1 > ks) GN = ldM(sF + 6 * NP + o + k - 1, NP), hN = ldV(sV + o + k - 1);
        v = hk - m3Vec(Gk, v);
        stV(sV + o + k, v);
        if (k == ke - 1) vE = v;
        Gk = GN, hk = hN;
      }
    }
    if (mlen >= 3) vS = v;
    stV(qr + 2 * lane, ldV(sR + o + ks) - m3Vec(ldM(sF + o + ks, NP), vS));
    stV(qr + 2 * lane + 1, ldV(sR + o + ke) - m3Vec(ldM(sF + o + ke, NP), vE));
  }
  __syncthreads();

  // ---- the end unknowns: x = inverse . r, thread o on output o (3Q of them)
  for (int o = tid; o < 3 * Q; o += nt) {
    const float* row = dense + o;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (int q = 0; q < Q; ++q) {
      const float4 rq = qr[q];
      a0 = fmaf(row[(3 * q) * QS], rq.x, a0);
      a1 = fmaf(row[(3 * q + 1) * QS], rq.y, a1);
      a2 = fmaf(row[(3 * q + 2) * QS], rq.z, a2);
    }
    reinterpret_cast<float*>(qx)[4 * (o / 3) + o % 3] = (a0 + a1) + a2;
  }
  __syncthreads();

  // ---- recovery and write-back, every node in parallel (fixed rows keep their unknowns)
  for (int k = tid; k < len; k += nt) {
    const int t = ch.of(k);
    const int ks = ch.start(t), ke = ks + ch.size(t) - 1;
    const int ix = t * S + (k - ks);
    if (sF[2 * NP + ix].z != 0.f) continue;
    const float3 xs = ldV(qx + 2 * t), xe = ldV(qx + 2 * t + 1);
    float3 x;
    if (k == ks)
      x = xs;
    else if (k == ke)
      x = xe;
    else
      x = ldV(sV + ix) + m3Vec(ldM(sF + 9 * NP + ix, NP), xs) + m3Vec(ldM(sF + 12 * NP + ix, NP), xe);
    L.X[n0 + k * st] = make_float4(x.x, x.y, x.z, 0.f);
  }
}


template <class Rows, int FAM>
__global__ void __launch_bounds__(SM_SWEEP_THREADS, 1) k_smooth(DLevel L, LineGeom g, const int4* __restrict__ lines, const int* __restrict__ base,
                                                       const float4* __restrict__ fac, int T, uint32_t* err) {
  __shared__ uint64_t bar;
  extern __shared__ float4 sm4[];
  LineAt a;
  if (g.table) {
    const int4 line = lines[g.first + blockIdx.x];
    a.n0 = line.x, a.st = line.y, a.len = line.z;
    a.ly = L.layers[line.w >> 1];
    a.fb = base[g.first + blockIdx.x];
    a.ch = Chunks(a.len);
    a.across0 = FAM == 0 ? (a.n0 - a.ly.offset) / a.ly.nx : (a.n0 - a.ly.offset) % a.ly.nx;
  } else {
    a = lineAt(g, blockIdx.x);
  }
  // the line's factors and coupling copies (written by the factorisation, launches back) stream in
  // while the kernel before this one may still run; its unknowns are read after the wait
  if (threadIdx.x == 0) {
    mbarInit(&bar, 1);
    issueLineCopies<Rows>(a, fac, T, sm4, &bar);
  }
  pdlWait();
  pdlLaunchNext();
  __syncthreads();
  unsigned phase = 0;
  sweepLine<Rows, FAM>(L, a, fac, T, err, sm4, &bar, phase, true);
}

}  // namespace btd
