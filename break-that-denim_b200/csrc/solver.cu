// Host side of the CUDA solve: the B200 counterpart of the reference's GpuSolver
// (src/simulation/gpu/solver.ts:194-838) behind the C ABI of include/btd.h.
//
// A solver owns its device memory and one CUDA stream. A substep (encodeSubstep, solver.ts:737-760)
// is captured once into a CUDA graph: predictor, Newton iterations (assembly, Galerkin hierarchy on
// the first iteration, PCG with a V-cycle preconditioner, line search, bounded update), commit,
// damage field and crossing slip. PCG's convergence test runs on the device and drives a graph
// while-node, so a whole substep is one graph launch with no host round trip.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "btd.h"
#include "common.cuh"
#include "k_contact.cuh"
#include "k_grip.cuh"
#include "k_learned.cuh"
#include "k_xcontact.cuh"
#include "k_history.cuh"
#include "k_mg.cuh"
#include "k_pcg.cuh"
#include "k_rigid.cuh"
#include "k_smooth.cuh"
#include "k_step.cuh"

namespace btd {
void setError(const std::string& msg);

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define CK(call)                                                                                            \
  do {                                                                                                      \
    cudaError_t e_ = (call);                                                                                \
    if (e_ != cudaSuccess) throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

static int blocksFor(int n, int t) { return (n + t - 1) / t; }

// ------------------------------------------------------------------------------------------ levels

struct Level {
  int N = 0;
  bool fine = false;
  std::vector<DLevelLayer> layers;
  std::vector<int4> lines;  // (start, stride, length, family) grouped by colour
  int colourStart[7] = {0, 0, 0, 0, 0, 0, 0};
  int maxLine = 0;
  DLevelLayer* dLayers = nullptr;
  uint2* dCoord = nullptr;
  int4* dLines = nullptr;
  // line factors (k_line_factor): each line's region starts at facBase[line]
  std::vector<int> facBase;
  int tile = 0;          // sweep staging tile (nodes)
  int threads = 0;       // sweep CTA size
  LineGeom geom[6] = {};  // launch geometry per colour
  int* dFacBase = nullptr;
  float4* fac = nullptr;
  size_t facF4 = 0;
  float4* op = nullptr;
  uint32_t* fixed = nullptr;
  float4 *X = nullptr, *B = nullptr, *R = nullptr, *pw = nullptr;
  DLevel dev() const {
    DLevel d;
    d.N = N;
    d.nLayers = (int)layers.size();
    d.one = layers.size() == 1 ? layers[0] : DLevelLayer{0, 0, 0, 0};
    d.layers = dLayers;
    d.coord = dCoord;
    d.op = op;
    d.fixed = fixed;
    d.X = X;
    d.B = B;
    d.R = R;
    d.pw = pw;
    return d;
  }
};

// Line tables (lineTable, lattice.ts:330-350): v-lines coloured i mod 3, then u-lines j mod 3;
// entry (start node, stride, length, family | layer << 1). Then each line's factor region, and per
// colour the launch geometry (computed from the block index on a single layer).
static void buildLines(Level& L) {
  std::vector<int4> byColour[6];
  for (size_t l = 0; l < L.layers.size(); ++l) {
    const auto& ly = L.layers[l];
    const int tag = (int)(l << 1);
    for (int i = 0; i < ly.nx; ++i) byColour[i % 3].push_back(make_int4(ly.offset + i, ly.nx, ly.ny, 1 | tag));
    for (int j = 0; j < ly.ny; ++j) byColour[3 + j % 3].push_back(make_int4(ly.offset + j * ly.nx, 1, ly.nx, 0 | tag));
    L.maxLine = std::max(L.maxLine, std::max(ly.nx, ly.ny));
  }
  L.lines.clear();
  for (int c = 0; c < 6; ++c) {
    L.colourStart[c] = (int)L.lines.size();
    L.lines.insert(L.lines.end(), byColour[c].begin(), byColour[c].end());
  }
  L.colourStart[6] = (int)L.lines.size();
  auto regionF4 = [&](int len) { return L.fine ? lineFactorF4<FineRows>(len) : lineFactorF4<CoarseRows>(len); };
  L.facBase.clear();
  size_t off = 0;
  for (const int4& ln : L.lines) {
    L.facBase.push_back((int)off);
    off += regionF4(ln.z);
  }
  L.facF4 = off;
  L.tile = L.fine ? smoothTile<FineRows>(L.maxLine) : smoothTile<CoarseRows>(L.maxLine);
  L.threads = sweepThreads(L.maxLine);
  for (int c = 0; c < 6; ++c) {
    LineGeom& g = L.geom[c];
    g = LineGeom{};
    g.first = L.colourStart[c];
    g.table = 1;
    if (L.layers.size() != 1 || L.colourStart[c + 1] == L.colourStart[c]) continue;
    const DLevelLayer& ly = L.layers[0];
    const int fam = c < 3 ? 1 : 0, c3 = c % 3;
    g.ly = ly;
    g.start0 = ly.offset + (fam == 1 ? c3 : c3 * ly.nx);
    g.startStep = fam == 1 ? 3 : 3 * ly.nx;
    g.stride = fam == 1 ? ly.nx : 1;
    g.len = fam == 1 ? ly.ny : ly.nx;
    g.base0 = L.facBase[g.first];
    g.baseStep = regionF4(g.len);
    g.across0 = c3;
    const Chunks ch(g.len);
    g.P = ch.P, g.chunkBase = ch.base, g.chunkExtra = ch.extra, g.S = ch.S;
    bool same = true;
    for (int b = 0; b < L.colourStart[c + 1] - g.first; ++b) {
      const int4 ln = L.lines[g.first + b];
      same = same && ln.x == g.start0 + b * g.startStep && ln.y == g.stride && ln.z == g.len &&
             L.facBase[g.first + b] == g.base0 + b * g.baseStep;
    }
    g.table = same ? 0 : 1;
  }
}

}  // namespace btd

using namespace btd;

struct btd_solver {
  int device = 0;
  cudaStream_t stream = nullptr, bodyStream = nullptr, gateStream = nullptr;
  btd_params params{};
  SimParams hostP{};
  int N = 0, C = 0, nLayers = 0;
  int redBlocks = 1;
  std::vector<void*> allocs;
  // scene copies for resetState
  std::vector<float4> x0;
  std::vector<Seg> segs0;
  std::vector<float> soft0, fail0, tails0;
  std::vector<uint8_t> damage0;
  // device state
  SimParams* dP = nullptr;
  Scalars* dScal = nullptr;
  uint32_t* dCounters = nullptr;
  double* dPartials = nullptr;
  unsigned* dTicket = nullptr;
  NodeStatic* dNodes = nullptr;
  DLayer* dLayers = nullptr;
  float4 *x = nullptr, *v = nullptr, *dx = nullptr, *pred = nullptr, *ext = nullptr, *delta = nullptr, *p = nullptr,
         *Ap = nullptr, *b0 = nullptr;
  double* deltaD = nullptr;
  // the fine operator in FP64, the operator PCG solves with (null when the solve takes the fp32 rows)
  double2* op64 = nullptr;
  bool opFp64 = true;
  float4* zPrev = nullptr;
  Seg* segs = nullptr;
  float *softening = nullptr, *failSite = nullptr, *tails = nullptr, *strain = nullptr, *strength = nullptr;
  uint8_t *damage = nullptr, *area = nullptr, *sep = nullptr, *marks = nullptr;
  std::vector<Level> levels;
  std::vector<DLayer> hostLayers;
  // grips (interaction.ts attachPatch/setTarget/release): device slots + entries, host mirror of
  // the slots, the base stiffness of each (setHold scales it) and the slot holding each node
  // self-contact (selfcontact.ts): hash table, hashed faces, candidates and bound keys, bounds,
  // fixed-point accumulators; allocated when params.self_contact
  unsigned* ctCells = nullptr;
  unsigned* ctScanTiles = nullptr;  // the contact scan's tile sums
  float4* ctItems = nullptr;
  unsigned* ctPairs = nullptr;
  float4* cmeta = nullptr;
  int* ctAcc = nullptr;
  bool contactOn() const { return params.self_contact != 0 && cmeta != nullptr; }
  // cross-layer contact in place of self-contact (solver.ts:364)
  unsigned* xcCells = nullptr;
  int* xcItems = nullptr;
  bool xcOn() const { return contactOn() && xcCells != nullptr; }
  float xcDist[4] = {0, 0, 0, 0};
  XcArgs xcArgs() const {
    XcArgs a;
    a.N = N;
    a.nodes = dNodes;
    a.P = dP;
    a.x = x;
    a.dx = dx;
    a.cells = xcCells;
    a.items = xcItems;
    a.cand = reinterpret_cast<int*>(ctPairs);
    a.cmeta = cmeta;
    a.ext = ext;
    a.flag = lcEnabled ? lcCtFlag : nullptr;
    for (int q = 0; q < 4; ++q) a.dist[q] = xcDist[q];
    return a;
  }
  ContactArgs contactArgs() const {
    ContactArgs a;
    a.N = N;
    a.nodes = dNodes;
    a.layers = dLayers;
    a.P = dP;
    a.pinned = levels[0].fixed;
    a.x = x;
    a.dx = dx;
    a.segs = segs;
    a.cells = ctCells;
    a.items = ctItems;
    a.pairs = ctPairs;
    a.cmeta = cmeta;
    a.acc = ctAcc;
    a.ext = ext;
    // SELF_CONTACT (selfcontact.ts:7-33)
    a.law = ContactLaw{12e-3f, 3e-3f, 1.0e-3f, 500.f, 0.45f, 0.002f, 0.45f, (1u << CT_TABLE_BITS) - 1u};
    a.flag = lcOn() ? lcCtFlag : nullptr;
    return a;
  }
  // learned coarse correction (extension): network, state, basis, flags per level, training log
  LcState* dLc = nullptr;
  MlpPacked* dNet = nullptr;
  float* dLcW = nullptr;       // the flat FP32 weights as given (packed into dNet)
  float* lcPhi = nullptr;      // 3 M x LC_K
  uint8_t* lcCtFlag = nullptr; // per fine node
  uint8_t* lcBasisFlags = nullptr;  // the coarsest flags of the current learned basis
  std::vector<uint8_t*> lcFlags;  // per level
  LcLog lcLog{};
  bool lcEnabled = false;
  bool lcOn() const { return lcEnabled; }
  LcArgs lcArgs() const { return LcArgs{dLc, dNet, lcPhi, lcLog, lcBasisFlags}; }
  GripSlot* dGripSlots = nullptr;
  GripEntry* dGripEntries = nullptr;
  float4* dGripGoal = nullptr;
  GripSlot hostGrip[GRIPS] = {};
  float gripStiffness[GRIPS] = {};
  std::vector<int8_t> gripOwner;
  bool gripsOn() const {
    for (int g = 0; g < GRIPS; ++g)
      if (hostGrip[g].goal.w > 0.f) return true;
    return false;
  }
  // graphs: substep graphs keyed by Newton iteration count and whether grips are held; the
  // standalone PCG graph
  std::map<int, cudaGraphExec_t> substepExec;
  cudaGraphExec_t pcgExec = nullptr;
  bool useGraphs = true;
  bool batchGrips = false;  // grips held when a batch graph holding this solver was captured
  void* flushBuf = nullptr;  // profiling only: rewritten to evict L2 between timed launches

  template <class T>
  T* alloc(size_t count) {
    void* ptr = nullptr;
    CK(cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T)));
    CK(cudaMemsetAsync(ptr, 0, std::max<size_t>(count, 1) * sizeof(T), stream));
    allocs.push_back(ptr);
    return static_cast<T*>(ptr);
  }

  StepArgs stepArgs() const {
    StepArgs a;
    a.P = dP;
    a.N = N;
    a.nodes = dNodes;
    a.pinned = levels[0].fixed;
    a.layers = dLayers;
    a.x = x;
    a.v = v;
    a.dx = dx;
    a.pred = pred;
    a.segs = segs;
    a.ext = ext;
    a.cmeta = contactOn() ? cmeta : nullptr;
    a.counters = dCounters;
    a.scal = dScal;
    a.pieceCount = pieceCount;
    a.pieceOf = dPieceOf;
    a.kx = dKx;
    a.curveW = pieceCount > 0 ? dCurveW : nullptr;
    a.curveR = pieceCount > 0 ? dCurveR : nullptr;
    return a;
  }
  // detached pieces (setPieces, solver.ts:664-676): piece of each node, node lists, rigid frames and steps
  int pieceCount = 0;
  uint32_t *dPieceOf = nullptr, *dPieceStart = nullptr, *dPieceNodes = nullptr;
  size_t pieceNodesCap = 0;
  float *dKx = nullptr, *dKr = nullptr;
  double *dFrame = nullptr, *dStep = nullptr;
  float4 *dCurveW = nullptr, *dCurveR = nullptr;
  RigidArgs rigidArgs() const {
    return RigidArgs{pieceCount, dPieceOf, dPieceStart, dPieceNodes, dKx, dKr, dFrame, dStep, dCurveW, dCurveR};
  }
  Reduce reduce() const { return {dPartials, dTicket}; }
  GripArgs gripArgs() const {
    GripArgs a;
    a.slots = dGripSlots;
    a.entries = dGripEntries;
    a.goal = dGripGoal;
    a.x = x;
    a.dx = dx;
    a.ext = ext;
    a.adds = params.self_contact ? 1 : 0;
    return a;
  }
  PcgArgs pcgArgs(cudaGraphConditionalHandle h, int useCond) const {
    PcgArgs a;
    a.F = levels[0].dev();
    a.p = p;
    a.Ap = Ap;
    a.delta = delta;
    a.b0 = b0;
    a.dd = deltaD;
    a.scal = dScal;
    a.P = dP;
    a.counters = dCounters;
    a.red = reduce();
    a.cond = h;
    a.useCond = useCond;
    a.lc = lcOn() ? dLc : nullptr;
    a.op64 = opFp64 ? op64 : nullptr;
    a.zPrev = zPrev;
    return a;
  }
  HistArgs histArgs() const {
    HistArgs a;
    a.S = stepArgs();
    a.nSpans = 2 * N;
    a.nCross = C;
    a.nLayers = nLayers;
    a.strain = strain;
    a.softening = softening;
    a.failSite = failSite;
    a.tails = tails;
    a.damage = damage;
    a.area = area;
    a.strength = strength;
    a.sep = sep;
    a.marks = marks;
    a.segsW = segs;
    return a;
  }

  // ---------------------------------------------------------------- stage encoders (stream s)

  // encodePredict + preSubstep (solver.ts:742): predictor, then each held grip's lead from the
  // committed positions, then the start of the projected iterate.
  // encodePredict, preSubstep and contact detection (solver.ts:738-745): predictor, each held grip's
  // lead from the committed positions, the face hash and contact bounds at the predicted iterate,
  // then the start of the projected iterate.
  void encPredict(cudaStream_t s, bool grips) {
    k_predict<<<blocksFor(N, 128), 128, 0, s>>>(stepArgs());
    if (pieceCount > 0) {  // detached pieces start from their rotation over the substep (solver.ts:698-704)
      k_spin_reduce<<<pieceCount, RIGID_THREADS, 0, s>>>(stepArgs(), rigidArgs());
      k_spin_apply<<<blocksFor(N, 128), 128, 0, s>>>(stepArgs(), rigidArgs());
    }
    if (grips) k_grip_lead<<<GRIPS, 256, 0, s>>>(gripArgs());
    if (contactOn()) encDetect(s);
    k_project_start<<<blocksFor(N, 128), 128, 0, s>>>(stepArgs());
  }

  // The exclusive scan of T cell counts in place (two launches over the GPU).
  void encScan(cudaStream_t s, unsigned* cells, int T) {
    const int tiles = (T + CT_SCAN_TILE - 1) / CT_SCAN_TILE;
    if (tiles > CT_SCAN_MAX_TILES) throw std::logic_error("contact table larger than the scan's tile sums");
    k_ct_scan_tiles<<<tiles, CT_SCAN_THREADS, 0, s>>>(cells, T, ctScanTiles);
    k_ct_scan_apply<<<tiles, CT_SCAN_THREADS, 0, s>>>(cells, T, ctScanTiles);
  }

  // SelfContact.encodeClear + encodeDetect (selfcontact.ts:137-152).
  void encDetect(cudaStream_t s) {
    if (xcOn()) {  // contact.ts encodeDetect: count, scan, fill, detect on the (cell, layer) hash
      const XcArgs a = xcArgs();
      const int T = (int)XC_MASK + 1;
      CK(cudaMemsetAsync(xcCells, 0, sizeof(unsigned) * 2 * (size_t)T, s));
      k_xc_count<<<blocksFor(N, 128), 128, 0, s>>>(a);
      encScan(s, xcCells, T);
      k_xc_fill<<<blocksFor(N, 128), 128, 0, s>>>(a);
      k_xc_detect<<<blocksFor(N, 128), 128, 0, s>>>(a, nLayers);
      return;
    }
    const ContactArgs a = contactArgs();
    const int T = 1 << CT_TABLE_BITS;
    CK(cudaMemsetAsync(ctCells, 0, sizeof(unsigned) * 2 * (size_t)T, s));
    k_ct_face_count<<<blocksFor(N, 128), 128, 0, s>>>(a);
    encScan(s, ctCells, T);
    k_ct_face_fill<<<blocksFor(N, 128), 128, 0, s>>>(a);
    k_ct_damage_row<<<blocksFor(N, 128), 128, 0, s>>>(a);
    k_ct_detect<<<blocksFor(N, 128), 128, 0, s>>>(a);
    k_ct_resolve<<<blocksFor(N, 128), 128, 0, s>>>(a);
  }

  // SelfContact.encodeTerms (selfcontact.ts:155-161): contact and friction at the current iterate,
  // written over ext (grips add theirs after).
  void encContactTerms(cudaStream_t s) {
    if (!contactOn()) return;
    if (xcOn()) {
      k_xc_terms<<<blocksFor(N, 128), 128, 0, s>>>(xcArgs());
      return;
    }
    const ContactArgs a = contactArgs();
    k_ct_terms<<<blocksFor(N, 128), 128, 0, s>>>(a);
    k_ct_gather<<<blocksFor(N, 128), 128, 0, s>>>(a);
  }

  // preAssemble (solver.ts:690): grip terms at the current iterate into ext.
  void encGripTerms(cudaStream_t s, bool grips) {
    if (grips) k_grip_terms<<<GRIPS * GRIP_ENTRIES / 128, 128, 0, s>>>(gripArgs());
  }

  void encHierarchy(cudaStream_t s) {
    for (size_t k = 0; k + 1 < levels.size(); ++k) {
      DLevel F = levels[k].dev(), Cl = levels[k + 1].dev();
      if (k == 0) {
        k_prolong_weights<FineRows, true><<<blocksFor(F.N, 128), 128, 0, s>>>(F, segs);
        k_rap<FineRows><<<blocksFor(Cl.N, RAP_THREADS), RAP_THREADS, 0, s>>>(F, Cl);
      } else {
        k_prolong_weights<CoarseRows, false><<<blocksFor(F.N, 128), 128, 0, s>>>(F, segs);
        k_rap<CoarseRows><<<blocksFor(Cl.N, RAP_THREADS), RAP_THREADS, 0, s>>>(F, Cl);
      }
      encFactor(s, (int)k + 1);
    }
    if (lcOn()) k_lc_bump<<<1, 1, 0, s>>>(dLc);
  }

  // The learned coarse space of this PCG solve: damage and contact flags restricted to the coarsest
  // level, then the basis (once per solve; the correction itself runs inside every V-cycle).
  void encLearnedBasis(cudaStream_t s) {
    if (!lcOn()) return;
    k_lc_flags_fine<<<blocksFor(N, 128), 128, 0, s>>>(N, dNodes, dLayers, segs, contactOn() ? lcCtFlag : nullptr, lcFlags[0]);
    for (size_t k = 0; k + 1 < levels.size(); ++k)
      k_lc_flags_restrict<<<blocksFor(levels[k + 1].N, 128), 128, 0, s>>>(levels[k].dev(), levels[k + 1].dev(), lcFlags[k],
                                                                          lcFlags[k + 1]);
    const Level& C = levels.back();
    k_lc_basis<<<1, LC_THREADS, lcBasisSmem(C.N), s>>>(C.dev(), lcFlags.back(), lcArgs());
  }

  void encAssemble(cudaStream_t s, bool coarse) {
    k_assemble<<<blocksFor(N, 128), 128, 0, s>>>(stepArgs(), levels[0].op, levels[0].B, opFp64 ? op64 : nullptr);
    if (pieceCount > 0) {  // the pieces' rigid frames at this iterate (encodeAssemble, solver.ts:615-616)
      k_rigid_rotation<<<blocksFor(N, 128), 128, 0, s>>>(stepArgs(), rigidArgs());
      k_rigid_frame<<<pieceCount, RIGID_THREADS, 0, s>>>(stepArgs(), rigidArgs());
    }
    encFactor(s, 0);
    if (coarse) encHierarchy(s);
  }
  // PCG's start: zero, or each detached piece's rigid response (encodeRigidStart, solver.ts:651-657).
  void encPcgInit(cudaStream_t s, const PcgArgs& a) {
    if (pieceCount > 0) {
      k_rigid_start<<<pieceCount, RIGID_THREADS, 0, s>>>(stepArgs(), rigidArgs(), levels[0].B);
      k_pcg_init_rigid<<<redBlocks, RED_THREADS, 0, s>>>(a, stepArgs(), rigidArgs());
    } else {
      k_pcg_init<<<redBlocks, RED_THREADS, 0, s>>>(a);
    }
  }

  // Line factors of level k, every line in one launch (after its operator changed).
  void encFactor(cudaStream_t s, int k) {
    Level& L = levels[k];
    const int count = (int)L.lines.size();
    if (L.fine)
      k_line_factor<FineRows><<<count, SM_THREADS, factorSmemBytes<FineRows>(L.maxLine), s>>>(L.dev(), L.dLines, L.dFacBase, L.fac);
    else
      k_line_factor<CoarseRows><<<count, SM_THREADS, factorSmemBytes<CoarseRows>(L.maxLine), s>>>(L.dev(), L.dLines, L.dFacBase, L.fac);
  }

  // One sweep of level k: the six colours, v-lines first (reversed for the post-smoother).
  // A kernel of the PCG loop on `s`: with programmatic stream serialisation when the solver overlaps
  // launches (each such kernel waits for its predecessor before reading its output; pdlWait).
  template <typename... P, typename... A>
  void launch(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &at;
    cfg.numAttrs = params.overlap_launches ? 1 : 0;
    CK(cudaLaunchKernelEx(&cfg, k, args...));
  }

  void encSmooth(cudaStream_t s, int k, bool reverse) {
    Level& L = levels[k];
    const size_t smem = L.fine ? smoothSmemBytes<FineRows>(L.maxLine, L.tile) : smoothSmemBytes<CoarseRows>(L.maxLine, L.tile);
    const DLevel d = L.dev();
    for (int q = 0; q < 6; ++q) {
      const int c = reverse ? 5 - q : q;
      const int count = L.colourStart[c + 1] - L.colourStart[c];
      if (count == 0) continue;
      const LineGeom& g = L.geom[c];
      if (L.fine) {
        if (c < 3)
          launch(k_smooth<FineRows, 1>, count, L.threads, smem, s, d, g, (const int4*)L.dLines, (const int*)L.dFacBase, (const float4*)L.fac, L.tile, dCounters + CNT_ERROR);
        else
          launch(k_smooth<FineRows, 0>, count, L.threads, smem, s, d, g, (const int4*)L.dLines, (const int*)L.dFacBase, (const float4*)L.fac, L.tile, dCounters + CNT_ERROR);
      } else {
        if (c < 3)
          launch(k_smooth<CoarseRows, 1>, count, L.threads, smem, s, d, g, (const int4*)L.dLines, (const int*)L.dFacBase, (const float4*)L.fac, L.tile, dCounters + CNT_ERROR);
        else
          launch(k_smooth<CoarseRows, 0>, count, L.threads, smem, s, d, g, (const int4*)L.dLines, (const int*)L.dFacBase, (const float4*)L.fac, L.tile, dCounters + CNT_ERROR);
      }
    }
  }

  // encodeVCycle (solver.ts:584-598): X of level k = V(B) with X zero on entry.
  void encVCycle(cudaStream_t s, int k) {
    int last = (int)levels.size() - 1;
    if (k == last) {
      if (lcOn()) {
        // the learned coarse space half-way through the coarsest sweeps, which mirror around it
        const int half = params.coarse_sweeps / 2;
        for (int sw = 0; sw < half; ++sw) encSmooth(s, k, (sw & 1) == 1);
        launch(k_lc_correct, 1, LC_THREADS, 0, s, levels[k].dev(), lcArgs());
        for (int sw = half; sw < params.coarse_sweeps; ++sw) encSmooth(s, k, (sw & 1) == 1);
        return;
      }
      for (int sw = 0; sw < params.coarse_sweeps; ++sw) encSmooth(s, k, (sw & 1) == 1);
      return;
    }
    Level& F = levels[k];
    Level& Cl = levels[k + 1];
    encSmooth(s, k, false);
    if (F.fine && opFp64)
      launch(k_residual_fine64, blocksFor(F.N, 128), 128, 0, s, F.dev(), (const double2*)op64);
    else if (F.fine)
      launch(k_residual_fine, blocksFor(F.N, 128), 128, 0, s, F.dev());
    else
      launch(k_residual_coarse, blocksFor(8 * F.N, 128), 128, 0, s, F.dev());
    launch(k_restrict, blocksFor(Cl.N, 128), 128, 0, s, F.dev(), Cl.dev());
    encVCycle(s, k + 1);
    launch(k_prolong, blocksFor(F.N, 128), 128, 0, s, F.dev(), Cl.dev());
    encSmooth(s, k, true);
  }

  void encPcgBody(cudaStream_t s, const PcgArgs& a) {
    encVCycle(s, 0);
    launch(k_pcg_dot_rz, redBlocks, RED_THREADS, 0, s, a, 0);
    launch(k_pcg_update_p, blocksFor(N, 256), 256, 0, s, a, 0);
    launch(k_pcg_matvec, redBlocks, RED_THREADS, 0, s, a);
    launch(k_pcg_update_xr, redBlocks, RED_THREADS, 0, s, a);
    launch(k_pcg_true_residual, redBlocks, RED_THREADS, 0, s, a);
  }

  // encodePCG (solver.ts:625-644) with the device-side stop: prologue, then a while-node whose
  // condition k_pcg_update_xr sets. Must be called while `s` is capturing.
  void encPCG(cudaStream_t s) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g;
    const cudaGraphNode_t* deps = nullptr;
    size_t nDeps = 0;
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nDeps));
    if (st != cudaStreamCaptureStatusActive)
      throw std::runtime_error("PCG must be encoded into a graph capture (capture status " + std::to_string((int)st) + ", last error " +
                               cudaGetErrorString(cudaPeekAtLastError()) + ")");
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    PcgArgs a = pcgArgs(h, 1);
    encLearnedBasis(s);
    encPcgInit(s, a);
    encVCycle(s, 0);
    launch(k_pcg_dot_rz, redBlocks, RED_THREADS, 0, s, a, 1);
    launch(k_pcg_update_p, blocksFor(N, 256), 256, 0, s, a, 1);
    launch(k_pcg_matvec, redBlocks, RED_THREADS, 0, s, a);
    launch(k_pcg_update_xr, redBlocks, RED_THREADS, 0, s, a);
    launch(k_pcg_true_residual, redBlocks, RED_THREADS, 0, s, a);
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nDeps));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nDeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    CK(cudaStreamBeginCaptureToGraph(bodyStream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    encPcgBody(bodyStream, a);
    cudaGraph_t out;
    CK(cudaStreamEndCapture(bodyStream, &out));
  }

  // The same PCG launched kernel by kernel, the stop read back after every iteration.
  void runPCGEager(cudaStream_t s) {
    PcgArgs a = pcgArgs(0, 0);
    encLearnedBasis(s);
    encPcgInit(s, a);
    encVCycle(s, 0);
    launch(k_pcg_dot_rz, redBlocks, RED_THREADS, 0, s, a, 1);
    launch(k_pcg_update_p, blocksFor(N, 256), 256, 0, s, a, 1);
    launch(k_pcg_matvec, redBlocks, RED_THREADS, 0, s, a);
    launch(k_pcg_update_xr, redBlocks, RED_THREADS, 0, s, a);
    launch(k_pcg_true_residual, redBlocks, RED_THREADS, 0, s, a);
    for (;;) {
      int conv = 0;
      CK(cudaMemcpyAsync(&conv, &dScal->converged, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      if (conv) break;
      encPcgBody(s, a);
    }
  }

  // The substep launched kernel by kernel; a gated iteration runs when the host reads that the one
  // before moved some node by more than the tolerance.
  void runSubstepEager(int newtonIterations, int newtonMax) {
    cudaStream_t s = stream;
    const bool grips = gripsOn();
    CK(cudaMemsetAsync(dCounters + CNT_UPDATE, 0, sizeof(uint32_t) * MAX_NEWTON, s));
    encPredict(s, grips);
    for (int it = 0; it < newtonMax; ++it) {
      if (it >= newtonIterations) {
        uint32_t moved = 0;
        CK(cudaMemcpyAsync(&moved, dCounters + CNT_UPDATE + it - 1, sizeof moved, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        float m;
        std::memcpy(&m, &moved, sizeof m);
        if (!(m > hostP.newtonTol)) break;
      }
      encContactTerms(s);
      encGripTerms(s, grips);
      encAssemble(s, it == 0 || !params.lag_coarse);
      runPCGEager(s);
      encLineSearch(s);
      encApply(s, it);
    }
    encFinalize(s);
    CK(cudaGetLastError());
  }

  void encLineSearch(cudaStream_t s) {
    // pieces step along the rotation of their rigid start (encodeLineSearch, solver.ts:680-681)
    if (pieceCount > 0) k_rigid_curves<<<blocksFor(N, 128), 128, 0, s>>>(stepArgs(), rigidArgs());
    if (params.line_search) {
      EnergyArgs e;
      e.S = stepArgs();
      e.delta = delta;
      e.red = reduce();
      e.curveW = pieceCount > 0 ? dCurveW : nullptr;
      e.curveR = pieceCount > 0 ? dCurveR : nullptr;
      k_energy<<<redBlocks, RED_THREADS, 0, s>>>(e);
    } else {
      k_set_alpha<<<1, 1, 0, s>>>(dScal, dCounters, 1.f);
    }
  }

  void encApply(cudaStream_t s, int it) {
    k_newton_apply<<<blocksFor(N, 128), 128, 0, s>>>(stepArgs(), delta, std::min(it, MAX_NEWTON - 1));
  }

  // encodeNewtonIteration (solver.ts:687-696).
  void encNewton(cudaStream_t s, int it, bool grips) {
    encContactTerms(s);
    encGripTerms(s, grips);
    encAssemble(s, it == 0 || !params.lag_coarse);
    encPCG(s);
    encLineSearch(s);
    encApply(s, it);
  }

  void encDamage(cudaStream_t s) {
    HistArgs h = histArgs();
    k_span_strain<<<blocksFor(2 * N, 256), 256, 0, s>>>(h);
    k_sep_snapshot<<<blocksFor(2 * C, 256), 256, 0, s>>>(h);
    k_field_update<<<blocksFor(2 * N, 128), 128, 0, s>>>(h);
    for (int l = 0; l < nLayers; ++l)
      k_pull_mark<<<blocksFor(hostLayers[l].K * hostLayers[l].M, 128), 128, 0, s>>>(h, l);
    k_pull_apply<<<blocksFor(2 * C, 256), 256, 0, s>>>(h);
    k_couple<<<blocksFor(2 * N, 128), 128, 0, s>>>(h);
  }

  // encodeFinalize (solver.ts:723-728); history passes check SimParams.historyOn on the device.
  void encFinalize(cudaStream_t s) {
    k_commit<<<blocksFor(N, 128), 128, 0, s>>>(stepArgs());
    encDamageGated(s);
    HistArgs h = histArgs();
    for (int f = 0; f < 2; ++f)
      for (int par = 0; par < 2; ++par) k_slip<<<blocksFor(N, 128), 128, 0, s>>>(h, f, par);
  }
  void encDamageGated(cudaStream_t s);

  // Gated Newton iteration `it` (encodeSubstep's optional iterations, solver.ts:744-757; gate.wgsl):
  // a conditional node runs it only while iteration it - 1 still moved some node by more than the
  // tolerance. A skipped iteration leaves its update slot at zero, so every later one stays off.
  // Must be called while `s` is capturing.
  void encGatedNewton(cudaStream_t s, int it, bool grips) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g;
    const cudaGraphNode_t* deps = nullptr;
    size_t nDeps = 0;
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nDeps));
    if (st != cudaStreamCaptureStatusActive) throw std::runtime_error("gated Newton iterations must be encoded into a graph capture");
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    k_gate<<<1, 1, 0, s>>>(dCounters, it - 1, dP, h);
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nDeps));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nDeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    CK(cudaStreamBeginCaptureToGraph(gateStream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    encNewton(gateStream, it, grips);
    cudaGraph_t out;
    CK(cudaStreamEndCapture(gateStream, &out));
  }

  void encSubstep(cudaStream_t s, int newtonIterations, int newtonMax, bool grips) {
    CK(cudaMemsetAsync(dCounters + CNT_UPDATE, 0, sizeof(uint32_t) * MAX_NEWTON, s));
    encPredict(s, grips);
    for (int it = 0; it < newtonIterations; ++it) encNewton(s, it, grips);
    for (int it = newtonIterations; it < newtonMax; ++it) encGatedNewton(s, it, grips);
    encFinalize(s);
  }

  cudaGraphExec_t capture(const std::function<void(cudaStream_t)>& fn) {
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
    try {
      fn(stream);
    } catch (...) {
      cudaGraph_t g;
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cudaGraph_t g;
    CK(cudaStreamEndCapture(stream, &g));
    cudaGraphExec_t ex;
    CK(cudaGraphInstantiate(&ex, g, 0));
    CK(cudaGraphDestroy(g));
    return ex;
  }

  // Newton iterations of a substep asked for min / max iterations (encodeSubstep, solver.ts:744-746).
  int unconditional(int minIterations) const { return std::min(MAX_NEWTON, std::max(params.newton_iterations, minIterations)); }
  int gatedBound(int minIterations, int maxIterations) const {
    return std::min(MAX_NEWTON, std::max(std::max(params.newton_max, unconditional(minIterations)), maxIterations));
  }

  cudaGraphExec_t substepGraph(int iters, int itersMax) {
    const bool grips = gripsOn();
    const int key = (iters * (MAX_NEWTON + 1) + itersMax) * 2 + (grips ? 1 : 0);
    auto it = substepExec.find(key);
    if (it != substepExec.end()) return it->second;
    cudaGraphExec_t ex = capture([&](cudaStream_t s) { encSubstep(s, iters, itersMax, grips); });
    substepExec[key] = ex;
    return ex;
  }
  void runSubstep(int minIterations, int maxIterations) {
    const int iters = unconditional(minIterations), itersMax = gatedBound(minIterations, maxIterations);
    if (useGraphs)
      CK(cudaGraphLaunch(substepGraph(iters, itersMax), stream));
    else
      runSubstepEager(iters, itersMax);
  }

  void pushParams() {
    CK(cudaMemcpyAsync(dP, &hostP, sizeof(SimParams), cudaMemcpyHostToDevice, stream));
  }
  void sync() { CK(cudaStreamSynchronize(stream)); }

  ~btd_solver() {
    for (auto& kv : substepExec) cudaGraphExecDestroy(kv.second);
    if (pcgExec) cudaGraphExecDestroy(pcgExec);
    if (flushBuf) cudaFree(flushBuf);
    for (void* q : allocs) cudaFree(q);
    if (stream) cudaStreamDestroy(stream);
    if (bodyStream) cudaStreamDestroy(bodyStream);
    if (gateStream) cudaStreamDestroy(gateStream);
  }
};

// The damage passes early-out inside the kernels when history is off, except the span strain and
// snapshot passes, which are cheap and harmless.
void btd_solver::encDamageGated(cudaStream_t s) { encDamage(s); }

namespace {

// A bounded device-side wait ran out (the kernel raised a flag in the counters and went on).
struct DeviceTimeout : std::runtime_error {
  using std::runtime_error::runtime_error;
};

int fail(const std::exception& e) {
  if (dynamic_cast<const DeviceTimeout*>(&e)) {
    btd::setError(e.what());
    return BTD_E_TIMEOUT;
  }
  if (dynamic_cast<const CudaError*>(&e)) {
    btd::setError(e.what());
    return BTD_E_CUDA;
  }
  btd::setError(e.what());
  return BTD_E_INVALID;
}

#define GUARD(...)                         \
  try {                                    \
    __VA_ARGS__;                           \
    return BTD_OK;                         \
  } catch (const std::exception& e) {      \
    return fail(e);                        \
  }

DYarn toDYarn(const btd_yarn& y) {
  return {(float)y.ea_low, (float)y.ea_high, (float)y.crimp_strain, (float)y.ea_compress, (float)y.axial_viscosity,
          (float)y.bend_rigidity, (float)y.bend_viscosity, (float)(y.yarns_per_span > 0 ? y.yarns_per_span : 1)};
}

void checkSolver(btd_solver* s) {
  if (!s) throw std::invalid_argument("null solver");
}

}  // namespace

extern "C" {

static float4* vectorPtr(btd_solver* s, int which, int level, size_t* count);

int btd_default_params(btd_params* out) {
  if (!out) return BTD_E_INVALID;
  btd_params p{};
  p.h = 1.0 / 120;
  p.gravity[0] = 0;
  p.gravity[1] = 0;
  p.gravity[2] = -9.81;
  p.newton_iterations = 2;
  p.newton_max = 2;
  p.newton_tolerance = 1e-5;
  p.history_tolerance = 1;
  p.pcg_iterations = 2;
  p.coarse_sweeps = 2;
  p.max_coarsest_nodes = 400;
  p.self_contact = 1;
  p.pcg_rel_tol = 0;
  p.line_search = 1;
  p.lag_coarse = 1;
  p.overlap_launches = 1;
  p.cross_layer = 0;
  *out = p;
  return BTD_OK;
}

int btd_create(const btd_scene* sc, const btd_params* prm, btd_solver** out) {
  if (!sc || !prm || !out) {
    btd::setError("btd_create: null argument");
    return BTD_E_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    btd::setError("btd_create: no CUDA device (the solve has no CPU fallback)");
    return BTD_E_NO_DEVICE;
  }
  std::unique_ptr<btd_solver> s(new btd_solver());
  try {
    if (prm->newton_iterations < 1 || prm->newton_iterations > MAX_NEWTON || prm->newton_max < prm->newton_iterations ||
        prm->newton_max > MAX_NEWTON)
      throw std::invalid_argument("invalid Newton iteration bounds");
    if (prm->pcg_iterations < 1) throw std::invalid_argument("pcg_iterations must be >= 1");
    if (prm->coarse_sweeps < 1) throw std::invalid_argument("coarse_sweeps must be >= 1");
    if (!(prm->h > 0)) throw std::invalid_argument("h must be positive");
    if (prm->self_contact && sc->node_count >= (1 << 20))
      throw std::invalid_argument("self-contact bound keys hold at most 2^20 - 1 nodes");
    CK(cudaGetDevice(&s->device));
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&s->bodyStream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&s->gateStream, cudaStreamNonBlocking));
    s->params = *prm;
    const int N = sc->node_count, C = sc->crossing_count;
    s->N = N;
    s->C = C;
    s->nLayers = sc->n_layers;
    if (N < 4 || sc->n_layers < 1) throw std::invalid_argument("empty scene");

    // ---- layers and per-node static data
    std::vector<NodeStatic> nodes(N);
    std::vector<uint32_t> pinned(N);
    std::vector<uint2> coord(N);
    for (int l = 0; l < sc->n_layers; ++l) {
      const btd_layer_info& L = sc->layers[l];
      if (L.nx < 2 || L.ny < 2 || L.nx > 65535 || L.ny > 65535) throw std::invalid_argument("lattice extent out of range");
      if (std::max(L.nx, L.ny) > SM_MAX_LINE) throw std::invalid_argument("yarn line longer than " + std::to_string(SM_MAX_LINE));
      if (L.bundle[0] > 32 || L.bundle[1] > 32) throw std::invalid_argument("bundles of more than 32 yarns are not supported");
      DLayer d{};
      d.offset = L.node_offset;
      d.nx = L.nx;
      d.ny = L.ny;
      d.nodeCount = L.node_count;
      d.yarn[0] = toDYarn(L.material.yarns[0]);
      d.yarn[1] = toDYarn(L.material.yarns[1]);
      d.shearStiffness = (float)L.material.shear_stiffness;
      d.crossingFriction = (float)L.material.crossing_friction;
      d.crossingWrap = (float)L.material.crossing_wrap;
      d.pitchU = (float)L.material.pitch_u;
      d.pitchV = (float)L.material.pitch_v;
      d.airDrag = (float)L.material.air_drag;
      d.crossingNormal0 = (float)L.material.crossing_normal0;
      d.thickness = (float)L.material.thickness;
      d.fOffset = L.field_offset;
      d.K = L.field_k;
      d.M = L.field_m;
      d.bu = L.bundle[0];
      d.bv = L.bundle[1];
      d.reachU = std::max(1, (int)std::lround(1.2e-3 / L.weave.pitch_u));
      d.reachV = std::max(1, (int)std::lround(1.2e-3 / L.weave.pitch_v));
      d.weavePitchU = (float)L.weave.pitch_u;
      d.weavePitchV = (float)L.weave.pitch_v;
      s->hostLayers.push_back(d);
      for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
          int n = L.node_offset + j * L.nx + i;
          nodes[n] = {(uint32_t)i | ((uint32_t)j << 16), (uint32_t)l, (float)sc->mass[n], (float)sc->crossing_normal0[n]};
          pinned[n] = sc->pinned[n] ? 1u : 0u;
          coord[n] = make_uint2((uint32_t)i | ((uint32_t)j << 16), (uint32_t)l);
        }
    }
    cudaStream_t st = s->stream;
    s->dP = s->alloc<SimParams>(1);
    s->dScal = s->alloc<Scalars>(1);
    s->dCounters = s->alloc<uint32_t>(CNT_SIZE);
    s->redBlocks = std::max(1, std::min(blocksFor(N, RED_THREADS), 4 * 148));
    s->dPartials = s->alloc<double>(8 * (size_t)s->redBlocks);
    s->dTicket = s->alloc<unsigned>(1);
    s->dNodes = s->alloc<NodeStatic>(N);
    s->dLayers = s->alloc<DLayer>(s->hostLayers.size());
    CK(cudaMemcpyAsync(s->dNodes, nodes.data(), sizeof(NodeStatic) * N, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->dLayers, s->hostLayers.data(), sizeof(DLayer) * s->hostLayers.size(), cudaMemcpyHostToDevice, st));
    s->x = s->alloc<float4>(N);
    s->v = s->alloc<float4>(N);
    s->dx = s->alloc<float4>(N);
    s->pred = s->alloc<float4>(N);
    s->ext = s->alloc<float4>(3 * (size_t)N);
    if (prm->self_contact) {
      s->ctCells = s->alloc<unsigned>(2 * ((size_t)1 << CT_TABLE_BITS));
      s->ctScanTiles = s->alloc<unsigned>(CT_SCAN_MAX_TILES);
      s->ctItems = s->alloc<float4>(4 * (size_t)N);
      s->ctPairs = s->alloc<unsigned>((CT_K + 2) * (size_t)N);
      s->cmeta = s->alloc<float4>(2 * (size_t)N);
      s->ctAcc = s->alloc<int>(CT_ACC * (size_t)N);
      if (prm->cross_layer && sc->n_layers > 1) {
        s->xcCells = s->alloc<unsigned>(2 * ((size_t)XC_MASK + 1));
        s->xcItems = s->alloc<int>(N);
        // contact distance of a layer pair: the mean of their thicknesses (contact.ts:49-50)
        auto thick = [&](int l) { return l < sc->n_layers ? sc->layers[l].material.thickness : 0.0; };
        s->xcDist[0] = (float)(0.5 * (thick(0) + thick(1)));
        s->xcDist[1] = (float)(0.5 * (thick(0) + thick(2)));
        s->xcDist[2] = (float)(0.5 * (thick(1) + thick(2)));
        s->xcDist[3] = 0.f;
      }
    }
    s->dGripSlots = s->alloc<GripSlot>(GRIPS);
    s->dGripEntries = s->alloc<GripEntry>((size_t)GRIPS * GRIP_ENTRIES);
    s->dGripGoal = s->alloc<float4>(3 * GRIPS);
    s->gripOwner.assign(N, -1);
    s->delta = s->alloc<float4>(N);
    s->p = s->alloc<float4>(N);
    s->Ap = s->alloc<float4>(N);
    s->b0 = s->alloc<float4>(N);
    s->deltaD = s->alloc<double>(3 * (size_t)N);
    s->op64 = s->alloc<double2>((size_t)FINE64_PLANES * N);
    s->zPrev = s->alloc<float4>(N);
    s->segs = s->alloc<Seg>(2 * (size_t)N);
    s->softening = s->alloc<float>(2 * (size_t)N);
    s->failSite = s->alloc<float>(2 * (size_t)N);
    s->tails = s->alloc<float>(4 * (size_t)N);
    s->strain = s->alloc<float>(2 * (size_t)N);
    s->damage = s->alloc<uint8_t>(2 * (size_t)C);
    s->area = s->alloc<uint8_t>(2 * (size_t)C);
    s->sep = s->alloc<uint8_t>(2 * (size_t)C);
    s->marks = s->alloc<uint8_t>(2 * (size_t)C);
    s->strength = s->alloc<float>(2 * (size_t)C);

    // ---- scene state (kept on the host for resetState)
    s->x0.resize(N);
    for (int n = 0; n < N; ++n)
      s->x0[n] = make_float4((float)sc->position[3 * n], (float)sc->position[3 * n + 1], (float)sc->position[3 * n + 2], 0.f);
    s->segs0.resize(2 * (size_t)N);
    s->soft0.resize(2 * (size_t)N);
    s->fail0.resize(2 * (size_t)N);
    for (size_t q = 0; q < 2 * (size_t)N; ++q) {
      s->segs0[q] = {(float)sc->rest_length[q], (float)sc->intact[q], sc->cut_mask[q], (uint32_t)sc->seg_flags[q]};
      s->soft0[q] = (float)sc->softening[q];
      s->fail0[q] = sc->fail_site[q];
    }
    s->tails0.resize(4 * (size_t)N);
    for (size_t q = 0; q < 4 * (size_t)N; ++q) s->tails0[q] = (float)sc->tails[q];
    s->damage0.assign(sc->field_damage, sc->field_damage + 2 * (size_t)C);
    CK(cudaMemcpyAsync(s->softening, s->soft0.data(), sizeof(float) * 2 * N, cudaMemcpyHostToDevice, st));
    if (C > 0) {
      CK(cudaMemcpyAsync(s->area, sc->field_area, 2 * (size_t)C, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(s->strength, sc->field_strength, sizeof(float) * 2 * (size_t)C, cudaMemcpyHostToDevice, st));
    }

    // ---- multigrid levels (levelLayers, lattice.ts:302-310)
    std::vector<DLevelLayer> cur;
    for (int l = 0; l < sc->n_layers; ++l)
      cur.push_back({sc->layers[l].node_offset, sc->layers[l].nx, sc->layers[l].ny, 0});
    for (;;) {
      Level L;
      L.layers = cur;
      for (auto& ly : cur) L.N += ly.nx * ly.ny;
      L.fine = s->levels.empty();
      buildLines(L);
      s->levels.push_back(L);
      bool can = true;
      for (auto& ly : cur) can = can && ly.nx * ly.ny > 48 && ly.nx >= 5 && ly.ny >= 5;
      if (L.N <= prm->max_coarsest_nodes || !can) break;
      std::vector<DLevelLayer> nxt;
      int off = 0;
      for (auto& ly : cur) {
        DLevelLayer c{off, ly.nx / 2 + 1, ly.ny / 2 + 1, 0};
        off += c.nx * c.ny;
        nxt.push_back(c);
      }
      cur = nxt;
    }
    for (size_t k = 0; k < s->levels.size(); ++k) {
      Level& L = s->levels[k];
      L.dLayers = s->alloc<DLevelLayer>(L.layers.size());
      CK(cudaMemcpyAsync(L.dLayers, L.layers.data(), sizeof(DLevelLayer) * L.layers.size(), cudaMemcpyHostToDevice, st));
      std::vector<uint2> cc(L.N);
      for (size_t l = 0; l < L.layers.size(); ++l) {
        auto& ly = L.layers[l];
        for (int j = 0; j < ly.ny; ++j)
          for (int i = 0; i < ly.nx; ++i) cc[ly.offset + j * ly.nx + i] = make_uint2((uint32_t)i | ((uint32_t)j << 16), (uint32_t)l);
      }
      L.dCoord = s->alloc<uint2>(L.N);
      CK(cudaMemcpyAsync(L.dCoord, cc.data(), sizeof(uint2) * L.N, cudaMemcpyHostToDevice, st));
      L.dLines = s->alloc<int4>(L.lines.size());
      CK(cudaMemcpyAsync(L.dLines, L.lines.data(), sizeof(int4) * L.lines.size(), cudaMemcpyHostToDevice, st));
      L.dFacBase = s->alloc<int>(L.facBase.size());
      CK(cudaMemcpyAsync(L.dFacBase, L.facBase.data(), sizeof(int) * L.facBase.size(), cudaMemcpyHostToDevice, st));
      L.fac = s->alloc<float4>(L.facF4);
      L.op = s->alloc<float4>((size_t)(L.fine ? FINE_PLANES : COARSE_PLANES) * L.N);
      L.fixed = s->alloc<uint32_t>(L.N);
      if (k == 0) CK(cudaMemcpyAsync(L.fixed, pinned.data(), sizeof(uint32_t) * N, cudaMemcpyHostToDevice, st));
      L.X = s->alloc<float4>(L.N);
      L.B = s->alloc<float4>(L.N);
      L.R = s->alloc<float4>(L.N);
      L.pw = s->alloc<float4>(L.N);
      const size_t smem = L.fine ? smoothSmemBytes<FineRows>(L.maxLine, L.tile) : smoothSmemBytes<CoarseRows>(L.maxLine, L.tile);
      const size_t fsmem = L.fine ? factorSmemBytes<FineRows>(L.maxLine) : factorSmemBytes<CoarseRows>(L.maxLine);
      // (227 KB of opt-in shared memory a block, less the kernels' few bytes of static shared memory)
      if (L.maxLine > SM_MAX_LINE || smem > 226 * 1024 || fsmem > 226 * 1024)
        throw std::invalid_argument("yarn lines of " + std::to_string(L.maxLine) + " nodes exceed the smoother's shared memory");
    }

    // the smoother's dynamic shared memory: a kernel's limit is an attribute of the function, shared
    // by every solver of the process, so it is raised once to what the device allows beside the
    // kernel's static shared memory (a permission, not an allocation; each launch asks for what its
    // level's lines need, checked against the same bound above)
    {
      static std::once_flag smemOnce;
      static cudaError_t smemErr = cudaSuccess;
      std::call_once(smemOnce, [] {
        int dev = 0, optin = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        auto set = [&](const void* f) {
          cudaFuncAttributes fa;
          if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, f);
          if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
        };
        set((const void*)k_smooth<FineRows, 0>);
        set((const void*)k_smooth<FineRows, 1>);
        set((const void*)k_smooth<CoarseRows, 0>);
        set((const void*)k_smooth<CoarseRows, 1>);
        set((const void*)k_line_factor<FineRows>);
        set((const void*)k_line_factor<CoarseRows>);
        smemErr = e;
      });
      CK(smemErr);
    }

    // ---- parameters
    SimParams& P = s->hostP;
    P.h = (float)prm->h;
    P.gx = (float)prm->gravity[0];
    P.gy = (float)prm->gravity[1];
    P.gz = (float)prm->gravity[2];
    P.historyOn = 1;
    P.historyTol = (float)prm->history_tolerance;
    P.floorOn = 0;
    P.floorZ = 0;
    P.floorBulge = 0.3e-3f;
    P.floorStiffness = 1300.f;
    P.floorFriction = 0.35f;
    P.floorFrictionSpeed = 0.002f;
    P.pcgMax = prm->pcg_iterations;
    P.lineSearch = prm->line_search;
    P.pcgTol = prm->pcg_rel_tol;
    P.newtonTol = (float)prm->newton_tolerance;
    P.gradFp64 = 1;
    s->pushParams();

    // ---- initial state (resetState)
    CK(cudaMemcpyAsync(s->x, s->x0.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->segs, s->segs0.data(), sizeof(Seg) * 2 * N, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->failSite, s->fail0.data(), sizeof(float) * 2 * N, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->tails, s->tails0.data(), sizeof(float) * 4 * N, cudaMemcpyHostToDevice, st));
    if (C > 0) CK(cudaMemcpyAsync(s->damage, s->damage0.data(), 2 * (size_t)C, cudaMemcpyHostToDevice, st));
    s->sync();
    s->substepGraph(s->unconditional(0), s->gatedBound(0, 0));
    s->pcgExec = s->capture([&](cudaStream_t q) { s->encPCG(q); });
    s->sync();
    *out = s.release();
    return BTD_OK;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int btd_destroy(btd_solver* s) {
  if (!s) return BTD_OK;
  cudaStreamSynchronize(s->stream);
  delete s;
  return BTD_OK;
}

int btd_substep(btd_solver* s, int32_t min_iterations, int32_t max_iterations) {
  GUARD({
    checkSolver(s);
    s->runSubstep(min_iterations, max_iterations);
  });
}

int btd_substeps(btd_solver* s, int32_t count) {
  GUARD({
    checkSolver(s);
    if (!s->useGraphs) {
      for (int k = 0; k < count; ++k) s->runSubstepEager(s->unconditional(0), s->gatedBound(0, 0));
    } else {
      cudaGraphExec_t ex = s->substepGraph(s->unconditional(0), s->gatedBound(0, 0));
      for (int k = 0; k < count; ++k) CK(cudaGraphLaunch(ex, s->stream));
    }
  });
}

int btd_batch_substeps(btd_solver* const* solvers, int32_t count, int32_t substeps) {
  GUARD({
    if (!solvers || count < 0 || substeps < 0) throw std::invalid_argument("bad batch");
    std::vector<cudaGraphExec_t> graphs(count, nullptr);
    for (int b = 0; b < count; ++b) {
      btd_solver* s = solvers[b];
      checkSolver(s);
      if (s->useGraphs) graphs[b] = s->substepGraph(s->unconditional(0), s->gatedBound(0, 0));
    }
    // round robin: every patch's next substep is queued before any patch's one after, so all
    // streams have work from the start
    for (int k = 0; k < substeps; ++k)
      for (int b = 0; b < count; ++b) {
        btd_solver* s = solvers[b];
        if (graphs[b])
          CK(cudaGraphLaunch(graphs[b], s->stream));
        else
          s->runSubstepEager(s->unconditional(0), s->gatedBound(0, 0));
      }
  });
}

}  // extern "C"

// A batch of solvers stepped by one graph: one substep of every solver, each on its own stream inside
// one capture (forked from and joined to the batch stream), so a whole batch substep is one
// cudaGraphLaunch whose branches the device runs side by side (each with its own device-side PCG loops).
struct btd_batch {
  std::vector<btd_solver*> solvers;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  std::vector<cudaEvent_t> ready, done;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
  ~btd_batch() {
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    for (cudaEvent_t e : ready) cudaEventDestroy(e);
    for (cudaEvent_t e : done) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (stream) cudaStreamDestroy(stream);
  }
  void capture() {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
    try {
      CK(cudaEventRecord(fork, stream));
      for (size_t b = 0; b < solvers.size(); ++b) {
        btd_solver* s = solvers[b];
        CK(cudaStreamWaitEvent(s->stream, fork, 0));
        s->encSubstep(s->stream, s->unconditional(0), s->gatedBound(0, 0), s->gripsOn());
        CK(cudaEventRecord(done[b], s->stream));
        CK(cudaStreamWaitEvent(stream, done[b], 0));
      }
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cudaGraph_t g;
    CK(cudaStreamEndCapture(stream, &g));
    cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    CK(e);
  }
};

extern "C" {

int btd_batch_create(btd_solver* const* solvers, int32_t count, btd_batch** out) {
  if (!solvers || count < 1 || !out) {
    btd::setError("btd_batch_create: solvers, count >= 1 and an output");
    return BTD_E_INVALID;
  }
  std::unique_ptr<btd_batch> b(new btd_batch());
  GUARD({
    for (int k = 0; k < count; ++k) {
      checkSolver(solvers[k]);
      if (!solvers[k]->useGraphs) throw std::invalid_argument("btd_batch_create: a solver in eager mode");
      for (int q = 0; q < k; ++q)
        if (solvers[q] == solvers[k]) throw std::invalid_argument("btd_batch_create: a solver twice");
    }
    b->solvers.assign(solvers, solvers + count);
    CK(cudaGetDevice(&b->device));
    CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming));
    b->ready.resize(count);
    b->done.resize(count);
    for (int k = 0; k < count; ++k) {
      CK(cudaEventCreateWithFlags(&b->ready[k], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&b->done[k], cudaEventDisableTiming));
    }
    for (btd_solver* s : b->solvers) s->sync();
    b->capture();
    for (btd_solver* s : b->solvers) s->batchGrips = s->gripsOn();
    *out = b.release();
  });
}

int btd_batch_destroy(btd_batch* b) {
  delete b;
  return BTD_OK;
}

int btd_batch_run(btd_batch* b, int32_t substeps) {
  GUARD({
    if (!b || substeps < 0) throw std::invalid_argument("btd_batch_run: null batch or negative count");
    // a grip attached or released since the capture changes a solver's substep: capture again
    bool stale = false;
    for (btd_solver* s : b->solvers) stale = stale || s->gripsOn() != s->batchGrips;
    if (stale) {
      for (btd_solver* s : b->solvers) s->sync();
      b->capture();
      for (btd_solver* s : b->solvers) s->batchGrips = s->gripsOn();
    }
    for (int k = 0; k < substeps; ++k) {
      // the batch stream waits for what each solver's stream holds (grip targets, state writes),
      // then every solver's stream waits for the batch substep
      for (size_t q = 0; q < b->solvers.size(); ++q) {
        CK(cudaEventRecord(b->ready[q], b->solvers[q]->stream));
        CK(cudaStreamWaitEvent(b->stream, b->ready[q], 0));
      }
      CK(cudaGraphLaunch(b->exec, b->stream));
      CK(cudaEventRecord(b->join, b->stream));
      for (btd_solver* s : b->solvers) CK(cudaStreamWaitEvent(s->stream, b->join, 0));
    }
  });
}

int btd_synchronize(btd_solver* s) {
  GUARD({
    checkSolver(s);
    uint32_t flags = 0;
    CK(cudaMemcpyAsync(&flags, s->dCounters + CNT_ERROR, sizeof flags, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    if (flags) {
      CK(cudaMemsetAsync(s->dCounters + CNT_ERROR, 0, sizeof flags, s->stream));
      s->sync();
      throw DeviceTimeout("a bounded device-side wait ran out (flags 0x" + std::to_string(flags) + "); results since the last synchronize are unreliable");
    }
  });
}

int btd_set_state(btd_solver* s, const float* pos4, const float* vel4) {
  GUARD({
    checkSolver(s);
    if (!pos4) throw std::invalid_argument("null positions");
    CK(cudaMemcpyAsync(s->x, pos4, sizeof(float4) * s->N, cudaMemcpyHostToDevice, s->stream));
    if (vel4)
      CK(cudaMemcpyAsync(s->v, vel4, sizeof(float4) * s->N, cudaMemcpyHostToDevice, s->stream));
    else
      CK(cudaMemsetAsync(s->v, 0, sizeof(float4) * s->N, s->stream));
    s->sync();
  });
}

int btd_get_state(btd_solver* s, float* pos4, float* vel4) {
  GUARD({
    checkSolver(s);
    if (pos4) CK(cudaMemcpyAsync(pos4, s->x, sizeof(float4) * s->N, cudaMemcpyDeviceToHost, s->stream));
    if (vel4) CK(cudaMemcpyAsync(vel4, s->v, sizeof(float4) * s->N, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
  });
}

int btd_set_segments(btd_solver* s, const float* rest, const float* intact, const uint32_t* cut, const uint32_t* flags,
                     const float* fail_site, const float* tails) {
  GUARD({
    checkSolver(s);
    const size_t n2 = 2 * (size_t)s->N;
    std::vector<Seg> sg(n2);
    CK(cudaMemcpyAsync(sg.data(), s->segs, sizeof(Seg) * n2, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    for (size_t q = 0; q < n2; ++q) {
      if (rest) sg[q].rest = rest[q];
      if (intact) sg[q].intact = intact[q];
      if (cut) sg[q].cutMask = cut[q];
      if (flags) sg[q].flags = flags[q];
    }
    CK(cudaMemcpyAsync(s->segs, sg.data(), sizeof(Seg) * n2, cudaMemcpyHostToDevice, s->stream));
    if (fail_site) CK(cudaMemcpyAsync(s->failSite, fail_site, sizeof(float) * n2, cudaMemcpyHostToDevice, s->stream));
    if (tails) CK(cudaMemcpyAsync(s->tails, tails, sizeof(float) * 4 * s->N, cudaMemcpyHostToDevice, s->stream));
    s->sync();
  });
}

int btd_get_segments(btd_solver* s, float* rest, float* intact, uint32_t* cut, uint32_t* flags, float* fail_site, float* tails) {
  GUARD({
    checkSolver(s);
    const size_t n2 = 2 * (size_t)s->N;
    std::vector<Seg> sg(n2);
    CK(cudaMemcpyAsync(sg.data(), s->segs, sizeof(Seg) * n2, cudaMemcpyDeviceToHost, s->stream));
    if (fail_site) CK(cudaMemcpyAsync(fail_site, s->failSite, sizeof(float) * n2, cudaMemcpyDeviceToHost, s->stream));
    if (tails) CK(cudaMemcpyAsync(tails, s->tails, sizeof(float) * 4 * s->N, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    for (size_t q = 0; q < n2; ++q) {
      if (rest) rest[q] = sg[q].rest;
      if (intact) intact[q] = sg[q].intact;
      if (cut) cut[q] = sg[q].cutMask;
      if (flags) flags[q] = sg[q].flags;
    }
  });
}

int btd_set_field(btd_solver* s, const uint8_t* damage) {
  GUARD({
    checkSolver(s);
    if (s->C > 0) CK(cudaMemcpyAsync(s->damage, damage, 2 * (size_t)s->C, cudaMemcpyHostToDevice, s->stream));
    s->sync();
  });
}

int btd_get_field(btd_solver* s, uint8_t* damage) {
  GUARD({
    checkSolver(s);
    if (s->C > 0) CK(cudaMemcpyAsync(damage, s->damage, 2 * (size_t)s->C, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
  });
}

int btd_reset_state(btd_solver* s) {
  GUARD({
    checkSolver(s);
    const int N = s->N;
    CK(cudaMemcpyAsync(s->x, s->x0.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemsetAsync(s->v, 0, sizeof(float4) * N, s->stream));
    CK(cudaMemcpyAsync(s->segs, s->segs0.data(), sizeof(Seg) * 2 * N, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->failSite, s->fail0.data(), sizeof(float) * 2 * N, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->tails, s->tails0.data(), sizeof(float) * 4 * N, cudaMemcpyHostToDevice, s->stream));
    if (s->C > 0) CK(cudaMemcpyAsync(s->damage, s->damage0.data(), 2 * (size_t)s->C, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemsetAsync(s->ext, 0, sizeof(float4) * 3 * N, s->stream));
    s->sync();
  });
}

int btd_set_floor(btd_solver* s, int32_t enabled, float z) {
  GUARD({
    checkSolver(s);
    s->hostP.floorOn = enabled ? 1 : 0;
    s->hostP.floorZ = z;
    s->pushParams();
    s->sync();
  });
}

int btd_set_timestep(btd_solver* s, float h) {
  GUARD({
    checkSolver(s);
    if (!(h > 0)) throw std::invalid_argument("h must be positive");
    s->hostP.h = h;
    s->params.h = h;
    s->pushParams();
    s->sync();
  });
}

int btd_set_history(btd_solver* s, int32_t on) {
  GUARD({
    checkSolver(s);
    s->hostP.historyOn = on ? 1 : 0;
    s->pushParams();
    s->sync();
  });
}

int btd_set_newton_tolerance(btd_solver* s, float tol) {
  GUARD({
    checkSolver(s);
    s->hostP.newtonTol = tol;
    s->params.newton_tolerance = tol;
    s->pushParams();
    s->sync();
  });
}

int btd_set_graph_mode(btd_solver* s, int32_t use_graphs) {
  GUARD({
    checkSolver(s);
    s->useGraphs = use_graphs != 0;
  });
}

int btd_set_gradient_precision(btd_solver* s, int32_t fp64) {
  GUARD({
    checkSolver(s);
    s->hostP.gradFp64 = fp64 ? 1 : 0;
    s->pushParams();
    s->sync();
  });
}

int btd_set_pcg_flexible(btd_solver* s, int32_t on) {
  GUARD({
    checkSolver(s);
    s->hostP.pcgFlex = on ? 1 : 0;
    s->pushParams();
    s->sync();
  });
}

static void resetGraphs(btd_solver* s);

int btd_set_operator_precision(btd_solver* s, int32_t fp64) {
  GUARD({
    checkSolver(s);
    if ((fp64 != 0) != s->opFp64) {
      s->opFp64 = fp64 != 0;
      resetGraphs(s);
    }
  });
}

int btd_set_pcg(btd_solver* s, int32_t max_iterations, double rel_tol) {
  GUARD({
    checkSolver(s);
    if (max_iterations < 1) throw std::invalid_argument("max_iterations must be >= 1");
    s->hostP.pcgMax = max_iterations;
    s->hostP.pcgTol = rel_tol;
    s->params.pcg_iterations = max_iterations;
    s->params.pcg_rel_tol = rel_tol;
    s->pushParams();
    s->sync();
  });
}

int btd_read_counters(btd_solver* s, uint32_t* out, int32_t n) {
  GUARD({
    checkSolver(s);
    if (!out || n < 0 || n > CNT_SIZE) throw std::invalid_argument("bad counter count");
    CK(cudaMemcpyAsync(out, s->dCounters, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
  });
}

// settleDrape (settle.ts:24-62): 420 substeps of 5 Newton iterations with a fixed 2 PCG iterations,
// history off (pre-tension must not tear), velocities cleared after every tenth of the first 360
// (kinetic damping), then velocities and counters cleared; the solver's settings come back after.
int btd_settle_drape(btd_solver* s) {
  GUARD({
    checkSolver(s);
    constexpr int SETTLE_STEPS = 420, SETTLE_DAMPED = 360, SETTLE_NEWTON = 5, SETTLE_PCG = 2;
    const SimParams savedP = s->hostP;
    const btd_params savedPrm = s->params;
    auto restore = [&] {
      s->hostP = savedP;
      s->params = savedPrm;
      s->pushParams();
    };
    s->hostP.pcgMax = SETTLE_PCG;
    s->hostP.pcgTol = 0.0;
    s->hostP.historyOn = 0;
    s->params.pcg_iterations = SETTLE_PCG;
    s->params.pcg_rel_tol = 0.0;
    s->pushParams();
    try {
      for (int k = 0; k < SETTLE_STEPS; ++k) {
        s->runSubstep(SETTLE_NEWTON, SETTLE_NEWTON);
        if (k % 10 == 9 && k < SETTLE_DAMPED) CK(cudaMemsetAsync(s->v, 0, sizeof(float4) * s->N, s->stream));
      }
      CK(cudaMemsetAsync(s->v, 0, sizeof(float4) * s->N, s->stream));
      CK(cudaMemsetAsync(s->dCounters, 0, sizeof(uint32_t) * CNT_SIZE, s->stream));
    } catch (...) {
      restore();
      throw;
    }
    restore();
    s->sync();
  });
}

int btd_clear_counters(btd_solver* s) {
  GUARD({
    checkSolver(s);
    CK(cudaMemsetAsync(s->dCounters, 0, sizeof(uint32_t) * CNT_SIZE, s->stream));
    s->sync();
  });
}

int btd_stage_predict(btd_solver* s) {
  GUARD({
    checkSolver(s);
    s->encPredict(s->stream, s->gripsOn());
    CK(cudaGetLastError());
    s->sync();
  });
}

int btd_stage_assemble(btd_solver* s, int32_t coarse) {
  GUARD({
    checkSolver(s);
    s->encAssemble(s->stream, coarse != 0);
    CK(cudaGetLastError());
    s->sync();
  });
}

int btd_stage_vcycle(btd_solver* s) {
  GUARD({
    checkSolver(s);
    CK(cudaMemsetAsync(s->levels[0].X, 0, sizeof(float4) * s->N, s->stream));
    s->encVCycle(s->stream, 0);
    CK(cudaGetLastError());
    s->sync();
  });
}

int btd_stage_smooth(btd_solver* s, int32_t level, int32_t reverse) {
  GUARD({
    checkSolver(s);
    if (level < 0 || level >= (int)s->levels.size()) throw std::invalid_argument("level out of range");
    s->encSmooth(s->stream, level, reverse != 0);
    CK(cudaGetLastError());
    s->sync();
  });
}

int btd_stage_pcg(btd_solver* s) {
  GUARD({
    checkSolver(s);
    CK(cudaGraphLaunch(s->pcgExec, s->stream));
    s->sync();
  });
}

int btd_stage_linesearch(btd_solver* s, double* e4, double* m4) {
  GUARD({
    checkSolver(s);
    s->encLineSearch(s->stream);
    CK(cudaGetLastError());
    Scalars sc;
    CK(cudaMemcpyAsync(&sc, s->dScal, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    for (int k = 0; k < 4; ++k) {
      if (e4) e4[k] = sc.e[k];
      if (m4) m4[k] = sc.m[k];
    }
  });
}

int btd_stage_apply(btd_solver* s, int32_t it) {
  GUARD({
    checkSolver(s);
    s->encApply(s->stream, it);
    CK(cudaGetLastError());
    s->sync();
  });
}

int btd_stage_newton(btd_solver* s, int32_t it) {
  GUARD({
    checkSolver(s);
    cudaGraphExec_t ex = s->capture([&](cudaStream_t q) { s->encNewton(q, it, s->gripsOn()); });
    cudaError_t e = cudaGraphLaunch(ex, s->stream);
    cudaError_t e2 = cudaStreamSynchronize(s->stream);
    cudaGraphExecDestroy(ex);
    CK(e);
    CK(e2);
  });
}

int btd_stage_finalize(btd_solver* s) {
  GUARD({
    checkSolver(s);
    s->encFinalize(s->stream);
    CK(cudaGetLastError());
    s->sync();
  });
}

int btd_stage_damage(btd_solver* s) {
  GUARD({
    checkSolver(s);
    s->encDamage(s->stream);
    CK(cudaGetLastError());
    s->sync();
  });
}

// ---------------------------------------------------------------- grips (interaction.ts:223-318)

static_assert(GRIPS == BTD_GRIPS && GRIP_ENTRIES == BTD_GRIP_ENTRIES, "grip limits differ from btd.h");
static_assert(LC_WEIGHTS == BTD_LEARNED_WEIGHTS && LC_K == BTD_LEARNED_K && LC_MAX_NODES == BTD_LEARNED_MAX_NODES,
              "learned correction sizes differ from btd.h");
static_assert(sizeof(GripEntry) == 32 && sizeof(GripSlot) == 64, "grip layout");

static void checkSlot(btd_solver* s, int32_t slot) {
  checkSolver(s);
  if (slot < 0 || slot >= GRIPS) throw std::invalid_argument("grip slot " + std::to_string(slot) + " outside [0, " + std::to_string(GRIPS) + ")");
}

static void pushGrip(btd_solver* s, int32_t slot) {
  k_grip_set_slot<<<1, 1, 0, s->stream>>>(s->dGripSlots, slot, s->hostGrip[slot]);
  CK(cudaGetLastError());
}

// release (interaction.ts:302-313): the slot's count drops to zero; without contact the grips own
// ext, which is cleared (the remaining grips rewrite their entries every iteration).
static void releaseGrip(btd_solver* s, int32_t slot) {
  if (s->hostGrip[slot].goal.w <= 0.f) return;
  for (int n = 0; n < s->N; ++n)
    if (s->gripOwner[n] == slot) s->gripOwner[n] = -1;
  s->hostGrip[slot].goal.w = 0.f;
  pushGrip(s, slot);
  if (!s->params.self_contact) CK(cudaMemsetAsync(s->ext, 0, sizeof(float4) * 3 * (size_t)s->N, s->stream));
}

int btd_set_grip(btd_solver* s, int32_t slot, const int32_t* nodes, const float* weights, const float* sides, int32_t count,
                 int32_t picked, const float* anchor, float stiffness, float max_lead, float pad_pitch, float slip) {
  GUARD({
    checkSlot(s, slot);
    if (!nodes || !weights || !anchor) throw std::invalid_argument("null grip nodes, weights or anchor");
    if (count < 1 || count > GRIP_ENTRIES)
      throw std::invalid_argument("grip entry count " + std::to_string(count) + " outside [1, " + std::to_string(GRIP_ENTRIES) + "]");
    if (picked < 0 || picked >= s->N) throw std::invalid_argument("picked node outside the lattice");
    if (!(std::isfinite(stiffness) && stiffness >= 0.f)) throw std::invalid_argument("grip stiffness must be finite and >= 0");
    if (!(max_lead > 0.f)) throw std::invalid_argument("grip max_lead must be > 0");
    if (!(std::isfinite(pad_pitch) && pad_pitch >= 0.f) || !(std::isfinite(slip) && slip >= 0.f))
      throw std::invalid_argument("grip pad_pitch and slip must be finite and >= 0");
    for (int q = 0; q < 3; ++q)
      if (!std::isfinite(anchor[q])) throw std::invalid_argument("grip anchor must be finite");
    releaseGrip(s, slot);
    // a node belongs to one patch at most, so every ext entry has one writer (interact.wgsl:4-6)
    std::vector<GripEntry> entries(count);
    std::vector<int> sorted(nodes, nodes + count);
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end()) throw std::invalid_argument("a node appears twice in one grip patch");
    for (int k = 0; k < count; ++k) {
      const int n = nodes[k];
      const float sd = sides ? sides[k] : 0.f;
      if (n < 0 || n >= s->N) throw std::invalid_argument("grip node " + std::to_string(n) + " outside the lattice");
      if (s->gripOwner[n] >= 0) throw std::invalid_argument("node " + std::to_string(n) + " is held by grip " + std::to_string(s->gripOwner[n]));
      if (!(std::isfinite(weights[k]) && weights[k] >= 0.f)) throw std::invalid_argument("grip weights must be finite and >= 0");
      if (sd != 0.f && sd != 1.f && sd != -1.f) throw std::invalid_argument("grip sides must be -1, 0 or +1");
      entries[k] = GripEntry{(uint32_t)n, weights[k], sd, 0.f, make_float4(0, 0, 0, 0)};
    }
    for (int k = 0; k < count; ++k) s->gripOwner[nodes[k]] = (int8_t)slot;
    GripSlot& S = s->hostGrip[slot];
    uint32_t pk = (uint32_t)picked;
    float pkBits;
    std::memcpy(&pkBits, &pk, sizeof pkBits);
    S.goal = make_float4(anchor[0], anchor[1], anchor[2], (float)count);
    S.params = make_float4(stiffness, max_lead, pkBits, 1.f);
    S.anchor = make_float4(anchor[0], anchor[1], anchor[2], pad_pitch);
    S.hold = make_float4(slip, 0.f, 0.f, 0.f);
    s->gripStiffness[slot] = stiffness;
    CK(cudaMemcpyAsync(s->dGripEntries + (size_t)slot * GRIP_ENTRIES, entries.data(), sizeof(GripEntry) * count,
                       cudaMemcpyHostToDevice, s->stream));
    pushGrip(s, slot);
    k_grip_init<<<blocksFor(count, 64), 64, 0, s->stream>>>(s->gripArgs(), slot);
    CK(cudaGetLastError());
    s->sync();
  });
}

int btd_set_grip_target(btd_solver* s, int32_t slot, const float* target) {
  GUARD({
    checkSlot(s, slot);
    if (!target) throw std::invalid_argument("null grip target");
    GripSlot& S = s->hostGrip[slot];
    if (S.goal.w <= 0.f) return BTD_OK;
    S.goal = make_float4(target[0], target[1], target[2], S.goal.w);
    pushGrip(s, slot);
  });
}

int btd_set_grip_pinch(btd_solver* s, int32_t slot, float scale) {
  GUARD({
    checkSlot(s, slot);
    if (s->hostGrip[slot].goal.w <= 0.f) return BTD_OK;
    s->hostGrip[slot].params.w = scale;
    pushGrip(s, slot);
  });
}

int btd_set_grip_hold(btd_solver* s, int32_t slot, float fraction) {
  GUARD({
    checkSlot(s, slot);
    if (s->hostGrip[slot].goal.w <= 0.f) return BTD_OK;
    s->hostGrip[slot].params.x = s->gripStiffness[slot] * fraction;
    pushGrip(s, slot);
  });
}

int btd_release_grip(btd_solver* s, int32_t slot) {
  GUARD({
    checkSlot(s, slot);
    releaseGrip(s, slot);
    s->sync();
  });
}

int btd_read_grip(btd_solver* s, int32_t slot, int32_t* nodes, float* weights, int32_t capacity, float* handle12,
                  int32_t* count) {
  GUARD({
    checkSlot(s, slot);
    const int n = (int)s->hostGrip[slot].goal.w;
    if (count) *count = n;
    std::vector<GripEntry> e(std::max(n, 1));
    float4 goal[3];
    if (n > 0)
      CK(cudaMemcpyAsync(e.data(), s->dGripEntries + (size_t)slot * GRIP_ENTRIES, sizeof(GripEntry) * n, cudaMemcpyDeviceToHost,
                         s->stream));
    CK(cudaMemcpyAsync(goal, s->dGripGoal + 3 * slot, sizeof goal, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    for (int k = 0; k < std::min(n, (int)capacity); ++k) {
      if (nodes) nodes[k] = (int32_t)e[k].node;
      if (weights) weights[k] = e[k].w;
    }
    if (handle12) std::memcpy(handle12, goal, sizeof goal);
  });
}

static void resetGraphs(btd_solver* s);

// The sweep's launch shape per level, chosen by measurement: for every level the CTA size (a multiple of
// 32 from 64 to SM_SWEEP_THREADS) and, on lines longer than 128 nodes, the staging tile (the whole line
// or 128 nodes) are timed on the level's current operator with CUDA events (the mean of `reps` sweeps
// after one untimed), and the fastest is kept. A sweep's arithmetic does not depend on either (every
// loop strides by the CTA size; a tile only changes how much of the line is staged at once), so the
// results are the same bit for bit. The captured graphs are dropped and captured again with the choice.
int btd_autotune(btd_solver* s, int32_t reps, int32_t* threads_out, int32_t* tile_out, float* ms_out) {
  GUARD({
    checkSolver(s);
    if (reps < 1) throw std::invalid_argument("btd_autotune: reps >= 1");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (size_t k = 0; k < s->levels.size(); ++k) {
      Level& L = s->levels[k];
      std::vector<int> tiles{L.tile};
      if (L.maxLine > 128 && L.tile != 128) tiles.push_back(128);
      int bestT = L.threads, bestTile = L.tile;
      float best = 1e30f;
      for (int tile : tiles)
        for (int T = 64; T <= SM_SWEEP_THREADS; T += 32) {
          L.tile = tile;
          L.threads = T;
          s->encSmooth(s->stream, (int)k, false);  // untimed: first touch
          CK(cudaEventRecord(e0, s->stream));
          for (int r = 0; r < reps; ++r) s->encSmooth(s->stream, (int)k, false);
          CK(cudaEventRecord(e1, s->stream));
          CK(cudaEventSynchronize(e1));
          float t = 0.f;
          CK(cudaEventElapsedTime(&t, e0, e1));
          t /= reps;
          if (t < best) best = t, bestT = T, bestTile = tile;
        }
      L.threads = bestT;
      L.tile = bestTile;
      if (threads_out) threads_out[k] = bestT;
      if (tile_out) tile_out[k] = bestTile;
      if (ms_out) ms_out[k] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaGetLastError());
    resetGraphs(s);
  });
}

int btd_profile_stage(btd_solver* s, int32_t which, int32_t reps, int32_t flush, float* ms) {
  GUARD({
    checkSolver(s);
    if (!ms || reps < 1 || which < 0 || which > 5) throw std::invalid_argument("bad profile request");
    const size_t flushBytes = size_t(256) << 20;
    if (flush && !s->flushBuf) CK(cudaMalloc(&s->flushBuf, flushBytes));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float total = 0.f;
    PcgArgs pa = s->pcgArgs(0, 0);
    for (int r = 0; r < reps; ++r) {
      if (flush) CK(cudaMemsetAsync(s->flushBuf, r & 0xff, flushBytes, s->stream));
      CK(cudaEventRecord(e0, s->stream));
      switch (which) {
        case BTD_STAGE_MATVEC:
          k_pcg_matvec<<<s->redBlocks, RED_THREADS, 0, s->stream>>>(pa);
          break;
        case BTD_STAGE_SMOOTH:
          s->encSmooth(s->stream, 0, false);
          break;
        case BTD_STAGE_ASSEMBLE:
          s->encAssemble(s->stream, false);
          break;
        case BTD_STAGE_VCYCLE:
          CK(cudaMemsetAsync(s->levels[0].X, 0, sizeof(float4) * s->N, s->stream));
          s->encVCycle(s->stream, 0);
          break;
        case BTD_STAGE_HIERARCHY:
          s->encHierarchy(s->stream);
          break;
        default:
          s->runSubstep(0, 0);
      }
      CK(cudaEventRecord(e1, s->stream));
      CK(cudaEventSynchronize(e1));
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, e0, e1));
      total += t;
    }
    CK(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = total / reps;
  });
}

int btd_launch_count(btd_solver* s, int32_t substeps, int32_t newton, int32_t pcg, int64_t* out) {
  GUARD({
    checkSolver(s);
    if (!out) throw std::invalid_argument("null output");
    auto colours = [&](int k) {
      int c = 0;
      for (int q = 0; q < 6; ++q) c += s->levels[k].colourStart[q + 1] > s->levels[k].colourStart[q];
      return (int64_t)c;
    };
    const int L = (int)s->levels.size();
    const int64_t lc = s->lcOn() ? 1 : 0;
    int64_t V = s->params.coarse_sweeps * colours(L - 1) + lc;
    for (int k = 0; k + 1 < L; ++k) V += 2 * colours(k) + 3;
    // per Newton iteration: assembly, PCG prologue (init + V-cycle + 5), line search, apply; the
    // hierarchy (weights + RAP per coarse level) on the first iteration; V-cycle + 5 per extra PCG pass
    // held grips add their lead once per substep and their terms once per Newton iteration; the
    // assembly and every Galerkin product are followed by their level's line factorisation
    const int64_t grips = s->gripsOn() ? 1 : 0;
    // self-contact adds detection (7 kernels, the scan two of them) once per substep and terms + gather
    // per Newton iteration
    const int64_t contact = s->contactOn() ? 1 : 0;
    // detached pieces add rotation + frame after the assembly, start (+ the init it replaces) and curves
    const int64_t rigid = s->pieceCount > 0 ? 1 : 0;
    const int64_t xc = s->xcOn() ? 1 : 0;  // cross-layer contact: terms in one kernel, detection in five
    // the learned correction adds its flags (fine, then one a coarse level) and basis to every solve
    const int64_t perNewton = 2 + (1 + V + 5) + 1 + 1 + grips + (2 - xc) * contact + 4 * rigid + lc * (L + 1);
    const int64_t hierarchy = 3 * (L - 1);
    const int64_t hierPerSubstep = s->params.lag_coarse ? hierarchy : hierarchy * (newton / std::max(1, substeps));
    const int64_t perSubstep = 2 + 1 + 5 + s->nLayers + 4 + grips + (7 - 2 * xc) * contact + 2 * rigid;
    // each optional (gated) Newton iteration slot adds its gate kernel, run or not
    const int64_t gates = s->gatedBound(0, 0) - s->unconditional(0);
    *out = (int64_t)substeps * (perSubstep + hierPerSubstep + gates) + (int64_t)newton * perNewton + (int64_t)(pcg - newton) * (V + 5);
  });
}

// ---------------------------------------------------------------- learned coarse correction (extension)

// Drops the captured graphs (they are captured again with the current settings on their next use).
static void resetGraphs(btd_solver* s) {
  s->sync();
  for (auto& kv : s->substepExec) cudaGraphExecDestroy(kv.second);
  s->substepExec.clear();
  if (s->pcgExec) cudaGraphExecDestroy(s->pcgExec);
  s->pcgExec = s->capture([&](cudaStream_t q) { s->encPCG(q); });
}

static void learnedAlloc(btd_solver* s) {
  if (s->dLc) return;
  const Level& C = s->levels.back();
  if (C.layers.size() != 1) throw std::invalid_argument("the learned coarse correction needs a single-layer lattice");
  if (C.N > LC_MAX_NODES)
    throw std::invalid_argument("the coarsest level has " + std::to_string(C.N) + " nodes; the learned coarse correction holds at most " +
                                std::to_string(LC_MAX_NODES) + " (lower max_coarsest_nodes)");
  static std::once_flag once;
  static cudaError_t err = cudaSuccess;
  std::call_once(once, [] {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void*)k_lc_basis);
    if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)k_lc_basis, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    err = e;
  });
  CK(err);
  s->dLc = s->alloc<LcState>(1);
  s->dNet = s->alloc<MlpPacked>(1);
  s->dLcW = s->alloc<float>(LC_WEIGHTS);
  s->lcPhi = s->alloc<float>((size_t)3 * C.N * LC_K);
  s->lcCtFlag = s->alloc<uint8_t>(s->N);
  s->lcBasisFlags = s->alloc<uint8_t>(C.N);
  for (const Level& L : s->levels) s->lcFlags.push_back(s->alloc<uint8_t>(L.N));
}

extern "C" int btd_set_learned(btd_solver* s, const float* weights, int32_t count, int32_t on, double guard) {
  GUARD({
    checkSolver(s);
    if (on && (!weights || count != LC_WEIGHTS))
      throw std::invalid_argument("btd_set_learned: the network needs " + std::to_string(LC_WEIGHTS) + " weights");
    if (weights) {
      if (count != LC_WEIGHTS) throw std::invalid_argument("btd_set_learned: the network needs " + std::to_string(LC_WEIGHTS) + " weights");
      for (int q = 0; q < count; ++q)
        if (!std::isfinite(weights[q])) throw std::invalid_argument("btd_set_learned: non-finite weight");
    }
    if (!(guard > 0.0)) throw std::invalid_argument("btd_set_learned: guard must be positive");
    const bool wasOn = s->lcEnabled;
    if (on || weights) learnedAlloc(s);
    if (weights) {
      CK(cudaMemcpyAsync(s->dLcW, weights, sizeof(float) * LC_WEIGHTS, cudaMemcpyHostToDevice, s->stream));
      k_mlp_pack<<<1, 256, 0, s->stream>>>(s->dLcW, s->dNet);
      CK(cudaGetLastError());
    }
    if (s->dLc) {
      LcState st;
      CK(cudaMemcpyAsync(&st, s->dLc, sizeof st, cudaMemcpyDeviceToHost, s->stream));
      s->sync();
      st.on = on ? 1 : 0;
      st.guard = (float)guard;
      if (weights) st.basisGen = -1;  // a new network: the next solve builds its basis
      CK(cudaMemcpyAsync(s->dLc, &st, sizeof st, cudaMemcpyHostToDevice, s->stream));
    }
    // the kernels stay in the graphs while logging, so a solver that only logs keeps them too
    s->lcEnabled = on != 0 || (s->dLc && s->lcLog.R);
    if (s->lcEnabled != wasOn) resetGraphs(s);
    s->sync();
  });
}

extern "C" int btd_learned_stats(btd_solver* s, int64_t* out) {
  GUARD({
    checkSolver(s);
    if (!out) throw std::invalid_argument("null output");
    LcState st{};
    if (s->dLc) {
      CK(cudaMemcpyAsync(&st, s->dLc, sizeof st, cudaMemcpyDeviceToHost, s->stream));
      s->sync();
    }
    out[0] = st.solves, out[1] = st.applied, out[2] = st.fallbacks, out[3] = st.nOps, out[4] = st.nCalls;
  });
}

extern "C" int btd_learned_basis(btd_solver* s, float* phi, double* G, int32_t* dead, uint8_t* flags, int32_t* nodes) {
  GUARD({
    checkSolver(s);
    if (!s->dLc) throw std::invalid_argument("btd_learned_basis: the learned correction was never set");
    const Level& C = s->levels.back();
    if (nodes) *nodes = C.N;
    LcState st;
    CK(cudaMemcpyAsync(&st, s->dLc, sizeof st, cudaMemcpyDeviceToHost, s->stream));
    if (phi) CK(cudaMemcpyAsync(phi, s->lcPhi, sizeof(float) * 3 * (size_t)C.N * LC_K, cudaMemcpyDeviceToHost, s->stream));
    if (flags) CK(cudaMemcpyAsync(flags, s->lcFlags.back(), C.N, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    if (G) std::memcpy(G, st.G, sizeof st.G);
    if (dead)
      for (int k = 0; k < LC_K; ++k) dead[k] = st.basisOk ? st.dead[k] : -1;
  });
}

extern "C" int btd_learned_log(btd_solver* s, int32_t on, int32_t cap_ops, int32_t cap_calls) {
  GUARD({
    checkSolver(s);
    if (on && (cap_ops < 1 || cap_calls < 1)) throw std::invalid_argument("btd_learned_log: capacities must be >= 1");
    learnedAlloc(s);
    const int M = s->levels.back().N;
    const bool wasOn = s->lcEnabled;
    LcState st;
    CK(cudaMemcpyAsync(&st, s->dLc, sizeof st, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    if (on) {
      auto fits = [](int cap, size_t each) { return (size_t)cap * each <= (size_t(8) << 30); };
      if (!fits(cap_ops, sizeof(float4) * COARSE_PLANES * M) || !fits(cap_calls, sizeof(float) * 3 * M))
        throw std::invalid_argument("btd_learned_log: capacities above 8 GiB of log");
      if (s->lcLog.R) {  // a new log replaces the old one
        for (void* q : {(void*)s->lcLog.rows, (void*)s->lcLog.fixed, (void*)s->lcLog.X, (void*)s->lcLog.R, (void*)s->lcLog.opOf}) {
          s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), q), s->allocs.end());
          cudaFree(q);
        }
        s->lcLog = LcLog{};
      }
      s->lcLog.rows = s->alloc<float4>((size_t)cap_ops * COARSE_PLANES * M);
      s->lcLog.fixed = s->alloc<uint32_t>((size_t)cap_ops * M);
      s->lcLog.X = s->alloc<float>((size_t)cap_ops * M * LC_IN);
      s->lcLog.R = s->alloc<float>((size_t)cap_calls * 3 * M);
      s->lcLog.opOf = s->alloc<int>(cap_calls);
      st.nOps = st.nCalls = 0;
      st.capOps = cap_ops;
      st.capCalls = cap_calls;
      st.loggedGen = st.gen - 1;
      st.curOp = -1;
    }
    st.log = on ? 1 : 0;
    CK(cudaMemcpyAsync(s->dLc, &st, sizeof st, cudaMemcpyHostToDevice, s->stream));
    s->lcEnabled = st.on != 0 || on != 0;
    resetGraphs(s);  // the log's buffers are kernel arguments of the graphs
    (void)wasOn;
    s->sync();
  });
}

extern "C++" {
namespace btd {
// The solver's learned log as device pointers and counts, for the trainer (trainer.cu).
struct LearnedLogView {
  const float4* rows;
  const uint32_t* fixed;
  const float* X;
  const float* R;
  const int* opOf;
  int M, nx, ny, ops, calls;
  cudaStream_t stream;
};
int learnedLogView(btd_solver* s, LearnedLogView* v) {
  if (!s || !s->dLc || !s->lcLog.R) return -1;
  LcState st;
  if (cudaMemcpyAsync(&st, s->dLc, sizeof st, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess) return -1;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return -1;
  const Level& C = s->levels.back();
  *v = LearnedLogView{s->lcLog.rows, s->lcLog.fixed, s->lcLog.X, s->lcLog.R, s->lcLog.opOf, C.N, C.layers[0].nx, C.layers[0].ny,
                      st.nOps, std::min(st.nCalls, st.capCalls), s->stream};
  return 0;
}
}  // namespace btd
}  // extern "C++"

// Test hook: the FP64 eigen-clamp of symmetric 3 x 3 blocks (mode 0: in = 6 doubles xx xy xz yy yz zz per
// block) or the spring block of a near-degenerate element (mode 1: in = K, f, dx, dy, dz, unused).
__global__ void k_debug_projection(const double* in, double* out, int count, int mode) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const double* a = in + 6 * q;
  double* o = out + 6 * q;
  if (mode == 0) {
    const double m[6] = {a[0], a[1], a[2], a[3], a[4], a[5]};
    double r[6];
    eigenClamp3(m, r);
    for (int k = 0; k < 6; ++k) o[k] = r[k];
  } else {
    const Sym S = springBlockFP64(a[0], a[1], a[2], a[3], a[4]);
    o[0] = S.xx, o[1] = S.xy, o[2] = S.xz, o[3] = S.yy, o[4] = S.yz, o[5] = S.zz;
  }
}

extern "C" int btd_debug_projection(const double* in, double* out, int32_t count, int32_t mode) {
  GUARD({
    if (!in || !out || count < 1 || count > (1 << 20) || (mode != 0 && mode != 1))
      throw std::invalid_argument("btd_debug_projection: 1..2^20 blocks, mode 0 or 1");
    double *din = nullptr, *dout = nullptr;
    const size_t bytes = sizeof(double) * 6 * (size_t)count;
    CK(cudaMalloc(&din, bytes));
    cudaError_t e = cudaMalloc(&dout, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(din, in, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      k_debug_projection<<<(count + 127) / 128, 128>>>(din, dout, count, mode);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost);
    cudaFree(din);
    if (dout) cudaFree(dout);
    CK(e);
  });
}

extern "C" int btd_set_wait_bound(int32_t first_tries) {
  GUARD({
    const int v = first_tries < 0 ? MBAR_TRIES : std::min<int>(first_tries, MBAR_TRIES);
    CK(cudaMemcpyToSymbol(g_mbarFirstTries, &v, sizeof v));
  });
}

// setPieces (solver.ts:664-676; topology.ts:7-22): the detached pieces of the topology analysis.
int btd_set_pieces(btd_solver* s, const uint32_t* piece_of, const uint32_t* start, const uint32_t* nodes, int32_t count) {
  GUARD({
    checkSolver(s);
    if (count < 0 || count > MAX_PIECES) throw std::invalid_argument("btd_set_pieces: 0.." + std::to_string(MAX_PIECES) + " pieces");
    const int N = s->N;
    if (count > 0) {
      if (!piece_of || !start || !nodes) throw std::invalid_argument("btd_set_pieces: null piece arrays");
      if (start[0] != 0) throw std::invalid_argument("btd_set_pieces: start[0] must be 0");
      for (int p = 0; p < count; ++p)
        if (start[p + 1] < start[p]) throw std::invalid_argument("btd_set_pieces: start must not decrease");
      const uint32_t total = start[count];
      if (total > (uint32_t)N) throw std::invalid_argument("btd_set_pieces: more piece nodes than nodes");
      for (int p = 0; p < count; ++p)
        for (uint32_t k = start[p]; k < start[p + 1]; ++k) {
          if (nodes[k] >= (uint32_t)N) throw std::invalid_argument("btd_set_pieces: node out of range");
          if (piece_of[nodes[k]] != (uint32_t)p) throw std::invalid_argument("btd_set_pieces: piece_of disagrees with the node lists");
        }
      for (int n = 0; n < N; ++n)
        if (piece_of[n] != NO_PIECE && piece_of[n] >= (uint32_t)count)
          throw std::invalid_argument("btd_set_pieces: piece_of names a piece beyond count");
      if (!s->dPieceOf) {
        s->dPieceOf = s->alloc<uint32_t>(N);
        s->dPieceStart = s->alloc<uint32_t>(MAX_PIECES + 1);
        s->dKx = s->alloc<float>(6 * (size_t)N);
        s->dKr = s->alloc<float>(6 * (size_t)N);
        s->dFrame = s->alloc<double>(40 * (size_t)MAX_PIECES);
        s->dStep = s->alloc<double>(6 * (size_t)MAX_PIECES);
        s->dCurveW = s->alloc<float4>(N);
        s->dCurveR = s->alloc<float4>(N);
      }
      if (total > s->pieceNodesCap) {
        if (s->dPieceNodes) {
          s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), (void*)s->dPieceNodes), s->allocs.end());
          cudaFree(s->dPieceNodes);
        }
        s->pieceNodesCap = std::max<size_t>(total, 1);
        s->dPieceNodes = s->alloc<uint32_t>(s->pieceNodesCap);
      }
      CK(cudaMemcpyAsync(s->dPieceOf, piece_of, sizeof(uint32_t) * N, cudaMemcpyHostToDevice, s->stream));
      CK(cudaMemcpyAsync(s->dPieceStart, start, sizeof(uint32_t) * (count + 1), cudaMemcpyHostToDevice, s->stream));
      if (total) CK(cudaMemcpyAsync(s->dPieceNodes, nodes, sizeof(uint32_t) * total, cudaMemcpyHostToDevice, s->stream));
    }
    const bool changed = count != s->pieceCount || count > 0;
    s->pieceCount = count;
    if (changed) resetGraphs(s);  // the piece count is a launch dimension of the captured kernels
    s->sync();
  });
}

int btd_level_count(btd_solver* s, int32_t* out) {
  GUARD({
    checkSolver(s);
    *out = (int32_t)s->levels.size();
  });
}

int btd_level_nodes(btd_solver* s, int32_t level, int32_t* out) {
  GUARD({
    checkSolver(s);
    if (level < 0 || level >= (int)s->levels.size()) throw std::invalid_argument("level out of range");
    *out = s->levels[level].N;
  });
}

int btd_read_operator(btd_solver* s, int32_t level, double* out, uint8_t* fixed) {
  GUARD({
    checkSolver(s);
    if (level < 0 || level >= (int)s->levels.size()) throw std::invalid_argument("level out of range");
    Level& L = s->levels[level];
    const int planes = L.fine ? FINE_PLANES : COARSE_PLANES;
    std::vector<float4> op((size_t)planes * L.N);
    std::vector<uint32_t> fx(L.N);
    CK(cudaMemcpyAsync(op.data(), L.op, sizeof(float4) * op.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(fx.data(), L.fixed, sizeof(uint32_t) * L.N, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    auto flt = [&](int n, int f) {
      const float4& v = op[(size_t)(f >> 2) * L.N + n];
      int c = f & 3;
      return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
    };
    if (out) {
      std::fill(out, out + (size_t)L.N * 225, 0.0);
      for (int n = 0; n < L.N; ++n) {
        auto put = [&](int o, int f) {
          double xx = flt(n, f), xy = flt(n, f + 1), xz = flt(n, f + 2), yy = flt(n, f + 3), yz = flt(n, f + 4), zz = flt(n, f + 5);
          double* b = out + ((size_t)n * 25 + o) * 9;
          b[0] = xx, b[1] = xy, b[2] = xz, b[3] = xy, b[4] = yy, b[5] = yz, b[6] = xz, b[7] = yz, b[8] = zz;
        };
        auto scal = [&](int o, double v) {
          double* b = out + ((size_t)n * 25 + o) * 9;
          b[0] = v, b[4] = v, b[8] = v;
        };
        if (L.fine) {
          const int di[8] = {1, -1, 0, 0, 1, -1, -1, 1}, dj[8] = {0, 0, 1, -1, 1, -1, 1, -1};
          put(12, 0);
          for (int k = 0; k < 8; ++k) put((dj[k] + 2) * 5 + di[k] + 2, 6 * (k + 1));
          scal(14, flt(n, 54));
          scal(10, flt(n, 55));
          scal(22, flt(n, 56));
          scal(2, flt(n, 57));
        } else {
          for (int o = 0; o < 25; ++o) put(o, 6 * o);
        }
      }
    }
    if (fixed)
      for (int n = 0; n < L.N; ++n) fixed[n] = fx[n] ? 1 : 0;
  });
}

int btd_device_buffer(btd_solver* s, int32_t which, int32_t level, void** ptr, size_t* bytes) {
  GUARD({
    checkSolver(s);
    if (!ptr) throw std::invalid_argument("null output");
    size_t b = 0;
    void* p = nullptr;
    if (which == BTD_BUF_X) {
      p = s->x, b = sizeof(float4) * s->N;
    } else if (which == BTD_BUF_V) {
      p = s->v, b = sizeof(float4) * s->N;
    } else if (which == BTD_BUF_CONTACT) {
      if (!s->contactOn()) throw std::invalid_argument("self-contact is off: no contact bounds");
      p = s->cmeta, b = sizeof(float4) * 2 * (size_t)s->N;
    } else if (which == BTD_BUF_OP || which == BTD_BUF_FIXED) {
      if (level < 0 || level >= (int)s->levels.size()) throw std::invalid_argument("level out of range");
      Level& L = s->levels[level];
      if (which == BTD_BUF_OP)
        p = L.op, b = sizeof(float4) * (size_t)(L.fine ? FINE_PLANES : COARSE_PLANES) * L.N;
      else
        p = L.fixed, b = sizeof(uint32_t) * L.N;
    } else {
      size_t n = 0;
      p = vectorPtr(s, which, level, &n);
      b = sizeof(float4) * n;
    }
    *ptr = p;
    if (bytes) *bytes = b;
  });
}

int btd_stage_matvec(btd_solver* s, const float* x4, float* y4, double* xy) {
  GUARD({
    checkSolver(s);
    if (!x4) throw std::invalid_argument("null input");
    const Level& F = s->levels[0];
    CK(cudaMemcpyAsync(s->p, x4, sizeof(float4) * s->N, cudaMemcpyHostToDevice, s->stream));
    MatvecArgs a;
    a.N = s->N;
    a.nx = F.layers[0].nx;
    a.ny = F.layers[0].ny;
    a.coord = F.dCoord;
    a.layers = F.dLayers;
    a.op = F.op;
    a.fixed = F.fixed;
    a.x = s->p;
    a.y = s->Ap;
    a.xy = &s->dScal->pAp;
    a.red = s->reduce();
    k_matvec_dot<<<s->redBlocks, RED_THREADS, 0, s->stream>>>(a);
    CK(cudaGetLastError());
    if (y4) CK(cudaMemcpyAsync(y4, s->Ap, sizeof(float4) * s->N, cudaMemcpyDeviceToHost, s->stream));
    double v = 0;
    CK(cudaMemcpyAsync(&v, &s->dScal->pAp, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    s->sync();
    if (xy) *xy = v;
  });
}

static float4* vectorPtr(btd_solver* s, int which, int level, size_t* count) {
  if (which <= BTD_VEC_R) {
    if (level < 0 || level >= (int)s->levels.size()) throw std::invalid_argument("level out of range");
    Level& L = s->levels[level];
    *count = L.N;
    return which == BTD_VEC_X ? L.X : which == BTD_VEC_B ? L.B : L.R;
  }
  *count = s->N;
  if (which == BTD_VEC_DELTA) return s->delta;
  if (which == BTD_VEC_DX) return s->dx;
  if (which == BTD_VEC_PRED) return s->pred;
  throw std::invalid_argument("unknown vector");
}

int btd_read_vector(btd_solver* s, int32_t which, int32_t level, float* out4) {
  GUARD({
    checkSolver(s);
    size_t n;
    float4* p = vectorPtr(s, which, level, &n);
    CK(cudaMemcpyAsync(out4, p, sizeof(float4) * n, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
  });
}

int btd_read_delta_f64(btd_solver* s, double* out3) {
  GUARD({
    checkSolver(s);
    if (!out3) throw std::invalid_argument("null output");
    CK(cudaMemcpyAsync(out3, s->deltaD, sizeof(double) * 3 * (size_t)s->N, cudaMemcpyDeviceToHost, s->stream));
    s->sync();
  });
}

int btd_write_vector(btd_solver* s, int32_t which, int32_t level, const float* in4) {
  GUARD({
    checkSolver(s);
    size_t n;
    float4* p = vectorPtr(s, which, level, &n);
    CK(cudaMemcpyAsync(p, in4, sizeof(float4) * n, cudaMemcpyHostToDevice, s->stream));
    s->sync();
  });
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Allocation-free matvec. Some callers cannot allocate device memory at the point where they call
// into the solve: a host that owns a fixed device pool (a game engine's or a plugin host's
// allocator), a real-time or frame-budgeted thread where cudaMalloc's implicit synchronisation is
// not allowed, or code running while another component captures the stream into a CUDA graph.
// btd_matvec_noalloc serves them: its reduction scratch is the file-scope array below, sized for
// NOALLOC_MAX_NODES nodes and resident on every GPU that loads this library until the process
// exits. Every call shares that array and leaves its last contents there; calls that overlap on the
// GPU (different streams, threads or devices sharing a context) race on it and must be serialised
// by the caller.

namespace {

constexpr int NOALLOC_MAX_BLOCKS = 2048;                              // one partial per 256-node block
constexpr int NOALLOC_MAX_NODES = NOALLOC_MAX_BLOCKS * RED_THREADS;  // 524,288 nodes
constexpr size_t NOALLOC_TICKET_BYTES = 256;
constexpr size_t NOALLOC_BYTES = NOALLOC_TICKET_BYTES + sizeof(double) * 8 * NOALLOC_MAX_BLOCKS;  // 131,328 bytes

static __device__ __align__(256) unsigned char g_noallocScratch[NOALLOC_BYTES];

std::mutex g_noallocMutex;
void* g_noallocAddr[256] = {};

// Device address of the scratch array on the current device, looked up once per device.
void* noallocScratch() {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) throw std::runtime_error("device index out of range");
  std::lock_guard<std::mutex> lock(g_noallocMutex);
  if (!g_noallocAddr[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noallocScratch));
    g_noallocAddr[dev] = p;
  }
  return g_noallocAddr[dev];
}

}  // namespace

extern "C" int btd_matvec_noalloc(int32_t nx, int32_t ny, const void* op, const void* fixed, const void* x, void* y,
                                  double* xy, void* stream) {
  GUARD({
    if (nx < 2 || ny < 2) throw std::invalid_argument("btd_matvec_noalloc: the lattice needs nx, ny >= 2");
    const long long N = (long long)nx * ny;
    if (N > NOALLOC_MAX_NODES)
      throw std::invalid_argument("btd_matvec_noalloc: " + std::to_string(N) + " nodes exceed the allocation-free maximum of " +
                                  std::to_string(NOALLOC_MAX_NODES));
    if (!op || !fixed || !x || !y || !xy) throw std::invalid_argument("btd_matvec_noalloc: null device pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* scratch = static_cast<unsigned char*>(noallocScratch());
    // the reduction ticket must start at zero; the partials are written before they are read
    CK(cudaMemsetAsync(scratch, 0, sizeof(unsigned), st));
    MatvecArgs a;
    a.N = (int)N;
    a.nx = nx;
    a.ny = ny;
    a.coord = nullptr;
    a.layers = nullptr;
    a.op = static_cast<const float4*>(op);
    a.fixed = static_cast<const uint32_t*>(fixed);
    a.x = static_cast<const float4*>(x);
    a.y = static_cast<float4*>(y);
    a.xy = xy;
    a.red = {reinterpret_cast<double*>(scratch + NOALLOC_TICKET_BYTES), reinterpret_cast<unsigned*>(scratch)};
    k_matvec_dot<<<blocksFor((int)N, RED_THREADS), RED_THREADS, 0, st>>>(a);
    CK(cudaGetLastError());
  });
}
