/*
 * btd.h - C ABI of the B200-native implicit cloth solve.
 *
 * The solve replaces the reference's WebGPU `GpuSolver` (src/simulation/gpu/solver.ts:194-838):
 * one projected-Newton substep over the woven crossing lattice, with the linear system solved by
 * Galerkin-multigrid-preconditioned PCG whose smoother solves each yarn line exactly. Every entry
 * point here corresponds to a member of `GpuSolver` (cited per function) or to the host-side scene
 * compilation it is constructed from (`compileScene`, src/simulation/scene.ts:233-278).
 *
 * Conventions: every function returns 0 on success and a negative BTD_E* code on failure; no C++
 * exception crosses this boundary. `btd_last_error` returns the message of the last failure on the
 * calling thread. Arrays are plain host pointers with the sizes stated; positions and velocities are
 * 4 floats per node (x, y, z, w), as the reference's vec4 buffers. A solver owns all its device
 * memory and works on its own CUDA stream; one solver must not be used from two threads at once.
 */
#ifndef BTD_H
#define BTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BTD_OK 0
#define BTD_E_INVALID (-1)     /* bad argument or unsupported size (the reference constructor throws) */
#define BTD_E_CUDA (-2)        /* a CUDA call failed (device lost, out of memory, ...) */
#define BTD_E_NO_DEVICE (-3)   /* no CUDA device: the library never falls back to the CPU */
#define BTD_E_STATE (-4)       /* call out of order (e.g. a stage that needs an assembled system) */
#define BTD_E_TIMEOUT (-5)     /* a bounded device-side wait ran out */

/* ------------------------------------------------------------------------------------------------
 * Scene description (src/simulation/material.ts:18-85, scene.ts:27-125)
 * ---------------------------------------------------------------------------------------------- */

/* YarnFamily (material.ts:18-54). yarns_per_span = 0 means "not bundled" (the field is absent). */
typedef struct btd_yarn {
  double linear_density, ea_low, ea_high, crimp_strain, ea_compress, axial_viscosity;
  double bend_rigidity, bend_viscosity, strength, softening_opening, width, height, crimp_amplitude;
  int32_t yarns_per_span;
  int32_t pad_;
} btd_yarn;

/* WeaveMaterial (material.ts:56-85). */
typedef struct btd_material {
  int32_t id;
  char name[60];
  double pitch_u, pitch_v;
  btd_yarn yarns[2];
  int32_t twill_repeat, twill_warp_over;
  double shear_stiffness, crossing_friction, crossing_normal0, crossing_wrap;
  double thickness, cloth_friction, air_drag;
} btd_material;

/* WearSpec (scene.ts:27-46). */
typedef struct btd_wear {
  double center[2], axis[2], radii[2];
  double amount, cell_size, feature_scale, defect_threshold, defect_density, sparse_from;
} btd_wear;

/* LayerSpec (scene.ts:48-71). bundle = {1, 1} when the reference leaves it undefined. */
typedef struct btd_layer_spec {
  btd_material material;
  int32_t bundle[2];
  double size_u, size_v, z, angle, compress_u, compress_v, shear;
  int32_t collar_rows;
  int32_t seed;
  btd_wear wear;
  double wear_strength_loss[2];
  double perturbation;
} btd_layer_spec;

/* LayerInfo (scene.ts:73-89) plus its yarn-field layout (yarnField.ts:47-66). */
typedef struct btd_layer_info {
  int32_t index, nx, ny, node_offset, node_count;
  int32_t bundle[2];
  int32_t field_offset, field_k, field_m;
  btd_material material; /* bundled (mechanical) */
  btd_material weave;    /* individual yarns */
  double map_a[4], map_origin[3], rest_center[2];
} btd_layer_info;

/*
 * CompiledScene (scene.ts:91-125). N = node_count, C = crossing_count. Spans are indexed 2 n + f
 * (f = 0: u-family span to (i + 1, j); f = 1: v-family span to (i, j + 1)); crossings 2 c + f.
 * Either filled by btd_scene_compile (library-owned arrays, freed by btd_scene_free) or assembled
 * by the caller over its own arrays.
 */
typedef struct btd_scene {
  int32_t n_layers;
  int32_t node_count;
  int32_t crossing_count;
  int32_t pad_;
  btd_layer_info* layers;
  double* rest_uv;          /* 2N */
  double* position;         /* 3N */
  double* mass;             /* N */
  uint8_t* pinned;          /* N */
  float* wear;              /* N */
  float* structural_wear;   /* N */
  double* rest_length;      /* 2N */
  double* softening;        /* 2N */
  uint16_t* seg_flags;      /* 2N: SEG_EXISTS 1, SEG_BROKEN 2, SEG_INITIAL_DEFECT 4, SEG_SLIPPED 8 */
  double* intact;           /* 2N */
  uint32_t* cut_mask;       /* 2N */
  float* fail_site;         /* 2N */
  float* field_strength;    /* 2C */
  uint8_t* field_damage;    /* 2C */
  uint8_t* field_area;      /* 2C */
  double* crossing_normal0; /* N */
  double* tails;            /* 4N */
} btd_scene;

/* compileScene (scene.ts:233-278): compile layer specs into a scene (host only, no GPU needed). */
int btd_scene_compile(const btd_layer_spec* specs, int32_t n_specs, btd_scene** out);
/* Free a scene returned by btd_scene_compile. */
int btd_scene_free(btd_scene* scene);
/* sceneHash (scene.ts:134-150): FNV-style content hash validating precomputed drapes. */
int btd_scene_hash(const btd_scene* scene, uint32_t* out);
/* The reference's materials DENIM / BACKING (material.ts:88-187); index 0 or 1. */
int btd_material_preset(int32_t index, btd_material* out);
/* bundleWeave (material.ts:198-226). */
int btd_bundle_weave(const btd_material* m, int32_t bu, int32_t bv, btd_material* out);
/* defaultSceneSpecs (scene.ts:438-469): the shipped 182 x 115 coupon. */
int btd_default_scene_spec(btd_layer_spec* out);

/* ------------------------------------------------------------------------------------------------
 * Solver (GpuSolver, src/simulation/gpu/solver.ts:194-838)
 * ---------------------------------------------------------------------------------------------- */

/* GpuSolverParams (solver.ts:26-53) with the multigrid schedule (newtonMultigrid.ts:20-34). */
typedef struct btd_params {
  double h;
  double gravity[3];
  int32_t newton_iterations; /* always performed per substep */
  int32_t newton_max;        /* gated upper bound (gate.wgsl) */
  double newton_tolerance;   /* m, largest nodal update that ends the gated iterations */
  double history_tolerance;  /* m, last update above which a node does not advance slip */
  int32_t pcg_iterations;    /* PCG iterations (reference: a fixed count) or the cap with pcg_rel_tol */
  int32_t coarse_sweeps;
  int32_t max_coarsest_nodes;
  int32_t self_contact;
  double pcg_rel_tol;        /* extension: stop at ||r_k|| / ||r_0|| <= tol (0: fixed count) */
  int32_t line_search;       /* choose the step among {1, 1/2, 1/4, 1/8} (energy.wgsl); 1 in the reference */
  int32_t lag_coarse;        /* reuse the coarse levels after a substep's first Newton iteration; 1 */
  int32_t overlap_launches;  /* extension: kernels of the PCG loop start while their predecessor drains
                                (programmatic dependent launch; the smoother stages its line factors
                                meanwhile); 0 serialises them; 1 */
  int32_t cross_layer;       /* with self_contact on a scene of several layers: node-node contact between
                                the layers in place of self-contact, as the reference does (solver.ts:364;
                                contact.ts, contact.wgsl); 0 */
} btd_params;

/* GPU_DEFAULTS (solver.ts:61-72). */
int btd_default_params(btd_params* out);

typedef struct btd_solver btd_solver;

/* Counters (solver.ts:218-225): [0] ruptures, [1] pulled-out spans, [2] max speed (f32 bits),
 * [3] line-search alpha (f32 bits), [4 + k] largest update of Newton iteration k (f32 bits),
 * [12] rejected directions. Slots 16.. are solver statistics: [16] PCG iterations of the last
 * Newton iteration, [17] PCG iterations summed since the last clear, [18] Newton iterations run,
 * [19] relative residual of the last PCG solve (f32 bits), [20] device-side error flags. */
#define BTD_COUNTERS 32

/* GpuSolver constructor (solver.ts:275-385). Throws there on unsupported sizes; BTD_E_INVALID here. */
int btd_create(const btd_scene* scene, const btd_params* params, btd_solver** out);
int btd_destroy(btd_solver* s);

/* encodeSubstep (solver.ts:737-760): predict, Newton iterations, commit, damage, slip. */
int btd_substep(btd_solver* s, int32_t min_iterations, int32_t max_iterations);
/* The engine's per-frame loop of substeps (worker.ts:664-674), stream-ordered, one launch each. */
int btd_substeps(btd_solver* s, int32_t count);
/* A batch of independent solvers (one patch each; the batched configuration): `substeps` substeps
 * of every solver, each on its own stream, queued round robin with no host synchronisation, so the
 * patches run concurrently on the GPU. Each patch's results are those of btd_substeps on it alone.
 * With more patches than CUDA_DEVICE_MAX_CONNECTIONS (8 unless the process sets it, at most 32)
 * streams share hardware queues. Synchronise each solver (btd_synchronize) before reading it. */
int btd_batch_substeps(btd_solver* const* solvers, int32_t count, int32_t substeps);
/* A batch as one graph (no counterpart in the reference): one substep of every solver, each on its own
 * stream inside one capture, so a batch substep is a single cudaGraphLaunch whose branches run side by
 * side, each with its own device-side PCG loops. btd_batch_run launches it `substeps` times, each after
 * the work already queued on every solver's stream (grip targets, state writes) and before what comes
 * after it there; its results are those of btd_substeps on each solver alone. The batch graph holds the
 * solvers' settings at creation: create it again after a solver's learned correction, pieces or graph
 * mode change (a grip attached or released is picked up by itself). Solvers must outlive the batch. */
typedef struct btd_batch btd_batch;
int btd_batch_create(btd_solver* const* solvers, int32_t count, btd_batch** out);
int btd_batch_run(btd_batch* b, int32_t substeps);
int btd_batch_destroy(btd_batch* b);
/* Wait for all submitted work (the reference's onSubmittedWorkDone). */
/* Wait for the solver's stream (onSubmittedWorkDone). Returns BTD_E_TIMEOUT, once, when a bounded
 * device-side wait (a staging copy's completion) ran out since the last call: the kernels never hang
 * on one; they flag it in counter slot 20 and go on. */
int btd_synchronize(btd_solver* s);

/* setState (solver.ts:833-837): positions (4 floats per node) and velocities (NULL: zero). */
int btd_set_state(btd_solver* s, const float* position4, const float* velocity4);
int btd_get_state(btd_solver* s, float* position4, float* velocity4);
/* setSegments (solver.ts:821-824): per span rest length, intact fraction, cut mask, flags, fail
 * site (2N each) and tails (4N). btd_get_segments reads them back (any pointer may be NULL). */
int btd_set_segments(btd_solver* s, const float* rest_length, const float* intact, const uint32_t* cut_mask,
                     const uint32_t* seg_flags, const float* fail_site, const float* tails);
int btd_get_segments(btd_solver* s, float* rest_length, float* intact, uint32_t* cut_mask, uint32_t* seg_flags,
                     float* fail_site, float* tails);
/* setField (solver.ts:827-830): damage codes, 2 per crossing. */
int btd_set_field(btd_solver* s, const uint8_t* damage);
int btd_get_field(btd_solver* s, uint8_t* damage);
/* resetState (solver.ts:810-818). */
int btd_reset_state(btd_solver* s);

/* setFloor (solver.ts:796-801): enabled = 0 removes the floor. */
int btd_set_floor(btd_solver* s, int32_t enabled, float z);
/* setTimestep (solver.ts:804-807). */
int btd_set_timestep(btd_solver* s, float h);
/* setHistoryEnabled (solver.ts:777-779). */
int btd_set_history(btd_solver* s, int32_t enabled);
/* setNewtonTolerance (solver.ts:782-785). */
int btd_set_newton_tolerance(btd_solver* s, float tolerance);
/* Execution mode: 1 (default) launches each substep as one captured CUDA graph whose PCG loop is a
 * device-side while-node; 0 launches the same kernels one by one with the PCG stop read back by
 * the host after every iteration (for per-kernel profilers, which cannot see into such graphs). */
int btd_set_graph_mode(btd_solver* s, int32_t use_graphs);
/* Extension: precision of the Newton right-hand side (the nonlinear residual -grad Phi): 1 (default)
 * evaluates its terms in FP64 from the FP32 state, so each Newton iteration refines in FP64 what the
 * FP32 operator and PCG solve for; 0 evaluates them in FP32 as the reference's shader does
 * (assemble.wgsl:152-334). The operator stays FP32 either way. */
int btd_set_gradient_precision(btd_solver* s, int32_t fp64);
/* Extension: precision of the operator PCG solves with. 1 (default): the fine operator is also assembled
 * in FP64 - each span's block formed from its FP64 element vector (exactly PSD), every row summed in
 * FP64 - and PCG's products, its true residual, the rigid start's residual and the V-cycle's fine
 * residual take it, while the smoothers, transfers and coarse levels keep the FP32 rows. In FP32 a row's large span terms
 * cancel on a rigid motion only to ~6e-8 of their size, which on torn cloth (loose strands held by
 * inertia alone, ~3e7 times softer than a span) leaves the FP32 operator indefinite and PCG breaks down
 * short of rel-res 1e-6. 0: the FP32 rows throughout, as the reference's shaders. */
int btd_set_operator_precision(btd_solver* s, int32_t fp64);
/* Extension: PCG's beta in the flexible (Polak-Ribiere) form, max(r' . (z' - z), 0) / (r . z), which
 * equals the plain form in exact arithmetic with a fixed SPD preconditioner and stays a descent method
 * when the preconditioner is applied inexactly (FP32 V-cycle, learned correction); 0 (default) the
 * reference's form r' . z' / (r . z). */
int btd_set_pcg_flexible(btd_solver* s, int32_t on);
/* Extension: PCG cap and relative-residual stop (0 = fixed count as the reference). */
int btd_set_pcg(btd_solver* s, int32_t max_iterations, double rel_tol);

/* settleDrape (settle.ts:24-62): settle the authored drape before interaction - 420 substeps of 5
 * Newton iterations with a fixed 2 PCG iterations each, history off, velocities cleared after every
 * tenth of the first 360 substeps, then velocities and counters cleared. The solver's Newton, PCG and
 * history settings are restored afterwards. Blocking. The drape file (settle.ts:4-22: a 16-byte
 * header [magic 0x50415244, version 1, node count, sceneHash] then 4 floats a node) is host code
 * around btd_get_state / btd_set_state and btd_scene_hash. */
int btd_settle_drape(btd_solver* s);
/* Counters (solver.ts:218-225); n <= BTD_COUNTERS. btd_clear_counters zeroes them. Slots: 0 ruptures,
 * 1 pull-outs, 2 max speed (f32), 3 line-search step (f32), 4-11 Newton updates (f32), 12 rejected,
 * 16 last PCG count, 17 PCG total, 18 Newton iterations, 19 last relative residual (f32), 20 errors;
 * extensions: 21 the largest relative residual a PCG solve stopped at (f32), 22 the solves that stopped
 * short of the relative-residual tolerance (at the cap or on a breakdown). */
int btd_read_counters(btd_solver* s, uint32_t* out, int32_t n);
int btd_clear_counters(btd_solver* s);

/* ---- stage encoders used by parity tests and profilers (solver.ts:574-728) ---- */
int btd_stage_predict(btd_solver* s);                  /* encodePredict */
int btd_stage_assemble(btd_solver* s, int32_t coarse); /* encodeAssemble(pass, coarse) */
int btd_stage_vcycle(btd_solver* s);                   /* encodeVCycle(pass, 0): X0 = V(B0), X0 zeroed first */
/* encodeSmooth (solver.ts:601-622): one yarn-line sweep of level `level` in place, X <- S(X, B);
 * reverse runs the colours backwards (the post-smoother). */
int btd_stage_smooth(btd_solver* s, int32_t level, int32_t reverse);
int btd_stage_pcg(btd_solver* s);                      /* encodePCG: delta = PCG(B0) */
/* encodeLineSearch: energy changes e[4] and magnitude sums m[4] along delta, alpha chosen on device. */
int btd_stage_linesearch(btd_solver* s, double* e4, double* m4);
int btd_stage_apply(btd_solver* s, int32_t iteration); /* newtonApply */
int btd_stage_newton(btd_solver* s, int32_t iteration);/* encodeNewtonIteration */
int btd_stage_finalize(btd_solver* s);                 /* encodeFinalize: commit, damage, slip */
int btd_stage_damage(btd_solver* s);                   /* encodeDamage */

/* setPieces (solver.ts:664-676): the detached pieces found by the topology analysis (topology.ts:7-22),
 * as piece_of (N: the piece of each node, 0xFFFFFFFF for none), start (count + 1 offsets into nodes) and
 * nodes (each piece's nodes). Each piece's six rigid modes then give PCG its start, its nodes step along
 * the rotation of that start in the line search and update, and each substep starts a spinning piece on
 * its rotation (rigid_frame.wgsl, rigid_apply.wgsl, rigid_spin.wgsl). count = 0 clears; at most 4096
 * pieces. BTD_E_INVALID when the arrays disagree. */
int btd_set_pieces(btd_solver* s, const uint32_t* piece_of, const uint32_t* start, const uint32_t* nodes, int32_t count);

/* Multigrid levels (solver.ts:105-118, 333-352). */
int btd_level_count(btd_solver* s, int32_t* out);
int btd_level_nodes(btd_solver* s, int32_t level, int32_t* out);
/* Operator of a level in the 25-offset layout of the CPU reference (newtonMultigrid.ts:38-48):
 * N * 25 * 9 doubles, offset index (dj + 2) * 5 + (di + 2), row-major 3x3 blocks; fixed flags N. */
int btd_read_operator(btd_solver* s, int32_t level, double* out, uint8_t* fixed);
/* Vectors (4 floats per node): which = 0 X, 1 B, 2 R of a level; 3 delta, 4 dx, 5 pred, 6 ext (3 vec4/node). */
#define BTD_VEC_X 0
#define BTD_VEC_B 1
#define BTD_VEC_R 2
#define BTD_VEC_DELTA 3
#define BTD_VEC_DX 4
#define BTD_VEC_PRED 5
int btd_read_vector(btd_solver* s, int32_t which, int32_t level, float* out4);
/* The last PCG solve's iterate as accumulated in FP64 (3 doubles per node); delta (BTD_VEC_DELTA) is
 * its fp32 copy. The outer residual that stops PCG at pcg_rel_tol is b - A x computed from it. */
int btd_read_delta_f64(btd_solver* s, double* out3);
/* Zero-copy access for consumers that bind the solver's buffers (the renderer and tools read
 * GpuSolver.x, .levels[k].op etc. directly, solver.ts:198-263): device pointer and size in bytes of
 * buffer `which` (BTD_VEC_* above, or BTD_BUF_*) of `level`. The pointer stays valid until
 * btd_destroy. Fine operator rows are 15 float4 planes, plane p of node n at op[p * N + n]: nine
 * symmetric blocks (xx xy xz yy yz zz) diag, +u, -u, +v, -v, +u+v, -u-v, -u+v, +u-v, then the scalar
 * couplings +2u, -2u, +2v, -2v; coarse rows are 38 planes of 25 blocks in offset order. */
#define BTD_BUF_OP 16
#define BTD_BUF_FIXED 17
#define BTD_BUF_X 18
#define BTD_BUF_V 19
/* contact.meta (solver.ts:263): 2 float4 per node, the node's own bound (unit normal away from the
 * face, largest approach along it) and the reciprocal bound of a face corner; w >= 1e8: none.
 * Only with self_contact. */
#define BTD_BUF_CONTACT 20
int btd_device_buffer(btd_solver* s, int32_t which, int32_t level, void** ptr, size_t* bytes);
/* Stage: y = A x and x . y with the fine operator of the last assembly (the PCG matvec, pcg.wgsl:268-287),
 * x and y 4 floats per node on the host. Uses the solver's own reduction scratch. */
int btd_stage_matvec(btd_solver* s, const float* x4, float* y4, double* xy);
int btd_write_vector(btd_solver* s, int32_t which, int32_t level, const float* in4);

/* ---- Grips (Interaction, src/simulation/gpu/interaction.ts:223-318; interact.wgsl:96-197).
 * Up to BTD_GRIPS grips, each a patch of at most BTD_GRIP_ENTRIES material nodes pulled by springs of
 * stiffness `stiffness` x weight toward a handle. No node is in two patches. Held grips add one
 * launch per substep (the lead) and one per Newton iteration (the terms); no held grip, no launch.
 *
 * btd_set_grip replaces attachPatch(slot, picked, patch, anchor, maxLead) (interaction.ts:223-261):
 * `nodes`/`weights`/`sides` are GripPatch.nodes/weights/sides (sides may be null: a radial patch),
 * `pad_pitch` and `slip` are GripPatch.padPitch and .slip (0: the hold does not slip), `anchor` is
 * where the caller takes the picked material to be. Entry offsets and the handle's origin are taken
 * on the device from node `picked`'s current position, so a target equal to the anchor moves nothing.
 * Errors (BTD_E_INVALID): slot, count or node out of range, a node twice or held by another grip,
 * negative or non-finite weight/stiffness, max_lead <= 0, a side other than -1/0/+1. */
#define BTD_GRIPS 4
#define BTD_GRIP_ENTRIES 512
int btd_set_grip(btd_solver* s, int32_t slot, const int32_t* nodes, const float* weights, const float* sides, int32_t count,
                 int32_t picked, const float* anchor3, float stiffness, float max_lead, float pad_pitch, float slip);
/* setTarget (interaction.ts:276-281): requested handle in the frame of the attach anchor. */
int btd_set_grip_target(btd_solver* s, int32_t slot, const float* target3);
/* setPinch (interaction.ts:263-267): spread of the patch relative to grab time (1: as grabbed). */
int btd_set_grip_pinch(btd_solver* s, int32_t slot, float scale);
/* setHold (interaction.ts:269-274): stiffness = attach stiffness x fraction. */
int btd_set_grip_hold(btd_solver* s, int32_t slot, float fraction);
/* release (interaction.ts:302-313); without self-contact it also clears ext. Target, pinch and hold
 * calls on a slot that holds nothing do nothing and return BTD_OK, like the reference's. */
int btd_release_grip(btd_solver* s, int32_t slot);
/* Readback for tests (the reference's tests read the grip buffer, tests/gpu/interaction.ts:318-324):
 * the entry count, up to `capacity` entries' nodes and current weights (0 once slipped out), and
 * 12 floats: the effective handle, the origin and the closing axis of the last lead, xyz + pad. */
int btd_read_grip(btd_solver* s, int32_t slot, int32_t* nodes, float* weights, int32_t capacity, float* handle12,
                  int32_t* count);

/* Per-stage timing (the reference's tools/gpu/scripts/profile.ts: timestamp queries per pass):
 * launches stage `which` `reps` times on the solver's stream on the current system and returns the
 * mean device time of one launch in ms, from CUDA events recorded on that stream. With flush != 0 a
 * 256 MiB buffer is rewritten before every launch (outside the events) so each launch starts with a
 * cold L2. which: 0 fine matvec (SpMV + dot), 1 fine smoother sweep (6 colour launches), 2 fine
 * assembly, 3 V-cycle, 4 Galerkin hierarchy (prolongation weights + RAP of every level), 5 substep. */
#define BTD_STAGE_MATVEC 0
#define BTD_STAGE_SMOOTH 1
#define BTD_STAGE_ASSEMBLE 2
#define BTD_STAGE_VCYCLE 3
#define BTD_STAGE_HIERARCHY 4
#define BTD_STAGE_SUBSTEP 5 /* a whole substep: one launch of the captured substep graph */
int btd_profile_stage(btd_solver* s, int32_t which, int32_t reps, int32_t flush, float* ms_per_launch);
/* Kernel launches of substeps that ran `newton_iterations` Newton iterations and `pcg_iterations`
 * PCG iterations in total (the graph's nodes that are kernels, loop bodies counted per pass). */
int btd_launch_count(btd_solver* s, int32_t substeps, int32_t newton_iterations, int32_t pcg_iterations, int64_t* out);
/* Autotuner of the yarn-line sweeps' launch shapes (no counterpart in the reference, whose workgroup
 * size is fixed at 128, smooth.wgsl:86): for every multigrid level the CTA size (multiples of 32 from 64
 * to 256) and, on lines longer than 128 nodes, the staging tile (whole line or 128 nodes) are timed on
 * the level's current operator (CUDA events, the mean of `reps` sweeps) and the fastest is kept for
 * every later sweep; results are unchanged bit for bit. Needs an assembled system (after a substep or
 * btd_stage_assemble). Per level (btd_level_count entries, any pointer may be NULL): the chosen CTA
 * size, tile, and the sweep's time in ms. */
int btd_autotune(btd_solver* s, int32_t reps, int32_t* threads, int32_t* tile, float* ms);

/* y = A x and x . y for a single-layer nx x ny fine operator on caller-owned DEVICE buffers (op in
 * the fine-row layout of btd_device_buffer, fixed flags as uint32, x and y 4 floats per node, xy one
 * double), enqueued on `stream` (a cudaStream_t; NULL: the legacy default stream); the results are
 * ready when that stream reaches this point. No counterpart in the reference: this entry point
 * allocates nothing, for callers that cannot call cudaMalloc (a host with its own fixed device
 * pool, a frame-budgeted thread where cudaMalloc's implicit synchronisation is not allowed, code
 * running while a stream is being captured). Its reduction scratch is a static device array of
 * 131,328 bytes that every GPU loading the library holds until exit; lattices of more than
 * 524,288 nodes are rejected with BTD_E_INVALID. The first call on each device looks the array's
 * address up (cudaGetSymbolAddress) and should come before any stream capture; that address is kept
 * for the life of the process, so this entry point must not be used after a cudaDeviceReset of the
 * device it ran on. All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int btd_matvec_noalloc(int32_t nx, int32_t ny, const void* op, const void* fixed, const void* x, void* y, double* xy,
                       void* stream);

/* ---- Learned coarse correction (no counterpart in the reference; the reference's coarsest V-cycle
 * level is two alternating line sweeps, newtonMultigrid.ts:495-502, solver.ts:584-598). Half-way through
 * the coarsest sweeps the V-cycle adds the Galerkin correction Phi (Phi^T A Phi)^-1 Phi^T (b - A x) on a
 * basis of BTD_LEARNED_K vectors that a 3-layer MLP (20 -> 64 -> 64 -> 24, tanh, BF16 weights and
 * activations, FP32 accumulation, evaluated on the tensor cores) builds per coarsest node from local
 * data: lattice position, the node's diagonal block, the fraction of fixed neighbours, and damage and
 * contact flags restricted from the fine lattice. The basis is built once per PCG solve. Single-layer
 * lattices whose coarsest level has at most BTD_LEARNED_MAX_NODES nodes. */
#define BTD_LEARNED_WEIGHTS 7064 /* W1[20][64] b1[64] W2[64][64] b2[64] W3[64][24] b3[24], row-major [in][out] */
#define BTD_LEARNED_K 8
#define BTD_LEARNED_MAX_NODES 576
/* Sets the network (weights: BTD_LEARNED_WEIGHTS floats, or NULL to keep the current ones) and turns the
 * correction on or off. guard: a PCG solve whose mean contraction per iteration (||r_k|| / ||r_0||)^(1/k)
 * exceeds it after three iterations goes on with the plain V-cycle, PCG restarted from its iterate.
 * BTD_E_INVALID for a wrong count, non-finite weights, a multi-layer lattice or too large a coarsest level. */
int btd_set_learned(btd_solver* s, const float* weights, int32_t count, int32_t on, double guard);
/* out[5]: PCG solves with the correction on, corrections applied, solves that fell back, logged
 * operators, logged calls. */
int btd_learned_stats(btd_solver* s, int64_t* out);
/* The last solve's basis: phi (3 M x 8 floats, row 3 n + c), the Cholesky factor of Phi^T A Phi (64
 * doubles, lower, row-major), dead columns (8; all -1 when no basis was built), the coarsest nodes'
 * flags (M bytes: 1 damage, 2 contact); any pointer may be NULL; nodes receives M. */
int btd_learned_basis(btd_solver* s, float* phi, double* G, int32_t* dead, uint8_t* flags, int32_t* nodes);
/* Logs training material on the device while on: every new coarsest operator (its rows, fixed flags and
 * the network inputs of its nodes; at most cap_ops) and the coarsest residual at every correction call
 * (at most cap_calls). Turning it on starts a new log. The log feeds btd_trainer_add_log. */
int btd_learned_log(btd_solver* s, int32_t on, int32_t cap_ops, int32_t cap_calls);

/* ---- Training of the learned correction's network on the GPU (no counterpart in the reference).
 * Material: per coarsest operator its whitened form At = L^-1 A L^-T over the free unknowns (D_i = L_i
 * L_i^T the diagonal blocks) and its nodes' network inputs; per correction call the whitened residual r
 * and the exact correction d = At^-1 r. Objective: the mean over calls of 1 - q, q = u^T G^-1 u / r^T d
 * the share of the call's error energy the basis captures (u = Psi^T r, G = Psi^T At Psi). The network
 * runs forward and backward in BF16 on the tensor cores with FP32 accumulation; Adam on FP32 weights. */
typedef struct btd_trainer btd_trainer;
int btd_trainer_create(btd_trainer** out);
int btd_trainer_destroy(btd_trainer* t);
/* Adds one operator of host material (FP64): At (3n x 3n), X (n x 20), R and D (calls x 3n). `group`
 * labels it for btd_trainer_train's group weights. */
int btd_trainer_add_op(btd_trainer* t, int32_t nodes, const double* At, const double* X, int32_t calls, const double* R,
                       const double* D, int32_t group);
/* Adds the solver's learned log (btd_learned_log) on the device: whitens every logged operator, factors it
 * (dense Cholesky, FP64) and solves every logged call's exact correction. Operators whose free diagonal
 * blocks are not all positive definite, or whose whitened form is not, are dropped (as are their calls). */
int btd_trainer_add_log(btd_trainer* t, btd_solver* s, int32_t group, int32_t* ops_added);
int btd_trainer_counts(btd_trainer* t, int32_t* ops, int32_t* calls);
/* Reads operator `op`'s material back (any pointer may be NULL; sizes as in btd_trainer_add_op, FP32). */
int btd_trainer_read_op(btd_trainer* t, int32_t op, int32_t* nodes, int32_t* calls, float* At, float* X, float* R, float* D,
                        double* E);
/* Loss and gradient (BTD_LEARNED_WEIGHTS floats) over all calls of the listed operators (1..16). */
int btd_trainer_loss_grad(btd_trainer* t, const float* weights, const int32_t* ops, int32_t n_ops, double* loss, float* grad);
/* `steps` Adam steps (lr decaying tenfold over the run) on minibatches of `batch_ops` operators (all
 * their calls), drawn without replacement within a step in proportion to group_weights[group] / the
 * group's operator count (all alike when group_weights is NULL); weights in and out; loss_history
 * (steps floats, may be NULL) receives each step's minibatch loss. */
int btd_trainer_train(btd_trainer* t, float* weights, int32_t steps, int32_t batch_ops, float lr, uint64_t seed,
                      const float* group_weights, int32_t n_groups, float* loss_history);

/* Test hook for the PSD projection of near-degenerate element blocks (no counterpart in the reference,
 * whose projections are closed forms, newtonMultigrid.ts:127-157): runs the device routine on `count`
 * blocks of 6 doubles. mode 0: the FP64 eigen-clamp (cyclic Jacobi) of symmetric 3 x 3 blocks given as
 * xx xy xz yy yz zz; mode 1: the spring block of a near-degenerate element from (K, f, dx, dy, dz, -),
 * the eigen-clamp of K e e^T + (f / l) (I - e e^T). Output: 6 doubles per block. */
int btd_debug_projection(const double* in, double* out, int32_t count, int32_t mode);

/* Test hook for the bounded device-side waits (no counterpart in the reference): the first bound of
 * the smoother's wait for its staging copies, in tries (negative: the default, 2^20). With 0 the
 * wait's error flag is raised at once while the copies still land under its second bound, so results
 * stay correct and the next btd_synchronize returns BTD_E_TIMEOUT once. Process-wide (every solver on
 * the current device). */
int btd_set_wait_bound(int32_t first_tries);

/* Last error message of the calling thread (always NUL-terminated when n > 0). */
int btd_last_error(char* buf, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* BTD_H */
