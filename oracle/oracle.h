/*
 * oracle.h - TEST INFRASTRUCTURE ONLY. The FP64 CPU restatement of the reference's own solver
 * (src/simulation/reference/{solver,newtonMultigrid}.ts with laws.ts, axial.ts, lattice.ts and
 * yarnField.ts). It is the correctness oracle for the CUDA path and the timed CPU baseline; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it. The product library
 * never links or calls it.
 *
 * Parity is pinned by restating the reference's own property tests (tests/unit/newtonMultigrid.test.ts,
 * referenceSolver.test.ts, yarnField.test.ts, laws.test.ts, axial.test.ts) against this code; the
 * reference ships no golden vectors for the solve.
 *
 * Extensions flagged as not in the reference: a PCG relative-residual stop, several grips, the
 * floor contact of the GPU shaders restated on the CPU, the learned coarse space on the coarsest
 * V-cycle level (with its training material logging), and BF16 storage of the coarse levels as a
 * precision study.
 */
#ifndef BTD_ORACLE_H
#define BTD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "btd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_params {
  double h;
  double gravity[3];
  int32_t newton_iterations;
  int32_t pcg_iterations;    /* fixed count, or the cap when pcg_rel_tol > 0 */
  double pcg_rel_tol;        /* extension: stop at ||r_k|| / ||r_0|| <= tol */
  int32_t max_coarsest_nodes;/* MGConfig (newtonMultigrid.ts:20-34) */
  int32_t coarse_sweeps;
  int32_t line_colors;
  int32_t lag_coarse;
  int32_t line_search;
  int32_t threads;           /* OpenMP threads (0: all) */
  int32_t self_contact;      /* node-face self-contact restated from selfcontact.wgsl (the f64 reference has none) */
  int32_t cross_layer;       /* with contact on, a scene of several layers gets the cross-layer node contact of
                                contact.wgsl in place of self-contact, as the reference does (solver.ts:364);
                                0 keeps self-contact on every scene */
  int32_t coarse_bf16;       /* extension (precision study): every coarse level's operator rounded to BF16
                                (nearest, ties to even) as it is built, the next level built from the rounded one;
                                1 all 25 blocks, 2 the 24 coupling blocks (the diagonal block kept) */
  int32_t fp32_rows;         /* extension (precision study): the operator as float32 storage would hold it
                                (nearest); units digit the fine level (after assembly), tens digit every coarse
                                level (after the Galerkin product): 0 kept, 1 every block rounded, 2 the row-sum
                                form - the couplings and each row's block sum rounded, the diagonal block the
                                rounded sum less the rounded couplings */
} ora_params;

typedef struct ora_solver ora_solver;

ora_solver* ora_create(const btd_scene* scene, const ora_params* params);
void ora_destroy(ora_solver* s);
const char* ora_last_error(void);

/* ReferenceSolver state (solver.ts(ref):41-119); 3 doubles per node. */
int ora_set_state(ora_solver* s, const double* x, const double* v);
int ora_get_state(ora_solver* s, double* x, double* v, double* dx, double* pred);
int ora_set_dx(ora_solver* s, const double* dx, const double* pred);
int ora_set_segments(ora_solver* s, const double* rest, const double* intact, const uint32_t* cut_mask,
                     const uint16_t* flags, const double* fail_site, const double* tails);
int ora_get_segments(ora_solver* s, double* rest, double* intact, uint32_t* cut_mask, uint16_t* flags,
                     double* fail_site, double* tails);
int ora_set_field(ora_solver* s, const uint8_t* damage);
int ora_get_field(ora_solver* s, uint8_t* damage);
int ora_set_history(ora_solver* s, int32_t on);
int ora_counts(ora_solver* s, int32_t* broken, int32_t* pulled);

/* Grips (ReferenceGrip, solver.ts(ref):29-37), any number (extension: the reference has one). */
int ora_clear_grips(ora_solver* s);
int ora_add_grip(ora_solver* s, const int32_t* nodes, const double* w, const double* offset, int32_t count,
                 const double* goal, double k);
int ora_set_grip_goal(ora_solver* s, int32_t grip, const double* goal);
/* Floor (GPU shader math, common.wgsl:251-270, restated; extension). */
/* The detached pieces (GpuSolver.setPieces, solver.ts:664-677): per node its piece or 0xFFFFFFFF, piece p's
   nodes nodes[start[p] .. start[p + 1]); count pieces (start has count + 1 entries), 0 removes them. Each
   piece's rigid modes then start PCG, curve its line search and start its substeps (rigid_*.wgsl). */
int ora_set_pieces(ora_solver* s, const uint32_t* piece_of, const uint32_t* start, int32_t count, const uint32_t* nodes);
int ora_set_floor(ora_solver* s, int32_t enabled, double z, double bulge, double stiffness, double friction,
                  double friction_speed);

/* Substep and its parts (solver.ts(ref):602-632, newtonMultigrid.ts:610-645). */
int ora_predict(ora_solver* s);
int ora_newton_step(ora_solver* s, double* max_update, int32_t* pcg_iterations, double* rel_residual,
                    double* alpha);
int ora_finalize(ora_solver* s);
/* updateDamage (solver.ts(ref):659-666): field update, pull-out and span coupling at the current x. */
int ora_update_damage(ora_solver* s);
int ora_substep(ora_solver* s);

/* Energies (solver.ts(ref):387-595). */
int ora_node_gradient(ora_solver* s, int32_t n, double* g3);
double ora_potential(ora_solver* s);
int ora_energy_change(ora_solver* s, const double* d, double* e4, double* m4);
double ora_yarn_material_length(ora_solver* s);

/* Multigrid stages on the solver's current system (newtonMultigrid.ts:169-576). A: N*25*9. */
int ora_assemble(ora_solver* s, double* A, uint8_t* fixed, double* b);
/* Build the hierarchy from a given fine operator (the current state's links), as correctness.ts does. */
int ora_build_levels(ora_solver* s, const double* A_fine);
int ora_level_count(ora_solver* s);
int ora_level_nodes(ora_solver* s, int32_t level);
int ora_read_level(ora_solver* s, int32_t level, double* A, uint8_t* fixed);
int ora_read_prolongation(ora_solver* s, int32_t level, int32_t* idx, double* w);
int ora_apply(ora_solver* s, int32_t level, const double* x, double* y);
int ora_smooth(ora_solver* s, int32_t level, double* x, const double* b, int32_t reverse);
int ora_vcycle(ora_solver* s, const double* b, double* z);
int ora_pcg(ora_solver* s, const double* b, double* x, int32_t iterations, double rel_tol, int32_t* done,
            double* rel_residual);

/* Learned coarse correction (extension; no counterpart in the reference): a learned coarse space on the
   coarsest V-cycle level. A 20-64-64-24 tanh MLP maps each coarsest node's inputs (lattice position with
   sin/cos features, its normalised diagonal block, fixed-neighbour fraction, damage and contact flags)
   to 8 basis values per coordinate; half-way through the coarsest sweeps the V-cycle adds the Galerkin
   correction on that basis. A solve whose mean contraction per iteration exceeds `guard` after three
   iterations restarts from its iterate with the plain V-cycle. Weights W1[20][64], b1, W2[64][64], b2,
   W3[64][24], b3, row-major [in][out]. Logging keeps, per coarsest operator, its whitened dense form
   over the free unknowns and the node inputs, and per call the whitened residual and exact correction
   (the training material). */
int32_t ora_learned_size(void);
int32_t ora_learned_dims(int32_t* in_hidden_basis);
int ora_learned_set(ora_solver* s, const double* weights, int32_t count, int32_t on, double guard);
int ora_learned_log(ora_solver* s, int32_t on, int64_t capacity_calls);
int32_t ora_learned_ops(ora_solver* s);
int32_t ora_learned_op_nodes(ora_solver* s, int32_t k);
int ora_learned_op(ora_solver* s, int32_t k, double* At, double* X);
int32_t ora_learned_calls(ora_solver* s);
int ora_learned_call(ora_solver* s, int32_t q, int32_t* op, double* r, double* d);
int ora_learned_stats(ora_solver* s, int64_t* applied_fallbacks_solves);
int ora_learned_forward(const double* weights, const double* X, int64_t rows, double* out);
/* Test instrumentation: per (crossing, family) the last damage update's relative distance to the
 * separation threshold (cut: eps / (eps_peak + eps_soft) - 1; pull-out: delta / ((d - 1/2) pitch) - 1). */
int ora_break_margins(ora_solver* s, double* out);
int ora_learned_basis_of(ora_solver* s, const double* weights, const double* A, const uint8_t* fixed, int32_t nx, int32_t ny,
                         const float* flags, double* X, double* phi, double* G, int32_t* dead);

/* Block pentadiagonal solve (newtonMultigrid.ts:435-473). */
int ora_solve_penta(int32_t n, const double* D, const double* E, const double* F, const double* r, double* x,
                    double shift);

/* The constitutive laws on their own (axial.ts, laws.ts); yarn = {eaLow, eaHigh, crimpStrain, eaCompress}. */
void ora_law_axial(const double* yarn, double eps, double* tension_stiffness_energy);
double ora_law_strain_at_tension(const double* yarn, double t);
double ora_law_yarn_damage(const double* yarn, double yarns, double area, double peak, double soft, double eps);
void ora_law_bend_psi(double q, double a, double* psi3);
double ora_law_bend_psi_delta(double q0, double q1, double dq, double a);
void ora_law_bend_geometry(double La, double Lc, double* wa_wc_kperb_fold);
double ora_law_bend_scale(double ia, double ic, uint32_t maskA, uint32_t maskC, int32_t B);
double ora_law_shear_jam(double area);
double ora_law_cell_area(double cu, double tu, double cv, double rv);
void ora_law_shear(double ks, double Ld, double l, double jam, double* force_stiffness_energy);
void ora_law_constants(double* bend_s0_shear_jam_shear_ramp);

/* The yarn damage field's steps on a solver's own field and spans (yarnField.ts). */
int ora_field_layer(ora_solver* o, int32_t layer, int32_t* foff_K_M_bu_bv_nx_ny_nodeoff);
int32_t ora_field_span_crossing(ora_solver* o, int32_t layer, int32_t i, int32_t j, int32_t f, int32_t q, int32_t p);
int32_t ora_field_own_span(ora_solver* o, int32_t layer, int32_t k, int32_t m, int32_t f, int32_t* ij);
double ora_field_interpolated_strain(ora_solver* o, int32_t layer, int32_t f, int32_t k, int32_t m, const double* strain);
int32_t ora_field_couple(ora_solver* o);
int ora_field_update(ora_solver* o, const double* strain);
int32_t ora_field_pull_out(ora_solver* o, const double* strain);
double ora_field_recoil_length(const double* yarn, double B, double area, double peak, double eps, double mu, double n0, double wrap,
                               double t_cross, double pitch);
int32_t ora_field_share_reach(ora_solver* o, int32_t layer, int32_t f);
double ora_field_share_factor(ora_solver* o, int32_t layer, const uint8_t* sep, int32_t f, int32_t k, int32_t m, int32_t reach, double cap);
double ora_field_share_cap(int32_t reach, double mu, double n0, double wrap, double t_cross, double peak);
void ora_field_constants(double* share_fraction_cut_pulled);

#ifdef __cplusplus
}
#endif

#endif
