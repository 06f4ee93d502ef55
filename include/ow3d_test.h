/*
 * ow3d_test.h -- probe entry points used by the parity tests. They expose the
 * set-up tables and the individual multigrid components of a handle so that
 * each can be compared with the CPU restatement of the reference; they have no
 * counterpart in the reference program and are not part of the drop-in API.
 * They are exported only by the testing build of the library
 * (libow3d_dev.so, the same objects linked without the product's export
 * list); libow3d.so exports the functions of ow3d.h alone.
 */
#ifndef OW3D_TEST_H
#define OW3D_TEST_H
#include "ow3d.h"
#ifdef __cplusplus
extern "C" {
#endif

/* n deviates of the incident-wave generator (Park-Miller with the
 * Bays-Durham shuffle, RAN1_b.f90) started from idum, and the final idum. */
int ow3d_test_ran1(int idum, int n, float* out, int* idum_out);
/* The pressure-damping zone a 2-D deck sets up (host only, flat bottom):
 * its first point i1 (1-based, ghosts included) and its nd points, gamma_phi
 * and gamma_eta over the row (Nxg each), and for type 0 the zone matrix L
 * (Dirichlet row, Laplacian rows, Neumann row; nd x nd, row-major) and the
 * inverse the device applies. Arrays may be null. */
int ow3d_test_pdamp_setup(const ow3d_params* p, int* i1, int* nd, double* gamPhi, double* gamEta, double* L,
                          double* Linv);
/* eta_x and eta_y of the current state as the device holds them (Nxg*Nyg
 * each; on the ghost rows they are the derivatives taken before that
 * direction's ghost update, as DifferentiationsFreeSurfacePlane leaves them). */
int ow3d_test_surface_derivs(ow3d_handle* h, double* Ex, double* Ey);
/* High-order stencil tables [order-1][pos][7] for x (2*Nxg*7), y (2*Nyg*7), sigma (2*Nzg*7). */
int ow3d_test_stencils(const ow3d_handle* h, double* SX, double* SY, double* SZ);
int ow3d_test_level_z(const ow3d_handle* h, int level, double* z);
int ow3d_test_zone_gamma(const ow3d_handle* h, int zone, double* gamma);
int ow3d_test_filter_coeffs(const ow3d_handle* h, double* centre, double* boundary);
/* Multigrid component on level `level` (0 = coarsest), in the handle's precision:
 * op 0: out = A_l in1;  op 1: out = smoothed in1 with rhs in2 (nu steps);
 * op 2: out = restriction of the fine residual in1 to level-1;
 * op 3: out = prolongation of the level-1 vector in1 (added to zero);
 * op 4: out = coarsest-level solve of in1 (level 0 only);
 * op 5: out = in1 after one smoother phase with rhs in2: colour pass `nu`, or
 *       the bottom-row pass when nu < 0 (levels with mixed-derivative terms). */
int ow3d_test_level_op(ow3d_handle* h, int level, int op, int nu, const double* in1, const double* in2, double* out);

/* Tuning knob for measurements: cap on the number of blocks of the fused
 * coarse-level multigrid kernel (0 = one block per SM, the default). Returns
 * the previous value. Process-wide. */
int ow3d_test_set_coarse_blocks(int blocks);

/* Tuning knob for measurements: levels with at most this many points run in
 * the fused coarse-level kernel (default 160000; 0 = none, every level above
 * the dense one as separate launches). Read when a V-cycle is launched, so it
 * applies to handles created after the change (and to captures made after
 * it). Returns the previous value. Process-wide. */
long long ow3d_test_set_coop_max_points(long long points);
/* Levels of at most `points` points run in the cluster (tail) kernel of the
 * fused coarse cycle (0: no tail), and the cluster's block count (8 or 16);
 * each returns the previous value. Process-wide. */
/* Programmatic dependent launch between the solver's kernels (1, the
 * default) or plain launches (0). Applies to launches made after the call:
 * captured graphs keep what they were captured with. Returns the previous
 * value. Process-wide. */
int ow3d_test_set_pdl(int on);
long long ow3d_test_set_tail_max_points(long long points);
int ow3d_test_set_tail_cluster(int blocks);

/* Levels without mixed-derivative terms that cover at least `min_tiles`
 * tiles of 32 x 8 columns take the tiled colour pass (columns away from the
 * walls solved from shared-memory tiles); 0: the per-column colour pass on
 * every level, the default. Both give bitwise-identical results. Returns the
 * previous value. Process-wide. */
int ow3d_test_set_colour_tiles(int min_tiles);

/* Per-level colour pass launch form: 0 one pass over the columns with up to
 * 32 blocks per SM; 1 the grid capped at the resident blocks per SM, each
 * warp prefetching its next group of columns into L1; 2 the capped grid
 * alone; -1 (the default) 2 on FP64 levels and 0 on FP32 ones. Results are
 * bitwise the same. Returns the previous value. Process-wide. */
int ow3d_test_set_colour_prefetch(int mode);

/* Number of captured Arnoldi-step graphs the handle holds, or -1 when a
 * capture failed and the handle launches kernels directly. */
int ow3d_test_graph_count(const ow3d_handle* h);

/* Number of whole-step graphs the handle holds (0..2, one per step parity),
 * or -1 when a step capture failed and the handle steps directly. */
int ow3d_test_step_graph_count(const ow3d_handle* h);

/* The relaxation target of generation zone `zone` as the device holds it:
 * nt x box samples each of eta and phis (either may be NULL). */
int ow3d_test_relax_target(const ow3d_handle* h, int zone, double* eta, double* phis);

/* The roller breaking model's state: tan(phi) per column (the angle carried
 * between steps) and the Qr_x of its last call, Nxg each (either may be NULL).
 * OW3D_ERR_BAD_INPUT when the handle runs no breaking model. */
int ow3d_test_breaking_state(ow3d_handle* h, double* tan_phi, double* Qr_x);
/* One call of the breaking model on the surface E (Nxg values; update: the
 * call after a step, with the roller-angle update and the roller record).
 * Uses the handle's stage buffer for E. */
int ow3d_test_detect_breaking(ow3d_handle* h, const double* E, int update);
/* The last step's local smoothing (accel_tol_fact <= 100): the surface
 * Lagrangian dw/dt and the flags of the points where -dw/dt reached the
 * limit, Nxg*Nyg each (either may be NULL; both zero before the third step). */
int ow3d_test_accel_state(ow3d_handle* h, double* Wt, int* flags);

/* sizeof the C structs: 0 ow3d_params, 1 ow3d_zone, 2 ow3d_stats. */
int ow3d_test_sizeof(int which);

#ifdef __cplusplus
}
#endif
#endif
