/* CPU restatement (plain C, FP64) of OctLB's per-level time step, used as the
 * test oracle and as the "port" CPU baseline.  TEST INFRASTRUCTURE: only the
 * tests, __graft_entry__.smoke() and bench.py's CPU legs load it; the product
 * never does.
 *
 * Every function restates a reference function; the citation (path:line,
 * relative to the gezengran/octlb tree) sits next to it in octlb_oracle.c.
 * The block layout is the reference's own: populations of one block stored
 * AoS as [(nx+2)][(ny+2)][(nz+2)][19] including a one-cell halo
 * (src/solver/lbm/block_lattice.h:294-304); BcKind codes are those of
 * src/solver/lbm/bc_kind.h:14-23. */
#ifndef OCTLB_ORACLE_H_
#define OCTLB_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_block orc_block;

orc_block* orc_block_new(int nx, int ny, int nz);
void orc_block_free(orc_block* b);
void orc_block_initialize(orc_block* b, double rho, double ux, double uy, double uz);
void orc_block_set_kinds(orc_block* b, const uint8_t* kinds);
void orc_block_get_padded(const orc_block* b, double* out);
void orc_block_set_padded(orc_block* b, const double* in);
void orc_block_collide(orc_block* b, double omega);
void orc_block_fill_periodic(orc_block* b);
void orc_block_stream(orc_block* b);
void orc_block_snapshot(orc_block* b);
void orc_block_set_links(orc_block* b, int n_links, const int* cell_pop, const double* q);
void orc_block_add_moving_wall(orc_block* b, const uint8_t* moving, const double* uw);
void orc_block_run_periodic(orc_block* b, double omega, int steps);
void orc_block_run_walls(orc_block* b, double omega, int steps, const uint8_t* moving,
                         const double* uw);
void orc_block_drag(const orc_block* b, const uint8_t* mask, double out[3]);
/* orc_block_run_periodic on `threads` POSIX threads, bitwise equal to it
 * (blocks without a link table; -1 otherwise). */
int orc_block_run_periodic_mt(orc_block* b, double omega, int steps, int threads);
/* rho [nx][ny][nz] and u [nx][ny][nz][3] of the core cells. */
void orc_block_fields(const orc_block* b, double* rho, double* u);

/* Periodic box as independent slabs (z-slices of the full box each own a
 * periodic halo), run on `threads` POSIX threads: the multi-core CPU
 * baseline (one slab per core, no halo exchange between slabs). */
double orc_periodic_slabs_mlups(int nx, int ny, int nz, int slabs, int threads,
                                double omega, int steps);

double orc_feq(int i, double rho, double ux, double uy, double uz);
double orc_bouzidi_pull(double f_bb, double f_q, double f_same, double q);

/* Octree sim: same forest description as the reference oracle's ref_sim_new. */
typedef struct orc_sim orc_sim;
orc_sim* orc_sim_new(int n_oct, const int* levels, const double* bounds, int n_sl,
                     const int* sl, int n_cf, const int* cf, const double* cf_bounds,
                     int n_tb, const int* tb, const double* tb_spec, int n, double omega,
                     const uint8_t* kinds, const double* core_pops, int n_links,
                     const int* link_cells, const double* link_q, int link_mode);
void orc_sim_free(orc_sim* s);
void orc_sim_advance(orc_sim* s, int steps);
void orc_sim_get_core(const orc_sim* s, double* out);
void orc_sim_drag(const orc_sim* s, const uint8_t* mask, double out[3]);
int orc_sim_plan(const orc_sim* s, int* out, int max_pts);

#ifdef __cplusplus
}
#endif
#endif
