/* CPU restatement (plain C, FP64) of OctLB's per-level time step.
 * TEST INFRASTRUCTURE ONLY -- see octlb_oracle.h.  Citations are path:line in
 * the gezengran/octlb tree. */
#include "octlb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <pthread.h>

#define Q 19

/* D3Q19 lattice: velocities, opposites, weights
 * (src/solver/lbm/descriptor/definition/common.h:165-197). */
static const int C[Q][3] = {
    {0, 0, 0},   {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {-1, -1, 0}, {-1, 1, 0}, {-1, 0, -1},
    {-1, 0, 1},  {0, -1, -1}, {0, -1, 1}, {1, 0, 0},  {0, 1, 0},   {0, 0, 1},  {1, 1, 0},
    {1, -1, 0},  {1, 0, 1},  {1, 0, -1}, {0, 1, 1},  {0, 1, -1}};
static const int OPP[Q] = {0, 10, 11, 12, 13, 14, 15, 16, 17, 18, 1, 2, 3, 4, 5, 6, 7, 8, 9};
static const double W[Q] = {1.0 / 3,  1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 36, 1.0 / 36, 1.0 / 36,
                            1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 18, 1.0 / 18, 1.0 / 18, 1.0 / 36,
                            1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};

/* BcKind codes (src/solver/lbm/bc_kind.h:14-23). */
enum { K_BULK = 0, K_SOLID = 1, K_BOUNCE = 2, K_MOVING = 3, K_BOUZIDI = 4, K_VEL = 5, K_PRES = 6, K_OUT = 7 };

/* BcKindReflectsOnPull (src/solver/lbm/bc_kind.h:30-33). */
static int reflects_on_pull(int k) { return k == K_VEL || k == K_PRES || k == K_BOUZIDI; }

/* Shifted second-order equilibrium (src/solver/lbm/dynamics/lbm.h:50-64):
 * rho t_i (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u^2) - t_i. */
double orc_feq(int i, double rho, double ux, double uy, double uz) {
  const double cu = C[i][0] * ux + C[i][1] * uy + C[i][2] * uz;
  const double usq = ux * ux + uy * uy + uz * uz;
  return rho * W[i] * (1.0 + 3.0 * cu + 9.0 * 0.5 * cu * cu - 3.0 * 0.5 * usq) - W[i];
}

/* Moments of shifted populations (src/solver/lbm/block_lattice.h:113-125):
 * rho = 1 + sum f, u = sum f c / rho. */
static void rho_u(const double* f, double* rho, double u[3]) {
  double r = 1.0, jx = 0, jy = 0, jz = 0;
  for (int i = 0; i < Q; ++i) {
    r += f[i];
    jx += f[i] * C[i][0];
    jy += f[i] * C[i][1];
    jz += f[i] * C[i][2];
  }
  *rho = r;
  u[0] = jx / r; u[1] = jy / r; u[2] = jz / r;
}

/* BGK on one cell, f += omega (feq - f)
 * (src/solver/lbm/block_lattice.cpp:328-341). */
static void bgk(double* f, double omega) {
  double rho, u[3];
  rho_u(f, &rho, u);
  for (int i = 0; i < Q; ++i) f[i] += omega * (orc_feq(i, rho, u[0], u[1], u[2]) - f[i]);
}

/* Bouzidi interpolated bounce-back, the reference's argument roles
 * (src/solver/lbm/boundary/bouzidi_pull.h:8-26). */
double orc_bouzidi_pull(double f_bb, double f_q, double f_same, double q) {
  if (q >= 1.0 - 1.0e-14 || q <= 1.0e-14) return f_bb;
  if (q >= 0.5 - 1.0e-14) {
    const double inv2q = 1.0 / (2.0 * q);
    return inv2q * f_bb + (1.0 - inv2q) * f_q;
  }
  return 2.0 * q * f_bb + (1.0 - 2.0 * q) * f_same;
}

struct orc_block {
  int nx, ny, nz, NX, NY, NZ;
  double* f;     /* padded AoS */
  double* tmp;   /* stream target (stream_tmp_) */
  double* snap;  /* post-collide snapshot or NULL */
  uint8_t* kind; /* core cells [nx][ny][nz] */
  double* q;     /* dense link table [nx][ny][nz][19] (default 1.0) or NULL */
  int q_shared;  /* q points into a table owned elsewhere */
};

static size_t hidx(const orc_block* b, int hx, int hy, int hz) {
  return ((size_t)(hx * b->NY + hy) * b->NZ + hz) * Q;
}
static int kidx(const orc_block* b, int x, int y, int z) { return (x * b->ny + y) * b->nz + z; }

orc_block* orc_block_new(int nx, int ny, int nz) {
  orc_block* b = (orc_block*)calloc(1, sizeof(orc_block));
  b->nx = nx; b->ny = ny; b->nz = nz;
  b->NX = nx + 2; b->NY = ny + 2; b->NZ = nz + 2;
  const size_t m = (size_t)b->NX * b->NY * b->NZ * Q;
  b->f = (double*)calloc(m, sizeof(double));
  b->tmp = (double*)calloc(m, sizeof(double));
  b->kind = (uint8_t*)calloc((size_t)nx * ny * nz, 1);
  return b;
}
void orc_block_free(orc_block* b) {
  if (!b) return;
  free(b->f); free(b->tmp); free(b->snap); free(b->kind);
  if (!b->q_shared) free(b->q);
  free(b);
}

/* Equilibrium initialisation of the core (block_lattice.cpp:272-285). */
void orc_block_initialize(orc_block* b, double rho, double ux, double uy, double uz) {
  for (int x = 0; x < b->nx; ++x)
    for (int y = 0; y < b->ny; ++y)
      for (int z = 0; z < b->nz; ++z) {
        double* f = b->f + hidx(b, x + 1, y + 1, z + 1);
        for (int i = 0; i < Q; ++i) f[i] = orc_feq(i, rho, ux, uy, uz);
      }
}
void orc_block_set_kinds(orc_block* b, const uint8_t* kinds) {
  memcpy(b->kind, kinds, (size_t)b->nx * b->ny * b->nz);
}
void orc_block_get_padded(const orc_block* b, double* out) {
  memcpy(out, b->f, (size_t)b->NX * b->NY * b->NZ * Q * sizeof(double));
}
void orc_block_set_padded(orc_block* b, const double* in) {
  memcpy(b->f, in, (size_t)b->NX * b->NY * b->NZ * Q * sizeof(double));
}

/* collide(): BGK on kBulk core cells only; overlap padding has no dynamics by
 * default (block_lattice.cpp:376-417, block_lattice.h:315-316). */
void orc_block_collide(orc_block* b, double omega) {
  for (int x = 0; x < b->nx; ++x)
    for (int y = 0; y < b->ny; ++y)
      for (int z = 0; z < b->nz; ++z)
        if (b->kind[kidx(b, x, y, z)] == K_BULK) bgk(b->f + hidx(b, x + 1, y + 1, z + 1), omega);
}

/* fill_periodic_halo(): x faces over the core y,z range, then y faces over
 * all x, then z faces over all x,y (block_lattice.cpp:918-964). */
void orc_block_fill_periodic(orc_block* b) {
  const int nx = b->nx, ny = b->ny, nz = b->nz, sz = Q * (int)sizeof(double);
  for (int y = 1; y <= ny; ++y)
    for (int z = 1; z <= nz; ++z) {
      memcpy(b->f + hidx(b, 0, y, z), b->f + hidx(b, nx, y, z), sz);
      memcpy(b->f + hidx(b, nx + 1, y, z), b->f + hidx(b, 1, y, z), sz);
    }
  for (int x = 0; x < b->NX; ++x)
    for (int z = 1; z <= nz; ++z) {
      memcpy(b->f + hidx(b, x, 0, z), b->f + hidx(b, x, ny, z), sz);
      memcpy(b->f + hidx(b, x, ny + 1, z), b->f + hidx(b, x, 1, z), sz);
    }
  for (int x = 0; x < b->NX; ++x)
    for (int y = 0; y < b->NY; ++y) {
      memcpy(b->f + hidx(b, x, y, 0), b->f + hidx(b, x, y, nz), sz);
      memcpy(b->f + hidx(b, x, y, nz + 1), b->f + hidx(b, x, y, 1), sz);
    }
}

void orc_block_snapshot(orc_block* b) {
  const size_t m = (size_t)b->NX * b->NY * b->NZ * Q;
  if (!b->snap) b->snap = (double*)malloc(m * sizeof(double));
  memcpy(b->snap, b->f, m * sizeof(double));
}

/* Torus pull over the padded block's linear index
 * (block_lattice.h:70-89): src = (dst - (cx NY NZ + cy NZ + cz)) mod cells. */
static size_t rotate_src(const orc_block* b, long dst_lin, int i) {
  const long cells = (long)b->NX * b->NY * b->NZ;
  const long off = (long)C[i][0] * b->NY * b->NZ + (long)C[i][1] * b->NZ + C[i][2];
  long s = (dst_lin - off) % cells;
  if (s < 0) s += cells;
  return (size_t)s * Q + i;
}

static int kind_at_halo(const orc_block* b, int hx, int hy, int hz) {
  const int x = hx - 1, y = hy - 1, z = hz - 1;
  if (x < 0 || y < 0 || z < 0 || x >= b->nx || y >= b->ny || z >= b->nz) return K_BULK;
  return b->kind[kidx(b, x, y, z)];
}
static int in_core_h(const orc_block* b, int hx, int hy, int hz) {
  return hx >= 1 && hy >= 1 && hz >= 1 && hx <= b->nx && hy <= b->ny && hz <= b->nz;
}

/* stream(): without a link table every padded slot is torus-pulled
 * (block_lattice.cpp:554-557,676-688); with one, halo slots pull directly (torus
 * when the source leaves the block), solid core cells are skipped, reflecting
 * kinds bounce back when the source is not interior, and solid / Bouzidi
 * sources are bounced back or Bouzidi-interpolated (block_lattice.cpp:579-720). */
void orc_block_stream(orc_block* b) {
  const double* f = b->f;
  double* t = b->tmp;
  const int NX = b->NX, NY = b->NY, NZ = b->NZ;
  if (!b->q) {
    for (int hx = 0; hx < NX; ++hx)
      for (int hy = 0; hy < NY; ++hy)
        for (int hz = 0; hz < NZ; ++hz) {
          const long lin = ((long)hx * NY + hy) * NZ + hz;
          for (int i = 0; i < Q; ++i) t[lin * Q + i] = f[rotate_src(b, lin, i)];
        }
    memcpy(b->f, b->tmp, (size_t)NX * NY * NZ * Q * sizeof(double));
    return;
  }
  for (int hx = 0; hx < NX; ++hx)
    for (int hy = 0; hy < NY; ++hy)
      for (int hz = 0; hz < NZ; ++hz) {
        const int core = in_core_h(b, hx, hy, hz);
        const int kind = core ? b->kind[kidx(b, hx - 1, hy - 1, hz - 1)] : K_BULK;
        if (core && kind == K_SOLID) continue;
        const long lin = ((long)hx * NY + hy) * NZ + hz;
        const size_t dst = (size_t)lin * Q;
        for (int i = 0; i < Q; ++i) {
          const int sx = hx - C[i][0], sy = hy - C[i][1], sz = hz - C[i][2];
          const int in_blk = sx >= 0 && sy >= 0 && sz >= 0 && sx < NX && sy < NY && sz < NZ;
          if (!core) { /* overlap padding: direct pull, torus outside */
            t[dst + i] = in_blk ? f[hidx(b, sx, sy, sz) + i] : f[rotate_src(b, lin, i)];
            continue;
          }
          /* core sources are always inside the padded block (halo 1) */
          if (reflects_on_pull(kind) && !in_core_h(b, sx, sy, sz)) {
            t[dst + i] = f[dst + OPP[i]];
            continue;
          }
          const int sk = kind_at_halo(b, sx, sy, sz);
          if (sk == K_SOLID || sk == K_BOUZIDI) {
            const double q = b->q[(size_t)kidx(b, hx - 1, hy - 1, hz - 1) * Q + i];
            if (q > 1.0e-10 && q < 1.0 - 1.0e-10) {
              double f_q = f[dst + i];
              const int nx_ = hx + C[i][0], ny_ = hy + C[i][1], nz_ = hz + C[i][2];
              if (kind_at_halo(b, nx_, ny_, nz_) == K_BULK) f_q = f[hidx(b, nx_, ny_, nz_) + i];
              t[dst + i] = orc_bouzidi_pull(f[dst + OPP[i]], f_q, f[dst + i], q);
            } else {
              t[dst + i] = f[dst + OPP[i]];
            }
            continue;
          }
          t[dst + i] = f[hidx(b, sx, sy, sz) + i];
        }
      }
  for (int hx = 0; hx < NX; ++hx)
    for (int hy = 0; hy < NY; ++hy)
      for (int hz = 0; hz < NZ; ++hz) {
        if (in_core_h(b, hx, hy, hz) && b->kind[kidx(b, hx - 1, hy - 1, hz - 1)] == K_SOLID) continue;
        const size_t d = hidx(b, hx, hy, hz);
        memcpy(b->f + d, b->tmp + d, Q * sizeof(double));
      }
}

/* Dense q table with default 1.0 and the given cut links
 * (src/solver/lbm/bouzidi_link_data.cpp:107-137). */
void orc_block_set_links(orc_block* b, int n_links, const int* cp, const double* q) {
  const size_t m = (size_t)b->nx * b->ny * b->nz * Q;
  if (!b->q || b->q_shared) { b->q = (double*)malloc(m * sizeof(double)); b->q_shared = 0; }
  for (size_t k = 0; k < m; ++k) b->q[k] = 1.0;
  for (int k = 0; k < n_links; ++k)
    b->q[(size_t)kidx(b, cp[4 * k], cp[4 * k + 1], cp[4 * k + 2]) * Q + cp[4 * k + 3]] = q[k];
}

/* Moving-wall momentum term (Ladd 1994), restated -- the reference has no
 * runtime arm for kMovingBounceBack (bc_dispatcher.h:75-79): a link pulled from
 * a moving solid / Bouzidi core cell s gains 6 w_i (c_i . u_w(s)). */
void orc_block_add_moving_wall(orc_block* b, const uint8_t* moving, const double* uw) {
  for (int x = 0; x < b->nx; ++x)
    for (int y = 0; y < b->ny; ++y)
      for (int z = 0; z < b->nz; ++z) {
        if (b->kind[kidx(b, x, y, z)] == K_SOLID) continue;
        double* f = b->f + hidx(b, x + 1, y + 1, z + 1);
        for (int i = 1; i < Q; ++i) {
          const int sx = x - C[i][0], sy = y - C[i][1], sz = z - C[i][2];
          if (sx < 0 || sy < 0 || sz < 0 || sx >= b->nx || sy >= b->ny || sz >= b->nz) continue;
          const int s = kidx(b, sx, sy, sz);
          if (b->kind[s] != K_SOLID && b->kind[s] != K_BOUZIDI) continue;
          if (!moving[s]) continue;
          f[i] += 6.0 * W[i] * (C[i][0] * uw[3 * s] + C[i][1] * uw[3 * s + 1] + C[i][2] * uw[3 * s + 2]);
        }
      }
}

/* collide -> fill_periodic_halo -> stream
 * (tests/unit/solver/test_collision_bgk.cpp:56-60). */
void orc_block_run_periodic(orc_block* b, double omega, int steps) {
  for (int t = 0; t < steps; ++t) {
    orc_block_collide(b, omega);
    orc_block_fill_periodic(b);
    orc_block_stream(b);
  }
}
void orc_block_run_walls(orc_block* b, double omega, int steps, const uint8_t* moving,
                         const double* uw) {
  for (int t = 0; t < steps; ++t) {
    orc_block_collide(b, omega);
    orc_block_stream(b);
    if (moving) orc_block_add_moving_wall(b, moving, uw);
  }
}

/* Momentum-exchange force on the fluid: -sum (f_i^snap + f_opp^live) c_i over
 * kBulk cells and in-block solid / Bouzidi neighbours passing the obstacle
 * predicate (src/solver/lbm/drag_postprocessor.h:67-115). */
void orc_block_drag(const orc_block* b, const uint8_t* mask, double out[3]) {
  double F[3] = {0, 0, 0};
  for (int z = 0; z < b->nz; ++z)
    for (int y = 0; y < b->ny; ++y)
      for (int x = 0; x < b->nx; ++x) {
        if (b->kind[kidx(b, x, y, z)] != K_BULK) continue;
        const double* live = b->f + hidx(b, x + 1, y + 1, z + 1);
        const double* snap = b->snap ? b->snap + hidx(b, x + 1, y + 1, z + 1) : live;
        for (int i = 1; i < Q; ++i) {
          const int nx_ = x + C[i][0], ny_ = y + C[i][1], nz_ = z + C[i][2];
          if (nx_ < 0 || ny_ < 0 || nz_ < 0 || nx_ >= b->nx || ny_ >= b->ny || nz_ >= b->nz) continue;
          const int nk = b->kind[kidx(b, nx_, ny_, nz_)];
          if (nk != K_SOLID && nk != K_BOUZIDI) continue;
          if (mask && !mask[kidx(b, nx_, ny_, nz_)]) continue;
          const double s = snap[i] + live[OPP[i]];
          F[0] += s * C[i][0]; F[1] += s * C[i][1]; F[2] += s * C[i][2];
        }
      }
  out[0] = -F[0]; out[1] = -F[1]; out[2] = -F[2];
}

/* Multi-core CPU baseline: `slabs` independent periodic boxes of nx*ny*(nz/slabs),
 * stepped with the loop above, `threads` POSIX threads taking slabs round-robin. */
typedef struct { orc_block** bl; int first, stride, n; double omega; int steps; } slab_job;
static void* slab_worker(void* arg) {
  slab_job* j = (slab_job*)arg;
  for (int s = j->first; s < j->n; s += j->stride) orc_block_run_periodic(j->bl[s], j->omega, j->steps);
  return NULL;
}
double orc_periodic_slabs_mlups(int nx, int ny, int nz, int slabs, int threads, double omega,
                                int steps) {
  const int nzs = nz / slabs;
  orc_block** bl = (orc_block**)calloc((size_t)slabs, sizeof(*bl));
  for (int s = 0; s < slabs; ++s) {
    bl[s] = orc_block_new(nx, ny, nzs);
    orc_block_initialize(bl[s], 1.0, 0.01, 0.0, 0.0);
  }
  if (threads < 1) threads = 1;
  pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
  slab_job* jobs = (slab_job*)calloc((size_t)threads, sizeof(slab_job));
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (int k = 0; k < threads; ++k) {
    jobs[k] = (slab_job){bl, k, threads, slabs, omega, steps};
    pthread_create(&th[k], NULL, slab_worker, &jobs[k]);
  }
  for (int k = 0; k < threads; ++k) pthread_join(th[k], NULL);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  const double sec = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
  for (int s = 0; s < slabs; ++s) orc_block_free(bl[s]);
  free(bl); free(th); free(jobs);
  return (double)nx * ny * (double)(nzs * slabs) * steps / sec / 1e6;
}

/* The periodic loop above (collide -> fill_periodic_halo -> stream) with the
 * collide and the torus stream split over `threads` POSIX threads by x
 * planes: every cell gets the same arithmetic as in the serial loop, so the
 * result is bitwise the serial one (only the work is shared).  For boxes the
 * serial loop takes minutes on (the 256^3 throughput box). */
typedef struct { orc_block* b; double omega; int phase, x0, x1; } mt_job;
static void* mt_worker(void* arg) {
  mt_job* j = (mt_job*)arg;
  orc_block* b = j->b;
  const int NY = b->NY, NZ = b->NZ;
  if (j->phase == 0) {
    for (int x = j->x0; x < j->x1; ++x)
      for (int y = 0; y < b->ny; ++y)
        for (int z = 0; z < b->nz; ++z)
          if (b->kind[kidx(b, x, y, z)] == K_BULK) bgk(b->f + hidx(b, x + 1, y + 1, z + 1), j->omega);
  } else if (j->phase == 1) {
    for (int hx = j->x0; hx < j->x1; ++hx)
      for (int hy = 0; hy < NY; ++hy)
        for (int hz = 0; hz < NZ; ++hz) {
          const long lin = ((long)hx * NY + hy) * NZ + hz;
          for (int i = 0; i < Q; ++i) b->tmp[lin * Q + i] = b->f[rotate_src(b, lin, i)];
        }
  } else {
    const size_t plane = (size_t)NY * NZ * Q;
    memcpy(b->f + (size_t)j->x0 * plane, b->tmp + (size_t)j->x0 * plane,
           (size_t)(j->x1 - j->x0) * plane * sizeof(double));
  }
  return NULL;
}
static void mt_phase(orc_block* b, double omega, int phase, int planes, int threads) {
  pthread_t th[256];
  mt_job jobs[256];
  if (threads > 256) threads = 256;
  if (threads > planes) threads = planes;
  for (int k = 0; k < threads; ++k) {
    jobs[k] = (mt_job){b, omega, phase, planes * k / threads, planes * (k + 1) / threads};
    pthread_create(&th[k], NULL, mt_worker, &jobs[k]);
  }
  for (int k = 0; k < threads; ++k) pthread_join(th[k], NULL);
}
int orc_block_run_periodic_mt(orc_block* b, double omega, int steps, int threads) {
  if (b->q) return -1; /* the torus stream only (no link table) */
  if (threads < 1) threads = 1;
  for (int t = 0; t < steps; ++t) {
    mt_phase(b, omega, 0, b->nx, threads);
    orc_block_fill_periodic(b);
    mt_phase(b, omega, 1, b->NX, threads);
    mt_phase(b, omega, 2, b->NX, threads);
  }
  return 0;
}

/* rho and u of every core cell, [nx][ny][nz] and [nx][ny][nz][3]
 * (block_lattice.h:113-125), without a padded copy. */
void orc_block_fields(const orc_block* b, double* rho, double* u) {
  for (int x = 0; x < b->nx; ++x)
    for (int y = 0; y < b->ny; ++y)
      for (int z = 0; z < b->nz; ++z) {
        const size_t k = (size_t)kidx(b, x, y, z);
        rho_u(b->f + hidx(b, x + 1, y + 1, z + 1), &rho[k], &u[3 * k]);
      }
}
