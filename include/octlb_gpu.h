/* octlb_gpu.h -- C ABI of the B200 (sm_100a) per-level LBM time step.
 *
 * This is the drop-in boundary for OctLB's per-level time step: one context
 * holds, on one GPU, every octree level's blocks (SoA populations in HBM), the
 * flattened topology the reference keeps in FacePairList / GhostSchedule /
 * LevelCoupler, and the TimeLoop recursion.  Plain C99: no C++ or torch types,
 * no exceptions across the boundary.  0 = OK, negative = error; the message of
 * the last error is available from octlb_gpu_last_error().
 *
 * Reference interfaces each entry point replaces (paths in gezengran/octlb):
 *   octlb_gpu_create    TimeLoop ctor + BlockCollection factory + GhostSchedule
 *                       ctor + LevelCoupler ctor + BouzidiLinkData
 *                       (src/solver/lbm/time_loop/time_loop.h:49-54,123-164;
 *                        src/solver/field/ghost_schedule.h:23-119;
 *                        src/solver/lbm/level_coupler.cpp:216-307;
 *                        src/solver/lbm/bouzidi_link_data.cpp:107-137)
 *   octlb_gpu_advance   TimeLoop::advance_one (time_loop.h:242-246), n times
 *   octlb_gpu_force     MomentumExchangeDrag::force_on_fluid_if summed over
 *                       blocks (src/solver/lbm/drag_postprocessor.h:67-115,
 *                        examples/cylinder3d/cylinder3d_case.h:473-517)
 *   octlb_gpu_audit     Cylinder3dCase::total_mass (cylinder3d_case.h:601-622)
 *                       plus total momentum
 *   octlb_gpu_get_fields / _get_populations / _set_populations
 *                       BlockLattice::get(...).computeRhoU and direct
 *                       population access (block_lattice.h:113-125,226-256)
 *   octlb_gpu_counters  TimeLoop::counters (time_loop.h:30-34,76)
 */
#ifndef OCTLB_GPU_H_
#define OCTLB_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OCTLB_OK 0
#define OCTLB_EINVAL (-1)   /* table / argument validation failed */
#define OCTLB_ENOMEM (-2)   /* device allocation failed */
#define OCTLB_ECUDA (-3)    /* CUDA runtime error */
#define OCTLB_ENAN (-4)     /* non-finite populations detected (audit) */
#define OCTLB_ETIMEOUT (-5) /* a bounded device wait gave up (no hang) */
#define OCTLB_ESTATE (-6)   /* call not valid in the context's state */

/* Population storage.  FP32 stores the shifted populations f - w as float;
 * FP16_SHIFTED stores (f - w) * scale[level] as IEEE half.  Arithmetic is
 * FP32 in both; audits and forces accumulate in FP64. */
#define OCTLB_FP32 0
#define OCTLB_FP16_SHIFTED 1

/* Stream rule (reference BlockLattice::stream, block_lattice.cpp:554-557):
 * ROTATE = no link table attached (every padded slot is torus-pulled);
 * LINKS = a BouzidiLinkData is attached (per-cell pull with half-way
 * bounce-back / Bouzidi on solid sources, default q = 1). */
#define OCTLB_STREAM_ROTATE 0
#define OCTLB_STREAM_LINKS 1

/* Tree-boundary face conditions (restated; applied as halo fills before the
 * same-level exchange, i.e. at DomainBoundaryHandler::apply()). */
#define OCTLB_TB_NONE 0
#define OCTLB_TB_WALL 1     /* half-way bounce-back wall, optionally moving */
#define OCTLB_TB_OUTFLOW 2  /* zero-gradient ghost copy (outflow_bc.h:15-21) */

/* Flattened mesh + per-cell data.  All arrays are host memory owned by the
 * caller and copied at create.  Cell order inside a block is the reference's
 * (ix * n + iy) * n + iz (block_lattice.h:290-296). */
typedef struct octlb_tables {
  int n;                          /* cells per block edge: even, or odd (>= 3) on a mesh without coarse-fine faces */
  int n_blocks;                   /* leaves (OctantId 0..n_blocks-1) */
  const int* levels;              /* [n_blocks] quadrant level */
  const double* bounds;           /* [n_blocks][6] xmin,ymin,zmin,xmax,ymax,zmax */
  const uint8_t* kinds;           /* [n_blocks][n^3] BcKind (bc_kind.h:14-23) */
  int n_same_level;               /* FacePairList::same_level_faces() */
  const int* same_level;          /* [n][3] local_id, dir, remote_id */
  int n_coarse_fine;              /* FacePairList::coarse_fine_faces() */
  const int* coarse_fine;         /* [n][8] coarse, fine0..3, normal, clevel, flevel */
  const double* coarse_fine_bounds; /* [n][30] coarse box, then 4 fine boxes */
  int n_tree_boundary;            /* FacePairList::tree_boundary_faces() */
  const int* tree_boundary;       /* [n][2] octant_id, face_dir */
  const double* tree_boundary_spec; /* [n][8] type, u[3], prof_axis, lo, hi, 0 */
  int n_links;                    /* Bouzidi cut links (q in (0,1)) */
  const int* link_cells;          /* [n][5] octant, ix, iy, iz, pop */
  const double* link_q;           /* [n] fractional link length q */
  const uint8_t* moving;          /* [n_blocks][n^3] moving solid cells or NULL */
  const double* wall_u;           /* [n_blocks][n^3][3] their velocity or NULL */
  const uint8_t* obstacle;        /* [n_blocks][n^3] MEM obstacle mask or NULL */
  int periodic;                   /* 1: single block, periodic in x, y, z */
} octlb_tables;

/* Coupler / relaxation mode.  REFERENCE (parity with the reference): one
 * global omega collides every level (time_loop.h:183-187) and the Lagrava
 * scales are (tau - 1/4) / tau and tau / (tau - 1/4) of that tau
 * (level_coupler.cpp:226-228).  PHYSICAL: every level relaxes with its own
 * tau_l, tau_{l+1} - 1/2 = 2 (tau_l - 1/2) (the viscosity is the same on every
 * level under the 2:1 time step), and the coupler rescales the
 * non-equilibrium part by tau_f / (2 tau_c) coarse -> fine and 2 tau_c / tau_f
 * fine -> coarse (Dupuis and Chopard), which is the reference's pair of
 * scales with tau = tau_c. */
#define OCTLB_COUPLER_REFERENCE 0
#define OCTLB_COUPLER_PHYSICAL 1

/* Stream order (the storage pattern of the pull; the results do not depend on
 * it): AB keeps two population buffers, AA one (Bailey et al., "Accelerating
 * lattice Boltzmann fluid flow simulations using graphics processors", 2009). */
#define OCTLB_ORDER_AB 0
#define OCTLB_ORDER_AA 1

typedef struct octlb_params {
  double omega;                   /* REFERENCE: the global BGK rate; PHYSICAL: the
                                     rate of the coarsest level with blocks */
  int precision;                  /* OCTLB_FP32 or OCTLB_FP16_SHIFTED */
  int stream_mode;                /* OCTLB_STREAM_ROTATE or OCTLB_STREAM_LINKS */
  int drag;                       /* 1: MEM force every coarse step */
  double fp16_scale[32];          /* per-level scale; 0 = default 2^16 */
  int coupler_mode;               /* OCTLB_COUPLER_REFERENCE (0) or _PHYSICAL */
  double omega_level[32];         /* PHYSICAL: explicit rate of level l, or 0 for
                                     the rescaled one */
  int stream_order;               /* OCTLB_ORDER_AB (0): two population buffers,
                                     pull from one into the other; OCTLB_ORDER_AA:
                                     one buffer updated in place, alternating a
                                     step that pulls from and writes back to the
                                     neighbours with one that reads and writes the
                                     cell's own slots (uniform periodic box only:
                                     one level, every cell kBulk, one context, no
                                     body force, ConstRhoBGK, drag or adjoint);
                                     half the memory, the same results bitwise */
} octlb_params;

typedef struct octlb_ctx octlb_ctx;

/* init_pops: [n_blocks][n^3][19] shifted populations (the reference state
 * before a step), or NULL for equilibrium at rho = 1, u = 0. */
int octlb_gpu_create(const octlb_tables* tables, const octlb_params* params,
                     const double* init_pops, octlb_ctx** out);
void octlb_gpu_destroy(octlb_ctx* ctx);
const char* octlb_gpu_last_error(const octlb_ctx* ctx);

/* Bind the context to a caller's cudaStream_t (NULL = the context's own). */
int octlb_gpu_set_stream(octlb_ctx* ctx, void* cuda_stream);

/* n_coarse_steps x TimeLoop::advance_one(), asynchronously on the stream. */
int octlb_gpu_advance(octlb_ctx* ctx, int n_coarse_steps);
int octlb_gpu_synchronize(octlb_ctx* ctx);

/* Body force F per core cell, [n_blocks][n^3][3] doubles (stored as FP32),
 * or NULL to remove it: the forcing term 3 w_i (c_i . F) is added to the
 * post-collision populations of every kBulk cell once per step of its level
 * (no reference counterpart: the reference has no body force; this is the
 * adjoint's per-cell control). */
int octlb_gpu_set_body_force(octlb_ctx* ctx, const double* force);

/* ConstRhoBGK on (1) or off (0): the TimeLoop constructor argument
 * use_const_rho_bgk with ConstRhoStatsScope::kFluidAndBoundary
 * (time_loop.h:47-54; collide block_lattice.cpp:441-455 and
 * block_lattice.h:134-151; statistics time_loop.h:201-222).  Every kBulk
 * cell collides with ratio_rho = 1 + (1 - average_rho) / rho, and after each
 * step average_rho becomes the mean of rho + (1 - average_rho) over the kBulk
 * cells of that collide (the reference starts at 1).  On a multi-level mesh
 * the statistics are the finest level's and every level collides at the
 * average: the levels above the finest then stream in their step and collide
 * after their coupling (one launch more per level step; a prolongation into
 * the finest level takes its target's collide and statistic).  Before the
 * first advance only (OCTLB_ESTATE after it); one context, not rank contexts
 * (OCTLB_EINVAL).  The adjoint refuses a ConstRhoBGK context.  get_fields returns the
 * reference's post-stream rho (the stored post-collision state minus the
 * 1 - average_rho the collide added to each kBulk cell; u is unchanged). */
int octlb_gpu_set_const_rho(octlb_ctx* ctx, int on);

/* TimeLoop::average_rho() (time_loop.h:87-88): the average density the next
 * ConstRhoBGK collide uses; 1 without ConstRhoBGK.  Synchronises the stream. */
int octlb_gpu_average_rho(octlb_ctx* ctx, double* out);

/* ---- Finite-difference domain boundary conditions -------------------------
 * The reference's ConcreteDomainBoundaryHandler (domain_boundary_handler.cpp:
 * 55-89) on the tree-boundary faces, types as DomainBcType
 * (domain_boundary_handler.h:16-22): 2 InterpolatedVelocity, 4
 * InterpolatedPressure (the finite-difference conditions), 0 no-slip (its
 * kBounceBack cells take the dispatcher's full-way swap at collide,
 * bc_dispatcher.h:55-67), 1 moving lid and 3 outflow (kinds with no
 * collide-time action there, streamed as they are).  Every step, after the pull and the
 * collide of the fluid cells, the velocity- and pressure-Dirichlet cells are
 * rebuilt from the finite-difference stencil of Skordos' method (plane, edge
 * and corner cells by their block's extents, in the reference's walk order,
 * interpolated_velocity.h:571-1037) and the velocity cells then collide at
 * their prescribed velocity (bc_dispatcher.h:55-72).  Prescribed velocity:
 * the inlet field of the first face the cell touches that has one (uniform
 * inlet_u[face] ramped by 10x^3 - 15x^4 + 6x^5, x = t / ramp_end_t), else
 * u_wall of the y+ face on the interior top-face cells (cavity3d's lid);
 * pressure cells hold rho_target[face].  The cells must carry their kinds in
 * the tables (octlb_fd_stamp_kinds), the faces no restated fill
 * (OCTLB_TB_NONE).  One context, the rotate stream rule, blocks of
 * n >= 4; before the first advance.  Any number of levels, as the reference
 * runs it: after every level's stream (an empty level's included) the pass
 * rewrites the Dirichlet cells of every level's tree-boundary blocks, and
 * each level's boundary cells collide at the start of its step; on a
 * multi-level mesh the coarse-fine interfaces must stay away from the
 * domain faces (every coupler source and target a kBulk cell; OCTLB_EINVAL
 * otherwise).  With ConstRhoBGK (octlb_gpu_set_const_rho, called first; any
 * number of levels) the finest level's velocity cells' collide densities join
 * the average's statistics, as the reference's kFluidAndBoundary scope does
 * (cavity3d's configuration). */
#define OCTLB_FD_NO_SLIP 0
#define OCTLB_FD_MOVING_LID 1
#define OCTLB_FD_VELOCITY 2
#define OCTLB_FD_OUTFLOW 3
#define OCTLB_FD_PRESSURE 4
int octlb_gpu_set_fd_boundary(octlb_ctx* ctx, const int types[6], const double u_wall[18],
                              const double rho_target[6], const double* inlet_u /* [18] or NULL */,
                              double ramp_end_t);
/* bc::StampTreeBoundaryCells (bc_installer.h:95-138): kinds_out = the
 * tables' kinds with the face slab of every tree-boundary face set to the
 * kind of that face's type (types as above, plus 0 no-slip, 1 moving lid, 3
 * outflow), solid cells kept; [n_blocks][n^3].  Host only. */
int octlb_fd_stamp_kinds(const octlb_tables* tables, const int types[6], uint8_t* kinds_out);
/* Host-only dry run of octlb_gpu_set_fd_boundary on the tables (every block
 * at forest level 0, kinds stamped): the per-cell records of the pass (one
 * per velocity / pressure Dirichlet cell, octlb_fd_record_bytes() bytes
 * each, the library's internal layout) -- for checking the stencil
 * resolution on the host.  Returns the number of records, or a negative
 * error code. */
int octlb_fd_plan(const octlb_tables* tables, const int types[6], const double u_wall[18],
                  const double rho_target[6], const double* inlet_u, double ramp_end_t, void* records,
                  int max_records);
int octlb_fd_record_bytes(void);

/* Inlet velocity fields of the velocity faces, the reference's
 * InletVelocityField kinds (inlet_velocity_field.h), each ramped by
 * 10x^3 - 15x^4 + 6x^5, x = t / ramp_end_t (none for ramp_end_t <= 0):
 *   UNIFORM             u = u (UniformInletProfile, :131-159);
 *   POISEUILLE          u = u_peak p(i0, n_inplane[0]) p(i1, n_inplane[1]) u,
 *                       p(i, n) = 4 c (1 - c), c = (i + 1/2) / n, i0 / i1 the
 *                       cell's block-local in-plane indices (y, z on x faces;
 *                       x, z on y faces; x, y on z faces) (PoiseuilleInletProfile,
 *                       :38-129);
 *   CHANNEL_POISEUILLE  the same from the cell's physical position, block
 *                       origin + (index + 1/2) cell width, on the patch
 *                       [patch[0], patch[1]] x [patch[2], patch[3]] of the in-plane
 *                       coordinates, c clamped to [0, 1]
 *                       (ChannelPoiseuilleInletProfile, :163-269).
 * u is the flow direction for the Poiseuille kinds. */
#define OCTLB_INLET_NONE 0
#define OCTLB_INLET_UNIFORM 1
#define OCTLB_INLET_POISEUILLE 2
#define OCTLB_INLET_CHANNEL_POISEUILLE 3
typedef struct octlb_fd_inlet {
  int kind;
  int n_inplane[2];
  double u[3];
  double u_peak;
  double patch[4];
  double ramp_end_t;
} octlb_fd_inlet;
/* octlb_gpu_set_fd_boundary with an inlet field per face (inlets[6], NULL:
 * none), in place of the uniform inlet_u; the cell's prescribed velocity is
 * the field of the first face it touches that has one. */
int octlb_gpu_set_fd_boundary_inlets(octlb_ctx* ctx, const int types[6], const double u_wall[18],
                                     const double rho_target[6], const octlb_fd_inlet* inlets);
/* octlb_fd_plan with inlet fields. */
int octlb_fd_plan_inlets(const octlb_tables* tables, const int types[6], const double u_wall[18],
                         const double rho_target[6], const octlb_fd_inlet* inlets, void* records, int max_records);

/* ---- VTK output (src/solver/io/vtk_writer/) ------------------------------
 * The files of the reference's writer, byte for byte for the same values: an
 * XML StructuredGrid .vts per block with binary (base64, UInt32 header)
 * Float64 cell data and vertex coordinates (WriteStructuredGridVts,
 * structured_grid_writer.cpp:49-100), a vtkMultiBlockDataSet .vtm per
 * timestep and a Collection .pvd series (WriteVtmIndex / AppendPvdTimestep,
 * parallel_vtk_index.cpp:117-172). */
#define OCTLB_VTK_VELOCITY 1 /* "velocity", 3 components (VtkVelocityField) */
#define OCTLB_VTK_DENSITY 2  /* "density" (VtkDensityField) */
#define OCTLB_VTK_PRESSURE 4 /* "pressure" = rho c_s^2 (VtkPressureField) */

/* AmrVtkWriter::WriteTimestep + WriteVtmAndPvd (amr_vtk_writer.h:25-33), each
 * block with its own fields: one file output_dir/base_r<rank>_oct<block>_T<step,
 * 5 digits>.vts per block, with the chosen fields (a mask of OCTLB_VTK_*, in
 * the order velocity, density, pressure) from the reference's post-stream
 * rho and u (as octlb_gpu_get_fields); with write_index, also
 * base_T<step>.vtm listing them and the step appended to base.pvd (a run of
 * several ranks writes the index once, with octlb_vtk_write_index).
 * Creates output_dir.  Synchronises the stream. */
int octlb_gpu_write_vtk(octlb_ctx* ctx, const char* output_dir, const char* base_name, int step, int rank,
                        int fields, int write_index);

/* WriteStructuredGridVts for one block of nx x ny x nz cells on
 * bounds = {x_min, y_min, z_min, x_max, y_max, z_max}: nfields cell fields,
 * field f named names[f] with comps[f] (1..3) components, values data[f] in
 * the file's cell order (i fastest, then j, then k).  Host only. */
int octlb_vtk_write_block(const char* path, int nx, int ny, int nz, const double bounds[6], int nfields,
                          const char* const* names, const int* comps, const double* const* data);

/* WriteVtmIndex + AppendPvdTimestep for one timestep: output_dir/base_T<step>.vtm
 * listing the .vts paths (relative to output_dir), and its entry appended to
 * output_dir/base.pvd (created on first use).  Host only. */
int octlb_vtk_write_index(const char* output_dir, const char* base_name, int step, int n_files,
                          const char* const* vts_relative_paths);

/* Discrete adjoint (reverse mode) of n coarse steps.  Objective J = the
 * `component` of octlb_gpu_force averaged over the last `window` coarse
 * steps.  Runs the forward from the context's current state with a
 * checkpoint every `checkpoint_interval` coarse steps (0: ceil(sqrt(n))),
 * then recomputes each segment from its checkpoint and runs the hand-written
 * adjoint kernels through it in reverse (a segment's recomputation on a
 * stream of its own beside the next-later segment's reverse).  Device memory
 * it allocates and keeps with the context: ceil(n / interval) + 1 states and
 * 2 x interval coarse steps of step inputs.  Outputs J, grad[0] = dJ/du_max
 * (u_max = the largest moving tree-boundary wall speed; all wall velocities
 * scale with it), grad[1] = dJ/dtau (tau = 1/omega, including the coupler
 * scales), and, when grad_force is not NULL, dJ/dF for the body force of
 * every core cell ([n_blocks][n^3][3]; at the current force, zero if none).
 * FP32 storage, drag enabled, slot-map levels (n a multiple of 8, <= 16).
 * The context ends in the forward's final state (as after advance(n)).
 * No reference counterpart: the reference has no adjoint. */
typedef struct octlb_adj_params {
  int coarse_steps;
  int window;
  int checkpoint_interval;
  int component;
} octlb_adj_params;
int octlb_gpu_adjoint(octlb_ctx* ctx, const octlb_adj_params* params, double* objective, double grad[2],
                      double* grad_force);

/* Reference state f (post-stream, pre-collision) -> context; the next step
 * starts by colliding it. */
int octlb_gpu_set_populations(octlb_ctx* ctx, const double* pops);
/* Equilibrium initialisation from per-cell fields: every core cell takes
 * f_i = feq_i(rho, u) (the shifted second-order equilibrium) and the next
 * step starts by colliding it -- BlockLattice::initialize(rho0, u0)
 * (block_lattice.cpp:273-285) and initialize_from_material
 * (lattice_material_init.cpp:11-33) with a rho and u per cell instead of one
 * pair.  rho [n_blocks][n^3], u [n_blocks][n^3][3]; equal to
 * octlb_gpu_set_populations of that equilibrium, at a fifth of its upload. */
int octlb_gpu_set_equilibrium(octlb_ctx* ctx, const double* rho, const double* u);
/* Post-collision populations the next stream reads (what the reference's
 * take_post_collide_snapshot holds after the next collide), core cells. */
int octlb_gpu_get_populations(octlb_ctx* ctx, double* pops);
/* rho [n_blocks][n^3] and u [n_blocks][n^3][3] of every core cell. */
int octlb_gpu_get_fields(octlb_ctx* ctx, double* rho, double* u);

/* MEM force on the fluid after the last coarse step, FP64. */
int octlb_gpu_force(octlb_ctx* ctx, double out[3]);
/* Sum of that force over every coarse step since create / reset, and count. */
int octlb_gpu_force_sum(octlb_ctx* ctx, double out[3], long long* steps);
int octlb_gpu_force_reset(octlb_ctx* ctx);
/* out[0] = sum rho, out[1..3] = sum rho u over kBulk core cells (FP64);
 * returns OCTLB_ENAN if any population is not finite. */
int octlb_gpu_audit(octlb_ctx* ctx, double out[4]);

/* Mass / momentum audit that allocates nothing on the device: same result as
 * octlb_gpu_audit, for callers that must not call cudaMalloc / cudaFree (an
 * application whose device memory is owned by another allocator, or a
 * per-step monitoring loop that cannot afford their implicit device
 * synchronisation).  It has no counterpart in the reference (whose audit is
 * a host loop).  Its partial sums live in one fixed file-scope device array of
 * 16,385 x 5 doubles (~640 KB), held by every GPU that loads the library until
 * the process exits; levels of more than 33,554,432 cells are rejected with
 * OCTLB_EINVAL.  The first call made on a device looks up that array's device
 * address (cudaGetSymbolAddress), so make that first call before any stream
 * capture; call with the context's device current.  The address is kept for
 * the life of the process: after a cudaDeviceReset of that device the entry
 * point must not be used again.  Like octlb_gpu_audit it first reports a
 * bounded device wait that gave up (OCTLB_ETIMEOUT).  All calls share the
 * array: calls that overlap on the GPU race. */
int octlb_gpu_audit_noalloc(octlb_ctx* ctx, double out[4]);

/* ---- Ranks: the leaves shared over several contexts -----------------------
 * The reference runs one MPI rank per core: p4est partitions the leaves by
 * weight (OctreeForest::partition with make_level_weight_fn, weight 2^level,
 * octree_forest.cpp:273-280, weighted_load_balancer.cpp:7-12), GhostSchedule
 * exchanges face and edge layers between ranks before every level step
 * (ghost_schedule.h:121-255), LevelCoupler sends its interface payloads
 * across ranks (level_coupler.cpp:325-436, 492-585) and the cases sum the
 * force and mass with MPI_Allreduce (cylinder3d_case.h:502, 620).  Here one
 * context per GPU (a "rank context") steps the leaves its rank owns; it keeps
 * the same-level neighbours of its leaves that other ranks own as mirror
 * blocks, refreshed before every step of their level, and receives the save
 * rows (pre-collision populations of coupler source cells) its coupler items
 * read after every step of their level.  Forces and audits come back summed
 * over the ranks.  Every rank passes the same global tables and initial
 * state; get_fields / get_populations / set_* / write_vtk touch the rank's
 * own blocks only.  ConstRhoBGK and the adjoint are single-context only. */

/* The reference's partition: leaves in the forest's order, weight 2^level;
 * rank k owns the leaves whose weight prefix lies in [k W / P, (k+1) W / P). */
int octlb_gpu_partition(const octlb_tables* tables, int nranks, int* owner);

/* Transport between the rank contexts.  Every rank context makes the same
 * exchanges in the same order (its octlb_gpu_advance calls), so every rank
 * must advance by the same number of steps. */
typedef struct octlb_comm octlb_comm;
/* The rank contexts of one process, each driven by its own host thread (on
 * one device or several): device copies ordered by events, two host barriers
 * per exchange; a rank that does not arrive within OCTLB_COMM_TIMEOUT_S
 * seconds (default 60) ends the others' calls with OCTLB_ETIMEOUT. */
int octlb_comm_create_local(int nranks, octlb_comm** out);
/* One process per GPU over NCCL (opened at run time): rank 0 makes the id,
 * every rank passes it (through the caller's launcher) to create_nccl with
 * its device current.  Synchronising calls give up after
 * OCTLB_COMM_TIMEOUT_S seconds (default 300) and abort the communicator. */
int octlb_comm_nccl_unique_id(unsigned char id[128]);
int octlb_comm_create_nccl(const unsigned char id[128], int nranks, int rank, octlb_comm** out);
/* After every context using it is destroyed. */
void octlb_comm_destroy(octlb_comm* comm);
/* Why the NCCL transport could not be opened (empty if it could). */
const char* octlb_comm_last_error(void);

typedef struct octlb_partition {
  int rank;                       /* this context's rank */
  int nranks;
  const int* owner;               /* [n_blocks] owning rank of every leaf */
  octlb_comm* comm;
} octlb_partition;

/* octlb_gpu_create for one rank of a partition. */
int octlb_gpu_create_part(const octlb_tables* tables, const octlb_params* params, const double* init_pops,
                          const octlb_partition* part, octlb_ctx** out);

/* Host-only dry run of octlb_gpu_create: validates and flattens the tables
 * (every index the kernels derive is bounds-checked) without touching a
 * device, and reports the plan: stats[0] = levels, then per level 10 values
 * (blocks, halo pages, open blocks, boundary-fill writes, prolongation items,
 * restriction items, saved cells, link records, drag cells, slots).  Returns
 * the number of values, or a negative error code. */
int octlb_gpu_plan(const octlb_tables* tables, const octlb_params* params, long long* stats, int max_stats);

/* Host-only dry run of octlb_gpu_create_part for `rank` (no comm, no
 * device): validates and flattens the tables as that rank would and writes
 * its exchange lists as records of 4 values -- level, kind (0 cells sent, 1
 * cells received before each step of the level; 2 save rows sent, 3 save
 * rows received after it), peer rank, global cell (block * n^3 + cell) -- in
 * the order they travel.  Returns the number of records (at most
 * max_records are written), or a negative error code. */
int octlb_gpu_plan_part(const octlb_tables* tables, const octlb_params* params, int rank, int nranks,
                        const int* owner, long long* records, long long max_records);

/* Per-level collide / stream counts and max level (TimeLoop::counters). */
int octlb_gpu_counters(const octlb_ctx* ctx, int* collide, int* stream, int max_levels);
int octlb_gpu_max_level(const octlb_ctx* ctx);
/* Kernel launches one coarse step issues (as counted when the last
 * advance_one was issued; before the first, without shared coupler launches),
 * and lattice updates it performs. */
int octlb_gpu_step_stats(const octlb_ctx* ctx, long long* launches, long long* lattice_updates);

#ifdef __cplusplus
}
#endif
#endif
