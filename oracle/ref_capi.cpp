// C entry points over the reference's OWN hot-path classes, compiled from the
// reference sources (BlockLattice, BouzidiLinkData, LevelCoupler, GhostSchedule,
// TimeLoop, MomentumExchangeDrag) into oracle/_ref/liboctlb_ref.so.  Used by the
// tests and by bench.py's reference arm as the checker / CPU baseline; never by
// the product.
//
// Two things here are restatements rather than reference code, because the
// reference has no runtime for them (kMovingBounceBack has no collide or stream
// arm, src/solver/lbm/bc_dispatcher.h:75-79, bc_kind.h:30-33; the zero-gradient
// helper src/solver/lbm/boundary/outflow_bc.h:15-21 is never called):
//   * the moving-wall momentum term of Ladd (1994): a population pulled from a
//     wall moving with u_w gains 2 w_i rho_w (c_i . u_w) / c_s^2, rho_w = 1;
//   * tree-boundary ghost fills (RestatedBoundary below): half-way bounce-back
//     walls (optionally moving) and the zero-gradient outflow ghost copy of
//     outflow_bc.h, written into the halo before the same-level exchange, at the
//     DomainBoundaryHandler::apply() hook (time_loop.h:207-211);
//   * an optional body force, the forcing term 3 w_i (c_i . F) added to the
//     post-collision populations of kBulk cells of the level just collided, at
//     the same hook before the fills (the reference has no body force; the
//     adjoint's finite-difference checks need one).
//
// The same file also builds the tangent-linear library (ref_tlm.cpp, with the
// reference's floating type replaced by a forward-mode dual number): the C
// ABI therefore uses f64 (always a plain double) and copies its buffers
// element by element, and omega and the wall velocities pass through the
// seed hooks, identities in this build.
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "src/solver/lbm/block_lattice.h"
#include "src/solver/lbm/bouzidi_link_data.h"
#include "src/solver/lbm/boundary/bouzidi_pull.h"
#include "src/solver/lbm/drag_postprocessor.h"
#include "src/solver/lbm/level_coupler.h"
#include "src/solver/lbm/domain_boundary_handler.h"
#include "src/solver/lbm/time_loop/time_loop.h"
#include "src/solver/field/ghost_schedule.h"
#include "src/mesh/topology/face_pair_list.h"
#ifndef OCTLB_REF_TLM
#include "src/solver/lbm/bc_installer.h"
#endif

namespace octlb {
void OracleForestInject(OctreeForest& forest, const std::vector<int>& levels,
                        const std::vector<BoundingBox>& bounds,
                        const std::vector<SameLevelFace>& sl,
                        const std::vector<CoarseFineFace>& cf,
                        const std::vector<TreeBoundaryFace>& tb);
}

using namespace octlb;
using D = olb::descriptors::D3Q19<>;
using Lat = BlockLattice<double, D>;
static constexpr int Q = 19;

#ifndef OCTLB_REF_TLM
using f64 = double;
inline f64 to_f64(double x) { return x; }
inline double seed_omega(double omega) { return omega; }
inline double seed_wall(double u) { return u; }
#endif

namespace {

inline int cc(int i, int d) { return olb::descriptors::c<D>(i, d); }
inline int opp(int i) { return olb::descriptors::opposite<D>(i); }
inline double wt(int i) { return olb::descriptors::t<double, D>(i); }

struct Block {
  std::unique_ptr<Lat> lat;
  std::unique_ptr<BouzidiLinkData> links;
  int nx, ny, nz;
};

// Ladd moving-wall term for every link pulled from a moving solid cell
// (restated; see header).  Applies to cells the reference streams on its
// per-cell path (block_lattice.cpp:536-548,639-670): non-solid core cells
// whose source x-c_i is a solid / Bouzidi core cell.
void AddMovingWallTerm(Lat& lat, int nx, int ny, int nz, const uint8_t* moving,
                       const f64* uw) {
  auto cidx = [&](int x, int y, int z) { return (x * ny + y) * nz + z; };
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        if (lat.bc_kind(x, y, z) == BcKind::kSolid) continue;
        double* f = lat.populations_at_halo(x + 1, y + 1, z + 1);
        for (int i = 1; i < Q; ++i) {
          const int sx = x - cc(i, 0), sy = y - cc(i, 1), sz = z - cc(i, 2);
          if (sx < 0 || sy < 0 || sz < 0 || sx >= nx || sy >= ny || sz >= nz) continue;
          const int s = cidx(sx, sy, sz);
          const BcKind sk = lat.bc_kind(sx, sy, sz);
          if (sk != BcKind::kSolid && sk != BcKind::kBouzidi) continue;
          if (!moving[s]) continue;
          const double cu = cc(i, 0) * uw[3 * s] + cc(i, 1) * uw[3 * s + 1] +
                            cc(i, 2) * uw[3 * s + 2];
          f[i] += 6.0 * wt(i) * cu;
        }
      }
}

// Restated tree-boundary conditions, applied as halo fills (see header).
struct FaceSpec {
  int type;        // 0 none, 1 wall (bounce-back, optionally moving), 2 outflow
  double u[3];     // wall velocity scale
  int prof_axis;   // -1: uniform u; else u *= 4 s (1-s), s along this axis
  double lo, hi;   // physical extent of the profile coordinate
};

double ProfileShape(const FaceSpec& s, const double p[3]) {
  if (s.prof_axis < 0) return 1.0;
  const double t = (p[s.prof_axis] - s.lo) / (s.hi - s.lo);
  return (t <= 0.0 || t >= 1.0) ? 0.0 : 4.0 * t * (1.0 - t);
}

class RestatedBoundary : public DomainBoundaryHandler {
 public:
  RestatedBoundary(BlockCollection<Lat>& blocks, const OctreeForest& forest,
                   std::vector<TreeBoundaryFace> faces, std::vector<FaceSpec> specs,
                   int n)
      : blocks_(blocks), forest_(forest), faces_(std::move(faces)),
        specs_(std::move(specs)), n_(n) {}

  void apply(CollideRhoStats*, double, bool) override {
    if (!force_.empty() && loop_) AddForce();
    for (std::size_t k = 0; k < faces_.size(); ++k) Fill(faces_[k], specs_[k]);
  }

  // Body force [oct][n^3][3]; the level collided just before apply() is the
  // one whose collide counter moved since the previous call.
  void set_force(const TimeLoop* loop, const double* f) {
    loop_ = loop;
    const std::size_t n3 = static_cast<std::size_t>(n_) * n_ * n_;
    if (f) force_.assign(f, f + static_cast<std::size_t>(blocks_.size()) * n3 * 3); else force_.clear();
    seen_.assign(loop->counters().collide.begin(), loop->counters().collide.end());
  }

 private:
  void AddForce() {
    const auto& c = loop_->counters().collide;
    int level = -1;
    if (seen_.size() < c.size()) seen_.resize(c.size(), 0);
    for (std::size_t l = 0; l < c.size(); ++l)
      if (c[l] != seen_[l]) { level = static_cast<int>(l); seen_[l] = c[l]; }
    if (level < 0) return;
    const std::size_t n3 = static_cast<std::size_t>(n_) * n_ * n_;
    for (label id = 0; id < blocks_.size(); ++id) {
      if (forest_.quadrant_level(id) != level) continue;
      Lat& lat = blocks_[id];
      for (int x = 0; x < n_; ++x)
        for (int y = 0; y < n_; ++y)
          for (int z = 0; z < n_; ++z) {
            if (lat.bc_kind(x, y, z) != BcKind::kBulk) continue;
            const double* F = force_.data() + ((std::size_t)id * n3 + (x * n_ + y) * n_ + z) * 3;
            double* f = lat.populations_at_halo(x + 1, y + 1, z + 1);
            for (int i = 0; i < Q; ++i)
              f[i] += 3.0 * wt(i) * (cc(i, 0) * F[0] + cc(i, 1) * F[1] + cc(i, 2) * F[2]);
          }
    }
  }

  void Fill(const TreeBoundaryFace& f, const FaceSpec& s) {
    if (s.type == 0) return;
    Lat& lat = blocks_[f.octant_id];
    const BoundingBox b = forest_.quadrant_bounds(f.octant_id);
    const double dx = (b.x_max - b.x_min) / n_;
    const double org[3] = {b.x_min, b.y_min, b.z_min};
    const int dir = static_cast<int>(f.face_dir);
    const int ax = dir / 2, t0 = (ax + 1) % 3, t1 = (ax + 2) % 3;
    const bool is_max = (dir & 1) != 0;
    const int hl = is_max ? n_ + 1 : 0;
    const int nin = is_max ? -1 : 1;
    for (int a = 0; a < n_ + 2; ++a)
      for (int bb = 0; bb < n_ + 2; ++bb) {
        int h[3];
        h[ax] = hl; h[t0] = a; h[t1] = bb;
        double* dst = lat.populations_at_halo(h[0], h[1], h[2]);
        if (s.type == 1) {
          double p[3];
          for (int d = 0; d < 3; ++d) p[d] = org[d] + (h[d] - 1 + 0.5) * dx;
          const double shape = ProfileShape(s, p);
          for (int i = 1; i < Q; ++i) {
            if (cc(i, ax) != nin) continue;
            const int x = h[0] + cc(i, 0), y = h[1] + cc(i, 1), z = h[2] + cc(i, 2);
            if (x < 1 || y < 1 || z < 1 || x > n_ || y > n_ || z > n_) continue;
            const double* src = lat.populations_at_halo(x, y, z);
            const double cu = (cc(i, 0) * s.u[0] + cc(i, 1) * s.u[1] +
                               cc(i, 2) * s.u[2]) * shape;
            dst[i] = src[opp(i)] + 6.0 * wt(i) * cu;
          }
        } else if (s.type == 2) {
          int src[3];
          src[ax] = hl + nin;
          src[t0] = std::min(std::max(a, 1), n_);
          src[t1] = std::min(std::max(bb, 1), n_);
          const double* sp = lat.populations_at_halo(src[0], src[1], src[2]);
          std::memcpy(dst, sp, sizeof(double) * Q);
        }
      }
  }

  BlockCollection<Lat>& blocks_;
  const OctreeForest& forest_;
  std::vector<TreeBoundaryFace> faces_;
  std::vector<FaceSpec> specs_;
  int n_;
  const TimeLoop* loop_ = nullptr;
  std::vector<double> force_;
  std::vector<int> seen_;
};

struct Sim {
  int n = 0;
  std::unique_ptr<OctreeForest> forest;
  std::unique_ptr<FacePairList> faces;
  std::unique_ptr<BlockCollection<Lat>> blocks;
  std::vector<std::unique_ptr<BouzidiLinkData>> links;  // 0 or 1 shared table
  std::unique_ptr<GhostSchedule<Lat>> ghosts;
  std::unique_ptr<LevelCoupler> coupler;
  std::unique_ptr<DomainBoundaryHandler> bc;
  std::unique_ptr<TimeLoop> loop;
  double omega = 0.0;
  std::vector<TreeBoundaryFace> tree_faces;
  // Physical coupler mode (ref_sim_set_physical): per-level rates and one
  // LevelCoupler per level pair, built with the coarse level's rate.
  bool physical = false;
  std::vector<double> omega_level;
  std::vector<std::unique_ptr<LevelCoupler>> pair_couplers;
  std::vector<std::vector<label>> by_level;
  int max_level = 0;
  long long step = 0;
};

// TimeLoop::advance (time_loop.h:201-240) restated for the physical mode:
// the same phase order, each level collided with its own rate omega_level[l],
// and the pair (l, l + 1) coupled by the LevelCoupler built with omega_level[l]
// -- whose scales (tau_c - 1/4) / tau_c and tau_c / (tau_c - 1/4)
// (level_coupler.cpp:226-228) are the Dupuis-Chopard factors tau_f / (2 tau_c)
// and 2 tau_c / tau_f for tau_f = 2 tau_c - 1/2.  Not the reference's loop: the
// reference collides every level with one rate.
void PhysicalAdvance(Sim* s, int level) {
  const auto& ids = s->by_level[static_cast<std::size_t>(level)];
  for (label id : ids) (*s->blocks)[id].collide(s->omega_level[static_cast<std::size_t>(level)]);
  s->bc->apply(nullptr, 1.0, false);
  s->ghosts->exchange();
  for (label id : ids) (*s->blocks)[id].take_post_collide_snapshot();
  for (label id : ids) (*s->blocks)[id].stream();
  s->bc->apply_post_stream();
  if (level >= s->max_level) return;
  LevelCoupler& c = *s->pair_couplers[static_cast<std::size_t>(level)];
  c.apply_half_time(level);
  PhysicalAdvance(s, level + 1);
  c.apply_full_time(level);
  PhysicalAdvance(s, level + 1);
  c.restrict(level + 1);
}

// Sum of MomentumExchangeDrag::force_on_fluid_if over all blocks (see
// ref_sim_drag).
std::array<double, 3> SimDrag(Sim* s, const uint8_t* mask) {
  const int n = s->n, n3 = n * n * n;
  std::array<double, 3> out{0.0, 0.0, 0.0};
  for (label id = 0; id < s->blocks->size(); ++id) {
    MomentumExchangeDrag drag((*s->blocks)[id]);
    const uint8_t* m = mask ? mask + (std::size_t)id * n3 : nullptr;
    auto f = drag.force_on_fluid_if([&](int x, int y, int z) {
      return m == nullptr || m[(x * n + y) * n + z] != 0;
    });
    out[0] += f[0]; out[1] += f[1]; out[2] += f[2];
  }
  return out;
}
}  // namespace

extern "C" {

// ---------------------------------------------------------------- one block
void* ref_block_new(int nx, int ny, int nz) {
  auto* b = new Block;
  b->lat = std::make_unique<Lat>(nx, ny, nz, 1);
  b->nx = nx; b->ny = ny; b->nz = nz;
  return b;
}
void ref_block_free(void* h) { delete static_cast<Block*>(h); }

void ref_block_initialize(void* h, f64 rho, f64 ux, f64 uy, f64 uz) {
  const double u[3] = {ux, uy, uz};
  static_cast<Block*>(h)->lat->initialize(rho, u);
}
void ref_block_set_kinds(void* h, const uint8_t* kinds) {
  auto* b = static_cast<Block*>(h);
  for (int x = 0; x < b->nx; ++x)
    for (int y = 0; y < b->ny; ++y)
      for (int z = 0; z < b->nz; ++z)
        b->lat->set_bc_kind(x, y, z, static_cast<BcKind>(kinds[(x * b->ny + y) * b->nz + z]));
}
// Padded storage [(nx+2)][(ny+2)][(nz+2)][19], the reference's own layout
// (block_lattice.h:294-304).
void ref_block_get_padded(void* h, f64* out) {
  auto* b = static_cast<Block*>(h);
  const std::size_t n = (std::size_t)(b->nx + 2) * (b->ny + 2) * (b->nz + 2) * Q;
  const double* p = b->lat->populations_at_halo(0, 0, 0);
  for (std::size_t k = 0; k < n; ++k) out[k] = to_f64(p[k]);
}
void ref_block_set_padded(void* h, const f64* in) {
  auto* b = static_cast<Block*>(h);
  const std::size_t n = (std::size_t)(b->nx + 2) * (b->ny + 2) * (b->nz + 2) * Q;
  double* p = b->lat->populations_at_halo(0, 0, 0);
  for (std::size_t k = 0; k < n; ++k) p[k] = in[k];
}
void ref_block_collide(void* h, f64 omega) { static_cast<Block*>(h)->lat->collide(omega); }
void ref_block_fill_periodic(void* h) { static_cast<Block*>(h)->lat->fill_periodic_halo(); }
void ref_block_stream(void* h) { static_cast<Block*>(h)->lat->stream(); }
void ref_block_snapshot(void* h) { static_cast<Block*>(h)->lat->take_post_collide_snapshot(); }

// Attach a BouzidiLinkData table (q defaults to 1.0 = half-way bounce-back,
// bouzidi_link_data.cpp:107-116) with the given cut links overriding it.
void ref_block_set_links(void* h, int n_links, const int* cell_pop, const f64* q) {
  auto* b = static_cast<Block*>(h);
  b->links = std::make_unique<BouzidiLinkData>(1, b->nx, b->ny, b->nz, Q);
  for (int k = 0; k < n_links; ++k)
    b->links->set_q_frac(0, cell_pop[4 * k], cell_pop[4 * k + 1], cell_pop[4 * k + 2],
                         cell_pop[4 * k + 3], q[k]);
  b->lat->set_bouzidi_links(b->links.get());
}
void ref_block_add_moving_wall(void* h, const uint8_t* moving, const f64* uw) {
  auto* b = static_cast<Block*>(h);
  AddMovingWallTerm(*b->lat, b->nx, b->ny, b->nz, moving, uw);
}

// Periodic box: collide -> fill_periodic_halo -> stream, the loop of
// tests/unit/solver/test_collision_bgk.cpp:56-60.
void ref_block_run_periodic(void* h, f64 omega, int steps) {
  auto* b = static_cast<Block*>(h);
  for (int t = 0; t < steps; ++t) {
    b->lat->collide(omega);
    b->lat->fill_periodic_halo();
    b->lat->stream();
  }
}
// Walled box (solid shell + q table): collide -> stream -> moving-wall term.
void ref_block_run_walls(void* h, f64 omega, int steps, const uint8_t* moving,
                         const f64* uw) {
  auto* b = static_cast<Block*>(h);
  for (int t = 0; t < steps; ++t) {
    b->lat->collide(omega);
    b->lat->stream();
    if (moving) AddMovingWallTerm(*b->lat, b->nx, b->ny, b->nz, moving, uw);
  }
}
// MomentumExchangeDrag::force_on_fluid_if over this block
// (drag_postprocessor.h:67-115); obstacle mask over core cells or null.
void ref_block_drag(void* h, const uint8_t* mask, f64* out) {
  auto* b = static_cast<Block*>(h);
  MomentumExchangeDrag drag(*b->lat);
  const int ny = b->ny, nz = b->nz;
  auto f = drag.force_on_fluid_if([&](int x, int y, int z) {
    return mask == nullptr || mask[(x * ny + y) * nz + z] != 0;
  });
  out[0] = to_f64(f[0]); out[1] = to_f64(f[1]); out[2] = to_f64(f[2]);
}

// ------------------------------------------------------------- octree + loop
// Forest description: leaves (level, bounds), and the FacePairList lists.
void* ref_sim_new(int n_oct, const int* levels, const f64* bounds, int n_sl,
                  const int* sl /* local, dir, remote */, int n_cf,
                  const int* cf /* coarse, f0..f3, normal, clevel, flevel */,
                  const f64* cf_bounds /* coarse 6 + 4 x fine 6 */, int n_tb,
                  const int* tb /* oct, dir */, const f64* tb_spec /* 7 per face */,
                  int n, f64 omega_in, const uint8_t* kinds /* [oct][n^3] */,
                  const f64* core_pops /* [oct][n^3][19] or null */,
                  int n_links, const int* link_cells /* oct,x,y,z,pop */,
                  const f64* link_q, int link_mode) {
  const double omega = seed_omega(omega_in);
  auto* s = new Sim;
  s->n = n;
  s->forest = std::make_unique<OctreeForest>(MPI_COMM_WORLD, BoundingBox{});
  std::vector<int> lv(levels, levels + n_oct);
  std::vector<BoundingBox> bx(n_oct);
  for (int i = 0; i < n_oct; ++i)
    bx[i] = {bounds[6 * i], bounds[6 * i + 1], bounds[6 * i + 2],
             bounds[6 * i + 3], bounds[6 * i + 4], bounds[6 * i + 5]};
  std::vector<SameLevelFace> slv(n_sl);
  for (int i = 0; i < n_sl; ++i)
    slv[i] = {sl[3 * i], static_cast<FaceDir>(sl[3 * i + 1]), sl[3 * i + 2], 0, 0};
  std::vector<CoarseFineFace> cfv(n_cf);
  for (int i = 0; i < n_cf; ++i) {
    CoarseFineFace e{};
    const int* r = cf + 8 * i;
    const f64* bd = cf_bounds + 30 * i;
    e.coarse_id = r[0];
    for (int k = 0; k < 4; ++k) { e.fine_ids[k] = r[1 + k]; e.remote_ranks[k] = 0; e.comm_tags[k] = 0; }
    e.normal = static_cast<FaceDir>(r[5]);
    e.coarse_level = r[6];
    e.fine_level = r[7];
    e.coarse_remote_rank = 0;
    e.coarse_bounds = {bd[0], bd[1], bd[2], bd[3], bd[4], bd[5]};
    for (int k = 0; k < 4; ++k) {
      const f64* fb = bd + 6 + 6 * k;
      e.fine_bounds[k] = {fb[0], fb[1], fb[2], fb[3], fb[4], fb[5]};
    }
    cfv[i] = e;
  }
  std::vector<TreeBoundaryFace> tbv(n_tb);
  std::vector<FaceSpec> specs(n_tb);
  for (int i = 0; i < n_tb; ++i) {
    tbv[i] = {tb[2 * i], static_cast<FaceDir>(tb[2 * i + 1])};
    const f64* p = tb_spec + 8 * i;
    specs[i] = {static_cast<int>(p[0]), {seed_wall(p[1]), seed_wall(p[2]), seed_wall(p[3])},
                static_cast<int>(p[4]), p[5], p[6]};
  }
  OracleForestInject(*s->forest, lv, bx, slv, cfv, tbv);
  s->faces = std::make_unique<FacePairList>(*s->forest);

  const int n3 = n * n * n;
  if (link_mode) {
    s->links.push_back(std::make_unique<BouzidiLinkData>(n_oct, n, n, n, Q));
    for (int k = 0; k < n_links; ++k) {
      const int* c = link_cells + 5 * k;
      s->links[0]->set_q_frac(c[0], c[1], c[2], c[3], c[4], link_q[k]);
    }
  }
  BouzidiLinkData* lp = link_mode ? s->links[0].get() : nullptr;
  s->blocks = std::make_unique<BlockCollection<Lat>>(n_oct, [&](OctantId id) {
    Lat lat(n, n, n, 1);
    for (int x = 0; x < n; ++x)
      for (int y = 0; y < n; ++y)
        for (int z = 0; z < n; ++z) {
          const int c = (x * n + y) * n + z;
          lat.set_bc_kind(x, y, z, static_cast<BcKind>(kinds[(std::size_t)id * n3 + c]));
          if (core_pops) {
            double* f = lat.populations_at_halo(x + 1, y + 1, z + 1);
            const f64* src = core_pops + ((std::size_t)id * n3 + c) * Q;
            for (int i = 0; i < Q; ++i) f[i] = src[i];
          }
        }
    if (!core_pops) {
      const double u0[3] = {0, 0, 0};
      lat.initialize(1.0, u0);
    }
    lat.set_octant_id(id);
    lat.set_bouzidi_links(lp);
#ifndef OCTLB_REF_TLM
    // the block's physical origin and cell width, as cylinder3d sets them
    // (cylinder3d_case.h:405-415): physical inlet fields read them
    lat.set_phys_origin({bx[id].x_min, bx[id].y_min, bx[id].z_min}, (bx[id].x_max - bx[id].x_min) / n);
#endif
    return lat;
  });
  s->ghosts = std::make_unique<GhostSchedule<Lat>>(MPI_COMM_WORLD, *s->faces, *s->blocks, n, n, n);
  s->coupler = std::make_unique<LevelCoupler>(MPI_COMM_WORLD, *s->faces, *s->forest,
                                              *s->blocks, n, n, n, omega);
  s->bc = std::make_unique<RestatedBoundary>(*s->blocks, *s->forest, tbv, specs, n);
  s->loop = std::make_unique<TimeLoop>(*s->forest, *s->blocks, *s->ghosts, *s->coupler,
                                       *s->bc, omega);
  s->loop->set_snapshot_post_collide(true);
  s->omega = omega;
  s->tree_faces = tbv;
  return s;
}
// The TimeLoop rebuilt with use_const_rho_bgk (ConstRhoStatsScope::
// kFluidAndBoundary, the constructor's default); before the first advance
// and before ref_sim_set_body_force.
void ref_sim_set_const_rho(void* h, int on) {
  auto* s = static_cast<Sim*>(h);
  s->loop = std::make_unique<TimeLoop>(*s->forest, *s->blocks, *s->ghosts, *s->coupler,
                                       *s->bc, s->omega, on != 0);
  s->loop->set_snapshot_post_collide(true);
}
f64 ref_sim_average_rho(void* h) { return to_f64(static_cast<Sim*>(h)->loop->average_rho()); }

#ifndef OCTLB_REF_TLM
// The reference's own domain boundary conditions in place of the restated
// fills: a ConcreteDomainBoundaryHandler (domain_boundary_handler.cpp) over
// every tree-boundary face, face f in FaceDir order (x-, x+, y-, y+, z-, z+)
// with spec type types[f] (DomainBcType), wall velocity u_wall[3f .. 3f + 2]
// and target density rho_target[f]; the face cells stamped with the spec's
// BcKind (bc::StampTreeBoundaryCells, bc_installer.h:96-140) and the TimeLoop
// rebuilt around the handler, optionally with ConstRhoBGK -- the cavity3d
// construction (cavity3d_case.h:152-197).  padding_mode: OverlapPaddingMode.
// inlet_u (null: none): faces with a nonzero row take a UniformInletProfile
// of that velocity ramped over ramp_end_t steps (inlet_velocity_field.h:
// 128-162).  Before the first advance.
static void install_fd(Sim* s, const std::vector<DomainBcSpec>& specs, int padding_mode, int const_rho);

void ref_sim_set_fd_boundary(void* h, const int* types, const f64* u_wall, const f64* rho_target,
                             int padding_mode, int const_rho, const f64* inlet_u, f64 ramp_end_t) {
  auto* s = static_cast<Sim*>(h);
  std::vector<DomainBcSpec> specs(6);
  for (int f = 0; f < 6; ++f) {
    specs[f].face = static_cast<FaceDir>(f);
    specs[f].type = static_cast<DomainBcType>(types[f]);
    specs[f].u_wall = {u_wall[3 * f], u_wall[3 * f + 1], u_wall[3 * f + 2]};
    specs[f].rho_target = rho_target[f];
    if (inlet_u && (inlet_u[3 * f] != 0.0 || inlet_u[3 * f + 1] != 0.0 || inlet_u[3 * f + 2] != 0.0))
      specs[f].inlet_field = std::make_shared<boundary::UniformInletProfile>(
          std::array<double, 3>{inlet_u[3 * f], inlet_u[3 * f + 1], inlet_u[3 * f + 2]}, ramp_end_t);
  }
  install_fd(s, specs, padding_mode, const_rho);
}

// The same with one of the reference's inlet fields per face: kind[f] 0
// none, 1 UniformInletProfile(u), 2 PoiseuilleInletProfile(face, n0, n1,
// u_peak, u), 3 ChannelPoiseuilleInletProfile(face, patch, u_peak, u);
// par[11 f ..] = u[3], u_peak, n0, n1, patch[4], ramp_end_t.
void ref_sim_set_fd_boundary_inlets(void* h, const int* types, const f64* u_wall, const f64* rho_target,
                                    int padding_mode, int const_rho, const int* kind, const f64* par) {
  auto* s = static_cast<Sim*>(h);
  std::vector<DomainBcSpec> specs(6);
  for (int f = 0; f < 6; ++f) {
    specs[f].face = static_cast<FaceDir>(f);
    specs[f].type = static_cast<DomainBcType>(types[f]);
    specs[f].u_wall = {u_wall[3 * f], u_wall[3 * f + 1], u_wall[3 * f + 2]};
    specs[f].rho_target = rho_target[f];
    const f64* p = par + 11 * f;
    const std::array<double, 3> u{p[0], p[1], p[2]};
    const FaceDir dir = static_cast<FaceDir>(f);
    if (kind[f] == 1)
      specs[f].inlet_field = std::make_shared<boundary::UniformInletProfile>(u, p[10]);
    else if (kind[f] == 2)
      specs[f].inlet_field = std::make_shared<boundary::PoiseuilleInletProfile>(
          dir, static_cast<int>(p[4]), static_cast<int>(p[5]), p[3], u, p[10]);
    else if (kind[f] == 3)
      specs[f].inlet_field =
          std::make_shared<boundary::ChannelPoiseuilleInletProfile>(dir, p[6], p[7], p[8], p[9], p[3], u, p[10]);
  }
  install_fd(s, specs, padding_mode, const_rho);
}

static void install_fd(Sim* s, const std::vector<DomainBcSpec>& specs, int padding_mode, int const_rho) {
  bc::StampTreeBoundaryCells(*s->blocks, s->tree_faces, specs, s->n, s->n, s->n);
  s->loop.reset();
  s->bc = std::make_unique<ConcreteDomainBoundaryHandler>(*s->blocks, s->tree_faces, specs, s->n, s->n, s->n,
                                                          s->omega, static_cast<OverlapPaddingMode>(padding_mode));
  s->loop = std::make_unique<TimeLoop>(*s->forest, *s->blocks, *s->ghosts, *s->coupler, *s->bc, s->omega,
                                       const_rho != 0);
  s->loop->set_snapshot_post_collide(true);
}

void ref_sim_get_core(void* h, f64* out);
void ref_sim_get_padded(void* h, f64* out);

// One advance_one of a single-level mesh with the padded block populations
// (halo 1, [oct][(n+2)^3][19]) at the start and after each phase of
// TimeLoop::advance_one_with_hooks: out[0] start, [1] collide (boundary cells
// first, the OpenLB order), [2] ghost exchange, [3] stream, [4] post-stream
// boundary pass.
void ref_sim_advance_phases_padded(void* h, f64* out) {
  auto* s = static_cast<Sim*>(h);
  const std::size_t m = (std::size_t)s->blocks->size() * (s->n + 2) * (s->n + 2) * (s->n + 2) * Q;
  ref_sim_get_padded(h, out);
  s->loop->advance_one_with_hooks([&](TimeLoop::FlatPhase ph) {
    if (ph == TimeLoop::FlatPhase::kAfterCollide) ref_sim_get_padded(h, out + m);
    if (ph == TimeLoop::FlatPhase::kAfterGhostExchange) ref_sim_get_padded(h, out + 2 * m);
    if (ph == TimeLoop::FlatPhase::kAfterStream) ref_sim_get_padded(h, out + 3 * m);
    if (ph == TimeLoop::FlatPhase::kAfterPostStream) ref_sim_get_padded(h, out + 4 * m);
  });
}

// BcKind of every core cell, [oct][n^3] (after set_fd_boundary's stamping).
void ref_sim_get_kinds(void* h, uint8_t* out) {
  auto* s = static_cast<Sim*>(h);
  const int n = s->n, n3 = n * n * n;
  for (label id = 0; id < s->blocks->size(); ++id)
    for (int x = 0; x < n; ++x)
      for (int y = 0; y < n; ++y)
        for (int z = 0; z < n; ++z)
          out[(std::size_t)id * n3 + (x * n + y) * n + z] = static_cast<uint8_t>((*s->blocks)[id].bc_kind(x, y, z));
}

// One advance_one of a single-level mesh through TimeLoop::advance_one_with_hooks
// (time_loop.h:278-310), with the core populations after the stream
// (after_stream) and after the post-stream boundary pass (after_post_stream),
// [oct][n^3][19] each: the two sides of the FD reconstruction.
void ref_sim_advance_phases(void* h, f64* after_stream, f64* after_post_stream) {
  auto* s = static_cast<Sim*>(h);
  s->loop->advance_one_with_hooks([&](TimeLoop::FlatPhase ph) {
    if (ph == TimeLoop::FlatPhase::kAfterStream) ref_sim_get_core(h, after_stream);
    if (ph == TimeLoop::FlatPhase::kAfterPostStream) ref_sim_get_core(h, after_post_stream);
  });
}
#endif
void ref_sim_free(void* h) {
  auto* s = static_cast<Sim*>(h);
  // TimeLoop / coupler / ghosts hold references: tear down in reverse order.
  s->loop.reset(); s->pair_couplers.clear(); s->bc.reset(); s->coupler.reset(); s->ghosts.reset();
  s->blocks.reset(); s->faces.reset(); s->forest.reset();
  delete s;
}
void ref_sim_advance(void* h, int steps) {
  auto* s = static_cast<Sim*>(h);
  for (int t = 0; t < steps; ++t) {
    if (!s->physical) {
      s->loop->advance_one();
      continue;
    }
    s->bc->set_time(static_cast<double>(s->step));  // TimeLoop::advance_one (time_loop.h:242-246)
    PhysicalAdvance(s, 0);
    ++s->step;
  }
}
// The physical coupler mode: omega_level[l] the rate of level l (nlev
// levels); before the first advance.
void ref_sim_set_physical(void* h, const f64* omega_level, int nlev) {
  auto* s = static_cast<Sim*>(h);
  s->physical = true;
  s->omega_level.assign(omega_level, omega_level + nlev);
  s->max_level = nlev - 1;
  s->by_level.assign(static_cast<std::size_t>(nlev), {});
  for (label id = 0; id < s->blocks->size(); ++id)
    s->by_level[static_cast<std::size_t>(s->forest->quadrant_level(id))].push_back(id);
  s->pair_couplers.clear();
  for (int l = 0; l + 1 < nlev; ++l)
    s->pair_couplers.push_back(std::make_unique<LevelCoupler>(MPI_COMM_WORLD, *s->faces, *s->forest, *s->blocks,
                                                              s->n, s->n, s->n, to_f64(omega_level[l])));
}
void ref_sim_set_body_force(void* h, const f64* force) {
  auto* s = static_cast<Sim*>(h);
  std::vector<double> f;
  if (force) {
    const std::size_t m = static_cast<std::size_t>(s->blocks->size()) * s->n * s->n * s->n * 3;
    f.assign(force, force + m);
  }
  static_cast<RestatedBoundary*>(s->bc.get())->set_force(s->loop.get(), force ? f.data() : nullptr);
}
int ref_sim_max_level(void* h) { return static_cast<Sim*>(h)->loop->max_level(); }
// Collide / stream counters per level and the coupler call sequence.
int ref_sim_counters(void* h, int* collide, int* stream, int* calls, int max_calls) {
  auto* s = static_cast<Sim*>(h);
  const auto& c = s->loop->counters();
  for (std::size_t l = 0; l < c.collide.size(); ++l) { collide[l] = c.collide[l]; stream[l] = c.stream[l]; }
  int k = 0;
  for (const auto& call : c.coupler_calls) {
    if (k >= max_calls) break;
    calls[2 * k] = static_cast<int>(call.phase);
    calls[2 * k + 1] = call.coarse_level;
    ++k;
  }
  return static_cast<int>(c.coupler_calls.size());
}
void ref_sim_get_core(void* h, f64* out) {
  auto* s = static_cast<Sim*>(h);
  const int n = s->n, n3 = n * n * n;
  for (label id = 0; id < s->blocks->size(); ++id)
    for (int x = 0; x < n; ++x)
      for (int y = 0; y < n; ++y)
        for (int z = 0; z < n; ++z) {
          f64* o = out + ((std::size_t)id * n3 + (x * n + y) * n + z) * Q;
          const double* f = (*s->blocks)[id].populations_at_halo(x + 1, y + 1, z + 1);
          for (int i = 0; i < Q; ++i) o[i] = to_f64(f[i]);
        }
}
void ref_sim_get_padded(void* h, f64* out) {
  auto* s = static_cast<Sim*>(h);
  const std::size_t m = (std::size_t)(s->n + 2) * (s->n + 2) * (s->n + 2) * Q;
  for (label id = 0; id < s->blocks->size(); ++id) {
    const double* f = (*s->blocks)[id].populations_at_halo(0, 0, 0);
    for (std::size_t k = 0; k < m; ++k) out[id * m + k] = to_f64(f[k]);
  }
}
// Sum of MomentumExchangeDrag::force_on_fluid_if over all blocks with an
// obstacle mask [oct][n^3] (or null = every solid / Bouzidi neighbour), the
// aggregation of examples/cylinder3d/cylinder3d_case.h:473-517 on one rank.
void ref_sim_drag(void* h, const uint8_t* mask, f64* out) {
  const std::array<double, 3> f = SimDrag(static_cast<Sim*>(h), mask);
  out[0] = to_f64(f[0]); out[1] = to_f64(f[1]); out[2] = to_f64(f[2]);
}
// Number of coupling points and the plan itself (coarse id,ci,cj,ck, fine
// id,fi,fj,fk, coarse level, fine level) for topology checks.
int ref_sim_plan(void* h, int* out, int max_pts) {
  auto* s = static_cast<Sim*>(h);
  const auto& plan = s->coupler->coupling_plan();
  int k = 0;
  for (const CouplingPoint& p : plan) {
    if (k >= max_pts) break;
    int* o = out + 10 * k;
    o[0] = p.coarse_id; o[1] = p.ci; o[2] = p.cj; o[3] = p.ck;
    o[4] = p.fine_id; o[5] = p.fi; o[6] = p.fj; o[7] = p.fk;
    o[8] = p.coarse_level; o[9] = p.fine_level;
    ++k;
  }
  return static_cast<int>(plan.size());
}

// Coupler phases alone, for the reference's coupler unit tests
// (tests/unit/solver/test_lagrava_coupler.cpp:194-248).
void ref_sim_coupler_full(void* h, int coarse_level) { static_cast<Sim*>(h)->coupler->apply_full_time(coarse_level); }
void ref_sim_coupler_half(void* h, int coarse_level) { static_cast<Sim*>(h)->coupler->apply_half_time(coarse_level); }
void ref_sim_coupler_restrict(void* h, int fine_level) { static_cast<Sim*>(h)->coupler->restrict(fine_level); }

// Reference arithmetic atoms for known-answer checks.
f64 ref_bouzidi_pull(f64 f_bb, f64 f_q, f64 f_same, f64 q) {
  return to_f64(boundary::BouzidiPostCollisionPull(double(f_bb), double(f_q), double(f_same), double(q)));
}
f64 ref_feq(int i, f64 rho, f64 ux, f64 uy, f64 uz) {
  const double u[3] = {ux, uy, uz};
  return to_f64(olb::equilibrium<D>::secondOrder(i, double(rho), u, double(ux * ux + uy * uy + uz * uz)));
}

}  // extern "C"
