// Host side of the finite-difference domain boundary conditions
// (octlb_gpu_set_fd_boundary): the reference's ConcreteDomainBoundaryHandler
// (domain_boundary_handler.cpp:55-89) with InterpolatedVelocity and
// InterpolatedPressure faces.  Every velocity / pressure Dirichlet cell's
// stencil (ApplyInterpolatedVelocityBoundaryCells,
// interpolated_velocity.h:951-1037) is resolved here into an FdCell record:
// the cell's role from its block's extents (plane, edge, corner), its
// prescribed velocity (PrescribedBoundaryU, :69-117: the first touched face
// with an inlet field, else the y+ face's wall velocity on interior top-face
// cells), and each velocity and density read -- inside the block, in the
// overlap padding (rho = 1, u = 0 within min(halo, 2) = 1 cell of the
// block), or mirrored back inside with the crossed components negated, as
// the BoundaryLatticeView reads them (:213-445).  A density read of a
// boundary cell takes the rewritten populations when the reference's in-place
// (ix, iy, iz) walk has rewritten that cell before the reader.
#include "octlb_ctx.h"

namespace octlb_gpu {
template <typename T>
cudaError_t launch_fd_reconstruct(const void*, long long, float, const FdCell*, const int*, int, float*,
                                  const double*, float, const float*, cudaStream_t);
template <typename T>
cudaError_t launch_fd_collide(void*, long long, float, float, const FdCell*, int, float*, const double*,
                              double, float, double*, cudaStream_t);
unsigned fd_collide_parts(int n);
cudaError_t launch_fd_tick(double*, cudaStream_t);
template <typename T>
cudaError_t launch_fd_rows_from_state(const void*, long long, float, const FdCell*, int, float*, cudaStream_t);
cudaError_t launch_fd_fields(const FdCell*, int, const float*, double*, double*, cudaStream_t);
template <typename T>
cudaError_t launch_fd_store(void*, long long, float, const FdCell*, int, const float*, double*, cudaStream_t);
}  // namespace octlb_gpu

using namespace octlb_gpu;
using namespace octlb_host;

namespace {

struct Pos {
  int x, y, z;
  int& operator[](int a) { return a == 0 ? x : (a == 1 ? y : z); }
  int operator[](int a) const { return a == 0 ? x : (a == 1 ? y : z); }
  bool operator<(const Pos& o) const { return x != o.x ? x < o.x : (y != o.y ? y < o.y : z < o.z); }
};

struct Builder {
  octlb_ctx* ctx;
  int n, lb;                       // block edge, local block
  const uint8_t* kinds;            // this block's kinds [n^3]
  const std::vector<int>* row_of;  // this block's cell -> row (-1: not a boundary cell)
  const std::vector<FdCell>* cells;
  std::vector<int>* role_of;       // row -> role
  const double* rho_target;        // [6]

  bool inside(const Pos& p) const { return p.x >= 0 && p.y >= 0 && p.z >= 0 && p.x < n && p.y < n && p.z < n; }
  // The overlap padding the view reads as rest (halo 1: one cell outside).
  bool padding(const Pos& p) const {
    return !inside(p) && p.x >= -1 && p.y >= -1 && p.z >= -1 && p.x <= n && p.y <= n && p.z <= n;
  }
  Pos mirror(const Pos& p) const {
    Pos m = p;
    for (int a = 0; a < 3; ++a) {
      if (m[a] < 0) m[a] = -m[a];
      else if (m[a] >= n) m[a] = 2 * (n - 1) - m[a];
    }
    return m;
  }
  int cell(const Pos& p) const { return (p.x * n + p.y) * n + p.z; }
  long long slot(const Pos& p) const { return core_slot_of(n, lb, p.x, p.y, p.z); }
  int kind(const Pos& p) const { return kinds[cell(p)]; }
  // the single face a cell lies on, or none (axis -1)
  void flat(const Pos& p, int& d, int& o) const {
    int cnt = 0;
    d = -1;
    o = 0;
    for (int a = 0; a < 3; ++a) {
      if (p[a] == 0) { d = a; o = -1; ++cnt; }
      else if (p[a] == n - 1) { d = a; o = 1; ++cnt; }
    }
    if (cnt != 1) d = -1;
  }

  int resolve_u(Pos p, int flips, FdURead& out, int depth = 0) const {
    if (depth > 8) return fail(ctx, OCTLB_EINVAL, "fd boundary: velocity read does not resolve");
    if (!inside(p)) {
      if (padding(p)) {
        out = {0, kFdZero, flips};
        return OCTLB_OK;
      }
      int f = flips;
      for (int a = 0; a < 3; ++a)
        if (p[a] < 0 || p[a] >= n) f ^= 1 << a;
      return resolve_u(mirror(p), f, out, depth + 1);
    }
    const int k = kind(p);
    if (k == kVelocityDirichlet) {
      out = {(*row_of)[cell(p)], kFdPrescribed, flips};
      return OCTLB_OK;
    }
    if (k == kPressureDirichlet) {  // ExtrapolatedU: the inward neighbour's velocity
      int d, o;
      flat(p, d, o);
      if (d < 0) {  // a block-rim cell (an edge or corner of its block): u = 0 (interpolated_velocity.h:297-305)
        out = {0, kFdZero, flips};
        return OCTLB_OK;
      }
      p[d] -= o;
      return resolve_u(p, flips, out, depth + 1);
    }
    out = {slot(p), kFdFluid, flips};
    return OCTLB_OK;
  }

  int resolve_rho(Pos p, const Pos& reader, int reader_role, FdRRead& out, int depth = 0) const {
    if (depth > 8) return fail(ctx, OCTLB_EINVAL, "fd boundary: density read does not resolve");
    if (!inside(p)) {
      if (padding(p)) {
        out = {0, 1.f, kFdRhoConst, 0, 0, 0};
        return OCTLB_OK;
      }
      return resolve_rho(mirror(p), reader, reader_role, out, depth + 1);
    }
    const int k = kind(p);
    int d, o;
    flat(p, d, o);
    if (k == kPressureDirichlet) {  // PrescribedRho (interpolated_velocity.h:320-330): 1 off a flat face
      out = {0, d < 0 ? 1.f : static_cast<float>(rho_target[2 * d + (o > 0)]), kFdRhoConst, 0, 0, 0};
      return OCTLB_OK;
    }
    const int row = (*row_of)[cell(p)];
    bool fresh = false;
    if (row >= 0 && (*role_of)[row] >= 1 && p < reader) {  // a cell the pass rewrites
      const int pr = (*role_of)[row];
      if (pr == reader_role) return fail(ctx, OCTLB_EINVAL, "fd boundary: blocks of n >= 4 only");
      fresh = pr < reader_role;
    }
    if (k == kVelocityDirichlet && d >= 0) {
      out = {fresh ? row : slot(p), 0.f, fresh ? kFdRhoBmNew : kFdRhoBmPre, row, d, o};
    } else {
      // urow = 1 marks a kBulk cell (its stored density carries ConstRhoBGK's shift)
      out = {fresh ? row : slot(p), 0.f, fresh ? kFdRhoSumNew : kFdRhoSumPre, k == kBulk && !fresh ? 1 : 0, 0, 0};
    }
    return OCTLB_OK;
  }
};

}  // namespace

namespace octlb_host {

// The pass after a step of level S: the reference's apply_post_stream()
// after each level's stream -- an empty level's too -- runs it on every
// tree-boundary block of every level (domain_boundary_handler.cpp:81-93,
// time_loop.h:201-214), so every level's records run:
// planes, edges, corners into the rows, then the rows into the state,
// uncollided, as the reference rewrites the cells in place -- a later pass
// on a level that has not stepped since reads them as its "pre" values.
template <typename T>
int fd_after_step(octlb_ctx* ctx, Level& S) {
  (void)S;
  if (!ctx->fd_on) return OCTLB_OK;
  const double* time = ctx->fd_time.as<double>();
  for (Level& L : ctx->levels) {
    if (L.nblk == 0 || L.fd_rows == 0) continue;
    void* state = cur_buf(L);
    const FdCell* cells = L.fd_cells.as<FdCell>();
    float* fnew = L.fd_new.as<float>();
    const float omega = static_cast<float>(ctx->omega_l[L.lvl]);
    for (int role = 1; role <= 3; ++role) {
      const int n = L.fd_count[role];
      if (n == 0) continue;
      CK(launch_fd_reconstruct<T>(state, L.nslots, L.inv_scale, cells, L.fd_lists.as<int>() + L.fd_first[role], n,
                                  fnew, time, omega, ctx->const_rho ? ctx->cr_shift.as<float>() + L.lvl : nullptr,
                                  ctx->stream));
      ++ctx->launch_count;
    }
    // on a single-level mesh this is the step's only pass: the store ticks
    // the boundary clock in place of a launch of its own
    CK(launch_fd_store<T>(state, L.nslots, L.scale, cells, L.fd_rows, fnew,
                          ctx->fd_single ? ctx->fd_time.as<double>() : nullptr, ctx->stream));
    ++ctx->launch_count;
  }
  return OCTLB_OK;
}

// The collide of level L's boundary cells at the start of its step
// (collide_level's per-cell dispatch, domain_boundary_handler.cpp:60-79), at
// this advance_one's time, from the rows the last pass left.  Under
// ConstRhoBGK the velocity cells' collide densities go to the partials the
// average update then reads.
template <typename T>
int fd_before_step(octlb_ctx* ctx, Level& L) {
  if (!ctx->fd_on || L.nblk == 0 || L.fd_rows == 0) return OCTLB_OK;
  CK(launch_fd_collide<T>(cur_buf(L), L.nslots, L.scale, L.inv_scale, L.fd_cells.as<FdCell>(), L.fd_rows,
                          L.fd_new.as<float>(), ctx->fd_time.as<double>(), 0.0,
                          static_cast<float>(ctx->omega_l[L.lvl]),
                          ctx->const_rho && L.lvl == ctx->cr_level ? ctx->fd_cr_part.as<double>() : nullptr,
                          ctx->stream));
  ++ctx->launch_count;
  return OCTLB_OK;
}
template int fd_before_step<float>(octlb_ctx*, Level&);
template int fd_before_step<__half>(octlb_ctx*, Level&);
template int fd_after_step<float>(octlb_ctx*, Level&);
template int fd_after_step<__half>(octlb_ctx*, Level&);

// get_fields: the Dirichlet cells' rho and u from their rows (level L's
// staging arrays, indexed by local core slot).
int fd_fix_fields(octlb_ctx* ctx, Level& L, double* rho, double* u) {
  if (!ctx->fd_on || L.nblk == 0 || L.fd_rows == 0) return OCTLB_OK;
  CK(launch_fd_fields(L.fd_cells.as<FdCell>(), L.fd_rows, L.fd_new.as<float>(), rho, u, ctx->stream));
  return OCTLB_OK;
}

int fd_end_of_step(octlb_ctx* ctx) {
  if (!ctx->fd_on || ctx->fd_single) return OCTLB_OK;  // (a single level's store ticked it)
  CK(launch_fd_tick(ctx->fd_time.as<double>(), ctx->stream));
  ++ctx->launch_count;
  return OCTLB_OK;
}

}  // namespace octlb_host

extern "C" {

int octlb_fd_stamp_kinds(const octlb_tables* t, const int types[6], uint8_t* kinds) {
  if (!t || !types || !kinds || !t->tree_boundary || t->n < 1) return OCTLB_EINVAL;
  const int n = t->n;
  const long long n3 = static_cast<long long>(n) * n * n;
  std::memcpy(kinds, t->kinds, static_cast<size_t>(n3 * t->n_blocks));
  // BcKindFromSpecType (bc_installer.h:44-58) and StampTreeBoundaryCells
  // (:95-138): the face slab of every tree-boundary face, solid cells kept.
  static const uint8_t kind_of[5] = {kBounceBack, kMovingBounceBack, kVelocityDirichlet, kOutflow,
                                     kPressureDirichlet};
  for (int f = 0; f < 6; ++f)
    if (types[f] < 0 || types[f] > 4) return OCTLB_EINVAL;
  for (int k = 0; k < t->n_tree_boundary; ++k) {
    const int b = t->tree_boundary[2 * k], dir = t->tree_boundary[2 * k + 1];
    if (b < 0 || b >= t->n_blocks || dir < 0 || dir > 5) return OCTLB_EINVAL;
    const int ax = dir / 2, side = (dir & 1) ? n - 1 : 0;
    for (int a = 0; a < n; ++a)
      for (int c = 0; c < n; ++c) {
        int p[3];
        p[ax] = side;
        p[(ax + 1) % 3] = a;
        p[(ax + 2) % 3] = c;
        const long long g = b * n3 + (static_cast<long long>(p[0]) * n + p[1]) * n + p[2];
        if (kinds[g] != kSolid) kinds[g] = kind_of[types[dir]];
      }
  }
  return OCTLB_OK;
}

}  // extern "C"

namespace octlb_host {

int check_inlets(octlb_ctx* ctx, const octlb_fd_inlet* inlets) {
  if (!inlets) return OCTLB_OK;
  for (int f = 0; f < 6; ++f) {
    const octlb_fd_inlet& in = inlets[f];
    if (in.kind < OCTLB_INLET_NONE || in.kind > OCTLB_INLET_CHANNEL_POISEUILLE)
      return fail(ctx, OCTLB_EINVAL, "fd boundary: inlet kind outside 0..3");
    if (in.kind == OCTLB_INLET_POISEUILLE && (in.n_inplane[0] < 1 || in.n_inplane[1] < 1))
      return fail(ctx, OCTLB_EINVAL, "fd boundary: a Poiseuille inlet needs n_inplane >= 1");
    if (in.kind == OCTLB_INLET_CHANNEL_POISEUILLE && !(in.patch[1] > in.patch[0] && in.patch[3] > in.patch[2]))
      return fail(ctx, OCTLB_EINVAL, "fd boundary: a channel inlet patch needs hi > lo");
  }
  return OCTLB_OK;
}

// The inlet field of face `face` at cell p of a block with bounds bd (x0, y0,
// z0, x1, y1, z1), before the ramp (inlet_velocity_field.h: UniformInletProfile
// :131-159, PoiseuilleInletProfile :38-129 from block-local indices,
// ChannelPoiseuilleInletProfile :163-269 from the physical position origin +
// (index + 1/2) cell width, as PrescribedBoundaryU supplies it,
// interpolated_velocity.h:69-117).  In-plane axes: y, z on x faces; x, z on y
// faces; x, y on z faces.
void inlet_velocity(const octlb_fd_inlet& in, int face, const Pos& p, int n, const double* bd, double u[3]) {
  if (in.kind == OCTLB_INLET_UNIFORM) {
    for (int d = 0; d < 3; ++d) u[d] = in.u[d];
    return;
  }
  const int ax = face / 2, a0 = ax == 0 ? 1 : 0, a1 = ax == 2 ? 1 : 2;
  double p0, p1;
  if (in.kind == OCTLB_INLET_POISEUILLE) {
    const double c0 = (p[a0] + 0.5) / in.n_inplane[0], c1 = (p[a1] + 0.5) / in.n_inplane[1];
    p0 = 4.0 * c0 * (1.0 - c0);
    p1 = 4.0 * c1 * (1.0 - c1);
  } else {
    const double cw = (bd[3] - bd[0]) / n;
    auto clamp01 = [](double c) { return c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c); };
    const double c0 = clamp01((bd[a0] + (p[a0] + 0.5) * cw - in.patch[0]) / (in.patch[1] - in.patch[0]));
    const double c1 = clamp01((bd[a1] + (p[a1] + 0.5) * cw - in.patch[2]) / (in.patch[3] - in.patch[2]));
    p0 = 4.0 * c0 * (1.0 - c0);
    p1 = 4.0 * c1 * (1.0 - c1);
  }
  const double mag = in.u_peak * p0 * p1;
  for (int d = 0; d < 3; ++d) u[d] = mag * in.u[d];
}

// The uniform inlets of octlb_gpu_set_fd_boundary / octlb_fd_plan: face f
// has one where inlet_u[3 f ..] is nonzero.
std::vector<octlb_fd_inlet> uniform_inlets(const double* inlet_u, double ramp_end_t) {
  std::vector<octlb_fd_inlet> v(6);
  for (int f = 0; f < 6; ++f) {
    v[f] = octlb_fd_inlet{};
    if (!inlet_u) continue;
    const double* iu = inlet_u + 3 * f;
    if (iu[0] == 0.0 && iu[1] == 0.0 && iu[2] == 0.0) continue;
    v[f].kind = OCTLB_INLET_UNIFORM;
    for (int d = 0; d < 3; ++d) v[f].u[d] = iu[d];
    v[f].ramp_end_t = ramp_end_t;
  }
  return v;
}

// The records of the pass for the blocks `blocks` (global ids, all of forest
// level 0, in local order) with the given kinds: cells in (block, x, y, z)
// order, and per role the rows of that role.  Host only.
int fd_build(octlb_ctx* ctx, int n, const std::vector<int>& blocks, const uint8_t* kinds, const double* bounds,
             const int types[6], const double* u_wall, const double* rho_target, const octlb_fd_inlet* inlets,
             std::vector<FdCell>& cells, std::vector<int>& lists, std::vector<int>& first, std::vector<int>& count) {
  for (int f = 0; f < 6; ++f)
    if (types[f] < 0 || types[f] > 4) return fail(ctx, OCTLB_EINVAL, "fd boundary: face type outside 0..4");
  if (int rc = check_inlets(ctx, inlets)) return rc;
  for (int f = 0; f < 6 && inlets; ++f)
    if (inlets[f].kind == OCTLB_INLET_CHANNEL_POISEUILLE && !bounds)
      return fail(ctx, OCTLB_EINVAL, "fd boundary: a channel inlet needs the blocks' bounds in the tables");
  if (n < 4) return fail(ctx, OCTLB_EINVAL, "fd boundary: blocks of n >= 4 only");
  const long long n3 = static_cast<long long>(n) * n * n;
  const int nblk = static_cast<int>(blocks.size());
  // rows: boundary cells in (block, x, y, z) order
  cells.clear();
  std::vector<std::vector<int>> row_of(static_cast<size_t>(nblk), std::vector<int>(static_cast<size_t>(n3), -1));
  for (int lb = 0; lb < nblk; ++lb) {
    const uint8_t* kb = kinds + static_cast<size_t>(blocks[lb]) * n3;
    for (long long c = 0; c < n3; ++c)
      if (kb[c] == kVelocityDirichlet || kb[c] == kPressureDirichlet || kb[c] == kBounceBack) {
        row_of[lb][c] = static_cast<int>(cells.size());
        FdCell fc{};
        fc.slot = lb * n3 + c;
        fc.kind = kb[c];
        cells.push_back(fc);
      }
  }
  std::vector<int> role(cells.size());
  for (int lb = 0; lb < nblk; ++lb)
    for (long long c = 0; c < n3; ++c) {
      const int r = row_of[lb][c];
      if (r < 0) continue;
      const int x = static_cast<int>(c / (n * n)), y = static_cast<int>((c / n) % n), z = static_cast<int>(c % n);
      int cnt = 0;
      for (int v : {x, y, z}) cnt += (v == 0 || v == n - 1) ? 1 : 0;
      if (cells[r].kind == kBounceBack) cnt = 0;  // no reconstruction: the collide's full-way swap only
      else if (cnt == 0) return fail(ctx, OCTLB_EINVAL, "fd boundary: a Dirichlet cell off its block's faces");
      role[r] = cnt;
    }
  for (int lb = 0; lb < nblk; ++lb) {
    Builder B{ctx, n, lb, kinds + static_cast<size_t>(blocks[lb]) * n3, &row_of[lb], &cells, &role, rho_target};
    for (long long c = 0; c < n3; ++c) {
      const int r = row_of[lb][c];
      if (r < 0) continue;
      FdCell& fc = cells[r];
      const Pos p{static_cast<int>(c / (n * n)), static_cast<int>((c / n) % n), static_cast<int>(c % n)};
      fc.role = role[r];
      if (fc.role == 0) continue;
      // prescribed velocity
      const bool on[6] = {p.x == 0, p.x == n - 1, p.y == 0, p.y == n - 1, p.z == 0, p.z == n - 1};
      bool done = false;
      for (int f = 0; f < 6 && !done; ++f) {
        if (!on[f] || !inlets || inlets[f].kind == OCTLB_INLET_NONE) continue;
        double iu[3];
        inlet_velocity(inlets[f], f, p, n, bounds + 6LL * blocks[lb], iu);
        for (int a = 0; a < 3; ++a) fc.u_base[a] = static_cast<float>(iu[a]);
        fc.ramp_end = static_cast<float>(inlets[f].ramp_end_t);
        done = true;
      }
      if (!done && p.y == n - 1 && p.x > 0 && p.x < n - 1 && p.z > 0 && p.z < n - 1)
        for (int a = 0; a < 3; ++a) fc.u_base[a] = static_cast<float>(u_wall[3 * 3 + a]);
      int side[3];
      for (int a = 0; a < 3; ++a) side[a] = p[a] == 0 ? -1 : (p[a] == n - 1 ? 1 : 0);
      auto at = [&](std::initializer_list<std::pair<int, int>> steps) {
        Pos q = p;
        for (const auto& s : steps) q[s.first] += s.second;
        return q;
      };
      int rc = OCTLB_OK;
      if (fc.role == 1) {
        int d, o;
        B.flat(p, d, o);
        fc.d = d;
        fc.o = o;
        if (fc.kind == kPressureDirichlet) fc.rho_target = static_cast<float>(rho_target[2 * d + (o > 0)]);
        const int t0 = std::min((d + 1) % 3, (d + 2) % 3), t1 = 3 - d - t0;
        const Pos q[7] = {p, at({{d, -o}}), at({{d, -2 * o}}), at({{t0, 1}}), at({{t0, -1}}), at({{t1, 1}}),
                          at({{t1, -1}})};
        for (int j = 0; j < 7 && !rc; ++j) rc = B.resolve_u(q[j], 0, fc.u[j]);
      } else if (fc.role == 2) {
        // ApplyInterpolatedVelocityBoundaryCells' pairing of the edge's two
        // normals (interpolated_velocity.h:991-1012): x & y -> axis z,
        // x & z -> axis y with d1 = z, d2 = x, y & z -> axis x.
        int plane, n1, n2;
        if (side[0] && side[1]) { plane = 2; n1 = side[0]; n2 = side[1]; }
        else if (side[0] && side[2]) { plane = 1; n1 = side[0]; n2 = side[2]; }
        else { plane = 0; n1 = side[1]; n2 = side[2]; }
        const int d1 = (plane + 1) % 3, d2 = (plane + 2) % 3;
        fc.ax[0] = plane; fc.ax[1] = d1; fc.ax[2] = d2;
        fc.nrm[0] = n1; fc.nrm[1] = n2;
        const Pos q[7] = {p, at({{plane, 1}}), at({{plane, -1}}), at({{d1, -n1}}), at({{d1, -2 * n1}}),
                          at({{d2, -n2}}), at({{d2, -2 * n2}})};
        for (int j = 0; j < 7 && !rc; ++j) rc = B.resolve_u(q[j], 0, fc.u[j]);
        const Pos rq[4] = {at({{d2, -n2}}), at({{d1, -n1}}), at({{d2, -2 * n2}}), at({{d1, -2 * n1}})};
        for (int j = 0; j < 4 && !rc; ++j) rc = B.resolve_rho(rq[j], p, 2, fc.r[j]);
      } else {
        for (int a = 0; a < 3; ++a) fc.nrm[a] = side[a];
        const Pos q[7] = {p, at({{0, -side[0]}}), at({{0, -2 * side[0]}}), at({{1, -side[1]}}),
                          at({{1, -2 * side[1]}}), at({{2, -side[2]}}), at({{2, -2 * side[2]}})};
        for (int j = 0; j < 7 && !rc; ++j) rc = B.resolve_u(q[j], 0, fc.u[j]);
        const Pos rq[6] = {at({{2, -side[2]}}), at({{1, -side[1]}}), at({{0, -side[0]}}),
                           at({{2, -2 * side[2]}}), at({{1, -2 * side[1]}}), at({{0, -2 * side[0]}})};
        for (int j = 0; j < 6 && !rc; ++j) rc = B.resolve_rho(rq[j], p, 3, fc.r[j]);
      }
      if (rc) return rc;
    }
  }
  const long long ncore_owned = nblk * n3;
  // every index the kernels derive
  const long long nrows = static_cast<long long>(cells.size());
  for (const FdCell& fc : cells) {
    if (fc.slot < 0 || fc.slot >= ncore_owned) return fail(ctx, OCTLB_EINVAL, "internal: fd slot");
    for (const FdURead& u : fc.u) {
      if (u.code == kFdFluid && (u.idx < 0 || u.idx >= ncore_owned)) return fail(ctx, OCTLB_EINVAL, "internal: fd u");
      if (u.code == kFdPrescribed && (u.idx < 0 || u.idx >= nrows)) return fail(ctx, OCTLB_EINVAL, "internal: fd u");
    }
    for (int j = 0; j < (fc.role == 2 ? 4 : fc.role == 3 ? 6 : 0); ++j) {
      const FdRRead& r = fc.r[j];
      const bool pre = r.code == kFdRhoSumPre || r.code == kFdRhoBmPre;
      const bool nw = r.code == kFdRhoSumNew || r.code == kFdRhoBmNew;
      if ((pre && (r.idx < 0 || r.idx >= ncore_owned)) || (nw && (r.idx < 0 || r.idx >= nrows)))
        return fail(ctx, OCTLB_EINVAL, "internal: fd density read");
      if ((r.code == kFdRhoBmPre || r.code == kFdRhoBmNew) && (r.urow < 0 || r.urow >= nrows || r.d < 0 || r.d > 2))
        return fail(ctx, OCTLB_EINVAL, "internal: fd density read");
    }
  }
  lists.clear();
  first.assign(4, 0);
  count.assign(4, 0);
  for (int rl = 1; rl <= 3; ++rl) {
    first[rl] = static_cast<int>(lists.size());
    for (size_t r = 0; r < cells.size(); ++r)
      if (cells[r].role == rl) lists.push_back(static_cast<int>(r));
    count[rl] = static_cast<int>(lists.size()) - first[rl];
  }
  return OCTLB_OK;
}

}  // namespace octlb_host

extern "C" {

int octlb_gpu_set_fd_boundary(octlb_ctx* ctx, const int types[6], const double* u_wall, const double* rho_target,
                              const double* inlet_u, double ramp_end_t) {
  const std::vector<octlb_fd_inlet> inlets = uniform_inlets(inlet_u, ramp_end_t);
  return octlb_gpu_set_fd_boundary_inlets(ctx, types, u_wall, rho_target, inlets.data());
}

int octlb_gpu_set_fd_boundary_inlets(octlb_ctx* ctx, const int types[6], const double* u_wall,
                                     const double* rho_target, const octlb_fd_inlet* inlets) {
  if (!ctx || !types || !u_wall || !rho_target) return OCTLB_EINVAL;
  if (ctx->levels.empty()) return fail(ctx, OCTLB_ESTATE, "context not initialised");
  for (int c : ctx->counters_collide)
    if (c != 0) return fail(ctx, OCTLB_ESTATE, "set_fd_boundary comes before the first advance");
  if (ctx->fd_on) return fail(ctx, OCTLB_ESTATE, "fd boundary already set");
  if (ctx->stream_mode != OCTLB_STREAM_ROTATE || ctx->periodic || ctx->comm)
    return fail(ctx, OCTLB_EINVAL, "fd boundary: one context, rotate stream rule, not periodic");
  int used = 0;
  for (const Level& L : ctx->levels) {
    if (L.nblk == 0) continue;
    ++used;
    if (L.n_bb > 0) return fail(ctx, OCTLB_EINVAL, "fd boundary: the tree-boundary faces must carry no restated fill");
  }
  if (used > 1 && !ctx->cpl_cells_bulk)
    return fail(ctx, OCTLB_EINVAL,
                "fd boundary on a multi-level mesh: every coupler source and target must be a kBulk cell "
                "(the coarse-fine interfaces away from the domain faces)");
  std::vector<std::vector<FdCell>> cells(ctx->levels.size());
  for (size_t l = 0; l < ctx->levels.size(); ++l) {
    Level& L = ctx->levels[l];
    if (L.nblk == 0) continue;
    std::vector<int> lists;
    const double* bounds = ctx->bounds.size() == 6 * static_cast<size_t>(ctx->n_blocks) ? ctx->bounds.data() : nullptr;
    if (int rc = fd_build(ctx, ctx->n, L.blocks, ctx->kinds.data(), bounds, types, u_wall, rho_target,
                          inlets, cells[l], lists, L.fd_first, L.fd_count))
      return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(upload(L.fd_cells, cells[l]));
    CK(upload(L.fd_lists, lists));
    CK(L.fd_new.alloc(cells[l].size() * kQ * sizeof(float)));
    L.fd_rows = static_cast<int>(cells[l].size());
  }
  size_t total = 0;
  for (const auto& c : cells) total += c.size();
  if (total == 0) return fail(ctx, OCTLB_EINVAL, "fd boundary: no Dirichlet or bounce-back cells");
  CK(upload(ctx->fd_time, std::vector<double>{0.0}));
  // ConstRhoBGK (chosen before): the finest level's velocity cells'
  // collide densities join its statistics (the reference's
  // kFluidAndBoundary scope, collected where level >= max_level_,
  // time_loop.h:201-222)
  if (ctx->const_rho) {
    ctx->fd_vel = 0;
    int rows = 0;
    if (ctx->cr_level >= 0 && ctx->cr_level < static_cast<int>(cells.size())) {
      rows = static_cast<int>(cells[ctx->cr_level].size());
      for (const FdCell& fc : cells[ctx->cr_level]) ctx->fd_vel += fc.kind == kVelocityDirichlet ? 1 : 0;
    }
    ctx->fd_cr_parts = static_cast<int>(fd_collide_parts(std::max(rows, 1)));
    CK(ctx->fd_cr_part.alloc(static_cast<size_t>(ctx->fd_cr_parts) * sizeof(double)));
    CK(cudaMemsetAsync(ctx->fd_cr_part.p, 0, static_cast<size_t>(ctx->fd_cr_parts) * sizeof(double), ctx->stream));
  }
  // The rows start as the stored initial state of the boundary cells,
  // which the initial collide left uncollided (it takes kBulk cells only):
  // the first step's collide starts from them (and the fields before any
  // step read them).
  for (Level& L : ctx->levels) {
    if (L.nblk == 0 || L.fd_rows == 0) continue;
    const FdCell* dc = L.fd_cells.as<FdCell>();
    float* rows = L.fd_new.as<float>();
    if (ctx->precision == OCTLB_FP32)
      CK(launch_fd_rows_from_state<float>(L.buf[L.cur].p, L.nslots, L.inv_scale, dc, L.fd_rows, rows, ctx->stream));
    else
      CK(launch_fd_rows_from_state<__half>(L.buf[L.cur].p, L.nslots, L.inv_scale, dc, L.fd_rows, rows,
                                           ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->fd_on = true;
  // one level in the recursion: one pass per advance_one (a mesh whose
  // blocks sit on a finer forest level also steps its empty coarser levels,
  // each with a pass)
  ctx->fd_single = ctx->levels.size() == 1;
  clear_graphs(ctx);  // the captured launch sequence changes
  return OCTLB_OK;
}

int octlb_fd_plan(const octlb_tables* t, const int types[6], const double* u_wall, const double* rho_target,
                  const double* inlet_u, double ramp_end_t, void* records, int max_records) {
  const std::vector<octlb_fd_inlet> inlets = uniform_inlets(inlet_u, ramp_end_t);
  return octlb_fd_plan_inlets(t, types, u_wall, rho_target, inlets.data(), records, max_records);
}

int octlb_fd_plan_inlets(const octlb_tables* t, const int types[6], const double* u_wall, const double* rho_target,
                         const octlb_fd_inlet* inlets, void* records, int max_records) {
  if (!t || !types || !u_wall || !rho_target || t->n_blocks < 1) return OCTLB_EINVAL;
  std::vector<int> blocks(t->n_blocks);
  for (int b = 0; b < t->n_blocks; ++b) {
    if (t->levels[b] != 0) return OCTLB_EINVAL;
    blocks[b] = b;
  }
  octlb_ctx ctx;
  std::vector<FdCell> cells;
  std::vector<int> lists, first, count;
  if (int rc = fd_build(&ctx, t->n, blocks, t->kinds, t->bounds, types, u_wall, rho_target, inlets, cells, lists,
                        first, count))
    return rc;
  if (cells.empty()) return OCTLB_EINVAL;  // no Dirichlet or bounce-back cells
  if (records)
    std::memcpy(records, cells.data(), sizeof(FdCell) * std::min<size_t>(cells.size(), max_records));
  return static_cast<int>(cells.size());
}

int octlb_fd_record_bytes(void) { return static_cast<int>(sizeof(FdCell)); }

}  // extern "C"
