// Host side of the C ABI (include/octlb_gpu.h): flattens the forest tables
// into per-level device tables, owns every device allocation, and drives the
// reference's recursive subcycling (TimeLoop::advance, time_loop.h:201-240) as
// a sequence of kernel launches on one stream.
#include "octlb_ctx.h"

namespace octlb_host {

int fail(octlb_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}
int cuda_fail(octlb_ctx* c, cudaError_t e, const char* where) {
  return fail(c, OCTLB_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Coupling plan of the reference (AppendFaceCouplingPoints,
// level_coupler.cpp:70-139): for each hanging face and fine slot, the fine
// block's quadrant of the coarse face decides which (n/2)^2 coarse face cells
// pair 1:1 with the fine block's first (n/2)^2 interface cells.
std::vector<PlanPoint> build_plan(const octlb_tables* t) {
  std::vector<PlanPoint> plan;
  const int n = t->n, half = n / 2;
  for (int f = 0; f < t->n_coarse_fine; ++f) {
    const int* r = t->coarse_fine + 8 * f;
    const double* bd = t->coarse_fine_bounds + 30 * f;
    const int normal = r[5], ax = normal / 2, tan0 = (ax + 1) % 3, tan1 = (ax + 2) % 3;
    const bool is_max = (normal & 1) != 0;
    const double cc[3] = {0.5 * (bd[0] + bd[3]), 0.5 * (bd[1] + bd[4]), 0.5 * (bd[2] + bd[5])};
    for (int s = 0; s < 4; ++s) {
      const double* fb = bd + 6 + 6 * s;
      const double fc[3] = {0.5 * (fb[0] + fb[3]), 0.5 * (fb[1] + fb[4]), 0.5 * (fb[2] + fb[5])};
      const int q0 = fc[tan0] < cc[tan0] ? 0 : 1, q1 = fc[tan1] < cc[tan1] ? 0 : 1;
      for (int a = q0 * half; a < q0 * half + half; ++a)
        for (int b = q1 * half; b < q1 * half + half; ++b) {
          int ci[3], fi[3];
          ci[ax] = is_max ? n - 1 : 0;
          fi[ax] = is_max ? 0 : n - 1;
          ci[tan0] = a; ci[tan1] = b;
          fi[tan0] = a - q0 * half; fi[tan1] = b - q1 * half;
          plan.push_back({r[0], ci[0], ci[1], ci[2], r[1 + s], fi[0], fi[1], fi[2], normal, r[6], r[7], s});
        }
    }
  }
  return plan;
}

// ReadMacro of a double-precision cell (level_coupler.cpp:183-189), as floats
// (rho - 1, u, f_neq).
void host_macro(const double* f, float out[23]) {
  double drho = 0, j[3] = {0, 0, 0};
  for (int i = 0; i < kQ; ++i) {
    drho += f[i]; j[0] += cx(i) * f[i]; j[1] += cy(i) * f[i]; j[2] += cz(i) * f[i];
  }
  const double rho = 1.0 + drho, u[3] = {j[0] / rho, j[1] / rho, j[2] / rho};
  const double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  out[0] = static_cast<float>(drho);
  for (int d = 0; d < 3; ++d) out[1 + d] = static_cast<float>(u[d]);
  for (int i = 0; i < kQ; ++i) {
    const double cu = cx(i) * u[0] + cy(i) * u[1] + cz(i) * u[2];
    const double feq = rho * wd(i) * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq) - wd(i);
    out[4 + i] = static_cast<float>(f[i] - feq);
  }
}

template <typename T>
int do_advance_level(octlb_ctx* ctx, int l);

// Launches the pending restrictions (two per launch).
template <typename T>
int flush_restricts(octlb_ctx* ctx) {
  auto& P = ctx->pending_restrict;
  const ProlongOp none_p{};
  const RestrictOp none_r{};
  for (size_t k = 0; k < P.size(); k += 2) {
    CK(launch_couple<T>(none_p, P[k].op, k + 1 < P.size() ? P[k + 1].op : none_r, ctx->stream));
    ++ctx->launch_count;
  }
  P.clear();
  return OCTLB_OK;
}

template <typename T>
int launch_level_step(octlb_ctx* ctx, Level& L) {
  if (L.nblk == 0) {
    // A rank context with no block on this level still takes part in the
    // level's two exchanges (it may receive save rows for its coupler items).
    // The finite-difference pass runs after an empty level's step too.
    if (int rc = exchange_cells<T>(ctx, L)) return rc;
    if (int rc = fd_after_step<T>(ctx, L)) return rc;
    return exchange_rows(ctx, L);  // (slab contexts own every level's block)
  }
  { const int rc = flush_restricts<T>(ctx); if (rc) return rc; }  // the step reads what they write
  // Body force on the stored post-collision state (the reference's apply()
  // hook after collide, time_loop.h:207-211).  The boundary fills and the
  // same-level exchange that follow there need no launch: the step reads
  // neighbour cores through the slot map and fill targets from their
  // sources.  Rank contexts then refresh their mirror blocks: the cells of
  // other ranks' blocks this level's pulls read.
  T* cur = static_cast<T*>(cur_buf(L));
  if (L.has_force) {
    CK(launch_add_force<T>(L.args, cur, L.body_force.as<float>(), ctx->stream));
    ++ctx->launch_count;
  }
  if (int rc = ctx->slab ? exchange_slab<T>(ctx, L) : exchange_cells<T>(ctx, L)) return rc;
  // the finite-difference boundary cells' collide (the step pulls from them)
  if (int rc = fd_before_step<T>(ctx, L)) return rc;

  StepArgs a = L.args;
  a.src = cur;
  a.dst = L.buf[1 - L.cur].p;
  StepRecord* rec = nullptr;
  void* next_cur = nullptr;
  if (ctx->adj && ctx->adj->recording) {
    // Record the step: its input buffer is the record's (the previous step
    // of the level wrote there, or the segment's checkpoint was restored
    // there), its output goes to the next record of the level, its save rows
    // to the record's.
    AdjointState& A = *ctx->adj;
    if (A.nrec >= A.recs.size() || A.recs[A.nrec].level != L.lvl)
      return fail(ctx, OCTLB_ESTATE, "adjoint: step record pool out of order");
    rec = &A.recs[A.nrec];
    if (rec->snap.p != a.src)
      CK(cudaMemcpyAsync(rec->snap.p, a.src, rec->snap.bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    a.src = rec->snap.p;
    const int nx = A.next_same[A.nrec];
    if (nx >= 0) a.dst = next_cur = A.recs[nx].snap.p;
    a.save_buf = rec->save.as<float>();
    L.rec_save = rec->save.p;
    rec->drag = ctx->drag && L.n_drag > 0 && L.substep + 1 == (1 << L.lvl);
    A.last_rec[L.lvl] = static_cast<int>(A.nrec++);
  }
  // The force after advance_one reads the input of each level's last step
  // (the reference computes MomentumExchangeDrag once, after advance_one):
  // launched on the side stream before that step, so it overlaps the step
  // and what follows it.  (The adjoint's recomputation needs no force: it
  // records the inputs.)
  if (ctx->drag && L.n_drag > 0 && L.substep + 1 == (1 << L.lvl) && !rec) {
    CK(cudaEventRecord(ctx->ev_fork, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
    CK(launch_drag<T>(a, ctx->stream_mode == OCTLB_STREAM_LINKS, L.drag_items.as<DragItem>(), L.n_drag,
                      ctx->drag_partial.as<double>() + 3 * L.drag_off, ctx->side));
    ctx->side_busy = true;
    ++ctx->launch_count;
  }
  if (ctx->const_rho && L.lvl != ctx->cr_level) {
    // ConstRhoBGK, a level above the finest: the step only streams (and
    // saves the coupler's rows); the level collides in do_advance_level once
    // its coupling is done, at the average density the finest level's last
    // collide gives (the stored state of every level is again one collide
    // ahead after advance_one)
    const bool links = ctx->stream_mode == OCTLB_STREAM_LINKS;
    if (L.use_map && ctx->map_global && ctx->map_cells == (links ? 1 : 2)) {
      CK(launch_step_map_nc<T>(a, L.near, links, L.has_flags, ctx->stream));
    } else {
      CK(launch_step_nc<T>(a, L.near, links, L.has_flags, ctx->stream));
      if (L.near.n > 0) ++ctx->launch_count;
    }
    // the level's kBulk cells are post-stream now: no density shift
    if (ctx->fd_on) CK(cudaMemsetAsync(ctx->cr_shift.as<float>() + L.lvl, 0, sizeof(float), ctx->stream));
  } else if (ctx->const_rho) {
    // ConstRhoBGK: average_rho from the last collide's statistics
    // (time_loop.h:220-222), then the step whose collide uses it
    CK(launch_cr_update(ctx->cr_avg.as<double>(), ctx->cr_part.as<double>(), ctx->cr_nparts + ctx->cr_pparts,
                        ctx->cr_count, ctx->fd_cr_part.as<double>(), ctx->fd_cr_parts, ctx->fd_vel,
                        ctx->cr_shift.as<float>() + L.lvl, ctx->stream));
    const bool links = ctx->stream_mode == OCTLB_STREAM_LINKS;
    if (L.use_map && ctx->map_global && ctx->map_cells == (links ? 1 : 2)) {
      CK(launch_step_map_cr<T>(a, L.near, links, L.has_flags, ctx->stream));
      ++ctx->launch_count;
    } else {
      CK(launch_step_cr<T>(a, L.near, links, L.has_flags, ctx->stream));
      ctx->launch_count += 1 + (L.near.n > 0 ? 1 : 0);
    }
  } else if (L.aa) {
    // AA order: cur is the layout (1: reversed), both buffers the same memory
    if (L.cur == 0 && L.use_aa_rows) CK(launch_step_aa_rows<T>(a, ctx->aa_rows, L.aa_rows_grid, ctx->stream));
    else if (L.cur == 1 && L.use_aa_local_rows)
      CK(launch_step_rows_h(a, ctx->fp16_rows, L.aa_local_grid, true, ctx->stream));
    else CK(launch_step_aa<T>(a, L.cur == 1, ctx->stream));
  } else if (L.use_bulk) {
    CK(launch_step_bulk<T>(a, L.bulk_grid, ctx->stream));
  } else if (L.use_rows) {
    CK(launch_step_rows_h(a, ctx->fp16_rows, L.rows_grid, false, ctx->stream));
  } else if (L.use_pair) {
    CK(launch_step_pair<T>(a, ctx->stream));
  } else if (L.use_map) {
    CK(launch_step_map<T>(a, L.near, ctx->stream_mode == OCTLB_STREAM_LINKS, L.has_flags, ctx->map_cells,
                          ctx->map_global, ctx->stream));
  } else {
    CK(launch_step<T>(a, ctx->periodic != 0, ctx->stream_mode == OCTLB_STREAM_LINKS, L.has_flags,
                      ctx->stream));
    CK(launch_step_near<T>(a, L.near, ctx->stream));
    if (L.near.n > 0) ++ctx->launch_count;
  }
  if (L.args.nitems > 0) ++ctx->launch_count;  // the step
  ++L.substep;
  L.cur = 1 - L.cur;
  if (rec) L.rec_cur = next_cur;
  // the finite-difference domain boundary pass on the new state
  if (int rc = fd_after_step<T>(ctx, L)) return rc;
  // the save rows other ranks' coupler items read, and those this rank's read
  return exchange_rows(ctx, L);
}

template <typename T>
int do_advance_level(octlb_ctx* ctx, int l) {
  Level& L = ctx->levels[l];
  int rc = launch_level_step<T>(ctx, L);
  if (rc) return rc;
  ++ctx->counters_collide[l];
  ++ctx->counters_stream[l];
  if (l >= ctx->max_level) return OCTLB_OK;
  Level& F = ctx->levels[l + 1];
  // Recording: the half-time prolongation copies the prev-macro rows it
  // reads into the step record (its adjoint needs them).
  float* rec_prev = nullptr;
  if (ctx->adj && ctx->adj->recording && L.n_prolong > 0)
    rec_prev = ctx->adj->recs[ctx->adj->last_rec[l]].prev.as<float>();
  // apply_half_time(l) -> advance(l+1) -> apply_full_time(l) -> advance(l+1)
  // -> restrict(l+1)  (time_loop.h:228-239)
  // A restriction is not launched where the recursion reaches it: it shares
  // the next coupler launch (the parent's full-time prolongation, or another
  // restriction), and is launched before the next step otherwise -- nothing
  // in between reads what it writes.
  auto& pend = ctx->pending_restrict;
  for (int phase = 0; phase < 2; ++phase) {
    if (L.n_prolong > 0) {
      ProlongOp p{};
      p.items = L.prolong_items.as<ProlongItem>();
      p.n = L.n_prolong;
      p.half = phase == 0 ? 1 : 0;
      p.coarse_save = save_ptr(L);
      p.prev = L.prev.as<float>();
      p.rec_prev = phase == 0 ? rec_prev : nullptr;
      p.fine = cur_buf(F);
      p.fine_qs = F.nslots;
      p.scale = ctx->pscale_l[l];
      p.omega = static_cast<float>(ctx->omega_l[l + 1]);  // the written fine cell collides with its level's rate
      p.fscale = F.scale;
      if (ctx->cr_multi) {
        // ConstRhoBGK: the target takes the collide the reference's next
        // collide_level(l + 1) gives it, at the average now in effect (no
        // finest step runs in between).  On the finest level the step's
        // collide of the cell is replaced and the statistic is this one; on
        // a level above it, the level's own collide pass has already run.
        p.cmode = kCollConstRho;
        p.cr_avg = ctx->cr_avg.as<double>();
        if (l + 1 == ctx->cr_level) p.cr_part = ctx->cr_part.as<double>() + ctx->cr_nparts;
      }
      bool share = pend.size() <= 2;
      for (const auto& q : pend)
        if (q.level == l + 1 && !F.fuse_restrict) share = false;
      if (!share) { rc = flush_restricts<T>(ctx); if (rc) return rc; }
      RestrictOp r0{}, r1{};
      if (!pend.empty()) r0 = pend[0].op;
      if (pend.size() > 1) r1 = pend[1].op;
      pend.clear();
      CK(launch_couple<T>(p, r0, r1, ctx->stream));
      ++ctx->launch_count;
    }
    rc = do_advance_level<T>(ctx, l + 1);
    if (rc) return rc;
  }
  if (F.n_restrict > 0) {
    if (pend.size() >= 2) { rc = flush_restricts<T>(ctx); if (rc) return rc; }
    RestrictOp r{};
    r.items = F.restrict_items.as<RestrictItem>();
    r.n = F.n_restrict;
    r.fine_save = save_ptr(F);
    r.coarse = cur_buf(L);
    r.coarse_qs = L.nslots;
    r.scale = ctx->rscale_l[l];
    r.omega = static_cast<float>(ctx->omega_l[l]);
    r.cscale = L.scale;
    r.cmode = ctx->cr_multi ? kCollNone : kCollBgk;  // under ConstRhoBGK the level collides below
    pend.push_back({r, l});
  }
  if (ctx->cr_multi && L.nblk > 0) {
    // ConstRhoBGK on a multi-level mesh: this level's collide (the
    // reference's next collide_level(l), time_loop.h:201-205), after the
    // restriction wrote its targets
    rc = flush_restricts<T>(ctx);
    if (rc) return rc;
    StepArgs a = L.args;
    a.dst = cur_buf(L);
    CK(launch_collide_cr<T>(a, ctx->cr_shift.as<float>() + L.lvl, ctx->stream));
    ++ctx->launch_count;
  }
  return OCTLB_OK;
}

int validate(octlb_ctx* ctx, const octlb_tables* t, const octlb_params* p) {
  if (!t || !p) return fail(ctx, OCTLB_EINVAL, "null tables or params");
  if (t->n < 2) return fail(ctx, OCTLB_EINVAL, "block edge n must be >= 2");
  // 2:1 coupling pairs n / 2 coarse face cells with each fine block's
  // (level_coupler.cpp:70-139): an odd n serves single-level meshes (the
  // reference's cavity3d runs one 31^3 block)
  if (t->n % 2 != 0 && (t->n < 3 || t->n_coarse_fine > 0))
    return fail(ctx, OCTLB_EINVAL, "odd block edge n: n >= 3 and a mesh without coarse-fine faces only");
  if (t->n_blocks < 1 || !t->levels || !t->kinds) return fail(ctx, OCTLB_EINVAL, "no blocks / levels / kinds");
  if (p->precision != OCTLB_FP32 && p->precision != OCTLB_FP16_SHIFTED)
    return fail(ctx, OCTLB_EINVAL, "unknown precision");
  if (p->stream_mode != OCTLB_STREAM_ROTATE && p->stream_mode != OCTLB_STREAM_LINKS)
    return fail(ctx, OCTLB_EINVAL, "unknown stream mode");
  if (!(p->omega > 0.0 && p->omega < 2.0)) return fail(ctx, OCTLB_EINVAL, "omega must lie in (0, 2)");
  if (p->coupler_mode != OCTLB_COUPLER_REFERENCE && p->coupler_mode != OCTLB_COUPLER_PHYSICAL)
    return fail(ctx, OCTLB_EINVAL, "unknown coupler mode");
  if (p->stream_order != OCTLB_ORDER_AB && p->stream_order != OCTLB_ORDER_AA)
    return fail(ctx, OCTLB_EINVAL, "unknown stream order");
  if (p->stream_order == OCTLB_ORDER_AA && (!t->periodic || p->drag))
    return fail(ctx, OCTLB_EINVAL, "AA stream order needs a uniform periodic box without drag");
  for (int l = 0; l < 32 && p->coupler_mode == OCTLB_COUPLER_PHYSICAL; ++l)
    if (p->omega_level[l] != 0.0 && !(p->omega_level[l] > 0.0 && p->omega_level[l] < 2.0))
      return fail(ctx, OCTLB_EINVAL, "omega_level must be 0 or lie in (0, 2)");
  for (int b = 0; b < t->n_blocks; ++b)
    if (t->levels[b] < 0 || t->levels[b] > 30) return fail(ctx, OCTLB_EINVAL, "block level out of range");
  const long long n3 = static_cast<long long>(t->n) * t->n * t->n;
  for (long long k = 0; k < n3 * t->n_blocks; ++k)
    if (t->kinds[k] > kOutflow) return fail(ctx, OCTLB_EINVAL, "BcKind out of range");
  if (t->periodic) {
    if (t->n_blocks != 1) return fail(ctx, OCTLB_EINVAL, "periodic mode needs exactly one block");
    if (p->stream_mode != OCTLB_STREAM_ROTATE)
      return fail(ctx, OCTLB_EINVAL, "periodic mode uses the rotate stream rule");
    if (t->n_same_level || t->n_coarse_fine || t->n_tree_boundary)
      return fail(ctx, OCTLB_EINVAL, "periodic mode takes no face lists");
  }
  for (int k = 0; k < t->n_same_level; ++k) {
    const int* r = t->same_level + 3 * k;
    if (r[0] < 0 || r[0] >= t->n_blocks || r[2] < 0 || r[2] >= t->n_blocks || r[1] < 0 || r[1] > 5)
      return fail(ctx, OCTLB_EINVAL, "same-level face entry out of range");
    if (t->levels[r[0]] != t->levels[r[2]]) return fail(ctx, OCTLB_EINVAL, "same-level face joins two levels");
  }
  for (int k = 0; k < t->n_coarse_fine; ++k) {
    const int* r = t->coarse_fine + 8 * k;
    if (r[0] < 0 || r[0] >= t->n_blocks || r[5] < 0 || r[5] > 5)
      return fail(ctx, OCTLB_EINVAL, "coarse-fine face entry out of range");
    for (int s = 0; s < 4; ++s)
      if (r[1 + s] < 0 || r[1 + s] >= t->n_blocks || t->levels[r[1 + s]] != t->levels[r[0]] + 1)
        return fail(ctx, OCTLB_EINVAL, "coarse-fine face: fine block must be one level finer");
    if (r[6] != t->levels[r[0]] || r[7] != r[6] + 1)
      return fail(ctx, OCTLB_EINVAL, "coarse-fine face levels disagree with the block levels");
  }
  for (int k = 0; k < t->n_tree_boundary; ++k) {
    const int* r = t->tree_boundary + 2 * k;
    if (r[0] < 0 || r[0] >= t->n_blocks || r[1] < 0 || r[1] > 5)
      return fail(ctx, OCTLB_EINVAL, "tree-boundary entry out of range");
    if (t->tree_boundary_spec) {
      const double ty = t->tree_boundary_spec[8 * k];
      if (ty != OCTLB_TB_NONE && ty != OCTLB_TB_WALL && ty != OCTLB_TB_OUTFLOW)
        return fail(ctx, OCTLB_EINVAL, "unknown tree-boundary condition");
    }
  }
  for (int k = 0; k < t->n_links; ++k) {
    const int* c = t->link_cells + 5 * k;
    if (c[0] < 0 || c[0] >= t->n_blocks || c[1] < 0 || c[2] < 0 || c[3] < 0 || c[1] >= t->n ||
        c[2] >= t->n || c[3] >= t->n || c[4] < 0 || c[4] >= kQ)
      return fail(ctx, OCTLB_EINVAL, "link cell out of range");
  }
  if (t->n_links && p->stream_mode != OCTLB_STREAM_LINKS)
    return fail(ctx, OCTLB_EINVAL, "Bouzidi links need the links stream rule");
  return OCTLB_OK;
}

template <typename T>
int create_impl(octlb_ctx* ctx, const octlb_tables* t, const octlb_params* p, const double* init) {
  const int n = t->n, nb = t->n_blocks;
  const long long n3 = static_cast<long long>(n) * n * n;
  const bool links = p->stream_mode == OCTLB_STREAM_LINKS;
  ctx->kinds.assign(t->kinds, t->kinds + n3 * nb);
  CK(ctx->dev_err.alloc(sizeof(int)));
  for (int b = 0; b < nb; ++b) ctx->max_level = std::max(ctx->max_level, t->levels[b]);
  const int nlev = ctx->max_level + 1;
  ctx->levels.resize(nlev);
  ctx->blk_level.resize(nb);
  ctx->blk_local.resize(nb);
  ctx->counters_collide.assign(nlev, 0);
  ctx->counters_stream.assign(nlev, 0);
  const double tau = 1.0 / p->omega;
  ctx->prolong_scale = static_cast<float>((tau - 0.25) / tau);   // level_coupler.cpp:226-228
  ctx->restrict_scale = static_cast<float>(tau / (tau - 0.25));
  // Per-level rates and coupler scales: the reference's global ones, or the
  // physical rescaling from the coarsest level with blocks.
  ctx->coupler_mode = p->coupler_mode;
  ctx->omega_l.assign(nlev, p->omega);
  ctx->pscale_l.assign(nlev, ctx->prolong_scale);
  ctx->rscale_l.assign(nlev, ctx->restrict_scale);
  if (p->coupler_mode == OCTLB_COUPLER_PHYSICAL) {
    int lmin = nlev;
    for (int b = 0; b < nb; ++b) lmin = std::min(lmin, t->levels[b]);
    std::vector<double> tl(nlev);
    for (int l = 0; l < nlev; ++l) {
      const double given = p->omega_level[l < 32 ? l : 31];
      tl[l] = given > 0.0 ? 1.0 / given : std::ldexp(tau - 0.5, l - lmin) + 0.5;
      ctx->omega_l[l] = 1.0 / tl[l];
    }
    for (int l = 0; l + 1 < nlev; ++l) {
      ctx->pscale_l[l] = static_cast<float>(tl[l + 1] / (2.0 * tl[l]));
      ctx->rscale_l[l] = static_cast<float>(2.0 * tl[l] / tl[l + 1]);
    }
  }
  for (int l = 0; l < nlev; ++l) ctx->levels[l].lvl = l;
  std::vector<int> face_nbr(static_cast<size_t>(nb) * 6, -1);
  for (int k = 0; k < t->n_same_level; ++k) {
    const int* r = t->same_level + 3 * k;
    face_nbr[static_cast<size_t>(r[0]) * 6 + r[1]] = r[2];
  }
  if (ctx->periodic)
    for (int d = 0; d < 6; ++d) face_nbr[d] = 0;  // fill_periodic_halo: the block is its own neighbour
  // Diagonal (edge) neighbour: two face steps in either order, the
  // composition GhostSchedule uses for its same-level edge exchange.
  auto edge_nbr = [&](int a, int d1, int d2) {
    int b = face_nbr[static_cast<size_t>(a) * 6 + d1];
    if (b >= 0 && face_nbr[static_cast<size_t>(b) * 6 + d2] >= 0) return face_nbr[static_cast<size_t>(b) * 6 + d2];
    b = face_nbr[static_cast<size_t>(a) * 6 + d2];
    if (b >= 0 && face_nbr[static_cast<size_t>(b) * 6 + d1] >= 0) return face_nbr[static_cast<size_t>(b) * 6 + d1];
    return -1;
  };
  // Same-level neighbour of global block gb in halo direction (ox, oy, oz):
  // itself (centre), the face neighbour, the composed edge neighbour, or -1
  // (corners: the exchange fills no corner ghosts, D3Q19 has no corner links).
  auto nbr_dir = [&](int gb, int ox, int oy, int oz) {
    const int o[3] = {ox, oy, oz};
    int dirs[3], nd = 0;
    for (int a = 0; a < 3; ++a)
      if (o[a]) dirs[nd++] = 2 * a + (o[a] > 0 ? 1 : 0);
    if (nd == 0) return gb;
    if (nd == 1) return face_nbr[static_cast<size_t>(gb) * 6 + dirs[0]];
    if (nd == 2) return edge_nbr(gb, dirs[0], dirs[1]);
    return -1;
  };
  // Owned blocks first (global order), then the mirror blocks: neighbours
  // (face or edge) of owned blocks that another rank owns.
  std::vector<char> mirror(static_cast<size_t>(nb), 0);
  for (int b = 0; b < nb; ++b) {
    ctx->blk_level[b] = t->levels[b];
    if (!ctx->owns(b)) continue;
    for (int d = 0; d < 27; ++d) {
      if (d == 13) continue;
      const int v = nbr_dir(b, d / 9 - 1, (d / 3) % 3 - 1, d % 3 - 1);
      if (v >= 0 && !ctx->owns(v)) mirror[v] = 1;
    }
  }
  std::fill(ctx->blk_local.begin(), ctx->blk_local.end(), -1);
  for (int b = 0; b < nb; ++b) {
    if (!ctx->owns(b)) continue;
    Level& L = ctx->levels[t->levels[b]];
    ctx->blk_local[b] = static_cast<int>(L.blocks.size());
    L.blocks.push_back(b);
  }
  for (auto& L : ctx->levels) L.nblk = static_cast<int>(L.blocks.size());
  for (int b = 0; b < nb; ++b) {
    if (!mirror[b]) continue;
    Level& L = ctx->levels[t->levels[b]];
    ctx->blk_local[b] = static_cast<int>(L.blocks.size());
    L.blocks.push_back(b);
  }
  // Equilibrium at rest when no initial state is given (block_lattice.cpp:272-285):
  // shifted populations f - w = 0, whose collision is 0 too, so the
  // zero-filled buffers already hold it and nothing is uploaded.

  // ---- per-level storage and flags
  for (int l = 0; l < nlev; ++l) {
    Level& L = ctx->levels[l];
    L.nmir = static_cast<int>(L.blocks.size()) - L.nblk;
    L.n = n;
    L.ncore = L.nblk * n3;
    L.core_end = static_cast<long long>(L.nblk + L.nmir) * n3;
    double sc = p->fp16_scale[l < 32 ? l : 31];
    if (!(sc > 0)) sc = 65536.0;
    L.scale = p->precision == OCTLB_FP16_SHIFTED ? static_cast<float>(sc) : 1.f;
    L.inv_scale = 1.f / L.scale;
    if (L.nblk == 0) continue;
    if (L.core_end >= (1LL << 31)) return fail(ctx, OCTLB_EINVAL, "level has more than 2^31 cells");
  }

  // Link records: q per direction (1 = half-way bounce-back) and the moving-wall
  // term per direction, for core cells with a cut link or a moving neighbour.
  std::map<long long, std::vector<float>> recs;  // global cell -> 38 floats
  auto rec_for = [&](long long gcell) -> std::vector<float>& {
    auto it = recs.find(gcell);
    if (it == recs.end()) {
      std::vector<float> r(38, 0.f);
      for (int i = 0; i < kQ; ++i) r[i] = 1.f;
      it = recs.emplace(gcell, std::move(r)).first;
    }
    return it->second;
  };
  if (links) {
    for (int k = 0; k < t->n_links; ++k) {
      const int* c = t->link_cells + 5 * k;
      const double q = t->link_q[k];
      // Reference thresholds (block_lattice.cpp:652, bouzidi_pull.h:11-16):
      // q outside (1e-10, 1-1e-10) or within 1e-14 of 0 / 1 is plain bounce-back.
      float qf = 1.f;
      if (q > 1.0e-10 && q < 1.0 - 1.0e-10 && q > 1.0e-14 && q < 1.0 - 1.0e-14) {
        qf = static_cast<float>(q);
        if (qf >= 1.f) qf = std::nextafter(1.f, 0.f);
        if (q >= 0.5 - 1.0e-14 && qf < 0.5f) qf = 0.5f;
      }
      rec_for(c[0] * n3 + (static_cast<long long>(c[1]) * n + c[2]) * n + c[3])[c[4]] = qf;
    }
    if (t->moving && t->wall_u) {
      for (int b = 0; b < nb; ++b)
        for (int x = 0; x < n; ++x)
          for (int y = 0; y < n; ++y)
            for (int z = 0; z < n; ++z) {
              const long long g = b * n3 + (static_cast<long long>(x) * n + y) * n + z;
              if (t->kinds[g] == kSolid) continue;
              for (int i = 1; i < kQ; ++i) {
                const int sx = x - cx(i), sy = y - cy(i), sz = z - cz(i);
                if (sx < 0 || sy < 0 || sz < 0 || sx >= n || sy >= n || sz >= n) continue;
                const long long s = b * n3 + (static_cast<long long>(sx) * n + sy) * n + sz;
                if ((t->kinds[s] != kSolid && t->kinds[s] != kBouzidi) || !t->moving[s]) continue;
                const double cu = cx(i) * t->wall_u[3 * s] + cy(i) * t->wall_u[3 * s + 1] +
                                  cz(i) * t->wall_u[3 * s + 2];
                if (cu == 0.0) continue;
                rec_for(g)[kQ + i] += static_cast<float>(6.0 * wd(i) * cu);
              }
            }
    }
  }
  // ---- coupler plan (reference order) and level ranges
  const std::vector<PlanPoint> plan = build_plan(t);
  {
    // LevelRangeBegin/End take min/max plan index per coarse level
    // (level_coupler.cpp:238-250); the flattened path requires the ranges not
    // to interleave, which holds when hanging faces are listed level by level.
    std::vector<int> lo(nlev, 1 << 30), hi(nlev, -1);
    for (size_t k = 0; k < plan.size(); ++k) {
      lo[plan[k].coarse_level] = std::min(lo[plan[k].coarse_level], static_cast<int>(k));
      hi[plan[k].coarse_level] = std::max(hi[plan[k].coarse_level], static_cast<int>(k));
    }
    for (size_t k = 0; k < plan.size(); ++k)
      for (int l = 0; l < nlev; ++l)
        if (l != plan[k].coarse_level && static_cast<int>(k) >= lo[l] && static_cast<int>(k) <= hi[l])
          return fail(ctx, OCTLB_EINVAL, "coarse-fine faces must be grouped by coarse level");
  }
  auto core_slot = [&](int gblk, int x, int y, int z) { return core_slot_of(n, ctx->blk_local[gblk], x, y, z); };
  auto gcell = [&](int gblk, int x, int y, int z) {
    return gblk * n3 + (static_cast<long long>(x) * n + y) * n + z;
  };
  auto owner_of = [&](long long g) { return ctx->owner.empty() ? ctx->rank : ctx->owner[g / n3]; };
  std::vector<float> prev(plan.size() * 23, 0.f);
  if (init)
    for (size_t k = 0; k < plan.size(); ++k)
      host_macro(init + gcell(plan[k].coarse_id, plan[k].ci, plan[k].cj, plan[k].ck) * kQ, &prev[k * 23]);
  // Coupler items of the whole forest, by global cell.  Prolongation writes a
  // fine cell per point and restriction a coarse cell per point from the fine
  // cell and its in-block D3Q19 neighbours; a later point writing the same
  // cell wins (plan order, level_coupler.cpp:440-477, 613-654).  An item runs
  // on the rank owning the cell it writes.
  struct PSrc { long long fine_g, coarse_g; int k; };
  struct RSrc { long long coarse_g, fine_g; int nnb; long long nb_g[18]; };
  std::vector<std::vector<PSrc>> pall(nlev);   // by coarse level
  std::vector<std::vector<RSrc>> rall(nlev);   // by fine level
  {
    std::vector<std::map<long long, size_t>> last(nlev), lastc(nlev);
    for (size_t k = 0; k < plan.size(); ++k) {
      last[plan[k].coarse_level][gcell(plan[k].fine_id, plan[k].fi, plan[k].fj, plan[k].fk)] = k;
      lastc[plan[k].fine_level][gcell(plan[k].coarse_id, plan[k].ci, plan[k].cj, plan[k].ck)] = k;
    }
    for (size_t k = 0; k < plan.size(); ++k) {
      const PlanPoint& pt = plan[k];
      const long long fg = gcell(pt.fine_id, pt.fi, pt.fj, pt.fk), cg = gcell(pt.coarse_id, pt.ci, pt.cj, pt.ck);
      if (last[pt.coarse_level][fg] == k) pall[pt.coarse_level].push_back({fg, cg, static_cast<int>(k)});
      if (lastc[pt.fine_level][cg] == k) {
        RSrc r{cg, fg, 0, {}};
        for (int j = 1; j < kQ; ++j) {
          const int x = pt.fi + cx(j), y = pt.fj + cy(j), z = pt.fk + cz(j);
          if (x < 0 || y < 0 || z < 0 || x >= n || y >= n || z >= n) continue;
          r.nb_g[r.nnb++] = gcell(pt.fine_id, x, y, z);
        }
        rall[pt.fine_level].push_back(r);
      }
    }
  }
  for (int l = 0; l < nlev; ++l) {
    for (const PSrc& it : pall[l])
      if (t->kinds[it.fine_g] != kBulk || t->kinds[it.coarse_g] != kBulk) ctx->cpl_cells_bulk = false;
    for (const RSrc& it : rall[l]) {
      if (t->kinds[it.fine_g] != kBulk || t->kinds[it.coarse_g] != kBulk) ctx->cpl_cells_bulk = false;
      for (int j = 0; j < it.nnb; ++j)
        if (t->kinds[it.nb_g[j]] != kBulk) ctx->cpl_cells_bulk = false;
    }
  }
  // Save rows per source level, keyed by global cell: first every owned cell
  // some item (on any rank) reads, sorted; then the cells of other ranks that
  // this rank's items read, grouped by owner rank and sorted -- each peer's
  // rows arrive as one contiguous run.  Rows of owned cells that a peer's
  // items read are sent to it after every step of the level.
  std::vector<std::map<long long, int>> save_rows(nlev);   // owned: local slot -> row
  std::vector<std::map<long long, int>> row_of(nlev);      // global cell -> row
  std::vector<int> n_save_all(nlev, 0);
  std::vector<std::map<int, std::vector<long long>>> row_send_g(nlev), row_recv_g(nlev);  // peer -> cells
  for (int l = 0; l < nlev; ++l) {
    std::set<long long> own;
    std::map<int, std::set<long long>> remote, send;
    auto use = [&](long long g, int exec) {
      const int o = owner_of(g);
      if (o == ctx->rank) {
        own.insert(g);
        if (exec != ctx->rank) send[exec].insert(g);
      } else if (exec == ctx->rank) {
        remote[o].insert(g);
      }
    };
    for (const PSrc& it : pall[l]) use(it.coarse_g, owner_of(it.fine_g));
    for (const RSrc& it : rall[l]) {
      const int exec = owner_of(it.coarse_g);
      use(it.fine_g, exec);
      for (int j = 0; j < it.nnb; ++j) use(it.nb_g[j], exec);
    }
    int r = 0;
    for (long long g : own) {
      row_of[l][g] = r;
      save_rows[l][core_slot(static_cast<int>(g / n3), 0, 0, 0) + g % n3] = r;
      ++r;
    }
    for (auto& [peer, cells] : remote) {
      for (long long g : cells) row_of[l][g] = r++;
      row_recv_g[l][peer].assign(cells.begin(), cells.end());
    }
    for (auto& [peer, cells] : send) row_send_g[l][peer].assign(cells.begin(), cells.end());
    n_save_all[l] = r;
    ctx->levels[l].n_save_own = static_cast<int>(own.size());
  }
  std::vector<std::vector<ProlongItem>> prolong(nlev);
  std::vector<std::vector<RestrictItem>> restrict_items(nlev);
  for (int l = 0; l < nlev; ++l) {
    for (const PSrc& ps : pall[l]) {
      if (owner_of(ps.fine_g) != ctx->rank) continue;
      const int fb = static_cast<int>(ps.fine_g / n3);
      ProlongItem it{};
      it.fine_slot = core_slot(fb, 0, 0, 0) + ps.fine_g % n3;
      it.coarse_save = row_of[l].at(ps.coarse_g);
      it.prev = ps.k;
      it.fine_kind = t->kinds[ps.fine_g];
      prolong[l].push_back(it);
    }
    for (const RSrc& rs : rall[l]) {
      if (owner_of(rs.coarse_g) != ctx->rank) continue;
      const int cb = static_cast<int>(rs.coarse_g / n3);
      RestrictItem it{};
      it.coarse_slot = core_slot(cb, 0, 0, 0) + rs.coarse_g % n3;
      it.coarse_kind = t->kinds[rs.coarse_g];
      it.fine_save = row_of[l].at(rs.fine_g);
      it.nnb = rs.nnb;
      for (int j = 0; j < rs.nnb; ++j) it.nb_save[j] = row_of[l].at(rs.nb_g[j]);
      restrict_items[l].push_back(it);
    }
  }

  // ---- per-level flags, links, neighbour bases, halo pages, boundary fills,
  //      drag items
  const int np = n + 2, np3 = np * np * np;
  // Velocity scale of the moving tree-boundary walls (the largest wall speed,
  // e.g. the inlet u_max): every wall velocity is taken proportional to it
  // for the adjoint's d/du_max.
  double wall_vscale = 0.0;
  for (int k = 0; k < t->n_tree_boundary && t->tree_boundary_spec; ++k) {
    const double* sp = t->tree_boundary_spec + 8 * k;
    if (static_cast<int>(sp[0]) == OCTLB_TB_WALL)
      wall_vscale = std::max(wall_vscale, std::sqrt(sp[1] * sp[1] + sp[2] * sp[2] + sp[3] * sp[3]));
  }
  ctx->wall_vscale = wall_vscale;
  std::vector<int> hmap(static_cast<size_t>(np3), -1), hpos;
  for (int X = 0; X < np; ++X)
    for (int Y = 0; Y < np; ++Y)
      for (int Z = 0; Z < np; ++Z) {
        const bool core = X >= 1 && Y >= 1 && Z >= 1 && X <= n && Y <= n && Z <= n;
        if (!core) {
          hmap[(X * np + Y) * np + Z] = static_cast<int>(hpos.size());
          hpos.push_back((X * np + Y) * np + Z);
        }
      }
  const int H = static_cast<int>(hpos.size());
  auto dir27 = [&](int X, int Y, int Z) {
    const int ox = X == 0 ? -1 : (X == n + 1 ? 1 : 0), oy = Y == 0 ? -1 : (Y == n + 1 ? 1 : 0),
              oz = Z == 0 ? -1 : (Z == n + 1 ? 1 : 0);
    return (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1);
  };
  for (int l = 0; l < nlev; ++l) {
    Level& L = ctx->levels[l];
    if (L.nblk == 0) {
      // No owned block on this level (rank contexts): only the save rows
      // received for this rank's coupler items and those items.
      L.n_save = n_save_all[l];
      CK(L.save_buf.alloc(static_cast<size_t>(L.n_save) * kQ * sizeof(float)));
      CK(upload(L.prolong_items, prolong[l]));
      CK(upload(L.restrict_items, restrict_items[l]));
      L.n_prolong = static_cast<int>(prolong[l].size());
      L.n_restrict = static_cast<int>(restrict_items[l].size());
      L.args = StepArgs{};
      L.args.save_buf = L.save_buf.as<float>();
      L.args.err = ctx->dev_err.as<int>();
      continue;
    }
    L.has_flags = !ctx->periodic || !save_rows[l].empty() || (l >= 1 && !prolong[l - 1].empty());
    if (ctx->periodic) {
      for (long long k = 0; k < n3; ++k) if (t->kinds[k] != kBulk) L.has_flags = true;
    }
    const long long ncore = L.ncore, core_end = L.core_end;
    std::vector<uint8_t> flags(static_cast<size_t>(ncore), 0);
    std::vector<int> lidx, sidx;
    std::vector<float> lrec;
    for (int lb = 0; lb < L.nblk; ++lb)
      std::memcpy(&flags[static_cast<size_t>(lb * n3)], t->kinds + static_cast<size_t>(L.blocks[lb]) * n3,
                  static_cast<size_t>(n3));
    L.n_bulk = std::count(flags.begin(), flags.end(), static_cast<uint8_t>(kBulk));
    for (const auto& kv : recs) {
      const int gb = static_cast<int>(kv.first / n3);
      if (ctx->blk_level[gb] != l || !ctx->owns(gb)) continue;
      const long long s = static_cast<long long>(ctx->blk_local[gb]) * n3 + kv.first % n3;
      if (lidx.empty()) lidx.assign(static_cast<size_t>(ncore), -1);
      lidx[s] = static_cast<int>(lrec.size() / 38);
      lrec.insert(lrec.end(), kv.second.begin(), kv.second.end());
      flags[s] |= kFlagLink;
    }
    L.n_links = static_cast<int>(lrec.size() / 38);
    if (links) {
      // kFlagNear: the cell's pull needs the link rule -- a link record, a
      // solid / Bouzidi source in the own core, or a reflecting kind with a
      // source in the halo (block_lattice.cpp:624-670).
      for (int lb = 0; lb < L.nblk; ++lb)
        for (int x = 0; x < n; ++x)
          for (int y = 0; y < n; ++y)
            for (int z = 0; z < n; ++z) {
              const long long sc = core_slot_of(n, lb, x, y, z);
              const int kind = flags[sc] & kKindMask;
              bool near = (flags[sc] & kFlagLink) != 0;
              for (int i = 1; i < kQ && !near; ++i) {
                const int sx = x - cx(i), sy = y - cy(i), sz = z - cz(i);
                const bool halo = sx < 0 || sy < 0 || sz < 0 || sx >= n || sy >= n || sz >= n;
                if (halo) {
                  near = reflects_on_pull(kind);
                } else {
                  const int sk = flags[core_slot_of(n, lb, sx, sy, sz)] & kKindMask;
                  near = sk == kSolid || sk == kBouzidi;
                }
              }
              if (near && kind != kSolid) flags[sc] |= kFlagNear;
            }
    }
    std::vector<int> near_cells;
    for (long long k = 0; k < ncore; ++k)
      if (flags[k] & kFlagNear) near_cells.push_back(static_cast<int>(k));
    L.n_near = static_cast<int>(near_cells.size());
    if (!save_rows[l].empty()) {
      sidx.assign(static_cast<size_t>(ncore), -1);
      for (const auto& kv : save_rows[l]) {
        sidx[kv.first] = kv.second;
        flags[kv.first] |= kFlagSave;
      }
    }
    if (l >= 1)
      for (const ProlongItem& it : prolong[l - 1]) flags[static_cast<size_t>(it.fine_slot)] |= kFlagProlong;
    L.n_save = n_save_all[l];

    // Same-level neighbour of each of the 27 halo directions (faces and edges
    // only: the exchange fills no corner ghosts), global ids, -1 for none.
    std::vector<int> nbr27(static_cast<size_t>(L.nblk) * 27, -1);
    for (int lb = 0; lb < L.nblk; ++lb)
      for (int d = 0; d < 27; ++d)
        nbr27[static_cast<size_t>(lb) * 27 + d] = nbr_dir(L.blocks[lb], d / 9 - 1, (d / 3) % 3 - 1, d % 3 - 1);

    // Tree-boundary fills (DomainBoundaryHandler::apply(), before the
    // exchange), in list order; a later write of the same halo population
    // wins.  Keyed by (block, padded position, population).
    struct BB { int lb, hlin, pop; long long src; int src_pop; float add, dadd; };
    std::map<std::tuple<int, int, int>, size_t> bbidx;
    std::vector<BB> bbl;
    auto put_bb = [&](int lb, int hlin, int pop, long long src, int src_pop, float add, float dadd) {
      const auto key = std::make_tuple(lb, hlin, pop);
      auto it = bbidx.find(key);
      if (it == bbidx.end()) { bbidx.emplace(key, bbl.size()); bbl.push_back({lb, hlin, pop, src, src_pop, add, dadd}); }
      else bbl[it->second] = {lb, hlin, pop, src, src_pop, add, dadd};
    };
    for (int k = 0; k < t->n_tree_boundary; ++k) {
      const int gb = t->tree_boundary[2 * k], dir = t->tree_boundary[2 * k + 1];
      if (ctx->blk_level[gb] != l || !t->tree_boundary_spec || !ctx->owns(gb)) continue;
      const double* sp = t->tree_boundary_spec + 8 * k;
      const int type = static_cast<int>(sp[0]);
      if (type == OCTLB_TB_NONE) continue;
      const int lb = ctx->blk_local[gb];
      const double* bd = t->bounds + 6 * gb;
      const double dx = (bd[3] - bd[0]) / n;
      const int ax = dir / 2, t0 = (ax + 1) % 3, t1 = (ax + 2) % 3;
      const bool is_max = (dir & 1) != 0;
      const int hl = is_max ? n + 1 : 0, nin = is_max ? -1 : 1;
      for (int a = 0; a < n + 2; ++a)
        for (int b2 = 0; b2 < n + 2; ++b2) {
          int h[3];
          h[ax] = hl; h[t0] = a; h[t1] = b2;
          const int hlin = (h[0] * np + h[1]) * np + h[2];
          if (type == OCTLB_TB_WALL) {
            double shape = 1.0;
            const int pax = static_cast<int>(sp[4]);
            if (pax >= 0) {
              const double pc = bd[pax] + (h[pax] - 1 + 0.5) * dx;
              const double tt = (pc - sp[5]) / (sp[6] - sp[5]);
              shape = (tt <= 0.0 || tt >= 1.0) ? 0.0 : 4.0 * tt * (1.0 - tt);
            }
            for (int i = 1; i < kQ; ++i) {
              const int ci[3] = {cx(i), cy(i), cz(i)};
              if (ci[ax] != nin) continue;
              const int xx = h[0] + ci[0], yy = h[1] + ci[1], zz = h[2] + ci[2];
              if (xx < 1 || yy < 1 || zz < 1 || xx > n || yy > n || zz > n) continue;
              const double cu = (ci[0] * sp[1] + ci[1] * sp[2] + ci[2] * sp[3]) * shape;
              put_bb(lb, hlin, i, core_slot_of(n, lb, xx - 1, yy - 1, zz - 1), opp(i),
                     static_cast<float>(6.0 * wd(i) * cu),
                     wall_vscale > 0.0 ? static_cast<float>(6.0 * wd(i) * cu / wall_vscale) : 0.f);
            }
          } else {  // outflow: copy the adjacent interior cell, tangentially clamped
            int src[3];
            src[ax] = hl + nin;
            src[t0] = std::min(std::max(a, 1), n);
            src[t1] = std::min(std::max(b2, 1), n);
            const long long ss = core_slot_of(n, lb, src[0] - 1, src[1] - 1, src[2] - 1);
            for (int i = 0; i < kQ; ++i) put_bb(lb, hlin, i, ss, i, 0.f, 0.f);
          }
        }
    }

    // Open blocks: a halo population some core read depends on is neither a
    // same-level neighbour cell nor rewritten by a boundary fill, so it carries
    // the reference's torus stream from step to step.
    std::vector<char> is_open(static_cast<size_t>(L.nblk), 0), needs_page(static_cast<size_t>(L.nblk), 0);
    for (const BB& op : bbl) needs_page[op.lb] = 1;
    if (!ctx->periodic) {
      auto covered = [&](int lb, int X, int Y, int Z, int pop) {
        const int d = dir27(X, Y, Z);
        if (nbr27[static_cast<size_t>(lb) * 27 + d] >= 0) return true;
        return bbidx.count(std::make_tuple(lb, (X * np + Y) * np + Z, pop)) > 0;
      };
      for (int lb = 0; lb < L.nblk; ++lb) {
        bool open = false;
        for (int x = 1; x <= n && !open; ++x)
          for (int y = 1; y <= n && !open; ++y)
            for (int z = 1; z <= n && !open; ++z) {
              if (x > 1 && y > 1 && z > 1 && x < n && y < n && z < n) continue;
              const long long s = core_slot_of(n, lb, x - 1, y - 1, z - 1);
              const int kind = flags[s] & kKindMask;
              for (int i = 1; i < kQ && !open; ++i) {
                const int hx = x - cx(i), hy = y - cy(i), hz = z - cz(i);
                const bool halo = hx < 1 || hy < 1 || hz < 1 || hx > n || hy > n || hz > n;
                if (halo) {
                  const bool reads = !links || !(kind == kSolid || reflects_on_pull(kind));
                  if (reads && !covered(lb, hx, hy, hz, i)) open = true;
                }
                if (links && (flags[s] & kFlagLink)) {
                  const int nx_ = x + cx(i), ny_ = y + cy(i), nz_ = z + cz(i);
                  const bool nhalo = nx_ < 1 || ny_ < 1 || nz_ < 1 || nx_ > n || ny_ > n || nz_ > n;
                  if (nhalo && !covered(lb, nx_, ny_, nz_, i)) open = true;
                }
              }
            }
        is_open[lb] = open;
        if (open) needs_page[lb] = 1;
      }
    }
    std::vector<int> page_of(static_cast<size_t>(L.nblk), -1), open_pages;
    for (int lb = 0; lb < L.nblk; ++lb)
      if (needs_page[lb]) page_of[lb] = L.n_pages++;
    // Torus-streamed halo populations of open blocks: the (slot, population)
    // pairs a core read needs, closed under "slot h's population i is pulled
    // from slot rot_i(h)" while the source is an uncovered own-halo slot
    // (block_lattice.cpp:565-577).  Items: page, block, halo index, population.
    std::vector<int> halo_items;
    if (!ctx->periodic) {
      auto covered = [&](int lb, int hlin, int pop) {
        const int X = hlin / (np * np), Y = (hlin / np) % np, Z = hlin % np;
        if (nbr27[static_cast<size_t>(lb) * 27 + dir27(X, Y, Z)] >= 0) return true;
        return bbidx.count(std::make_tuple(lb, hlin, pop)) > 0;
      };
      for (int lb = 0; lb < L.nblk; ++lb) {
        if (!is_open[lb]) continue;
        std::set<std::pair<int, int>> need;
        std::vector<std::pair<int, int>> work;
        auto add = [&](int hlin, int pop) {
          if (hmap[hlin] < 0 || covered(lb, hlin, pop)) return;
          if (need.insert({hlin, pop}).second) work.push_back({hlin, pop});
        };
        for (int x = 1; x <= n; ++x)
          for (int y = 1; y <= n; ++y)
            for (int z = 1; z <= n; ++z) {
              if (x > 1 && y > 1 && z > 1 && x < n && y < n && z < n) continue;
              const long long sc = core_slot_of(n, lb, x - 1, y - 1, z - 1);
              const int kind = flags[sc] & kKindMask;
              for (int i = 1; i < kQ; ++i) {
                const bool reads = !links || !(kind == kSolid || reflects_on_pull(kind));
                if (reads) add(((x - cx(i)) * np + (y - cy(i))) * np + (z - cz(i)), i);
                if (links && (flags[sc] & kFlagLink)) add(((x + cx(i)) * np + (y + cy(i))) * np + (z + cz(i)), i);
              }
            }
        while (!work.empty()) {
          const auto [hlin, pop] = work.back();
          work.pop_back();
          int src = hlin - (cx(pop) * np * np + cy(pop) * np + cz(pop));
          src = ((src % np3) + np3) % np3;
          add(src, pop);
        }
        for (const auto& hp : need) {
          halo_items.push_back(page_of[lb]);
          halo_items.push_back(lb);
          halo_items.push_back(hmap[hp.first]);
          halo_items.push_back(hp.second);
        }
      }
    }
    open_pages = halo_items;
    L.n_open = static_cast<int>(halo_items.size() / 4);
    L.n_halo = L.n_pages > 0 ? H : 0;
    // even slot count: population rows start on 2-element boundaries
    L.nslots = core_end + static_cast<long long>(L.n_pages) * H;
    if (ctx->slab) L.nslots = core_end + 2LL * n * n;  // the two ghost x planes
    L.nslots += L.nslots & 1;
    std::vector<BBOp> bbv;
    for (const BB& op : bbl)
      bbv.push_back(BBOp{core_end + static_cast<long long>(page_of[op.lb]) * H + hmap[op.hlin], op.src, op.pop,
                         op.src_pop, op.add, op.dadd});
    L.n_bb = static_cast<uint32_t>(bbv.size());
    std::vector<int> fill_of_h(static_cast<size_t>(L.n_pages) * H * kQ, -1);
    for (size_t k = 0; k < bbv.size(); ++k)
      fill_of_h[static_cast<size_t>(bbv[k].dst - core_end) * kQ + bbv[k].pop] = static_cast<int>(k);

    // Slot bases of the 27 directions: own core (centre), the neighbour's core
    // shifted by one block edge, or the own halo page.
    std::vector<long long> nbase(static_cast<size_t>(L.nblk) * 27, kOwnPage);
    for (int lb = 0; lb < L.nblk; ++lb)
      for (int d = 0; d < 27; ++d) {
        const int v = nbr27[static_cast<size_t>(lb) * 27 + d];
        if (v < 0) continue;
        const int ox = d / 9 - 1, oy = (d / 3) % 3 - 1, oz = d % 3 - 1;
        const long long vl = ctx->blk_local[v];
        nbase[static_cast<size_t>(lb) * 27 + d] = (vl - ox) * n3 - static_cast<long long>(oy) * n * n - oz * n;
      }

    // Slot of every padded position of every block (the slot-map step's
    // table): own core, the neighbour core the same-level exchange copies,
    // or the own halo page.  Positions nothing resolves (the padded box's
    // corners, and halo positions of closed blocks no table covers) point at
    // the block's first core slot and must never be pulled: checked below
    // for every cell the step kernel streams.
    auto resolve_slot = [&](int lb, int X, int Y, int Z) -> long long {
      const int P = (X * np + Y) * np + Z;
      const long long lin = (static_cast<long long>(X - 1) * n + (Y - 1)) * n + (Z - 1);
      const int d = dir27(X, Y, Z);
      if (d == 13) return static_cast<long long>(lb) * n3 + lin;
      const long long b0 = nbase[static_cast<size_t>(lb) * 27 + d];
      if (b0 != kOwnPage) return b0 + lin;
      if (page_of[lb] >= 0) return core_end + static_cast<long long>(page_of[lb]) * H + hmap[P];
      return -1;
    };
    std::vector<int> slot_map;
    std::vector<float> wall_add, wall_dadd;  // per moving-wall position: the 19 wall terms, their velocity derivative
    if (map_step_eligible(n, L.nslots) && !(ctx->periodic && !L.has_flags)) {
      slot_map.assign(static_cast<size_t>(L.nblk) * np3, 0);
      std::vector<uint8_t> unresolved(static_cast<size_t>(np3));
      for (int lb = 0; lb < L.nblk; ++lb) {
        int* m = slot_map.data() + static_cast<size_t>(lb) * np3;
        for (int X = 0; X < np; ++X)
          for (int Y = 0; Y < np; ++Y)
            for (int Z = 0; Z < np; ++Z) {
              const int P = (X * np + Y) * np + Z;
              const long long sl = resolve_slot(lb, X, Y, Z);
              unresolved[P] = sl < 0;
              if (sl >= L.nslots) return fail(ctx, OCTLB_EINVAL, "internal: slot map out of range");
              m[P] = sl < 0 ? static_cast<int>(static_cast<long long>(lb) * n3) : static_cast<int>(sl);
              if (sl < core_end) continue;
              // A halo-page position whose pulled populations are boundary
              // fills: an outflow copy becomes its source cell's slot, a
              // bounce-back wall the marker -1 (at rest) or -(2 + k) (moving,
              // row k of the wall-term table); the pull then reads the
              // cell's own opposite population.
              int nfill = 0, npull = 0, ncopy = 0, nbb = 0;
              long long copy_src = -1;
              bool moving = false;
              for (int i = 1; i < kQ; ++i) {
                const int Xs = X + cx(i), Ys = Y + cy(i), Zs = Z + cz(i);
                if (Xs < 1 || Ys < 1 || Zs < 1 || Xs > n || Ys > n || Zs > n) continue;
                ++npull;
                const int fo = fill_of_h[static_cast<size_t>(sl - core_end) * kQ + i];
                if (fo < 0) continue;
                ++nfill;
                const BBOp& op = bbv[fo];
                if (op.src_pop == i) {
                  if (copy_src >= 0 && copy_src != op.src) return fail(ctx, OCTLB_EINVAL, "internal: mixed fill position");
                  copy_src = op.src;
                  ++ncopy;
                } else if (op.src_pop == opp(i) && op.src == core_slot_of(n, lb, Xs - 1, Ys - 1, Zs - 1)) {
                  ++nbb;
                  moving = moving || op.add != 0.f;
                } else {
                  return fail(ctx, OCTLB_EINVAL, "internal: unexpected fill source");
                }
              }
              if (nfill == 0) continue;
              if (nfill != npull || (ncopy > 0 && nbb > 0)) return fail(ctx, OCTLB_EINVAL, "internal: mixed fill position");
              if (ncopy > 0) {
                m[P] = static_cast<int>(copy_src);
              } else if (!moving) {
                m[P] = -1;
              } else {
                const int k = static_cast<int>(wall_add.size() / kQ);
                wall_add.resize(wall_add.size() + kQ, 0.f);
                wall_dadd.resize(wall_dadd.size() + kQ, 0.f);
                for (int i = 1; i < kQ; ++i) {
                  const int fo = fill_of_h[static_cast<size_t>(sl - core_end) * kQ + i];
                  if (fo < 0) continue;
                  wall_add[static_cast<size_t>(k) * kQ + i] = bbv[fo].add;
                  wall_dadd[static_cast<size_t>(k) * kQ + i] = bbv[fo].dadd;
                }
                m[P] = -(2 + k);
              }
            }
        for (int x = 0; x < n; ++x)
          for (int y = 0; y < n; ++y)
            for (int z = 0; z < n; ++z) {
              const uint8_t f = flags[static_cast<size_t>(core_slot_of(n, lb, x, y, z))];
              if (ctx->stream_mode == OCTLB_STREAM_LINKS && ((f & kKindMask) == kSolid || (f & kFlagNear))) continue;
              for (int i = 1; i < kQ; ++i)
                if (unresolved[((x + 1 - cx(i)) * np + (y + 1 - cy(i))) * np + (z + 1 - cz(i))])
                  return fail(ctx, OCTLB_EINVAL, "internal: pulled halo position without a source");
            }
      }
    }

    // Link rule of the near cells (block_lattice.cpp:613-672), resolved per
    // direction: pull source, reflect-on-pull at a reflecting kind's block
    // edge, half-way bounce-back or Bouzidi on a solid / Bouzidi source.
    std::vector<uint32_t> nmask(near_cells.size(), 0);
    std::vector<int> nslot(near_cells.size() * kQ);
    std::vector<float> nq(near_cells.size() * kQ, 1.f), nadd(near_cells.size() * kQ, -0.f);
    {
      const size_t nn = near_cells.size();
      for (size_t k = 0; k < nn; ++k) {
        const long long tc = near_cells[k];
        const int lb = static_cast<int>(tc / n3);
        const int r = static_cast<int>(tc % n3), x = r / (n * n), y = (r / n) % n, z = r % n;
        const int kind = flags[tc] & kKindMask;
        const int li = (flags[tc] & kFlagLink) ? lidx[tc] : -1;
        for (int i = 0; i < kQ; ++i) {
          const int X = x + 1 - cx(i), Y = y + 1 - cy(i), Z = z + 1 - cz(i);
          const bool halo = X < 1 || Y < 1 || Z < 1 || X > n || Y > n || Z > n;
          long long sl = resolve_slot(lb, X, Y, Z);
          if (sl < 0) return fail(ctx, OCTLB_EINVAL, "internal: pulled halo position without a source");
          const int sk = halo ? kBulk : (flags[sl] & kKindMask);
          if (i > 0 && reflects_on_pull(kind) && halo) {
            nmask[k] |= 1u << i;  // own[opp(i)], nothing added
          } else if (i > 0 && (sk == kSolid || sk == kBouzidi)) {
            nmask[k] |= 1u << i;
            if (li >= 0) {
              const float q = lrec[static_cast<size_t>(li) * 38 + i];
              nq[i * nn + k] = q;
              nadd[i * nn + k] = lrec[static_cast<size_t>(li) * 38 + kQ + i];
              if (q < 1.0f) {
                // f_q: population i of x + c_i when that cell is kBulk (a halo
                // position counts as kBulk), else the cell's own
                const int Xn = x + 1 + cx(i), Yn = y + 1 + cy(i), Zn = z + 1 + cz(i);
                const bool nh = Xn < 1 || Yn < 1 || Zn < 1 || Xn > n || Yn > n || Zn > n;
                const long long nbs = resolve_slot(lb, Xn, Yn, Zn);
                if (nbs < 0) return fail(ctx, OCTLB_EINVAL, "internal: Bouzidi neighbour without a source");
                const int nk = nh ? kBulk : (flags[nbs] & kKindMask);
                sl = nk == kBulk ? nbs : tc;
              }
            }
          }
          if (sl >= (1LL << 31)) return fail(ctx, OCTLB_EINVAL, "level has more than 2^31 slots");
          nslot[i * nn + k] = static_cast<int>(sl);
        }
      }
    }

    // Drag cells (drag_postprocessor.h:73-110).
    std::vector<DragItem> drag;
    if (ctx->drag) {
      for (int lb = 0; lb < L.nblk; ++lb) {
        const int gb = L.blocks[lb];
        for (int x = 0; x < n; ++x)
          for (int y = 0; y < n; ++y)
            for (int z = 0; z < n; ++z) {
              if (t->kinds[gcell(gb, x, y, z)] != kBulk) continue;
              uint32_t mask = 0;
              for (int i = 1; i < kQ; ++i) {
                const int xx = x + cx(i), yy = y + cy(i), zz = z + cz(i);
                if (xx < 0 || yy < 0 || zz < 0 || xx >= n || yy >= n || zz >= n) continue;
                const long long g = gcell(gb, xx, yy, zz);
                if (t->kinds[g] != kSolid && t->kinds[g] != kBouzidi) continue;
                if (t->obstacle && !t->obstacle[g]) continue;
                mask |= 1u << i;
              }
              if (!mask) continue;
              DragItem it{};
              it.slot = core_slot_of(n, lb, x, y, z);
              it.mask = mask;
              drag.push_back(it);
            }
      }
    }
    L.n_drag = static_cast<int>(drag.size());

    // Bounds of every index a kernel derives from these tables, checked on the
    // host before anything runs on the device.
    {
      const long long ns = L.nslots;
      auto in = [&](long long v, long long hi) { return v >= 0 && v < hi; };
      for (const BBOp& op : bbv)
        if (!in(op.dst, ns) || op.dst < core_end || !in(op.src, ncore) || !in(op.pop, kQ) || !in(op.src_pop, kQ))
          return fail(ctx, OCTLB_EINVAL, "internal: boundary fill out of range");
      for (int v : lidx) if (v < -1 || v >= L.n_links) return fail(ctx, OCTLB_EINVAL, "internal: link index");
      for (int v : sidx) if (v < -1 || v >= L.n_save) return fail(ctx, OCTLB_EINVAL, "internal: save index");
      for (size_t k = 0; k < open_pages.size(); k += 4)
        if (!in(open_pages[k], L.n_pages) || !in(open_pages[k + 1], L.nblk) || !in(open_pages[k + 2], H) ||
            !in(open_pages[k + 3], kQ))
          return fail(ctx, OCTLB_EINVAL, "internal: halo item");
      for (int lb = 0; lb < L.nblk; ++lb)
        for (int d = 0; d < 27; ++d) {
          const long long b0 = nbase[static_cast<size_t>(lb) * 27 + d];
          if (b0 == kOwnPage) continue;
          // extreme core-linear offsets of the halo region of direction d
          const int o[3] = {d / 9 - 1, (d / 3) % 3 - 1, d % 3 - 1};
          long long lo = 0, hi = 0;
          const long long w[3] = {static_cast<long long>(n) * n, n, 1};
          for (int a = 0; a < 3; ++a) {
            const long long cmin = o[a] < 0 ? -1 : (o[a] > 0 ? n : 0);
            const long long cmax = o[a] < 0 ? -1 : (o[a] > 0 ? n : n - 1);
            lo += cmin * w[a];
            hi += cmax * w[a];
          }
          if (!in(b0 + lo, core_end) || !in(b0 + hi, core_end))
            return fail(ctx, OCTLB_EINVAL, "internal: neighbour base out of range");
        }
      for (const DragItem& it : drag) if (!in(it.slot, ncore)) return fail(ctx, OCTLB_EINVAL, "internal: drag slot");
      for (const RestrictItem& it : restrict_items[l]) {
        if (!in(it.fine_save, L.n_save) || it.nnb < 0 || it.nnb > 18)
          return fail(ctx, OCTLB_EINVAL, "internal: restriction source");
        for (int k = 0; k < it.nnb; ++k)
          if (!in(it.nb_save[k], L.n_save)) return fail(ctx, OCTLB_EINVAL, "internal: restriction source");
      }
      if (static_cast<long long>(L.n_open) + ncore >= (1LL << 32))
        return fail(ctx, OCTLB_EINVAL, "level work exceeds 2^32 items");
      if (L.nslots * static_cast<long long>(kQ) >= (1LL << 40)) return fail(ctx, OCTLB_EINVAL, "level too large");
      if (!L.has_flags && (L.n_save > 0 || !ctx->periodic))
        return fail(ctx, OCTLB_EINVAL, "internal: flags required");
    }

    // allocations and uploads; AA order: one population buffer, the second
    // an alias of it (the step kernels update it in place)
    L.aa = ctx->stream_order == OCTLB_ORDER_AA;
    if (L.aa && !(ctx->periodic && !L.has_flags && L.nblk == 1 && n % 2 == 0 && !ctx->comm))
      return fail(ctx, OCTLB_EINVAL,
                  "AA stream order needs a uniform periodic box (one all-kBulk block, even n) in one context");
    CK(L.buf[0].alloc(static_cast<size_t>(L.nslots) * kQ * sizeof(T)));
    if (L.aa) L.buf[1].alias(L.buf[0]);
    else CK(L.buf[1].alloc(static_cast<size_t>(L.nslots) * kQ * sizeof(T)));
    if (L.has_flags) CK(upload(L.flags, flags));
    CK(upload(L.link_idx, lidx));
    CK(upload(L.link_rec, lrec));
    CK(upload(L.save_idx, sidx));
    CK(L.save_buf.alloc(static_cast<size_t>(L.n_save) * kQ * sizeof(float)));
    CK(upload(L.nbase, nbase));
    CK(upload(L.page_of, page_of));
    CK(upload(L.hmap, hmap));
    CK(upload(L.hpos, hpos));
    CK(upload(L.open_pages, open_pages));
    CK(upload(L.near_cells, near_cells));
    CK(upload(L.near_mask, nmask));
    CK(upload(L.near_slot, nslot));
    CK(upload(L.near_q, nq));
    CK(upload(L.near_add, nadd));
    L.near = NearTables{L.near_cells.as<int>(), L.near_mask.as<uint32_t>(), L.near_slot.as<int>(),
                        L.near_q.as<float>(), L.near_add.as<float>(), L.n_near};
    CK(upload(L.bb_ops, bbv));
    CK(upload(L.fill_of, fill_of_h));
    CK(upload(L.prolong_items, prolong[l]));
    CK(upload(L.restrict_items, restrict_items[l]));
    if (l >= 1 && l + 1 < nlev) {
      std::unordered_set<long long> ptarget;
      for (const ProlongItem& it : prolong[l - 1]) ptarget.insert(it.fine_slot);
      L.fuse_restrict = true;
      for (const RestrictItem& it : restrict_items[l + 1])
        if (ptarget.count(it.coarse_slot)) L.fuse_restrict = false;
    }
    L.n_prolong = static_cast<int>(prolong[l].size());
    L.n_restrict = static_cast<int>(restrict_items[l].size());
    CK(upload(L.drag_items, drag));
    if (L.n_drag > 0) {
      L.drag_off = ctx->drag_parts;
      ctx->drag_parts += static_cast<int>(drag_partials(L.n_drag));
    }

    StepArgs& A = L.args;
    A = StepArgs{};
    A.qs = L.nslots;
    A.flags = L.has_flags ? L.flags.as<uint8_t>() : nullptr;
    A.link_idx = L.link_idx.as<int>();
    A.link_rec = L.link_rec.as<float>();
    A.save_idx = L.save_idx.as<int>();
    A.save_buf = L.save_buf.as<float>();
    A.nbase = L.nbase.as<long long>();
    A.page_of = L.page_of.as<int>();
    A.hmap = L.hmap.as<int>();
    A.hpos = L.hpos.as<int>();
    A.open_pages = L.open_pages.as<int>();
    A.n_open = L.n_open;
    A.n_halo = L.n_halo;
    A.nblk = L.nblk; A.n = n; A.np = np;
    A.halo_base = core_end;
    A.ncore = static_cast<uint32_t>(ncore);
    A.nitems = A.ncore + static_cast<uint32_t>(L.n_open);
    A.div_n = FastDiv(n);
    A.div_n2 = FastDiv(n * n);
    A.div_n3 = FastDiv(static_cast<uint32_t>(n3));
    A.div_halo = FastDiv(L.n_halo > 0 ? L.n_halo : 1);
    A.div_np = FastDiv(np);
    A.div_np2 = FastDiv(np * np);
    A.omega = static_cast<float>(ctx->omega_l[l]);
    A.scale = L.scale;
    A.inv_scale = L.inv_scale;
    for (int i = 0; i < kQ; ++i) {
      A.off[i] = cx(i) * n * n + cy(i) * n + cz(i);
      A.off_pad[i] = cx(i) * np * np + cy(i) * np + cz(i);
    }
    A.err = ctx->dev_err.as<int>();
    A.wait_ns = ctx->wait_ns;
    A.stall_first_row = ctx->stall_first_row;
    A.fill_of = L.n_bb > 0 ? L.fill_of.as<int>() : nullptr;
    A.fills = L.bb_ops.as<BBOp>();
    // One all-kBulk periodic block: paired vector step by default, the
    // pipelined bulk-copy step on request (OCTLB_STEP_KERNEL=bulk), the plain
    // one-cell-per-thread step with OCTLB_STEP_KERNEL=plain.
    const bool uniform = ctx->periodic && !L.has_flags;
    if (uniform && ctx->step_kernel == 0 && pair_step_eligible(n)) L.use_pair = true;
    A.wrap_lo = ctx->slab ? n : n - 1;
    A.wrap_hi = ctx->slab ? n + 1 : 0;
    if (ctx->slab && !L.use_pair)
      return fail(ctx, OCTLB_EINVAL, "a periodic block shared over ranks needs the paired step (all kBulk, even n)");
    // Any other level: the slot-map step by default, the one-cell-per-thread
    // k_step with OCTLB_STEP_KERNEL=plain (or bulk, which only periodic
    // blocks take) or where the map does not fit.
    if (!uniform && ctx->step_kernel == 0 && map_step_eligible(n, L.nslots)) {
      L.use_map = true;
      CK(upload(L.slot_map, slot_map));
      CK(upload(L.wall_add, wall_add));
      CK(upload(L.wall_dadd, wall_dadd));
      std::vector<uint8_t> moving(static_cast<size_t>(L.nblk), 0);
      for (int lb = 0; lb < L.nblk; ++lb)
        for (int k = 0; k < np3 && !moving[lb]; ++k)
          if (slot_map[static_cast<size_t>(lb) * np3 + k] < -1) moving[lb] = 1;
      CK(upload(L.blk_moving, moving));
      A.blk_moving = L.blk_moving.as<uint8_t>();
      A.slot_map = L.slot_map.as<int>();
      A.wall_add = L.wall_add.as<float>();
      A.wall_dadd = L.wall_dadd.as<float>();
    }
    // FP16: the four-cell step fed by bulk async copies where its shape
    // fits (OCTLB_FP16_ROWS=off keeps k_step_quad_h; bitwise equal)
    if (L.use_pair && sizeof(T) == 2 && ctx->fp16_rows >= 0 &&
        rows_step_eligible(n, L.ncore, L.nslots, ctx->fp16_rows) && !g_dry_run) {
      const int per_sm = rows_prepare(ctx->fp16_rows, false);
      int dev = 0, sms = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      if (per_sm > 0) {
        L.use_rows = true;
        L.rows_grid = static_cast<int>(std::min<long long>(static_cast<long long>(per_sm) * sms,
                                                           L.ncore / rows_stage_cells(ctx->fp16_rows)));
      }
    }
    // AA order: the pull step fed and drained by bulk async copies where its
    // shape fits (OCTLB_AA_ROWS=off keeps the unstaged ones; bitwise equal)
    if (L.aa && ctx->aa_rows >= 0 && aa_rows_eligible(n, L.ncore, L.nslots, sizeof(T), ctx->aa_rows) &&
        !g_dry_run) {
      const int per_sm = aa_rows_prepare<T>(ctx->aa_rows);
      int dev = 0, sms = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      if (per_sm > 0) {
        L.use_aa_rows = true;
        L.aa_rows_grid = static_cast<int>(std::min<long long>(static_cast<long long>(per_sm) * sms,
                                                              L.ncore / aa_rows_stage_cells(ctx->aa_rows, sizeof(T))));
      }
    }
    // ... and its local step (from the reversed layout) staged as the AB step
    if (L.aa && sizeof(T) == 2 && ctx->fp16_rows >= 0 && rows_step_eligible(n, L.ncore, L.nslots, ctx->fp16_rows) &&
        !g_dry_run) {
      const int per_sm = rows_prepare(ctx->fp16_rows, true);
      int dev = 0, sms = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      if (per_sm > 0) {
        L.use_aa_local_rows = true;
        L.aa_local_grid = static_cast<int>(std::min<long long>(static_cast<long long>(per_sm) * sms,
                                                               L.ncore / rows_stage_cells(ctx->fp16_rows)));
      }
    }
    if (uniform && ctx->step_kernel == 1 && bulk_step_eligible(n, sizeof(T)) && !g_dry_run) {
      const int per_sm = bulk_prepare<T>(n);
      int dev = 0, sms = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      if (per_sm > 0) {
        L.use_bulk = true;
        L.bulk_grid = std::min(per_sm * sms, n * n);
      }
    }
  }
  // ---- cross-rank exchange tables (rank contexts).  For every pair of
  // same-level blocks b, m = neighbour of b in a face or edge direction with
  // different owners: the cells of m in b's halo region of that direction
  // travel from m's owner to b's owner before every step of the level (the
  // face layer of n^2 or the edge row of n cells, all 19 populations, as
  // GhostSchedule sends them).  Both ends list them in global cell order.
  if (!ctx->owner.empty()) {
    for (int l = 0; l < nlev; ++l) {
      Level& L = ctx->levels[l];
      std::map<int, std::vector<long long>> send_c, recv_c;
      for (int b = 0; b < nb; ++b) {
        if (t->levels[b] != l) continue;
        const int ob = ctx->owner[b];
        for (int d = 0; d < 27; ++d) {
          if (d == 13) continue;
          const int o[3] = {d / 9 - 1, (d / 3) % 3 - 1, d % 3 - 1};
          const int m = nbr_dir(b, o[0], o[1], o[2]);
          if (m < 0) continue;
          const int om = ctx->owner[m];
          const bool recv = ob == ctx->rank && om != ctx->rank, send = om == ctx->rank && ob != ctx->rank;
          if (!recv && !send) continue;
          std::vector<long long>& dst = recv ? recv_c[om] : send_c[ob];
          int lo[3], hi[3];
          for (int a = 0; a < 3; ++a) {
            lo[a] = o[a] < 0 ? n - 1 : 0;
            hi[a] = o[a] > 0 ? 0 : n - 1;
          }
          for (int x = lo[0]; x <= hi[0]; ++x)
            for (int y = lo[1]; y <= hi[1]; ++y)
              for (int z = lo[2]; z <= hi[2]; ++z) dst.push_back(gcell(m, x, y, z));
        }
      }
      auto record = [&](int kind, const std::map<int, std::vector<long long>>& by_peer) {
        if (!ctx->plan_lists) return;
        for (const auto& [peer, v] : by_peer)
          for (long long g : v) ctx->plan_lists->insert(ctx->plan_lists->end(), {l, kind, peer, g});
      };
      auto to_slots = [&](std::map<int, std::vector<long long>>& by_peer) {
        for (auto& [peer, v] : by_peer) {
          std::sort(v.begin(), v.end());
          v.erase(std::unique(v.begin(), v.end()), v.end());
          for (long long& g : v) g = core_slot(static_cast<int>(g / n3), 0, 0, 0) + g % n3;
        }
      };
      for (auto* m : {&send_c, &recv_c})
        for (auto& [peer, v] : *m) {
          std::sort(v.begin(), v.end());
          v.erase(std::unique(v.begin(), v.end()), v.end());
        }
      record(0, send_c);
      record(1, recv_c);
      record(2, row_send_g[l]);
      record(3, row_recv_g[l]);
      to_slots(send_c);
      to_slots(recv_c);
      const size_t cell_bytes = kQ * sizeof(T);
      if (int rc = setup_xfer(ctx, L.cell_send, send_c, cell_bytes, true)) return rc;
      if (int rc = setup_xfer(ctx, L.cell_recv, recv_c, cell_bytes, true)) return rc;
      // save rows: rows of owned cells out, runs of received rows in
      std::map<int, std::vector<long long>> rsend, rrecv;
      for (const auto& [peer, cells] : row_send_g[l])
        for (long long g : cells) rsend[peer].push_back(row_of[l].at(g));
      L.row_recv_first.clear();
      for (const auto& [peer, cells] : row_recv_g[l]) {
        for (long long g : cells) rrecv[peer].push_back(row_of[l].at(g));
        const std::vector<long long>& rows = rrecv[peer];
        for (size_t k = 1; k < rows.size(); ++k)
          if (rows[k] != rows[0] + static_cast<long long>(k))
            return fail(ctx, OCTLB_EINVAL, "internal: received save rows not contiguous");
        if (!rows.empty()) L.row_recv_first.push_back(rows[0]);
      }
      if (int rc = setup_xfer(ctx, L.row_send, rsend, kQ * sizeof(float), true)) return rc;
      if (int rc = setup_xfer(ctx, L.row_recv, rrecv, kQ * sizeof(float), false)) return rc;
      // every index the pack / unpack kernels derive
      for (const auto& [peer, v] : send_c)
        for (long long sl : v)
          if (sl < 0 || sl >= L.ncore) return fail(ctx, OCTLB_EINVAL, "internal: sent cell not owned");
      for (const auto& [peer, v] : recv_c)
        for (long long sl : v)
          if (sl < L.ncore || sl >= L.core_end) return fail(ctx, OCTLB_EINVAL, "internal: received cell not a mirror");
      for (const auto& [peer, v] : rsend)
        for (long long r : v)
          if (r < 0 || r >= L.n_save_own) return fail(ctx, OCTLB_EINVAL, "internal: sent save row");
      for (const auto& [peer, v] : rrecv)
        for (long long r : v)
          if (r < L.n_save_own || r >= L.n_save) return fail(ctx, OCTLB_EINVAL, "internal: received save row");
    }
  }

  // Cross-level coupler indices: prolongation targets live on level l+1,
  // restriction targets on level l-1.
  for (int l = 0; l < nlev; ++l) {
    for (const ProlongItem& it : prolong[l]) {
      if (l + 1 >= nlev || it.fine_slot < 0 || it.fine_slot >= ctx->levels[l + 1].nslots ||
          it.coarse_save < 0 || it.coarse_save >= ctx->levels[l].n_save || it.prev < 0 ||
          it.prev >= static_cast<int>(plan.size()))
        return fail(ctx, OCTLB_EINVAL, "internal: prolongation item out of range");
    }
    for (const RestrictItem& it : restrict_items[l]) {
      if (l < 1 || it.coarse_slot < 0 || it.coarse_slot >= ctx->levels[l - 1].nslots)
        return fail(ctx, OCTLB_EINVAL, "internal: restriction target out of range");
    }
  }
  // prev macros live with the coarse level
  for (int l = 0; l < nlev; ++l) {
    if (ctx->levels[l].n_prolong == 0) continue;
    CK(upload(ctx->levels[l].prev, prev));
  }
  CK(ctx->drag_partial.alloc(static_cast<size_t>(std::max(ctx->drag_parts, 1)) * 3 * sizeof(double)));
  CK(ctx->force.alloc(3 * sizeof(double)));
  CK(ctx->force_sum.alloc(3 * sizeof(double)));
  CK(ctx->audit_out.alloc(5 * sizeof(double)));

  // ---- initial state: g = C(f0) on kBulk cells
  for (int l = 0; l < nlev && !g_dry_run && init; ++l) {
    Level& L = ctx->levels[l];
    if (L.nblk == 0) continue;
    std::vector<double> dense(static_cast<size_t>(L.nblk * n3 * kQ));
    for (int lb = 0; lb < L.nblk; ++lb)
      std::memcpy(&dense[static_cast<size_t>(lb * n3 * kQ)], init + static_cast<size_t>(L.blocks[lb] * n3 * kQ),
                  sizeof(double) * n3 * kQ);
    DevBuf d;
    CK(upload(d, dense));
    StepArgs a = L.args;
    a.dst = L.buf[L.cur].p;
    CK(launch_scatter<T>(a, d.as<double>(), 0, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  long long lups = 0;
  for (int l = 0; l < nlev; ++l) lups += static_cast<long long>(ctx->levels[l].nblk) * n3 << l;
  ctx->lups_per_step = lups;
  return OCTLB_OK;
}

// Reads the device error word (after the stream has drained).
int check_device_error(octlb_ctx* ctx) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, ctx->dev_err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (h == kErrBulkTimeout)
    return fail(ctx, OCTLB_ETIMEOUT,
                "bulk-copy wait gave up after " + std::to_string(ctx->wait_ns / 1000000ull) + " ms");
  if (h == kErrBulkDrainTimeout) {
    ctx->unusable = true;
    return fail(ctx, OCTLB_ECUDA,
                "bulk-copy wait gave up and its copies in flight did not drain either: context unusable");
  }
  if (h != 0) return fail(ctx, OCTLB_ECUDA, "device error word set");
  return OCTLB_OK;
}

// One advance_one: the TimeLoop recursion from level 0, then the force total.
template <typename T>
int advance_one_launches(octlb_ctx* ctx) {
  for (auto& L : ctx->levels) L.substep = 0;
  ctx->launch_count = 0;
  int rc = do_advance_level<T>(ctx, 0);
  if (rc) return rc;
  rc = flush_restricts<T>(ctx);
  if (rc) return rc;
  if (ctx->side_busy) {
    CK(launch_drag_total(ctx->drag_partial.as<double>(), ctx->drag_parts, ctx->force.as<double>(),
                         ctx->force_sum.as<double>(), ctx->side));
    CK(cudaEventRecord(ctx->ev_join, ctx->side));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
    ctx->side_busy = false;
    ++ctx->launch_count;
  }
  if (int rc2 = fd_end_of_step(ctx)) return rc2;
  if (!(ctx->adj && ctx->adj->recording)) ctx->launches_per_step = ctx->launch_count;
  return OCTLB_OK;
}

uint64_t parity_mask(const octlb_ctx* ctx) {
  uint64_t m = 0;
  for (size_t l = 0; l < ctx->levels.size(); ++l)
    if (ctx->levels[l].cur) m |= 1ull << l;
  return m;
}

// Programmatic launches for the duration of one advance call on this thread.
struct ProgrammaticScope {
  explicit ProgrammaticScope(bool on) { set_programmatic_launch(on); }
  ~ProgrammaticScope() { set_programmatic_launch(false); }
};

template <typename T>
int advance_impl(octlb_ctx* ctx, int steps) {
  const ProgrammaticScope pdl(ctx->use_pdl);
  for (int s = 0; s < steps; ++s) {
    if (!ctx->use_graphs) {
      int rc = advance_one_launches<T>(ctx);
      if (rc) return rc;
    } else {
      const uint64_t mask = parity_mask(ctx);
      auto it = ctx->graphs.find(mask);
      if (it == ctx->graphs.end()) {
        // Capture this parity's advance_one (the host bookkeeping runs once
        // during capture), then launch it.
        const std::vector<int> c0 = ctx->counters_collide;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = advance_one_launches<T>(ctx);
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &g);
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (ee != cudaSuccess) return cuda_fail(ctx, ee, "cudaStreamEndCapture");
        octlb_ctx::GraphEntry e;
        const cudaError_t ei = cudaGraphInstantiate(&e.exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return cuda_fail(ctx, ei, "cudaGraphInstantiate");
        e.out_mask = parity_mask(ctx);
        e.dcollide.resize(ctx->counters_collide.size());
        for (size_t l = 0; l < e.dcollide.size(); ++l) e.dcollide[l] = ctx->counters_collide[l] - c0[l];
        it = ctx->graphs.emplace(mask, e).first;
        CK(cudaGraphLaunch(it->second.exec, ctx->stream));
      } else {
        CK(cudaGraphLaunch(it->second.exec, ctx->stream));
        for (size_t l = 0; l < ctx->levels.size(); ++l) ctx->levels[l].cur = (it->second.out_mask >> l) & 1;
        for (size_t l = 0; l < it->second.dcollide.size(); ++l) {
          ctx->counters_collide[l] += it->second.dcollide[l];
          ctx->counters_stream[l] += it->second.dcollide[l];
        }
      }
    }
    if (ctx->drag) ++ctx->force_steps;
  }
  return OCTLB_OK;
}

// ------------------------------------------------------------------ adjoint
// Discrete adjoint of n coarse steps (advance_one) by a reverse sweep with
// checkpoints every K coarse steps and recomputation in between: the forward
// pass stores the state at every checkpoint and evaluates the objective; then,
// segment by segment from the last, the forward is recomputed from the
// segment's checkpoint with every level step's input recorded, and the
// adjoint kernels run through those steps in reverse (TimeLoop::advance's
// recursion mirrored: restriction, second child, full-time prolongation,
// first child, half-time prolongation, then the level's own step).

int count_records(const octlb_ctx* ctx, int l) {
  int c = ctx->levels[l].nblk > 0 ? 1 : 0;
  if (l < ctx->max_level) c += 2 * count_records(ctx, l + 1);
  return c;
}

int adj_step(octlb_ctx* ctx, int l, const StepRecord& R, float coef) {
  Level& L = ctx->levels[l];
  AdjointState& A = *ctx->adj;
  AdjointState::Lv& V = A.lv[l];
  const bool links = ctx->stream_mode == OCTLB_STREAM_LINKS;
  StepArgs a = L.args;
  a.src = R.snap.p;
  a.dst = nullptr;
  a.slot_map = L.slot_map.as<int>();
  float* lamY = V.lam[V.cur].as<float>();
  float* lamX = V.lam[1 - V.cur].as<float>();
  double* g = A.g.as<double>();
  // lamX starts zeroed: the adjoint kernels clear every cotangent entry they
  // consume (lamY, the save rows, the coupler targets), so each buffer is
  // back to zero when it becomes the accumulator again.  The body-force
  // gradient of the state this step read is taken where its cotangent is
  // consumed (the previous step's k_adj_step, the coupler
  // kernels for their targets, and a final pass for the initial state).
  CK(launch_adj_step(a, L.near, links, L.has_flags, lamY, lamX, V.lam_save.as<float>(), g, V.gF.as<double>(),
                     ctx->stream));
  if (R.drag && coef != 0.f)
    CK(launch_adj_drag(a, links, L.drag_items.as<DragItem>(), L.n_drag, lamX, coef, A.comp, g, ctx->stream));
  V.cur = 1 - V.cur;
  return OCTLB_OK;
}

int adj_level(octlb_ctx* ctx, int l, size_t start, float coef) {
  Level& L = ctx->levels[l];
  AdjointState& A = *ctx->adj;
  const bool own = L.nblk > 0;
  const size_t c0 = start + (own ? 1 : 0);
  const float omega = static_cast<float>(ctx->omega);
  if (own && (start >= A.nrec || A.recs[start].level != l))
    return fail(ctx, OCTLB_ESTATE, "adjoint: step record out of order");
  if (l < ctx->max_level) {
    Level& F = ctx->levels[l + 1];
    const size_t cc = static_cast<size_t>(count_records(ctx, l + 1));
    const size_t s1 = c0, s2 = c0 + cc;
    AdjointState::Lv& V = A.lv[l];
    AdjointState::Lv& VF = A.lv[l + 1];
    double* g = A.g.as<double>();
    if (F.n_restrict > 0)
      CK(launch_adj_restrict(F.restrict_items.as<RestrictItem>(), F.n_restrict, A.recs[s2].save.as<float>(),
                             V.lam[V.cur].as<float>(), L.nslots, ctx->restrict_scale, omega,
                             VF.lam_save.as<float>(), g, V.gF.as<double>(), L.ncore, ctx->stream));
    int rc = adj_level(ctx, l + 1, s2, coef);
    if (rc) return rc;
    if (L.n_prolong > 0)
      CK(launch_adj_prolong(L.prolong_items.as<ProlongItem>(), L.n_prolong, A.recs[start].save.as<float>(),
                            A.recs[start].prev.as<float>(), 0, VF.lam[VF.cur].as<float>(), F.nslots,
                            ctx->prolong_scale, omega, V.lam_m.as<float>(), V.lam_prev.as<float>(),
                            V.lam_save.as<float>(), g, VF.gF.as<double>(), F.ncore, ctx->stream));
    rc = adj_level(ctx, l + 1, s1, coef);
    if (rc) return rc;
    if (L.n_prolong > 0) {
      CK(launch_adj_prolong(L.prolong_items.as<ProlongItem>(), L.n_prolong, A.recs[start].save.as<float>(),
                            A.recs[start].prev.as<float>(), 1, VF.lam[VF.cur].as<float>(), F.nslots,
                            ctx->prolong_scale, omega, V.lam_m.as<float>(), V.lam_prev.as<float>(),
                            V.lam_save.as<float>(), g, VF.gF.as<double>(), F.ncore, ctx->stream));
    }
  }
  if (own) return adj_step(ctx, l, A.recs[start], coef);
  return OCTLB_OK;
}

// Levels of the step records of one coarse step, in forward order.
void record_levels(const octlb_ctx* ctx, int l, std::vector<int>& out) {
  if (ctx->levels[l].nblk > 0) out.push_back(l);
  if (l < ctx->max_level) {
    record_levels(ctx, l + 1, out);
    record_levels(ctx, l + 1, out);
  }
}

// The record pool for `steps` coarse steps, allocated before any capture.
template <typename T>
int prealloc_records(octlb_ctx* ctx, int steps) {
  AdjointState& A = *ctx->adj;
  std::vector<int> seq;
  record_levels(ctx, 0, seq);
  const size_t need = seq.size() * static_cast<size_t>(steps);
  if (A.set_size != need) {  // the two sets' layout: set 1 = set 0 shifted by need
    A.recs.clear();
    A.recs.resize(2 * need);
    A.set_size = need;
  }
  A.next_same.assign(A.recs.size(), -1);
  A.first_rec.assign(ctx->levels.size(), -1);
  for (int set = 0; set < 2; ++set) {
    std::vector<int> last(ctx->levels.size(), -1);
    for (size_t r = 0; r < need; ++r) {
      const int l = seq[r % seq.size()];
      const int abs_r = static_cast<int>(set * need + r);
      if (last[l] >= 0) A.next_same[last[l]] = abs_r;
      else if (set == 0) A.first_rec[l] = abs_r;
      last[l] = abs_r;
    }
  }
  for (size_t r = 0; r < 2 * need; ++r) {
    StepRecord& R = A.recs[r];
    const int l = seq[r % seq.size()];
    if (R.level == l) continue;
    Level& L = ctx->levels[l];
    CK(R.snap.alloc(static_cast<size_t>(L.nslots) * kQ * sizeof(T)));
    CK(R.save.alloc(static_cast<size_t>(L.n_save) * kQ * sizeof(float)));
    CK(R.prev.alloc(L.n_prolong > 0 ? L.prev.bytes : 0));
    R.level = l;
  }
  return OCTLB_OK;
}

uint64_t lam_mask(const AdjointState& A) {
  uint64_t m = 0;
  for (size_t l = 0; l < A.lv.size(); ++l)
    if (A.lv[l].cur) m |= 1ull << l;
  return m;
}

// Runs body() on stream s (the context's stream is pointed at s meanwhile),
// through a CUDA graph captured on first use for `key` when graphs are
// enabled; set_out applies the captured run's final host-side parity to the
// context on replay.
template <typename Body, typename GetMask, typename SetMask>
int run_captured(octlb_ctx* ctx, const std::array<long long, 4>& key, Body body, GetMask get_mask,
                 SetMask set_mask, cudaStream_t s) {
  struct StreamSwap {
    octlb_ctx* c;
    cudaStream_t keep;
    ~StreamSwap() { c->stream = keep; }
  } swap_back{ctx, ctx->stream};
  ctx->stream = s;
  AdjointState& A = *ctx->adj;
  if (!ctx->use_graphs) return body();
  auto it = A.graphs.find(key);
  if (it == A.graphs.end()) {
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (ee != cudaSuccess) return cuda_fail(ctx, ee, "cudaStreamEndCapture");
    AdjointState::Graph e;
    const cudaError_t ei = cudaGraphInstantiate(&e.exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return cuda_fail(ctx, ei, "cudaGraphInstantiate");
    e.out_mask = get_mask();
    A.graphs.emplace(key, e);
    CK(cudaGraphLaunch(e.exec, ctx->stream));
    return OCTLB_OK;
  }
  CK(cudaGraphLaunch(it->second.exec, ctx->stream));
  set_mask(it->second.out_mask);
  return OCTLB_OK;
}

template <typename T>
int checkpoint_copy(octlb_ctx* ctx, AdjointState::Checkpoint& c, bool save) {
  const size_t nl = ctx->levels.size();
  if (save && c.buf.size() != nl) {
    c.buf.resize(nl);
    c.prev.resize(nl);
    c.cur.assign(nl, 0);
    for (size_t l = 0; l < nl; ++l) {
      Level& L = ctx->levels[l];
      CK(c.buf[l].alloc(static_cast<size_t>(L.nslots) * kQ * sizeof(T)));
      CK(c.prev[l].alloc(L.n_prolong > 0 ? L.prev.bytes : 0));
    }
  }
  for (size_t l = 0; l < nl; ++l) {
    Level& L = ctx->levels[l];
    if (L.nblk == 0) continue;
    if (save) {
      c.cur[l] = L.cur;
      CK(cudaMemcpyAsync(c.buf[l].p, L.buf[L.cur].p, c.buf[l].bytes, cudaMemcpyDeviceToDevice, ctx->stream));
      if (L.n_prolong > 0)
        CK(cudaMemcpyAsync(c.prev[l].p, L.prev.p, c.prev[l].bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
      L.cur = c.cur[l];
      CK(cudaMemcpyAsync(L.buf[L.cur].p, c.buf[l].p, c.buf[l].bytes, cudaMemcpyDeviceToDevice, ctx->stream));
      if (L.n_prolong > 0)
        CK(cudaMemcpyAsync(L.prev.p, c.prev[l].p, c.prev[l].bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    }
  }
  return OCTLB_OK;
}

template <typename T>
int adjoint_impl(octlb_ctx* ctx, const octlb_adj_params* p, double* objective, double* grad,
                 double* grad_force) {
  if (ctx->precision != OCTLB_FP32) return fail(ctx, OCTLB_EINVAL, "the adjoint differentiates FP32 storage only");
  if (!ctx->drag) return fail(ctx, OCTLB_ESTATE, "the adjoint's objective needs a context created with drag");
  const int NT = p->coarse_steps, W = p->window;
  if (NT < 1 || W < 1 || W > NT || p->component < 0 || p->component > 2 || p->checkpoint_interval < 0)
    return fail(ctx, OCTLB_EINVAL, "adjoint: need coarse_steps >= 1, 1 <= window <= coarse_steps, component 0..2");
  for (auto& L : ctx->levels)
    if (L.nblk > 0 && !L.slot_map.p)
      return fail(ctx, OCTLB_EINVAL, "adjoint: every level needs the slot-map layout (n a multiple of 8, <= 16)");
  const int K = p->checkpoint_interval > 0 ? p->checkpoint_interval
                                           : std::max(1, static_cast<int>(std::ceil(std::sqrt(static_cast<double>(NT)))));
  const int nck = (NT + K - 1) / K;
  if (!ctx->adj) ctx->adj = std::make_unique<AdjointState>();
  AdjointState& A = *ctx->adj;
  A.comp = p->component;
  const size_t nl = ctx->levels.size();
  if (A.lv.size() != nl) {
    A.lv.clear();
    A.lv.resize(nl);
    for (size_t l = 0; l < nl; ++l) {
      Level& L = ctx->levels[l];
      AdjointState::Lv& V = A.lv[l];
      for (int k = 0; k < 2; ++k) CK(V.lam[k].alloc(static_cast<size_t>(L.nslots) * kQ * sizeof(float)));
      CK(V.lam_save.alloc(static_cast<size_t>(L.n_save) * kQ * sizeof(float)));
      CK(V.lam_m.alloc(static_cast<size_t>(L.n_prolong) * 23 * sizeof(float)));
      CK(V.lam_prev.alloc(L.n_prolong > 0 ? L.prev.bytes : 0));
      CK(V.gF.alloc(static_cast<size_t>(3 * L.ncore) * sizeof(double)));
    }
    CK(A.g.alloc(kGradSlots * sizeof(double)));
  }
  if (A.ck.size() < static_cast<size_t>(nck + 1)) A.ck.resize(nck + 1);
  const std::vector<int> c0 = ctx->counters_collide, s0 = ctx->counters_stream;

  // Forward: checkpoints, objective over the window.
  for (int k = 0; k < NT; ++k) {
    if (k % K == 0) { int rc = checkpoint_copy<T>(ctx, A.ck[k / K], true); if (rc) return rc; }
    if (k == NT - W) {
      CK(cudaMemsetAsync(ctx->force_sum.p, 0, 3 * sizeof(double), ctx->stream));
      ctx->force_steps = 0;
    }
    int rc = advance_impl<T>(ctx, 1);
    if (rc) return rc;
  }
  double fs[3];
  CK(cudaMemcpyAsync(fs, ctx->force_sum.p, sizeof(fs), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (int rc = check_device_error(ctx)) return rc;
  const double J = fs[p->component] / W;
  const long long fsteps = ctx->force_steps;
  { int rc = checkpoint_copy<T>(ctx, A.ck[nck], true); if (rc) return rc; }
  DevBuf keep_force, keep_sum;
  CK(keep_force.alloc(3 * sizeof(double)));
  CK(keep_sum.alloc(3 * sizeof(double)));
  CK(cudaMemcpyAsync(keep_force.p, ctx->force.p, 3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(keep_sum.p, ctx->force_sum.p, 3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));

  // Reverse sweep.
  for (auto& V : A.lv) {
    for (int k = 0; k < 2; ++k) if (V.lam[k].p) CK(cudaMemsetAsync(V.lam[k].p, 0, V.lam[k].bytes, ctx->stream));
    if (V.lam_save.p) CK(cudaMemsetAsync(V.lam_save.p, 0, V.lam_save.bytes, ctx->stream));
    if (V.lam_m.p) CK(cudaMemsetAsync(V.lam_m.p, 0, V.lam_m.bytes, ctx->stream));
    if (V.lam_prev.p) CK(cudaMemsetAsync(V.lam_prev.p, 0, V.lam_prev.bytes, ctx->stream));
    if (V.gF.p) CK(cudaMemsetAsync(V.gF.p, 0, V.gF.bytes, ctx->stream));
    V.cur = 0;
  }
  CK(cudaMemsetAsync(A.g.p, 0, A.g.bytes, ctx->stream));
  const size_t per = static_cast<size_t>(count_records(ctx, 0));
  const float coef = static_cast<float>(1.0 / W);
  const std::array<long long, 4> gp{NT, W, K, p->component};
  if (gp != A.graph_params) {
    A.clear_graphs();
    A.graph_params = gp;
  }
  { int rc = prealloc_records<T>(ctx, K); if (rc) return rc; }
  const ProgrammaticScope pdl(ctx->use_pdl);
  auto set_parity = [&](uint64_t m) {
    for (size_t l = 0; l < nl; ++l) ctx->levels[l].cur = (m >> l) & 1;
  };
  auto set_lam = [&](uint64_t m) {
    for (size_t l = 0; l < nl; ++l) A.lv[l].cur = (m >> l) & 1;
  };
  // Segments from the last: segment c's recomputation fills record set c % 2
  // on rstream; its reverse reads that set on the context's stream while
  // segment c - 1 is recomputed into the other set.  Events order each
  // reverse after its recomputation and each recomputation after the reverse
  // that last read its set.
  if (!A.rstream) {
    CK(cudaStreamCreateWithFlags(&A.rstream, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&A.ev_fwd, &A.ev_rec[0], &A.ev_rec[1], &A.ev_rev[0], &A.ev_rev[1]})
      CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  CK(cudaEventRecord(A.ev_fwd, ctx->stream));
  CK(cudaStreamWaitEvent(A.rstream, A.ev_fwd, 0));
  bool rev_used[2] = {false, false};
  auto recompute = [&](int c) -> int {
    const int set = c & 1;
    const size_t base = static_cast<size_t>(set) * A.set_size;
    const int k0 = c * K, k1 = std::min(NT, k0 + K);
    if (rev_used[set]) CK(cudaStreamWaitEvent(A.rstream, A.ev_rev[set], 0));
    // the segment's checkpoint goes straight into each level's first record
    for (size_t l = 0; l < nl; ++l) {
      Level& L = ctx->levels[l];
      if (L.nblk == 0) continue;
      AdjointState::Checkpoint& ck = A.ck[c];
      L.cur = ck.cur[l];
      L.rec_cur = A.recs[base + A.first_rec[l]].snap.p;
      CK(cudaMemcpyAsync(L.rec_cur, ck.buf[l].p, ck.buf[l].bytes, cudaMemcpyDeviceToDevice, A.rstream));
      if (L.n_prolong > 0)
        CK(cudaMemcpyAsync(L.prev.p, ck.prev[l].p, ck.prev[l].bytes, cudaMemcpyDeviceToDevice, A.rstream));
    }
    // recompute the segment, recording every level step
    const int rc = run_captured(
        ctx, {2 * set, static_cast<long long>(parity_mask(ctx)), k1 - k0, 0},
        [&]() {
          A.recording = true;
          A.nrec = base;
          for (int k = k0; k < k1; ++k) {
            const int r = advance_one_launches<T>(ctx);
            if (r) { A.recording = false; return r; }
          }
          A.recording = false;
          if (A.nrec != base + per * static_cast<size_t>(k1 - k0))
            return fail(ctx, OCTLB_ESTATE, "adjoint: record count mismatch");
          return static_cast<int>(OCTLB_OK);
        },
        [&]() { return parity_mask(ctx); }, set_parity, A.rstream);
    for (auto& L : ctx->levels) L.rec_cur = L.rec_save = nullptr;
    if (rc) return rc;
    CK(cudaEventRecord(A.ev_rec[set], A.rstream));
    return OCTLB_OK;
  };
  auto reverse = [&](int c) -> int {
    const int set = c & 1;
    const size_t base = static_cast<size_t>(set) * A.set_size;
    const int k0 = c * K, k1 = std::min(NT, k0 + K);
    const int nwin = std::max(0, k1 - std::max(k0, NT - W));
    CK(cudaStreamWaitEvent(ctx->stream, A.ev_rec[set], 0));
    A.nrec = base + per * static_cast<size_t>(k1 - k0);
    const int rc = run_captured(
        ctx, {2 * set + 1, static_cast<long long>(lam_mask(A)), k1 - k0, nwin},
        [&]() {
          for (int k = k1 - 1; k >= k0; --k) {
            const int r = adj_level(ctx, 0, base + per * static_cast<size_t>(k - k0), k >= NT - W ? coef : 0.f);
            if (r) return r;
          }
          return static_cast<int>(OCTLB_OK);
        },
        [&]() { return lam_mask(A); }, set_lam, ctx->stream);
    if (rc) return rc;
    CK(cudaEventRecord(A.ev_rev[set], ctx->stream));
    rev_used[set] = true;
    return OCTLB_OK;
  };
  { const int rc = recompute(nck - 1); if (rc) return rc; }
  for (int c = nck - 1; c >= 0; --c) {
    if (c >= 1) { const int rc = recompute(c - 1); if (rc) return rc; }
    const int rc = reverse(c);
    if (rc) return rc;
  }

  // Body-force gradient of the initial state (consumed by no earlier step).
  for (size_t l = 0; l < nl; ++l) {
    Level& L = ctx->levels[l];
    if (L.nblk == 0) continue;
    CK(launch_adj_force(L.args, A.lv[l].lam[A.lv[l].cur].as<float>(), A.lv[l].gF.as<double>(), ctx->stream));
  }

  // Leave the context as the forward left it.
  { int rc = checkpoint_copy<T>(ctx, A.ck[nck], false); if (rc) return rc; }
  CK(cudaMemcpyAsync(ctx->force.p, keep_force.p, 3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->force_sum.p, keep_sum.p, 3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  ctx->force_steps = fsteps;
  ctx->counters_collide = c0;
  ctx->counters_stream = s0;
  for (size_t l = 0; l < nl; ++l) {
    ctx->counters_collide[l] += NT << l;
    ctx->counters_stream[l] += NT << l;
  }

  double gv[kGradSlots];
  CK(cudaMemcpyAsync(gv, A.g.p, sizeof(gv), cudaMemcpyDeviceToHost, ctx->stream));
  const long long n3 = static_cast<long long>(ctx->n) * ctx->n * ctx->n;
  std::vector<std::vector<double>> gF(nl);
  if (grad_force) {
    for (size_t l = 0; l < nl; ++l) {
      Level& L = ctx->levels[l];
      if (L.nblk == 0) continue;
      gF[l].resize(static_cast<size_t>(3 * L.ncore));
      CK(cudaMemcpyAsync(gF[l].data(), A.lv[l].gF.p, gF[l].size() * sizeof(double), cudaMemcpyDeviceToHost,
                         ctx->stream));
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  if (int rc = check_device_error(ctx)) return rc;
  const double tau = 1.0 / ctx->omega;
  // omega = 1/tau; prolongation scale (tau - 1/4)/tau; restriction scale
  // tau/(tau - 1/4) (level_coupler.cpp:226-228)
  const double dtau = gv[0] * (-1.0 / (tau * tau)) + gv[1] * (0.25 / (tau * tau)) +
                      gv[2] * (-0.25 / ((tau - 0.25) * (tau - 0.25)));
  if (objective) *objective = J;
  if (grad) {
    grad[0] = gv[3];
    grad[1] = dtau;
  }
  if (grad_force) {
    for (size_t l = 0; l < nl; ++l) {
      Level& L = ctx->levels[l];
      for (int lb = 0; lb < L.nblk; ++lb)
        for (long long c = 0; c < n3; ++c)
          for (int a = 0; a < 3; ++a)
            grad_force[(static_cast<size_t>(L.blocks[lb]) * n3 + c) * 3 + a] =
                gF[l][static_cast<size_t>(a * L.ncore + lb * n3 + c)];
    }
  }
  return OCTLB_OK;
}

void clear_graphs(octlb_ctx* ctx) {
  for (auto& kv : ctx->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  ctx->graphs.clear();
}

// Level-local block order equals a contiguous run of global ids: host
// arrays can be copied without reordering.
bool contiguous(const Level& L) {
  for (int k = 1; k < L.nblk; ++k)
    if (L.blocks[k] != L.blocks[0] + k) return false;
  return true;
}

template <typename T>
int gather_impl(octlb_ctx* ctx, double* pops, double* rho, double* u) {
  const long long n3 = static_cast<long long>(ctx->n) * ctx->n * ctx->n;
  for (auto& L : ctx->levels) {
    if (L.nblk == 0) continue;
    const long long cells = L.nblk * n3;
    const int mode = pops ? 0 : 1;
    DevBuf& d = ctx->stage_a;
    DevBuf& du = ctx->stage_b;
    const size_t bytes0 = static_cast<size_t>(cells * (mode == 0 ? kQ : 1)) * sizeof(double);
    const size_t bytes1 = static_cast<size_t>(cells * 3) * sizeof(double);
    CK(d.reserve(bytes0));
    if (mode == 1) CK(du.reserve(bytes1));
    StepArgs a = L.args;
    a.src = L.buf[L.cur].p;
    a.aa_rev = L.aa && L.cur;
    CK(launch_gather<T>(a, d.as<double>(), du.as<double>(), mode, ctx->stream));
    if (mode == 1)  // the FD pass's Dirichlet cells: the fields of their rewritten rows
      if (int rc = fd_fix_fields(ctx, L, d.as<double>(), du.as<double>())) return rc;
    const bool direct = contiguous(L);
    const long long off = static_cast<long long>(L.blocks[0]) * n3;
    std::vector<double> h0, h1;
    double* o0 = mode == 0 ? pops + off * kQ : rho + off;
    double* o1 = mode == 0 ? nullptr : u + off * 3;
    if (!direct) {
      h0.resize(static_cast<size_t>(cells * (mode == 0 ? kQ : 1)));
      o0 = h0.data();
      if (mode == 1) { h1.resize(static_cast<size_t>(cells * 3)); o1 = h1.data(); }
    }
    CK(cudaMemcpyAsync(o0, d.p, bytes0, cudaMemcpyDeviceToHost, ctx->stream));
    if (mode == 1) CK(cudaMemcpyAsync(o1, du.p, bytes1, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (!direct) {
      for (int lb = 0; lb < L.nblk; ++lb) {
        const long long g = static_cast<long long>(L.blocks[lb]) * n3, l0 = lb * n3;
        if (mode == 0) {
          std::memcpy(pops + g * kQ, &h0[static_cast<size_t>(l0 * kQ)], sizeof(double) * n3 * kQ);
        } else {
          std::memcpy(rho + g, &h0[static_cast<size_t>(l0)], sizeof(double) * n3);
          std::memcpy(u + g * 3, &h1[static_cast<size_t>(l0 * 3)], sizeof(double) * n3 * 3);
        }
      }
    }
  }
  return OCTLB_OK;
}

template <typename T>
int scatter_impl(octlb_ctx* ctx, const double* in) {
  const long long n3 = static_cast<long long>(ctx->n) * ctx->n * ctx->n;
  for (auto& L : ctx->levels) {
    if (L.nblk == 0) continue;
    const long long cells = L.nblk * n3;
    DevBuf& d = ctx->stage_a;
    const size_t bytes = static_cast<size_t>(cells * kQ) * sizeof(double);
    CK(d.reserve(bytes));
    if (contiguous(L)) {
      CK(cudaMemcpyAsync(d.p, in + static_cast<long long>(L.blocks[0]) * n3 * kQ, bytes,
                         cudaMemcpyHostToDevice, ctx->stream));
    } else {
      for (int lb = 0; lb < L.nblk; ++lb)
        CK(cudaMemcpyAsync(d.as<double>() + lb * n3 * kQ, in + static_cast<long long>(L.blocks[lb]) * n3 * kQ,
                           sizeof(double) * n3 * kQ, cudaMemcpyHostToDevice, ctx->stream));
    }
    StepArgs a = L.args;
    a.dst = L.buf[L.cur].p;
    CK(launch_scatter<T>(a, d.as<double>(), a.cr_part ? ctx->cr_near : 0, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (L.aa) L.cur = 0;  // the natural layout again
  }
  return OCTLB_OK;
}

// Equilibrium from per-cell rho [n_blocks][n^3] and u [n_blocks][n^3][3]:
// per level, the level's rows of both are staged as [rho | u] and
// k_scatter_eq forms, collides and stores the state.  One stream sync at
// the end (the staging buffer is reused per level, each level's copies are
// ordered after the previous level's kernel on the same stream).
template <typename T>
int scatter_eq_impl(octlb_ctx* ctx, const double* rho, const double* u) {
  const long long n3 = static_cast<long long>(ctx->n) * ctx->n * ctx->n;
  for (auto& L : ctx->levels) {
    if (L.nblk == 0) continue;
    const long long cells = L.nblk * n3;
    DevBuf& d = ctx->stage_a;
    CK(d.reserve(static_cast<size_t>(cells * 4) * sizeof(double)));
    double* dr = d.as<double>();
    double* du = dr + cells;
    if (contiguous(L)) {
      const long long b0 = static_cast<long long>(L.blocks[0]) * n3;
      CK(cudaMemcpyAsync(dr, rho + b0, sizeof(double) * cells, cudaMemcpyHostToDevice, ctx->stream));
      CK(cudaMemcpyAsync(du, u + 3 * b0, sizeof(double) * 3 * cells, cudaMemcpyHostToDevice, ctx->stream));
    } else {
      for (int lb = 0; lb < L.nblk; ++lb) {
        const long long b0 = static_cast<long long>(L.blocks[lb]) * n3;
        CK(cudaMemcpyAsync(dr + lb * n3, rho + b0, sizeof(double) * n3, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(du + 3 * lb * n3, u + 3 * b0, sizeof(double) * 3 * n3, cudaMemcpyHostToDevice,
                           ctx->stream));
      }
    }
    StepArgs a = L.args;
    a.dst = L.buf[L.cur].p;
    CK(launch_scatter_eq<T>(a, dr, a.cr_part ? ctx->cr_near : 0, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (L.aa) L.cur = 0;  // the natural layout again
  }
  return OCTLB_OK;
}

template <typename T>
int audit_impl(octlb_ctx* ctx, double out[4]) {
  double tot[5] = {0, 0, 0, 0, 0};
  for (auto& L : ctx->levels) {
    if (L.nblk == 0) continue;
    StepArgs a = L.args;
    a.src = L.buf[L.cur].p;
    a.aa_rev = L.aa && L.cur;
    DevBuf part;
    CK(part.alloc(audit_partials(a) * 5 * sizeof(double)));
    CK(launch_audit<T>(a, part.as<double>(), ctx->audit_out.as<double>(), ctx->stream));
    double h[5];
    CK(cudaMemcpyAsync(h, ctx->audit_out.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 5; ++k) tot[k] += h[k];
  }
  if (int rc = comm_allreduce(ctx, tot, 5)) return rc;  // rank contexts: the sum over ranks
  for (int k = 0; k < 4; ++k) out[k] = tot[k];
  if (tot[4] != 0.0) return fail(ctx, OCTLB_ENAN, "non-finite populations");
  return OCTLB_OK;
}

}  // namespace octlb_host

using namespace octlb_host;

// ====================================================================== C ABI
extern "C" {

static int create_common(const octlb_tables* t, const octlb_params* p, const double* init,
                         const octlb_partition* part, octlb_ctx** out) {
  if (!out) return OCTLB_EINVAL;
  *out = nullptr;
  auto ctx = std::make_unique<octlb_ctx>();
  int rc = validate(ctx.get(), t, p);
  if (rc) { *out = ctx.release(); return rc; }
  if (part) {
    if (part->nranks < 1 || part->rank < 0 || part->rank >= part->nranks || (!part->owner && !t->periodic) ||
        !part->comm) {
      *out = ctx.release();
      return fail(*out, OCTLB_EINVAL, "partition: rank, nranks, owner and comm are required");
    }
    if (comm_nranks(part->comm) != part->nranks) {
      *out = ctx.release();
      return fail(*out, OCTLB_EINVAL, "partition: the comm has another number of ranks");
    }
    for (int b = 0; b < t->n_blocks && !t->periodic; ++b)
      if (part->owner[b] < 0 || part->owner[b] >= part->nranks) {
        *out = ctx.release();
        return fail(*out, OCTLB_EINVAL, "partition: owner out of range");
      }
    // A periodic block: rank r owns x slab r (owner is not read); one rank
    // exchanges its ghost planes with itself.
    if (t->periodic) ctx->slab = true;
    ctx->rank = part->rank;
    ctx->nranks = part->nranks;
    if (!t->periodic) ctx->owner.assign(part->owner, part->owner + t->n_blocks);
    ctx->comm = part->comm;
  }
  ctx->n = t->n;
  ctx->n_blocks = t->n_blocks;
  if (t->bounds) ctx->bounds.assign(t->bounds, t->bounds + 6 * static_cast<size_t>(t->n_blocks));
  ctx->precision = p->precision;
  ctx->stream_mode = p->stream_mode;
  ctx->stream_order = p->stream_order;
  ctx->periodic = t->periodic;
  ctx->drag = p->drag;
  ctx->omega = p->omega;
  if (const char* ng = std::getenv("OCTLB_NO_GRAPH")) ctx->use_graphs = ng[0] != '1';
  if (const char* np = std::getenv("OCTLB_NO_PDL")) ctx->use_pdl = np[0] != '1';
  if (const char* sk = std::getenv("OCTLB_STEP_KERNEL")) {
    const std::string v(sk);
    ctx->step_kernel = v == "bulk" ? 1 : (v == "plain" ? 2 : 0);
  }
  ctx->map_cells = p->stream_mode == OCTLB_STREAM_LINKS ? 1 : 2;
  if (const char* mc = std::getenv("OCTLB_MAP_CELLS")) ctx->map_cells = mc[0] == '1' ? 1 : 2;
  if (const char* ms = std::getenv("OCTLB_MAP_SMEM")) ctx->map_global = ms[0] != '1';
  if (const char* wm = std::getenv("OCTLB_WAIT_MS")) {
    const long long ms = std::atoll(wm);
    if (ms >= 1 && ms <= 60000) ctx->wait_ns = static_cast<unsigned long long>(ms) * 1000000ull;
  }
  if (const char* st = std::getenv("OCTLB_TEST_BULK_STALL")) ctx->stall_first_row = st[0] == '1' ? 1 : 0;
  if (const char* fr = std::getenv("OCTLB_FP16_ROWS")) {
    const std::string v(fr);
    ctx->fp16_rows = v == "off" ? -1 : (v.size() == 1 && v[0] >= '0' && v[0] <= '7' ? v[0] - '0' : ctx->fp16_rows);
  }
  if (const char* ar = std::getenv("OCTLB_AA_ROWS")) {
    const std::string v(ar);
    ctx->aa_rows = v == "off" ? -1 : (v.size() == 1 && v[0] >= '0' && v[0] <= '2' ? v[0] - '0' : ctx->aa_rows);
  }
  // OCTLB_AA_PULL picks one of the unstaged pull steps (scalar, quad)
  if (const char* ap = std::getenv("OCTLB_AA_PULL")) ctx->aa_rows = ap[0] ? -1 : ctx->aa_rows;
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { rc = cuda_fail(ctx.get(), e, "cudaStreamCreate"); *out = ctx.release(); return rc; }
  ctx->own_stream = true;
  e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
  if (e != cudaSuccess) { rc = cuda_fail(ctx.get(), e, "side stream"); *out = ctx.release(); return rc; }
  if (ctx->comm) {
    // The exchanges sit between the launches of a level step and the local
    // transport meets the other ranks on the host: launched one by one, in
    // plain stream order.
    ctx->use_graphs = false;
    ctx->use_pdl = false;
    rc = comm_attach(ctx.get());
    if (rc) { *out = ctx.release(); return rc; }
  }
  rc = p->precision == OCTLB_FP32 ? create_impl<float>(ctx.get(), t, p, init)
                                  : create_impl<__half>(ctx.get(), t, p, init);
  *out = ctx.release();
  return rc;
}

int octlb_gpu_create(const octlb_tables* t, const octlb_params* p, const double* init, octlb_ctx** out) {
  return create_common(t, p, init, nullptr, out);
}

int octlb_gpu_create_part(const octlb_tables* t, const octlb_params* p, const double* init,
                          const octlb_partition* part, octlb_ctx** out) {
  if (!part) return OCTLB_EINVAL;
  return create_common(t, p, init, part, out);
}

void octlb_gpu_destroy(octlb_ctx* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  comm_detach(ctx);
  clear_graphs(ctx);
  cudaStream_t s = ctx->own_stream ? ctx->stream : nullptr;
  ctx->levels.clear();
  if (s) cudaStreamDestroy(s);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  delete ctx;
}

const char* octlb_gpu_last_error(const octlb_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int octlb_gpu_set_stream(octlb_ctx* ctx, void* s) {
  if (!ctx) return OCTLB_EINVAL;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  if (s) {
    ctx->stream = static_cast<cudaStream_t>(s);
    ctx->own_stream = false;
  } else {
    cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    ctx->own_stream = true;
  }
  return OCTLB_OK;
}

int octlb_gpu_advance(octlb_ctx* ctx, int steps) {
  if (!ctx || steps < 0) return OCTLB_EINVAL;
  if (ctx->levels.empty()) return fail(ctx, OCTLB_ESTATE, "context not initialised");
  if (ctx->unusable) return fail(ctx, OCTLB_ESTATE, "context unusable after a failed drain of a bounded wait");
  return ctx->precision == OCTLB_FP32 ? advance_impl<float>(ctx, steps) : advance_impl<__half>(ctx, steps);
}

int octlb_gpu_adjoint(octlb_ctx* ctx, const octlb_adj_params* p, double* objective, double* grad,
                      double* grad_force) {
  if (!ctx || !p) return OCTLB_EINVAL;
  if (ctx->levels.empty()) return fail(ctx, OCTLB_ESTATE, "context not initialised");
  if (ctx->unusable) return fail(ctx, OCTLB_ESTATE, "context unusable after a failed drain of a bounded wait");
  if (ctx->precision != OCTLB_FP32) return fail(ctx, OCTLB_EINVAL, "the adjoint differentiates FP32 storage only");
  if (ctx->comm) return fail(ctx, OCTLB_EINVAL, "the adjoint runs on one context, not rank contexts");
  if (ctx->coupler_mode != OCTLB_COUPLER_REFERENCE)
    return fail(ctx, OCTLB_EINVAL, "the adjoint differentiates the reference coupler mode (one global tau)");
  if (ctx->fd_on) return fail(ctx, OCTLB_EINVAL, "the adjoint does not differentiate the fd boundary pass");
  if (ctx->const_rho) return fail(ctx, OCTLB_EINVAL, "the adjoint differentiates the BGK collide, not ConstRhoBGK");
  if (ctx->stream_order != OCTLB_ORDER_AB) return fail(ctx, OCTLB_EINVAL, "the adjoint records two-buffer (AB) steps");
  return adjoint_impl<float>(ctx, p, objective, grad, grad_force);
}

int octlb_gpu_set_const_rho(octlb_ctx* ctx, int on) {
  if (!ctx) return OCTLB_EINVAL;
  if (ctx->levels.empty()) return fail(ctx, OCTLB_ESTATE, "context not initialised");
  if (ctx->comm && on) return fail(ctx, OCTLB_EINVAL, "ConstRhoBGK is built for one context, not rank contexts");
  if (ctx->stream_order != OCTLB_ORDER_AB && on)
    return fail(ctx, OCTLB_EINVAL, "ConstRhoBGK runs with the two-buffer (AB) stream order");
  if (ctx->fd_on && on)
    return fail(ctx, OCTLB_ESTATE, "ConstRhoBGK is chosen before octlb_gpu_set_fd_boundary");
  for (int c : ctx->counters_collide)
    if (c != 0) return fail(ctx, OCTLB_ESTATE, "ConstRhoBGK is chosen before the first advance");
  if ((on != 0) == ctx->const_rho) return OCTLB_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  clear_graphs(ctx);  // the captured launch sequence changes
  int lev = -1, used = 0;
  for (size_t l = 0; l < ctx->levels.size(); ++l)
    if (ctx->levels[l].nblk > 0) { lev = static_cast<int>(l); ++used; }
  if (!on) {
    for (auto& L : ctx->levels) {
      L.args.cr_avg = nullptr;
      L.args.cr_part = nullptr;
    }
    ctx->const_rho = ctx->cr_multi = false;
    ctx->cr_level = -1;
    ctx->cr_pparts = 0;
    return OCTLB_OK;
  }
  // The statistics are the finest level's (TimeLoop::advance collects them
  // when level >= max_level_, time_loop.h:201-222) and every level collides
  // at the average density.  The stored state is one collide ahead of the
  // reference's; a coarser level's collide needs the average of finest
  // steps that come after its step, so with more than one level the coarser
  // levels' steps only stream and each collides after its coupling
  // (do_advance_level).  On the finest level a prolongation's target takes
  // the collide and statistic the step gave it.
  Level& L = ctx->levels[lev];
  CK(upload(ctx->cr_avg, std::vector<double>{1.0}));  // TimeLoop starts at average_rho_ = 1
  CK(upload(ctx->cr_shift, std::vector<float>(ctx->levels.size(), 0.f)));  // BGK-collided: no shift
  const uint32_t core = cr_core_parts(L.args), near = cr_near_parts(L.near);
  ctx->cr_multi = used > 1;
  ctx->cr_nparts = static_cast<int>(core + near);
  ctx->cr_near = static_cast<int>(near);
  ctx->cr_pparts = ctx->cr_multi && lev >= 1 ? static_cast<int>(couple_prolong_ctas(ctx->levels[lev - 1].n_prolong)) : 0;
  ctx->cr_count = L.n_bulk;
  const size_t nparts = static_cast<size_t>(std::max(ctx->cr_nparts + ctx->cr_pparts, 1));
  CK(ctx->cr_part.alloc(nparts * sizeof(double)));
  CK(cudaMemsetAsync(ctx->cr_part.p, 0, nparts * sizeof(double), ctx->stream));
  for (auto& C : ctx->levels)
    if (C.nblk > 0) C.args.cr_avg = ctx->cr_avg.as<double>();  // every level collides at the average
  L.args.cr_part = ctx->cr_part.as<double>();
  L.args.cr_total = ctx->cr_nparts;
  // The stored state was collided by BGK, which is ConstRhoBGK at
  // average_rho = 1 and keeps each cell's density: its statistics are the
  // stored densities.
  StepArgs a = L.args;
  a.src = cur_buf(L);
  CK(ctx->precision == OCTLB_FP32 ? launch_cr_seed<float>(a, ctx->cr_near, ctx->stream)
                                  : launch_cr_seed<__half>(a, ctx->cr_near, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->const_rho = true;
  ctx->cr_level = lev;
  return OCTLB_OK;
}

int octlb_gpu_average_rho(octlb_ctx* ctx, double* out) {
  if (!ctx || !out) return OCTLB_EINVAL;
  if (!ctx->const_rho) {
    *out = 1.0;
    return OCTLB_OK;
  }
  CK(cudaMemcpyAsync(out, ctx->cr_avg.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return OCTLB_OK;
}

int octlb_gpu_synchronize(octlb_ctx* ctx) {
  if (!ctx) return OCTLB_EINVAL;
  if (int rc = comm_synchronize(ctx)) return rc;  // bounded for the NCCL transport
  return check_device_error(ctx);
}

int octlb_gpu_set_body_force(octlb_ctx* ctx, const double* force) {
  if (!ctx) return OCTLB_EINVAL;
  if (force && ctx->stream_order != OCTLB_ORDER_AB)
    return fail(ctx, OCTLB_EINVAL, "a body force needs the two-buffer (AB) stream order");
  CK(cudaStreamSynchronize(ctx->stream));
  clear_graphs(ctx);  // the captured launch sequence changes
  const long long n3 = static_cast<long long>(ctx->n) * ctx->n * ctx->n;
  for (auto& L : ctx->levels) {
    L.has_force = false;
    CK(L.body_force.alloc(0));
    if (!force || L.nblk == 0) continue;
    std::vector<float> f(static_cast<size_t>(3 * L.ncore));
    bool any = false;
    for (int lb = 0; lb < L.nblk; ++lb)
      for (long long c = 0; c < n3; ++c) {
        const double* g = force + (static_cast<size_t>(L.blocks[lb]) * n3 + c) * 3;
        if (!std::isfinite(g[0]) || !std::isfinite(g[1]) || !std::isfinite(g[2]))
          return fail(ctx, OCTLB_EINVAL, "non-finite body force");
        for (int a = 0; a < 3; ++a) {
          f[static_cast<size_t>(a * L.ncore + lb * n3 + c)] = static_cast<float>(g[a]);
          any = any || g[a] != 0.0;
        }
      }
    if (!any) continue;
    CK(upload(L.body_force, f));
    L.has_force = true;
  }
  return OCTLB_OK;
}

int octlb_gpu_set_populations(octlb_ctx* ctx, const double* pops) {
  if (!ctx || !pops) return OCTLB_EINVAL;
  return ctx->precision == OCTLB_FP32 ? scatter_impl<float>(ctx, pops) : scatter_impl<__half>(ctx, pops);
}

int octlb_gpu_set_equilibrium(octlb_ctx* ctx, const double* rho, const double* u) {
  if (!ctx || !rho || !u) return OCTLB_EINVAL;
  if (ctx->levels.empty()) return fail(ctx, OCTLB_ESTATE, "context not initialised");
  return ctx->precision == OCTLB_FP32 ? scatter_eq_impl<float>(ctx, rho, u) : scatter_eq_impl<__half>(ctx, rho, u);
}

int octlb_gpu_get_populations(octlb_ctx* ctx, double* pops) {
  if (!ctx || !pops) return OCTLB_EINVAL;
  if (int rc = check_device_error(ctx)) return rc;
  return ctx->precision == OCTLB_FP32 ? gather_impl<float>(ctx, pops, nullptr, nullptr)
                                      : gather_impl<__half>(ctx, pops, nullptr, nullptr);
}

int octlb_gpu_get_fields(octlb_ctx* ctx, double* rho, double* u) {
  if (!ctx || !rho || !u) return OCTLB_EINVAL;
  if (int rc = check_device_error(ctx)) return rc;
  return ctx->precision == OCTLB_FP32 ? gather_impl<float>(ctx, nullptr, rho, u)
                                      : gather_impl<__half>(ctx, nullptr, rho, u);
}

int octlb_gpu_write_vtk(octlb_ctx* ctx, const char* output_dir, const char* base_name, int step, int rank,
                        int fields, int write_index) {
  if (!ctx || !output_dir || !base_name || rank < 0) return OCTLB_EINVAL;
  if (fields <= 0 || (fields & ~(OCTLB_VTK_VELOCITY | OCTLB_VTK_DENSITY | OCTLB_VTK_PRESSURE)))
    return fail(ctx, OCTLB_EINVAL, "write_vtk: fields is a nonzero mask of OCTLB_VTK_*");
  if (ctx->bounds.size() != 6 * static_cast<size_t>(ctx->n_blocks))
    return fail(ctx, OCTLB_EINVAL, "write_vtk: the tables gave no block bounds");
  const int n = ctx->n;
  const long long n3 = static_cast<long long>(n) * n * n;
  std::vector<double> rho(static_cast<size_t>(ctx->n_blocks * n3)), u(rho.size() * 3);
  if (int rc = octlb_gpu_get_fields(ctx, rho.data(), u.data())) return rc;
  std::error_code ec;
  std::filesystem::create_directories(output_dir, ec);
  // AmrVtkWriter's names (amr_vtk_writer.cpp): base_r<rank>_oct<id>_T<step, 5 digits>.vts
  char tag[16];
  std::snprintf(tag, sizeof(tag), "%05d", step);
  std::vector<std::string> rel;
  std::vector<double> vel(static_cast<size_t>(n3) * 3), den(static_cast<size_t>(n3)), pre(static_cast<size_t>(n3));
  for (int b = 0; b < ctx->n_blocks; ++b) {
    if (!ctx->owns(b)) continue;  // rank contexts write their own blocks
    // cell (i, j, k) of the file (i fastest) is core cell (x, y, z) = (i, j, k)
    size_t c = 0;
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i, ++c) {
          const size_t s = static_cast<size_t>(b * n3 + (static_cast<long long>(i) * n + j) * n + k);
          for (int d = 0; d < 3; ++d) vel[3 * c + d] = u[3 * s + d];
          den[c] = rho[s];
          pre[c] = rho[s] * (1.0 / 3.0);  // p = rho c_s^2 (VtkPressureField)
        }
    const char* names[3];
    int comps[3];
    const double* data[3];
    int nf = 0;
    if (fields & OCTLB_VTK_VELOCITY) { names[nf] = "velocity"; comps[nf] = 3; data[nf++] = vel.data(); }
    if (fields & OCTLB_VTK_DENSITY) { names[nf] = "density"; comps[nf] = 1; data[nf++] = den.data(); }
    if (fields & OCTLB_VTK_PRESSURE) { names[nf] = "pressure"; comps[nf] = 1; data[nf++] = pre.data(); }
    const std::string name = std::string(base_name) + "_r" + std::to_string(rank) + "_oct" + std::to_string(b) +
                             "_T" + tag + ".vts";
    const int rc = octlb_vtk_write_block((std::string(output_dir) + "/" + name).c_str(), n, n, n,
                                         &ctx->bounds[6 * static_cast<size_t>(b)], nf, names, comps, data);
    if (rc) return fail(ctx, rc, "write_vtk: cannot write " + name);
    rel.push_back(name);
  }
  if (write_index) {
    std::vector<const char*> p;
    for (const std::string& r : rel) p.push_back(r.c_str());
    const int rc = octlb_vtk_write_index(output_dir, base_name, step, static_cast<int>(p.size()), p.data());
    if (rc) return fail(ctx, rc, "write_vtk: cannot write the .vtm / .pvd index");
  }
  return OCTLB_OK;
}

int octlb_gpu_force(octlb_ctx* ctx, double out[3]) {
  if (!ctx || !out) return OCTLB_EINVAL;
  if (!ctx->drag) return fail(ctx, OCTLB_ESTATE, "context created without drag");
  CK(cudaMemcpyAsync(out, ctx->force.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return comm_allreduce(ctx, out, 3);  // rank contexts: the sum over ranks
}

int octlb_gpu_force_sum(octlb_ctx* ctx, double out[3], long long* steps) {
  if (!ctx || !out) return OCTLB_EINVAL;
  if (!ctx->drag) return fail(ctx, OCTLB_ESTATE, "context created without drag");
  CK(cudaMemcpyAsync(out, ctx->force_sum.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (steps) *steps = ctx->force_steps;
  return comm_allreduce(ctx, out, 3);
}

int octlb_gpu_force_reset(octlb_ctx* ctx) {
  if (!ctx) return OCTLB_EINVAL;
  if (ctx->force_sum.p) CK(cudaMemsetAsync(ctx->force_sum.p, 0, 3 * sizeof(double), ctx->stream));
  ctx->force_steps = 0;
  return OCTLB_OK;
}

int octlb_gpu_audit(octlb_ctx* ctx, double out[4]) {
  if (!ctx || !out) return OCTLB_EINVAL;
  if (int rc = check_device_error(ctx)) return rc;
  return ctx->precision == OCTLB_FP32 ? audit_impl<float>(ctx, out) : audit_impl<__half>(ctx, out);
}

int octlb_gpu_counters(const octlb_ctx* ctx, int* collide, int* stream, int max_levels) {
  if (!ctx) return OCTLB_EINVAL;
  const int nl = static_cast<int>(ctx->counters_collide.size());
  for (int l = 0; l < nl && l < max_levels; ++l) {
    if (collide) collide[l] = ctx->counters_collide[l];
    if (stream) stream[l] = ctx->counters_stream[l];
  }
  return nl;
}

int octlb_gpu_max_level(const octlb_ctx* ctx) { return ctx ? ctx->max_level : OCTLB_EINVAL; }

int octlb_gpu_plan(const octlb_tables* t, const octlb_params* p, long long* stats, int max_stats) {
  octlb_ctx ctx;
  int rc = validate(&ctx, t, p);
  if (rc) return rc;
  ctx.n = t->n;
  ctx.n_blocks = t->n_blocks;
  ctx.precision = p->precision;
  ctx.stream_mode = p->stream_mode;
  ctx.periodic = t->periodic;
  ctx.drag = p->drag;
  ctx.omega = p->omega;
  g_dry_run = true;
  rc = p->precision == OCTLB_FP32 ? create_impl<float>(&ctx, t, p, nullptr)
                                  : create_impl<__half>(&ctx, t, p, nullptr);
  g_dry_run = false;
  if (rc) return rc;
  const int nl = static_cast<int>(ctx.levels.size());
  std::vector<long long> v;
  v.push_back(nl);
  for (const Level& L : ctx.levels) {
    const long long row[10] = {L.nblk, L.n_pages, L.n_open, L.n_bb, L.n_prolong, L.n_restrict,
                               L.n_save, L.n_links, L.n_drag, L.nslots};
    v.insert(v.end(), row, row + 10);
  }
  for (int k = 0; k < max_stats && k < static_cast<int>(v.size()); ++k) stats[k] = v[k];
  return static_cast<int>(v.size());
}

int octlb_gpu_plan_part(const octlb_tables* t, const octlb_params* p, int rank, int nranks, const int* owner,
                        long long* records, long long max_records) {
  if (!owner || nranks < 1 || rank < 0 || rank >= nranks) return OCTLB_EINVAL;
  octlb_ctx ctx;
  int rc = validate(&ctx, t, p);
  if (rc) return rc;
  for (int b = 0; b < t->n_blocks; ++b)
    if (owner[b] < 0 || owner[b] >= nranks) return OCTLB_EINVAL;
  if (t->periodic) return OCTLB_EINVAL;
  ctx.n = t->n;
  ctx.n_blocks = t->n_blocks;
  ctx.precision = p->precision;
  ctx.stream_mode = p->stream_mode;
  ctx.periodic = t->periodic;
  ctx.drag = p->drag;
  ctx.omega = p->omega;
  ctx.rank = rank;
  ctx.nranks = nranks;
  ctx.owner.assign(owner, owner + t->n_blocks);
  std::vector<long long> lists;
  ctx.plan_lists = &lists;
  g_dry_run = true;
  rc = p->precision == OCTLB_FP32 ? create_impl<float>(&ctx, t, p, nullptr)
                                  : create_impl<__half>(&ctx, t, p, nullptr);
  g_dry_run = false;
  if (rc) return rc;
  const long long nrec = static_cast<long long>(lists.size() / 4);
  if (records)
    for (long long k = 0; k < 4 * std::min(nrec, max_records); ++k) records[k] = lists[k];
  return static_cast<int>(std::min<long long>(nrec, 2147483647LL));
}

// Host-only check of the multiply-high divider the kernels use for index
// decomposition (no device work).
unsigned octlb_gpu_debug_fastdiv(unsigned d, unsigned n) { return FastDiv(d).div(n); }

int octlb_gpu_step_stats(const octlb_ctx* ctx, long long* launches, long long* lups) {
  if (!ctx) return OCTLB_EINVAL;
  if (ctx->launches_per_step > 0) {  // counted while the last advance_one was issued
    if (launches) *launches = ctx->launches_per_step;
    if (lups) *lups = ctx->lups_per_step;
    return OCTLB_OK;
  }
  long long total = 0;  // before any advance: the unfused count
  // Per level advance: ghost fill (if any ops) + step (+ drag + partial sum);
  // per coarse level: two prolongations, per fine level: one restriction.
  std::vector<long long> per(ctx->levels.size(), 0);
  for (size_t l = 0; l < ctx->levels.size(); ++l) {
    const Level& L = ctx->levels[l];
    if (L.nblk == 0) continue;
    per[l] = (L.args.nitems > 0 ? 1 : 0) + (L.n_near > 0 && !L.use_pair && !L.use_bulk && !L.use_map ? 1 : 0) + (L.has_force ? 1 : 0);
    if (ctx->drag && L.n_drag > 0) total += 1;  // once per advance_one, last step of the level
  }
  for (size_t l = 0; l < ctx->levels.size(); ++l) {
    const Level& L = ctx->levels[l];
    long long mult = 1LL << l;
    total += per[l] * mult;
    if (l + 1 < ctx->levels.size()) {
      total += (L.n_prolong > 0 ? 2 : 0) * mult;
      total += (ctx->levels[l + 1].n_restrict > 0 ? 1 : 0) * mult;
    }
  }
  if (ctx->drag && ctx->drag_parts > 0) total += 1;
  if (launches) *launches = total;
  if (lups) *lups = ctx->lups_per_step;
  return OCTLB_OK;
}

}  // extern "C"

// ==================================================== allocation-free audit
// octlb_gpu_audit_noalloc: the mass / momentum audit with its per-CTA
// partial sums in a fixed, file-scope device array instead of a cudaMalloc'd
// buffer, for callers that must not allocate device memory.  The array holds
// kNoAllocRows partial rows (one per CTA of 256 threads x 8 cells) plus one
// result row; every GPU that loads this library keeps it until exit.  Its
// device address is looked up with cudaGetSymbolAddress once per device, on
// the first call made with that device current.  Every call overwrites the
// whole array (no state carries over), so calls that overlap on the GPU race.
namespace octlb_host {

constexpr int kNoAllocRows = 16384;                 // partial rows (640 KB)
constexpr int kNoAllocCellsPerCta = 256 * 8;
constexpr long long kNoAllocMaxCells = static_cast<long long>(kNoAllocRows) * kNoAllocCellsPerCta;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[(kNoAllocRows + 1) * 5];
// Device address of the array per device, looked up once under the mutex (two
// host threads making their first call at once look it up once).
static double* g_noalloc_ptr[kNoAllocMaxDevices] = {};
static std::mutex g_noalloc_mutex;

template <typename T>
__global__ void __launch_bounds__(256) k_audit_noalloc(const StepArgs a, double* rows) {
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int k = 0; k < 8; ++k) {
    const uint32_t t = blockIdx.x * kNoAllocCellsPerCta + k * 256 + threadIdx.x;
    if (t >= a.ncore) break;
    const long long slot = t;  // compact core slot
    const T* src = static_cast<const T*>(a.src);
    double drho = 0, jx = 0, jy = 0, jz = 0;
    bool finite = true;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const float v = Store<T>::ld(src + (a.aa_rev ? aa_rev_slot(a, i, t) : i * a.qs + slot), a.inv_scale);
      finite = finite && isfinite(v);
      drho += v; jx += cx(i) * static_cast<double>(v);
      jy += cy(i) * static_cast<double>(v); jz += cz(i) * static_cast<double>(v);
    }
    if (!finite) acc[4] = 1.0;
    const int kind = a.flags ? (a.flags[slot] & kKindMask) : kBulk;
    if (kind == kBulk) {
      acc[0] += 1.0 + drho; acc[1] += jx; acc[2] += jy; acc[3] += jz;
    }
  }
  __shared__ double sm[8][5];
  for (int c = 0; c < 5; ++c)
    for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 5; ++c) sm[threadIdx.x >> 5][c] = acc[c];
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += sm[w][threadIdx.x];
    rows[blockIdx.x * 5 + threadIdx.x] = s;
  }
}

// Fixed-order sum of the partial rows into the result row: strided
// per-thread sums, then a fixed shuffle tree (deterministic).
__global__ void __launch_bounds__(256) k_audit_noalloc_sum(double* rows, int nrows) {
  __shared__ double sm[8];
  for (int c = 0; c < 5; ++c) {
    double v = 0.0;
    for (int r = threadIdx.x; r < nrows; r += 256) v += rows[r * 5 + c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < 8; ++w) s += sm[w];
      rows[kNoAllocRows * 5 + c] = s;
    }
    __syncthreads();
  }
}

template <typename T>
int audit_noalloc_impl(octlb_ctx* ctx, double* scratch, double out[4]) {
  double tot[5] = {0, 0, 0, 0, 0};
  for (auto& L : ctx->levels) {
    if (L.nblk == 0) continue;
    StepArgs a = L.args;
    a.src = L.buf[L.cur].p;
    a.aa_rev = L.aa && L.cur;
    const int nrows = static_cast<int>((a.ncore + kNoAllocCellsPerCta - 1) / kNoAllocCellsPerCta);
    k_audit_noalloc<T><<<nrows, 256, 0, ctx->stream>>>(a, scratch);
    CK(cudaGetLastError());
    k_audit_noalloc_sum<<<1, 256, 0, ctx->stream>>>(scratch, nrows);
    CK(cudaGetLastError());
    double h[5];
    CK(cudaMemcpyAsync(h, scratch + kNoAllocRows * 5, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 5; ++k) tot[k] += h[k];
  }
  for (int k = 0; k < 4; ++k) out[k] = tot[k];
  if (tot[4] != 0.0) return fail(ctx, OCTLB_ENAN, "non-finite populations");
  return OCTLB_OK;
}

}  // namespace octlb_host

extern "C" int octlb_gpu_audit_noalloc(octlb_ctx* ctx, double out[4]) {
  if (!ctx || !out) return OCTLB_EINVAL;
  if (ctx->levels.empty()) return fail(ctx, OCTLB_ESTATE, "context not initialised");
  for (const auto& L : ctx->levels) {
    if (static_cast<long long>(L.args.ncore) > kNoAllocMaxCells)
      return fail(ctx, OCTLB_EINVAL,
                  "octlb_gpu_audit_noalloc: a level has " + std::to_string(L.args.ncore) +
                      " cells, more than the " + std::to_string(kNoAllocMaxCells) +
                      " its fixed device scratch covers");
  }
  // The context's buffers must live on the current device.
  int dev = 0;
  CK(cudaGetDevice(&dev));
  for (const auto& L : ctx->levels) {
    if (!L.buf[0].p) continue;
    cudaPointerAttributes attr{};
    CK(cudaPointerGetAttributes(&attr, L.buf[0].p));
    if (attr.device != dev)
      return fail(ctx, OCTLB_EINVAL, "octlb_gpu_audit_noalloc: make the context's device current first");
    break;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(ctx, OCTLB_EINVAL, "device ordinal out of range");
  // A bounded device wait that gave up left a partly written state: report
  // it as octlb_gpu_audit does instead of summing that state.
  if (int rc = check_device_error(ctx)) return rc;
  // One-time set-up on this device: the scratch array's device address.  In
  // host code the array's name is only a host-side stand-in, never a device
  // address, so the kernels receive this pointer.
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
      g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_noalloc_ptr[dev];
  }
  return ctx->precision == OCTLB_FP32 ? audit_noalloc_impl<float>(ctx, scratch, out)
                                      : audit_noalloc_impl<__half>(ctx, scratch, out);
}
