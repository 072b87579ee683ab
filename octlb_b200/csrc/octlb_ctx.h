// Host-side state of one context (struct octlb_ctx of the C ABI) and the
// device-buffer helpers, shared by the translation units of the context:
// octlb_ctx.cu (tables, recursion, graphs, entry points) and octlb_part.cu
// (partition over ranks, cross-rank exchange).  Not part of the C ABI.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <unordered_set>
#include <vector>

#include "octlb_internal.h"
#include "../../include/octlb_gpu.h"

namespace octlb_gpu {

template <typename T> cudaError_t launch_step(const StepArgs&, bool, bool, bool, cudaStream_t);
template <typename T>
cudaError_t launch_couple(const ProlongOp&, const RestrictOp&, const RestrictOp&, cudaStream_t);
template <typename T>
cudaError_t launch_drag(const StepArgs&, bool, const DragItem*, int, double*, cudaStream_t);
cudaError_t launch_drag_total(const double*, int, double*, double*, cudaStream_t);
template <typename T> cudaError_t launch_audit(const StepArgs&, double*, double*, cudaStream_t);
template <typename T> cudaError_t launch_gather(const StepArgs&, double*, double*, int, cudaStream_t);
template <typename T> cudaError_t launch_scatter(const StepArgs&, const double*, int, cudaStream_t);
template <typename T> cudaError_t launch_scatter_eq(const StepArgs&, const double*, int, cudaStream_t);
template <typename T>
cudaError_t launch_step_cr(const StepArgs&, const NearTables&, bool, bool, cudaStream_t);
template <typename T> cudaError_t launch_cr_seed(const StepArgs&, int, cudaStream_t);
template <typename T>
cudaError_t launch_step_map_cr(const StepArgs&, const NearTables&, bool, bool, cudaStream_t);
template <typename T>
cudaError_t launch_step_map_nc(const StepArgs&, const NearTables&, bool, bool, cudaStream_t);
template <typename T>
cudaError_t launch_step_nc(const StepArgs&, const NearTables&, bool, bool, cudaStream_t);
template <typename T> cudaError_t launch_collide_cr(const StepArgs&, float*, cudaStream_t);
template <typename T> cudaError_t launch_step_aa(const StepArgs&, bool, cudaStream_t);
cudaError_t launch_cr_update(double*, const double*, int, long long, const double*, int, long long, float*,
                             cudaStream_t);
uint32_t cr_core_parts(const StepArgs& a);
uint32_t cr_near_parts(const NearTables& nt);
uint32_t couple_prolong_ctas(int n);
template <typename T> cudaError_t launch_step_bulk(const StepArgs&, int, cudaStream_t);
template <typename T> int bulk_prepare(int n);
bool rows_step_eligible(int n, long long ncore, long long qs, int variant);
long long rows_stage_cells(int variant);
int rows_prepare(int variant, bool local);
cudaError_t launch_step_rows_h(const StepArgs&, int variant, int grid, bool local, cudaStream_t);
bool aa_rows_eligible(int n, long long ncore, long long qs, int elem_bytes, int variant);
long long aa_rows_stage_cells(int variant, int elem_bytes);
template <typename T> int aa_rows_prepare(int variant);
template <typename T> cudaError_t launch_step_aa_rows(const StepArgs&, int variant, int grid, cudaStream_t);
template <typename T> cudaError_t launch_step_pair(const StepArgs&, cudaStream_t);
template <typename T> cudaError_t launch_step_near(const StepArgs&, const NearTables&, cudaStream_t);
template <typename T> cudaError_t launch_add_force(const StepArgs&, T*, const float*, cudaStream_t);
template <typename T> cudaError_t launch_step_map(const StepArgs&, const NearTables&, bool, bool, int, bool, cudaStream_t);
bool pair_step_eligible(int n);
bool map_step_eligible(int n, long long nslots);
void set_programmatic_launch(bool on);
cudaError_t launch_adj_step(const StepArgs&, const NearTables&, bool, bool, float*, float*, float*, double*, double*,
                            cudaStream_t);
cudaError_t launch_adj_force(const StepArgs&, const float*, double*, cudaStream_t);
cudaError_t launch_adj_drag(const StepArgs&, bool, const DragItem*, int, float*, float, int, double*, cudaStream_t);
cudaError_t launch_adj_prolong(const ProlongItem*, int, const float*, const float*, int, float*, long long, float,
                               float, float*, float*, float*, double*, double*, long long, cudaStream_t);
cudaError_t launch_adj_restrict(const RestrictItem*, int, const float*, float*, long long, float, float, float*,
                                double*, double*, long long, cudaStream_t);
bool bulk_step_eligible(int n, int elem_bytes);
uint32_t drag_partials(int n);
uint32_t audit_partials(const StepArgs& a);

// Host-only planning (octlb_gpu_plan): every allocation, upload and launch is
// skipped while the tables are flattened and checked.
inline thread_local bool g_dry_run = false;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool owned = true;        // false: an alias of another buffer (not freed here)
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes), owned(o.owned) { o.p = nullptr; o.bytes = 0; }
  ~DevBuf() { if (p && owned) cudaFree(p); }
  // The same memory as o, which keeps it.
  void alias(const DevBuf& o) {
    if (p && owned) cudaFree(p);
    p = o.p;
    bytes = o.bytes;
    owned = false;
  }
  cudaError_t alloc(size_t b) {
    if (p && owned) cudaFree(p);
    p = nullptr;
    owned = true;
    bytes = b;
    if (g_dry_run) return cudaSuccess;
    if (b == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) e = cudaMemset(p, 0, b);
    // The zero fill runs on the legacy default stream, which the context's
    // non-blocking streams do not wait for: it must land before any of them
    // touches the buffer.
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    return e;
  }
  // Capacity of at least b bytes, kept across calls and not zero-filled:
  // staging that every use overwrites before it is read.
  cudaError_t reserve(size_t b) {
    if (p && owned && bytes >= b) return cudaSuccess;
    if (p && owned) cudaFree(p);
    p = nullptr;
    owned = true;
    bytes = b;
    if (g_dry_run || b == 0) return cudaSuccess;
    return cudaMalloc(&p, b);
  }
  template <typename U> U* as() const { return static_cast<U*>(p); }
};

template <typename U>
inline cudaError_t upload(DevBuf& d, const std::vector<U>& h) {
  cudaError_t e = d.alloc(h.size() * sizeof(U));
  if (e != cudaSuccess || h.empty() || g_dry_run) return e;
  e = cudaMemcpy(d.p, h.data(), h.size() * sizeof(U), cudaMemcpyHostToDevice);
  // From pageable memory cudaMemcpy may return before its last DMA chunk has
  // landed (on the legacy stream, which the context's non-blocking streams do
  // not wait for); a kernel on those streams would read the buffer's tail
  // early.
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
  return e;
}

struct PlanPoint {  // CouplingPoint (level_coupler.h:18-30)
  int coarse_id, ci, cj, ck, fine_id, fi, fj, fk, normal, coarse_level, fine_level, slot;
};

struct Level {
  int lvl = 0;
  std::vector<int> blocks;          // global block ids, level-local order
  int nblk = 0, n = 0;
  long long ncore = 0, nslots = 0;  // core slots, core + halo-page slots
  DevBuf buf[2];
  int cur = 0;
  DevBuf flags, link_idx, link_rec, save_idx, save_buf;
  DevBuf nbase, page_of, hmap, hpos, open_pages, near_cells, slot_map;
  DevBuf near_mask, near_slot, near_q, near_add;
  NearTables near{};
  int n_near = 0;
  int n_open = 0, n_halo = 0, n_pages = 0, n_save = 0, n_links = 0;
  long long n_bulk = 0;             // kBulk core cells
  bool has_flags = false;
  // tree-boundary halo fills
  DevBuf bb_ops, fill_of;           // fills, and per (page slot, population) the fill index or -1
  DevBuf wall_add, wall_dadd;       // slot-map wall markers' terms
  DevBuf blk_moving;                // per block: its map holds a moving-wall marker
  uint32_t n_bb = 0;
  // coupler: this level as coarse (prolong) and as fine (restrict)
  DevBuf prolong_items, prev, restrict_items;
  // The restriction into this level (from level + 1) may share a launch with
  // the full-time prolongation into it (from level - 1): their target cells
  // are disjoint.
  bool fuse_restrict = false;
  int n_prolong = 0, n_restrict = 0;
  // drag
  DevBuf drag_items;
  int n_drag = 0;
  long long drag_off = 0;           // this level's rows in the context's drag partials
  int substep = 0;                  // steps of this level within the current advance_one
  float scale = 1.f, inv_scale = 1.f;
  bool use_bulk = false;            // pipelined bulk-copy step (periodic block)
  bool use_pair = false;            // two-cells-per-thread step (periodic block)
  bool use_map = false;             // slot-map step (forest level)
  bool aa = false;                  // AA stream order: buf[1] aliases buf[0], cur = layout parity
  // The finite-difference pass on this level's tree-boundary blocks: one
  // record per Dirichlet cell, the cells of each role (plane, edge, corner)
  // as runs of fd_lists, and their rewritten rows.
  DevBuf fd_cells, fd_lists, fd_new;
  int fd_rows = 0;
  std::vector<int> fd_first, fd_count;
  int bulk_grid = 0;
  bool use_rows = false;            // staged FP16 four-cell step (periodic block)
  int rows_grid = 0;
  bool use_aa_rows = false;         // staged AA pull step
  int aa_rows_grid = 0;
  bool use_aa_local_rows = false;   // staged FP16 AA local step
  int aa_local_grid = 0;
  DevBuf body_force;                // [3][ncore] float, or empty
  bool has_force = false;
  // Rank contexts (octlb_gpu_create_part): after the nblk owned blocks come
  // nmir mirror blocks -- same-level face / edge neighbours of owned blocks
  // that another rank owns -- stored like cores but never stepped; their
  // cells the owned blocks read are refreshed before every step of the level.
  // Halo pages start after them, at core_end.
  int nmir = 0;
  long long core_end = 0;
  int n_save_own = 0;               // save rows of owned cells; rows received from peers follow
  // One direction of a cross-rank exchange: items grouped by peer rank
  // (segment k: peer[k], items off[k] .. off[k + 1]), their local slots
  // (cells) or save rows, and the staging buffer ([19][items] in the storage
  // type for cells, [items][19] float for save rows).
  struct Xfer {
    std::vector<int> peer;
    std::vector<long long> off{0};
    DevBuf idx, buf;
    long long items() const { return off.back(); }
  };
  Xfer cell_send, cell_recv, row_send, row_recv;
  std::vector<long long> row_recv_first;  // first save row of each receive segment
  // While the adjoint recomputes a segment, the level's state and save rows
  // live in the step records' buffers (null otherwise).
  void* rec_cur = nullptr;
  void* rec_save = nullptr;
  StepArgs args{};
};

inline void* cur_buf(Level& L) { return L.rec_cur ? L.rec_cur : L.buf[L.cur].p; }
inline float* save_ptr(Level& L) { return static_cast<float*>(L.rec_save ? L.rec_save : L.save_buf.p); }

// Forward state of one level step kept for the reverse sweep: the step's
// input after the body force and the boundary fills, the save rows it wrote,
// and (coarse levels) the prev-macro store before its half-time prolongation.
constexpr int kGradSlots = 4;       // d/d omega, d/d prolong scale, d/d restrict scale, d/d wall velocity

struct StepRecord {
  int level = -1;
  DevBuf snap, save, prev;
  bool drag = false;                // the objective's force is taken from this input
};

// Adjoint sweep state (octlb_gpu_adjoint): cotangents per level, the
// checkpoints of one run and the step records of one recomputed segment.
struct AdjointState {
  struct Lv {
    DevBuf lam[2];                  // cotangent of the level's populations ([19][slots] FP32)
    int cur = 0;
    DevBuf lam_save, lam_m, lam_prev, gF;
  };
  std::vector<Lv> lv;
  // Two record sets, one per segment parity: the recomputation of the next
  // segment (set (c - 1) % 2) runs on rstream beside the reverse of the
  // current one (set c % 2) on the context's stream.
  std::vector<StepRecord> recs;     // [2][set_size]
  size_t set_size = 0;
  std::vector<int> next_same;       // next record of the same level in the same set, or -1
  std::vector<int> first_rec;       // first record of each level in set 0, or -1 (set 1: + set_size)
  size_t nrec = 0;
  cudaStream_t rstream = nullptr;
  cudaEvent_t ev_fwd = nullptr, ev_rec[2] = {nullptr, nullptr}, ev_rev[2] = {nullptr, nullptr};
  bool recording = false;
  int last_rec[32] = {};
  DevBuf g;                         // parameter-gradient accumulators (FP64)
  struct Checkpoint {
    std::vector<DevBuf> buf, prev;
    std::vector<int> cur;
  };
  std::vector<Checkpoint> ck;
  int comp = 0;
  // Recomputation (kind 0) and reverse (kind 1) of one segment captured as
  // CUDA graphs, keyed by (kind, buffer or cotangent parity, steps, steps in
  // the objective's window); valid for one adjoint call.
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    uint64_t out_mask = 0;
  };
  std::map<std::array<long long, 4>, Graph> graphs;
  std::array<long long, 4> graph_params{};  // (steps, window, interval, component) the graphs were made for
  void clear_graphs() {
    for (auto& kv : graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    graphs.clear();
  }
  AdjointState() = default;
  AdjointState(const AdjointState&) = delete;
  AdjointState& operator=(const AdjointState&) = delete;
  ~AdjointState() {
    if (rstream) cudaStreamSynchronize(rstream);
    clear_graphs();
    for (cudaEvent_t e : {ev_fwd, ev_rec[0], ev_rec[1], ev_rev[0], ev_rev[1]})
      if (e) cudaEventDestroy(e);
    if (rstream) cudaStreamDestroy(rstream);
  }
};

}  // namespace octlb_gpu

using namespace octlb_gpu;

struct octlb_ctx {
  std::string err;
  int n = 0, n_blocks = 0, precision = 0, stream_mode = 0, periodic = 0, drag = 0;
  double omega = 1.0;
  int max_level = 0;
  std::vector<Level> levels;
  std::vector<int> blk_level, blk_local;
  std::vector<uint8_t> kinds;
  std::vector<double> bounds;       // [n_blocks][6] leaf bounds (VTK output)
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // Restrictions not launched yet: each shares the next coupler launch unless
  // a step comes first (then they are launched alone, two per launch).
  struct PendingRestrict {
    RestrictOp op;
    int level;  // the coarse level written
  };
  std::vector<PendingRestrict> pending_restrict;
  // The momentum-exchange force runs on a forked stream inside advance_one
  // (it only reads the last finest step's input) and joins at its end.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool side_busy = false;
  DevBuf drag_partial, force, force_sum, audit_out, audit_partial, host_tmp, dev_err;
  // FP64 host-layout staging of set/get_populations and get_fields (grown on
  // demand, kept until destroy: no allocation per call)
  DevBuf stage_a, stage_b;
  int drag_parts = 0;
  long long force_steps = 0;
  std::vector<int> counters_collide, counters_stream;
  long long launches_per_step = 0, lups_per_step = 0;
  long long launch_count = 0;       // kernels issued by the advance_one being built
  int step_kernel = 0;              // OCTLB_STEP_KERNEL: 0 pair (default), 1 bulk, 2 plain
  int fp16_rows = 0;                // OCTLB_FP16_ROWS: the staged FP16 step's launch shape (off: -1)
  int aa_rows = 0;                  // OCTLB_AA_ROWS: the staged AA pull step's launch shape (off: -1)
  bool map_global = true;           // slot map read through L1 (OCTLB_MAP_SMEM=1: staged in shared memory)
  // Bounded device waits: their limit (OCTLB_WAIT_MS, default 1 s) and the
  // test of the give-up path (OCTLB_TEST_BULK_STALL=1: one CTA of the bulk
  // step waits for a row it never requested).  After a give-up whose own
  // copies did not drain either, the context refuses further work.
  unsigned long long wait_ns = 1000000000ull;
  int stall_first_row = 0;
  bool unusable = false;
  int map_cells = 0;                // cells per thread of the slot-map step (OCTLB_MAP_CELLS 1 or 2;
                                    // default 2, 1 under the links rule whose variant spills at 2)
  // advance_one captured as CUDA graphs, keyed by the A/B parity of every
  // level's buffers (the launch arguments depend on it)
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    uint64_t out_mask = 0;
    std::vector<int> dcollide;
  };
  std::map<uint64_t, GraphEntry> graphs;
  bool use_graphs = true;           // OCTLB_NO_GRAPH=1 launches kernel by kernel
  bool use_pdl = true;              // OCTLB_NO_PDL=1: plain stream order between the step's kernels
  float prolong_scale = 0.f, restrict_scale = 0.f;
  // Per level: the BGK rate, and the Lagrava scales of the pair (l, l + 1)
  // (all equal in the reference coupler mode).
  int coupler_mode = 0;
  std::vector<double> omega_l;
  std::vector<float> pscale_l, rscale_l;
  double wall_vscale = 0.0;         // largest moving-wall speed (adjoint velocity parameter)
  std::unique_ptr<AdjointState> adj;
  // ConstRhoBGK (TimeLoop's use_const_rho_bgk): the average density on the
  // device (TimeLoop::average_rho_) and the partial sums of the last collide
  // of the finest level cr_level, over its cr_count kBulk cells: cr_nparts
  // from its step, then cr_pparts from the prolongation into it.  cr_multi:
  // levels above cr_level exist; their steps only stream, and each collides
  // (k_collide_cr) once its coupling is done.
  int stream_order = 0;             // OCTLB_ORDER_AB or OCTLB_ORDER_AA
  bool const_rho = false, cr_multi = false;
  DevBuf cr_avg, cr_part;
  int cr_level = -1, cr_nparts = 0, cr_near = 0, cr_pparts = 0;
  long long cr_count = 0;
  // Ranks (octlb_gpu_create_part): this context steps the blocks with
  // owner[b] == rank and exchanges with the other ranks' contexts through
  // comm (empty owner: one rank owns every block).
  int rank = 0, nranks = 1;
  std::vector<int> owner;
  struct octlb_comm* comm = nullptr;
  // A periodic block shared over ranks: rank r holds x slab r of the
  // periodic (nranks n) x n x n box, with two ghost x planes after its core
  // that the neighbouring slabs fill before every step.
  bool slab = false;
  // Finite-difference domain boundary conditions (octlb_gpu_set_fd_boundary):
  // the records per level (Level::fd_*) and the time of the current
  // advance_one (the inlet ramp's clock).  cpl_cells_bulk: every coupler
  // source and target cell is kBulk (the pass on multi-level meshes needs
  // its interfaces away from the domain faces).
  bool fd_on = false;
  DevBuf fd_time;
  bool cpl_cells_bulk = true;
  // ConstRhoBGK with the pass: per-CTA sums of the velocity cells' collide
  // densities (the boundary part of the statistics), over fd_vel cells
  bool fd_single = false;           // the pass on one level: its store ticks the clock
  DevBuf fd_cr_part;
  // ConstRhoBGK: per level the density shift 1 - average_rho its kBulk
  // cells' stored state carries (0 after a stream-only step), which the
  // finite-difference pass removes from the densities it reads
  DevBuf cr_shift;
  int fd_cr_parts = 0;
  long long fd_vel = 0;
  bool owns(int b) const { return owner.empty() || owner[b] == rank; }
  // Host-only planning of a rank context (octlb_gpu_plan_part): the exchange
  // lists as (level, kind, peer, global cell) records, kind 0 / 1 cells sent /
  // received, 2 / 3 save rows sent / received.
  std::vector<long long>* plan_lists = nullptr;
};


namespace octlb_host {

int fail(octlb_ctx* c, int code, const std::string& msg);
int cuda_fail(octlb_ctx* c, cudaError_t e, const char* where);
#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);       \
  } while (0)

// Cross-rank exchange of rank contexts (octlb_part.cu).
int setup_xfer(octlb_ctx* ctx, Level::Xfer& x, const std::map<int, std::vector<long long>>& by_peer,
               size_t item_bytes, bool staging);
template <typename T> int exchange_cells(octlb_ctx* ctx, Level& L);
template <typename T> int exchange_slab(octlb_ctx* ctx, Level& L);
int exchange_rows(octlb_ctx* ctx, Level& L);
int comm_allreduce(octlb_ctx* ctx, double* v, int n);
int comm_synchronize(octlb_ctx* ctx);
int comm_attach(octlb_ctx* ctx);
int comm_nranks(const octlb_comm* comm);
// Finite-difference domain boundary pass (octlb_fd.cu).
template <typename T> int fd_after_step(octlb_ctx* ctx, Level& L);
template <typename T> int fd_before_step(octlb_ctx* ctx, Level& L);
int fd_end_of_step(octlb_ctx* ctx);
int fd_fix_fields(octlb_ctx* ctx, Level& L, double* rho, double* u);
void clear_graphs(octlb_ctx* ctx);
void comm_detach(octlb_ctx* ctx);

inline long long core_slot_of(int n, int local_blk, int x, int y, int z) {
  const long long n3 = static_cast<long long>(n) * n * n;
  return local_blk * n3 + (static_cast<long long>(x) * n + y) * n + z;
}

}  // namespace octlb_host
