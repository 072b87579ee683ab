// Ranks: the weighted Morton partition of the leaves, the exchange tables of a
// rank context, and the two transports between rank contexts.
//
// A rank context (octlb_gpu_create_part) steps the blocks its rank owns.  Per
// level step it refreshes its mirror blocks (the same-level neighbours of its
// blocks that other ranks own) with the cells those ranks send, and after the
// step it sends the save rows (pre-collision populations of coupler source
// cells) that other ranks' coupler items read.  The reference's counterparts:
// OctreeForest::partition with make_level_weight_fn (octree_forest.cpp:
// 273-280, weighted_load_balancer.cpp:7-12), GhostSchedule's cross-rank face /
// edge messages (ghost_schedule.h:121-255), LevelCoupler's coarse -> fine and
// fine -> coarse MPI batches (level_coupler.cpp:325-436, 492-585) and the
// force / mass MPI_Allreduce of the cases (cylinder3d_case.h:502, 620).
//
// Transports:
//  * local  -- the rank contexts of one process, one host thread each (on one
//              or several devices): a sender's staging buffer is copied into
//              the receiver's with cudaMemcpyAsync on the receiver's stream,
//              ordered by events and two host barriers per exchange (bounded
//              waits: a rank that never arrives ends the others' calls with
//              OCTLB_ETIMEOUT).
//  * nccl   -- one process per GPU: grouped ncclSend / ncclRecv on the
//              context's stream, FP64 ncclAllReduce for the force and audit
//              sums.  libnccl is opened at run time (dlopen), so the library
//              loads where NCCL is absent.
#include <chrono>
#include <condition_variable>
#include <thread>
#include <dlfcn.h>
#include <nccl.h>

#include "octlb_ctx.h"

namespace octlb_gpu {
template <typename T>
cudaError_t launch_pack_cells(const void*, long long, const long long*, long long, void*, cudaStream_t);
template <typename T>
cudaError_t launch_unpack_cells(void*, long long, const long long*, long long, const void*, cudaStream_t);
cudaError_t launch_pack_rows(const float*, const long long*, long long, float*, cudaStream_t);
}  // namespace octlb_gpu

using namespace octlb_gpu;
using namespace octlb_host;

struct XSeg {
  int peer;
  void* ptr;
  size_t bytes;
};

struct octlb_comm {
  int nranks = 1;
  virtual ~octlb_comm() = default;
  virtual int attach(octlb_ctx* ctx, int rank) = 0;
  virtual void detach(octlb_ctx* ctx, int rank) = 0;
  // Every rank context calls exchange() at the same points of the time step
  // (once before and once after every level step), with what it sends and
  // receives there (possibly nothing).
  // Segments between two ranks are matched in order: the k-th one a rank
  // lists for a peer is the k-th one the peer lists for it.
  virtual int exchange(octlb_ctx* ctx, const std::vector<XSeg>& sends, const std::vector<XSeg>& recvs) = 0;
  virtual int allreduce_sum(octlb_ctx* ctx, double* v, int n) = 0;
  virtual int synchronize(octlb_ctx* ctx) = 0;
};

namespace {

// ----------------------------------------------------------------- local
struct LocalComm final : octlb_comm {
  std::mutex m;
  std::condition_variable cv;
  int arrived = 0;
  long long generation = 0;
  bool broken = false;
  double timeout_s = 60.0;
  struct Pub {
    octlb_ctx* ctx = nullptr;
    std::vector<XSeg> sends;
    cudaEvent_t ev_pack = nullptr, ev_copy = nullptr;
    std::vector<double> red;
  };
  std::vector<Pub> pub;

  explicit LocalComm(int n) {
    nranks = n;
    pub.resize(n);
    if (const char* e = std::getenv("OCTLB_COMM_TIMEOUT_S")) {
      const double v = std::atof(e);
      if (v > 0) timeout_s = v;
    }
  }
  ~LocalComm() override {
    for (Pub& p : pub) {
      if (p.ev_pack) cudaEventDestroy(p.ev_pack);
      if (p.ev_copy) cudaEventDestroy(p.ev_copy);
    }
  }
  // All ranks meet; false after timeout_s (the comm is then broken for all).
  bool barrier() {
    std::unique_lock<std::mutex> lk(m);
    if (broken) return false;
    const long long gen = generation;
    if (++arrived == nranks) {
      arrived = 0;
      ++generation;
      cv.notify_all();
      return true;
    }
    const bool ok = cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                [&] { return generation != gen || broken; });
    if (!ok || broken) {
      broken = true;
      cv.notify_all();
      return false;
    }
    return true;
  }
  int attach(octlb_ctx* ctx, int rank) override {
    std::lock_guard<std::mutex> lk(m);
    Pub& p = pub[rank];
    if (p.ctx) return fail(ctx, OCTLB_EINVAL, "local comm: rank " + std::to_string(rank) + " is already attached");
    CK(cudaEventCreateWithFlags(&p.ev_pack, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&p.ev_copy, cudaEventDisableTiming));
    p.ctx = ctx;
    return OCTLB_OK;
  }
  void detach(octlb_ctx* ctx, int rank) override {
    std::lock_guard<std::mutex> lk(m);
    if (rank >= 0 && rank < nranks && pub[rank].ctx == ctx) pub[rank].ctx = nullptr;
  }
  int exchange(octlb_ctx* ctx, const std::vector<XSeg>& sends, const std::vector<XSeg>& recvs) override {
    const int r = ctx->rank;
    Pub& me = pub[r];
    me.sends = sends;
    CK(cudaEventRecord(me.ev_pack, ctx->stream));
    if (!barrier()) return fail(ctx, OCTLB_ETIMEOUT, "local comm: a rank did not reach the exchange");
    // The k-th segment this rank receives from a peer is the k-th segment
    // that peer sends to this rank.
    std::vector<size_t> cursor(nranks, 0);
    for (const XSeg& in : recvs) {
      const Pub& src = pub[in.peer];
      const XSeg* out = nullptr;
      for (size_t k = cursor[in.peer]; k < src.sends.size(); ++k)
        if (src.sends[k].peer == r) {
          out = &src.sends[k];
          cursor[in.peer] = k + 1;
          break;
        }
      if (!out || out->bytes != in.bytes) {
        std::lock_guard<std::mutex> lk(m);
        broken = true;
        cv.notify_all();
        return fail(ctx, OCTLB_EINVAL, "local comm: rank " + std::to_string(in.peer) + " sends " +
                                           std::to_string(out ? out->bytes : 0) + " bytes, rank " +
                                           std::to_string(r) + " expects " + std::to_string(in.bytes));
      }
      CK(cudaStreamWaitEvent(ctx->stream, src.ev_pack, 0));
      CK(cudaMemcpyAsync(in.ptr, out->ptr, in.bytes, cudaMemcpyDefault, ctx->stream));
    }
    CK(cudaEventRecord(me.ev_copy, ctx->stream));
    if (!barrier()) return fail(ctx, OCTLB_ETIMEOUT, "local comm: a rank did not finish the exchange");
    // The receivers' copies out of this rank's staging buffer come before
    // anything this rank's stream does next (the next pack rewrites it).
    for (const XSeg& s : sends) CK(cudaStreamWaitEvent(ctx->stream, pub[s.peer].ev_copy, 0));
    return OCTLB_OK;
  }
  int allreduce_sum(octlb_ctx* ctx, double* v, int n) override {
    const int r = ctx->rank;
    pub[r].red.assign(v, v + n);
    if (!barrier()) return fail(ctx, OCTLB_ETIMEOUT, "local comm: a rank did not reach the reduction");
    std::vector<double> sum(n, 0.0);
    for (int k = 0; k < nranks; ++k) {
      if (static_cast<int>(pub[k].red.size()) != n) {
        std::lock_guard<std::mutex> lk(m);
        broken = true;
        cv.notify_all();
        return fail(ctx, OCTLB_EINVAL, "local comm: reduction sizes differ between ranks");
      }
      for (int j = 0; j < n; ++j) sum[j] += pub[k].red[j];  // rank order: the same sum on every rank
    }
    if (!barrier()) return fail(ctx, OCTLB_ETIMEOUT, "local comm: a rank did not finish the reduction");
    std::copy(sum.begin(), sum.end(), v);
    return OCTLB_OK;
  }
  int synchronize(octlb_ctx* ctx) override {
    CK(cudaStreamSynchronize(ctx->stream));
    return OCTLB_OK;
  }
};

// ------------------------------------------------------------------ nccl
struct NcclApi {
  void* h = nullptr;
  decltype(&ncclGetUniqueId) get_unique_id = nullptr;
  decltype(&ncclCommInitRank) init_rank = nullptr;
  decltype(&ncclCommDestroy) destroy = nullptr;
  decltype(&ncclCommAbort) abort = nullptr;
  decltype(&ncclCommGetAsyncError) async_error = nullptr;
  decltype(&ncclGetErrorString) error_string = nullptr;
  decltype(&ncclGroupStart) group_start = nullptr;
  decltype(&ncclGroupEnd) group_end = nullptr;
  decltype(&ncclSend) send = nullptr;
  decltype(&ncclRecv) recv = nullptr;
  decltype(&ncclAllReduce) allreduce = nullptr;
  std::string error;
  bool load() {
    if (h) return true;
    for (const char* name : {"libnccl.so.2", "libnccl.so"}) {
      h = dlopen(name, RTLD_NOW | RTLD_GLOBAL);
      if (h) break;
    }
    if (!h) {
      error = std::string("libnccl not found: ") + dlerror();
      return false;
    }
    bool ok = true;
    auto sym = [&](auto& fn, const char* name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
      if (!fn) { ok = false; error = std::string("libnccl lacks ") + name; }
    };
    sym(get_unique_id, "ncclGetUniqueId");
    sym(init_rank, "ncclCommInitRank");
    sym(destroy, "ncclCommDestroy");
    sym(abort, "ncclCommAbort");
    sym(async_error, "ncclCommGetAsyncError");
    sym(error_string, "ncclGetErrorString");
    sym(group_start, "ncclGroupStart");
    sym(group_end, "ncclGroupEnd");
    sym(send, "ncclSend");
    sym(recv, "ncclRecv");
    sym(allreduce, "ncclAllReduce");
    return ok;
  }
};
NcclApi& nccl() {
  static NcclApi api;
  return api;
}
std::mutex g_nccl_mutex;

struct NcclComm final : octlb_comm {
  ncclComm_t comm = nullptr;
  int rank = 0;
  DevBuf red;
  double timeout_s = 300.0;
  bool aborted = false;
  ~NcclComm() override {
    if (comm) (aborted ? nccl().abort : nccl().destroy)(comm);
  }
  int check(octlb_ctx* ctx, ncclResult_t r, const char* where) {
    if (r == ncclSuccess) return OCTLB_OK;
    return fail(ctx, OCTLB_ECUDA, std::string(where) + ": " + nccl().error_string(r));
  }
  int attach(octlb_ctx* ctx, int r) override {
    if (r != rank) return fail(ctx, OCTLB_EINVAL, "nccl comm: the context's rank differs from the comm's");
    return OCTLB_OK;
  }
  void detach(octlb_ctx*, int) override {}
  int exchange(octlb_ctx* ctx, const std::vector<XSeg>& sends, const std::vector<XSeg>& recvs) override {
    if (sends.empty() && recvs.empty()) return OCTLB_OK;  // point-to-point: nothing to match
    if (int rc = check(ctx, nccl().group_start(), "ncclGroupStart")) return rc;
    for (const XSeg& s : sends)
      if (int rc = check(ctx, nccl().send(s.ptr, s.bytes, ncclUint8, s.peer, comm, ctx->stream), "ncclSend"))
        return rc;
    for (const XSeg& s : recvs)
      if (int rc = check(ctx, nccl().recv(s.ptr, s.bytes, ncclUint8, s.peer, comm, ctx->stream), "ncclRecv"))
        return rc;
    return check(ctx, nccl().group_end(), "ncclGroupEnd");
  }
  int allreduce_sum(octlb_ctx* ctx, double* v, int n) override {
    CK(red.reserve(static_cast<size_t>(n) * sizeof(double)));
    CK(cudaMemcpyAsync(red.p, v, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    if (int rc = check(ctx, nccl().allreduce(red.p, red.p, n, ncclFloat64, ncclSum, comm, ctx->stream),
                       "ncclAllReduce"))
      return rc;
    CK(cudaMemcpyAsync(v, red.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    return synchronize(ctx);
  }
  // Waits for the stream with a limit: a peer that died leaves NCCL's kernels
  // waiting, so the wait polls the communicator's error state and aborts it
  // (which ends those kernels) after timeout_s.
  int synchronize(octlb_ctx* ctx) override {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      const cudaError_t q = cudaStreamQuery(ctx->stream);
      if (q == cudaSuccess) return OCTLB_OK;
      if (q != cudaErrorNotReady) return cuda_fail(ctx, q, "cudaStreamQuery");
      ncclResult_t ae = ncclSuccess;
      nccl().async_error(comm, &ae);
      const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (ae != ncclSuccess || el > timeout_s) {
        aborted = true;
        nccl().abort(comm);
        comm = nullptr;
        return fail(ctx, OCTLB_ETIMEOUT, ae != ncclSuccess ? std::string("nccl: ") + nccl().error_string(ae)
                                                           : std::string("nccl: exchange did not complete"));
      }
      std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
  }
};

}  // namespace

namespace octlb_host {

// Staging and index tables of one exchange direction: items grouped by peer
// (ascending rank), idx[k] the local slot (cells) or save row of item k.
int setup_xfer(octlb_ctx* ctx, Level::Xfer& x, const std::map<int, std::vector<long long>>& by_peer,
               size_t item_bytes, bool staging) {
  x.peer.clear();
  x.off.assign(1, 0);
  std::vector<long long> idx;
  for (const auto& [peer, items] : by_peer) {
    if (items.empty()) continue;
    x.peer.push_back(peer);
    idx.insert(idx.end(), items.begin(), items.end());
    x.off.push_back(static_cast<long long>(idx.size()));
  }
  CK(upload(x.idx, idx));
  if (staging) CK(x.buf.alloc(idx.size() * item_bytes));
  return OCTLB_OK;
}

// Before a step of level L: the owned cells the peers mirror, out; this
// rank's mirror cells, in.  Called by every rank context at every level step.
template <typename T>
int exchange_cells(octlb_ctx* ctx, Level& L) {
  if (!ctx->comm) return OCTLB_OK;
  const size_t ib = kQ * sizeof(T);
  void* cur = L.nblk > 0 ? cur_buf(L) : nullptr;
  std::vector<XSeg> sends, recvs;
  if (L.cell_send.items() > 0) {
    CK(launch_pack_cells<T>(cur, L.nslots, L.cell_send.idx.as<long long>(), L.cell_send.items(), L.cell_send.buf.p,
                            ctx->stream));
    ++ctx->launch_count;
    for (size_t k = 0; k < L.cell_send.peer.size(); ++k)
      sends.push_back({L.cell_send.peer[k], L.cell_send.buf.as<char>() + L.cell_send.off[k] * ib,
                       static_cast<size_t>(L.cell_send.off[k + 1] - L.cell_send.off[k]) * ib});
  }
  for (size_t k = 0; k < L.cell_recv.peer.size(); ++k)
    recvs.push_back({L.cell_recv.peer[k], L.cell_recv.buf.as<char>() + L.cell_recv.off[k] * ib,
                     static_cast<size_t>(L.cell_recv.off[k + 1] - L.cell_recv.off[k]) * ib});
  if (int rc = ctx->comm->exchange(ctx, sends, recvs)) return rc;
  if (L.cell_recv.items() > 0) {
    CK(launch_unpack_cells<T>(cur, L.nslots, L.cell_recv.idx.as<long long>(), L.cell_recv.items(),
                              L.cell_recv.buf.p, ctx->stream));
    ++ctx->launch_count;
  }
  return OCTLB_OK;
}

// After a step of level L: the save rows other ranks' coupler items read,
// out; the rows this rank's items read from other ranks, in (straight into
// the save-row buffer, one contiguous run per peer).
int exchange_rows(octlb_ctx* ctx, Level& L) {
  if (!ctx->comm || ctx->slab) return OCTLB_OK;
  const size_t ib = kQ * sizeof(float);
  float* save = save_ptr(L);
  std::vector<XSeg> sends, recvs;
  if (L.row_send.items() > 0) {
    CK(launch_pack_rows(save, L.row_send.idx.as<long long>(), L.row_send.items(), L.row_send.buf.as<float>(),
                        ctx->stream));
    ++ctx->launch_count;
    for (size_t k = 0; k < L.row_send.peer.size(); ++k)
      sends.push_back({L.row_send.peer[k], L.row_send.buf.as<char>() + L.row_send.off[k] * ib,
                       static_cast<size_t>(L.row_send.off[k + 1] - L.row_send.off[k]) * ib});
  }
  for (size_t k = 0; k < L.row_recv.peer.size(); ++k)
    recvs.push_back({L.row_recv.peer[k], save + L.row_recv_first[k] * kQ,
                     static_cast<size_t>(L.row_recv.off[k + 1] - L.row_recv.off[k]) * ib});
  return ctx->comm->exchange(ctx, sends, recvs);
}

// Before a step of an x slab of a periodic box: its two ghost x planes (after
// the core, planes n and n + 1) from the neighbouring slabs, straight from and
// into the state buffer -- every population's plane is one contiguous run of
// n^2 values.  A cell at x = 0 pulls the populations with c_x = +1 from the
// left neighbour's last plane, a cell at x = n - 1 those with c_x = -1 from
// the right neighbour's first plane.  Segments are listed by (peer,
// population) on both ends, which matches them when the two neighbours are
// the same rank (two slabs).
template <typename T>
int exchange_slab(octlb_ctx* ctx, Level& L) {
  const int P = ctx->nranks, r = ctx->rank, left = (r + P - 1) % P, right = (r + 1) % P;
  const long long n = L.n, n2 = n * n;
  T* cur = static_cast<T*>(cur_buf(L));
  const size_t bytes = static_cast<size_t>(n2) * sizeof(T);
  struct K { int peer, pop; XSeg s; };
  std::vector<K> sends, recvs;
  for (int i = 0; i < kQ; ++i) {
    if (cx(i) == -1) {  // my first plane -> left's hi ghost; right's first plane -> my hi ghost
      sends.push_back({left, i, {left, cur + i * L.nslots, bytes}});
      recvs.push_back({right, i, {right, cur + i * L.nslots + (n + 1) * n2, bytes}});
    } else if (cx(i) == 1) {  // my last plane -> right's lo ghost; left's last plane -> my lo ghost
      sends.push_back({right, i, {right, cur + i * L.nslots + (n - 1) * n2, bytes}});
      recvs.push_back({left, i, {left, cur + i * L.nslots + n * n2, bytes}});
    }
  }
  auto by_peer_pop = [](const K& a, const K& b) { return a.peer != b.peer ? a.peer < b.peer : a.pop < b.pop; };
  std::sort(sends.begin(), sends.end(), by_peer_pop);
  std::sort(recvs.begin(), recvs.end(), by_peer_pop);
  std::vector<XSeg> s, v;
  for (const K& k : sends) s.push_back(k.s);
  for (const K& k : recvs) v.push_back(k.s);
  return ctx->comm->exchange(ctx, s, v);
}

int comm_allreduce(octlb_ctx* ctx, double* v, int n) {
  if (!ctx->comm) return OCTLB_OK;
  return ctx->comm->allreduce_sum(ctx, v, n);
}

int comm_synchronize(octlb_ctx* ctx) {
  if (!ctx->comm) {
    CK(cudaStreamSynchronize(ctx->stream));
    return OCTLB_OK;
  }
  return ctx->comm->synchronize(ctx);
}

int comm_nranks(const octlb_comm* comm) { return comm->nranks; }

int comm_attach(octlb_ctx* ctx) { return ctx->comm ? ctx->comm->attach(ctx, ctx->rank) : OCTLB_OK; }
void comm_detach(octlb_ctx* ctx) {
  if (ctx->comm) ctx->comm->detach(ctx, ctx->rank);
}

template int exchange_cells<float>(octlb_ctx*, Level&);
template int exchange_cells<__half>(octlb_ctx*, Level&);
template int exchange_slab<float>(octlb_ctx*, Level&);
template int exchange_slab<__half>(octlb_ctx*, Level&);

}  // namespace octlb_host

// ====================================================================== C ABI
extern "C" {

int octlb_gpu_partition(const octlb_tables* t, int nranks, int* owner) {
  if (!t || !owner || nranks < 1 || t->n_blocks < 1 || !t->levels) return OCTLB_EINVAL;
  // Leaves in the forest's order (trees, then Morton order inside a tree),
  // weight 2^level: rank k takes the leaves whose weight prefix lies in
  // [k W / P, (k + 1) W / P) -- contiguous runs of equal weight.
  long long W = 0;
  for (int b = 0; b < t->n_blocks; ++b) {
    if (t->levels[b] < 0 || t->levels[b] > 30) return OCTLB_EINVAL;
    W += 1LL << t->levels[b];
  }
  long long S = 0;
  for (int b = 0; b < t->n_blocks; ++b) {
    const long long r = (static_cast<__int128>(S) * nranks) / W;
    owner[b] = static_cast<int>(std::min<long long>(r, nranks - 1));
    S += 1LL << t->levels[b];
  }
  return OCTLB_OK;
}

int octlb_comm_create_local(int nranks, octlb_comm** out) {
  if (!out || nranks < 1) return OCTLB_EINVAL;
  *out = new LocalComm(nranks);
  return OCTLB_OK;
}

int octlb_comm_nccl_unique_id(unsigned char id[128]) {
  if (!id) return OCTLB_EINVAL;
  std::lock_guard<std::mutex> lk(g_nccl_mutex);
  if (!nccl().load()) return OCTLB_ECUDA;
  ncclUniqueId u;
  if (nccl().get_unique_id(&u) != ncclSuccess) return OCTLB_ECUDA;
  std::memcpy(id, u.internal, NCCL_UNIQUE_ID_BYTES);
  return OCTLB_OK;
}

int octlb_comm_create_nccl(const unsigned char id[128], int nranks, int rank, octlb_comm** out) {
  if (!out || !id || nranks < 1 || rank < 0 || rank >= nranks) return OCTLB_EINVAL;
  *out = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_nccl_mutex);
    if (!nccl().load()) return OCTLB_ECUDA;
  }
  ncclUniqueId u;
  std::memcpy(u.internal, id, NCCL_UNIQUE_ID_BYTES);
  auto c = std::make_unique<NcclComm>();
  c->nranks = nranks;
  c->rank = rank;
  if (const char* e = std::getenv("OCTLB_COMM_TIMEOUT_S")) {
    const double v = std::atof(e);
    if (v > 0) c->timeout_s = v;
  }
  if (nccl().init_rank(&c->comm, nranks, u, rank) != ncclSuccess) return OCTLB_ECUDA;
  *out = c.release();
  return OCTLB_OK;
}

void octlb_comm_destroy(octlb_comm* comm) { delete comm; }

const char* octlb_comm_last_error(void) { return nccl().error.c_str(); }

}  // extern "C"
