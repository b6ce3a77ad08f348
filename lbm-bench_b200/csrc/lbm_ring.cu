// Native ring of x-slabs (lbm_ring_* in include/lbm_b200.h): the halo
// exchange of lbm_create_slab solvers between ring neighbours over NCCL
// point-to-point, ordered on the solver's stream, and the step loop around
// it issued from C. Per exchange: lbm_halo_pack writes the two messages,
// one grouped ncclSend/ncclRecv pair per neighbour moves them, and
// lbm_halo_unpack reads what arrived. Nothing on the host waits per step.
//
// NCCL is loaded at run time, so the library itself does not depend on it.
// The communicator is non-blocking (ncclConfig_t::blocking = 0) and every
// wait on it is bounded: creation, the completion of each group, and the
// stream (the run loop keeps at most two windows of kWindow steps queued).
// When a wait runs out the communicator is aborted - ncclCommAbort ends NCCL
// kernels that wait for a peer that is gone - and the ring is marked failed.
//
// LBM-Bench has no decomposition (single-node OpenMP, src/main.c).
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>

#include "lbm_b200.h"
#include "lbm_internal.h"

using namespace lbm;

namespace {

// The NCCL entry points the ring uses (all present since NCCL 2.14).
struct NcclApi {
  void *h = nullptr;
  ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
  ncclResult_t (*init_rank_config)(ncclComm_t *, int, ncclUniqueId, int, ncclConfig_t *) = nullptr;
  ncclResult_t (*finalize)(ncclComm_t) = nullptr;
  ncclResult_t (*destroy)(ncclComm_t) = nullptr;
  ncclResult_t (*abort)(ncclComm_t) = nullptr;
  ncclResult_t (*async_error)(ncclComm_t, ncclResult_t *) = nullptr;
  ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*group_start)() = nullptr;
  ncclResult_t (*group_end)() = nullptr;
  const char *(*error_string)(ncclResult_t) = nullptr;
};

NcclApi g_api;
char g_load_err[384] = "";
std::once_flag g_once;

template <class F> bool bind(void *h, const char *name, F &f)
{
  f = reinterpret_cast<F>(dlsym(h, name));
  return f != nullptr;
}

void load_nccl()
{
  const char *env = getenv("LBM_B200_NCCL");
  const char *path = env && *env ? env : "libnccl.so.2";
  void *h = dlopen(path, RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    snprintf(g_load_err, sizeof g_load_err, "cannot load NCCL (%s): %s", path, dlerror());
    return;
  }
  NcclApi a;
  a.h = h;
  bool ok = bind(h, "ncclGetUniqueId", a.get_unique_id) &&
            bind(h, "ncclCommInitRankConfig", a.init_rank_config) &&
            bind(h, "ncclCommFinalize", a.finalize) && bind(h, "ncclCommDestroy", a.destroy) &&
            bind(h, "ncclCommAbort", a.abort) && bind(h, "ncclCommGetAsyncError", a.async_error) &&
            bind(h, "ncclSend", a.send) && bind(h, "ncclRecv", a.recv) &&
            bind(h, "ncclGroupStart", a.group_start) && bind(h, "ncclGroupEnd", a.group_end) &&
            bind(h, "ncclGetErrorString", a.error_string);
  if (!ok) {
    snprintf(g_load_err, sizeof g_load_err,
        "NCCL at %s lacks an entry point of the non-blocking API (2.14 or later needed)", path);
    dlclose(h);
    return;
  }
  g_api = a;
}

const NcclApi *nccl()
{
  std::call_once(g_once, load_nccl);
  return g_api.h ? &g_api : nullptr;
}

constexpr int kWindow = 16; // run loop: steps per window, two windows queued at most
constexpr int kDefaultTimeoutMs = 60000;

using Clock = std::chrono::steady_clock;

} // namespace

struct lbm_ring {
  lbm_solver *s = nullptr;
  const NcclApi *api = nullptr;
  ncclComm_t comm = nullptr; // nullptr: ring of one with device copies
  int rank = 0, nranks = 1, left = 0, right = 0;
  int planes = 0, device = 0;
  size_t bytes = 0;  // one message
  size_t stride = 0; // message slots, 256-byte aligned
  unsigned char *buf = nullptr; // to_left, to_right, from_left, from_right
  int timeout_ms = kDefaultTimeoutMs;
  int failed = 0;
  cudaEvent_t window_ev[2] = {nullptr, nullptr};
  cudaEvent_t sync_ev = nullptr;
  long long steps_issued = 0;
  long long exchanges = 0;

  void *slot(int i) const { return buf + (size_t)i * stride; }
};

namespace {

int ring_fail(lbm_ring *r, int code, const char *what, const char *detail)
{
  if (r->comm) {
    r->api->abort(r->comm);
    r->comm = nullptr;
  }
  r->failed = 1;
  return record_error(code, "%s: %s", what, detail);
}

double elapsed_ms(Clock::time_point t0)
{
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// Polls the communicator until no operation is in progress, bounded.
int wait_comm(lbm_ring *r, const char *what)
{
  auto t0 = Clock::now();
  for (;;) {
    ncclResult_t st = ncclSuccess;
    ncclResult_t rc = r->api->async_error(r->comm, &st);
    if (rc != ncclSuccess)
      st = rc;
    if (st == ncclSuccess)
      return LBM_OK;
    if (st != ncclInProgress)
      return ring_fail(r, LBM_ERR_COMM, what, r->api->error_string(st));
    if (elapsed_ms(t0) > r->timeout_ms) {
      char msg[128];
      snprintf(msg, sizeof msg, "no completion within %d ms (communicator aborted)", r->timeout_ms);
      return ring_fail(r, LBM_ERR_TIMEOUT, what, msg);
    }
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

// Waits for an event on the solver's stream, bounded, watching the
// communicator for asynchronous errors meanwhile.
int wait_event(lbm_ring *r, cudaEvent_t e, const char *what)
{
  auto t0 = Clock::now();
  for (;;) {
    cudaError_t q = cudaEventQuery(e);
    if (q == cudaSuccess)
      return LBM_OK;
    if (q != cudaErrorNotReady)
      return ring_fail(r, LBM_ERR_CUDA, what, cudaGetErrorString(q));
    if (r->comm) {
      ncclResult_t st = ncclSuccess;
      ncclResult_t rc = r->api->async_error(r->comm, &st);
      if (rc != ncclSuccess)
        st = rc;
      if (st != ncclSuccess && st != ncclInProgress)
        return ring_fail(r, LBM_ERR_COMM, what, r->api->error_string(st));
    }
    if (elapsed_ms(t0) > r->timeout_ms) {
      char msg[128];
      snprintf(msg, sizeof msg, "stream not done within %d ms (communicator aborted)",
          r->timeout_ms);
      return ring_fail(r, LBM_ERR_TIMEOUT, what, msg);
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

int usable(lbm_ring *r, const char *what)
{
  if (!r)
    return record_error(LBM_ERR_ARG, "%s: NULL ring", what);
  if (r->failed)
    return record_error(LBM_ERR_STATE, "%s: the ring failed earlier and must be destroyed", what);
  cudaError_t e = cudaSetDevice(r->device);
  if (e != cudaSuccess)
    return record_error(LBM_ERR_CUDA, "%s: cudaSetDevice: %s", what, cudaGetErrorString(e));
  return LBM_OK;
}

// One exchange: pack, move the two messages each way, unpack. Every rank
// posts send-right, send-left, receive-from-left, receive-from-right in
// this order, so with two ranks (both neighbours the same peer) the i-th
// send to a peer meets that peer's i-th receive from it: what travels right
// arrives as the receiver's from_left.
int exchange(lbm_ring *r, int when)
{
  cudaStream_t st = (cudaStream_t)lbm_stream(r->s);
  int rc = lbm_halo_pack(r->s, when, r->slot(0), r->slot(1));
  if (rc)
    return rc;
  if (!r->comm) {
    cudaError_t e = cudaMemcpyAsync(r->slot(2), r->slot(1), r->bytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(r->slot(3), r->slot(0), r->bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess)
      return ring_fail(r, LBM_ERR_CUDA, "lbm_ring exchange", cudaGetErrorString(e));
  } else {
    const NcclApi *a = r->api;
    ncclResult_t n = a->group_start();
    if (n == ncclSuccess || n == ncclInProgress)
      n = a->send(r->slot(1), r->bytes, ncclUint8, r->right, r->comm, st);
    if (n == ncclSuccess || n == ncclInProgress)
      n = a->send(r->slot(0), r->bytes, ncclUint8, r->left, r->comm, st);
    if (n == ncclSuccess || n == ncclInProgress)
      n = a->recv(r->slot(2), r->bytes, ncclUint8, r->left, r->comm, st);
    if (n == ncclSuccess || n == ncclInProgress)
      n = a->recv(r->slot(3), r->bytes, ncclUint8, r->right, r->comm, st);
    ncclResult_t g = a->group_end();
    if (n == ncclSuccess || n == ncclInProgress)
      n = g;
    if (n == ncclInProgress)
      rc = wait_comm(r, "lbm_ring exchange");
    else if (n != ncclSuccess)
      rc = ring_fail(r, LBM_ERR_COMM, "lbm_ring exchange", a->error_string(n));
    if (rc)
      return rc;
  }
  rc = lbm_halo_unpack(r->s, when, r->slot(2), r->slot(3));
  if (rc)
    return rc;
  ++r->exchanges;
  return LBM_OK;
}

int one_step(lbm_ring *r, int overlap)
{
  lbm_solver *s = r->s;
  int need = lbm_halo_needs(s);
  int rc;
  if (!overlap) {
    if ((need & LBM_HALO_BEFORE) && (rc = exchange(r, LBM_HALO_BEFORE)))
      return rc;
    if ((rc = lbm_run(s, 1)))
      return rc;
    if ((need & LBM_HALO_AFTER) && (rc = exchange(r, LBM_HALO_AFTER)))
      return rc;
    return LBM_OK;
  }
  // interior planes on the side stream, the exchanges and the boundary
  // planes on the solver's stream
  const int nx = r->planes;
  if ((rc = lbm_step_begin(s)))
    return rc;
  if (nx > 2 && (rc = lbm_step_planes(s, 1, nx - 1, 1)))
    return rc;
  if ((need & LBM_HALO_BEFORE) && (rc = exchange(r, LBM_HALO_BEFORE)))
    return rc;
  if ((rc = lbm_step_planes(s, 0, 1, 0)))
    return rc;
  if (nx > 1 && (rc = lbm_step_planes(s, nx - 1, nx, 0)))
    return rc;
  if ((need & LBM_HALO_AFTER) && (rc = exchange(r, LBM_HALO_AFTER)))
    return rc;
  return lbm_step_end(s);
}

} // namespace

extern "C" int lbm_ring_unique_id(unsigned char *id)
{
  if (!id)
    return record_error(LBM_ERR_ARG, "lbm_ring_unique_id: NULL id");
  const NcclApi *a = nccl();
  if (!a)
    return record_error(LBM_ERR_COMM, "lbm_ring_unique_id: %s", g_load_err);
  ncclUniqueId u;
  ncclResult_t n = a->get_unique_id(&u);
  if (n != ncclSuccess)
    return record_error(LBM_ERR_COMM, "lbm_ring_unique_id: %s", a->error_string(n));
  static_assert(sizeof(u.internal) == LBM_RING_ID_BYTES, "NCCL unique id size");
  memcpy(id, u.internal, LBM_RING_ID_BYTES);
  return LBM_OK;
}

extern "C" int lbm_ring_create(lbm_ring **out, lbm_solver *s, int rank, int nranks,
    const unsigned char *id, int timeout_ms)
{
  if (!out || !s)
    return record_error(LBM_ERR_ARG, "lbm_ring_create: NULL argument");
  *out = nullptr;
  if (nranks < 1 || rank < 0 || rank >= nranks || timeout_ms < 0)
    return record_error(LBM_ERR_ARG, "lbm_ring_create: rank %d of %d, timeout %d ms", rank,
        nranks, timeout_ms);
  if (!id && nranks != 1)
    return record_error(LBM_ERR_ARG, "lbm_ring_create: %d ranks need an NCCL id", nranks);
  size_t bytes = lbm_halo_bytes(s);
  if (bytes == 0)
    return record_error(LBM_ERR_ARG, "lbm_ring_create: not a slab solver (lbm_create_slab)");
  const NcclApi *a = nullptr;
  if (id && !(a = nccl()))
    return record_error(LBM_ERR_COMM, "lbm_ring_create: %s", g_load_err);

  lbm_ring *r = new (std::nothrow) lbm_ring;
  if (!r)
    return record_error(LBM_ERR_ALLOC, "lbm_ring_create: host allocation failed");
  r->s = s;
  r->api = a;
  r->rank = rank;
  r->nranks = nranks;
  r->left = (rank + nranks - 1) % nranks;
  r->right = (rank + 1) % nranks;
  r->planes = solver_planes(s);
  r->device = solver_device(s);
  r->bytes = bytes;
  r->stride = (bytes + 255) / 256 * 256;
  r->timeout_ms = timeout_ms ? timeout_ms : kDefaultTimeoutMs;

  int rc = LBM_OK;
  cudaError_t e = cudaSetDevice(r->device);
  if (e == cudaSuccess)
    e = cudaMalloc(&r->buf, 4 * r->stride);
  if (e == cudaSuccess)
    e = cudaMemset(r->buf, 0, 4 * r->stride);
  for (int i = 0; i < 2 && e == cudaSuccess; ++i)
    e = cudaEventCreateWithFlags(&r->window_ev[i], cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaEventCreateWithFlags(&r->sync_ev, cudaEventDisableTiming);
  if (e != cudaSuccess)
    rc = record_error(e == cudaErrorMemoryAllocation ? LBM_ERR_ALLOC : LBM_ERR_CUDA,
        "lbm_ring_create: %s", cudaGetErrorString(e));

  if (!rc && id) {
    ncclUniqueId u;
    memcpy(u.internal, id, LBM_RING_ID_BYTES);
    ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
    cfg.blocking = 0;
    ncclResult_t n = a->init_rank_config(&r->comm, nranks, u, rank, &cfg);
    if (n == ncclInProgress || (n == ncclSuccess && r->comm))
      rc = wait_comm(r, "lbm_ring_create");
    else
      rc = ring_fail(r, LBM_ERR_COMM, "lbm_ring_create", a->error_string(n));
  }
  if (rc) {
    lbm_ring_destroy(r);
    return rc;
  }
  *out = r;
  return LBM_OK;
}

extern "C" int lbm_ring_run(lbm_ring *r, int steps, int overlap)
{
  int rc = usable(r, "lbm_ring_run");
  if (rc)
    return rc;
  if (steps < 0)
    return record_error(LBM_ERR_ARG, "lbm_ring_run: %d steps", steps);
  cudaStream_t st = (cudaStream_t)lbm_stream(r->s);
  for (int i = 0; i < steps; ++i) {
    if (r->steps_issued % kWindow == 0) {
      // the event of two windows ago must have passed before a new window
      // is queued: the host never runs more than 2 * kWindow steps ahead,
      // and a peer that stopped is noticed within the timeout
      long long w = r->steps_issued / kWindow;
      cudaEvent_t e = r->window_ev[w & 1];
      if (w >= 2 && (rc = wait_event(r, e, "lbm_ring_run")))
        return rc;
      cudaError_t ce = cudaEventRecord(e, st);
      if (ce != cudaSuccess)
        return ring_fail(r, LBM_ERR_CUDA, "lbm_ring_run", cudaGetErrorString(ce));
    }
    if ((rc = one_step(r, overlap)))
      return rc;
    ++r->steps_issued;
  }
  return LBM_OK;
}

extern "C" int lbm_ring_gather(lbm_ring *r)
{
  int rc = usable(r, "lbm_ring_gather");
  if (rc)
    return rc;
  return lbm_halo_shifted(r->s) == 1 ? exchange(r, LBM_HALO_BEFORE) : LBM_OK;
}

extern "C" int lbm_ring_scatter(lbm_ring *r)
{
  int rc = usable(r, "lbm_ring_scatter");
  if (rc)
    return rc;
  return lbm_halo_shifted(r->s) == 1 ? exchange(r, LBM_HALO_SCATTER) : LBM_OK;
}

extern "C" int lbm_ring_synchronize(lbm_ring *r)
{
  int rc = usable(r, "lbm_ring_synchronize");
  if (rc)
    return rc;
  cudaError_t e = cudaEventRecord(r->sync_ev, (cudaStream_t)lbm_stream(r->s));
  if (e != cudaSuccess)
    return ring_fail(r, LBM_ERR_CUDA, "lbm_ring_synchronize", cudaGetErrorString(e));
  return wait_event(r, r->sync_ev, "lbm_ring_synchronize");
}

extern "C" long long lbm_ring_exchanges(const lbm_ring *r) { return r ? r->exchanges : -1; }

extern "C" int lbm_ring_uses_nccl(const lbm_ring *r) { return r ? (r->api ? 1 : 0) : -1; }

extern "C" int lbm_ring_destroy(lbm_ring *r)
{
  if (!r)
    return LBM_OK;
  int rc = LBM_OK;
  cudaSetDevice(r->device);
  if (!r->failed && r->sync_ev && r->steps_issued + r->exchanges > 0)
    rc = lbm_ring_synchronize(r); // bounded; aborts the communicator if a peer is gone
  if (r->comm && !r->failed) {
    ncclResult_t n = r->api->finalize(r->comm);
    if (n == ncclInProgress)
      rc = rc ? rc : wait_comm(r, "lbm_ring_destroy");
    else if (n != ncclSuccess && !rc)
      rc = ring_fail(r, LBM_ERR_COMM, "lbm_ring_destroy", r->api->error_string(n));
    if (r->comm) {
      r->api->destroy(r->comm);
      r->comm = nullptr;
    }
  }
  for (cudaEvent_t &ev : r->window_ev)
    if (ev)
      cudaEventDestroy(ev);
  if (r->sync_ev)
    cudaEventDestroy(r->sync_ev);
  if (r->buf)
    cudaFree(r->buf);
  delete r;
  return rc;
}
