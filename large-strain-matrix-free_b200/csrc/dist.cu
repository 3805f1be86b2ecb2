// Distributed (z-slab partitioned) operator application and CG: the
// reference's MPI pattern of NeoHookOperator::vmult (mf_nh_operator.h:
// 680-700: src.update_ghost_values(), cell loop, dst.compress(add)) and of
// SolverCG's all-reduced scalars (mf_elasticity.h:3175-3180), over one of two
// transports:
//   group  all parts driven from one process (one or several devices), the
//          interface buffers moved with cudaMemcpyAsync between the parts'
//          streams, reductions summed on the host in part order;
//   nccl   one part per process and GPU, ncclSend / ncclRecv to the two slab
//          neighbours and ncclAllReduce of the CG scalars (libnccl.so.2 is
//          loaded when such an object is created; the library has no link
//          dependency on it).
// Interface data move as packed buffers of 3 values per shared node in the
// order of the PartLayout lists, which both sides enumerate identically.
//
// Fused exchange (group transport, the default where every part can reach
// its upper neighbour's memory): no packed buffers at all.  Each part's cell
// loop runs on an index map in which its ghost nodes carry PEER_BIT and the
// upper neighbour's node numbers, so the interface cells read the owners'
// src values and add their contributions to the owners' dst over peer
// memory (NVLink P2P loads and atomics between GPUs; plain device memory
// when the parts share a GPU).  Ordering is by events between the parts'
// streams: part r's cell loop starts after part r + 1 has zeroed its dst,
// and part r + 1 continues after part r's cell loop.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "op_dispatch.h"
#include "solver_internal.h"

namespace lsmf {
namespace {

__global__ void pack_kernel(const double *__restrict__ v, const int *__restrict__ idx, int n,
                            const uint8_t *__restrict__ cmask, int zero_constrained, double *__restrict__ buf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x) {
    const size_t dof = 3 * (size_t)idx[i / 3] + i % 3;
    buf[i] = (zero_constrained && cmask[dof]) ? 0.0 : v[dof];
  }
}
// mode 0: v = buf; 1: v += buf; 2: v = 0
__global__ void unpack_kernel(double *__restrict__ v, const int *__restrict__ idx, int n,
                              const double *__restrict__ buf, int mode) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x) {
    const size_t dof = 3 * (size_t)idx[i / 3] + i % 3;
    if (mode == 0) v[dof] = buf[i];
    else if (mode == 1) v[dof] += buf[i];
    else v[dof] = 0.0;
  }
}
__global__ void invert_all_kernel(double *inv, const double *d, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    inv[i] = 1.0 / d[i];
}

// makes a part's device current for the scope (parts of a group may live
// on different GPUs; streams and allocations belong to their device)
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
    else if (prev == dev) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int grid_of(size_t n) {
  const size_t b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 1184 ? 1184 : b));
}

// the NCCL entry points used here, resolved from libnccl.so.2 at run time
struct Nccl {
  void *h = nullptr;
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
  bool load() {
    if (h) return true;
    h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return false;
    GetUniqueId = (decltype(GetUniqueId))dlsym(h, "ncclGetUniqueId");
    CommInitRank = (decltype(CommInitRank))dlsym(h, "ncclCommInitRank");
    CommDestroy = (decltype(CommDestroy))dlsym(h, "ncclCommDestroy");
    Send = (decltype(Send))dlsym(h, "ncclSend");
    Recv = (decltype(Recv))dlsym(h, "ncclRecv");
    AllReduce = (decltype(AllReduce))dlsym(h, "ncclAllReduce");
    GroupStart = (decltype(GroupStart))dlsym(h, "ncclGroupStart");
    GroupEnd = (decltype(GroupEnd))dlsym(h, "ncclGroupEnd");
    GetErrorString = (decltype(GetErrorString))dlsym(h, "ncclGetErrorString");
    return GetUniqueId && CommInitRank && CommDestroy && Send && Recv && AllReduce && GroupStart && GroupEnd &&
           GetErrorString;
  }
};
Nccl g_nccl;

#define LSMF_NCCL(...)                                                                   \
  do {                                                                                   \
    ncclResult_t r_ = (__VA_ARGS__);                                                     \
    if (r_ != ncclSuccess) {                                                             \
      ::lsmf::set_error(std::string(#__VA_ARGS__) + ": " + g_nccl.GetErrorString(r_));   \
      return LSMF_ERR_CUDA;                                                              \
    }                                                                                    \
  } while (0)

}  // namespace
}  // namespace lsmf

using namespace lsmf;

// one partition held by this object
struct lsmf_dist_part {
  lsmf_op *op = nullptr;
  int part = 0;
  int n_lower = 0, n_upper = 0;
  DevBuf<int> d_lower, d_upper;
  DevBuf<double> send_lo, send_up, recv_lo, recv_up;
  DevBuf<double> g, h, d, sc, partial, inv_diag;
  cudaEvent_t ev = nullptr;
  // fused exchange: the index map with the ghost nodes in the upper
  // neighbour's numbering (PEER_BIT set; parts with an upper neighbour), the
  // owned constrained dofs, and the events that order the neighbours' streams
  DevBuf<int> peer_nodes, con_owned;
  int n_con_owned = 0;
  cudaEvent_t ev_zero = nullptr, ev_done = nullptr;
  cudaStream_t stream() const { return op->stream; }
  size_t n() const { return (size_t)op->L().n_dofs(); }
  ~lsmf_dist_part() {
    for (cudaEvent_t e : {ev, ev_zero, ev_done})
      if (e) cudaEventDestroy(e);
  }
};

struct lsmf_dist {
  int n_parts = 1;
  bool nccl = false;
  bool fused_capable = false;  // group: peer maps built, every part reaches its upper neighbour
  bool fused = false;          // vmults use the fused exchange
  ncclComm_t comm = nullptr;
  std::vector<lsmf_dist_part *> parts;  // group: every part in order; nccl: this process's part
  ~lsmf_dist() {
    for (auto *p : parts) delete p;
    if (comm) g_nccl.CommDestroy(comm);
  }
};

namespace lsmf {
namespace {

lsmf_status init_part(lsmf_dist_part &P, lsmf_op *op) {
  if (!op || op->precision != LSMF_FP64) { set_error("distributed operators must be FP64"); return LSMF_ERR_INVALID_ARG; }
  const PartLayout &Lay = op->mesh->layout;
  if (op->level != (int)op->mesh->levels.size() - 1) { set_error("the operator must be on the finest level"); return LSMF_ERR_INVALID_ARG; }
  DeviceGuard dg(op->device);
  P.op = op;
  P.part = Lay.part;
  P.n_lower = (int)Lay.lower_shared.size();
  P.n_upper = (int)Lay.upper_shared.size();
  LSMF_TRY(P.d_lower.upload(Lay.lower_shared.data(), Lay.lower_shared.size()));
  LSMF_TRY(P.d_upper.upload(Lay.upper_shared.data(), Lay.upper_shared.size()));
  for (auto *b : {&P.send_lo, &P.recv_lo}) LSMF_TRY(b->alloc(3 * (size_t)P.n_lower + 1));
  for (auto *b : {&P.send_up, &P.recv_up}) LSMF_TRY(b->alloc(3 * (size_t)P.n_upper + 1));
  const size_t n = P.n();
  for (auto *b : {&P.g, &P.h, &P.d, &P.inv_diag}) LSMF_TRY(b->alloc(n));
  LSMF_TRY(P.sc.alloc(SC_N));
  LSMF_TRY(P.partial.alloc(reduce_blocks()));
  for (cudaEvent_t *e : {&P.ev, &P.ev_zero, &P.ev_done}) LSMF_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return LSMF_OK;
}

// run f(i, part) for every part this object holds, each with its device current
template <typename F>
lsmf_status each_part(lsmf_dist *D, F &&f) {
  for (size_t i = 0; i < D->parts.size(); ++i) {
    DeviceGuard dg(D->parts[i]->op->device);
    LSMF_TRY(f(i, *D->parts[i]));
  }
  return LSMF_OK;
}

lsmf_status pack(lsmf_dist_part &P, const double *v, bool upper, bool zero_constrained) {
  const int n = upper ? P.n_upper : P.n_lower;
  if (!n) return LSMF_OK;
  DeviceGuard dg(P.op->device);
  pack_kernel<<<grid_of(3 * (size_t)n), 256, 0, P.stream()>>>(v, upper ? P.d_upper.ptr : P.d_lower.ptr, n,
                                                                P.op->L().d_cmask.ptr, zero_constrained ? 1 : 0,
                                                                upper ? P.send_up.ptr : P.send_lo.ptr);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

lsmf_status unpack(lsmf_dist_part &P, double *v, bool upper, int mode) {
  const int n = upper ? P.n_upper : P.n_lower;
  if (!n) return LSMF_OK;
  DeviceGuard dg(P.op->device);
  unpack_kernel<<<grid_of(3 * (size_t)n), 256, 0, P.stream()>>>(v, upper ? P.d_upper.ptr : P.d_lower.ptr, n,
                                                                  upper ? P.recv_up.ptr : P.recv_lo.ptr, mode);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

// Move the packed interface buffers one slab down (send_lo of part r ->
// recv_up of part r - 1) or up (send_up of part r -> recv_lo of part r + 1).
lsmf_status transfer(lsmf_dist *D, bool down) {
  if (D->nccl) {
    lsmf_dist_part &P = *D->parts[0];
    const int r = P.part;
    LSMF_NCCL(g_nccl.GroupStart());
    if (down) {
      if (r > 0) LSMF_NCCL(g_nccl.Send(P.send_lo.ptr, 3 * (size_t)P.n_lower, ncclDouble, r - 1, D->comm, P.stream()));
      if (r < D->n_parts - 1)
        LSMF_NCCL(g_nccl.Recv(P.recv_up.ptr, 3 * (size_t)P.n_upper, ncclDouble, r + 1, D->comm, P.stream()));
    } else {
      if (r < D->n_parts - 1)
        LSMF_NCCL(g_nccl.Send(P.send_up.ptr, 3 * (size_t)P.n_upper, ncclDouble, r + 1, D->comm, P.stream()));
      if (r > 0) LSMF_NCCL(g_nccl.Recv(P.recv_lo.ptr, 3 * (size_t)P.n_lower, ncclDouble, r - 1, D->comm, P.stream()));
    }
    LSMF_NCCL(g_nccl.GroupEnd());
    return LSMF_OK;
  }
  // group: the receiving part's stream waits for the sender's pack, copies,
  // and the sender's stream waits for the copy before it may pack again
  LSMF_TRY(each_part(D, [&](size_t, lsmf_dist_part &P) -> lsmf_status {
    LSMF_CUDA(cudaEventRecord(P.ev, P.stream()));
    return LSMF_OK;
  }));
  std::vector<cudaEvent_t> done;
  lsmf_status st = each_part(D, [&](size_t r, lsmf_dist_part &Rv) -> lsmf_status {
    const int from = down ? (int)r + 1 : (int)r - 1;
    if (from < 0 || from >= D->n_parts) return LSMF_OK;
    lsmf_dist_part &Sd = *D->parts[from];
    const int n = down ? Rv.n_upper : Rv.n_lower;
    if ((down ? Sd.n_lower : Sd.n_upper) != n) { set_error("interface lists of neighbouring parts differ"); return LSMF_ERR_INVALID_ARG; }
    LSMF_CUDA(cudaStreamWaitEvent(Rv.stream(), Sd.ev, 0));
    if (n)
      LSMF_CUDA(cudaMemcpyAsync(down ? Rv.recv_up.ptr : Rv.recv_lo.ptr, down ? Sd.send_lo.ptr : Sd.send_up.ptr,
                                3 * (size_t)n * sizeof(double), cudaMemcpyDefault, Rv.stream()));
    cudaEvent_t e;
    LSMF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    done.push_back(e);
    LSMF_CUDA(cudaEventRecord(e, Rv.stream()));
    return LSMF_OK;
  });
  size_t k = 0;
  if (st == LSMF_OK)
    st = each_part(D, [&](size_t r, lsmf_dist_part &) -> lsmf_status {
      const int from = down ? (int)r + 1 : (int)r - 1;
      if (from < 0 || from >= D->n_parts) return LSMF_OK;
      // (a stream may wait on an event of another device)
      LSMF_CUDA(cudaStreamWaitEvent(D->parts[from]->stream(), done[k++], 0));
      return LSMF_OK;
    });
  for (cudaEvent_t e : done) cudaEventDestroy(e);
  return st;
}

// sum the scalar slot over all parts (every part holds the total afterwards)
lsmf_status allreduce(lsmf_dist *D, int slot) {
  if (D->nccl) {
    lsmf_dist_part &P = *D->parts[0];
    LSMF_NCCL(g_nccl.AllReduce(P.sc.ptr + slot, P.sc.ptr + slot, 1, ncclDouble, ncclSum, D->comm, P.stream()));
    return LSMF_OK;
  }
  double s = 0;
  LSMF_TRY(each_part(D, [&](size_t, lsmf_dist_part &P) -> lsmf_status {
    double v = 0;
    LSMF_CUDA(cudaMemcpyAsync(&v, P.sc.ptr + slot, sizeof(double), cudaMemcpyDeviceToHost, P.stream()));
    LSMF_CUDA(cudaStreamSynchronize(P.stream()));
    s += v;
    return LSMF_OK;
  }));
  LSMF_TRY(each_part(D, [&](size_t, lsmf_dist_part &P) -> lsmf_status {
    LSMF_CUDA(cudaMemcpyAsync(P.sc.ptr + slot, &s, sizeof(double), cudaMemcpyHostToDevice, P.stream()));
    return LSMF_OK;
  }));
  return each_part(D, [&](size_t, lsmf_dist_part &P) -> lsmf_status {
    LSMF_CUDA(cudaStreamSynchronize(P.stream()));
    return LSMF_OK;
  });
}

// ghost entries (upper-shared nodes) of v from their owners
lsmf_status update_ghosts(lsmf_dist *D, double *const *v) {
  for (size_t i = 0; i < D->parts.size(); ++i) LSMF_TRY(pack(*D->parts[i], v[i], false, false));
  LSMF_TRY(transfer(D, true));
  for (size_t i = 0; i < D->parts.size(); ++i) LSMF_TRY(unpack(*D->parts[i], v[i], true, 0));
  return LSMF_OK;
}

// compress(add): the ghosts' partial sums (constrained entries dropped: their
// rows are the identity on the owner) are added on the owners and the ghost
// entries cleared
lsmf_status compress_add(lsmf_dist *D, double *const *v) {
  for (size_t i = 0; i < D->parts.size(); ++i) {
    LSMF_TRY(pack(*D->parts[i], v[i], true, true));
    LSMF_TRY(unpack(*D->parts[i], v[i], true, 2));
  }
  LSMF_TRY(transfer(D, false));
  for (size_t i = 0; i < D->parts.size(); ++i) LSMF_TRY(unpack(*D->parts[i], v[i], false, 1));
  return LSMF_OK;
}

// Build the fused exchange of a group: every part's upper neighbour must be
// reachable (same GPU, or peer access enabled between the two GPUs); the
// index map of a part with an upper neighbour renumbers its ghost nodes
// into the neighbour's numbering (the interface lists of both sides are in
// the same order).  Leaves D->fused_capable false when it does not apply.
lsmf_status setup_fused(lsmf_dist *D) {
  const int n = (int)D->parts.size();
  if (D->nccl || n < 2) return LSMF_OK;
  for (int r = 0; r + 1 < n; ++r) {
    const int da = D->parts[r]->op->device, db = D->parts[r + 1]->op->device;
    if (da == db) continue;
    int can = 0;
    LSMF_CUDA(cudaDeviceCanAccessPeer(&can, da, db));
    if (!can) return LSMF_OK;
    DeviceGuard dg(da);
    const cudaError_t e = cudaDeviceEnablePeerAccess(db, 0);
    if (e == cudaErrorPeerAccessAlreadyEnabled) (void)cudaGetLastError();
    else if (e != cudaSuccess) { (void)cudaGetLastError(); return LSMF_OK; }
  }
  for (int r = 0; r < n; ++r) {
    lsmf_dist_part &P = *D->parts[r];
    const Level &L = P.op->L();
    if (L.n_nodes > PEER_NODE_MASK) return LSMF_OK;
    const PartLayout &Lay = P.op->mesh->layout;
    std::vector<int> ghost_of(L.n_nodes, -1);
    for (size_t j = 0; j < Lay.upper_shared.size(); ++j) ghost_of[Lay.upper_shared[j]] = (int)j;
    DeviceGuard dg(P.op->device);
    // identity rows of the owned constrained dofs (a ghost's row is its owner's)
    std::vector<int> con;
    for (int dof : L.constrained)
      if (ghost_of[dof / 3] < 0) con.push_back(dof);
    P.n_con_owned = (int)con.size();
    LSMF_TRY(P.con_owned.upload(con.data(), con.size()));
    if (r + 1 == n) continue;
    const std::vector<int> &owner = D->parts[r + 1]->op->mesh->layout.lower_shared;
    if (owner.size() != Lay.upper_shared.size()) { set_error("interface lists of neighbouring parts differ"); return LSMF_ERR_INVALID_ARG; }
    std::vector<int> packed(L.cell_nodes.size());
    for (size_t i = 0; i < packed.size(); ++i) {
      const int node = L.cell_nodes[i];
      const int cm = L.cmask[3 * (size_t)node] | (L.cmask[3 * (size_t)node + 1] << 1) |
                     (L.cmask[3 * (size_t)node + 2] << 2);
      const int j = ghost_of[node];
      packed[i] = (j < 0 ? node : (PEER_BIT | owner[j])) | (cm << NODE_BITS);
    }
    LSMF_TRY(P.peer_nodes.upload(packed.data(), packed.size()));
  }
  D->fused_capable = true;
  D->fused = true;
  return LSMF_OK;
}

// the fused exchange serves operators with the fast kernel and atomic scatter
bool fused_applies(const lsmf_dist *D) {
  if (!D->fused) return false;
  for (auto *P : D->parts)
    if (P->op->basic || P->op->scatter != LSMF_SCATTER_ATOMIC) return false;
  return true;
}

// dst = A src with the interface exchange done by the cell loops (fused):
// zero every dst; part r's cell loop, once part r + 1 has zeroed its dst,
// gathers its ghosts from src[r + 1] and adds their contributions to
// dst[r + 1]; part r + 1 continues after it.  dst's ghost entries stay zero
// and src's ghost entries are not read.
lsmf_status dist_vmult_fused(lsmf_dist *D, double *const *dst, double *const *src) {
  const int n = (int)D->parts.size();
  LSMF_TRY(each_part(D, [&](size_t r, lsmf_dist_part &P) -> lsmf_status {
    LSMF_CUDA(cudaMemsetAsync(dst[r], 0, P.n() * sizeof(double), P.stream()));
    LSMF_CUDA(cudaEventRecord(P.ev_zero, P.stream()));
    return LSMF_OK;
  }));
  LSMF_TRY(each_part(D, [&](size_t r, lsmf_dist_part &P) -> lsmf_status {
    if ((int)r + 1 < n) {
      lsmf_dist_part &U = *D->parts[r + 1];
      LSMF_CUDA(cudaStreamWaitEvent(P.stream(), U.ev_zero, 0));
      CellRange rg;
      rg.peer_nodes = P.peer_nodes.ptr;
      rg.peer_src = src[r + 1];
      rg.peer_dst = dst[r + 1];
      rg.peer_u = U.op->d_u;
      LSMF_TRY(launch_apply_peer(P.op, dst[r], src[r], rg, P.con_owned.ptr, P.n_con_owned));
    } else {
      // the top part has no ghosts: the plain cell loop, dst already zero
      LSMF_TRY(launch_apply(P.op, dst[r], src[r], LSMF_MASK_DEFAULT, true));
    }
    LSMF_CUDA(cudaEventRecord(P.ev_done, P.stream()));
    return LSMF_OK;
  }));
  return each_part(D, [&](size_t r, lsmf_dist_part &P) -> lsmf_status {
    if (r > 0) LSMF_CUDA(cudaStreamWaitEvent(P.stream(), D->parts[r - 1]->ev_done, 0));
    return LSMF_OK;
  });
}

lsmf_status dist_vmult(lsmf_dist *D, double *const *dst, double *const *src) {
  if (fused_applies(D)) return dist_vmult_fused(D, dst, src);
  LSMF_TRY(update_ghosts(D, src));
  LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
    return launch_apply(P.op, dst[i], src[i], LSMF_MASK_DEFAULT, false);
  }));
  return compress_add(D, dst);
}

}  // namespace
}  // namespace lsmf

extern "C" {

lsmf_status lsmf_dist_create_group(int n_parts, lsmf_op *const *ops, lsmf_dist **out) {
  if (!ops || !out || n_parts < 1) { set_error("bad arguments"); return LSMF_ERR_INVALID_ARG; }
  *out = nullptr;
  lsmf_dist *D = new (std::nothrow) lsmf_dist();
  if (!D) return LSMF_ERR_ALLOC;
  D->n_parts = n_parts;
  for (int r = 0; r < n_parts; ++r) {
    if (!ops[r] || (n_parts > 1 && (ops[r]->mesh->layout.n_parts != n_parts || ops[r]->mesh->layout.part != r))) {
      set_error("ops[r] must be the operator of part r of an n_parts partition");
      delete D;
      return LSMF_ERR_INVALID_ARG;
    }
    D->parts.push_back(new lsmf_dist_part());
    lsmf_status s = init_part(*D->parts.back(), ops[r]);
    if (s != LSMF_OK) { delete D; return s; }
  }
  lsmf_status s = setup_fused(D);
  if (s != LSMF_OK) { delete D; return s; }
  *out = D;
  return LSMF_OK;
}

lsmf_status lsmf_dist_set_exchange(lsmf_dist *D, int mode) {
  if (!D || (mode != LSMF_DIST_EXCHANGE_PACKED && mode != LSMF_DIST_EXCHANGE_FUSED)) {
    set_error("bad arguments");
    return LSMF_ERR_INVALID_ARG;
  }
  if (mode == LSMF_DIST_EXCHANGE_FUSED && !D->fused_capable) {
    set_error("the fused exchange needs every part in this process with its upper neighbour reachable (same GPU "
              "or peer access) and fewer than 2^28 nodes per part");
    return LSMF_ERR_UNSUPPORTED;
  }
  D->fused = mode == LSMF_DIST_EXCHANGE_FUSED;
  return LSMF_OK;
}

lsmf_status lsmf_dist_get_exchange(const lsmf_dist *D, int *mode) {
  if (!D || !mode) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  *mode = fused_applies(D) ? LSMF_DIST_EXCHANGE_FUSED : LSMF_DIST_EXCHANGE_PACKED;
  return LSMF_OK;
}

lsmf_status lsmf_dist_nccl_unique_id(unsigned char *id128) {
  if (!id128) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!g_nccl.load()) { set_error("libnccl.so.2 could not be loaded"); return LSMF_ERR_UNSUPPORTED; }
  ncclUniqueId id;
  LSMF_NCCL(g_nccl.GetUniqueId(&id));
  static_assert(sizeof(id) == 128, "ncclUniqueId is 128 bytes");
  std::memcpy(id128, &id, sizeof(id));
  return LSMF_OK;
}

lsmf_status lsmf_dist_create_nccl(lsmf_op *op, const unsigned char *id128, lsmf_dist **out) {
  if (!op || !id128 || !out) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  *out = nullptr;
  if (!g_nccl.load()) { set_error("libnccl.so.2 could not be loaded"); return LSMF_ERR_UNSUPPORTED; }
  const PartLayout &Lay = op->mesh->layout;
  lsmf_dist *D = new (std::nothrow) lsmf_dist();
  if (!D) return LSMF_ERR_ALLOC;
  D->n_parts = Lay.n_parts;
  D->nccl = true;
  D->parts.push_back(new lsmf_dist_part());
  lsmf_status s = init_part(*D->parts[0], op);
  if (s != LSMF_OK) { delete D; return s; }
  ncclUniqueId id;
  std::memcpy(&id, id128, sizeof(id));
  DeviceGuard dg(op->device);
  const ncclResult_t r = g_nccl.CommInitRank(&D->comm, Lay.n_parts, id, Lay.part);
  if (r != ncclSuccess) {
    set_error(std::string("ncclCommInitRank: ") + g_nccl.GetErrorString(r));
    D->comm = nullptr;
    delete D;
    return LSMF_ERR_CUDA;
  }
  *out = D;
  return LSMF_OK;
}

void lsmf_dist_destroy(lsmf_dist *d) { delete d; }

lsmf_status lsmf_dist_vmult(lsmf_dist *D, double *const *dst, double *const *src) {
  if (!D || !dst || !src) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  for (auto *P : D->parts)
    if (!P->op->cached) { set_error("cache() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  return dist_vmult(D, dst, src);
}

lsmf_status lsmf_dist_dot(lsmf_dist *D, const double *const *a, const double *const *b, double *out) {
  if (!D || !a || !b || !out) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  // owned entries only: b is copied into a work vector whose ghost entries
  // are cleared, so each part sums over the entries it owns
  LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
    LSMF_CUDA(cudaMemcpyAsync(P.g.ptr, b[i], P.n() * sizeof(double), cudaMemcpyDeviceToDevice, P.stream()));
    LSMF_TRY(pack(P, P.g.ptr, true, false));
    LSMF_TRY(unpack(P, P.g.ptr, true, 2));
    return dot_async(a[i], P.g.ptr, false, P.n(), P.partial.ptr, P.sc.ptr, SC_TMP, P.stream());
  }));
  LSMF_TRY(allreduce(D, SC_TMP));
  lsmf_dist_part &P0 = *D->parts[0];
  DeviceGuard dg(P0.op->device);
  LSMF_CUDA(cudaMemcpyAsync(out, P0.sc.ptr + SC_TMP, sizeof(double), cudaMemcpyDeviceToHost, P0.stream()));
  LSMF_CUDA(cudaStreamSynchronize(P0.stream()));
  return LSMF_OK;
}

// SolverCG over the partitions (deal.II form, as lsmf_cg_solve): the ghost
// entries of g and h are kept zero, so each part's dot products are sums over
// its owned entries and one all-reduce completes them.
lsmf_status lsmf_dist_cg_solve(lsmf_dist *D, int precond, double omega, double *const *x, const double *const *b,
                               double tol_abs, int max_it, lsmf_solve_info *info) {
  if (!D || !x || !b) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (precond != 0 && precond != 1) { set_error("distributed CG supports precond 0 (none) and 1 (Jacobi)"); return LSMF_ERR_UNSUPPORTED; }
  const size_t np = D->parts.size();
  for (auto *P : D->parts)
    if (!P->op->cached) { set_error("cache() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  std::vector<double *> g(np), h(np), d(np), invd(np);
  for (size_t i = 0; i < np; ++i) {
    g[i] = D->parts[i]->g.ptr; h[i] = D->parts[i]->h.ptr; d[i] = D->parts[i]->d.ptr; invd[i] = D->parts[i]->inv_diag.ptr;
  }
  if (precond == 1) {
    // the diagonal of the whole operator on the owned entries: each part's
    // cell contributions, compress(add) across the interfaces, then inverted
    LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
      LSMF_TRY(lsmf_operator_compute_diagonal(P.op));
      LSMF_CUDA(cudaMemcpyAsync(h[i], P.op->d_diag.ptr, P.n() * sizeof(double), cudaMemcpyDeviceToDevice, P.stream()));
      return LSMF_OK;
    }));
    LSMF_TRY(compress_add(D, h.data()));
    LSMF_TRY(update_ghosts(D, h.data()));
    LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
      invert_all_kernel<<<grid_of(P.n()), 256, 0, P.stream()>>>(invd[i], h[i], P.n());
      LSMF_CUDA(cudaGetLastError());
      return LSMF_OK;
    }));
  }
  auto prec = [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
    if (precond == 0) {
      LSMF_CUDA(cudaMemcpyAsync(h[i], g[i], P.n() * sizeof(double), cudaMemcpyDeviceToDevice, P.stream()));
      return LSMF_OK;
    }
    return jacobi_async<double>(h[i], invd[i], g[i], omega, P.n(), P.stream());
  };
  auto read = [&](int slot, double &v) -> lsmf_status {
    lsmf_dist_part &P = *D->parts[0];
    DeviceGuard dg(P.op->device);
    LSMF_CUDA(cudaMemcpyAsync(&v, P.sc.ptr + slot, sizeof(double), cudaMemcpyDeviceToHost, P.stream()));
    LSMF_CUDA(cudaStreamSynchronize(P.stream()));
    return LSMF_OK;
  };
  // g = A x - b with zero ghost entries
  LSMF_TRY(dist_vmult(D, h.data(), x));
  LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
    LSMF_TRY(neg_residual_async<double>(g[i], h[i], b[i], P.n(), P.stream()));
    LSMF_TRY(pack(P, g[i], true, false));
    LSMF_TRY(unpack(P, g[i], true, 2));
    return dot_async(g[i], g[i], false, P.n(), P.partial.ptr, P.sc.ptr, SC_RES2, P.stream());
  }));
  LSMF_TRY(allreduce(D, SC_RES2));
  double res2 = 0;
  LSMF_TRY(read(SC_RES2, res2));
  double res = std::sqrt(res2);
  int it = 0;
  bool conv = res <= tol_abs;
  if (!conv && max_it > 0) {
    LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
      LSMF_TRY(prec(i, P));
      return dot_async(g[i], h[i], false, P.n(), P.partial.ptr, P.sc.ptr, SC_GH0, P.stream());
    }));
    LSMF_TRY(allreduce(D, SC_GH0));
    LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
      return cg_dir_async(d[i], h[i], P.n(), P.sc.ptr, SC_GH0, SC_GH0, true, P.stream());
    }));
    int k = 0;
    while (true) {
      ++it;
      LSMF_TRY(dist_vmult(D, h.data(), d.data()));
      LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
        return dot_async(d[i], h[i], false, P.n(), P.partial.ptr, P.sc.ptr, SC_DH, P.stream());
      }));
      LSMF_TRY(allreduce(D, SC_DH));
      LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
        return cg_update_async(x[i], g[i], d[i], h[i], P.n(), P.sc.ptr, SC_GH0 + (k & 1), P.partial.ptr, P.stream());
      }));
      LSMF_TRY(allreduce(D, SC_RES2));
      LSMF_TRY(read(SC_RES2, res2));
      res = std::sqrt(res2);
      if (!(res == res)) break;
      if (res <= tol_abs) { conv = true; break; }
      if (it >= max_it) break;
      LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
        LSMF_TRY(prec(i, P));
        return dot_async(g[i], h[i], false, P.n(), P.partial.ptr, P.sc.ptr, SC_GH0 + ((k + 1) & 1), P.stream());
      }));
      LSMF_TRY(allreduce(D, SC_GH0 + ((k + 1) & 1)));
      LSMF_TRY(each_part(D, [&](size_t i, lsmf_dist_part &P) -> lsmf_status {
        return cg_dir_async(d[i], h[i], P.n(), P.sc.ptr, SC_GH0 + ((k + 1) & 1), SC_GH0 + (k & 1), false, P.stream());
      }));
      ++k;
    }
  }
  // the owners' values in the ghost entries of the solution
  LSMF_TRY(update_ghosts(D, x));
  LSMF_TRY(each_part(D, [&](size_t, lsmf_dist_part &P) -> lsmf_status {
    LSMF_CUDA(cudaStreamSynchronize(P.stream()));
    return LSMF_OK;
  }));
  if (info) { info->iterations = it; info->residual = res; info->converged = conv ? 1 : 0; }
  if (!conv) { set_error("CG did not reach the tolerance"); return LSMF_ERR_CG_NOT_CONVERGED; }
  return LSMF_OK;
}

}  // extern "C"
