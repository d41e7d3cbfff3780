// api.cu -- the C ABI (include/fmm_b200.h): contexts, fmm!, direct!, parity
// exports and single-operator entry points.
//
// fmm_solve follows the reference driver (src/fmm.jl:807-1176): trees for the
// targets and the sources, interaction lists, the influence estimate for the
// relative error methods, then nearfield -> upward -> horizontal -> downward
// passes and the unsort of the target buffer.  The trees, the lists, the near field
// and the unsort run on the context's stream; the far field (upward pass, M2L,
// downward pass) runs on a second high-priority stream concurrently with the near
// field, and the influence estimate's sub-solve on a third; the tree and list
// builders synchronise with the host once per level (trees) or per build (lists).
#include <algorithm>
#include <cstring>
#include <string>

#include <cub/cub.cuh>

#include "context.cuh"

using namespace fmmb;

namespace {

// One source system's bodies inside a tuple's shared octree (Tree(systems::Tuple, ...),
// src/tree.jl:3-122 keeps one buffer per system and per branch one body range per system):
// the system's bodies in tree order, and per branch the range of them it holds.
struct SysView {
  int kind = FMM_POINT_SOURCE;
  int64_t n = 0;
  DevBuf<double4> pos, str;
  DevBuf<int> start, count, pre;
};

struct Workspace {
  DevTree tree[2];  // [0] target role, [1] source role (aliased when shared)
  DevLists lists;
  DevBuf<int> sys_orig, sys_sorted;  // tuples: system of every source body (input / tree order)
  SysView views[8];
  DevBuf<double> acc13;      // target buffer rows 4..16, sorted order: near field (the whole field
                             // when the far field runs on the same stream)
  DevBuf<double> acc13_far;  // far field (L2P) when it runs on the far-field stream
  bool shared = false;
  DevTree& target() { return shared ? tree[1] : tree[0]; }
  DevTree& source() { return tree[1]; }
};

// far (may be null): the far field of the solve, added to the near field here with the
// single addition the L2P makes when it accumulates into the near-field rows itself
__global__ void k_unsort(const double* __restrict__ acc13, const int* __restrict__ sort_index,
                         const double4* __restrict__ pos, int64_t n, double* __restrict__ out16,
                         const double* __restrict__ far = nullptr) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t o = sort_index ? sort_index[i] : i;
    double4 p = pos[i];
    double* d = out16 + 16 * o;
    d[0] = p.x;
    d[1] = p.y;
    d[2] = p.z;
    const double* a = acc13 + 13 * i;
    if (far) {
      const double* f = far + 13 * i;
#pragma unroll
      for (int k = 0; k < 13; ++k) d[3 + k] = a[k] + f[k];
    } else {
#pragma unroll
      for (int k = 0; k < 13; ++k) d[3 + k] = a[k];
    }
  }
}

// the influence estimate's output: |grad| of every body in the caller's order (the
// one quantity the relative error methods read, get_influence, src/fmm.jl:1180-1183)
// get_influence (src/fmm.jl:1180-1187) per body, caller's order: |gradient|, or the scalar
// potential itself (potential != 0, PowerRelativePotential)
__global__ void k_unsort_gradnorm(const double* __restrict__ acc13, const int* __restrict__ sort_index, int64_t n,
                                  double* __restrict__ gnorm, int potential = 0) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* a = acc13 + 13 * i;
    gnorm[sort_index ? sort_index[i] : i] = potential ? a[0] : sqrt(a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
  }
}

// rows of the target buffer whose cotangents the adjoint does not propagate: the gradient and
// Hessian of point sources (they would need dipole sources), the potential row and the
// velocity gradient of vortex particles
__device__ __host__ inline bool vjp_unsupported_row(int kind, int r) {
  return kind == FMM_POINT_SOURCE ? r >= 4 : (r == 3 || r >= 7);
}

__global__ void k_check_cotangents(int64_t n, int kind, const double* __restrict__ dout16, int* __restrict__ flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 16 * n; i += (int64_t)gridDim.x * blockDim.x)
    if (vjp_unsupported_row(kind, (int)(i % 16)) && dout16[i] != 0.0) atomicExch(flag, 1);
}

// tuple of systems: system k's bodies into the shared body arrays at offset off (rows of
// the reference buffer: x, y, z, radius, strength), with the system index of each
__global__ void k_unpack_system(const double* __restrict__ buf, int64_t n, int d, int kind, int64_t off, int k,
                                double4* __restrict__ pos, double4* __restrict__ str, int* __restrict__ sys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* b = buf + i * d;
    pos[off + i] = make_double4(b[0], b[1], b[2], b[3]);
    str[off + i] = kind == FMM_POINT_VORTEX ? make_double4(b[4], b[5], b[6], 0.0) : make_double4(b[4], 0.0, 0.0, 0.0);
    sys[off + i] = k;
  }
}

__global__ void k_gather_int(const int* __restrict__ in, const int* __restrict__ idx, int64_t n, int* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[idx[i]];
}

__global__ void k_flag_system(const int* __restrict__ sys, int64_t n, int k, int* __restrict__ flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = i < n && sys[i] == k;
}

// system k's bodies in tree order (pre = exclusive count of its bodies before each position)
__global__ void k_split_system(const int* __restrict__ sys, const int* __restrict__ pre, int64_t n, int k,
                               const double4* __restrict__ pos, const double4* __restrict__ str,
                               double4* __restrict__ pos_k, double4* __restrict__ str_k) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (sys[i] == k) {
      pos_k[pre[i]] = pos[i];
      str_k[pre[i]] = str[i];
    }
}

// per branch, the range of system k's bodies (contiguous in its tree-ordered array)
__global__ void k_branch_ranges(const int* __restrict__ body_start, const int* __restrict__ body_count, int nb,
                                const int* __restrict__ pre, int* __restrict__ start, int* __restrict__ count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    const int a = pre[body_start[i]], e = pre[body_start[i] + body_count[i]];
    start[i] = a;
    count[i] = e - a;
  }
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }

// out += in on rows 4..16 of the target buffer (rows 1..3 are the positions)
__global__ void k_add_rows(int64_t n, const double* __restrict__ in, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 13 * n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / 13, r = 3 + i % 13;
    out[16 * b + r] += in[16 * b + r];
  }
}

// adjoint sources: at the targets (or the sources themselves), strengths = cotangents
__global__ void k_adj_sources(int64_t n, const double* __restrict__ pos, int64_t stride, bool radius_from_pos,
                              const double* __restrict__ dout16, int kind, double* __restrict__ buf) {
  const int d = kind == FMM_POINT_SOURCE ? 5 : 7;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double* b = buf + d * i;
    const double* x = pos + stride * i;
    b[0] = x[0];
    b[1] = x[1];
    b[2] = x[2];
    b[3] = radius_from_pos ? x[3] : 0.0;
    if (kind == FMM_POINT_SOURCE) {
      b[4] = dout16[16 * i + 3];
    } else {
      b[4] = dout16[16 * i + 4];
      b[5] = dout16[16 * i + 5];
      b[6] = dout16[16 * i + 6];
    }
  }
}

// dL/dstrength and dL/dx at the sources from the adjoint solve (adj16, at the sources)
// and, when the sources are the targets, the forward solve and the cotangents
__global__ void k_vjp_sources(int64_t n, int kind, const double* __restrict__ src, int d,
                              const double* __restrict__ adj16, const double* __restrict__ fwd16,
                              const double* __restrict__ dout16, double* __restrict__ dstr,
                              double* __restrict__ dpos) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* a = adj16 + 16 * i;
    if (kind == FMM_POINT_SOURCE) {
      const double q = src[d * i + 4];
      dstr[i] = a[3];
      for (int k = 0; k < 3; ++k) {
        double v = -q * a[4 + k];
        if (fwd16) v += dout16[16 * i + k] - dout16[16 * i + 3] * fwd16[16 * i + 4 + k];
        dpos[3 * i + k] = v;
      }
    } else {
      const double* G = src + d * i + 4;
      for (int c = 0; c < 3; ++c) dstr[3 * i + c] = a[4 + c];
      for (int k = 0; k < 3; ++k) {
        double v = 0.0;
        for (int c = 0; c < 3; ++c) v += G[c] * a[7 + c + 3 * k];
        if (fwd16) {
          v += dout16[16 * i + k];
          for (int c = 0; c < 3; ++c) v += dout16[16 * i + 4 + c] * fwd16[16 * i + 7 + c + 3 * k];
        }
        dpos[3 * i + k] = v;
      }
    }
  }
}

// dL/dy at a separate target system, from the forward solve (rows 1..3 of the target
// buffer are the target positions themselves: their cotangents pass through)
__global__ void k_vjp_targets(int64_t n, int kind, const double* __restrict__ fwd16, const double* __restrict__ dout16,
                              double* __restrict__ dtp) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* f = fwd16 + 16 * i;
    const double* w = dout16 + 16 * i;
    for (int k = 0; k < 3; ++k) {
      double v = w[k];
      if (kind == FMM_POINT_SOURCE)
        v -= w[3] * f[4 + k];
      else
        for (int c = 0; c < 3; ++c) v += w[4 + c] * f[7 + c + 3 * k];
      dtp[3 * i + k] = v;
    }
  }
}

}  // namespace

struct fmm_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool timing = false;
  size_t budget = 0;
  std::string err;
  Workspace main, est;
  Scratch sc;
  DevTables tables;
  DevBuf<double> stage_s, stage_t, out16, est_out16;
  DevBuf<double> adj_src, adj_out16, stage_d, vjp_out;  // fmm_vjp
  DevBuf<double> multi16;                                // fmm_solve_multi
  // influence estimate on its own stream (run_fmm)
  cudaStream_t est_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // far field (upward, M2L, downward) on its own stream, concurrent with the near field
  cudaStream_t far_stream = nullptr;
  cudaEvent_t ev_far = nullptr, ev_up = nullptr;
  Scratch est_sc;
  DevBuf<int> est_stats;
  DevBuf<int> stats;
  bool have_solve = false;
  int last_p = 0;
  int last_kind = 1;
  void* serve = nullptr;  // serving state (serve.cpp)
};

namespace {
cudaStream_t est_stream(fmm_ctx* c) {
  if (!c->est_stream) {
    int least = 0, greatest = 0;
    FMM_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    FMM_CUDA_TRY(cudaStreamCreateWithPriority(&c->est_stream, cudaStreamNonBlocking, greatest));
  }
  return c->est_stream;
}
cudaEvent_t fork_event(fmm_ctx* c) {
  if (!c->ev_fork) FMM_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  return c->ev_fork;
}
cudaEvent_t join_event(fmm_ctx* c) {
  if (!c->ev_join) FMM_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  return c->ev_join;
}
// one priority level below the influence estimate's stream (when the device has one):
// the M2L waits for the estimate, so the estimate's kernels go first
cudaStream_t far_stream(fmm_ctx* c) {
  if (!c->far_stream) {
    int least = 0, greatest = 0;
    FMM_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const int prio = greatest < least ? greatest + 1 : greatest;
    FMM_CUDA_TRY(cudaStreamCreateWithPriority(&c->far_stream, cudaStreamNonBlocking, prio));
  }
  return c->far_stream;
}
cudaEvent_t far_event(fmm_ctx* c) {
  if (!c->ev_far) FMM_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_far, cudaEventDisableTiming));
  return c->ev_far;
}
cudaEvent_t up_event(fmm_ctx* c) {
  if (!c->ev_up) FMM_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_up, cudaEventDisableTiming));
  return c->ev_up;
}
Scratch& est_scratch(fmm_ctx* c) { return c->est_sc; }
DevBuf<int>& est_stats(fmm_ctx* c) { return c->est_stats; }
}  // namespace

namespace fmmb {
void*& ctx_serve_slot(fmm_ctx* c) { return c->serve; }
int ctx_device(fmm_ctx* c) { return c->device; }
// device memory of a request's solve (an estimate from its sizes and options) and the
// release of a context's device buffers (serving: memory handed back to the shared account)
size_t request_footprint(const fmm_request* r);
void ctx_release_buffers(fmm_ctx* c);
}  // namespace fmmb

namespace {

int fail(fmm_ctx* c, const Error& e) {
  if (c) c->err = e.msg;
  return e.code;
}

constexpr int kMaxSystems = 8;  // source systems of one tuple

struct SysIn {
  const double* buf;  // device, body-major d*n
  int d;
  int kind;
  int64_t n;
};

struct SolveIn {
  const double* src;  // device, body-major d*n_s
  int d;
  int kind;
  int64_t n_s;
  const double* tpos;  // device, stride (nullptr: the sources are the targets)
  int64_t t_stride;
  int64_t n_t;
  // a tuple of source systems (n_sys > 1): one octree over all their bodies (n_s in total);
  // src, d and kind are then unused
  int n_sys = 1;
  SysIn sys[kMaxSystems] = {};
};

size_t footprint(const SolveIn& in, const fmm_options& o) {
  int64_t nt = in.tpos ? in.n_t : in.n_s;
  int64_t ls = std::max(1, o.leaf_size_source);
  int64_t nbr = 2 * (nt + in.n_s) / ls + 1024;
  size_t exp = (size_t)nbr * 4 * nh(o.expansion_order) * 8 * 2;
  size_t bodies = (size_t)(nt + in.n_s) * (32 + 32 + 8) + (size_t)nt * (13 + 13 + 16) * 8;
  size_t lists = (size_t)nbr * (256 + 64) * 8;
  size_t scratch = (size_t)(nt + in.n_s) * 48;
  return exp + bodies + lists + scratch;
}

// stream of the influence estimate: non-blocking, highest priority, so that its small
// kernels take SM slots as soon as the solve's near-field CTAs retire
cudaStream_t est_stream(fmm_ctx* c);
cudaEvent_t fork_event(fmm_ctx* c);
cudaEvent_t join_event(fmm_ctx* c);
cudaStream_t far_stream(fmm_ctx* c);
cudaEvent_t far_event(fmm_ctx* c);
cudaEvent_t up_event(fmm_ctx* c);
Scratch& est_scratch(fmm_ctx* c);
DevBuf<int>& est_stats(fmm_ctx* c);

// one fmm! evaluation into out16 (device, original target order), queued on st.
// The far field runs on the far-field stream (M2L waiting for the influence estimate of
// the relative error methods, src/fmm.jl:1189-1276, which runs on its own stream) while
// the near field runs on st; st waits for the far field before the unsort.  The
// estimate's own sub-solve keeps every stage on its stream.
// ---- tuples of source systems: one octree over every system's bodies
// the bodies of all systems, concatenated in tuple order, with the system of each
void unpack_tuple(Workspace& W, DevTree& S, const SolveIn& in, cudaStream_t st) {
  S.n_bodies = in.n_s;
  S.pos.grow(in.n_s);
  S.str.grow(in.n_s);
  W.sys_orig.grow(in.n_s);
  int64_t off = 0;
  for (int k = 0; k < in.n_sys; ++k) {
    const SysIn& y = in.sys[k];
    if (y.n > 0) {
      note_launch();
      k_unpack_system<<<grid_for(y.n), 256, 0, st>>>(y.buf, y.n, y.d, y.kind, off, k, S.pos.ptr, S.str.ptr,
                                                     W.sys_orig.ptr);
      FMM_CUDA_TRY(cudaGetLastError());
    }
    off += y.n;
  }
}

// after the tree: every system's bodies in tree order and its body range per branch (the
// reference's per-system bodies_index; within a leaf the tree keeps input order, so the
// systems come one after another)
void build_views(Workspace& W, const DevTree& S, const SolveIn& in, Scratch& sc, cudaStream_t st) {
  const int64_t n = S.n_bodies;
  W.sys_sorted.grow(n);
  note_launch();
  k_gather_int<<<grid_for(n), 256, 0, st>>>(W.sys_orig.ptr, S.sort_index.ptr, n, W.sys_sorted.ptr);
  FMM_CUDA_TRY(cudaGetLastError());
  sc.tmp_i.grow((size_t)n + 1);
  for (int k = 0; k < in.n_sys; ++k) {
    SysView& v = W.views[k];
    v.kind = in.sys[k].kind;
    v.n = in.sys[k].n;
    v.pre.grow((size_t)n + 1);
    v.pos.grow(std::max<int64_t>(v.n, 1));
    v.str.grow(std::max<int64_t>(v.n, 1));
    v.start.grow((size_t)S.n_branches);
    v.count.grow((size_t)S.n_branches);
    note_launch();
    k_flag_system<<<grid_for(n + 1), 256, 0, st>>>(W.sys_sorted.ptr, n, k, sc.tmp_i.ptr);
    size_t tb = 0;
    FMM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, sc.tmp_i.ptr, v.pre.ptr, (int)(n + 1), st));
    sc.cub.grow(tb);
    note_launch();
    FMM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(sc.cub.ptr, tb, sc.tmp_i.ptr, v.pre.ptr, (int)(n + 1), st));
    note_launch();
    k_split_system<<<grid_for(n), 256, 0, st>>>(W.sys_sorted.ptr, v.pre.ptr, n, k, S.pos.ptr, S.str.ptr, v.pos.ptr,
                                                v.str.ptr);
    note_launch();
    k_branch_ranges<<<grid_for(S.n_branches), 256, 0, st>>>(S.body_start.ptr, S.body_count.ptr, (int)S.n_branches,
                                                            v.pre.ptr, v.start.ptr, v.count.ptr);
    FMM_CUDA_TRY(cudaGetLastError());
  }
}

// the shared source tree seen through one system's bodies (a non-owning copy: its buffers
// are never grown or released)
DevTree view_tree(const DevTree& S, const SysView& v) {
  DevTree t = S;
  t.n_bodies = v.n;
  t.body_start.ptr = v.start.ptr;
  t.body_count.ptr = v.count.ptr;
  t.pos.ptr = v.pos.ptr;
  t.str.ptr = v.str.ptr;
  return t;
}

// is_estimate: the influence estimate's sub-solve, whose out16 receives one value per body
// (get_influence: the scalar potential when influence_potential, else |gradient|)
void run_fmm(fmm_ctx* c, Workspace& W, const SolveIn& in, const fmm_options& o, double* out16, fmm_result* res,
             bool is_estimate, cudaStream_t st, Scratch& sc, DevBuf<int>& stats, bool influence_potential = false) {
  const int p = o.expansion_order;
  const bool multi = in.n_sys > 1;
  // lamb_helmholtz = has_vector_potential(source_systems) (src/fmm.jl:927)
  bool lh = in.kind == FMM_POINT_VORTEX;
  if (multi) {
    lh = false;
    for (int k = 0; k < in.n_sys; ++k) lh = lh || in.sys[k].kind == FMM_POINT_VORTEX;
  }
  const int64_t ls_s = o.leaf_size_source;
  const int64_t ls_t = o.leaf_size_target > 0 ? o.leaf_size_target : ls_s;
  const bool ps = o.scalar_potential != 0, gs = o.gradient != 0, hs = o.hessian != 0;
  const int64_t launches0 = g_launches;
  cudaEvent_t ev[8] = {}, eve[2] = {};
  const bool timing = c->timing && !is_estimate && res;
  if (timing) {
    for (auto& e : ev) FMM_CUDA_TRY(cudaEventCreate(&e));
    for (auto& e : eve) FMM_CUDA_TRY(cudaEventCreate(&e));
  }
  auto mark = [&](int k) {
    if (timing) FMM_CUDA_TRY(cudaEventRecord(ev[k], st));
  };
  mark(0);
  // ---- trees (src/tree.jl:3-122)
  DevTree& S = W.tree[1];
  if (multi)
    unpack_tuple(W, S, in, st);
  else
    unpack_bodies(S, in.src, in.n_s, in.d, in.kind, true, st);
  build_tree(S, sc, st, ls_s, o.list_method, o.shrink_recenter != 0);
  if (multi) build_views(W, S, in, sc, st);
  // body_to_multipole! and direct! run per source system (src/fmm.jl:291-346, 3-40)
  auto p2m_all = [&](cudaStream_t s_) {
    if (!multi) return launch_p2m(S, p, in.kind, c->tables, s_);
    for (int k = 0; k < in.n_sys; ++k) {
      DevTree v = view_tree(S, W.views[k]);
      launch_p2m(v, p, W.views[k].kind, c->tables, s_);
    }
  };
  W.shared = (in.tpos == nullptr) && (ls_t == ls_s);
  if (!W.shared) {
    DevTree& T = W.tree[0];
    const double* tp = in.tpos ? in.tpos : in.src;
    int64_t stride = in.tpos ? in.t_stride : in.d;
    int64_t nt = in.tpos ? in.n_t : in.n_s;
    unpack_bodies(T, tp, nt, stride, 0, false, st);
    build_tree(T, sc, st, ls_t, o.list_method, o.shrink_recenter != 0);
  }
  DevTree& T = W.target();
  mark(1);
  // a solve runs its far field (upward pass, M2L, downward pass) on a second high-priority
  // stream, concurrently with the lists and the near field on st, into its own accumulator;
  // the influence estimate's sub-solve runs everything on its own stream
  const bool split = !is_estimate;
  cudaStream_t fs = split ? far_stream(c) : st;
  cudaEvent_t evf[5] = {};
  if (timing && split)
    for (auto& e : evf) FMM_CUDA_TRY(cudaEventCreate(&e));
  auto markf = [&](int k) {
    if (timing && split) FMM_CUDA_TRY(cudaEventRecord(evf[k], fs));
  };
  const int64_t NH4 = 4 * nh(p);
  upload_tables(c->tables, p, st);
  S.multipole.grow(NH4 * S.n_branches);
  FMM_CUDA_TRY(cudaMemsetAsync(S.multipole.ptr, 0, NH4 * S.n_branches * sizeof(double), st));
  // ---- upward pass: needs the source tree only
  if (split) {
    FMM_CUDA_TRY(cudaEventRecord(up_event(c), st));
    FMM_CUDA_TRY(cudaStreamWaitEvent(fs, up_event(c), 0));
  }
  markf(0);
  if (o.upward_pass && split) {
    p2m_all(fs);
    launch_m2m(S, p, lh, c->tables, fs);
  }
  markf(1);
  // ---- interaction lists (src/interaction_list.jl:3-19, 183-213)
  // error-controlled M2L: rows ordered by separation, so that the 32 pairs of a pass stop at similar orders
  build_lists(W.lists, T, S, sc, st, ls_s, o.multipole_acceptance, o.farfield != 0, o.nearfield != 0,
              o.self_induced != 0, o.list_method, o.error_method != FMM_ERROR_NONE);
  mark(2);
  FMM_CUDA_TRY(cudaMemsetAsync(T.max_influence.ptr, 0, T.n_branches * sizeof(double), st));
  const bool estimate = o.error_method == FMM_POWER_RELATIVE_GRADIENT ||
                        o.error_method == FMM_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT ||
                        o.error_method == FMM_POWER_RELATIVE_POTENTIAL;
  // ---- evaluation passes (src/fmm.jl:1028-1089)
  T.local.grow(NH4 * T.n_branches);
  FMM_CUDA_TRY(cudaMemsetAsync(T.local.ptr, 0, NH4 * T.n_branches * sizeof(double), st));
  W.acc13.grow(13 * (size_t)T.n_bodies);
  FMM_CUDA_TRY(cudaMemsetAsync(W.acc13.ptr, 0, 13 * T.n_bodies * sizeof(double), st));
  double* far13 = W.acc13.ptr;
  if (split) {
    W.acc13_far.grow(13 * (size_t)T.n_bodies);
    FMM_CUDA_TRY(cudaMemsetAsync(W.acc13_far.ptr, 0, 13 * T.n_bodies * sizeof(double), st));
    far13 = W.acc13_far.ptr;
  }
  stats.grow(8);
  FMM_CUDA_TRY(cudaMemsetAsync(stats.ptr, 0, 8 * sizeof(int), st));
  if (res) count_p2p_pairs(T, S, W.lists, reinterpret_cast<unsigned long long*>(stats.ptr + 4), st);
  // trees, lists and zeroed accumulators are ready: fork the rest of the far field and the estimate
  if (estimate || split) FMM_CUDA_TRY(cudaEventRecord(fork_event(c), st));
  if (split) FMM_CUDA_TRY(cudaStreamWaitEvent(fs, fork_event(c), 0));
  // near field
  auto near = [&] {
    if (!multi) {
      launch_p2p(T, S, W.lists, W.acc13.ptr, in.kind, ps, gs, hs, o.precision, st, !is_estimate);
    } else {
      for (int k = 0; k < in.n_sys; ++k) {
        if (W.views[k].n == 0) continue;
        DevTree v = view_tree(S, W.views[k]);
        launch_p2p(T, v, W.lists, W.acc13.ptr, W.views[k].kind, ps, gs, hs, o.precision, st, !is_estimate);
      }
    }
  };
  near();
  mark(3);
  if (o.upward_pass && !split) {
    p2m_all(st);
    launch_m2m(S, p, lh, c->tables, st);
  }
  if (!split) mark(4);
  // ---- relative error methods: influence estimate on its own stream, joined before the M2L
  if (estimate) {
    fmm_options e = o;
    e.leaf_size_source = 5;
    e.leaf_size_target = 5;
    e.expansion_order = 3;
    e.multipole_acceptance = 0.6;
    e.error_method = FMM_ERROR_NONE;
    e.shrink_recenter = 1;
    e.list_method = FMM_LIST_SELF_TUNING_TREE_STOP;
    e.farfield = e.nearfield = e.self_induced = 1;
    e.upward_pass = e.horizontal_pass = e.downward_pass = 1;
    // the relative gradient methods read only |grad| of the estimate (get_influence,
    // src/fmm.jl:1180-1183): its potential, which the reference also computes, is skipped;
    // PowerRelativePotential reads the potential (:1185-1187)
    e.scalar_potential = o.error_method == FMM_POWER_RELATIVE_POTENTIAL ? 1 : 0;
    e.gradient = 1;
    e.hessian = 0;
    e.precision = o.precision;  // the mixed solve estimates with its FP32 near field
    int64_t nt = in.tpos ? in.n_t : in.n_s;
    c->est_out16.grow((size_t)nt);  // |grad| per body
    cudaStream_t es = est_stream(c);
    FMM_CUDA_TRY(cudaStreamWaitEvent(es, fork_event(c), 0));
    if (timing) FMM_CUDA_TRY(cudaEventRecord(eve[0], es));
    run_fmm(c, c->est, in, e, c->est_out16.ptr, nullptr, true, es, est_scratch(c), est_stats(c),
            o.error_method == FMM_POWER_RELATIVE_POTENTIAL);
    branch_max_influence(T, c->est_out16.ptr, es);
    if (timing) FMM_CUDA_TRY(cudaEventRecord(eve[1], es));
    FMM_CUDA_TRY(cudaEventRecord(join_event(c), es));
    FMM_CUDA_TRY(cudaStreamWaitEvent(fs, join_event(c), 0));
  }
  markf(2);
  if (!split) mark(5);
  if (o.horizontal_pass)
    launch_m2l(T, S, W.lists, p, lh, o.error_method, o.error_tolerance, o.bonus_expansion, nullptr, stats.ptr,
               c->tables, o.precision, fs);
  markf(3);
  if (!split) mark(6);
  if (o.downward_pass) {
    launch_l2l(T, p, lh, c->tables, fs);
    launch_l2p(T, p, lh, ps, gs, hs, far13, fs);
  }
  markf(4);
  if (split) {
    FMM_CUDA_TRY(cudaEventRecord(far_event(c), fs));
    FMM_CUDA_TRY(cudaStreamWaitEvent(st, far_event(c), 0));
  }
  // ---- unsort into the caller's order (buffer_to_target!, src/compatibility.jl:324-338)
  note_launch();
  if (is_estimate)  // out16 receives |grad| per body (n doubles)
    k_unsort_gradnorm<<<grid_for(T.n_bodies), 256, 0, st>>>(W.acc13.ptr, T.sort_index.ptr, T.n_bodies, out16,
                                                             influence_potential ? 1 : 0);
  else
    k_unsort<<<grid_for(T.n_bodies), 256, 0, st>>>(W.acc13.ptr, T.sort_index.ptr, T.pos.ptr, T.n_bodies, out16,
                                                    split ? far13 : nullptr);
  FMM_CUDA_TRY(cudaGetLastError());
  mark(7);
  if (res) {
    int h[6] = {0, 0, 0, 0, 0, 0};
    FMM_CUDA_TRY(cudaMemcpyAsync(h, stats.ptr, 6 * sizeof(int), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaStreamSynchronize(st));
    unsigned long long fl, pairs;
    std::memcpy(&fl, &h[2], 8);
    std::memcpy(&pairs, &h[4], 8);
    res->p_max = h[0] + (h[1] ? 1 : 0);
    res->error_success = h[1] ? 0 : 1;
    res->n_target_branches = T.n_branches;
    res->n_source_branches = S.n_branches;
    res->n_target_leaves = T.n_leaves;
    res->n_source_leaves = S.n_leaves;
    res->n_m2l = W.lists.n_m2l;
    res->n_direct = W.lists.n_direct;
    res->m2l_flops = (int64_t)fl;
    res->n_p2p_pairs = (int64_t)pairs;
    res->n_kernel_launches = g_launches - launches0;
    if (timing) {
      float ms[3], tot = 0.0f, fup = 0.0f, fh = 0.0f, fd = 0.0f;
      for (int k = 0; k < 3; ++k) FMM_CUDA_TRY(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]));
      FMM_CUDA_TRY(cudaEventElapsedTime(&tot, ev[0], ev[7]));
      // far field on its own stream: upward (evf 0-1), horizontal (2-3, after the wait for the
      // influence estimate), downward (3-4)
      FMM_CUDA_TRY(cudaEventElapsedTime(&fup, evf[0], evf[1]));
      FMM_CUDA_TRY(cudaEventElapsedTime(&fh, evf[2], evf[3]));
      FMM_CUDA_TRY(cudaEventElapsedTime(&fd, evf[3], evf[4]));
      res->t_tree_ms = ms[0];
      res->t_lists_ms = ms[1];
      res->t_nearfield_ms = ms[2];
      res->t_upward_ms = fup;
      res->t_horizontal_ms = fh;
      res->t_downward_ms = fd;
      float me = 0.0f;
      if (estimate) FMM_CUDA_TRY(cudaEventElapsedTime(&me, eve[0], eve[1]));
      res->t_influence_ms = me;  // on its own stream, overlapping the near field and the upward pass
      res->t_total_ms = tot;
    }
  }
  if (timing) {
    for (auto& e : ev) cudaEventDestroy(e);
    for (auto& e : eve) cudaEventDestroy(e);
    for (auto& e : evf)
      if (e) cudaEventDestroy(e);
  }
}

void check_options(const fmm_options& o) {
  FMM_CHECK(o.expansion_order >= 1 && o.expansion_order <= kMaxP, FMM_ERR_ARGUMENT,
            "expansion_order must be in [1, 20]");
  FMM_CHECK(o.leaf_size_source >= 1, FMM_ERR_ARGUMENT, "leaf_size_source must be >= 1");
  FMM_CHECK(o.multipole_acceptance > 0, FMM_ERR_ARGUMENT, "multipole_acceptance must be > 0");
  FMM_CHECK(o.error_method >= 0 && o.error_method <= 6, FMM_ERR_ARGUMENT, "unknown error_method");
  FMM_CHECK(o.list_method >= 0 && o.list_method <= 2, FMM_ERR_ARGUMENT, "unknown list_method");
  FMM_CHECK(o.precision == FMM_PRECISION_F64 || o.precision == FMM_PRECISION_MIXED, FMM_ERR_ARGUMENT,
            "unknown precision");
}

void check_source(const fmm_source_system* s) {
  FMM_CHECK(s != nullptr, FMM_ERR_ARGUMENT, "source system is NULL");
  FMM_CHECK(s->kind == FMM_POINT_SOURCE || s->kind == FMM_POINT_VORTEX, FMM_ERR_ARGUMENT,
            "source kind must be FMM_POINT_SOURCE or FMM_POINT_VORTEX");
  FMM_CHECK(s->n_bodies >= 0, FMM_ERR_ARGUMENT, "negative n_bodies");
  FMM_CHECK(s->data_per_body >= 4 + s->kind, FMM_ERR_ARGUMENT, "data_per_body too small for the strength");
  FMM_CHECK(s->n_bodies == 0 || s->buffer, FMM_ERR_ARGUMENT, "source buffer is NULL");
}

// stage a caller buffer on the device (no copy for device memory)
const double* stage(fmm_ctx* c, DevBuf<double>& buf, const double* ptr, size_t n_doubles, int memory) {
  if (memory == FMM_MEMORY_DEVICE) return ptr;
  buf.grow(n_doubles);
  FMM_CUDA_TRY(cudaMemcpyAsync(buf.ptr, ptr, n_doubles * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return buf.ptr;
}

size_t tree_bytes(const DevTree& t) {
  return (t.body_start.cap + t.body_count.cap + t.child_start.cap + t.n_children.cap + t.parent.cap + t.i_leaf.cap +
          t.level.cap + t.leaf_index.cap + t.sort_index.cap) *
             4 +
         (t.gcenter.cap + t.gbox.cap + t.gradius.cap + t.tcenter.cap + t.scenter.cap + t.tradius.cap + t.sradius.cap +
          t.tbox.cap + t.sbox.cap + t.max_influence.cap + t.multipole.cap + t.local.cap) *
             8 +
         (t.pos.cap + t.str.cap) * 32;
}

size_t lists_bytes(const DevLists& l) {
  return (l.m2l_t.cap + l.m2l_s.cap + l.dir_t.cap + l.dir_s.cap + l.m2l_tgt.cap + l.m2l_off.cap + l.dir_tgt.cap +
          l.dir_off.cap) *
             4 +
         (l.p2p_chunks.cap + l.p2p_rowtab.cap) * sizeof(int4) + l.p2p_part.cap * 8;
}

template <class T>
void rel(DevBuf<T>& b) {
  b.release();
}

void release_tree(DevTree& t) {
  rel(t.body_start); rel(t.body_count); rel(t.child_start); rel(t.n_children); rel(t.parent); rel(t.i_leaf);
  rel(t.level); rel(t.gcenter); rel(t.gbox); rel(t.gradius); rel(t.tcenter); rel(t.scenter); rel(t.tradius);
  rel(t.sradius); rel(t.tbox); rel(t.sbox); rel(t.max_influence); rel(t.leaf_index); rel(t.sort_index);
  rel(t.pos); rel(t.str); rel(t.multipole); rel(t.local);
}

void release_lists(DevLists& l) {
  rel(l.m2l_t); rel(l.m2l_s); rel(l.dir_t); rel(l.dir_s); rel(l.m2l_tgt); rel(l.m2l_off); rel(l.dir_tgt);
  rel(l.dir_off); rel(l.p2p_chunks); rel(l.p2p_rowtab); rel(l.p2p_part);
}

void release_scratch(Scratch& s) {
  rel(s.cub); rel(s.keys_a); rel(s.keys_b); rel(s.vals_a); rel(s.vals_b); rel(s.tmp_i); rel(s.tmp_j); rel(s.tmp_k);
  rel(s.front_a); rel(s.front_b); rel(s.dir_raw); rel(s.m2l_raw); rel(s.cnt_a); rel(s.cnt_b); rel(s.counts);
  rel(s.tmp_d); rel(s.staging); rel(s.out16); rel(s.flag);
}

}  // namespace

namespace fmmb {
size_t request_footprint(const fmm_request* r) {
  SolveIn in;
  in.d = r->source.data_per_body;
  in.kind = r->source.kind;
  in.n_s = std::max<int64_t>(0, r->source.n_bodies);
  in.src = nullptr;
  in.tpos = r->target.positions;
  in.t_stride = r->target.stride;
  in.n_t = r->target.positions ? std::max<int64_t>(0, r->target.n_bodies) : in.n_s;
  return footprint(in, r->options);
}

void ctx_release_buffers(fmm_ctx* c) {
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (Workspace* w : {&c->main, &c->est}) {
    release_tree(w->tree[0]);
    release_tree(w->tree[1]);
    release_lists(w->lists);
    w->acc13.release();
    w->acc13_far.release();
  }
  release_scratch(c->sc);
  release_scratch(c->est_sc);
  for (DevBuf<double>* b : {&c->stage_s, &c->stage_t, &c->out16, &c->est_out16, &c->adj_src, &c->adj_out16,
                            &c->stage_d, &c->vjp_out, &c->multi16})
    b->release();
  c->have_solve = false;
}
}  // namespace fmmb

extern "C" {

void fmm_default_options(fmm_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->expansion_order = 5;
  o->leaf_size_source = 20;
  o->leaf_size_target = 0;
  o->multipole_acceptance = 0.4;
  o->error_method = FMM_ERROR_NONE;
  o->error_tolerance = 0.0;
  o->bonus_expansion = 1;
  o->shrink_recenter = 1;
  o->list_method = FMM_LIST_SELF_TUNING_TREE_STOP;
  o->farfield = o->nearfield = o->self_induced = 1;
  o->upward_pass = o->horizontal_pass = o->downward_pass = 1;
  o->scalar_potential = 0;
  o->gradient = 1;
  o->hessian = 0;
  o->precision = FMM_PRECISION_F64;
}

int fmm_ctx_create(fmm_ctx** out, int device) {
  if (!out) return FMM_ERR_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) return FMM_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return FMM_ERR_NO_DEVICE;
  if (prop.major != 10) return FMM_ERR_NO_DEVICE;  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return FMM_ERR_CUDA;
  fmm_ctx* c = new fmm_ctx();
  c->device = device;
  *out = c;
  return FMM_OK;
}

int fmm_ctx_destroy(fmm_ctx* c) {
  if (!c) return FMM_OK;
  if (c->serve) fmm_serve_stop(c);
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (Workspace* w : {&c->main, &c->est}) {
    release_tree(w->tree[0]);
    release_tree(w->tree[1]);
    release_lists(w->lists);
    w->acc13.release();
    w->acc13_far.release();
  }
  release_scratch(c->sc);
  release_scratch(c->est_sc);
  c->est_stats.release();
  if (c->est_stream) {
    cudaStreamSynchronize(c->est_stream);
    cudaStreamDestroy(c->est_stream);
  }
  if (c->far_stream) {
    cudaStreamSynchronize(c->far_stream);
    cudaStreamDestroy(c->far_stream);
  }
  if (c->ev_far) cudaEventDestroy(c->ev_far);
  if (c->ev_up) cudaEventDestroy(c->ev_up);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  c->tables.Hs.release();
  c->tables.zeta.release();
  c->tables.eta.release();
  c->tables.Mt.release();
  c->tables.Lt.release();
  c->stage_s.release();
  c->stage_t.release();
  c->out16.release();
  c->est_out16.release();
  c->adj_src.release();
  c->adj_out16.release();
  c->stage_d.release();
  c->vjp_out.release();
  c->multi16.release();
  c->stats.release();
  delete c;
  return FMM_OK;
}

int fmm_ctx_set_stream(fmm_ctx* c, void* stream) {
  if (!c) return FMM_ERR_ARGUMENT;
  c->stream = reinterpret_cast<cudaStream_t>(stream);
  return FMM_OK;
}

int fmm_ctx_set_timing(fmm_ctx* c, int enabled) {
  if (!c) return FMM_ERR_ARGUMENT;
  c->timing = enabled != 0;
  return FMM_OK;
}

int fmm_ctx_set_hbm_budget(fmm_ctx* c, size_t bytes) {
  if (!c) return FMM_ERR_ARGUMENT;
  c->budget = bytes;
  return FMM_OK;
}

size_t fmm_ctx_device_bytes(const fmm_ctx* c) {
  if (!c) return 0;
  size_t b = 0;
  for (const Workspace* w : {&c->main, &c->est}) {
    b += tree_bytes(w->tree[0]) + tree_bytes(w->tree[1]) + lists_bytes(w->lists) +
         (w->acc13.cap + w->acc13_far.cap) * 8;
  }
  const Scratch& s = c->sc;
  b += s.cub.cap + (s.keys_a.cap + s.keys_b.cap) * 8 +
       (s.vals_a.cap + s.vals_b.cap + s.tmp_i.cap + s.tmp_j.cap + s.tmp_k.cap + s.cnt_a.cap + s.cnt_b.cap) * 4 +
       (s.front_a.cap + s.front_b.cap + s.dir_raw.cap + s.m2l_raw.cap) * 8 + s.tmp_d.cap * 8;
  b += (c->stage_s.cap + c->stage_t.cap + c->out16.cap + c->est_out16.cap) * 8;
  b += (c->adj_src.cap + c->adj_out16.cap + c->stage_d.cap + c->vjp_out.cap + c->multi16.cap) * 8;
  return b;
}

const char* fmm_ctx_last_error(const fmm_ctx* c) { return c ? c->err.c_str() : "no context"; }

int fmm_solve(fmm_ctx* c, const fmm_target_system* target, const fmm_source_system* source, const fmm_options* opt,
              fmm_result* result) {
  if (!c) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(opt != nullptr, FMM_ERR_ARGUMENT, "options are NULL");
    check_options(*opt);
    check_source(source);
    FMM_CHECK(target != nullptr, FMM_ERR_ARGUMENT, "target system is NULL (it carries the output buffer)");
    const bool self = target->positions == nullptr;  // fmm!(system): the sources are the targets
    FMM_CHECK(self || target->stride >= 3, FMM_ERR_ARGUMENT, "target stride must be >= 3");
    FMM_CHECK(self || target->n_bodies >= 0, FMM_ERR_ARGUMENT, "negative target n_bodies");
    FMM_CUDA_TRY(cudaSetDevice(c->device));
    if (result) std::memset(result, 0, sizeof(*result));
    SolveIn in;
    in.d = source->data_per_body;
    in.kind = source->kind;
    in.n_s = source->n_bodies;
    in.src = nullptr;
    in.tpos = nullptr;
    in.t_stride = 0;
    in.n_t = self ? source->n_bodies : target->n_bodies;
    FMM_CHECK(in.n_t == 0 || target->out, FMM_ERR_ARGUMENT, "target out buffer is NULL");
    FMM_CHECK(self || in.n_t == 0 || target->positions, FMM_ERR_ARGUMENT, "target positions are NULL");
    if (c->budget) FMM_CHECK(footprint(in, *opt) <= c->budget, FMM_ERR_MEMORY, "request exceeds the context's HBM budget");
    c->have_solve = false;
    if (in.n_s == 0 || in.n_t == 0) {
      // fmm! warns and foregoes the calculation (src/fmm.jl:1155-1158): rows 4..16 are zero
      if (in.n_t > 0) {
        if (target->memory == FMM_MEMORY_DEVICE) {
          FMM_CUDA_TRY(cudaMemset2DAsync(target->out + 3, 16 * sizeof(double), 0, 13 * sizeof(double), in.n_t,
                                         c->stream));
          FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        } else {
          for (int64_t i = 0; i < in.n_t; ++i) std::memset(target->out + 16 * i + 3, 0, 13 * sizeof(double));
        }
      }
      if (result) result->error_success = 1;
      return FMM_OK;
    }
    in.src = stage(c, c->stage_s, source->buffer, (size_t)in.d * in.n_s, source->memory);
    if (!self) {
      in.tpos = stage(c, c->stage_t, target->positions, (size_t)target->stride * target->n_bodies, target->memory);
      in.t_stride = target->stride;
    }
    c->out16.grow(16 * (size_t)in.n_t);
    run_fmm(c, c->main, in, *opt, c->out16.ptr, result, false, c->stream, c->sc, c->stats);
    // write the target buffer (rows 1..3 = positions, 4..16 = phi, gradient, hessian)
    int mem = target->memory;
    double* dst = target->out;
    if (mem == FMM_MEMORY_DEVICE)
      FMM_CUDA_TRY(cudaMemcpyAsync(dst, c->out16.ptr, 16 * in.n_t * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    else
      FMM_CUDA_TRY(cudaMemcpyAsync(dst, c->out16.ptr, 16 * in.n_t * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->have_solve = true;
    c->last_p = opt->expansion_order;
    c->last_kind = source->kind;
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

int fmm_solve_multi(fmm_ctx* c, const fmm_target_system* target, const fmm_source_system* sources, int n_sources,
                    const fmm_options* opt, fmm_result* result) {
  if (!c) return FMM_ERR_ARGUMENT;
  if (n_sources == 1 && sources) return fmm_solve(c, target, sources, opt, result);
  try {
    FMM_CHECK(sources && n_sources > 1, FMM_ERR_ARGUMENT, "fmm_solve_multi: no source systems");
    FMM_CHECK(n_sources <= kMaxSystems, FMM_ERR_ARGUMENT, "fmm_solve_multi: at most 8 source systems");
    FMM_CHECK(target && target->positions, FMM_ERR_ARGUMENT,
              "fmm_solve_multi: several source systems need explicit target positions");
    FMM_CHECK(target->stride >= 3, FMM_ERR_ARGUMENT, "target stride must be >= 3");
    FMM_CHECK(opt != nullptr, FMM_ERR_ARGUMENT, "options are NULL");
    check_options(*opt);
    FMM_CHECK(opt->list_method != FMM_LIST_BARBA, FMM_ERR_ARGUMENT,
              "fmm_solve_multi: the Barba rule splits on per-system counts, which is not supported");
    const int64_t nt = target->n_bodies;
    FMM_CHECK(nt >= 0, FMM_ERR_ARGUMENT, "negative target n_bodies");
    FMM_CHECK(nt == 0 || target->out, FMM_ERR_ARGUMENT, "target out buffer is NULL");
    SolveIn in;
    in.n_sys = n_sources;
    in.n_s = 0;
    for (int k = 0; k < n_sources; ++k) {
      check_source(&sources[k]);
      in.n_s += sources[k].n_bodies;
    }
    FMM_CUDA_TRY(cudaSetDevice(c->device));
    if (result) std::memset(result, 0, sizeof(*result));
    in.kind = sources[0].kind;
    in.d = sources[0].data_per_body;
    in.src = nullptr;
    in.n_t = nt;
    in.t_stride = target->stride;
    in.tpos = nullptr;
    if (c->budget) FMM_CHECK(footprint(in, *opt) <= c->budget, FMM_ERR_MEMORY, "request exceeds the context's HBM budget");
    c->have_solve = false;
    if (in.n_s == 0 || nt == 0) {
      if (nt > 0) {
        if (target->memory == FMM_MEMORY_DEVICE) {
          FMM_CUDA_TRY(cudaMemset2DAsync(target->out + 3, 16 * sizeof(double), 0, 13 * sizeof(double), nt,
                                         c->stream));
          FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
        } else {
          for (int64_t i = 0; i < nt; ++i) std::memset(target->out + 16 * i + 3, 0, 13 * sizeof(double));
        }
      }
      if (result) result->error_success = 1;
      return FMM_OK;
    }
    // every system's buffer on the device (one staging area, systems back to back)
    size_t total = 0;
    for (int k = 0; k < n_sources; ++k) total += (size_t)sources[k].data_per_body * sources[k].n_bodies;
    const bool any_host = [&] {
      for (int k = 0; k < n_sources; ++k)
        if (sources[k].memory != FMM_MEMORY_DEVICE) return true;
      return false;
    }();
    if (any_host) c->stage_s.grow(total + 1);
    size_t at = 0;
    for (int k = 0; k < n_sources; ++k) {
      const fmm_source_system& y = sources[k];
      const size_t nd = (size_t)y.data_per_body * y.n_bodies;
      const double* dev = y.buffer;
      if (y.memory != FMM_MEMORY_DEVICE && nd > 0) {
        FMM_CUDA_TRY(cudaMemcpyAsync(c->stage_s.ptr + at, y.buffer, nd * sizeof(double), cudaMemcpyHostToDevice,
                                     c->stream));
        dev = c->stage_s.ptr + at;
      }
      in.sys[k] = SysIn{dev, y.data_per_body, y.kind, y.n_bodies};
      at += nd;
    }
    in.tpos = stage(c, c->stage_t, target->positions, (size_t)target->stride * nt, target->memory);
    c->out16.grow(16 * (size_t)nt);
    run_fmm(c, c->main, in, *opt, c->out16.ptr, result, false, c->stream, c->sc, c->stats);
    const cudaMemcpyKind dir = target->memory == FMM_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    FMM_CUDA_TRY(cudaMemcpyAsync(target->out, c->out16.ptr, 16 * (size_t)nt * sizeof(double), dir, c->stream));
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->have_solve = true;
    c->last_p = opt->expansion_order;
    c->last_kind = in.kind;
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

int fmm_vjp(fmm_ctx* c, const fmm_target_system* target, const fmm_source_system* source, const fmm_options* opt,
            const double* d_out, double* d_strength, double* d_source_position, double* d_target_position,
            fmm_result* result) {
  if (!c) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(opt != nullptr, FMM_ERR_ARGUMENT, "options are NULL");
    check_options(*opt);
    check_source(source);
    FMM_CHECK(target != nullptr, FMM_ERR_ARGUMENT, "target system is NULL (it carries the forward output)");
    const bool self = target->positions == nullptr;
    FMM_CHECK(self || target->stride >= 3, FMM_ERR_ARGUMENT, "target stride must be >= 3");
    FMM_CHECK(self || target->n_bodies >= 0, FMM_ERR_ARGUMENT, "negative target n_bodies");
    const int64_t ns = source->n_bodies, nt = self ? source->n_bodies : target->n_bodies;
    FMM_CHECK(ns > 0 && nt > 0, FMM_ERR_ARGUMENT, "fmm_vjp needs sources and targets");
    FMM_CHECK(target->out && d_out && d_strength && d_source_position, FMM_ERR_ARGUMENT,
              "fmm_vjp: target->out, d_out, d_strength and d_source_position are required");
    FMM_CHECK(target->memory == source->memory, FMM_ERR_ARGUMENT, "fmm_vjp: source and target memory must agree");
    const int mem = source->memory;
    FMM_CUDA_TRY(cudaSetDevice(c->device));
    if (result) std::memset(result, 0, sizeof(*result));
    const int kind = source->kind, d = source->data_per_body, sdim = kind == FMM_POINT_SOURCE ? 1 : 3;
    c->have_solve = false;
    // forward solve (the reference's fmm!): potential and gradient (point sources), velocity and its
    // gradient (vortex particles)
    fmm_options of = *opt;
    of.scalar_potential = kind == FMM_POINT_SOURCE ? 1 : of.scalar_potential;
    of.gradient = 1;
    of.hessian = kind == FMM_POINT_VORTEX ? 1 : of.hessian;
    SolveIn in;
    in.d = d;
    in.kind = kind;
    in.n_s = ns;
    in.n_t = nt;
    in.src = stage(c, c->stage_s, source->buffer, (size_t)d * ns, mem);
    in.tpos = nullptr;
    in.t_stride = 0;
    if (!self) {
      in.tpos = stage(c, c->stage_t, target->positions, (size_t)target->stride * nt, mem);
      in.t_stride = target->stride;
    }
    const double* dout = stage(c, c->stage_d, d_out, 16 * (size_t)nt, mem);
    {
      // a cotangent the adjoint would ignore is an error, not a silently wrong gradient
      c->sc.flag.grow(1);
      FMM_CUDA_TRY(cudaMemsetAsync(c->sc.flag.ptr, 0, sizeof(int), c->stream));
      note_launch();
      k_check_cotangents<<<grid_for(16 * nt), 256, 0, c->stream>>>(nt, kind, dout, c->sc.flag.ptr);
      FMM_CUDA_TRY(cudaGetLastError());
      int bad = 0;
      FMM_CUDA_TRY(cudaMemcpyAsync(&bad, c->sc.flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
      FMM_CHECK(!bad, FMM_ERR_ARGUMENT,
                kind == FMM_POINT_SOURCE
                    ? "fmm_vjp: point sources propagate cotangents of rows 1..4 (positions, potential) only"
                    : "fmm_vjp: vortex particles propagate cotangents of rows 1..3 and 5..7 (positions, velocity) only");
    }
    c->out16.grow(16 * (size_t)nt);
    run_fmm(c, c->main, in, of, c->out16.ptr, result, false, c->stream, c->sc, c->stats);
    // adjoint solve: sources at the targets with the cotangents as strengths, targets at the sources
    const int da = kind == FMM_POINT_SOURCE ? 5 : 7;
    c->adj_src.grow((size_t)da * nt);
    note_launch();
    k_adj_sources<<<grid_for(nt), 256, 0, c->stream>>>(nt, self ? in.src : in.tpos, self ? d : in.t_stride, self,
                                                        dout, kind, c->adj_src.ptr);
    FMM_CUDA_TRY(cudaGetLastError());
    SolveIn ia;
    ia.d = da;
    ia.kind = kind;
    ia.n_s = nt;
    ia.n_t = ns;
    ia.src = c->adj_src.ptr;
    ia.tpos = self ? nullptr : in.src;
    ia.t_stride = self ? 0 : d;
    fmm_options oa = of;
    c->adj_out16.grow(16 * (size_t)ns);
    run_fmm(c, c->main, ia, oa, c->adj_out16.ptr, nullptr, false, c->stream, c->sc, c->stats);
    // combine
    const size_t n_res = (size_t)sdim * ns + 3 * (size_t)ns + (self ? 0 : 3 * (size_t)nt);
    c->vjp_out.grow(n_res);
    double* r_str = c->vjp_out.ptr;
    double* r_pos = r_str + (size_t)sdim * ns;
    double* r_tpos = r_pos + 3 * (size_t)ns;
    note_launch();
    k_vjp_sources<<<grid_for(ns), 256, 0, c->stream>>>(ns, kind, in.src, d, c->adj_out16.ptr,
                                                        self ? c->out16.ptr : nullptr, self ? dout : nullptr, r_str,
                                                        r_pos);
    FMM_CUDA_TRY(cudaGetLastError());
    if (!self) {
      note_launch();
      k_vjp_targets<<<grid_for(nt), 256, 0, c->stream>>>(nt, kind, c->out16.ptr, dout, r_tpos);
      FMM_CUDA_TRY(cudaGetLastError());
    }
    const cudaMemcpyKind dir = mem == FMM_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    FMM_CUDA_TRY(cudaMemcpyAsync(target->out, c->out16.ptr, 16 * (size_t)nt * sizeof(double), dir, c->stream));
    FMM_CUDA_TRY(cudaMemcpyAsync(d_strength, r_str, (size_t)sdim * ns * sizeof(double), dir, c->stream));
    FMM_CUDA_TRY(cudaMemcpyAsync(d_source_position, r_pos, 3 * (size_t)ns * sizeof(double), dir, c->stream));
    if (!self && d_target_position)
      FMM_CUDA_TRY(cudaMemcpyAsync(d_target_position, r_tpos, 3 * (size_t)nt * sizeof(double), dir, c->stream));
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

int fmm_direct(fmm_ctx* c, const fmm_target_system* target, const fmm_source_system* source, int ps, int gs, int hs,
               int precision) {
  if (!c) return FMM_ERR_ARGUMENT;
  try {
    check_source(source);
    FMM_CHECK(target != nullptr, FMM_ERR_ARGUMENT, "direct! needs a target buffer");
    const bool self = target->positions == nullptr;
    const int64_t nt = self ? source->n_bodies : target->n_bodies;
    FMM_CHECK(self || target->stride >= 3, FMM_ERR_ARGUMENT, "target stride must be >= 3");
    FMM_CHECK(nt >= 0, FMM_ERR_ARGUMENT, "negative target n_bodies");
    FMM_CHECK(nt == 0 || target->out, FMM_ERR_ARGUMENT, "target out buffer is NULL");
    FMM_CHECK(precision == FMM_PRECISION_F64 || precision == FMM_PRECISION_MIXED, FMM_ERR_ARGUMENT,
              "unknown precision");
    FMM_CUDA_TRY(cudaSetDevice(c->device));
    c->have_solve = false;
    if (nt == 0) return FMM_OK;
    const double* src = stage(c, c->stage_s, source->buffer, (size_t)source->data_per_body * source->n_bodies + 1,
                              source->memory);
    const double* tp = self ? src
                            : stage(c, c->stage_t, target->positions, (size_t)target->stride * target->n_bodies,
                                    target->memory);
    DevTree& S = c->main.tree[1];
    DevTree& T = c->main.tree[0];
    unpack_bodies(S, src, source->n_bodies, source->data_per_body, source->kind, true, c->stream);
    unpack_bodies(T, tp, nt, self ? source->data_per_body : target->stride, 0, false, c->stream);
    c->main.acc13.grow(13 * (size_t)nt + 1);
    FMM_CUDA_TRY(cudaMemsetAsync(c->main.acc13.ptr, 0, 13 * nt * sizeof(double), c->stream));
    launch_direct(T.pos.ptr, nt, S.pos.ptr, S.str.ptr, source->n_bodies, c->main.acc13.ptr, source->kind, gs != 0,
                  hs != 0, precision, c->stream);
    (void)ps;
    c->out16.grow(16 * (size_t)nt + 1);
    note_launch();
    k_unsort<<<grid_for(nt), 256, 0, c->stream>>>(c->main.acc13.ptr, nullptr, T.pos.ptr, nt, c->out16.ptr);
    FMM_CUDA_TRY(cudaGetLastError());
    auto kind = target->memory == FMM_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    FMM_CUDA_TRY(cudaMemcpyAsync(target->out, c->out16.ptr, 16 * nt * sizeof(double), kind, c->stream));
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->have_solve = false;
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

int fmm_get_tree(fmm_ctx* c, int which, fmm_tree_view* v) {
  if (!c || !v) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(c->have_solve, FMM_ERR_STATE, "no solve to export");
    FMM_CHECK(which == 0 || which == 1, FMM_ERR_ARGUMENT, "which must be 0 (target) or 1 (source)");
    DevTree& t = which == 0 ? c->main.target() : c->main.source();
    const int64_t nb = t.n_branches;
    v->n_branches = nb;
    v->n_levels = t.n_levels;
    v->n_leaves = t.n_leaves;
    v->n_bodies = t.n_bodies;
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    auto get_i = [&](const DevBuf<int>& d, int64_t n, int64_t* dst) {
      if (!dst || n == 0) return;
      std::vector<int> h(n);
      FMM_CUDA_TRY(cudaMemcpy(h.data(), d.ptr, n * sizeof(int), cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < n; ++i) dst[i] = h[i];
    };
    auto get_d = [&](const DevBuf<double>& d, int64_t n, double* dst) {
      if (!dst || n == 0) return;
      FMM_CUDA_TRY(cudaMemcpy(dst, d.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
    };
    get_i(t.body_start, nb, v->body_start);
    get_i(t.body_count, nb, v->body_count);
    get_i(t.child_start, nb, v->child_start);
    get_i(t.n_children, nb, v->n_children);
    get_i(t.parent, nb, v->parent);
    get_i(t.i_leaf, nb, v->i_leaf);
    // The reference's target tree reads body radii from its target buffer, where
    // that row is zero, so its source centre/box/radius equal the target ones.
    const bool target_role = (which == 0);
    get_d(t.tcenter, 3 * nb, v->target_center);
    get_d(target_role ? t.tcenter : t.scenter, 3 * nb, v->source_center);
    get_d(t.tradius, nb, v->target_radius);
    get_d(target_role ? t.tradius : t.sradius, nb, v->source_radius);
    get_d(t.tbox, 3 * nb, v->target_box);
    get_d(target_role ? t.tbox : t.sbox, 3 * nb, v->source_box);
    get_d(t.max_influence, nb, v->max_influence);
    get_i(t.sort_index, t.n_bodies, v->sort_index);
    get_i(t.leaf_index, t.n_leaves, v->leaf_index);
    if (v->levels_start)
      for (int l = 0; l < t.n_levels; ++l) v->levels_start[l] = t.levels_start[l];
    if (v->levels_end)
      for (int l = 0; l < t.n_levels; ++l) v->levels_end[l] = t.levels_end[l];
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

int fmm_get_lists(fmm_ctx* c, int32_t* m2l, int64_t* n_m2l, int32_t* direct, int64_t* n_direct) {
  if (!c) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(c->have_solve, FMM_ERR_STATE, "no solve to export");
    DevLists& L = c->main.lists;
    if (n_m2l) *n_m2l = L.n_m2l;
    if (n_direct) *n_direct = L.n_direct;
    if (m2l || direct) {
      FMM_CUDA_TRY(cudaSetDevice(c->device));
      export_lists_reference_order(L, c->main.target(), c->main.source(), c->sc, c->stream, m2l, direct);
    }
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

int fmm_get_expansions(fmm_ctx* c, int which, double* out, int64_t n_doubles) {
  if (!c || !out) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(c->have_solve, FMM_ERR_STATE, "no solve to export");
    DevTree& t = which == 0 ? c->main.target() : c->main.source();
    const DevBuf<double>& e = which == 0 ? t.local : t.multipole;
    int64_t need = 4 * nh(c->last_p) * t.n_branches;
    FMM_CHECK(n_doubles >= need, FMM_ERR_ARGUMENT, "output too small for the expansions");
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    FMM_CUDA_TRY(cudaMemcpy(out, e.ptr, need * sizeof(double), cudaMemcpyDeviceToHost));
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

// ---- single operators ----------------------------------------------------------
int fmm_op_p2m(fmm_ctx* c, int kind, const double* buf, int d, int64_t n, const double* center, int p,
               double* expansion) {
  if (!c) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(p >= 1 && p <= kMaxP, FMM_ERR_ARGUMENT, "p must be in [1, 20]");
    FMM_CHECK(kind == FMM_POINT_SOURCE || kind == FMM_POINT_VORTEX, FMM_ERR_ARGUMENT, "bad kind");
    FMM_CHECK(d >= 4 + kind && n >= 0 && buf && center && expansion, FMM_ERR_ARGUMENT, "bad p2m arguments");
    FMM_CUDA_TRY(cudaSetDevice(c->device));
    const double* src = stage(c, c->stage_s, buf, (size_t)d * n + 1, FMM_MEMORY_HOST);
    DevTree& S = c->main.tree[1];
    unpack_bodies(S, src, n, d, kind, true, c->stream);
    int64_t NH4 = 4 * nh(p);
    c->sc.tmp_d.grow(NH4);
    FMM_CUDA_TRY(cudaMemcpyAsync(c->sc.tmp_d.ptr, expansion, NH4 * 8, cudaMemcpyHostToDevice, c->stream));
    launch_op_p2m(kind, S.pos.ptr, S.str.ptr, n, center, p, c->sc.tmp_d.ptr, c->stream);
    FMM_CUDA_TRY(cudaMemcpyAsync(expansion, c->sc.tmp_d.ptr, NH4 * 8, cudaMemcpyDeviceToHost, c->stream));
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->have_solve = false;
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

namespace {
struct OpBufs {
  DevBuf<double> a, b, cc, dd, e, f, g;
  DevBuf<int> pu;
  ~OpBufs() {
    a.release(); b.release(); cc.release(); dd.release(); e.release(); f.release(); g.release(); pu.release();
  }
};
double* up(DevBuf<double>& d, const double* h, size_t n, cudaStream_t st) {
  if (!h) return nullptr;
  d.grow(n);
  FMM_CUDA_TRY(cudaMemcpyAsync(d.ptr, h, n * 8, cudaMemcpyHostToDevice, st));
  return d.ptr;
}
}  // namespace

static int op_pairs(fmm_ctx* c, int64_t n, double* target, const double* tc, const double* src, const double* sc,
                    int p, int lh, bool local) {
  if (!c) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(p >= 1 && p <= kMaxP, FMM_ERR_ARGUMENT, "p must be in [1, 20]");
    FMM_CHECK(n >= 0 && target && tc && src && sc, FMM_ERR_ARGUMENT, "bad operator arguments");
    FMM_CUDA_TRY(cudaSetDevice(c->device));
    upload_tables(c->tables, p, c->stream);
    OpBufs B;
    size_t NH4 = 4 * nh(p);
    double* dt = up(B.a, target, NH4 * n, c->stream);
    double* dtc = up(B.b, tc, 3 * n, c->stream);
    double* ds = up(B.cc, src, NH4 * n, c->stream);
    double* dsc = up(B.dd, sc, 3 * n, c->stream);
    launch_op_m2m(n, dt, dtc, ds, dsc, p, lh != 0, local, c->tables, c->stream);
    FMM_CUDA_TRY(cudaMemcpyAsync(target, dt, NH4 * n * 8, cudaMemcpyDeviceToHost, c->stream));
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

int fmm_op_m2m(fmm_ctx* c, int64_t n, double* target, const double* tc, const double* src, const double* sc, int p,
               int lh) {
  return op_pairs(c, n, target, tc, src, sc, p, lh, false);
}

int fmm_op_l2l(fmm_ctx* c, int64_t n, double* target, const double* tc, const double* src, const double* sc, int p,
               int lh) {
  return op_pairs(c, n, target, tc, src, sc, p, lh, true);
}

int fmm_op_m2l(fmm_ctx* c, int64_t n, double* target, const double* tc, const double* tbox, const double* trad,
               const double* maxinf, const double* src, const double* sc, int p, int lh, int em, double eps, int be,
               int* p_used) {
  if (!c) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(p >= 1 && p <= kMaxP, FMM_ERR_ARGUMENT, "p must be in [1, 20]");
    FMM_CHECK(n >= 0 && target && tc && src && sc, FMM_ERR_ARGUMENT, "bad operator arguments");
    FMM_CHECK(em >= 0 && em <= 6, FMM_ERR_ARGUMENT, "unknown error method");
    FMM_CUDA_TRY(cudaSetDevice(c->device));
    upload_tables(c->tables, p, c->stream);
    OpBufs B;
    size_t NH4 = 4 * nh(p);
    double* dt = up(B.a, target, NH4 * n, c->stream);
    double* dtc = up(B.b, tc, 3 * n, c->stream);
    double* dtb = up(B.e, tbox, 3 * n, c->stream);
    double* dtr = up(B.f, trad, n, c->stream);
    double* dmi = up(B.g, maxinf, n, c->stream);
    double* ds = up(B.cc, src, NH4 * n, c->stream);
    double* dsc = up(B.dd, sc, 3 * n, c->stream);
    int* dpu = nullptr;
    if (p_used) {
      B.pu.grow(n + 1);
      dpu = B.pu.ptr;
    }
    launch_op_m2l(n, dt, dtc, dtb, dtr, dmi, ds, dsc, p, lh != 0, em, eps, be, dpu, c->tables, c->stream);
    FMM_CUDA_TRY(cudaMemcpyAsync(target, dt, NH4 * n * 8, cudaMemcpyDeviceToHost, c->stream));
    if (p_used) FMM_CUDA_TRY(cudaMemcpyAsync(p_used, dpu, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

int fmm_op_l2p(fmm_ctx* c, int64_t n, const double* dx, const double* local, int p, int lh, int ps, int gs, int hs,
               double* out13) {
  if (!c) return FMM_ERR_ARGUMENT;
  try {
    FMM_CHECK(p >= 1 && p <= kMaxP, FMM_ERR_ARGUMENT, "p must be in [1, 20]");
    FMM_CHECK(n >= 0 && dx && local && out13, FMM_ERR_ARGUMENT, "bad operator arguments");
    FMM_CUDA_TRY(cudaSetDevice(c->device));
    OpBufs B;
    double* ddx = up(B.a, dx, 3 * n, c->stream);
    double* dl = up(B.b, local, 4 * nh(p), c->stream);
    B.cc.grow(13 * n + 1);
    FMM_CUDA_TRY(cudaMemsetAsync(B.cc.ptr, 0, 13 * n * 8, c->stream));
    launch_op_l2p(n, ddx, dl, p, lh != 0, ps != 0, gs != 0, hs != 0, B.cc.ptr, c->stream);
    FMM_CUDA_TRY(cudaMemcpyAsync(out13, B.cc.ptr, 13 * n * 8, cudaMemcpyDeviceToHost, c->stream));
    FMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return FMM_OK;
  } catch (const Error& e) {
    return fail(c, e);
  }
}

}  // extern "C"
