// lists.cu -- dual-tree traversal in HBM (replaces src/interaction_list.jl:3-213).
//
// The reference recurses from (root, root) and, per (target, source) branch
// pair, either records a P2P pair, records an M2L pair (multipole acceptance
// criterion d^2 * mac^2 > (r_s + r_t)^2) or descends into the children of one
// side, with three rule sets (Barba, SelfTuning, SelfTuningTreeStop).  Here the
// same per-pair decision runs on a breadth-first frontier of pairs: every step
// classifies the whole frontier, scans the output counts and writes the P2P
// pairs, M2L pairs and the next frontier in order.  The decisions are the
// reference's, with the same FP64 operations (-fmad=false), so the resulting
// pair sets are identical; a stable radix sort by target then gives the
// target-sorted lists of sort_by_target (src/interaction_list.jl:183-213).
// Within one target the pairs are in frontier order (the reference's are in
// depth-first order); every consumer of the lists is order independent up to
// floating-point summation order.
#include <cub/cub.cuh>

#include "context.cuh"

namespace fmmb {

namespace {

enum : int { A_NONE = 0, A_DIRECT = 1, A_M2L = 2, A_SPLIT_T = 3, A_SPLIT_S = 4 };

struct Cnt3 {
  int d, m, n;
};
struct Cnt3Sum {
  __device__ __forceinline__ Cnt3 operator()(const Cnt3& a, const Cnt3& b) const {
    return Cnt3{a.d + b.d, a.m + b.m, a.n + b.n};
  }
};

struct TreeRef {
  const int* n_children;
  const int* child_start;
  const int* body_count;
  const double* center;  // target centre (target tree) or source centre (source tree)
  const double* radius;
};

struct Rule {
  double mac;
  int64_t ls;  // source leaf size (SelfTuning)
  int method;
  bool ff, nf, si;
};

__device__ __forceinline__ bool mac_accept(const TreeRef& T, int t, const TreeRef& S, int s, double mac) {
  double dx = T.center[3 * t] - S.center[3 * s];
  double dy = T.center[3 * t + 1] - S.center[3 * s + 1];
  double dz = T.center[3 * t + 2] - S.center[3 * s + 2];
  double sep2 = dx * dx + dy * dy + dz * dz;
  double summed = S.radius[s] + T.radius[t];
  return sep2 * mac * mac > summed * summed;
}

// one step of build_interaction_lists! for the three rule sets
// (src/interaction_list.jl:23-64, 66-120, 122-166)
__device__ int decide(const TreeRef& T, int t, const TreeRef& S, int s, const Rule& R, int& n_next) {
  n_next = 0;
  int nct = T.n_children[t], ncs = S.n_children[s];
  int bt = T.body_count[t], bs = S.body_count[s];
  bool both_leaves = (nct == 0) && (ncs == 0);
  bool dir_ok = (R.nf || (t == s && R.si)) && (t != s || R.si);
  if (R.method == FMM_LIST_BARBA) {
    if (mac_accept(T, t, S, s, R.mac)) return R.ff ? A_M2L : A_NONE;
    if (both_leaves) return dir_ok ? A_DIRECT : A_NONE;
    // target radius decides the side (src/interaction_list.jl:48)
    double tr = T.radius[t], sr = S.radius[s];
    if (ncs == 0 || (tr >= sr && nct != 0)) {
      n_next = nct;
      return A_SPLIT_T;
    }
    n_next = ncs;
    return A_SPLIT_S;
  }
  if (R.method == FMM_LIST_SELF_TUNING) {
    double fraction = 0.0;
    fraction = fraction + (double)bs / (double)(R.ls * R.ls);
    fraction = fraction * (double)bt;
    if (fraction < 1.0 || both_leaves) return (R.nf && (t != s || R.si)) ? A_DIRECT : A_NONE;
    if (mac_accept(T, t, S, s, R.mac)) return R.ff ? A_M2L : A_NONE;
  } else {  // SelfTuningTreeStop
    if (both_leaves) return dir_ok ? A_DIRECT : A_NONE;
    if (mac_accept(T, t, S, s, R.mac)) return R.ff ? A_M2L : A_NONE;
  }
  if (ncs == 0 || (bt >= bs && nct != 0)) {
    n_next = nct;
    return A_SPLIT_T;
  }
  n_next = ncs;
  return A_SPLIT_S;
}

__global__ void k_classify(const int2* __restrict__ front, int nf, TreeRef T, TreeRef S, Rule R, Cnt3* __restrict__ cnt) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > nf) return;
  if (k == nf) {
    cnt[k] = Cnt3{0, 0, 0};
    return;
  }
  int2 p = front[k];
  int nn;
  int a = decide(T, p.x, S, p.y, R, nn);
  cnt[k] = Cnt3{a == A_DIRECT, a == A_M2L, nn};
}

__global__ void k_emit(const int2* __restrict__ front, int nf, TreeRef T, TreeRef S, Rule R,
                       const Cnt3* __restrict__ off, int2* __restrict__ dir, int dir_base, int2* __restrict__ m2l,
                       int m2l_base, int2* __restrict__ next) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nf) return;
  int2 p = front[k];
  int nn;
  int a = decide(T, p.x, S, p.y, R, nn);
  Cnt3 o = off[k];
  if (a == A_DIRECT) {
    dir[dir_base + o.d] = p;
  } else if (a == A_M2L) {
    m2l[m2l_base + o.m] = p;
  } else if (a == A_SPLIT_T) {
    int c0 = T.child_start[p.x];
    for (int c = 0; c < nn; ++c) next[o.n + c] = make_int2(c0 + c, p.y);
  } else if (a == A_SPLIT_S) {
    int c0 = S.child_start[p.y];
    for (int c = 0; c < nn; ++c) next[o.n + c] = make_int2(p.x, c0 + c);
  }
}

__global__ void k_split(const int2* __restrict__ in, int n, int* __restrict__ t, int* __restrict__ s) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    t[k] = in[k].x;
    s[k] = in[k].y;
  }
}

template <class T>
void grow_keep_l(DevBuf<T>& b, size_t n, cudaStream_t st) {
  if (n <= b.cap) return;
  DevBuf<T> nb;
  nb.grow(n);
  if (b.ptr && b.cap) FMM_CUDA_TRY(cudaMemcpyAsync(nb.ptr, b.ptr, b.cap * sizeof(T), cudaMemcpyDeviceToDevice, st));
  FMM_CUDA_TRY(cudaStreamSynchronize(st));
  b.release();
  b = nb;
  nb.ptr = nullptr;
  nb.cap = 0;
}

// stable sort of (target, source) pairs by target and the per-target CSR
void finish_list(DevBuf<int2>& raw, int64_t n, int nbits, DevBuf<int>& out_t, DevBuf<int>& out_s,
                 DevBuf<int>& tgt, DevBuf<int>& off, int64_t& n_targets, Scratch& sc, cudaStream_t st) {
  out_t.grow(n + 1);
  out_s.grow(n + 1);
  if (n == 0) {
    n_targets = 0;
    tgt.grow(1);
    off.grow(2);
    FMM_CUDA_TRY(cudaMemsetAsync(off.ptr, 0, 2 * sizeof(int), st));
    return;
  }
  sc.tmp_i.grow(n);
  sc.tmp_j.grow(n);
  note_launch();
  k_split<<<(int)((n + 255) / 256), 256, 0, st>>>(raw.ptr, (int)n, sc.tmp_i.ptr, sc.tmp_j.ptr);
  size_t tb = 0;
  unsigned int* ki = reinterpret_cast<unsigned int*>(sc.tmp_i.ptr);
  unsigned int* ko = reinterpret_cast<unsigned int*>(out_t.ptr);
  cub::DeviceRadixSort::SortPairs(nullptr, tb, ki, ko, sc.tmp_j.ptr, out_s.ptr, (int)n, 0, nbits, st);
  sc.cub.grow(tb);
  FMM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(sc.cub.ptr, tb, ki, ko, sc.tmp_j.ptr, out_s.ptr, (int)n, 0, nbits, st));
  // run-length encode the targets -> unique targets + counts -> offsets
  tgt.grow(n + 1);
  off.grow(n + 2);
  sc.tmp_k.grow(n + 2);
  sc.counts.grow(4);
  tb = 0;
  cub::DeviceRunLengthEncode::Encode(nullptr, tb, out_t.ptr, tgt.ptr, sc.tmp_k.ptr, sc.counts.ptr, (int)n, st);
  sc.cub.grow(tb);
  FMM_CUDA_TRY(cub::DeviceRunLengthEncode::Encode(sc.cub.ptr, tb, out_t.ptr, tgt.ptr, sc.tmp_k.ptr, sc.counts.ptr,
                                                  (int)n, st));
  int runs = 0;
  FMM_CUDA_TRY(cudaMemcpyAsync(&runs, sc.counts.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  FMM_CUDA_TRY(cudaStreamSynchronize(st));
  n_targets = runs;
  FMM_CUDA_TRY(cudaMemsetAsync(sc.tmp_k.ptr + runs, 0, sizeof(int), st));
  tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, sc.tmp_k.ptr, off.ptr, runs + 1, st);
  sc.cub.grow(tb);
  FMM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(sc.cub.ptr, tb, sc.tmp_k.ptr, off.ptr, runs + 1, st));
}

}  // namespace

void build_lists(DevLists& L, const DevTree& tt, const DevTree& stt, Scratch& sc, cudaStream_t st,
                 int64_t leaf_size_source, double mac, bool ff, bool nf, bool si, int method) {
  TreeRef T{tt.n_children.ptr, tt.child_start.ptr, tt.body_count.ptr, tt.tcenter.ptr, tt.tradius.ptr};
  TreeRef S{stt.n_children.ptr, stt.child_start.ptr, stt.body_count.ptr, stt.scenter.ptr, stt.sradius.ptr};
  Rule R{mac, leaf_size_source, method, ff, nf, si};

  DevBuf<int2>& dir_raw = sc.dir_raw;
  DevBuf<int2>& m2l_raw = sc.m2l_raw;
  int64_t n_dir = 0, n_m2l = 0;
  sc.front_a.grow(1024);
  sc.front_b.grow(1024);
  int2 root = make_int2(0, 0);
  FMM_CUDA_TRY(cudaMemcpyAsync(sc.front_a.ptr, &root, sizeof(int2), cudaMemcpyHostToDevice, st));
  int nfront = 1;
  dir_raw.grow(std::max<size_t>(1024, (size_t)tt.n_leaves * 32));
  m2l_raw.grow(std::max<size_t>(1024, (size_t)tt.n_branches * 64));
  while (nfront > 0) {
    sc.cnt_a.grow(3 * (size_t)(nfront + 1));
    sc.cnt_b.grow(3 * (size_t)(nfront + 1));
    Cnt3* cnt = reinterpret_cast<Cnt3*>(sc.cnt_a.ptr);
    Cnt3* off = reinterpret_cast<Cnt3*>(sc.cnt_b.ptr);
    int g = (nfront + 1 + 255) / 256;
    note_launch();
    k_classify<<<g, 256, 0, st>>>(sc.front_a.ptr, nfront, T, S, R, cnt);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveScan(nullptr, tb, cnt, off, Cnt3Sum(), Cnt3{0, 0, 0}, nfront + 1, st);
    sc.cub.grow(tb);
    FMM_CUDA_TRY(cub::DeviceScan::ExclusiveScan(sc.cub.ptr, tb, cnt, off, Cnt3Sum(), Cnt3{0, 0, 0},
                                                nfront + 1, st));
    Cnt3 tot;
    FMM_CUDA_TRY(cudaMemcpyAsync(&tot, off + nfront, sizeof(Cnt3), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaStreamSynchronize(st));
    grow_keep_l(dir_raw, (size_t)(n_dir + tot.d + 1), st);
    grow_keep_l(m2l_raw, (size_t)(n_m2l + tot.m + 1), st);
    sc.front_b.grow((size_t)tot.n + 1);
    note_launch();
    k_emit<<<(nfront + 255) / 256, 256, 0, st>>>(sc.front_a.ptr, nfront, T, S, R, off, dir_raw.ptr, (int)n_dir,
                                                 m2l_raw.ptr, (int)n_m2l, sc.front_b.ptr);
    FMM_CUDA_TRY(cudaGetLastError());
    n_dir += tot.d;
    n_m2l += tot.m;
    nfront = tot.n;
    std::swap(sc.front_a, sc.front_b);
  }
  int nbits = 1;
  while ((1ll << nbits) <= tt.n_branches) ++nbits;
  L.n_direct = n_dir;
  L.n_m2l = n_m2l;
  finish_list(dir_raw, n_dir, nbits, L.dir_t, L.dir_s, L.dir_tgt, L.dir_off, L.n_dir_targets, sc, st);
  finish_list(m2l_raw, n_m2l, nbits, L.m2l_t, L.m2l_s, L.m2l_tgt, L.m2l_off, L.n_m2l_targets, sc, st);
}

}  // namespace fmmb
