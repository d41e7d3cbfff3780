// tree.cu -- octree construction in HBM (replaces src/tree.jl:3-122).
//
// The reference builds its octree top-down, sorting each splitting branch's
// bodies into octants with a stable counting sort, where the octant of a body
// is decided by strict `>` comparisons against the branch's FP64 centre, and
// child centres are parent_centre +- parent_box/2 (src/tree.jl:433-592).
// Here every body computes its whole octant path at once: the centre
// recursion is replayed per body with the same FP64 operations (this file is
// compiled with -fmad=false, so every product and sum is rounded exactly as
// in the reference), giving a 63-bit key (21 levels x 3 bits).  One radix sort
// of the keys then yields the branch structure level by level: a branch
// splits iff exceeds(n_bodies) (src/tree.jl:492-569), its children are the
// runs of the next key digit, emitted in octant order, so branches come out in
// the reference's breadth-first order with identical body ranges.  Finally the
// bodies inside each leaf are put back in input order (the reference's
// per-level sorts are stable and leaves are never sorted).
#include <cub/cub.cuh>

#include "context.cuh"

namespace fmmb {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n, int t = kThreads) {
  int64_t b = (n + t - 1) / t;
  if (b < 1) b = 1;
  if (b > 148 * 64) b = 148 * 64;
  return (int)b;
}

struct RootGeom {
  double c[3];
  double bmax;
  double radius;
};

__global__ void k_unpack(const double* __restrict__ buf, int64_t n, int64_t stride, int ns, int has_r,
                         double4* __restrict__ pos, double4* __restrict__ str) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* b = buf + i * stride;
    pos[i] = make_double4(b[0], b[1], b[2], has_r ? b[3] : 0.0);
    double4 s = make_double4(0, 0, 0, 0);
    if (ns >= 1) s.x = b[4];
    if (ns >= 3) {
      s.y = b[5];
      s.z = b[6];
    }
    str[i] = s;
  }
}

__global__ void k_bbox_partial(const double4* __restrict__ pos, int64_t n, double* __restrict__ part) {
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double4 p = pos[i];
    mn[0] = fmin(mn[0], p.x); mx[0] = fmax(mx[0], p.x);
    mn[1] = fmin(mn[1], p.y); mx[1] = fmax(mx[1], p.y);
    mn[2] = fmin(mn[2], p.z); mx[2] = fmax(mx[2], p.z);
  }
  __shared__ double s[6][kThreads];
  for (int k = 0; k < 3; ++k) {
    s[k][threadIdx.x] = mn[k];
    s[3 + k][threadIdx.x] = mx[k];
  }
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = fmin(s[k][threadIdx.x], s[k][threadIdx.x + w]);
        s[3 + k][threadIdx.x] = fmax(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) part[6 * blockIdx.x + k] = s[k][0];
}

// center_box / get_center_box (src/tree.jl:894-924) and the cubic root cell (src/tree.jl:20-26)
// one warp: lanes reduce strided partials, then shuffles (min/max are exact in any order)
__global__ void k_bbox_final(const double* __restrict__ part, int nb, RootGeom* root) {
  if (blockIdx.x != 0) return;
  const int lane = threadIdx.x;
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int b = lane; b < nb; b += 32)
    for (int k = 0; k < 3; ++k) {
      mn[k] = fmin(mn[k], part[6 * b + k]);
      mx[k] = fmax(mx[k], part[6 * b + 3 + k]);
    }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; ++k) {
      mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
      mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
    }
  if (lane != 0) return;
  double box[3];
  for (int k = 0; k < 3; ++k) {
    root->c[k] = (mx[k] + mn[k]) * 0.5;
    box[k] = mx[k] - root->c[k];
  }
  double bmax = fmax(fmax(box[0], box[1]), box[2]);
  root->bmax = bmax;
  root->radius = sqrt(bmax * bmax * 3.0);
}

// octant path of every body: get_octant (src/tree.jl:474-480) applied level by
// level with the child-centre recursion of get_child_center (src/tree.jl:581-592)
__global__ void k_keys(const double4* __restrict__ pos, int64_t n, const RootGeom* __restrict__ root,
                       unsigned long long* __restrict__ keys, int* __restrict__ vals) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double4 p = pos[i];
    double cx = root->c[0], cy = root->c[1], cz = root->c[2];
    double box = root->bmax;
    unsigned long long key = 0;
    for (int d = 0; d < kMaxDepth; ++d) {
      int o = (p.x > cx ? 1 : 0) | (p.y > cy ? 2 : 0) | (p.z > cz ? 4 : 0);
      key = (key << 3) | (unsigned long long)o;
      double delta = box * 0.5;
      cx = cx + ((o & 1) ? delta : -delta);
      cy = cy + ((o & 2) ? delta : -delta);
      cz = cz + ((o & 4) ? delta : -delta);
      box = box * 0.5;
    }
    keys[i] = key;
    vals[i] = (int)i;
  }
}

__device__ __forceinline__ int key_digit(unsigned long long k, int l) {
  return (int)((k >> (3 * (kMaxDepth - 1 - l))) & 7ull);
}

// first position in [lo, hi) whose level-l digit is >= o
__device__ int lower_bound_digit(const unsigned long long* keys, int lo, int hi, int l, int o) {
  while (lo < hi) {
    int mid = lo + ((hi - lo) >> 1);
    if (key_digit(keys[mid], l) < o)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// exceeds(..., method), src/tree.jl:492-569 (same FP operations)
__device__ __forceinline__ bool exceeds(int n, int64_t ls, int method) {
  if (method == FMM_LIST_BARBA) return n > ls;
  double fraction = 0.0;
  fraction = fraction + (double)n / (double)(ls * ls);
  fraction = fraction * (double)ls;
  if (method == FMM_LIST_SELF_TUNING) return fraction > 0.5 && n > 1;
  return fraction > 2.8284271247461903 && n > 1;
}

// The children of a splitting level-l branch are the runs of key digit l among its
// bodies.  Eight lanes per branch: lane o finds where octant o starts (a binary search
// over the branch's keys, in parallel instead of seven chained searches), lane o + 1
// where it ends.
constexpr unsigned kFullMask = 0xffffffffu;
struct Octants {
  int k;       // branch
  int o;       // this lane's octant
  bool split;  // the branch splits
  int b, e;    // bodies of octant o: [b, e)
  unsigned nonempty;  // bit q: octant q holds bodies (all lanes of the group)
};
__device__ __forceinline__ Octants octants_of(const unsigned long long* __restrict__ keys, int ls_node, int le_node,
                                              int level, int64_t leaf_size, int method,
                                              const int* __restrict__ body_start, const int* __restrict__ body_count,
                                              int* __restrict__ err) {
  Octants r;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  r.k = ls_node + (g >> 3);
  r.o = g & 7;
  const bool in = r.k < le_node;
  const int cnt = in ? body_count[r.k] : 0;
  r.split = in && exceeds(cnt, leaf_size, method);
  if (r.split && level >= kMaxDepth) {
    if (r.o == 0) atomicExch(err, 1);
    r.split = false;
  }
  const int lo = r.split ? body_start[r.k] : 0, hi = lo + (r.split ? cnt : 0);
  r.b = r.o == 0 ? lo : lower_bound_digit(keys, lo, hi, level, r.o);
  const int nb = __shfl_down_sync(kFullMask, r.b, 1, 8);
  r.e = r.o == 7 ? hi : nb;
  const unsigned ball = __ballot_sync(kFullMask, r.split && r.e > r.b);
  r.nonempty = (ball >> ((threadIdx.x & 31) & ~7)) & 0xffu;
  return r;
}

__global__ void k_count_children(const unsigned long long* __restrict__ keys, int ls_node, int le_node, int level,
                                 int64_t leaf_size, int method, const int* __restrict__ body_start,
                                 const int* __restrict__ body_count, int* __restrict__ nch, int* __restrict__ err) {
  const Octants r = octants_of(keys, ls_node, le_node, level, leaf_size, method, body_start, body_count, err);
  if (r.k < le_node && r.o == 0) nch[r.k - ls_node] = __popc(r.nonempty);
}

__global__ void k_emit_children(const unsigned long long* __restrict__ keys, int ls_node, int le_node, int level,
                                int64_t leaf_size, int method, const int* __restrict__ off, int* body_start,
                                int* body_count, int* child_start, int* n_children, int* parent, int* lev,
                                double* gcenter, double* gbox, double* gradius, int* __restrict__ err) {
  const Octants r = octants_of(keys, ls_node, le_node, level, leaf_size, method, body_start, body_count, err);
  if (r.k >= le_node) return;
  const int k = r.k, o = r.o;
  const int base = le_node + off[k - ls_node];
  if (o == 0) {
    child_start[k] = base;
    n_children[k] = __popc(r.nonempty);
  }
  if (!((r.nonempty >> o) & 1u)) return;
  const int c = base + __popc(r.nonempty & ((1u << o) - 1u));
  const double pbox = gbox[k], prad = gradius[k];
  body_start[c] = r.b;
  body_count[c] = r.e - r.b;
  parent[c] = k;
  lev[c] = level + 1;
  const double delta = pbox * 0.5;  // get_child_center: parent box is a cube of half width pbox
  gcenter[3 * c] = gcenter[3 * k] + ((o & 1) ? delta : -delta);
  gcenter[3 * c + 1] = gcenter[3 * k + 1] + ((o & 2) ? delta : -delta);
  gcenter[3 * c + 2] = gcenter[3 * k + 2] + ((o & 4) ? delta : -delta);
  gbox[c] = pbox * 0.5;
  gradius[c] = prad * 0.5;
}

__global__ void k_root(const RootGeom* root, int64_t n, int* body_start, int* body_count, int* parent, int* lev,
                       double* gcenter, double* gbox, double* gradius) {
  body_start[0] = 0;
  body_count[0] = (int)n;
  parent[0] = -1;
  lev[0] = 0;
  for (int k = 0; k < 3; ++k) gcenter[k] = root->c[k];
  gbox[0] = root->bmax;
  gradius[0] = root->radius;
}

__global__ void k_leaf_flags(const int* __restrict__ n_children, int nb, int* __restrict__ flag) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nb) flag[k] = n_children[k] == 0;
}

__global__ void k_leaf_index(const int* __restrict__ n_children, const int* __restrict__ scan, int nb,
                             int* __restrict__ i_leaf, int* __restrict__ leaf_index) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  if (n_children[k] == 0) {
    i_leaf[k] = scan[k];
    leaf_index[scan[k]] = k;
  } else {
    i_leaf[k] = -1;
  }
}

// key of the final order: the body_start of the leaf holding sorted position i,
// scattered to the body's input index
__global__ void k_leaf_keys(const int* __restrict__ leaf_index, int n_leaves, const int* __restrict__ body_start,
                            const int* __restrict__ body_count, const int* __restrict__ perm,
                            unsigned int* __restrict__ key_by_input) {
  int lane = threadIdx.x & 31;
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n_leaves) return;
  int b = leaf_index[w];
  int s = body_start[b], c = body_count[b];
  for (int i = lane; i < c; i += 32) key_by_input[perm[s + i]] = (unsigned int)s;
}

__global__ void k_iota(int* v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (int)i;
}

__global__ void k_permute(const double4* __restrict__ in_pos, const double4* __restrict__ in_str,
                          const int* __restrict__ sort_index, int64_t n, double4* __restrict__ pos,
                          double4* __restrict__ str) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int j = sort_index[i];
    pos[i] = in_pos[j];
    str[i] = in_str[j];
  }
}

// geometric cells without shrinking
__global__ void k_copy_geometry(int nb, const double* gcenter, const double* gbox, const double* gradius,
                                double* tc, double* sc, double* tr, double* sr, double* tb, double* sb) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  for (int d = 0; d < 3; ++d) {
    tc[3 * k + d] = sc[3 * k + d] = gcenter[3 * k + d];
    tb[3 * k + d] = sb[3 * k + d] = gbox[k];
  }
  tr[k] = sr[k] = gradius[k];
}

// min / max over an aligned group of G lanes (exact, so the grouping does not matter)
template <int G = 32>
__device__ __forceinline__ double wmin(double v) {
  for (int o = G / 2; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <int G = 32>
__device__ __forceinline__ double wmax(double v) {
  for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// shrink_leaf! (src/tree.jl:1141-1161): a group of G lanes per leaf (32, or 8 when the
// leaves hold a few bodies)
template <int G>
__global__ void k_shrink_leaves(const int* __restrict__ leaf_index, int n_leaves, const int* __restrict__ body_start,
                                const int* __restrict__ body_count, const double4* __restrict__ pos, double* tc,
                                double* sc, double* tr, double* sr, double* tb, double* sb) {
  const int lane = threadIdx.x & (G - 1);
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool valid = w < n_leaves;  // the groups past the end repeat the last leaf and write nothing
  const int b = leaf_index[valid ? w : n_leaves - 1];
  const int s = body_start[b], c = body_count[b];
  double4 p0 = pos[s];
  double tmn[3] = {p0.x, p0.y, p0.z}, tmx[3] = {p0.x, p0.y, p0.z};
  double smn[3] = {p0.x, p0.y, p0.z}, smx[3] = {p0.x, p0.y, p0.z};
  for (int i = lane; i < c; i += G) {
    double4 p = pos[s + i];
    double x[3] = {p.x, p.y, p.z};
    for (int d = 0; d < 3; ++d) {
      tmn[d] = fmin(tmn[d], x[d]);
      tmx[d] = fmax(tmx[d], x[d]);
      smn[d] = fmin(smn[d], x[d] - p.w);
      smx[d] = fmax(smx[d], x[d] + p.w);
    }
  }
  double tcen[3], scen[3];
  for (int d = 0; d < 3; ++d) {
    tmn[d] = wmin<G>(tmn[d]);
    tmx[d] = wmax<G>(tmx[d]);
    smn[d] = wmin<G>(smn[d]);
    smx[d] = wmax<G>(smx[d]);
    tcen[d] = (tmx[d] + tmn[d]) * 0.5;
    scen[d] = (smx[d] + smn[d]) * 0.5;
  }
  double trad = 0.0, srad = 0.0;
  for (int i = lane; i < c; i += G) {
    double4 p = pos[s + i];
    double dx = p.x - tcen[0], dy = p.y - tcen[1], dz = p.z - tcen[2];
    trad = fmax(trad, sqrt(dx * dx + dy * dy + dz * dz));
    dx = p.x - scen[0];
    dy = p.y - scen[1];
    dz = p.z - scen[2];
    srad = fmax(srad, sqrt(dx * dx + dy * dy + dz * dz) + p.w);
  }
  trad = wmax<G>(trad);
  srad = wmax<G>(srad);
  if (valid && lane == 0) {
    for (int d = 0; d < 3; ++d) {
      tc[3 * b + d] = tcen[d];
      sc[3 * b + d] = scen[d];
      tb[3 * b + d] = tmx[d] - tcen[d];
      sb[3 * b + d] = smx[d] - scen[d];
    }
    tr[b] = trad;
    sr[b] = srad;
  }
}

// shrink_branch! (src/tree.jl:1163-1174) for the non-leaf branches of one level
__global__ void k_shrink_branches(int l0, int l1, const int* __restrict__ child_start, const int* __restrict__ n_children,
                                  double* tc, double* sc, double* tr, double* sr, double* tb, double* sb) {
  int k = l0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= l1) return;
  int nc = n_children[k];
  if (nc == 0) return;
  int c0 = child_start[k];
  double tmn[3], tmx[3], smn[3], smx[3];
  for (int d = 0; d < 3; ++d) {
    tmn[d] = tmx[d] = tc[3 * c0 + d];
    smn[d] = smx[d] = sc[3 * c0 + d];
  }
  for (int c = c0; c < c0 + nc; ++c)
    for (int d = 0; d < 3; ++d) {
      tmn[d] = fmin(tmn[d], tc[3 * c + d] - tb[3 * c + d]);
      tmx[d] = fmax(tmx[d], tc[3 * c + d] + tb[3 * c + d]);
      smn[d] = fmin(smn[d], sc[3 * c + d] - sb[3 * c + d]);
      smx[d] = fmax(smx[d], sc[3 * c + d] + sb[3 * c + d]);
    }
  double tcen[3], scen[3];
  for (int d = 0; d < 3; ++d) {
    tcen[d] = (tmn[d] + tmx[d]) * 0.5;
    scen[d] = (smn[d] + smx[d]) * 0.5;
  }
  double trad = 0.0, srad = 0.0;
  for (int c = c0; c < c0 + nc; ++c) {
    double dx = tc[3 * c] - tcen[0], dy = tc[3 * c + 1] - tcen[1], dz = tc[3 * c + 2] - tcen[2];
    trad = fmax(trad, sqrt(dx * dx + dy * dy + dz * dz) + tr[c]);
    dx = sc[3 * c] - scen[0];
    dy = sc[3 * c + 1] - scen[1];
    dz = sc[3 * c + 2] - scen[2];
    srad = fmax(srad, sqrt(dx * dx + dy * dy + dz * dz) + sr[c]);
  }
  for (int d = 0; d < 3; ++d) {
    tc[3 * k + d] = tcen[d];
    sc[3 * k + d] = scen[d];
    tb[3 * k + d] = tmx[d] - tcen[d];
    sb[3 * k + d] = smx[d] - scen[d];
  }
  tr[k] = trad;
  sr[k] = srad;
}

// estimate_influence! tail (src/fmm.jl:1236-1262): max |grad| over each branch's bodies
__global__ void k_leaf_maxinf(const int* __restrict__ leaf_index, int n_leaves, const int* __restrict__ body_start,
                              const int* __restrict__ body_count, const int* __restrict__ sort_index,
                              const double* __restrict__ gnorm, double* __restrict__ mi) {
  int lane = threadIdx.x & 31;
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n_leaves) return;
  int b = leaf_index[w];
  int s = body_start[b], c = body_count[b];
  double m = 0.0;
  for (int i = lane; i < c; i += 32) {
    m = fmax(m, gnorm[sort_index[s + i]]);
  }
  m = wmax(m);
  if (lane == 0) mi[b] = m;
}

__global__ void k_branch_maxinf(int l0, int l1, const int* __restrict__ child_start, const int* __restrict__ n_children,
                                double* mi) {
  int k = l0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= l1) return;
  int nc = n_children[k];
  if (nc == 0) return;
  double m = 0.0;
  for (int c = child_start[k]; c < child_start[k] + nc; ++c) m = fmax(m, mi[c]);
  mi[k] = m;
}

template <class T>
void grow_keep(DevBuf<T>& b, size_t n, cudaStream_t st) {
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

}  // namespace

void unpack_bodies(DevTree& t, const double* dev_buf, int64_t n, int64_t stride, int n_strength, bool has_radius,
                   cudaStream_t st) {
  t.n_bodies = n;
  t.pos.grow(n);
  t.str.grow(n);
  if (n == 0) return;
  note_launch();
  k_unpack<<<blocks_for(n), kThreads, 0, st>>>(dev_buf, n, stride, n_strength, has_radius ? 1 : 0, t.pos.ptr,
                                               t.str.ptr);
  FMM_CUDA_TRY(cudaGetLastError());
}

void build_tree(DevTree& t, Scratch& sc, cudaStream_t st, int64_t leaf_size, int method, bool shrink) {
  const int64_t n = t.n_bodies;
  FMM_CHECK(n > 0, FMM_ERR_ARGUMENT, "build_tree: empty system");
  FMM_CHECK(n < (1ll << 31) - 64, FMM_ERR_ARGUMENT, "build_tree: more than 2^31 bodies");
  FMM_CHECK(leaf_size >= 1, FMM_ERR_ARGUMENT, "leaf_size must be >= 1");

  // root cell
  int nb_part = (int)std::min<int64_t>(blocks_for(n), 148 * 8);
  sc.tmp_d.grow(6 * (size_t)nb_part + 8);
  double* part = sc.tmp_d.ptr;
  RootGeom* root = reinterpret_cast<RootGeom*>(part + 6 * nb_part);
  note_launch();
  k_bbox_partial<<<nb_part, kThreads, 0, st>>>(t.pos.ptr, n, part);
  note_launch();
  k_bbox_final<<<1, 32, 0, st>>>(part, nb_part, root);

  // octant-path keys, sorted (stable) with the body index
  sc.keys_a.grow(n);
  sc.keys_b.grow(n);
  sc.vals_a.grow(n);
  sc.vals_b.grow(n);
  note_launch();
  k_keys<<<blocks_for(n), kThreads, 0, st>>>(t.pos.ptr, n, root, sc.keys_a.ptr, sc.vals_a.ptr);
  size_t tmp_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, sc.keys_a.ptr, sc.keys_b.ptr, sc.vals_a.ptr, sc.vals_b.ptr,
                                  (int)n, 0, 3 * kMaxDepth, st);
  sc.cub.grow(tmp_bytes);
  FMM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(sc.cub.ptr, tmp_bytes, sc.keys_a.ptr, sc.keys_b.ptr, sc.vals_a.ptr,
                                               sc.vals_b.ptr, (int)n, 0, 3 * kMaxDepth, st));
  const unsigned long long* keys = sc.keys_b.ptr;
  int* perm = sc.vals_b.ptr;

  // branches, level by level
  size_t cap = (size_t)(2 * n / std::max<int64_t>(leaf_size, 1) + 1024);
  auto ensure = [&](size_t need) {
    if (need <= t.body_start.cap && t.body_start.ptr) return;
    size_t want = std::max(need, 2 * std::max<size_t>(t.body_start.cap, cap));
    grow_keep(t.body_start, want, st);
    grow_keep(t.body_count, want, st);
    grow_keep(t.child_start, want, st);
    grow_keep(t.n_children, want, st);
    grow_keep(t.parent, want, st);
    grow_keep(t.level, want, st);
    grow_keep(t.gcenter, 3 * want, st);
    grow_keep(t.gbox, want, st);
    grow_keep(t.gradius, want, st);
  };
  ensure(cap);
  sc.counts.grow(4);
  sc.flag.grow(1);
  FMM_CUDA_TRY(cudaMemsetAsync(sc.flag.ptr, 0, sizeof(int), st));
  note_launch();
  k_root<<<1, 1, 0, st>>>(root, n, t.body_start.ptr, t.body_count.ptr, t.parent.ptr, t.level.ptr, t.gcenter.ptr,
                          t.gbox.ptr, t.gradius.ptr);
  FMM_CUDA_TRY(cudaGetLastError());
  t.levels_start.assign(1, 0);
  t.levels_end.assign(1, 1);
  int ls_node = 0, le_node = 1, level = 0;
  for (;;) {
    int nl = le_node - ls_node;
    sc.tmp_i.grow(nl + 1);
    sc.tmp_j.grow(nl + 1);
    const int g = (int)((8ll * nl + 127) / 128);  // eight lanes per branch
    note_launch();
    k_count_children<<<g, 128, 0, st>>>(keys, ls_node, le_node, level, leaf_size, method, t.body_start.ptr,
                                        t.body_count.ptr, sc.tmp_i.ptr, sc.flag.ptr);
    FMM_CUDA_TRY(cudaMemsetAsync(sc.tmp_i.ptr + nl, 0, sizeof(int), st));
    size_t sb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, sb, sc.tmp_i.ptr, sc.tmp_j.ptr, nl + 1, st);
    sc.cub.grow(sb);
    FMM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(sc.cub.ptr, sb, sc.tmp_i.ptr, sc.tmp_j.ptr, nl + 1, st));
    int h[2] = {0, 0};
    FMM_CUDA_TRY(cudaMemcpyAsync(&h[0], sc.tmp_j.ptr + nl, sizeof(int), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaMemcpyAsync(&h[1], sc.flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaStreamSynchronize(st));
    FMM_CHECK(h[1] == 0, FMM_ERR_TREE_DEPTH,
              "octree deeper than 21 levels: bodies are (nearly) coincident; spread them or raise leaf_size");
    int total = h[0];
    ensure((size_t)le_node + total + 1);
    note_launch();
    k_emit_children<<<g, 128, 0, st>>>(keys, ls_node, le_node, level, leaf_size, method, sc.tmp_j.ptr,
                                       t.body_start.ptr, t.body_count.ptr, t.child_start.ptr, t.n_children.ptr,
                                       t.parent.ptr, t.level.ptr, t.gcenter.ptr, t.gbox.ptr, t.gradius.ptr,
                                       sc.flag.ptr);
    FMM_CUDA_TRY(cudaGetLastError());
    if (total == 0) break;
    ls_node = le_node;
    le_node += total;
    ++level;
    t.levels_start.push_back(ls_node);
    t.levels_end.push_back(le_node);
  }
  const int nb = le_node;
  t.n_branches = nb;
  t.n_levels = (int)t.levels_start.size();

  // leaves (branch order) -> i_leaf, leaf_index
  t.i_leaf.grow(nb);
  sc.tmp_i.grow(nb + 1);
  sc.tmp_j.grow(nb + 1);
  int gb = (nb + 255) / 256;
  note_launch();
  k_leaf_flags<<<gb, 256, 0, st>>>(t.n_children.ptr, nb, sc.tmp_i.ptr);
  FMM_CUDA_TRY(cudaMemsetAsync(sc.tmp_i.ptr + nb, 0, sizeof(int), st));
  size_t sb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, sb, sc.tmp_i.ptr, sc.tmp_j.ptr, nb + 1, st);
  sc.cub.grow(sb);
  FMM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(sc.cub.ptr, sb, sc.tmp_i.ptr, sc.tmp_j.ptr, nb + 1, st));
  int nleaves = 0;
  FMM_CUDA_TRY(cudaMemcpyAsync(&nleaves, sc.tmp_j.ptr + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
  FMM_CUDA_TRY(cudaStreamSynchronize(st));
  t.n_leaves = nleaves;
  t.leaf_index.grow(nleaves);
  note_launch();
  k_leaf_index<<<gb, 256, 0, st>>>(t.n_children.ptr, sc.tmp_j.ptr, nb, t.i_leaf.ptr, t.leaf_index.ptr);

  // final body order: by leaf (key order), input order inside each leaf
  unsigned int* key_in = reinterpret_cast<unsigned int*>(sc.keys_a.ptr);
  unsigned int* key_out = key_in + n;
  note_launch();
  k_leaf_keys<<<(int)((nleaves * 32ll + 255) / 256), 256, 0, st>>>(t.leaf_index.ptr, nleaves, t.body_start.ptr,
                                                                    t.body_count.ptr, perm, key_in);
  note_launch();
  k_iota<<<blocks_for(n), kThreads, 0, st>>>(sc.vals_a.ptr, n);
  t.sort_index.grow(n);
  int bits = 1;
  while ((1ll << bits) <= n) ++bits;
  tmp_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key_in, key_out, sc.vals_a.ptr, t.sort_index.ptr, (int)n, 0,
                                  bits, st);
  sc.cub.grow(tmp_bytes);
  FMM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(sc.cub.ptr, tmp_bytes, key_in, key_out, sc.vals_a.ptr,
                                               t.sort_index.ptr, (int)n, 0, bits, st));
  // permute bodies into sorted order (through scratch copies of the input order)
  sc.tmp_d.grow(8 * (size_t)n);
  double4* in_pos = reinterpret_cast<double4*>(sc.tmp_d.ptr);
  double4* in_str = in_pos + n;
  FMM_CUDA_TRY(cudaMemcpyAsync(in_pos, t.pos.ptr, n * sizeof(double4), cudaMemcpyDeviceToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyAsync(in_str, t.str.ptr, n * sizeof(double4), cudaMemcpyDeviceToDevice, st));
  note_launch();
  k_permute<<<blocks_for(n), kThreads, 0, st>>>(in_pos, in_str, t.sort_index.ptr, n, t.pos.ptr, t.str.ptr);

  // branch geometry: shrink_recenter! (src/tree.jl:1176-1188) or the geometric cells
  t.tcenter.grow(3 * nb);
  t.scenter.grow(3 * nb);
  t.tradius.grow(nb);
  t.sradius.grow(nb);
  t.tbox.grow(3 * nb);
  t.sbox.grow(3 * nb);
  t.max_influence.grow(nb);
  FMM_CUDA_TRY(cudaMemsetAsync(t.max_influence.ptr, 0, nb * sizeof(double), st));
  note_launch();
  k_copy_geometry<<<gb, 256, 0, st>>>(nb, t.gcenter.ptr, t.gbox.ptr, t.gradius.ptr, t.tcenter.ptr, t.scenter.ptr,
                                      t.tradius.ptr, t.sradius.ptr, t.tbox.ptr, t.sbox.ptr);
  if (shrink) {
    note_launch();
    if (n <= 8 * (int64_t)nleaves)
      k_shrink_leaves<8><<<(int)((nleaves * 8ll + 255) / 256), 256, 0, st>>>(
          t.leaf_index.ptr, nleaves, t.body_start.ptr, t.body_count.ptr, t.pos.ptr, t.tcenter.ptr, t.scenter.ptr,
          t.tradius.ptr, t.sradius.ptr, t.tbox.ptr, t.sbox.ptr);
    else
      k_shrink_leaves<32><<<(int)((nleaves * 32ll + 255) / 256), 256, 0, st>>>(
          t.leaf_index.ptr, nleaves, t.body_start.ptr, t.body_count.ptr, t.pos.ptr, t.tcenter.ptr, t.scenter.ptr,
          t.tradius.ptr, t.sradius.ptr, t.tbox.ptr, t.sbox.ptr);
    for (int l = t.n_levels - 1; l >= 0; --l) {
      int l0 = (int)t.levels_start[l], l1 = (int)t.levels_end[l];
      note_launch();
      k_shrink_branches<<<(l1 - l0 + 127) / 128, 128, 0, st>>>(l0, l1, t.child_start.ptr, t.n_children.ptr,
                                                               t.tcenter.ptr, t.scenter.ptr, t.tradius.ptr,
                                                               t.sradius.ptr, t.tbox.ptr, t.sbox.ptr);
    }
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

void branch_max_influence(DevTree& t, const double* gnorm_orig, cudaStream_t st) {
  int nl = (int)t.n_leaves;
  note_launch();
  k_leaf_maxinf<<<(int)((nl * 32ll + 255) / 256), 256, 0, st>>>(t.leaf_index.ptr, nl, t.body_start.ptr,
                                                                t.body_count.ptr, t.sort_index.ptr, gnorm_orig,
                                                                t.max_influence.ptr);
  for (int l = t.n_levels - 1; l >= 0; --l) {
    int l0 = (int)t.levels_start[l], l1 = (int)t.levels_end[l];
    note_launch();
    k_branch_maxinf<<<(l1 - l0 + 127) / 128, 128, 0, st>>>(l0, l1, t.child_start.ptr, t.n_children.ptr,
                                                           t.max_influence.ptr);
  }
  FMM_CUDA_TRY(cudaGetLastError());
}

}  // namespace fmmb
