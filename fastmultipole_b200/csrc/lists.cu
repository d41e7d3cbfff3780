// lists.cu -- dual-tree traversal in HBM (replaces src/interaction_list.jl:3-213).
//
// The reference recurses from (root, root) and, per (target, source) branch
// pair, either records a P2P pair, records an M2L pair (multipole acceptance
// criterion d^2 * mac^2 > (r_s + r_t)^2) or descends into the children of one
// side, with three rule sets (Barba, SelfTuning, SelfTuningTreeStop).  Here the
// same per-pair decision runs on a breadth-first frontier of pairs, one kernel
// per step with no host round trip in between: a pair at step k has depth(t) +
// depth(s) = k, so (levels of the target tree + levels of the source tree - 1)
// steps exhaust the recursion.  Outputs and the next frontier take their slots
// with warp-aggregated atomics, and the pairs of every target are counted.  The
// decisions are the reference's, with the same FP64 operations (-fmad=false), so
// the pair sets are identical.  A scan of the per-target counts, a scatter into
// the target rows and a segmented sort of every row give the target-sorted lists
// of sort_by_target (src/interaction_list.jl:183-213) with a canonical order inside
// each target (the reference's is depth-first): by source index, or, for the M2L
// rows of an error-controlled solve, by decreasing (r_s + r_t) / separation and then
// source index, so that the pairs of one lane-per-pair pass stop at similar orders.
// The result does not depend on the order in which the atomics were served.
// The host synchronises twice per build: after the traversal (totals, capacity
// check) and after the row compaction (row counts).
#include <climits>

#include <cub/cub.cuh>
#include <cub/block/block_merge_sort.cuh>
#include <cub/warp/warp_merge_sort.cuh>

#include "context.cuh"

namespace fmmb {

namespace {

enum : int { A_NONE = 0, A_DIRECT = 1, A_M2L = 2, A_SPLIT_T = 3, A_SPLIT_S = 4 };

// per branch of one tree in its role: centre and radius (target ones for the target
// tree, source ones for the source tree), and (n_children, child_start, body_count)
struct TreeRef {
  const double4* geo;
  const int4* info;
};

struct Rule {
  double mac;
  int64_t ls;  // source leaf size (SelfTuning)
  int method;
  bool ff, nf, si;
};

__device__ __forceinline__ bool mac_accept(const double4& tg, const double4& sg, double mac) {
  double dx = tg.x - sg.x;
  double dy = tg.y - sg.y;
  double dz = tg.z - sg.z;
  double sep2 = dx * dx + dy * dy + dz * dz;
  double summed = sg.w + tg.w;
  return sep2 * mac * mac > summed * summed;
}

// one step of build_interaction_lists! for the three rule sets
// (src/interaction_list.jl:23-64, 66-120, 122-166); for a split, n_next children
// starting at child0 (of the target for A_SPLIT_T, of the source for A_SPLIT_S)
__device__ int decide(const TreeRef& T, int t, const TreeRef& S, int s, const Rule& R, int& n_next, int& child0) {
  n_next = 0;
  child0 = 0;
  const int4 ti = T.info[t], si = S.info[s];
  const int nct = ti.x, ncs = si.x;
  const int bt = ti.z, bs = si.z;
  bool both_leaves = (nct == 0) && (ncs == 0);
  bool dir_ok = (R.nf || (t == s && R.si)) && (t != s || R.si);
  if (R.method == FMM_LIST_BARBA) {
    const double4 tg = T.geo[t], sg = S.geo[s];
    if (mac_accept(tg, sg, R.mac)) return R.ff ? A_M2L : A_NONE;
    if (both_leaves) return dir_ok ? A_DIRECT : A_NONE;
    // target radius decides the side (src/interaction_list.jl:48)
    if (ncs == 0 || (tg.w >= sg.w && nct != 0)) {
      n_next = nct;
      child0 = ti.y;
      return A_SPLIT_T;
    }
    n_next = ncs;
    child0 = si.y;
    return A_SPLIT_S;
  }
  if (R.method == FMM_LIST_SELF_TUNING) {
    double fraction = 0.0;
    fraction = fraction + (double)bs / (double)(R.ls * R.ls);
    fraction = fraction * (double)bt;
    if (fraction < 1.0 || both_leaves) return (R.nf && (t != s || R.si)) ? A_DIRECT : A_NONE;
    if (mac_accept(T.geo[t], S.geo[s], R.mac)) return R.ff ? A_M2L : A_NONE;
  } else {  // SelfTuningTreeStop
    if (both_leaves) return dir_ok ? A_DIRECT : A_NONE;
    if (mac_accept(T.geo[t], S.geo[s], R.mac)) return R.ff ? A_M2L : A_NONE;
  }
  if (ncs == 0 || (bt >= bs && nct != 0)) {
    n_next = nct;
    child0 = ti.y;
    return A_SPLIT_T;
  }
  n_next = ncs;
  child0 = si.y;
  return A_SPLIT_S;
}

__global__ void k_pack_nodes(int n, const double* __restrict__ center, const double* __restrict__ radius,
                             const int* __restrict__ n_children, const int* __restrict__ child_start,
                             const int* __restrict__ body_count, double4* __restrict__ geo, int4* __restrict__ info) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    geo[i] = make_double4(center[3 * i], center[3 * i + 1], center[3 * i + 2], radius[i]);
    info[i] = make_int4(n_children[i], child_start[i], body_count[i], 0);
  }
}

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxSteps = 64;  // frontier counters; a traversal takes levels_t + levels_s - 1 steps
enum : int { C_DIR = kMaxSteps, C_M2L, C_FLAG, C_ROWS_DIR, C_ROWS_M2L = C_ROWS_DIR + 8, C_N = 128 };
constexpr int kStepThreads = 128;
constexpr int kStepMaxBlocks = 148 * 16;

__global__ void k_root_pair(int2* front, int* ctr) {
  front[0] = make_int2(0, 0);
  ctr[0] = 1;
}

// Add one to cnt[t] for the lanes that pass, one atomic per distinct target of the warp.
__device__ __forceinline__ void count_targets(bool on, int t, int lane, int* __restrict__ cnt) {
  const unsigned grp = __match_any_sync(kFull, on ? t : -1 - lane);
  if (on && lane == __ffs(grp) - 1) atomicAdd(cnt + t, __popc(grp));
}

constexpr int kStepItems = 4;                              // pairs per thread and chunk
constexpr int kStepChunk = kStepThreads * kStepItems;      // pairs per block and chunk

// Step k of the traversal: every pair of the frontier (ctr[k] pairs) is decided;
// direct and M2L pairs go to the raw lists and count for their target, split
// pairs put their children into the next frontier (ctr[k + 1] pairs).  A block
// takes the slots of a whole chunk with one atomic per counter.  Slots past a
// capacity are not written and raise the flag, which stops the later steps (the
// host grows the buffers and repeats).
__global__ void __launch_bounds__(kStepThreads) k_step(const int2* __restrict__ fin, int2* __restrict__ fout, int k,
                                                      TreeRef T, TreeRef S, Rule R, int2* __restrict__ rdir,
                                                      int2* __restrict__ rm2l, int* __restrict__ cdir,
                                                      int* __restrict__ cm2l, int* __restrict__ ctr, int cap_f,
                                                      int cap_d, int cap_m) {
  constexpr int NW = kStepThreads / 32;
  __shared__ int wsum[3][NW];
  __shared__ int bbase[3];
  __shared__ int stop;
  // after an overflow the frontier holds unwritten slots: the steps that follow do
  // nothing, and the host grows the buffers and repeats the traversal.  Another block
  // of this step may raise the flag meanwhile, so one thread reads it for the block:
  // the block leaves or stays as a whole (its barriers and block sums need every warp)
  if (threadIdx.x == 0) stop = *reinterpret_cast<volatile int*>(ctr + C_FLAG);
  __syncthreads();
  if (stop) return;
  const int n = min(ctr[k], cap_f);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  bool bad = false;
  for (int c0 = blockIdx.x * kStepChunk; c0 < n; c0 += gridDim.x * kStepChunk) {
    int2 p[kStepItems];
    int a[kStepItems], nn[kStepItems], ch[kStepItems];
    int cd = 0, cm = 0, cf = 0;
#pragma unroll
    for (int r = 0; r < kStepItems; ++r) {
      const int i = c0 + r * kStepThreads + threadIdx.x;
      p[r] = make_int2(0, 0);
      a[r] = A_NONE;
      nn[r] = 0;
      ch[r] = 0;
      if (i < n) {
        p[r] = fin[i];
        a[r] = decide(T, p[r].x, S, p[r].y, R, nn[r], ch[r]);
      }
      if (a[r] != A_SPLIT_T && a[r] != A_SPLIT_S) nn[r] = 0;
      cd += a[r] == A_DIRECT;
      cm += a[r] == A_M2L;
      cf += nn[r];
    }
    // block exclusive scan of (cd, cm, cf)
    int id = cd, im = cm, jf = cf;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(kFull, id, o), y = __shfl_up_sync(kFull, im, o), z = __shfl_up_sync(kFull, jf, o);
      if (lane >= o) id += x, im += y, jf += z;
    }
    if (lane == 31) wsum[0][w] = id, wsum[1][w] = im, wsum[2][w] = jf;
    __syncthreads();
    if (threadIdx.x < 3) {
      int tot = 0;
      for (int q = 0; q < NW; ++q) tot += wsum[threadIdx.x][q];
      const int slot = threadIdx.x == 0 ? C_DIR : threadIdx.x == 1 ? C_M2L : k + 1;
      bbase[threadIdx.x] = tot ? atomicAdd(ctr + slot, tot) : 0;
    }
    __syncthreads();
    int od = bbase[0] + id - cd, om = bbase[1] + im - cm, of = bbase[2] + jf - cf;
    for (int q = 0; q < w; ++q) od += wsum[0][q], om += wsum[1][q], of += wsum[2][q];
#pragma unroll
    for (int r = 0; r < kStepItems; ++r) {
      if (a[r] == A_DIRECT) {
        if (od < cap_d)
          rdir[od] = p[r];
        else
          bad = true;
        ++od;
      } else if (a[r] == A_M2L) {
        if (om < cap_m)
          rm2l[om] = p[r];
        else
          bad = true;
        ++om;
      } else if (nn[r]) {
        if (of + nn[r] > cap_f) {
          bad = true;
        } else if (a[r] == A_SPLIT_T) {
          for (int c = 0; c < nn[r]; ++c) fout[of + c] = make_int2(ch[r] + c, p[r].y);
        } else {
          for (int c = 0; c < nn[r]; ++c) fout[of + c] = make_int2(p[r].x, ch[r] + c);
        }
        of += nn[r];
      }
      count_targets(a[r] == A_DIRECT, p[r].x, lane, cdir);
      count_targets(a[r] == A_M2L, p[r].x, lane, cm2l);
    }
    __syncthreads();  // wsum / bbase are rewritten by the next chunk
  }
  if (bad) atomicOr(ctr + C_FLAG, 1);
}

// per target: (count << 32) | (count > 0), so that one exclusive scan gives both the
// row offset (high word) and the row ordinal among the non-empty targets (low word)
__global__ void k_pack_counts(const int* __restrict__ cnt, int n, unsigned long long* __restrict__ pk) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int c = cnt[t];
    pk[t] = ((unsigned long long)(unsigned)c << 32) | (c > 0 ? 1ull : 0ull);
  }
}

constexpr int kSmallRow = 256;  // rows up to this length: one warp each (merge sort in registers)
constexpr int kMidRow = 4096;   // up to this length: one block each; longer: segmented radix sort
constexpr int kMidClasses = 4;  // block sorts of 512, 1024, 2048 and 4096 keys
constexpr int kRowCtr = 2 + kMidClasses;  // per list: rows, rows per block class, big rows

__host__ __device__ constexpr int mid_class(int c) { return c <= 512 ? 0 : c <= 1024 ? 1 : c <= 2048 ? 2 : 3; }

// offsets of all targets (off, n + 1), the CSR of the non-empty ones (tgt, roff),
// and the rows too long for a warp sort: row ordinals per block class (mid, n + 1
// per class) and the bounds of the longer rows (big)
__global__ void k_rows(const int* __restrict__ cnt, const unsigned long long* __restrict__ ex, int n,
                       int* __restrict__ off, int* __restrict__ tgt, int* __restrict__ roff, int* __restrict__ ctr,
                       int* __restrict__ mid, int* __restrict__ big_b, int* __restrict__ big_e,
                       int* __restrict__ big_r) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= n; t += gridDim.x * blockDim.x) {
    const unsigned long long e = ex[t];
    const int o = (int)(e >> 32), r = (int)(e & 0xffffffffu);
    off[t] = o;
    if (t < n) {
      const int c = cnt[t];
      if (c > 0) {
        tgt[r] = t;
        roff[r] = o;
      }
      if (c > kMidRow) {
        const int q = atomicAdd(ctr + 1 + kMidClasses, 1);
        big_b[q] = o;
        big_e[q] = o + c;
        big_r[q] = r;
      } else if (c > kSmallRow) {
        const int k = mid_class(c);
        mid[(size_t)k * (n + 1) + atomicAdd(ctr + 1 + k, 1)] = r;
      }
    } else {
      roff[r] = o;
      ctr[0] = r;
    }
  }
}

// raw pairs into their target's row, sources only (order inside a row fixed by the
// sort that follows); one cursor atomic per distinct target of a warp
__global__ void k_scatter(const int2* __restrict__ raw, int n, const int* __restrict__ off, int* __restrict__ cursor,
                          int* __restrict__ out_s) {
  const int lane = threadIdx.x & 31;
  for (int w0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); w0 < n; w0 += gridDim.x * blockDim.x) {
    const int i = w0 + lane;
    const bool on = i < n;
    const int2 p = on ? raw[i] : make_int2(-1 - lane, 0);
    const unsigned grp = __match_any_sync(kFull, p.x);
    const int leader = __ffs(grp) - 1;
    int b = 0;
    if (on && lane == leader) b = atomicAdd(cursor + p.x, __popc(grp));
    b = __shfl_sync(kFull, b, leader);
    if (on) out_s[off[p.x] + b + __popc(grp & ((1u << lane) - 1u))] = p.y;
  }
}

struct KeyLess {
  __device__ __forceinline__ bool operator()(unsigned a, unsigned b) const { return a < b; }
};

// Sort key of a row entry: its source index, or, for M2L rows ordered by separation,
// (4095 - q) << 20 | source with q = floor(4095 (r_s + r_t) / |c_t - c_s|) clamped to
// [0, 4095]: the pairs of one target that need high expansion orders come first and
// neighbouring pairs need similar orders (source indices < 2^20 on that path).
constexpr int kSepShift = 20;
struct RowKey {
  const double4* sgeo;  // null: source order
  double4 tg;
  __device__ __forceinline__ unsigned enc(int s) const {
    if (!sgeo) return (unsigned)s;
    const double4 sg = sgeo[s];
    const double dx = tg.x - sg.x, dy = tg.y - sg.y, dz = tg.z - sg.z;
    const double rho = (sg.w + tg.w) / sqrt(dx * dx + dy * dy + dz * dz);
    const int q = (int)fmin(4095.0, fmax(0.0, rho * 4095.0));
    return ((unsigned)(4095 - q) << kSepShift) | (unsigned)s;
  }
  __device__ __forceinline__ int dec(unsigned k) const {
    return sgeo ? (int)(k & ((1u << kSepShift) - 1u)) : (int)k;
  }
};
__device__ __forceinline__ RowKey row_key(const double4* tgeo, const double4* sgeo, int t) {
  RowKey k;
  k.sgeo = sgeo;
  k.tg = sgeo ? tgeo[t] : make_double4(0, 0, 0, 0);
  return k;
}

constexpr int kSortWarps = 8;

// rows of 32 (ITEMS / 2) + 1 .. 32 ITEMS entries (1 .. 32 for ITEMS = 1): one warp per row
template <int ITEMS>
__global__ void __launch_bounds__(kSortWarps * 32) k_sort_warp(const int* __restrict__ tgt,
                                                                const int* __restrict__ roff, int n_rows,
                                                                const int* __restrict__ in, int* __restrict__ out_t,
                                                                int* __restrict__ out_s, const double4* tgeo,
                                                                const double4* sgeo) {
  using WMS = cub::WarpMergeSort<unsigned, ITEMS, 32>;
  __shared__ typename WMS::TempStorage tmp[kSortWarps];
  constexpr int lo = ITEMS == 1 ? 1 : 16 * ITEMS + 1, hi = 32 * ITEMS;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WMS ws(tmp[w]);
  for (int r = blockIdx.x * kSortWarps + w; r < n_rows; r += gridDim.x * kSortWarps) {
    const int b = roff[r], len = roff[r + 1] - b;
    if (len < lo || len > hi) continue;
    const int t = tgt[r];
    if (len == 1) {
      if (lane == 0) out_t[b] = t, out_s[b] = in[b];
      continue;
    }
    const RowKey rk = row_key(tgeo, sgeo, t);
    unsigned keys[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int i = lane * ITEMS + j;
      keys[j] = i < len ? rk.enc(in[b + i]) : UINT_MAX;
    }
    ws.Sort(keys, KeyLess(), len, UINT_MAX);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const int i = lane * ITEMS + j;
      if (i < len) out_t[b + i] = t, out_s[b + i] = rk.dec(keys[j]);
    }
    __syncwarp();
  }
}

// rows of one block class: one block of THREADS x ITEMS keys per row
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) k_sort_block(const int* __restrict__ mid, const int* __restrict__ tgt,
                                                      const int* __restrict__ roff, const int* __restrict__ in,
                                                      int* __restrict__ out_t, int* __restrict__ out_s,
                                                      const double4* tgeo, const double4* sgeo) {
  using BMS = cub::BlockMergeSort<unsigned, THREADS, ITEMS>;
  __shared__ typename BMS::TempStorage tmp;
  const int r = mid[blockIdx.x];
  const int b = roff[r], len = roff[r + 1] - b, t = tgt[r];
  const RowKey rk = row_key(tgeo, sgeo, t);
  unsigned keys[ITEMS];
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = threadIdx.x * ITEMS + j;
    keys[j] = i < len ? rk.enc(in[b + i]) : UINT_MAX;
  }
  BMS(tmp).Sort(keys, KeyLess(), len, UINT_MAX);
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = threadIdx.x * ITEMS + j;
    if (i < len) out_t[b + i] = t, out_s[b + i] = rk.dec(keys[j]);
  }
}

// target column of the rows sorted by the segmented radix sort
__global__ void k_fill_rows(const int* __restrict__ big_r, const int* __restrict__ tgt, const int* __restrict__ roff,
                            int* __restrict__ out_t) {
  const int r = big_r[blockIdx.x];
  const int b = roff[r], e = roff[r + 1], t = tgt[r];
  for (int i = b + threadIdx.x; i < e; i += blockDim.x) out_t[i] = t;
}

int blocks_for(int64_t n, int threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, kStepMaxBlocks));
}

// one list (direct or M2L) being turned into target rows
struct RowBuild {
  const int* cnt;
  const int2* raw;
  int n;
  DevBuf<int>*out_t, *out_s, *tgt, *roff;
  DevBuf<int>* off;
  DevBuf<int>* tmp;
  int* ctr;  // rows, rows per block class, big rows (kRowCtr ints)
  const double4* tgeo = nullptr;  // non-null: rows up to kMidRow ordered by separation (RowKey)
  const double4* sgeo = nullptr;
};

// offsets and row CSR (before the host reads the row counts)
void rows_of(RowBuild& B, int nt, Scratch& sc, cudaStream_t st) {
  B.out_t->grow((size_t)B.n + 1);
  B.out_s->grow((size_t)B.n + 1);
  B.tgt->grow((size_t)nt + 1);
  B.roff->grow((size_t)nt + 2);
  B.off->grow((size_t)nt + 1);
  sc.keys_a.grow((size_t)nt + 1);
  sc.keys_b.grow((size_t)nt + 1);
  note_launch();
  k_pack_counts<<<blocks_for(nt + 1, 256), 256, 0, st>>>(B.cnt, nt + 1, sc.keys_a.ptr);
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, sc.keys_a.ptr, sc.keys_b.ptr, nt + 1, st);
  sc.cub.grow(tb);
  FMM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(sc.cub.ptr, tb, sc.keys_a.ptr, sc.keys_b.ptr, nt + 1, st));
  note_launch();
  k_rows<<<blocks_for(nt + 1, 256), 256, 0, st>>>(B.cnt, sc.keys_b.ptr, nt, B.off->ptr, B.tgt->ptr, B.roff->ptr,
                                                  B.ctr, sc.row_mid.ptr, sc.row_big_b.ptr, sc.row_big_e.ptr,
                                                  sc.row_big_r.ptr);
  FMM_CUDA_TRY(cudaGetLastError());
}

// scatter into rows and sort every row by source index (after the host read the counts:
// h = rows, rows per block class, big rows)
void sort_rows(RowBuild& B, int nt, const int* h, int nbits, Scratch& sc, cudaStream_t st) {
  if (B.n == 0) return;
  const int rows = h[0], n_big = h[1 + kMidClasses];
  B.tmp->grow((size_t)B.n + 1);
  sc.row_cur.grow((size_t)nt + 1);
  FMM_CUDA_TRY(cudaMemsetAsync(sc.row_cur.ptr, 0, (size_t)nt * sizeof(int), st));
  note_launch();
  k_scatter<<<blocks_for(B.n, 256), 256, 0, st>>>(B.raw, B.n, B.off->ptr, sc.row_cur.ptr, B.tmp->ptr);
  const int gw = blocks_for((int64_t)rows * 32, kSortWarps * 32);
  note_launch();
  k_sort_warp<1><<<gw, kSortWarps * 32, 0, st>>>(B.tgt->ptr, B.roff->ptr, rows, B.tmp->ptr, B.out_t->ptr, B.out_s->ptr,
                                                  B.tgeo, B.sgeo);
  note_launch();
  k_sort_warp<2><<<gw, kSortWarps * 32, 0, st>>>(B.tgt->ptr, B.roff->ptr, rows, B.tmp->ptr, B.out_t->ptr, B.out_s->ptr,
                                                  B.tgeo, B.sgeo);
  note_launch();
  k_sort_warp<4><<<gw, kSortWarps * 32, 0, st>>>(B.tgt->ptr, B.roff->ptr, rows, B.tmp->ptr, B.out_t->ptr, B.out_s->ptr,
                                                  B.tgeo, B.sgeo);
  note_launch();
  k_sort_warp<8><<<gw, kSortWarps * 32, 0, st>>>(B.tgt->ptr, B.roff->ptr, rows, B.tmp->ptr, B.out_t->ptr, B.out_s->ptr,
                                                  B.tgeo, B.sgeo);
  FMM_CUDA_TRY(cudaGetLastError());
  const int* mid = sc.row_mid.ptr;
  const size_t stride = (size_t)nt + 1;
  if (h[1] > 0) {
    note_launch();
    k_sort_block<128, 4><<<h[1], 128, 0, st>>>(mid, B.tgt->ptr, B.roff->ptr, B.tmp->ptr, B.out_t->ptr, B.out_s->ptr,
                                               B.tgeo, B.sgeo);
  }
  if (h[2] > 0) {
    note_launch();
    k_sort_block<256, 4><<<h[2], 256, 0, st>>>(mid + stride, B.tgt->ptr, B.roff->ptr, B.tmp->ptr, B.out_t->ptr,
                                               B.out_s->ptr, B.tgeo, B.sgeo);
  }
  if (h[3] > 0) {
    note_launch();
    k_sort_block<256, 8><<<h[3], 256, 0, st>>>(mid + 2 * stride, B.tgt->ptr, B.roff->ptr, B.tmp->ptr, B.out_t->ptr,
                                               B.out_s->ptr, B.tgeo, B.sgeo);
  }
  if (h[4] > 0) {
    note_launch();
    k_sort_block<256, 16><<<h[4], 256, 0, st>>>(mid + 3 * stride, B.tgt->ptr, B.roff->ptr, B.tmp->ptr, B.out_t->ptr,
                                                B.out_s->ptr, B.tgeo, B.sgeo);
  }
  FMM_CUDA_TRY(cudaGetLastError());
  if (n_big > 0) {
    size_t tb = 0;
    cub::DeviceSegmentedRadixSort::SortKeys(nullptr, tb, B.tmp->ptr, B.out_s->ptr, B.n, n_big, sc.row_big_b.ptr,
                                            sc.row_big_e.ptr, 0, nbits, st);
    sc.cub.grow(tb);
    FMM_CUDA_TRY(cub::DeviceSegmentedRadixSort::SortKeys(sc.cub.ptr, tb, B.tmp->ptr, B.out_s->ptr, B.n, n_big,
                                                         sc.row_big_b.ptr, sc.row_big_e.ptr, 0, nbits, st));
    note_launch();
    k_fill_rows<<<n_big, 256, 0, st>>>(sc.row_big_r.ptr, B.tgt->ptr, B.roff->ptr, B.out_t->ptr);
    FMM_CUDA_TRY(cudaGetLastError());
  }
}

}  // namespace

void build_lists(DevLists& L, const DevTree& tt, const DevTree& stt, Scratch& sc, cudaStream_t st,
                 int64_t leaf_size_source, double mac, bool ff, bool nf, bool si, int method,
                 bool m2l_by_separation) {
  const int nt = (int)tt.n_branches, ns = (int)stt.n_branches;
  sc.node_geo_t.grow((size_t)nt);
  sc.node_info_t.grow((size_t)nt);
  sc.node_geo_s.grow((size_t)ns);
  sc.node_info_s.grow((size_t)ns);
  note_launch();
  k_pack_nodes<<<blocks_for(nt, 256), 256, 0, st>>>(nt, tt.tcenter.ptr, tt.tradius.ptr, tt.n_children.ptr,
                                                     tt.child_start.ptr, tt.body_count.ptr, sc.node_geo_t.ptr,
                                                     sc.node_info_t.ptr);
  note_launch();
  k_pack_nodes<<<blocks_for(ns, 256), 256, 0, st>>>(ns, stt.scenter.ptr, stt.sradius.ptr, stt.n_children.ptr,
                                                     stt.child_start.ptr, stt.body_count.ptr, sc.node_geo_s.ptr,
                                                     sc.node_info_s.ptr);
  FMM_CUDA_TRY(cudaGetLastError());
  TreeRef T{sc.node_geo_t.ptr, sc.node_info_t.ptr};
  TreeRef S{sc.node_geo_s.ptr, sc.node_info_s.ptr};
  Rule R{mac, leaf_size_source, method, ff, nf, si};
  const int n_steps = tt.n_levels + stt.n_levels - 1;
  FMM_CHECK(n_steps + 1 < kMaxSteps, FMM_ERR_TREE_DEPTH, "interaction-list traversal deeper than supported");
  sc.counts.grow(C_N);
  int* ctr = sc.counts.ptr;
  sc.cnt_a.grow((size_t)nt + 1);
  sc.cnt_b.grow((size_t)nt + 1);
  // capacities: kept from earlier builds, grown when a traversal reports more
  size_t cap_f = std::max<size_t>(4096, (size_t)nt * 32), cap_d = std::max<size_t>(4096, (size_t)tt.n_leaves * 64);
  size_t cap_m = std::max<size_t>(4096, (size_t)nt * 96);
  std::vector<int> h(C_N, 0);
  for (int attempt = 0;; ++attempt) {
    FMM_CHECK(attempt < 8, FMM_ERR_MEMORY, "interaction-list capacities did not converge");
    sc.front_a.grow(cap_f);
    sc.front_b.grow(cap_f);
    sc.dir_raw.grow(cap_d);
    sc.m2l_raw.grow(cap_m);
    const int cf = (int)std::min<size_t>(sc.front_a.cap, sc.front_b.cap);
    const int cd = (int)sc.dir_raw.cap, cm = (int)sc.m2l_raw.cap;
    FMM_CUDA_TRY(cudaMemsetAsync(ctr, 0, C_N * sizeof(int), st));
    FMM_CUDA_TRY(cudaMemsetAsync(sc.cnt_a.ptr, 0, ((size_t)nt + 1) * sizeof(int), st));
    FMM_CUDA_TRY(cudaMemsetAsync(sc.cnt_b.ptr, 0, ((size_t)nt + 1) * sizeof(int), st));
    note_launch();
    k_root_pair<<<1, 1, 0, st>>>(sc.front_a.ptr, ctr);
    for (int k = 0; k < n_steps; ++k) {
      const int2* fin = (k & 1) ? sc.front_b.ptr : sc.front_a.ptr;
      int2* fout = (k & 1) ? sc.front_a.ptr : sc.front_b.ptr;
      // grid from this scratch's previous build (the kernel strides over any frontier)
      const int64_t hint = k < (int)sc.step_hint.size() ? sc.step_hint[k] : (int64_t)kStepChunk * kStepMaxBlocks;
      note_launch();
      k_step<<<blocks_for(hint + hint / 4 + 32, kStepChunk), kStepThreads, 0, st>>>(
          fin, fout, k, T, S, R, sc.dir_raw.ptr, sc.m2l_raw.ptr, sc.cnt_a.ptr, sc.cnt_b.ptr, ctr, cf, cd, cm);
      FMM_CUDA_TRY(cudaGetLastError());
    }
    FMM_CUDA_TRY(cudaMemcpyAsync(h.data(), ctr, C_N * sizeof(int), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaStreamSynchronize(st));
    size_t max_f = 0;
    for (int k = 0; k <= n_steps; ++k) max_f = std::max(max_f, (size_t)(unsigned)h[k]);
    const size_t nd = (size_t)(unsigned)h[C_DIR], nm = (size_t)(unsigned)h[C_M2L];
    if (h[C_FLAG] || max_f > (size_t)cf || nd > (size_t)cd || nm > (size_t)cm) {
      // the counts after an overflow are partial: grow past them and at least double
      cap_f = std::max(2 * (size_t)cf, max_f + max_f / 4 + 64);
      cap_d = std::max(nd > (size_t)cd ? 2 * (size_t)cd : (size_t)cd, nd + nd / 4 + 64);
      cap_m = std::max(nm > (size_t)cm ? 2 * (size_t)cm : (size_t)cm, nm + nm / 4 + 64);
      continue;
    }
    FMM_CHECK(h[n_steps] == 0, FMM_ERR_TREE_DEPTH, "interaction-list traversal did not terminate");
    sc.step_hint.assign(h.begin(), h.begin() + n_steps);
    break;
  }
  const int n_dir = h[C_DIR], n_m2l = h[C_M2L];
  int nbits = 1;
  while ((1ll << nbits) <= stt.n_branches) ++nbits;
  // the row classes of one list are built (k_rows) and consumed (sort_rows) before the
  // next list's k_rows reuses the class arrays, so the lists take turns
  sc.row_mid.grow((size_t)kMidClasses * (nt + 1));
  sc.row_big_b.grow((size_t)nt + 1);
  sc.row_big_e.grow((size_t)nt + 1);
  sc.row_big_r.grow((size_t)nt + 1);
  RowBuild lists[2] = {
      {sc.cnt_a.ptr, sc.dir_raw.ptr, n_dir, &L.dir_t, &L.dir_s, &L.dir_tgt, &L.dir_off, &sc.row_off_a, &sc.row_tmp_a,
       ctr + C_ROWS_DIR},
      {sc.cnt_b.ptr, sc.m2l_raw.ptr, n_m2l, &L.m2l_t, &L.m2l_s, &L.m2l_tgt, &L.m2l_off, &sc.row_off_b, &sc.row_tmp_b,
       ctr + C_ROWS_M2L}};
  if (m2l_by_separation && ns < (1 << kSepShift)) {
    lists[1].tgeo = sc.node_geo_t.ptr;
    lists[1].sgeo = sc.node_geo_s.ptr;
  }
  int rows[2] = {0, 0};
  for (int q = 0; q < 2; ++q) {
    rows_of(lists[q], nt, sc, st);
    int hq[kRowCtr];
    FMM_CUDA_TRY(cudaMemcpyAsync(hq, lists[q].ctr, kRowCtr * sizeof(int), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaStreamSynchronize(st));
    rows[q] = hq[0];
    sort_rows(lists[q], nt, hq, nbits, sc, st);
  }
  L.n_direct = n_dir;
  L.n_m2l = n_m2l;
  L.n_dir_targets = rows[0];
  L.n_m2l_targets = rows[1];
  L.rule_mac = mac;
  L.rule_ls = leaf_size_source;
  L.rule_method = method;
  L.rule_ff = ff;
  L.rule_nf = nf;
  L.rule_si = si;
}

namespace {

constexpr int kMaxDepth = 24;      // ancestor chain of a branch (the octant key allows 21 levels)
constexpr int kStepsPerWord = 21;  // 3 bits per step, 63 bits per key word

// Depth-first rank of every pair: the reference's recursion (src/interaction_list.jl:3-166)
// reaches (t, s) from (root, root) by one split per step, each into the child that is an
// ancestor of t (target split) or of s (source split); the side is the rule's decision at
// that pair.  The child ordinals along the way (3 bits each, first step most significant)
// order the pairs as the recursion emits them (no emitted pair's path is a prefix of
// another's, so zero padding keeps the order).  An inconsistent path raises the flag.
__global__ void k_dfs_keys(const int* __restrict__ lt, const int* __restrict__ ls, int n, TreeRef T, TreeRef S,
                           const int* __restrict__ parent_t, const int* __restrict__ parent_s, Rule R,
                           unsigned long long* __restrict__ khi, unsigned long long* __restrict__ klo,
                           int* __restrict__ perm, int* __restrict__ flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int ct[kMaxDepth], cs[kMaxDepth];
    int nt = 0, ns = 0;
    for (int a = lt[i]; a >= 0 && nt < kMaxDepth; a = parent_t[a]) ct[nt++] = a;
    for (int b = ls[i]; b >= 0 && ns < kMaxDepth; b = parent_s[b]) cs[ns++] = b;
    unsigned long long hi = 0, lo = 0;
    bool bad = ct[nt - 1] != 0 || cs[ns - 1] != 0;
    int it = nt - 1, is = ns - 1, step = 0;
    while (!bad && (it > 0 || is > 0)) {
      int nn, c0;
      const int act = decide(T, ct[it], S, cs[is], R, nn, c0);
      int ord;
      if (act == A_SPLIT_T && it > 0) {
        ord = ct[it - 1] - c0;
        --it;
      } else if (act == A_SPLIT_S && is > 0) {
        ord = cs[is - 1] - c0;
        --is;
      } else {
        bad = true;
        break;
      }
      if (ord < 0 || ord >= nn || ord > 7 || step >= 2 * kStepsPerWord) {
        bad = true;
        break;
      }
      if (step < kStepsPerWord)
        hi |= (unsigned long long)ord << (3 * (kStepsPerWord - 1 - step));
      else
        lo |= (unsigned long long)ord << (3 * (2 * kStepsPerWord - 1 - step));
      ++step;
    }
    if (bad) atomicExch(flag, 1);
    khi[i] = hi;
    klo[i] = lo;
    perm[i] = i;
  }
}

__global__ void k_permute_u64(const unsigned long long* __restrict__ in, const int* __restrict__ perm, int n,
                              unsigned long long* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[perm[i]];
}

__global__ void k_gather_pairs(const int* __restrict__ lt, const int* __restrict__ ls, const int* __restrict__ perm,
                               int n, int2* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int j = perm[i];
    out[i] = make_int2(lt[j], ls[j]);
  }
}

}  // namespace

void export_lists_reference_order(const DevLists& L, const DevTree& tt, const DevTree& stt, Scratch& sc,
                                  cudaStream_t st, int32_t* m2l, int32_t* direct) {
  const int nt = (int)tt.n_branches, ns = (int)stt.n_branches;
  sc.node_geo_t.grow((size_t)nt);
  sc.node_info_t.grow((size_t)nt);
  sc.node_geo_s.grow((size_t)ns);
  sc.node_info_s.grow((size_t)ns);
  note_launch();
  k_pack_nodes<<<blocks_for(nt, 256), 256, 0, st>>>(nt, tt.tcenter.ptr, tt.tradius.ptr, tt.n_children.ptr,
                                                     tt.child_start.ptr, tt.body_count.ptr, sc.node_geo_t.ptr,
                                                     sc.node_info_t.ptr);
  note_launch();
  k_pack_nodes<<<blocks_for(ns, 256), 256, 0, st>>>(ns, stt.scenter.ptr, stt.sradius.ptr, stt.n_children.ptr,
                                                     stt.child_start.ptr, stt.body_count.ptr, sc.node_geo_s.ptr,
                                                     sc.node_info_s.ptr);
  FMM_CUDA_TRY(cudaGetLastError());
  const TreeRef T{sc.node_geo_t.ptr, sc.node_info_t.ptr};
  const TreeRef S{sc.node_geo_s.ptr, sc.node_info_s.ptr};
  const Rule R{L.rule_mac, L.rule_ls, L.rule_method, L.rule_ff, L.rule_nf, L.rule_si};
  struct One {
    const DevBuf<int>*t, *s, *off;
    int64_t n, rows;
    int32_t* dst;
  } lists[2] = {{&L.m2l_t, &L.m2l_s, &L.m2l_off, L.n_m2l, L.n_m2l_targets, m2l},
                {&L.dir_t, &L.dir_s, &L.dir_off, L.n_direct, L.n_dir_targets, direct}};
  sc.flag.grow(1);
  for (const One& q : lists) {
    if (!q.dst || q.n == 0) continue;
    const int n = (int)q.n, rows = (int)q.rows;
    sc.keys_a.grow(2 * (size_t)n);
    sc.keys_b.grow(2 * (size_t)n);
    sc.vals_a.grow((size_t)n);
    sc.vals_b.grow((size_t)n);
    unsigned long long *hi = sc.keys_a.ptr, *lo = sc.keys_a.ptr + n, *k1 = sc.keys_b.ptr, *k2 = sc.keys_b.ptr + n;
    FMM_CUDA_TRY(cudaMemsetAsync(sc.flag.ptr, 0, sizeof(int), st));
    note_launch();
    k_dfs_keys<<<blocks_for(n, 256), 256, 0, st>>>(q.t->ptr, q.s->ptr, n, T, S, tt.parent.ptr, stt.parent.ptr, R, hi,
                                                  lo, sc.vals_a.ptr, sc.flag.ptr);
    FMM_CUDA_TRY(cudaGetLastError());
    // lexicographic (hi, lo) inside every row: stable sort by lo, then stable sort by hi
    const int* beg = q.off->ptr;
    const int* end = q.off->ptr + 1;
    size_t tb = 0, tb2 = 0;
    FMM_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(nullptr, tb, lo, k1, sc.vals_a.ptr, sc.vals_b.ptr, n, rows,
                                                           beg, end, st));
    FMM_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(nullptr, tb2, hi, k2, sc.vals_b.ptr, sc.vals_a.ptr, n,
                                                           rows, beg, end, st));
    sc.cub.grow(std::max(tb, tb2));
    note_launch();
    FMM_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(sc.cub.ptr, tb, lo, k1, sc.vals_a.ptr, sc.vals_b.ptr, n,
                                                           rows, beg, end, st));
    // the second pass needs the hi keys in the order of the first: gather them
    note_launch();
    k_permute_u64<<<blocks_for(n, 256), 256, 0, st>>>(hi, sc.vals_b.ptr, n, lo);
    note_launch();
    FMM_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(sc.cub.ptr, tb2, lo, k2, sc.vals_b.ptr, sc.vals_a.ptr, n,
                                                           rows, beg, end, st));
    sc.front_a.grow((size_t)n);
    note_launch();
    k_gather_pairs<<<blocks_for(n, 256), 256, 0, st>>>(q.t->ptr, q.s->ptr, sc.vals_a.ptr, n, sc.front_a.ptr);
    FMM_CUDA_TRY(cudaGetLastError());
    int bad = 0;
    FMM_CUDA_TRY(cudaMemcpyAsync(&bad, sc.flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaMemcpyAsync(q.dst, sc.front_a.ptr, (size_t)n * sizeof(int2), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaStreamSynchronize(st));
    FMM_CHECK(!bad, FMM_ERR_STATE, "a list pair is not reachable by the traversal rule (reference-order export)");
  }
}

}  // namespace fmmb
