// context.cuh -- device-resident data of one FMM solve and the launch interfaces
// of the tree, list and evaluation stages.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace fmmb {

// An octree in HBM (the reference's Tree/Branch, src/containers.jl:150-195),
// struct-of-arrays, branches in breadth-first order.
struct DevTree {
  int64_t n_bodies = 0, n_branches = 0, n_leaves = 0;
  int n_levels = 0;
  std::vector<int64_t> levels_start, levels_end;  // host copy of levels_index
  // branch fields
  DevBuf<int> body_start, body_count, child_start, n_children, parent, i_leaf, level;
  DevBuf<double> gcenter;                // geometric cell centre (3 per branch)
  DevBuf<double> gbox, gradius;          // geometric half width / radius (per branch)
  DevBuf<double> tcenter, scenter;       // target / source centre (3 per branch)
  DevBuf<double> tradius, sradius;
  DevBuf<double> tbox, sbox;             // 3 per branch
  DevBuf<double> max_influence;
  DevBuf<int> leaf_index;                // leaf ordinal -> branch
  DevBuf<int> sort_index;                // sorted position -> original body index
  // bodies in sorted order
  DevBuf<double4> pos;                   // x y z radius
  DevBuf<double4> str;                   // strength (1 or 3 components)
  // expansions, 4*Nh doubles per branch: multipole (source role) and local (target role);
  // one tree can play both roles when the targets are the sources
  DevBuf<double> multipole, local;
  int p = 0;
};

// Interaction lists (pairs of branch indices), sorted by target, plus the
// per-target CSR used by the target-owned kernels.
struct DevLists {
  int64_t n_m2l = 0, n_direct = 0;
  DevBuf<int> m2l_t, m2l_s, dir_t, dir_s;
  int64_t n_m2l_targets = 0, n_dir_targets = 0;
  DevBuf<int> m2l_tgt, m2l_off;   // unique targets, offsets (n+1)
  DevBuf<int> dir_tgt, dir_off;
  // near field of launches of few rows: rows cut into chunks of source leaves (row, leaf range,
  // offset of the chunk's partial sums), their partial sums, and each row's chunk range
  DevBuf<int4> p2p_chunks, p2p_rowtab;
  DevBuf<double> p2p_part;
  // the traversal's rule (for the reference-order export)
  double rule_mac = 0.5;
  int64_t rule_ls = 1;
  int rule_method = 0;
  bool rule_ff = true, rule_nf = true, rule_si = true;
};

// Scratch shared by the stages of one solve.
struct Scratch {
  DevBuf<unsigned char> cub;            // CUB temporary storage
  DevBuf<unsigned long long> keys_a, keys_b;
  DevBuf<int> vals_a, vals_b, tmp_i, tmp_j, tmp_k;
  DevBuf<int2> front_a, front_b;        // traversal frontiers
  DevBuf<int2> dir_raw, m2l_raw;        // list pairs of the traversal in arrival order
  DevBuf<int> cnt_a, cnt_b;             // pairs per target (direct, M2L)
  DevBuf<int> counts;                   // small host-visible counters
  DevBuf<double> tmp_d;
  DevBuf<double> staging;               // raw caller buffers copied to HBM
  DevBuf<double> out16;                 // target buffer in original order
  DevBuf<int> flag;
  std::vector<int> step_hint;           // frontier sizes of the previous list build (launch shapes)
  // target rows of the lists: offsets of all targets, unsorted rows, row classes
  DevBuf<int> row_off_a, row_off_b, row_tmp_a, row_tmp_b, row_cur, row_mid, row_big_b, row_big_e, row_big_r;
  // branch records of the two trees for the traversal (centre + radius, counts)
  DevBuf<double4> node_geo_t, node_geo_s;
  DevBuf<int4> node_info_t, node_info_s;
};

struct DevTables {
  int p = -1;
  DevBuf<double> Hs, zeta, eta, Mt, Lt;
};

struct Stream {
  cudaStream_t s = nullptr;
};

// ---- tree.cu ----
// Build `t` from bodies already unpacked to t.pos / t.str (original order);
// sorts them, creates branches, shrinks (optional) and permutes the bodies.
void build_tree(DevTree& t, Scratch& sc, cudaStream_t st, int64_t leaf_size, int method, bool shrink);
// Unpack a caller buffer (body-major, stride doubles) into pos/str (original order).
void unpack_bodies(DevTree& t, const double* dev_buf, int64_t n, int64_t stride, int n_strength,
                   bool has_radius, cudaStream_t st);
// max_influence of every branch from |gradient| of the original bodies (one per body, caller's order).
void branch_max_influence(DevTree& t, const double* gnorm_orig, cudaStream_t st);

// ---- lists.cu ----
// m2l_by_separation: M2L rows ordered by decreasing (r_s + r_t) / separation (pairs that
// need similar expansion orders side by side), else every row by source index
void build_lists(DevLists& L, const DevTree& tt, const DevTree& stt, Scratch& sc, cudaStream_t st,
                 int64_t leaf_size_source, double mac, bool ff, bool nf, bool si, int method,
                 bool m2l_by_separation);
// The lists of the last build in the reference's order: target rows ascending and, inside a
// row, the order in which the depth-first recursion emitted the pairs (host arrays of
// (target, source) pairs, n_m2l / n_direct of them; either may be null).
void export_lists_reference_order(const DevLists& L, const DevTree& tt, const DevTree& stt, Scratch& sc,
                                  cudaStream_t st, int32_t* m2l, int32_t* direct);

// ---- p2p.cu ----
// Near field over the direct list; accumulates into acc13 (sorted target order, 13 per body).
// exact_self: on the mixed path, evaluate the batch holding the target's own leaf in FP64
void launch_p2p(const DevTree& tt, const DevTree& stt, DevLists& L, double* acc13, int kind, bool ps,
                bool gs, bool hs, int precision, cudaStream_t st, bool exact_self = true);
// sum over the direct list of n_target * n_source (atomically added to *out)
void count_p2p_pairs(const DevTree& tt, const DevTree& stt, const DevLists& L, unsigned long long* out,
                     cudaStream_t st);
// All pairs (direct!): targets in pos order, sources; writes acc13.
void launch_direct(const double4* tpos, int64_t nt, const double4* spos, const double4* sstr, int64_t ns,
                   double* acc13, int kind, bool gs, bool hs, int precision, cudaStream_t st);

// ---- expansions.cu ----
void upload_tables(DevTables& dt, int p, cudaStream_t st);
void launch_p2m(DevTree& s, int p, int kind, const DevTables& tb, cudaStream_t st);
void launch_m2m(DevTree& s, int p, bool lh, const DevTables& tb, cudaStream_t st);
// per-pair orders go to p_used (device, one per m2l entry) when non-null; stats (device,
// 4 ints, zeroed by the caller) receives the max order, a failure flag and the flop count
// lane-per-pair M2L (m2l_lane.cu): point sources, orders 1..12; false = not handled
// lane-per-child M2M (orders 1..12) / L2L (orders 1..6), point sources (m2l_lane.cu); false = not handled
bool launch_m2m_lane(DevTree& s, int p, bool lh, cudaStream_t st);
bool launch_l2l_lane(DevTree& t, int p, bool lh, cudaStream_t st);
bool launch_m2l_lane(DevTree& t, const DevTree& s, const DevLists& L, int p, bool lh, int em, double eps, int be,
                     int* p_used, int* stats, int precision, cudaStream_t st);
void launch_m2l(DevTree& t, const DevTree& s, const DevLists& L, int p, bool lh, int error_method, double eps,
                int be, int* p_used, int* stats, const DevTables& tb, int precision, cudaStream_t st);
void launch_l2l(DevTree& t, int p, bool lh, const DevTables& tb, cudaStream_t st);
void launch_l2p(DevTree& t, int p, bool lh, bool ps, bool gs, bool hs, double* acc13, cudaStream_t st);
// unit operators over explicit pair lists (device arrays)
void launch_op_m2m(int64_t n, double* target, const double* tc, const double* src, const double* sc, int p,
                   bool lh, bool local, const DevTables& tb, cudaStream_t st);
void launch_op_m2l(int64_t n, double* target, const double* tc, const double* tbox, const double* trad,
                   const double* maxinf, const double* src, const double* sc, int p, bool lh, int error_method,
                   double eps, int be, int* p_used, const DevTables& tb, cudaStream_t st);
void launch_op_p2m(int kind, const double4* pos, const double4* str, int64_t n, const double* center, int p,
                   double* expansion, cudaStream_t st);
void launch_op_l2p(int64_t n, const double* dx, const double* local, int p, bool lh, bool ps, bool gs, bool hs,
                   double* out13, cudaStream_t st);

}  // namespace fmmb
