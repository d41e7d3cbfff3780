// fmm.cpp -- TEST INFRASTRUCTURE ONLY (see fmm_oracle.h).
// FP64 restatement of the reference's octree (src/tree.jl), dual-tree
// interaction lists (src/interaction_list.jl), the P2P kernels of the
// reference's test systems (test/gravitational.jl, test/vortex.jl) and the
// fmm!/direct! drivers (src/fmm.jl, src/direct.jl), parallelised with threads
// over target-owned units exactly as the reference's threaded passes are
// (a target branch is only ever written by one thread).
#include <algorithm>
#include <atomic>
#include <thread>
#include <chrono>
#include <cstring>
#include <memory>

#include "fmm_oracle.h"
#include "internal.h"

namespace orc {

static int g_threads = 0;  // <= 0: hardware concurrency

static int n_workers() {
  int n = g_threads > 0 ? g_threads : (int)std::thread::hardware_concurrency();
  return n > 0 ? n : 1;
}

// Dynamic-schedule parallel for over [0, n): fn(i, worker_id).  Each index is
// one ownership unit (a target branch, a leaf, a parent), as in the reference's
// threaded passes.
template <class F>
static void parallel_for(int64_t n, int64_t chunk, F&& fn) {
  int nw = n_workers();
  if (nw <= 1 || n <= chunk) {
    for (int64_t i = 0; i < n; ++i) fn(i, 0);
    return;
  }
  std::atomic<int64_t> next(0);
  auto body = [&](int wid) {
    for (;;) {
      int64_t s = next.fetch_add(chunk);
      if (s >= n) break;
      int64_t e = std::min(n, s + chunk);
      for (int64_t i = s; i < e; ++i) fn(i, wid);
    }
  };
  std::vector<std::thread> th;
  for (int w = 1; w < nw; ++w) th.emplace_back(body, w);
  body(0);
  for (auto& t : th) t.join();
}

static const double ONE_OVER_4PI = 1.0 / (4.0 * 3.141592653589793);

struct Branch {
  int64_t body_start = 0, body_count = 0, n_branches = 0, child_start = 0, parent = -1, i_leaf = -1;
  double source_center[3], target_center[3];
  double source_radius = 0, target_radius = 0;
  double source_box[3], target_box[3];
  double max_influence = 0;
};

struct Tree {
  std::vector<Branch> branches;
  std::vector<int64_t> levels_start, levels_end, leaf_index;
  std::vector<int64_t> sort_index, inverse_sort_index;
  std::vector<double> buf;  // sorted buffer: 16 rows (target) or d rows (source)
  int rows = 16;
  int64_t n = 0;
  std::vector<double> expansions;
};

// exceeds(..., ::SelfTuning / ::SelfTuningTreeStop / ::Barba), src/tree.jl:492-569
static bool exceeds(int64_t n, int64_t ls, int method) {
  if (method == ORACLE_LIST_BARBA) return n > ls;
  double fraction = 0.0;
  fraction += (double)n / (double)(ls * ls);
  fraction *= (double)ls;
  if (method == ORACLE_LIST_SELF_TUNING) return fraction > 0.5 && n > 1;
  return fraction > 2.8284271247461903 && n > 1;
}

// get_octant, src/tree.jl:474-480 (0-based octant)
static inline int get_octant(const double* x, const double* c) {
  int o = 0;
  if (x[0] > c[0]) o += 1;
  if (x[1] > c[1]) o += 2;
  if (x[2] > c[2]) o += 4;
  return o;
}

// get_child_center, src/tree.jl:581-592
static void get_child_center(const double* pc, const double* pbox, int o, double* cc) {
  double delta = pbox[0] * 0.5;
  double dx = (o % 2 == 0) ? -delta : delta;
  delta = pbox[1] * 0.5;
  o >>= 1;
  double dy = (o % 2 == 0) ? -delta : delta;
  delta = pbox[2] * 0.5;
  o >>= 1;
  double dz = (o % 2 == 0) ? -delta : delta;
  cc[0] = pc[0] + dx;
  cc[1] = pc[1] + dy;
  cc[2] = pc[2] + dz;
}

// get_center_box, src/tree.jl:899-904
static void center_from_minmax(double xmn, double xmx, double ymn, double ymx, double zmn, double zmx,
                               double* c, double* box) {
  c[0] = (xmx + xmn) * 0.5;
  c[1] = (ymx + ymn) * 0.5;
  c[2] = (zmx + zmn) * 0.5;
  box[0] = xmx - c[0];
  box[1] = ymx - c[1];
  box[2] = zmx - c[2];
}

struct Builder {
  Tree& T;
  std::vector<double> pos;  // sorted positions (3 per body)
  std::vector<double> small;
  std::vector<int64_t> sort_buf;
  int64_t ls;
  int method;
  int64_t i_leaf = 0;

  // branch!, src/tree.jl:433-463: census, split decision, stable octant sort
  Branch branch(int64_t start, int64_t count, const double* c, double radius, const double* box,
                int64_t parent, int64_t i_first_branch, int64_t& n_children) {
    int64_t cnt[8] = {0};
    for (int64_t i = start; i < start + count; ++i) cnt[get_octant(&pos[3 * i], c)]++;
    n_children = 0;
    if (exceeds(count, ls, method))
      for (int o = 0; o < 8; ++o) n_children += cnt[o] > 0;
    if (n_children > 0) {  // sort_bodies!, src/tree.jl:712-737
      int64_t idx[8];
      int64_t acc = start;
      for (int o = 0; o < 8; ++o) {
        idx[o] = acc;
        acc += cnt[o];
      }
      for (int64_t i = start; i < start + count; ++i) {
        int o = get_octant(&pos[3 * i], c);
        int64_t j = idx[o]++;
        std::memcpy(&small[3 * j], &pos[3 * i], 3 * sizeof(double));
        sort_buf[j] = T.sort_index[i];
      }
      for (int64_t i = start; i < start + count; ++i) {
        std::memcpy(&pos[3 * i], &small[3 * i], 3 * sizeof(double));
        T.sort_index[i] = sort_buf[i];
      }
    }
    Branch b;
    b.body_start = start;
    b.body_count = count;
    b.n_branches = n_children;
    b.child_start = i_first_branch;
    b.parent = parent;
    b.i_leaf = (n_children == 0) ? i_leaf++ : -1;
    for (int k = 0; k < 3; ++k) {
      b.source_center[k] = b.target_center[k] = c[k];
      b.source_box[k] = b.target_box[k] = box[k];
    }
    b.source_radius = b.target_radius = radius;
    return b;
  }
};

static double get_radius(const Tree& T, int64_t i) { return T.buf[(int64_t)T.rows * i + 3]; }
static const double* get_pos(const Tree& T, int64_t i) { return &T.buf[(int64_t)T.rows * i]; }

// shrink_leaf! / shrink_branch! / shrink_recenter!, src/tree.jl:1141-1188
static void shrink_recenter(Tree& T) {
  for (int64_t lev = (int64_t)T.levels_start.size() - 1; lev >= 0; --lev) {
    for (int64_t ib = T.levels_start[lev]; ib < T.levels_end[lev]; ++ib) {
      Branch& b = T.branches[ib];
      double tc[3], tb[3], sc[3], sbx[3];
      if (b.n_branches == 0) {
        const double* x0 = get_pos(T, b.body_start);
        double xmn = x0[0], xmx = x0[0], ymn = x0[1], ymx = x0[1], zmn = x0[2], zmx = x0[2];
        for (int64_t i = b.body_start; i < b.body_start + b.body_count; ++i) {
          const double* x = get_pos(T, i);
          xmn = std::min(xmn, x[0]); xmx = std::max(xmx, x[0]);
          ymn = std::min(ymn, x[1]); ymx = std::max(ymx, x[1]);
          zmn = std::min(zmn, x[2]); zmx = std::max(zmx, x[2]);
        }
        center_from_minmax(xmn, xmx, ymn, ymx, zmn, zmx, tc, tb);
        xmn = x0[0]; xmx = x0[0]; ymn = x0[1]; ymx = x0[1]; zmn = x0[2]; zmx = x0[2];
        for (int64_t i = b.body_start; i < b.body_start + b.body_count; ++i) {
          const double* x = get_pos(T, i);
          double r = get_radius(T, i);
          xmn = std::min(xmn, x[0] - r); ymn = std::min(ymn, x[1] - r); zmn = std::min(zmn, x[2] - r);
          xmx = std::max(xmx, x[0] + r); ymx = std::max(ymx, x[1] + r); zmx = std::max(zmx, x[2] + r);
        }
        center_from_minmax(xmn, xmx, ymn, ymx, zmn, zmx, sc, sbx);
        double trad = 0, srad = 0;
        for (int64_t i = b.body_start; i < b.body_start + b.body_count; ++i) {
          const double* x = get_pos(T, i);
          double br = get_radius(T, i);
          double dx = x[0] - tc[0], dy = x[1] - tc[1], dz = x[2] - tc[2];
          trad = std::max(trad, std::sqrt(dx * dx + dy * dy + dz * dz));
          dx = x[0] - sc[0]; dy = x[1] - sc[1]; dz = x[2] - sc[2];
          srad = std::max(srad, std::sqrt(dx * dx + dy * dy + dz * dz) + br);
        }
        b.target_radius = trad;
        b.source_radius = srad;
      } else {
        const Branch& f = T.branches[b.child_start];
        double xmn = f.target_center[0], xmx = xmn, ymn = f.target_center[1], ymx = ymn,
               zmn = f.target_center[2], zmx = zmn;
        for (int64_t c = b.child_start; c < b.child_start + b.n_branches; ++c) {
          const Branch& ch = T.branches[c];
          xmn = std::min(xmn, ch.target_center[0] - ch.target_box[0]);
          xmx = std::max(xmx, ch.target_center[0] + ch.target_box[0]);
          ymn = std::min(ymn, ch.target_center[1] - ch.target_box[1]);
          ymx = std::max(ymx, ch.target_center[1] + ch.target_box[1]);
          zmn = std::min(zmn, ch.target_center[2] - ch.target_box[2]);
          zmx = std::max(zmx, ch.target_center[2] + ch.target_box[2]);
        }
        tc[0] = (xmn + xmx) * 0.5; tc[1] = (ymn + ymx) * 0.5; tc[2] = (zmn + zmx) * 0.5;
        tb[0] = xmx - tc[0]; tb[1] = ymx - tc[1]; tb[2] = zmx - tc[2];
        xmn = f.source_center[0]; xmx = xmn; ymn = f.source_center[1]; ymx = ymn;
        zmn = f.source_center[2]; zmx = zmn;
        for (int64_t c = b.child_start; c < b.child_start + b.n_branches; ++c) {
          const Branch& ch = T.branches[c];
          xmn = std::min(xmn, ch.source_center[0] - ch.source_box[0]);
          xmx = std::max(xmx, ch.source_center[0] + ch.source_box[0]);
          ymn = std::min(ymn, ch.source_center[1] - ch.source_box[1]);
          ymx = std::max(ymx, ch.source_center[1] + ch.source_box[1]);
          zmn = std::min(zmn, ch.source_center[2] - ch.source_box[2]);
          zmx = std::max(zmx, ch.source_center[2] + ch.source_box[2]);
        }
        sc[0] = (xmn + xmx) * 0.5; sc[1] = (ymn + ymx) * 0.5; sc[2] = (zmn + zmx) * 0.5;
        sbx[0] = xmx - sc[0]; sbx[1] = ymx - sc[1]; sbx[2] = zmx - sc[2];
        double trad = 0, srad = 0;
        for (int64_t c = b.child_start; c < b.child_start + b.n_branches; ++c) {
          const Branch& ch = T.branches[c];
          double dx = ch.target_center[0] - tc[0], dy = ch.target_center[1] - tc[1],
                 dz = ch.target_center[2] - tc[2];
          trad = std::max(trad, std::sqrt(dx * dx + dy * dy + dz * dz) + ch.target_radius);
          dx = ch.source_center[0] - sc[0]; dy = ch.source_center[1] - sc[1]; dz = ch.source_center[2] - sc[2];
          srad = std::max(srad, std::sqrt(dx * dx + dy * dy + dz * dz) + ch.source_radius);
        }
        b.target_radius = trad;
        b.source_radius = srad;
      }
      for (int k = 0; k < 3; ++k) {
        b.target_center[k] = tc[k];
        b.target_box[k] = tb[k];
        b.source_center[k] = sc[k];
        b.source_box[k] = sbx[k];
      }
    }
  }
}

// Tree(systems, target; leaf_size, shrink_recenter, interaction_list_method), src/tree.jl:3-122.
// data: body-major rows (stride doubles per body); positions in the first 3.
static bool build_tree(Tree& T, const double* data, int stride, int64_t n, bool target, int rows,
                       int64_t leaf_size, int method, bool shrink) {
  T = Tree();
  T.n = n;
  T.rows = rows;
  if (n == 0) return true;  // EmptyTree
  Builder B{T, {}, {}, {}, 0, 0};
  B.ls = leaf_size;
  B.method = method;
  B.pos.resize(3 * n);
  B.small.resize(3 * n);
  B.sort_buf.resize(n);
  T.sort_index.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    T.sort_index[i] = i;
    for (int k = 0; k < 3; ++k) B.pos[3 * i + k] = data[stride * i + k];
  }
  // center_box, src/tree.jl:917-924
  double xmn = B.pos[0], xmx = xmn, ymn = B.pos[1], ymx = ymn, zmn = B.pos[2], zmx = zmn;
  for (int64_t i = 0; i < n; ++i) {
    xmn = std::min(xmn, B.pos[3 * i]); xmx = std::max(xmx, B.pos[3 * i]);
    ymn = std::min(ymn, B.pos[3 * i + 1]); ymx = std::max(ymx, B.pos[3 * i + 1]);
    zmn = std::min(zmn, B.pos[3 * i + 2]); zmx = std::max(zmx, B.pos[3 * i + 2]);
  }
  double c[3], box[3];
  center_from_minmax(xmn, xmx, ymn, ymx, zmn, zmx, c, box);
  double bmax = std::max(std::max(box[0], box[1]), box[2]);
  double radius = std::sqrt(bmax * bmax * 3.0);
  double cube[3] = {bmax, bmax, bmax};
  int64_t n_children = 0;
  T.branches.push_back(B.branch(0, n, c, radius, cube, -1, 1, n_children));
  T.levels_start.push_back(0);
  T.levels_end.push_back(1);
  int64_t ps = 0, pe = 1;
  const int max_levels = 64;  // the reference's while loop is unbounded; degenerate (coincident) bodies stop here
  while (n_children > 0) {
    if ((int)T.levels_start.size() >= max_levels) return false;
    int64_t i_first = pe + n_children;  // child_branches!, src/tree.jl:346-376
    for (int64_t ip = ps; ip < pe; ++ip) {
      Branch P = T.branches[ip];
      if (P.n_branches == 0) continue;
      double crad = P.target_radius * 0.5;
      double cbox[3] = {P.target_box[0] * 0.5, P.target_box[1] * 0.5, P.target_box[2] * 0.5};
      int64_t cnt[8] = {0};
      for (int64_t i = P.body_start; i < P.body_start + P.body_count; ++i)
        cnt[get_octant(&B.pos[3 * i], P.target_center)]++;
      if (!exceeds(P.body_count, leaf_size, method)) continue;
      int64_t acc = P.body_start;
      for (int o = 0; o < 8; ++o) {
        if (cnt[o] > 0) {
          double cc[3];
          get_child_center(P.target_center, P.target_box, o, cc);
          int64_t ng = 0;
          Branch ch = B.branch(acc, cnt[o], cc, crad, cbox, ip, i_first, ng);
          i_first += ng;
          T.branches.push_back(ch);
        }
        acc += cnt[o];
      }
    }
    n_children = i_first - (int64_t)T.branches.size();
    ps = pe;
    pe = (int64_t)T.branches.size();
    T.levels_start.push_back(ps);
    T.levels_end.push_back(pe);
  }
  // fill buffers in sorted order (target_to_buffer! / system_to_buffer!, src/tree.jl:81-84)
  T.buf.assign((int64_t)rows * n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    const double* src = data + stride * T.sort_index[i];
    if (target) {
      for (int k = 0; k < 3; ++k) T.buf[(int64_t)rows * i + k] = src[k];
    } else {
      for (int k = 0; k < rows; ++k) T.buf[(int64_t)rows * i + k] = src[k];
    }
  }
  T.inverse_sort_index.resize(n);  // invert_index!, src/tree.jl:748-752
  for (int64_t i = 0; i < n; ++i) T.inverse_sort_index[T.sort_index[i]] = i;
  if (shrink) shrink_recenter(T);
  for (int64_t ib = 0; ib < (int64_t)T.branches.size(); ++ib)
    if (T.branches[ib].n_branches == 0) T.leaf_index.push_back(ib);
  return true;
}

// ---------------------------------------------------------------------------
// build_interaction_lists!, src/interaction_list.jl:23-166
struct ListBuilder {
  const std::vector<Branch>& tb;
  const std::vector<Branch>& sb;
  int64_t ls;
  double mac;
  bool ff, nf, si;
  int method;
  std::vector<int32_t> m2l, direct;  // pairs (target, source), 0-based

  bool mac_ok(const Branch& t, const Branch& s) const {
    double dx = t.target_center[0] - s.source_center[0];
    double dy = t.target_center[1] - s.source_center[1];
    double dz = t.target_center[2] - s.source_center[2];
    double sep2 = dx * dx + dy * dy + dz * dz;
    double summed = s.source_radius + t.target_radius;
    return sep2 * mac * mac > summed * summed;
  }
  void push(std::vector<int32_t>& v, int64_t it, int64_t js) {
    v.push_back((int32_t)it);
    v.push_back((int32_t)js);
  }
  void recurse(int64_t it, int64_t js) {
    const Branch& s = sb[js];
    const Branch& t = tb[it];
    bool both_leaves = s.n_branches == 0 && t.n_branches == 0;
    if (method == ORACLE_LIST_SELF_TUNING_TREE_STOP) {
      if (both_leaves) {
        if ((nf || (it == js && si)) && (it != js || si)) push(direct, it, js);
        return;
      }
      if (mac_ok(t, s)) {
        if (ff) push(m2l, it, js);
        return;
      }
      if (s.n_branches == 0 || (t.body_count >= s.body_count && t.n_branches != 0)) {
        for (int64_t c = t.child_start; c < t.child_start + t.n_branches; ++c) recurse(c, js);
      } else {
        for (int64_t c = s.child_start; c < s.child_start + s.n_branches; ++c) recurse(it, c);
      }
    } else if (method == ORACLE_LIST_BARBA) {
      if (mac_ok(t, s)) {
        if (ff) push(m2l, it, js);
        return;
      }
      if (both_leaves) {
        if ((nf || (it == js && si)) && (it != js || si)) push(direct, it, js);
        return;
      }
      if (s.n_branches == 0 || (t.target_radius >= s.source_radius && t.n_branches != 0)) {
        for (int64_t c = t.child_start; c < t.child_start + t.n_branches; ++c) recurse(c, js);
      } else {
        for (int64_t c = s.child_start; c < s.child_start + s.n_branches; ++c) recurse(it, c);
      }
    } else {  // SelfTuning
      double fraction = 0.0;
      fraction += (double)s.body_count / (double)(ls * ls);
      fraction *= (double)t.body_count;
      if (fraction < 1.0 || both_leaves) {
        if (nf && (it != js || si)) push(direct, it, js);
        return;
      }
      if (mac_ok(t, s)) {
        if (ff) push(m2l, it, js);
        return;
      }
      if (s.n_branches == 0 || (t.body_count >= s.body_count && t.n_branches != 0)) {
        for (int64_t c = t.child_start; c < t.child_start + t.n_branches; ++c) recurse(c, js);
      } else {
        for (int64_t c = s.child_start; c < s.child_start + s.n_branches; ++c) recurse(it, c);
      }
    }
  }
};

// sort_by_target, src/interaction_list.jl:183-213 (stable counting sort)
static void sort_by_target(std::vector<int32_t>& list, int64_t n_targets) {
  int64_t L = (int64_t)list.size() / 2;
  std::vector<int64_t> cnt(n_targets + 1, 0);
  for (int64_t k = 0; k < L; ++k) cnt[list[2 * k] + 1]++;
  for (int64_t i = 0; i < n_targets; ++i) cnt[i + 1] += cnt[i];
  std::vector<int32_t> out(list.size());
  for (int64_t k = 0; k < L; ++k) {
    int64_t d = cnt[list[2 * k]]++;
    out[2 * d] = list[2 * k];
    out[2 * d + 1] = list[2 * k + 1];
  }
  list.swap(out);
}

// ---------------------------------------------------------------------------
// direct! of the reference's test systems
// Laplace point source: test/gravitational.jl:80-104 (phi and gradient, no hessian)
static inline void p2p_source(const double* t, double* acc, const double* s) {
  double dx = t[0] - s[0], dy = t[1] - s[1], dz = t[2] - s[2];
  double r2 = dx * dx + dy * dy + dz * dz;
  if (r2 > 0) {
    double q = s[4];
    double r = std::sqrt(r2);
    acc[0] += q / r * ONE_OVER_4PI;
    double den = r2 * r;
    acc[1] += dx * q / den * ONE_OVER_4PI;
    acc[2] += dy * q / den * ONE_OVER_4PI;
    acc[3] += dz * q / den * ONE_OVER_4PI;
  }
}

// vortex particle: test/vortex.jl:83-128 (velocity and velocity gradient)
static inline void p2p_vortex(const double* t, double* acc, const double* s, bool gs, bool hs) {
  double dx = t[0] - s[0], dy = t[1] - s[1], dz = t[2] - s[2];
  double r2 = dx * dx + dy * dy + dz * dz;
  if (r2 > 0) {
    double gx = s[4], gy = s[5], gz = s[6];
    double r = std::sqrt(r2), rinv = 1 / r, rinv2 = rinv * rinv;
    double denom = ONE_OVER_4PI * rinv * rinv2;
    if (gs) {
      acc[1] += (dz * gy - dy * gz) * denom;
      acc[2] += (dx * gz - dz * gx) * denom;
      acc[3] += (dy * gx - dx * gy) * denom;
    }
    if (hs) {
      denom *= rinv2;
      acc[4] += -3 * dx * (gy * dz - gz * dy) * denom;
      acc[5] += (-3 * dx * (gz * dx - gx * dz) + gz * r2) * denom;
      acc[6] += (-3 * dx * (gx * dy - gy * dx) - gy * r2) * denom;
      acc[7] += (-3 * dy * (gy * dz - gz * dy) - gz * r2) * denom;
      acc[8] += -3 * dy * (gz * dx - gx * dz) * denom;
      acc[9] += (-3 * dy * (gx * dy - gy * dx) + gx * r2) * denom;
      acc[10] += (-3 * dz * (gy * dz - gz * dy) + gy * r2) * denom;
      acc[11] += (-3 * dz * (gz * dx - gx * dz) - gx * r2) * denom;
      acc[12] += -3 * dz * (gx * dy - gy * dx) * denom;
    }
  }
}

static inline void p2p(int kind, const double* tpos, double* acc13, const double* s, bool gs, bool hs) {
  if (kind == ORACLE_POINT_VORTEX)
    p2p_vortex(tpos, acc13, s, gs, hs);
  else
    p2p_source(tpos, acc13, s);
}

}  // namespace orc

using namespace orc;

struct oracle_run {
  Tree target, source;
  bool same = false;
  std::vector<int32_t> m2l, direct;
  std::vector<double> out16;  // original order
  int pmax = 0, success = 1;
  double times[6] = {0, 0, 0, 0, 0, 0};
};

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void fill_view(const Tree& T, oracle_tree_view* v, std::vector<int64_t>& i64, std::vector<double>& f64) {
  int64_t nb = (int64_t)T.branches.size();
  i64.assign(6 * nb, 0);
  f64.assign(17 * nb, 0);
  for (int64_t b = 0; b < nb; ++b) {
    const Branch& B = T.branches[b];
    i64[b] = B.body_start;
    i64[nb + b] = B.body_count;
    i64[2 * nb + b] = B.child_start;
    i64[3 * nb + b] = B.n_branches;
    i64[4 * nb + b] = B.parent;
    i64[5 * nb + b] = B.i_leaf;
    for (int k = 0; k < 3; ++k) {
      f64[3 * b + k] = B.target_center[k];
      f64[3 * nb + 3 * b + k] = B.source_center[k];
      f64[8 * nb + 3 * b + k] = B.target_box[k];
      f64[11 * nb + 3 * b + k] = B.source_box[k];
    }
    f64[6 * nb + b] = B.target_radius;
    f64[7 * nb + b] = B.source_radius;
    f64[14 * nb + b] = B.max_influence;
  }
  v->n_branches = nb;
  v->n_levels = (int64_t)T.levels_start.size();
  v->n_leaves = (int64_t)T.leaf_index.size();
  v->n_bodies = T.n;
  v->body_start = i64.data();
  v->body_count = i64.data() + nb;
  v->child_start = i64.data() + 2 * nb;
  v->n_children = i64.data() + 3 * nb;
  v->parent = i64.data() + 4 * nb;
  v->i_leaf = i64.data() + 5 * nb;
  v->target_center = f64.data();
  v->source_center = f64.data() + 3 * nb;
  v->target_radius = f64.data() + 6 * nb;
  v->source_radius = f64.data() + 7 * nb;
  v->target_box = f64.data() + 8 * nb;
  v->source_box = f64.data() + 11 * nb;
  v->max_influence = f64.data() + 14 * nb;
  v->sort_index = T.sort_index.data();
  v->levels_start = T.levels_start.data();
  v->levels_end = T.levels_end.data();
  v->leaf_index = T.leaf_index.data();
}

// views keep their backing storage alive with the run
struct view_store {
  std::vector<int64_t> i64;
  std::vector<double> f64;
};
static thread_local view_store g_vs_t, g_vs_s;

static oracle_run* fmm_impl(const double* target_pos, int64_t n_t, const double* source_buf, int d,
                            int kind, int64_t n_s, const oracle_options& o,
                            const std::vector<double>* influence_by_body);

// estimate_influence!, src/fmm.jl:1193-1276: a cheap p=3 FMM gives |grad| per target body
static void estimate_influence(oracle_run* run, const double* target_pos, int64_t n_t, const double* source_buf,
                               int d, int kind, int64_t n_s, const oracle_options& o) {
  oracle_options e = o;
  e.leaf_size_source = 5;
  e.leaf_size_target = 5;
  e.expansion_order = 3;
  e.multipole_acceptance = 0.6;
  e.error_method = ORACLE_ERR_NONE;
  e.shrink_recenter = 1;
  e.list_method = ORACLE_LIST_SELF_TUNING_TREE_STOP;
  e.farfield = e.nearfield = e.self_induced = 1;
  e.upward_pass = e.horizontal_pass = e.downward_pass = 1;
  e.scalar_potential = 1;
  e.gradient = 1;
  e.hessian = 0;
  oracle_run* est = fmm_impl(target_pos, n_t, source_buf, d, kind, n_s, e, nullptr);
  if (!est) return;
  // get_influence (src/fmm.jl:1180-1187): |gradient|, or the scalar potential itself for
  // PowerRelativePotential
  const bool potential = o.error_method == ORACLE_ERR_POWER_RELATIVE_POTENTIAL;
  Tree& T = run->target;
  for (auto& b : T.branches) {
    double mi = b.max_influence;
    for (int64_t i = b.body_start; i < b.body_start + b.body_count; ++i) {
      const double* g = &est->out16[16 * T.sort_index[i] + 3];
      mi = std::max(mi, potential ? g[0] : std::sqrt(g[1] * g[1] + g[2] * g[2] + g[3] * g[3]));
    }
    b.max_influence = mi;
  }
  delete est;
}

static oracle_run* fmm_impl(const double* target_pos, int64_t n_t, const double* source_buf, int d,
                            int kind, int64_t n_s, const oracle_options& o,
                            const std::vector<double>*) {
  if (!source_buf && n_s > 0) return nullptr;
  // a tuple of systems (Tree(systems::Tuple, ...), src/tree.jl:3-122): one octree over the
  // bodies of every system, concatenated in tuple order, each body with its kind in row 8.
  // The octree splits on the total count, as the reference's TreeStop/SelfTuning rules do for
  // systems of one leaf size; Barba splits on per-system counts and is not restated here.
  const bool per_body = kind == ORACLE_KIND_PER_BODY;
  if (kind != ORACLE_POINT_SOURCE && kind != ORACLE_POINT_VORTEX && !per_body) return nullptr;
  if (d < (per_body ? 8 : 4 + kind)) return nullptr;
  if (per_body && o.list_method == ORACLE_LIST_BARBA) return nullptr;
  if (o.expansion_order < 1 || o.expansion_order > 40) return nullptr;
  auto run = std::make_unique<oracle_run>();
  run->same = (target_pos == nullptr);
  const double* tp = run->same ? source_buf : target_pos;
  int tstride = run->same ? d : 3;
  if (run->same) n_t = n_s;
  int p = o.expansion_order;
  int64_t ls_s = o.leaf_size_source, ls_t = o.leaf_size_target > 0 ? o.leaf_size_target : ls_s;
  // lamb_helmholtz = has_vector_potential(source_systems) (src/fmm.jl:927): any vortex system
  bool lh = (kind == ORACLE_POINT_VORTEX);
  if (per_body)
    for (int64_t j = 0; j < n_s && !lh; ++j) lh = source_buf[(int64_t)d * j + 7] == ORACLE_POINT_VORTEX;
  bool ps = o.scalar_potential, gs = o.gradient, hs = o.hessian;
  g_threads = o.n_threads;
  tables(p);  // grow the constant tables before the threaded passes

  double t0 = now_s();
  if (!build_tree(run->target, tp, tstride, n_t, true, 16, ls_t, o.list_method, o.shrink_recenter)) return nullptr;
  if (!build_tree(run->source, source_buf, d, n_s, false, d, ls_s, o.list_method, o.shrink_recenter)) return nullptr;
  double t1 = now_s();
  {
    ListBuilder L{run->target.branches, run->source.branches, ls_s, o.multipole_acceptance,
                  o.farfield != 0, o.nearfield != 0, o.self_induced != 0, o.list_method, {}, {}};
    if (!run->target.branches.empty() && !run->source.branches.empty()) L.recurse(0, 0);
    sort_by_target(L.m2l, (int64_t)run->target.branches.size());
    sort_by_target(L.direct, (int64_t)run->target.branches.size());
    run->m2l.swap(L.m2l);
    run->direct.swap(L.direct);
  }
  double t2 = now_s();
  run->times[0] = t1 - t0;
  run->times[1] = t2 - t1;
  if (o.error_method == ORACLE_ERR_POWER_RELATIVE_GRADIENT ||
      o.error_method == ORACLE_ERR_ROTATED_COEFFICIENTS_RELATIVE_GRADIENT ||
      o.error_method == ORACLE_ERR_POWER_RELATIVE_POTENTIAL)
    estimate_influence(run.get(), target_pos, n_t, source_buf, d, kind, n_s, o);

  Tree& TT = run->target;
  Tree& ST = run->source;
  run->out16.assign(16 * (size_t)n_t, 0.0);
  if (n_t > 0 && n_s > 0) {
    int64_t NH = nh(p);
    TT.expansions.assign(4 * NH * TT.branches.size(), 0.0);
    ST.expansions.assign(4 * NH * ST.branches.size(), 0.0);
    // ---- nearfield (src/fmm.jl:3-40, 112-181): one target branch per task
    double tn0 = now_s();
    auto groups = [](const std::vector<int32_t>& list) {
      std::vector<int64_t> g;
      int64_t L = (int64_t)list.size() / 2;
      for (int64_t k = 0; k < L; ++k)
        if (k == 0 || list[2 * k] != list[2 * k - 2]) g.push_back(k);
      g.push_back(L);
      return g;
    };
    if (o.nearfield || o.self_induced) {
      std::vector<int64_t> g = groups(run->direct);
      parallel_for((int64_t)g.size() - 1, 1, [&](int64_t gi, int) {
        for (int64_t k = g[gi]; k < g[gi + 1]; ++k) {
          const Branch& tb = TT.branches[run->direct[2 * k]];
          const Branch& sb = ST.branches[run->direct[2 * k + 1]];
          for (int64_t j = sb.body_start; j < sb.body_start + sb.body_count; ++j) {
            const double* s = &ST.buf[(int64_t)d * j];
            for (int64_t i = tb.body_start; i < tb.body_start + tb.body_count; ++i)
              p2p(per_body ? (int)s[7] : kind, &TT.buf[16 * i], &TT.buf[16 * i + 3], s, gs, hs);
          }
        }
      });
    }
    double tn1 = now_s();
    std::vector<Work> works(n_workers());
    for (auto& w : works) w.resize(p);
    // ---- upward pass (src/fmm.jl:252-447)
    if (o.upward_pass) {
      parallel_for((int64_t)ST.leaf_index.size(), 4, [&](int64_t li, int wid) {
        Work& w = works[wid];
        const Branch& b = ST.branches[ST.leaf_index[li]];
        double* M = &ST.expansions[4 * NH * ST.leaf_index[li]];
        for (int64_t j = b.body_start; j < b.body_start + b.body_count; ++j) {
          const double* s = &ST.buf[(int64_t)d * j];
          double dx = s[0] - b.source_center[0], dy = s[1] - b.source_center[1], dz = s[2] - b.source_center[2];
          // body_to_multipole! of the body's own system (src/bodytomultipole.jl:387-489)
          if ((per_body ? (int)s[7] : kind) == ORACLE_POINT_VORTEX)
            p2m_point_vortex(M, w.harm.data(), dx, dy, dz, s[4], s[5], s[6], p);
          else
            p2m_point_source(M, w.harm.data(), dx, dy, dz, s[4], p);
        }
      });
      for (int64_t lev = (int64_t)ST.levels_start.size() - 2; lev >= 0; --lev) {
        int64_t l0 = ST.levels_start[lev];
        parallel_for(ST.levels_end[lev] - l0, 4, [&](int64_t k, int wid) {
          int64_t ib = l0 + k;
          const Branch& b = ST.branches[ib];
          for (int64_t c = b.child_start; c < b.child_start + b.n_branches; ++c)
            m2m(&ST.expansions[4 * NH * ib], b.source_center, &ST.expansions[4 * NH * c],
                ST.branches[c].source_center, p, lh, works[wid]);
        });
      }
    }
    double tn2 = now_s();
    // ---- horizontal pass (src/fmm.jl:455-598)
    int pmax = 0;
    int success = 1;
    if (o.horizontal_pass && !run->m2l.empty()) {
      std::vector<int64_t> g = groups(run->m2l);
      std::vector<int> wp(works.size(), 0), ws(works.size(), 1);
      parallel_for((int64_t)g.size() - 1, 1, [&](int64_t gi, int wid) {
        for (int64_t k = g[gi]; k < g[gi + 1]; ++k) {
          int64_t it = run->m2l[2 * k], js = run->m2l[2 * k + 1];
          const Branch& tb = TT.branches[it];
          const Branch& sb = ST.branches[js];
          M2LTarget tg{tb.target_center, tb.target_box, tb.target_radius, tb.max_influence};
          bool ok = true;
          int P = m2l(&TT.expansions[4 * NH * it], tg, &ST.expansions[4 * NH * js], sb.source_center, p, lh,
                      o.error_method, o.error_tolerance, o.bonus_expansion, ok, works[wid]);
          wp[wid] = std::max(wp[wid], P);
          ws[wid] = ws[wid] && ok;
        }
      });
      for (size_t k = 0; k < works.size(); ++k) {
        pmax = std::max(pmax, wp[k]);
        success = success && ws[k];
      }
    }
    if (!success) pmax += 1;
    run->pmax = pmax;
    run->success = success;
    double tn3 = now_s();
    // ---- downward pass (src/fmm.jl:602-757)
    if (o.downward_pass) {
      for (int64_t lev = 0; lev < (int64_t)TT.levels_start.size(); ++lev) {
        int64_t l0 = TT.levels_start[lev];
        parallel_for(TT.levels_end[lev] - l0, 4, [&](int64_t k, int wid) {
          int64_t ib = l0 + k;
          const Branch& b = TT.branches[ib];
          for (int64_t c = b.child_start; c < b.child_start + b.n_branches; ++c)
            l2l(&TT.expansions[4 * NH * c], TT.branches[c].target_center, &TT.expansions[4 * NH * ib],
                b.target_center, p, lh, works[wid]);
        });
      }
      parallel_for((int64_t)TT.leaf_index.size(), 4, [&](int64_t li, int wid) {
        const Branch& b = TT.branches[TT.leaf_index[li]];
        const double* L = &TT.expansions[4 * NH * TT.leaf_index[li]];
        for (int64_t i = b.body_start; i < b.body_start + b.body_count; ++i) {
          double* x = &TT.buf[16 * i];
          double dx[3] = {x[0] - b.target_center[0], x[1] - b.target_center[1], x[2] - b.target_center[2]};
          double phi, g[3], H[9];
          evaluate_local(dx, L, p, lh, ps, gs, hs, phi, g, H, works[wid]);
          if (ps) x[3] += phi;
          if (gs) {
            x[4] += g[0];
            x[5] += g[1];
            x[6] += g[2];
          }
          if (hs)
            for (int c = 0; c < 9; ++c) x[7 + c] += H[c];
        }
      });
    }
    double tn4 = now_s();
    run->times[2] = tn1 - tn0;
    run->times[3] = tn2 - tn1;
    run->times[4] = tn3 - tn2;
    run->times[5] = tn4 - tn3;
    // buffer_to_target!, src/compatibility.jl:324-338 (unsort)
    for (int64_t i = 0; i < n_t; ++i)
      std::memcpy(&run->out16[16 * TT.sort_index[i]], &TT.buf[16 * i], 16 * sizeof(double));
  } else {
    for (int64_t i = 0; i < n_t; ++i)
      for (int k = 0; k < 3; ++k) run->out16[16 * i + k] = tp[tstride * i + k];
  }
  return run.release();
}

extern "C" {

oracle_run* oracle_fmm_run(const double* target_pos, int64_t n_t, const double* source_buf, int d, int kind,
                           int64_t n_s, const oracle_options* opt) {
  if (!opt) return nullptr;
  return fmm_impl(target_pos, n_t, source_buf, d, kind, n_s, *opt, nullptr);
}

int oracle_run_output(const oracle_run* run, double* out16) {
  if (!run || !out16) return 1;
  std::memcpy(out16, run->out16.data(), run->out16.size() * sizeof(double));
  return 0;
}

int oracle_run_target_tree(const oracle_run* run, oracle_tree_view* v) {
  if (!run || !v) return 1;
  fill_view(run->target, v, g_vs_t.i64, g_vs_t.f64);
  return 0;
}

int oracle_run_source_tree(const oracle_run* run, oracle_tree_view* v) {
  if (!run || !v) return 1;
  fill_view(run->source, v, g_vs_s.i64, g_vs_s.f64);
  return 0;
}

int64_t oracle_run_n_m2l(const oracle_run* run) { return run ? (int64_t)run->m2l.size() / 2 : 0; }
int64_t oracle_run_n_direct(const oracle_run* run) { return run ? (int64_t)run->direct.size() / 2 : 0; }

int oracle_run_lists(const oracle_run* run, int32_t* m2l, int32_t* direct) {
  if (!run) return 1;
  if (m2l) std::memcpy(m2l, run->m2l.data(), run->m2l.size() * sizeof(int32_t));
  if (direct) std::memcpy(direct, run->direct.data(), run->direct.size() * sizeof(int32_t));
  return 0;
}

int oracle_run_pmax(const oracle_run* run, int* pmax, int* success) {
  if (!run) return 1;
  if (pmax) *pmax = run->pmax;
  if (success) *success = run->success;
  return 0;
}

int oracle_run_times(const oracle_run* run, double* t6) {
  if (!run || !t6) return 1;
  std::memcpy(t6, run->times, 6 * sizeof(double));
  return 0;
}

void oracle_run_free(oracle_run* run) { delete run; }

int oracle_direct(const double* target_pos, int64_t n_t, const double* source_buf, int d, int kind, int64_t n_s,
                  int ps, int gs, int hs, int n_threads, double* out16) {
  (void)ps;
  if (!source_buf || !out16) return 1;
  const double* tp = target_pos ? target_pos : source_buf;
  int ts = target_pos ? 3 : d;
  if (!target_pos) n_t = n_s;
  g_threads = n_threads;
  parallel_for(n_t, 64, [&](int64_t i, int) {
    double* o = out16 + 16 * i;
    std::memset(o, 0, 16 * sizeof(double));
    for (int k = 0; k < 3; ++k) o[k] = tp[ts * i + k];
    for (int64_t j = 0; j < n_s; ++j) p2p(kind, o, o + 3, source_buf + (int64_t)d * j, gs != 0, hs != 0);
  });
  return 0;
}

int oracle_direct_subset(const double* target_pos, int64_t n_t, const int64_t* ids, int64_t n_ids,
                         const double* source_buf, int d, int kind, int64_t n_s, int n_threads, double* out16) {
  if (!source_buf || !out16 || !ids) return 1;
  const double* tp = target_pos ? target_pos : source_buf;
  int ts = target_pos ? 3 : d;
  if (!target_pos) n_t = n_s;
  g_threads = n_threads;
  parallel_for(n_ids, 16, [&](int64_t k, int) {
    int64_t i = ids[k];
    double* o = out16 + 16 * k;
    std::memset(o, 0, 16 * sizeof(double));
    if (i < 0 || i >= n_t) return;
    for (int c = 0; c < 3; ++c) o[c] = tp[ts * i + c];
    for (int64_t j = 0; j < n_s; ++j) p2p(kind, o, o + 3, source_buf + (int64_t)d * j, true, true);
  });
  return 0;
}

// ---- unit-level entry points ----
int oracle_tables(int p, double* Hs, double* zeta, double* eta, double* Mt, double* Lt) {
  const Tables& t = tables(p);
  if (Hs) std::memcpy(Hs, t.Hs.data(), length_Hs(p) * sizeof(double));
  if (zeta) std::memcpy(zeta, t.zeta.data(), length_Ts(p) * sizeof(double));
  if (eta) std::memcpy(eta, t.eta.data(), length_Ts(p) * sizeof(double));
  if (Mt) std::memcpy(Mt, t.Mt.data(), nh(p) * sizeof(double));
  if (Lt) std::memcpy(Lt, t.Lt.data(), nh(p) * sizeof(double));
  return 0;
}
int64_t oracle_length_Hs(int p) { return length_Hs(p); }
int64_t oracle_length_Ts(int p) { return length_Ts(p); }
int oracle_update_Ts(int p, double beta, double* Ts) {
  update_Ts(Ts, tables(p).Hs.data(), beta, p);
  return 0;
}
int oracle_compute_Pnms(int p, double s, double c, double* out) {
  compute_Pnms(p, s, c, out);
  return 0;
}
int oracle_regular_harmonics(double rho, double theta, double phi, int p, double* h) {
  regular_harmonics(h, rho, theta, phi, p);
  return 0;
}
int oracle_irregular_harmonics(double rho, double theta, double phi, int p, double* h) {
  irregular_harmonics(h, rho, theta, phi, p);
  return 0;
}
int oracle_translate_multipole_z(const double* src, double t, int p, int lh, double* out) {
  translate_multipole_z(out, src, t, p, lh != 0);
  return 0;
}
int oracle_translate_multipole_to_local_z(const double* src, double t, int p, int lh, double* out) {
  translate_multipole_to_local_z(out, src, t, p, lh != 0);
  return 0;
}
int oracle_translate_local_z(const double* src, double t, int p, int lh, double* out) {
  translate_local_z(out, src, t, p, lh != 0);
  return 0;
}
int oracle_lh_transform(double* e, double r, int p, int local) {
  if (local)
    lh_local(e, r, p);
  else
    lh_multipole(e, r, p);
  return 0;
}
int oracle_m2m(double* target, const double* tc, const double* src, const double* sc, int p, int lh) {
  Work w;
  w.resize(p);
  m2m(target, tc, src, sc, p, lh != 0, w);
  return 0;
}
int oracle_m2l(double* target, const double* tc, const double* tbox, double trad, double maxinf, const double* src,
               const double* sc, int p, int lh, int em, double eps, int be, int* p_used, int* success) {
  Work w;
  w.resize(p);
  M2LTarget tg{tc, tbox, trad, maxinf};
  bool ok = true;
  int P = m2l(target, tg, src, sc, p, lh != 0, em, eps, be, ok, w);
  if (p_used) *p_used = P;
  if (success) *success = ok;
  return 0;
}
int oracle_l2l(double* target, const double* tc, const double* src, const double* sc, int p, int lh) {
  Work w;
  w.resize(p);
  l2l(target, tc, src, sc, p, lh != 0, w);
  return 0;
}
int oracle_l2p(const double* dx, const double* local, int p, int lh, int ps, int gs, int hs, double* phi,
               double* grad3, double* hess9) {
  Work w;
  w.resize(p);
  evaluate_local(dx, local, p, lh != 0, ps != 0, gs != 0, hs != 0, *phi, grad3, hess9, w);
  return 0;
}
int oracle_p2m(int kind, const double* buf, int d, int64_t n, const double* center, int p, double* expansion) {
  Work w;
  w.resize(p);
  for (int64_t j = 0; j < n; ++j) {
    const double* s = buf + (int64_t)d * j;
    double dx = s[0] - center[0], dy = s[1] - center[1], dz = s[2] - center[2];
    if (kind == ORACLE_POINT_VORTEX)
      p2m_point_vortex(expansion, w.harm.data(), dx, dy, dz, s[4], s[5], s[6], p);
    else
      p2m_point_source(expansion, w.harm.data(), dx, dy, dz, s[4], p);
  }
  return 0;
}
int oracle_cartesian_to_spherical(double x, double y, double z, double* rtp) {
  cartesian_to_spherical(x, y, z, rtp[0], rtp[1], rtp[2]);
  return 0;
}

}  // extern "C"
