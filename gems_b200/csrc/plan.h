// plan.h -- execution order and on-chip plan of a traversal op list (host C++, no CUDA).
//
// Shared by the session layer (which plans every uploaded list) and the traversal kernels
// (which decode the plan word); a CPU test compiles it with g++ and checks the plans by
// simulation.
#pragma once

#include <algorithm>
#include <cstring>
#include <utility>
#include <vector>

#include "gems_b200.h"

#ifdef __CUDACC__
#define GEMS_HD __host__ __device__
#else
#define GEMS_HD
#endif

namespace gems {

// On-chip plan of a traversal op, in DevOp::pad_ of the uploaded list (the caller's pad_ is
// ignored).  The session reorders a hazard-free list so that each node's children run
// larger-subtree-first (Sethi-Ullman order: the live set of produced-but-unconsumed partials
// stays at a few entries), then assigns each partial produced and consumed within the list a
// place: forwarded in registers when its consumer is the next op, else a position of a small
// per-thread stack in shared memory, else (stack full) global memory only.  Every output is
// also stored to its slot.  Kernels without a stack ignore the plan.
//   bits 0-1 left source, 2-3 right source (kSrcGlobal: tip byte or slot in HBM; kSrcStack;
//   kSrcFwd), 4-5 output (kSrcGlobal: not kept; kSrcStack; kSrcFwd), 6 left kind, 7 right
//   kind (GEMS_CHILD_*), 8-15 left position, 16-23 right position, 24-31 output position.
enum : int { kSrcGlobal = 0, kSrcStack = 1, kSrcFwd = 2 };
constexpr int kPlanMaxPos = 16;  // stack positions a plan may use
GEMS_HD inline int plan_lsrc(int w) { return w & 3; }
GEMS_HD inline int plan_rsrc(int w) { return (w >> 2) & 3; }
GEMS_HD inline int plan_out(int w) { return (w >> 4) & 3; }
GEMS_HD inline int plan_lkind(int w) { return (w >> 6) & 1; }
GEMS_HD inline int plan_rkind(int w) { return (w >> 7) & 1; }
GEMS_HD inline int plan_lpos(int w) { return (w >> 8) & 255; }
GEMS_HD inline int plan_rpos(int w) { return (w >> 16) & 255; }
GEMS_HD inline int plan_opos(int w) { return (w >> 24) & 255; }

// Execution order and on-chip plan of an op list: writes the ops in execution order into dst
// with their plans in pad_ and returns the stack positions used (dst must not alias ops).
// Reordering keeps every op after the ops producing its children; it is skipped when a slot is
// written twice or read before being overwritten in the list, or a partial has two consumers
// (then the list runs in the caller's order, with the same kind of plan).
inline int plan_ops(const gems_op *ops, int nops, int nslots, gems_op *dst) {
  std::vector<int> last(nslots, -1), ncons(nops, 0), prod(2 * (size_t)nops, -1);
  std::vector<char> read_old(nslots, 0);
  bool keep_order = false;
  for (int j = 0; j < nops; j++) {
    const int kind[2] = {ops[j].left_kind, ops[j].right_kind};
    const int id[2] = {ops[j].left_id, ops[j].right_id};
    for (int sd = 0; sd < 2; sd++) {
      if (kind[sd] != GEMS_CHILD_PARTIAL) continue;
      const int i = last[id[sd]];
      if (i >= 0) {
        prod[2 * j + sd] = i;
        if (++ncons[i] > 1) keep_order = true;
      } else {
        read_old[id[sd]] = 1;
      }
    }
    const int d = ops[j].dst_slot;
    if (last[d] >= 0 || read_old[d]) keep_order = true;
    last[d] = j;
  }
  std::vector<int> order;
  order.reserve(nops);
  if (keep_order) {
    for (int j = 0; j < nops; j++) order.push_back(j);
  } else {
    // stack need of each op's subtree: the larger child first, the smaller's evaluation with
    // the larger's output waiting (the last child's output is forwarded, needing no position)
    std::vector<int> need(nops, 0);
    for (int j = 0; j < nops; j++) {
      const int a = prod[2 * j], b = prod[2 * j + 1];
      const int na = a >= 0 ? need[a] : -1, nb = b >= 0 ? need[b] : -1;
      if (a >= 0 && b >= 0)
        need[j] = std::max(std::max(na, nb), std::min(na, nb) + 1);
      else
        need[j] = std::max(0, std::max(na, nb));
    }
    std::vector<std::pair<int, int>> work;  // (op, children emitted?)
    for (int r = 0; r < nops; r++) {
      if (ncons[r]) continue;  // not a root of the list's forest
      work.push_back({r, 0});
      while (!work.empty()) {
        auto [j, done] = work.back();
        work.pop_back();
        if (done) {
          order.push_back(j);
          continue;
        }
        work.push_back({j, 1});
        int a = prod[2 * j], b = prod[2 * j + 1];
        if (a >= 0 && b >= 0 && need[b] > need[a]) std::swap(a, b);
        // pushed in reverse: a (the larger) is emitted first
        if (b >= 0) work.push_back({b, 0});
        if (a >= 0) work.push_back({a, 0});
      }
    }
  }
  // positions, in execution order
  std::vector<int> at(nops), pos(nops, -1), last_use(nops, -1);
  for (int t = 0; t < nops; t++) at[order[t]] = t;
  for (int j = 0; j < nops; j++)
    for (int sd = 0; sd < 2; sd++)
      if (prod[2 * j + sd] >= 0)
        last_use[prod[2 * j + sd]] = std::max(last_use[prod[2 * j + sd]], at[j]);
  std::vector<char> fwd(nops, 0);
  unsigned used = 0;  // bitmask of occupied positions
  int depth = 0;
  for (int t = 0; t < nops; t++) {
    const int j = order[t];
    const gems_op &o = ops[j];
    int w = (o.left_kind & 1) << 6 | (o.right_kind & 1) << 7;
    for (int sd = 0; sd < 2; sd++) {
      const int i = prod[2 * j + sd];
      int src = kSrcGlobal, p = 0;
      if (i >= 0 && fwd[i]) {
        src = kSrcFwd;
      } else if (i >= 0 && pos[i] >= 0) {
        src = kSrcStack;
        p = pos[i];
      }
      w |= src << (2 * sd) | p << (8 + 8 * sd);
    }
    for (int sd = 0; sd < 2; sd++) {  // positions whose last reader is this op are free again
      const int i = prod[2 * j + sd];
      if (i >= 0 && pos[i] >= 0 && last_use[i] == t) used &= ~(1u << pos[i]);
    }
    if (last_use[j] >= 0) {
      if (ncons[j] == 1 && last_use[j] == t + 1) {
        fwd[j] = 1;
        w |= kSrcFwd << 4;
      } else {
        int p = 0;
        while (p < kPlanMaxPos && (used >> p & 1u)) p++;
        if (p < kPlanMaxPos) {
          used |= 1u << p;
          pos[j] = p;
          depth = std::max(depth, p + 1);
          w |= kSrcStack << 4 | p << 24;
        }
      }
    }
    dst[t] = o;
    dst[t].pad_ = w;
  }
  return depth;
}

}  // namespace gems
