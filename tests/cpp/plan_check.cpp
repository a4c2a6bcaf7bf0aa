// plan_check.cpp -- CPU check of the traversal plans (gems_b200/csrc/plan.h), compiled with g++
// (test infrastructure).
//
// Random binary trees give postorder op lists like the tree mirror's (children in random
// adjacency order, some subtrees already computed so that their partials are read as they
// are, some lists with a slot written twice); each list is planned, then executed symbolically:
// every op produces a distinct value, global memory holds slot contents, the stack and the
// forwarding register hold what the plan says.  Every child an op reads through its plan must
// be the value the caller's order would have given it, and global memory must end the same.
// Prints "OK <lists> <max depth>" or the first failure.
#include <cstdio>
#include <random>
#include <vector>

#include "plan.h"

using gems::plan_ops;

namespace {

struct Tree {
  int ntaxa;
  std::vector<std::vector<int>> adj;
};

Tree random_tree(int ntaxa, std::mt19937 &rng) {
  Tree t;
  t.ntaxa = ntaxa;
  t.adj.assign(2 * ntaxa - 2, {});
  auto link = [&](int a, int b) {
    t.adj[a].push_back(b);
    t.adj[b].push_back(a);
  };
  int next = ntaxa;
  std::vector<std::pair<int, int>> edges;
  const int r = next++;
  for (int i = 0; i < 3; i++) edges.push_back({r, i});
  for (int leaf = 3; leaf < ntaxa; leaf++) {
    std::uniform_int_distribution<size_t> pick(0, edges.size() - 1);
    const size_t e = pick(rng);
    const int a = edges[e].first, b = edges[e].second, m = next++;
    edges[e] = {a, m};
    edges.push_back({m, b});
    edges.push_back({m, leaf});
  }
  for (auto &e : edges) link(e.first, e.second);
  for (auto &a : t.adj) std::shuffle(a.begin(), a.end(), rng);
  return t;
}

// postorder ops towards node `root_dad` -> `root`, one slot per internal node; nodes in `done`
// are taken as already computed (their slot is read as it is)
void collect(const Tree &t, int dad, int node, const std::vector<char> &done,
             std::vector<gems_op> &ops) {
  if (node < t.ntaxa || done[node]) return;
  int kids[2], nk = 0;
  for (int c : t.adj[node])
    if (c != dad) {
      collect(t, node, c, done, ops);
      kids[nk++] = c;
    }
  gems_op op{};
  op.dst_slot = node - t.ntaxa;
  auto child = [&](int c, int &kind, int &id) {
    kind = c < t.ntaxa ? GEMS_CHILD_TIP : GEMS_CHILD_PARTIAL;
    id = c < t.ntaxa ? c : c - t.ntaxa;
  };
  child(kids[0], op.left_kind, op.left_id);
  child(kids[1], op.right_kind, op.right_id);
  ops.push_back(op);
}

// symbolic execution: slot contents after running `ops` in order, reading children from
// global memory; returns the child values each op reads (by op index of the caller's list)
std::vector<long> run_plain(const std::vector<gems_op> &ops, int nslots,
                            std::vector<long> &mem) {
  std::vector<long> reads;
  for (size_t j = 0; j < ops.size(); j++) {
    const gems_op &o = ops[j];
    reads.push_back(o.left_kind == GEMS_CHILD_TIP ? -1 - o.left_id : mem[o.left_id]);
    reads.push_back(o.right_kind == GEMS_CHILD_TIP ? -1 - o.right_id : mem[o.right_id]);
    mem[o.dst_slot] = 1000000 + (long)j;
  }
  return reads;
}

bool check(const std::vector<gems_op> &ops, int nslots, int &depth, const char *what) {
  const int n = (int)ops.size();
  std::vector<long> mem0(nslots);
  for (int i = 0; i < nslots; i++) mem0[i] = 5000000 + i;  // old contents
  std::vector<long> mem_ref = mem0;
  const std::vector<long> reads = run_plain(ops, nslots, mem_ref);
  std::vector<gems_op> plan(n);
  depth = plan_ops(ops.data(), n, nslots, plan.data());
  if (depth > gems::kPlanMaxPos) {
    std::printf("FAIL %s: depth %d\n", what, depth);
    return false;
  }
  // op identity: the planned list is a permutation of the caller's list
  std::vector<int> orig(n, -1);
  std::vector<char> taken(n, 0);
  for (int t = 0; t < n; t++) {
    for (int j = 0; j < n; j++)
      if (!taken[j] && ops[j].dst_slot == plan[t].dst_slot && ops[j].left_id == plan[t].left_id &&
          ops[j].right_id == plan[t].right_id && ops[j].left_kind == plan[t].left_kind &&
          ops[j].right_kind == plan[t].right_kind) {
        orig[t] = j;
        taken[j] = 1;
        break;
      }
    if (orig[t] < 0) {
      std::printf("FAIL %s: op %d is not from the list\n", what, t);
      return false;
    }
  }
  std::vector<long> mem = mem0, stack(gems::kPlanMaxPos, -7);
  long fwd = -9;
  for (int t = 0; t < n; t++) {
    const gems_op &o = plan[t];
    const int w = o.pad_;
    const int src[2] = {gems::plan_lsrc(w), gems::plan_rsrc(w)};
    const int kind[2] = {gems::plan_lkind(w), gems::plan_rkind(w)};
    const int id[2] = {o.left_id, o.right_id};
    const int pos[2] = {gems::plan_lpos(w), gems::plan_rpos(w)};
    if (kind[0] != o.left_kind || kind[1] != o.right_kind) {
      std::printf("FAIL %s: kinds not encoded\n", what);
      return false;
    }
    for (int sd = 0; sd < 2; sd++) {
      long v;
      if (kind[sd] == GEMS_CHILD_TIP) {
        if (src[sd] != gems::kSrcGlobal) {
          std::printf("FAIL %s: tip from the stack\n", what);
          return false;
        }
        v = -1 - id[sd];
      } else if (src[sd] == gems::kSrcFwd) {
        v = fwd;
      } else if (src[sd] == gems::kSrcStack) {
        if (pos[sd] >= depth) {
          std::printf("FAIL %s: position %d >= depth %d\n", what, pos[sd], depth);
          return false;
        }
        v = stack[pos[sd]];
      } else {
        v = mem[id[sd]];
      }
      // values are named by the producing op's index in the caller's list
      if (v != reads[2 * orig[t] + sd]) {
        std::printf("FAIL %s: op %d side %d reads %ld, expected %ld\n", what, t, sd, v,
                    reads[2 * orig[t] + sd]);
        return false;
      }
    }
    const long out = 1000000 + orig[t];
    mem[o.dst_slot] = out;
    if (gems::plan_out(w) == gems::kSrcFwd) fwd = out;
    if (gems::plan_out(w) == gems::kSrcStack) {
      if (gems::plan_opos(w) >= depth) {
        std::printf("FAIL %s: output position beyond depth\n", what);
        return false;
      }
      stack[gems::plan_opos(w)] = out;
    }
  }
  if (mem != mem_ref) {
    std::printf("FAIL %s: final slot contents differ\n", what);
    return false;
  }
  return true;
}

}  // namespace

int main() {
  std::mt19937 rng(12345);
  int lists = 0, max_depth = 0, max_depth_full = 0;
  for (int rep = 0; rep < 300; rep++) {
    const int ntaxa = 3 + (int)(rng() % (rep < 100 ? 20 : 600));
    Tree t = random_tree(ntaxa, rng);
    const int nint = ntaxa - 2;
    // a branch (leaf 0 and its neighbour) and the whole traversal towards it
    std::vector<char> done(t.adj.size(), 0);
    std::vector<gems_op> ops;
    const int root = t.adj[0][0];
    collect(t, 0, root, done, ops);
    int depth = 0;
    if (!check(ops, nint, depth, "full")) return 1;
    max_depth_full = std::max(max_depth_full, depth);
    lists++;
    // part of the tree already computed
    for (size_t v = ntaxa; v < t.adj.size(); v++) done[v] = (rng() % 4 == 0);
    done[root] = 0;
    ops.clear();
    collect(t, 0, root, done, ops);
    if (!check(ops, nint, depth, "partial")) return 1;
    lists++;
    // a slot written twice (hazard: kept in the caller's order)
    if (ops.size() >= 2) {
      std::vector<gems_op> h = ops;
      h.push_back(h[0]);
      if (!check(h, nint, depth, "hazard")) return 1;
      lists++;
    }
    max_depth = std::max(max_depth, depth);
  }
  std::printf("OK lists=%d max_depth_full=%d max_depth=%d\n", lists, max_depth_full, max_depth);
  return 0;
}
