// phylotree.cpp -- host C++ mirror of the PhyloTree calls on the likelihood path, driving the
// kernel set of gems_b200.h.  The tree owns topology, branch lengths and cache flags; the
// device session owns every buffer.  Each method names the reference member it restates
// (paths relative to the IQ-TREE 3 source tree).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/gems_b200.h"

namespace {

struct Tree {
  gems_session *s = nullptr;
  int ntaxa = 0, nnode = 0, nedges = 0, nslots = 0;
  bool per_branch = false;  // one slot per directed branch (no re-orientation)
  // LM_MEM_SAVE (tree/memslot.cpp, tree/phylotree.cpp:1026-1040): fewer slots than internal
  // nodes; directed branches get a slot when their partial is computed, and a full pool gives
  // up the unlocked slot whose partial is cheapest to recompute (smallest subtree)
  bool pool = false;
  int pool_free = 0;               // slots not handed out yet (MemSlotVector::free_count)
  std::vector<char> slot_locked;   // per slot (MEM_LOCKED)
  std::vector<int> sub_size;       // per directed branch: leaves of the subtree it points to
  int pool_status = GEMS_OK;       // GEMS_ERR_ADMISSION when a traversal found no slot
  std::vector<int> deg, adj, eu, ev;
  std::vector<double> len;
  // directed branch d = u*3+k: u -> adj[u*3+k]; its partial is the subtree at adj[u*3+k]
  std::vector<char> computed;
  std::vector<int> dslot;      // per_branch and pool: slot of directed branch (-1: none)
  std::vector<int> node_slot;  // per node: slot of internal node (LM_PER_NODE)
  std::vector<int> owner;      // per slot: directed branch currently holding it, -1 if none
  int cur_u = -1, cur_k = 0;
  bool theta_computed = false;
  double min_bl = 1e-6, max_bl = 10.0;
  long long partial_ops = 0;
  int newton_evals = 0;
  std::vector<gems_op> ops;
  std::vector<char> *track = nullptr;  // when set: the slots every traversal writes

  int find(int u, int v) const {
    for (int k = 0; k < deg[u]; k++)
      if (adj[u * 3 + k] == v) return k;
    return -1;
  }
  bool leaf(int u) const { return deg[u] == 1; }
  int dir(int u, int v) const { return u * 3 + find(u, v); }

  // slot for directed branch d (u -> v, v internal).  In LM_PER_NODE mode the node's single
  // buffer moves to d, invalidating the branch that held it (reorientPartialLh + takeover,
  // tree/phylotree.cpp:6011, tree/memslot.cpp:213-229).
  int acquire(int d) {
    const int v = adj[d];
    int sl = per_branch ? dslot[d] : node_slot[v];
    if (owner[sl] != d) {
      if (owner[sl] >= 0) computed[owner[sl]] = 0;
      owner[sl] = d;
    }
    return sl;
  }
  int slot_of(int d) const { return per_branch || pool ? dslot[d] : node_slot[adj[d]]; }

  // PhyloNode::computeSize (tree/phylonode.cpp:91): leaves below every directed branch
  int size_below(int u, int k) {
    const int d = u * 3 + k, v = adj[d];
    if (sub_size[d] > 0) return sub_size[d];
    int n = 0;
    if (leaf(v)) {
      n = 1;
    } else {
      for (int j = 0; j < deg[v]; j++)
        if (adj[v * 3 + j] != u) n += size_below(v, j);
    }
    return sub_size[d] = n;
  }
  void compute_sizes() {
    sub_size.assign(nnode * 3, 0);
    for (int u = 0; u < nnode; u++)
      for (int k = 0; k < deg[u]; k++) size_below(u, k);
  }

  // MemSlotVector::lock / unlock (tree/memslot.cpp:92-121): a partial in use by the traversal
  // being built keeps its slot
  bool lock(int d) {
    if (!pool || leaf(adj[d]) || dslot[d] < 0 || slot_locked[dslot[d]]) return false;
    slot_locked[dslot[d]] = 1;
    return true;
  }
  void unlock(int d) {
    if (pool && dslot[d] >= 0) slot_locked[dslot[d]] = 0;
  }
  void give_slot(int d, int sl) {
    if (owner[sl] >= 0 && owner[sl] != d) {
      computed[owner[sl]] = 0;  // clearPartialLh of the branch that held it
      dslot[owner[sl]] = -1;
    }
    if (dslot[d] >= 0 && dslot[d] != sl) owner[dslot[d]] = -1;  // d's old slot is free again
    owner[sl] = d;
    dslot[d] = sl;
  }
  // MemSlotVector::allocate (tree/memslot.cpp:138-175): a free slot, else the unlocked slot of
  // the smallest subtree
  bool allocate(int d) {
    if (pool_free < nslots) {
      give_slot(d, pool_free++);
      return true;
    }
    for (int sl = 0; sl < nslots; sl++)
      if (!slot_locked[sl] && owner[sl] < 0) {
        give_slot(d, sl);
        return true;
      }
    int best = -1, best_size = 1 << 30;
    for (int sl = 0; sl < nslots; sl++) {
      if (slot_locked[sl] || owner[sl] < 0) continue;
      if (sub_size[owner[sl]] < best_size) {
        best = sl;
        best_size = sub_size[owner[sl]];
        if (best_size == 2) break;  // the smallest subtree an internal partial can have
      }
    }
    if (best < 0) return false;
    give_slot(d, best);
    return true;
  }

  // computeTraversalInfo with LM_MEM_SAVE (tree/phylotree.cpp:6031-6140): children in
  // descending subtree size, the partial re-oriented from a back-neighbour's slot when it has
  // none, else a slot allocated; children locked until their parent's op is listed.  Returns
  // whether the partial of (dad -> node) was locked.
  bool collect_pool(int dad, int node) {
    const int d = dir(dad, node);
    if (computed[d] || leaf(node)) return lock(d);
    int kids[2], nk = 0;
    for (int k = 0; k < deg[node]; k++)
      if (adj[node * 3 + k] != dad) kids[nk++] = adj[node * 3 + k];
    if (sub_size[dir(node, kids[0])] < sub_size[dir(node, kids[1])]) std::swap(kids[0], kids[1]);
    bool lk[2];
    for (int i = 0; i < 2; i++) lk[i] = collect_pool(node, kids[i]);
    computed[d] = 1;
    // reorientPartialLh (:6011): take over the slot of a back-neighbour (an unlocked one)
    if (dslot[d] < 0) {
      for (int i = 0; i < 2; i++) {
        const int back = dir(kids[i], node);
        if (dslot[back] >= 0 && !slot_locked[dslot[back]]) {
          give_slot(d, dslot[back]);
          break;
        }
      }
    }
    if ((dslot[d] < 0 || slot_locked[dslot[d]]) && !allocate(d)) pool_status = GEMS_ERR_ADMISSION;
    for (int i = 0; i < 2; i++)
      if (lk[i]) unlock(dir(node, kids[i]));
    gems_op op{};
    op.dst_slot = dslot[d] < 0 ? 0 : dslot[d];
    auto child = [&](int c, int &kind, int &id, double &l) {
      l = len[node * 3 + find(node, c)];
      kind = leaf(c) ? GEMS_CHILD_TIP : GEMS_CHILD_PARTIAL;
      id = leaf(c) ? c : dslot[dir(node, c)];
    };
    child(kids[0], op.left_kind, op.left_id, op.left_len);
    child(kids[1], op.right_kind, op.right_id, op.right_len);
    ops.push_back(op);
    partial_ops++;
    return lock(d);
  }

  // computeTraversalInfo (tree/phylotree.cpp:6031-6140): postorder list of stale partials
  void collect(int dad, int node) {
    const int d = dir(dad, node);
    if (computed[d] || leaf(node)) return;
    int kids[2], nk = 0;
    for (int k = 0; k < deg[node]; k++) {
      const int c = adj[node * 3 + k];
      if (c == dad) continue;
      collect(node, c);
      kids[nk++] = c;
    }
    computed[d] = 1;
    gems_op op{};
    op.dst_slot = acquire(d);
    auto child = [&](int c, int &kind, int &id, double &l) {
      l = len[node * 3 + find(node, c)];
      if (leaf(c)) {
        kind = GEMS_CHILD_TIP;
        id = c;
      } else {
        kind = GEMS_CHILD_PARTIAL;
        id = slot_of(dir(node, c));
      }
    };
    child(kids[0], op.left_kind, op.left_id, op.left_len);
    child(kids[1], op.right_kind, op.right_id, op.right_len);
    ops.push_back(op);
    partial_ops++;
  }

  // the branch (node, dad) after the reference's leaf swap (phylokernelnew.h:2671-2678)
  gems_branch branch(int &node, int &dad) {
    if (leaf(node)) std::swap(node, dad);
    ops.clear();
    if (pool) {
      // the larger side first (phylokernelnew.h:1176-1190); both ends stay locked until the
      // list is complete
      pool_status = GEMS_OK;
      int a = dad, b = node;
      if (sub_size[dir(dad, node)] < sub_size[dir(node, dad)]) std::swap(a, b);
      const bool la = collect_pool(a, b);
      const bool lb = collect_pool(b, a);
      if (la) unlock(dir(a, b));
      if (lb) unlock(dir(b, a));
    } else {
      collect(dad, node);
      if (!leaf(dad)) collect(node, dad);
    }
    if (track)
      for (const gems_op &o : ops) (*track)[o.dst_slot] = 1;
    gems_branch br{};
    br.dad_slot = slot_of(dir(dad, node));
    if (leaf(dad)) {
      br.node_kind = GEMS_CHILD_TIP;
      br.node_id = dad;
    } else {
      br.node_kind = GEMS_CHILD_PARTIAL;
      br.node_id = slot_of(dir(node, dad));
    }
    br.length = len[dad * 3 + find(dad, node)];
    return br;
  }

  void set_len(int u, int v, double x) {
    len[u * 3 + find(u, v)] = x;
    len[v * 3 + find(v, u)] = x;
  }

  // PhyloNode::clearReversePartialLh (tree/phylonode.cpp:22)
  void clear_reverse(int node, int dad) {
    for (int k = 0; k < deg[node]; k++) {
      const int c = adj[node * 3 + k];
      if (c == dad) continue;
      computed[dir(c, node)] = 0;
      clear_reverse(c, node);
    }
  }

  // MTree::findFarthestLeaf (tree/mtree.cpp:3040)
  int far_leaf(int node, int dad, std::vector<int> &h) const {
    if (dad >= 0 && leaf(node)) {
      h[node] = 0;
      return node;
    }
    int res = -1;
    h[node] = 0;
    for (int k = 0; k < deg[node]; k++) {
      const int c = adj[node * 3 + k];
      if (c == dad) continue;
      const int lf = far_leaf(c, node, h);
      if (h[node] < h[c] + 1) {
        h[node] = h[c] + 1;
        res = lf;
      }
    }
    return res;
  }

  // MTree::getPreOrderBranches (tree/mtree.cpp:3062)
  void preorder(int node, int dad, const std::vector<int> &h, std::vector<int> &n1,
                std::vector<int> &n2) const {
    if (dad >= 0) {
      n1.push_back(node);
      n2.push_back(dad);
    }
    int nv[3], nd = deg[node];
    for (int i = 0; i < nd; i++) nv[i] = adj[node * 3 + i];
    for (int i = 0; i < nd; i++)
      for (int j = i + 1; j < nd; j++)
        if (h[nv[i]] > h[nv[j]]) std::swap(nv[i], nv[j]);
    for (int i = 0; i < nd; i++)
      if (nv[i] != dad) preorder(nv[i], node, h, n1, n2);
  }

  int lh_branch(int node, int dad, double *lnl, double *pattern_lh) {
    gems_branch br = branch(node, dad);
    if (pool_status) return pool_status;
    return gems_branch_lnl(s, ops.data(), (int)ops.size(), &br, lnl, pattern_lh);
  }

  int derv(int node, int dad, double *df, double *ddf) {
    int st;
    if (!theta_computed) {
      gems_branch br = branch(node, dad);
      if (pool_status) return pool_status;
      st = gems_branch_derv(s, ops.data(), (int)ops.size(), &br, 1, df, ddf, nullptr);
      if (st == GEMS_OK) theta_computed = true;
    } else {
      if (leaf(node)) std::swap(node, dad);
      gems_branch br{};
      br.length = len[dad * 3 + find(dad, node)];
      br.dad_slot = slot_of(dir(dad, node));
      br.node_kind = leaf(dad) ? GEMS_CHILD_TIP : GEMS_CHILD_PARTIAL;
      br.node_id = leaf(dad) ? dad : slot_of(dir(node, dad));
      st = gems_branch_derv(s, nullptr, 0, &br, 0, df, ddf, nullptr);
    }
    return st;
  }

  int from_buffer(double *lnl) {
    if (cur_u < 0 || !theta_computed) {
      // computeLikelihoodFromBuffer falls back to computeLikelihoodBranch
      const int u = cur_u < 0 ? 0 : cur_u;
      const int v = adj[u * 3 + (cur_u < 0 ? 0 : cur_k)];
      return lh_branch(v, u, lnl, nullptr);
    }
    return gems_lnl_from_buffer(s, len[cur_u * 3 + cur_k], lnl, nullptr);
  }

  // PhyloTree::optimizeOneBranch (tree/phylotree.cpp:2620-2670) with the Newton loop of
  // Optimization::minimizeNewton (utils/optimization.cpp:422-499) run on the device, in two
  // halves: the traversal, theta and Newton loop enqueued on the session's stream, then the
  // result applied (the divergence check, the new length, clearReversePartialLh).
  double pending_len = 0;
  int optimize_begin(int node1, int node2, int max_nr) {
    const int k = find(node1, node2);
    if (k < 0) return GEMS_ERR_BAD_ARG;
    cur_u = node1;
    cur_k = k;
    pending_len = len[node1 * 3 + k];
    theta_computed = false;
    int n = node2, d = node1;
    gems_branch br = branch(n, d);
    if (pool_status) return pool_status;
    return gems_newton_branch_async(s, ops.data(), (int)ops.size(), &br, 1, min_bl, max_bl,
                                    min_bl, max_nr);
  }
  int optimize_finish(int node1, int node2, int clear_lh) {
    const double cur = pending_len;
    double optx = cur;
    int nev = 0;
    int st = gems_newton_branch_wait(s, &optx, &nev);
    newton_evals = nev;
    if (st != GEMS_OK) return st;
    theta_computed = true;
    if (optx > max_bl * 0.95) {
      double opt_lh = 0, orig_lh = 0;
      if ((st = gems_lnl_from_buffer(s, optx, &opt_lh, nullptr))) return st;
      if ((st = gems_lnl_from_buffer(s, cur, &orig_lh, nullptr))) return st;
      if (orig_lh > opt_lh) optx = cur;
    }
    set_len(node1, node2, optx);
    if (clear_lh && cur != optx) {
      clear_reverse(node1, node2);
      clear_reverse(node2, node1);
    }
    return GEMS_OK;
  }
  int optimize_one(int node1, int node2, int clear_lh, int max_nr) {
    if (int st = optimize_begin(node1, node2, max_nr)) return st;
    return optimize_finish(node1, node2, clear_lh);
  }

  // PhyloTree::optimizeAllBranches(my_iterations, tolerance, maxNRStep)
  // (tree/phylotree.cpp:2724-2800) with computeBestTraversal (:2710)
  int optimize_all(int iterations, double tol, int max_nr, double *out) {
    std::vector<int> h(nnode, 0), n1, n2;
    const int far = far_leaf(0, -1, h);
    far_leaf(far, -1, h);
    preorder(far, -1, h, n1, n2);
    double tree_lh = 0;
    int st = lh_branch(n2[0], n1[0], &tree_lh, nullptr);
    if (st) return st;
    std::vector<double> saved(nedges);
    for (int it = 0; it < iterations; it++) {
      for (int e = 0; e < nedges; e++) saved[e] = len[eu[e] * 3 + find(eu[e], ev[e])];
      for (size_t j = 0; j < n1.size(); j++)
        if ((st = optimize_one(n1[j], n2[j], 1, max_nr))) return st;
      double new_lh = 0;
      if ((st = from_buffer(&new_lh))) return st;
      if (new_lh < tree_lh - tol * 0.1) {
        std::fill(computed.begin(), computed.end(), 0);
        theta_computed = false;
        for (int e = 0; e < nedges; e++) set_len(eu[e], ev[e], saved[e]);
        if ((st = compute_likelihood(&new_lh, nullptr))) return st;
        *out = new_lh;
        return GEMS_OK;
      }
      if (tree_lh <= new_lh && new_lh <= tree_lh + tol) {
        tree_lh = new_lh;
        break;
      }
      tree_lh = new_lh;
    }
    *out = tree_lh;
    return GEMS_OK;
  }

  // the branch order of optimizeAllBranches (computeBestTraversal, tree/phylotree.cpp:2710)
  void best_traversal(std::vector<int> &n1, std::vector<int> &n2) const {
    std::vector<int> h(nnode, 0);
    const int far = far_leaf(0, -1, h);
    far_leaf(far, -1, h);
    preorder(far, -1, h, n1, n2);
  }

  // PhyloTree::doNNI (tree/phylotree.cpp:4059-4125): exchange subtree a (at u) with subtree b
  // (at v) across the internal branch (u, v).  The neighbour entries move with their lengths
  // and partials (the subtrees at a and b are unchanged); the central partials and every
  // partial looking back towards u or v are invalidated.
  int nni(int u, int v, int a, int b) {
    const int ku_a = find(u, a), kv_b = find(v, b), ka_u = find(a, u), kb_v = find(b, v);
    if (leaf(u) || leaf(v) || find(u, v) < 0 || ku_a < 0 || kv_b < 0 || a == v || b == u)
      return GEMS_ERR_BAD_ARG;
    const int du = u * 3 + ku_a, dv = v * 3 + kv_b;
    if (per_branch || pool) {
      std::swap(dslot[du], dslot[dv]);
      if (pool) {  // the slots follow their subtrees: their owners are re-pointed
        if (dslot[du] >= 0) owner[dslot[du]] = du;
        if (dslot[dv] >= 0) owner[dslot[dv]] = dv;
      }
    } else {
      // the buffers of a and b stay with their subtrees: re-point their owners
      const bool own_a = !leaf(a) && owner[node_slot[a]] == du;
      const bool own_b = !leaf(b) && owner[node_slot[b]] == dv;
      if (own_a) owner[node_slot[a]] = dv;
      if (own_b) owner[node_slot[b]] = du;
    }
    std::swap(adj[du], adj[dv]);
    std::swap(len[du], len[dv]);
    std::swap(computed[du], computed[dv]);
    adj[a * 3 + ka_u] = v;
    adj[b * 3 + kb_v] = u;
    computed[u * 3 + find(u, v)] = 0;
    computed[v * 3 + find(v, u)] = 0;
    clear_reverse(v, u);
    clear_reverse(u, v);
    // edge list: the edges (u, a) and (v, b) become (v, a) and (u, b)
    for (int e = 0; e < nedges; e++) {
      if ((eu[e] == u && ev[e] == a) || (eu[e] == a && ev[e] == u)) {
        eu[e] = v;
        ev[e] = a;
      } else if ((eu[e] == v && ev[e] == b) || (eu[e] == b && ev[e] == v)) {
        eu[e] = u;
        ev[e] = b;
      }
    }
    theta_computed = false;
    cur_u = -1;
    if (pool) compute_sizes();
    return GEMS_OK;
  }

  // the nodes of the subtree at v (away from u)
  void mark(int v, int u, std::vector<char> &m) const {
    m[v] = 1;
    for (int k = 0; k < deg[v]; k++)
      if (adj[v * 3 + k] != u) mark(adj[v * 3 + k], v, m);
  }
  // every partial whose subtree holds node x (the directed branches pointing at x)
  void clear_toward(int x) {
    for (int k = 0; k < deg[x]; k++) {
      const int c = adj[x * 3 + k];
      computed[dir(c, x)] = 0;
      clear_reverse(c, x);
    }
  }

  // SPR with the geometry of assessSPRMove (tree/phylotree.cpp:4822-4880): the subtree at
  // `node` is pruned from internal `dad`, whose other neighbours s1 < s2 (by node id; the
  // reference takes them in its neighbour order) are joined by one branch of their summed
  // length, and dad is inserted into the branch (node2, dad2): its entry that pointed at s1 now
  // points at dad2, the one that pointed at s2 at node2, each half the branch's length.  Edges:
  // (dad, s1) -> (s1, s2), (dad, s2) -> (dad, dad2), (node2, dad2) -> (dad, node2).
  // Partials: the four neighbour entries whose subtree moves unchanged keep theirs (slot and
  // validity: (s1->s2) takes (dad->s2)'s, (s2->s1) (dad->s1)'s, (dad->dad2) (node2->dad2)'s,
  // (dad->node2) (dad2->node2)'s), the two new entries pointing at dad take the slots of the
  // two old ones (one slot per directed branch and pool modes), and every partial whose subtree
  // holds dad before or after the move is invalidated, which also covers any of the four whose
  // subtree did change (a regraft next to s1 or s2).
  int spr(int node, int dad, int node2, int dad2) {
    auto bad = [&](int x) { return x < 0 || x >= nnode; };
    if (bad(node) || bad(dad) || bad(node2) || bad(dad2)) return GEMS_ERR_BAD_ARG;
    const int kn = find(dad, node);
    if (leaf(dad) || kn < 0 || find(node2, dad2) < 0 || node2 == dad || dad2 == dad)
      return GEMS_ERR_BAD_ARG;
    std::vector<char> in_s(nnode, 0);
    mark(node, dad, in_s);
    if (in_s[node2] || in_s[dad2]) return GEMS_ERR_BAD_ARG;
    int ks[2], nk = 0;
    for (int k = 0; k < 3; k++)
      if (k != kn) ks[nk++] = k;
    if (adj[dad * 3 + ks[0]] > adj[dad * 3 + ks[1]]) std::swap(ks[0], ks[1]);
    const int s1 = adj[dad * 3 + ks[0]], s2 = adj[dad * 3 + ks[1]];
    const int ia = dad * 3 + ks[0], ib = dad * 3 + ks[1];
    const int ic = dir(s1, dad), id = dir(s2, dad);
    const int ie = dir(node2, dad2), iff = dir(dad2, node2);
    const double l1 = len[ia], l2 = len[ib], l = len[ie];
    clear_toward(dad);
    // contents: idx[i] takes src[i]'s (validity, and its slot in per-branch and pool modes)
    const int idx[6] = {ic, id, ia, ib, ie, iff}, src[6] = {ib, ia, ie, iff, ic, id};
    char cm[6];
    int ds[6];
    for (int i = 0; i < 6; i++) {
      cm[i] = computed[src[i]];
      ds[i] = dslot.empty() ? -1 : dslot[src[i]];
    }
    // LM_PER_NODE: a node's buffer owned by a moved entry follows it (the first four moves keep
    // their target node); dad's buffer was owned by an entry that now points elsewhere or by one
    // just invalidated, so it is released.  Every new owner is decided on the old owners.
    std::vector<std::pair<int, int>> reown;  // (slot, new owner)
    if (!per_branch && !pool) {
      for (int i = 0; i < 4; i++) {
        const int v = adj[src[i]];
        if (!leaf(v) && owner[node_slot[v]] == src[i]) reown.push_back({node_slot[v], idx[i]});
      }
      reown.push_back({node_slot[dad], -1});
    }
    adj[ic] = s2;
    adj[id] = s1;
    len[ic] = len[id] = l1 + l2;
    adj[ia] = dad2;
    adj[ib] = node2;
    adj[ie] = dad;
    adj[iff] = dad;
    len[ia] = len[ib] = len[ie] = len[iff] = l / 2;
    for (int i = 0; i < 6; i++) computed[idx[i]] = cm[i];
    if (per_branch || pool) {
      for (int i = 0; i < 6; i++) dslot[idx[i]] = ds[i];
      for (int i = 0; i < 6; i++)
        if (ds[i] >= 0) owner[ds[i]] = idx[i];
    } else {
      for (const auto &r : reown) owner[r.first] = r.second;
    }
    clear_toward(dad);
    int e_s1 = -1, e_s2 = -1, e_r = -1;
    for (int e = 0; e < nedges; e++) {
      const int a = eu[e], b = ev[e];
      if ((a == dad && b == s1) || (a == s1 && b == dad)) e_s1 = e;
      else if ((a == dad && b == s2) || (a == s2 && b == dad)) e_s2 = e;
      else if ((a == node2 && b == dad2) || (a == dad2 && b == node2)) e_r = e;
    }
    eu[e_s1] = s1;
    ev[e_s1] = s2;
    eu[e_s2] = dad;
    ev[e_s2] = dad2;
    eu[e_r] = dad;
    ev[e_r] = node2;
    theta_computed = false;
    cur_u = -1;
    if (pool) compute_sizes();
    return GEMS_OK;
  }

  // PhyloTree::getBestNNIForBran's evaluation (tree/phylotree.cpp:4176-4420, NNI-5 with one
  // evaluation round): both NNIs of the internal branch (u, v) -- u's neighbour a (the smaller
  // of its two other neighbours) swapped with each of v's other neighbours b (in id order) --
  // each evaluated by Newton on u's two outer branches, the central one and v's two outer ones
  // (outer branches in id order; the reference takes its neighbour order), the partial looking
  // back across each branch cleared before it is optimised, then the lnL from the buffers; the
  // swap is undone after each, and the lengths travel with the subtrees from the first move to
  // the second, as in the reference.  The tree is left as it was: its host state is restored,
  // and a partial held in a slot the evaluation wrote is recomputed when next needed.  With one
  // slot per internal node and two spare slots (nslots = internal nodes + 2), u's and v's
  // partials are computed in the spares (the reference's nni_partial_lh), so the tree's own
  // partials survive.  moves[2][2] = (a, b); lnl[2]; lens[2][5] = central, u's outer, v's outer.
  int nni_evaluate(int u, int v, int max_nr, int *moves, double *lnl, double *lens) {
    if (leaf(u) || leaf(v) || find(u, v) < 0) return GEMS_ERR_BAD_ARG;
    auto others = [&](int x, int y) {
      std::array<int, 2> o{};
      int n = 0;
      for (int k = 0; k < 3; k++)
        if (adj[x * 3 + k] != y) o[n++] = adj[x * 3 + k];
      if (o[0] > o[1]) std::swap(o[0], o[1]);
      return o;
    };
    const auto s_adj = adj, s_eu = eu, s_ev = ev, s_dslot = dslot, s_node = node_slot,
               s_owner = owner, s_sub = sub_size;
    const auto s_len = len;
    const auto s_comp = computed;
    const auto s_lock = slot_locked;
    const int s_free = pool_free, s_cur_u = cur_u, s_cur_k = cur_k;
    std::vector<char> written(nslots, 0);
    track = &written;
    const int ninternal = nnode - ntaxa;
    const bool spare = !per_branch && !pool && nslots >= ninternal + 2;
    if (spare) {  // u's and v's partials go to the two spare slots
      node_slot[u] = nslots - 2;
      node_slot[v] = nslots - 1;
      owner[nslots - 2] = owner[nslots - 1] = -1;
      for (int x = 0; x < nnode; x++)
        for (int k = 0; k < deg[x]; k++)
          if (adj[x * 3 + k] == u || adj[x * 3 + k] == v) computed[x * 3 + k] = 0;
    }
    const int a = others(u, v)[0];
    const auto bs = others(v, u);
    int st = GEMS_OK;
    for (int cnt = 0; cnt < 2 && st == GEMS_OK; cnt++) {
      const int b = bs[cnt];
      moves[2 * cnt] = a;
      moves[2 * cnt + 1] = b;
      if ((st = nni(u, v, a, b))) break;
      double *L = lens + 5 * cnt;
      int i = 1;
      for (int x : others(u, v)) {
        computed[dir(x, u)] = 0;
        if ((st = optimize_one(u, x, 0, max_nr))) break;
        L[i++] = len[u * 3 + find(u, x)];
      }
      if (st) break;
      computed[dir(v, u)] = 0;
      if ((st = optimize_one(u, v, 0, max_nr))) break;
      L[0] = len[u * 3 + find(u, v)];
      for (int y : others(v, u)) {
        computed[dir(y, v)] = 0;
        if ((st = optimize_one(v, y, 0, max_nr))) break;
        L[i++] = len[v * 3 + find(v, y)];
      }
      if (st) break;
      computed[dir(u, v)] = 0;
      if ((st = from_buffer(&lnl[cnt]))) break;
      st = nni(u, v, b, a);
    }
    track = nullptr;
    adj = s_adj;
    eu = s_eu;
    ev = s_ev;
    dslot = s_dslot;
    node_slot = s_node;
    owner = s_owner;
    sub_size = s_sub;
    len = s_len;
    computed = s_comp;
    slot_locked = s_lock;
    pool_free = s_free;
    cur_u = s_cur_u;
    cur_k = s_cur_k;
    theta_computed = false;  // the session's theta now belongs to the evaluation
    // a partial of the tree held in a slot the evaluation wrote is stale
    for (int d = 0; d < (int)computed.size(); d++) {
      if (!computed[d] || leaf(adj[d])) continue;
      const int sl = slot_of(d);
      if (sl < 0 || written[sl]) computed[d] = 0;
    }
    return st;
  }

  // PhyloTree::computeLikelihood (tree/phylotree.cpp:1258-1295)
  int compute_likelihood(double *lnl, double *pattern_lh) {
    if (cur_u < 0) {
      std::vector<int> h(nnode, 0);
      cur_u = far_leaf(0, -1, h);
      cur_k = 0;
    }
    const int v = adj[cur_u * 3 + cur_k];
    return lh_branch(v, cur_u, lnl, pattern_lh);
  }

  // computeLikelihood on new data: every partial is stale, the session's tips, weights and +I
  // terms are replaced, and the upload overlaps the traversal (gems_branch_lnl_from_host)
  int compute_likelihood_from_host(const uint8_t *states, const double *ptn_freq,
                                   const double *ptn_invar, int nchunks, double *lnl,
                                   double *pattern_lh) {
    std::fill(computed.begin(), computed.end(), 0);
    theta_computed = false;
    if (cur_u < 0) {
      std::vector<int> h(nnode, 0);
      cur_u = far_leaf(0, -1, h);
      cur_k = 0;
    }
    int node = adj[cur_u * 3 + cur_k], dad = cur_u;
    gems_branch br = branch(node, dad);
    if (pool_status) return pool_status;
    const int st = gems_branch_lnl_from_host(s, states, ptn_freq, ptn_invar, ops.data(),
                                             (int)ops.size(), &br, nchunks, lnl, pattern_lh);
    if (st) std::fill(computed.begin(), computed.end(), 0);
    return st;
  }
};

}  // namespace

struct gems_tree : public Tree {};

namespace {

// optimizeAllBranches on trees of one topology (ModelFinder's candidate models on one tree),
// each tree exactly as gems_tree_optimize_all_branches runs it, in lock-step over the common
// branch order: every tree's Newton loop on a branch is enqueued before any result is read,
// so the candidates' device work overlaps
int optimize_all_batch(gems_tree *const *ts, int n, int iterations, double tol, int max_nr,
                       double *out) {
  std::vector<int> n1, n2;
  ts[0]->best_traversal(n1, n2);
  std::vector<double> tree_lh(n, 0.0);
  std::vector<char> active(n, 1);
  std::vector<std::vector<double>> saved(n);
  for (int i = 0; i < n; i++) {
    if (int st = ts[i]->lh_branch(n2[0], n1[0], &tree_lh[i], nullptr)) return st;
    saved[i].resize(ts[i]->nedges);
  }
  for (int it = 0; it < iterations; it++) {
    bool any = false;
    for (int i = 0; i < n; i++) {
      if (!active[i]) continue;
      any = true;
      Tree &t = *ts[i];
      for (int e = 0; e < t.nedges; e++) saved[i][e] = t.len[t.eu[e] * 3 + t.find(t.eu[e], t.ev[e])];
    }
    if (!any) break;
    for (size_t j = 0; j < n1.size(); j++) {
      for (int i = 0; i < n; i++)
        if (active[i])
          if (int st = ts[i]->optimize_begin(n1[j], n2[j], max_nr)) return st;
      for (int i = 0; i < n; i++)
        if (active[i])
          if (int st = ts[i]->optimize_finish(n1[j], n2[j], 1)) return st;
    }
    for (int i = 0; i < n; i++) {
      if (!active[i]) continue;
      Tree &t = *ts[i];
      double new_lh = 0;
      if (int st = t.from_buffer(&new_lh)) return st;
      if (new_lh < tree_lh[i] - tol * 0.1) {
        std::fill(t.computed.begin(), t.computed.end(), 0);
        t.theta_computed = false;
        for (int e = 0; e < t.nedges; e++) t.set_len(t.eu[e], t.ev[e], saved[i][e]);
        if (int st = t.compute_likelihood(&new_lh, nullptr)) return st;
        tree_lh[i] = new_lh;
        active[i] = 0;
      } else if (tree_lh[i] <= new_lh && new_lh <= tree_lh[i] + tol) {
        tree_lh[i] = new_lh;
        active[i] = 0;
      } else {
        tree_lh[i] = new_lh;
      }
    }
  }
  for (int i = 0; i < n; i++) out[i] = tree_lh[i];
  return GEMS_OK;
}

}  // namespace

extern "C" {

int gems_tree_create(gems_session *s, int nedges, const int *eu, const int *ev,
                     const double *len, gems_tree **out) {
  if (!s || !eu || !ev || !len || !out || nedges < 3) return GEMS_ERR_BAD_ARG;
  gems_tree *t = new gems_tree();
  t->s = s;
  t->nedges = nedges;
  t->nnode = nedges + 1;
  t->ntaxa = (t->nnode + 2) / 2;
  t->deg.assign(t->nnode, 0);
  t->adj.assign(t->nnode * 3, -1);
  t->len.assign(t->nnode * 3, 0.0);
  t->eu.assign(eu, eu + nedges);
  t->ev.assign(ev, ev + nedges);
  for (int e = 0; e < nedges; e++) {
    const int u = eu[e], v = ev[e];
    if (u < 0 || v < 0 || u >= t->nnode || v >= t->nnode || u == v || t->deg[u] >= 3 ||
        t->deg[v] >= 3 || !(len[e] >= 0)) {
      delete t;
      return GEMS_ERR_BAD_ARG;
    }
    t->adj[u * 3 + t->deg[u]] = v;
    t->len[u * 3 + t->deg[u]++] = len[e];
    t->adj[v * 3 + t->deg[v]] = u;
    t->len[v * 3 + t->deg[v]++] = len[e];
  }
  for (int u = 0; u < t->nnode; u++) {
    const bool is_leaf_id = u < t->ntaxa;
    if ((is_leaf_id && t->deg[u] != 1) || (!is_leaf_id && t->deg[u] != 3)) {
      delete t;
      return GEMS_ERR_BAD_ARG;  // binary unrooted tree with leaves 0..ntaxa-1 required
    }
  }
  const int ninternal = t->nnode - t->ntaxa;
  // the number of slots the session holds decides the memory mode
  t->computed.assign(t->nnode * 3, 0);
  t->node_slot.assign(t->nnode, -1);
  t->dslot.assign(t->nnode * 3, -1);
  gems_session_desc desc{};
  if (gems_session_info(s, &desc) != GEMS_OK || desc.ntaxa != t->ntaxa) {
    delete t;
    return GEMS_ERR_BAD_ARG;
  }
  const int nslots = desc.nslots;
  // LM_MEM_SAVE's floor: log2(leafNum) + LH_MIN_CONST slots (tree/phylotree.cpp:42,1026-1040)
  const int min_slots = (int)std::log2((double)t->ntaxa) + 1;
  if (nslots < ninternal && nslots < min_slots) {
    delete t;
    return GEMS_ERR_ADMISSION;
  }
  t->nslots = nslots;
  int next = 0;
  if (nslots < ninternal) {
    t->pool = true;
    t->slot_locked.assign(nslots, 0);
    t->compute_sizes();
  } else if (nslots >= 3 * ninternal) {
    t->per_branch = true;
    for (int u = 0; u < t->nnode; u++)
      for (int k = 0; k < t->deg[u]; k++)
        if (!t->leaf(t->adj[u * 3 + k])) t->dslot[u * 3 + k] = next++;
  } else {
    for (int u = t->ntaxa; u < t->nnode; u++) t->node_slot[u] = next++;
  }
  t->owner.assign(nslots, -1);
  *out = t;
  return GEMS_OK;
}

int gems_tree_destroy(gems_tree *t) {
  delete t;
  return GEMS_OK;
}

int gems_tree_set_branch_limits(gems_tree *t, double min_len, double max_len) {
  if (!t || !(min_len >= 0) || !(max_len > min_len)) return GEMS_ERR_BAD_ARG;
  t->min_bl = min_len;
  t->max_bl = max_len;
  return GEMS_OK;
}

int gems_tree_set_length(gems_tree *t, int u, int v, double x) {
  if (!t || u < 0 || v < 0 || u >= t->nnode || v >= t->nnode || t->find(u, v) < 0 || !(x >= 0))
    return GEMS_ERR_BAD_ARG;
  t->set_len(u, v, x);
  // a changed length invalidates partials looking across the branch
  t->clear_reverse(u, v);
  t->clear_reverse(v, u);
  t->theta_computed = false;
  return GEMS_OK;
}

int gems_tree_get_lengths(gems_tree *t, double *out) {
  if (!t || !out) return GEMS_ERR_BAD_ARG;
  for (int e = 0; e < t->nedges; e++) out[e] = t->len[t->eu[e] * 3 + t->find(t->eu[e], t->ev[e])];
  return GEMS_OK;
}

int gems_tree_clear_all_partial_lh(gems_tree *t) {
  if (!t) return GEMS_ERR_BAD_ARG;
  std::fill(t->computed.begin(), t->computed.end(), 0);
  t->theta_computed = false;
  return GEMS_OK;
}

int gems_tree_compute_likelihood(gems_tree *t, double *lnl, double *pattern_lh) {
  if (!t || !lnl) return GEMS_ERR_BAD_ARG;
  return t->compute_likelihood(lnl, pattern_lh);
}

int gems_tree_compute_likelihood_from_host(gems_tree *t, const uint8_t *states,
                                           const double *ptn_freq, const double *ptn_invar,
                                           int nchunks, double *lnl, double *pattern_lh) {
  if (!t || !states || !ptn_freq || !lnl || nchunks < 1) return GEMS_ERR_BAD_ARG;
  return t->compute_likelihood_from_host(states, ptn_freq, ptn_invar, nchunks, lnl, pattern_lh);
}

int gems_tree_compute_likelihood_branch(gems_tree *t, int node, int dad, double *lnl,
                                        double *pattern_lh) {
  if (!t || !lnl || node < 0 || dad < 0 || node >= t->nnode || dad >= t->nnode ||
      t->find(node, dad) < 0)
    return GEMS_ERR_BAD_ARG;
  return t->lh_branch(node, dad, lnl, pattern_lh);
}

int gems_tree_compute_likelihood_derv(gems_tree *t, int node, int dad, double *df, double *ddf) {
  if (!t || !df || !ddf || node < 0 || dad < 0 || node >= t->nnode || dad >= t->nnode ||
      t->find(node, dad) < 0)
    return GEMS_ERR_BAD_ARG;
  return t->derv(node, dad, df, ddf);
}

int gems_tree_compute_likelihood_from_buffer(gems_tree *t, double *lnl) {
  if (!t || !lnl) return GEMS_ERR_BAD_ARG;
  return t->from_buffer(lnl);
}

int gems_tree_optimize_one_branch(gems_tree *t, int node1, int node2, int clear_lh,
                                  int max_nr_step) {
  if (!t || node1 < 0 || node2 < 0 || node1 >= t->nnode || node2 >= t->nnode ||
      max_nr_step < 1)
    return GEMS_ERR_BAD_ARG;
  return t->optimize_one(node1, node2, clear_lh, max_nr_step);
}

int gems_tree_optimize_all_branches(gems_tree *t, int iterations, double tolerance,
                                    int max_nr_step, double *lnl) {
  if (!t || !lnl || iterations < 1 || max_nr_step < 1) return GEMS_ERR_BAD_ARG;
  return t->optimize_all(iterations, tolerance, max_nr_step, lnl);
}

int gems_tree_optimize_all_branches_batch(gems_tree *const *trees, int ntrees, int iterations,
                                          double tolerance, int max_nr_step, double *lnl) {
  if (!trees || ntrees < 1 || !lnl || iterations < 1 || max_nr_step < 1) return GEMS_ERR_BAD_ARG;
  for (int i = 0; i < ntrees; i++) {
    if (!trees[i]) return GEMS_ERR_BAD_ARG;
    if (trees[i]->adj != trees[0]->adj || trees[i]->deg != trees[0]->deg) return GEMS_ERR_BAD_ARG;
    for (int j = 0; j < i; j++)
      if (trees[j] == trees[i] || trees[j]->s == trees[i]->s) return GEMS_ERR_BAD_ARG;
  }
  return optimize_all_batch(trees, ntrees, iterations, tolerance, max_nr_step, lnl);
}

int gems_tree_compute_likelihood_batch(gems_tree *const *trees, int ntrees, double *lnl) {
  if (!trees || ntrees <= 0 || !lnl) return GEMS_ERR_BAD_ARG;
  std::vector<gems_session *> ss(ntrees);
  std::vector<gems_branch> br(ntrees);
  std::vector<const gems_op *> ops(ntrees);
  std::vector<int> nops(ntrees);
  for (int i = 0; i < ntrees; i++) {
    gems_tree *t = trees[i];
    if (!t) return GEMS_ERR_BAD_ARG;
    // the branch computeLikelihood evaluates (compute_likelihood)
    if (t->cur_u < 0) {
      std::vector<int> h(t->nnode, 0);
      t->cur_u = t->far_leaf(0, -1, h);
      t->cur_k = 0;
    }
    int node = t->adj[t->cur_u * 3 + t->cur_k], dad = t->cur_u;
    br[i] = t->branch(node, dad);
    if (t->pool_status) return t->pool_status;
    ss[i] = t->s;
    ops[i] = t->ops.data();
    nops[i] = (int)t->ops.size();
  }
  const int st =
      gems_branch_lnl_batch_ops(ss.data(), ntrees, ops.data(), nops.data(), br.data(), lnl);
  if (st) {
    // the op lists marked their partials computed, but nothing (or not all of it) ran: every
    // tree recomputes from scratch at its next evaluation
    for (int i = 0; i < ntrees; i++) std::fill(trees[i]->computed.begin(), trees[i]->computed.end(), 0);
  }
  return st;
}

int gems_tree_nni(gems_tree *t, int u, int v, int a, int b) {
  if (!t || u < 0 || v < 0 || a < 0 || b < 0 || u >= t->nnode || v >= t->nnode ||
      a >= t->nnode || b >= t->nnode)
    return GEMS_ERR_BAD_ARG;
  return t->nni(u, v, a, b);
}

int gems_tree_nni_evaluate(gems_tree *t, int u, int v, int max_nr_step, int *moves,
                           double *lnl, double *lens) {
  if (!t || !moves || !lnl || !lens || u < 0 || v < 0 || u >= t->nnode || v >= t->nnode ||
      max_nr_step < 1)
    return GEMS_ERR_BAD_ARG;
  return t->nni_evaluate(u, v, max_nr_step, moves, lnl, lens);
}

int gems_tree_spr(gems_tree *t, int node, int dad, int node2, int dad2) {
  if (!t) return GEMS_ERR_BAD_ARG;
  return t->spr(node, dad, node2, dad2);
}

int gems_tree_get_edges(gems_tree *t, int *eu, int *ev) {
  if (!t || !eu || !ev) return GEMS_ERR_BAD_ARG;
  for (int e = 0; e < t->nedges; e++) {
    eu[e] = t->eu[e];
    ev[e] = t->ev[e];
  }
  return GEMS_OK;
}

int gems_tree_compute_func_derv(gems_tree *t, int node1, int node2, double value,
                                int new_branch, double *f, double *df) {
  if (!t || !f || !df || node1 < 0 || node2 < 0 || node1 >= t->nnode || node2 >= t->nnode ||
      t->find(node1, node2) < 0 || !(value >= 0))
    return GEMS_ERR_BAD_ARG;
  // PhyloTree::computeFuncDerv (tree/phylotree.cpp:2555): current_it = node1 -> node2, both
  // lengths set to value without invalidating partials (theta does not depend on the length)
  t->cur_u = node1;
  t->cur_k = t->find(node1, node2);
  if (new_branch) t->theta_computed = false;
  t->set_len(node1, node2, value);
  double d1 = 0, d2 = 0;
  const int st = t->derv(node2, node1, &d1, &d2);
  if (st) return st;
  *f = -d1;
  *df = -d2;
  return GEMS_OK;
}

int gems_tree_get_partial(gems_tree *t, int node, int dad, double *partial, uint16_t *scale) {
  if (!t || node < 0 || dad < 0 || node >= t->nnode || dad >= t->nnode ||
      t->find(dad, node) < 0 || t->leaf(node))
    return GEMS_ERR_BAD_ARG;
  const int d = t->dir(dad, node);
  if (!t->computed[d]) return GEMS_ERR_STATE;
  return gems_get_partial(t->s, t->slot_of(d), partial, scale);
}

int gems_tree_stats(gems_tree *t, long long *partial_ops, int *last_newton_evals) {
  if (!t) return GEMS_ERR_BAD_ARG;
  if (partial_ops) *partial_ops = t->partial_ops;
  if (last_newton_evals) *last_newton_evals = t->newton_evals;
  return GEMS_OK;
}

}  // extern "C"
