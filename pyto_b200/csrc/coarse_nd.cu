// Sparse coarse solver of the deflated PCG: nested dissection of W_f^T K_ff W_f on a
// regular box grid of node groups (the direct coarse solve of src/deflation.py:517-521,
// 577, for coarse spaces far beyond a dense matrix).
//
// Symbolic phase (host, pyto_coarse_nd_plan).  The box [0,gx) x [0,gy) x [0,gz) of group
// indices is split recursively: a box of more than `leaf` groups is cut across its longest
// side by a separator plane of groups (thickness 1, enough for the 27-neighbour block
// pattern) into two sub-boxes; the separator (or a leaf box) is the node's own set, and its
// unknowns are eliminated after those of both sub-trees (post-order).  Every group adjacent
// to a node's box but outside it belongs to an ancestor separator (siblings are two planes
// apart), so a node's boundary is exactly the one-group shell around its box.  The front of
// a node is the dense matrix over [own groups, boundary groups] x modes; a child's boundary
// lies inside its parent's front.
//
// Numeric phase (per pyto_dpcg_setup, fully on the device, no host synchronisation).  The
// coarse matrix is assembled block-sparse in the deflation's neighbour-slot order (64-bit
// fixed point per row group, as the dense path), converted, its diagonal blocks
// symmetrised and shifted.  Then for each tree level, deepest first: zero the level's
// fronts; push each coarse block into the one front that eliminates the earlier of its two
// groups (block and transpose; every front entry receives at most one block); add each
// child's Schur complement into its parent's front (first children, then second children:
// no two writes meet); sweep the node's own pivots with the blocked Gauss-Jordan kernels of
// the dense inverse (batched over the level's fronts); mirror the lower tiles into the
// upper ones, so that a front is stored in full.  A front then holds -A_ss^-1 (own x own),
// L = A_bs A_ss^-1 (boundary x own), its transpose (own x boundary) and the Schur
// complement (boundary x boundary).
//
// Solve (per coarse correction): up the tree, a node's own part is its entries of v plus
// what its children left in its two incoming slots (one per child: no two writes meet,
// and the sum runs in a fixed order); each boundary row, incoming slots - L . own part,
// goes straight into the parent's slot of this child through the child's map.  Down the
// tree, the own unknowns are -[rows of own] . [own part ; solution at the boundary
// groups], one GEMV over full front rows.  One kernel per level and direction, a warp per
// front row.
#include <algorithm>
#include <cstring>
#include <vector>

#include "krylov.cuh"
#include "sweep.cuh"

namespace pyto {

struct NdNode {
  int box[6];  // x0, x1, y0, y1, z0, z1 (half-open group index ranges)
  int parent = -1, nchild = 0, depth = 0;
  int child[2] = {-1, -1};
  std::vector<int> own, bnd;  // group ids: own (box / separator order), boundary (elimination order)
};

constexpr int kNdRows = 32;       // front rows per CTA of the solve kernels (8 warps, 4 rows each)
constexpr int kNdThreads = 256;
constexpr int kNdMaxFront = 8192;  // largest front (unknowns) staged in shared memory by the solves
constexpr int kNdDiagBlocks = 256;  // blocks of the diagonal pass (partial sums of |diag|)

}  // namespace pyto

// Host plan: tree, device layout and the host copies of the device tables.
struct pyto_coarse_nd {
  int gx = 0, gy = 0, gz = 0, M = 0, leaf = 0, ng = 0;
  long long nslots = 0;  // blocks of the neighbour lists
  std::vector<pyto::NdNode> node;
  std::vector<int> order;                // post-order
  std::vector<std::vector<int>> lvl;     // nodes by depth
  int depth = 0, maxF = 0;
  double flops = 0.0, solve_bytes = 0.0;
  // per node (host): front size, own unknowns, offsets
  std::vector<long long> front_off, fv_off, scr_off;
  std::vector<int> F, own, fg_off, nfg, emap_off, cslot, child0, child1, parent;
  std::vector<int> fgroups, emap, diag_slot;
  // coarse block pushes (sorted by level)
  std::vector<long long> push_dst1, push_dst2;
  std::vector<int> push_slot, push_ld, push_lo;  // push_lo[level .. level+1]
  // per level: extend-add children (pass 0 then pass 1), sweep and solve work items
  std::vector<int> ext_child, ext_lo;       // ext_lo[2 level + pass]
  std::vector<int> piv_node, piv_lo;        // nodes of the level (pivot kernel)
  std::vector<int> pan_item, pan_lo;        // (node, column chunk) pairs
  std::vector<int> tile_item, tile_lo;      // (node, ti, tj) triples, lower tiles
  std::vector<int> fwd_item, fwd_lo;        // (node, first boundary row)
  std::vector<int> bwd_item, bwd_lo;        // (node, first own row)
  std::vector<int> lvl_maxown;              // largest own count of each level
  std::vector<long long> lvl_front_lo, lvl_front_hi;
  long long fronts_doubles = 0, fv_doubles = 0, scr_doubles = 0;
  // device layout: byte offsets in the bound buffer
  size_t o_E = 0, o_fronts = 0, o_fv = 0, o_in = 0, o_scr = 0, o_i64 = 0, o_i32 = 0, bytes = 0;
  std::vector<long long> i64;  // packed 64-bit tables
  std::vector<int> i32;        // packed 32-bit tables
  // offsets of each table inside i64 / i32
  size_t t_front_off, t_fv_off, t_scr_off, t_push_dst1, t_push_dst2;
  size_t t_F, t_own, t_fg_off, t_nfg, t_emap_off, t_cslot, t_child0, t_child1, t_parent, t_fgroups, t_emap,
      t_push_slot, t_push_ld, t_ext_child, t_piv_node, t_pan_item, t_tile_item, t_fwd_item, t_bwd_item,
      t_diag_slot;
  char* dev = nullptr;
};

namespace pyto {
namespace {

int nd_rec(pyto_coarse_nd* P, const int (&box)[6], int depth, int parent) {
  const int me = (int)P->node.size();
  P->node.emplace_back();
  {
    NdNode& n = P->node[me];
    for (int i = 0; i < 6; ++i) n.box[i] = box[i];
    n.parent = parent;
    n.depth = depth;
  }
  const int ext[3] = {box[1] - box[0], box[3] - box[2], box[5] - box[4]};
  const long long vol = (long long)ext[0] * ext[1] * ext[2];
  int own_box[6];
  for (int i = 0; i < 6; ++i) own_box[i] = box[i];
  if (vol > P->leaf) {
    int ax = 0;
    for (int d = 1; d < 3; ++d)
      if (ext[d] > ext[ax]) ax = d;
    const int lo = box[2 * ax], hi = box[2 * ax + 1], mid = (lo + hi) / 2;
    int sub[2][6];
    for (int s = 0; s < 2; ++s)
      for (int i = 0; i < 6; ++i) sub[s][i] = box[i];
    sub[0][2 * ax + 1] = mid;
    sub[1][2 * ax] = mid + 1;
    own_box[2 * ax] = mid;
    own_box[2 * ax + 1] = mid + 1;
    for (int s = 0; s < 2; ++s) {
      if (sub[s][2 * ax + 1] <= sub[s][2 * ax]) continue;
      const int c = nd_rec(P, sub[s], depth + 1, me);
      NdNode& n = P->node[me];
      n.child[n.nchild++] = c;
    }
  }
  std::vector<int> own;
  for (int k = own_box[4]; k < own_box[5]; ++k)
    for (int j = own_box[2]; j < own_box[3]; ++j)
      for (int i = own_box[0]; i < own_box[1]; ++i) own.push_back(i + P->gx * (j + P->gy * k));
  P->node[me].own.swap(own);
  return me;
}

void nd_post(const pyto_coarse_nd* P, int n, std::vector<int>& out) {
  for (int c = 0; c < P->node[n].nchild; ++c) nd_post(P, P->node[n].child[c], out);
  out.push_back(n);
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

// Tree, boundary shells, front layout and the device tables; 0 or an error message.
const char* nd_build(pyto_coarse_nd* P, const int32_t* nptr, const int32_t* nlist) {
  const int M = P->M;
  const int top[6] = {0, P->gx, 0, P->gy, 0, P->gz};
  nd_rec(P, top, 0, -1);
  const int nn = (int)P->node.size();
  nd_post(P, 0, P->order);
  std::vector<int> pos(P->ng, -1), owner(P->ng, -1);
  int p = 0;
  for (int n : P->order)
    for (int g : P->node[n].own) {
      pos[g] = p++;
      owner[g] = n;
    }
  if (p != P->ng) return "nested dissection did not cover every group";
  P->depth = 0;
  for (auto& n : P->node) P->depth = std::max(P->depth, n.depth);
  for (auto& n : P->node) {
    for (int k = std::max(0, n.box[4] - 1); k < std::min(P->gz, n.box[5] + 1); ++k)
      for (int j = std::max(0, n.box[2] - 1); j < std::min(P->gy, n.box[3] + 1); ++j)
        for (int i = std::max(0, n.box[0] - 1); i < std::min(P->gx, n.box[1] + 1); ++i) {
          if (i >= n.box[0] && i < n.box[1] && j >= n.box[2] && j < n.box[3] && k >= n.box[4] && k < n.box[5])
            continue;
          n.bnd.push_back(i + P->gx * (j + P->gy * k));
        }
    std::sort(n.bnd.begin(), n.bnd.end(), [&](int a, int b) { return pos[a] < pos[b]; });
  }
  P->lvl.assign(P->depth + 1, {});
  for (int n = 0; n < nn; ++n) P->lvl[P->node[n].depth].push_back(n);
  // per node sizes and the front group lists
  P->F.assign(nn, 0);
  P->own.assign(nn, 0);
  P->fg_off.assign(nn, 0);
  P->nfg.assign(nn, 0);
  P->child0.assign(nn, -1);
  P->child1.assign(nn, -1);
  P->parent.assign(nn, -1);
  for (int n = 0; n < nn; ++n) {
    const NdNode& d = P->node[n];
    P->nfg[n] = (int)(d.own.size() + d.bnd.size());
    P->F[n] = M * P->nfg[n];
    P->own[n] = M * (int)d.own.size();
    P->fg_off[n] = (int)P->fgroups.size();
    P->fgroups.insert(P->fgroups.end(), d.own.begin(), d.own.end());
    P->fgroups.insert(P->fgroups.end(), d.bnd.begin(), d.bnd.end());
    P->child0[n] = d.child[0];
    P->child1[n] = d.child[1];
    P->parent[n] = d.parent;
    P->maxF = std::max(P->maxF, P->F[n]);
    P->flops += 2.0 * P->own[n] * (double)P->F[n] * P->F[n];
    P->solve_bytes += 8.0 * ((double)P->own[n] * P->F[n] + (double)(P->F[n] - P->own[n]) * P->own[n]);
  }
  if (P->maxF > kNdMaxFront) return "a frontal matrix exceeds the solve kernels' limit";
  // fronts, frontal vectors and sweep scratch, level by level (deepest first)
  P->front_off.assign(nn, 0);
  P->fv_off.assign(nn, 0);
  P->scr_off.assign(nn, 0);
  P->lvl_front_lo.assign(P->depth + 1, 0);
  P->lvl_front_hi.assign(P->depth + 1, 0);
  long long fo = 0, vo = 0;
  for (int l = P->depth; l >= 0; --l) {
    P->lvl_front_lo[l] = fo;
    long long so = 0;
    for (int n : P->lvl[l]) {
      P->front_off[n] = fo;
      fo += (long long)P->F[n] * P->F[n];
      P->fv_off[n] = vo;
      vo += P->F[n];
      P->scr_off[n] = so;
      so += (long long)kSweepB * kSweepB + 2LL * kSweepB * P->F[n];
    }
    P->lvl_front_hi[l] = fo;
    P->scr_doubles = std::max(P->scr_doubles, so);
  }
  P->fronts_doubles = fo;
  P->fv_doubles = vo;
  // children's boundary groups in the parent's front, and which child each node is
  P->emap_off.assign(nn, -1);
  P->cslot.assign(nn, -1);
  std::vector<int> loc(P->ng, -1);
  for (int n = 0; n < nn; ++n) {
    const NdNode& d = P->node[n];
    if (d.nchild == 0) continue;
    for (int r = 0; r < P->nfg[n]; ++r) loc[P->fgroups[P->fg_off[n] + r]] = r;
    for (int c = 0; c < d.nchild; ++c) {
      const int ch = d.child[c];
      P->emap_off[ch] = (int)P->emap.size();
      P->cslot[ch] = c;
      for (int g : P->node[ch].bnd) {
        const int r = loc[g];
        if (r < 0) return "a child's boundary group is outside its parent's front";
        P->emap.push_back(r);
      }
    }
    for (int r = 0; r < P->nfg[n]; ++r) loc[P->fgroups[P->fg_off[n] + r]] = -1;
  }
  // coarse blocks E[G, H] (H <= G, as assembled) into the front eliminating the earlier group
  P->nslots = nptr[P->ng];
  std::vector<std::vector<int>> lvl_items(P->depth + 1);
  std::vector<long long> d1(P->nslots, -1), d2(P->nslots, -1);
  std::vector<int> ld(P->nslots, 0);
  P->diag_slot.assign(P->ng, -1);
  for (int G = 0; G < P->ng; ++G) {
    const int gi = G % P->gx, gj = (G / P->gx) % P->gy, gk = G / (P->gx * P->gy);
    for (int sl = nptr[G]; sl < nptr[G + 1]; ++sl)
      if (nlist[sl] == G) P->diag_slot[G] = sl;
    if (P->diag_slot[G] < 0) return "a group is missing from its own neighbour list";
    for (int sl = nptr[G]; sl < nptr[G + 1]; ++sl) {
      const int H = nlist[sl];
      if (H < 0 || H >= P->ng) return "neighbour list entry out of range";
      const int hi = H % P->gx, hj = (H / P->gx) % P->gy, hk = H / (P->gx * P->gy);
      if (std::abs(hi - gi) > 1 || std::abs(hj - gj) > 1 || std::abs(hk - gk) > 1)
        return "a neighbour group is not adjacent on the box grid";
      if (H > G) continue;
      const int first = pos[G] <= pos[H] ? G : H, other = first == G ? H : G;
      const int n = owner[first];
      int lf = -1, lo2 = -1;
      for (int r = 0; r < P->nfg[n]; ++r) {
        const int g = P->fgroups[P->fg_off[n] + r];
        if (g == G) lf = r;
        if (g == H) lo2 = r;
      }
      (void)other;
      if (lf < 0 || lo2 < 0) return "a coarse block falls outside the front that eliminates it";
      const long long F = P->F[n];
      d1[sl] = P->front_off[n] + (long long)lf * M * F + (long long)lo2 * M;
      d2[sl] = (G == H) ? -1 : P->front_off[n] + (long long)lo2 * M * F + (long long)lf * M;
      ld[sl] = (int)F;
      lvl_items[P->node[n].depth].push_back(sl);
    }
  }
  P->push_lo.assign(P->depth + 2, 0);
  for (int l = 0; l <= P->depth; ++l) {
    P->push_lo[l] = (int)P->push_slot.size();
    for (int sl : lvl_items[l]) {
      P->push_slot.push_back(sl);
      P->push_dst1.push_back(d1[sl]);
      P->push_dst2.push_back(d2[sl]);
      P->push_ld.push_back(ld[sl]);
    }
  }
  P->push_lo[P->depth + 1] = (int)P->push_slot.size();
  return nullptr;
}

// Work lists of the level kernels and the packed device tables.
void nd_items(pyto_coarse_nd* P) {
  const int L = P->depth + 1;
  P->ext_lo.assign(2 * L + 1, 0);
  P->piv_lo.assign(L + 1, 0);
  P->pan_lo.assign(L + 1, 0);
  P->tile_lo.assign(L + 1, 0);
  P->fwd_lo.assign(L + 1, 0);
  P->bwd_lo.assign(L + 1, 0);
  P->lvl_maxown.assign(L, 0);
  for (int l = 0; l < L; ++l) {  // indexed by level; lists kept in level order
    for (int pass = 0; pass < 2; ++pass) {
      P->ext_lo[2 * l + pass] = (int)P->ext_child.size();
      for (int n : P->lvl[l])
        if (P->node[n].nchild > pass) P->ext_child.push_back(P->node[n].child[pass]);
    }
    P->piv_lo[l] = (int)P->piv_node.size();
    P->pan_lo[l] = (int)P->pan_item.size() / 2;
    P->tile_lo[l] = (int)P->tile_item.size() / 3;
    P->fwd_lo[l] = (int)P->fwd_item.size() / 2;
    P->bwd_lo[l] = (int)P->bwd_item.size() / 2;
    for (int n : P->lvl[l]) {
      const int F = P->F[n], own = P->own[n];
      P->lvl_maxown[l] = std::max(P->lvl_maxown[l], own);
      P->piv_node.push_back(n);
      for (int j = 0; j < F; j += 16) {
        P->pan_item.push_back(n);
        P->pan_item.push_back(j);
      }
      const int nt = (F + 63) / 64;
      for (int ti = 0; ti < nt; ++ti)
        for (int tj = 0; tj <= ti; ++tj) {
          P->tile_item.push_back(n);
          P->tile_item.push_back(ti);
          P->tile_item.push_back(tj);
        }
      const int nb = F - own;
      for (int r = 0; r < std::max(nb, 1); r += kNdRows) {
        P->fwd_item.push_back(n);
        P->fwd_item.push_back(r);
      }
      for (int r = 0; r < own; r += kNdRows) {
        P->bwd_item.push_back(n);
        P->bwd_item.push_back(r);
      }
    }
  }
  P->ext_lo[2 * L] = (int)P->ext_child.size();
  P->piv_lo[L] = (int)P->piv_node.size();
  P->pan_lo[L] = (int)P->pan_item.size() / 2;
  P->tile_lo[L] = (int)P->tile_item.size() / 3;
  P->fwd_lo[L] = (int)P->fwd_item.size() / 2;
  P->bwd_lo[L] = (int)P->bwd_item.size() / 2;
  // packed tables
  auto put64 = [&](const std::vector<long long>& v) {
    const size_t o = P->i64.size();
    P->i64.insert(P->i64.end(), v.begin(), v.end());
    return o;
  };
  auto put32 = [&](const std::vector<int>& v) {
    const size_t o = P->i32.size();
    P->i32.insert(P->i32.end(), v.begin(), v.end());
    P->i32.resize((P->i32.size() + 3) & ~(size_t)3, 0);  // 16-byte aligned tables
    return o;
  };
  P->t_front_off = put64(P->front_off);
  P->t_fv_off = put64(P->fv_off);
  P->t_scr_off = put64(P->scr_off);
  P->t_push_dst1 = put64(P->push_dst1);
  P->t_push_dst2 = put64(P->push_dst2);
  P->t_F = put32(P->F);
  P->t_own = put32(P->own);
  P->t_fg_off = put32(P->fg_off);
  P->t_nfg = put32(P->nfg);
  P->t_emap_off = put32(P->emap_off);
  P->t_cslot = put32(P->cslot);
  P->t_child0 = put32(P->child0);
  P->t_child1 = put32(P->child1);
  P->t_parent = put32(P->parent);
  P->t_fgroups = put32(P->fgroups);
  P->t_emap = put32(P->emap);
  P->t_push_slot = put32(P->push_slot);
  P->t_push_ld = put32(P->push_ld);
  P->t_ext_child = put32(P->ext_child);
  P->t_piv_node = put32(P->piv_node);
  P->t_pan_item = put32(P->pan_item);
  P->t_tile_item = put32(P->tile_item);
  P->t_fwd_item = put32(P->fwd_item);
  P->t_bwd_item = put32(P->bwd_item);
  P->t_diag_slot = put32(P->diag_slot);
  size_t o = 0;
  P->o_E = o;
  o = align256(o + (size_t)P->nslots * P->M * P->M * sizeof(double));
  P->o_fronts = o;
  o = align256(o + (size_t)P->fronts_doubles * sizeof(double));
  P->o_fv = o;
  o = align256(o + (size_t)P->fv_doubles * sizeof(double));
  P->o_in = o;  // the children's contributions to each front (two slots)
  o = align256(o + 2 * (size_t)P->fv_doubles * sizeof(double));
  P->o_scr = o;
  o = align256(o + (size_t)(P->scr_doubles + kNdDiagBlocks) * sizeof(double));  // + the diagonal partials
  P->o_i64 = o;
  o = align256(o + P->i64.size() * sizeof(long long));
  P->o_i32 = o;
  o = align256(o + P->i32.size() * sizeof(int));
  P->bytes = o;
}

}  // namespace pyto

namespace pyto {

// Device view of a bound plan.
struct NdDev {
  double *E, *fronts, *fv, *in0, *in1, *scr, *mean;
  const long long *front_off, *fv_off, *scr_off, *push_dst1, *push_dst2;
  const int *F, *own, *fg_off, *emap_off, *cslot, *child0, *child1, *parent, *fgroups, *emap, *push_slot, *push_ld, *ext_child, *piv_node, *pan_item, *tile_item, *fwd_item, *bwd_item, *diag_slot;
  int M, ng;
};

static NdDev nd_dev(const pyto_coarse_nd* P) {
  NdDev d;
  char* b = P->dev;
  d.E = (double*)(b + P->o_E);
  d.fronts = (double*)(b + P->o_fronts);
  d.fv = (double*)(b + P->o_fv);
  d.in0 = (double*)(b + P->o_in);
  d.in1 = d.in0 + P->fv_doubles;
  d.scr = (double*)(b + P->o_scr);
  d.mean = d.scr + P->scr_doubles;
  const long long* i64 = (const long long*)(b + P->o_i64);
  const int* i32 = (const int*)(b + P->o_i32);
  d.front_off = i64 + P->t_front_off;
  d.fv_off = i64 + P->t_fv_off;
  d.scr_off = i64 + P->t_scr_off;
  d.push_dst1 = i64 + P->t_push_dst1;
  d.push_dst2 = i64 + P->t_push_dst2;
  d.F = i32 + P->t_F;
  d.own = i32 + P->t_own;
  d.fg_off = i32 + P->t_fg_off;
  d.emap_off = i32 + P->t_emap_off;
  d.cslot = i32 + P->t_cslot;
  d.child0 = i32 + P->t_child0;
  d.child1 = i32 + P->t_child1;
  d.parent = i32 + P->t_parent;
  d.fgroups = i32 + P->t_fgroups;
  d.emap = i32 + P->t_emap;
  d.push_slot = i32 + P->t_push_slot;
  d.push_ld = i32 + P->t_push_ld;
  d.ext_child = i32 + P->t_ext_child;
  d.piv_node = i32 + P->t_piv_node;
  d.pan_item = i32 + P->t_pan_item;
  d.tile_item = i32 + P->t_tile_item;
  d.fwd_item = i32 + P->t_fwd_item;
  d.bwd_item = i32 + P->t_bwd_item;
  d.diag_slot = i32 + P->t_diag_slot;
  d.M = P->M;
  d.ng = P->ng;
  return d;
}

// Block-sparse coarse matrix: 64-bit fixed-point sums -> FP64 (row group scale 2^gexp[G]);
// blocks above the group diagonal (H > G, not assembled) are 0; diagonal blocks
// symmetrised.  One CTA per row group.
__global__ void __launch_bounds__(128) k_nd_from_fixed(NdDev d, const int32_t* __restrict__ nptr,
                                                       const int32_t* __restrict__ nlist,
                                                       const int* __restrict__ gexp) {
  const int G = blockIdx.x, M2 = d.M * d.M;
  const int s0 = nptr[G], s1 = nptr[G + 1];
  const int e = gexp[G];
  for (int t = threadIdx.x; t < (s1 - s0) * M2; t += blockDim.x) {
    const long long i = (long long)s0 * M2 + t;
    const long long q = reinterpret_cast<const long long*>(d.E)[i];
    d.E[i] = nlist[s0 + t / M2] <= G ? ldexp((double)q, -e) : 0.0;
  }
  __syncthreads();
  for (int s = s0; s < s1; ++s) {
    if (nlist[s] != G) continue;
    double* B = d.E + (long long)s * M2;
    for (int t = threadIdx.x; t < M2; t += blockDim.x) {
      const int a = t / d.M, b = t - a * d.M;
      if (a < b) {
        const double v = 0.5 * (B[a * d.M + b] + B[b * d.M + a]);
        B[a * d.M + b] = v;
        B[b * d.M + a] = v;
      }
    }
  }
}

// diagonal: zero -> 1 (a mode that vanishes on the free DOFs), + shift (relative: times
// the mean |diagonal|).  Pass 1: partial sums of |diag| over fixed chunks of the
// unknowns; pass 2: every block sums the partials in order (the same mean in all
// blocks) and updates its chunk.
__global__ void __launch_bounds__(256) k_nd_diag_sum(NdDev d) {
  __shared__ double sred[8];
  const long long nc = (long long)d.ng * d.M, per = (nc + gridDim.x - 1) / gridDim.x;
  const long long i0 = blockIdx.x * per, i1 = min(nc, i0 + per);
  double acc = 0.0;
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int G = (int)(i / d.M), a = (int)(i - (long long)G * d.M);
    acc += fabs(d.E[((long long)d.diag_slot[G] * d.M + a) * d.M + a]);
  }
  const double t = block_sum<256>(acc, sred);
  if (threadIdx.x == 0) d.mean[blockIdx.x] = t;
}

__global__ void __launch_bounds__(256) k_nd_diag_apply(NdDev d, double shift, int relative) {
  __shared__ double s_sh;
  const long long nc = (long long)d.ng * d.M, per = (nc + gridDim.x - 1) / gridDim.x;
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) t += d.mean[b];
    s_sh = relative ? shift * (t / (double)nc) : shift;
  }
  __syncthreads();
  const double sh = s_sh;
  const long long i0 = blockIdx.x * per, i1 = min(nc, i0 + per);
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int G = (int)(i / d.M), a = (int)(i - (long long)G * d.M);
    double* p = d.E + ((long long)d.diag_slot[G] * d.M + a) * d.M + a;
    double v = *p;
    if (v == 0.0) v = 1.0;
    *p = v + sh;
  }
}

// coarse blocks into the fronts of one level (block and, off the group diagonal, transpose)
__global__ void k_nd_push(NdDev d, int lo, int hi) {
  const int M2 = d.M * d.M;
  const long long n = (long long)(hi - lo) * M2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int it = lo + (int)(t / M2), e = (int)(t % M2);
    const int a = e / d.M, b = e - a * d.M;
    const double v = d.E[(long long)d.push_slot[it] * M2 + e];
    const long long ld = d.push_ld[it];
    d.fronts[d.push_dst1[it] + a * ld + b] = v;
    const long long t2 = d.push_dst2[it];
    if (t2 >= 0) d.fronts[t2 + b * ld + a] = v;
  }
}

// Schur complements of one pass of children into their parents' fronts (blockIdx.y: child)
__global__ void k_nd_extend(NdDev d, int lo) {
  const int C = d.ext_child[lo + blockIdx.y];
  const int P = d.parent[C];
  const int FC = d.F[C], oc = d.own[C], nb = FC - oc, FP = d.F[P], M = d.M;
  const double* src = d.fronts + d.front_off[C] + (long long)oc * FC + oc;
  double* dst = d.fronts + d.front_off[P];
  const int* em = d.emap + d.emap_off[C];
  const long long n = (long long)nb * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / nb), j = (int)(t - (long long)i * nb);
    const int gi = i / M, gj = j / M;
    const long long r = (long long)em[gi] * M + (i - gi * M), c = (long long)em[gj] * M + (j - gj * M);
    dst[r * FP + c] += src[(long long)i * FC + j];
  }
}

// batched blocked Gauss-Jordan over the own pivots of a level's fronts (pivot block at k0)
__global__ void __launch_bounds__(256) k_nd_pivot(NdDev d, int lo, int k0) {
  const int n = d.piv_node[lo + blockIdx.x];
  const int bk = min(kSweepB, d.own[n] - k0);
  if (bk <= 0) return;
  sweep_pivot_block(d.F[n], k0, bk, d.fronts + d.front_off[n], d.scr + d.scr_off[n]);
}

__global__ void __launch_bounds__(256) k_nd_panel(NdDev d, int lo, int k0) {
  const int* it = d.pan_item + 2LL * (lo + blockIdx.x);
  const int n = it[0];
  const int bk = min(kSweepB, d.own[n] - k0);
  if (bk <= 0) return;
  const long long F = d.F[n];
  double* P = d.scr + d.scr_off[n];
  double* Rp = P + kSweepB * kSweepB;
  sweep_panel_cols(F, k0, bk, d.fronts + d.front_off[n], P, Rp, Rp + kSweepB * F, it[1]);
}

__global__ void __launch_bounds__(256, 2) k_nd_update(NdDev d, int lo, int k0) {
  const int* it = d.tile_item + 3LL * (lo + blockIdx.x);
  const int n = it[0];
  const int bk = min(kSweepB, d.own[n] - k0);
  if (bk <= 0) return;
  const long long F = d.F[n];
  double* P = d.scr + d.scr_off[n];
  double* Rp = P + kSweepB * kSweepB;
  sweep_update_tile(F, k0, bk, d.fronts + d.front_off[n], P, Rp, Rp + kSweepB * F, it[1], it[2], -1, nullptr, 0);
}

// lower tiles -> upper tiles (the fronts are stored in full after their sweep)
__global__ void __launch_bounds__(256) k_nd_mirror(NdDev d, int lo) {
  const int* it = d.tile_item + 3LL * (lo + blockIdx.x);
  if (it[1] == it[2]) return;
  const int n = it[0];
  const long long F = d.F[n];
  double* A = d.fronts + d.front_off[n];
  for (int t = threadIdx.x; t < 64 * 64; t += blockDim.x) {
    const long long i = it[1] * 64LL + t / 64, j = it[2] * 64LL + t % 64;
    if (i < F && j < F) A[j * F + i] = A[i * F + j];
  }
}

// dot of a front row with the staged vector w (one warp; four independent partial sums,
// fixed order: every lane, then a xor butterfly)
__device__ __forceinline__ double nd_row_dot(const double* __restrict__ a, const double* w, int len, int lane) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int i = lane;
  for (; i + 96 < len; i += 128) {
    s0 = fma(a[i], w[i], s0);
    s1 = fma(a[i + 32], w[i + 32], s1);
    s2 = fma(a[i + 64], w[i + 64], s2);
    s3 = fma(a[i + 96], w[i + 96], s3);
  }
  for (; i < len; i += 32) s0 = fma(a[i], w[i], s0);
  double acc = (s0 + s1) + (s2 + s3);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

// up the tree, one level; blockIdx.x: (node, first boundary row).  The node's own part is
// its entries of v plus what its children left in its two incoming slots; each boundary
// row (incoming slots - L . own part) goes to the parent's incoming slot of this child.
__global__ void __launch_bounds__(kNdThreads) k_nd_fwd(NdDev d, const double* __restrict__ v, int lo,
                                                       const KrylovState* S) {
  if (S && S->done) return;
  extern __shared__ double nd_w[];
  const int* it = d.fwd_item + 2LL * (lo + blockIdx.x);
  const int n = it[0], r0 = it[1];
  const int F = d.F[n], own = d.own[n], M = d.M;
  const long long off = d.fv_off[n];
  const int* fg = d.fgroups + d.fg_off[n];
  for (int i = threadIdx.x; i < own; i += blockDim.x) {
    const int g = i / M;
    nd_w[i] = (v[(long long)fg[g] * M + (i - g * M)] + d.in0[off + i]) + d.in1[off + i];
  }
  __syncthreads();
  if (r0 == 0)
    for (int i = threadIdx.x; i < own; i += blockDim.x) d.fv[off + i] = nd_w[i];
  const int P = d.parent[n];
  if (P < 0) return;
  double* dst = (d.cslot[n] == 0 ? d.in0 : d.in1) + d.fv_off[P];
  const int* em = d.emap + d.emap_off[n];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double* A = d.fronts + d.front_off[n];
  for (int k = r0 + wid; k < min(r0 + kNdRows, F - own); k += kNdThreads / 32) {
    const double acc = nd_row_dot(A + (long long)(own + k) * F, nd_w, own, lane);
    if (lane == 0) {
      const int gk = k / M;
      dst[(long long)em[gk] * M + (k - gk * M)] = (d.in0[off + own + k] + d.in1[off + own + k]) - acc;
    }
  }
}

// down the tree, one level: own unknowns = -(front rows of own) . [own part; solution at
// the boundary groups]; blockIdx.x: (node, first own row)
__global__ void __launch_bounds__(kNdThreads) k_nd_bwd(NdDev d, double* __restrict__ mu, int lo,
                                                       const KrylovState* S) {
  if (S && S->done) return;
  extern __shared__ double nd_w[];
  const int* it = d.bwd_item + 2LL * (lo + blockIdx.x);
  const int n = it[0], r0 = it[1];
  const int F = d.F[n], own = d.own[n], M = d.M;
  const double* fvn = d.fv + d.fv_off[n];
  const int* fg = d.fgroups + d.fg_off[n];
  for (int i = threadIdx.x; i < F; i += blockDim.x) {
    if (i < own) {
      nd_w[i] = fvn[i];
    } else {
      const int g = i / M;
      nd_w[i] = mu[(long long)fg[g] * M + (i - g * M)];
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double* A = d.fronts + d.front_off[n];
  for (int r = r0 + wid; r < min(r0 + kNdRows, own); r += kNdThreads / 32) {
    const double acc = nd_row_dot(A + (long long)r * F, nd_w, F, lane);
    if (lane == 0) {
      const int g = r / M;
      mu[(long long)fg[g] * M + (r - g * M)] = -acc;
    }
  }
}

}  // namespace pyto

namespace pyto {

// device block-sparse coarse matrix of a bound plan (int64 fixed-point bits during assembly)
double* nd_matrix(const pyto_coarse_nd* P) { return P->dev ? (double*)(P->dev + P->o_E) : nullptr; }
long long nd_matrix_bytes(const pyto_coarse_nd* P) { return P->nslots * P->M * P->M * (long long)sizeof(double); }

// Numeric factorisation of the assembled coarse matrix (fixed point in nd_matrix).
int nd_factor(const pyto_coarse_nd* P, const int32_t* nptr, const int32_t* nlist, const int* gexp, double shift,
              int relative, cudaStream_t st) {
  if (!P->dev) return PYTO_ERR_ARG;
  const NdDev d = nd_dev(P);
  static PerDevice attr;
  if (attr.needed()) {
    PYTO_CUDA(cudaFuncSetAttribute(k_nd_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(kNdMaxFront * sizeof(double))));
    PYTO_CUDA(cudaFuncSetAttribute(k_nd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(kNdMaxFront * sizeof(double))));
    attr.done();
  }
  static PerDevice attr_u;
  if (attr_u.needed()) {
    PYTO_CUDA(cudaFuncSetAttribute(k_nd_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSweepTileSmem));
    attr_u.done();
  }
  k_nd_from_fixed<<<P->ng, 128, 0, st>>>(d, nptr, nlist, gexp);
  k_nd_diag_sum<<<kNdDiagBlocks, 256, 0, st>>>(d);
  k_nd_diag_apply<<<kNdDiagBlocks, 256, 0, st>>>(d, shift, relative);
  PYTO_COUNT(3);
  for (int l = P->depth; l >= 0; --l) {
    const long long f0 = P->lvl_front_lo[l], f1 = P->lvl_front_hi[l];
    PYTO_CUDA(cudaMemsetAsync(d.fronts + f0, 0, (size_t)(f1 - f0) * sizeof(double), st));
    const int p0 = P->push_lo[l], p1 = P->push_lo[l + 1];
    if (p1 > p0) {
      const long long work = (long long)(p1 - p0) * P->M * P->M;
      k_nd_push<<<(int)std::min<long long>((work + 255) / 256, 16 * kNumSMs), 256, 0, st>>>(d, p0, p1);
      PYTO_COUNT(1);
    }
    for (int pass = 0; pass < 2; ++pass) {
      const int e0 = P->ext_lo[2 * l + pass], e1 = P->ext_lo[2 * l + pass + 1];
      if (e1 <= e0) continue;
      long long mx = 0;
      for (int e = e0; e < e1; ++e) {
        const int C = P->ext_child[e];
        const long long nb = P->F[C] - P->own[C];
        mx = std::max(mx, nb * nb);
      }
      const int bx = (int)std::max<long long>(1, std::min<long long>((mx + 255) / 256, 64));
      k_nd_extend<<<dim3(bx, e1 - e0), 256, 0, st>>>(d, e0);
      PYTO_COUNT(1);
    }
    const int pv0 = P->piv_lo[l], pv1 = P->piv_lo[l + 1];
    const int pa0 = P->pan_lo[l], pa1 = P->pan_lo[l + 1];
    const int t0 = P->tile_lo[l], t1 = P->tile_lo[l + 1];
    for (int k0 = 0; k0 < P->lvl_maxown[l]; k0 += kSweepB) {
      k_nd_pivot<<<pv1 - pv0, 256, 0, st>>>(d, pv0, k0);
      k_nd_panel<<<pa1 - pa0, 256, 0, st>>>(d, pa0, k0);
      k_nd_update<<<t1 - t0, 256, kSweepTileSmem, st>>>(d, t0, k0);
      PYTO_COUNT(3);
    }
    k_nd_mirror<<<t1 - t0, 256, 0, st>>>(d, t0);
    PYTO_COUNT(1);
  }
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

// mu = E^-1 v with the factorisation of nd_factor (S: skip once the solver's state is done)
int nd_solve(const pyto_coarse_nd* P, const double* v, double* mu, const KrylovState* S, cudaStream_t st) {
  if (!P->dev) return PYTO_ERR_ARG;
  const NdDev d = nd_dev(P);
  const size_t shm = (size_t)P->maxF * sizeof(double);
  PYTO_CUDA(cudaMemsetAsync(d.in0, 0, 2 * (size_t)P->fv_doubles * sizeof(double), st));
  for (int l = P->depth; l >= 0; --l) {
    const int a = P->fwd_lo[l], b = P->fwd_lo[l + 1];
    if (b > a) {
      k_nd_fwd<<<b - a, kNdThreads, shm, st>>>(d, v, a, S);
      PYTO_COUNT(1);
    }
  }
  for (int l = 0; l <= P->depth; ++l) {
    const int a = P->bwd_lo[l], b = P->bwd_lo[l + 1];
    if (b > a) {
      k_nd_bwd<<<b - a, kNdThreads, shm, st>>>(d, mu, a, S);
      PYTO_COUNT(1);
    }
  }
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

}  // namespace pyto

using namespace pyto;

extern "C" pyto_coarse_nd_t* pyto_coarse_nd_plan(int32_t gx, int32_t gy, int32_t gz, int32_t modes, int32_t leaf,
                                                 const int32_t* nbr_ptr, const int32_t* nbr_list) {
  if (gx < 1 || gy < 1 || gz < 1 || (modes != 3 && modes != 6) || leaf < 1 || !nbr_ptr || !nbr_list ||
      (long long)gx * gy * gz > (1LL << 24)) {
    record_error(cudaErrorInvalidValue, "pyto_coarse_nd_plan: invalid grid, modes, leaf or lists", __FILE__,
                 __LINE__);
    return nullptr;
  }
  pyto_coarse_nd* P = new pyto_coarse_nd();
  P->gx = gx;
  P->gy = gy;
  P->gz = gz;
  P->M = modes;
  P->leaf = leaf;
  P->ng = gx * gy * gz;
  const char* err = nd_build(P, nbr_ptr, nbr_list);
  if (err) {
    record_error(cudaErrorInvalidValue, err, __FILE__, __LINE__);
    delete P;
    return nullptr;
  }
  nd_items(P);
  return P;
}

extern "C" size_t pyto_coarse_nd_bytes(const pyto_coarse_nd_t* P, double* info) {
  if (!P) return 0;
  if (info) {
    info[0] = (double)P->node.size();
    info[1] = (double)P->depth;
    info[2] = (double)P->maxF;
    info[3] = P->flops;
    info[4] = P->solve_bytes;
  }
  return P->bytes;
}

extern "C" int pyto_coarse_nd_bind(pyto_coarse_nd_t* P, void* dev_buf, size_t bytes, void* stream) {
  if (!P || !dev_buf || bytes < P->bytes || ((uintptr_t)dev_buf & 255)) return PYTO_ERR_ARG;
  const cudaStream_t st = (cudaStream_t)stream;
  P->dev = (char*)dev_buf;
  PYTO_CUDA(cudaMemcpyAsync(P->dev + P->o_i64, P->i64.data(), P->i64.size() * sizeof(long long),
                            cudaMemcpyHostToDevice, st));
  PYTO_CUDA(cudaMemcpyAsync(P->dev + P->o_i32, P->i32.data(), P->i32.size() * sizeof(int),
                            cudaMemcpyHostToDevice, st));
  return PYTO_OK;
}

extern "C" int pyto_coarse_nd_solve(const pyto_coarse_nd_t* P, const double* v, double* mu, void* stream) {
  if (!P || !v || !mu) return PYTO_ERR_ARG;
  return nd_solve(P, v, mu, nullptr, (cudaStream_t)stream);
}

extern "C" void pyto_coarse_nd_free(pyto_coarse_nd_t* P) { delete P; }
