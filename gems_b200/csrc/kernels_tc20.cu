// kernels_tc20.cu -- 20-state mixed-precision traversal on the 5th-generation tensor cores.
//
// Node update per category c (real space, FP32 storage):
//     out[p][c][:] = (P_c(t_L) . L[p][c][:]) (*) (P_c(t_R) . R[p][c][:])
// For a tile of 128 patterns each child product is a GEMM  D[128 x 32] = A[128 x 24] . B^T,
// A = the child partial rows of category c (K = 20 states padded to 24), B = P_c (20 x 20
// padded to 32 x 24, zero padding).  FP32 accuracy comes from split TF32 ("3xTF32"):
//     A.B ~= A_hi.B_hi + A_hi.B_lo + A_lo.B_hi,  x_hi = rna_tf32(x), x_lo = rna_tf32(x - x_hi)
// issued as tcgen05.mma kind::tf32 (M=128, N=32, K=8) by one thread, accumulators in TMEM
// (2 sides x C categories x 32 columns), read back with tcgen05.ld for the epilogue (product,
// 2^64 rescaling, FP32 store).
//
// Operands in shared memory use the no-swizzle K-major core-matrix layout: 16-byte chunks of
// 4 states x 128 rows, LBO = 2048 B between K chunks, SBO = 128 B between 8-row groups.  The
// 20-state mixed partials are stored in global memory in exactly this layout (tile-major,
// see mix_off), so a child's tile is one contiguous 5C x 2 KB block brought by one
// cp.async.bulk, and the output rows go out as coalesced 16-byte stores (a warp writes 512
// contiguous bytes per chunk).  The split B images are precomputed per op in the same layout.
//
// Pipeline per op (one CTA per SM, 8 warps; warps w and w+4 share TMEM lane quadrant w%4 and
// each handles two of the four categories of a row):
//   wait(copies of this op) -> split the loaded tiles into hi/lo -> MMAs -> wait(MMA)
//   -> epilogue part 1 (TMEM / tip-table reads, products) -> barrier
//   -> issue the next op's bulk copies (operand buffers and tables are free again)
//   -> epilogue part 2 (rescaling, split, stores); when the next op consumes this op's output,
//      the split row also goes into the next op's operand buffer (no round trip through
//      global memory), and its counters stay in registers
//   -> loads of the next op's tip bytes and counters, issued a whole op ahead of their use.
// Tip children need no product: the message is a row of the op's tip table, which the same
// bulk copy brings into the side's table region.  The op descriptors are read two ops ahead.
//
// Every mbarrier wait is bounded by a clock budget; on expiry the CTA records
// GEMS_ERR_TIMEOUT, stops issuing work, waits (bounded) for what it has in flight, frees its
// TMEM and returns.
#include <cmath>
#include <cstring>
#include <string>

#include "gems_internal.cuh"
#include "tc_common.cuh"

namespace gems {

namespace {

using namespace tc;

constexpr int kN = 20;                          // states
constexpr int kNP = 32;                         // MMA N (padded states)
constexpr int kKP = 24;                         // padded K (3 x 8)
constexpr int kTile = 128;                      // patterns per CTA = MMA M
constexpr int kThreadsTc = 256;                 // 2 threads per pattern row
constexpr int kRowChunks = 20;                  // 16-byte chunks per row (4 categories x 5)
constexpr int kAChunk = kTile * 16;             // one chunk of an A tile (128 rows x 16 B)
constexpr int kABytes = (kRowChunks + 1) * kAChunk;  // + a zero chunk for the last category
constexpr int kBImg = (kKP / 4) * kNP * 16;     // 6 chunks x 32 rows x 16 B = 3072
// TMEM columns: accumulators D[side][category] (32 columns each) in [0, 256), the hi part of
// the operand rows A_hi[side][category] (K = 24 columns each) in [256, 448)
constexpr int kTmemCols = 512;
constexpr int kAhiCol = 256;
// tip tables: one row of C x 20 floats per state code, padded by 4 floats so that rows of
// consecutive state codes start in different shared-memory bank groups
__host__ __device__ constexpr int tip_row_floats(int C) { return C * kN + 4; }

// instruction descriptor: D f32, A/B tf32, both K-major, N = 32, M = 128
constexpr uint32_t kIdesc = tc::idesc_tf32(kNP);
__device__ __forceinline__ void mma_tf32(uint32_t dtm, uint64_t a, uint64_t b, uint32_t acc) {
  tc::mma_ss(dtm, a, b, kIdesc, acc);
}
__device__ __forceinline__ void mma_tf32_ta(uint32_t dtm, uint32_t atm, uint64_t b, uint32_t acc) {
  tc::mma_ts(dtm, atm, b, kIdesc, acc);
}
__device__ __forceinline__ void tc_fence_after() { tc::fence_after(); }
__device__ __forceinline__ void tc_fence_before() { tc::fence_before(); }

// the 20 state columns of one accumulator (columns 20..31 are padding) of this thread's lane;
// the registers are valid after tmem_ld_wait on them
__device__ __forceinline__ void tmem_ld20(uint32_t taddr, uint32_t (&r)[20]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19])
               : "r"(taddr + 16));
}
// waits for this thread's TMEM loads; the register operands make every later use of the
// loaded values depend on the wait
__device__ __forceinline__ void tmem_ld_wait(uint32_t (&r)[20]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                 "+r"(r[18]), "+r"(r[19])
               :
               : "memory");
}
// the hi part of a row of one category (20 states and 4 zero columns of K padding) into its
// 24 TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_st_row(uint32_t taddr, const float4 (&h)[5]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};" ::"r"(taddr),
      "f"(h[0].x), "f"(h[0].y), "f"(h[0].z), "f"(h[0].w), "f"(h[1].x), "f"(h[1].y), "f"(h[1].z),
      "f"(h[1].w), "f"(h[2].x), "f"(h[2].y), "f"(h[2].z), "f"(h[2].w), "f"(h[3].x), "f"(h[3].y),
      "f"(h[3].z), "f"(h[3].w)
      : "memory");
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %5, %5, %5};" ::"r"(
          taddr + 16),
      "f"(h[4].x), "f"(h[4].y), "f"(h[4].z), "f"(h[4].w), "f"(0.f)
      : "memory");
}
// ---------------------------------------------------------------------------------------
// Per-op tables for the tensor-core path (floats, per op):
//   B images [2 sides][C][hi, lo][6 chunks][32 rows][4]   (row n = target state x, K = y)
//   tip tables [2 sides][U1][C][20]
// ---------------------------------------------------------------------------------------
__global__ void k_prep_ops_tc(DevCtx c, const DevOp *ops, float *tab, size_t stride_f) {
  extern __shared__ double sm[];
  double *ex = sm;                                        // [C][n]
  float *Pm = reinterpret_cast<float *>(ex + c.C * kN);  // [C][n][n]
  const int k = blockIdx.x, side = blockIdx.y;
  const DevOp op = ops[k];
  const int kind = side ? op.r_kind : op.l_kind;
  const double len = side ? op.r_len : op.l_len;
  const int C = c.C, n = kN;
  for (int idx = threadIdx.x; idx < C * n; idx += blockDim.x) {
    const int cc = idx / n, i = idx - cc * n;
    ex[idx] = exp(c.eval[i] * (c.rates[cc] * len));
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < C * n * n; idx += blockDim.x) {
    const int cc = idx / (n * n), r = idx - cc * n * n, x = r / n, y = r - x * n;
    double acc = 0.0;
    for (int i = 0; i < n; i++) acc = fma(c.evec[x * n + i] * ex[cc * n + i], c.inv_evec[i * n + y], acc);
    Pm[idx] = (float)fmax(acc, 0.0);
  }
  __syncthreads();
  float *img = tab + (size_t)k * stride_f + (size_t)side * C * 2 * (kBImg / 4);
  for (int idx = threadIdx.x; idx < C * (kBImg / 4); idx += blockDim.x) {
    const int cc = idx / (kBImg / 4), r = idx - cc * (kBImg / 4);
    const int chunk = r / (kNP * 4), rr = r - chunk * kNP * 4, row = rr / 4, e = rr - row * 4;
    const int x = row, y = chunk * 4 + e;
    const float v = (x < n && y < n) ? Pm[(cc * n + x) * n + y] : 0.f;
    const float hi = tf32_rna(v);
    const float lo = tf32_rna(v - hi);
    img[(size_t)cc * 2 * (kBImg / 4) + r] = hi;
    img[(size_t)cc * 2 * (kBImg / 4) + (kBImg / 4) + r] = lo;
  }
  if (kind != GEMS_CHILD_TIP) return;
  const int trow = tip_row_floats(C);
  float *leaf = tab + (size_t)k * stride_f + (size_t)2 * C * 2 * (kBImg / 4) +
                (size_t)side * (c.unknown + 1) * trow;
  for (int idx = threadIdx.x; idx < (c.unknown + 1) * trow; idx += blockDim.x) {
    const int s = idx / trow, r = idx - s * trow, cc = r / n, x = r - cc * n;
    if (cc >= C) {  // row padding
      leaf[idx] = 0.f;
      continue;
    }
    const double *ind = c.tip_real + (size_t)s * n;
    float acc = 0.f;
    for (int y = 0; y < n; y++) acc = fmaf(Pm[(cc * n + x) * n + y], (float)ind[y], acc);
    leaf[idx] = acc;
  }
}

// MMAs of one side: for each category, D[128 x 32] = A_hi.B_hi + A_hi.B_lo + A_lo.B_hi over
// three K steps (A_hi in TMEM, A_lo and the B images in shared memory)
__device__ __forceinline__ void issue_side_mmas(int s, int C, uint32_t tmem, uint64_t dB0,
                                                uint64_t dL0s) {
#pragma unroll
  for (int cc = 0; cc < 4; cc++) {
    if (cc >= C) break;
    const uint32_t dtm = tmem + (uint32_t)((s * C + cc) * kNP);
    const uint32_t atm = tmem + (uint32_t)(kAhiCol + (s * 4 + cc) * kKP);
    const uint64_t bh = dB0 + (uint64_t)((((s * C + cc) * 2) * kBImg) >> 4);
    const uint64_t bl = bh + (uint64_t)(kBImg >> 4);
#pragma unroll
    for (int ks = 0; ks < kKP / 8; ks++) {
      const uint64_t ko = (uint64_t)(((cc * 5 + 2 * ks) * kAChunk) >> 4);
      const uint64_t kb = (uint64_t)((2 * ks * kNP * 16) >> 4);
      mma_tf32_ta(dtm, atm + 8 * ks, bh + kb, ks > 0 ? 1u : 0u);
      mma_tf32_ta(dtm, atm + 8 * ks, bl + kb, 1u);
      mma_tf32(dtm, dL0s + ko, bh + kb, 1u);
    }
  }
}

struct TcShared {
  uint64_t bar_tile;  // operand tiles of the next op (landing buffers)
  uint64_t bar_tab;   // tables of the next op (B images / tip tables)
  uint64_t bar_mma;
  uint32_t tmem_base;
  float rowmax[2][kTile];
};

// which children of op `nx` the TMA must bring (the one equal to `fwd_slot` is forwarded)
__device__ __forceinline__ int tma_mask(const DevOp &nx, int fwd_slot) {
  int m = 0;
  if (nx.l_kind == GEMS_CHILD_PARTIAL && nx.l_id != fwd_slot) m |= 1;
  if (nx.r_kind == GEMS_CHILD_PARTIAL && nx.r_id != fwd_slot) m |= 2;
  return m;
}

// bytes of a side's op table: split B images (internal child) or its tip table (tip child)
__device__ __forceinline__ uint32_t side_table_bytes(bool internal, int C, int unknown) {
  return internal ? (uint32_t)C * 2 * kBImg : (uint32_t)(unknown + 1) * tip_row_floats(C) * 4;
}

// Copies for op `nx`, issued by one thread.  issue_tiles: the tiles of the children in `mask`
// (one contiguous block of the tile-major slot each) into the landing buffers; it runs as soon
// as the current op no longer reads those.  issue_tables: for each side its op table (B
// images of an internal child, tip table of a tip child) into that side's region, once the
// current op's MMAs and table reads are done.  Each completes its barrier once per op.
__device__ __forceinline__ void issue_tiles(const DevCtx &c, const DevOp &nx, int mask,
                                            uint32_t sA0, uint32_t sA1, int tile, uint32_t bar) {
  const int C = c.C;
  const uint32_t tb = 5 * C * kAChunk;
  mbar_expect_tx(bar, (uint32_t)__popc(mask) * tb);
  for (int s = 0; s < 2; s++) {
    if (!(mask & (1 << s))) continue;
    const float *src = static_cast<const float *>(c.partials) +
                       (size_t)(s ? nx.r_id : nx.l_id) * c.slot_elems + (size_t)tile * (tb / 4);
    bulk_g2s(s ? sA1 : sA0, src, tb, bar);
  }
}
__device__ __forceinline__ void issue_tables(const DevCtx &c, const DevOp &nx, const float *tk,
                                             unsigned char *Bbase, uint32_t bar) {
  const int C = c.C;
  const size_t imgf = kBImg / 4;
  uint32_t bytes = 0;
  for (int s = 0; s < 2; s++)
    bytes += side_table_bytes((s ? nx.r_kind : nx.l_kind) == GEMS_CHILD_PARTIAL, C, c.unknown);
  mbar_expect_tx(bar, bytes);
  for (int s = 0; s < 2; s++) {
    const bool in = (s ? nx.r_kind : nx.l_kind) == GEMS_CHILD_PARTIAL;
    const float *src = in ? tk + (size_t)s * C * 2 * imgf
                          : tk + (size_t)2 * C * 2 * imgf +
                                (size_t)s * (c.unknown + 1) * tip_row_floats(C);
    bulk_g2s(sptr(Bbase + (size_t)s * C * 2 * kBImg), src, side_table_bytes(in, C, c.unknown),
             bar);
  }
}

// what a thread loads for an op before its products are ready: tip bytes and the counters of
// internal children (a forwarded child's counters come from the previous op's registers).
// Plain named scalars, so that everything stays in registers and the loads stay in flight
// until their first use a whole op later.
struct SideIn {
  int st;        // tip state code (tip child)
  int sc0, sc1;  // counters of this thread's two categories (internal child)
};
struct OpIn {
  SideIn L, R;
};

template <bool SAFE>
__device__ __forceinline__ SideIn load_side(const DevCtx &c, int kind, int id, bool fwd,
                                            int fs0, int fs1, long p, int half, bool act) {
  SideIn r{0, 0, 0};
  if (!act) return r;
  if (kind == GEMS_CHILD_TIP) {
    r.st = c.tips[(size_t)id * c.P + p];
  } else if (fwd) {
    r.sc0 = fs0;
    r.sc1 = fs1;
  } else {
    const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
    if (SAFE) {
      if (2 * half < c.C) r.sc0 = sc[(size_t)p * c.C + 2 * half];
      if (2 * half + 1 < c.C) r.sc1 = sc[(size_t)p * c.C + 2 * half + 1];
    } else {
      r.sc0 = r.sc1 = sc[p];
    }
  }
  return r;
}

template <bool SAFE>
__device__ __forceinline__ void load_op_inputs(const DevCtx &c, const DevOp &op, int fwd_side,
                                               int fs0, int fs1, long p, int half, bool act,
                                               OpIn &in) {
  in.L = load_side<SAFE>(c, op.l_kind, op.l_id, fwd_side == 0, fs0, fs1, p, half, act);
  in.R = load_side<SAFE>(c, op.r_kind, op.r_id, fwd_side == 1, fs0, fs1, p, half, act);
}

template <bool SAFE>
__global__ void __launch_bounds__(kThreadsTc, 1)
    k_traverse_tc20(DevCtx c, const DevOp *__restrict__ ops, int nops,
                    const float *__restrict__ tab, size_t stride_f, int *flag, int tile0) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = smem_raw;
  float *A[2], *Alo[2];
  A[0] = reinterpret_cast<float *>(base);
  A[1] = reinterpret_cast<float *>(base + kABytes);
  Alo[0] = reinterpret_cast<float *>(base + 2 * kABytes);
  Alo[1] = reinterpret_cast<float *>(base + 3 * kABytes);
  const int C = c.C;
  unsigned char *Bbase = base + 4 * kABytes;
  TcShared *ctl = reinterpret_cast<TcShared *>(Bbase + (size_t)2 * C * 2 * kBImg);

  const int t = threadIdx.x, warp = t >> 5;
  const int row = ((warp & 3) << 5) | (t & 31);  // TMEM lane = pattern row of the tile
  const int half = warp >> 2;                    // categories {2h, 2h+1}
  const int tile = tile0 + blockIdx.x;  // pattern tile of this CTA
  const int p0 = tile * kTile;
  const long p = p0 + row;
  const bool act = p < c.P;
  const uint32_t bar_tile = sptr(&ctl->bar_tile), bar_tab = sptr(&ctl->bar_tab);
  const uint32_t bar_mma = sptr(&ctl->bar_mma);

  if (t == 0) {
    mbar_init(bar_tile, 1);
    mbar_init(bar_tab, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // chunks 5C..20 of every operand buffer stay zero for the whole kernel (the K padding of
  // the last category, and categories the session does not have): nothing writes them again
  for (int i = t; i < (kRowChunks + 1 - 5 * C) * kTile; i += kThreadsTc) {
    const int off = 5 * C * kTile + i;
    for (int s = 0; s < 2; s++) {
      reinterpret_cast<float4 *>(A[s])[off] = make_float4(0.f, 0.f, 0.f, 0.f);
      reinterpret_cast<float4 *>(Alo[s])[off] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     sptr(&ctl->tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = ctl->tmem_base;
  const uint32_t lane_off = (uint32_t)((warp & 3) * 32) << 16;
  // MMA descriptors of the first K step of category 0; the others are these plus offsets
  // (the 14-bit address field counts 16-byte units and the whole buffer is < 256 KiB)
  const uint64_t dL0[2] = {sdesc(sptr(Alo[0]), kAChunk, 128), sdesc(sptr(Alo[1]), kAChunk, 128)};
  const uint64_t dB0 = sdesc(sptr(Bbase), kNP * 16, 128);
  uint32_t ph_tile = 0, ph_tab = 0, ph_mma = 0;
  bool ok = true, tile_pending = false, tab_pending = false, mma_pending = false;
  const uint32_t sA0 = sptr(A[0]), sA1 = sptr(A[1]);
  const bool inv0 = act ? c.invar[p] == 0.0 : false;

  DevOp cur = ops[0];
  DevOp nxt = nops > 1 ? ops[1] : cur;
  int cur_mask = tma_mask(cur, -1);
  if (warp == 0 && elect_one()) {
    issue_tiles(c, cur, cur_mask, sA0, sA1, tile, bar_tile);
    issue_tables(c, cur, tab, Bbase, bar_tab);
  }
  tile_pending = tab_pending = true;
  OpIn in;
  load_op_inputs<SAFE>(c, cur, -1, 0, 0, p, half, act, in);

  for (int k = 0; k < nops && ok; k++) {
    const bool inL = cur.l_kind == GEMS_CHILD_PARTIAL, inR = cur.r_kind == GEMS_CHILD_PARTIAL;
    const bool has_next = k + 1 < nops;
    // the op after next: its descriptor is needed one op from now
    const DevOp nxt2 = (k + 2 < nops) ? ops[k + 2] : nxt;
    if (__syncthreads_or(!mbar_wait(bar_tile, ph_tile) || !mbar_wait(bar_tab, ph_tab))) {
      ok = false;
      if (t == 0) atomicExch(flag, GEMS_ERR_TIMEOUT);
      break;
    }
    tile_pending = tab_pending = false;
    ph_tile ^= 1;
    ph_tab ^= 1;
    // the next op's children: the one this op produces is forwarded, the others are copied
    int nxt_mask = 0, nxt_fwd = -1;
    if (has_next) {
      nxt_mask = tma_mask(nxt, cur.dst_slot);
      if (nxt.l_kind == GEMS_CHILD_PARTIAL && nxt.l_id == cur.dst_slot) nxt_fwd = 0;
      if (nxt.r_kind == GEMS_CHILD_PARTIAL && nxt.r_id == cur.dst_slot) nxt_fwd = 1;
    }
    if (inL || inR) {
      // The forwarded child's operands are already in place (written by the previous op's
      // epilogue): its MMAs go first and run while the loaded child is split.
      const int fwd_side = (inL && !(cur_mask & 1)) ? 0 : ((inR && !(cur_mask & 2)) ? 1 : -1);
      if (warp == 0 && elect_one()) {
        if (fwd_side >= 0) issue_side_mmas(fwd_side, C, tmem, dB0, fwd_side ? dL0[1] : dL0[0]);
        if (cur_mask == 0) {
          mma_commit(bar_mma);
          // nothing to split: the landing buffers are free for the next op's tiles
          if (has_next) issue_tiles(c, nxt, nxt_mask, sA0, sA1, tile, bar_tile);
        }
      }
      if (cur_mask) {
        // split the tiles the bulk copies brought: hi -> the side's TMEM operand columns,
        // lo -> Alo (shared memory)
        for (int s = 0; s < 2; s++) {
          if (!(cur_mask & (1 << s))) continue;
          const float4 *a4 = reinterpret_cast<const float4 *>(s ? A[1] : A[0]);
          float4 *l4 = reinterpret_cast<float4 *>(s ? Alo[1] : Alo[0]);
#pragma unroll
          for (int j = 0; j < 2; j++) {
            const int cc = 2 * half + j;
            if (cc >= C) continue;
            float4 h[5];
#pragma unroll
            for (int i = 0; i < 5; i++) {
              float4 l;
              split4(a4[(cc * 5 + i) * kTile + row], h[i], l);
              l4[(cc * 5 + i) * kTile + row] = l;
            }
            tmem_st_row(tmem + lane_off + (uint32_t)(kAhiCol + (s * 4 + cc) * kKP), h);
          }
        }
        tmem_st_wait();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // the same elected lane (the lowest) commits every MMA of this op
        if (warp == 0 && elect_one()) {
          if (cur_mask & 1) issue_side_mmas(0, C, tmem, dB0, dL0[0]);
          if (cur_mask & 2) issue_side_mmas(1, C, tmem, dB0, dL0[1]);
          mma_commit(bar_mma);
          // the split has read the landing buffers: the next op's tiles can come in
          if (has_next) issue_tiles(c, nxt, nxt_mask, sA0, sA1, tile, bar_tile);
        }
      }
      tile_pending = has_next;
      mma_pending = true;
      if (__syncthreads_or(!mbar_wait(bar_mma, ph_mma))) {
        ok = false;
        if (t == 0) atomicExch(flag, GEMS_ERR_TIMEOUT);
        break;
      }
      mma_pending = false;
      ph_mma ^= 1;
      tc_fence_after();
    } else {
      if (has_next && warp == 0 && elect_one())
        issue_tiles(c, nxt, nxt_mask, sA0, sA1, tile, bar_tile);
      tile_pending = has_next;
    }
    // ---- epilogue, part 1: messages and products into registers (the tip tables of this op
    // are in the side regions of shared memory; read them before the next copies land)
    float out[2][kN];
    float mx[2] = {0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int cc = 2 * half + j;
      if (cc >= C) {
#pragma unroll
        for (int x = 0; x < kN; x++) out[j][x] = 0.f;
        continue;
      }
      float m[2][kN];
      // both sides' accumulator loads in flight together, then the wait
      uint32_t r[2][20];
#pragma unroll
      for (int s = 0; s < 2; s++)
        if (s ? inR : inL) tmem_ld20(tmem + lane_off + (uint32_t)((s * C + cc) * kNP), r[s]);
#pragma unroll
      for (int s = 0; s < 2; s++) {
        if (s ? inR : inL) {
          tmem_ld_wait(r[s]);
#pragma unroll
          for (int x = 0; x < kN; x++) m[s][x] = __uint_as_float(r[s][x]);
        } else {
          const float4 *lt = reinterpret_cast<const float4 *>(
              Bbase + (size_t)s * C * 2 * kBImg +
              ((size_t)(s ? in.R.st : in.L.st) * tip_row_floats(C) + (size_t)cc * kN) * 4);
#pragma unroll
          for (int i = 0; i < kN / 4; i++) {
            const float4 v = lt[i];
            m[s][4 * i] = v.x;
            m[s][4 * i + 1] = v.y;
            m[s][4 * i + 2] = v.z;
            m[s][4 * i + 3] = v.w;
          }
        }
      }
#pragma unroll
      for (int x = 0; x < kN; x++) {
        const float v = fmaxf(m[0][x], 0.f) * fmaxf(m[1][x], 0.f);
        out[j][x] = v;
        mx[j] = fmaxf(mx[j], v);
      }
    }
    const bool tiptip = !inL && !inR;
    if (!SAFE) ctl->rowmax[half][row] = fmaxf(mx[0], mx[1]);  // the row max spans both halves
    tc_fence_before();
    __syncthreads();  // operand buffers, tables and TMEM of this op are no longer read
    tc_fence_after();
    // the tables of this op are no longer read: the next op's tables come in under the rest
    // of this epilogue
    if (has_next) {
      if (warp == 0 && elect_one())
        issue_tables(c, nxt, tab + (size_t)(k + 1) * stride_f, Bbase, bar_tab);
      tab_pending = true;
    }
    // ---- epilogue, part 2: rescaling, counters, stores, forwarding
    float f[2] = {1.f, 1.f};
    int s_out[2];
    if (SAFE) {
      s_out[0] = in.L.sc0 + in.R.sc0;
      s_out[1] = in.L.sc1 + in.R.sc1;
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int cc = 2 * half + j;
        if (cc < C && !tiptip && mx[j] < kScaleThrF && inv0) {
          f[j] = 18446744073709551616.0f;  // 2^64
          s_out[j] += 1;
        }
      }
    } else {
      const float m = fmaxf(ctl->rowmax[0][row], ctl->rowmax[1][row]);
      s_out[0] = in.L.sc0 + in.R.sc0;
      if (!tiptip && m < kScaleThrF && inv0) {
        f[0] = f[1] = 18446744073709551616.0f;  // 2^64
        s_out[0] += 1;
      }
      s_out[1] = s_out[0];
    }
    // The output rows are stored as computed, straight into the tile-major slot: for one chunk
    // a warp writes 32 consecutive rows, 512 contiguous bytes.  When the next op consumes this
    // output, the split of the same values goes into its operand buffers: exactly what a later
    // copy of the stored rows splits into, so a forwarded and a copied child give the same bits.
    float *dtile = static_cast<float *>(c.partials) + (size_t)cur.dst_slot * c.slot_elems +
                   (size_t)tile * (5 * C * kAChunk / 4);
    float *fl = nxt_fwd == 1 ? Alo[1] : Alo[0];
    {
      uint16_t *sd = c.scale + (size_t)cur.dst_slot * c.slot_scale;
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int cc = 2 * half + j;
        if (cc >= C) continue;
        float4 h[5];
#pragma unroll
        for (int i = 0; i < kN / 4; i++) {
          const float4 v = make_float4(out[j][4 * i] * f[j], out[j][4 * i + 1] * f[j],
                                       out[j][4 * i + 2] * f[j], out[j][4 * i + 3] * f[j]);
          const int idx = (cc * 5 + i) * kTile + row;
          reinterpret_cast<float4 *>(dtile)[idx] = v;
          if (nxt_fwd >= 0) {
            float4 l;
            split4(v, h[i], l);
            reinterpret_cast<float4 *>(fl)[idx] = l;
          }
        }
        if (nxt_fwd >= 0)
          tmem_st_row(tmem + lane_off + (uint32_t)(kAhiCol + (nxt_fwd * 4 + cc) * kKP), h);
        if (SAFE && act) sd[(size_t)p * C + cc] = (uint16_t)s_out[j];
      }
      if (!SAFE && act && half == 0) sd[p] = (uint16_t)s_out[0];
    }
    // next op's tip bytes and counters (a forwarded child's counters are this op's s_out)
    if (has_next) load_op_inputs<SAFE>(c, nxt, nxt_fwd, s_out[0], s_out[1], p, half, act, in);
    // later ops bulk-copy this output from global memory, and the next MMA reads the forwarded
    // operands: both through the async proxy
    if (nxt_fwd >= 0) tmem_st_wait();
    asm volatile("fence.proxy.async.global;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    cur = nxt;
    nxt = nxt2;
    cur_mask = nxt_mask;
  }
  if (!ok && t == 0) {
    if (tile_pending) mbar_wait(bar_tile, ph_tile);
    if (tab_pending) mbar_wait(bar_tab, ph_tab);
    if (mma_pending) mbar_wait(bar_mma, ph_mma);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
}


// ---------------------------------------------------------------------------------------
// Two CTAs per SM, in half-steps (GEMS_OPT_TC20_HALVES).  A CTA of 128 threads (one per
// pattern row) runs its tile's op list two categories at a time: per half-step a side's operand
// tile is 10 chunks (20 KB), its B images 12 KB, and the CTA needs 113 KB of shared memory and
// 256 TMEM columns, so two CTAs share an SM and one's copy, MMA and barrier waits are covered by
// the other's work.  No child is forwarded: every internal child is copied from the slot
// (usually from L2), the copy of the op that just wrote it issued after its stores.  NORM
// scaling spans every category of a row: the first half-step's rows are stored as computed and,
// when the row needs scaling (rare), re-read and scaled after the last half-step; SAFE scaling
// is per category.  Values are those of the one-CTA kernel bit for bit (same products, same
// split, same summation order); only the schedule differs.
// ---------------------------------------------------------------------------------------
constexpr int kThreadsH = kTile;                       // one thread per pattern row
constexpr int kHalfChunks = 10;                        // chunks of two categories
constexpr int kLandH = (kHalfChunks + 1) * kAChunk;    // + a chunk that stays zero: 22 KB
constexpr int kBSideH = 2 * 2 * kBImg;                 // two categories' hi and lo: 12 KB
constexpr int kTmemColsH = 256;
constexpr int kAhiColH = 128;                          // A_hi[side][j] at 128 + (2 side + j) 24

struct TcSharedH {
  uint64_t bar_land, bar_tab, bar_mma;
  uint32_t tmem_base;
};
size_t tc_smem_h() { return 4 * (size_t)kLandH + 2 * (size_t)kBSideH + sizeof(TcSharedH) + 64; }

// categories of half-step h (2 or, for the last half of an odd C, 1)
__device__ __forceinline__ int half_cats(int C, int h) { return min(2, C - 2 * h); }

// the child tiles of half-step h of op `o` (all but `late`) into the landing buffers; the
// barrier expects every child's bytes, `late`'s included (its copy is issued by issue_late_h)
__device__ __forceinline__ void issue_land_h(const DevCtx &c, const DevOp &o, int h, int late,
                                             uint32_t sL0, uint32_t sL1, int tile, uint32_t bar) {
  const uint32_t bytes = (uint32_t)half_cats(c.C, h) * 5 * kAChunk;
  uint32_t total = 0;
  for (int s = 0; s < 2; s++)
    if ((s ? o.r_kind : o.l_kind) == GEMS_CHILD_PARTIAL) total += bytes;
  mbar_expect_tx(bar, total);
  for (int s = 0; s < 2; s++) {
    const int kind = s ? o.r_kind : o.l_kind, id = s ? o.r_id : o.l_id;
    if (kind != GEMS_CHILD_PARTIAL || id == late) continue;
    const float *src = static_cast<const float *>(c.partials) + (size_t)id * c.slot_elems +
                       (size_t)tile * (5 * c.C * kAChunk / 4) + (size_t)10 * h * (kAChunk / 4);
    bulk_g2s(s ? sL1 : sL0, src, bytes, bar);
  }
}
__device__ __forceinline__ void issue_late_h(const DevCtx &c, const DevOp &o, int h, int late,
                                             uint32_t sL0, uint32_t sL1, int tile, uint32_t bar) {
  const uint32_t bytes = (uint32_t)half_cats(c.C, h) * 5 * kAChunk;
  for (int s = 0; s < 2; s++) {
    const int kind = s ? o.r_kind : o.l_kind, id = s ? o.r_id : o.l_id;
    if (kind != GEMS_CHILD_PARTIAL || id != late) continue;
    const float *src = static_cast<const float *>(c.partials) + (size_t)id * c.slot_elems +
                       (size_t)tile * (5 * c.C * kAChunk / 4) + (size_t)10 * h * (kAChunk / 4);
    bulk_g2s(s ? sL1 : sL0, src, bytes, bar);
  }
}
// the tables of half-step h of op `o`, per side: an internal child's B images of the half's
// categories, a tip child's whole tip table
__device__ __forceinline__ void issue_tab_h(const DevCtx &c, const DevOp &o, const float *tk,
                                            int h, unsigned char *Bbase, uint32_t bar) {
  const int C = c.C, nc = half_cats(C, h);
  uint32_t bytes[2];
  for (int s = 0; s < 2; s++)
    bytes[s] = (s ? o.r_kind : o.l_kind) == GEMS_CHILD_PARTIAL
                   ? (uint32_t)nc * 2 * kBImg
                   : (uint32_t)(c.unknown + 1) * tip_row_floats(C) * 4;
  mbar_expect_tx(bar, bytes[0] + bytes[1]);
  const size_t imgf = kBImg / 4;
  for (int s = 0; s < 2; s++) {
    const bool in = (s ? o.r_kind : o.l_kind) == GEMS_CHILD_PARTIAL;
    const float *src = in ? tk + ((size_t)(s * C + 2 * h) * 2) * imgf
                          : tk + (size_t)2 * C * 2 * imgf +
                                (size_t)s * (c.unknown + 1) * tip_row_floats(C);
    bulk_g2s(sptr(Bbase + (size_t)s * kBSideH), src, bytes[s], bar);
  }
}

template <bool SAFE>
__global__ void __launch_bounds__(kThreadsH, 2)
    k_traverse_tc20h(DevCtx c, const DevOp *__restrict__ ops, int nops,
                     const float *__restrict__ tab, size_t stride_f, int *flag, int tile0) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *land[2] = {smem_raw, smem_raw + kLandH};
  unsigned char *alo[2] = {smem_raw + 2 * kLandH, smem_raw + 3 * kLandH};
  unsigned char *Bbase = smem_raw + 4 * kLandH;
  TcSharedH *ctl = reinterpret_cast<TcSharedH *>(Bbase + 2 * kBSideH);
  const int t = threadIdx.x, warp = t >> 5, row = t;
  const int C = c.C, H = (C + 1) / 2, nsteps = nops * H;
  const int tile = tile0 + blockIdx.x;
  const long p = (long)tile * kTile + row;
  const bool act = p < c.P;
  const uint32_t bar_land = sptr(&ctl->bar_land), bar_tab = sptr(&ctl->bar_tab),
                 bar_mma = sptr(&ctl->bar_mma);
  if (t == 0) {
    mbar_init(bar_land, 1);
    mbar_init(bar_tab, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // every landing and lo buffer starts at zero: chunks a half-step does not fill (the K padding
  // chunk, and the second category's chunks of a one-category half) hold finite values
  for (int i = t; i < 4 * kLandH / 16; i += kThreadsH)
    reinterpret_cast<float4 *>(smem_raw)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (warp == 0) tmem_alloc(sptr(&ctl->tmem_base), kTmemColsH);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = ctl->tmem_base;
  const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
  const uint32_t sL[2] = {sptr(land[0]), sptr(land[1])};
  const uint64_t dLo[2] = {sdesc(sptr(alo[0]), kAChunk, 128), sdesc(sptr(alo[1]), kAChunk, 128)};
  const uint64_t dB[2] = {sdesc(sptr(Bbase), kNP * 16, 128),
                          sdesc(sptr(Bbase + kBSideH), kNP * 16, 128)};
  const bool inv0 = act ? c.invar[p] == 0.0 : false;
  float *part = static_cast<float *>(c.partials);
  uint32_t ph_land = 0, ph_tab = 0, ph_mma = 0;
  bool ok = true, land_pending = false, tab_pending = false, mma_pending = false;

  DevOp cur = ops[0];
  if (warp == 0 && elect_one()) {
    issue_land_h(c, cur, 0, -1, sL[0], sL[1], tile, bar_land);
    issue_tab_h(c, cur, tab, 0, Bbase, bar_tab);
  }
  land_pending = tab_pending = true;
  int st_l = 0, st_r = 0;  // tip state codes of the current op
  if (act) {
    if (cur.l_kind == GEMS_CHILD_TIP) st_l = min((int)c.tips[(size_t)cur.l_id * c.P + p], c.unknown);
    if (cur.r_kind == GEMS_CHILD_TIP) st_r = min((int)c.tips[(size_t)cur.r_id * c.P + p], c.unknown);
  }
  float mx_prev = 0.f;  // NORM: the row maximum over the op's earlier half-steps

  for (int step = 0; step < nsteps && ok; step++) {
    const int k = step / H, h = step - k * H, nc = half_cats(C, h);
    const bool last_half = h == H - 1;
    const bool inL = cur.l_kind == GEMS_CHILD_PARTIAL, inR = cur.r_kind == GEMS_CHILD_PARTIAL;
    const bool tiptip = !inL && !inR;
    const bool has_next = step + 1 < nsteps;
    DevOp nxt = cur;
    int nh = h + 1;
    if (last_half) {
      nh = 0;
      if (has_next) nxt = ops[k + 1];
    }
    // the next op's child that this op writes is copied after this op's last stores
    const int late = (has_next && last_half) ? cur.dst_slot : -1;
    // children's counters of this half-step's categories (NORM: per pattern)
    int scl[2] = {0, 0}, scr[2] = {0, 0};
    if (act) {
#pragma unroll
      for (int j = 0; j < 2; j++) {
        if (j >= nc) continue;
        const size_t o = SAFE ? (size_t)p * C + 2 * h + j : (size_t)p;
        if (inL) scl[j] = c.scale[(size_t)cur.l_id * c.slot_scale + o];
        if (inR) scr[j] = c.scale[(size_t)cur.r_id * c.slot_scale + o];
      }
    }
    if (__syncthreads_or(!mbar_wait(bar_land, ph_land) || !mbar_wait(bar_tab, ph_tab))) {
      ok = false;
      if (t == 0) atomicExch(flag, GEMS_ERR_TIMEOUT);
      break;
    }
    land_pending = tab_pending = false;
    ph_land ^= 1;
    ph_tab ^= 1;
    // internal children: hi -> TMEM, lo -> shared memory; tip children: the row's tip-table
    // entries of the half's categories into the side's lo buffer (which it does not use)
#pragma unroll
    for (int s = 0; s < 2; s++) {
      float4 *l4 = reinterpret_cast<float4 *>(alo[s]);
      if (!(s ? inR : inL)) {
        const int stc = s ? st_r : st_l;
        const float4 *lt = reinterpret_cast<const float4 *>(
            Bbase + (size_t)s * kBSideH + (size_t)stc * tip_row_floats(C) * 4);
#pragma unroll
        for (int j = 0; j < 2; j++) {
          if (j >= nc) continue;
#pragma unroll
          for (int i = 0; i < 5; i++) l4[(j * 5 + i) * kTile + row] = lt[(2 * h + j) * 5 + i];
        }
        continue;
      }
      const float4 *a4 = reinterpret_cast<const float4 *>(land[s]);
#pragma unroll
      for (int j = 0; j < 2; j++) {
        if (j >= nc) continue;
        float4 hv[5];
#pragma unroll
        for (int i = 0; i < 5; i++) {
          float4 lv;
          split4(a4[(j * 5 + i) * kTile + row], hv[i], lv);
          l4[(j * 5 + i) * kTile + row] = lv;
        }
        tmem_st_row(tmem + lane_off + (uint32_t)(kAhiColH + (2 * s + j) * kKP), hv);
      }
    }
    tmem_st_wait();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0 && elect_one()) {
      // the landing buffers have been read: the next half-step's tiles come in
      if (has_next) issue_land_h(c, nxt, nh, late, sL[0], sL[1], tile, bar_land);
#pragma unroll
      for (int s = 0; s < 2; s++) {
        if (!(s ? inR : inL)) continue;
#pragma unroll
        for (int j = 0; j < 2; j++) {
          if (j >= nc) continue;
          const uint32_t dtm = tmem + (uint32_t)((2 * s + j) * kNP);
          const uint32_t atm = tmem + (uint32_t)(kAhiColH + (2 * s + j) * kKP);
          const uint64_t bh = dB[s] + (uint64_t)((j * 2 * kBImg) >> 4);
          const uint64_t bl = bh + (uint64_t)(kBImg >> 4);
#pragma unroll
          for (int ks = 0; ks < kKP / 8; ks++) {
            const uint64_t ko = (uint64_t)(((j * 5 + 2 * ks) * kAChunk) >> 4);
            const uint64_t kb = (uint64_t)((2 * ks * kNP * 16) >> 4);
            mma_tf32_ta(dtm, atm + 8 * ks, bh + kb, ks > 0 ? 1u : 0u);
            mma_tf32_ta(dtm, atm + 8 * ks, bl + kb, 1u);
            mma_tf32(dtm, dLo[s] + ko, bh + kb, 1u);
          }
        }
      }
      if (!tiptip) mma_commit(bar_mma);
    }
    land_pending = has_next;
    if (!tiptip) {
      mma_pending = true;
      if (__syncthreads_or(!mbar_wait(bar_mma, ph_mma))) {
        ok = false;
        if (t == 0) atomicExch(flag, GEMS_ERR_TIMEOUT);
        break;
      }
      mma_pending = false;
      ph_mma ^= 1;
      tc_fence_after();
    }
    // the tables of this half-step are no longer read (MMAs done, tip rows copied out)
    if (has_next) {
      if (warp == 0 && elect_one())
        issue_tab_h(c, nxt, tab + (size_t)(last_half ? k + 1 : k) * stride_f, nh, Bbase, bar_tab);
      tab_pending = true;
    }
    // ---- epilogue: messages, products, scaling, stores
    float out[2][kN];
    float mx[2] = {0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 2; j++) {
      if (j >= nc) continue;
      float m[2][kN];
      uint32_t r[2][20];
#pragma unroll
      for (int s = 0; s < 2; s++)
        if (s ? inR : inL) tmem_ld20(tmem + lane_off + (uint32_t)((2 * s + j) * kNP), r[s]);
#pragma unroll
      for (int s = 0; s < 2; s++) {
        if (s ? inR : inL) {
          tmem_ld_wait(r[s]);
#pragma unroll
          for (int x = 0; x < kN; x++) m[s][x] = __uint_as_float(r[s][x]);
        } else {
          const float4 *l4 = reinterpret_cast<const float4 *>(alo[s]);
#pragma unroll
          for (int i = 0; i < 5; i++) {
            const float4 v = l4[(j * 5 + i) * kTile + row];
            m[s][4 * i] = v.x;
            m[s][4 * i + 1] = v.y;
            m[s][4 * i + 2] = v.z;
            m[s][4 * i + 3] = v.w;
          }
        }
      }
#pragma unroll
      for (int x = 0; x < kN; x++) {
        const float v = fmaxf(m[0][x], 0.f) * fmaxf(m[1][x], 0.f);
        out[j][x] = v;
        mx[j] = fmaxf(mx[j], v);
      }
    }
    float f[2] = {1.f, 1.f};
    bool up_all = false;  // NORM: the row is scaled (decided at the op's last half-step)
    if (SAFE) {
#pragma unroll
      for (int j = 0; j < 2; j++)
        if (j < nc && !tiptip && mx[j] < kScaleThrF && inv0) f[j] = 18446744073709551616.0f;
    } else {
      const float m = fmaxf(mx_prev, fmaxf(mx[0], mx[1]));
      if (last_half) {
        up_all = !tiptip && m < kScaleThrF && inv0;
        if (up_all) f[0] = f[1] = 18446744073709551616.0f;  // 2^64
        mx_prev = 0.f;
      } else {
        mx_prev = m;
      }
    }
    float *dtile = part + (size_t)cur.dst_slot * c.slot_elems + (size_t)tile * (5 * C * kAChunk / 4);
    uint16_t *sd = c.scale + (size_t)cur.dst_slot * c.slot_scale;
#pragma unroll
    for (int j = 0; j < 2; j++) {
      if (j >= nc) continue;
      const int cc = 2 * h + j;
#pragma unroll
      for (int i = 0; i < kN / 4; i++) {
        const float4 v = make_float4(out[j][4 * i] * f[j], out[j][4 * i + 1] * f[j],
                                     out[j][4 * i + 2] * f[j], out[j][4 * i + 3] * f[j]);
        reinterpret_cast<float4 *>(dtile)[(cc * 5 + i) * kTile + row] = v;
      }
      if (SAFE && act)
        sd[(size_t)p * C + cc] =
            (uint16_t)(scl[j] + scr[j] + (f[j] != 1.f ? 1 : 0));
    }
    if (!SAFE && last_half) {
      if (up_all) {  // the earlier half-steps' rows of this op, stored unscaled: scale them
        for (int cc = 0; cc < 2 * h; cc++)
#pragma unroll
          for (int i = 0; i < kN / 4; i++) {
            float4 *q = reinterpret_cast<float4 *>(dtile) + (cc * 5 + i) * kTile + row;
            float4 v = *q;
            v.x *= 18446744073709551616.0f;
            v.y *= 18446744073709551616.0f;
            v.z *= 18446744073709551616.0f;
            v.w *= 18446744073709551616.0f;
            *q = v;
          }
      }
      if (act) sd[p] = (uint16_t)(scl[0] + scr[0] + (up_all ? 1 : 0));
    }
    // later steps bulk-copy these rows from global memory (through the async proxy)
    asm volatile("fence.proxy.async.global;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (late >= 0 && warp == 0 && elect_one())
      issue_late_h(c, nxt, nh, late, sL[0], sL[1], tile, bar_land);
    if (has_next && last_half) {  // the next op: its tip state codes
      st_l = st_r = 0;
      if (act) {
        if (nxt.l_kind == GEMS_CHILD_TIP)
          st_l = min((int)c.tips[(size_t)nxt.l_id * c.P + p], c.unknown);
        if (nxt.r_kind == GEMS_CHILD_TIP)
          st_r = min((int)c.tips[(size_t)nxt.r_id * c.P + p], c.unknown);
      }
    }
    cur = nxt;
  }
  if (!ok && t == 0) {
    if (land_pending) mbar_wait(bar_land, ph_land);
    if (tab_pending) mbar_wait(bar_tab, ph_tab);
    if (mma_pending) mbar_wait(bar_mma, ph_mma);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemColsH);
}

}  // namespace

size_t tc20_op_floats(int ncat, int unknown) {
  return (size_t)2 * ncat * 2 * (kBImg / 4) + (size_t)2 * (unknown + 1) * tip_row_floats(ncat);
}

bool tc20_supported(const Session *s) {
  return s->desc.nstates == 20 && s->desc.precision == GEMS_PREC_MIXED && s->desc.ncat <= 4 &&
         s->tc_enabled && s->tiled;
}

static size_t tc_smem(int C) {
  return 4 * (size_t)kABytes + (size_t)2 * C * 2 * kBImg + sizeof(TcShared) + 64;
}

int launch_prep_ops_tc20(Session *s, int nops) {
  if (nops <= 0) return GEMS_OK;
  DevCtx c = s->ctx();
  const size_t smem = sizeof(double) * s->desc.ncat * kN + sizeof(float) * s->desc.ncat * kN * kN;
  k_prep_ops_tc<<<dim3(nops, 2), 256, smem, s->stream>>>(
      c, s->d_ops, reinterpret_cast<float *>(s->d_opmats), s->op_stride_tc);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

int launch_traverse_tc20(Session *s, int nops, int p0, int p1) {
  if (nops <= 0 || p1 <= p0) return GEMS_OK;
  if (p0 % kTile != 0 || (p1 % kTile != 0 && p1 != s->P)) {
    set_error("tcgen05 20-state traversal: pattern range not aligned to its 128-pattern tiles");
    return GEMS_ERR_BAD_ARG;
  }
  DevCtx c = s->ctx();
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  if (s->tc20_halves) {  // two CTAs per SM in half-steps
    void *fh = safe ? (void *)k_traverse_tc20h<true> : (void *)k_traverse_tc20h<false>;
    GEMS_CUDA(cudaFuncSetAttribute(fh, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem_h()));
    GEMS_CUDA(cudaMemsetAsync(s->d_flag, 0, sizeof(int), s->stream));
    const int tile0 = p0 / kTile;
    const int grid = (p1 + kTile - 1) / kTile - tile0;
    cudaEvent_t ev0;
    if (int st = prof_begin(s, 0, &ev0)) return st;
    const float *tab = reinterpret_cast<const float *>(s->d_opmats);
    if (safe)
      k_traverse_tc20h<true><<<grid, kThreadsH, tc_smem_h(), s->stream>>>(
          c, s->d_ops, nops, tab, s->op_stride_tc, s->d_flag, tile0);
    else
      k_traverse_tc20h<false><<<grid, kThreadsH, tc_smem_h(), s->stream>>>(
          c, s->d_ops, nops, tab, s->op_stride_tc, s->d_flag, tile0);
    s->launches++;
    GEMS_CUDA(cudaGetLastError());
    if (int st = prof_end(s, 0, ev0)) return st;
    int flag = 0;
    GEMS_CUDA(cudaMemcpyAsync(&flag, s->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    GEMS_CUDA(cudaStreamSynchronize(s->stream));
    if (flag) {
      set_error("tensor-core traversal: bounded wait expired");
      return GEMS_ERR_TIMEOUT;
    }
    return GEMS_OK;
  }
  const size_t smem = tc_smem(s->desc.ncat);
  void *fn = safe ? (void *)k_traverse_tc20<true> : (void *)k_traverse_tc20<false>;
  // the limit is a property of the kernel, shared by every session and host thread: set it to
  // the largest size any session needs (4 categories), so that a concurrent setting for another
  // session never lowers it below this launch's size
  GEMS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem(4)));
  GEMS_CUDA(cudaMemsetAsync(s->d_flag, 0, sizeof(int), s->stream));
  const int tile0 = p0 / kTile;
  const int grid = (p1 + kTile - 1) / kTile - tile0;
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 0, &ev0)) return st;
  const float *tab = reinterpret_cast<const float *>(s->d_opmats);
  if (safe)
    k_traverse_tc20<true><<<grid, kThreadsTc, smem, s->stream>>>(c, s->d_ops, nops, tab,
                                                                  s->op_stride_tc, s->d_flag,
                                                                  tile0);
  else
    k_traverse_tc20<false><<<grid, kThreadsTc, smem, s->stream>>>(c, s->d_ops, nops, tab,
                                                                   s->op_stride_tc, s->d_flag,
                                                                   tile0);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  if (int st = prof_end(s, 0, ev0)) return st;
  int flag = 0;
  GEMS_CUDA(cudaMemcpyAsync(&flag, s->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  GEMS_CUDA(cudaStreamSynchronize(s->stream));
  if (flag) {
    set_error("tensor-core traversal: bounded wait expired");
    return GEMS_ERR_TIMEOUT;
  }
  return GEMS_OK;
}

}  // namespace gems
