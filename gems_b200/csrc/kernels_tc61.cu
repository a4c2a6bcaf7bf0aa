// kernels_tc61.cu -- 61-state (codon) mixed-precision traversal on the tcgen05 tensor cores.
//
// Node update per category c (real space, FP32 storage, SAFE scaling per category -- the
// reference always uses SAFE for 61 states, phylotreesse.cpp:95-96):
//     out[p][c][:] = (P_c(t_L) . L[p][c][:]) (*) (P_c(t_R) . R[p][c][:])
// For a tile of 128 patterns each child product is D[128 x 64] = A[128 x 64] . B^T (61 states
// padded to 64 in K and N; the padding rows of B are zero), issued as tcgen05.mma kind::tf32
// M=128 N=64 K=8, FP32 accuracy from split TF32 (A.B ~ A_hi.B_hi + A_hi.B_lo + A_lo.B_hi).
// A tip child needs no product: its message is a row of the op's tip table (column s of
// P_c(t) for a tip in state s, the row sums for the unknown state), which the table copy brings
// in place of that side's B images.
//
// The work of one op is done category by category ("steps"): one category of a child tile is
// 16 chunks x 2 KB = 32 KB, contiguous in the tile-major layout (mix_off<61>), brought by one
// cp.async.bulk.  Per step (one CTA per SM, 256 threads, 2 per pattern row):
//   wait(operand tiles, tables of this step)
//   -> split of internal children: hi -> TMEM operand columns (tcgen05.st), lo -> shared
//      memory; a tip child's table row is copied into its side's (unused) lo buffer
//   -> the next step's operand tiles start copying (landing buffers free)
//   -> MMAs of internal children (issued by an elected lane), wait -> the next step's tables
//      start copying
//   -> epilogue: tcgen05.ld of the accumulators, products, SAFE rescaling by 2^64 with uint16
//      counters, coalesced stores of the rows (as computed; every consumer splits the stored
//      values the same way)
// The step after the last category of an op may need that op's output of the same category
// (one category: C = 1); that copy is issued after the epilogue's stores instead.
//
// The kernel takes an array of jobs (sessions that share one tree: ModelFinder's candidate
// models on one alignment; each job has its own op list), grid (tiles, jobs), so many small
// sessions fill the GPU
// in one launch.  Every mbarrier wait is bounded; on expiry the CTA records GEMS_ERR_TIMEOUT,
// waits (bounded) for its copies in flight, frees its TMEM and returns.
#include <cstring>
#include <string>
#include <vector>

#include "gems_internal.cuh"
#include "tc_common.cuh"

namespace gems {

namespace {

using namespace tc;

constexpr int kN = 61;
constexpr int kNP = 64;                   // MMA N and K (padded states)
constexpr int kTile = 128;                // patterns per CTA = MMA M
constexpr int kThreads61 = 256;           // 2 threads per pattern row, 32 states each
constexpr int kK = 16;                    // 4-state chunks per category row
constexpr int kAChunk = kTile * 16;       // one chunk of a tile (128 rows x 16 B)
constexpr int kATile = kK * kAChunk;      // one category of one child tile: 32 KB
constexpr int kBImg = (kNP / 4) * kNP * 16;  // 16 K chunks x 64 rows x 16 B = 16 KB
constexpr int kBSide = 2 * kBImg;         // hi + lo images of one side: 32 KB
constexpr uint32_t kIdesc61 = idesc_tf32(kNP);
constexpr int kTmemCols61 = 256;          // D[side] at side*64, A_hi[side] at 128 + side*64
constexpr int kAhi61 = 128;

// op tables: per side and category a 32 KB region.  An internal child's: the B images
// [hi, lo][16 K chunks][64 rows][4] (row = target state x, K = source state y).  A tip child's:
// its tip table [62 state codes][64 target states + 4 padding] -- row s < 61 is column s of P_c(t), the
// message of a tip in state s; row 61 the row sums, the message of the unknown state (every
// code >= 61) -- so a tip side needs neither MMAs nor B images.  Floats per op:
__host__ __device__ constexpr size_t op_floats61(int C) { return (size_t)2 * C * (kBSide / 4); }
constexpr int kTipRows61 = kN + 1;  // 61 states + unknown
// a tip table row: 64 target states padded by 4 floats, so that the rows of different state
// codes (the lanes of a warp read their own patterns' rows) start in different bank groups
constexpr int kTipRow61 = kNP + 4;
constexpr uint32_t kTipBytes61 = kTipRows61 * kTipRow61 * 4;  // 16,864 bytes

// The op tables of a job's op k and side (blockIdx.x, blockIdx.y; job blockIdx.z of `jobs`, or
// `one` when jobs is null).  P_c(t) = evec . diag(exp(eval * rate_c * t)) . inv_evec in FP64,
// clamped at 0, then split into TF32 hi and lo images.  Register-tiled: a thread owns target
// states 4xq..4xq+3 by the source-state quads jo and jo + 8 (4 x 8 outputs; float4s of the
// image rows it writes), so each term of the sum costs 13 shared-memory reads for 32 FMAs; the
// sum over i runs in index order with the same fma(evec * exp, inv_evec, acc) steps as a scalar
// loop.  Shared memory: exp terms [C][n]; evec as [64][n] (rows 61..63 zero); inv_evec as
// [n][4 e][16 j] = inv_evec[i][4j + e] (columns 61..63 zero), so that the 8 lanes of a row quad
// read 8 consecutive doubles.  A tip side's unknown-state row sums add the quads j and j + 8 in
// the thread, then the 8 lanes of the row quad by a fixed shuffle tree: the same bits in every
// launch.
// two halves of 128 threads (16 row quads x 8 pairs of column quads) take alternate categories
constexpr int kPrepThreads = 256;
__host__ __device__ constexpr size_t prep61_smem_doubles(int C) {
  return (size_t)C * kN + (size_t)kNP * kN + (size_t)kN * kNP;
}
__global__ void __launch_bounds__(kPrepThreads, 2)
    k_prep_ops_tc61(const __grid_constant__ TcJob one, const TcJob *__restrict__ jobs,
                    size_t stride_f) {
  extern __shared__ double ex[];
  const TcJob &job = jobs ? jobs[blockIdx.z] : one;
  const DevCtx &c = job.c;
  const int k = blockIdx.x, side = blockIdx.y;
  const DevOp op = job.ops[k];
  const double len = side ? op.r_len : op.l_len;
  const int C = c.C, n = kN;
  double *ev = ex + C * n, *iv = ev + kNP * n;
  for (int idx = threadIdx.x; idx < C * n; idx += blockDim.x) {
    const int cc = idx / n, i = idx - cc * n;
    ex[idx] = exp(c.eval[i] * (c.rates[cc] * len));
  }
  for (int idx = threadIdx.x; idx < kNP * n; idx += blockDim.x) {
    const int x = idx / n;
    ev[idx] = x < n ? c.evec[idx] : 0.0;
    const int i = idx / kNP, r = idx - i * kNP, e = r >> 4, j = r & 15, y = 4 * j + e;
    iv[idx] = y < n ? c.inv_evec[i * n + y] : 0.0;
  }
  __syncthreads();
  // the job's own table, written here and read by its traversal
  float *img = const_cast<float *>(job.tab) + (size_t)k * stride_f + (size_t)side * C * (kBSide / 4);
  const int per = kBImg / 4;  // floats of one image
  // thread: row quad xq (rows 4xq..4xq+3) and the column quads jo and jo + 8, in the half of
  // the block that takes categories sub, sub + 2, ...
  const int lt = threadIdx.x & 127, sub = threadIdx.x >> 7;
  const int jo = lt & 7, xq = lt >> 3;
  const bool tip = (side ? op.r_kind : op.l_kind) == GEMS_CHILD_TIP;
  for (int cc = sub; cc < C; cc += 2) {
    double acc[4][2][4];  // [row][column quad jo, jo + 8][column in quad]
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[r][h][e] = 0.0;
    const double *exc = ex + cc * n;
    for (int i = 0; i < n; i++) {
      const double xi = exc[i];
      double a[4], b[2][4];
#pragma unroll
      for (int r = 0; r < 4; r++) a[r] = ev[(4 * xq + r) * n + i] * xi;
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int e = 0; e < 4; e++) b[h][e] = iv[i * kNP + e * 16 + jo + 8 * h];
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
          for (int e = 0; e < 4; e++) acc[r][h][e] = fma(a[r], b[h][e], acc[r][h][e]);
    }
    if (tip) {
      // tip table: row s = column s of P_c (target states x consecutive), then the row sums
      float *tt = img + (size_t)cc * 2 * per;
      double rs[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = jo + 8 * h;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int y = 4 * j + e;
          float v[4];
#pragma unroll
          for (int r = 0; r < 4; r++) {
            const int x = 4 * xq + r;
            const double a = (x < n && y < n) ? fmax(acc[r][h][e], 0.0) : 0.0;
            rs[h][r] += a;
            v[r] = (float)a;
          }
          if (y < n)
            *reinterpret_cast<float4 *>(tt + (size_t)y * kTipRow61 + 4 * xq) =
                make_float4(v[0], v[1], v[2], v[3]);
        }
      }
      // the sums of the 16 column quads by a fixed tree: quads j and j + 8 first (in this
      // thread), then across the 8 lanes of the row quad
      double t4[4];
#pragma unroll
      for (int r = 0; r < 4; r++) t4[r] = rs[0][r] + rs[1][r];
#pragma unroll
      for (int o = 4; o >= 1; o >>= 1)
#pragma unroll
        for (int r = 0; r < 4; r++) t4[r] += __shfl_xor_sync(0xffffffffu, t4[r], o);
      if (jo == 0)
        *reinterpret_cast<float4 *>(tt + (size_t)n * kTipRow61 + 4 * xq) =
            make_float4((float)t4[0], (float)t4[1], (float)t4[2], (float)t4[3]);
      continue;
    }
    // image element (row x, K index y) at chunk y / 4, row x, lane y % 4
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int x = 4 * xq + r;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = jo + 8 * h;
        float v[4];
#pragma unroll
        for (int e = 0; e < 4; e++)
          v[e] = (x < n && 4 * j + e < n) ? (float)fmax(acc[r][h][e], 0.0) : 0.f;
        const float4 hi = make_float4(tf32_rna(v[0]), tf32_rna(v[1]), tf32_rna(v[2]), tf32_rna(v[3]));
        const float4 lo = make_float4(tf32_rna(v[0] - hi.x), tf32_rna(v[1] - hi.y),
                                      tf32_rna(v[2] - hi.z), tf32_rna(v[3] - hi.w));
        const size_t o = (size_t)cc * 2 * per + ((size_t)j * kNP + x) * 4;
        *reinterpret_cast<float4 *>(img + o) = hi;
        *reinterpret_cast<float4 *>(img + o + per) = lo;
      }
    }
  }
}

struct Tc61Shared {
  uint64_t bar_land, bar_b, bar_mma;
  uint32_t tmem_base;
  float rowmax[2][kTile];
};

// 32 TMEM columns of this thread's lane; valid after tmem_ld32_wait on the same registers
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld32_wait(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                 "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                 "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                 "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}
// 32 consecutive TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, "
      "%29, %30, %31, %32};" ::"r"(taddr),
      "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]),
      "f"(v[8]), "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]),
      "f"(v[15]), "f"(v[16]), "f"(v[17]), "f"(v[18]), "f"(v[19]), "f"(v[20]), "f"(v[21]),
      "f"(v[22]), "f"(v[23]), "f"(v[24]), "f"(v[25]), "f"(v[26]), "f"(v[27]), "f"(v[28]),
      "f"(v[29]), "f"(v[30]), "f"(v[31])
      : "memory");
}


// step t of an op list: op t / C, category t % C
struct Step {
  DevOp op;
  int cat;
};

// copies of the operand tiles of step `st` (internal children, category st.cat) into the
// landing buffers; `late_slot`: a child equal to it is left for a late copy (issued by the
// caller after the current step's stores); the barrier expects all bytes now
__device__ __forceinline__ void issue_land(const DevCtx &c, const Step &st, int late_slot,
                                           uint32_t sL0, uint32_t sL1, int tile, uint32_t bar) {
  uint32_t bytes = 0;
  for (int s = 0; s < 2; s++)
    if ((s ? st.op.r_kind : st.op.l_kind) == GEMS_CHILD_PARTIAL) bytes += kATile;
  mbar_expect_tx(bar, bytes);
  for (int s = 0; s < 2; s++) {
    const int kind = s ? st.op.r_kind : st.op.l_kind, id = s ? st.op.r_id : st.op.l_id;
    if (kind != GEMS_CHILD_PARTIAL || id == late_slot) continue;
    const float *src = static_cast<const float *>(c.partials) + (size_t)id * c.slot_elems +
                       mix_off<61>(c, (long)tile * kTile, st.cat);
    bulk_g2s(s ? sL1 : sL0, src, kATile, bar);
  }
}
__device__ __forceinline__ void issue_late(const DevCtx &c, const Step &st, int late_slot,
                                           uint32_t sL0, uint32_t sL1, int tile, uint32_t bar) {
  for (int s = 0; s < 2; s++) {
    const int kind = s ? st.op.r_kind : st.op.l_kind, id = s ? st.op.r_id : st.op.l_id;
    if (kind != GEMS_CHILD_PARTIAL || id != late_slot) continue;
    const float *src = static_cast<const float *>(c.partials) + (size_t)id * c.slot_elems +
                       mix_off<61>(c, (long)tile * kTile, st.cat);
    bulk_g2s(s ? sL1 : sL0, src, kATile, bar);
  }
}
// the tables of step (op, cat): per side the B images (hi and lo) of an internal child or the
// tip table of a tip child
__device__ __forceinline__ void issue_b(const float *tab_op, int C, int cat, const DevOp &op,
                                        unsigned char *Bbase, uint32_t bar) {
  uint32_t bytes[2];
  for (int s = 0; s < 2; s++)
    bytes[s] = (s ? op.r_kind : op.l_kind) == GEMS_CHILD_PARTIAL ? (uint32_t)kBSide : kTipBytes61;
  mbar_expect_tx(bar, bytes[0] + bytes[1]);
  for (int s = 0; s < 2; s++)
    bulk_g2s(sptr(Bbase + (size_t)s * kBSide),
             tab_op + ((size_t)s * C + cat) * (kBSide / 4), bytes[s], bar);
}

__global__ void __launch_bounds__(kThreads61, 1)
    k_traverse_tc61(const TcJob *__restrict__ jobs, int nops, size_t stride_f, int *flag,
                    int tile0) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ TcJob sj;
  unsigned char *land = smem_raw;                     // [2][32 KB] raw operand tiles
  unsigned char *alo = smem_raw + 2 * kATile;         // [2][32 KB] lo parts
  unsigned char *Bbase = smem_raw + 4 * kATile;       // [2][hi 16 KB, lo 16 KB]
  Tc61Shared *ctl = reinterpret_cast<Tc61Shared *>(smem_raw + 4 * kATile + 2 * kBSide);

  const int t = threadIdx.x, warp = t >> 5;
  const int row = ((warp & 3) << 5) | (t & 31);
  const int half = warp >> 2;  // states [32h, 32h + 32) = chunks [8h, 8h + 8)
  if (t == 0) sj = jobs[blockIdx.y];
  const uint32_t bar_land = sptr(&ctl->bar_land), bar_b = sptr(&ctl->bar_b),
                 bar_mma = sptr(&ctl->bar_mma);
  if (t == 0) {
    mbar_init(bar_land, 1);
    mbar_init(bar_b, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(sptr(&ctl->tmem_base), kTmemCols61);
  fence_before();
  __syncthreads();
  fence_after();
  const DevCtx &c = sj.c;
  const DevOp *ops = sj.ops;
  const float *tab = sj.tab;
  const int C = c.C;
  const int tile = tile0 + blockIdx.x;
  const long p = (long)tile * kTile + row;
  const bool act = p < c.P;
  const bool inv0 = act ? c.invar[p] == 0.0 : false;
  const uint32_t tmem = ctl->tmem_base;
  const uint32_t lane_off = (uint32_t)((warp & 3) * 32) << 16;
  const uint32_t sL0 = sptr(land), sL1 = sptr(land + kATile);
  const uint64_t dLo[2] = {sdesc(sptr(alo), kAChunk, 128), sdesc(sptr(alo + kATile), kAChunk, 128)};
  const uint64_t dB[2] = {sdesc(sptr(Bbase), kNP * 16, 128),
                          sdesc(sptr(Bbase + kBSide), kNP * 16, 128)};
  float *part = static_cast<float *>(c.partials);
  const int nsteps = nops * C;
  uint32_t ph_land = 0, ph_b = 0, ph_mma = 0;
  bool ok = true, land_pending = false, b_pending = false, mma_pending = false;

  Step cur{ops[0], 0};
  if (warp == 0 && elect_one()) {
    issue_land(c, cur, -1, sL0, sL1, tile, bar_land);
    issue_b(tab, C, 0, cur.op, Bbase, bar_b);
  }
  land_pending = b_pending = true;
  int st_l = 0, st_r = 0;  // tip state codes of the current op
  if (act) {
    if (cur.op.l_kind == GEMS_CHILD_TIP) st_l = c.tips[(size_t)cur.op.l_id * c.P + p];
    if (cur.op.r_kind == GEMS_CHILD_TIP) st_r = c.tips[(size_t)cur.op.r_id * c.P + p];
  }

  for (int step = 0; step < nsteps && ok; step++) {
    const int k = step / C;
    const bool inL = cur.op.l_kind == GEMS_CHILD_PARTIAL, inR = cur.op.r_kind == GEMS_CHILD_PARTIAL;
    const bool has_next = step + 1 < nsteps;
    Step nxt = cur;
    if (has_next) {
      if (cur.cat + 1 < C) {
        nxt.cat = cur.cat + 1;
      } else {
        nxt.op = ops[k + 1];
        nxt.cat = 0;
      }
    }
    // the next step needs this step's output (same slot and category): copied after the stores
    const int late = (has_next && nxt.cat == cur.cat) ? cur.op.dst_slot : -1;
    // children's counters of this category (SAFE: per pattern and category)
    int scl = 0, scr = 0;
    if (act) {
      if (inL) scl = c.scale[(size_t)cur.op.l_id * c.slot_scale + (size_t)p * C + cur.cat];
      if (inR) scr = c.scale[(size_t)cur.op.r_id * c.slot_scale + (size_t)p * C + cur.cat];
    }
    if (__syncthreads_or(!mbar_wait(bar_land, ph_land) || !mbar_wait(bar_b, ph_b))) {
      ok = false;
      if (t == 0) atomicExch(flag, GEMS_ERR_TIMEOUT);
      break;
    }
    land_pending = b_pending = false;
    ph_land ^= 1;
    ph_b ^= 1;
    // operand rows of internal children: hi -> TMEM, lo -> shared memory.  A tip child's
    // message is its tip table's row: copied into the side's lo buffer (which its side does not
    // use), so that the next step's tables can overwrite the table region during the epilogue
#pragma unroll
    for (int s = 0; s < 2; s++) {
      float4 *l4 = reinterpret_cast<float4 *>(alo + (size_t)s * kATile);
      if (!(s ? inR : inL)) {
        const int st = s ? st_r : st_l;
        const float4 *tr = reinterpret_cast<const float4 *>(
                               Bbase + (size_t)s * kBSide + (size_t)(st < kN ? st : kN) * kTipRow61 * 4) +
                           8 * half;
#pragma unroll
        for (int i = 0; i < 8; i++) l4[(8 * half + i) * kTile + row] = tr[i];
        continue;
      }
      float h[32];
      const float4 *a4 = reinterpret_cast<const float4 *>(land + (size_t)s * kATile);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int ch = 8 * half + i;
        float4 hv, lv;
        split4(a4[ch * kTile + row], hv, lv);
        l4[ch * kTile + row] = lv;
        h[4 * i] = hv.x;
        h[4 * i + 1] = hv.y;
        h[4 * i + 2] = hv.z;
        h[4 * i + 3] = hv.w;
      }
      tmem_st32(tmem + lane_off + (uint32_t)(kAhi61 + s * kNP + 32 * half), h);
    }
    tmem_st_wait();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    const bool any_in = inL || inR;
    if (warp == 0 && elect_one()) {
      // the landing buffers have been read: the next step's tiles come in
      if (has_next) issue_land(c, nxt, late, sL0, sL1, tile, bar_land);
#pragma unroll
      for (int s = 0; s < 2; s++) {
        if (!(s ? inR : inL)) continue;
        const uint32_t dtm = tmem + (uint32_t)(s * kNP);
        const uint32_t atm = tmem + (uint32_t)(kAhi61 + s * kNP);
#pragma unroll
        for (int ks = 0; ks < kNP / 8; ks++) {
          const uint64_t kb = (uint64_t)((2 * ks * kNP * 16) >> 4);
          const uint64_t ko = (uint64_t)((2 * ks * kAChunk) >> 4);
          const uint64_t bh = dB[s] + kb, bl = dB[s] + kb + (uint64_t)(kBImg >> 4);
          mma_ts(dtm, atm + 8 * ks, bh, kIdesc61, ks > 0 ? 1u : 0u);
          mma_ts(dtm, atm + 8 * ks, bl, kIdesc61, 1u);
          mma_ss(dtm, dLo[s] + ko, bh, kIdesc61, 1u);
        }
      }
      if (any_in) mma_commit(bar_mma);
    }
    land_pending = has_next;
    if (any_in) {
      mma_pending = true;
      if (__syncthreads_or(!mbar_wait(bar_mma, ph_mma))) {
        ok = false;
        if (t == 0) atomicExch(flag, GEMS_ERR_TIMEOUT);
        break;
      }
      mma_pending = false;
      ph_mma ^= 1;
      fence_after();
    }
    // the tables of this step are no longer read (the MMAs are done, the tip rows copied out):
    // the next step's come in under the epilogue
    if (has_next) {
      if (warp == 0 && elect_one())
        issue_b(tab + (size_t)(cur.cat + 1 < C ? k : k + 1) * stride_f, C, nxt.cat, nxt.op,
                Bbase, bar_b);
      b_pending = true;
    }
    // ---- epilogue: products, SAFE rescaling of this category, stores
    // messages: an internal child's from its accumulator, a tip's from its table row
    uint32_t rm[2][32];
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (s ? inR : inL) tmem_ld32(tmem + lane_off + (uint32_t)(s * kNP + 32 * half), rm[s]);
#pragma unroll
    for (int s = 0; s < 2; s++) {
      if (s ? inR : inL) {
        tmem_ld32_wait(rm[s]);
      } else {
        const float4 *tr = reinterpret_cast<const float4 *>(alo + (size_t)s * kATile);
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const float4 q = tr[(8 * half + i) * kTile + row];
          rm[s][4 * i] = __float_as_uint(q.x);
          rm[s][4 * i + 1] = __float_as_uint(q.y);
          rm[s][4 * i + 2] = __float_as_uint(q.z);
          rm[s][4 * i + 3] = __float_as_uint(q.w);
        }
      }
    }
    float v[32];
    float mx = 0.f;
#pragma unroll
    for (int i = 0; i < 32; i++) {
      v[i] = fmaxf(__uint_as_float(rm[0][i]), 0.f) * fmaxf(__uint_as_float(rm[1][i]), 0.f);
      mx = fmaxf(mx, v[i]);
    }
    ctl->rowmax[half][row] = mx;
    __syncthreads();
    const float m = fmaxf(ctl->rowmax[0][row], ctl->rowmax[1][row]);
    int s_out = scl + scr;
    float f = 1.f;
    if ((inL || inR) && m < kScaleThrF && inv0) {
      f = 18446744073709551616.0f;  // 2^64
      s_out += 1;
    }
    float *dst = part + (size_t)cur.op.dst_slot * c.slot_elems + mix_off<61>(c, (long)tile * kTile, cur.cat);
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int x = 32 * half + 4 * i;
      float4 w = make_float4(v[4 * i] * f, v[4 * i + 1] * f, v[4 * i + 2] * f, v[4 * i + 3] * f);
      if (x + 3 >= kN) {  // padding states stored as zeros
        if (x + 1 >= kN) w.y = 0.f;
        if (x + 2 >= kN) w.z = 0.f;
        if (x + 3 >= kN) w.w = 0.f;
        if (x >= kN) w.x = 0.f;
      }
      reinterpret_cast<float4 *>(dst)[(8 * half + i) * kTile + row] = w;
    }
    if (act && half == 0)
      c.scale[(size_t)cur.op.dst_slot * c.slot_scale + (size_t)p * C + cur.cat] = (uint16_t)s_out;
    // later steps bulk-copy this output from global memory
    asm volatile("fence.proxy.async.global;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    if (late >= 0 && warp == 0 && elect_one()) issue_late(c, nxt, late, sL0, sL1, tile, bar_land);
    if (has_next && nxt.cat == 0 && act) {  // the next op's tip state codes
      st_l = nxt.op.l_kind == GEMS_CHILD_TIP ? c.tips[(size_t)nxt.op.l_id * c.P + p] : 0;
      st_r = nxt.op.r_kind == GEMS_CHILD_TIP ? c.tips[(size_t)nxt.op.r_id * c.P + p] : 0;
    }
    cur = nxt;
  }
  if (!ok && t == 0) {
    if (land_pending) mbar_wait(bar_land, ph_land);
    if (b_pending) mbar_wait(bar_b, ph_b);
    if (mma_pending) mbar_wait(bar_mma, ph_mma);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols61);
}

size_t tc61_smem() { return 4 * (size_t)kATile + 2 * (size_t)kBSide + sizeof(Tc61Shared) + 64; }

// ---------------------------------------------------------------------------------------
// Warp-role form: the parts of a step run in different warps, on different steps at once, so
// that the split of step s+1, the MMAs of step s and the epilogue of step s-1 overlap (the form
// above runs them one after the other in every warp, and the tensor pipe idles through the split
// and the epilogue).
//   warps 0-3, split: one thread per pattern row.  Waits for the operand tiles of step s in
//     landing buffer s&1 and splits each internal child's row: hi -> TMEM A_hi[s&1][side], lo
//     written back in place (the landing buffer is then the lo operand of the MMAs).
//   warps 4-11, epilogue: two threads per pattern row, 32 states each (warps w and w+4 share
//     TMEM lane quadrant w%4).  A tip child's message is its tip table row, read from global
//     memory (L1-cached: the rows of one table are shared by the patterns of a tile) before the
//     wait; waits for the MMAs of step s, reads D[s&1] and frees it; products, the row maximum
//     over both halves (exchanged in shared memory), SAFE rescaling.  The rows go into a 32 KB
//     staging buffer, so that no per-thread global store sits in the SM's memory path beside
//     the copies and MMAs.  The epilogue is the longest part of a step, so it has the most
//     warps.
//   warp 14, stores: one bulk store of the staged rows per step; once it has read the staging
//     buffer the epilogue may fill it again, and once it has completed the number of steps
//     stored is published.
//   warp 12, copies: the operand tiles of step s into landing buffer s&1, once the MMAs of
//     step s-2 are done with it and every step that wrote one of those children has published
//     its stores; the B images of internal sides, in step order, into a ring of two 32 KB slots.
//   warp 13, MMAs: step s into D[s&1] once its split is done, its B images have landed and the
//     epilogue of step s-2 has read D[s&1]; a commit per side frees its ring slot, a commit per
//     step signals the epilogue and the copies.
// TMEM: D[b][side] at columns b*128 + side*64, A_hi[b][side] at 256 + b*128 + side*64 (512).
// Shared memory: landing buffers [2][2 sides][32 KB], the ring [2][32 KB] and the staging
// buffer: 224 KB; 480 threads.  The products, the split and the summation order are those of
// the form above: the same bits.  Every wait is bounded and also gives up once another role has
// failed (err); on failure the copy, MMA and store warps wait (bounded) for what they have in
// flight before TMEM and shared memory are released.
// ---------------------------------------------------------------------------------------
constexpr int kWsThreads = 480;
constexpr int kWsEpi = 256;  // epilogue threads
constexpr int kWsSlots = 2;
constexpr int kWsTmemCols = 512;
constexpr int kWsAhi = 256;

struct Ws61Shared {
  uint64_t full_land[2], split_done[2], mma_done[2], epi_done[2];
  uint64_t full_slot[kWsSlots], slot_free[kWsSlots];
  uint64_t drain;  // MMAs in flight when a role failed
  uint64_t staged, stage_free;  // the staging buffer holds a step's rows / has been read
  uint32_t tmem_base;
  int n_stored;  // steps whose rows are stored and fenced for the async proxy
  int err;       // set by the first role whose wait expired
  float rowmax[2][2][kTile];  // epilogue: each half's row maximum, by step parity
};

__device__ __forceinline__ void ws_fail(int *err, int *flag) {
  *(volatile int *)err = 1;
  atomicExch(flag, GEMS_ERR_TIMEOUT);
}
// (op, category) of consecutive steps
struct StepIt {
  int k, cat;
  DevOp op;
};
__device__ __forceinline__ void step_next(StepIt &it, const DevOp *ops, int nops, int C) {
  if (++it.cat == C) {
    it.cat = 0;
    if (++it.k < nops) it.op = ops[it.k];
  }
}

__global__ void __launch_bounds__(kWsThreads, 1)
    k_traverse_tc61ws(const TcJob *__restrict__ jobs, int nops, size_t stride_f, int *flag,
                      int tile0) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *land = smem_raw;               // [buffer][side][32 KB]
  unsigned char *ring = smem_raw + 4 * kATile;  // [slot][hi 16 KB, lo 16 KB]
  unsigned char *stage = ring + kWsSlots * kBSide;  // output rows of one step (epilogue)
  Ws61Shared *ctl = reinterpret_cast<Ws61Shared *>(stage + kATile);
  const int t = threadIdx.x, warp = t >> 5;
  if (t == 0) {
    for (int b = 0; b < 2; b++) {
      mbar_init(sptr(&ctl->full_land[b]), 1);
      mbar_init(sptr(&ctl->split_done[b]), kTile);
      mbar_init(sptr(&ctl->mma_done[b]), 1);
      mbar_init(sptr(&ctl->epi_done[b]), kWsEpi);
    }
    for (int q = 0; q < kWsSlots; q++) {
      mbar_init(sptr(&ctl->full_slot[q]), 1);
      mbar_init(sptr(&ctl->slot_free[q]), 1);
    }
    mbar_init(sptr(&ctl->drain), 1);
    mbar_init(sptr(&ctl->staged), kWsEpi);
    mbar_init(sptr(&ctl->stage_free), 1);
    ctl->n_stored = 0;
    ctl->err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(sptr(&ctl->tmem_base), kWsTmemCols);
  fence_before();
  __syncthreads();
  fence_after();
  const TcJob &job = jobs[blockIdx.y];  // read in place: the shared memory is all in use
  const DevCtx &c = job.c;
  const DevOp *ops = job.ops;
  const float *tab = job.tab;
  const int C = c.C;
  const int tile = tile0 + blockIdx.x;
  const uint32_t tmem = ctl->tmem_base;
  const int nsteps = nops * C;
  int *err = &ctl->err;

  if (warp < 4) {
    // ---- split
    const int row = t;
    const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
    StepIt it{0, 0, ops[0]};
    for (int s = 0; s < nsteps; s++) {
      const int b = s & 1;
      const bool inL = it.op.l_kind == GEMS_CHILD_PARTIAL, inR = it.op.r_kind == GEMS_CHILD_PARTIAL;
      if (__any_sync(0xffffffffu, !ws_wait(sptr(&ctl->full_land[b]), (s >> 1) & 1, err))) {
        ws_fail(err, flag);
        break;
      }
      fence_after();
#pragma unroll
      for (int side = 0; side < 2; side++) {
        if (!(side ? inR : inL)) continue;
        float4 *a4 = reinterpret_cast<float4 *>(land + (size_t)(2 * b + side) * kATile);
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
          float h[32];
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const int ch = 8 * hh + i;
            float4 hv, lv;
            split4(a4[ch * kTile + row], hv, lv);
            a4[ch * kTile + row] = lv;
            h[4 * i] = hv.x;
            h[4 * i + 1] = hv.y;
            h[4 * i + 2] = hv.z;
            h[4 * i + 3] = hv.w;
          }
          tmem_st32(tmem + lane_off + (uint32_t)(kWsAhi + b * 128 + side * kNP + 32 * hh), h);
        }
      }
      tmem_st_wait();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      fence_before();
      mbar_arrive(sptr(&ctl->split_done[b]));
      step_next(it, ops, nops, C);
    }
  } else if (warp < 12) {
    // ---- epilogue
    const int ew = warp - 4;
    const int row = ((ew & 3) << 5) | (t & 31);
    const int half = ew >> 2;  // states [32 half, 32 half + 32)
    const uint32_t lane_off = (uint32_t)((ew & 3) * 32) << 16;
    const long p = (long)tile * kTile + row;
    const bool act = p < c.P;
    const bool inv0 = act ? c.invar[p] == 0.0 : false;
    StepIt it{0, 0, ops[0]};
    int st_l = 0, st_r = 0;
    bool stale_prev = false;  // the previous step's staging wait failed
    for (int s = 0; s < nsteps; s++) {
      const int b = s & 1;
      const DevOp op = it.op;
      const bool inL = op.l_kind == GEMS_CHILD_PARTIAL, inR = op.r_kind == GEMS_CHILD_PARTIAL;
      if (it.cat == 0 && act) {  // tip state codes of a new op
        st_l = inL ? 0 : c.tips[(size_t)op.l_id * c.P + p];
        st_r = inR ? 0 : c.tips[(size_t)op.r_id * c.P + p];
      }
      int scl = 0, scr = 0;
      if (act) {
        if (inL) scl = c.scale[(size_t)op.l_id * c.slot_scale + (size_t)p * C + it.cat];
        if (inR) scr = c.scale[(size_t)op.r_id * c.slot_scale + (size_t)p * C + it.cat];
      }
      // messages: a tip child's from its table row (loaded before the wait), an internal
      // child's from its accumulator
      uint32_t rm[2][32];
      const float *tk = tab + (size_t)it.k * stride_f;
#pragma unroll
      for (int side = 0; side < 2; side++) {
        if (side ? inR : inL) continue;
        const int st = side ? st_r : st_l;
        const float4 *tr = reinterpret_cast<const float4 *>(
                               tk + ((size_t)side * C + it.cat) * (kBSide / 4) +
                               (size_t)(st < kN ? st : kN) * kTipRow61) + 8 * half;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const float4 q = __ldg(tr + i);
          rm[side][4 * i] = __float_as_uint(q.x);
          rm[side][4 * i + 1] = __float_as_uint(q.y);
          rm[side][4 * i + 2] = __float_as_uint(q.z);
          rm[side][4 * i + 3] = __float_as_uint(q.w);
        }
      }
      const bool bad = __any_sync(0xffffffffu, !ws_wait(sptr(&ctl->mma_done[b]), (s >> 1) & 1, err));
      float v[32];
      if (!bad) {
        fence_after();
#pragma unroll
        for (int side = 0; side < 2; side++)
          if (side ? inR : inL)
            tmem_ld32(tmem + lane_off + (uint32_t)(b * 128 + side * kNP + 32 * half), rm[side]);
#pragma unroll
        for (int side = 0; side < 2; side++)
          if (side ? inR : inL) tmem_ld32_wait(rm[side]);
        // D[b] has been read: the MMAs of step s+2 may overwrite it
        fence_before();
        mbar_arrive(sptr(&ctl->epi_done[b]));
        float mx = 0.f;
#pragma unroll
        for (int i = 0; i < 32; i++) {
          v[i] = fmaxf(__uint_as_float(rm[0][i]), 0.f) * fmaxf(__uint_as_float(rm[1][i]), 0.f);
          mx = fmaxf(mx, v[i]);
        }
        ctl->rowmax[b][half][row] = mx;
      }
      // every thread agrees on a failure; both halves' maxima are in place
      if (bar_or<1, kWsEpi>(bad || stale_prev)) {
        ws_fail(err, flag);
        break;
      }
      const float m = fmaxf(ctl->rowmax[b][0][row], ctl->rowmax[b][1][row]);
      int s_out = scl + scr;
      float f = 1.f;
      if ((inL || inR) && m < kScaleThrF && inv0) {
        f = 18446744073709551616.0f;  // 2^64
        s_out += 1;
      }
      if (act && half == 0)
        c.scale[(size_t)op.dst_slot * c.slot_scale + (size_t)p * C + it.cat] = (uint16_t)s_out;
      // the rows go out through the staging buffer and one bulk store (issued by the store
      // warp), which keeps the global stores out of the epilogue's way; the next steps' copies
      // read them through the same (async) proxy.  The previous step's store has read the
      // staging buffer first.
      const bool stale = s > 0 && __any_sync(0xffffffffu, !ws_wait(sptr(&ctl->stage_free), (s - 1) & 1, err));
      if (stale) ws_fail(err, flag);
#pragma unroll
      for (int i = 0; i < 8 && !stale; i++) {
        const int x = 32 * half + 4 * i;
        float4 w = make_float4(v[4 * i] * f, v[4 * i + 1] * f, v[4 * i + 2] * f, v[4 * i + 3] * f);
        if (x + 3 >= kN) {  // padding states stored as zeros
          if (x + 1 >= kN) w.y = 0.f;
          if (x + 2 >= kN) w.z = 0.f;
          if (x + 3 >= kN) w.w = 0.f;
          if (x >= kN) w.x = 0.f;
        }
        reinterpret_cast<float4 *>(stage)[(8 * half + i) * kTile + row] = w;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      // this thread's rows are staged: the store warp waits for all of them (a failed wait is
      // agreed on at the next step's barrier)
      mbar_arrive(sptr(&ctl->staged));
      stale_prev = stale;
      step_next(it, ops, nops, C);
    }
  } else if (warp == 14) {
    // ---- bulk stores of the staged rows, and the count of steps stored
    if (elect_one()) {
      float *part = static_cast<float *>(c.partials);
      StepIt it{0, 0, ops[0]};
      for (int s = 0; s < nsteps; s++) {
        if (!ws_wait(sptr(&ctl->staged), s & 1, err)) {
          ws_fail(err, flag);
          break;
        }
        bulk_s2g(part + (size_t)it.op.dst_slot * c.slot_elems + mix_off<61>(c, (long)tile * kTile, it.cat),
                 sptr(stage), kATile);
        bulk_commit();
        bulk_wait_read<0>();
        mbar_arrive(sptr(&ctl->stage_free));
        // the rows are in global memory: publish the step (this warp has nothing else to do
        // until the next step is staged)
        bulk_wait<0>();
        asm volatile("fence.proxy.async.global;" ::: "memory");
        st_release_s(&ctl->n_stored, s + 1);
        step_next(it, ops, nops, C);
      }
      bulk_wait<0>();
    }
    __syncwarp();
  } else if (warp == 12) {
    // ---- copies
    if (elect_one()) {
      float *part = static_cast<float *>(c.partials);
      StepIt it{0, 0, ops[0]};
      int d1 = -1, d2 = -1, d3 = -1;  // destination slots of the three previous ops
      int nimg = 0;
      bool ok = true;
      bool land_armed[2] = {false, false}, slot_armed[kWsSlots] = {};
      uint32_t land_par[2] = {0, 0}, slot_par[kWsSlots] = {};
      for (int s = 0; s < nsteps && ok; s++) {
        const int b = s & 1, u = s >> 1;
        const DevOp &op = it.op;
        const bool in[2] = {op.l_kind == GEMS_CHILD_PARTIAL, op.r_kind == GEMS_CHILD_PARTIAL};
        const int id[2] = {op.l_id, op.r_id};
        // landing buffer b: the MMAs of step s-2 have read it
        if (u >= 1 && !ws_wait(sptr(&ctl->mma_done[b]), (u - 1) & 1, err)) {
          ok = false;
          break;
        }
        // the children's rows of this category: stored by the step that wrote them (an op at
        // most three back is waited for exactly, older ones by the step four ops back)
        int need = 0;
        for (int side = 0; side < 2; side++) {
          if (!in[side]) continue;
          const int back = id[side] == d1 ? 1 : (id[side] == d2 ? 2 : (id[side] == d3 ? 3 : 4));
          need = max(need, s - back * C + 1);
        }
        if (need > 0 && !wait_count(&ctl->n_stored, need, err)) {
          ok = false;
          break;
        }
        const uint32_t fl = sptr(&ctl->full_land[b]);
        mbar_expect_tx(fl, (uint32_t)((in[0] ? kATile : 0) + (in[1] ? kATile : 0)));
        land_armed[b] = true;
        land_par[b] = u & 1;
        for (int side = 0; side < 2; side++)
          if (in[side])
            bulk_g2s(sptr(land + (size_t)(2 * b + side) * kATile),
                     part + (size_t)id[side] * c.slot_elems + mix_off<61>(c, (long)tile * kTile, it.cat),
                     kATile, fl);
        // B images of the internal sides, in ring order
        for (int side = 0; side < 2 && ok; side++) {
          if (!in[side]) continue;
          const int q = nimg % kWsSlots, uu = nimg / kWsSlots;
          if (uu >= 1 && !ws_wait(sptr(&ctl->slot_free[q]), (uu - 1) & 1, err)) {
            ok = false;
            break;
          }
          const uint32_t fs = sptr(&ctl->full_slot[q]);
          mbar_expect_tx(fs, (uint32_t)kBSide);
          slot_armed[q] = true;
          slot_par[q] = uu & 1;
          bulk_g2s(sptr(ring + (size_t)q * kBSide),
                   tab + (size_t)it.k * stride_f + ((size_t)side * C + it.cat) * (kBSide / 4),
                   kBSide, fs);
          nimg++;
        }
        if (it.cat + 1 == C) {
          d3 = d2;
          d2 = d1;
          d1 = op.dst_slot;
        }
        step_next(it, ops, nops, C);
      }
      if (!ok) {
        ws_fail(err, flag);
        // the copies issued must land before the CTA's shared memory is released
        for (int b = 0; b < 2; b++)
          if (land_armed[b]) mbar_wait(sptr(&ctl->full_land[b]), land_par[b]);
        for (int q = 0; q < kWsSlots; q++)
          if (slot_armed[q]) mbar_wait(sptr(&ctl->full_slot[q]), slot_par[q]);
      }
    }
    __syncwarp();
  } else if (warp == 13) {
    // ---- MMAs
    if (elect_one()) {
      StepIt it{0, 0, ops[0]};
      int nimg = 0;
      bool ok = true;
      bool slot_used[kWsSlots] = {};
      uint32_t slot_par[kWsSlots] = {};
      for (int s = 0; s < nsteps && ok; s++) {
        const int b = s & 1, u = s >> 1;
        const bool in[2] = {it.op.l_kind == GEMS_CHILD_PARTIAL, it.op.r_kind == GEMS_CHILD_PARTIAL};
        if (!ws_wait(sptr(&ctl->split_done[b]), u & 1, err) ||
            (u >= 1 && !ws_wait(sptr(&ctl->epi_done[b]), (u - 1) & 1, err))) {
          ok = false;
          break;
        }
        fence_after();
        for (int side = 0; side < 2; side++) {
          if (!in[side]) continue;
          const int q = nimg % kWsSlots, uu = nimg / kWsSlots;
          if (!ws_wait(sptr(&ctl->full_slot[q]), uu & 1, err)) {
            ok = false;
            break;
          }
          const uint32_t dtm = tmem + (uint32_t)(b * 128 + side * kNP);
          const uint32_t atm = tmem + (uint32_t)(kWsAhi + b * 128 + side * kNP);
          const uint64_t dB = sdesc(sptr(ring + (size_t)q * kBSide), kNP * 16, 128);
          const uint64_t dLo = sdesc(sptr(land + (size_t)(2 * b + side) * kATile), kAChunk, 128);
#pragma unroll
          for (int ks = 0; ks < kNP / 8; ks++) {
            const uint64_t kb = (uint64_t)((2 * ks * kNP * 16) >> 4);
            const uint64_t ko = (uint64_t)((2 * ks * kAChunk) >> 4);
            const uint64_t bh = dB + kb, bl = dB + kb + (uint64_t)(kBImg >> 4);
            mma_ts(dtm, atm + 8 * ks, bh, kIdesc61, ks > 0 ? 1u : 0u);
            mma_ts(dtm, atm + 8 * ks, bl, kIdesc61, 1u);
            mma_ss(dtm, dLo + ko, bh, kIdesc61, 1u);
          }
          mma_commit(sptr(&ctl->slot_free[q]));
          slot_used[q] = true;
          slot_par[q] = uu & 1;
          nimg++;
        }
        if (!ok) break;
        mma_commit(sptr(&ctl->mma_done[b]));
        step_next(it, ops, nops, C);
      }
      if (!ok) ws_fail(err, flag);
      // every MMA has completed (and every commit has arrived) before TMEM and shared memory
      // are released
      for (int q = 0; q < kWsSlots; q++)
        if (slot_used[q]) mbar_wait(sptr(&ctl->slot_free[q]), slot_par[q]);
      mma_commit(sptr(&ctl->drain));
      mbar_wait(sptr(&ctl->drain), 0);
    }
    __syncwarp();
  }
  fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kWsTmemCols);
}

size_t tc61ws_smem() {
  return 5 * (size_t)kATile + kWsSlots * (size_t)kBSide + sizeof(Ws61Shared) + 64;
}

}  // namespace

size_t tc61_op_floats(int ncat) { return op_floats61(ncat); }

bool tc61_supported(const Session *s) {
  return s->desc.nstates == 61 && s->desc.precision == GEMS_PREC_MIXED &&
         s->desc.scaling == GEMS_SCALE_SAFE && s->tc_enabled && s->tiled;
}

// op tables of `njobs` sessions that share one op list and category count, one launch on s0's
// stream: jobs on the device (njobs > 1) or the single job `one`
static int prep61(Session *s0, const TcJob &one, const TcJob *jobs, int njobs, int nops) {
  const size_t smem = sizeof(double) * prep61_smem_doubles(s0->desc.ncat);
  // the limit is a per-kernel attribute shared by every thread of the process: always set to
  // the largest size (kMaxCat categories)
  GEMS_CUDA(cudaFuncSetAttribute(k_prep_ops_tc61, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * prep61_smem_doubles(kMaxCat))));
  k_prep_ops_tc61<<<dim3(nops, 2, njobs), kPrepThreads, smem, s0->stream>>>(one, jobs,
                                                                            s0->op_stride_tc);
  s0->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

int launch_prep_ops_tc61(Session *s, int nops) {
  if (nops <= 0) return GEMS_OK;
  const TcJob one{s->ctx(), s->d_ops, reinterpret_cast<const float *>(s->d_opmats)};
  return prep61(s, one, nullptr, 1, nops);
}

// one launch over the tiles of every session in `ss` (all with the same op list, pattern
// count, categories and device), on the stream of ss[0]; with_tables: the sessions' op tables
// are built first, by one launch over every (session, op, side)
int launch_traverse_tc61_batch(Session *const *ss, int nsess, int nops, int p0, int p1,
                               bool with_tables) {
  if (nops <= 0 || nsess <= 0 || p1 <= p0) return GEMS_OK;
  Session *s0 = ss[0];
  if (p0 % kTile != 0 || (p1 % kTile != 0 && p1 != s0->P)) {
    set_error("tcgen05 61-state traversal: pattern range not aligned to its 128-pattern tiles");
    return GEMS_ERR_BAD_ARG;
  }
  if (nsess > Session::kMaxBatch) {
    set_error("too many sessions in one batched launch");
    return GEMS_ERR_BAD_ARG;
  }
  std::vector<TcJob> jobs(nsess);
  for (int i = 0; i < nsess; i++) {
    jobs[i].c = ss[i]->ctx();
    jobs[i].ops = ss[i]->d_ops;
    jobs[i].tab = reinterpret_cast<const float *>(ss[i]->d_opmats);
  }
  // host staging (pinned), then one copy; the previous launch that read it has completed
  GEMS_CUDA(cudaStreamSynchronize(s0->stream));
  std::memcpy(s0->h_jobs, jobs.data(), sizeof(TcJob) * nsess);
  GEMS_CUDA(cudaMemcpyAsync(s0->d_jobs, s0->h_jobs, sizeof(TcJob) * nsess,
                            cudaMemcpyHostToDevice, s0->stream));
  if (with_tables)
    if (int st = prep61(s0, jobs[0], nsess > 1 ? s0->d_jobs : nullptr, nsess, nops)) return st;
  const bool roles = s0->tc61_roles;
  const size_t smem = roles ? tc61ws_smem() : tc61_smem();
  if (roles)
    GEMS_CUDA(cudaFuncSetAttribute(k_traverse_tc61ws, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  else
    GEMS_CUDA(cudaFuncSetAttribute(k_traverse_tc61, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  GEMS_CUDA(cudaMemsetAsync(s0->d_flag, 0, sizeof(int), s0->stream));
  const int tile0 = p0 / kTile;
  const dim3 grid((p1 + kTile - 1) / kTile - tile0, nsess);
  cudaEvent_t ev0;
  if (int st = prof_begin(s0, 0, &ev0)) return st;
  if (roles)
    k_traverse_tc61ws<<<grid, kWsThreads, smem, s0->stream>>>(
        reinterpret_cast<const TcJob *>(s0->d_jobs), nops, s0->op_stride_tc, s0->d_flag, tile0);
  else
    k_traverse_tc61<<<grid, kThreads61, smem, s0->stream>>>(
        reinterpret_cast<const TcJob *>(s0->d_jobs), nops, s0->op_stride_tc, s0->d_flag, tile0);
  s0->launches++;
  GEMS_CUDA(cudaGetLastError());
  if (int st = prof_end(s0, 0, ev0)) return st;
  int flag = 0;
  GEMS_CUDA(cudaMemcpyAsync(&flag, s0->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s0->stream));
  GEMS_CUDA(cudaStreamSynchronize(s0->stream));
  if (flag) {
    set_error("tensor-core traversal: bounded wait expired");
    return GEMS_ERR_TIMEOUT;
  }
  return GEMS_OK;
}

int launch_traverse_tc61(Session *s, int nops, int p0, int p1) {
  Session *one[1] = {s};
  return launch_traverse_tc61_batch(one, 1, nops, p0, p1, false);
}

}  // namespace gems
