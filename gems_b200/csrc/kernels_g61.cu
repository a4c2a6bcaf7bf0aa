// kernels_g61.cu -- FP64 traversal for 61 states (codon models) as register-tiled GEMMs.
//
// The node update of the reference (tree/phylokernelnew.h:1911-2035) per (pattern, category)
// row is
//     out = inv_evec . ((E_L,c . L) * (E_R,c . R)),   E_c = evec . diag(exp(eval r_c t)).
// Over a tile of rows each product is a GEMM: V = L . E_c^T (K = N = 61) for the rows of
// category c, and out = T . inv_evec^T for all rows.  The products and their summation order
// are those of the per-row form (fma over the contraction index in ascending order), so the
// values are the generic kernel's bit for bit.  (The factored form evec . (d (*) L) of the 4- and
// 20-state kernels was tried here: with 61 states the eigen-space sums cancel heavily, and on
// a 160-taxon tree with long branches it moved partials by up to 2.5e-8 of their pattern's
// largest value, measured in plain FP64 numpy as well.)
//
// Two kernels share the per-op tables (prep) and the row layout of the partial slots:
// - k_traverse_g61m (SAFE scaling): the GEMMs on the FP64 tensor cores (mma.sync m8n8k4 f64),
//   one CTA per tile of 64 patterns of ONE category -- categories are independent under SAFE
//   scaling -- so that a CTA reads one E table per side and op (32 KB) instead of C of them;
// - k_traverse_g61 (NORM scaling, whose per-pattern maximum spans the categories): FP64 FMA,
//   one CTA per tile of up to 64 rows = tp patterns x C categories (tp = 64 / C rounded down to
//   a multiple of 8), stored category-major (row = c * tp + pattern), 128 threads as 8 x 16:
//   thread (ty, tx) owns rows ty*8..ty*8+7 -- all of one category -- and columns tx, tx+16,
//   tx+32, tx+48 (32 FP64 accumulators).
// Both: two CTAs per SM, so that one's loads overlap the other's GEMMs; the A operand of a child
// (its partial rows) staged k-major in shared memory; inv_evec^T in shared memory for the whole
// traversal; E_c^T read through L1 from the op table (stored [side][c][k][64 columns] by the
// prep kernel) and prefetched into L1 while the child's rows load.  A tip child's V is a row of
// the op's leaf table (E_c . tip vector), gathered by state.  The tensor-core products come out
// bit-identical to the FMA ones (the tests compare every partial).  Measured on one 200-taxon
// codon model (3,780 patterns): per-row kernel 26.6 ms (+G4); FMA tiles of 128 rows 7.0 ms, with
// the L1 prefetch 5.9 ms, 64-row tiles at two CTAs per SM 5.3 ms; tensor cores with mixed
// categories per tile 5.9 ms (spills), one category per tile 4.7 ms (+R8: 11.9 -> 9.6 ms).
#include <string>

#include "gems_internal.cuh"

namespace gems {

namespace {

constexpr int kN = 61;
constexpr int kK = 64;       // padded contraction length (MMA k-steps of 4)
constexpr int kNC = 64;      // padded output columns
constexpr int kRows = 64;    // rows per tile
constexpr int kSaLd = kRows + 2;
constexpr int kMaxCatG = 8;
constexpr int kThreadsG = 2 * kRows;  // 8 rows x 4 columns per thread
constexpr size_t kSmemG = sizeof(double) * ((size_t)kK * kNC + (size_t)kK * kSaLd + kRows);

// patterns per tile: 64 / C rounded down to a multiple of 8, so that the 8 rows of a thread
// (category-major rows) belong to one category
__host__ __device__ constexpr int tile_patterns(int C) { return kRows / C / 8 * 8; }

// per-op table (doubles): Et[2][C][kK][kNC] (Et[side][c][i][x] = E_c[x][i], zero padded), then
// leaf[2][unknown + 1][C][61]
__host__ __device__ constexpr size_t et_doubles(int C) { return (size_t)C * kK * kNC; }

__global__ void k_prep_ops_g61(DevCtx c, const DevOp *ops, double *tab, size_t stride) {
  __shared__ double dsh[kMaxCatG * kN];
  const int k = blockIdx.x, side = blockIdx.y;
  const DevOp op = ops[k];
  const int kind = side ? op.r_kind : op.l_kind;
  const double len = side ? op.r_len : op.l_len;
  const int C = c.C, blk = C * kN;
  for (int idx = threadIdx.x; idx < blk; idx += blockDim.x) {
    const int cc = idx / kN, i = idx - cc * kN;
    dsh[idx] = exp(c.eval[i] * (c.rates[cc] * len));
  }
  __syncthreads();
  double *et = tab + (size_t)k * stride + (size_t)side * et_doubles(C);
  for (int idx = threadIdx.x; idx < (int)et_doubles(C); idx += blockDim.x) {
    const int cc = idx / (kK * kNC), r = idx - cc * (kK * kNC), i = r / kNC, x = r - i * kNC;
    et[idx] = (i < kN && x < kN) ? c.evec[x * kN + i] * dsh[cc * kN + i] : 0.0;
  }
  if (kind != GEMS_CHILD_TIP) return;
  double *leaf = tab + (size_t)k * stride + 2 * et_doubles(C) + (size_t)side * (c.unknown + 1) * blk;
  const int rows = c.unknown * blk;
  for (int idx = threadIdx.x; idx < rows; idx += blockDim.x) {
    const int s = idx / blk, r = idx - s * blk, cc = r / kN, x = r - cc * kN;
    const double *t = c.tip + (size_t)s * kN;
    double acc = 0.0;
    for (int i = 0; i < kN; i++) acc = fma(c.evec[x * kN + i] * dsh[cc * kN + i], t[i], acc);
    leaf[idx] = acc;
  }
  for (int idx = threadIdx.x; idx < blk; idx += blockDim.x) leaf[rows + idx] = 1.0;
}

// acc[j][q] = sum_k sA[k][ty*8 + j] * B[k][tx + 16 q], k ascending; B in global memory (read
// through L1) or shared memory
template <bool GLOBAL_B>
__device__ __forceinline__ void gemm_tile(const double *__restrict__ sA,
                                          const double *__restrict__ B, int ty, int tx,
                                          double (&acc)[8][4]) {
#pragma unroll
  for (int j = 0; j < 8; j++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[j][q] = 0.0;
#pragma unroll 2
  for (int k = 0; k < kK; k++) {
    double b[4];
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = GLOBAL_B ? __ldg(B + k * kNC + tx + 16 * q) : B[k * kNC + tx + 16 * q];
    const double2 *a2 = reinterpret_cast<const double2 *>(sA + k * kSaLd + ty * 8);
    double a[8];
#pragma unroll
    for (int h = 0; h < 4; h++) {
      const double2 t = a2[h];
      a[2 * h] = t.x;
      a[2 * h + 1] = t.y;
    }
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[j][q] = fma(a[j], b[q], acc[j][q]);
  }
}

// tile row -> (category, pattern within the tile) and back to the slot's pattern-major rows
struct TileMap {
  int C, tp, nrow;
  long p0, P;
  __device__ int cat(int r) const { return r / tp; }
  __device__ long pattern(int r) const { return p0 + (r - (r / tp) * tp); }
  __device__ bool valid(int r) const { return r < nrow && pattern(r) < P; }
  // offset of the row's first state in the slot
  __device__ size_t off(int r) const { return ((size_t)pattern(r) * C + cat(r)) * kN; }
};

// SAFE only: a tile of 64 patterns of one category (categories are independent under SAFE
// scaling), so a CTA reads one E table per side instead of C
struct TileMap1 {
  int C, tp, nrow, c0;
  long p0, P;
  __device__ int cat(int) const { return c0; }
  __device__ long pattern(int r) const { return p0 + r; }
  __device__ bool valid(int r) const { return p0 + r < P; }
  __device__ size_t off(int r) const { return ((size_t)(p0 + r) * C + c0) * kN; }
  __device__ int tile_row(int g) const { return g < kRows ? g : -1; }
  __device__ bool row_ok(int g) const { return g < kRows && p0 + g < P; }
  __device__ size_t slot_row(int g) const { return (size_t)(p0 + g) * C + c0; }
};

// V of one child for the thread's rows and columns, and its scale counts (per row: SAFE; the
// pattern's: NORM).  A partial child's GEMM leaves sA in use: the caller synchronises before
// the next write of sA.
template <bool SAFE>
__device__ __forceinline__ void child_v(const DevCtx &c, const TileMap &tm, int kind, int id,
                                        const double *et, const double *leaf, double *sA, int ty,
                                        int tx, double (&v)[8][4], int (&s)[8]) {
  if (kind == GEMS_CHILD_TIP) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int r = ty * 8 + j;
      const bool ok = tm.valid(r);
      const int st = ok ? min((int)c.tips[(size_t)id * c.P + tm.pattern(r)], c.unknown) : 0;
      const double *row = leaf + ((size_t)st * tm.C + tm.cat(r)) * kN;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int col = tx + 16 * q;
        v[j][q] = ok && col < kN ? __ldg(row + col) : 0.0;
      }
      s[j] = 0;
    }
    return;
  }
  // the rows of E_c^T this CTA will read, pulled into L1 while the child's rows load (the
  // GEMM's first touch of each row otherwise waits on L2: 7.0 -> 5.9 ms with 128-row tiles)
  {
    const char *e0 = reinterpret_cast<const char *>(et);
    const int lines = (int)(et_doubles(tm.C) * sizeof(double) / 128);
    for (int l = threadIdx.x; l < lines; l += blockDim.x)
      asm volatile("prefetch.global.L1 [%0];" ::"l"(e0 + (size_t)l * 128));
  }
  // sA[k][r] = L[r][k] for k < 61, zero elsewhere.  idx runs over (pattern, category, k) in
  // the slot's order, so consecutive threads read consecutive doubles; every load of a thread
  // is issued before the first store.
  const double *src = static_cast<const double *>(c.partials) + (size_t)id * c.slot_elems;
  constexpr int kPer = kRows * kK / kThreadsG;
  static_assert(kRows * kK % kThreadsG == 0, "whole loads per thread");
  double a[kPer];
#pragma unroll
  for (int u = 0; u < kPer; u++) {
    const int idx = threadIdx.x + u * kThreadsG;
    const int g = idx / kK, k = idx - g * kK;  // g = pattern-major row within the tile
    const int lp = g / tm.C, cc = g - lp * tm.C;
    a[u] = (g < tm.nrow && tm.p0 + lp < tm.P && k < kN)
               ? __ldcg(src + ((size_t)(tm.p0 + lp) * tm.C + cc) * kN + k)
               : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kPer; u++) {
    const int idx = threadIdx.x + u * kThreadsG;
    const int g = idx / kK, k = idx - g * kK;
    const int lp = g / tm.C, cc = g - lp * tm.C;
    if (g < tm.nrow) sA[k * kSaLd + cc * tm.tp + lp] = a[u];
  }
  const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int r = ty * 8 + j;
    const long p = tm.pattern(r);
    s[j] = tm.valid(r) ? (SAFE ? sc[(size_t)p * tm.C + tm.cat(r)] : sc[p]) : 0;
  }
  __syncthreads();
  // rows past the tile's (64 % C) have no category: any table will do, their A rows are zero
  const int cat = min(tm.cat(ty * 8), tm.C - 1);
  gemm_tile<true>(sA, et + (size_t)cat * kK * kNC, ty, tx, v);
}

template <bool SAFE>
__global__ void __launch_bounds__(kThreadsG, 2)
    k_traverse_g61(DevCtx c, const DevOp *__restrict__ ops, int nops,
                   const double *__restrict__ tab, size_t stride, int tile0) {
  extern __shared__ __align__(16) double smem[];
  double *sIv = smem;                  // [kK][kNC]: inv_evec[j][x] at [x][j]
  double *sA = sIv + kK * kNC;         // [kK][kSaLd]
  double *sMax = sA + kK * kSaLd;      // [kRows] row maxima (NORM)
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  TileMap tm;
  tm.C = c.C;
  tm.tp = tile_patterns(c.C);
  tm.nrow = tm.tp * c.C;
  tm.p0 = (long)(tile0 + blockIdx.x) * tm.tp;
  tm.P = c.P;
  for (int idx = tid; idx < kK * kNC; idx += blockDim.x) {
    const int k = idx / kNC, x = idx - k * kNC;
    sIv[idx] = (k < kN && x < kN) ? c.inv_evec[x * kN + k] : 0.0;
  }
  // rows of sA past the tile's rows (64 % C) are never written: zero them once
  for (int idx = tid; idx < kK * kSaLd; idx += blockDim.x) sA[idx] = 0.0;
  double *part = static_cast<double *>(c.partials);
  const int blk = c.C * kN;
  for (int kop = 0; kop < nops; kop++) {
    const DevOp op = ops[kop];
    const double *tk = tab + (size_t)kop * stride;
    const double *leafL = tk + 2 * et_doubles(c.C);
    const double *leafR = leafL + (size_t)(c.unknown + 1) * blk;
    const bool tiptip = op.l_kind == GEMS_CHILD_TIP && op.r_kind == GEMS_CHILD_TIP;
    double vl[8][4], o[8][4];
    int sl[8], sr[8];
    __syncthreads();  // sA free (previous op's last GEMM, or the set-up)
    child_v<SAFE>(c, tm, op.l_kind, op.l_id, tk, leafL, sA, ty, tx, vl, sl);
    __syncthreads();
    child_v<SAFE>(c, tm, op.r_kind, op.r_id, tk + et_doubles(c.C), leafR, sA, ty, tx, o, sr);
    __syncthreads();
    // T = V_L (*) V_R into sA (k-major); columns >= 61 of V are zero, so row 61 of T is zero
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int x = tx + 16 * q;
      if (x < kK) {
#pragma unroll
        for (int j = 0; j < 8; j++) sA[x * kSaLd + ty * 8 + j] = vl[j][q] * o[j][q];
      }
    }
    __syncthreads();
    gemm_tile<false>(sA, sIv, ty, tx, o);
    double m[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      double x = 0.0;
#pragma unroll
      for (int q = 0; q < 4; q++) x = fmax(x, fabs(o[j][q]));
      for (int off = 1; off < 16; off <<= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, off));
      m[j] = x;
    }
    if (!SAFE) {
      // the pattern's maximum over its C rows (rows c * tp + lp, in other threads)
      if (tx == 0) {
#pragma unroll
        for (int j = 0; j < 8; j++) sMax[ty * 8 + j] = m[j];
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int lp = (ty * 8 + j) % tm.tp;
        double x = 0.0;
        for (int u = 0; u < tm.C; u++) x = fmax(x, sMax[u * tm.tp + lp]);
        m[j] = x;
      }
    }
    uint16_t *scd = c.scale + (size_t)op.dst_slot * c.slot_scale;
    double *dst = part + (size_t)op.dst_slot * c.slot_elems;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int r = ty * 8 + j;
      if (!tm.valid(r)) continue;
      const long p = tm.pattern(r);
      const int cat = tm.cat(r);
      int s_out = sl[j] + sr[j];
      if (!tiptip && m[j] < kScaleThr && c.invar[p] == 0.0) {
#pragma unroll
        for (int q = 0; q < 4; q++) o[j][q] = ldexp(o[j][q], kScaleExp);
        s_out += 1;
      }
      double *row = dst + tm.off(r);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int col = tx + 16 * q;
        if (col < kN) row[col] = o[j][q];
      }
      if (tx == 0) {
        if (SAFE)
          scd[(size_t)p * tm.C + cat] = (uint16_t)s_out;
        else if (cat == 0)
          scd[p] = (uint16_t)s_out;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// The same traversal with the GEMMs on the FP64 tensor cores (mma.sync m8n8k4 f64: one warp
// instruction does 8 x 8 x 4 multiply-adds).  Warp w owns rows 16w..16w+15 as two 8-row blocks
// (each of one category, tp being a multiple of 8) and all 64 columns as eight 8-column blocks;
// lane l holds rows l/4 and columns 2(l%4), 2(l%4)+1 of each 8 x 8 block (the instruction's
// accumulator layout).  Operand rows in shared memory are 72 doubles apart, so that the four
// k-rows of a fragment load fall in two bank halves.
// ---------------------------------------------------------------------------------------
constexpr int kLdM = 72;
constexpr size_t kSmemM = sizeof(double) * 2 * (size_t)kK * kLdM;

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// acc[rb][cb] = A[rows of row block rb][k] . B_rb[k][columns of block cb] over k < kK, with
// A k-major in shared memory (row stride kLdM) and B_rb = B0 or B1 (row stride ldb)
template <bool GLOBAL_B>
__device__ __forceinline__ void gemm_mma(const double *__restrict__ sA,
                                         const double *__restrict__ B0,
                                         const double *__restrict__ B1, int ldb, int w, int lane,
                                         double (&acc)[2][8][2]) {
#pragma unroll
  for (int rb = 0; rb < 2; rb++)
#pragma unroll
    for (int cb = 0; cb < 8; cb++) acc[rb][cb][0] = acc[rb][cb][1] = 0.0;
  const int kr = lane & 3, rc = lane >> 2;
  const bool same = B0 == B1;
#pragma unroll 2
  for (int k0 = 0; k0 < kK; k0 += 4) {
    const double *ar = sA + (k0 + kr) * kLdM + 16 * w + rc;
    const double a0 = ar[0], a1 = ar[8];
    const double *b0 = B0 + (size_t)(k0 + kr) * ldb + rc;
    double bv[8];
#pragma unroll
    for (int cb = 0; cb < 8; cb++) bv[cb] = GLOBAL_B ? __ldg(b0 + 8 * cb) : b0[8 * cb];
#pragma unroll
    for (int cb = 0; cb < 8; cb++) dmma(acc[0][cb], a0, bv[cb]);
    if (same) {
#pragma unroll
      for (int cb = 0; cb < 8; cb++) dmma(acc[1][cb], a1, bv[cb]);
    } else {
      const double *b1 = B1 + (size_t)(k0 + kr) * ldb + rc;
#pragma unroll
      for (int cb = 0; cb < 8; cb++) bv[cb] = GLOBAL_B ? __ldg(b1 + 8 * cb) : b1[8 * cb];
#pragma unroll
      for (int cb = 0; cb < 8; cb++) dmma(acc[1][cb], a1, bv[cb]);
    }
  }
}

template <bool SAFE>
__device__ __forceinline__ void child_v_mma(const DevCtx &c, const TileMap1 &tm, int kind, int id,
                                            const double *et, const double *leaf, double *sA,
                                            int w, int lane, double (&v)[2][8][2], int (&s)[2]) {
  const int kr = lane & 3, rc = lane >> 2;
  if (kind == GEMS_CHILD_TIP) {
#pragma unroll
    for (int rb = 0; rb < 2; rb++) {
      const int r = 16 * w + 8 * rb + rc;
      const bool ok = tm.valid(r);
      const int st = ok ? min((int)c.tips[(size_t)id * c.P + tm.pattern(r)], c.unknown) : 0;
      const double *row = leaf + ((size_t)st * tm.C + tm.cat(r)) * kN;
#pragma unroll
      for (int cb = 0; cb < 8; cb++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int col = 8 * cb + 2 * kr + e;
          v[rb][cb][e] = ok && col < kN ? __ldg(row + col) : 0.0;
        }
      s[rb] = 0;
    }
    return;
  }
  {
    const char *e0 = reinterpret_cast<const char *>(et);
    const int lines = (int)(et_doubles(tm.C) * sizeof(double) / 128);
    for (int l = threadIdx.x; l < lines; l += blockDim.x)
      asm volatile("prefetch.global.L1 [%0];" ::"l"(e0 + (size_t)l * 128));
  }
  const double *src = static_cast<const double *>(c.partials) + (size_t)id * c.slot_elems;
  constexpr int kPer = kRows * kK / kThreadsG;
  static_assert(kRows * kK % kThreadsG == 0, "whole loads per thread");
  double a[kPer];
#pragma unroll
  for (int u = 0; u < kPer; u++) {
    const int idx = threadIdx.x + u * kThreadsG;
    const int g = idx / kK, k = idx - g * kK;
    a[u] = (tm.row_ok(g) && k < kN) ? __ldcg(src + tm.slot_row(g) * kN + k) : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kPer; u++) {
    const int idx = threadIdx.x + u * kThreadsG;
    const int g = idx / kK, k = idx - g * kK;
    const int r = tm.tile_row(g);
    if (r >= 0) sA[k * kLdM + r] = a[u];
  }
  const uint16_t *sc = c.scale + (size_t)id * c.slot_scale;
#pragma unroll
  for (int rb = 0; rb < 2; rb++) {
    const int r = 16 * w + 8 * rb + rc;
    const long p = tm.pattern(r);
    s[rb] = tm.valid(r) ? (SAFE ? sc[(size_t)p * tm.C + tm.cat(r)] : sc[p]) : 0;
  }
  __syncthreads();
  const double *b = et + (size_t)tm.c0 * kK * kNC;
  gemm_mma<true>(sA, b, b, kNC, w, lane, v);
}

template <bool SAFE>
__global__ void __launch_bounds__(kThreadsG, 2)
    k_traverse_g61m(DevCtx c, const DevOp *__restrict__ ops, int nops,
                    const double *__restrict__ tab, size_t stride, int tile0) {
  static_assert(SAFE, "one category per tile: SAFE scaling only");
  extern __shared__ __align__(16) double smem[];
  double *sIv = smem;                  // [kK][kLdM]: inv_evec[j][x] at [x][j]
  double *sA = sIv + kK * kLdM;        // [kK][kLdM]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, kr = lane & 3, rc = lane >> 2;
  TileMap1 tm;
  tm.C = c.C;
  tm.tp = kRows;
  tm.nrow = kRows;
  tm.c0 = blockIdx.x % c.C;
  tm.p0 = (long)(tile0 + blockIdx.x / c.C) * kRows;
  tm.P = c.P;
  for (int idx = threadIdx.x; idx < kK * kLdM; idx += blockDim.x) {
    const int k = idx / kLdM, x = idx - k * kLdM;
    sIv[idx] = (k < kN && x < kN) ? c.inv_evec[x * kN + k] : 0.0;
    sA[idx] = 0.0;  // rows past the tile's rows (64 % C) are never written
  }
  double *part = static_cast<double *>(c.partials);
  const int blk = c.C * kN;
  for (int kop = 0; kop < nops; kop++) {
    const DevOp op = ops[kop];
    const double *tk = tab + (size_t)kop * stride;
    const double *leafL = tk + 2 * et_doubles(c.C);
    const double *leafR = leafL + (size_t)(c.unknown + 1) * blk;
    const bool tiptip = op.l_kind == GEMS_CHILD_TIP && op.r_kind == GEMS_CHILD_TIP;
    double vl[2][8][2], o[2][8][2];
    int sl[2], sr[2];
    __syncthreads();
    child_v_mma<SAFE>(c, tm, op.l_kind, op.l_id, tk, leafL, sA, w, lane, vl, sl);
    __syncthreads();
    child_v_mma<SAFE>(c, tm, op.r_kind, op.r_id, tk + et_doubles(c.C), leafR, sA, w, lane, o, sr);
    __syncthreads();
#pragma unroll
    for (int rb = 0; rb < 2; rb++)
#pragma unroll
      for (int cb = 0; cb < 8; cb++)
#pragma unroll
        for (int e = 0; e < 2; e++)
          sA[(8 * cb + 2 * kr + e) * kLdM + 16 * w + 8 * rb + rc] = vl[rb][cb][e] * o[rb][cb][e];
    __syncthreads();
    gemm_mma<false>(sA, sIv, sIv, kLdM, w, lane, o);
    double m[2];
#pragma unroll
    for (int rb = 0; rb < 2; rb++) {
      double x = 0.0;
#pragma unroll
      for (int cb = 0; cb < 8; cb++) x = fmax(x, fmax(fabs(o[rb][cb][0]), fabs(o[rb][cb][1])));
      x = fmax(x, __shfl_xor_sync(0xffffffffu, x, 1));
      x = fmax(x, __shfl_xor_sync(0xffffffffu, x, 2));
      m[rb] = x;
    }
    uint16_t *scd = c.scale + (size_t)op.dst_slot * c.slot_scale;
    double *dst = part + (size_t)op.dst_slot * c.slot_elems;
#pragma unroll
    for (int rb = 0; rb < 2; rb++) {
      const int r = 16 * w + 8 * rb + rc;
      if (!tm.valid(r)) continue;
      const long p = tm.pattern(r);
      const int cat = tm.cat(r);
      int s_out = sl[rb] + sr[rb];
      const bool scale = !tiptip && m[rb] < kScaleThr && c.invar[p] == 0.0;
      if (scale) s_out += 1;
      double *row = dst + tm.off(r);
#pragma unroll
      for (int cb = 0; cb < 8; cb++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int col = 8 * cb + 2 * kr + e;
          if (col < kN) row[col] = scale ? ldexp(o[rb][cb][e], kScaleExp) : o[rb][cb][e];
        }
      if (kr == 0) scd[(size_t)p * tm.C + cat] = (uint16_t)s_out;
    }
  }
}

}  // namespace

size_t g61_op_doubles(int ncat, int unknown) {
  return 2 * et_doubles(ncat) + 2 * (size_t)(unknown + 1) * ncat * kN;
}

bool g61_supported(const Session *s) {
  const int C = s->desc.ncat;
  return s->g61_enabled && s->desc.precision == GEMS_PREC_FP64 && s->desc.nstates == kN &&
         C >= 1 && C <= kMaxCatG;
}

int launch_prep_ops_g61(Session *s, int nops) {
  if (nops <= 0) return GEMS_OK;
  k_prep_ops_g61<<<dim3(nops, 2), 256, 0, s->stream>>>(s->ctx(), s->d_ops, s->d_opmats,
                                                        s->op_stride);
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return GEMS_OK;
}

int g61_pattern_granule(const Session *s) {
  return s->desc.scaling == GEMS_SCALE_SAFE ? kRows : tile_patterns(s->desc.ncat);
}

int launch_traverse_g61(Session *s, int nops, int p0, int p1) {
  if (nops <= 0 || p1 <= p0) return GEMS_OK;
  const int tp = tile_patterns(s->desc.ncat);
  const bool safe = s->desc.scaling == GEMS_SCALE_SAFE;
  const int gran = safe ? kRows : tp;
  if (p0 % gran != 0 || (p1 % gran != 0 && p1 != s->P)) {
    set_error("FP64 61-state traversal: pattern range not aligned to its pattern tiles");
    return GEMS_ERR_BAD_ARG;
  }
  cudaEvent_t ev0;
  if (int st = prof_begin(s, 0, &ev0)) return st;
  const int tile0 = p0 / gran;
  const int grid = (p1 + tp - 1) / tp - tile0;
  // the limit is a per-kernel attribute shared by every thread of the process: always the same
  // value
  if (safe) {  // FP64 tensor cores, one category per tile
    const int g = ((p1 + kRows - 1) / kRows - tile0) * s->desc.ncat;
    GEMS_CUDA(cudaFuncSetAttribute(k_traverse_g61m<true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemM));
    k_traverse_g61m<true><<<g, kThreadsG, kSmemM, s->stream>>>(s->ctx(), s->d_ops, nops,
                                                                s->d_opmats, s->op_stride,
                                                                tile0);
  } else {  // NORM: a pattern's categories in one tile, FP64 FMA
    GEMS_CUDA(cudaFuncSetAttribute(k_traverse_g61<false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemG));
    k_traverse_g61<false><<<grid, kThreadsG, kSmemG, s->stream>>>(s->ctx(), s->d_ops, nops,
                                                                   s->d_opmats, s->op_stride,
                                                                   tile0);
  }
  s->launches++;
  GEMS_CUDA(cudaGetLastError());
  return prof_end(s, 0, ev0);
}

}  // namespace gems
