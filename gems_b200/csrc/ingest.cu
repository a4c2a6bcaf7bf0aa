// ingest.cu -- alignment ingest on the device: state encoding and pattern compression.
//
// The reference builds patterns on the host, one site after another (Alignment::buildPattern,
// alignment/alignment.cpp:1240-1268): each site's column of state codes is looked up in a hash
// map; a new column becomes the next pattern, a repeated one adds to that pattern's frequency
// (addPatternLazy, :1511-1543), and every new pattern gets its constant state (computeConst,
// :1321-1420).  The result is first-appearance order, which this file reproduces exactly, in
// parallel:
//   encode   characters -> state codes by a 256-entry table (convertState, :1856-1958)
//   hash     FNV-1a over each column
//   insert   open-addressing table: the first column to claim a slot represents its group;
//            later columns compare hash and bytes; each group keeps its smallest site index
//   first    a site is a pattern's first appearance iff it is its group's smallest site
//   scan     prefix sum over first appearances -> pattern ids in first-appearance order
//   assign   per site: pattern id, frequency (integer atomics), the pattern's first site
//   gather   pattern columns; const   the constant state of each pattern
// Every loop is bounded (the table has at least twice as many slots as sites).
#include <cstring>
#include <string>
#include <vector>

#include "gems_internal.cuh"

namespace gems {
namespace {

constexpr unsigned long long kEmpty = ~0ULL;

__global__ void k_encode(uint8_t *codes, const uint8_t *chars, size_t n, const uint8_t *lut,
                         unsigned long long *bad) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint8_t v = lut[chars[i]];
    if (v == 0xFF) atomicMin(bad, (unsigned long long)i);  // first bad position
    codes[i] = v;
  }
}

// FNV-1a (64-bit) over the column of site s
__global__ void k_hash(const uint8_t *codes, int ntaxa, long long nsites, unsigned long long *h) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsites) return;
  unsigned long long v = 1469598103934665603ULL;
  for (int t = 0; t < ntaxa; t++) {
    v ^= codes[(size_t)t * nsites + s];
    v *= 1099511628211ULL;
  }
  h[s] = v;
}

__global__ void k_insert(const uint8_t *codes, int ntaxa, long long nsites,
                         const unsigned long long *h, unsigned long long *tab,
                         unsigned long long *minsite, unsigned long long mask, long long *grp) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsites) return;
  const unsigned long long hs = h[s];
  unsigned long long slot = hs & mask;
  for (unsigned long long probe = 0; probe <= mask; probe++) {
    const unsigned long long old = atomicCAS(&tab[slot], kEmpty, (unsigned long long)s);
    bool mine = old == kEmpty;
    if (!mine && h[old] == hs) {
      mine = true;
      for (int t = 0; t < ntaxa && mine; t++)
        mine = codes[(size_t)t * nsites + s] == codes[(size_t)t * nsites + old];
    }
    if (mine) {
      grp[s] = (long long)slot;
      atomicMin(&minsite[slot], (unsigned long long)s);
      return;
    }
    slot = (slot + 1) & mask;
  }
}

__global__ void k_first(const long long *grp, const unsigned long long *minsite,
                        long long nsites, unsigned int *flag) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsites) return;
  const long long g = grp[s];  // -1 only if a site found no slot, which the table size excludes
  flag[s] = (g >= 0 && minsite[g] == (unsigned long long)s) ? 1u : 0u;
}

// exclusive scan of flag[] in blocks of 1024 (one element per thread): in-block scan, then the
// block totals are scanned by one block, then added
__global__ void k_scan_block(const unsigned int *in, long long n, long long *out,
                             long long *block_sum) {
  __shared__ long long sh[1024];
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  const long long v = i < n ? in[i] : 0;
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const long long a = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += a;
    __syncthreads();
  }
  if (i < n) out[i] = sh[threadIdx.x] - v;
  if (threadIdx.x == 1023) block_sum[blockIdx.x] = sh[1023];
}
__global__ void k_scan_sums(long long *block_sum, long long nblocks, long long *total) {
  if (threadIdx.x != 0) return;
  long long run = 0;
  for (long long b = 0; b < nblocks; b++) {
    const long long v = block_sum[b];
    block_sum[b] = run;
    run += v;
  }
  *total = run;
}
__global__ void k_scan_add(long long *out, long long n, const long long *block_sum) {
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += block_sum[blockIdx.x];
}

__global__ void k_assign(const long long *grp, const unsigned long long *minsite,
                         const long long *pid_at, long long nsites, int *site_pattern,
                         unsigned int *count, long long *rep) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsites) return;
  const long long g = grp[s];
  if (g < 0) {
    site_pattern[s] = -1;
    return;
  }
  const long long f = (long long)minsite[g];
  const long long p = pid_at[f];
  site_pattern[s] = (int)p;
  atomicAdd(&count[p], 1u);
  if (f == s) rep[p] = s;
}

__global__ void k_gather(const uint8_t *codes, int ntaxa, long long nsites, long long npat,
                         const long long *rep, uint8_t *pat) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npat) return;
  const long long s = rep[p];
  for (int t = 0; t < ntaxa; t++) pat[(size_t)t * npat + p] = codes[(size_t)t * nsites + s];
}

// states a code stands for, as a bit set (getAppearance, alignment.cpp:5567-5600)
__device__ __forceinline__ unsigned long long appearance(int code, int n) {
  const int unk = n == 4 ? 18 : (n == 20 ? 23 : n);
  const unsigned long long all = n == 64 ? ~0ULL : ((1ULL << n) - 1);
  if (code >= unk) return all;
  if (code < n) return 1ULL << code;
  if (n == 4) return (unsigned long long)(code - 3);
  // protein B = {N, D}, Z = {Q, E}, J = {I, L}
  return code == 20 ? 0xCULL : (code == 21 ? 0x60ULL : 0x600ULL);
}

// constant state of each pattern (computeConst, alignment.cpp:1321-1420): the intersection of
// the states its codes stand for -- all states: unknown; one state: that state; DNA: the
// ambiguity code of the set; protein: B / Z / J; empty: unknown + 1 (not constant)
__global__ void k_const(const uint8_t *pat, int ntaxa, long long npat, int n, uint8_t *cc) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npat) return;
  const int unk = n == 4 ? 18 : (n == 20 ? 23 : n);
  unsigned long long app = n == 64 ? ~0ULL : ((1ULL << n) - 1);
  for (int t = 0; t < ntaxa; t++) app &= appearance(pat[(size_t)t * npat + p], n);
  const int k = __popcll(app);
  int v = unk + 1;
  if (k == n) {
    v = unk;
  } else if (k == 1) {
    v = __ffsll((long long)app) - 1;
  } else if (k > 1 && n == 4) {
    v = n - 1 + (int)app;
  } else if (k > 1 && n == 20) {
    v = (app == 0xCULL) ? 20 : (app == 0x60ULL ? 21 : 22);
  }
  cc[p] = (uint8_t)v;
}

// characters -> codes (convertState): gaps and unknown symbols -> unknown, invalid -> 0xFF;
// lower case is read as upper case, as the reference upper-cases its sequences
void build_lut(int n, uint8_t *lut) {
  std::memset(lut, 0xFF, 256);
  const int unk = n == 4 ? 18 : 23;
  auto both = [&](char c, int v) {
    lut[(unsigned char)c] = (uint8_t)v;
    if (c >= 'A' && c <= 'Z') lut[(unsigned char)(c - 'A' + 'a')] = (uint8_t)v;
  };
  for (char c : {'?', '-', '.', '~'}) both(c, unk);
  if (n == 4) {
    const char *s = "ACGT";
    for (int i = 0; i < 4; i++) both(s[i], i);
    both('U', 3);
    both('R', 1 + 4 + 3);
    both('Y', 2 + 8 + 3);
    both('W', 1 + 8 + 3);
    both('S', 2 + 4 + 3);
    both('M', 1 + 2 + 3);
    both('K', 4 + 8 + 3);
    both('B', 2 + 4 + 8 + 3);
    both('H', 1 + 2 + 8 + 3);
    both('D', 1 + 4 + 8 + 3);
    both('V', 1 + 2 + 4 + 3);
    for (char c : {'O', 'N', 'X'}) both(c, unk);
  } else {
    const char *s = "ARNDCQEGHILKMFPSTWYV";
    for (int i = 0; i < 20; i++) both(s[i], i);
    both('B', 20);
    both('Z', 21);
    both('J', 22);
    for (char c : {'*', 'U', 'O', 'X'}) both(c, unk);
  }
}

}  // namespace

// ptn_invar of each pattern from its constant state (computePtnInvar,
// tree/phylotreesse.cpp:549-612): p_invar times the frequency of the states it stands for
struct FreqPack {
  double f[64];
};
__global__ void k_ptn_invar(const uint8_t *cc, long long npat, int n, double p_invar,
                            FreqPack fr, double *invar) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npat) return;
  const int unk = n == 4 ? 18 : (n == 20 ? 23 : n);
  const int c = cc[p];
  double v = 0.0;
  if (p_invar != 0.0 && c <= unk) {
    if (c == unk) {
      v = p_invar;
    } else if (c < n) {
      v = p_invar * fr.f[c];
    } else {
      const unsigned long long app = appearance(c, n);
      double acc = 0.0;
      for (int x = 0; x < n; x++)
        if (app & (1ULL << x)) acc += fr.f[x];
      v = acc * p_invar;
    }
  }
  invar[p] = v;
}
__global__ void k_counts(const unsigned int *count, long long npat, double *w) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < npat) w[p] = (double)count[p];
}

}  // namespace gems

using namespace gems;

// compressed alignment kept on the device
struct gems_ingest {
  int device = 0, ntaxa = 0, nstates = 0;
  long long nsites = 0, npat = 0;
  uint8_t *d_pat = nullptr, *d_cc = nullptr;
  unsigned int *d_count = nullptr;
  int *d_sp = nullptr;
  cudaStream_t st = nullptr;
};

extern "C" void gems_ingest_destroy(gems_ingest *g) {
  if (!g) return;
  cudaSetDevice(g->device);
  cudaFree(g->d_pat);
  cudaFree(g->d_cc);
  cudaFree(g->d_count);
  cudaFree(g->d_sp);
  if (g->st) cudaStreamDestroy(g->st);
  delete g;
}

extern "C" int gems_ingest_create(int device, int ntaxa, long long nsites, int nstates,
                                  const uint8_t *seqs, int encoded, gems_ingest **out,
                                  long long *npat_out) {
  if (!out || !npat_out || ntaxa < 1 || nsites < 1 || nsites > 0x7FFFFFFFLL || !seqs ||
      (nstates != 4 && nstates != 20 && nstates != 61) || (!encoded && nstates == 61)) {
    set_error("ingest: bad arguments (characters are read for 4 and 20 states)");
    return GEMS_ERR_BAD_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    set_error("no CUDA device");
    return GEMS_ERR_NO_DEVICE;
  }
  GEMS_CUDA(cudaSetDevice(device));
  gems_ingest *g = new gems_ingest();
  g->device = device;
  g->ntaxa = ntaxa;
  g->nstates = nstates;
  g->nsites = nsites;
  const size_t cells = (size_t)ntaxa * nsites;
  unsigned long long cap = 1;
  while (cap < 2ULL * (unsigned long long)nsites) cap <<= 1;
  const long long nblk = (nsites + 1023) / 1024;
  // working buffers, freed before returning
  uint8_t *d_raw = nullptr, *d_codes = nullptr, *d_lut = nullptr;
  unsigned long long *d_h = nullptr, *d_tab = nullptr, *d_min = nullptr, *d_bad = nullptr;
  long long *d_grp = nullptr, *d_pid = nullptr, *d_bsum = nullptr, *d_rep = nullptr;
  unsigned int *d_flag = nullptr;
  auto release = [&]() {
    cudaFree(d_raw); cudaFree(d_codes); cudaFree(d_lut); cudaFree(d_h); cudaFree(d_tab);
    cudaFree(d_min); cudaFree(d_bad); cudaFree(d_grp); cudaFree(d_pid); cudaFree(d_bsum);
    cudaFree(d_rep); cudaFree(d_flag);
  };
  auto fail = [&](cudaError_t e, const char *what) {
    const int code = cuda_status(e, what);
    release();
    gems_ingest_destroy(g);
    return code;
  };
  cudaError_t e;
#define ALLOC(p, bytes) \
  if ((e = cudaMalloc((void **)&(p), (bytes))) != cudaSuccess) return fail(e, "cudaMalloc " #p);
  ALLOC(d_codes, cells);
  if (!encoded) {
    ALLOC(d_raw, cells);
    ALLOC(d_lut, 256);
  }
  ALLOC(d_h, sizeof(unsigned long long) * nsites);
  ALLOC(d_tab, sizeof(unsigned long long) * cap);
  ALLOC(d_min, sizeof(unsigned long long) * cap);
  ALLOC(d_bad, sizeof(unsigned long long));
  ALLOC(d_grp, sizeof(long long) * nsites);
  ALLOC(d_pid, sizeof(long long) * nsites);
  ALLOC(d_bsum, sizeof(long long) * (nblk + 1));
  ALLOC(d_rep, sizeof(long long) * nsites);
  ALLOC(d_flag, sizeof(unsigned int) * nsites);
  ALLOC(g->d_count, sizeof(unsigned int) * nsites);
  ALLOC(g->d_sp, sizeof(int) * nsites);
#undef ALLOC
  if ((e = cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(e, "cudaStreamCreate");
  cudaStream_t st = g->st;
  const int T = 256;
  const unsigned gs = (unsigned)((nsites + T - 1) / T);
  unsigned long long bad = kEmpty;
  if (!encoded) {
    uint8_t lut[256];
    build_lut(nstates, lut);
    if ((e = cudaMemcpyAsync(d_raw, seqs, cells, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(d_lut, lut, 256, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(d_bad, &bad, sizeof(bad), cudaMemcpyHostToDevice, st)))
      return fail(e, "ingest upload");
    k_encode<<<1184, T, 0, st>>>(d_codes, d_raw, cells, d_lut, d_bad);
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
      return fail(e, "ingest encode");
    if (bad != kEmpty) {
      release();
      gems_ingest_destroy(g);
      set_error("ingest: unrecognised character in sequence " + std::to_string(bad / nsites) +
                " at site " + std::to_string(bad % nsites + 1));
      return GEMS_ERR_BAD_ARG;
    }
  } else {
    if ((e = cudaMemcpyAsync(d_codes, seqs, cells, cudaMemcpyHostToDevice, st)))
      return fail(e, "ingest upload");
  }
  if ((e = cudaMemsetAsync(d_tab, 0xFF, sizeof(unsigned long long) * cap, st)) ||
      (e = cudaMemsetAsync(d_grp, 0xFF, sizeof(long long) * nsites, st)) ||
      (e = cudaMemsetAsync(d_min, 0xFF, sizeof(unsigned long long) * cap, st)) ||
      (e = cudaMemsetAsync(g->d_count, 0, sizeof(unsigned int) * nsites, st)))
    return fail(e, "ingest memset");
  k_hash<<<gs, T, 0, st>>>(d_codes, ntaxa, nsites, d_h);
  k_insert<<<gs, T, 0, st>>>(d_codes, ntaxa, nsites, d_h, d_tab, d_min, cap - 1, d_grp);
  k_first<<<gs, T, 0, st>>>(d_grp, d_min, nsites, d_flag);
  k_scan_block<<<(unsigned)nblk, 1024, 0, st>>>(d_flag, nsites, d_pid, d_bsum);
  k_scan_sums<<<1, 32, 0, st>>>(d_bsum, nblk, d_bsum + nblk);
  k_scan_add<<<(unsigned)nblk, 1024, 0, st>>>(d_pid, nsites, d_bsum);
  k_assign<<<gs, T, 0, st>>>(d_grp, d_min, d_pid, nsites, g->d_sp, g->d_count, d_rep);
  long long npat = 0;
  if ((e = cudaGetLastError()) ||
      (e = cudaMemcpyAsync(&npat, d_bsum + nblk, sizeof(npat), cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return fail(e, "ingest compress");
  g->npat = npat;
  if ((e = cudaMalloc((void **)&g->d_pat, (size_t)ntaxa * npat)) != cudaSuccess ||
      (e = cudaMalloc((void **)&g->d_cc, (size_t)npat)) != cudaSuccess)
    return fail(e, "cudaMalloc patterns");
  const unsigned gp = (unsigned)((npat + T - 1) / T);
  k_gather<<<gp, T, 0, st>>>(d_codes, ntaxa, nsites, npat, d_rep, g->d_pat);
  k_const<<<gp, T, 0, st>>>(g->d_pat, ntaxa, npat, nstates, g->d_cc);
  if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(st))) return fail(e, "ingest gather");
  release();
  *out = g;
  *npat_out = npat;
  return GEMS_OK;
}

extern "C" int gems_ingest_read(gems_ingest *g, uint8_t *patterns, double *weights,
                                int *site_pattern, uint8_t *const_char) {
  if (!g) return GEMS_ERR_BAD_ARG;
  GEMS_CUDA(cudaSetDevice(g->device));
  std::vector<unsigned int> cnt((size_t)g->npat);
  if (patterns)
    GEMS_CUDA(cudaMemcpyAsync(patterns, g->d_pat, (size_t)g->ntaxa * g->npat,
                              cudaMemcpyDeviceToHost, g->st));
  if (weights)
    GEMS_CUDA(cudaMemcpyAsync(cnt.data(), g->d_count, sizeof(unsigned int) * g->npat,
                              cudaMemcpyDeviceToHost, g->st));
  if (site_pattern)
    GEMS_CUDA(cudaMemcpyAsync(site_pattern, g->d_sp, sizeof(int) * g->nsites,
                              cudaMemcpyDeviceToHost, g->st));
  if (const_char)
    GEMS_CUDA(cudaMemcpyAsync(const_char, g->d_cc, (size_t)g->npat, cudaMemcpyDeviceToHost,
                              g->st));
  GEMS_CUDA(cudaStreamSynchronize(g->st));
  if (weights)
    for (long long p = 0; p < g->npat; p++) weights[p] = (double)cnt[(size_t)p];
  return GEMS_OK;
}

extern "C" int gems_ingest_to_session(gems_ingest *g, gems_session *s, double p_invar,
                                      const double *state_freq) {
  if (!g || !s || (p_invar != 0.0 && !state_freq) || p_invar < 0.0 || p_invar >= 1.0)
    return GEMS_ERR_BAD_ARG;
  if (s->desc.device != g->device || s->desc.ntaxa != g->ntaxa || s->desc.nptn != g->npat ||
      s->desc.nstates != g->nstates) {
    set_error("ingest_to_session: the session's device, taxa, patterns or states differ");
    return GEMS_ERR_BAD_ARG;
  }
  GEMS_CUDA(cudaSetDevice(g->device));
  GEMS_CUDA(cudaStreamSynchronize(g->st));  // the ingest's kernels have finished
  FreqPack fr{};
  for (int x = 0; x < g->nstates && state_freq; x++) fr.f[x] = state_freq[x];
  const unsigned gp = (unsigned)((g->npat + 255) / 256);
  k_counts<<<gp, 256, 0, s->stream>>>(g->d_count, g->npat, s->d_freq);
  k_ptn_invar<<<gp, 256, 0, s->stream>>>(g->d_cc, g->npat, g->nstates, p_invar, fr, s->d_invar);
  s->launches += 2;
  GEMS_CUDA(cudaGetLastError());
  s->theta_valid = false;
  return load_tips(s, g->d_pat, (size_t)g->npat, cudaMemcpyDeviceToDevice);
}

extern "C" int gems_compress_alignment(int device, int ntaxa, long long nsites, int nstates,
                                       const uint8_t *seqs, int encoded, uint8_t *patterns,
                                       double *weights, int *site_pattern, uint8_t *const_char,
                                       long long *npat_out) {
  if (!patterns || !weights || !npat_out) return GEMS_ERR_BAD_ARG;
  gems_ingest *g = nullptr;
  long long npat = 0;
  if (int st = gems_ingest_create(device, ntaxa, nsites, nstates, seqs, encoded, &g, &npat))
    return st;
  const int st = gems_ingest_read(g, patterns, weights, site_pattern, const_char);
  gems_ingest_destroy(g);
  if (!st) *npat_out = npat;
  return st;
}
