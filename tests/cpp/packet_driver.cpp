// packet_driver.cpp -- a C++ caller of the C-ABI, compiled with g++ against include/gems_b200.h
// and linked to libgems_b200.so (test infrastructure).
//
// It drives one session the way the reference drives computePartialLikelihood: the pattern
// range split into packets (waves of 3/4 of the remaining patterns, each wave split evenly over
// the threads, bounds rounded to the kernel's granule, as computeBounds does,
// tree/phylokernelnew.h:1118-1146), then for every packet every traversal entry in postorder
// (tree/phylokernelnew.h:1274-1281) -> gems_compute_partial.  A second session runs the same
// op list as one gems_traverse call.  Every slot's partial and scale counters and the branch
// lnL must be identical, bit for bit.
//
// usage: packet_driver <input file> <threads>
// input (little endian): int32 ntaxa, nptn, nstates, ncat, nslots, precision, scaling, nops;
// uint8 tips[ntaxa][nptn]; float64 freq[nptn], eval[n], evec[n*n], inv_evec[n*n], rates[ncat],
// props[ncat]; gems_op ops[nops]; gems_branch br.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gems_b200.h"

namespace {

bool ok(int st, const char *what) {
  if (st != GEMS_OK) std::fprintf(stderr, "%s: status %d: %s\n", what, st, gems_last_error());
  return st == GEMS_OK;
}

template <typename T>
bool read_vec(std::FILE *f, std::vector<T> &v, size_t n) {
  v.resize(n);
  return std::fread(v.data(), sizeof(T), n, f) == n;
}

// packet bounds over [0, elements): waves of 3/4 of what is left, each split over `threads`
size_t round_up(size_t x, size_t g) { return (x + g - 1) / g * g; }

std::vector<size_t> packet_bounds(int threads, int packets, size_t elements, size_t g) {
  std::vector<size_t> lim;
  elements = round_up(elements, g);
  size_t start = 0;
  for (int wave = packets / threads; wave >= 1; --wave) {
    size_t this_wave = elements - start;
    if (wave > 1) this_wave = this_wave * 3 / 4;
    this_wave = round_up(this_wave, g);
    const size_t stop = start + this_wave;
    for (int left = threads; left >= 1; --left) {
      lim.push_back(start);
      start += round_up((stop - start) / left, g);
    }
  }
  lim.push_back(elements);
  return lim;
}

gems_session *open_session(const gems_session_desc &d, const std::vector<uint8_t> &tips,
                           const std::vector<double> &freq, const std::vector<double> &eval,
                           const std::vector<double> &evec, const std::vector<double> &ivec,
                           const std::vector<double> &rates, const std::vector<double> &props) {
  gems_session *s = nullptr;
  if (!ok(gems_session_create(&d, &s), "gems_session_create")) return nullptr;
  if (!ok(gems_upload_tips(s, tips.data()), "gems_upload_tips") ||
      !ok(gems_upload_patterns(s, freq.data(), nullptr), "gems_upload_patterns") ||
      !ok(gems_set_model(s, eval.data(), evec.data(), ivec.data(), rates.data(), props.data()),
          "gems_set_model")) {
    gems_session_destroy(s);
    return nullptr;
  }
  return s;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <input> <threads>\n", argv[0]);
    return 2;
  }
  std::FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  int32_t hdr[8];
  if (std::fread(hdr, sizeof(int32_t), 8, f) != 8) return 2;
  gems_session_desc d{};
  d.ntaxa = hdr[0];
  d.nptn = hdr[1];
  d.nstates = hdr[2];
  d.ncat = hdr[3];
  d.nslots = hdr[4];
  d.precision = hdr[5];
  d.scaling = hdr[6];
  d.device = 0;
  const int nops = hdr[7], n = d.nstates;
  std::vector<uint8_t> tips;
  std::vector<double> freq, eval, evec, ivec, rates, props;
  std::vector<gems_op> ops;
  gems_branch br{};
  if (!read_vec(f, tips, (size_t)d.ntaxa * d.nptn) || !read_vec(f, freq, d.nptn) ||
      !read_vec(f, eval, n) || !read_vec(f, evec, (size_t)n * n) ||
      !read_vec(f, ivec, (size_t)n * n) || !read_vec(f, rates, d.ncat) ||
      !read_vec(f, props, d.ncat) || !read_vec(f, ops, nops) ||
      std::fread(&br, sizeof(br), 1, f) != 1)
    return 2;
  std::fclose(f);
  const int threads = std::atoi(argv[2]);

  gems_session *whole = open_session(d, tips, freq, eval, evec, ivec, rates, props);
  gems_session *packed = open_session(d, tips, freq, eval, evec, ivec, rates, props);
  if (!whole || !packed) return 1;
  if (!ok(gems_traverse(whole, ops.data(), nops), "gems_traverse")) return 1;

  int g = 1;
  if (!ok(gems_session_pattern_granule(packed, &g), "gems_session_pattern_granule")) return 1;
  const std::vector<size_t> lim = packet_bounds(threads, 2 * threads, d.nptn, g);
  int calls = 0;
  for (size_t k = 0; k + 1 < lim.size(); k++) {
    const size_t lo = lim[k], hi = lim[k + 1] < (size_t)d.nptn ? lim[k + 1] : d.nptn;
    if (lo >= hi) continue;  // a packet past the last pattern (bounds are rounded up)
    for (int i = 0; i < nops; i++) {
      if (!ok(gems_compute_partial(packed, &ops[i], (int)lo, (int)hi), "gems_compute_partial"))
        return 1;
      calls++;
    }
  }

  const size_t elems = (size_t)d.nptn * d.ncat * n;
  const size_t nsc = (size_t)d.nptn * (d.scaling == GEMS_SCALE_SAFE ? d.ncat : 1);
  std::vector<double> a(elems), b(elems);
  std::vector<uint16_t> sa(nsc), sb(nsc);
  int written = 0;
  for (int i = 0; i < nops; i++) {
    const int slot = ops[i].dst_slot;
    if (!ok(gems_get_partial(whole, slot, a.data(), sa.data()), "gems_get_partial") ||
        !ok(gems_get_partial(packed, slot, b.data(), sb.data()), "gems_get_partial"))
      return 1;
    if (std::memcmp(a.data(), b.data(), elems * sizeof(double)) != 0 ||
        std::memcmp(sa.data(), sb.data(), nsc * sizeof(uint16_t)) != 0) {
      std::printf("MISMATCH slot %d\n", slot);
      return 1;
    }
    written++;
  }
  double la = 0, lb = 0;
  if (!ok(gems_branch_lnl(whole, nullptr, 0, &br, &la, nullptr), "gems_branch_lnl") ||
      !ok(gems_branch_lnl(packed, nullptr, 0, &br, &lb, nullptr), "gems_branch_lnl"))
    return 1;
  if (std::memcmp(&la, &lb, sizeof(double)) != 0) {
    std::printf("MISMATCH lnl %.17g %.17g\n", la, lb);
    return 1;
  }
  std::printf("OK slots=%d packets=%zu granule=%d calls=%d lnl=%.17g\n", written,
              lim.size() - 1, g, calls, la);
  gems_session_destroy(whole);
  gems_session_destroy(packed);
  return 0;
}
