// Host-side check of the per-vertex cull word (cp_cull.cuh): the library's
// vertex_word_hi against a plain statement of the same definition -- bits
// 0..2 component j strongly positive (|v_j| > kappa' b), bits 3..5 strongly
// negative, bit 6 tiny (b below the tiny bound), bits 7.. the band mask of
// b's exponent -- on random and special high words, for float and double and
// 2 or 3 components.  Prints the first mismatch and exits 1, else exits 0.
#include <cstdio>
#include <cstdint>
#include <random>

#include "../../ftk2_b200/csrc/cp_cull.cuh"

using namespace ftk2b;

template <typename T, int M>
static unsigned word_plain(const unsigned h[M], const unsigned* tbl) {
  using P = CullParams<T>;
  unsigned a[M], b = 0;
  for (int j = 0; j < M; ++j) {
    a[j] = h[j] & 0x7FFFFFFFu;
    if (a[j] > b) b = a[j];
  }
  const unsigned kexp = (unsigned)P::kappa_exp << P::mant;
  const unsigned thr = (b > kexp ? b : kexp) - kexp;
  unsigned w = 0;
  for (int j = 0; j < M; ++j) {
    if (a[j] > thr) w |= (h[j] >> 31) ? (8u << j) : (1u << j);
  }
  if (b < P::tiny_hi) w |= 1u << 6;
  const long long rel1 = (long long)(b >> P::mant) - P::bias - kElo + 1;
  const long long ri = (rel1 < 0 || rel1 > kBandTable - 1) ? kBandTable - 1 : rel1;
  return w | tbl[ri];
}

template <typename T, int M>
static int check(std::mt19937_64& rng, long long n) {
  unsigned tbl[kBandTable];
  fill_band_table<T>(tbl, 0, 1);
  const unsigned special[] = {0u, 0x80000000u, 0x7F800000u, 0xFF800000u, 0x7FC00000u, 0x7FF00000u, 0xFFF00000u,
                              0x7FF80000u, 0x00000001u, 0x80000001u, CullParams<T>::tiny_hi,
                              CullParams<T>::tiny_hi - 1, CullParams<T>::tiny_hi + 1, 0x3F800000u, 0xBF800000u,
                              0x3FF00000u, 0xBFF00000u, (unsigned)CullParams<T>::kappa_exp << CullParams<T>::mant};
  const int ns = (int)(sizeof(special) / sizeof(special[0]));
  for (long long it = 0; it < n; ++it) {
    unsigned h[M];
    const int mode = (int)(it % 4);
    const unsigned base = (unsigned)rng();
    for (int j = 0; j < M; ++j) {
      unsigned x = (unsigned)rng();
      if (mode == 1) x = special[rng() % ns] ^ (unsigned)(rng() % 3);
      // near-equal magnitudes: the strong test's boundary
      if (mode == 2) x = (base & 0x7FFFFFFFu) + (unsigned)(rng() % 64) - 32u + ((unsigned)(rng() & 1) << 31);
      // magnitudes kappa' apart: the threshold itself
      if (mode == 3 && j > 0)
        x = (((h[0] & 0x7FFFFFFFu) - ((unsigned)CullParams<T>::kappa_exp << CullParams<T>::mant)) +
             (unsigned)(rng() % 5) - 2u) | ((unsigned)(rng() & 1) << 31);
      h[j] = x;
    }
    const unsigned got = vertex_word_hi<T, M>(h, tbl), want = word_plain<T, M>(h, tbl);
    if (got != want) {
      std::printf("mismatch (sizeof(T) %d, M %d):", (int)sizeof(T), M);
      for (int j = 0; j < M; ++j) std::printf(" %08x", h[j]);
      std::printf(" -> %08x, want %08x\n", got, want);
      return 1;
    }
  }
  return 0;
}

int main() {
  std::mt19937_64 rng(20240607);
  const long long n = 4000000;
  int bad = check<float, 2>(rng, n) | check<float, 3>(rng, n) | check<double, 2>(rng, n) | check<double, 3>(rng, n);
  if (!bad) std::printf("cull words agree on %lld x 4 cases\n", n);
  return bad;
}
