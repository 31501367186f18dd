// Host check of the population-plane index arithmetic (lattice.cuh), run by tests/test_layout_host.py: for the
// level-paired 16-bit planes and the plain 32-bit planes, lvl_nbr (the neighbour offset the step kernels form from a
// cell's own offset) equals lvl at the neighbour's level and row-column for every level, every lateral shift of the
// D3Q19 / D3Q7 velocities and every vertical shift, and the 38 pair slots (pair_slot) are a dense numbering of the
// first and second source words of a level pair. Compiled by nvcc as host code (no GPU involved). Prints "ok <checks>"
// or the first failure.
#include <cstdio>

#include "fused.cuh"

using namespace ahx;

template <class T>
static long check_planes(uint32_t px, uint32_t ny, int nz) {
  const uint32_t ps = px * ny;
  long n = 0;
  for (int k = 1; k < nz - 1; ++k)
    for (uint32_t j = 1; j + 1 < ny; ++j)
      for (uint32_t i = 1; i + 1 < px; i += 7) {
        const uint32_t m = j * px + i;
        const uint32_t own = lvl<T>(k, m, ps);
        for (int cz = -1; cz <= 1; ++cz)
          for (int cy = -1; cy <= 1; ++cy)
            for (int cx = -1; cx <= 1; ++cx) {
              const uint32_t d = (uint32_t)(cx + cy * (int)px);
              const uint32_t want = lvl<T>(k - cz, m - d, ps);
              const uint32_t got = lvl_nbr<T>(k, m, own, cz, d, ps);
              if (want != got) {
                printf("lvl_nbr mismatch (%zu-byte): k %d m %u c (%d, %d, %d): %u, want %u\n", sizeof(T), k, m, cx, cy,
                       cz, got, want);
                return -1;
              }
              ++n;
            }
      }
  return n;
}

int main() {
  long total = 0;
  for (uint32_t px : {64u, 640u})
    for (uint32_t ny : {5u, 12u}) {
      const long a = check_planes<__half>(px, ny, 10), b = check_planes<float>(px, ny, 10);
      if (a < 0 || b < 0) return 1;
      total += a + b;
    }
  // pair slots: each population's first word, then its second word when it moves vertically, densely numbered
  int expect = 0;
  for (int p = 0; p < 26; ++p) {
    if (pair_slot(p) != expect) {
      printf("pair_slot(%d) = %d, want %d\n", p, pair_slot(p), expect);
      return 1;
    }
    const int cz = p < 19 ? kC19[p][2] : kC7[p - 19][2];
    expect += cz != 0 ? 2 : 1;
  }
  if (expect != kPairSlots) {
    printf("%d pair slots, want %d\n", expect, kPairSlots);
    return 1;
  }
  printf("ok %ld\n", total + 26);
  return 0;
}
