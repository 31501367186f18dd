// Coverage check of the column split of a step launch (split.h), run by tests/test_split_host.py: for each
// configuration on the command line (nx ny jg0 nyg jlo jhi jbase ws rows staged) it walks every thread of the launch
// grid the step launcher builds (staged = 1: the TMA-staged paired step's grid, main blocks from row m0) and checks
// that each column of the step's rows is taken by exactly one thread, that no main
// warp holds a lateral-face column when ws > 0, and that the lanes of a main warp are 32 consecutive columns of one
// row. Prints "ok <columns>" or the first failure.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "split.h"

using namespace ahx;

static int check(int nx, int ny, int jg0, int nyg, int jlo, int jhi, int jbase, int ws, int rows, int staged) {
  const StepSplit P = step_split(nx, jlo, jhi, jbase, jg0, nyg, ws);
  const int main_by = staged ? staged_main_blocks_y(P, rows) : main_blocks_y(jhi, jbase, rows);
  const int gy = main_by + strip_blocks_y(P, rows);
  std::vector<int> seen((size_t)nx * ny, 0);
  for (int by = 0; by < gy; ++by)
    for (int bx = 0; bx < P.gx; ++bx)
      for (int ty = 0; ty < rows; ++ty) {
        int row = -1, first = -1;
        for (int tx = 0; tx < 32; ++tx) {
          int i, j;
          const bool got = staged ? staged_block_column(P, nx, rows, bx, by, tx, ty, i, j)
                                  : block_column(P, nx, jbase, jhi, rows, bx, by, tx, ty, i, j);
          if (!got) continue;
          if (i < 0 || i >= nx || j < 0 || j >= ny) {
            printf("column (%d, %d) outside the domain\n", i, j);
            return 1;
          }
          ++seen[(size_t)j * nx + i];
          const bool main = by < main_by;
          if (main && ws > 0) {
            const int jg = j + jg0;
            if (i == 0 || i == nx - 1 || jg == 0 || jg == nyg - 1) {
              printf("face column (%d, %d) in a main warp\n", i, j);
              return 1;
            }
          }
          if (main) {
            if (row < 0) {
              row = j;
              first = i - tx;
            } else if (j != row || i != first + tx) {
              printf("main warp lanes not consecutive columns of one row at (%d, %d)\n", i, j);
              return 1;
            }
          }
        }
      }
  const int r0 = jlo > jbase ? jlo : jbase;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const int want = (j >= r0 && j < jhi) ? 1 : 0;
      if (seen[(size_t)j * nx + i] != want) {
        printf("column (%d, %d) taken %d times, want %d\n", i, j, seen[(size_t)j * nx + i], want);
        return 1;
      }
    }
  return 0;
}

int main(int argc, char** argv) {
  if ((argc - 1) % 10 != 0) {
    printf("usage: split_check (nx ny jg0 nyg jlo jhi jbase ws rows staged)...\n");
    return 2;
  }
  int n = 0;
  for (int a = 1; a < argc; a += 10) {
    int v[10];
    for (int t = 0; t < 10; ++t) v[t] = atoi(argv[a + t]);
    if (check(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9])) {
      printf("failed: nx %d ny %d jg0 %d nyg %d jlo %d jhi %d jbase %d ws %d rows %d staged %d\n", v[0], v[1], v[2],
             v[3], v[4], v[5], v[6], v[7], v[8], v[9]);
      return 1;
    }
    ++n;
  }
  printf("ok %d\n", n);
  return 0;
}
