// Column split of a step launch of the B200 live solver: which column of the domain each thread of a step launch
// updates. Plain C++ (host and device), so the host-side tests check the split's coverage directly.
#pragma once

#ifdef __CUDACC__
#define AHX_HD __host__ __device__
#else
#define AHX_HD
#endif

namespace ahx {

// Split of a step's columns between main blocks and strip blocks. The step updates local rows [r0, r1) =
// [max(jlo, jbase), jhi); among them can be the global south row (local row -jg0, which is r0 when present) and the
// global north row (local nyg - 1 - jg0, which is r1 - 1 when present). With strip width ws = 0 the main blocks cover
// every column of every row, as warps of 32 consecutive columns from column 0, and there are no strip blocks. With
// ws > 0 the main blocks cover the columns [we, ea) of the rows [m0, m1) between the south and north rows, as warps of
// 32 consecutive columns from column we (ea - we a multiple of 32), and the strip blocks after them give each thread
// one column of: the west strips (columns [0, we) of those rows), the east strips ([ea, nx)), then the south and north
// rows whole. Every lateral-face column is then in a strip, so every main warp can take the interior paths; a warp of
// the west strips covers 32 / ws rows of ws consecutive columns (whole 32-byte sectors when ws elements are 32 bytes).
struct StepSplit {
  int r0, r1;       // rows of the step
  int m0, m1;       // rows of the main blocks
  int we, ea;       // columns of the main blocks
  int gx;           // blocks in x of a launch
  int nw, ne, nsn;  // strip columns: west strips, east strips, south and north rows
  bool south, north;
};
AHX_HD inline StepSplit step_split(int nx, int jlo, int jhi, int jbase, int jg0, int nyg, int ws) {
  StepSplit P;
  P.r0 = jlo > jbase ? jlo : jbase;
  P.r1 = jhi > P.r0 ? jhi : P.r0;
  P.south = P.north = false;
  P.m0 = P.r0;
  P.m1 = P.r1;
  P.we = 0;
  P.ea = nx;
  P.gx = (nx + 31) / 32;
  P.nw = P.ne = P.nsn = 0;
  if (ws <= 0 || P.r1 == P.r0) return P;
  P.south = -jg0 == P.r0;
  P.north = nyg - 1 - jg0 == P.r1 - 1 && !(P.south && P.r1 - 1 == P.r0);
  P.m0 = P.r0 + (P.south ? 1 : 0);
  P.m1 = P.r1 - (P.north ? 1 : 0);
  if (P.m1 < P.m0) P.m1 = P.m0;
  P.we = ws < nx ? ws : nx;
  P.ea = nx - 1 < P.we ? P.we : P.we + 32 * ((nx - 1 - P.we) / 32);
  P.gx = P.ea - P.we >= 32 ? (P.ea - P.we) / 32 : 1;
  const int rows = P.m1 - P.m0;
  P.nw = rows * P.we;
  P.ne = rows * (nx - P.ea);
  P.nsn = ((P.south ? 1 : 0) + (P.north ? 1 : 0)) * nx;
  return P;
}
// strip column number c (west strips, east strips, south row, north row) as (i, j); false past the end
AHX_HD inline bool strip_column(const StepSplit& P, int nx, int c, int& i, int& j) {
  i = 0;
  j = P.r0;
  if (c < 0) return false;
  if (c < P.nw) {
    j = P.m0 + c / P.we;
    i = c - (j - P.m0) * P.we;
    return true;
  }
  c -= P.nw;
  if (c < P.ne) {
    const int ew = nx - P.ea;
    j = P.m0 + c / ew;
    i = P.ea + (c - (j - P.m0) * ew);
    return true;
  }
  c -= P.ne;
  if (P.south) {
    if (c < nx) { i = c; j = P.r0; return true; }
    c -= nx;
  }
  if (P.north && c < nx) { i = c; j = P.r1 - 1; return true; }
  return false;
}
// blocks in y of a step launch with `rows` rows of 32 columns per block: the main blocks over rows [jbase, jhi), then
// the strip blocks (gx blocks in x, one strip column per thread)
AHX_HD inline int main_blocks_y(int jhi, int jbase, int rows) { return (jhi - jbase + rows - 1) / rows; }
AHX_HD inline int strip_blocks_y(const StepSplit& P, int rows) {
  const int per = P.gx * 32 * rows, n = P.nw + P.ne + P.nsn;
  return (n + per - 1) / per;
}
// strip width of a storage on a grid nx columns wide: for 2-byte population elements 8 or 16 columns, whichever leaves
// fewer columns to the strips (the 16-bit planes keep two levels of a column in one 4-byte word, so 8 columns are
// one 32-byte sector; the main path of the 16-bit storages is bound by instruction issue, so taking its face columns
// off the main warps pays; ties keep 16), else none (the 4- and 8-byte storages are bound by DRAM bandwidth, and
// sector-aligned main warps keep every write a whole sector)
AHX_HD constexpr int strip_columns(int nx, int we) { return nx - 1 < we ? nx : nx - 32 * ((nx - 1 - we) / 32); }
AHX_HD constexpr int strip_width(int esize_f, int nx) {
  return esize_f != 2 ? 0 : (strip_columns(nx, 8) < strip_columns(nx, 16) ? 8 : 16);
}

// the column (i, j) of thread (tx, ty) of block (bx, by) of a step launch with `rows` rows per block over rows
// [jbase, jhi): main blocks first (by < main_blocks_y), strip blocks after them; false for a thread without a column
AHX_HD inline bool block_column(const StepSplit& P, int nx, int jbase, int jhi, int rows, int bx, int by, int tx,
                                int ty, int& i, int& j) {
  const int main_by = main_blocks_y(jhi, jbase, rows);
  if (by < main_by) {
    i = P.we + bx * 32 + tx;
    j = jbase + by * rows + ty;
    return i < P.ea && j >= P.m0 && j < P.m1;
  }
  return strip_column(P, nx, ((by - main_by) * P.gx + bx) * 32 * rows + ty * 32 + tx, i, j);
}

// The TMA-staged paired step (ws > 0 only) tiles the main columns from row m0 instead of jbase, so a block's rows are
// rows of main columns only (its staged boxes then never start on a strip row): main blocks over rows [m0, m1), then
// the same strip blocks as block_column.
AHX_HD inline int staged_main_blocks_y(const StepSplit& P, int rows) { return (P.m1 - P.m0 + rows - 1) / rows; }
AHX_HD inline bool staged_block_column(const StepSplit& P, int nx, int rows, int bx, int by, int tx, int ty, int& i,
                                       int& j) {
  const int main_by = staged_main_blocks_y(P, rows);
  if (by < main_by) {
    i = P.we + bx * 32 + tx;
    j = P.m0 + by * rows + ty;
    return i < P.ea && j < P.m1;
  }
  return strip_column(P, nx, ((by - main_by) * P.gx + bx) * 32 * rows + ty * 32 + tx, i, j);
}


}  // namespace ahx
