// Host-side check of the LU-SGS sweep-record layout (device/layout.cuh),
// compiled and run on the CPU by tests/test_sweep_layout.py: for each grid,
// sweep_slot maps the ni nj cells one-to-one onto [0, ni nj); diagonal d is
// the contiguous range [diag_cells(d), diag_cells(d + 1)) holding rows
// max(0, d - ni + 1) .. min(d, nj - 1) in order; and the chunk ranges the
// sweep's producer copies (K diagonals, forward from diagonal 0, backward
// ending at the last) stay inside the case and within K * min(ni, nj)
// records, the buffer size. Also the sweep's launch shape (sweep_shape):
// within a CTA's share of shared memory the longest chunk of up to 8
// diagonals in at least two buffers, then up to four buffers, and the
// smallest shape when not even one diagonal in two buffers fits the share. Prints "ok" or the first failure.
#include <cstdio>
#include <vector>

#include "device/layout.cuh"
#include "device/sweep.cuh"

static int check(int ni, int nj) {
  const int ndiag = ni + nj - 1;
  const long long cells = (long long)ni * nj;
  if (bsd::sweep_slots(ni, nj) != cells) return printf("%d x %d: sweep_slots %lld\n", ni, nj, (long long)bsd::sweep_slots(ni, nj)), 1;
  if ((long long)bsd::diag_cells(ni, nj, ndiag) != cells) return printf("%d x %d: diag_cells(end)\n", ni, nj), 1;
  std::vector<char> seen(cells, 0);
  for (int j = 0; j < nj; j++)
    for (int i = 0; i < ni; i++) {
      const long long s = bsd::sweep_slot(ni, nj, i, j);
      if (s < 0 || s >= cells || seen[s]) return printf("%d x %d: cell (%d, %d) slot %lld\n", ni, nj, i, j, s), 1;
      seen[s] = 1;
      const int d = i + j, jlo = d - ni + 1 > 0 ? d - ni + 1 : 0;
      if (s != (long long)bsd::diag_cells(ni, nj, d) + (j - jlo)) return printf("%d x %d: diagonal order at (%d, %d)\n", ni, nj, i, j), 1;
    }
  const int len_max = ni < nj ? ni : nj;
  for (int d = 0; d < ndiag; d++) {
    const int jlo = d - ni + 1 > 0 ? d - ni + 1 : 0, jhi = d < nj - 1 ? d : nj - 1;
    const unsigned len = bsd::diag_cells(ni, nj, d + 1) - bsd::diag_cells(ni, nj, d);
    if (len != unsigned(jhi - jlo + 1) || len > unsigned(len_max)) return printf("%d x %d: diagonal %d length\n", ni, nj, d), 1;
  }
  for (int K = 1; K <= 16; K *= 2) {
    const int nch = (ndiag + K - 1) / K;
    for (int pass = 0; pass < 2; pass++)
      for (int cc = 0; cc < nch; cc++) {
        const int n = ndiag - cc * K < K ? ndiag - cc * K : K;
        const int dlo = pass == 0 ? cc * K : ndiag - cc * K - n;
        const unsigned lo = bsd::diag_cells(ni, nj, dlo), hi = bsd::diag_cells(ni, nj, dlo + n);
        if (dlo < 0 || hi > cells || hi < lo || hi - lo > unsigned(K) * unsigned(len_max))
          return printf("%d x %d: K %d pass %d chunk %d\n", ni, nj, K, pass, cc), 1;
      }
  }
  return 0;
}

static int check_shape(int max_len, int warps, int cases, int want_chunk, int want_buffers) {
  const bsd::SweepShape s = bsd::sweep_shape(max_len, warps, cases);
  const size_t bytes = bsd::sweep_smem_bytes(max_len, warps, s.chunk, s.buffers);
  if (s.chunk != want_chunk || s.buffers != want_buffers || bytes > 220 * 1024)
    return printf("shape(%d, %d, %d): K %d NB %d, %zu bytes\n", max_len, warps, cases, s.chunk, s.buffers, bytes), 1;
  return 0;
}

int main() {
  // The drag curve (160 x 80, 16 cases): K 8 in four buffers, 208 KB.
  if (check_shape(80, 3, 16, 8, 4)) return 1;
  // 640 x 320 alone: 25.6 KB a diagonal, the longest chunk first: K 4 in two buffers.
  if (check_shape(320, 10, 16, 4, 2)) return 1;
  // 300 cases of 160 x 80 (three an SM): K 4 in two buffers within 73 KB.
  if (check_shape(80, 3, 300, 4, 2)) return 1;
  // 873 cases of 640 x 320, 1,988 mixed up to 320 x 160: no shape fits a
  // CTA's share of an SM, so the smallest.
  if (check_shape(320, 10, 873, 1, 2)) return 1;
  if (check_shape(160, 5, 1988, 1, 2)) return 1;
  // A case of up to 32 rows: one consumer warp, K 8 in four buffers.
  if (check_shape(20, 1, 16, 8, 4)) return 1;
  const int grids[][2] = {{2, 2},   {3, 5},    {5, 3},    {40, 20},  {20, 40},   {160, 80}, {7, 33},
                          {33, 97}, {2, 512},  {512, 2},  {96, 48},  {640, 320}, {512, 128}, {64, 512},
                          {1000, 7}, {7, 1000}, {1280, 512}};
  for (const auto& g : grids)
    if (check(g[0], g[1])) return 1;
  // The largest grid the 32-bit diagonal arithmetic allows (ni + nj = 65536):
  // the slot count and the last diagonal's offset only.
  const int ni = 65024, nj = 512;
  if ((long long)bsd::diag_cells(ni, nj, ni + nj - 1) != (long long)ni * nj) return printf("limit grid\n"), 1;
  printf("ok\n");
  return 0;
}
