// Host check of the reverse-pass early stop of the full-alignment kernels
// (PassStop in ipuma-lib_b200/csrc/sw_device.cuh).  A strip-wise reverse
// pass that (a) ends a strip after the first row where a cell reaches the
// target (= the forward score) and (b) runs later strips only on the rows
// above the best row found so far must give the same (score, row, column)
// as the full reverse pass, under the reference's first-strict-maximum
// tie-break (codelet_batch_affine.cpp:79-83, 89-115), for any strip width.
// The recurrence is the codelet's (E along A, F along B, H floor 0).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
typedef struct { int s, i, j; } Best;
static int better(int s1, int i1, int j1, int s2, int i2, int j2) {
  return s1 > s2 || (s1 == s2 && (i1 < i2 || (i1 == i2 && j1 < j2)));
}
static int gI, gE;
static int sim[4][4];
static inline int mx(int a, int b) { return a > b ? a : b; }
// Full DP over a (len la, columns) x b (len lb, rows): first strict max, row-major.
static Best full(const int* a, int la, const int* b, int lb) {
  int* H = calloc(la + 1, sizeof(int)); int* F = calloc(la + 1, sizeof(int));
  Best bst = {0, 0, 0};
  for (int i = 0; i < lb; ++i) {
    int E = gI, Hleft = 0, Hdiag = 0;
    for (int j = 0; j < la; ++j) {
      E = mx(Hleft + gI + gE, E + gE);
      F[j] = mx(H[j] + gI + gE, F[j] + gE);
      int h = mx(mx(Hdiag + sim[a[j]][b[i]], E), mx(F[j], 0));
      Hdiag = H[j]; H[j] = h; Hleft = h;
      if (h > bst.s) { bst.s = h; bst.i = i; bst.j = j; }
    }
  }
  free(H); free(F); return bst;
}
// Strip-wise with early stop; rows processed counted in *work.
static Best stripped(const int* a, int la, const int* b, int lb, int SW, int target, long* work) {
  int* Hb = calloc(lb, sizeof(int)); int* Eb = malloc(lb * sizeof(int));  // boundary column per row
  for (int i = 0; i < lb; ++i) Eb[i] = gI;  // row init before column 0 (E starts at gI)
  int* H = calloc(SW, sizeof(int)); int* F = calloc(SW, sizeof(int));
  int* nHb = calloc(lb, sizeof(int)); int* nEb = malloc(lb * sizeof(int));
  Best bst = {0, 0, 0};
  int cap = lb;
  for (int c0 = 0; c0 < la; c0 += SW) {
    const int w = (la - c0 < SW) ? la - c0 : SW;
    memset(H, 0, SW * sizeof(int)); memset(F, 0, SW * sizeof(int));
    Best sb = {0, 0, 0};
    int rows = cap;
    for (int i = 0; i < rows; ++i) {
      int E = Eb[i], Hleft = Hb[i], Hdiag = (i > 0) ? Hb[i - 1] : 0;
      for (int j = 0; j < w; ++j) {
        E = mx(Hleft + gI + gE, E + gE);
        F[j] = mx(H[j] + gI + gE, F[j] + gE);
        int h = mx(mx(Hdiag + sim[a[c0 + j]][b[i]], E), mx(F[j], 0));
        Hdiag = H[j]; H[j] = h; Hleft = h;
        if (h > sb.s) { sb.s = h; sb.i = i; sb.j = c0 + j; }
      }
      nHb[i] = Hleft; nEb[i] = E;
      ++*work;
      if (sb.s == target && rows > i + 1) rows = i + 1;  // finish this row, then stop
    }
    if (better(sb.s, sb.i, sb.j, bst.s, bst.i, bst.j)) bst = sb;
    if (bst.s == target && bst.i < cap) cap = bst.i;  // later strips: rows above the best only
    memcpy(Hb, nHb, lb * sizeof(int)); memcpy(Eb, nEb, lb * sizeof(int));
    if (cap == 0) break;
  }
  free(Hb); free(Eb); free(H); free(F); free(nHb); free(nEb); return bst;
}
int main(void) {
  srand(7);
  long cases = 0, fails = 0, workFull = 0, workStop = 0;
  const int scorings[][4] = {{0, -1, 1, -1}, {-1, -1, 1, -1}, {-10, -1, 2, -3}, {-3, -2, 1, -1}, {0, -1, 2, -1}};
  for (int sc = 0; sc < 5; ++sc) {
    gI = scorings[sc][0]; gE = scorings[sc][1];
    for (int x = 0; x < 4; ++x) for (int y = 0; y < 4; ++y) sim[x][y] = (x == y) ? scorings[sc][2] : scorings[sc][3];
    for (int t = 0; t < 8000; ++t) {
      int la = 1 + rand() % 120, lb = 1 + rand() % 120;
      int a[128], b[128];
      const int related = rand() % 2;
      for (int j = 0; j < la; ++j) a[j] = rand() % 4;
      for (int i = 0; i < lb; ++i) b[i] = (related && i < la && rand() % 10) ? a[i] : rand() % 4;
      Best fw = full(a, la, b, lb);
      if (fw.s <= 0) continue;
      // reverse rectangle, reversed reads
      int ra[128], rb[128];
      for (int j = 0; j <= fw.j; ++j) ra[j] = a[fw.j - j];
      for (int i = 0; i <= fw.i; ++i) rb[i] = b[fw.i - i];
      Best rv = full(ra, fw.j + 1, rb, fw.i + 1);
      workFull += (long)(fw.i + 1) * ((fw.j + 1 + 15) / 16);
      for (int SW = 1; SW <= 64; SW *= 4) {
        long w = 0;
        Best st = stripped(ra, fw.j + 1, rb, fw.i + 1, SW, fw.s, &w);
        if (SW == 16) workStop += w;
        ++cases;
        if (st.s != rv.s || st.i != rv.i || st.j != rv.j) {
          if (fails < 5) printf("mismatch sc=%d SW=%d: full (%d,%d,%d) stop (%d,%d,%d)\n", sc, SW, rv.s, rv.i, rv.j, st.s, st.i, st.j);
          ++fails;
        }
      }
      if (rv.s != fw.s) { printf("reverse max %d != forward %d\n", rv.s, fw.s); ++fails; }
    }
  }
  printf("cases %ld, mismatches %ld, strip-rows with stop / without (SW=16): %.3f\n", cases, fails,
         (double)workStop / workFull);
  return fails != 0;
}
