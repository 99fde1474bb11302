/*
 * sw_oracle.c -- CPU oracle for the batched affine-gap Smith-Waterman path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only
 * as the checker.  The product (ipuma-lib_b200/) never links or calls it.
 *
 * It restates, in plain C and int32 arithmetic, the per-pair recurrence of
 * the ipuma IPU codelet `SWAffine::compute`
 * (src/codelets/codelet_batch_affine.cpp:37-127; identical recurrence in
 * `MultiSWAffine::compute`, src/codelets/codelet_multi_affine.cpp:37-126):
 *
 *   for i over B (outer), j over A (inner):
 *     E     = max(Hleft + gI + gE, E + gE)          E reset to gI per row
 *     F[j]  = max(H[j] + gI + gE, F[j] + gE)        F zeroed per pair
 *     Hnew  = max(diag + sim[a[j]][b[i]], E, F[j], 0)
 *     if (Hnew > best) { Aend = j; Bend = i; best = Hnew; }   (strict >)
 *
 * and the optional reverse pass over [Bend..0] x [Aend..0] that yields the
 * start coordinates with the same strict-> rule in reverse order
 * (codelet_batch_affine.cpp:89-115).  Ranges are packed as
 * `start | end << 16` with uint16 halves (codelet_batch_affine.cpp:117-123).
 *
 * One intentional deviation, shared with the product: a pair with an empty
 * sequence yields score 0 / ranges 0 and does not stop the processing of the
 * following pairs (the codelet `break`s out of its tile loop at :60).
 *
 * Parity of this restatement is pinned by tests/test_oracle_golden.py against
 * the reference's known answers (test/simple-test.cpp:25-45,
 * test/mn_cmp-test.cpp:29-57) and against outputs of the reference codelet
 * itself, compiled for the host by oracle/Makefile (fixtures in tests/golden/).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static inline int imax(int a, int b) { return a > b ? a : b; }

/*
 * One pass of the recurrence over a (length alen, stride da from a0) and
 * b (length blen, stride db from b0).  A stride of -1 walks a sequence
 * backwards, which is how the reverse pass of the codelet reads a[Aend..0]
 * and b[Bend..0].  Returns the best score and writes the (j, i) step counts
 * of the first strict maximum in (i, j) row-major order.
 */
static int oracle_pass(const uint8_t* a0, int alen, int da, const uint8_t* b0, int blen, int db,
                       const int8_t* sim, int simN, int gI, int gE, int32_t* C, int32_t* F,
                       int* bestJ, int* bestI) {
  int s = 0;
  int bj = 0, bi = 0;
  memset(C, 0, sizeof(int32_t) * (size_t)alen);
  memset(F, 0, sizeof(int32_t) * (size_t)alen);
  for (int i = 0; i < blen; ++i) {
    const int bc = b0[(long)i * db];
    int e = gI;
    int hleft = 0;
    int diag = 0;
    for (int j = 0; j < alen; ++j) {
      const int ac = a0[(long)j * da];
      e = imax(hleft + gI + gE, e + gE);
      F[j] = imax(C[j] + gI + gE, F[j] + gE);
      int h = imax(diag + sim[ac * simN + bc], e);
      h = imax(h, F[j]);
      h = imax(h, 0);
      diag = C[j];
      C[j] = h;
      hleft = h;
      if (h > s) {
        bj = j;
        bi = i;
        s = h;
      }
    }
  }
  *bestJ = bj;
  *bestI = bi;
  return s;
}

/* Packs a (start, end) range with uint16 halves like codelet_batch_affine.cpp:117-123. */
static inline int32_t pack_range(int start, int end) {
  uint32_t v = (uint32_t)(uint16_t)start | ((uint32_t)(uint16_t)end << 16);
  return (int32_t)v;
}

/*
 * Aligns one pair.  `scratch` holds 2*alen int32.  Writes score, arange and
 * brange like one slot of the codelet.
 */
void oracle_sw_pair(const uint8_t* a, int alen, const uint8_t* b, int blen, const int8_t* sim,
                    int simN, int gI, int gE, int forwardOnly, int32_t* scratch, int32_t* score,
                    int32_t* arange, int32_t* brange) {
  if (alen <= 0 || blen <= 0) {
    *score = 0;
    *arange = 0;
    *brange = 0;
    return;
  }
  int32_t* C = scratch;
  int32_t* F = scratch + alen;
  int aend = 0, bend = 0, astart = 0, bstart = 0;
  int s = oracle_pass(a, alen, 1, b, blen, 1, sim, simN, gI, gE, C, F, &aend, &bend);
  if (!forwardOnly) {
    int rj = 0, ri = 0;
    oracle_pass(a + aend, aend + 1, -1, b + bend, bend + 1, -1, sim, simN, gI, gE, C, F, &rj, &ri);
    astart = aend - rj;
    bstart = bend - ri;
  }
  /* uint16 truncation of the coordinates, as in the codelet. */
  *score = s;
  *arange = pack_range(astart, aend);
  *brange = pack_range(bstart, bend);
}

/*
 * Aligns n pairs.  Pair p reads a = codes + a_off[p] (a_len[p] codes) and
 * b = codes + b_off[p].  `nthreads` <= 0 uses all OpenMP threads.
 */
void oracle_sw_batch(const uint8_t* codes, const int64_t* a_off, const int32_t* a_len,
                     const int64_t* b_off, const int32_t* b_len, int64_t n, const int8_t* sim,
                     int simN, int gI, int gE, int forwardOnly, int nthreads, int32_t* score,
                     int32_t* arange, int32_t* brange) {
  int maxA = 1;
  for (int64_t p = 0; p < n; ++p) maxA = imax(maxA, a_len[p]);
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    int32_t* scratch = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)maxA);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
    for (int64_t p = 0; p < n; ++p) {
      oracle_sw_pair(codes + a_off[p], a_len[p], codes + b_off[p], b_len[p], sim, simN, gI, gE,
                     forwardOnly, scratch, &score[p], &arange[p], &brange[p]);
    }
    free(scratch);
  }
}

/* Number of OpenMP threads the batch call uses by default. */
int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
