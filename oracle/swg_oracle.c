/*
 * ORACLE - test infrastructure only.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this code, and
 * only as the checker or the timed CPU reference.  The product path (csharp_b200) never calls it.
 *
 * A CPU restatement, in plain C, of the reference's all-pairs alignment -> distance path
 * (DSC-SPIDAL/csharp, directory SalsaTPL/):
 *
 *   swo_align            Salsa.CoreTPL/Bio/Algorithms/SmithWaterman/SmithWatermanGotoh.cs:52-340
 *                        (Align :52-110, Construct :119-219, Traceback :229-332, Max :337-340,
 *                         Cell init score -inf Cell.cs:39-44, Directions enum Directions.cs:26-32)
 *   swo_distance_i16     Salsa.SmithWatermanMPI/Program.cs:259-285 (USE_INT16 ComputeDistance)
 *                        with PercentIdentity/PercentSimilarity Alignment.cs:187-195,
 *                        Kimura2 Alignment.cs:254-302, JukesCantor Alignment.cs:314-348
 *   swo_ms_distance_i16  Salsa.SmithWatermanMS/Program.cs:417-446, :479-495, :521-541, :555-668
 *   swo_block            Salsa.SmithWatermanMPI/Program.cs:203-257 (diagonal: j < i, mirrored)
 *                        Salsa.SmithWatermanMS/Program.cs:341-375 (full block, both orientations)
 *   nwo_align            documented restatement of the global (Needleman-Wunsch, affine) aligner
 *                        that Salsa.NeedlemanWunschTPL/Program.cs:210-263 calls in the closed
 *                        MBF Bio.dll 2.0; parity with Bio.dll is unpinned (its source is absent)
 *   nwo_distance_i16     Salsa.NeedlemanWunschTPL/Program.cs:270-300, :547-571, :583-604
 *   swo_parse_matrix     Salsa.CoreTPL/Bio/Algorithms/ScoringMatrix.cs:145-196
 *   swo_indp_align       the in-DP (no traceback) integer formulation the CUDA kernels use;
 *                        equal to swo_align on every pair (checked by the tests)
 *
 * Float semantics follow the source: IEEE binary32 with no contraction (build with
 * -ffp-contract=off -fno-fast-math), +-infinity as in the source, and the .NET x64 conv.i2
 * rule for (short)float: truncate toward zero through a 32-bit integer, NaN/out-of-range
 * giving 0x80000000, then keep the low 16 bits.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SWO_SIZE 127

enum { DIR_STOP = 0, DIR_LEFT = 1, DIR_DIAGONAL = 2, DIR_UP = 3 };
enum { ALN_PROTEIN = 0, ALN_NUCLEIC = 1 };
enum { DF_PERCENT_IDENTITY = 0, DF_KIMURA2 = 1, DF_JUKES_CANTOR = 2 };

typedef struct {
  float score;
  int end1, end2;     /* traceback start cell (Cell.Row, Cell.Column), DP coordinates */
  int start1, start2; /* PairwiseAlignment.Start1/Start2 */
  int identity, similarity, gaps, length;
} swo_result;

/* .NET x64 conv.i2 / conv.i4 of a float or double: cvtts*2si to int32, then truncate. */
static int32_t cs_conv_i4(double x) {
  if (!(x > -2147483649.0 && x < 2147483648.0)) return INT32_MIN;
  return (int32_t)x; /* C truncates toward zero */
}
static int16_t cs_conv_i2(double x) { return (int16_t)(uint16_t)(uint32_t)cs_conv_i4(x); }

/* Math.Max(float,float) in .NET: val1 > val2 ? val1 : (IsNaN(val1) ? val1 : val2). */
static float cs_maxf(float a, float b) { return (a > b) ? a : (isnan(a) ? a : b); }

/* ---- ScoringMatrix.Load (ScoringMatrix.cs:145-196) ------------------------------------------
 * Skip lines whose trimmed first char is '#'; the first other line holds the column letters
 * (whitespace-separated tokens, first char of each); every following line is "<row letter>
 * <score per column letter>".  Cells not named stay 0.  scores is [127][127] row-major. */
static int is_delim(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f'; }

static const char* next_token(const char* p, const char* end, const char** tok, int* toklen) {
  while (p < end && is_delim(*p)) p++;
  if (p >= end) return NULL;
  *tok = p;
  while (p < end && !is_delim(*p)) p++;
  *toklen = (int)(p - *tok);
  return p;
}

int swo_parse_matrix(const char* text, long textlen, float* scores) {
  memset(scores, 0, sizeof(float) * SWO_SIZE * SWO_SIZE);
  const char* p = text;
  const char* end = text + textlen;
  char acids[SWO_SIZE];
  memset(acids, 0, sizeof(acids));
  int header_done = 0;
  while (p < end) {
    const char* nl = memchr(p, '\n', (size_t)(end - p));
    const char* le = nl ? nl : end;
    const char* q = p;
    while (q < le && is_delim(*q)) q++;
    if (!header_done) {
      if (q < le && *q == '#') { p = nl ? nl + 1 : end; continue; }
      const char* t;
      int tl, j = 0;
      const char* r = q;
      while ((r = next_token(r, le, &t, &tl)) != NULL) {
        if (j >= SWO_SIZE) return -1;
        acids[j++] = t[0];
      }
      header_done = 1;
    } else if (q < le) {
      const char* t;
      int tl;
      const char* r = next_token(q, le, &t, &tl);
      unsigned char acid = (unsigned char)t[0];
      if (acid >= SWO_SIZE) return -2;
      for (int i = 0; i < SWO_SIZE; i++) {
        if (acids[i] == 0) continue;
        r = r ? next_token(r, le, &t, &tl) : NULL;
        if (!r) return -3;
        char buf[32];
        int n = tl < 31 ? tl : 31;
        memcpy(buf, t, (size_t)n);
        buf[n] = 0;
        unsigned char col = (unsigned char)acids[i];
        if (col >= SWO_SIZE) return -2;
        scores[acid * SWO_SIZE + col] = strtof(buf, NULL);
      }
    }
    p = nl ? nl + 1 : end;
  }
  return header_done ? 0 : -4;
}

/* ---- SmithWatermanGotoh.Align + Traceback --------------------------------------------------
 * aln1/aln2 (optional, capacity m+n) receive the aligned strings in forward order. */
int swo_align(const uint8_t* s1, int m0, const uint8_t* s2, int n0, const float* scores, float o,
              float e, swo_result* res, char* aln1, char* aln2) {
  const int m = m0 + 1, n = n0 + 1;
  uint8_t* pointers = (uint8_t*)malloc((size_t)m * n);
  int16_t* vgap = (int16_t*)malloc(sizeof(int16_t) * (size_t)m * n);
  int16_t* hgap = (int16_t*)malloc(sizeof(int16_t) * (size_t)m * n);
  float* g = (float*)malloc(sizeof(float) * (size_t)n);
  float* v = (float*)malloc(sizeof(float) * (size_t)n);
  char* r1 = (char*)malloc((size_t)(m0 + n0) + 1);
  char* r2 = (char*)malloc((size_t)(m0 + n0) + 1);
  if (!pointers || !vgap || !hgap || !g || !v || !r1 || !r2) {
    free(pointers); free(vgap); free(hgap); free(g); free(v); free(r1); free(r2);
    return -1;
  }
  memset(pointers, DIR_STOP, (size_t)m * n); /* default(Directions) is STOP; boundaries STOP */
  for (long k = 0; k < (long)m * n; k++) vgap[k] = hgap[k] = 1;

  /* Construct (:119-219) */
  float best = -INFINITY;
  int bi = 0, bj = 0;
  g[0] = -INFINITY;
  v[0] = 0;
  for (int j = 1; j < n; j++) { g[j] = -INFINITY; v[j] = 0; }
  for (int i = 1, k = n; i < m; i++, k += n) {
    float h = -INFINITY;
    float vdiag = v[0];
    for (int j = 1, l = k + 1; j < n; j++, l++) {
      float sim = scores[s1[i - 1] * SWO_SIZE + s2[j - 1]];
      float f = vdiag + sim;
      float g1 = g[j] - e, g2 = v[j] - o;
      if (g1 > g2) { g[j] = g1; vgap[l] = (int16_t)(vgap[l - n] + 1); }
      else g[j] = g2;
      float h1 = h - e, h2 = v[j - 1] - o;
      if (h1 > h2) { h = h1; hgap[l] = (int16_t)(hgap[l - 1] + 1); }
      else h = h2;
      vdiag = v[j];
      v[j] = cs_maxf(cs_maxf(f, g[j]), cs_maxf(h, 0.0f));
      if (v[j] == 0) pointers[l] = DIR_STOP;
      else if (v[j] == f) pointers[l] = DIR_DIAGONAL;
      else if (v[j] == g[j]) pointers[l] = DIR_UP;
      else pointers[l] = DIR_LEFT;
      if (v[j] > best) { best = v[j]; bi = i; bj = j; }
    }
  }

  /* Traceback (:229-332) */
  int i = bi, j = bj, k = i * n, len = 0, identity = 0, similarity = 0, gaps = 0;
  for (int going = 1; going;) {
    switch (pointers[k + j]) {
      case DIR_UP:
        for (int l = 0, L = vgap[k + j]; l < L; l++) {
          r1[len] = (char)s1[--i]; r2[len] = '-'; len++; k -= n; gaps++;
        }
        break;
      case DIR_DIAGONAL: {
        char c1 = (char)s1[--i], c2 = (char)s2[--j];
        k -= n;
        r1[len] = c1; r2[len] = c2; len++;
        if (c1 == c2) { identity++; similarity++; }
        else if (scores[(unsigned char)c1 * SWO_SIZE + (unsigned char)c2] > 0) similarity++;
        break;
      }
      case DIR_LEFT:
        for (int l = 0, L = hgap[k + j]; l < L; l++) {
          r1[len] = '-'; r2[len] = (char)s2[--j]; len++; gaps++;
        }
        break;
      default:
        going = 0;
        break;
    }
  }
  res->score = best;
  res->end1 = bi; res->end2 = bj;
  res->start1 = i; res->start2 = j;
  res->identity = identity; res->similarity = similarity; res->gaps = gaps; res->length = len;
  if (aln1 && aln2)
    for (int t = 0; t < len; t++) { aln1[t] = r1[len - 1 - t]; aln2[t] = r2[len - 1 - t]; }
  free(pointers); free(vgap); free(hgap); free(g); free(v); free(r1); free(r2);
  return 0;
}

/* ---- PairwiseAlignment distances (Alignment.cs:187-195, :254-348) ------------------------------ */
static double kimura2(const char* a, const char* b, int len) {
  double length = 0, gapc = 0, ts = 0, tv = 0;
  for (int i = 0; i < len; i++) {
    length++;
    char x = a[i], y = b[i];
    if (x != y) {
      if (x == '-' || y == '-') gapc++;
      else if ((x == 'A' && y == 'G') || (x == 'G' && y == 'A') || (x == 'C' && y == 'T') ||
               (x == 'T' && y == 'C'))
        ts++;
      else tv++;
    }
  }
  double P = ts / (length - gapc), Q = tv / (length - gapc);
  const double eps = 4.9406564584124654e-324; /* System.Double.Epsilon */
  if (1.0 - (2.0 * P + Q) <= eps) return 10;
  if (1.0 - (2.0 * Q) <= eps) return 10;
  return (-0.5 * log(1.0 - 2.0 * P - Q) - 0.25 * log(1.0 - 2.0 * Q));
}

/* Returns 0 and sets *d, or -1 where the reference throws ("Log(Zero)"). */
static int jukes_cantor(const char* a, const char* b, int len, double* out) {
  double length = 0, gapc = 0, diff = 0;
  for (int i = 0; i < len; i++) {
    length++;
    if (a[i] != b[i]) {
      if (a[i] == '-' || b[i] == '-') gapc++;
      else diff++;
    }
  }
  double d = 1.0 - ((4.0 / 3.0) * (diff / (length - gapc)));
  if (d <= 4.9406564584124654e-324) return -1;
  *out = (-0.75 * log(d));
  return 0;
}

/* ComputeDistance, USE_INT16 (SWG-MPI Program.cs:259-285).  Returns 0 and sets *out, or -1
 * where the reference would throw. */
int swo_distance_i16(const swo_result* r, const char* aln1, const char* aln2, int alignment_type,
                     int dist_fn, int16_t* out) {
  if (alignment_type == ALN_NUCLEIC) {
    if (dist_fn == DF_PERCENT_IDENTITY) {
      float pi = (float)r->identity / ((float)r->length * 1.0f);
      *out = cs_conv_i2((float)((1.0f - pi) * (float)32767));
      return 0;
    }
    if (dist_fn == DF_KIMURA2) {
      *out = cs_conv_i2(kimura2(aln1, aln2, r->length) * 32767);
      return 0;
    }
    if (dist_fn == DF_JUKES_CANTOR) {
      double d;
      if (jukes_cantor(aln1, aln2, r->length, &d)) return -1;
      *out = cs_conv_i2(d * 32767);
      return 0;
    }
    *out = 0; /* MinMaxNormScore is not a case of the SWG-MPI switch: result stays 0 */
    return 0;
  }
  float ps = (float)r->similarity / ((float)r->length * 1.0f);
  *out = cs_conv_i2((float)((1.0f - ps) * (float)32767));
  return 0;
}

/* SWG-MS ComputeDistance (MS Program.cs:417-446): identity over the full aligned length for
 * nucleotides (:479-495), similarity = non-gap pairs with positive score over the aligned
 * length for protein (:521-541).  Kimura2 adds the cap at 10 (:555-614); JukesCantor maps an
 * undefined log to 10 (:625-668). */
int swo_ms_distance_i16(const char* a, const char* b, int len, const float* scores,
                        int protein, int dist_fn, int16_t* out) {
  if (!protein) {
    if (dist_fn == DF_PERCENT_IDENTITY) {
      float id = 0.0f;
      for (int i = 0; i < len; i++) if (a[i] == b[i]) id++;
      float pi = id / (float)len;
      *out = cs_conv_i2((float)((1.0f - pi) * (float)32767));
      return 0;
    }
    if (dist_fn == DF_KIMURA2) {
      double k = kimura2(a, b, len);
      if (k > 10) k = 10;
      *out = cs_conv_i2(k * 32767);
      return 0;
    }
    if (dist_fn == DF_JUKES_CANTOR) {
      double d;
      if (jukes_cantor(a, b, len, &d)) d = 10;
      *out = cs_conv_i2(d * 32767);
      return 0;
    }
    return -1;
  }
  float sim = 0.0f;
  for (int i = 0; i < len; i++)
    if (a[i] != '-' && b[i] != '-' && scores[(unsigned char)a[i] * SWO_SIZE + (unsigned char)b[i]] > 0)
      sim++;
  float ps = sim / (float)len;
  *out = cs_conv_i2((float)((1.0f - ps) * (float)32767));
  return 0;
}

/* ---- Block loops (SWG-MPI Program.cs:203-257, SWG-MS Program.cs:341-375) ---------------------
 * seqs/offsets: concatenated sequences.  out is row-major over the block with leading dimension
 * ld (rows row_start..row_end, columns col_start..col_end).  mode 0 = SWG-MPI (diagonal blocks
 * compute j < i and mirror), mode 1 = SWG-MS (full block).  Returns pairs computed or < 0. */
long swo_block(const uint8_t* seqs, const int64_t* offsets, int row_start, int row_end,
               int col_start, int col_end, int is_diagonal, int mode, const float* scores,
               float o, float e, int alignment_type, int dist_fn, int16_t* out, long ld) {
  long count = 0;
  int cap = 0;
  char *a = NULL, *b = NULL;
  for (int i = row_start; i <= row_end; i++) {
    int jend = (mode == 0 && is_diagonal) ? i - 1 : col_end;
    for (int j = col_start; j <= jend; j++) {
      const uint8_t* si = seqs + offsets[i];
      const uint8_t* sj = seqs + offsets[j];
      int mi = (int)(offsets[i + 1] - offsets[i]), nj = (int)(offsets[j + 1] - offsets[j]);
      if (mi + nj + 1 > cap) {
        cap = mi + nj + 1;
        a = (char*)realloc(a, (size_t)cap);
        b = (char*)realloc(b, (size_t)cap);
      }
      swo_result r;
      if (swo_align(si, mi, sj, nj, scores, o, e, &r, a, b)) { free(a); free(b); return -1; }
      int16_t d;
      int rc = (mode == 0) ? swo_distance_i16(&r, a, b, alignment_type, dist_fn, &d)
                           : swo_ms_distance_i16(a, b, r.length, scores,
                                                 alignment_type == ALN_PROTEIN, dist_fn, &d);
      if (rc) { free(a); free(b); return -2; }
      out[(long)(i - row_start) * ld + (j - col_start)] = d;
      if (mode == 0 && is_diagonal) out[(long)(j - row_start) * ld + (i - col_start)] = d;
      count++;
    }
  }
  free(a);
  free(b);
  return count;
}

/* ---- Needleman-Wunsch (global, affine) restatement ---------------------------------------------
 * Same Gotoh recurrences and tie rules as SmithWatermanGotoh.Construct without the 0 floor:
 * gap of length L costs o + (L-1)e; a gap extends only when strictly better than reopening;
 * pointer priority DIAGONAL > UP > LEFT.  Boundaries: V(i,0) is an UP gap of length i, V(0,j) a
 * LEFT gap of length j.  Traceback runs from (m,n) to (0,0). */
int nwo_align(const uint8_t* s1, int m0, const uint8_t* s2, int n0, const float* scores, float o,
              float e, float* score_out, char* aln1, char* aln2, int* len_out) {
  const int m = m0 + 1, n = n0 + 1;
  uint8_t* pointers = (uint8_t*)malloc((size_t)m * n);
  int16_t* vgap = (int16_t*)malloc(sizeof(int16_t) * (size_t)m * n);
  int16_t* hgap = (int16_t*)malloc(sizeof(int16_t) * (size_t)m * n);
  float* g = (float*)malloc(sizeof(float) * (size_t)n);
  float* v = (float*)malloc(sizeof(float) * (size_t)n);
  char* r1 = (char*)malloc((size_t)(m0 + n0) + 1);
  char* r2 = (char*)malloc((size_t)(m0 + n0) + 1);
  if (!pointers || !vgap || !hgap || !g || !v || !r1 || !r2) {
    free(pointers); free(vgap); free(hgap); free(g); free(v); free(r1); free(r2);
    return -1;
  }
  pointers[0] = DIR_STOP;
  for (long k = 0; k < (long)m * n; k++) vgap[k] = hgap[k] = 1;
  v[0] = 0;
  g[0] = -INFINITY;
  for (int j = 1; j < n; j++) {
    v[j] = -o - (float)(j - 1) * e;
    g[j] = -INFINITY;
    pointers[j] = DIR_LEFT;
    hgap[j] = (int16_t)j;
  }
  for (int i = 1, k = n; i < m; i++, k += n) {
    float vleft = -o - (float)(i - 1) * e; /* V(i,0) */
    pointers[k] = DIR_UP;
    vgap[k] = (int16_t)i;
    float h = -INFINITY;
    float vdiag = v[0];
    v[0] = vleft;
    for (int j = 1, l = k + 1; j < n; j++, l++) {
      float sim = scores[s1[i - 1] * SWO_SIZE + s2[j - 1]];
      float f = vdiag + sim;
      float g1 = g[j] - e, g2 = v[j] - o;
      if (g1 > g2) { g[j] = g1; vgap[l] = (int16_t)(vgap[l - n] + 1); }
      else g[j] = g2;
      float h1 = h - e, h2 = v[j - 1] - o;
      if (h1 > h2) { h = h1; hgap[l] = (int16_t)(hgap[l - 1] + 1); }
      else h = h2;
      vdiag = v[j];
      v[j] = cs_maxf(cs_maxf(f, g[j]), h);
      if (v[j] == f) pointers[l] = DIR_DIAGONAL;
      else if (v[j] == g[j]) pointers[l] = DIR_UP;
      else pointers[l] = DIR_LEFT;
    }
  }
  *score_out = v[n - 1];
  int i = m - 1, j = n - 1, k = i * n, len = 0;
  while (i > 0 || j > 0) {
    switch (pointers[k + j]) {
      case DIR_UP:
        for (int l = 0, L = vgap[k + j]; l < L; l++) { r1[len] = (char)s1[--i]; r2[len] = '-'; len++; k -= n; }
        break;
      case DIR_DIAGONAL:
        r1[len] = (char)s1[--i]; r2[len] = (char)s2[--j]; len++; k -= n;
        break;
      case DIR_LEFT:
        for (int l = 0, L = hgap[k + j]; l < L; l++) { r1[len] = '-'; r2[len] = (char)s2[--j]; len++; }
        break;
      default:
        i = j = 0;
        break;
    }
  }
  for (int t = 0; t < len; t++) { aln1[t] = r1[len - 1 - t]; aln2[t] = r2[len - 1 - t]; }
  *len_out = len;
  free(pointers); free(vgap); free(hgap); free(g); free(v); free(r1); free(r2);
  return 0;
}

/* NW ComputeDistance (NW Program.cs:270-300): identity over the aligned region with leading and
 * trailing end gaps trimmed (:547-571), or similarity = non-gap positive-score pairs over the
 * full aligned length for protein (:583-604).  IndexOfNonGap returns -1 when a row is all gaps. */
int nwo_distance_i16(const char* a, const char* b, int len, const float* scores, int protein,
                     int16_t* out) {
  if (!protein) {
    long fa = -1, fb = -1, la = -1, lb = -1;
    for (int i = 0; i < len; i++) if (a[i] != '-') { fa = i; break; }
    for (int i = 0; i < len; i++) if (b[i] != '-') { fb = i; break; }
    for (int i = len - 1; i >= 0; i--) if (a[i] != '-') { la = i; break; }
    for (int i = len - 1; i >= 0; i--) if (b[i] != '-') { lb = i; break; }
    long first = fa > fb ? fa : fb, last = la < lb ? la : lb;
    float id = 0.0f;
    for (long i = first; i <= last; i++) if (a[i] == b[i]) id++;
    float pi = id / (float)((last - first) + 1);
    *out = cs_conv_i2((float)((1.0f - pi) * (float)32767));
    return 0;
  }
  float sim = 0.0f;
  for (int i = 0; i < len; i++)
    if (a[i] != '-' && b[i] != '-' && scores[(unsigned char)a[i] * SWO_SIZE + (unsigned char)b[i]] > 0)
      sim++;
  float ps = sim / (float)len;
  *out = cs_conv_i2((float)((1.0f - ps) * (float)32767));
  return 0;
}

/* NW distances of many pairs (s1 = sequence rows[k], s2 = cols[k]), OpenMP over host cores:
 * nwo_align then nwo_distance_i16 per pair.  Returns the number of pairs that failed. */
long nwo_pairs(const uint8_t* seqs, const int64_t* offsets, const int32_t* rows, const int32_t* cols,
               long npairs, const float* scores, float o, float e, int protein, int16_t* out,
               int threads) {
  long bad = 0;
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads) reduction(+ : bad)
  for (long k = 0; k < npairs; k++) {
    const int i = rows[k], j = cols[k];
    const int mi = (int)(offsets[i + 1] - offsets[i]), nj = (int)(offsets[j + 1] - offsets[j]);
    char* a = (char*)malloc((size_t)(mi + nj) + 1);
    char* b = (char*)malloc((size_t)(mi + nj) + 1);
    float score;
    int len = 0;
    if (!a || !b || nwo_align(seqs + offsets[i], mi, seqs + offsets[j], nj, scores, o, e, &score, a, b, &len)) {
      bad++;
    } else {
      nwo_distance_i16(a, b, len, scores, protein, &out[k]);
    }
    free(a);
    free(b);
  }
  return bad;
}

/* ---- In-DP integer formulation (what the CUDA kernels compute) ---------------------------------
 * Row-major Gotoh over int32 scores with, per state X in {V, G(up), H(left)}, the counters of the
 * path that reaches X: identity, similarity, aligned columns, DP start cell.  G/H take the
 * counters of the extended gap state or of V above/left, plus one column; V takes STOP->empty,
 * DIAGONAL->V(i-1,j-1)+column, UP->G, LEFT->H, in the source's priority.  The traceback start is
 * the first strictly greater V in row-major order.  Scores and penalties must be integers. */
typedef struct { int id, sim, len, si, sj; } cnt5;

int swo_indp_align(const uint8_t* s1, int m, const uint8_t* s2, int n, const int* iscores, int o,
                   int e, swo_result* res) {
  const int NEG = -(1 << 28);
  int* vrow = (int*)malloc(sizeof(int) * (size_t)(n + 1));
  int* grow = (int*)malloc(sizeof(int) * (size_t)(n + 1));
  cnt5* cv = (cnt5*)malloc(sizeof(cnt5) * (size_t)(n + 1));
  cnt5* cg = (cnt5*)malloc(sizeof(cnt5) * (size_t)(n + 1));
  if (!vrow || !grow || !cv || !cg) { free(vrow); free(grow); free(cv); free(cg); return -1; }
  for (int j = 0; j <= n; j++) {
    vrow[j] = 0; grow[j] = NEG;
    cv[j] = (cnt5){0, 0, 0, 0, j};
    cg[j] = cv[j];
  }
  int best = NEG, bi = 0, bj = 0;
  cnt5 bc = {0, 0, 0, 0, 0};
  for (int i = 1; i <= m; i++) {
    int h = NEG, vdiag = vrow[0], vleft = 0;
    cnt5 ch = {0, 0, 0, i, 0}, cdiag = cv[0], cleft = {0, 0, 0, i, 0};
    vrow[0] = 0;
    cv[0] = cleft;
    for (int j = 1; j <= n; j++) {
      int a = s1[i - 1], b = s2[j - 1];
      int f = vdiag + iscores[a * SWO_SIZE + b];
      cnt5 cf = cdiag;
      cf.len++;
      if (a == b) { cf.id++; cf.sim++; }
      else if (iscores[a * SWO_SIZE + b] > 0) cf.sim++;
      /* vertical gap */
      int g1 = grow[j] - e, g2 = vrow[j] - o, g;
      cnt5 cgn;
      if (g1 > g2) { g = g1; cgn = cg[j]; } else { g = g2; cgn = cv[j]; }
      cgn.len++;
      /* horizontal gap */
      int h1 = h - e, h2 = vleft - o;
      cnt5 chn;
      if (h1 > h2) { h = h1; chn = ch; } else { h = h2; chn = cleft; }
      chn.len++;
      ch = chn;
      int v = f > g ? f : g;
      v = v > h ? v : h;
      v = v > 0 ? v : 0;
      cnt5 cvn;
      if (v == 0) cvn = (cnt5){0, 0, 0, i, j};
      else if (v == f) cvn = cf;
      else if (v == g) cvn = cgn;
      else cvn = chn;
      vdiag = vrow[j];
      cdiag = cv[j];
      vrow[j] = v; grow[j] = g; cv[j] = cvn; cg[j] = cgn;
      vleft = v; cleft = cvn;
      if (v > best) { best = v; bi = i; bj = j; bc = cvn; }
    }
  }
  res->score = (m == 0 || n == 0) ? -INFINITY : (float)best; /* Cell.Score stays -inf */
  res->end1 = bi; res->end2 = bj;
  res->start1 = bc.si; res->start2 = bc.sj;
  res->identity = bc.id; res->similarity = bc.sim; res->length = bc.len;
  /* gap columns = aligned columns - diagonal columns; diagonal columns = (bi-si)+(bj-sj)-len */
  res->gaps = bc.len - ((bi - bc.si) + (bj - bc.sj) - bc.len);
  free(vrow); free(grow); free(cv); free(cg);
  return 0;
}

/* Many pairs in parallel: CPU baseline timing and big-sample parity.  Pair k aligns
 * (rows[k], cols[k]) with the source aligner (traceback, float) and writes the SWG-MPI
 * PercentIdentity/PercentSimilarity distance. */
long swo_pairs(const uint8_t* seqs, const int64_t* offsets, const int32_t* rows, const int32_t* cols,
               long npairs, const float* scores, float o, float e, int alignment_type, int16_t* out,
               int threads) {
  long bad = 0;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads) reduction(+ : bad)
  for (long k = 0; k < npairs; k++) {
    int i = rows[k], j = cols[k];
    int mi = (int)(offsets[i + 1] - offsets[i]), nj = (int)(offsets[j + 1] - offsets[j]);
    swo_result r;
    if (swo_align(seqs + offsets[i], mi, seqs + offsets[j], nj, scores, o, e, &r, NULL, NULL)) {
      bad++;
      continue;
    }
    int16_t d;
    swo_distance_i16(&r, NULL, NULL, alignment_type, DF_PERCENT_IDENTITY, &d);
    out[k] = d;
  }
  return bad;
}

/* SWG-MPI distances of many pairs with the in-DP integer formulation (pinned to the traceback
 * restatement and to the reference's golden vectors by the tests), OpenMP over host cores: the
 * fast checker for whole configurations.  Returns the number of pairs that failed. */
long swo_indp_pairs(const uint8_t* seqs, const int64_t* offsets, const int32_t* rows, const int32_t* cols,
                    long npairs, const int* iscores, int o, int e, int alignment_type, int16_t* out,
                    int threads) {
  long bad = 0;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads) reduction(+ : bad)
  for (long k = 0; k < npairs; k++) {
    const int i = rows[k], j = cols[k];
    const int mi = (int)(offsets[i + 1] - offsets[i]), nj = (int)(offsets[j + 1] - offsets[j]);
    swo_result r;
    if (swo_indp_align(seqs + offsets[i], mi, seqs + offsets[j], nj, iscores, o, e, &r)) {
      bad++;
      continue;
    }
    swo_distance_i16(&r, NULL, NULL, alignment_type, DF_PERCENT_IDENTITY, &out[k]);
  }
  return bad;
}

/* The same in-DP formulation with one counter word per state (aligned columns << 16 | counted
 * columns, counted = identical for nucleic, identical or positive-scoring for protein: the columns
 * ComputeDistance divides, SWG-MPI Program.cs:259-285), for checking whole configurations fast.
 * Pinned to swo_indp_align and the traceback restatement by the tests. */
long swo_count_pairs(const uint8_t* seqs, const int64_t* offsets, const int32_t* rows, const int32_t* cols,
                     long npairs, const int* iscores, int o, int e, int alignment_type, int16_t* out,
                     int threads) {
  long bad = 0;
  const int NEG = -(1 << 28);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads) reduction(+ : bad)
  for (long k = 0; k < npairs; k++) {
    const uint8_t* s1 = seqs + offsets[rows[k]];
    const uint8_t* s2 = seqs + offsets[cols[k]];
    const int m = (int)(offsets[rows[k] + 1] - offsets[rows[k]]), n = (int)(offsets[cols[k] + 1] - offsets[cols[k]]);
    int* V = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    int* G = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    uint32_t* CV = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n + 1));
    uint32_t* CG = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n + 1));
    if (!V || !G || !CV || !CG) {
      bad++;
      free(V); free(G); free(CV); free(CG);
      continue;
    }
    for (int j = 0; j <= n; j++) { V[j] = 0; G[j] = NEG; CV[j] = CG[j] = 0u; }
    int best = NEG;
    uint32_t bc = 0u;
    for (int i = 1; i <= m; i++) {
      const int a = s1[i - 1];
      const int* row = iscores + a * SWO_SIZE;
      int vdiag = 0, vleft = 0, h = NEG;
      uint32_t cdiag = 0u, cleft = 0u, ch = 0u;
      for (int j = 1; j <= n; j++) {
        const int b = s2[j - 1], sc = row[b];
        const uint32_t fl = (a == b || (alignment_type == ALN_PROTEIN && sc > 0)) ? 1u : 0u;
        const int f = vdiag + sc;
        const uint32_t cf = cdiag + 0x10000u + fl;
        /* selects written as masks: the data-dependent decisions do not branch */
        const int g1 = G[j] - e, g2 = V[j] - o;
        const uint32_t mg = 0u - (uint32_t)(g1 > g2);
        const int g = (int)(((uint32_t)g1 & mg) | ((uint32_t)g2 & ~mg));
        const uint32_t cg = ((CG[j] & mg) | (CV[j] & ~mg)) + 0x10000u;
        const int h1 = h - e, h2 = vleft - o;
        const uint32_t mh = 0u - (uint32_t)(h1 > h2);
        h = (int)(((uint32_t)h1 & mh) | ((uint32_t)h2 & ~mh));
        ch = ((ch & mh) | (cleft & ~mh)) + 0x10000u;
        int v = f > g ? f : g;
        v = v > h ? v : h;
        v = v > 0 ? v : 0;
        const uint32_t mf = 0u - (uint32_t)(v == f), mgv = 0u - (uint32_t)(v == g), mz = 0u - (uint32_t)(v != 0);
        const uint32_t cv = ((cf & mf) | (((cg & mgv) | (ch & ~mgv)) & ~mf)) & mz;
        vdiag = V[j]; cdiag = CV[j];
        V[j] = v; G[j] = g; CV[j] = cv; CG[j] = cg;
        vleft = v; cleft = cv;
        if (v > best) { best = v; bc = cv; }
      }
    }
    swo_result r;
    memset(&r, 0, sizeof(r));
    r.score = (m == 0 || n == 0) ? -INFINITY : (float)best;
    r.identity = r.similarity = (int)(bc & 0xFFFFu);
    r.length = (int)(bc >> 16);
    swo_distance_i16(&r, NULL, NULL, alignment_type, DF_PERCENT_IDENTITY, &out[k]);
    free(V); free(G); free(CV); free(CG);
  }
  return bad;
}
