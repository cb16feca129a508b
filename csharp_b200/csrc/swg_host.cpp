// Host-side part of the C ABI: the formats and index arithmetic around the block handler.
//   scoring matrices  Salsa.CoreTPL/Bio/Algorithms/ScoringMatrix.cs:145-196
//   FASTA             Salsa.CoreTPL/Bio/IO/Parser.cs:123-180, FastaRecord.cs:112-118
//   partitioning      Salsa.CoreTPL/RangePartitioner.cs:17-55, BlockPartitioner.cs:10-28
//   block ownership   Salsa.SmithWatermanMPI/Program.cs:628-639
//   full matrix file  Salsa.SmithWatermanMPI/Program.cs:786-888, Blas/MatrixBinaryWriter.cs:73-92
//   MS block files    Salsa.SmithWatermanMS/Program.cs:1081-1160
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/swgb200.h"

namespace {

bool is_delim(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f'; }

// Splits [p, end) on the tokenizer's delimiters.
std::vector<std::string> tokens(const char* p, const char* end) {
  std::vector<std::string> out;
  while (p < end) {
    while (p < end && is_delim(*p)) p++;
    const char* s = p;
    while (p < end && !is_delim(*p)) p++;
    if (p > s) out.emplace_back(s, p);
  }
  return out;
}

// Letters and scores of the matrices shipped built in.  These are the standard published
// tables (NCBI NUC.4.4 "EDNAFULL" and BLOSUM62) in the reference's letter order; they must be
// identical to the reference's embedded resources of the same names for the distances to match.
const char kEdnaLetters[] = "ATGCSWRYKMBVHDNU";
const signed char kEdnaFull[16][16] = {
    {5, -4, -4, -4, -4, 1, 1, -4, -4, 1, -4, -1, -1, -1, -2, -4},
    {-4, 5, -4, -4, -4, 1, -4, 1, 1, -4, -1, -4, -1, -1, -2, 5},
    {-4, -4, 5, -4, 1, -4, 1, -4, 1, -4, -1, -1, -4, -1, -2, -4},
    {-4, -4, -4, 5, 1, -4, -4, 1, -4, 1, -1, -1, -1, -4, -2, -4},
    {-4, -4, 1, 1, -1, -4, -2, -2, -2, -2, -1, -1, -3, -3, -1, -4},
    {1, 1, -4, -4, -4, -1, -2, -2, -2, -2, -3, -3, -1, -1, -1, 1},
    {1, -4, 1, -4, -2, -2, -1, -4, -2, -2, -3, -1, -3, -1, -1, -4},
    {-4, 1, -4, 1, -2, -2, -4, -1, -2, -2, -1, -3, -1, -3, -1, 1},
    {-4, 1, 1, -4, -2, -2, -2, -2, -1, -4, -1, -3, -3, -1, -1, 1},
    {1, -4, -4, 1, -2, -2, -2, -2, -4, -1, -3, -1, -1, -3, -1, -4},
    {-4, -1, -1, -1, -1, -3, -3, -1, -1, -3, -1, -2, -2, -2, -1, -1},
    {-1, -4, -1, -1, -1, -3, -1, -3, -3, -1, -2, -1, -2, -2, -1, -4},
    {-1, -1, -4, -1, -3, -1, -3, -1, -3, -1, -2, -2, -1, -2, -1, -1},
    {-1, -1, -1, -4, -3, -1, -1, -3, -1, -3, -2, -2, -2, -1, -1, -1},
    {-2, -2, -2, -2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -2},
    {-4, 5, -4, -4, -4, 1, -4, 1, 1, -4, -1, -4, -1, -1, -2, 5},
};
const char kBlosumLetters[] = "ARNDCQEGHILKMFPSTWYVBZX*";
const signed char kBlosum62[24][24] = {
    {4, -1, -2, -2, 0, -1, -1, 0, -2, -1, -1, -1, -1, -2, -1, 1, 0, -3, -2, 0, -2, -1, 0, -4},
    {-1, 5, 0, -2, -3, 1, 0, -2, 0, -3, -2, 2, -1, -3, -2, -1, -1, -3, -2, -3, -1, 0, -1, -4},
    {-2, 0, 6, 1, -3, 0, 0, 0, 1, -3, -3, 0, -2, -3, -2, 1, 0, -4, -2, -3, 3, 0, -1, -4},
    {-2, -2, 1, 6, -3, 0, 2, -1, -1, -3, -4, -1, -3, -3, -1, 0, -1, -4, -3, -3, 4, 1, -1, -4},
    {0, -3, -3, -3, 9, -3, -4, -3, -3, -1, -1, -3, -1, -2, -3, -1, -1, -2, -2, -1, -3, -3, -2, -4},
    {-1, 1, 0, 0, -3, 5, 2, -2, 0, -3, -2, 1, 0, -3, -1, 0, -1, -2, -1, -2, 0, 3, -1, -4},
    {-1, 0, 0, 2, -4, 2, 5, -2, 0, -3, -3, 1, -2, -3, -1, 0, -1, -3, -2, -2, 1, 4, -1, -4},
    {0, -2, 0, -1, -3, -2, -2, 6, -2, -4, -4, -2, -3, -3, -2, 0, -2, -2, -3, -3, -1, -2, -1, -4},
    {-2, 0, 1, -1, -3, 0, 0, -2, 8, -3, -3, -1, -2, -1, -2, -1, -2, -2, 2, -3, 0, 0, -1, -4},
    {-1, -3, -3, -3, -1, -3, -3, -4, -3, 4, 2, -3, 1, 0, -3, -2, -1, -3, -1, 3, -3, -3, -1, -4},
    {-1, -2, -3, -4, -1, -2, -3, -4, -3, 2, 4, -2, 2, 0, -3, -2, -1, -2, -1, 1, -4, -3, -1, -4},
    {-1, 2, 0, -1, -3, 1, 1, -2, -1, -3, -2, 5, -1, -3, -1, 0, -1, -3, -2, -2, 0, 1, -1, -4},
    {-1, -1, -2, -3, -1, 0, -2, -3, -2, 1, 2, -1, 5, 0, -2, -1, -1, -1, -1, 1, -3, -1, -1, -4},
    {-2, -3, -3, -3, -2, -3, -3, -3, -1, 0, 0, -3, 0, 6, -4, -2, -2, 1, 3, -1, -3, -3, -1, -4},
    {-1, -2, -2, -1, -3, -1, -1, -2, -2, -3, -3, -1, -2, -4, 7, -1, -1, -4, -3, -2, -2, -1, -2, -4},
    {1, -1, 1, 0, -1, 0, 0, 0, -1, -2, -2, 0, -1, -2, -1, 4, 1, -3, -2, -2, 0, 0, 0, -4},
    {0, -1, 0, -1, -1, -1, -1, -2, -2, -1, -1, -1, -1, -2, -1, 1, 5, -2, -2, 0, -1, -1, 0, -4},
    {-3, -3, -4, -4, -2, -2, -3, -2, -2, -3, -2, -3, -1, 1, -4, -3, -2, 11, 2, -3, -4, -3, -2, -4},
    {-2, -2, -2, -3, -2, -1, -2, -3, 2, -1, -1, -2, -1, 3, -3, -2, -2, 2, 7, -1, -3, -2, -1, -4},
    {0, -3, -3, -3, -1, -2, -2, -3, -3, 3, 1, -2, 1, -1, -2, -2, 0, -3, -1, 4, -3, -2, -1, -4},
    {-2, -1, 3, 4, -3, 0, 1, -1, 0, -3, -4, 0, -3, -3, -2, 0, -1, -4, -3, -3, 4, 1, -1, -4},
    {-1, 0, 0, 1, -3, 3, 4, -2, 0, -3, -3, 1, -1, -3, -1, 0, -1, -3, -2, -2, 1, 4, -1, -4},
    {0, -1, -1, -1, -2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -2, 0, 0, -2, -1, -1, -1, -1, -1, -4},
    {-4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, 1},
};
// IDENTITY and MATCH: 24 letters; +1 on the diagonal except X-X and *-* (0); off-diagonal
// -10000 (IDENTITY) or -1 (MATCH).
const char kIdLetters[] = "ARNBDCQZEGHILKMFPSTWYVX*";

void fill_rule_matrix(int16_t out[128][128], int off) {
  std::memset(out, 0, sizeof(int16_t) * 128 * 128);
  for (int a = 0; kIdLetters[a]; a++)
    for (int b = 0; kIdLetters[b]; b++) {
      const unsigned char ca = (unsigned char)kIdLetters[a], cb = (unsigned char)kIdLetters[b];
      int v = (a == b) ? 1 : off;
      if (a == b && (ca == 'X' || ca == '*')) v = 0;
      out[ca][cb] = (int16_t)v;
    }
}

}  // namespace

extern "C" {

int sw_parse_scoring_matrix(const char* text, int64_t text_len, int16_t out[128][128]) {
  if (!text || !out || text_len < 0) return SW_E_ARG;
  std::memset(out, 0, sizeof(int16_t) * 128 * 128);
  const char* p = text;
  const char* end = text + text_len;
  std::vector<char> acids;
  bool header = false;
  while (p < end) {
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
    const char* le = nl ? nl : end;
    std::vector<std::string> t = tokens(p, le);
    p = nl ? nl + 1 : end;
    if (!header) {
      // leading lines whose trimmed text starts with '#' are comments (ScoringMatrix.cs:167)
      if (!t.empty() && t[0][0] == '#') continue;
      if (t.empty()) return SW_E_ARG;  // the reference indexes [0] of an empty line and throws
      for (auto& s : t) acids.push_back(s[0]);
      if (acids.size() > 127) return SW_E_ARG;
      header = true;
      continue;
    }
    if (t.empty()) return SW_E_ARG;
    const unsigned char a = (unsigned char)t[0][0];
    if (a >= 127) return SW_E_ARG;
    size_t k = 1;
    for (size_t c = 0; c < acids.size(); c++) {
      if (acids[c] == 0) continue;
      if (k >= t.size()) return SW_E_ARG;  // NextToken throws past the last token
      char* ep = nullptr;
      const double v = std::strtod(t[k++].c_str(), &ep);
      if (!ep || *ep != 0) return SW_E_ARG;
      if (v != std::floor(v) || std::fabs(v) > 16383) return SW_E_UNSUPPORTED;
      const unsigned char b = (unsigned char)acids[c];
      if (b >= 127) return SW_E_ARG;
      out[a][b] = (int16_t)v;
    }
  }
  return header ? SW_OK : SW_E_ARG;
}

int sw_builtin_scoring_matrix(const char* name, int16_t out[128][128]) {
  if (!name || !out) return SW_E_ARG;
  std::memset(out, 0, sizeof(int16_t) * 128 * 128);
  if (!std::strcmp(name, "EDNAFULL")) {
    for (int a = 0; a < 16; a++)
      for (int b = 0; b < 16; b++)
        out[(unsigned char)kEdnaLetters[a]][(unsigned char)kEdnaLetters[b]] = kEdnaFull[a][b];
    return SW_OK;
  }
  if (!std::strcmp(name, "BLOSUM62")) {
    for (int a = 0; a < 24; a++)
      for (int b = 0; b < 24; b++)
        out[(unsigned char)kBlosumLetters[a]][(unsigned char)kBlosumLetters[b]] = kBlosum62[a][b];
    return SW_OK;
  }
  if (!std::strcmp(name, "IDENTITY")) { fill_rule_matrix(out, -10000); return SW_OK; }
  if (!std::strcmp(name, "MATCH")) { fill_rule_matrix(out, -1); return SW_OK; }
  return SW_E_ARG;
}

int sw_parse_fasta(const char* text, int64_t text_len, uint8_t* concat, int64_t* offsets,
                   int32_t* count, int64_t* residues) {
  if (!text || text_len < 0 || !count || !residues) return SW_E_ARG;
  const bool fill = concat && offsets;
  int32_t n = 0;
  int64_t r = 0;
  bool in_record = false;
  const char* p = text;
  const char* end = text + text_len;
  while (p < end) {
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
    const char* le = nl ? nl : end;
    const char* a = p;
    const char* b = le;
    p = nl ? nl + 1 : end;
    while (a < b && (*a == ' ' || *a == '\t' || *a == '\r')) a++;
    while (b > a && (b[-1] == ' ' || b[-1] == '\t' || b[-1] == '\r')) b--;
    if (a == b) continue;
    if (*a == '>') {
      if (fill) offsets[n] = r;
      n++;
      in_record = true;
      continue;
    }
    if (!in_record) return SW_E_ARG;  // residues before the first label do not parse
    for (const char* q = a; q < b; q++) {
      char c = *q;
      if (c >= 'a' && c <= 'z') c = (char)(c - 'a' + 'A');  // Residues += residues.ToUpper()
      if (fill) concat[r] = (uint8_t)c;
      r++;
    }
  }
  if (fill) offsets[n] = r;
  *count = n;
  *residues = r;
  return SW_OK;
}

int sw_partition_ranges(int32_t start, int32_t length, int32_t parts, int32_t* starts,
                        int32_t* ends) {
  if (parts < 1 || !starts || !ends) return SW_E_ARG;  // ArgumentOutOfRangeException
  const int32_t chunk = length / parts;
  int32_t rem = length % parts;
  for (int32_t i = 0; i < parts; i++) {
    if (rem > 0) {
      starts[i] = start;
      ends[i] = start + chunk;
      start += chunk + 1;
      rem--;
    } else {
      starts[i] = start;
      ends[i] = start + chunk - 1;
      start += chunk;
    }
  }
  return SW_OK;
}

int sw_block_is_computed(int32_t r, int32_t c) {
  if (r == c) return 1;
  const int odd = (r + c) & 1;
  return (r > c && !odd) || (r < c && odd);
}

int sw_write_full_matrix(const char* path, const int16_t* m, int64_t rows, int64_t cols,
                         int64_t ld) {
  if (!path || (!m && rows * cols > 0) || rows < 0 || cols < 0 || ld < cols) return SW_E_ARG;
  FILE* f = std::fopen(path, "wb");
  if (!f) return SW_E_IO;
  std::vector<uint8_t> buf((size_t)cols * 2);
  for (int64_t i = 0; i < rows; i++) {
    const int16_t* row = m + i * ld;
    for (int64_t j = 0; j < cols; j++) {  // BinaryWriter.Write(short): little-endian
      const uint16_t v = (uint16_t)row[j];
      buf[(size_t)j * 2] = (uint8_t)(v & 0xFF);
      buf[(size_t)j * 2 + 1] = (uint8_t)(v >> 8);
    }
    if (cols && std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) {
      std::fclose(f);
      return SW_E_IO;
    }
  }
  return std::fclose(f) == 0 ? SW_OK : SW_E_IO;
}

namespace {
void put_u16(std::vector<uint8_t>& b, uint32_t v) { b.push_back((uint8_t)(v & 0xFF)); b.push_back((uint8_t)((v >> 8) & 0xFF)); }
void put_u32(std::vector<uint8_t>& b, uint32_t v) { for (int k = 0; k < 4; k++) b.push_back((uint8_t)((v >> (8 * k)) & 0xFF)); }
void put_str(std::vector<uint8_t>& b, const char* s) {
  const size_t n = s ? std::strlen(s) : 0;
  put_u16(b, (uint32_t)n);  // (UInt16) length then the ASCII bytes
  for (size_t k = 0; k < n; k++) b.push_back((uint8_t)s[k]);
}
bool get_u16(FILE* f, uint32_t* v) { uint8_t x[2]; if (std::fread(x, 1, 2, f) != 2) return false; *v = x[0] | (x[1] << 8); return true; }
bool get_u32(FILE* f, uint32_t* v) { uint8_t x[4]; if (std::fread(x, 1, 4, f) != 4) return false; *v = x[0] | (x[1] << 8) | (x[2] << 16) | ((uint32_t)x[3] << 24); return true; }
bool skip_str(FILE* f) { uint32_t n; if (!get_u16(f, &n)) return false; return std::fseek(f, (long)n, SEEK_CUR) == 0; }

struct MsDims { uint32_t rank, rb, cb, rs, re, cs, ce; };
bool read_ms_header(FILE* f, MsDims* d) {
  if (!skip_str(f) || !get_u16(f, &d->rank) || !skip_str(f) || !skip_str(f)) return false;
  if (!get_u16(f, &d->rb) || !get_u16(f, &d->cb)) return false;
  if (!get_u32(f, &d->rs) || !get_u32(f, &d->re) || !get_u32(f, &d->cs) || !get_u32(f, &d->ce)) return false;
  for (int k = 0; k < 4; k++) if (!skip_str(f)) return false;
  return d->re >= d->rs && d->ce >= d->cs;
}
}  // namespace

int sw_write_ms_block(const char* path, const sw_ms_block_header* h, const int16_t* values,
                      int64_t ld) {
  if (!path || !h || !values) return SW_E_ARG;
  if (h->row_end < h->row_start || h->col_end < h->col_start) return SW_E_ARG;
  const int64_t cols = (int64_t)h->col_end - h->col_start + 1;
  const int64_t rows = (int64_t)h->row_end - h->row_start + 1;
  if (ld < cols) return SW_E_ARG;
  std::vector<uint8_t> b;
  put_str(b, h->project);
  put_u16(b, (uint32_t)h->rank);
  put_str(b, h->system);
  put_str(b, h->fasta);
  put_u16(b, (uint32_t)h->row_block);
  put_u16(b, (uint32_t)h->col_block);
  put_u32(b, (uint32_t)h->row_start);
  put_u32(b, (uint32_t)h->row_end);
  put_u32(b, (uint32_t)h->col_start);
  put_u32(b, (uint32_t)h->col_end);
  put_str(b, h->row_start_id);
  put_str(b, h->row_end_id);
  put_str(b, h->col_start_id);
  put_str(b, h->col_end_id);
  for (int64_t i = 0; i < rows; i++)
    for (int64_t j = 0; j < cols; j++) put_u16(b, (uint16_t)values[i * ld + j]);
  FILE* f = std::fopen(path, "wb");
  if (!f) return SW_E_IO;
  const bool ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
  return (std::fclose(f) == 0 && ok) ? SW_OK : SW_E_IO;
}

int sw_read_ms_block_dims(const char* path, int32_t* rank, int32_t* row_block, int32_t* col_block,
                          int32_t* row_start, int32_t* row_end, int32_t* col_start,
                          int32_t* col_end) {
  if (!path) return SW_E_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return SW_E_IO;
  MsDims d;
  const bool ok = read_ms_header(f, &d);
  std::fclose(f);
  if (!ok) return SW_E_IO;
  if (rank) *rank = (int32_t)d.rank;
  if (row_block) *row_block = (int32_t)d.rb;
  if (col_block) *col_block = (int32_t)d.cb;
  if (row_start) *row_start = (int32_t)d.rs;
  if (row_end) *row_end = (int32_t)d.re;
  if (col_start) *col_start = (int32_t)d.cs;
  if (col_end) *col_end = (int32_t)d.ce;
  return SW_OK;
}

int sw_read_ms_block_values(const char* path, int16_t* values, int64_t ld) {
  if (!path || !values) return SW_E_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return SW_E_IO;
  MsDims d;
  if (!read_ms_header(f, &d)) { std::fclose(f); return SW_E_IO; }
  const int64_t rows = (int64_t)d.re - d.rs + 1, cols = (int64_t)d.ce - d.cs + 1;
  if (ld < cols) { std::fclose(f); return SW_E_ARG; }
  for (int64_t i = 0; i < rows; i++)
    for (int64_t j = 0; j < cols; j++) {
      uint32_t v;
      if (!get_u16(f, &v)) { std::fclose(f); return SW_E_IO; }
      values[i * ld + j] = (int16_t)(uint16_t)v;
    }
  std::fclose(f);
  return SW_OK;
}

}  // extern "C"
