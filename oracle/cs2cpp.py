"""Build oracle/_ref: the reference's own C# alignment path, mechanically rewritten to C++.

ORACLE - test infrastructure only.  Nothing in the product imports this file.

No C# toolchain exists on this machine (no mono / dotnet / csc), so the reference cannot be run
as-is.  This script reads the reference sources where they lie (default
``/root/reference/SalsaTPL``, or ``$SWG_REFERENCE_ROOT``) and applies a fixed list of *syntactic*
substitutions -- no semantic edits -- to the files that carry the SWG-MPI hot path:

* ``Salsa.CoreTPL/Bio/Algorithms/SmithWaterman/SmithWatermanGotoh.cs``  (whole class)
* ``Salsa.CoreTPL/Bio/Algorithms/SmithWaterman/{Cell,Directions,Markups}.cs``
* ``Salsa.CoreTPL/Bio/Algorithms/Alignment.cs``  (PairwiseAlignment; Summary text dropped)
* ``Salsa.CoreTPL/Bio/Algorithms/AlignmentType.cs``
* ``Salsa.CoreTPL/Bio/Algorithms/ScoringMatrix.cs``  (``Load``)
* ``Salsa.SmithWatermanMPI/Program.cs``  (``ComputeBlock`` and the USE_INT16 ``ComputeDistance``)

The output (``oracle/_ref/ref_swg.cpp`` and the shared library ``oracle/_ref/libref_swg.so``) is
generated, git-ignored and never committed; it travels to the GPU host as a built file.  The
small C++ runtime shim below (strings, arrays, the 127x127 grid, the tokenizer, resource lookup,
.NET conversion rules) stands in for the .NET base library the C# code calls.

Usage: python oracle/cs2cpp.py [--out oracle/_ref]
"""
import argparse
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
DEFAULT_REF = Path(os.environ.get("SWG_REFERENCE_ROOT", "/root/reference")) / "SalsaTPL"

PRELUDE = r'''
// Generated by oracle/cs2cpp.py from the reference's C# sources -- do not edit, do not commit.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>
#include <map>
#include <stdexcept>

typedef uint16_t CsChar;  // System.Char (UTF-16 code unit)
typedef int16_t TDistance;  // USE_INT16 (all hot-path csproj files define it)
static const double CS_DOUBLE_EPSILON = 4.9406564584124654e-324;  // System.Double.Epsilon

struct CsNull {};
static const CsNull null = {};

// .NET x64 conv.i4 / conv.i2: cvtts*2si to int32 (0x80000000 on NaN / overflow), keep 16 bits.
static inline int32_t cs_conv_i4(double x) {
  if (!(x > -2147483649.0 && x < 2147483648.0)) return INT32_MIN;
  return (int32_t)x;
}
static inline TDistance cs_conv_i2(double x) { return (TDistance)(uint16_t)(uint32_t)cs_conv_i4(x); }
static inline TDistance cs_conv_i2(float x) { return cs_conv_i2((double)x); }

template <class T> struct Arr {  // reference-typed T[] (zero-initialised like new T[n])
  std::shared_ptr<std::vector<T>> p;
  int Length = 0;
  Arr() {}
  explicit Arr(long n) : p(std::make_shared<std::vector<T>>((size_t)n)), Length((int)n) {}
  T& operator[](long i) const { return (*p)[(size_t)i]; }
  bool operator==(CsNull) const { return !p; }
  bool operator!=(CsNull) const { return !!p; }
};

template <class T> struct Grid2D {  // reference-typed T[,]
  std::shared_ptr<std::vector<T>> p;
  int n0 = 0, n1 = 0;
  Grid2D() {}
  Grid2D(int a, int b) : p(std::make_shared<std::vector<T>>((size_t)a * b)), n0(a), n1(b) {}
  T& operator()(long i, long j) const {
    if (i < 0 || i >= n0 || j < 0 || j >= n1) throw std::out_of_range("IndexOutOfRangeException");
    return (*p)[(size_t)i * n1 + j];
  }
};

struct CsString {  // System.String (null-able); code units stored as CsChar
  std::vector<CsChar> s;
  bool isnull = false;
  int Length = 0;
  CsString() {}
  CsString(CsNull) : isnull(true) {}
  CsString(const char* c) { for (; *c; ++c) s.push_back((unsigned char)*c); Length = (int)s.size(); }
  CsChar operator[](long i) const {
    if (i < 0 || i >= Length) throw std::out_of_range("IndexOutOfRangeException");
    return s[(size_t)i];
  }
  bool operator==(CsNull) const { return isnull; }
  bool operator!=(CsNull) const { return !isnull; }
  static bool ws(CsChar c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v'; }
  CsString Trim() const {
    CsString r;
    size_t a = 0, b = s.size();
    while (a < b && ws(s[a])) a++;
    while (b > a && ws(s[b - 1])) b--;
    r.s.assign(s.begin() + a, s.begin() + b);
    r.Length = (int)r.s.size();
    return r;
  }
  std::string narrow() const { std::string r; for (CsChar c : s) r.push_back((char)c); return r; }
};
static inline bool operator!=(CsNull, CsNull) { return false; }
// String concatenation only feeds Console.WriteLine (a no-op here); values are not formatted.
template <class T> static inline CsString operator+(const CsString& a, const T&) { return a; }
static inline CsString operator+(const char* a, const CsString& b) { CsString r(a); r.s.insert(r.s.end(), b.s.begin(), b.s.end()); r.Length = (int)r.s.size(); return r; }

struct CsMathT {
  // System.Math.Max(float, float): val1 > val2 ? val1 : (IsNaN(val1) ? val1 : val2)
  float Max(float a, float b) const { return (a > b) ? a : (std::isnan(a) ? a : b); }
  double Log(double x) const { return std::log(x); }
};
static const CsMathT Math = {};
struct CsConsoleT { template <class... A> void WriteLine(A&&...) const {} };
static const CsConsoleT Console = {};
struct CsSingleT { float Parse(const CsString& t) const { return std::strtof(t.narrow().c_str(), nullptr); } };
static const CsSingleT Single = {};
struct Exception : std::runtime_error { explicit Exception(const char* m) : std::runtime_error(m) {} };
struct SmithWatermanGotohException : std::runtime_error { explicit SmithWatermanGotohException(const char* m) : std::runtime_error(m) {} };

// Embedded resources "Salsa.Core.Bio.Algorithms.Matrices.<name>" (Salsa.CoreTPL.csproj).
static std::string g_matrix_dir;
struct Stream { std::vector<std::string> lines; size_t pos = 0; };
struct CsAssembly {
  Stream GetManifestResourceStream(const CsString& name) const {
    std::string n = name.narrow();
    const std::string pre = "Salsa.Core.Bio.Algorithms.Matrices.";
    if (n.compare(0, pre.size(), pre) != 0) throw std::runtime_error("no such resource");
    std::string path = g_matrix_dir + "/" + n.substr(pre.size());
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("resource stream is null");
    Stream st;
    std::string cur;
    int c;
    while ((c = std::fgetc(f)) != EOF) {
      if (c == '\n') { if (!cur.empty() && cur.back() == '\r') cur.pop_back(); st.lines.push_back(cur); cur.clear(); }
      else cur.push_back((char)c);
    }
    if (!cur.empty()) st.lines.push_back(cur);
    std::fclose(f);
    return st;
  }
};
struct CsAssemblyT { CsAssembly GetExecutingAssembly() const { return CsAssembly(); } };
static const CsAssemblyT Assembly = {};
struct StreamReader {
  Stream* st;
  explicit StreamReader(Stream& s) : st(&s) {}
  CsString ReadLine() { if (st->pos >= st->lines.size()) return CsString(null); return CsString(st->lines[st->pos++].c_str()); }
};
// ScoringMatrixTokenizer: a StringTokenizer over " \t\n\r\f" (ScoringMatrixTokenizer.cs:20,116-191).
struct ScoringMatrixTokenizer {
  std::vector<CsString> toks;
  size_t pos = 0;
  ScoringMatrixTokenizer() {}
  explicit ScoringMatrixTokenizer(const CsString& src) {
    CsString cur;
    auto flush = [&]() { if (!cur.s.empty()) { cur.Length = (int)cur.s.size(); toks.push_back(cur); cur = CsString(); } };
    for (CsChar c : src.s) {
      if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f') flush(); else cur.s.push_back(c);
    }
    flush();
  }
  bool HasMoreTokens() const { return pos < toks.size(); }
  CsString NextToken() { if (pos >= toks.size()) throw std::out_of_range("ArgumentOutOfRangeException"); return toks[pos++]; }
};

struct Sequence {  // Salsa.Core.Bio.Algorithms.Sequence (Sequence.cs:30-87): label + residues
  CsString Residues, Label;
  int Length = 0;
  bool isnull = false;
  CsChar operator[](long i) const { return Residues[i]; }
  bool operator==(CsNull) const { return isnull; }
};

struct ScoringMatrix;  // forward
'''

SCORING_MATRIX_SHELL_HEAD = r'''
struct ScoringMatrix {  // ScoringMatrix.cs:31-196 (fields and properties; Load is transliterated)
  static const int SIZE = 127;
  static const CsChar COMMENT_STARTER = '#';
  CsString _matrixName, Name;
  Grid2D<float> _scores, Scores;
  ScoringMatrix() {}
  ScoringMatrix(CsString matrixName, Grid2D<float> scores) : _matrixName(matrixName), Name(matrixName), _scores(scores), Scores(scores) {}
'''

POSTLUDE = r'''
// ---- ambient state of Salsa.SmithWatermanMPI.Program (Program.cs:28-66) --------------------
typedef int AlignmentTypeInt;
static AlignmentType _alignmentType = AlignmentType::Nucleic;
static DistanceFunctionType _distanceFunction = DistanceFunctionType::PercentIdentity;
static float _gapOpen = 14, _gapExtension = 4;
static CsString _scoringMatrixName = "EDNAFULL";
static std::vector<Sequence> _sequences;
static bool _writeAlignments = false;
static CsNull _writeAlignmentsWriter;
template <class W, class A> static void WriteAlignment(W, A) {}

struct Range { int StartIndex, EndIndex, Length; Range(int s, int e) : StartIndex(s), EndIndex(e), Length(e - s + 1) {} };
struct Block { Range RowRange, ColumnRange; Block(Range r, Range c) : RowRange(r), ColumnRange(c) {} };
template <class T> struct PartialMatrix {  // PartialMatrix.cs:59-63 indexer with global indices
  int r0, c0, cols;
  std::vector<T> el;
  PartialMatrix(int rs, int re, int cs, int ce) : r0(rs), c0(cs), cols(ce - cs + 1), el((size_t)(re - rs + 1) * (ce - cs + 1)) {}
  T& operator()(long i, long j) {
    long a = i - r0, b = j - c0;
    if (a < 0 || b < 0 || b >= cols || (size_t)(a * cols + b) >= el.size()) throw std::out_of_range("IndexOutOfRangeException");
    return el[(size_t)(a * cols + b)];
  }
};
'''

EXPORTS = r'''
// ---- C entry points for the tests (ctypes) ----------------------------------------------------
static Sequence make_seq(const uint8_t* p, int n) {
  Sequence s;
  for (int i = 0; i < n; i++) s.Residues.s.push_back(p[i]);
  s.Residues.Length = n;
  s.Length = n;
  return s;
}
extern "C" {
int ref_set_matrix_dir(const char* d) { g_matrix_dir = d; return 0; }

// SmithWatermanGotoh.Align on one pair; fills the PairwiseAlignment fields the path uses.
int ref_align(const char* matrix, const uint8_t* s1, int m, const uint8_t* s2, int n, float o, float e,
              float* score, int* identity, int* similarity, int* length, int* start1, int* start2, int* gaps,
              char* aln1, char* aln2) {
  try {
    ScoringMatrix sm = ScoringMatrix::Load(CsString(matrix));
    SmithWatermanGotoh aligner(AlignmentType::Nucleic);
    PairwiseAlignment a = aligner.Align(make_seq(s1, m), make_seq(s2, n), sm, o, e);
    *score = a.Score; *identity = a.Identity; *similarity = a.Similarity; *length = a.Sequence1.Length;
    *start1 = a.Start1; *start2 = a.Start2; *gaps = a.Gaps;
    if (aln1 && aln2) for (int i = 0; i < a.Sequence1.Length; i++) { aln1[i] = (char)a.Sequence1[i]; aln2[i] = (char)a.Sequence2[i]; }
    return 0;
  } catch (...) { return -1; }
}

// The body of ComputeBlock's loop (Align, then ComputeDistance) over an explicit pair list with
// one ScoringMatrix.Load, as one ComputeBlock call does: the timed CPU reference.
long ref_distances(const char* matrix, int alignment_type, int dist_fn, float o, float e,
                   const uint8_t* seqs, const int64_t* offsets, const int32_t* rows,
                   const int32_t* cols, long npairs, int16_t* out) {
  try {
    _alignmentType = alignment_type ? AlignmentType::Nucleic : AlignmentType::Protein;
    _distanceFunction = (DistanceFunctionType)dist_fn;
    ScoringMatrix scoringMatrix = ScoringMatrix::Load(CsString(matrix));
    SmithWatermanGotoh aligner(_alignmentType);
    for (long k = 0; k < npairs; k++) {
      const int i = rows[k], j = cols[k];
      Sequence si = make_seq(seqs + offsets[i], (int)(offsets[i + 1] - offsets[i]));
      Sequence sj = make_seq(seqs + offsets[j], (int)(offsets[j + 1] - offsets[j]));
      PairwiseAlignment alignment = aligner.Align(si, sj, scoringMatrix, o, e);
      out[k] = ComputeDistance(alignment);
    }
    return npairs;
  } catch (...) { return -1; }
}

// Program.ComputeBlock (SWG-MPI) over one block; out is an N x N row-major Int16 matrix that
// receives matrix[i,j] (and matrix[j,i] for diagonal blocks) at global indices.
long ref_compute_block(const char* matrix, int alignment_type, int dist_fn, float o, float e,
                       const uint8_t* seqs, const int64_t* offsets, int nseq,
                       int rs, int re, int cs, int ce, int is_diag, int16_t* out) {
  try {
    _scoringMatrixName = CsString(matrix);
    _alignmentType = alignment_type ? AlignmentType::Nucleic : AlignmentType::Protein;
    _distanceFunction = (DistanceFunctionType)dist_fn;
    _gapOpen = o; _gapExtension = e;
    _sequences.clear();
    for (int i = 0; i < nseq; i++) _sequences.push_back(make_seq(seqs + offsets[i], (int)(offsets[i + 1] - offsets[i])));
    PartialMatrix<TDistance> pm(0, nseq - 1, 0, nseq - 1);
    Block b(Range(rs, re), Range(cs, ce));
    long cnt = ComputeBlock(b, pm, is_diag != 0);
    for (size_t k = 0; k < pm.el.size(); k++) if (pm.el[k] != 0) out[k] = pm.el[k];
    return cnt;
  } catch (...) { return -1; }
}
}
'''


# ------------------------------------------------------------------------------------------------
# C# source helpers
def read(p: Path) -> str:
    t = p.read_text(encoding="utf-8-sig")
    return t.replace("\r\n", "\n")


def strip_comments_regions(code: str) -> str:
    code = re.sub(r"^\s*#(region|endregion)[^\n]*$", "", code, flags=re.M)
    code = re.sub(r"/\*.*?\*/", "", code, flags=re.S)
    code = re.sub(r"//[^\n]*", "", code)
    return code


def match_brace(s: str, i: int, open_c="{", close_c="}") -> int:
    """Index of the bracket closing the one at s[i] (string/char literals respected)."""
    depth, k = 0, i
    while k < len(s):
        c = s[k]
        if c in "\"'":
            q = c
            k += 1
            while s[k] != q:
                k += 2 if s[k] == "\\" else 1
        elif c == open_c:
            depth += 1
        elif c == close_c:
            depth -= 1
            if depth == 0:
                return k
        k += 1
    raise ValueError("unbalanced")


def class_body(code: str, header_regex: str) -> str:
    m = re.search(header_regex, code)
    if not m:
        raise ValueError(f"not found: {header_regex}")
    i = code.index("{", m.end() - 1)
    return code[i + 1: match_brace(code, i)]


def split_members(body: str):
    """Split a class body into (header, block_or_None) members at brace depth 0."""
    out, k, start = [], 0, 0
    while k < len(body):
        c = body[k]
        if c in "\"'":
            q = c
            k += 1
            while body[k] != q:
                k += 2 if body[k] == "\\" else 1
            k += 1
            continue
        if c == ";":
            out.append((body[start:k].strip(), None))
            start = k + 1
        elif c == "{":
            end = match_brace(body, k)
            out.append((body[start:k].strip(), body[k: end + 1]))
            start = end + 1
            k = end
        k += 1
    return [(h, b) for h, b in out if h or b]


def strip_attrs(h: str) -> str:
    return re.sub(r"^\s*\[[^\]]*\]\s*", "", h)


# ------------------------------------------------------------------------------------------------
# syntactic substitutions
def rewrite_2d_index(code: str) -> str:
    """a[x, y] -> a(x, y) for a top-level comma inside the brackets (C# rectangular arrays)."""
    out, k = [], 0
    while k < len(code):
        m = re.compile(r"\b([A-Za-z_]\w*)\s*\[").search(code, k)
        if not m:
            out.append(code[k:])
            break
        ob = m.end() - 1
        cb = match_brace(code, ob, "[", "]")
        inner = code[ob + 1: cb]
        depth, comma = 0, -1
        for i, c in enumerate(inner):
            if c in "([":
                depth += 1
            elif c in ")]":
                depth -= 1
            elif c == "," and depth == 0:
                comma = i
                break
        if comma >= 0 and inner.strip() != ",":
            out.append(code[k: m.start()])
            out.append(m.group(1) + "(" + rewrite_2d_index(inner) + ")")
        else:
            out.append(code[k: ob + 1])
            out.append(rewrite_2d_index(inner))
            out.append("]")
        k = cb + 1
    return "".join(out)


def rewrite_using_blocks(code: str) -> str:
    """using (decl) { ... }  ->  { decl; ... }"""
    while True:
        m = re.search(r"\busing\s*\(", code)
        if not m:
            return code
        op = m.end() - 1
        cp = match_brace(code, op, "(", ")")
        decl = code[op + 1: cp].strip()
        rest = code[cp + 1:]
        ob = rest.index("{")
        code = code[: m.start()] + "{ " + decl + ";" + rest[ob + 1:]


PROPERTY_CALLS = ("PercentIdentity", "PercentSimilarity", "PercentGaps")


def rewrite(code: str) -> str:
    code = strip_comments_regions(code)
    code = rewrite_using_blocks(code)
    code = re.sub(r"\bfloat\.NegativeInfinity\b", "(-INFINITY)", code)
    code = re.sub(r"\bdouble\.Epsilon\b", "CS_DOUBLE_EPSILON", code)
    code = re.sub(r"\bnew\s+(\w+)\s*\[\s*([^\],\[]+?)\s*,\s*([^\]\[]+?)\s*\]", r"Grid2D<\1>(\2, \3)", code)
    code = re.sub(r"\bnew\s+(\w+)\s*\[([^\]]+)\]", r"Arr<\1>(\2)", code)
    code = re.sub(r"\bnew\s+(\w+(?:<\w+>)?)\s*\(", r"\1(", code)
    code = re.sub(r"\bthrow\s+(\w+\()", r"throw \1", code)
    code = re.sub(r"\b(public|private|internal|protected|readonly|sealed|abstract|override)\s+", "", code)
    code = re.sub(r"\bfloat\s*\[\s*,\s*\]", "Grid2D<float>", code)
    code = re.sub(r"\b(char|short|float|int|Directions)\s*\[\s*\]", r"Arr<\1>", code)
    code = rewrite_2d_index(code)
    code = re.sub(r"\bchar\b", "CsChar", code)
    code = re.sub(r"\b(string|String)\b", "CsString", code)
    code = re.sub(r"\bvar\b", "auto", code)
    code = re.sub(r"\bbool\s+isDiagonal\b", "bool isDiagonal", code)
    code = re.sub(r"\b(Directions|Markups|AlignmentType|DistanceFunctionType)\.(\w+)", r"\1::\2", code)
    code = re.sub(r"\bPairwiseAlignment\.GAP\b", "PairwiseAlignment::GAP", code)
    code = re.sub(r"\bScoringMatrix\.Load\b", "ScoringMatrix::Load", code)
    code = re.sub(r"\(TDistance\)\s*\(", "cs_conv_i2(", code)
    code = re.sub(r"\bTDistance\.MaxValue\b", "((TDistance)32767)", code)
    code = re.sub(r"\bthis\.", "this->", code)
    for p in PROPERTY_CALLS:
        code = re.sub(r"\.\s*" + p + r"\b(?!\s*\()", "." + p + "()", code)
    return code


# ------------------------------------------------------------------------------------------------
def translate_enum(src: str, name: str) -> str:
    m = re.search(r"enum\s+" + name + r"\s*(:\s*byte)?\s*\{", src)
    i = src.index("{", m.start())
    body = src[i + 1: match_brace(src, i)]
    body = strip_comments_regions(body)
    base = " : uint8_t" if m.group(1) else ""
    return f"enum class {name}{base} {{{body}}};\n"


def translate_class(src: str, name: str, kind="struct", drop=(), collapse_trivial=True,
                    extra_head="", force_fields=()):
    """C# class -> C++ struct.  Trivial properties (get { return f; } / set { f = value; })
    collapse onto their backing field, which takes the property's name class-wide; other
    getter-only properties become methods."""
    body = class_body(src, r"class\s+" + name + r"\b[^{]*\{")
    members = split_members(strip_comments_regions(body))
    renames, methods, fields, getters = {}, [], [], []
    for h, b in members:
        h = strip_attrs(h)
        if b is None:
            fields.append(h)
            continue
        if "(" in h:
            methods.append((h, b))
            continue
        pname = h.split()[-1]
        if pname in drop:
            continue
        g = re.search(r"get\s*\{\s*return\s+(\w+)\s*;\s*\}", b)
        s = re.search(r"set\s*\{\s*(\w+)\s*=\s*value\s*;\s*\}", b)
        backing = (g.group(1) if g else None) or (s.group(1) if s else None)
        if collapse_trivial and backing and (g or s) and (pname in force_fields or g):
            renames[backing] = pname
        else:
            gm = re.search(r"\bget\s*\{", b)
            gi = b.index("{", gm.start())
            getters.append((h, b[gi: match_brace(b, gi) + 1]))
    out = [f"{kind} {name} {{\n{extra_head}"]

    def ren(t):
        for a, bb in renames.items():
            t = re.sub(r"\b" + a + r"\b", bb, t)
        return t

    for f in fields:
        f = rewrite(ren(f))
        f = re.sub(r"^\s*const\s+(CsChar|int|float)\s+", r"static const \1 ", f)
        f = re.sub(r"^\s*const\s+CsString\s+(\w+)\s*=", r"static constexpr const char* \1 =", f)
        f = re.sub(r"^\s*static\s+CsString\[\]\s+\w+", "", f)
        if f.strip():
            out.append("  " + f + ";\n")
    for h, b in getters:
        h = rewrite(ren(h))
        out.append(f"  {h}() const {rewrite(ren(b))}\n")
    for h, b in methods:
        hh = rewrite(ren(h))
        if re.search(r"\bstatic\s+" + name + r"\s*\(", hh):  # static constructor
            continue
        out.append(f"  {hh} {rewrite(ren(b))}\n")
    out.append("};\n")
    return "".join(out)


def extract_method(src: str, header_regex: str) -> str:
    m = re.search(header_regex, src)
    i = src.index("{", m.end() - 1)
    return src[m.start(): match_brace(src, i) + 1]


def build(ref: Path, outdir: Path) -> Path:
    core = ref / "Salsa.CoreTPL" / "Bio" / "Algorithms"
    swdir = core / "SmithWaterman"
    prog = read(ref / "Salsa.SmithWatermanMPI" / "Program.cs")
    parts = [PRELUDE]
    parts.append(translate_enum(read(swdir / "Directions.cs"), "Directions"))
    at = read(core / "AlignmentType.cs")
    parts.append(translate_enum(at, "AlignmentType"))
    parts.append(translate_enum(at, "DistanceFunctionType"))
    parts.append(translate_class(read(swdir / "Markups.cs"), "Markups"))
    parts.append(translate_class(read(swdir / "Cell.cs"), "Cell"))
    parts.append(translate_class(read(core / "Alignment.cs"), "PairwiseAlignment",
                                 drop=("Summary",), force_fields=("Name1", "Name2")))
    # ScoringMatrix: data members in the shell, Load transliterated.
    sm = read(core / "ScoringMatrix.cs")
    load = extract_method(strip_comments_regions(sm), r"public\s+static\s+ScoringMatrix\s+Load\s*\(")
    parts.append(SCORING_MATRIX_SHELL_HEAD + "  " + rewrite(load) + "\n};\n")
    parts.append(translate_class(read(swdir / "SmithWatermanGotoh.cs"), "SmithWatermanGotoh",
                                 kind="struct"))
    parts.append(POSTLUDE)
    p2 = strip_comments_regions(prog)
    cd_start = p2.index("#if USE_UINT16 || USE_INT16")
    cd_end = p2.index("#else", cd_start)
    compute_distance = p2[cd_start + len("#if USE_UINT16 || USE_INT16"): cd_end]
    parts.append(rewrite(compute_distance).replace("static TDistance ComputeDistance", "static TDistance ComputeDistance") + "\n")
    cb = extract_method(p2, r"static\s+int\s+ComputeBlock\s*\(")
    cb = rewrite(cb).replace("PartialMatrix<TDistance> matrix", "PartialMatrix<TDistance>& matrix")
    parts.append(cb + "\n")
    parts.append(EXPORTS)
    outdir.mkdir(parents=True, exist_ok=True)
    cpp = outdir / "ref_swg.cpp"
    cpp.write_text("".join(parts))
    mdir = outdir / "Matrices"
    mdir.mkdir(exist_ok=True)
    for f in (core / "Matrices").iterdir():
        shutil.copyfile(f, mdir / f.name)
    so = outdir / "libref_swg.so"
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-w", "-o", str(so), str(cpp)]
    subprocess.run(cmd, check=True)
    return so


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=str(DEFAULT_REF))
    ap.add_argument("--out", default=str(HERE / "_ref"))
    a = ap.parse_args()
    ref = Path(a.ref)
    if not ref.exists():
        print(f"reference sources not found at {ref}; oracle/_ref not rebuilt", file=sys.stderr)
        return 1
    so = build(ref, Path(a.out))
    print(so)
    return 0


if __name__ == "__main__":
    sys.exit(main())
