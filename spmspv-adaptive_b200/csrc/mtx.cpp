// MatrixMarket reader and the binary CSR cache (host only).
//
// spmx_mtx_read restates the reading half of the reference's ReadMTX
// (hice-spmspv/hice/la/include/spmspv/mtx.hpp:218-333) with the same meaning:
//   - indices are 1-based in the file and 0-based in the output;
//   - field "real" keeps the value (parsed as double, then rounded to float,
//     like fscanf("%lf") followed by the cast), "integer" converts the
//     integer, "pattern" stores 1, "complex" reads both parts and stores 1;
//   - symmetry "symmetric" appends the mirror (c, r, v) right after every
//     off-diagonal entry (r, c, v); "skew-symmetric" and "hermitian" are NOT
//     expanded, as in the reference;
//   - duplicates are kept.
// The (row, col) sort that follows in the reference (mtx.hpp:335-360,
// std::sort) is not done here: spmx_input_coo sorts on the GPU.
//
// Departures, all on malformed input where the reference reads on blindly:
// out-of-range indices, a short or long entry section, a missing size line
// and "array" files are reported as SPMX_ERR_INVALID_VALUE with the line
// number.  Qualifiers compare case-insensitively (the MatrixMarket format
// defines them so; the reference compares lowercase only).
//
// The parser maps the file and splits the entry section into chunks that
// start at line starts.  Pass 1 counts the entry lines of every chunk, pass 2
// parses each chunk into its slice of the output, pass 3 (symmetric files)
// spreads the entries and their mirrors.  Positions come from prefix sums, so
// the output does not depend on the thread count.
//
// spmx_csr_store / _load_header / _load write and read the reference's
// binary cache (mtx.hpp:706-808): 9 magic bytes "Hola\1CSR\1", 3 bytes of
// padding (the struct's alignment), int32 rows, cols, nnz, then float
// val[nnz], int32 col[nnz], int32 rowptr[rows + 1].
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <charconv>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "spmx.h"

namespace spmx {
int set_error(int code, const std::string& msg);
}
using spmx::set_error;

namespace {

struct MappedFile {
  const char* p = nullptr;
  size_t n = 0;
  int fd = -1;
  ~MappedFile() {
    if (p && n) munmap((void*)p, n);
    if (fd >= 0) close(fd);
  }
};

int map_file(const char* path, MappedFile* f) {
  f->fd = open(path, O_RDONLY);
  if (f->fd < 0) return set_error(SPMX_ERR_INVALID_VALUE, std::string("cannot open ") + path);
  struct stat st;
  if (fstat(f->fd, &st) != 0) return set_error(SPMX_ERR_INVALID_VALUE, std::string("cannot stat ") + path);
  f->n = (size_t)st.st_size;
  if (f->n == 0) return SPMX_SUCCESS;
  void* q = mmap(nullptr, f->n, PROT_READ, MAP_PRIVATE, f->fd, 0);
  if (q == MAP_FAILED) {
    f->n = 0;
    return set_error(SPMX_ERR_INVALID_VALUE, std::string("cannot map ") + path);
  }
  madvise(q, f->n, MADV_SEQUENTIAL);
  f->p = (const char*)q;
  return SPMX_SUCCESS;
}

inline bool is_blank(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\f' || c == '\v'; }

inline const char* skip_blank(const char* p, const char* e) {
  while (p < e && is_blank(*p)) ++p;
  return p;
}

inline const char* end_of_line(const char* p, const char* e) {
  const void* q = std::memchr(p, '\n', (size_t)(e - p));
  return q ? (const char*)q : e;
}

// one whitespace-delimited token of [p, e); advances p past it
bool next_token(const char*& p, const char* e, std::string* tok) {
  p = skip_blank(p, e);
  const char* s = p;
  while (p < e && !is_blank(*p) && *p != '\n') ++p;
  if (p == s) return false;
  tok->assign(s, (size_t)(p - s));
  for (char& c : *tok) c = (char)std::tolower((unsigned char)c);
  return true;
}

inline bool at_token_end(const char* p, const char* e) { return p == e || is_blank(*p) || *p == '\n'; }

// integer token (fscanf "%d" accepts a leading '+')
inline bool parse_int(const char*& p, const char* e, long long* v) {
  p = skip_blank(p, e);
  if (p < e && *p == '+') {
    ++p;
    if (p < e && *p == '-') return false;
  }
  auto r = std::from_chars(p, e, *v);
  if (r.ec != std::errc() || !at_token_end(r.ptr, e)) return false;
  p = r.ptr;
  return true;
}

// floating token, correctly rounded to double like strtod / fscanf("%lf")
inline bool parse_real(const char*& p, const char* e, double* v) {
  p = skip_blank(p, e);
  if (p < e && *p == '+') {
    ++p;
    if (p < e && *p == '-') return false;
  }
  auto r = std::from_chars(p, e, *v, std::chars_format::general);
  if (r.ec == std::errc::result_out_of_range) {
    // from_chars leaves v unset on overflow/underflow; strtod's answer is
    // what fscanf gives (inf or a rounded subnormal/zero)
    std::string s(p, r.ptr);
    *v = std::strtod(s.c_str(), nullptr);
  } else if (r.ec != std::errc()) {
    return false;
  }
  if (!at_token_end(r.ptr, e)) return false;
  p = r.ptr;
  return true;
}

enum Field { kReal = 0, kInteger = 1, kPattern = 2, kComplex = 3 };
enum Symmetry { kGeneral = 0, kSymmetric = 1, kSkew = 2, kHermitian = 3 };

struct Chunk {
  const char* b = nullptr;
  const char* e = nullptr;
  long long entries = 0;   // entry lines in this chunk
  long long lines = 0;     // newlines in this chunk
  long long diag = 0;      // diagonal entries
  long long bad_line = -1; // first malformed line (chunk-local, 0-based)
  const char* bad_why = nullptr;
};

}  // namespace

extern "C" int spmx_mtx_read(const char* path, int* m_out, int* n_out, long long* nnz_out,
                             int** row_out, int** col_out, float** val_out, int* info) {
  if (!path || !m_out || !n_out || !nnz_out || !row_out || !col_out || !val_out)
    return set_error(SPMX_ERR_INVALID_VALUE, "NULL argument to spmx_mtx_read");
  *row_out = nullptr;
  *col_out = nullptr;
  *val_out = nullptr;
  MappedFile f;
  if (int rc = map_file(path, &f)) return rc;
  const char* p = f.p;
  const char* e = f.p + f.n;
  auto bad = [&](long long line, const std::string& why) {
    return set_error(SPMX_ERR_INVALID_VALUE,
                     std::string(path) + ":" + std::to_string(line) + ": " + why);
  };
  // banner: %%MatrixMarket object format field symmetry
  if (f.n < 14 || std::strncmp(p, "%%MatrixMarket", 14) != 0)
    return bad(1, "no %%MatrixMarket banner");
  const char* le = end_of_line(p, e);
  const char* q = p + 14;
  std::string obj, fmt, fld, sym;
  if (!next_token(q, le, &obj) || !next_token(q, le, &fmt) || !next_token(q, le, &fld) ||
      !next_token(q, le, &sym))
    return bad(1, "banner needs object, format, field and symmetry");
  if (obj != "matrix") return bad(1, "object '" + obj + "' is not 'matrix'");
  if (fmt != "coordinate") return bad(1, "format '" + fmt + "' is not supported (only 'coordinate')");
  Field field;
  if (fld == "real" || fld == "double") field = kReal;
  else if (fld == "integer") field = kInteger;
  else if (fld == "pattern") field = kPattern;
  else if (fld == "complex") field = kComplex;
  else return bad(1, "unknown field '" + fld + "'");
  Symmetry symm;
  if (sym == "general") symm = kGeneral;
  else if (sym == "symmetric") symm = kSymmetric;
  else if (sym == "skew-symmetric") symm = kSkew;
  else if (sym == "hermitian") symm = kHermitian;
  else return bad(1, "unknown symmetry '" + sym + "'");
  // comments and blank lines, then the size line
  long long line = 1;
  p = le < e ? le + 1 : e;
  long long M = -1, N = -1, L = -1;
  while (p < e) {
    ++line;
    le = end_of_line(p, e);
    const char* s = skip_blank(p, le);
    if (s < le && *s != '%') {
      const char* t = s;
      if (!parse_int(t, le, &M) || !parse_int(t, le, &N) || !parse_int(t, le, &L))
        return bad(line, "size line must hold rows, columns and entries");
      if (skip_blank(t, le) != le) return bad(line, "extra tokens on the size line");
      p = le < e ? le + 1 : e;
      break;
    }
    p = le < e ? le + 1 : e;
  }
  if (M < 0) return bad(line, "no size line");
  if (M > INT_MAX || N > INT_MAX || N < 0 || L < 0)
    return bad(line, "sizes out of range (rows and columns must fit int32)");
  const long long size_line = line;

  // chunks of the entry section, each starting at a line start
  const char* d0 = p;
  const size_t len = (size_t)(e - d0);
  const int threads = std::max(1, omp_get_max_threads());
  const size_t target = 4u << 20;
  int nch = (int)std::min<size_t>(std::max<size_t>(1, len / target), (size_t)threads * 8);
  if (len == 0) nch = 1;
  std::vector<Chunk> ch(nch);
  for (int k = 0; k < nch; ++k) {
    const char* b = d0 + (size_t)((unsigned __int128)len * k / nch);
    if (k > 0 && b > d0 && b[-1] != '\n') {
      b = end_of_line(b, e);
      if (b < e) ++b;
    }
    ch[k].b = b;
  }
  for (int k = 0; k < nch; ++k) ch[k].e = (k + 1 < nch) ? std::max(ch[k + 1].b, ch[k].b) : e;

  // pass 1: entry lines and newlines per chunk
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < nch; ++k) {
    long long ent = 0, nl = 0;
    for (const char* r = ch[k].b; r < ch[k].e;) {
      const char* l2 = end_of_line(r, ch[k].e);
      const char* s = skip_blank(r, l2);
      if (s < l2 && *s != '%') ++ent;
      if (l2 < ch[k].e) ++nl;
      r = l2 < ch[k].e ? l2 + 1 : ch[k].e;
    }
    ch[k].entries = ent;
    ch[k].lines = nl;
  }
  std::vector<long long> eoff(nch + 1, 0), loff(nch + 1, 0);
  for (int k = 0; k < nch; ++k) {
    eoff[k + 1] = eoff[k] + ch[k].entries;
    loff[k + 1] = loff[k] + ch[k].lines;
  }
  if (eoff[nch] != L)
    return bad(size_line, "size line declares " + std::to_string(L) + " entries, the file holds " +
                              std::to_string(eoff[nch]));
  const bool expand = symm == kSymmetric;

  // pass 2: parse.  Symmetric files go to scratch first (pass 3 spreads them).
  int *r1 = nullptr, *c1 = nullptr;
  float* v1 = nullptr;
  const size_t nL = (size_t)std::max<long long>(L, 1);
  r1 = (int*)std::malloc(4 * nL);
  c1 = (int*)std::malloc(4 * nL);
  v1 = (float*)std::malloc(4 * nL);
  if (!r1 || !c1 || !v1) {
    std::free(r1); std::free(c1); std::free(v1);
    return set_error(SPMX_ERR_ALLOC, "host allocation for the entries");
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < nch; ++k) {
    long long i = eoff[k], ln = 0, dg = 0;
    for (const char* r = ch[k].b; r < ch[k].e; ++ln) {
      const char* l2 = end_of_line(r, ch[k].e);
      const char* s = skip_blank(r, l2);
      r = l2 < ch[k].e ? l2 + 1 : ch[k].e;
      if (s == l2 || *s == '%') continue;
      long long ri, ci;
      const char* why = nullptr;
      float v = 1.0f;  // pattern and complex entries store 1
      if (!parse_int(s, l2, &ri) || !parse_int(s, l2, &ci)) why = "entry needs a row and a column index";
      else if (ri < 1 || ri > M || ci < 1 || ci > N) why = "index out of range";
      else if (field == kReal) {
        double dv;
        if (!parse_real(s, l2, &dv)) why = "entry needs a real value";
        else v = (float)dv;
      } else if (field == kInteger) {
        long long iv;
        if (!parse_int(s, l2, &iv)) why = "entry needs an integer value";
        else v = (float)iv;
      } else if (field == kComplex) {
        double re, im;
        if (!parse_real(s, l2, &re) || !parse_real(s, l2, &im)) why = "entry needs two complex parts";
      }
      if (why) {
        if (ch[k].bad_line < 0) {
          ch[k].bad_line = ln;
          ch[k].bad_why = why;
        }
        ++i;
        continue;
      }
      r1[i] = (int)(ri - 1);
      c1[i] = (int)(ci - 1);
      v1[i] = v;
      dg += (ri == ci);
      ++i;
    }
    ch[k].diag = dg;
  }
  for (int k = 0; k < nch; ++k)
    if (ch[k].bad_line >= 0) {
      std::free(r1); std::free(c1); std::free(v1);
      return bad(size_line + 1 + loff[k] + ch[k].bad_line, ch[k].bad_why);
    }
  long long diag = 0;
  std::vector<long long> doff(nch + 1, 0);
  for (int k = 0; k < nch; ++k) doff[k + 1] = doff[k] + ch[k].diag;
  diag = doff[nch];
  long long total = L;
  if (expand) {
    total = 2 * L - diag;
    const size_t nt = (size_t)std::max<long long>(total, 1);
    int* r2 = (int*)std::malloc(4 * nt);
    int* c2 = (int*)std::malloc(4 * nt);
    float* v2 = (float*)std::malloc(4 * nt);
    if (!r2 || !c2 || !v2) {
      std::free(r1); std::free(c1); std::free(v1);
      std::free(r2); std::free(c2); std::free(v2);
      return set_error(SPMX_ERR_ALLOC, "host allocation for the mirrored entries");
    }
    // pass 3: entry i lands at 2 i - (diagonals before i); its mirror follows
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < nch; ++k) {
      long long o = 2 * eoff[k] - doff[k];
      for (long long i = eoff[k]; i < eoff[k + 1]; ++i) {
        r2[o] = r1[i];
        c2[o] = c1[i];
        v2[o] = v1[i];
        ++o;
        if (r1[i] != c1[i]) {
          r2[o] = c1[i];
          c2[o] = r1[i];
          v2[o] = v1[i];
          ++o;
        }
      }
    }
    std::free(r1); std::free(c1); std::free(v1);
    r1 = r2; c1 = c2; v1 = v2;
  }
  *m_out = (int)M;
  *n_out = (int)N;
  *nnz_out = total;
  if (total == 0) {
    std::free(r1); std::free(c1); std::free(v1);
  } else {
    *row_out = r1;
    *col_out = c1;
    *val_out = v1;
  }
  if (info) {
    info[0] = (int)field;
    info[1] = (int)symm;
  }
  return SPMX_SUCCESS;
}

// ---------------------------------------------------------------------------
// MatrixMarket writer: entries are formatted in parallel blocks (shortest
// round-trip float text from std::to_chars, so values read back exactly) and
// written in order.
// ---------------------------------------------------------------------------
extern "C" int spmx_mtx_write(const char* path, int m, int n, long long nnz, const int* row,
                              const int* col, const float* val, int symmetric) {
  if (!path || m < 0 || n < 0 || nnz < 0 || (nnz > 0 && (!row || !col)))
    return set_error(SPMX_ERR_INVALID_VALUE, "bad spmx_mtx_write arguments");
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(SPMX_ERR_INVALID_VALUE, std::string("cannot create ") + path);
  std::string head = std::string("%%MatrixMarket matrix coordinate ") + (val ? "real" : "pattern") +
                     (symmetric ? " symmetric\n" : " general\n") + std::to_string(m) + " " +
                     std::to_string(n) + " " + std::to_string(nnz) + "\n";
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  const long long block = 1 << 18;
  const long long nb = (nnz + block - 1) / block;
  std::vector<std::string> out((size_t)std::min<long long>(nb, 4LL * omp_get_max_threads() + 1));
  int bad = 0;
  for (long long b0 = 0; b0 < nb && ok; b0 += (long long)out.size()) {
    const long long b1 = std::min<long long>(nb, b0 + (long long)out.size());
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (long long b = b0; b < b1; ++b) {
      std::string& s = out[(size_t)(b - b0)];
      s.clear();
      const long long i0 = b * block, i1 = std::min(nnz, i0 + block);
      s.reserve((size_t)(i1 - i0) * 32);
      char buf[128];  // an entry needs at most 11 + 1 + 11 + 1 + 15 + 1 bytes
      for (long long i = i0; i < i1; ++i) {
        if ((unsigned)row[i] >= (unsigned)m || (unsigned)col[i] >= (unsigned)n) {
          bad = 1;
          break;
        }
        char* const end = buf + sizeof buf - 2;  // room for the separators
        char* p = std::to_chars(buf, end, (long long)row[i] + 1).ptr;
        *p++ = ' ';
        p = std::to_chars(p, end, (long long)col[i] + 1).ptr;
        if (val) {
          *p++ = ' ';
          p = std::to_chars(p, end, val[i]).ptr;
        }
        *p++ = '\n';
        s.append(buf, (size_t)(p - buf));
      }
    }
    if (bad) break;
    for (long long b = b0; b < b1 && ok; ++b) {
      const std::string& s = out[(size_t)(b - b0)];
      ok = std::fwrite(s.data(), 1, s.size(), f) == s.size();
    }
  }
  if (std::fclose(f) != 0) ok = false;
  if (bad) return set_error(SPMX_ERR_INVALID_VALUE, "index out of range in spmx_mtx_write");
  if (!ok) return set_error(SPMX_ERR_INVALID_VALUE, std::string("write failed: ") + path);
  return SPMX_SUCCESS;
}

// ---------------------------------------------------------------------------
// binary CSR cache
// ---------------------------------------------------------------------------
namespace {

constexpr char kCsrMagic[9] = {'H', 'o', 'l', 'a', 1, 'C', 'S', 'R', 1};
constexpr size_t kCsrHeader = 24;  // 9 magic + 3 padding + 3 x int32

struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) std::fclose(f);
  }
};

int read_csr_header(FILE* f, const char* path, int* m, int* n, int* nnz, long long* fsize) {
  unsigned char h[kCsrHeader];
  if (std::fread(h, 1, kCsrHeader, f) != kCsrHeader)
    return set_error(SPMX_ERR_INVALID_VALUE, std::string(path) + ": could not read the CSR header");
  if (std::memcmp(h, kCsrMagic, sizeof(kCsrMagic)) != 0)
    return set_error(SPMX_ERR_INVALID_VALUE, std::string(path) + ": not a CSR cache file (magic)");
  std::memcpy(m, h + 12, 4);
  std::memcpy(n, h + 16, 4);
  std::memcpy(nnz, h + 20, 4);
  if (*m < 0 || *n < 0 || *nnz < 0)
    return set_error(SPMX_ERR_INVALID_VALUE, std::string(path) + ": negative sizes in the header");
  struct stat st;
  if (fstat(fileno(f), &st) != 0) return set_error(SPMX_ERR_INVALID_VALUE, std::string(path) + ": stat");
  *fsize = (long long)st.st_size;
  const long long want = (long long)kCsrHeader + 8LL * *nnz + 4LL * (*m + 1LL);
  if (*fsize < want)
    return set_error(SPMX_ERR_INVALID_VALUE, std::string(path) + ": file is shorter than its header says");
  return SPMX_SUCCESS;
}

bool read_all(FILE* f, void* dst, size_t bytes) {
  char* d = (char*)dst;
  while (bytes) {
    const size_t step = std::min<size_t>(bytes, (size_t)1 << 30);
    if (std::fread(d, 1, step, f) != step) return false;
    d += step;
    bytes -= step;
  }
  return true;
}

bool write_all(FILE* f, const void* src, size_t bytes) {
  const char* s = (const char*)src;
  while (bytes) {
    const size_t step = std::min<size_t>(bytes, (size_t)1 << 30);
    if (std::fwrite(s, 1, step, f) != step) return false;
    s += step;
    bytes -= step;
  }
  return true;
}

}  // namespace

extern "C" int spmx_csr_store(const char* path, int m, int n, int nnz, const int* rowptr,
                              const int* col, const float* val) {
  if (!path || m < 0 || n < 0 || nnz < 0 || !rowptr || (nnz > 0 && (!col || !val)))
    return set_error(SPMX_ERR_INVALID_VALUE, "bad spmx_csr_store arguments");
  if (rowptr[m] != nnz) return set_error(SPMX_ERR_INVALID_VALUE, "rowptr[m] differs from nnz");
  FileCloser fc{std::fopen(path, "wb")};
  if (!fc.f) return set_error(SPMX_ERR_INVALID_VALUE, std::string("cannot create ") + path);
  unsigned char h[kCsrHeader] = {};
  std::memcpy(h, kCsrMagic, sizeof(kCsrMagic));
  std::memcpy(h + 12, &m, 4);
  std::memcpy(h + 16, &n, 4);
  std::memcpy(h + 20, &nnz, 4);
  bool ok = write_all(fc.f, h, kCsrHeader) && write_all(fc.f, val, 4 * (size_t)nnz) &&
            write_all(fc.f, col, 4 * (size_t)nnz) && write_all(fc.f, rowptr, 4 * ((size_t)m + 1));
  if (std::fclose(fc.f) != 0) ok = false;
  fc.f = nullptr;
  if (!ok) return set_error(SPMX_ERR_INVALID_VALUE, std::string("write failed: ") + path);
  return SPMX_SUCCESS;
}

extern "C" int spmx_csr_load_header(const char* path, int* m, int* n, int* nnz) {
  if (!path || !m || !n || !nnz) return set_error(SPMX_ERR_INVALID_VALUE, "NULL argument");
  FileCloser fc{std::fopen(path, "rb")};
  if (!fc.f) return set_error(SPMX_ERR_INVALID_VALUE, std::string("cannot open ") + path);
  long long fsize;
  return read_csr_header(fc.f, path, m, n, nnz, &fsize);
}

extern "C" int spmx_csr_load(const char* path, int m, int n, int nnz, int* rowptr, int* col,
                             float* val) {
  if (!path || m < 0 || n < 0 || nnz < 0 || !rowptr || (nnz > 0 && !col))
    return set_error(SPMX_ERR_INVALID_VALUE, "bad spmx_csr_load arguments");
  FileCloser fc{std::fopen(path, "rb")};
  if (!fc.f) return set_error(SPMX_ERR_INVALID_VALUE, std::string("cannot open ") + path);
  int fm, fn, fnnz;
  long long fsize;
  if (int rc = read_csr_header(fc.f, path, &fm, &fn, &fnnz, &fsize)) return rc;
  if (fm != m || fn != n || fnnz != nnz)
    return set_error(SPMX_ERR_INVALID_VALUE, std::string(path) + ": sizes differ from the header");
  bool ok;
  if (val) ok = read_all(fc.f, val, 4 * (size_t)nnz);
  else ok = std::fseek(fc.f, 4L * nnz, SEEK_CUR) == 0;
  ok = ok && read_all(fc.f, col, 4 * (size_t)nnz) && read_all(fc.f, rowptr, 4 * ((size_t)m + 1));
  if (!ok) return set_error(SPMX_ERR_INVALID_VALUE, std::string(path) + ": could not read the CSR arrays");
  return SPMX_SUCCESS;
}
