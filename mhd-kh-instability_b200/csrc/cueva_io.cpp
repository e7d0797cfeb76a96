// cueva_io.cpp -- the reference's backup text format for restarts.
//
// all_variables_NNNN.dat is written by the writer every hloc steps
// (22_writer.f95:1134-1150, DIM == 2) and read back by init_restart
// (03_restart_primitive.f95:51-57): one list-directed WRITE / READ per point,
// i = -6..imax+6 in the outer loop and j = -6..jmax+6 in the inner one, each
// with the 14 values psi phi Bx By Bz Vx Vy Vz Ex Ey Ez q rho p, ghost
// points included.
//
// The reader implements the list-directed input rules that such files can
// contain: blank or comma separators, repeat counts (r*c), null values (r*
// or empty fields between commas, which leave the variable unchanged), a
// slash ending the READ, every Fortran real form (E, D or Q exponent
// letters, exponents written without a letter as in 1.0-100, Infinity and
// NaN), and READs whose 14 values span several lines.  Files whose lines
// each hold one point (the writer's own output) are parsed in parallel; any
// other layout falls back to a sequential parse with the full rules.
#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "../../include/cueva.h"

int32_t cueva_fail(int32_t code, const std::string& msg);

namespace {

constexpr int NCOL = 14;
// file column -> primitive field id of enum cueva_field
const int kColField[NCOL] = {CUEVA_PSI, CUEVA_PHI, CUEVA_BX, CUEVA_BY, CUEVA_BZ, CUEVA_VX, CUEVA_VY,
                             CUEVA_VZ,  CUEVA_EX,  CUEVA_EY, CUEVA_EZ, CUEVA_Q,  CUEVA_RHO, CUEVA_P};

int nthreads_of(int32_t n) {
  if (n > 0) return n;
  const unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

bool is_sep(char c) { return c == ' ' || c == '\t' || c == ',' || c == '\r'; }

// one Fortran real constant; false if the token is not one
bool parse_real(const char* b, const char* e, double& out) {
  char buf[96];
  size_t n = 0;
  if (b < e && (*b == '+')) ++b;
  if (e - b <= 0 || e - b > 80) return false;
  bool seen_digit = false, seen_exp = false;
  for (const char* p = b; p < e; ++p) {
    char c = *p;
    if (c >= '0' && c <= '9') { seen_digit = true; buf[n++] = c; continue; }
    if (c == '.') { buf[n++] = c; continue; }
    if ((c == 'E' || c == 'e' || c == 'D' || c == 'd' || c == 'Q' || c == 'q') && seen_digit && !seen_exp) {
      buf[n++] = 'e';
      seen_exp = true;
      if (p + 1 < e && p[1] == '+') ++p;   // from_chars takes no '+' after the exponent letter
      continue;
    }
    if ((c == '+' || c == '-') && p > b) {
      // a sign after the mantissa without exponent letter: 1.0-100 = 1.0e-100
      if (!seen_exp && seen_digit) { buf[n++] = 'e'; seen_exp = true; }
      if (c == '-') buf[n++] = '-';
      continue;
    }
    if (c == '-' && p == b) { buf[n++] = c; continue; }
    // Infinity / Inf / NaN (optionally NaN(...)), any case
    std::string w(b, e);
    std::string lw;
    for (char ch : w) lw += (char)((ch >= 'A' && ch <= 'Z') ? ch - 'A' + 'a' : ch);
    bool neg = false;
    size_t s = 0;
    if (!lw.empty() && lw[0] == '-') { neg = true; s = 1; }
    const std::string body = lw.substr(s);
    if (body == "inf" || body == "infinity") { out = neg ? -HUGE_VAL : HUGE_VAL; return true; }
    if (body.compare(0, 3, "nan") == 0) { out = neg ? -std::nan("") : std::nan(""); return true; }
    return false;
  }
  if (!seen_digit) return false;
  const auto r = std::from_chars(buf, buf + n, out, std::chars_format::general);
  return r.ec == std::errc() && r.ptr == buf + n;
}

struct Text {
  std::vector<char> data;
  std::vector<size_t> line_start;   // offsets of the lines, plus data.size() at the end
};

int32_t load_text(const char* path, Text& t) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return cueva_fail(CUEVA_ERR_ARG, std::string("cannot open ") + path + ": " + std::strerror(errno));
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  t.data.resize(sz > 0 ? (size_t)sz : 0);
  const size_t got = sz > 0 ? std::fread(t.data.data(), 1, (size_t)sz, f) : 0;
  std::fclose(f);
  if ((long)got != sz) return cueva_fail(CUEVA_ERR_ARG, std::string("short read of ") + path);
  t.line_start.clear();
  t.line_start.push_back(0);
  const char* d = t.data.data();
  for (size_t k = 0; k < t.data.size();) {
    const void* nl = std::memchr(d + k, '\n', t.data.size() - k);
    if (!nl) break;
    k = (size_t)((const char*)nl - d) + 1;
    t.line_start.push_back(k);
  }
  if (t.line_start.back() != t.data.size()) t.line_start.push_back(t.data.size());
  return CUEVA_OK;
}

// fast form: line k holds exactly the 14 plain values of record k
bool parse_line_plain(const char* b, const char* e, double (&v)[NCOL]) {
  int n = 0;
  const char* p = b;
  while (p < e) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
    if (p >= e) break;
    const char* q = p;
    while (q < e && !is_sep(*q) && *q != '\n') ++q;
    if (n == NCOL) return false;
    for (const char* s = p; s < q; ++s)
      if (*s == '*' || *s == '/') return false;
    if (!parse_real(p, q, v[n])) return false;
    ++n;
    p = q;
    if (p < e && *p == ',') return false;   // commas may carry null values: full rules
  }
  return n == NCOL;
}

struct Grid {
  int imax, jmax;
  double* const* fields;
  size_t idx(size_t rec) const {
    const int i = (int)(rec / (size_t)(jmax + 13)) - 6, j = (int)(rec % (size_t)(jmax + 13)) - 6;
    return (size_t)(i + 6) + (size_t)(j + 6) * (size_t)(imax + 13);
  }
  void put(size_t rec, int col, double x) const { fields[kColField[col]][idx(rec)] = x; }
};

// sequential list-directed parse of nrec READ statements of 14 items
int32_t parse_general(const Text& t, const Grid& g, size_t nrec) {
  const char* d = t.data.data();
  const size_t nlines = t.line_start.size() - 1;
  size_t line = 0;
  for (size_t r = 0; r < nrec; ++r) {
    int item = 0;
    bool done = false;
    while (!done) {
      if (line >= nlines)
        return cueva_fail(CUEVA_ERR_ARG, "end of file in record " + std::to_string(r + 1) + " of " +
                                             std::to_string(nrec));
      const char* p = d + t.line_start[line];
      const char* e = d + t.line_start[line + 1];
      ++line;
      bool prev_comma = false, at_start = true;
      while (p < e && !done) {
        while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
        if (p >= e) break;
        if (*p == '/') { done = true; break; }            // slash: the READ ends, the rest keeps its value
        if (*p == ',') {
          if (prev_comma || at_start) ++item;             // empty field: null value
          if (item >= NCOL) done = true;
          prev_comma = true; at_start = false; ++p;
          continue;
        }
        const char* q = p;
        while (q < e && !is_sep(*q) && *q != '\n' && *q != '/') ++q;
        long rep = 1;
        const char* val = p;
        const char* star = (const char*)std::memchr(p, '*', (size_t)(q - p));
        if (star) {
          const auto rr = std::from_chars(p, star, rep);
          if (rr.ec != std::errc() || rr.ptr != star || rep < 1)
            return cueva_fail(CUEVA_ERR_ARG, "bad repeat count on line " + std::to_string(line));
          val = star + 1;
        }
        double x = 0.0;
        const bool null_value = (val == q);
        if (!null_value && !parse_real(val, q, x))
          return cueva_fail(CUEVA_ERR_ARG, "not a real number on line " + std::to_string(line) + ": '" +
                                               std::string(p, q) + "'");
        for (long k = 0; k < rep; ++k) {
          if (item >= NCOL) return cueva_fail(CUEVA_ERR_ARG, "repeat count overruns record " + std::to_string(r + 1));
          if (!null_value) g.put(r, item, x);
          ++item;
        }
        if (item >= NCOL) done = true;
        p = q;
        prev_comma = false; at_start = false;
        while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
        if (p < e && *p == ',') { ++p; prev_comma = true; }
      }
    }
  }
  return CUEVA_OK;
}

int32_t check_grid(int32_t imax, int32_t jmax, const void* fields) {
  if (imax < 1 || jmax < 1) return cueva_fail(CUEVA_ERR_ARG, "imax and jmax must be >= 1");
  if (!fields) return cueva_fail(CUEVA_ERR_ARG, "null field table");
  return CUEVA_OK;
}

}  // namespace

extern "C" {

int32_t cueva_read_all_variables(const char* path, int32_t imax, int32_t jmax, double* const* fields,
                                 int32_t nthreads) {
  if (int32_t e = check_grid(imax, jmax, fields)) return e;
  for (int c = 0; c < NCOL; ++c)
    if (!fields[kColField[c]]) return cueva_fail(CUEVA_ERR_ARG, "null field pointer");
  if (!path) return cueva_fail(CUEVA_ERR_ARG, "null path");
  Text t;
  if (int32_t e = load_text(path, t)) return e;
  const Grid g{imax, jmax, fields};
  const size_t nrec = (size_t)(imax + 13) * (size_t)(jmax + 13);
  const size_t nlines = t.line_start.size() - 1;
  // fast path: one point per line, nothing but blanks after the last one
  bool plain = nlines >= nrec;
  for (size_t k = nrec; plain && k < nlines; ++k)
    for (size_t c = t.line_start[k]; c < t.line_start[k + 1]; ++c)
      if (!(t.data[c] == ' ' || t.data[c] == '\t' || t.data[c] == '\r' || t.data[c] == '\n')) { plain = false; break; }
  if (plain) {
    const int nt = std::max(1, std::min<int>(nthreads_of(nthreads), (int)(nrec / 4096) + 1));
    std::vector<char> ok(nt, 1);
    std::vector<std::thread> th;
    for (int w = 0; w < nt; ++w)
      th.emplace_back([&, w] {
        const size_t a = nrec * w / nt, b = nrec * (w + 1) / nt;
        double v[NCOL];
        for (size_t r = a; r < b; ++r) {
          if (!parse_line_plain(t.data.data() + t.line_start[r], t.data.data() + t.line_start[r + 1], v)) {
            ok[w] = 0;
            return;
          }
          for (int c = 0; c < NCOL; ++c) g.put(r, c, v[c]);
        }
      });
    for (auto& x : th) x.join();
    if (std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; })) return CUEVA_OK;
  }
  return parse_general(t, g, nrec);
}

int32_t cueva_write_all_variables(const char* path, int32_t imax, int32_t jmax, const double* const* fields,
                                  int32_t overwrite, int32_t nthreads) {
  if (int32_t e = check_grid(imax, jmax, fields)) return e;
  for (int c = 0; c < NCOL; ++c)
    if (!fields[kColField[c]]) return cueva_fail(CUEVA_ERR_ARG, "null field pointer");
  if (!path) return cueva_fail(CUEVA_ERR_ARG, "null path");
  struct stat sb;
  if (!overwrite && stat(path, &sb) == 0)
    return cueva_fail(CUEVA_ERR_ARG, std::string(path) + " exists (the writer opens backups with status='new')");
  const size_t nrec = (size_t)(imax + 13) * (size_t)(jmax + 13);
  const int nt = std::max(1, std::min<int>(nthreads_of(nthreads), (int)(nrec / 4096) + 1));
  constexpr int W = 25;   // columns per value, 17 significant digits
  const size_t line_bytes = (size_t)NCOL * W + 1;
  std::vector<std::vector<char>> chunk(nt);
  const Grid g{imax, jmax, const_cast<double* const*>(fields)};
  std::vector<std::thread> th;
  for (int w = 0; w < nt; ++w)
    th.emplace_back([&, w] {
      const size_t a = nrec * w / nt, b = nrec * (w + 1) / nt;
      std::vector<char>& out = chunk[w];
      out.assign((b - a) * line_bytes, ' ');
      char* o = out.data();
      for (size_t r = a; r < b; ++r) {
        const size_t id = g.idx(r);
        for (int c = 0; c < NCOL; ++c) {
          char tmp[40];
          const double x = fields[kColField[c]][id];
          auto res = std::to_chars(tmp, tmp + sizeof tmp, x, std::chars_format::scientific, 16);
          size_t n = (size_t)(res.ptr - tmp);
          for (size_t k = 0; k < n; ++k) if (tmp[k] == 'e') tmp[k] = 'E';
          if (n > (size_t)W - 1) n = W - 1;   // never: 24 characters at most
          std::memcpy(o + (W - n), tmp, n);
          o += W;
        }
        *o++ = '\n';
      }
    });
  for (auto& x : th) x.join();
  const std::string tmp_path = std::string(path) + ".partial";
  FILE* f = std::fopen(tmp_path.c_str(), "wb");
  if (!f) return cueva_fail(CUEVA_ERR_ARG, "cannot create " + tmp_path + ": " + std::strerror(errno));
  for (const auto& cbuf : chunk)
    if (!cbuf.empty() && std::fwrite(cbuf.data(), 1, cbuf.size(), f) != cbuf.size()) {
      std::fclose(f);
      std::remove(tmp_path.c_str());
      return cueva_fail(CUEVA_ERR_ARG, "write failed: " + tmp_path);
    }
  if (std::fclose(f) != 0 || std::rename(tmp_path.c_str(), path) != 0) {
    std::remove(tmp_path.c_str());
    return cueva_fail(CUEVA_ERR_ARG, std::string("cannot finish ") + path);
  }
  return CUEVA_OK;
}

}  // extern "C"
