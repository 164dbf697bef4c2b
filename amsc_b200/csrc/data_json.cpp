// data_json.cpp -- DATA.json reader for large scenarios (host code).
//
// DATA.json (main/mpm_data.h:61-122; written by the Octave generators'
// v2j, data/dambreak/dambreak.m:146-165) is one JSON object whose values are
// numbers or flat arrays of numbers.  A 4M-particle scenario is ~1 GB of
// text; this reader streams the file in blocks and parses each number with
// std::from_chars, which rounds exactly as strtod does, straight into double
// arrays -- no per-number objects.  Nested arrays are flattened in reading
// order; strings, booleans and nulls are rejected with a message.
#include <charconv>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/dampm_cuda.h"

struct dampm_json {
  std::map<std::string, std::vector<double>> arrays;
  std::map<std::string, double> scalars;
  std::string err;
};

namespace {

class Reader {
 public:
  explicit Reader(FILE* f) : f_(f), buf_(1 << 22) {}

  // next character that is not white space, or -1 at the end
  int peek() {
    for (;;) {
      if (pos_ == len_ && !fill()) return -1;
      const char c = buf_[pos_];
      if (c == ' ' || c == '\n' || c == '\r' || c == '\t') {
        ++pos_;
        continue;
      }
      return (unsigned char)c;
    }
  }
  int get() {
    const int c = peek();
    if (c >= 0) ++pos_;
    return c;
  }
  bool expect(char c) { return get() == (unsigned char)c; }

  bool string(std::string& out) {
    if (!expect('"')) return false;
    out.clear();
    for (;;) {
      if (pos_ == len_ && !fill()) return false;
      const char c = buf_[pos_++];
      if (c == '"') return true;
      if (c == '\\') {  // keys are plain names; keep the escaped character
        if (pos_ == len_ && !fill()) return false;
        out.push_back(buf_[pos_++]);
      } else {
        out.push_back(c);
      }
    }
  }

  bool number(double& v) {
    peek();
    char tok[64];
    int n = 0;
    for (;;) {
      if (pos_ == len_ && !fill()) break;
      const char c = buf_[pos_];
      if ((c >= '0' && c <= '9') || c == '-' || c == '+' || c == '.' || c == 'e' ||
          c == 'E') {
        if (n == 63) return false;
        tok[n++] = c;
        ++pos_;
      } else {
        break;
      }
    }
    if (n == 0) return false;
    const char* b = tok;
    if (*b == '+') ++b;  // from_chars takes no leading '+'
    const auto r = std::from_chars(b, tok + n, v);
    return r.ec == std::errc() && r.ptr == tok + n;
  }

 private:
  bool fill() {
    len_ = std::fread(buf_.data(), 1, buf_.size(), f_);
    pos_ = 0;
    return len_ > 0;
  }
  FILE* f_;
  std::vector<char> buf_;
  size_t pos_ = 0, len_ = 0;
};

// value: number (scalar) or array of numbers, nested arrays flattened
bool read_array(Reader& r, std::vector<double>& out, int depth) {
  if (depth > 32 || !r.expect('[')) return false;
  if (r.peek() == ']') {
    r.get();
    return true;
  }
  for (;;) {
    if (r.peek() == '[') {
      if (!read_array(r, out, depth + 1)) return false;
    } else {
      double v;
      if (!r.number(v)) return false;
      out.push_back(v);
    }
    const int c = r.get();
    if (c == ']') return true;
    if (c != ',') return false;
  }
}

}  // namespace

extern "C" {

int dampm_json_read(const char* path, dampm_json** out) {
  if (!path || !out) return DAMPM_ERR_ARG;
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return DAMPM_ERR_ARG;
  dampm_json* j = new dampm_json();
  Reader r(f);
  bool ok = r.expect('{');
  std::string key;
  if (ok && r.peek() == '}') {
    r.get();
  } else {
    while (ok) {
      ok = r.string(key) && r.expect(':');
      if (!ok) break;
      if (r.peek() == '[') {
        std::vector<double>& a = j->arrays[key];
        a.clear();
        ok = read_array(r, a, 0);
      } else {
        double v;
        ok = r.number(v);
        if (ok) j->scalars[key] = v;
      }
      if (!ok) {
        j->err = "value of key '" + key + "' is not a number or an array of numbers";
        break;
      }
      const int c = r.get();
      if (c == '}') break;
      if (c != ',') {
        ok = false;
        j->err = "malformed object after key '" + key + "'";
      }
    }
  }
  std::fclose(f);
  if (!ok) {
    if (j->err.empty()) j->err = "malformed JSON";
    *out = j;  // the caller reads the message, then frees
    return DAMPM_ERR_ARG;
  }
  *out = j;
  return DAMPM_OK;
}

// n < 0: key absent.  Scalars count as length-1 arrays.
int dampm_json_size(const dampm_json* j, const char* key, long long* n) {
  if (!j || !key || !n) return DAMPM_ERR_ARG;
  auto a = j->arrays.find(key);
  if (a != j->arrays.end()) {
    *n = (long long)a->second.size();
    return DAMPM_OK;
  }
  *n = j->scalars.count(key) ? 1 : -1;
  return DAMPM_OK;
}

int dampm_json_get(const dampm_json* j, const char* key, double* out) {
  if (!j || !key || !out) return DAMPM_ERR_ARG;
  auto a = j->arrays.find(key);
  if (a != j->arrays.end()) {
    std::memcpy(out, a->second.data(), sizeof(double) * a->second.size());
    return DAMPM_OK;
  }
  auto s = j->scalars.find(key);
  if (s == j->scalars.end()) return DAMPM_ERR_UNKNOWN_FIELD;
  *out = s->second;
  return DAMPM_OK;
}

// is_array: 1 for an array value, 0 for a scalar
int dampm_json_kind(const dampm_json* j, const char* key, int* is_array) {
  if (!j || !key || !is_array) return DAMPM_ERR_ARG;
  if (j->arrays.count(key)) {
    *is_array = 1;
    return DAMPM_OK;
  }
  if (j->scalars.count(key)) {
    *is_array = 0;
    return DAMPM_OK;
  }
  return DAMPM_ERR_UNKNOWN_FIELD;
}

const char* dampm_json_error(const dampm_json* j) { return j ? j->err.c_str() : "null"; }

int dampm_json_free(dampm_json* j) {
  if (!j) return DAMPM_ERR_ARG;
  delete j;
  return DAMPM_OK;
}

}  // extern "C"
