// TEST INFRASTRUCTURE ONLY -- stand-in for the absent nlohmann/json submodule
// (.gitmodules:9-12 of the reference project), just large enough for the
// reference's main/mpm_data.h to compile unmodified: an object of numbers and
// flat number arrays (DATA.json), read with operator>>, at(), value() and
// get_to().  Written for this project; it restates the published JSON grammar,
// not nlohmann's code.
#pragma once
#include <cctype>
#include <charconv>
#include <cstdlib>
#include <istream>
#include <iterator>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace nlohmann {

class json {
 public:
  enum class kind { null, number, array, object, string, boolean };
  kind k = kind::null;
  double num = 0.0;
  std::vector<double> arr;  // arrays of numbers
  std::map<std::string, json> obj;
  std::string str;

  const json& at(const std::string& key) const {
    auto it = obj.find(key);
    if (it == obj.end()) throw std::out_of_range("DATA: key '" + key + "' not found");
    return it->second;
  }
  template <class T>
  T value(const std::string& key, T dflt) const {
    auto it = obj.find(key);
    if (it == obj.end()) return dflt;
    T v;
    it->second.get_to(v);
    return v;
  }
  void get_to(std::vector<double>& v) const {
    if (k == kind::array) v = arr;
    else if (k == kind::number) v.assign(1, num);
    else throw std::runtime_error("json: not an array");
  }
  void get_to(double& v) const {
    if (k != kind::number) throw std::runtime_error("json: not a number");
    v = num;
  }
  void get_to(int& v) const {
    if (k != kind::number) throw std::runtime_error("json: not a number");
    v = static_cast<int>(num);
  }
  // user types: from_json(const json&, T&) found by argument-dependent lookup
  template <class T>
  T& get_to(T& v) const {
    from_json(*this, v);
    return v;
  }
};

namespace detail {

struct parser {
  const char* p;
  const char* e;
  void ws() {
    while (p < e && std::isspace(static_cast<unsigned char>(*p))) ++p;
  }
  [[noreturn]] void fail(const char* what) { throw std::runtime_error(std::string("json: ") + what); }
  double number() {
    double v = 0.0;
    auto r = std::from_chars(p, e, v);
    if (r.ec != std::errc()) fail("bad number");
    p = r.ptr;
    return v;
  }
  std::string string() {
    if (*p != '"') fail("expected string");
    ++p;
    std::string s;
    while (p < e && *p != '"') {
      if (*p == '\\' && p + 1 < e) ++p;
      s.push_back(*p++);
    }
    if (p >= e) fail("unterminated string");
    ++p;
    return s;
  }
  void parse(json& j) {
    ws();
    if (p >= e) fail("unexpected end");
    const char c = *p;
    if (c == '{') {
      ++p;
      j.k = json::kind::object;
      ws();
      if (*p == '}') { ++p; return; }
      while (true) {
        ws();
        std::string key = string();
        ws();
        if (*p != ':') fail("expected ':'");
        ++p;
        parse(j.obj[key]);
        ws();
        if (*p == ',') { ++p; continue; }
        if (*p == '}') { ++p; return; }
        fail("expected ',' or '}'");
      }
    } else if (c == '[') {
      ++p;
      j.k = json::kind::array;
      ws();
      if (*p == ']') { ++p; return; }
      while (true) {
        ws();
        j.arr.push_back(number());
        ws();
        if (*p == ',') { ++p; continue; }
        if (*p == ']') { ++p; return; }
        fail("expected ',' or ']'");
      }
    } else if (c == '"') {
      j.k = json::kind::string;
      j.str = string();
    } else if (c == 't' || c == 'f') {
      j.k = json::kind::boolean;
      j.num = (c == 't') ? 1.0 : 0.0;
      p += (c == 't') ? 4 : 5;
    } else if (c == 'n') {
      j.k = json::kind::null;
      p += 4;
    } else {
      j.k = json::kind::number;
      j.num = number();
    }
  }
};

}  // namespace detail

inline std::istream& operator>>(std::istream& is, json& j) {
  std::string text((std::istreambuf_iterator<char>(is)), std::istreambuf_iterator<char>());
  detail::parser ps{text.data(), text.data() + text.size()};
  j = json();
  ps.parse(j);
  return is;
}

}  // namespace nlohmann
