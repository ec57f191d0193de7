// json.h -- minimal JSON reader for plan documents (objects, arrays,
// strings, integers, booleans, null).  Malformed input throws srdl::Error.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace srdl {

struct Json {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  long long num = 0;
  std::string str;
  std::vector<Json> arr;
  std::map<std::string, Json> obj;

  const Json& at(const std::string& k) const {
    auto it = obj.find(k);
    SRDL_REQUIRE(kind == Obj && it != obj.end(), kErrPlan, "plan: missing key '" + k + "'");
    return it->second;
  }
  bool has(const std::string& k) const { return kind == Obj && obj.count(k); }
  const std::string& s() const {
    SRDL_REQUIRE(kind == Str, kErrPlan, "plan: expected string");
    return str;
  }
  long long i() const {
    SRDL_REQUIRE(kind == Num, kErrPlan, "plan: expected integer");
    return num;
  }
  bool flag() const {
    SRDL_REQUIRE(kind == Bool, kErrPlan, "plan: expected boolean");
    return b;
  }
  const std::vector<Json>& a() const {
    SRDL_REQUIRE(kind == Arr, kErrPlan, "plan: expected array");
    return arr;
  }
  std::vector<int> ints() const {
    std::vector<int> v;
    for (auto& x : a()) v.push_back((int)x.i());
    return v;
  }
  std::vector<std::string> strs() const {
    std::vector<std::string> v;
    for (auto& x : a()) v.push_back(x.s());
    return v;
  }
};

class JsonParser {
 public:
  explicit JsonParser(const std::string& t) : t_(t) {}
  Json parse() {
    Json v = value();
    ws();
    SRDL_REQUIRE(p_ == t_.size(), kErrPlan, "plan: trailing characters");
    return v;
  }

 private:
  const std::string& t_;
  size_t p_ = 0;
  void ws() {
    while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\n' || t_[p_] == '\t' || t_[p_] == '\r')) p_++;
  }
  char peek() {
    ws();
    SRDL_REQUIRE(p_ < t_.size(), kErrPlan, "plan: unexpected end of input");
    return t_[p_];
  }
  void expect(char c) {
    SRDL_REQUIRE(peek() == c, kErrPlan, std::string("plan: expected '") + c + "'");
    p_++;
  }
  Json value() {
    char c = peek();
    Json v;
    if (c == '{') {
      v.kind = Json::Obj;
      p_++;
      if (peek() == '}') { p_++; return v; }
      for (;;) {
        std::string k = string();
        expect(':');
        v.obj[k] = value();
        if (peek() == ',') { p_++; continue; }
        expect('}');
        return v;
      }
    }
    if (c == '[') {
      v.kind = Json::Arr;
      p_++;
      if (peek() == ']') { p_++; return v; }
      for (;;) {
        v.arr.push_back(value());
        if (peek() == ',') { p_++; continue; }
        expect(']');
        return v;
      }
    }
    if (c == '"') {
      v.kind = Json::Str;
      v.str = string();
      return v;
    }
    if (t_.compare(p_, 4, "true") == 0) { p_ += 4; v.kind = Json::Bool; v.b = true; return v; }
    if (t_.compare(p_, 5, "false") == 0) { p_ += 5; v.kind = Json::Bool; v.b = false; return v; }
    if (t_.compare(p_, 4, "null") == 0) { p_ += 4; return v; }
    SRDL_REQUIRE(c == '-' || (c >= '0' && c <= '9'), kErrPlan, "plan: bad value");
    size_t s = p_;
    if (t_[p_] == '-') p_++;
    while (p_ < t_.size() && t_[p_] >= '0' && t_[p_] <= '9') p_++;
    v.kind = Json::Num;
    v.num = std::stoll(t_.substr(s, p_ - s));
    return v;
  }
  std::string string() {
    expect('"');
    std::string out;
    while (p_ < t_.size() && t_[p_] != '"') {
      char c = t_[p_++];
      if (c == '\\') {
        SRDL_REQUIRE(p_ < t_.size(), kErrPlan, "plan: bad escape");
        char e = t_[p_++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            SRDL_REQUIRE(p_ + 4 <= t_.size(), kErrPlan, "plan: bad \\u escape");
            unsigned cp = std::stoul(t_.substr(p_, 4), nullptr, 16);
            p_ += 4;
            SRDL_REQUIRE(cp < 0x80, kErrPlan, "plan: non-ASCII \\u escape");
            out += (char)cp;
            break;
          }
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    SRDL_REQUIRE(p_ < t_.size(), kErrPlan, "plan: unterminated string");
    p_++;
    return out;
  }
};

}  // namespace srdl
