// json_min.h -- a small JSON reader for sim_set.json.
//
// The reference vendors a general JSON library; the configuration file has
// a fixed, small schema, so this reader supports exactly what it needs:
// objects, arrays, strings (without \u escapes beyond ASCII), numbers
// (kept both as the literal text and as double), true/false/null.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace mcml {
namespace json {

struct Value {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0.0;
  bool is_integer = false;  // literal had no '.', 'e' or 'E'
  std::string text;         // number literal or string contents
  std::vector<Value> arr;
  std::vector<std::pair<std::string, Value>> obj;

  const Value *find(const std::string &key) const {
    for (const auto &kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
  // Text the reference's library would print for this value in messages.
  std::string repr() const {
    switch (kind) {
      case Null: return "null";
      case Bool: return b ? "true" : "false";
      case Number: return text;
      case String: return "\"" + text + "\"";
      case Array: return "[...]";
      default: return "{...}";
    }
  }
};

class Parser {
 public:
  explicit Parser(const std::string &s) : s_(s) {}
  Value parse() {
    Value v = value();
    ws();
    if (i_ != s_.size()) fail("trailing characters");
    return v;
  }

 private:
  const std::string &s_;
  size_t i_ = 0;

  [[noreturn]] void fail(const char *what) {
    throw std::runtime_error(std::string("JSON parse error at offset ") + std::to_string(i_) +
                             ": " + what);
  }
  void ws() {
    while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r'))
      ++i_;
  }
  bool lit(const char *w) {
    size_t n = 0;
    while (w[n]) ++n;
    if (s_.compare(i_, n, w) == 0) {
      i_ += n;
      return true;
    }
    return false;
  }
  Value value() {
    ws();
    if (i_ >= s_.size()) fail("unexpected end");
    const char c = s_[i_];
    Value v;
    if (c == '{') {
      v.kind = Value::Object;
      ++i_;
      ws();
      if (i_ < s_.size() && s_[i_] == '}') {
        ++i_;
        return v;
      }
      for (;;) {
        ws();
        if (i_ >= s_.size() || s_[i_] != '"') fail("expected key");
        std::string k = str();
        ws();
        if (i_ >= s_.size() || s_[i_] != ':') fail("expected ':'");
        ++i_;
        v.obj.emplace_back(std::move(k), value());
        ws();
        if (i_ < s_.size() && s_[i_] == ',') {
          ++i_;
          continue;
        }
        if (i_ < s_.size() && s_[i_] == '}') {
          ++i_;
          return v;
        }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind = Value::Array;
      ++i_;
      ws();
      if (i_ < s_.size() && s_[i_] == ']') {
        ++i_;
        return v;
      }
      for (;;) {
        v.arr.push_back(value());
        ws();
        if (i_ < s_.size() && s_[i_] == ',') {
          ++i_;
          continue;
        }
        if (i_ < s_.size() && s_[i_] == ']') {
          ++i_;
          return v;
        }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.kind = Value::String;
      v.text = str();
      return v;
    }
    if (lit("true")) {
      v.kind = Value::Bool;
      v.b = true;
      return v;
    }
    if (lit("false")) {
      v.kind = Value::Bool;
      return v;
    }
    if (lit("null")) return v;
    if (c == '-' || (c >= '0' && c <= '9')) {
      const size_t b = i_;
      bool integer = true;
      if (s_[i_] == '-') ++i_;
      while (i_ < s_.size()) {
        const char d = s_[i_];
        if (d >= '0' && d <= '9') {
          ++i_;
        } else if (d == '.' || d == 'e' || d == 'E' || d == '+' || d == '-') {
          integer = false;
          ++i_;
        } else {
          break;
        }
      }
      v.kind = Value::Number;
      v.text = s_.substr(b, i_ - b);
      v.is_integer = integer;
      char *end = nullptr;
      v.num = std::strtod(v.text.c_str(), &end);
      if (end == v.text.c_str()) fail("bad number");
      return v;
    }
    fail("unexpected character");
  }
  std::string str() {
    ++i_;  // opening quote
    std::string out;
    while (i_ < s_.size() && s_[i_] != '"') {
      char c = s_[i_++];
      if (c == '\\' && i_ < s_.size()) {
        const char e = s_[i_++];
        switch (e) {
          case 'n': c = '\n'; break;
          case 't': c = '\t'; break;
          case 'r': c = '\r'; break;
          case 'b': c = '\b'; break;
          case 'f': c = '\f'; break;
          case 'u': i_ += 4; c = '?'; break;
          default: c = e;
        }
      }
      out.push_back(c);
    }
    if (i_ >= s_.size()) fail("unterminated string");
    ++i_;
    return out;
  }
};

}  // namespace json
}  // namespace mcml
