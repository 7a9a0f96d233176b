// Minimal JSON value, parser and writer for the C-ABI request/response
// protocol (no third-party JSON library is available to the build).
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace qmbed {
namespace json {

struct ParseError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class Value {
 public:
  enum Kind { Null, Bool, Number, String, Array, Object };
  Value() = default;
  static Value null() { return Value(); }
  static Value boolean(bool b) { Value v; v.kind_ = Bool; v.b_ = b; return v; }
  static Value number(double d) { Value v; v.kind_ = Number; v.d_ = d; v.integral_ = false; return v; }
  static Value integer(long long i) { Value v; v.kind_ = Number; v.d_ = static_cast<double>(i); v.i_ = i; v.integral_ = true; return v; }
  static Value string(std::string s) { Value v; v.kind_ = String; v.s_ = std::move(s); return v; }
  static Value array() { Value v; v.kind_ = Array; return v; }
  static Value object() { Value v; v.kind_ = Object; return v; }

  Kind kind() const { return kind_; }
  bool is_null() const { return kind_ == Null; }
  bool is_number() const { return kind_ == Number; }
  bool is_string() const { return kind_ == String; }
  bool is_array() const { return kind_ == Array; }
  bool is_object() const { return kind_ == Object; }
  bool is_bool() const { return kind_ == Bool; }
  bool is_integral() const { return kind_ == Number && integral_; }

  bool as_bool() const { expect(Bool, "a boolean"); return b_; }
  double as_double() const { expect(Number, "a number"); return d_; }
  long long as_int() const {
    expect(Number, "an integer");
    if (integral_) return i_;
    if (std::floor(d_) != d_) throw ParseError("expected an integer");
    return static_cast<long long>(d_);
  }
  const std::string& as_string() const { expect(String, "a string"); return s_; }
  const std::vector<Value>& items() const { expect(Array, "an array"); return a_; }
  std::vector<Value>& items() { expect(Array, "an array"); return a_; }
  const std::vector<std::pair<std::string, Value>>& members() const { expect(Object, "an object"); return o_; }

  const Value* find(const std::string& key) const {
    if (kind_ != Object) return nullptr;
    for (auto& kv : o_)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
  bool has(const std::string& key) const {
    const Value* v = find(key);
    return v && !v->is_null();
  }
  const Value& at(const std::string& key) const {
    const Value* v = find(key);
    if (!v) throw ParseError("missing field `" + key + "`");
    return *v;
  }
  Value& set(const std::string& key, Value v) {
    kind_ = Object;
    for (auto& kv : o_)
      if (kv.first == key) {
        kv.second = std::move(v);
        return kv.second;
      }
    o_.emplace_back(key, std::move(v));
    return o_.back().second;
  }
  Value& push(Value v) {
    kind_ = Array;
    a_.push_back(std::move(v));
    return a_.back();
  }

  std::string dump() const {
    std::string out;
    write(out);
    return out;
  }

 private:
  void expect(Kind k, const char* what) const {
    if (kind_ != k) throw ParseError(std::string("expected ") + what);
  }
  void write(std::string& out) const {
    switch (kind_) {
      case Null: out += "null"; break;
      case Bool: out += b_ ? "true" : "false"; break;
      case Number: {
        if (integral_) {
          out += std::to_string(i_);
        } else if (!std::isfinite(d_)) {
          out += "null";
        } else {
          char buffer[32];
          std::snprintf(buffer, sizeof(buffer), "%.17g", d_);
          std::string text(buffer);
          if (text.find_first_of(".eE") == std::string::npos) text += ".0";
          out += text;
        }
        break;
      }
      case String: write_string(out, s_); break;
      case Array: {
        out += '[';
        for (size_t i = 0; i < a_.size(); ++i) {
          if (i) out += ',';
          a_[i].write(out);
        }
        out += ']';
        break;
      }
      case Object: {
        out += '{';
        for (size_t i = 0; i < o_.size(); ++i) {
          if (i) out += ',';
          write_string(out, o_[i].first);
          out += ':';
          o_[i].second.write(out);
        }
        out += '}';
        break;
      }
    }
  }
  static void write_string(std::string& out, const std::string& s) {
    out += '"';
    for (unsigned char c : s) {
      switch (c) {
        case '"': out += "\\\""; break;
        case '\\': out += "\\\\"; break;
        case '\n': out += "\\n"; break;
        case '\r': out += "\\r"; break;
        case '\t': out += "\\t"; break;
        default:
          if (c < 0x20) {
            char buffer[8];
            std::snprintf(buffer, sizeof(buffer), "\\u%04x", c);
            out += buffer;
          } else {
            out += static_cast<char>(c);
          }
      }
    }
    out += '"';
  }

  Kind kind_ = Null;
  bool b_ = false;
  double d_ = 0.0;
  long long i_ = 0;
  bool integral_ = false;
  std::string s_;
  std::vector<Value> a_;
  std::vector<std::pair<std::string, Value>> o_;
};

class Parser {
 public:
  explicit Parser(const std::string& text) : t_(text) {}
  Value parse() {
    Value v = value();
    skip();
    if (p_ != t_.size()) fail("trailing characters");
    return v;
  }

 private:
  [[noreturn]] void fail(const std::string& what) const {
    throw ParseError(what + " at position " + std::to_string(p_));
  }
  void skip() {
    while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\n' || t_[p_] == '\r' || t_[p_] == '\t')) ++p_;
  }
  Value value() {
    skip();
    if (p_ >= t_.size()) fail("unexpected end of input");
    char c = t_[p_];
    if (c == '{') return object();
    if (c == '[') return array();
    if (c == '"') return Value::string(string());
    if (c == 't') return literal("true", Value::boolean(true));
    if (c == 'f') return literal("false", Value::boolean(false));
    if (c == 'n') return literal("null", Value::null());
    return number();
  }
  Value literal(const char* word, Value v) {
    size_t len = std::string(word).size();
    if (t_.compare(p_, len, word) != 0) fail("invalid literal");
    p_ += len;
    return v;
  }
  Value number() {
    size_t start = p_;
    bool integral = true;
    if (p_ < t_.size() && (t_[p_] == '-' || t_[p_] == '+')) ++p_;
    while (p_ < t_.size()) {
      char c = t_[p_];
      if (c >= '0' && c <= '9') { ++p_; continue; }
      if (c == '.' || c == 'e' || c == 'E' || c == '-' || c == '+') { integral = false; ++p_; continue; }
      break;
    }
    std::string text = t_.substr(start, p_ - start);
    if (text.empty() || text == "-") fail("invalid number");
    char* end = nullptr;
    if (integral) {
      errno = 0;
      long long i = std::strtoll(text.c_str(), &end, 10);
      if (errno == 0 && end && *end == '\0') return Value::integer(i);
    }
    double d = std::strtod(text.c_str(), &end);
    if (!end || *end != '\0') fail("invalid number");
    return Value::number(d);
  }
  std::string string() {
    ++p_;  // opening quote
    std::string out;
    while (p_ < t_.size()) {
      char c = t_[p_++];
      if (c == '"') return out;
      if (c == '\\') {
        if (p_ >= t_.size()) fail("bad escape");
        char e = t_[p_++];
        switch (e) {
          case '"': out += '"'; break;
          case '\\': out += '\\'; break;
          case '/': out += '/'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'n': out += '\n'; break;
          case 'r': out += '\r'; break;
          case 't': out += '\t'; break;
          case 'u': {
            if (p_ + 4 > t_.size()) fail("bad unicode escape");
            unsigned code = static_cast<unsigned>(std::strtoul(t_.substr(p_, 4).c_str(), nullptr, 16));
            p_ += 4;
            if (code < 0x80) {
              out += static_cast<char>(code);
            } else if (code < 0x800) {
              out += static_cast<char>(0xC0 | (code >> 6));
              out += static_cast<char>(0x80 | (code & 0x3F));
            } else {
              out += static_cast<char>(0xE0 | (code >> 12));
              out += static_cast<char>(0x80 | ((code >> 6) & 0x3F));
              out += static_cast<char>(0x80 | (code & 0x3F));
            }
            break;
          }
          default: fail("bad escape");
        }
      } else {
        out += c;
      }
    }
    fail("unterminated string");
  }
  Value array() {
    ++p_;
    Value v = Value::array();
    skip();
    if (p_ < t_.size() && t_[p_] == ']') { ++p_; return v; }
    for (;;) {
      v.push(value());
      skip();
      if (p_ >= t_.size()) fail("unterminated array");
      if (t_[p_] == ',') { ++p_; continue; }
      if (t_[p_] == ']') { ++p_; return v; }
      fail("expected , or ]");
    }
  }
  Value object() {
    ++p_;
    Value v = Value::object();
    skip();
    if (p_ < t_.size() && t_[p_] == '}') { ++p_; return v; }
    for (;;) {
      skip();
      if (p_ >= t_.size() || t_[p_] != '"') fail("expected a key");
      std::string key = string();
      skip();
      if (p_ >= t_.size() || t_[p_] != ':') fail("expected :");
      ++p_;
      v.set(key, value());
      skip();
      if (p_ >= t_.size()) fail("unterminated object");
      if (t_[p_] == ',') { ++p_; continue; }
      if (t_[p_] == '}') { ++p_; return v; }
      fail("expected , or }");
    }
  }
  const std::string& t_;
  size_t p_ = 0;
};

inline Value parse(const std::string& text) { return Parser(text).parse(); }

}  // namespace json
}  // namespace qmbed
