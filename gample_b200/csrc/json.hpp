// json.hpp -- minimal JSON reader for gample condition files.
//
// Supports the subset the condition schema uses: objects, arrays, strings
// (with escapes), numbers, true/false/null. Parse errors throw json::Error.
#pragma once

#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace gample {
namespace json {

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct Value {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0.0;
  bool integral = false;  // the literal had no fraction/exponent
  std::string str;
  std::vector<Value> arr;
  std::vector<std::pair<std::string, Value>> obj;  // insertion order kept

  bool is_object() const { return kind == Object; }
  bool is_array() const { return kind == Array; }
  bool is_string() const { return kind == String; }
  bool is_number() const { return kind == Number; }
  const Value* find(const std::string& key) const {
    if (kind != Object) return nullptr;
    const Value* hit = nullptr;
    for (const auto& kv : obj)
      if (kv.first == key) hit = &kv.second;  // last duplicate wins
    return hit;
  }
};

class Parser {
 public:
  explicit Parser(const std::string& s) : s_(s) {}
  Value parse() {
    Value v = value();
    ws();
    if (i_ != s_.size()) fail("trailing characters");
    return v;
  }

 private:
  const std::string& s_;
  size_t i_ = 0;

  [[noreturn]] void fail(const char* what) {
    throw Error(std::string("JSON parse error at offset ") + std::to_string(i_) + ": " + what);
  }
  void ws() {
    while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
  }
  bool eat(char c) {
    ws();
    if (i_ < s_.size() && s_[i_] == c) {
      ++i_;
      return true;
    }
    return false;
  }
  Value value() {
    ws();
    if (i_ >= s_.size()) fail("unexpected end");
    char c = s_[i_];
    if (c == '{') return object();
    if (c == '[') return array();
    if (c == '"') {
      Value v;
      v.kind = Value::String;
      v.str = string();
      return v;
    }
    if (c == 't' || c == 'f' || c == 'n') return literal();
    return number();
  }
  Value object() {
    Value v;
    v.kind = Value::Object;
    ++i_;
    if (eat('}')) return v;
    do {
      ws();
      if (i_ >= s_.size() || s_[i_] != '"') fail("expected key");
      std::string k = string();
      if (!eat(':')) fail("expected ':'");
      v.obj.emplace_back(std::move(k), value());
    } while (eat(','));
    if (!eat('}')) fail("expected '}'");
    return v;
  }
  Value array() {
    Value v;
    v.kind = Value::Array;
    ++i_;
    if (eat(']')) return v;
    do {
      v.arr.push_back(value());
    } while (eat(','));
    if (!eat(']')) fail("expected ']'");
    return v;
  }
  std::string string() {
    std::string out;
    ++i_;  // opening quote
    while (i_ < s_.size() && s_[i_] != '"') {
      char c = s_[i_++];
      if (c == '\\') {
        if (i_ >= s_.size()) fail("bad escape");
        char e = s_[i_++];
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
            if (i_ + 4 > s_.size()) fail("bad \\u escape");
            unsigned cp = std::stoul(s_.substr(i_, 4), nullptr, 16);
            i_ += 4;
            if (cp < 0x80) {
              out += char(cp);
            } else if (cp < 0x800) {
              out += char(0xC0 | (cp >> 6));
              out += char(0x80 | (cp & 0x3F));
            } else {
              out += char(0xE0 | (cp >> 12));
              out += char(0x80 | ((cp >> 6) & 0x3F));
              out += char(0x80 | (cp & 0x3F));
            }
            break;
          }
          default: fail("bad escape");
        }
      } else {
        out += c;
      }
    }
    if (i_ >= s_.size()) fail("unterminated string");
    ++i_;
    return out;
  }
  Value literal() {
    Value v;
    if (s_.compare(i_, 4, "true") == 0) {
      v.kind = Value::Bool;
      v.b = true;
      i_ += 4;
    } else if (s_.compare(i_, 5, "false") == 0) {
      v.kind = Value::Bool;
      i_ += 5;
    } else if (s_.compare(i_, 4, "null") == 0) {
      i_ += 4;
    } else {
      fail("bad literal");
    }
    return v;
  }
  Value number() {
    size_t start = i_;
    if (i_ < s_.size() && (s_[i_] == '-' || s_[i_] == '+')) ++i_;
    bool frac = false;
    while (i_ < s_.size()) {
      char c = s_[i_];
      if (c >= '0' && c <= '9') {
        ++i_;
      } else if (c == '.' || c == 'e' || c == 'E' || ((c == '-' || c == '+') && (s_[i_ - 1] == 'e' || s_[i_ - 1] == 'E'))) {
        frac = true;
        ++i_;
      } else {
        break;
      }
    }
    if (i_ == start) fail("unexpected character");
    Value v;
    v.kind = Value::Number;
    std::string tok = s_.substr(start, i_ - start);
    char* end = nullptr;
    v.num = std::strtod(tok.c_str(), &end);
    if (!end || *end != '\0') fail("bad number");
    v.integral = !frac;
    return v;
  }
};

inline Value parse(const std::string& text) { return Parser(text).parse(); }

}  // namespace json
}  // namespace gample
