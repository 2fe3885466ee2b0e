// json.h -- a small JSON reader for the solver's parameter file.
//
// Objects, arrays, strings (with the standard escapes), numbers, true,
// false and null.  Enough for the par file of the forward run
// (src/forward/par_t.cu reads it with cJSON); errors throw
// std::runtime_error with the byte offset.
#pragma once
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace cgfd_json {

struct Value {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Value> arr;
  std::vector<std::pair<std::string, Value>> obj;   // file order kept

  const Value *get(const std::string &key) const {
    if (kind != Object) return nullptr;
    for (const auto &kv : obj) if (kv.first == key) return &kv.second;
    return nullptr;
  }
  // cJSON's valueint truncates the number
  int as_int() const { return (int)num; }
};

class Parser {
 public:
  explicit Parser(const std::string &s) : s_(s) {}
  Value parse() {
    Value v = value();
    ws();
    if (p_ != s_.size()) err("trailing characters");
    return v;
  }

 private:
  const std::string &s_;
  size_t p_ = 0;

  [[noreturn]] void err(const char *m) {
    throw std::runtime_error(std::string("par file: ") + m + " at byte " + std::to_string(p_));
  }
  void ws() {
    while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r')) p_++;
  }
  bool eat(char c) {
    ws();
    if (p_ < s_.size() && s_[p_] == c) { p_++; return true; }
    return false;
  }
  Value value() {
    ws();
    if (p_ >= s_.size()) err("unexpected end");
    const char c = s_[p_];
    Value v;
    if (c == '{') {
      p_++;
      v.kind = Value::Object;
      if (eat('}')) return v;
      do {
        ws();
        if (p_ >= s_.size() || s_[p_] != '"') err("expected a key");
        std::string k = string();
        if (!eat(':')) err("expected ':'");
        v.obj.emplace_back(k, value());
      } while (eat(','));
      if (!eat('}')) err("expected '}'");
    } else if (c == '[') {
      p_++;
      v.kind = Value::Array;
      if (eat(']')) return v;
      do v.arr.push_back(value()); while (eat(','));
      if (!eat(']')) err("expected ']'");
    } else if (c == '"') {
      v.kind = Value::String;
      v.str = string();
    } else if (s_.compare(p_, 4, "true") == 0) {
      p_ += 4; v.kind = Value::Bool; v.b = true;
    } else if (s_.compare(p_, 5, "false") == 0) {
      p_ += 5; v.kind = Value::Bool;
    } else if (s_.compare(p_, 4, "null") == 0) {
      p_ += 4;
    } else {
      const char *b = s_.c_str() + p_;
      char *e = nullptr;
      v.num = std::strtod(b, &e);
      if (e == b) err("unexpected character");
      v.kind = Value::Number;
      v.b = v.num != 0.0;
      p_ += (size_t)(e - b);
    }
    return v;
  }
  std::string string() {
    p_++;   // opening quote
    std::string out;
    while (p_ < s_.size() && s_[p_] != '"') {
      char c = s_[p_++];
      if (c == '\\') {
        if (p_ >= s_.size()) err("bad escape");
        const char e = s_[p_++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (p_ + 4 > s_.size()) err("bad \\u escape");
            const unsigned cp = (unsigned)std::strtoul(s_.substr(p_, 4).c_str(), nullptr, 16);
            p_ += 4;
            if (cp < 0x80) out += (char)cp;
            else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
            else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F)); }
            break;
          }
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (p_ >= s_.size()) err("unterminated string");
    p_++;
    return out;
  }
};

inline Value parse(const std::string &text) { return Parser(text).parse(); }

}  // namespace cgfd_json
