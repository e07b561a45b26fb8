// A small JSON reader (RFC 8259) for the library's host code: scene files and the
// autotuning cache.  Values are held as a tree of JVal; errors carry the byte offset.
#pragma once

#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <utility>
#include <vector>

namespace nd_json {

struct JVal {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;

  const JVal* get(const char* key) const {
    if (kind != OBJ) return nullptr;
    for (const auto& kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

class JsonParser {
 public:
  JsonParser(const char* s, size_t n) : s_(s), n_(n) {}

  bool parse(JVal* out) {
    ws();
    if (!value(out, 0)) return false;
    ws();
    if (i_ != n_) return fail("trailing characters");
    return true;
  }
  const std::string& error() const { return err_; }

 private:
  const char* s_;
  size_t n_, i_ = 0;
  std::string err_;

  bool fail(const char* what) {
    char buf[96];
    snprintf(buf, sizeof(buf), "JSON: %s at byte %zu", what, i_);
    err_ = buf;
    return false;
  }
  void ws() {
    while (i_ < n_ && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
  }
  bool lit(const char* w) {
    const size_t k = strlen(w);
    if (n_ - i_ < k || memcmp(s_ + i_, w, k) != 0) return false;
    i_ += k;
    return true;
  }
  bool value(JVal* v, int depth) {
    if (depth > 64) return fail("nesting too deep");
    if (i_ >= n_) return fail("unexpected end");
    const char c = s_[i_];
    if (c == '{') return object(v, depth);
    if (c == '[') return array(v, depth);
    if (c == '"') {
      v->kind = JVal::STR;
      return string(&v->str);
    }
    if (lit("true")) {
      v->kind = JVal::BOOL;
      v->b = true;
      return true;
    }
    if (lit("false")) {
      v->kind = JVal::BOOL;
      v->b = false;
      return true;
    }
    if (lit("null")) {
      v->kind = JVal::NUL;
      return true;
    }
    return number(v);
  }
  bool number(JVal* v) {
    const size_t start = i_;
    if (i_ < n_ && s_[i_] == '-') ++i_;
    bool digits = false;
    while (i_ < n_ && s_[i_] >= '0' && s_[i_] <= '9') ++i_, digits = true;
    if (i_ < n_ && s_[i_] == '.') {
      ++i_;
      while (i_ < n_ && s_[i_] >= '0' && s_[i_] <= '9') ++i_, digits = true;
    }
    if (!digits) return fail("bad value");
    if (i_ < n_ && (s_[i_] == 'e' || s_[i_] == 'E')) {
      ++i_;
      if (i_ < n_ && (s_[i_] == '+' || s_[i_] == '-')) ++i_;
      bool ed = false;
      while (i_ < n_ && s_[i_] >= '0' && s_[i_] <= '9') ++i_, ed = true;
      if (!ed) return fail("bad exponent");
    }
    v->kind = JVal::NUM;
    v->num = strtod(std::string(s_ + start, i_ - start).c_str(), nullptr);
    return true;
  }
  static void utf8(std::string* out, unsigned cp) {
    if (cp < 0x80) {
      out->push_back(char(cp));
    } else if (cp < 0x800) {
      out->push_back(char(0xC0 | (cp >> 6)));
      out->push_back(char(0x80 | (cp & 0x3F)));
    } else if (cp < 0x10000) {
      out->push_back(char(0xE0 | (cp >> 12)));
      out->push_back(char(0x80 | ((cp >> 6) & 0x3F)));
      out->push_back(char(0x80 | (cp & 0x3F)));
    } else {
      out->push_back(char(0xF0 | (cp >> 18)));
      out->push_back(char(0x80 | ((cp >> 12) & 0x3F)));
      out->push_back(char(0x80 | ((cp >> 6) & 0x3F)));
      out->push_back(char(0x80 | (cp & 0x3F)));
    }
  }
  bool hex4(unsigned* cp) {
    if (n_ - i_ < 4) return fail("bad \\u escape");
    unsigned v = 0;
    for (int k = 0; k < 4; ++k) {
      const char h = s_[i_++];
      v <<= 4;
      if (h >= '0' && h <= '9') v |= unsigned(h - '0');
      else if (h >= 'a' && h <= 'f') v |= unsigned(h - 'a' + 10);
      else if (h >= 'A' && h <= 'F') v |= unsigned(h - 'A' + 10);
      else return fail("bad \\u escape");
    }
    *cp = v;
    return true;
  }
  bool string(std::string* out) {
    ++i_;  // opening quote
    out->clear();
    while (i_ < n_) {
      const char c = s_[i_++];
      if (c == '"') return true;
      if (uint8_t(c) < 0x20) return fail("control character in string");
      if (c != '\\') {
        out->push_back(c);
        continue;
      }
      if (i_ >= n_) break;
      const char e = s_[i_++];
      switch (e) {
        case '"': out->push_back('"'); break;
        case '\\': out->push_back('\\'); break;
        case '/': out->push_back('/'); break;
        case 'b': out->push_back('\b'); break;
        case 'f': out->push_back('\f'); break;
        case 'n': out->push_back('\n'); break;
        case 'r': out->push_back('\r'); break;
        case 't': out->push_back('\t'); break;
        case 'u': {
          unsigned cp;
          if (!hex4(&cp)) return false;
          if (cp >= 0xD800 && cp < 0xDC00 && n_ - i_ >= 6 && s_[i_] == '\\' && s_[i_ + 1] == 'u') {
            i_ += 2;
            unsigned lo;
            if (!hex4(&lo)) return false;
            if (lo >= 0xDC00 && lo < 0xE000) cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          }
          utf8(out, cp);
          break;
        }
        default: return fail("bad escape");
      }
    }
    return fail("unterminated string");
  }
  bool array(JVal* v, int depth) {
    ++i_;
    v->kind = JVal::ARR;
    ws();
    if (i_ < n_ && s_[i_] == ']') {
      ++i_;
      return true;
    }
    while (true) {
      v->arr.emplace_back();
      ws();
      if (!value(&v->arr.back(), depth + 1)) return false;
      ws();
      if (i_ < n_ && s_[i_] == ',') {
        ++i_;
        continue;
      }
      if (i_ < n_ && s_[i_] == ']') {
        ++i_;
        return true;
      }
      return fail("expected , or ]");
    }
  }
  bool object(JVal* v, int depth) {
    ++i_;
    v->kind = JVal::OBJ;
    ws();
    if (i_ < n_ && s_[i_] == '}') {
      ++i_;
      return true;
    }
    while (true) {
      ws();
      if (i_ >= n_ || s_[i_] != '"') return fail("expected a key");
      std::string key;
      if (!string(&key)) return false;
      ws();
      if (i_ >= n_ || s_[i_] != ':') return fail("expected :");
      ++i_;
      ws();
      v->obj.emplace_back(std::move(key), JVal());
      if (!value(&v->obj.back().second, depth + 1)) return false;
      ws();
      if (i_ < n_ && s_[i_] == ',') {
        ++i_;
        continue;
      }
      if (i_ < n_ && s_[i_] == '}') {
        ++i_;
        return true;
      }
      return fail("expected , or }");
    }
  }
};

}  // namespace nd_json
