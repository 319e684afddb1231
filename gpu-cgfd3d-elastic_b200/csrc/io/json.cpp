// json.cpp -- recursive-descent JSON reader (RFC 8259 subset sufficient for parameter files).
#include "json.h"

#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace cgfd {
namespace json {

const Value *Value::get(const std::string &key) const {
  if (kind != OBJ) return nullptr;
  for (const auto &kv : obj)
    if (kv.first == key) return &kv.second;
  return nullptr;
}

namespace {

struct Parser {
  const std::string &s;
  size_t p = 0;
  explicit Parser(const std::string &t) : s(t) {}

  [[noreturn]] void fail(const char *what) {
    throw std::runtime_error(std::string("json: ") + what + " at byte " + std::to_string(p));
  }
  void ws() {
    while (p < s.size() && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n' || s[p] == '\r')) p++;
  }
  bool eat(char c) {
    ws();
    if (p < s.size() && s[p] == c) { p++; return true; }
    return false;
  }
  void expect(char c) {
    if (!eat(c)) fail("unexpected character");
  }
  std::string str() {
    ws();
    if (p >= s.size() || s[p] != '"') fail("expected string");
    p++;
    std::string out;
    while (p < s.size() && s[p] != '"') {
      char c = s[p++];
      if (c == '\\') {
        if (p >= s.size()) fail("bad escape");
        char e = s[p++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (p + 4 > s.size()) fail("bad \\u escape");
            unsigned cp = (unsigned)strtoul(s.substr(p, 4).c_str(), nullptr, 16);
            p += 4;
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
    if (p >= s.size()) fail("unterminated string");
    p++;
    return out;
  }
  Value value() {
    ws();
    if (p >= s.size()) fail("unexpected end");
    Value v;
    char c = s[p];
    if (c == '{') {
      p++;
      v.kind = Value::OBJ;
      if (eat('}')) return v;
      do {
        std::string k = str();
        expect(':');
        v.obj.emplace_back(k, value());
      } while (eat(','));
      expect('}');
    } else if (c == '[') {
      p++;
      v.kind = Value::ARR;
      if (eat(']')) return v;
      do v.arr.push_back(value());
      while (eat(','));
      expect(']');
    } else if (c == '"') {
      v.kind = Value::STR;
      v.str = str();
    } else if (s.compare(p, 4, "true") == 0) {
      p += 4; v.kind = Value::BOOL; v.b = true;
    } else if (s.compare(p, 5, "false") == 0) {
      p += 5; v.kind = Value::BOOL; v.b = false;
    } else if (s.compare(p, 4, "null") == 0) {
      p += 4;
    } else {
      const char *b = s.c_str() + p;
      char *e = nullptr;
      v.num = strtod(b, &e);
      if (e == b) fail("bad value");
      p += (size_t)(e - b);
      v.kind = Value::NUM;
    }
    return v;
  }
};

}  // namespace

Value parse(const std::string &text) {
  Parser ps(text);
  Value v = ps.value();
  ps.ws();
  if (ps.p != text.size()) ps.fail("trailing characters");
  return v;
}

Value parse_file(const std::string &path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parse(ss.str());
}

}  // namespace json
}  // namespace cgfd
