#include "json.h"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <strings.h>

namespace cgfdm {

namespace {

struct Parser {
  const std::string &s;
  size_t i = 0;
  std::string err;
  explicit Parser(const std::string &t) : s(t) {}

  void ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
  }
  bool fail(const char *m) {
    if (err.empty()) {
      char buf[128];
      std::snprintf(buf, sizeof buf, "%s at offset %zu", m, i);
      err = buf;
    }
    return false;
  }
  bool lit(const char *w) {
    size_t n = std::strlen(w);
    if (s.compare(i, n, w) != 0) return fail("bad literal");
    i += n;
    return true;
  }
  bool string(std::string &out) {
    if (i >= s.size() || s[i] != '"') return fail("expected string");
    ++i;
    while (i < s.size() && s[i] != '"') {
      char c = s[i++];
      if (c == '\\' && i < s.size()) {
        char e = s[i++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (i + 4 > s.size()) return fail("bad escape");
            unsigned v = std::strtoul(s.substr(i, 4).c_str(), nullptr, 16);
            i += 4;
            if (v < 0x80) out += (char)v;
            else if (v < 0x800) { out += (char)(0xC0 | (v >> 6)); out += (char)(0x80 | (v & 0x3F)); }
            else { out += (char)(0xE0 | (v >> 12)); out += (char)(0x80 | ((v >> 6) & 0x3F));
                   out += (char)(0x80 | (v & 0x3F)); }
          } break;
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (i >= s.size()) return fail("unterminated string");
    ++i;
    return true;
  }
  bool value(Json &v) {
    ws();
    if (i >= s.size()) return fail("unexpected end");
    char c = s[i];
    if (c == '{') {
      v.kind = Json::Object;
      ++i;
      ws();
      if (i < s.size() && s[i] == '}') { ++i; return true; }
      for (;;) {
        ws();
        std::string key;
        if (!string(key)) return false;
        ws();
        if (i >= s.size() || s[i] != ':') return fail("expected ':'");
        ++i;
        Json child;
        if (!value(child)) return false;
        v.members.emplace_back(std::move(key), std::move(child));
        ws();
        if (i < s.size() && s[i] == ',') { ++i; continue; }
        if (i < s.size() && s[i] == '}') { ++i; return true; }
        return fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind = Json::Array;
      ++i;
      ws();
      if (i < s.size() && s[i] == ']') { ++i; return true; }
      for (;;) {
        Json child;
        if (!value(child)) return false;
        v.items.push_back(std::move(child));
        ws();
        if (i < s.size() && s[i] == ',') { ++i; continue; }
        if (i < s.size() && s[i] == ']') { ++i; return true; }
        return fail("expected ',' or ']'");
      }
    }
    if (c == '"') { v.kind = Json::String; return string(v.str); }
    if (c == 't') { v.kind = Json::Bool; v.boolean = true; v.num = 1; return lit("true"); }
    if (c == 'f') { v.kind = Json::Bool; v.boolean = false; v.num = 0; return lit("false"); }
    if (c == 'n') { v.kind = Json::Null; return lit("null"); }
    return number(v);
  }
  // Decimal text to double the way the reference's reader does it
  // (cjson.c:96-115): mantissa digits accumulated in a double, then one
  // multiplication by pow(10, exponent).  Matching it keeps DT, DH, TMAX
  // bit-identical to the reference's values.
  bool number(Json &v) {
    size_t start = i;
    double n = 0, sign = 1, scale = 0;
    int subscale = 0, signsubscale = 1;
    auto dig = [&](size_t k) { return k < s.size() && s[k] >= '0' && s[k] <= '9'; };
    if (i < s.size() && s[i] == '-') sign = -1, ++i;
    if (i < s.size() && s[i] == '0') ++i;
    if (i < s.size() && s[i] >= '1' && s[i] <= '9')
      do n = (n * 10.0) + (s[i++] - '0'); while (dig(i));
    if (i < s.size() && s[i] == '.' && dig(i + 1)) {
      ++i;
      do n = (n * 10.0) + (s[i++] - '0'), scale--; while (dig(i));
    }
    if (i < s.size() && (s[i] == 'e' || s[i] == 'E')) {
      ++i;
      if (i < s.size() && s[i] == '+') ++i;
      else if (i < s.size() && s[i] == '-') signsubscale = -1, ++i;
      while (dig(i)) subscale = (subscale * 10) + (s[i++] - '0');
    }
    if (i == start) return fail("bad value");
    v.kind = Json::Number;
    v.num = sign * n * std::pow(10.0, (scale + subscale * signsubscale));
    return true;
  }
};

}  // namespace

const Json *Json::get(const char *key) const {
  if (kind != Object) return nullptr;
  for (const auto &m : members)
    if (strcasecmp(m.first.c_str(), key) == 0) return &m.second;
  return nullptr;
}

int Json::as_int() const {
  if (kind == Bool) return boolean ? 1 : 0;
  if (kind != Number) return 0;
  // Integer view of a number: saturating conversion, as the reference's JSON
  // library stores valueint.
  if (num >= 2147483647.0) return 2147483647;
  if (num <= -2147483648.0) return (int)-2147483648.0;
  return (int)num;
}

double Json::as_double() const { return kind == Number ? num : (kind == Bool ? (boolean ? 1 : 0) : 0.0); }

bool Json::parse(const std::string &text, Json &out, std::string &err) {
  Parser p(text);
  out = Json();
  if (!p.value(out)) {
    err = p.err;
    return false;
  }
  return true;
}

bool Json::parse_file(const std::string &path, Json &out, std::string &err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  return parse(ss.str(), out, err);
}

}  // namespace cgfdm
