#include "dat_parser.h"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <functional>

namespace akb {

namespace {

std::string trim(const std::string &s) {
  size_t b = 0, e = s.size();
  while (b < e && std::isspace((unsigned char)s[b])) ++b;
  while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
  return s.substr(b, e - b);
}

// recursive-descent arithmetic: expr := term (('+'|'-') term)*,
// term := power (('*'|'/') power)*, power := unary ('^' power)?,
// unary := ('+'|'-') unary | number | '(' expr ')'
struct Expr {
  const std::string &s;
  size_t p = 0;
  bool ok = true;
  explicit Expr(const std::string &str) : s(str) {}
  void ws() {
    while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
  }
  double expr() {
    double v = term();
    for (;;) {
      ws();
      if (p < s.size() && (s[p] == '+' || s[p] == '-')) {
        char op = s[p++];
        double r = term();
        v = op == '+' ? v + r : v - r;
      } else {
        return v;
      }
    }
  }
  double term() {
    double v = power();
    for (;;) {
      ws();
      if (p < s.size() && (s[p] == '*' || s[p] == '/')) {
        char op = s[p++];
        double r = power();
        v = op == '*' ? v * r : v / r;
      } else {
        return v;
      }
    }
  }
  double power() {
    double v = unary();
    ws();
    if (p < s.size() && s[p] == '^') {
      ++p;
      double r = power();
      v = std::pow(v, r);
    }
    return v;
  }
  double unary() {
    ws();
    if (p >= s.size()) {
      ok = false;
      return 0;
    }
    if (s[p] == '+') { ++p; return unary(); }
    if (s[p] == '-') { ++p; return -unary(); }
    if (s[p] == '(') {
      ++p;
      double v = expr();
      ws();
      if (p < s.size() && s[p] == ')') ++p;
      else ok = false;
      return v;
    }
    const char *b = s.c_str() + p;
    char *e = nullptr;
    double v = std::strtod(b, &e);
    if (e == b) {
      ok = false;
      return 0;
    }
    p += (size_t)(e - b);
    return v;
  }
};

}  // namespace

bool eval_value(const std::string &text, double &value) {
  std::string t = trim(text);
  if (t == "true") { value = 1.; return true; }
  if (t == "false") { value = 0.; return true; }
  Expr ex(t);
  double v = ex.expr();
  ex.ws();
  if (!ex.ok || ex.p != t.size()) return false;
  value = v;
  return true;
}

bool parse_dat(const std::string &text, ParsedFile &out, std::string &err) {
  // strip comments, keep line structure
  std::string src;
  src.reserve(text.size());
  bool in_comment = false;
  for (char c : text) {
    if (c == '#') in_comment = true;
    if (c == '\n') in_comment = false;
    if (!in_comment) src.push_back(c);
  }
  size_t p = 0;
  const size_t n = src.size();
  auto skip_ws = [&]() {
    while (p < n && std::isspace((unsigned char)src[p])) ++p;
  };
  auto read_word = [&]() {
    size_t b = p;
    while (p < n && (std::isalnum((unsigned char)src[p]) || src[p] == '_' || src[p] == '.' ||
                     src[p] == '-' || src[p] == '+'))
      ++p;
    return src.substr(b, p - b);
  };
  // value: rest of the logical line (until newline, ']' or '[' at depth 0),
  // or a bracketed matrix / vector "[...]" up to its closing bracket (it may
  // span lines)
  auto read_value = [&]() {
    size_t b = p;
    if (p < n && src[p] == '[') {
      int brackets = 0;
      while (p < n) {
        if (src[p] == '[') ++brackets;
        if (src[p] == ']' && --brackets == 0) {
          ++p;
          break;
        }
        ++p;
      }
      return trim(src.substr(b, p - b));
    }
    int depth = 0;
    while (p < n && src[p] != '\n') {
      if (src[p] == '(') ++depth;
      if (src[p] == ')') --depth;
      if (depth == 0 && (src[p] == ']' || src[p] == '[')) break;
      ++p;
    }
    return trim(src.substr(b, p - b));
  };
  // body of a section: key = value pairs and nested sections
  std::function<bool(ParsedMaterial *)> body = [&](ParsedMaterial *mat) -> bool {
    for (;;) {
      skip_ws();
      if (p >= n) {
        err = "unterminated section";
        return false;
      }
      if (src[p] == ']') {
        ++p;
        return true;
      }
      std::string key = read_word();
      if (key.empty()) {
        err = std::string("unexpected character '") + src[p] + "'";
        return false;
      }
      skip_ws();
      if (p < n && src[p] == '=') {
        ++p;
        skip_ws();
        std::string val = read_value();
        if (mat) {
          if (key == "name") mat->name = val;
          mat->raw[key] = val;
        }
        continue;
      }
      // nested section: key [name] [ ... ]
      std::string maybe_name;
      if (p < n && src[p] != '[') maybe_name = read_word();
      skip_ws();
      if (p >= n || src[p] != '[') {
        err = "expected '=' or '[' after '" + key + "'";
        return false;
      }
      ++p;
      if (!body(nullptr)) return false;
    }
  };
  for (;;) {
    skip_ws();
    if (p >= n) break;
    std::string key = read_word();
    if (key.empty()) {
      err = std::string("unexpected character '") + src[p] + "'";
      return false;
    }
    skip_ws();
    if (p < n && src[p] == '=') {
      ++p;
      skip_ws();
      out.globals[key] = read_value();
      continue;
    }
    std::string sub;
    if (p < n && src[p] != '[') {
      sub = read_word();
      skip_ws();
    }
    if (p >= n || src[p] != '[') {
      err = "expected '[' after section '" + key + "'";
      return false;
    }
    ++p;
    if (key == "material") {
      ParsedMaterial m;
      m.type = sub;
      if (!body(&m)) return false;
      out.materials.push_back(m);
    } else {
      if (!body(nullptr)) return false;
    }
  }
  return true;
}

}  // namespace akb
