#include "ecg_xml.h"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace ecg {
namespace xml {

std::string upper(std::string s) {
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

const Node* Node::child(const std::string& n) const {
  for (auto& c : children)
    if (c->name == n) return c.get();
  return nullptr;
}

std::vector<const Node*> Node::all(const std::string& n) const {
  std::vector<const Node*> v;
  for (auto& c : children)
    if (c->name == n) v.push_back(c.get());
  return v;
}

std::string Node::attr(const std::string& a) const {
  auto it = attrs.find(a);
  return it == attrs.end() ? std::string() : it->second;
}

bool Node::get_double(const std::string& a, double* v) const {
  auto it = attrs.find(a);
  if (it == attrs.end()) return false;
  // sscanf("%lf") semantics: leading whitespace skipped, longest numeric prefix, rest ignored
  return std::sscanf(it->second.c_str(), "%lf", v) == 1;
}

bool Node::get_int(const std::string& a, int* v) const {
  auto it = attrs.find(a);
  if (it == attrs.end()) return false;
  return std::sscanf(it->second.c_str(), "%d", v) == 1;
}

bool Node::get_bool(const std::string& a, bool* v) const {
  auto it = attrs.find(a);
  if (it == attrs.end()) return false;
  std::string s = upper(trim(it->second));
  if (s == "TRUE" || s == "1") { *v = true; return true; }
  if (s == "FALSE" || s == "0") { *v = false; return true; }
  return false;
}

namespace {

struct Parser {
  const std::string& s;
  size_t i = 0;
  std::string err;
  explicit Parser(const std::string& t) : s(t) {}

  bool eof() const { return i >= s.size(); }
  void ws() {
    while (!eof() && std::isspace((unsigned char)s[i])) i++;
  }
  bool starts(const char* p) const { return s.compare(i, std::char_traits<char>::length(p), p) == 0; }

  bool skip_misc() {  // comments, declarations, processing instructions
    for (;;) {
      ws();
      if (starts("<!--")) {
        size_t e = s.find("-->", i + 4);
        if (e == std::string::npos) { err = "unterminated comment"; return false; }
        i = e + 3;
      } else if (starts("<?")) {
        size_t e = s.find("?>", i + 2);
        if (e == std::string::npos) { err = "unterminated declaration"; return false; }
        i = e + 2;
      } else if (starts("<!")) {
        size_t e = s.find('>', i + 2);
        if (e == std::string::npos) { err = "unterminated directive"; return false; }
        i = e + 1;
      } else {
        return true;
      }
    }
  }

  std::string name() {
    size_t a = i;
    while (!eof() && (std::isalnum((unsigned char)s[i]) || s[i] == '_' || s[i] == '-' || s[i] == ':' || s[i] == '.'))
      i++;
    return s.substr(a, i - a);
  }

  static std::string unescape(const std::string& v) {
    std::string o;
    for (size_t k = 0; k < v.size(); k++) {
      if (v[k] == '&') {
        size_t e = v.find(';', k);
        if (e != std::string::npos) {
          std::string ent = v.substr(k + 1, e - k - 1);
          if (ent == "lt") { o += '<'; k = e; continue; }
          if (ent == "gt") { o += '>'; k = e; continue; }
          if (ent == "amp") { o += '&'; k = e; continue; }
          if (ent == "quot") { o += '"'; k = e; continue; }
          if (ent == "apos") { o += '\''; k = e; continue; }
        }
      }
      o += v[k];
    }
    return o;
  }

  std::unique_ptr<Node> element() {
    if (eof() || s[i] != '<') { err = "expected '<'"; return nullptr; }
    i++;
    auto n = std::make_unique<Node>();
    n->name = name();
    if (n->name.empty()) { err = "empty element name"; return nullptr; }
    for (;;) {
      ws();
      if (eof()) { err = "unterminated tag <" + n->name; return nullptr; }
      if (starts("/>")) { i += 2; return n; }
      if (s[i] == '>') { i++; break; }
      std::string an = name();
      if (an.empty()) { err = "bad attribute in <" + n->name + ">"; return nullptr; }
      ws();
      if (eof() || s[i] != '=') { err = "expected '=' after " + an; return nullptr; }
      i++;
      ws();
      if (eof() || (s[i] != '"' && s[i] != '\'')) { err = "expected quote for " + an; return nullptr; }
      char q = s[i++];
      size_t e = s.find(q, i);
      if (e == std::string::npos) { err = "unterminated attribute " + an; return nullptr; }
      n->attrs[an] = unescape(s.substr(i, e - i));
      i = e + 1;
    }
    // content
    for (;;) {
      if (eof()) { err = "unterminated element <" + n->name + ">"; return nullptr; }
      if (starts("</")) {
        i += 2;
        std::string cn = name();
        ws();
        if (cn != n->name || eof() || s[i] != '>') { err = "mismatched </" + cn + "> for <" + n->name + ">"; return nullptr; }
        i++;
        return n;
      }
      if (starts("<!--") || starts("<?") || starts("<!")) {
        if (!skip_misc()) return nullptr;
        continue;
      }
      if (s[i] == '<') {
        auto c = element();
        if (!c) return nullptr;
        n->children.push_back(std::move(c));
        continue;
      }
      size_t e = s.find('<', i);
      if (e == std::string::npos) e = s.size();
      n->text += unescape(s.substr(i, e - i));
      i = e;
    }
  }
};

}  // namespace

std::unique_ptr<Node> parse_string(const std::string& text, std::string* err) {
  Parser p(text);
  if (!p.skip_misc()) {
    if (err) *err = p.err;
    return nullptr;
  }
  auto root = p.element();
  if (!root && err) *err = p.err;
  return root;
}

std::unique_ptr<Node> parse_file(const std::string& path, std::string* err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    if (err) *err = "cannot open " + path;
    return nullptr;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string e;
  auto r = parse_string(ss.str(), &e);
  if (!r && err) *err = path + ": " + e;
  return r;
}

}  // namespace xml
}  // namespace ecg
