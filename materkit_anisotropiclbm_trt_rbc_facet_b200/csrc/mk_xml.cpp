// mk_xml.cpp — see mk_xml.hpp.
#include "mk_xml.hpp"

#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace mkx {

const Element* Element::child(const std::string& n) const {
  for (const auto& c : children)
    if (c->name == n) return c.get();
  return nullptr;
}

const Element* Element::path(const std::string& p) const {
  const Element* cur = this;
  size_t a = 0;
  while (cur && a <= p.size()) {
    size_t b = p.find('/', a);
    if (b == std::string::npos) b = p.size();
    const std::string part = p.substr(a, b - a);
    if (!part.empty()) cur = cur->child(part);
    a = b + 1;
  }
  return cur;
}

std::vector<const Element*> Element::all(const std::string& n) const {
  std::vector<const Element*> v;
  for (const auto& c : children)
    if (c->name == n) v.push_back(c.get());
  return v;
}

namespace {

struct Parser {
  const std::string& s;
  size_t i = 0;
  std::string err;
  explicit Parser(const std::string& src) : s(src) {}

  bool starts(const char* t) const { return s.compare(i, strlen(t), t) == 0; }

  bool skip_until(const char* t) {
    size_t j = s.find(t, i);
    if (j == std::string::npos) return false;
    i = j + strlen(t);
    return true;
  }

  static bool name_char(char c) {
    return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_' || c == '-' ||
           c == '.' || c == ':';
  }

  // Skips prolog, comments, doctype and processing instructions.  Returns
  // false only on an unterminated construct.
  bool skip_misc() {
    for (;;) {
      while (i < s.size() && isspace((unsigned char)s[i])) ++i;
      if (starts("<?")) {
        if (!skip_until("?>")) return fail("unterminated <?");
      } else if (starts("<!--")) {
        if (!skip_until("-->")) return fail("unterminated comment");
      } else if (starts("<!DOCTYPE") || starts("<!doctype")) {
        if (!skip_until(">")) return fail("unterminated DOCTYPE");
      } else {
        return true;
      }
    }
  }

  bool fail(const std::string& m) {
    std::ostringstream o;
    o << m << " at byte " << i;
    err = o.str();
    return false;
  }

  bool element(std::unique_ptr<Element>& out, int depth) {
    if (depth > 256) return fail("nesting too deep");
    if (i >= s.size() || s[i] != '<') return fail("expected '<'");
    ++i;
    size_t a = i;
    while (i < s.size() && name_char(s[i])) ++i;
    if (i == a) return fail("empty element name");
    out.reset(new Element());
    out->name = s.substr(a, i - a);
    // attributes (ignored)
    for (;;) {
      while (i < s.size() && isspace((unsigned char)s[i])) ++i;
      if (i >= s.size()) return fail("unterminated start tag");
      if (s[i] == '/') {
        if (i + 1 < s.size() && s[i + 1] == '>') {
          i += 2;
          return true;
        }
        return fail("bad '/' in tag");
      }
      if (s[i] == '>') {
        ++i;
        break;
      }
      if (s[i] == '"' || s[i] == '\'') {
        const char q = s[i++];
        while (i < s.size() && s[i] != q) ++i;
        if (i >= s.size()) return fail("unterminated attribute");
        ++i;
      } else {
        ++i;
      }
    }
    // content
    for (;;) {
      if (i >= s.size()) return fail("unterminated element <" + out->name + ">");
      if (starts("<!--")) {
        if (!skip_until("-->")) return fail("unterminated comment");
      } else if (starts("<![CDATA[")) {
        i += 9;
        size_t j = s.find("]]>", i);
        if (j == std::string::npos) return fail("unterminated CDATA");
        out->text += s.substr(i, j - i);
        i = j + 3;
      } else if (starts("<?")) {
        if (!skip_until("?>")) return fail("unterminated <?");
      } else if (starts("</")) {
        i += 2;
        size_t a2 = i;
        while (i < s.size() && name_char(s[i])) ++i;
        if (s.compare(a2, i - a2, out->name) != 0 || i - a2 != out->name.size())
          return fail("mismatched end tag for <" + out->name + ">");
        while (i < s.size() && isspace((unsigned char)s[i])) ++i;
        if (i >= s.size() || s[i] != '>') return fail("bad end tag");
        ++i;
        return true;
      } else if (s[i] == '<') {
        std::unique_ptr<Element> c;
        if (!element(c, depth + 1)) return false;
        out->children.push_back(std::move(c));
      } else {
        size_t j = s.find('<', i);
        if (j == std::string::npos) j = s.size();
        out->text += s.substr(i, j - i);
        i = j;
      }
    }
  }
};

}  // namespace

bool parse_string(const std::string& text, Document& doc, std::string& err) {
  Parser p(text);
  // optional UTF-8 byte-order mark
  if (text.size() >= 3 && (unsigned char)text[0] == 0xEF && (unsigned char)text[1] == 0xBB &&
      (unsigned char)text[2] == 0xBF)
    p.i = 3;
  if (!p.skip_misc()) {
    err = p.err;
    return false;
  }
  if (!p.element(doc.root, 0)) {
    err = p.err;
    return false;
  }
  return true;
}

bool parse_file(const std::string& path, Document& doc, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::ostringstream ss;
  ss << f.rdbuf();
  if (!parse_string(ss.str(), doc, err)) {
    err = path + ": " + err;
    return false;
  }
  return true;
}

std::string trimmed(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) ++a;
  while (b > a && isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

bool read_doubles(const Element* e, std::vector<double>& out, std::string& err) {
  out.clear();
  if (!e) {
    err = "missing element";
    return false;
  }
  std::istringstream in(e->text);
  std::string tok;
  while (in >> tok) {
    char* end = nullptr;
    errno = 0;
    double v = strtod(tok.c_str(), &end);
    if (end == tok.c_str() || *end != '\0' || errno == ERANGE) {
      // hexadecimal integers (seed values such as 0xB200)
      if (tok.size() > 2 && tok[0] == '0' && (tok[1] == 'x' || tok[1] == 'X')) {
        errno = 0;
        unsigned long long h = strtoull(tok.c_str(), &end, 16);
        if (*end == '\0' && errno == 0) {
          out.push_back((double)h);
          continue;
        }
      }
      err = "<" + e->name + ">: cannot read '" + tok + "' as a number";
      return false;
    }
    out.push_back(v);
  }
  return true;
}

bool read_double(const Element* e, double& out, std::string& err) {
  std::vector<double> v;
  if (!read_doubles(e, v, err)) return false;
  if (v.empty()) {
    err = "<" + e->name + ">: empty value";
    return false;
  }
  out = v[0];
  return true;
}

bool read_int(const Element* e, int& out, std::string& err) {
  double d;
  if (!read_double(e, d, err)) return false;
  out = (int)d;
  if ((double)out != d) {
    err = "<" + e->name + ">: not an integer";
    return false;
  }
  return true;
}

bool read_bool(const Element* e, bool& out, std::string& err) {
  if (!e) {
    err = "missing element";
    return false;
  }
  std::string t = trimmed(e->text);
  for (auto& c : t) c = (char)tolower((unsigned char)c);
  if (t == "true" || t == "1" || t == "yes") {
    out = true;
    return true;
  }
  if (t == "false" || t == "0" || t == "no") {
    out = false;
    return true;
  }
  err = "<" + e->name + ">: cannot read '" + t + "' as a boolean";
  return false;
}

}  // namespace mkx
