// mk_xml.hpp — minimal XML reader for the BoltzTechs case format.
//
// Replaces mkt::XMLreader / XMLreaderProxy (MaterKit/xml/mkTINYXMLIO.h:32-84),
// whose TinyXML parser body is inside the closed DLL.  Supports what the
// BoltzTechs*.xml files use: a prolog, nested elements with text, comments
// (any byte content, the shipped files carry GBK text in comments),
// attributes (ignored) and self-closing tags.  Values are whitespace-separated
// tokens read like XMLreaderProxy::read<T> (mkTINYXMLIO.hh:34-43), which
// fails when a token does not parse.
#ifndef MK_XML_HPP
#define MK_XML_HPP

#include <memory>
#include <string>
#include <vector>

namespace mkx {

struct Element {
  std::string name;
  std::string text;  // concatenated character data directly inside the element
  std::vector<std::unique_ptr<Element>> children;

  // First child with this name, or nullptr.
  const Element* child(const std::string& n) const;
  // Element at a '/'-separated path below this one, or nullptr.
  const Element* path(const std::string& p) const;
  // All children with this name.
  std::vector<const Element*> all(const std::string& n) const;
};

struct Document {
  std::unique_ptr<Element> root;
};

// Parse a file; returns false and sets err on failure.
bool parse_file(const std::string& path, Document& doc, std::string& err);
bool parse_string(const std::string& text, Document& doc, std::string& err);

// Token readers.  Return false (and set err) when a token is not a number.
bool read_doubles(const Element* e, std::vector<double>& out, std::string& err);
bool read_double(const Element* e, double& out, std::string& err);
bool read_int(const Element* e, int& out, std::string& err);
bool read_bool(const Element* e, bool& out, std::string& err);
std::string trimmed(const std::string& s);

}  // namespace mkx

#endif
