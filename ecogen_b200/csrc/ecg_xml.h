// Minimal XML reader for ECOGEN case files: elements, attributes, text and comments.
// Attribute values are read as doubles the way tinyxml2's QueryDoubleAttribute does (a leading
// number is accepted, trailing characters are ignored), which is how the reference reads e.g.
// energyRef="-1.15e6." in its own EOS files.
#pragma once
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace ecg {
namespace xml {

struct Node {
  std::string name;
  std::map<std::string, std::string> attrs;
  std::vector<std::unique_ptr<Node>> children;
  std::string text;

  const Node* child(const std::string& n) const;
  std::vector<const Node*> all(const std::string& n) const;
  bool has(const std::string& a) const { return attrs.count(a) != 0; }
  std::string attr(const std::string& a) const;
  bool get_double(const std::string& a, double* v) const;
  bool get_int(const std::string& a, int* v) const;
  bool get_bool(const std::string& a, bool* v) const;
};

// Parses a file; returns the root element or nullptr (err receives a message).
std::unique_ptr<Node> parse_file(const std::string& path, std::string* err);
std::unique_ptr<Node> parse_string(const std::string& text, std::string* err);

std::string upper(std::string s);
std::string trim(const std::string& s);

}  // namespace xml
}  // namespace ecg
