// Material-file reader for the subset of Akantu's .dat grammar the explicit
// path needs (src/io/parser/input_file_parser.hh:113-252, parser.hh:68-432):
//   # comments, `key = value` global parameters, sections
//   `material <type> [ key = value ... ]` (nested sections are skipped),
//   numeric values with + - * / ^, parentheses and unary signs, booleans
//   true/false, and bare strings (names).
#pragma once

#include <map>
#include <string>
#include <vector>

namespace akb {

struct ParsedMaterial {
  std::string type;  // elastic | neohookean | plastic_linear_isotropic_hardening
  std::string name;
  std::map<std::string, std::string> raw;  // key -> value text, in file order
};

struct ParsedFile {
  std::map<std::string, std::string> globals;
  std::vector<ParsedMaterial> materials;
};

// returns false and fills err on a syntax error
bool parse_dat(const std::string &text, ParsedFile &out, std::string &err);
// evaluates a numeric / boolean value text; returns false if it is neither
bool eval_value(const std::string &text, double &value);

}  // namespace akb
