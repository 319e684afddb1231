// json.h -- minimal JSON reader for the parameter file (objects, arrays, numbers, strings,
// true/false/null). Keys starting with '#' are kept and simply never looked up, which is how
// the reference's parameter files comment out options.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace cgfd {
namespace json {

struct Value {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  double num = 0.0;
  bool b = false;
  std::string str;
  std::vector<Value> arr;
  std::vector<std::pair<std::string, Value>> obj;  // insertion order kept

  const Value *get(const std::string &key) const;  // nullptr when absent / not an object
  bool is_obj() const { return kind == OBJ; }
  bool is_num() const { return kind == NUM || kind == BOOL; }
  double as_num(double def = 0.0) const { return kind == NUM ? num : (kind == BOOL ? (b ? 1.0 : 0.0) : def); }
  int as_int(int def = 0) const { return is_num() ? (int)as_num() : def; }
  std::string as_str(const std::string &def = "") const { return kind == STR ? str : def; }
};

// Parses `text`; throws std::runtime_error with the byte offset on malformed input.
Value parse(const std::string &text);
Value parse_file(const std::string &path);

}  // namespace json
}  // namespace cgfd
