// Minimal JSON reader for params.json and station.json.
//
// Behaviour matched to the reference's use of its JSON library
// (src-new-FP32-SVE/getParams.cpp:41-247, station.cpp:112-181): object keys
// are looked up case-insensitively and the first matching member wins;
// numbers expose both a double value and a truncated integer value; object
// members keep their file order.
#pragma once
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace cgfdm {

struct Json {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  double num = 0.0;
  bool boolean = false;
  std::string str;
  std::vector<Json> items;                               // Array
  std::vector<std::pair<std::string, Json>> members;     // Object, file order

  // Case-insensitive member lookup; nullptr when absent.
  const Json *get(const char *key) const;
  int as_int() const;   // integer value of a number (truncation toward zero), bool
  double as_double() const;

  // Parses text; returns false and sets err on malformed input.
  static bool parse(const std::string &text, Json &out, std::string &err);
  static bool parse_file(const std::string &path, Json &out, std::string &err);
};

}  // namespace cgfdm
