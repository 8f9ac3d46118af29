// Minimal JSON value, reader and pretty writer for the index manifest
// (serde_json output of src/power_merge/storage.rs:132-214). Integers keep
// full 64-bit precision; floats round-trip through shortest %.17g.
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace zx {

struct JsonValue {
  enum Kind { Null, Bool, Int, Float, Str, Arr, Obj } kind = Null;
  bool b = false;
  bool neg = false;
  uint64_t u = 0;
  double d = 0;
  std::string s;
  std::vector<JsonValue> arr;
  std::vector<std::pair<std::string, JsonValue>> obj;

  static JsonValue null() { return JsonValue(); }
  static JsonValue boolean(bool v) {
    JsonValue j;
    j.kind = Bool;
    j.b = v;
    return j;
  }
  static JsonValue uint(uint64_t v) {
    JsonValue j;
    j.kind = Int;
    j.u = v;
    j.d = (double)v;
    return j;
  }
  static JsonValue real(double v) {
    JsonValue j;
    j.kind = Float;
    j.d = v;
    return j;
  }
  static JsonValue str(std::string v) {
    JsonValue j;
    j.kind = Str;
    j.s = std::move(v);
    return j;
  }
  static JsonValue array() {
    JsonValue j;
    j.kind = Arr;
    return j;
  }
  static JsonValue object() {
    JsonValue j;
    j.kind = Obj;
    return j;
  }

  const JsonValue* find(const char* key) const;
  JsonValue& set(const std::string& key, JsonValue v);  // appends (object order kept)
  bool is_null() const { return kind == Null; }
};

// Throws zx::Error on malformed input.
JsonValue json_parse(const std::string& text);
std::string json_write_pretty(const JsonValue& v);

}  // namespace zx
