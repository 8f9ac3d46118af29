#include "json.h"

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "error.h"

namespace zx {

const JsonValue* JsonValue::find(const char* key) const {
  if (kind != Obj) return nullptr;
  for (auto& kv : obj)
    if (kv.first == key) return &kv.second;
  return nullptr;
}

JsonValue& JsonValue::set(const std::string& key, JsonValue v) {
  kind = Obj;
  obj.emplace_back(key, std::move(v));
  return obj.back().second;
}

namespace {

struct Reader {
  const char* p;
  const char* e;

  void ws() {
    while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  char peek() {
    ws();
    check_format(p < e, "manifest: unexpected end of JSON");
    return *p;
  }
  void expect(char c) {
    check_format(peek() == c, "manifest: malformed JSON");
    ++p;
  }
  static void utf8(std::string& out, unsigned cp) {
    if (cp < 0x80) {
      out += (char)cp;
    } else if (cp < 0x800) {
      out += (char)(0xC0 | (cp >> 6));
      out += (char)(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
      out += (char)(0xE0 | (cp >> 12));
      out += (char)(0x80 | ((cp >> 6) & 0x3F));
      out += (char)(0x80 | (cp & 0x3F));
    } else {
      out += (char)(0xF0 | (cp >> 18));
      out += (char)(0x80 | ((cp >> 12) & 0x3F));
      out += (char)(0x80 | ((cp >> 6) & 0x3F));
      out += (char)(0x80 | (cp & 0x3F));
    }
  }
  unsigned hex4() {
    check_format(e - p >= 4, "manifest: bad \\u escape");
    unsigned v = 0;
    for (int i = 0; i < 4; ++i) {
      char c = *p++;
      v <<= 4;
      if (c >= '0' && c <= '9') v |= (unsigned)(c - '0');
      else if (c >= 'a' && c <= 'f') v |= (unsigned)(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') v |= (unsigned)(c - 'A' + 10);
      else raise(kEFormat, "manifest: bad \\u escape");
    }
    return v;
  }
  std::string string() {
    expect('"');
    std::string out;
    while (true) {
      check_format(p < e, "manifest: unterminated string");
      char c = *p++;
      if (c == '"') break;
      if (c != '\\') {
        out += c;
        continue;
      }
      check_format(p < e, "manifest: bad escape");
      c = *p++;
      switch (c) {
        case '"': out += '"'; break;
        case '\\': out += '\\'; break;
        case '/': out += '/'; break;
        case 'b': out += '\b'; break;
        case 'f': out += '\f'; break;
        case 'n': out += '\n'; break;
        case 'r': out += '\r'; break;
        case 't': out += '\t'; break;
        case 'u': {
          unsigned cp = hex4();
          if (cp >= 0xD800 && cp < 0xDC00 && e - p >= 6 && p[0] == '\\' && p[1] == 'u') {
            p += 2;
            unsigned lo = hex4();
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          }
          utf8(out, cp);
          break;
        }
        default: raise(kEFormat, "manifest: bad escape");
      }
    }
    return out;
  }
  JsonValue value(int depth) {
    check_format(depth < 64, "manifest: JSON nesting too deep");
    char c = peek();
    if (c == '{') {
      ++p;
      JsonValue v = JsonValue::object();
      if (peek() == '}') {
        ++p;
        return v;
      }
      while (true) {
        std::string key = string();
        expect(':');
        v.obj.emplace_back(std::move(key), value(depth + 1));
        char n = peek();
        ++p;
        if (n == '}') break;
        check_format(n == ',', "manifest: malformed object");
      }
      return v;
    }
    if (c == '[') {
      ++p;
      JsonValue v = JsonValue::array();
      if (peek() == ']') {
        ++p;
        return v;
      }
      while (true) {
        v.arr.push_back(value(depth + 1));
        char n = peek();
        ++p;
        if (n == ']') break;
        check_format(n == ',', "manifest: malformed array");
      }
      return v;
    }
    if (c == '"') return JsonValue::str(string());
    if (e - p >= 4 && !strncmp(p, "true", 4)) {
      p += 4;
      return JsonValue::boolean(true);
    }
    if (e - p >= 5 && !strncmp(p, "false", 5)) {
      p += 5;
      return JsonValue::boolean(false);
    }
    if (e - p >= 4 && !strncmp(p, "null", 4)) {
      p += 4;
      return JsonValue::null();
    }
    const char* s = p;
    bool neg = false, integral = true;
    if (*p == '-') {
      neg = true;
      ++p;
    }
    while (p < e && ((*p >= '0' && *p <= '9') || *p == '.' || *p == 'e' || *p == 'E' ||
                     *p == '+' || *p == '-')) {
      if (*p == '.' || *p == 'e' || *p == 'E') integral = false;
      ++p;
    }
    std::string text(s, p);
    check_format(text.size() > (neg ? 1u : 0u), "manifest: malformed value");
    JsonValue v;
    if (integral) {
      v.kind = JsonValue::Int;
      v.neg = neg;
      errno = 0;
      v.u = strtoull(text.c_str() + (neg ? 1 : 0), nullptr, 10);
      check_format(errno == 0, "manifest: integer out of range");
      v.d = neg ? -(double)v.u : (double)v.u;
    } else {
      v.kind = JsonValue::Float;
      v.d = strtod(text.c_str(), nullptr);
    }
    return v;
  }
};

void escape(std::string& out, const std::string& s) {
  out += '"';
  for (unsigned char c : s) {
    switch (c) {
      case '"': out += "\\\""; break;
      case '\\': out += "\\\\"; break;
      case '\n': out += "\\n"; break;
      case '\r': out += "\\r"; break;
      case '\t': out += "\\t"; break;
      case '\b': out += "\\b"; break;
      case '\f': out += "\\f"; break;
      default:
        if (c < 0x20) {
          char buf[8];
          snprintf(buf, sizeof buf, "\\u%04x", c);
          out += buf;
        } else {
          out += (char)c;
        }
    }
  }
  out += '"';
}

void write(std::string& out, const JsonValue& v, int indent) {
  std::string pad((size_t)indent * 2, ' '), inner((size_t)(indent + 1) * 2, ' ');
  char buf[64];
  switch (v.kind) {
    case JsonValue::Null: out += "null"; break;
    case JsonValue::Bool: out += v.b ? "true" : "false"; break;
    case JsonValue::Int:
      snprintf(buf, sizeof buf, "%s%llu", v.neg ? "-" : "", (unsigned long long)v.u);
      out += buf;
      break;
    case JsonValue::Float: {
      snprintf(buf, sizeof buf, "%.17g", v.d);
      std::string t = buf;
      if (t.find_first_of(".eEn") == std::string::npos) t += ".0";
      out += t;
      break;
    }
    case JsonValue::Str: escape(out, v.s); break;
    case JsonValue::Arr:
      if (v.arr.empty()) {
        out += "[]";
        break;
      }
      out += "[\n";
      for (size_t i = 0; i < v.arr.size(); ++i) {
        out += inner;
        write(out, v.arr[i], indent + 1);
        out += i + 1 < v.arr.size() ? ",\n" : "\n";
      }
      out += pad + "]";
      break;
    case JsonValue::Obj:
      if (v.obj.empty()) {
        out += "{}";
        break;
      }
      out += "{\n";
      for (size_t i = 0; i < v.obj.size(); ++i) {
        out += inner;
        escape(out, v.obj[i].first);
        out += ": ";
        write(out, v.obj[i].second, indent + 1);
        out += i + 1 < v.obj.size() ? ",\n" : "\n";
      }
      out += pad + "}";
      break;
  }
}

}  // namespace

JsonValue json_parse(const std::string& text) {
  Reader r{text.data(), text.data() + text.size()};
  JsonValue v = r.value(0);
  r.ws();
  check_format(r.p == r.e, "manifest: trailing characters after JSON");
  return v;
}

std::string json_write_pretty(const JsonValue& v) {
  std::string out;
  write(out, v, 0);
  return out;
}

}  // namespace zx
