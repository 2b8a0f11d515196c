// Test infrastructure only (see core.h). The reference's file formats: little-endian arrays at 8-byte-aligned
// offsets described by a JSON manifest (io.rs:5-55), a flat JSON writer (io.rs:77-125), the key scanner
// (jsonscan.rs:3-26) and state files <prefix>.{json,bin} (e7_state.rs:9-40).
#pragma once
#include <cstring>
#include <fstream>
#include <sstream>

#include "core.h"

namespace oracle {

struct BinaryArrays {
  std::vector<uint8_t> bytes;
  std::vector<std::string> entries;
  size_t align() {
    while (bytes.size() % 8) bytes.push_back(0);
    return bytes.size();
  }
  template <class T> void push(const std::string& name, const char* dtype, const std::vector<T>& v) {
    size_t off = align();
    size_t n = v.size() * sizeof(T);
    bytes.resize(off + n);
    if (n) std::memcpy(bytes.data() + off, v.data(), n);
    entries.push_back("{\"name\":\"" + name + "\",\"dtype\":\"" + dtype + "\",\"length\":" + std::to_string(v.size()) +
                      ",\"offset\":" + std::to_string(off) + "}");
  }
  void push_u32(const std::string& n, const std::vector<uint32_t>& v) { push(n, "u32", v); }
  void push_f32(const std::string& n, const std::vector<float>& v) { push(n, "f32", v); }
  void push_f64(const std::string& n, const std::vector<double>& v) { push(n, "f64", v); }
  std::string manifest() const {
    std::string s = "[";
    for (size_t i = 0; i < entries.size(); ++i) s += (i ? "," : "") + entries[i];
    return s + "]";
  }
  void write(const std::string& path) const {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error(path + ": cannot write");
    f.write(reinterpret_cast<const char*>(bytes.data()), std::streamsize(bytes.size()));
  }
};

inline std::string render_number(double v) {
  if (!std::isfinite(v)) return "null";
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.17g", v);
  return buf;
}

struct Json {
  std::vector<std::string> fields;
  Json& number(const std::string& k, double v) {
    fields.push_back("\"" + k + "\":" + render_number(v));
    return *this;
  }
  Json& integer(const std::string& k, long long v) {
    fields.push_back("\"" + k + "\":" + std::to_string(v));
    return *this;
  }
  Json& text(const std::string& k, const std::string& v) {
    fields.push_back("\"" + k + "\":\"" + v + "\"");
    return *this;
  }
  Json& flag(const std::string& k, bool v) {
    fields.push_back("\"" + k + "\":" + (v ? "true" : "false"));
    return *this;
  }
  Json& raw(const std::string& k, const std::string& v) {
    fields.push_back("\"" + k + "\":" + v);
    return *this;
  }
  std::string render() const {
    std::string s = "{";
    for (size_t i = 0; i < fields.size(); ++i) s += (i ? "," : "") + fields[i];
    return s + "}";
  }
};

// jsonscan.rs:3-26: the first `"key":` after the first `"anchor"`.
inline bool json_raw(const std::string& text, const std::string& anchor, const std::string& key, std::string& out) {
  size_t start = 0;
  if (!anchor.empty()) {
    start = text.find("\"" + anchor + "\"");
    if (start == std::string::npos) return false;
  }
  std::string marker = "\"" + key + "\":";
  size_t at = text.find(marker, start);
  if (at == std::string::npos) return false;
  at += marker.size();
  while (at < text.size() && std::isspace(static_cast<unsigned char>(text[at]))) ++at;
  size_t end;
  if (at < text.size() && text[at] == '"') {
    end = text.find('"', at + 1);
    if (end == std::string::npos) return false;
    out = text.substr(at + 1, end - at - 1);
    return true;
  }
  end = text.find_first_of(",}\n", at);
  if (end == std::string::npos) end = text.size();
  out = text.substr(at, end - at);
  while (!out.empty() && std::isspace(static_cast<unsigned char>(out.back()))) out.pop_back();
  return true;
}
inline double json_number(const std::string& t, const std::string& a, const std::string& k) {
  std::string v;
  if (!json_raw(t, a, k, v)) return NAN;
  char* end = nullptr;
  double d = std::strtod(v.c_str(), &end);
  return end == v.c_str() ? NAN : d;
}
inline std::string json_string(const std::string& t, const std::string& a, const std::string& k) {
  std::string v;
  return json_raw(t, a, k, v) ? v : std::string();
}
inline bool json_flag(const std::string& t, const std::string& a, const std::string& k) {
  std::string v;
  return json_raw(t, a, k, v) && v == "true";
}

inline std::string read_text(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error(path + ": cannot read");
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}
inline void write_text(const std::string& path, const std::string& text) {
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error(path + ": cannot write");
  f << text;
}

// e7_state.rs:9-40
inline void write_state(const std::string& prefix, const std::vector<Vec3>& x, double final_h, bool single) {
  std::ofstream f(prefix + ".bin", std::ios::binary);
  for (auto& p : x)
    for (double v : p) {
      if (single) {
        float s = float(v);
        f.write(reinterpret_cast<const char*>(&s), 4);
      } else {
        f.write(reinterpret_cast<const char*>(&v), 8);
      }
    }
  Json j;
  j.integer("vertices", (long long)x.size()).number("final_h", final_h).text("dtype", single ? "f32" : "f64");
  write_text(prefix + ".json", j.render());
}

inline std::vector<Vec3> read_state(const std::string& prefix, double* final_h) {
  std::string text = read_text(prefix + ".json"), bin = read_text(prefix + ".bin");
  bool single = json_string(text, "", "dtype") == "f32";
  std::vector<double> vals;
  if (single)
    for (size_t i = 0; i + 4 <= bin.size(); i += 4) {
      float f;
      std::memcpy(&f, bin.data() + i, 4);
      vals.push_back(f);
    }
  else
    for (size_t i = 0; i + 8 <= bin.size(); i += 8) {
      double d;
      std::memcpy(&d, bin.data() + i, 8);
      vals.push_back(d);
    }
  std::vector<Vec3> x;
  for (size_t i = 0; i + 3 <= vals.size(); i += 3) x.push_back({vals[i], vals[i + 1], vals[i + 2]});
  if (final_h) *final_h = json_number(text, "", "final_h");
  return x;
}

}  // namespace oracle
