// Minimal JSON value, parser and compact writer for the manifest and the ONTC container.
//
// The writer reproduces the byte format upstream's .ntc files carry (libopenntc/
// openntc_runtime.cpp:188-227 serialises with nlohmann::json::dump()):
//   * objects print their keys in byte-lexicographic order (a std::map), compact,
//     no whitespace;
//   * integers print in decimal, floats print the shortest round-trip decimal digits
//     of the double, placed as 'ddd.d' / '0.000ddd' / 'd.dddde+XX' by the rules in
//     format_double() below.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace ontc {

class Json {
 public:
  enum class Type { Null, Bool, Int, Uint, Float, String, Array, Object };

  Json() = default;
  static Json make_int(int64_t v) { Json j; j.type_ = Type::Int; j.i_ = v; return j; }
  static Json make_uint(uint64_t v) { Json j; j.type_ = Type::Uint; j.u_ = v; return j; }
  static Json make_float(double v) { Json j; j.type_ = Type::Float; j.d_ = v; return j; }
  static Json make_bool(bool v) { Json j; j.type_ = Type::Bool; j.b_ = v; return j; }
  static Json make_string(std::string v) { Json j; j.type_ = Type::String; j.s_ = std::move(v); return j; }
  static Json make_array() { Json j; j.type_ = Type::Array; return j; }
  static Json make_object() { Json j; j.type_ = Type::Object; return j; }

  Type type() const { return type_; }
  bool is_object() const { return type_ == Type::Object; }
  bool is_array() const { return type_ == Type::Array; }
  bool is_string() const { return type_ == Type::String; }
  bool is_bool() const { return type_ == Type::Bool; }
  bool is_integer() const { return type_ == Type::Int || type_ == Type::Uint; }
  bool is_number() const { return is_integer() || type_ == Type::Float; }

  int64_t as_int() const { return type_ == Type::Uint ? (int64_t)u_ : type_ == Type::Int ? i_ : (int64_t)d_; }
  uint64_t as_uint() const { return type_ == Type::Int ? (uint64_t)i_ : type_ == Type::Uint ? u_ : (uint64_t)d_; }
  double as_double() const { return type_ == Type::Float ? d_ : type_ == Type::Int ? (double)i_ : (double)u_; }
  bool as_bool() const { return b_; }
  const std::string& as_string() const { return s_; }

  // Arrays
  size_t size() const { return type_ == Type::Array ? arr_.size() : type_ == Type::Object ? obj_.size() : 0; }
  const Json& at(size_t i) const { return arr_[i]; }
  void push_back(Json v) { arr_.push_back(std::move(v)); }
  const std::vector<Json>& items() const { return arr_; }

  // Objects
  const Json* find(const std::string& key) const;
  Json& set(const std::string& key, Json v) { return obj_[key] = std::move(v); }
  const std::map<std::string, Json>& members() const { return obj_; }
  // Members in document order (the manifest's texture semantics are read in that
  // order by upstream; std::map order is only used when writing).
  const std::vector<std::string>& key_order() const { return order_; }

  std::string dump() const;

  // Strict RFC 8259 parse of [begin, end).  Returns false on any syntax error.
  static bool parse(const char* begin, const char* end, Json& out);

 private:
  friend struct JsonParser;
  Type type_ = Type::Null;
  bool b_ = false;
  int64_t i_ = 0;
  uint64_t u_ = 0;
  double d_ = 0.0;
  std::string s_;
  std::vector<Json> arr_;
  std::map<std::string, Json> obj_;
  std::vector<std::string> order_;
  void dump_to(std::string& out) const;
};

// Shortest round-trip digits of `v` placed as described in the file comment.
std::string format_double(double v);

}  // namespace ontc
