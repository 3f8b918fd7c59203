// A small strict JSON value, reader and writer for parameter deltas, profiles and replies.
// Reader: RFC 8259 text, one top-level value, numbers as binary64, duplicate keys keep the last.
// Writer: objects with keys in bytewise order, numbers in the shortest round-trip form, non-finite as null.
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <string_view>
#include <variant>
#include <vector>

namespace spkb::json {

class Value;
using Array = std::vector<Value>;
using Object = std::map<std::string, Value, std::less<>>;

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

class Value {
public:
    Value() = default;
    Value(std::nullptr_t) {}
    Value(bool b) : v_(b) {}
    Value(double d) : v_(d) {}
    Value(int i) : v_(double(i)) {}
    Value(unsigned u) : v_(double(u)) {}
    Value(long long i) : v_(double(i)) {}
    Value(const char* s) : v_(std::string(s)) {}
    Value(std::string s) : v_(std::move(s)) {}
    Value(Array a) : v_(std::make_shared<Array>(std::move(a))) {}
    Value(Object o) : v_(std::make_shared<Object>(std::move(o))) {}

    bool is_null() const { return v_.index() == 0; }
    bool is_bool() const { return v_.index() == 1; }
    bool is_number() const { return v_.index() == 2; }
    bool is_string() const { return v_.index() == 3; }
    bool is_array() const { return v_.index() == 4; }
    bool is_object() const { return v_.index() == 5; }

    bool as_bool() const { return std::get<1>(v_); }
    double as_number() const { return std::get<2>(v_); }
    const std::string& as_string() const { return std::get<3>(v_); }
    const Array& as_array() const { return *std::get<4>(v_); }
    const Object& as_object() const { return *std::get<5>(v_); }
    Array& as_array() { return *std::get<4>(v_); }
    Object& as_object() { return *std::get<5>(v_); }

    // Object member lookup; nullptr when absent or not an object.
    const Value* find(std::string_view key) const;
    // Object member for writing; turns a null value into an empty object first.
    Value& operator[](const std::string& key);

    bool operator==(const Value& o) const;

private:
    std::variant<std::monostate, bool, double, std::string, std::shared_ptr<Array>, std::shared_ptr<Object>> v_;
};

Value parse(std::string_view text);
std::string write(const Value& v);

}  // namespace spkb::json
