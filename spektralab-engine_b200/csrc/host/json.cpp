#include "json.hpp"

#include <charconv>
#include <cmath>
#include <cstdio>

namespace spkb::json {

const Value* Value::find(std::string_view key) const {
    if (!is_object()) return nullptr;
    const Object& o = as_object();
    auto it = o.find(key);
    return it == o.end() ? nullptr : &it->second;
}

Value& Value::operator[](const std::string& key) {
    if (is_null()) v_ = std::make_shared<Object>();
    return as_object()[key];
}

bool Value::operator==(const Value& o) const {
    if (v_.index() != o.v_.index()) return false;
    switch (v_.index()) {
        case 0: return true;
        case 1: return as_bool() == o.as_bool();
        case 2: return as_number() == o.as_number();
        case 3: return as_string() == o.as_string();
        case 4: return as_array() == o.as_array();
        default: return as_object() == o.as_object();
    }
}

namespace {

class Reader {
public:
    explicit Reader(std::string_view t) : s_(t) {}

    Value run() {
        ws();
        Value v = value(0);
        ws();
        if (i_ != s_.size()) err("trailing characters");
        return v;
    }

private:
    std::string_view s_;
    size_t i_ = 0;

    [[noreturn]] void err(const char* what) const {
        throw ParseError(std::string("JSON: ") + what + " at offset " + std::to_string(i_));
    }
    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
    }
    bool lit(std::string_view w) {
        if (s_.substr(i_, w.size()) == w) {
            i_ += w.size();
            return true;
        }
        return false;
    }
    Value value(int depth) {
        if (depth > 256) err("nesting too deep");
        if (i_ >= s_.size()) err("unexpected end");
        const char c = s_[i_];
        if (c == '{') return object(depth);
        if (c == '[') return array(depth);
        if (c == '"') return Value(string());
        if (lit("true")) return Value(true);
        if (lit("false")) return Value(false);
        if (lit("null")) return Value();
        if (c == '-' || (c >= '0' && c <= '9')) return Value(number());
        err("unexpected character");
    }
    double number() {
        const size_t b = i_;
        if (s_[i_] == '-') ++i_;
        auto digits = [&] {
            const size_t d = i_;
            while (i_ < s_.size() && s_[i_] >= '0' && s_[i_] <= '9') ++i_;
            if (i_ == d) err("bad number");
        };
        if (i_ < s_.size() && s_[i_] == '0') {
            ++i_;
        } else {
            digits();
        }
        if (i_ < s_.size() && s_[i_] == '.') {
            ++i_;
            digits();
        }
        if (i_ < s_.size() && (s_[i_] == 'e' || s_[i_] == 'E')) {
            ++i_;
            if (i_ < s_.size() && (s_[i_] == '+' || s_[i_] == '-')) ++i_;
            digits();
        }
        double v = 0;
        auto r = std::from_chars(s_.data() + b, s_.data() + i_, v);
        if (r.ec == std::errc::result_out_of_range) {
            // overflow to infinity or underflow to zero, as strtod does
            v = std::strtod(std::string(s_.substr(b, i_ - b)).c_str(), nullptr);
        } else if (r.ec != std::errc()) {
            err("bad number");
        }
        return v;
    }
    static void put_utf8(std::string& o, uint32_t cp) {
        if (cp < 0x80) {
            o += char(cp);
        } else if (cp < 0x800) {
            o += char(0xC0 | (cp >> 6));
            o += char(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            o += char(0xE0 | (cp >> 12));
            o += char(0x80 | ((cp >> 6) & 0x3F));
            o += char(0x80 | (cp & 0x3F));
        } else {
            o += char(0xF0 | (cp >> 18));
            o += char(0x80 | ((cp >> 12) & 0x3F));
            o += char(0x80 | ((cp >> 6) & 0x3F));
            o += char(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (i_ + 4 > s_.size()) err("bad escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k) {
            const char c = s_[i_++];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= uint32_t(c - '0');
            else if (c >= 'a' && c <= 'f') v |= uint32_t(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= uint32_t(c - 'A' + 10);
            else err("bad escape");
        }
        return v;
    }
    std::string string() {
        ++i_;  // opening quote
        std::string o;
        while (true) {
            if (i_ >= s_.size()) err("unterminated string");
            const unsigned char c = static_cast<unsigned char>(s_[i_++]);
            if (c == '"') return o;
            if (c < 0x20) err("control character in string");
            if (c != '\\') {
                o += char(c);
                continue;
            }
            if (i_ >= s_.size()) err("bad escape");
            const char e = s_[i_++];
            switch (e) {
                case '"': o += '"'; break;
                case '\\': o += '\\'; break;
                case '/': o += '/'; break;
                case 'b': o += '\b'; break;
                case 'f': o += '\f'; break;
                case 'n': o += '\n'; break;
                case 'r': o += '\r'; break;
                case 't': o += '\t'; break;
                case 'u': {
                    uint32_t cp = hex4();
                    if (cp >= 0xD800 && cp < 0xDC00) {
                        if (!lit("\\u")) err("lone surrogate");
                        const uint32_t lo = hex4();
                        if (lo < 0xDC00 || lo >= 0xE000) err("bad surrogate pair");
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    } else if (cp >= 0xDC00 && cp < 0xE000) {
                        err("lone surrogate");
                    }
                    put_utf8(o, cp);
                    break;
                }
                default: err("bad escape");
            }
        }
    }
    Value array(int depth) {
        ++i_;
        Array a;
        ws();
        if (i_ < s_.size() && s_[i_] == ']') {
            ++i_;
            return Value(std::move(a));
        }
        while (true) {
            ws();
            a.push_back(value(depth + 1));
            ws();
            if (i_ >= s_.size()) err("unterminated array");
            if (s_[i_] == ',') {
                ++i_;
                continue;
            }
            if (s_[i_] == ']') {
                ++i_;
                return Value(std::move(a));
            }
            err("expected , or ]");
        }
    }
    Value object(int depth) {
        ++i_;
        Object o;
        ws();
        if (i_ < s_.size() && s_[i_] == '}') {
            ++i_;
            return Value(std::move(o));
        }
        while (true) {
            ws();
            if (i_ >= s_.size() || s_[i_] != '"') err("expected a key");
            std::string k = string();
            ws();
            if (i_ >= s_.size() || s_[i_] != ':') err("expected :");
            ++i_;
            ws();
            o[k] = value(depth + 1);
            ws();
            if (i_ >= s_.size()) err("unterminated object");
            if (s_[i_] == ',') {
                ++i_;
                continue;
            }
            if (s_[i_] == '}') {
                ++i_;
                return Value(std::move(o));
            }
            err("expected , or }");
        }
    }
};

void write_string(std::string& out, const std::string& s) {
    out += '"';
    for (unsigned char c : s) {
        switch (c) {
            case '"': out += "\\\""; break;
            case '\\': out += "\\\\"; break;
            case '\n': out += "\\n"; break;
            case '\r': out += "\\r"; break;
            case '\t': out += "\\t"; break;
            default:
                if (c < 0x20) {
                    char b[8];
                    std::snprintf(b, sizeof b, "\\u%04x", c);
                    out += b;
                } else {
                    out += char(c);
                }
        }
    }
    out += '"';
}

void write_value(std::string& out, const Value& v) {
    if (v.is_null()) {
        out += "null";
    } else if (v.is_bool()) {
        out += v.as_bool() ? "true" : "false";
    } else if (v.is_number()) {
        const double d = v.as_number();
        if (!std::isfinite(d)) {
            out += "null";
            return;
        }
        char b[32];
        auto r = std::to_chars(b, b + sizeof b, d);
        out.append(b, r.ptr);
    } else if (v.is_string()) {
        write_string(out, v.as_string());
    } else if (v.is_array()) {
        out += '[';
        bool first = true;
        for (const Value& e : v.as_array()) {
            if (!first) out += ',';
            first = false;
            write_value(out, e);
        }
        out += ']';
    } else {
        out += '{';
        bool first = true;
        for (const auto& [k, e] : v.as_object()) {
            if (!first) out += ',';
            first = false;
            write_string(out, k);
            out += ':';
            write_value(out, e);
        }
        out += '}';
    }
}

}  // namespace

Value parse(std::string_view text) { return Reader(text).run(); }

std::string write(const Value& v) {
    std::string s;
    write_value(s, v);
    return s;
}

}  // namespace spkb::json
