// Minimal JSON reader and writer helpers for the PGM IO module: the whole document is parsed
// into a tree of Json values (null, bool, number, string, array, object with keys in file
// order).  Numbers are doubles (strtod); strings support the standard escapes, \uXXXX up to
// U+FFFF encoded as UTF-8.  Errors throw std::runtime_error with the byte offset.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>
#include <vector>

namespace gapb200::json {

struct Json {
    enum class Kind { Null, Bool, Number, String, Array, Object };
    Kind kind = Kind::Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    bool is_object() const { return kind == Kind::Object; }
    bool is_array() const { return kind == Kind::Array; }
    bool is_number() const { return kind == Kind::Number; }
    // member lookup (first match); nullptr when absent or not an object
    const Json* get(std::string_view key) const {
        if (kind != Kind::Object) return nullptr;
        for (auto const& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    bool has(std::string_view key) const {
        const Json* v = get(key);
        return v && v->kind != Kind::Null;
    }
    // numeric member (booleans count as 0 / 1); `dflt` when absent or null
    double number(std::string_view key, double dflt) const {
        const Json* v = get(key);
        if (!v || v->kind == Kind::Null) return dflt;
        if (v->kind == Kind::Bool) return v->b ? 1.0 : 0.0;
        if (v->kind != Kind::Number)
            throw std::runtime_error("JSON member '" + std::string(key) + "' is not a number");
        return v->num;
    }
    double required(std::string_view key) const {
        const Json* v = get(key);
        if (!v || v->kind != Kind::Number)
            throw std::runtime_error("JSON member '" + std::string(key) + "' missing or not a number");
        return v->num;
    }
};

class Parser {
  public:
    explicit Parser(std::string_view text) : p_(text.data()), b_(text.data()), e_(text.data() + text.size()) {}

    Json parse() {
        Json v = value();
        ws();
        if (p_ != e_) fail("trailing characters");
        return v;
    }

  private:
    const char* p_;
    const char* b_;
    const char* e_;

    [[noreturn]] void fail(const char* what) const {
        throw std::runtime_error(std::string("JSON parse error at byte ") +
                                 std::to_string(p_ - b_) + ": " + what);
    }
    void ws() {
        while (p_ < e_ && (*p_ == ' ' || *p_ == '\n' || *p_ == '\r' || *p_ == '\t')) ++p_;
    }
    bool lit(const char* s) {
        const size_t n = std::strlen(s);
        if (static_cast<size_t>(e_ - p_) >= n && std::memcmp(p_, s, n) == 0) {
            p_ += n;
            return true;
        }
        return false;
    }
    Json value() {
        ws();
        if (p_ >= e_) fail("unexpected end");
        Json v;
        const char c = *p_;
        if (c == '{') {
            v.kind = Json::Kind::Object;
            ++p_;
            ws();
            if (p_ < e_ && *p_ == '}') {
                ++p_;
                return v;
            }
            for (;;) {
                ws();
                if (p_ >= e_ || *p_ != '"') fail("object key expected");
                std::string key = string();
                ws();
                if (p_ >= e_ || *p_ != ':') fail("':' expected");
                ++p_;
                v.obj.emplace_back(std::move(key), value());
                ws();
                if (p_ < e_ && *p_ == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < e_ && *p_ == '}') {
                    ++p_;
                    return v;
                }
                fail("',' or '}' expected");
            }
        }
        if (c == '[') {
            v.kind = Json::Kind::Array;
            ++p_;
            ws();
            if (p_ < e_ && *p_ == ']') {
                ++p_;
                return v;
            }
            for (;;) {
                v.arr.push_back(value());
                ws();
                if (p_ < e_ && *p_ == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < e_ && *p_ == ']') {
                    ++p_;
                    return v;
                }
                fail("',' or ']' expected");
            }
        }
        if (c == '"') {
            v.kind = Json::Kind::String;
            v.str = string();
            return v;
        }
        if (lit("true")) {
            v.kind = Json::Kind::Bool;
            v.b = true;
            return v;
        }
        if (lit("false")) {
            v.kind = Json::Kind::Bool;
            return v;
        }
        if (lit("null")) return v;
        // number
        std::string buf;
        while (p_ < e_ && *p_ != '\0' && (std::strchr("+-.eE", *p_) || (*p_ >= '0' && *p_ <= '9')))
            buf += *p_++;
        if (buf.empty()) fail("value expected");
        char* end = nullptr;
        v.kind = Json::Kind::Number;
        v.num = std::strtod(buf.c_str(), &end);
        if (!end || *end != '\0') fail("bad number");
        return v;
    }
    std::string string() {
        ++p_;  // opening quote
        std::string out;
        while (p_ < e_ && *p_ != '"') {
            char c = *p_++;
            if (c != '\\') {
                out += c;
                continue;
            }
            if (p_ >= e_) fail("bad escape");
            c = *p_++;
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
                    if (e_ - p_ < 4) fail("bad \\u escape");
                    const unsigned cp = static_cast<unsigned>(std::strtoul(std::string(p_, 4).c_str(), nullptr, 16));
                    p_ += 4;
                    if (cp < 0x80) {
                        out += static_cast<char>(cp);
                    } else if (cp < 0x800) {
                        out += static_cast<char>(0xC0 | (cp >> 6));
                        out += static_cast<char>(0x80 | (cp & 0x3F));
                    } else {
                        out += static_cast<char>(0xE0 | (cp >> 12));
                        out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F));
                        out += static_cast<char>(0x80 | (cp & 0x3F));
                    }
                    break;
                }
                default: fail("bad escape");
            }
        }
        if (p_ >= e_) fail("unterminated string");
        ++p_;
        return out;
    }
};

inline Json parse(std::string_view text) { return Parser(text).parse(); }

// Shortest round-trip decimal form of a double ("%.17g" then trimmed by re-parsing).
inline std::string number(double x) {
    char buf[40];
    for (int prec = 15; prec <= 17; ++prec) {
        std::snprintf(buf, sizeof(buf), "%.*g", prec, x);
        if (std::strtod(buf, nullptr) == x) break;
    }
    return buf;
}

}  // namespace gapb200::json
