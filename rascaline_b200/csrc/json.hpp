// Minimal JSON reader for calculator hyper-parameters: objects, arrays,
// strings (with escapes), numbers (integer-ness kept), booleans and null.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace fb200 {
namespace json {

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool boolean = false;
    double number = 0.0;
    bool is_integer = false;
    int64_t integer = 0;
    std::string string;
    std::vector<Value> array;
    std::vector<std::pair<std::string, Value>> object;  // keeps input order

    const Value* get(const std::string& key) const {
        for (auto& kv : object)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    const char* kind_name() const {
        switch (kind) {
            case Null: return "null";
            case Bool: return "boolean";
            case Number: return is_integer ? "integer" : "floating point";
            case String: return "string";
            case Array: return "sequence";
            case Object: return "map";
        }
        return "?";
    }
};

class Parser {
  public:
    explicit Parser(const std::string& s) : s_(s), i_(0) {}

    Value parse() {
        Value v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

  private:
    const std::string& s_;
    size_t i_;

    [[noreturn]] void fail(const std::string& what) {
        size_t line = 1, col = 1;
        for (size_t k = 0; k < i_ && k < s_.size(); k++) {
            if (s_[k] == '\n') { line++; col = 1; } else { col++; }
        }
        throw ParseError(what + " at line " + std::to_string(line) + " column " + std::to_string(col));
    }
    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\n' || s_[i_] == '\t' || s_[i_] == '\r')) i_++;
    }
    bool lit(const char* w) {
        size_t n = 0;
        while (w[n]) n++;
        if (s_.compare(i_, n, w) == 0) { i_ += n; return true; }
        return false;
    }
    Value value() {
        ws();
        if (i_ >= s_.size()) fail("EOF while parsing a value");
        char c = s_[i_];
        Value v;
        if (c == '{') return object();
        if (c == '[') return array();
        if (c == '"') { v.kind = Value::String; v.string = str(); return v; }
        if (lit("true")) { v.kind = Value::Bool; v.boolean = true; return v; }
        if (lit("false")) { v.kind = Value::Bool; v.boolean = false; return v; }
        if (lit("null")) { v.kind = Value::Null; return v; }
        if (c == '-' || (c >= '0' && c <= '9')) return number();
        fail("expected value");
    }
    Value number() {
        size_t start = i_;
        bool integer = true;
        if (s_[i_] == '-') i_++;
        if (i_ >= s_.size() || !(s_[i_] >= '0' && s_[i_] <= '9')) fail("invalid number");
        while (i_ < s_.size() && s_[i_] >= '0' && s_[i_] <= '9') i_++;
        if (i_ < s_.size() && s_[i_] == '.') {
            integer = false;
            i_++;
            if (i_ >= s_.size() || !(s_[i_] >= '0' && s_[i_] <= '9')) fail("invalid number");
            while (i_ < s_.size() && s_[i_] >= '0' && s_[i_] <= '9') i_++;
        }
        if (i_ < s_.size() && (s_[i_] == 'e' || s_[i_] == 'E')) {
            integer = false;
            i_++;
            if (i_ < s_.size() && (s_[i_] == '+' || s_[i_] == '-')) i_++;
            if (i_ >= s_.size() || !(s_[i_] >= '0' && s_[i_] <= '9')) fail("invalid number");
            while (i_ < s_.size() && s_[i_] >= '0' && s_[i_] <= '9') i_++;
        }
        Value v;
        v.kind = Value::Number;
        std::string text = s_.substr(start, i_ - start);
        v.number = std::strtod(text.c_str(), nullptr);
        v.is_integer = integer;
        if (integer) v.integer = std::strtoll(text.c_str(), nullptr, 10);
        return v;
    }
    static void utf8(std::string& out, uint32_t cp) {
        if (cp < 0x80) out += (char)cp;
        else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
        else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18)); out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (i_ + 4 > s_.size()) fail("invalid escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; k++) {
            char h = s_[i_++];
            v <<= 4;
            if (h >= '0' && h <= '9') v |= (uint32_t)(h - '0');
            else if (h >= 'a' && h <= 'f') v |= (uint32_t)(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F') v |= (uint32_t)(h - 'A' + 10);
            else fail("invalid escape");
        }
        return v;
    }
    std::string str() {
        i_++;  // opening quote
        std::string out;
        while (true) {
            if (i_ >= s_.size()) fail("EOF while parsing a string");
            char c = s_[i_++];
            if (c == '"') break;
            if (c == '\\') {
                if (i_ >= s_.size()) fail("EOF while parsing a string");
                char e = s_[i_++];
                switch (e) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        uint32_t cp = hex4();
                        if (cp >= 0xD800 && cp < 0xDC00 && i_ + 1 < s_.size() && s_[i_] == '\\' && s_[i_ + 1] == 'u') {
                            i_ += 2;
                            uint32_t lo = hex4();
                            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                        }
                        utf8(out, cp);
                        break;
                    }
                    default: fail("invalid escape");
                }
            } else if ((unsigned char)c < 0x20) {
                fail("control character while parsing a string");
            } else {
                out += c;
            }
        }
        return out;
    }
    Value array() {
        i_++;
        Value v;
        v.kind = Value::Array;
        ws();
        if (i_ < s_.size() && s_[i_] == ']') { i_++; return v; }
        while (true) {
            v.array.push_back(value());
            ws();
            if (i_ >= s_.size()) fail("EOF while parsing a list");
            if (s_[i_] == ',') { i_++; continue; }
            if (s_[i_] == ']') { i_++; break; }
            fail("expected `,` or `]`");
        }
        return v;
    }
    Value object() {
        i_++;
        Value v;
        v.kind = Value::Object;
        ws();
        if (i_ < s_.size() && s_[i_] == '}') { i_++; return v; }
        while (true) {
            ws();
            if (i_ >= s_.size() || s_[i_] != '"') fail("key must be a string");
            std::string key = str();
            ws();
            if (i_ >= s_.size() || s_[i_] != ':') fail("expected `:`");
            i_++;
            Value item = value();
            for (auto& kv : v.object)
                if (kv.first == key) fail("duplicate field `" + key + "`");
            v.object.emplace_back(key, std::move(item));
            ws();
            if (i_ >= s_.size()) fail("EOF while parsing an object");
            if (s_[i_] == ',') { i_++; continue; }
            if (s_[i_] == '}') { i_++; break; }
            fail("expected `,` or `}`");
        }
        return v;
    }
};

inline Value parse(const std::string& s) { return Parser(s).parse(); }

}  // namespace json
}  // namespace fb200
