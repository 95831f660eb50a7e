// ffb_json.hpp -- a small JSON reader/writer for the render-call boundary.
//
// The boundary speaks JSON: the `fae_call` request (`{"fn": ...}`), the
// `.fae` flame configuration inside it, and the info note it answers with
// (wasm/python/src/lib.rs:1-29).  Objects keep their key order, because the
// reference's per-transform variation order can come from the file.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace ffb {

struct Json;
using JsonPtr = std::shared_ptr<Json>;

struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<JsonPtr> arr;
    std::vector<std::pair<std::string, JsonPtr>> obj;

    const Json* get(const std::string& k) const {
        if (kind != Object) return nullptr;
        for (auto& kv : obj) if (kv.first == k) return kv.second.get();
        return nullptr;
    }
    bool has(const std::string& k) const { return get(k) != nullptr; }
    bool is_num() const { return kind == Number; }
    double number_or(const std::string& k, double d) const {
        const Json* v = get(k);
        return (v && v->kind == Number) ? v->num : d;
    }
    bool bool_or(const std::string& k, bool d) const {
        const Json* v = get(k);
        return (v && v->kind == Bool) ? v->b : d;
    }
    std::string string_or(const std::string& k, const std::string& d) const {
        const Json* v = get(k);
        return (v && v->kind == String) ? v->str : d;
    }
};

class JsonParser {
public:
    explicit JsonParser(const std::string& s) : s_(s), i_(0) {}
    JsonPtr parse() {
        JsonPtr v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string& s_;
    size_t i_;
    [[noreturn]] void fail(const char* what) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "%s at offset %zu", what, i_);
        throw std::runtime_error(buf);
    }
    void ws() { while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\n' || s_[i_] == '\r' || s_[i_] == '\t')) ++i_; }
    bool lit(const char* w) {
        size_t n = std::char_traits<char>::length(w);
        if (s_.compare(i_, n, w) == 0) { i_ += n; return true; }
        return false;
    }
    JsonPtr value() {
        ws();
        if (i_ >= s_.size()) fail("unexpected end of input");
        auto v = std::make_shared<Json>();
        char c = s_[i_];
        if (c == '{') {
            v->kind = Json::Object; ++i_; ws();
            if (i_ < s_.size() && s_[i_] == '}') { ++i_; return v; }
            for (;;) {
                ws();
                if (i_ >= s_.size() || s_[i_] != '"') fail("expected a key");
                std::string k = string();
                ws();
                if (i_ >= s_.size() || s_[i_] != ':') fail("expected ':'");
                ++i_;
                v->obj.emplace_back(std::move(k), value());
                ws();
                if (i_ < s_.size() && s_[i_] == ',') { ++i_; continue; }
                if (i_ < s_.size() && s_[i_] == '}') { ++i_; break; }
                fail("expected ',' or '}'");
            }
        } else if (c == '[') {
            v->kind = Json::Array; ++i_; ws();
            if (i_ < s_.size() && s_[i_] == ']') { ++i_; return v; }
            for (;;) {
                v->arr.push_back(value());
                ws();
                if (i_ < s_.size() && s_[i_] == ',') { ++i_; continue; }
                if (i_ < s_.size() && s_[i_] == ']') { ++i_; break; }
                fail("expected ',' or ']'");
            }
        } else if (c == '"') {
            v->kind = Json::String; v->str = string();
        } else if (lit("true")) { v->kind = Json::Bool; v->b = true; }
        else if (lit("false")) { v->kind = Json::Bool; v->b = false; }
        else if (lit("null")) { v->kind = Json::Null; }
        else {
            size_t st = i_;
            if (s_[i_] == '-' || s_[i_] == '+') ++i_;
            while (i_ < s_.size() && (std::isdigit((unsigned char)s_[i_]) || s_[i_] == '.' || s_[i_] == 'e' || s_[i_] == 'E' || s_[i_] == '-' || s_[i_] == '+')) ++i_;
            if (st == i_) fail("unexpected character");
            std::string t = s_.substr(st, i_ - st);
            char* end = nullptr;
            v->kind = Json::Number;
            v->num = std::strtod(t.c_str(), &end);
            if (!end || *end) fail("bad number");
        }
        return v;
    }
    static void put_utf8(std::string& o, uint32_t cp) {
        if (cp < 0x80) o += (char)cp;
        else if (cp < 0x800) { o += (char)(0xC0 | (cp >> 6)); o += (char)(0x80 | (cp & 0x3F)); }
        else if (cp < 0x10000) { o += (char)(0xE0 | (cp >> 12)); o += (char)(0x80 | ((cp >> 6) & 0x3F)); o += (char)(0x80 | (cp & 0x3F)); }
        else { o += (char)(0xF0 | (cp >> 18)); o += (char)(0x80 | ((cp >> 12) & 0x3F)); o += (char)(0x80 | ((cp >> 6) & 0x3F)); o += (char)(0x80 | (cp & 0x3F)); }
    }
    uint32_t hex4() {
        if (i_ + 4 > s_.size()) fail("bad \\u escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k) {
            char c = s_[i_++];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= c - '0';
            else if (c >= 'a' && c <= 'f') v |= c - 'a' + 10;
            else if (c >= 'A' && c <= 'F') v |= c - 'A' + 10;
            else fail("bad \\u escape");
        }
        return v;
    }
    std::string string() {
        ++i_;  // opening quote
        std::string o;
        while (i_ < s_.size()) {
            char c = s_[i_++];
            if (c == '"') return o;
            if (c != '\\') { o += c; continue; }
            if (i_ >= s_.size()) break;
            char e = s_[i_++];
            switch (e) {
            case '"': o += '"'; break; case '\\': o += '\\'; break; case '/': o += '/'; break;
            case 'b': o += '\b'; break; case 'f': o += '\f'; break; case 'n': o += '\n'; break;
            case 'r': o += '\r'; break; case 't': o += '\t'; break;
            case 'u': {
                uint32_t cp = hex4();
                if (cp >= 0xD800 && cp < 0xDC00 && i_ + 1 < s_.size() && s_[i_] == '\\' && s_[i_ + 1] == 'u') {
                    i_ += 2;
                    uint32_t lo = hex4();
                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                }
                put_utf8(o, cp);
                break;
            }
            default: fail("bad escape");
            }
        }
        fail("unterminated string");
    }
};

inline JsonPtr json_parse(const std::string& s) { return JsonParser(s).parse(); }

// Minimal writer for the info notes.
class JsonWriter {
public:
    JsonWriter& begin() { out_ += '{'; first_.push_back(1); return *this; }
    JsonWriter& end() { out_ += '}'; first_.pop_back(); return *this; }
    JsonWriter& key(const std::string& k) { sep(); out_ += quote(k); out_ += ':'; return *this; }
    JsonWriter& num(const std::string& k, double v) {
        key(k);
        char b[64];
        if (std::isfinite(v) && v == std::floor(v) && std::fabs(v) < 9.0e15) std::snprintf(b, sizeof b, "%.0f", v);
        else if (std::isfinite(v)) std::snprintf(b, sizeof b, "%.17g", v);
        else std::snprintf(b, sizeof b, "null");
        out_ += b; return *this;
    }
    JsonWriter& str(const std::string& k, const std::string& v) { key(k); out_ += quote(v); return *this; }
    JsonWriter& boolean(const std::string& k, bool v) { key(k); out_ += v ? "true" : "false"; return *this; }
    JsonWriter& raw(const std::string& k, const std::string& v) { key(k); out_ += v; return *this; }
    const std::string& s() const { return out_; }
    static std::string quote(const std::string& v) {
        std::string o = "\"";
        for (unsigned char c : v) {
            if (c == '"') o += "\\\""; else if (c == '\\') o += "\\\\";
            else if (c == '\n') o += "\\n"; else if (c < 0x20) { char b[8]; std::snprintf(b, sizeof b, "\\u%04x", c); o += b; }
            else o += (char)c;
        }
        return o + "\"";
    }

private:
    void sep() { if (!first_.empty()) { if (!first_.back()) out_ += ','; first_.back() = 0; } }
    std::string out_;
    std::vector<char> first_;
};

}  // namespace ffb
