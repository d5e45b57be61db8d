// Minimal JSON reader for the scene schema.  Accepts // and /* */ comments and
// trailing commas, as the reference's loader does (src/core/json_util.h:12-70).
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace vs {

class Json {
public:
    enum Kind { Null, Bool, Number, String, Array, Object };

    Json() = default;
    static Json number(double v) { Json j; j.kind_ = Number; j.num_ = v; return j; }
    static Json string(std::string s) { Json j; j.kind_ = String; j.str_ = std::move(s); return j; }

    Kind kind() const { return kind_; }
    bool is_null() const { return kind_ == Null; }
    bool is_number() const { return kind_ == Number; }
    bool is_string() const { return kind_ == String; }
    bool is_array() const { return kind_ == Array; }
    bool is_object() const { return kind_ == Object; }
    bool is_bool() const { return kind_ == Bool; }

    size_t size() const { return kind_ == Array ? arr_.size() : (kind_ == Object ? obj_.size() : 0); }
    const Json &operator[](size_t i) const {
        static const Json null_json;
        return (kind_ == Array && i < arr_.size()) ? arr_[i] : null_json;
    }
    const Json &operator[](const std::string &k) const {
        static const Json null_json;
        if (kind_ != Object) return null_json;
        auto it = obj_.find(k);
        return it == obj_.end() ? null_json : it->second;
    }
    bool contains(const std::string &k) const { return kind_ == Object && obj_.count(k) != 0; }
    // Sets (or adds) a member of an object.
    void set(const std::string &k, Json v) {
        if (kind_ != Object) throw std::runtime_error("json: set on a non-object");
        obj_[k] = std::move(v);
    }
    const std::map<std::string, Json> &items() const { return obj_; }
    const std::vector<Json> &elements() const { return arr_; }

    double as_number(double def = 0.0) const {
        if (kind_ == Number) return num_;
        if (kind_ == Bool) return b_ ? 1.0 : 0.0;
        return def;
    }
    float as_float(float def = 0.0f) const { return static_cast<float>(as_number(def)); }
    unsigned as_uint(unsigned def = 0) const { return kind_ == Number ? static_cast<unsigned>(num_) : (kind_ == Bool ? (b_ ? 1u : 0u) : def); }
    int as_int(int def = 0) const { return kind_ == Number ? static_cast<int>(num_) : def; }
    bool as_bool(bool def = false) const {
        if (kind_ == Bool) return b_;
        if (kind_ == Number) return num_ != 0.0;
        return def;
    }
    std::string as_string(const std::string &def = "") const { return kind_ == String ? str_ : def; }
    std::vector<float> as_floats() const {
        std::vector<float> v;
        if (kind_ == Number) v.push_back(static_cast<float>(num_));
        for (const auto &e : arr_) v.push_back(e.as_float());
        return v;
    }

    static Json parse(const std::string &text) {
        Parser p{text, 0};
        p.skip();
        Json j = p.value();
        p.skip();
        if (p.i != text.size()) throw std::runtime_error("json: trailing characters at offset " + std::to_string(p.i));
        return j;
    }

private:
    struct Parser {
        const std::string &s;
        size_t i;
        [[noreturn]] void fail(const char *what) const {
            throw std::runtime_error(std::string("json: ") + what + " at offset " + std::to_string(i));
        }
        void skip() {
            while (i < s.size()) {
                char c = s[i];
                if (c == ' ' || c == '\t' || c == '\n' || c == '\r') { ++i; continue; }
                if (c == '/' && i + 1 < s.size() && s[i + 1] == '/') {
                    while (i < s.size() && s[i] != '\n') ++i;
                    continue;
                }
                if (c == '/' && i + 1 < s.size() && s[i + 1] == '*') {
                    size_t e = s.find("*/", i + 2);
                    if (e == std::string::npos) fail("unterminated comment");
                    i = e + 2;
                    continue;
                }
                break;
            }
        }
        Json value() {
            skip();
            if (i >= s.size()) fail("unexpected end");
            char c = s[i];
            if (c == '{') return object();
            if (c == '[') return array();
            if (c == '"') { Json j; j.kind_ = String; j.str_ = str(); return j; }
            if (s.compare(i, 4, "true") == 0) { i += 4; Json j; j.kind_ = Bool; j.b_ = true; return j; }
            if (s.compare(i, 5, "false") == 0) { i += 5; Json j; j.kind_ = Bool; j.b_ = false; return j; }
            if (s.compare(i, 4, "null") == 0) { i += 4; return Json(); }
            return num();
        }
        std::string str() {
            ++i;
            std::string out;
            while (i < s.size() && s[i] != '"') {
                if (s[i] == '\\' && i + 1 < s.size()) {
                    char e = s[i + 1];
                    out.push_back(e == 'n' ? '\n' : e == 't' ? '\t' : e);
                    i += 2;
                } else {
                    out.push_back(s[i++]);
                }
            }
            if (i >= s.size()) fail("unterminated string");
            ++i;
            return out;
        }
        Json num() {
            size_t st = i;
            if (s[i] == '-' || s[i] == '+') ++i;
            while (i < s.size() && (isdigit(static_cast<unsigned char>(s[i])) || s[i] == '.' || s[i] == 'e' || s[i] == 'E' ||
                                    s[i] == '-' || s[i] == '+'))
                ++i;
            if (st == i) fail("bad value");
            return Json::number(std::stod(s.substr(st, i - st)));
        }
        Json array() {
            Json j;
            j.kind_ = Array;
            ++i;
            while (true) {
                skip();
                if (i >= s.size()) fail("unterminated array");
                if (s[i] == ']') { ++i; break; }
                j.arr_.push_back(value());
                skip();
                if (i < s.size() && s[i] == ',') ++i;
            }
            return j;
        }
        Json object() {
            Json j;
            j.kind_ = Object;
            ++i;
            while (true) {
                skip();
                if (i >= s.size()) fail("unterminated object");
                if (s[i] == '}') { ++i; break; }
                if (s[i] != '"') fail("expected key");
                std::string k = str();
                skip();
                if (i >= s.size() || s[i] != ':') fail("expected ':'");
                ++i;
                j.obj_[k] = value();
                skip();
                if (i < s.size() && s[i] == ',') ++i;
            }
            return j;
        }
    };

    Kind kind_ = Null;
    bool b_ = false;
    double num_ = 0.0;
    std::string str_;
    std::vector<Json> arr_;
    std::map<std::string, Json> obj_;
};

}  // namespace vs
