// A small JSON reader for pipeline documents and node manifests: objects,
// arrays, strings (with the standard escapes; \u escapes of the Basic
// Multilingual Plane are written as UTF-8), numbers, true / false / null.
// Object members keep their document order.
#pragma once

#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace cpb {
namespace json {

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double n = 0.0;
    std::string s;
    std::vector<Value> a;
    std::vector<std::pair<std::string, Value>> o;

    const Value* get(const char* key) const {
        if (kind != Object) return nullptr;
        for (const auto& kv : o)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    std::string str(const char* key, const std::string& def = std::string()) const {
        const Value* v = get(key);
        return v && v->kind == String ? v->s : def;
    }
    bool is_str() const { return kind == String; }
    bool is_num() const { return kind == Number; }
    bool is_obj() const { return kind == Object; }
    bool is_arr() const { return kind == Array; }
    // The strings of an array member (empty when absent or not an array).
    std::vector<std::string> strings(const char* key) const {
        std::vector<std::string> out;
        const Value* v = get(key);
        if (v && v->kind == Array)
            for (const auto& e : v->a)
                if (e.kind == String) out.push_back(e.s);
        return out;
    }
};

class Parser {
public:
    Parser(const char* text, size_t n) : p_(text), end_(text + n) {}
    // Parses one document; false with error() set on malformed input or
    // trailing characters.
    bool parse(Value* out) {
        skip();
        if (!value(out, 0)) return false;
        skip();
        if (p_ != end_) return fail("trailing characters after the document");
        return true;
    }
    const std::string& error() const { return err_; }

private:
    const char* p_;
    const char* end_;
    std::string err_;

    bool fail(const char* m) {
        if (err_.empty()) err_ = m;
        return false;
    }
    void skip() {
        while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) ++p_;
    }
    bool lit(const char* w) {
        const size_t k = std::strlen(w);
        if ((size_t)(end_ - p_) < k || std::strncmp(p_, w, k) != 0) return fail("invalid literal");
        p_ += k;
        return true;
    }
    static void utf8(unsigned cp, std::string* s) {
        if (cp < 0x80) {
            s->push_back((char)cp);
        } else if (cp < 0x800) {
            s->push_back((char)(0xC0 | (cp >> 6)));
            s->push_back((char)(0x80 | (cp & 0x3F)));
        } else {
            s->push_back((char)(0xE0 | (cp >> 12)));
            s->push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
            s->push_back((char)(0x80 | (cp & 0x3F)));
        }
    }
    bool string(std::string* s) {
        if (p_ >= end_ || *p_ != '"') return fail("expected a string");
        ++p_;
        while (p_ < end_ && *p_ != '"') {
            const char c = *p_++;
            if ((unsigned char)c < 0x20) return fail("control character in a string");
            if (c != '\\') {
                s->push_back(c);
                continue;
            }
            if (p_ >= end_) return fail("unterminated escape");
            const char e = *p_++;
            switch (e) {
                case '"': s->push_back('"'); break;
                case '\\': s->push_back('\\'); break;
                case '/': s->push_back('/'); break;
                case 'b': s->push_back('\b'); break;
                case 'f': s->push_back('\f'); break;
                case 'n': s->push_back('\n'); break;
                case 'r': s->push_back('\r'); break;
                case 't': s->push_back('\t'); break;
                case 'u': {
                    if (end_ - p_ < 4) return fail("short \\u escape");
                    unsigned cp = 0;
                    for (int i = 0; i < 4; ++i) {
                        const char h = *p_++;
                        cp <<= 4;
                        if (h >= '0' && h <= '9') cp |= (unsigned)(h - '0');
                        else if (h >= 'a' && h <= 'f') cp |= (unsigned)(h - 'a' + 10);
                        else if (h >= 'A' && h <= 'F') cp |= (unsigned)(h - 'A' + 10);
                        else return fail("bad \\u escape");
                    }
                    utf8(cp, s);
                    break;
                }
                default: return fail("unknown escape");
            }
        }
        if (p_ >= end_) return fail("unterminated string");
        ++p_;
        return true;
    }
    bool number(double* v) {
        const char* q = p_;
        if (q < end_ && (*q == '-' || *q == '+')) ++q;
        while (q < end_ && ((*q >= '0' && *q <= '9') || *q == '.' || *q == 'e' || *q == 'E' || *q == '-' || *q == '+')) ++q;
        if (q == p_) return fail("expected a value");
        const std::string tok(p_, q);
        char* used = nullptr;
        *v = std::strtod(tok.c_str(), &used);
        if (used == nullptr || *used != '\0') return fail("malformed number");
        p_ = q;
        return true;
    }
    bool value(Value* v, int depth) {
        if (depth > 64) return fail("document nested too deeply");
        skip();
        if (p_ >= end_) return fail("unexpected end of document");
        const char c = *p_;
        if (c == '{') {
            v->kind = Value::Object;
            ++p_;
            skip();
            if (p_ < end_ && *p_ == '}') {
                ++p_;
                return true;
            }
            for (;;) {
                skip();
                std::string k;
                if (!string(&k)) return false;
                skip();
                if (p_ >= end_ || *p_ != ':') return fail("expected ':'");
                ++p_;
                Value m;
                if (!value(&m, depth + 1)) return false;
                v->o.emplace_back(std::move(k), std::move(m));
                skip();
                if (p_ < end_ && *p_ == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < end_ && *p_ == '}') {
                    ++p_;
                    return true;
                }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v->kind = Value::Array;
            ++p_;
            skip();
            if (p_ < end_ && *p_ == ']') {
                ++p_;
                return true;
            }
            for (;;) {
                Value e;
                if (!value(&e, depth + 1)) return false;
                v->a.push_back(std::move(e));
                skip();
                if (p_ < end_ && *p_ == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < end_ && *p_ == ']') {
                    ++p_;
                    return true;
                }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v->kind = Value::String;
            return string(&v->s);
        }
        if (c == 't') {
            v->kind = Value::Bool;
            v->b = true;
            return lit("true");
        }
        if (c == 'f') {
            v->kind = Value::Bool;
            v->b = false;
            return lit("false");
        }
        if (c == 'n') {
            v->kind = Value::Null;
            return lit("null");
        }
        v->kind = Value::Number;
        return number(&v->n);
    }
};

inline bool parse(const char* text, size_t n, Value* out, std::string* error) {
    Parser p(text, n);
    if (p.parse(out)) return true;
    if (error) *error = p.error();
    return false;
}

}  // namespace json
}  // namespace cpb
