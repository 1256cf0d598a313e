// json.hpp -- minimal JSON reader for the reference's case decks.
//
// The reference parses decks with the vendored parson library
// (src/parson.c); only its value model matters here: objects, arrays,
// numbers (read as double, like json_object_get_number), strings, booleans
// and null.  A missing key reads as 0, which is what
// json_object_get_number returns for an absent key.
#pragma once
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace hp {

struct JVal {
    enum Kind { NUL, NUM, STR, BOOL, ARR, OBJ } kind = NUL;
    double num = 0.0;
    bool b = false;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;

    const JVal *get(const std::string &k) const {
        if (kind != OBJ) return nullptr;
        for (auto &kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
    // json_object_get_number semantics: 0 when absent or not a number
    double number(const std::string &k) const {
        const JVal *v = get(k);
        return (v && v->kind == NUM) ? v->num : 0.0;
    }
    const JVal &object(const std::string &k) const {
        static const JVal empty_obj = [] { JVal v; v.kind = OBJ; return v; }();
        const JVal *v = get(k);
        return (v && v->kind == OBJ) ? *v : empty_obj;
    }
    const std::vector<JVal> &array(const std::string &k) const {
        static const std::vector<JVal> empty;
        const JVal *v = get(k);
        return (v && v->kind == ARR) ? v->arr : empty;
    }
    bool has(const std::string &k) const { return get(k) != nullptr; }
};

class JParser {
  public:
    JParser(const char *s, size_t n) : p_(s), e_(s + n) {}
    JVal parse() {
        JVal v = value();
        ws();
        if (p_ != e_) fail("trailing characters");
        return v;
    }

  private:
    const char *p_, *e_;
    [[noreturn]] void fail(const char *what) { throw std::runtime_error(std::string("JSON: ") + what); }
    void ws() {
        while (p_ < e_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) p_++;
    }
    JVal value() {
        ws();
        if (p_ >= e_) fail("unexpected end");
        char c = *p_;
        if (c == '{') return object();
        if (c == '[') return array();
        if (c == '"') { JVal v; v.kind = JVal::STR; v.str = string(); return v; }
        if (c == 't' || c == 'f') return boolean();
        if (c == 'n') { expect("null"); return JVal(); }
        return number();
    }
    void expect(const char *lit) {
        for (const char *q = lit; *q; q++, p_++)
            if (p_ >= e_ || *p_ != *q) fail("bad literal");
    }
    JVal boolean() {
        JVal v; v.kind = JVal::BOOL;
        if (*p_ == 't') { expect("true"); v.b = true; } else { expect("false"); v.b = false; }
        return v;
    }
    JVal number() {
        std::string buf;
        while (p_ < e_ && (isdigit((unsigned char)*p_) || *p_ == '-' || *p_ == '+' || *p_ == '.' || *p_ == 'e' || *p_ == 'E'))
            buf.push_back(*p_++);
        if (buf.empty()) fail("bad value");
        char *end = nullptr;
        double d = strtod(buf.c_str(), &end);
        if (!end || *end) fail("bad number");
        JVal v; v.kind = JVal::NUM; v.num = d;
        return v;
    }
    std::string string() {
        std::string s;
        p_++; // opening quote
        while (p_ < e_ && *p_ != '"') {
            if (*p_ == '\\') {
                p_++;
                if (p_ >= e_) fail("bad escape");
                char c = *p_++;
                switch (c) {
                case 'n': s.push_back('\n'); break;
                case 't': s.push_back('\t'); break;
                case 'r': s.push_back('\r'); break;
                case 'b': s.push_back('\b'); break;
                case 'f': s.push_back('\f'); break;
                case 'u': {
                    if (e_ - p_ < 4) fail("bad \\u");
                    unsigned cp = (unsigned)strtoul(std::string(p_, p_ + 4).c_str(), nullptr, 16);
                    p_ += 4;
                    if (cp < 0x80) s.push_back((char)cp);
                    else if (cp < 0x800) { s.push_back((char)(0xC0 | (cp >> 6))); s.push_back((char)(0x80 | (cp & 0x3F))); }
                    else { s.push_back((char)(0xE0 | (cp >> 12))); s.push_back((char)(0x80 | ((cp >> 6) & 0x3F))); s.push_back((char)(0x80 | (cp & 0x3F))); }
                    break;
                }
                default: s.push_back(c);
                }
            } else {
                s.push_back(*p_++);
            }
        }
        if (p_ >= e_) fail("unterminated string");
        p_++;
        return s;
    }
    JVal array() {
        JVal v; v.kind = JVal::ARR;
        p_++;
        ws();
        if (p_ < e_ && *p_ == ']') { p_++; return v; }
        for (;;) {
            v.arr.push_back(value());
            ws();
            if (p_ >= e_) fail("unterminated array");
            if (*p_ == ',') { p_++; continue; }
            if (*p_ == ']') { p_++; break; }
            fail("expected , or ]");
        }
        return v;
    }
    JVal object() {
        JVal v; v.kind = JVal::OBJ;
        p_++;
        ws();
        if (p_ < e_ && *p_ == '}') { p_++; return v; }
        for (;;) {
            ws();
            if (p_ >= e_ || *p_ != '"') fail("expected key");
            std::string k = string();
            ws();
            if (p_ >= e_ || *p_ != ':') fail("expected :");
            p_++;
            JVal val = value();
            v.obj.emplace_back(std::move(k), std::move(val));
            ws();
            if (p_ >= e_) fail("unterminated object");
            if (*p_ == ',') { p_++; continue; }
            if (*p_ == '}') { p_++; break; }
            fail("expected , or }");
        }
        return v;
    }
};

} // namespace hp
