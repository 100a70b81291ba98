// cl_toml.hpp — the subset of TOML v1.0 that the run files (runs/*.toml) and
// material files (data/*.toml) of CryspLight use; header-only C++17.
//
// Supported: comments, [table] headers (dotted names kept as one string),
// `key = value` with bare or quoted keys, basic and literal strings,
// integers (sign, underscores, 0x/0o/0b), floats (fraction, exponent,
// underscores, inf, nan), booleans, and arrays of those values (nested
// arrays included, spanning lines).  Inline tables, multi-line strings and
// dates are rejected with an error naming the line.
#pragma once

#include <cctype>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace cltoml {

struct Value {
    enum Kind { STR, INT, FLOAT, BOOL, ARRAY } kind = STR;
    std::string s;
    int64_t i = 0;
    double f = 0.0;
    bool b = false;
    std::vector<Value> arr;

    bool is_number() const { return kind == INT || kind == FLOAT; }
    double num() const
    {
        if (kind == INT) return (double)i;
        if (kind == FLOAT) return f;
        throw std::runtime_error("not a number");
    }
};

// table name ("" = root) -> key -> value
using Table = std::map<std::string, Value>;
using Document = std::map<std::string, Table>;

class Parser {
public:
    explicit Parser(std::string text, std::string origin = "") : t_(std::move(text)), origin_(std::move(origin)) {}

    Document parse()
    {
        Document doc;
        doc[""];
        std::string table;
        for (;;) {
            skip_ws_comments_newlines();
            if (p_ >= t_.size()) break;
            if (t_[p_] == '[') {
                ++p_;
                if (p_ < t_.size() && t_[p_] == '[') fail("arrays of tables are not supported");
                skip_ws();
                std::string name = key();
                skip_ws();
                while (p_ < t_.size() && t_[p_] == '.') {
                    ++p_;
                    skip_ws();
                    name += "." + key();
                    skip_ws();
                }
                expect(']');
                end_of_line();
                if (doc.count(name) && !doc[name].empty()) fail("table [" + name + "] defined twice");
                doc[name];
                table = name;
                continue;
            }
            std::string k = key();
            skip_ws();
            if (p_ < t_.size() && t_[p_] == '.') fail("dotted keys are not supported");
            expect('=');
            skip_ws();
            Value v = value();
            end_of_line();
            if (doc[table].count(k)) fail("key '" + k + "' defined twice");
            doc[table][k] = std::move(v);
        }
        return doc;
    }

private:
    std::string t_, origin_;
    size_t p_ = 0;

    int line() const
    {
        int n = 1;
        for (size_t i = 0; i < p_ && i < t_.size(); ++i) n += t_[i] == '\n';
        return n;
    }
    [[noreturn]] void fail(const std::string& what) const
    {
        std::ostringstream o;
        o << (origin_.empty() ? "toml" : origin_) << ":" << line() << ": " << what;
        throw std::runtime_error(o.str());
    }
    void skip_ws()
    {
        while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\t')) ++p_;
    }
    void skip_comment()
    {
        if (p_ < t_.size() && t_[p_] == '#')
            while (p_ < t_.size() && t_[p_] != '\n') ++p_;
    }
    void skip_ws_comments_newlines()
    {
        for (;;) {
            skip_ws();
            skip_comment();
            if (p_ < t_.size() && (t_[p_] == '\n' || t_[p_] == '\r')) { ++p_; continue; }
            break;
        }
    }
    void end_of_line()
    {
        skip_ws();
        skip_comment();
        if (p_ < t_.size() && t_[p_] == '\r') ++p_;
        if (p_ < t_.size() && t_[p_] != '\n') fail("unexpected text after a value");
    }
    void expect(char c)
    {
        if (p_ >= t_.size() || t_[p_] != c) fail(std::string("expected '") + c + "'");
        ++p_;
    }
    std::string key()
    {
        if (p_ < t_.size() && (t_[p_] == '"' || t_[p_] == '\'')) return string_value();
        size_t s = p_;
        while (p_ < t_.size() && (std::isalnum((unsigned char)t_[p_]) || t_[p_] == '_' || t_[p_] == '-')) ++p_;
        if (p_ == s) fail("expected a key");
        return t_.substr(s, p_ - s);
    }
    std::string string_value()
    {
        const char q = t_[p_++];
        if (p_ + 1 < t_.size() && t_[p_] == q && t_[p_ + 1] == q) fail("multi-line strings are not supported");
        std::string out;
        while (p_ < t_.size() && t_[p_] != q) {
            char c = t_[p_++];
            if (c == '\n') fail("unterminated string");
            if (q == '"' && c == '\\') {
                if (p_ >= t_.size()) fail("bad escape");
                const char e = t_[p_++];
                switch (e) {
                case 'n': out += '\n'; break;
                case 't': out += '\t'; break;
                case 'r': out += '\r'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case 'u': case 'U': {
                    const int nd = e == 'u' ? 4 : 8;
                    if (p_ + nd > t_.size()) fail("bad unicode escape");
                    const uint32_t cp = (uint32_t)std::stoul(t_.substr(p_, nd), nullptr, 16);
                    p_ += nd;
                    utf8(out, cp);
                    break;
                }
                default: fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        expect(q);
        return out;
    }
    static void utf8(std::string& o, uint32_t cp)
    {
        if (cp < 0x80) { o += (char)cp; return; }
        if (cp < 0x800) { o += (char)(0xC0 | (cp >> 6)); o += (char)(0x80 | (cp & 0x3F)); return; }
        if (cp < 0x10000) {
            o += (char)(0xE0 | (cp >> 12)); o += (char)(0x80 | ((cp >> 6) & 0x3F)); o += (char)(0x80 | (cp & 0x3F));
            return;
        }
        o += (char)(0xF0 | (cp >> 18)); o += (char)(0x80 | ((cp >> 12) & 0x3F));
        o += (char)(0x80 | ((cp >> 6) & 0x3F)); o += (char)(0x80 | (cp & 0x3F));
    }
    Value value()
    {
        if (p_ >= t_.size()) fail("expected a value");
        Value v;
        const char c = t_[p_];
        if (c == '"' || c == '\'') { v.kind = Value::STR; v.s = string_value(); return v; }
        if (c == '[') {
            ++p_;
            v.kind = Value::ARRAY;
            for (;;) {
                skip_ws_comments_newlines();
                if (p_ < t_.size() && t_[p_] == ']') { ++p_; break; }
                v.arr.push_back(value());
                skip_ws_comments_newlines();
                if (p_ < t_.size() && t_[p_] == ',') { ++p_; continue; }
                skip_ws_comments_newlines();
                expect(']');
                break;
            }
            return v;
        }
        if (c == '{') fail("inline tables are not supported");
        size_t s = p_;
        while (p_ < t_.size() && !std::isspace((unsigned char)t_[p_]) && t_[p_] != ',' && t_[p_] != ']' &&
               t_[p_] != '#')
            ++p_;
        std::string w = t_.substr(s, p_ - s);
        if (w == "true" || w == "false") { v.kind = Value::BOOL; v.b = w == "true"; return v; }
        return number(w);
    }
    Value number(const std::string& w0)
    {
        Value v;
        std::string w;
        for (size_t i = 0; i < w0.size(); ++i) {
            if (w0[i] == '_') {
                if (i == 0 || i + 1 == w0.size() || !std::isalnum((unsigned char)w0[i - 1]) ||
                    !std::isalnum((unsigned char)w0[i + 1]))
                    fail("bad underscore in number '" + w0 + "'");
                continue;
            }
            w += w0[i];
        }
        if (w.empty()) fail("expected a value");
        std::string body = w;
        double sign = 1.0;
        if (body[0] == '+' || body[0] == '-') { sign = body[0] == '-' ? -1.0 : 1.0; body = body.substr(1); }
        if (body == "inf" || body == "nan") {
            v.kind = Value::FLOAT;
            v.f = body == "inf" ? sign * INFINITY : NAN;
            return v;
        }
        if (body.size() > 2 && body[0] == '0' && (body[1] == 'x' || body[1] == 'o' || body[1] == 'b')) {
            if (w[0] == '+' || w[0] == '-') fail("signed prefixed integer '" + w0 + "'");
            const int base = body[1] == 'x' ? 16 : (body[1] == 'o' ? 8 : 2);
            size_t used = 0;
            const unsigned long long u = std::stoull(body.substr(2), &used, base);
            if (used != body.size() - 2 || u > (unsigned long long)INT64_MAX) fail("bad integer '" + w0 + "'");
            v.kind = Value::INT;
            v.i = (int64_t)u;
            return v;
        }
        const bool is_float = w.find_first_of(".eE") != std::string::npos;
        for (char ch : body)
            if (!(std::isdigit((unsigned char)ch) || ch == '.' || ch == 'e' || ch == 'E' || ch == '+' || ch == '-'))
                fail("bad value '" + w0 + "'");
        try {
            size_t used = 0;
            if (is_float) {
                v.kind = Value::FLOAT;
                v.f = std::stod(w, &used);
            } else {
                v.kind = Value::INT;
                v.i = (int64_t)std::stoll(w, &used, 10);
            }
            if (used != w.size()) fail("bad number '" + w0 + "'");
        } catch (const std::logic_error&) {
            fail("bad number '" + w0 + "'");
        }
        return v;
    }
};

inline Document parse_file(const std::string& path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return Parser(ss.str(), path).parse();
}

}  // namespace cltoml
