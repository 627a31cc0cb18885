#include "json.hpp"

#include <cerrno>
#include <cstdlib>
#include <stdexcept>

namespace dq::json {
namespace {

struct Reader {
    const char* p;
    const char* end;
    const char* begin;
    int depth = 0;

    [[noreturn]] void error(const std::string& what) const {
        throw std::runtime_error(what + " at position " + std::to_string(p - begin));
    }
    void ws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    }
    bool lit(const char* w) {
        const char* q = p;
        for (; *w; ++w, ++q)
            if (q >= end || *q != *w) return false;
        p = q;
        return true;
    }
    static void put_utf8(std::string& out, uint32_t cp) {
        if (cp < 0x80) {
            out += char(cp);
        } else if (cp < 0x800) {
            out += char(0xC0 | (cp >> 6));
            out += char(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += char(0xE0 | (cp >> 12));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        } else {
            out += char(0xF0 | (cp >> 18));
            out += char(0x80 | ((cp >> 12) & 0x3F));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (end - p < 4) error("EOF while parsing a string");
        uint32_t v = 0;
        for (int i = 0; i < 4; i++) {
            char c = *p++;
            v <<= 4;
            if (c >= '0' && c <= '9') v |= uint32_t(c - '0');
            else if (c >= 'a' && c <= 'f') v |= uint32_t(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= uint32_t(c - 'A' + 10);
            else error("invalid escape");
        }
        return v;
    }
    std::string string() {
        // assumes *p == '"'
        p++;
        std::string out;
        while (true) {
            if (p >= end) error("EOF while parsing a string");
            unsigned char c = static_cast<unsigned char>(*p++);
            if (c == '"') break;
            if (c < 0x20) error("control character while parsing a string");
            if (c != '\\') {
                out += char(c);
                continue;
            }
            if (p >= end) error("EOF while parsing a string");
            char e = *p++;
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
                    if (cp >= 0xD800 && cp < 0xDC00) {
                        if (!(end - p >= 2 && p[0] == '\\' && p[1] == 'u')) error("lone leading surrogate");
                        p += 2;
                        uint32_t lo = hex4();
                        if (lo < 0xDC00 || lo >= 0xE000) error("invalid unicode surrogate");
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    } else if (cp >= 0xDC00 && cp < 0xE000) {
                        error("lone trailing surrogate");
                    }
                    put_utf8(out, cp);
                    break;
                }
                default: error("invalid escape");
            }
        }
        return out;
    }
    Value number() {
        const char* start = p;
        bool neg = false;
        if (*p == '-') {
            neg = true;
            p++;
        }
        if (p >= end) error("invalid number");
        if (*p == '0') {
            p++;
        } else if (*p >= '1' && *p <= '9') {
            while (p < end && *p >= '0' && *p <= '9') p++;
        } else {
            error("invalid number");
        }
        bool is_float = false;
        if (p < end && *p == '.') {
            is_float = true;
            p++;
            if (p >= end || !(*p >= '0' && *p <= '9')) error("invalid number");
            while (p < end && *p >= '0' && *p <= '9') p++;
        }
        if (p < end && (*p == 'e' || *p == 'E')) {
            is_float = true;
            p++;
            if (p < end && (*p == '+' || *p == '-')) p++;
            if (p >= end || !(*p >= '0' && *p <= '9')) error("invalid number");
            while (p < end && *p >= '0' && *p <= '9') p++;
        }
        std::string text(start, p);
        Value v;
        v.f = std::strtod(text.c_str(), nullptr);
        if (!is_float) {
            v.type = Type::Int;
            v.negative = neg;
            uint64_t mag = 0;
            bool overflow = false;
            for (const char* q = start + (neg ? 1 : 0); q < p; q++) {
                uint64_t d = uint64_t(*q - '0');
                if (mag > (~uint64_t(0) - d) / 10) overflow = true;
                mag = mag * 10 + d;
            }
            v.u = mag;
            v.int_overflow = overflow;
            if (neg && mag == 0) v.negative = false;  // -0 is the integer 0
        } else {
            v.type = Type::Float;
        }
        return v;
    }
    Value value() {
        ws();
        if (p >= end) error("EOF while parsing a value");
        Value v;
        char c = *p;
        if (c == '{') {
            if (++depth > 128) error("recursion limit exceeded");
            p++;
            v.type = Type::Object;
            ws();
            if (p < end && *p == '}') {
                p++;
                depth--;
                return v;
            }
            while (true) {
                ws();
                if (p >= end || *p != '"') error("key must be a string");
                std::string key = string();
                ws();
                if (p >= end || *p != ':') error("expected `:`");
                p++;
                Value item = value();
                v.obj.emplace_back(std::move(key), std::move(item));
                ws();
                if (p < end && *p == ',') {
                    p++;
                    continue;
                }
                if (p < end && *p == '}') {
                    p++;
                    break;
                }
                error("expected `,` or `}`");
            }
            depth--;
            return v;
        }
        if (c == '[') {
            if (++depth > 128) error("recursion limit exceeded");
            p++;
            v.type = Type::Array;
            ws();
            if (p < end && *p == ']') {
                p++;
                depth--;
                return v;
            }
            while (true) {
                v.arr.push_back(value());
                ws();
                if (p < end && *p == ',') {
                    p++;
                    continue;
                }
                if (p < end && *p == ']') {
                    p++;
                    break;
                }
                error("expected `,` or `]`");
            }
            depth--;
            return v;
        }
        if (c == '"') {
            v.type = Type::String;
            v.s = string();
            return v;
        }
        if (c == '-' || (c >= '0' && c <= '9')) return number();
        if (lit("true")) {
            v.type = Type::Bool;
            v.b = true;
            return v;
        }
        if (lit("false")) {
            v.type = Type::Bool;
            return v;
        }
        if (lit("null")) return v;
        error("expected value");
    }
};

}  // namespace

Value parse(const char* text, size_t len) {
    Reader r{text, text + len, text};
    Value v = r.value();
    r.ws();
    if (r.p != r.end) r.error("trailing characters");
    return v;
}

}  // namespace dq::json
