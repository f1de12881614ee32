#include "json.hpp"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace cgfdm {

static bool ieq(const std::string &a, const char *b)
{
    size_t n = std::strlen(b);
    if (a.size() != n) return false;
    for (size_t i = 0; i < n; i++)
        if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return false;
    return true;
}

const JsonValue *JsonValue::get(const char *key) const
{
    if (kind != Object) return nullptr;
    for (const auto &m : members)
        if (ieq(m.first, key)) return &m.second;
    return nullptr;
}

namespace {

struct Parser {
    const char *p, *end;
    std::string err;

    void ws()
    {
        while (p < end && (unsigned char)*p <= 32) p++;
    }
    bool fail(const char *msg)
    {
        if (err.empty()) err = msg;
        return false;
    }

    // Digit accumulation then one pow(10, e) scaling, as the reference's
    // cJSON does; keeps DT/DH/TMAX bit-identical to what it reads.
    bool number(JsonValue &v)
    {
        double n = 0, sign = 1, scale = 0;
        int subscale = 0, signsub = 1;
        if (p < end && *p == '-') sign = -1, p++;
        if (p < end && *p == '0') p++;
        if (p < end && *p >= '1' && *p <= '9')
            do n = (n * 10.0) + (*p++ - '0');
            while (p < end && *p >= '0' && *p <= '9');
        if (p + 1 < end && *p == '.' && p[1] >= '0' && p[1] <= '9') {
            p++;
            do n = (n * 10.0) + (*p++ - '0'), scale--;
            while (p < end && *p >= '0' && *p <= '9');
        }
        if (p < end && (*p == 'e' || *p == 'E')) {
            p++;
            if (p < end && *p == '+') p++;
            else if (p < end && *p == '-') signsub = -1, p++;
            while (p < end && *p >= '0' && *p <= '9') subscale = (subscale * 10) + (*p++ - '0');
        }
        v.kind = JsonValue::Number;
        v.num = sign * n * std::pow(10.0, (scale + subscale * signsub));
        return true;
    }

    bool string(std::string &s)
    {
        if (p >= end || *p != '"') return fail("expected string");
        p++;
        s.clear();
        while (p < end && *p != '"') {
            if (*p == '\\') {
                p++;
                if (p >= end) return fail("bad escape");
                switch (*p) {
                case 'b': s += '\b'; break;
                case 'f': s += '\f'; break;
                case 'n': s += '\n'; break;
                case 'r': s += '\r'; break;
                case 't': s += '\t'; break;
                case 'u': {
                    if (end - p < 5) return fail("bad \\u escape");
                    unsigned cp = (unsigned)std::strtoul(std::string(p + 1, p + 5).c_str(), nullptr, 16);
                    p += 4;
                    if (cp < 0x80) s += (char)cp;
                    else if (cp < 0x800) s += (char)(0xC0 | (cp >> 6)), s += (char)(0x80 | (cp & 0x3F));
                    else
                        s += (char)(0xE0 | (cp >> 12)), s += (char)(0x80 | ((cp >> 6) & 0x3F)),
                            s += (char)(0x80 | (cp & 0x3F));
                    break;
                }
                default: s += *p;
                }
                p++;
            } else {
                s += *p++;
            }
        }
        if (p >= end) return fail("unterminated string");
        p++;
        return true;
    }

    bool value(JsonValue &v, int depth)
    {
        if (depth > 64) return fail("nesting too deep");
        ws();
        if (p >= end) return fail("unexpected end");
        if (*p == '{') {
            p++;
            v.kind = JsonValue::Object;
            ws();
            if (p < end && *p == '}') return p++, true;
            for (;;) {
                ws();
                std::string k;
                if (!string(k)) return false;
                ws();
                if (p >= end || *p != ':') return fail("expected ':'");
                p++;
                JsonValue child;
                if (!value(child, depth + 1)) return false;
                v.members.emplace_back(std::move(k), std::move(child));
                ws();
                if (p < end && *p == ',') { p++; continue; }
                if (p < end && *p == '}') { p++; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (*p == '[') {
            p++;
            v.kind = JsonValue::Array;
            ws();
            if (p < end && *p == ']') return p++, true;
            for (;;) {
                JsonValue child;
                if (!value(child, depth + 1)) return false;
                v.items.push_back(std::move(child));
                ws();
                if (p < end && *p == ',') { p++; continue; }
                if (p < end && *p == ']') { p++; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (*p == '"') {
            v.kind = JsonValue::String;
            return string(v.str);
        }
        if (*p == '-' || (*p >= '0' && *p <= '9')) return number(v);
        if (end - p >= 4 && !std::strncmp(p, "null", 4)) return p += 4, v.kind = JsonValue::Null, true;
        if (end - p >= 4 && !std::strncmp(p, "true", 4)) return p += 4, v.kind = JsonValue::True, v.num = 1, true;
        if (end - p >= 5 && !std::strncmp(p, "false", 5)) return p += 5, v.kind = JsonValue::False, true;
        return fail("unexpected character");
    }
};

}  // namespace

bool json_parse(const std::string &text, JsonValue &out, std::string &err)
{
    Parser ps{text.data(), text.data() + text.size(), {}};
    out = JsonValue();
    if (!ps.value(out, 0)) {
        char buf[96];
        std::snprintf(buf, sizeof buf, " at byte %ld", (long)(ps.p - text.data()));
        err = ps.err + buf;
        return false;
    }
    return true;
}

bool json_parse_file(const std::string &path, JsonValue &out, std::string &err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    return json_parse(ss.str(), out, err);
}

}  // namespace cgfdm
