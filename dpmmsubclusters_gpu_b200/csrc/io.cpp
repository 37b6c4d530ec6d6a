// io.cpp -- JSON reader (comments allowed) and .npy reader/writer; see io.h.
#include "io.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace dpmm {
namespace io {

static const Json kNull;

const Json& Json::operator[](const std::string& key) const
{
    if (kind != Object) return kNull;
    auto it = obj.find(key);
    return it == obj.end() ? kNull : it->second;
}

const Json& Json::operator[](size_t i) const
{
    if (kind != Array || i >= arr.size()) return kNull;
    return arr[i];
}

double Json::as_double(double dflt) const
{
    if (kind == Number) return num;
    if (kind == Bool) return b ? 1.0 : 0.0;
    return dflt;
}

long long Json::as_int(long long dflt) const
{
    if (kind == Number) return (long long)num;
    if (kind == Bool) return b ? 1 : 0;
    return dflt;
}

bool Json::as_bool(bool dflt) const
{
    if (kind == Bool) return b;
    if (kind == Number) return num != 0;
    return dflt;
}

namespace {
struct Parser {
    const std::string& s;
    size_t i = 0;
    std::string err;
    explicit Parser(const std::string& t) : s(t) {}

    void skip()
    {
        for (;;) {
            while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
            if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/') {
                while (i < s.size() && s[i] != '\n') ++i;
            } else if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '*') {
                size_t e = s.find("*/", i + 2);
                i = e == std::string::npos ? s.size() : e + 2;
            } else {
                return;
            }
        }
    }
    bool fail(const std::string& m)
    {
        if (err.empty()) err = m + " at offset " + std::to_string(i);
        return false;
    }
    bool value(Json& v)
    {
        skip();
        if (i >= s.size()) return fail("unexpected end");
        char c = s[i];
        if (c == '{') return object(v);
        if (c == '[') return array(v);
        if (c == '"') {
            v.kind = Json::String;
            return string(v.str);
        }
        if (s.compare(i, 4, "true") == 0) { v.kind = Json::Bool; v.b = true; i += 4; return true; }
        if (s.compare(i, 5, "false") == 0) { v.kind = Json::Bool; v.b = false; i += 5; return true; }
        if (s.compare(i, 4, "null") == 0) { v.kind = Json::Null; i += 4; return true; }
        return number(v);
    }
    bool string(std::string& out)
    {
        ++i;
        out.clear();
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < s.size()) {
                char e = s[i + 1];
                out += e == 'n' ? '\n' : e == 't' ? '\t' : e;
                i += 2;
            } else {
                out += s[i++];
            }
        }
        if (i >= s.size()) return fail("unterminated string");
        ++i;
        return true;
    }
    bool number(Json& v)
    {
        const char* b = s.c_str() + i;
        char* e = nullptr;
        double d = std::strtod(b, &e);
        if (e == b) return fail("bad value");
        i += (size_t)(e - b);
        v.kind = Json::Number;
        v.num = d;
        return true;
    }
    bool array(Json& v)
    {
        v.kind = Json::Array;
        ++i;
        skip();
        if (i < s.size() && s[i] == ']') { ++i; return true; }
        for (;;) {
            Json e;
            if (!value(e)) return false;
            v.arr.push_back(std::move(e));
            skip();
            if (i < s.size() && s[i] == ',') { ++i; skip(); if (i < s.size() && s[i] == ']') { ++i; return true; } continue; }
            if (i < s.size() && s[i] == ']') { ++i; return true; }
            return fail("expected , or ]");
        }
    }
    bool object(Json& v)
    {
        v.kind = Json::Object;
        ++i;
        skip();
        if (i < s.size() && s[i] == '}') { ++i; return true; }
        for (;;) {
            skip();
            if (i >= s.size() || s[i] != '"') return fail("expected key");
            std::string key;
            if (!string(key)) return false;
            skip();
            if (i >= s.size() || s[i] != ':') return fail("expected :");
            ++i;
            Json e;
            if (!value(e)) return false;
            v.obj[key] = std::move(e);
            skip();
            if (i < s.size() && s[i] == ',') { ++i; skip(); if (i < s.size() && s[i] == '}') { ++i; return true; } continue; }
            if (i < s.size() && s[i] == '}') { ++i; return true; }
            return fail("expected , or }");
        }
    }
};
}  // namespace

bool parse_json(const std::string& text, Json& out, std::string& err)
{
    Parser p(text);
    out = Json();
    if (!p.value(out)) {
        err = p.err;
        return false;
    }
    p.skip();
    if (p.i != text.size()) {
        err = "trailing characters at offset " + std::to_string(p.i);
        return false;
    }
    return true;
}

bool read_file(const std::string& path, std::string& out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

static double bf16_to_double(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

bool read_npy(const std::string& path, std::vector<double>& data, int64_t& rows, int64_t& cols, std::string& err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path; return false; }
    char magic[6];
    f.read(magic, 6);
    if (!f || std::memcmp(magic, "\x93NUMPY", 6) != 0) { err = "not a .npy file"; return false; }
    uint8_t ver[2];
    f.read((char*)ver, 2);
    uint32_t hlen = 0;
    if (ver[0] == 1) {
        uint16_t h16;
        f.read((char*)&h16, 2);
        hlen = h16;
    } else {
        f.read((char*)&hlen, 4);
    }
    std::string header(hlen, ' ');
    f.read(&header[0], hlen);
    if (!f) { err = "truncated header"; return false; }
    auto field = [&](const char* key) -> std::string {
        size_t p = header.find(key);
        if (p == std::string::npos) return "";
        p = header.find(':', p);
        size_t q = p + 1;
        while (q < header.size() && header[q] == ' ') ++q;
        return header.substr(q);
    };
    std::string descr = field("'descr'");
    if (descr.size() < 3 || descr[0] != '\'') { err = "bad descr"; return false; }
    descr = descr.substr(1, descr.find('\'', 1) - 1);
    const bool fortran = field("'fortran_order'").compare(0, 4, "True") == 0;
    std::string shp = field("'shape'");
    if (shp.empty() || shp[0] != '(') { err = "bad shape"; return false; }
    std::vector<int64_t> dims;
    {
        size_t p = 1;
        while (p < shp.size() && shp[p] != ')') {
            while (p < shp.size() && (shp[p] == ' ' || shp[p] == ',')) ++p;
            if (shp[p] == ')') break;
            dims.push_back(std::strtoll(shp.c_str() + p, nullptr, 10));
            while (p < shp.size() && shp[p] != ',' && shp[p] != ')') ++p;
        }
    }
    if (dims.size() == 1) dims.push_back(1);
    if (dims.size() != 2) { err = "expected a 2-D array"; return false; }
    rows = dims[0];
    cols = dims[1];
    const size_t n = (size_t)(rows * cols);
    char endian = descr[0];
    if (endian == '>') { err = "big-endian .npy not supported"; return false; }
    std::string t = descr.substr(1);
    size_t wsize = 0;
    if (t == "f8" || t == "i8" || t == "u8") wsize = 8;
    else if (t == "f4" || t == "i4" || t == "u4") wsize = 4;
    else if (t == "i2" || t == "u2" || t == "V2" || t == "f2") wsize = 2;
    else if (t == "i1" || t == "u1" || t == "b1") wsize = 1;
    if (descr.find("bfloat16") != std::string::npos) { t = "V2"; wsize = 2; }
    if (!wsize) { err = "unsupported dtype " + descr; return false; }
    std::vector<unsigned char> raw(n * wsize);
    f.read((char*)raw.data(), (std::streamsize)raw.size());
    if (!f) { err = "truncated data"; return false; }
    data.resize(n);
    for (size_t e = 0; e < n; ++e) {
        const unsigned char* p = raw.data() + e * wsize;
        double v = 0;
        if (t == "f8") { double d; std::memcpy(&d, p, 8); v = d; }
        else if (t == "f4") { float d; std::memcpy(&d, p, 4); v = d; }
        else if (t == "i8") { int64_t d; std::memcpy(&d, p, 8); v = (double)d; }
        else if (t == "u8") { uint64_t d; std::memcpy(&d, p, 8); v = (double)d; }
        else if (t == "i4") { int32_t d; std::memcpy(&d, p, 4); v = d; }
        else if (t == "u4") { uint32_t d; std::memcpy(&d, p, 4); v = d; }
        else if (t == "i2") { int16_t d; std::memcpy(&d, p, 2); v = d; }
        else if (t == "u2") { uint16_t d; std::memcpy(&d, p, 2); v = d; }
        else if (t == "V2") { uint16_t d; std::memcpy(&d, p, 2); v = bf16_to_double(d); }
        else if (t == "f2") {
            uint16_t h; std::memcpy(&h, p, 2);
            int ex = (h >> 10) & 0x1f, mant = h & 0x3ff;
            double m = ex == 0 ? mant / 1024.0 * std::pow(2.0, -14) : (1 + mant / 1024.0) * std::pow(2.0, ex - 15);
            v = (h & 0x8000) ? -m : m;
        }
        else if (t == "i1") v = (int8_t)p[0];
        else v = p[0];
        // Fortran order: element e is (e % rows, e / rows)
        size_t dst = fortran ? (size_t)(e % rows) * cols + e / rows : e;
        data[dst] = v;
    }
    return true;
}

static bool write_npy_raw(const std::string& path, const void* data, size_t bytes, const char* descr, int64_t rows,
                          int64_t cols)
{
    std::string header = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (" +
                         std::to_string(rows) + ", " + std::to_string(cols) + "), }";
    size_t total = 10 + header.size() + 1;
    size_t pad = (64 - total % 64) % 64;
    header += std::string(pad, ' ') + "\n";
    std::ofstream f(path, std::ios::binary);
    if (!f) return false;
    f.write("\x93NUMPY\x01\x00", 8);
    uint16_t hl = (uint16_t)header.size();
    f.write((const char*)&hl, 2);
    f.write(header.data(), (std::streamsize)header.size());
    f.write((const char*)data, (std::streamsize)bytes);
    return (bool)f;
}

bool write_npy_f64(const std::string& path, const double* data, int64_t rows, int64_t cols)
{
    return write_npy_raw(path, data, sizeof(double) * rows * cols, "<f8", rows, cols);
}

bool write_npy_i32(const std::string& path, const int32_t* data, int64_t rows, int64_t cols)
{
    return write_npy_raw(path, data, sizeof(int32_t) * rows * cols, "<i4", rows, cols);
}

}  // namespace io
}  // namespace dpmm
