// scene_io.cpp -- scene.json loader and writer, the binary scene file, PNG and
// Radiance HDR output.
//
// Loader: drop-in for LoadSceneJSON (reference src/scene_loader.cpp:26-138)
// with the same schema (version 1; camera, sun, lights[], materials[],
// triangles[]), the same number conversion (a JSON integer converts to float
// directly, a JSON real is read as double then narrowed to float, as
// nlohmann::json's get<float>() does) and the same messages.  It is a
// schema-driven parser over the file bytes instead of a DOM.  The triangle
// array is parsed by several host threads at once, each from a guessed
// element boundary in its share of the bytes, the guesses checked to chain
// (parse_triangles_speculative); when they do not, the top level is scanned
// once recording each element's offset and the elements are then parsed in
// parallel from those offsets.  Where the
// reference lets nlohmann throw out of LoadSceneJSON on a missing key (the
// process terminates), this loader prints "[scene] ..." and returns false.
// Which documents load follows the reference's nlohmann::json read with
// `f >> j`: a leading UTF-8 byte-order mark is skipped, nothing after the
// top-level object is read, members the schema does not use are checked for
// syntax as they are skipped, strings must be well-formed UTF-8, and a number
// whose double overflows fails the load.
// A file that begins with the binary scene magic ("LGSCENE1", layout below)
// is read as a binary scene instead: same content, no text parsing.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include "bvh.h"
#include "common.h"
#include "scene.h"

namespace lg
{
namespace
{
// Sizes (or reserves) a triangle array for n records.  The storage is allocated first and,
// for its whole 2 MB-aligned stretches, the kernel is asked for transparent
// huge pages before the records are written: the first write to fresh memory
// then takes one page fault per 2 MB instead of one per 4 KB.  A scene of a
// million triangles is 105 MB; faulting it in 4 KB pages cost more than
// parsing its binary file.  The advice is a hint; without huge pages nothing
// changes.
void reserve_triangles(std::vector<Triangle>& v, size_t n)
{
    if (n <= v.capacity()) return;
    std::vector<Triangle>().swap(v);
    v.reserve(n);
#ifdef MADV_HUGEPAGE
    const uintptr_t huge = (uintptr_t)2 << 20;
    const uintptr_t a = (reinterpret_cast<uintptr_t>(v.data()) + huge - 1) & ~(huge - 1);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(v.data()) + n * sizeof(Triangle)) & ~(huge - 1);
    if (e > a) ::madvise(reinterpret_cast<void*>(a), e - a, MADV_HUGEPAGE);
#endif
}
// n default-valued records (Triangle{}: zero vertices, normals and uvs,
// material 0).  The value-initialisation writes every page once on the
// calling thread, which is where the huge-page hint above pays.
void size_triangles(std::vector<Triangle>& v, size_t n)
{
    reserve_triangles(v, n);
    v.clear();
    v.resize(n);
}

// Copies n triangle records with up to 16 host threads (the pages are
// already faulted in by size_triangles; the threads split the copy itself).
void copy_triangles(Triangle* dst, const void* src, size_t n)
{
    const size_t bytes = n * sizeof(Triangle);
    int nt = (int)std::min<size_t>(16, std::max<size_t>(1, std::thread::hardware_concurrency()));
    if (bytes < ((size_t)8 << 20)) nt = 1;
    if (nt == 1)
    {
        if (bytes) std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> pool;
    for (int k = 0; k < nt; ++k)
        pool.emplace_back([=] {
            const size_t a = n * (size_t)k / (size_t)nt, b = n * (size_t)(k + 1) / (size_t)nt;
            std::memcpy(dst + a, static_cast<const Triangle*>(src) + a, (b - a) * sizeof(Triangle));
        });
    for (auto& t : pool) t.join();
}

struct ParseError
{
    std::string msg;
};

// A cursor over a byte range of the document.
struct Cursor
{
    const char* beg;
    const char* p;
    const char* end;

    [[noreturn]] void fail(const char* what) const
    {
        char buf[256];
        std::snprintf(buf, sizeof buf, "syntax error at byte %lld: %s", (long long)(p - beg), what);
        throw ParseError{buf};
    }
    void ws()
    {
        while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    }
    char peek()
    {
        ws();
        if (p >= end) fail("unexpected end of input");
        return *p;
    }
    void expect(char c)
    {
        if (peek() != c)
        {
            char m[48];
            std::snprintf(m, sizeof m, "expected '%c'", c);
            fail(m);
        }
        ++p;
    }
    bool literal(const char* lit)
    {
        size_t n = std::strlen(lit);
        if ((size_t)(end - p) >= n && std::memcmp(p, lit, n) == 0) { p += n; return true; }
        return false;
    }

    static void put_utf8(std::string& s, uint32_t cp)
    {
        if (cp < 0x80) s += (char)cp;
        else if (cp < 0x800) { s += (char)(0xC0 | (cp >> 6)); s += (char)(0x80 | (cp & 0x3F)); }
        else if (cp < 0x10000)
        {
            s += (char)(0xE0 | (cp >> 12)); s += (char)(0x80 | ((cp >> 6) & 0x3F)); s += (char)(0x80 | (cp & 0x3F));
        }
        else
        {
            s += (char)(0xF0 | (cp >> 18)); s += (char)(0x80 | ((cp >> 12) & 0x3F));
            s += (char)(0x80 | ((cp >> 6) & 0x3F)); s += (char)(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4()
    {
        if (end - p < 4) fail("truncated \\u escape");
        uint32_t v = 0;
        for (int i = 0; i < 4; ++i)
        {
            char c = *p++;
            v <<= 4;
            if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
            else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
            else fail("bad \\u escape");
        }
        return v;
    }
    // A multi-byte UTF-8 sequence whose lead byte b0 was just read: the
    // well-formed sequences of RFC 3629 (no overlong forms, no UTF-16
    // surrogates, nothing above U+10FFFF), which nlohmann::json's lexer
    // accepts and no others.  Appends the sequence to s.
    void utf8_tail(unsigned char b0, std::string& s)
    {
        int n;
        unsigned char lo = 0x80, hi = 0xBF;  // range of the second byte
        if (b0 >= 0xC2 && b0 <= 0xDF) n = 1;
        else if (b0 == 0xE0) { n = 2; lo = 0xA0; }
        else if (b0 >= 0xE1 && b0 <= 0xEC) n = 2;
        else if (b0 == 0xED) { n = 2; hi = 0x9F; }
        else if (b0 >= 0xEE && b0 <= 0xEF) n = 2;
        else if (b0 == 0xF0) { n = 3; lo = 0x90; }
        else if (b0 >= 0xF1 && b0 <= 0xF3) n = 3;
        else if (b0 == 0xF4) { n = 3; hi = 0x8F; }
        else { --p; fail("ill-formed UTF-8 byte"); }
        s += (char)b0;
        for (int i = 0; i < n; ++i)
        {
            if (p >= end) fail("unterminated string");
            const unsigned char b = (unsigned char)*p;
            if (b < (i ? 0x80 : lo) || b > (i ? 0xBF : hi)) fail("ill-formed UTF-8 byte");
            s += (char)b;
            ++p;
        }
    }
    std::string string()
    {
        expect('"');
        std::string s;
        for (;;)
        {
            if (p >= end) fail("unterminated string");
            char c = *p++;
            if (c == '"') break;
            if ((unsigned char)c < 0x20) fail("control character in string");
            if ((unsigned char)c >= 0x80) { utf8_tail((unsigned char)c, s); continue; }
            if (c != '\\') { s += c; continue; }
            if (p >= end) fail("unterminated escape");
            char e = *p++;
            switch (e)
            {
            case '"': s += '"'; break;
            case '\\': s += '\\'; break;
            case '/': s += '/'; break;
            case 'b': s += '\b'; break;
            case 'f': s += '\f'; break;
            case 'n': s += '\n'; break;
            case 'r': s += '\r'; break;
            case 't': s += '\t'; break;
            case 'u':
            {
                uint32_t cp = hex4();
                if (cp >= 0xD800 && cp <= 0xDBFF)
                {
                    if (!literal("\\u")) fail("unpaired surrogate");
                    uint32_t lo = hex4();
                    if (lo < 0xDC00 || lo > 0xDFFF) fail("bad surrogate pair");
                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                }
                else if (cp >= 0xDC00 && cp <= 0xDFFF) fail("unpaired surrogate");
                put_utf8(s, cp);
                break;
            }
            default: fail("bad escape");
            }
        }
        return s;
    }
    // A JSON number token; sets is_int when it has no fraction or exponent.
    void number_token(const char*& tb, const char*& te, bool& is_int)
    {
        ws();
        tb = p;
        is_int = true;
        if (p < end && *p == '-') ++p;
        if (p >= end) fail("bad number");
        if (*p == '0') ++p;
        else if (*p >= '1' && *p <= '9') { while (p < end && *p >= '0' && *p <= '9') ++p; }
        else fail("bad number");
        if (p < end && *p == '.')
        {
            is_int = false;
            ++p;
            if (p >= end || !(*p >= '0' && *p <= '9')) fail("bad number");
            while (p < end && *p >= '0' && *p <= '9') ++p;
        }
        if (p < end && (*p == 'e' || *p == 'E'))
        {
            is_int = false;
            ++p;
            if (p < end && (*p == '+' || *p == '-')) ++p;
            if (p >= end || !(*p >= '0' && *p <= '9')) fail("bad number");
            while (p < end && *p >= '0' && *p <= '9') ++p;
        }
        te = p;
    }
    // nlohmann::json rejects a number whose double is not finite (an
    // exponent past 1e308, or an integer of more than 308 digits that it
    // reads as a double) with this error, wherever the number stands.
    [[noreturn]] static void overflow(const char* tb, const char* te)
    {
        throw ParseError{"[json.exception.out_of_range.406] number overflow parsing '" + std::string(tb, te) + "'"};
    }
    // The overflow check of a number that is not converted (a skipped value).
    static void check_finite(const char* tb, const char* te)
    {
        if (te - tb < 300 && !std::memchr(tb, 'e', (size_t)(te - tb)) && !std::memchr(tb, 'E', (size_t)(te - tb)))
            return;  // under 300 characters without an exponent: below 1e300
        if (!std::isfinite(std::strtod(std::string(tb, te).c_str(), nullptr))) overflow(tb, te);
    }
    // nlohmann get<float>(): integer -> (float)int64, real -> (float)strtod.
    float real()
    {
        const char *tb, *te;
        bool is_int;
        if (peek() != '-' && !(*p >= '0' && *p <= '9')) fail("expected a number");
        number_token(tb, te, is_int);
        if (is_int)
        {
            if (*tb == '-')
            {
                int64_t v;
                auto r = std::from_chars(tb, te, v);
                if (r.ec == std::errc()) return (float)v;
            }
            else
            {
                uint64_t v;
                auto r = std::from_chars(tb, te, v);
                if (r.ec == std::errc()) return (float)v;
            }
        }
        double d;
        auto r = std::from_chars(tb, te, d);
        if (r.ec == std::errc::result_out_of_range) d = std::strtod(std::string(tb, te).c_str(), nullptr);
        else if (r.ec != std::errc()) fail("bad number");
        if (!std::isfinite(d)) overflow(tb, te);
        return (float)d;
    }
    // nlohmann get<int>(): integer -> (int)int64, real -> (int)double.
    int integer()
    {
        const char *tb, *te;
        bool is_int;
        if (peek() != '-' && !(*p >= '0' && *p <= '9')) fail("expected a number");
        number_token(tb, te, is_int);
        if (is_int)
        {
            int64_t v;
            auto r = std::from_chars(tb, te, v);
            if (r.ec == std::errc()) return (int)v;
            uint64_t u;  // nlohmann keeps integers up to 2^64 - 1 as unsigned
            r = std::from_chars(tb, te, u);
            if (r.ec == std::errc()) return (int)u;
        }
        double d = std::strtod(std::string(tb, te).c_str(), nullptr);
        if (!std::isfinite(d)) overflow(tb, te);
        return (int)d;
    }
    // Skips one value, checking its syntax as nlohmann's parser does (an
    // explicit stack of the open containers, so nesting depth is unbounded).
    void skip_checked()
    {
        std::vector<char> open;
        for (;;)
        {
            const char c = peek();
            if (c == '{' || c == '[')
            {
                ++p;
                if (peek() == (c == '{' ? '}' : ']')) ++p;
                else
                {
                    open.push_back(c);
                    if (c == '{')
                    {
                        string();
                        expect(':');
                    }
                    continue;
                }
            }
            else scalar();
            // after a value: close containers, or go on to the next member or element
            for (;;)
            {
                if (open.empty()) return;
                const char d = peek();
                if (d == ',')
                {
                    ++p;
                    if (open.back() == '{')
                    {
                        string();
                        expect(':');
                    }
                    break;
                }
                if (d == (open.back() == '{' ? '}' : ']'))
                {
                    ++p;
                    open.pop_back();
                    continue;
                }
                fail(open.back() == '{' ? "expected ',' or '}'" : "expected ',' or ']'");
            }
        }
    }
    // A string, literal or number (checked for overflow).
    void scalar()
    {
        const char c = peek();
        if (c == '"') { string(); return; }
        if (c == 't') { if (!literal("true")) fail("bad literal"); return; }
        if (c == 'f') { if (!literal("false")) fail("bad literal"); return; }
        if (c == 'n') { if (!literal("null")) fail("bad literal"); return; }
        const char *tb, *te;
        bool is_int;
        number_token(tb, te, is_int);
        check_finite(tb, te);
    }
    // Skips one value.  When starts != null and the value is an array, the
    // offset of each element is appended (used for the triangle array, whose
    // elements are then parsed, and so checked, one by one); any other value
    // is checked as it is skipped.
    void skip(std::vector<const char*>* starts = nullptr)
    {
        if (!starts)
        {
            skip_checked();
            return;
        }
        char c = peek();
        if (c == '{' || c == '[')
        {
            // Iterative structural scan; strings are skipped with their escapes.
            int depth = 0;
            const bool record = starts && c == '[';
            const char* q = p;
            for (;;)
            {
                if (q >= end) { p = q; fail("unterminated container"); }
                char ch = *q;
                if (ch == '"')
                {
                    ++q;
                    while (q < end && *q != '"') q += (*q == '\\') ? 2 : 1;
                    if (q >= end) { p = q; fail("unterminated string"); }
                    ++q;
                    continue;
                }
                if (ch == '{' || ch == '[')
                {
                    ++depth;
                    ++q;
                    if (record && depth == 1)
                    {
                        const char* r = q;
                        while (r < end && (*r == ' ' || *r == '\n' || *r == '\r' || *r == '\t')) ++r;
                        if (r < end && *r != ']') starts->push_back(r);
                    }
                    continue;
                }
                if (ch == '}' || ch == ']')
                {
                    --depth;
                    ++q;
                    if (depth == 0) break;
                    continue;
                }
                if (record && depth == 1 && ch == ',')
                {
                    ++q;
                    while (q < end && (*q == ' ' || *q == '\n' || *q == '\r' || *q == '\t')) ++q;
                    starts->push_back(q);
                    continue;
                }
                ++q;
            }
            p = q;
            return;
        }
        scalar();
    }
};

// Object member iteration: calls fn(key, cursor) for each member.
template <class F>
void for_members(Cursor& c, F&& fn)
{
    c.expect('{');
    if (c.peek() == '}') { ++c.p; return; }
    for (;;)
    {
        std::string key = c.string();
        c.expect(':');
        fn(key, c);
        char d = c.peek();
        ++c.p;
        if (d == '}') return;
        if (d != ',') { --c.p; c.fail("expected ',' or '}'"); }
    }
}
template <class F>
void for_elements(Cursor& c, F&& fn)
{
    c.expect('[');
    if (c.peek() == ']') { ++c.p; return; }
    for (;;)
    {
        fn(c);
        char d = c.peek();
        ++c.p;
        if (d == ']') return;
        if (d != ',') { --c.p; c.fail("expected ',' or ']'"); }
    }
}

// Where an object stands for the lights, materials or triangles array, the
// reference's range-for over the json value visits the object's values in the
// order its std::map keeps them: by key, compared byte by byte, with the last
// of equal keys kept.  Returns the start of each such value; `c` ends after
// the object.
std::vector<const char*> object_values_in_key_order(Cursor& c)
{
    std::vector<std::pair<std::string, const char*>> m;
    for_members(c, [&](const std::string& k, Cursor& v) {
        v.ws();
        m.emplace_back(k, v.p);
        v.skip();
    });
    std::stable_sort(m.begin(), m.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<const char*> out;
    for (size_t i = 0; i < m.size(); ++i)
        if (i + 1 == m.size() || m[i + 1].first != m[i].first) out.push_back(m[i].second);
    return out;
}
// The elements of a lights or materials value as the reference's range-for
// visits them: an array's elements, an object's values in key order, none for
// null.
template <class F>
void for_values(Cursor& c, F&& fn)
{
    const char ch = c.peek();
    if (ch == 'n')
    {
        if (!c.literal("null")) c.fail("bad literal");
        return;
    }
    if (ch != '{')
    {
        for_elements(c, fn);
        return;
    }
    const std::vector<const char*> vals = object_values_in_key_order(c);
    for (const char* v : vals)
    {
        Cursor e{c.beg, v, c.end};
        fn(e);
    }
}

// Reads a JSON array of exactly `n` numbers (the reference reads j[0..n-1];
// extra elements are ignored, missing ones are an error).
void read_floats(Cursor& c, float* out, int n)
{
    int i = 0;
    for_elements(c, [&](Cursor& e) {
        if (i < n) out[i] = e.real();
        else e.skip();
        ++i;
    });
    if (i < n) c.fail("array too short");
}

struct Span
{
    const char* p = nullptr;
    const char* end = nullptr;
    bool present() const { return p != nullptr; }
};

[[noreturn]] void missing(const char* what) { throw ParseError{std::string("missing key \"") + what + "\""}; }

void parse_triangle(Cursor& c, Triangle& t)
{
    bool hv = false, hn = false, huv = false, hm = false;
    for_members(c, [&](const std::string& k, Cursor& v) {
        if (k == "v" || k == "n" || k == "uv")
        {
            const int dim = (k == "uv") ? 2 : 3;
            int i = 0;
            for_elements(v, [&](Cursor& e) {
                if (i < 3)
                {
                    float* dst = (k == "v") ? t.v[i] : (k == "n") ? t.n[i] : t.uv[i];
                    read_floats(e, dst, dim);
                }
                else e.skip();
                ++i;
            });
            if (i < 3) v.fail("vertex array too short");
            (k == "v" ? hv : k == "n" ? hn : huv) = true;
        }
        else if (k == "mat") { t.material = v.integer(); hm = true; }
        else v.skip();
    });
    if (!hv) missing("v");
    if (!hn) missing("n");
    if (!huv) missing("uv");
    if (!hm) missing("mat");
}

// The triangle array parsed by several threads without a serial pre-scan.
// The bytes from the array's '[' to the end of the file are cut into equal
// shares; share 0 starts at the array, every other share at the first '{'
// at or after its cut (a guessed element start), and each parses whole
// elements until the next element would start in the following share or the
// array closes.  The guesses are accepted only if every share begins exactly
// where the previous one stopped, so by induction from share 0 each share
// parsed the true elements and the result equals a serial parse.  Returns
// false, leaving `c` and `out` untouched, when a guess does not chain or a
// share meets a parse error; the caller then takes the serial path (which
// also produces the reference's error message).
bool parse_triangles_speculative(Cursor& c, std::vector<Triangle>& out, int nt)
{
    struct Share
    {
        const char* first = nullptr;  // first element start parsed (or guessed)
        const char* next = nullptr;   // element start where the share stopped
        const char* close = nullptr;  // just past ']' when the array ended here
        std::vector<Triangle> tris;
        bool bad = false;
    };
    const char* b = c.p;
    const size_t bytes = (size_t)(c.end - b);
    std::vector<const char*> cut((size_t)nt + 1);
    for (int k = 0; k <= nt; ++k) cut[(size_t)k] = b + bytes * (size_t)k / (size_t)nt;
    std::vector<Share> sh((size_t)nt);
    auto work = [&](int k) {
        Share& s = sh[(size_t)k];
        const char* hi = cut[(size_t)k + 1];
        Cursor q{c.beg, cut[(size_t)k], c.end};
        try
        {
            if (k == 0)
            {
                q.expect('[');
                if (q.peek() == ']') { s.first = q.p; s.close = q.p + 1; return; }
            }
            else
            {
                const void* f = std::memchr(q.p, '{', (size_t)(c.end - q.p));
                if (!f) { s.bad = true; return; }
                q.p = static_cast<const char*>(f);
                if (q.p >= hi) { s.first = s.next = q.p; return; }
            }
            s.first = q.p;
            reserve_triangles(s.tris, (size_t)(hi - q.p) / 200 + 16);
            for (;;)
            {
                if (q.peek() != '{') { s.bad = true; return; }
                Triangle t;
                parse_triangle(q, t);
                s.tris.push_back(t);
                const char d = q.peek();
                ++q.p;
                if (d == ']') { s.close = q.p; return; }
                if (d != ',') { s.bad = true; return; }
                q.ws();
                if (q.p >= hi) { s.next = q.p; return; }
            }
        }
        catch (const ParseError&) { s.bad = true; }
    };
    {
        std::vector<std::thread> pool;
        for (int k = 1; k < nt; ++k) pool.emplace_back(work, k);
        work(0);
        for (auto& t : pool) t.join();
    }
    size_t total = 0;
    int used = 0;
    const char* close = nullptr;
    for (int k = 0; k < nt; ++k)
    {
        const Share& s = sh[(size_t)k];
        if (s.bad || (k > 0 && s.first != sh[(size_t)k - 1].next)) return false;
        total += s.tris.size();
        used = k + 1;
        if (s.close) { close = s.close; break; }
    }
    if (!close) return false;
    size_triangles(out, total);
    std::vector<size_t> off((size_t)used + 1, 0);
    for (int k = 0; k < used; ++k) off[(size_t)k + 1] = off[(size_t)k] + sh[(size_t)k].tris.size();
    {
        std::vector<std::thread> pool;
        for (int k = 0; k < used; ++k)
            pool.emplace_back([&, k] {
                const auto& v = sh[(size_t)k].tris;
                if (!v.empty()) std::memcpy(&out[off[(size_t)k]], v.data(), v.size() * sizeof(Triangle));
            });
        for (auto& t : pool) t.join();
    }
    c.p = close;
    return true;
}

}  // namespace

// Parses a whole scene file held in memory.  Returns an empty string on
// success, else the message printed by LoadSceneJSON.
std::string parse_scene(const char* data, size_t size, Scene& out, int threads)
{
    Cursor c{data, data, data + size};
    // nlohmann's lexer skips a UTF-8 byte-order mark at the start of the input.
    if (size >= 3 && std::memcmp(data, "\xEF\xBB\xBF", 3) == 0) c.p += 3;
    try
    {
        Span sv, sc, ss, sl, sm, st;
        std::vector<const char*> tri_starts;
        bool tris_parsed = false;  // the speculative parallel parse succeeded
        unsigned hw = std::thread::hardware_concurrency();
        const int nt_all = threads > 0 ? threads : (int)(hw ? hw : 1);
        for_members(c, [&](const std::string& k, Cursor& v) {
            Span* s = nullptr;
            if (k == "version") s = &sv;
            else if (k == "camera") s = &sc;
            else if (k == "sun") s = &ss;
            else if (k == "lights") s = &sl;
            else if (k == "materials") s = &sm;
            else if (k == "triangles") { s = &st; tri_starts.clear(); }
            v.ws();
            const char* b = v.p;
            if (s == &st)
            {
                // Shares of at least 1 MB; small arrays take the serial scan.
                const int nt = (int)std::min<size_t>((size_t)nt_all, (size_t)(v.end - v.p) >> 20);
                tris_parsed = nt > 1 && v.peek() == '[' && parse_triangles_speculative(v, out.triangles, nt);
                if (tris_parsed) { st.p = b; st.end = v.p; return; }
            }
            v.skip(s == &st ? &tri_starts : nullptr);
            if (s) { s->p = b; s->end = v.p; }
        });
        // LoadSceneJSON reads the file with `f >> j` (scene_loader.cpp:38), a
        // non-strict parse: what follows the top-level object is not read.

        // "version" via j.value("version", 0): absent or not a number -> 0.
        int version = 0;
        if (sv.present())
        {
            Cursor v{data, sv.p, sv.end};
            char ch = v.peek();
            if (ch == '-' || (ch >= '0' && ch <= '9')) version = v.integer();
        }
        if (version != 1)
        {
            char m[96];
            std::snprintf(m, sizeof m, "unsupported version %d (expected 1)", version);
            return std::string("!") + m;  // '!' marks a non-parse failure
        }

        if (!sc.present()) missing("camera");
        {
            Cursor v{data, sc.p, sc.end};
            bool h[8] = {};
            for_members(v, [&](const std::string& k, Cursor& e) {
                if (k == "pos") { read_floats(e, out.camera.pos, 3); h[0] = true; }
                else if (k == "camera_to_world") { read_floats(e, out.camera.cameraToWorld, 16); h[1] = true; }
                else if (k == "fov_y_deg") { out.camera.fovYDeg = e.real(); h[2] = true; }
                else if (k == "aspect") { out.camera.aspect = e.real(); h[3] = true; }
                else if (k == "near") { out.camera.nearZ = e.real(); h[4] = true; }
                else if (k == "far") { out.camera.farZ = e.real(); h[5] = true; }
                else if (k == "image_width") { out.camera.imageWidth = e.integer(); h[6] = true; }
                else if (k == "image_height") { out.camera.imageHeight = e.integer(); h[7] = true; }
                else e.skip();
            });
            static const char* names[8] = {"pos", "camera_to_world", "fov_y_deg", "aspect", "near", "far",
                                           "image_width", "image_height"};
            for (int i = 0; i < 8; ++i) if (!h[i]) missing(names[i]);
        }
        if (!ss.present()) missing("sun");
        {
            Cursor v{data, ss.p, ss.end};
            bool h[3] = {};
            for_members(v, [&](const std::string& k, Cursor& e) {
                if (k == "direction") { read_floats(e, out.sun.dir, 3); h[0] = true; }
                else if (k == "color") { read_floats(e, out.sun.color, 3); h[1] = true; }
                else if (k == "intensity") { out.sun.intensity = e.real(); h[2] = true; }
                else e.skip();
            });
            if (!h[0]) missing("direction");
            if (!h[1]) missing("color");
            if (!h[2]) missing("intensity");
        }
        if (!sl.present()) missing("lights");
        {
            Cursor v{data, sl.p, sl.end};
            for_values(v, [&](Cursor& e) {
                // Members may come in any order: collect, then interpret by type.
                std::string type;
                bool htype = false, hdir = false, hcol = false, hint = false, hpos = false, hrad = false;
                float dir[3] = {}, col[3] = {}, pos[3] = {}, inten = 0, rad = 0;
                for_members(e, [&](const std::string& k, Cursor& m) {
                    if (k == "type")
                    {
                        if (m.peek() != '"') m.fail("light type must be a string");
                        type = m.string();
                        htype = true;
                    }
                    else if (k == "direction") { read_floats(m, dir, 3); hdir = true; }
                    else if (k == "color") { read_floats(m, col, 3); hcol = true; }
                    else if (k == "intensity") { inten = m.real(); hint = true; }
                    else if (k == "pos") { read_floats(m, pos, 3); hpos = true; }
                    else if (k == "radius") { rad = m.real(); hrad = true; }
                    else m.skip();
                });
                if (!htype) missing("type");
                if (type == "directional")
                {
                    if (!hdir) missing("direction");
                    if (!hcol) missing("color");
                    if (!hint) missing("intensity");
                    DirectionalLight d;
                    std::memcpy(d.dir, dir, sizeof dir);
                    std::memcpy(d.color, col, sizeof col);
                    d.intensity = inten;
                    out.directionals.push_back(d);
                }
                else if (type == "point")
                {
                    if (!hpos) missing("pos");
                    if (!hcol) missing("color");
                    if (!hint) missing("intensity");
                    if (!hrad) missing("radius");
                    PointLight pl;
                    std::memcpy(pl.pos, pos, sizeof pos);
                    std::memcpy(pl.color, col, sizeof col);
                    pl.intensity = inten;
                    pl.radius = rad;
                    out.points.push_back(pl);
                }
            });
        }
        if (!sm.present()) missing("materials");
        {
            Cursor v{data, sm.p, sm.end};
            for_values(v, [&](Cursor& e) {
                Material m;
                bool ha = false, he = false;
                for_members(e, [&](const std::string& k, Cursor& f) {
                    if (k == "albedo") { read_floats(f, m.albedo, 3); ha = true; }
                    else if (k == "emissive") { read_floats(f, m.emissive, 3); he = true; }
                    else if (k == "diffuse_tex")
                    {
                        if (f.peek() != '"') f.fail("diffuse_tex must be a string");
                        m.diffuseTex = f.string();
                    }
                    else f.skip();
                });
                if (!ha) missing("albedo");
                if (!he) missing("emissive");
                out.materials.push_back(std::move(m));
            });
        }
        if (!st.present()) missing("triangles");
        if (!tris_parsed)
        {
            Cursor v{data, st.p, st.end};
            // an object's values in key order, or none for null, as for lights and materials
            const char tc0 = v.peek();
            const bool tri_object = tc0 == '{' || tc0 == 'n';
            if (tc0 == '{') tri_starts = object_values_in_key_order(v);
            else if (tc0 == 'n')
            {
                if (!v.literal("null")) v.fail("bad literal");
                tri_starts.clear();
            }
            else if (tc0 != '[') v.fail("triangles must be an array");
            const size_t n = tri_starts.size();
            size_triangles(out.triangles, n);
            int nt = nt_all;
            const size_t min_per_thread = 16384;
            if ((size_t)nt > n / min_per_thread + 1) nt = (int)(n / min_per_thread + 1);
            std::vector<std::string> errs((size_t)nt);
            auto work = [&](int w) {
                const size_t b = n * (size_t)w / (size_t)nt, e = n * (size_t)(w + 1) / (size_t)nt;
                try
                {
                    for (size_t i = b; i < e; ++i)
                    {
                        Cursor tc{data, tri_starts[i], st.end};
                        if (tc.peek() != '{') tc.fail("triangle must be an object");
                        parse_triangle(tc, out.triangles[i]);
                        // the scan recorded starts only after commas: the element must end
                        // where the next one's comma (or the array's ']') follows
                        if (!tri_object && tc.peek() != (i + 1 < n ? ',' : ']')) tc.fail("expected ',' or ']'");
                    }
                }
                catch (const ParseError& pe) { errs[(size_t)w] = pe.msg; }
            };
            if (nt <= 1) work(0);
            else
            {
                std::vector<std::thread> pool;
                for (int w = 0; w < nt; ++w) pool.emplace_back(work, w);
                for (auto& t : pool) t.join();
            }
            for (auto& e : errs) if (!e.empty()) throw ParseError{e};
        }
    }
    catch (const ParseError& e)
    {
        return e.msg;
    }
    return std::string();
}

bool is_scene_bin(const char* data, size_t size);
std::string parse_scene_bin(const char* data, size_t size, Scene& out);

bool load_scene_file(const std::string& path, Scene& out, bool verbose, int threads, std::string& err)
{
    // The file is mapped read-only (pages prefaulted from the page cache) and
    // parsed in place; files that cannot be mapped are read into memory.
    const int fd = ::open(path.c_str(), O_RDONLY);
    struct stat stt;
    if (fd < 0 || ::fstat(fd, &stt) != 0)
    {
        if (fd >= 0) ::close(fd);
        err = "failed to open " + path;
        std::fprintf(stderr, "[scene] %s\n", err.c_str());
        set_error(LG_ERR_IO, "[scene] %s", err.c_str());
        return false;
    }
    const size_t sz = (size_t)stt.st_size;
    void* map = sz > 0 && S_ISREG(stt.st_mode) ? ::mmap(nullptr, sz, PROT_READ, MAP_PRIVATE | MAP_POPULATE, fd, 0)
                                               : MAP_FAILED;
    std::vector<char> copy;
    const char* data = nullptr;
    size_t got = 0;
    if (map != MAP_FAILED)
    {
        data = static_cast<const char*>(map);
        got = sz;
    }
    else
    {
        char chunk[1 << 16];
        ssize_t r;
        while ((r = ::read(fd, chunk, sizeof chunk)) > 0) copy.insert(copy.end(), chunk, chunk + r);
        if (r < 0)
        {
            ::close(fd);
            set_error(LG_ERR_IO, "[scene] read error on %s", path.c_str());
            std::fprintf(stderr, "[scene] read error on %s\n", path.c_str());
            return false;
        }
        data = copy.data();
        got = copy.size();
    }
    ::close(fd);
    struct Unmap
    {
        void* m;
        size_t n;
        ~Unmap() { if (m != MAP_FAILED) ::munmap(m, n); }
    } unmap{map, sz};
    Scene s;
    std::string msg = is_scene_bin(data, got) ? parse_scene_bin(data, got, s) : parse_scene(data, got, s, threads);
    if (!msg.empty())
    {
        if (msg[0] == '!')
        {
            std::fprintf(stderr, "[scene] %s\n", msg.c_str() + 1);
            set_error(LG_ERR_PARSE, "[scene] %s", msg.c_str() + 1);
        }
        else
        {
            std::fprintf(stderr, "[scene] JSON parse error: %s\n", msg.c_str());
            set_error(LG_ERR_PARSE, "[scene] JSON parse error: %s", msg.c_str());
        }
        err = msg;
        return false;
    }
    out = std::move(s);
    if (verbose)
    {
        std::printf("[scene] loaded %s\n", path.c_str());
        std::printf("  camera: %dx%d, fov %.1f deg, pos (%.2f,%.2f,%.2f)\n", out.camera.imageWidth,
                    out.camera.imageHeight, out.camera.fovYDeg, out.camera.pos[0], out.camera.pos[1],
                    out.camera.pos[2]);
        std::printf("  %zu directional + %zu point lights, %zu materials, %zu triangles\n", out.directionals.size(),
                    out.points.size(), out.materials.size(), out.triangles.size());
    }
    return true;
}

// ---------------------------------------------------------------------------
// Writer: 9 significant digits per float, which reads back to the same float
// through either strtof or strtod-then-narrow.
// ---------------------------------------------------------------------------
namespace
{
struct Out
{
    std::string s;
    void f(float x)
    {
        char b[32];
        if (!std::isfinite(x)) { s += "0"; return; }
        auto r = std::to_chars(b, b + sizeof b, x, std::chars_format::general, 9);
        s.append(b, r.ptr);
    }
    void i(long long v)
    {
        char b[24];
        auto r = std::to_chars(b, b + sizeof b, v);
        s.append(b, r.ptr);
    }
    void arr(const float* p, int n)
    {
        s += '[';
        for (int k = 0; k < n; ++k) { if (k) s += ','; f(p[k]); }
        s += ']';
    }
    void str(const std::string& v)
    {
        s += '"';
        for (char c : v)
        {
            if (c == '"' || c == '\\') { s += '\\'; s += c; }
            else if ((unsigned char)c < 0x20)
            {
                char b[8];
                std::snprintf(b, sizeof b, "\\u%04x", (unsigned char)c);
                s += b;
            }
            else s += c;
        }
        s += '"';
    }
};
}  // namespace

bool save_scene_file(const Scene& sc, const std::string& path, int threads)
{
    Out o;
    o.s.reserve(4096);
    o.s += "{\n\"version\": 1,\n\"camera\": {\"pos\": ";
    o.arr(sc.camera.pos, 3);
    o.s += ", \"camera_to_world\": ";
    o.arr(sc.camera.cameraToWorld, 16);
    o.s += ", \"fov_y_deg\": "; o.f(sc.camera.fovYDeg);
    o.s += ", \"aspect\": "; o.f(sc.camera.aspect);
    o.s += ", \"near\": "; o.f(sc.camera.nearZ);
    o.s += ", \"far\": "; o.f(sc.camera.farZ);
    o.s += ", \"image_width\": "; o.i(sc.camera.imageWidth);
    o.s += ", \"image_height\": "; o.i(sc.camera.imageHeight);
    o.s += "},\n\"sun\": {\"direction\": "; o.arr(sc.sun.dir, 3);
    o.s += ", \"color\": "; o.arr(sc.sun.color, 3);
    o.s += ", \"intensity\": "; o.f(sc.sun.intensity);
    o.s += "},\n\"lights\": [";
    bool first = true;
    for (const auto& d : sc.directionals)
    {
        if (!first) o.s += ",";
        first = false;
        o.s += "\n {\"type\": \"directional\", \"direction\": "; o.arr(d.dir, 3);
        o.s += ", \"color\": "; o.arr(d.color, 3);
        o.s += ", \"intensity\": "; o.f(d.intensity); o.s += "}";
    }
    for (const auto& p : sc.points)
    {
        if (!first) o.s += ",";
        first = false;
        o.s += "\n {\"type\": \"point\", \"pos\": "; o.arr(p.pos, 3);
        o.s += ", \"color\": "; o.arr(p.color, 3);
        o.s += ", \"intensity\": "; o.f(p.intensity);
        o.s += ", \"radius\": "; o.f(p.radius); o.s += "}";
    }
    o.s += "],\n\"materials\": [";
    for (size_t i = 0; i < sc.materials.size(); ++i)
    {
        const Material& m = sc.materials[i];
        if (i) o.s += ",";
        o.s += "\n {\"albedo\": "; o.arr(m.albedo, 3);
        o.s += ", \"emissive\": "; o.arr(m.emissive, 3);
        if (!m.diffuseTex.empty()) { o.s += ", \"diffuse_tex\": "; o.str(m.diffuseTex); }
        o.s += "}";
    }
    o.s += "],\n\"triangles\": [";
    // Triangles are formatted in parallel chunks, then written in order.
    const size_t n = sc.triangles.size();
    unsigned hw = std::thread::hardware_concurrency();
    int nt = threads > 0 ? threads : (int)(hw ? hw : 1);
    if ((size_t)nt > n / 4096 + 1) nt = (int)(n / 4096 + 1);
    std::vector<Out> parts((size_t)nt);
    auto work = [&](int w) {
        const size_t b = n * (size_t)w / (size_t)nt, e = n * (size_t)(w + 1) / (size_t)nt;
        Out& q = parts[(size_t)w];
        q.s.reserve((e - b) * 260);
        for (size_t i = b; i < e; ++i)
        {
            const Triangle& t = sc.triangles[i];
            if (i) q.s += ",";
            q.s += "\n{\"v\":[";
            for (int k = 0; k < 3; ++k) { if (k) q.s += ','; q.arr(t.v[k], 3); }
            q.s += "],\"n\":[";
            for (int k = 0; k < 3; ++k) { if (k) q.s += ','; q.arr(t.n[k], 3); }
            q.s += "],\"uv\":[";
            for (int k = 0; k < 3; ++k) { if (k) q.s += ','; q.arr(t.uv[k], 2); }
            q.s += "],\"mat\":"; q.i(t.material); q.s += "}";
        }
    };
    if (nt <= 1) work(0);
    else
    {
        std::vector<std::thread> pool;
        for (int w = 0; w < nt; ++w) pool.emplace_back(work, w);
        for (auto& t : pool) t.join();
    }
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fwrite(o.s.data(), 1, o.s.size(), f) == o.s.size();
    for (auto& q : parts) ok = ok && std::fwrite(q.s.data(), 1, q.s.size(), f) == q.s.size();
    const char tail[] = "\n]\n}\n";
    ok = ok && std::fwrite(tail, 1, sizeof tail - 1, f) == sizeof tail - 1;
    ok = (std::fclose(f) == 0) && ok;
    return ok;
}

// ---------------------------------------------------------------------------
// PNG (8-bit RGB, filter "none", zlib deflate) and Radiance RGBE (.hdr).
// ---------------------------------------------------------------------------
namespace
{
void be32(std::vector<unsigned char>& v, uint32_t x)
{
    v.push_back((unsigned char)(x >> 24)); v.push_back((unsigned char)(x >> 16));
    v.push_back((unsigned char)(x >> 8)); v.push_back((unsigned char)x);
}
void chunk(std::vector<unsigned char>& out, const char* type, const unsigned char* data, size_t n)
{
    be32(out, (uint32_t)n);
    size_t at = out.size();
    out.insert(out.end(), type, type + 4);
    if (n) out.insert(out.end(), data, data + n);
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, out.data() + at, (uInt)(n + 4));
    be32(out, (uint32_t)crc);
}
}  // namespace

bool write_png(const char* path, int w, int h, const uint8_t* rgb)
{
    if (w <= 0 || h <= 0 || !rgb) return false;
    const size_t row = (size_t)w * 3;
    std::vector<unsigned char> raw((row + 1) * (size_t)h);
    for (int y = 0; y < h; ++y)
    {
        raw[(row + 1) * (size_t)y] = 0;
        std::memcpy(&raw[(row + 1) * (size_t)y + 1], rgb + row * (size_t)y, row);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<unsigned char> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) return false;
    std::vector<unsigned char> out;
    const unsigned char sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    out.insert(out.end(), sig, sig + 8);
    std::vector<unsigned char> ihdr;
    be32(ihdr, (uint32_t)w);
    be32(ihdr, (uint32_t)h);
    ihdr.push_back(8);  // bit depth
    ihdr.push_back(2);  // colour type RGB
    ihdr.push_back(0); ihdr.push_back(0); ihdr.push_back(0);
    chunk(out, "IHDR", ihdr.data(), ihdr.size());
    chunk(out, "IDAT", z.data(), zlen);
    chunk(out, "IEND", nullptr, 0);
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return (std::fclose(f) == 0) && ok;
}

bool write_hdr(const char* path, int w, int h, const float* rgb)
{
    if (w <= 0 || h <= 0 || !rgb) return false;
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    std::fprintf(f, "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n", h, w);
    std::vector<unsigned char> line((size_t)w * 4);
    bool ok = true;
    for (int y = 0; y < h && ok; ++y)
    {
        for (int x = 0; x < w; ++x)
        {
            const float* p = rgb + ((size_t)y * w + x) * 3;
            float m = std::max(p[0], std::max(p[1], p[2]));
            unsigned char* q = &line[(size_t)x * 4];
            if (!(m > 1e-32f)) { q[0] = q[1] = q[2] = q[3] = 0; continue; }
            int e;
            float s = std::frexp(m, &e) * 256.0f / m;
            q[0] = (unsigned char)std::max(0.0f, p[0] * s);
            q[1] = (unsigned char)std::max(0.0f, p[1] * s);
            q[2] = (unsigned char)std::max(0.0f, p[2] * s);
            q[3] = (unsigned char)(e + 128);
        }
        ok = std::fwrite(line.data(), 1, line.size(), f) == line.size();
    }
    return (std::fclose(f) == 0) && ok;
}

// ---------------------------------------------------------------------------
// Binary scene file: the same content as scene.json with every record stored
// in its in-memory layout, so loading is one sequential read per array.
//
//   0   char[8]  "LGSCENE1"
//   8   u32      version (1), u32 flags (0)
//   16  i32      n_tris, n_mats, n_points, n_directionals
//   32  camera   pos[3], camera_to_world[16], fov_y_deg, aspect, near, far (f32),
//                image_width, image_height (i32)                      (100 B)
//   132 sun      direction[3], color[3], intensity (f32)               (28 B)
//   160 materials n_mats x {albedo[3], emissive[3] f32, u32 tex_len}, then the
//                texture paths (tex_len bytes each, no terminator)
//       points   n_points x 32 B, directionals n_directionals x 28 B
//       zero padding to a multiple of 64 bytes
//       triangles n_tris x 100 B (Triangle records)
// All values little-endian.
// ---------------------------------------------------------------------------
namespace
{
constexpr char kBinMagic[8] = {'L', 'G', 'S', 'C', 'E', 'N', 'E', '1'};

struct BinWriter
{
    std::vector<unsigned char> b;
    template <class T>
    void put(const T& v)
    {
        const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
        b.insert(b.end(), p, p + sizeof(T));
    }
    void raw(const void* p, size_t n)
    {
        const unsigned char* q = static_cast<const unsigned char*>(p);
        b.insert(b.end(), q, q + n);
    }
};

struct BinReader
{
    const unsigned char* p;
    const unsigned char* end;
    bool ok = true;
    void raw(void* dst, size_t n)
    {
        if ((size_t)(end - p) < n) { ok = false; return; }
        std::memcpy(dst, p, n);
        p += n;
    }
    template <class T>
    T get()
    {
        T v{};
        raw(&v, sizeof v);
        return v;
    }
};
}  // namespace

bool is_scene_bin(const char* data, size_t size) { return size >= 8 && std::memcmp(data, kBinMagic, 8) == 0; }

bool save_scene_bin(const Scene& sc, const std::string& path)
{
    BinWriter w;
    w.raw(kBinMagic, 8);
    w.put<uint32_t>(1);
    w.put<uint32_t>(0);
    w.put<int32_t>((int32_t)sc.triangles.size());
    w.put<int32_t>((int32_t)sc.materials.size());
    w.put<int32_t>((int32_t)sc.points.size());
    w.put<int32_t>((int32_t)sc.directionals.size());
    w.raw(sc.camera.pos, 12);
    w.raw(sc.camera.cameraToWorld, 64);
    w.put(sc.camera.fovYDeg);
    w.put(sc.camera.aspect);
    w.put(sc.camera.nearZ);
    w.put(sc.camera.farZ);
    w.put<int32_t>(sc.camera.imageWidth);
    w.put<int32_t>(sc.camera.imageHeight);
    w.raw(sc.sun.dir, 12);
    w.raw(sc.sun.color, 12);
    w.put(sc.sun.intensity);
    for (const Material& m : sc.materials)
    {
        w.raw(m.albedo, 12);
        w.raw(m.emissive, 12);
        w.put<uint32_t>((uint32_t)m.diffuseTex.size());
    }
    for (const Material& m : sc.materials) w.raw(m.diffuseTex.data(), m.diffuseTex.size());
    if (!sc.points.empty()) w.raw(sc.points.data(), sc.points.size() * sizeof(PointLight));
    if (!sc.directionals.empty()) w.raw(sc.directionals.data(), sc.directionals.size() * sizeof(DirectionalLight));
    while (w.b.size() % 64) w.b.push_back(0);
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fwrite(w.b.data(), 1, w.b.size(), f) == w.b.size();
    const size_t tb = sc.triangles.size() * sizeof(Triangle);
    ok = ok && (tb == 0 || std::fwrite(sc.triangles.data(), 1, tb, f) == tb);
    return (std::fclose(f) == 0) && ok;
}

// Parses a whole binary scene held in memory; returns "" or an error message.
std::string parse_scene_bin(const char* data, size_t size, Scene& out)
{
    BinReader r{reinterpret_cast<const unsigned char*>(data), reinterpret_cast<const unsigned char*>(data) + size};
    char magic[8];
    r.raw(magic, 8);
    const uint32_t version = r.get<uint32_t>();
    r.get<uint32_t>();
    if (!r.ok || version != 1) return "!unsupported binary scene version";
    const int32_t nt = r.get<int32_t>(), nm = r.get<int32_t>(), np = r.get<int32_t>(), nd = r.get<int32_t>();
    if (!r.ok || nt < 0 || nm < 0 || np < 0 || nd < 0) return "!corrupt binary scene header";
    r.raw(out.camera.pos, 12);
    r.raw(out.camera.cameraToWorld, 64);
    out.camera.fovYDeg = r.get<float>();
    out.camera.aspect = r.get<float>();
    out.camera.nearZ = r.get<float>();
    out.camera.farZ = r.get<float>();
    out.camera.imageWidth = r.get<int32_t>();
    out.camera.imageHeight = r.get<int32_t>();
    r.raw(out.sun.dir, 12);
    r.raw(out.sun.color, 12);
    out.sun.intensity = r.get<float>();
    if ((size_t)(r.end - r.p) < (size_t)nm * 28) return "!truncated binary scene";
    out.materials.resize((size_t)nm);
    std::vector<uint32_t> tl((size_t)nm);
    for (int32_t i = 0; i < nm; ++i)
    {
        r.raw(out.materials[(size_t)i].albedo, 12);
        r.raw(out.materials[(size_t)i].emissive, 12);
        tl[(size_t)i] = r.get<uint32_t>();
    }
    for (int32_t i = 0; i < nm && r.ok; ++i)
    {
        if ((size_t)(r.end - r.p) < tl[(size_t)i]) { r.ok = false; break; }
        out.materials[(size_t)i].diffuseTex.assign(reinterpret_cast<const char*>(r.p), tl[(size_t)i]);
        r.p += tl[(size_t)i];
    }
    if (!r.ok || (size_t)(r.end - r.p) < (size_t)np * sizeof(PointLight) + (size_t)nd * sizeof(DirectionalLight))
        return "!truncated binary scene";
    out.points.resize((size_t)np);
    if (np) r.raw(out.points.data(), (size_t)np * sizeof(PointLight));
    out.directionals.resize((size_t)nd);
    if (nd) r.raw(out.directionals.data(), (size_t)nd * sizeof(DirectionalLight));
    const size_t at = (size_t)(r.p - reinterpret_cast<const unsigned char*>(data));
    r.p += (64 - at % 64) % 64;
    const size_t tb = (size_t)nt * sizeof(Triangle);
    if (r.p > r.end || (size_t)(r.end - r.p) != tb) return "!truncated binary scene";
    if (!r.ok) return "!truncated binary scene";
    size_triangles(out.triangles, (size_t)nt);
    copy_triangles(out.triangles.data(), r.p, (size_t)nt);
    return std::string();
}

}  // namespace lg

// Drop-in C++ entry point (reference include/scene.h:58).
bool LoadSceneJSON(const std::string& path, Scene& out)
{
    std::string err;
    return lg::load_scene_file(path, out, true, 0, err);
}
