// scene_io.cpp -- scene.json loader and writer, PNG and Radiance HDR output.
//
// Loader: drop-in for LoadSceneJSON (reference src/scene_loader.cpp:26-138)
// with the same schema (version 1; camera, sun, lights[], materials[],
// triangles[]), the same number conversion (a JSON integer converts to float
// directly, a JSON real is read as double then narrowed to float, as
// nlohmann::json's get<float>() does) and the same messages.  It is a
// schema-driven parser over the file bytes instead of a DOM: the top level is
// scanned once, the triangle array's element offsets are recorded during that
// scan, and the elements are parsed by several host threads.  Where the
// reference lets nlohmann throw out of LoadSceneJSON on a missing key (the
// process terminates), this loader prints "[scene] ..." and returns false.
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

#include <zlib.h>

#include "bvh.h"
#include "common.h"
#include "scene.h"

namespace lg
{
namespace
{
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
        }
        double d = std::strtod(std::string(tb, te).c_str(), nullptr);
        return (int)d;
    }
    // Skips one value.  When starts != null and the value is an array, the
    // offset of each element is appended (used for the triangle array).
    void skip(std::vector<const char*>* starts = nullptr)
    {
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
        if (c == '"') { string(); return; }
        if (c == 't') { if (!literal("true")) fail("bad literal"); return; }
        if (c == 'f') { if (!literal("false")) fail("bad literal"); return; }
        if (c == 'n') { if (!literal("null")) fail("bad literal"); return; }
        const char *tb, *te;
        bool is_int;
        number_token(tb, te, is_int);
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

}  // namespace

// Parses a whole scene file held in memory.  Returns an empty string on
// success, else the message printed by LoadSceneJSON.
std::string parse_scene(const char* data, size_t size, Scene& out, int threads)
{
    Cursor c{data, data, data + size};
    try
    {
        Span sv, sc, ss, sl, sm, st;
        std::vector<const char*> tri_starts;
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
            v.skip(s == &st ? &tri_starts : nullptr);
            if (s) { s->p = b; s->end = v.p; }
        });
        c.ws();
        if (c.p != c.end) c.fail("trailing characters");

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
            for_elements(v, [&](Cursor& e) {
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
            for_elements(v, [&](Cursor& e) {
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
        {
            Cursor v{data, st.p, st.end};
            if (v.peek() != '[') v.fail("triangles must be an array");
            const size_t n = tri_starts.size();
            out.triangles.assign(n, Triangle{});
            unsigned hw = std::thread::hardware_concurrency();
            int nt = threads > 0 ? threads : (int)(hw ? hw : 1);
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

bool load_scene_file(const std::string& path, Scene& out, bool verbose, int threads, std::string& err)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f)
    {
        err = "failed to open " + path;
        std::fprintf(stderr, "[scene] %s\n", err.c_str());
        set_error(LG_ERR_IO, "[scene] %s", err.c_str());
        return false;
    }
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::unique_ptr<char[]> buf(new (std::nothrow) char[sz > 0 ? (size_t)sz : 1]);
    if (!buf)
    {
        std::fclose(f);
        set_error(LG_ERR_NOMEM, "[scene] out of memory reading %s", path.c_str());
        return false;
    }
    size_t got = sz > 0 ? std::fread(buf.get(), 1, (size_t)sz, f) : 0;
    std::fclose(f);
    if ((long)got != sz)
    {
        set_error(LG_ERR_IO, "[scene] short read on %s", path.c_str());
        std::fprintf(stderr, "[scene] short read on %s\n", path.c_str());
        return false;
    }
    Scene s;
    std::string msg = parse_scene(buf.get(), got, s, threads);
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

}  // namespace lg

// Drop-in C++ entry point (reference include/scene.h:58).
bool LoadSceneJSON(const std::string& path, Scene& out)
{
    std::string err;
    return lg::load_scene_file(path, out, true, 0, err);
}
