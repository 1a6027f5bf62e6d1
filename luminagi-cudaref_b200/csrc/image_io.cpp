// image_io.cpp -- PNG decoding to 8-bit RGBA for diffuse textures.
//
// The reference loads textures with stbi_load(path, &w, &h, &n, 4)
// (src/pathtracer.cu:553-560): any PNG becomes 8-bit RGBA, top row first,
// without gamma handling.  This decoder follows the PNG specification
// (ISO/IEC 15948): every colour type (grey, RGB, palette, grey+alpha, RGBA),
// every bit depth (1/2/4/8/16), the five scanline filters and Adam7
// interlacing, with zlib's inflate for the IDAT stream.  Conversions to
// 8-bit RGBA are the ones stb_image makes:
//   * samples of 1/2/4 bits scale by 255 / (2^depth - 1) (0xff, 0x55, 0x11);
//   * 16-bit samples keep their high byte;
//   * grey replicates into R, G and B;
//   * missing alpha is 255, and a tRNS colour key (grey or RGB, compared at the
//     file's bit depth) or tRNS palette alphas set it.
// Only the RGB channels reach the renderer (sample_albedo, :274-282).  Other
// formats stb_image reads (JPEG, BMP, TGA, ...) are not decoded: they fail
// with "not a PNG file" and the material stays untextured.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <zlib.h>

namespace lg
{
namespace
{
uint32_t rd32(const unsigned char* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

int paeth(int a, int b, int c)
{
    const int p = a + b - c;
    const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

// Reverses the per-scanline filters of one (sub-)image in place.  `in` holds
// rows of 1 filter byte + rowbytes; returns false on an unknown filter type.
bool unfilter(const unsigned char* in, unsigned char* out, size_t rowbytes, int rows, int bpp)
{
    for (int y = 0; y < rows; ++y)
    {
        const int f = in[(rowbytes + 1) * (size_t)y];
        const unsigned char* src = in + (rowbytes + 1) * (size_t)y + 1;
        unsigned char* cur = out + rowbytes * (size_t)y;
        const unsigned char* prev = y > 0 ? cur - rowbytes : nullptr;
        for (size_t i = 0; i < rowbytes; ++i)
        {
            const int a = i >= (size_t)bpp ? cur[i - bpp] : 0;
            const int b = prev ? prev[i] : 0;
            const int c = (prev && i >= (size_t)bpp) ? prev[i - bpp] : 0;
            int v;
            switch (f)
            {
            case 0: v = src[i]; break;
            case 1: v = src[i] + a; break;
            case 2: v = src[i] + b; break;
            case 3: v = src[i] + ((a + b) >> 1); break;
            case 4: v = src[i] + paeth(a, b, c); break;
            default: return false;
            }
            cur[i] = (unsigned char)v;
        }
    }
    return true;
}

struct Header
{
    int w = 0, h = 0, depth = 0, ctype = 0, interlace = 0;
    int channels() const
    {
        switch (ctype)
        {
        case 0: return 1;
        case 2: return 3;
        case 3: return 1;
        case 4: return 2;
        case 6: return 4;
        }
        return 0;
    }
};

// Sample `c` of pixel x in an unfiltered row, at the file's bit depth.
unsigned sample_at(const unsigned char* row, int x, int c, int channels, int depth)
{
    if (depth == 8) return row[(size_t)x * channels + c];
    if (depth == 16)
    {
        const unsigned char* p = row + ((size_t)x * channels + c) * 2;
        return (unsigned)p[0] << 8 | p[1];
    }
    // 1/2/4 bits: one channel (grey or palette index), packed from the MSB.
    const size_t bit = (size_t)x * depth;
    const unsigned byte = row[bit >> 3];
    const int shift = 8 - depth - (int)(bit & 7);
    return (byte >> shift) & ((1u << depth) - 1);
}

unsigned char to8(unsigned v, int depth)
{
    switch (depth)
    {
    case 16: return (unsigned char)(v >> 8);
    case 8: return (unsigned char)v;
    case 4: return (unsigned char)(v * 0x11);
    case 2: return (unsigned char)(v * 0x55);
    case 1: return (unsigned char)(v * 0xff);
    }
    return 0;
}
}  // namespace

bool decode_png(const char* path, int& out_w, int& out_h, std::vector<uint8_t>& rgba, std::string& err)
{
    FILE* f = std::fopen(path, "rb");
    if (!f)
    {
        err = "cannot open";
        return false;
    }
    std::vector<unsigned char> file;
    {
        unsigned char buf[1 << 16];
        size_t n;
        while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) file.insert(file.end(), buf, buf + n);
        std::fclose(f);
    }
    static const unsigned char kSig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (file.size() < 8 || std::memcmp(file.data(), kSig, 8) != 0)
    {
        err = "not a PNG file";
        return false;
    }
    Header hd;
    std::vector<unsigned char> idat, plte, trns;
    bool have_ihdr = false, have_iend = false;
    size_t pos = 8;
    while (pos + 12 <= file.size() && !have_iend)
    {
        const uint32_t len = rd32(&file[pos]);
        if (len > file.size() - pos - 12)
        {
            err = "truncated chunk";
            return false;
        }
        const unsigned char* type = &file[pos + 4];
        const unsigned char* data = &file[pos + 8];
        // The chunk CRC is skipped, not verified, as stb_image skips it: a file
        // the reference accepts is accepted here too.
        if (!std::memcmp(type, "IHDR", 4))
        {
            if (len != 13)
            {
                err = "bad IHDR";
                return false;
            }
            hd.w = (int)rd32(data);
            hd.h = (int)rd32(data + 4);
            hd.depth = data[8];
            hd.ctype = data[9];
            hd.interlace = data[12];
            if (data[10] != 0 || data[11] != 0 || hd.interlace > 1)
            {
                err = "unsupported compression, filter or interlace method";
                return false;
            }
            have_ihdr = true;
        }
        else if (!std::memcmp(type, "PLTE", 4)) plte.assign(data, data + len);
        else if (!std::memcmp(type, "tRNS", 4)) trns.assign(data, data + len);
        else if (!std::memcmp(type, "IDAT", 4)) idat.insert(idat.end(), data, data + len);
        else if (!std::memcmp(type, "IEND", 4)) have_iend = true;
        pos += 12 + (size_t)len;
    }
    if (!have_ihdr || idat.empty())
    {
        err = "missing IHDR or IDAT";
        return false;
    }
    const int ch = hd.channels();
    const bool depth_ok = (hd.ctype == 0 && (hd.depth == 1 || hd.depth == 2 || hd.depth == 4 || hd.depth == 8 ||
                                              hd.depth == 16)) ||
                          (hd.ctype == 3 && (hd.depth == 1 || hd.depth == 2 || hd.depth == 4 || hd.depth == 8)) ||
                          ((hd.ctype == 2 || hd.ctype == 4 || hd.ctype == 6) && (hd.depth == 8 || hd.depth == 16));
    if (!ch || !depth_ok || hd.w <= 0 || hd.h <= 0 || hd.w > (1 << 24) || hd.h > (1 << 24) ||
        (long long)hd.w * hd.h > (1ll << 30))
    {
        err = "unsupported colour type, bit depth or size";
        return false;
    }
    if (hd.ctype == 3 && (plte.empty() || plte.size() % 3))
    {
        err = "palette image without a valid PLTE";
        return false;
    }
    const int bits = ch * hd.depth;
    const int bpp = bits >= 8 ? bits / 8 : 1;

    // Adam7 passes: x0, y0, dx, dy.  A non-interlaced image is one pass.
    static const int kAdam7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                                     {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
    const int n_pass = hd.interlace ? 7 : 1;
    struct Pass { int x0, y0, dx, dy, pw, ph; size_t rowbytes; };
    std::vector<Pass> passes;
    size_t raw_size = 0;
    for (int p = 0; p < n_pass; ++p)
    {
        Pass ps;
        if (hd.interlace)
        {
            ps.x0 = kAdam7[p][0]; ps.y0 = kAdam7[p][1]; ps.dx = kAdam7[p][2]; ps.dy = kAdam7[p][3];
        }
        else
        {
            ps.x0 = 0; ps.y0 = 0; ps.dx = 1; ps.dy = 1;
        }
        ps.pw = hd.w > ps.x0 ? (hd.w - ps.x0 + ps.dx - 1) / ps.dx : 0;
        ps.ph = hd.h > ps.y0 ? (hd.h - ps.y0 + ps.dy - 1) / ps.dy : 0;
        ps.rowbytes = ((size_t)ps.pw * bits + 7) / 8;
        if (ps.pw && ps.ph) raw_size += (ps.rowbytes + 1) * (size_t)ps.ph;
        passes.push_back(ps);
    }

    std::vector<unsigned char> raw(raw_size);
    {
        z_stream zs{};
        if (inflateInit(&zs) != Z_OK)
        {
            err = "zlib init failed";
            return false;
        }
        zs.next_in = idat.data();
        zs.avail_in = (uInt)idat.size();
        zs.next_out = raw.data();
        zs.avail_out = (uInt)raw.size();
        const int zr = inflate(&zs, Z_FINISH);
        const size_t got = raw.size() - zs.avail_out;
        inflateEnd(&zs);
        if ((zr != Z_STREAM_END && zr != Z_BUF_ERROR && zr != Z_OK) || got != raw.size())
        {
            err = "corrupt image data";
            return false;
        }
    }

    rgba.assign((size_t)hd.w * hd.h * 4, 255);
    // Colour key from tRNS at the file's bit depth (grey or RGB images).
    bool key = false;
    unsigned key_v[3] = {0, 0, 0};
    if (!trns.empty() && hd.ctype == 0 && trns.size() >= 2)
    {
        key = true;
        key_v[0] = (unsigned)trns[0] << 8 | trns[1];
    }
    if (!trns.empty() && hd.ctype == 2 && trns.size() >= 6)
    {
        key = true;
        for (int k = 0; k < 3; ++k) key_v[k] = (unsigned)trns[2 * k] << 8 | trns[2 * k + 1];
    }
    const size_t n_pal = plte.size() / 3;
    size_t off = 0;
    std::vector<unsigned char> rows;
    for (const Pass& ps : passes)
    {
        if (!ps.pw || !ps.ph) continue;
        rows.resize(ps.rowbytes * (size_t)ps.ph);
        if (!unfilter(raw.data() + off, rows.data(), ps.rowbytes, ps.ph, bpp))
        {
            err = "bad scanline filter";
            return false;
        }
        off += (ps.rowbytes + 1) * (size_t)ps.ph;
        for (int y = 0; y < ps.ph; ++y)
        {
            const unsigned char* row = rows.data() + ps.rowbytes * (size_t)y;
            for (int x = 0; x < ps.pw; ++x)
            {
                unsigned char* o = &rgba[(((size_t)(ps.y0 + y * ps.dy)) * hd.w + ps.x0 + (size_t)x * ps.dx) * 4];
                switch (hd.ctype)
                {
                case 0:
                {
                    const unsigned g = sample_at(row, x, 0, 1, hd.depth);
                    o[0] = o[1] = o[2] = to8(g, hd.depth);
                    if (key && g == key_v[0]) o[3] = 0;
                    break;
                }
                case 2:
                {
                    unsigned v[3];
                    for (int k = 0; k < 3; ++k)
                    {
                        v[k] = sample_at(row, x, k, 3, hd.depth);
                        o[k] = to8(v[k], hd.depth);
                    }
                    if (key && v[0] == key_v[0] && v[1] == key_v[1] && v[2] == key_v[2]) o[3] = 0;
                    break;
                }
                case 3:
                {
                    const unsigned idx = sample_at(row, x, 0, 1, hd.depth);
                    if (idx >= n_pal)
                    {
                        err = "palette index out of range";
                        return false;
                    }
                    o[0] = plte[3 * idx];
                    o[1] = plte[3 * idx + 1];
                    o[2] = plte[3 * idx + 2];
                    o[3] = idx < trns.size() ? trns[idx] : 255;
                    break;
                }
                case 4:
                    o[0] = o[1] = o[2] = to8(sample_at(row, x, 0, 2, hd.depth), hd.depth);
                    o[3] = to8(sample_at(row, x, 1, 2, hd.depth), hd.depth);
                    break;
                case 6:
                    for (int k = 0; k < 4; ++k) o[k] = to8(sample_at(row, x, k, 4, hd.depth), hd.depth);
                    break;
                }
            }
        }
    }
    out_w = hd.w;
    out_h = hd.h;
    return true;
}

}  // namespace lg
