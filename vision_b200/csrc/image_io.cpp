// Image decoders for the `image` shader node (the reference loads textures
// through its image pool, src/render_core/shadernodes/image.cpp, on top of a
// third-party image library): PNG (RFC 2083, with a DEFLATE decoder after
// RFC 1951), baseline sequential JPEG (ITU-T T.81, JFIF colour) and Radiance
// HDR (RGBE).  Output: linear RGB as float, row 0 the top of the image.
#include "vs_image.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <stdexcept>

namespace vs {

namespace {

std::vector<uint8_t> read_file(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("image: cannot open '" + path + "'");
    return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

[[noreturn]] void bad(const std::string &what) { throw std::runtime_error("image: " + what); }
// Text taken from a file, for an error message: printable ASCII only.
std::string printable(const std::string &s) {
    std::string r = s.substr(0, 64);
    for (char &c : r)
        if (c < 0x20 || c > 0x7e) c = '?';
    return r;
}
// A valid file using a feature these decoders do not implement.
[[noreturn]] void not_supported(const std::string &what) { throw std::runtime_error("unsupported: image: " + what); }

// ---- DEFLATE (RFC 1951) ------------------------------------------------------

struct BitReader {
    const uint8_t *p;
    size_t n, pos = 0;
    uint32_t bitbuf = 0;
    int bitcnt = 0;
    uint32_t bits(int k) {
        while (bitcnt < k) {
            if (pos >= n) bad("deflate stream truncated");
            bitbuf |= static_cast<uint32_t>(p[pos++]) << bitcnt;
            bitcnt += 8;
        }
        uint32_t v = bitbuf & ((k == 32) ? 0xffffffffu : ((1u << k) - 1u));
        bitbuf >>= k;
        bitcnt -= k;
        return v;
    }
    void align() {
        bitbuf = 0;
        bitcnt = 0;
    }
};

// Canonical Huffman code from code lengths: decoded bit by bit with the
// counts per length (the construction of RFC 1951 section 3.2.2).
struct Huff {
    uint16_t count[16] = {};
    std::vector<uint16_t> symbol;
    void build(const uint8_t *len, int n) {
        std::memset(count, 0, sizeof(count));
        for (int i = 0; i < n; ++i) count[len[i]]++;
        count[0] = 0;
        uint16_t offs[16] = {};
        for (int i = 1; i < 16; ++i) offs[i] = offs[i - 1] + count[i - 1];
        symbol.assign(n, 0);
        for (int i = 0; i < n; ++i)
            if (len[i]) symbol[offs[len[i]]++] = static_cast<uint16_t>(i);
    }
    int decode(BitReader &br) const {
        int code = 0, first = 0, index = 0;
        for (int l = 1; l < 16; ++l) {
            code |= static_cast<int>(br.bits(1));
            const int c = count[l];
            if (code - c < first) return symbol[index + (code - first)];
            index += c;
            first += c;
            first <<= 1;
            code <<= 1;
        }
        bad("invalid Huffman code");
    }
};

const uint16_t kLenBase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31,
                               35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
const uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t kDistBase[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129,
                                193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
const uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

std::vector<uint8_t> inflate(const uint8_t *data, size_t n, size_t expect) {
    BitReader br{data, n};
    std::vector<uint8_t> out;
    out.reserve(expect);
    bool last = false;
    while (!last) {
        last = br.bits(1) != 0;
        const uint32_t type = br.bits(2);
        if (type == 0) {
            br.align();
            if (br.pos + 4 > n) bad("deflate stored block truncated");
            const uint32_t len = data[br.pos] | (data[br.pos + 1] << 8);
            br.pos += 4;
            if (br.pos + len > n) bad("deflate stored block truncated");
            out.insert(out.end(), data + br.pos, data + br.pos + len);
            br.pos += len;
            continue;
        }
        Huff lit, dist;
        if (type == 1) {
            uint8_t l[288], d[30];
            for (int i = 0; i < 144; ++i) l[i] = 8;
            for (int i = 144; i < 256; ++i) l[i] = 9;
            for (int i = 256; i < 280; ++i) l[i] = 7;
            for (int i = 280; i < 288; ++i) l[i] = 8;
            for (int i = 0; i < 30; ++i) d[i] = 5;
            lit.build(l, 288);
            dist.build(d, 30);
        } else if (type == 2) {
            const int hlit = static_cast<int>(br.bits(5)) + 257, hdist = static_cast<int>(br.bits(5)) + 1;
            const int hclen = static_cast<int>(br.bits(4)) + 4;
            static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
            uint8_t cl[19] = {};
            for (int i = 0; i < hclen; ++i) cl[order[i]] = static_cast<uint8_t>(br.bits(3));
            Huff ch;
            ch.build(cl, 19);
            uint8_t lens[320] = {};
            int i = 0;
            while (i < hlit + hdist) {
                const int sym = ch.decode(br);
                if (sym < 16) {
                    lens[i++] = static_cast<uint8_t>(sym);
                } else {
                    int rep = 0;
                    uint8_t v = 0;
                    if (sym == 16) {
                        if (i == 0) bad("deflate repeat without a previous length");
                        v = lens[i - 1];
                        rep = 3 + static_cast<int>(br.bits(2));
                    } else if (sym == 17) {
                        rep = 3 + static_cast<int>(br.bits(3));
                    } else {
                        rep = 11 + static_cast<int>(br.bits(7));
                    }
                    if (i + rep > hlit + hdist) bad("deflate code lengths overflow");
                    while (rep--) lens[i++] = v;
                }
            }
            lit.build(lens, hlit);
            dist.build(lens + hlit, hdist);
        } else {
            bad("deflate block type 3");
        }
        for (;;) {
            const int sym = lit.decode(br);
            if (sym < 256) {
                out.push_back(static_cast<uint8_t>(sym));
            } else if (sym == 256) {
                break;
            } else {
                const int li = sym - 257;
                if (li >= 29) bad("deflate length code");
                const size_t len = kLenBase[li] + br.bits(kLenExtra[li]);
                const int di = dist.decode(br);
                if (di >= 30) bad("deflate distance code");
                const size_t d = kDistBase[di] + br.bits(kDistExtra[di]);
                if (d > out.size()) bad("deflate distance beyond the output");
                const size_t from = out.size() - d;
                for (size_t k = 0; k < len; ++k) out.push_back(out[from + k]);
            }
        }
    }
    return out;
}

// ---- PNG -----------------------------------------------------------------------

uint32_t be32(const uint8_t *p) {
    return (static_cast<uint32_t>(p[0]) << 24) | (static_cast<uint32_t>(p[1]) << 16) |
           (static_cast<uint32_t>(p[2]) << 8) | p[3];
}

Image decode_png(const std::vector<uint8_t> &f) {
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (f.size() < 8 || std::memcmp(f.data(), sig, 8) != 0) bad("not a PNG file");
    uint32_t w = 0, h = 0;
    int depth = 0, ctype = 0, interlace = 0;
    std::vector<uint8_t> idat, plte, trns;
    size_t p = 8;
    while (p + 8 <= f.size()) {
        const uint32_t len = be32(&f[p]);
        const std::string type(reinterpret_cast<const char *>(&f[p + 4]), 4);
        if (p + 12 + len > f.size()) bad("PNG chunk truncated");
        const uint8_t *d = &f[p + 8];
        if (type == "IHDR") {
            w = be32(d);
            h = be32(d + 4);
            depth = d[8];
            ctype = d[9];
            interlace = d[12];
        } else if (type == "PLTE") {
            plte.assign(d, d + len);
        } else if (type == "tRNS") {
            trns.assign(d, d + len);
        } else if (type == "IDAT") {
            idat.insert(idat.end(), d, d + len);
        } else if (type == "IEND") {
            break;
        }
        p += 12 + len;
    }
    if (w == 0 || h == 0 || w > 65536 || h > 65536) bad("PNG size");
    if (interlace) not_supported("interlaced PNG");
    int channels = 0;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: bad("PNG colour type");
    }
    const bool low = depth == 1 || depth == 2 || depth == 4;
    if (!(depth == 8 || (depth == 16 && ctype != 3) || (low && (ctype == 0 || ctype == 3)))) bad("PNG bit depth");
    if (static_cast<uint64_t>(w) * h > (1ull << 28)) bad("PNG size");
    if (idat.size() < 2) bad("PNG without image data");
    const size_t bits_px = static_cast<size_t>(channels) * depth;
    const size_t stride = (bits_px * w + 7) / 8;
    const size_t bpp = std::max<size_t>(1, bits_px / 8);
    // zlib: 2-byte header, DEFLATE data, Adler-32.
    std::vector<uint8_t> raw = inflate(idat.data() + 2, idat.size() - 2, (stride + 1) * h);
    if (raw.size() < (stride + 1) * h) bad("PNG image data truncated");
    std::vector<uint8_t> img(stride * h);
    for (uint32_t y = 0; y < h; ++y) {
        const uint8_t filter = raw[y * (stride + 1)];
        const uint8_t *src = &raw[y * (stride + 1) + 1];
        uint8_t *dst = &img[y * stride];
        const uint8_t *up = y ? &img[(y - 1) * stride] : nullptr;
        for (size_t i = 0; i < stride; ++i) {
            const int a = i >= bpp ? dst[i - bpp] : 0;
            const int b = up ? up[i] : 0;
            const int c = (up && i >= bpp) ? up[i - bpp] : 0;
            int v = src[i];
            switch (filter) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) / 2; break;
                case 4: {
                    const int pp = a + b - c, pa = std::abs(pp - a), pb = std::abs(pp - b), pc = std::abs(pp - c);
                    v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
                    break;
                }
                default: bad("PNG filter type");
            }
            dst[i] = static_cast<uint8_t>(v);
        }
    }
    Image out;
    out.width = w;
    out.height = h;
    out.channels = (ctype == 3) ? (trns.empty() ? 3 : 4) : channels;
    out.data.assign(static_cast<size_t>(w) * h * out.channels, 0.0f);
    const float maxv = static_cast<float>((1 << depth) - 1);
    auto sample = [&](uint32_t x, uint32_t y, int ch) -> uint32_t {
        const uint8_t *row = &img[y * stride];
        if (depth == 8) return row[static_cast<size_t>(x) * channels + ch];
        if (depth == 16) {
            const size_t o = (static_cast<size_t>(x) * channels + ch) * 2;
            return (static_cast<uint32_t>(row[o]) << 8) | row[o + 1];
        }
        const size_t bit = static_cast<size_t>(x) * depth;
        return (row[bit / 8] >> (8 - depth - (bit % 8))) & ((1u << depth) - 1u);
    };
    for (uint32_t y = 0; y < h; ++y) {
        for (uint32_t x = 0; x < w; ++x) {
            float *o = &out.data[(static_cast<size_t>(y) * w + x) * out.channels];
            if (ctype == 3) {
                const uint32_t i = sample(x, y, 0);
                if (3 * i + 2 >= plte.size()) bad("PNG palette index");
                for (int c = 0; c < 3; ++c) o[c] = plte[3 * i + c] / 255.0f;
                if (out.channels == 4) o[3] = i < trns.size() ? trns[i] / 255.0f : 1.0f;
            } else {
                for (int c = 0; c < channels; ++c) o[c] = static_cast<float>(sample(x, y, c)) / maxv;
            }
        }
    }
    return out;
}

// ---- baseline JPEG (ITU-T T.81) ----------------------------------------------------

const uint8_t kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                             12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                             35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                             58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

struct JpegHuff {
    // Canonical code table of a DHT segment (T.81 annex C): the code of each
    // symbol from the counts per length.
    uint8_t counts[17] = {};
    std::vector<uint8_t> symbols;
    int maxcode[18] = {}, valptr[17] = {}, mincode[17] = {};
    bool defined = false;
    void build() {
        int code = 0, k = 0;
        for (int l = 1; l <= 16; ++l) {
            valptr[l] = k;
            mincode[l] = code;
            code += counts[l];
            k += counts[l];
            // More codes of this length than the code space holds.
            if (code > (1 << l)) bad("JPEG Huffman table over-subscribed");
            maxcode[l] = counts[l] ? code - 1 : -1;
            code <<= 1;
        }
        maxcode[17] = 0x7fffffff;
        defined = true;
    }
};

struct JpegBits {
    const uint8_t *p;
    size_t n, pos;
    uint32_t buf = 0;
    int cnt = 0;
    bool marker = false;
    int bit() {
        if (cnt == 0) {
            uint8_t b = 0;
            if (!marker && pos < n) {
                b = p[pos++];
                if (b == 0xff) {
                    const uint8_t nx = pos < n ? p[pos] : 0;
                    if (nx == 0x00) {
                        ++pos;
                    } else {
                        marker = true;  // a marker: feed zeros from here on
                        --pos;
                        b = 0;
                    }
                }
            }
            buf = b;
            cnt = 8;
        }
        --cnt;
        return (buf >> cnt) & 1;
    }
    int bits(int k) {
        int v = 0;
        for (int i = 0; i < k; ++i) v = (v << 1) | bit();
        return v;
    }
    int decode(const JpegHuff &h) {
        if (!h.defined) bad("JPEG scan uses an undefined Huffman table");
        int code = bit();
        for (int l = 1; l <= 16; ++l) {
            if (h.maxcode[l] >= 0 && code <= h.maxcode[l] && code >= h.mincode[l])
                return h.symbols[h.valptr[l] + code - h.mincode[l]];
            code = (code << 1) | bit();
        }
        bad("JPEG Huffman code");
    }
    // T.81 F.12: the value of a k-bit magnitude category.
    static int extend(int v, int k) { return (k && v < (1 << (k - 1))) ? v - (1 << k) + 1 : v; }
    void restart() {
        cnt = 0;
        marker = false;
        // Skip to the RSTn marker and past it.
        while (pos + 1 < n && !(p[pos] == 0xff && p[pos + 1] >= 0xd0 && p[pos + 1] <= 0xd7)) ++pos;
        if (pos + 1 < n) pos += 2;
    }
};

// 8 x 8 inverse DCT from its definition (T.81 A.3.3), separable, in float.
void idct8x8(const float *in, float *out) {
    static float cosv[8][8];
    static bool init = false;
    if (!init) {
        for (int x = 0; x < 8; ++x)
            for (int u = 0; u < 8; ++u)
                cosv[x][u] = (u == 0 ? std::sqrt(0.125f) : 0.5f) * std::cos((2 * x + 1) * u * 3.14159265358979323846 / 16.0);
        init = true;
    }
    float tmp[64];
    for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) {
            float s = 0.0f;
            for (int u = 0; u < 8; ++u) s += cosv[x][u] * in[y * 8 + u];
            tmp[y * 8 + x] = s;
        }
    for (int x = 0; x < 8; ++x)
        for (int y = 0; y < 8; ++y) {
            float s = 0.0f;
            for (int v = 0; v < 8; ++v) s += cosv[y][v] * tmp[v * 8 + x];
            out[y * 8 + x] = s;
        }
}

Image decode_jpeg(const std::vector<uint8_t> &f) {
    if (f.size() < 4 || f[0] != 0xff || f[1] != 0xd8) bad("not a JPEG file");
    uint16_t qt[4][64] = {};
    JpegHuff hdc[4], hac[4];
    struct Comp {
        int id, h, v, tq, td = 0, ta = 0;
        int bw, bh;  // blocks across / down, padded to whole MCUs
        std::vector<float> plane;
        int pred = 0;
    };
    std::vector<Comp> comps;
    int width = 0, height = 0, hmax = 1, vmax = 1, restart = 0;
    size_t p = 2;
    bool frame = false;
    while (p + 4 <= f.size()) {
        if (f[p] != 0xff) bad("JPEG marker expected");
        const uint8_t m = f[p + 1];
        p += 2;
        if (m == 0xd8 || (m >= 0xd0 && m <= 0xd7) || m == 0x01) continue;
        if (m == 0xd9) break;
        const size_t len = (static_cast<size_t>(f[p]) << 8) | f[p + 1];
        if (len < 2 || p + len > f.size()) bad("JPEG segment truncated");
        const uint8_t *d = &f[p + 2];
        const size_t dl = len - 2;
        if (m == 0xdb) {
            for (size_t i = 0; i < dl;) {
                const int pq = d[i] >> 4, tq = d[i] & 15;
                ++i;
                if (tq > 3 || pq > 1) bad("JPEG quantisation table id");
                if (i + (pq ? 128u : 64u) > dl) bad("JPEG quantisation table truncated");
                for (int k = 0; k < 64; ++k) {
                    qt[tq][k] = pq ? static_cast<uint16_t>((d[i] << 8) | d[i + 1]) : d[i];
                    i += pq ? 2 : 1;
                }
            }
        } else if (m == 0xc4) {
            for (size_t i = 0; i < dl;) {
                const int tc = d[i] >> 4, th = d[i] & 15;
                ++i;
                if (th > 3 || tc > 1) bad("JPEG Huffman table id");
                if (i + 16 > dl) bad("JPEG Huffman table truncated");
                JpegHuff &t = tc ? hac[th] : hdc[th];
                int total = 0;
                for (int l = 1; l <= 16; ++l) total += (t.counts[l] = d[i++]);
                if (i + static_cast<size_t>(total) > dl) bad("JPEG Huffman table truncated");
                t.symbols.assign(d + i, d + i + total);
                i += total;
                t.build();
            }
        } else if (m == 0xc0 || m == 0xc1) {
            if (frame) bad("JPEG with two frames");
            if (dl < 6) bad("JPEG frame header truncated");
            if (d[0] != 8) bad("JPEG sample precision other than 8 bits");
            height = (d[1] << 8) | d[2];
            width = (d[3] << 8) | d[4];
            if (static_cast<uint64_t>(width) * height > (1ull << 28)) bad("JPEG size");
            const int nc = d[5];
            if (nc != 1 && nc != 3) bad("JPEG component count");
            if (dl < 6u + 3u * nc) bad("JPEG frame header truncated");
            for (int c = 0; c < nc; ++c) {
                Comp k;
                k.id = d[6 + 3 * c];
                k.h = d[7 + 3 * c] >> 4;
                k.v = d[7 + 3 * c] & 15;
                k.tq = d[8 + 3 * c];
                if (k.h < 1 || k.v < 1 || k.h > 4 || k.v > 4 || k.tq > 3) bad("JPEG sampling factors");
                hmax = std::max(hmax, k.h);
                vmax = std::max(vmax, k.v);
                comps.push_back(k);
            }
            frame = true;
        } else if (m >= 0xc2 && m <= 0xcf && m != 0xc4 && m != 0xc8 && m != 0xcc) {
            not_supported("progressive, lossless or arithmetic-coded JPEG");
        } else if (m == 0xdd) {
            if (dl < 2) bad("JPEG restart interval truncated");
            restart = (d[0] << 8) | d[1];
        } else if (m == 0xda) {
            if (!frame || width == 0 || height == 0) bad("JPEG scan before its frame");
            if (dl < 1) bad("JPEG scan header truncated");
            const int ns = d[0];
            if (dl < 1u + 2u * ns) bad("JPEG scan header truncated");
            std::vector<int> order;
            for (int s = 0; s < ns; ++s) {
                const int id = d[1 + 2 * s], t = d[2 + 2 * s];
                if ((t >> 4) > 3 || (t & 15) > 3) bad("JPEG Huffman table id");
                for (size_t c = 0; c < comps.size(); ++c)
                    if (comps[c].id == id) {
                        comps[c].td = t >> 4;
                        comps[c].ta = t & 15;
                        order.push_back(static_cast<int>(c));
                    }
            }
            if (ns != static_cast<int>(comps.size())) bad("JPEG non-interleaved scans are not supported");
            const int mcux = (width + 8 * hmax - 1) / (8 * hmax), mcuy = (height + 8 * vmax - 1) / (8 * vmax);
            for (Comp &k : comps) {
                k.bw = mcux * k.h;
                k.bh = mcuy * k.v;
                k.plane.assign(static_cast<size_t>(k.bw) * 8 * k.bh * 8, 0.0f);
                k.pred = 0;
            }
            JpegBits br{f.data(), f.size(), p + len};
            int mcus = 0;
            float coef[64], blk[64];
            for (int my = 0; my < mcuy; ++my) {
                for (int mx = 0; mx < mcux; ++mx) {
                    if (restart && mcus && mcus % restart == 0) {
                        br.restart();
                        for (Comp &k : comps) k.pred = 0;
                    }
                    ++mcus;
                    for (int ci : order) {
                        Comp &k = comps[ci];
                        for (int by = 0; by < k.v; ++by)
                            for (int bx = 0; bx < k.h; ++bx) {
                                // T.81 F.2.2: DC difference, then AC run / size pairs.
                                std::memset(coef, 0, sizeof(coef));
                                const int t = br.decode(hdc[k.td]);
                                // 8-bit baseline: DC categories up to 11, AC sizes up to 10.
                                if (t > 11) bad("JPEG DC difference category");
                                const int diff = t ? JpegBits::extend(br.bits(t), t) : 0;
                                k.pred += diff;
                                coef[0] = static_cast<float>(k.pred * qt[k.tq][0]);
                                for (int i = 1; i < 64;) {
                                    const int rs = br.decode(hac[k.ta]);
                                    const int r = rs >> 4, sz = rs & 15;
                                    if (sz > 10) bad("JPEG AC coefficient size");
                                    if (sz == 0) {
                                        if (r == 15) {
                                            i += 16;
                                            continue;
                                        }
                                        break;
                                    }
                                    i += r;
                                    if (i > 63) bad("JPEG coefficient index");
                                    coef[kZigzag[i]] = static_cast<float>(JpegBits::extend(br.bits(sz), sz) * qt[k.tq][i]);
                                    ++i;
                                }
                                idct8x8(coef, blk);
                                const int ox = (mx * k.h + bx) * 8, oy = (my * k.v + by) * 8;
                                for (int y = 0; y < 8; ++y)
                                    for (int x = 0; x < 8; ++x) {
                                        const float v = std::round(blk[y * 8 + x] + 128.0f);
                                        k.plane[static_cast<size_t>(oy + y) * (k.bw * 8) + ox + x] =
                                            std::min(255.0f, std::max(0.0f, v));
                                    }
                            }
                    }
                }
            }
            // Colour: upsample chroma (linear, sample-centred), JFIF YCbCr -> RGB.
            Image out;
            out.width = static_cast<uint32_t>(width);
            out.height = static_cast<uint32_t>(height);
            out.channels = 3;
            out.data.assign(static_cast<size_t>(width) * height * 3, 0.0f);
            auto at = [&](const Comp &k, int x, int y) {
                // Sample (x, y) of the full-resolution grid from component k.
                const float sx = (static_cast<float>(x) + 0.5f) * k.h / hmax - 0.5f;
                const float sy = (static_cast<float>(y) + 0.5f) * k.v / vmax - 0.5f;
                const int w = k.bw * 8, hgt = k.bh * 8;
                const int x0 = static_cast<int>(std::floor(sx)), y0 = static_cast<int>(std::floor(sy));
                const float tx = sx - x0, ty = sy - y0;
                auto px = [&](int xx, int yy) {
                    xx = std::min(std::max(xx, 0), std::min(w, (width * k.h + hmax - 1) / hmax) - 1);
                    yy = std::min(std::max(yy, 0), std::min(hgt, (height * k.v + vmax - 1) / vmax) - 1);
                    return k.plane[static_cast<size_t>(yy) * w + xx];
                };
                if (k.h == hmax && k.v == vmax) return px(x, y);
                const float a = px(x0, y0), b = px(x0 + 1, y0), c = px(x0, y0 + 1), e = px(x0 + 1, y0 + 1);
                return (a * (1 - tx) + b * tx) * (1 - ty) + (c * (1 - tx) + e * tx) * ty;
            };
            for (int y = 0; y < height; ++y)
                for (int x = 0; x < width; ++x) {
                    float *o = &out.data[(static_cast<size_t>(y) * width + x) * 3];
                    const float Y = at(comps[0], x, y);
                    if (comps.size() == 1) {
                        o[0] = o[1] = o[2] = Y / 255.0f;
                        continue;
                    }
                    const float cb = at(comps[1], x, y) - 128.0f, cr = at(comps[2], x, y) - 128.0f;
                    const float rgb[3] = {Y + 1.402f * cr, Y - 0.344136f * cb - 0.714136f * cr, Y + 1.772f * cb};
                    for (int c = 0; c < 3; ++c) o[c] = std::min(255.0f, std::max(0.0f, std::round(rgb[c]))) / 255.0f;
                }
            return out;
        }
        p += len;
    }
    bad("JPEG without a scan");
}

// ---- Radiance HDR (RGBE) -----------------------------------------------------------

Image decode_hdr(const std::vector<uint8_t> &f) {
    size_t p = 0;
    auto line = [&]() {
        std::string s;
        while (p < f.size() && f[p] != '\n') s.push_back(static_cast<char>(f[p++]));
        if (p < f.size()) ++p;
        return s;
    };
    const std::string magic = line();
    if (magic.rfind("#?", 0) != 0) bad("not a Radiance HDR file");
    for (;;) {
        if (p >= f.size()) bad("HDR header truncated");
        const std::string s = line();
        if (s.empty()) break;
        if (s.rfind("FORMAT=", 0) == 0 && s != "FORMAT=32-bit_rle_rgbe") bad("HDR format " + printable(s));
    }
    const std::string res = line();
    int w = 0, h = 0;
    char ys[3] = {}, xs[3] = {};
    if (std::sscanf(res.c_str(), "%2s %d %2s %d", ys, &h, xs, &w) != 4 || std::string(ys) != "-Y" ||
        std::string(xs) != "+X" || w <= 0 || h <= 0)
        bad("HDR resolution line '" + printable(res) + "' (only -Y H +X W)");
    std::vector<uint8_t> rgbe(static_cast<size_t>(w) * h * 4);
    for (int y = 0; y < h; ++y) {
        uint8_t *row = &rgbe[static_cast<size_t>(y) * w * 4];
        if (p + 4 <= f.size() && f[p] == 2 && f[p + 1] == 2 && ((f[p + 2] << 8) | f[p + 3]) == w && w >= 8 &&
            w < 32768) {
            // New-style run-length scanline: four channel planes.
            p += 4;
            for (int c = 0; c < 4; ++c) {
                int x = 0;
                while (x < w) {
                    if (p >= f.size()) bad("HDR scanline truncated");
                    int count = f[p++];
                    if (count > 128) {
                        count -= 128;
                        if (x + count > w || p >= f.size()) bad("HDR run overflow");
                        const uint8_t v = f[p++];
                        for (int k = 0; k < count; ++k) row[4 * (x++) + c] = v;
                    } else {
                        if (count == 0 || x + count > w || p + count > f.size()) bad("HDR literal overflow");
                        for (int k = 0; k < count; ++k) row[4 * (x++) + c] = f[p++];
                    }
                }
            }
        } else {
            if (p + static_cast<size_t>(w) * 4 > f.size()) bad("HDR flat scanline truncated");
            std::memcpy(row, &f[p], static_cast<size_t>(w) * 4);
            p += static_cast<size_t>(w) * 4;
        }
    }
    Image out;
    out.width = static_cast<uint32_t>(w);
    out.height = static_cast<uint32_t>(h);
    out.channels = 3;
    out.data.resize(static_cast<size_t>(w) * h * 3);
    for (size_t i = 0; i < static_cast<size_t>(w) * h; ++i) {
        const uint8_t *e = &rgbe[4 * i];
        // RGBE: mantissa * 2^(exponent - 136); exponent 0 is black.
        const float s = e[3] ? std::ldexp(1.0f, static_cast<int>(e[3]) - 136) : 0.0f;
        for (int c = 0; c < 3; ++c) out.data[3 * i + c] = e[c] * s;
    }
    return out;
}

// ---- OpenEXR -------------------------------------------------------------------
// Single-part scanline files as the OpenEXR file layout defines them: magic
// 20000630, version 2, header attributes (name, type, size, value) up to an
// empty name, a table of chunk offsets, and chunks of {first line, packed
// size, data}.  Channels HALF, FLOAT or UINT at full resolution, stored per
// line in the channel list's (alphabetical) order.  Compression NONE, RLE
// (runs), ZIPS (one line) or ZIP (16 lines): a zlib stream, after which the
// byte-delta predictor and the split into two halves of the byte stream are
// undone.  PIZ, PXR24, B44 and DWA files, tiled, deep and multi-part files
// are refused.

uint32_t le32(const uint8_t *p) {
    return p[0] | (static_cast<uint32_t>(p[1]) << 8) | (static_cast<uint32_t>(p[2]) << 16) |
           (static_cast<uint32_t>(p[3]) << 24);
}

// IEEE 754 binary16 to binary32 (exact).
float half_bits_to_float(uint16_t h) {
    const uint32_t sign = static_cast<uint32_t>(h >> 15) << 31;
    const uint32_t e = (h >> 10) & 31u, m = h & 1023u;
    uint32_t bits;
    if (e == 0) {
        const float v = std::ldexp(static_cast<float>(m), -24);
        return sign ? -v : v;
    }
    bits = e == 31 ? (sign | 0x7f800000u | (m << 13)) : (sign | ((e + 112u) << 23) | (m << 13));
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// Undo ZIP / RLE preprocessing: deltas of successive bytes (biased by 128),
// then the first and second halves of the stream interleaved back.
void exr_unpredict(std::vector<uint8_t> &t) {
    for (size_t i = 1; i < t.size(); ++i) t[i] = static_cast<uint8_t>(t[i - 1] + t[i] - 128);
    std::vector<uint8_t> out(t.size());
    const size_t half = (t.size() + 1) / 2;
    for (size_t i = 0; i < t.size(); ++i) out[i] = (i & 1) ? t[half + i / 2] : t[i / 2];
    t.swap(out);
}

std::vector<uint8_t> exr_unrle(const uint8_t *d, size_t n, size_t expect) {
    std::vector<uint8_t> out;
    out.reserve(expect);
    size_t p = 0;
    while (p < n) {
        const int8_t c = static_cast<int8_t>(d[p++]);
        if (c < 0) {
            const size_t k = static_cast<size_t>(-c);
            if (p + k > n) bad("EXR RLE run truncated");
            out.insert(out.end(), d + p, d + p + k);
            p += k;
        } else {
            if (p >= n) bad("EXR RLE run truncated");
            out.insert(out.end(), static_cast<size_t>(c) + 1, d[p++]);
        }
        if (out.size() > expect) bad("EXR RLE data too long");
    }
    return out;
}

Image decode_exr(const std::vector<uint8_t> &f) {
    if (f.size() < 8 || le32(f.data()) != 20000630u) bad("not an OpenEXR file");
    const uint32_t version = le32(f.data() + 4);
    if ((version & 0xffu) != 2u) bad("EXR version");
    if (version & 0x200u) not_supported("tiled EXR");
    if (version & 0x1800u) not_supported("deep or multi-part EXR");
    size_t p = 8;
    auto cstr = [&]() {
        const size_t start = p;
        while (p < f.size() && f[p] != 0) ++p;
        if (p >= f.size() || p - start > 255) bad("EXR header truncated");
        return std::string(reinterpret_cast<const char *>(&f[start]), (p++) - start);
    };
    struct Chan {
        std::string name;
        uint32_t type;
        int32_t xs, ys;
    };
    std::vector<Chan> chans;
    int compression = -1;
    int32_t dw[4] = {0, 0, -1, -1};
    bool have_dw = false;
    for (;;) {
        const std::string name = cstr();
        if (name.empty()) break;
        cstr();  // attribute type
        if (p + 4 > f.size()) bad("EXR header truncated");
        const uint32_t size = le32(&f[p]);
        p += 4;
        if (size > f.size() - p) bad("EXR header truncated");
        const uint8_t *v = &f[p];
        if (name == "channels") {
            size_t q = 0;
            while (q < size && v[q] != 0) {
                size_t e = q;
                while (e < size && v[e] != 0) ++e;
                if (e + 17 > size) bad("EXR channel list truncated");
                Chan c{std::string(reinterpret_cast<const char *>(v + q), e - q), le32(v + e + 1),
                       static_cast<int32_t>(le32(v + e + 9)), static_cast<int32_t>(le32(v + e + 13))};
                chans.push_back(c);
                q = e + 17;
            }
        } else if (name == "compression") {
            if (size < 1) bad("EXR compression attribute");
            compression = v[0];
        } else if (name == "dataWindow") {
            if (size < 16) bad("EXR dataWindow attribute");
            for (int k = 0; k < 4; ++k) dw[k] = static_cast<int32_t>(le32(v + 4 * k));
            have_dw = true;
        }
        p += size;
    }
    if (!have_dw || chans.empty() || compression < 0) bad("EXR header lacks channels, compression or dataWindow");
    const int64_t w64 = static_cast<int64_t>(dw[2]) - dw[0] + 1, h64 = static_cast<int64_t>(dw[3]) - dw[1] + 1;
    if (w64 <= 0 || h64 <= 0 || w64 > 65536 || h64 > 65536) bad("EXR size");
    const uint32_t w = static_cast<uint32_t>(w64), h = static_cast<uint32_t>(h64);
    static const char *kNames[10] = {"NONE", "RLE", "ZIPS", "ZIP", "PIZ", "PXR24", "B44", "B44A", "DWAA", "DWAB"};
    uint32_t lines = 0;
    if (compression == 0 || compression == 1 || compression == 2) lines = 1;
    else if (compression == 3) lines = 16;
    else not_supported(std::string("EXR compression ") + (compression < 10 ? kNames[compression] : "unknown"));
    size_t pixel_bytes = 0;
    int rgb[3] = {-1, -1, -1}, grey = -1;
    for (size_t c = 0; c < chans.size(); ++c) {
        if (chans[c].type > 2) bad("EXR channel type");
        if (chans[c].xs != 1 || chans[c].ys != 1) not_supported("sub-sampled EXR channels");
        pixel_bytes += chans[c].type == 1 ? 2 : 4;
        const std::string &n = chans[c].name;
        if (n == "R") rgb[0] = static_cast<int>(c);
        else if (n == "G") rgb[1] = static_cast<int>(c);
        else if (n == "B") rgb[2] = static_cast<int>(c);
        else if (n == "Y") grey = static_cast<int>(c);
    }
    const bool colour = rgb[0] >= 0 && rgb[1] >= 0 && rgb[2] >= 0;
    if (!colour && grey < 0) not_supported("EXR without R, G, B or Y channels");
    Image out;
    out.width = w;
    out.height = h;
    out.channels = colour ? 3 : 1;
    out.data.assign(static_cast<size_t>(w) * h * out.channels, 0.0f);
    const size_t line_bytes = pixel_bytes * w;
    const uint32_t chunks = (h + lines - 1) / lines;
    if (p + 8ull * chunks > f.size()) bad("EXR offset table truncated");
    std::vector<bool> seen(chunks, false);
    for (uint32_t k = 0; k < chunks; ++k) {
        uint64_t off = 0;
        for (int b = 7; b >= 0; --b) off = (off << 8) | f[p + 8 * k + b];
        if (off + 8 > f.size()) bad("EXR chunk offset");
        const int64_t y0 = static_cast<int64_t>(static_cast<int32_t>(le32(&f[off]))) - dw[1];
        const uint32_t packed = le32(&f[off + 4]);
        if (y0 < 0 || y0 >= h64 || y0 % lines != 0 || packed > f.size() - off - 8) bad("EXR chunk header");
        const uint32_t ci = static_cast<uint32_t>(y0 / lines);
        if (seen[ci]) bad("EXR chunk repeated");
        seen[ci] = true;
        const uint32_t n_lines = std::min<uint32_t>(lines, h - static_cast<uint32_t>(y0));
        const size_t expect = line_bytes * n_lines;
        const uint8_t *d = &f[off + 8];
        std::vector<uint8_t> raw;
        if (compression == 0 || packed == expect) {
            if (packed != expect) bad("EXR chunk size");
            raw.assign(d, d + packed);
        } else {
            if (compression == 1) {
                raw = exr_unrle(d, packed, expect);
            } else {
                if (packed < 2) bad("EXR zlib stream");
                raw = inflate(d + 2, packed - 2, expect);
            }
            if (raw.size() != expect) bad("EXR chunk decodes to the wrong size");
            exr_unpredict(raw);
        }
        for (uint32_t l = 0; l < n_lines; ++l) {
            const uint8_t *row = raw.data() + l * line_bytes;
            float *dst = out.data.data() + (static_cast<size_t>(y0) + l) * w * out.channels;
            size_t at = 0;
            for (size_t c = 0; c < chans.size(); ++c) {
                const uint32_t t = chans[c].type;
                const int slot = colour ? (static_cast<int>(c) == rgb[0] ? 0 : static_cast<int>(c) == rgb[1] ? 1
                                                                          : static_cast<int>(c) == rgb[2] ? 2 : -1)
                                        : (static_cast<int>(c) == grey ? 0 : -1);
                for (uint32_t x = 0; x < w; ++x) {
                    float v;
                    if (t == 1) {
                        v = half_bits_to_float(static_cast<uint16_t>(row[at] | (row[at + 1] << 8)));
                        at += 2;
                    } else if (t == 2) {
                        const uint32_t b = le32(row + at);
                        std::memcpy(&v, &b, 4);
                        at += 4;
                    } else {
                        v = static_cast<float>(le32(row + at));
                        at += 4;
                    }
                    if (slot >= 0) dst[x * out.channels + slot] = v;
                }
            }
        }
    }
    return out;
}

std::string lower_ext(const std::string &path) {
    const size_t dot = path.find_last_of('.');
    std::string e = dot == std::string::npos ? "" : path.substr(dot + 1);
    for (char &c : e) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    return e;
}

}  // namespace

Image load_image(const std::string &path) {
    const std::vector<uint8_t> f = read_file(path);
    const std::string e = lower_ext(path);
    if (e == "png") return decode_png(f);
    if (e == "jpg" || e == "jpeg") return decode_jpeg(f);
    if (e == "hdr") return decode_hdr(f);
    if (e == "exr") return decode_exr(f);
    throw std::runtime_error("unsupported: image: format of '" + path + "' (PNG, JPEG, Radiance HDR, OpenEXR)");
}

float srgb_to_linear(float c) {
    return c <= 0.04045f ? c / 12.92f : std::pow((c + 0.055f) / 1.055f, 2.4f);
}

}  // namespace vs
